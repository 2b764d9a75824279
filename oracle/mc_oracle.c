/*
 * CPU restatement of the miniCOMBUST flow-solver SIMPLE pass.  TEST
 * INFRASTRUCTURE ONLY (see mc_oracle.h): the checker for the CUDA path and the
 * timed CPU baseline, never part of the product.
 *
 * Every function names the reference lines it restates.  Arithmetic is written
 * in the reference's operation order (vec<T> helpers of utils.hpp:195-354,
 * std::min/std::max argument order) and the library is built with FMA
 * contraction off, so compat mode reproduces the reference bit for bit.
 */
#include "mc_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define MESH_BOUNDARY UINT64_MAX
enum { FRONT = 0, BACK = 1, LEFT = 2, RIGHT = 3, DOWN = 4, UP = 5 };
enum { WALL = 1, INLET = 2, OUTLET = 3 };
enum { VA = 0, VB = 1, VC = 2, VD = 3, VE = 4, VF = 5, VG = 6, VH = 7 };

/* CUBE_FACE_VERTEX_MAP, Mesh.hpp:20-28 */
static const int face_vertex_map[6][4] = {
    {VA, VB, VC, VD}, {VE, VF, VG, VH}, {VA, VC, VE, VG},
    {VB, VD, VF, VH}, {VA, VB, VE, VF}, {VC, VD, VG, VH},
};

/* std::min / std::max semantics (argument order matters for signed zeros). */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }

typedef struct { double x, y, z; } v3;
static inline v3 mk(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vscale(v3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 vdiv(v3 a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline double vmag(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline v3 vnorm(v3 a) { return vdiv(a, vmag(a)); }
static inline v3 vcross(v3 a, v3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double vcos(v3 a, v3 b) { return vdot(a, b) / (vmag(a) * vmag(b)); }
static inline v3 ld3(const double *p, uint64_t i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
static inline void st3(double *p, uint64_t i, v3 v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }

struct mco_solver {
    mco_params prm;
    uint64_t N, F, P;
    const uint64_t *faces;      /* borrowed from the mesh: [F][2] */
    const uint64_t *cell_faces; /* [N][6] */
    const double *cc;           /* [N][3] */
    const uint64_t *cell_nbrs;  /* [N][6], MESH_BOUNDARY on the domain boundary */
    uint64_t btype[6];
    double *farea, *flam, *frl, *fnorm, *fcen; /* face geometry */
    double *vol, *rho;
    double *phi[MCO_NFIELDS];   /* [N + 6] */
    double *grad[MCO_NFIELDS];  /* [N][3]; allocated for U, V, W, P, PP, TEM */
    double *AU, *AV, *AW, *SU, *SV, *SW; /* [N + 6] */
    double *ff;                 /* face_fields [F][2] */
    double *mdot;               /* [F] */
    double *src;                /* particle_aos [N][5] */
    /* sparse pattern {diag} U {internal neighbours}, ascending columns */
    int *rp, *col;
    int nnz;
    double *valA, *valP;        /* A and Pressure_A values */
    double *bA, *bP;            /* b and Pressure_b */
    double eff_visc, inlet_eff_visc;
    int first_pressure;
    uint64_t timestep_count;
    int pass_in_step;
    int sources_set;
    double p_bnorm_ref;         /* simple mode: norm of the first corrector's right-hand side */
    mco_stats stats;
};

/* ------------------------------------------------------------------ params */

void mco_default_params(mco_params *p, int mode)
{
    memset(p, 0, sizeof(*p));
    p->mode = mode;
    p->delta = 1.0e-5;
    p->density = 1.2;
    p->inlet_u = 50.0;
    p->pressure0 = 4000.0;
    p->flux_corr = 0.8;
    p->urf_temperature = 0.95;
    p->max_iters = 100000;
    if (mode == MCO_MODE_COMPAT) {
        p->viscosity = 0.000014;
        p->temperature0 = 2000.0;
        p->urf_momentum = 0.5;
        p->urf_pressure = 0.2;
        p->u_rtol = 1e-13;
        p->p_rtol = 1e-13;
    } else {
        p->viscosity = 1.8e-5;
        p->temperature0 = 1500.0;
        p->urf_momentum = 0.7;
        p->urf_pressure = 0.3;
        p->u_rtol = 1e-13;
        p->p_rtol = 1e-13;
    }
}

/* -------------------------------------------------------------------- mesh */

/* load_mesh (mesh_examples.cpp:120-571) for a single flow rank: one block,
 * cells in x-fastest order, neighbours as in fill_neighbours (:13-118), faces
 * created in cell order with the partner slot f^1 (:510-561). */
int mco_mesh_box(uint64_t ex, uint64_t ey, uint64_t ez, double lx, double ly, double lz, mco_mesh *m)
{
    memset(m, 0, sizeof(*m));
    const uint64_t px = ex + 1, py = ey + 1, pz = ez + 1;
    const uint64_t N = ex * ey * ez;
    const double dx = lx / (double)ex, dy = ly / (double)ey, dz = lz / (double)ez;
    m->ex = ex; m->ey = ey; m->ez = ez;
    m->cells = N;
    m->points = px * py * pz;
    m->faces = (ex + 1) * ey * ez + (ey + 1) * ex * ez + (ez + 1) * ex * ey;
    m->points_xyz = (double *)malloc(3 * m->points * sizeof(double));
    m->cell_nodes = (uint64_t *)malloc(8 * N * sizeof(uint64_t));
    m->face_cells = (uint64_t *)malloc(2 * m->faces * sizeof(uint64_t));
    m->cell_faces = (uint64_t *)malloc(6 * N * sizeof(uint64_t));
    m->cell_neighbours = (uint64_t *)malloc(6 * N * sizeof(uint64_t));
    m->cell_centers = (double *)malloc(3 * N * sizeof(double));
    if (!m->points_xyz || !m->cell_nodes || !m->face_cells || !m->cell_faces || !m->cell_neighbours || !m->cell_centers) return -1;

    for (uint64_t idx = 0; idx < m->points; idx++) { /* :286-302 */
        const uint64_t x = idx % px, y = (idx / px) % py, z = idx / (px * py);
        m->points_xyz[3 * idx] = (double)x * dx;
        m->points_xyz[3 * idx + 1] = (double)y * dy;
        m->points_xyz[3 * idx + 2] = (double)z * dz;
    }
    for (uint64_t z = 0; z < ez; z++) /* :305-384 */
        for (uint64_t y = 0; y < ey; y++)
            for (uint64_t x = 0; x < ex; x++) {
                const uint64_t c = z * ex * ey + y * ex + x;
                const uint64_t g = x + y * px + z * px * py;
                uint64_t *n = m->cell_nodes + 8 * c;
                n[VA] = g;
                n[VH] = g + px * py + px + 1;
                n[VB] = g + 1;
                n[VC] = g + px;
                n[VD] = g + px + 1;
                n[VE] = g + px * py;
                n[VF] = g + px * py + 1;
                n[VG] = g + px * py + px;
                uint64_t *nb = m->cell_neighbours + 6 * c; /* fill_neighbours, :13-118 */
                nb[FRONT] = (z == 0) ? MESH_BOUNDARY : c - ex * ey;
                nb[BACK] = (z == ez - 1) ? MESH_BOUNDARY : c + ex * ey;
                nb[LEFT] = (x == 0) ? MESH_BOUNDARY : c - 1;
                nb[RIGHT] = (x == ex - 1) ? MESH_BOUNDARY : c + 1;
                nb[DOWN] = (y == 0) ? MESH_BOUNDARY : c - ex;
                nb[UP] = (y == ey - 1) ? MESH_BOUNDARY : c + ex;
            }
    m->boundary_types[FRONT] = WALL; /* :469-474 */
    m->boundary_types[BACK] = WALL;
    m->boundary_types[LEFT] = INLET;
    m->boundary_types[RIGHT] = OUTLET;
    m->boundary_types[DOWN] = WALL;
    m->boundary_types[UP] = WALL;

    uint64_t *face_index = (uint64_t *)malloc(6 * N * sizeof(uint64_t));
    for (uint64_t i = 0; i < 6 * N; i++) face_index[i] = UINT64_MAX;
    uint64_t count = 0;
    for (uint64_t c = 0; c < N; c++)
        for (uint64_t f = 0; f < 6; f++) {
            uint64_t nb = m->cell_neighbours[6 * c + f];
            if (face_index[6 * c + f] == UINT64_MAX) {
                const uint64_t nb_block = nb; /* block-relative id (:520) */
                if (nb == MESH_BOUNDARY) nb = N + f;
                m->face_cells[2 * count] = c < nb ? c : nb;
                m->face_cells[2 * count + 1] = c < nb ? nb : c;
                if (nb_block < N) face_index[6 * nb_block + (f ^ 1)] = count;
                m->cell_faces[6 * c + f] = count;
                count++;
            } else {
                m->cell_faces[6 * c + f] = face_index[6 * c + f];
            }
        }
    free(face_index);
    if (count != m->faces) return -2;

    for (uint64_t c = 0; c < N; c++) { /* calculate_cell_centers, Mesh.hpp:54-67 */
        v3 s = mk(0.0, 0.0, 0.0);
        for (int i = 0; i < 8; i++) s = vadd(s, ld3(m->points_xyz, m->cell_nodes[8 * c + i]));
        st3(m->cell_centers, c, vdiv(s, 8.0));
    }
    return 0;
}

void mco_mesh_free(mco_mesh *m)
{
    free(m->points_xyz);
    free(m->cell_nodes);
    free(m->face_cells);
    free(m->cell_faces);
    free(m->cell_neighbours);
    free(m->cell_centers);
    memset(m, 0, sizeof(*m));
}

/* ----------------------------------------------------------------- matrix */

static void build_pattern(mco_solver *s)
{
    const uint64_t N = s->N;
    int *cnt = (int *)calloc(N, sizeof(int));
    for (uint64_t i = 0; i < N; i++) cnt[i] = 1;
    for (uint64_t f = 0; f < s->F; f++) {
        const uint64_t c0 = s->faces[2 * f], c1 = s->faces[2 * f + 1];
        if (c1 >= N) continue;
        cnt[c0]++;
        cnt[c1]++;
    }
    s->rp = (int *)malloc((N + 1) * sizeof(int));
    s->rp[0] = 0;
    for (uint64_t i = 0; i < N; i++) s->rp[i + 1] = s->rp[i] + cnt[i];
    s->nnz = s->rp[N];
    s->col = (int *)malloc((size_t)s->nnz * sizeof(int));
    for (uint64_t i = 0; i < N; i++) cnt[i] = 0;
    for (uint64_t i = 0; i < N; i++) s->col[s->rp[i] + cnt[i]++] = (int)i;
    for (uint64_t f = 0; f < s->F; f++) {
        const uint64_t c0 = s->faces[2 * f], c1 = s->faces[2 * f + 1];
        if (c1 >= N) continue;
        s->col[s->rp[c0] + cnt[c0]++] = (int)c1;
        s->col[s->rp[c1] + cnt[c1]++] = (int)c0;
    }
    for (uint64_t i = 0; i < N; i++) { /* insertion sort, <= 7 entries */
        int *c = s->col + s->rp[i];
        const int n = s->rp[i + 1] - s->rp[i];
        for (int a = 1; a < n; a++) {
            const int v = c[a];
            int b = a - 1;
            while (b >= 0 && c[b] > v) { c[b + 1] = c[b]; b--; }
            c[b + 1] = v;
        }
    }
    free(cnt);
    s->valA = (double *)calloc((size_t)s->nnz, sizeof(double));
    s->valP = (double *)calloc((size_t)s->nnz, sizeof(double));
    s->bA = (double *)calloc(N, sizeof(double));
    s->bP = (double *)calloc(N, sizeof(double));
}

/* MatSetValue(..., INSERT_VALUES) on the fixed pattern. */
static void mat_set(const mco_solver *s, double *val, uint64_t r, uint64_t c, double v)
{
    for (int k = s->rp[r]; k < s->rp[r + 1]; k++)
        if ((uint64_t)s->col[k] == c) { val[k] = v; return; }
    abort();
}

/* Threads of the linear solves (mco_set_threads).  With one thread every
 * sum runs in index order, as in the reference's shim solvers; with more, the
 * loops are split across POSIX threads and dot products are summed in a
 * fixed number of chunks (a result that does not depend on the thread count,
 * but is not the serial rounding). */
static int g_threads = 1;
#define MCO_CHUNKS 512

void mco_set_threads(int n) { g_threads = n > 1 ? (n < 256 ? n : 256) : 1; }

typedef void (*range_fn)(void *ctx, uint64_t lo, uint64_t hi, int chunk);
typedef struct { range_fn fn; void *ctx; uint64_t n; int chunks, first, step; } par_job;

static void *par_worker(void *arg)
{
    const par_job *j = (const par_job *)arg;
    for (int c = j->first; c < j->chunks; c += j->step)
        j->fn(j->ctx, j->n * (uint64_t)c / (uint64_t)j->chunks, j->n * (uint64_t)(c + 1) / (uint64_t)j->chunks, c);
    return NULL;
}

/* fn over `chunks` equal ranges of [0, n): serially in order with one thread,
 * else chunk c on thread c mod g_threads. */
static void par_for(uint64_t n, int chunks, range_fn fn, void *ctx)
{
    if (g_threads <= 1) {
        for (int c = 0; c < chunks; c++) fn(ctx, n * (uint64_t)c / (uint64_t)chunks, n * (uint64_t)(c + 1) / (uint64_t)chunks, c);
        return;
    }
    const int T = g_threads;
    pthread_t th[256];
    par_job jobs[256];
    int joined[256] = {0};
    for (int t = 0; t < T; t++) jobs[t] = (par_job){fn, ctx, n, chunks, t, T};
    for (int t = 1; t < T; t++) {
        if (pthread_create(&th[t], NULL, par_worker, &jobs[t]) == 0)
            joined[t] = 1;
        else
            par_worker(&jobs[t]); /* could not start a thread: run its share here */
    }
    par_worker(&jobs[0]);
    for (int t = 1; t < T; t++)
        if (joined[t]) pthread_join(th[t], NULL);
}

typedef struct { const mco_solver *s; const double *val, *x; double *y; } spmv_ctx;
static void spmv_range(void *vc, uint64_t lo, uint64_t hi, int chunk)
{
    const spmv_ctx *c = (const spmv_ctx *)vc;
    (void)chunk;
    for (uint64_t i = lo; i < hi; i++) {
        double acc = 0.0;
        for (int k = c->s->rp[i]; k < c->s->rp[i + 1]; k++) acc += c->val[k] * c->x[c->s->col[k]];
        c->y[i] = acc;
    }
}

static void spmv(const mco_solver *s, const double *val, const double *x, double *y)
{
    spmv_ctx c = {s, val, x, y};
    par_for(s->N, g_threads <= 1 ? 1 : 4 * g_threads, spmv_range, &c);
}

typedef struct { const double *a, *b; double *part; } dot_ctx;
static void dot_range(void *vc, uint64_t lo, uint64_t hi, int chunk)
{
    const dot_ctx *c = (const dot_ctx *)vc;
    double acc = 0.0;
    if (c->b)
        for (uint64_t i = lo; i < hi; i++) acc += c->a[i] * c->b[i];
    else
        for (uint64_t i = lo; i < hi; i++) acc += c->a[i];
    c->part[chunk] = acc;
}

/* sum of a[i] * b[i] (b null: sum of a[i]) */
static double sumn(const double *a, const double *b, uint64_t n)
{
    if (g_threads <= 1) {
        double acc = 0.0;
        if (b)
            for (uint64_t i = 0; i < n; i++) acc += a[i] * b[i];
        else
            for (uint64_t i = 0; i < n; i++) acc += a[i];
        return acc;
    }
    double part[MCO_CHUNKS];
    dot_ctx c = {a, b, part};
    par_for(n, MCO_CHUNKS, dot_range, &c);
    double acc = 0.0;
    for (int k = 0; k < MCO_CHUNKS; k++) acc += part[k];
    return acc;
}

static double dotn(const double *a, const double *b, uint64_t n) { return sumn(a, b, n); }

static void project_mean_zero(double *v, uint64_t n)
{
    const double acc = sumn(v, NULL, n);
    const double m = acc / (double)n;
    for (uint64_t i = 0; i < n; i++) v[i] -= m;
}

/* Vector updates of the Krylov loops, split like spmv. */
typedef struct { int op; double a, b; double *x, *y, *z; const double *u, *v, *w; } axpy_ctx;
static void axpy_range(void *vc, uint64_t lo, uint64_t hi, int chunk)
{
    const axpy_ctx *c = (const axpy_ctx *)vc;
    (void)chunk;
    switch (c->op) {
    case 0: /* p = r + beta (p - omega v) */
        for (uint64_t i = lo; i < hi; i++) c->x[i] = c->u[i] + c->a * (c->x[i] - c->b * c->v[i]);
        break;
    case 1: /* s = r - alpha v */
        for (uint64_t i = lo; i < hi; i++) c->x[i] = c->u[i] - c->a * c->v[i];
        break;
    case 2: /* x += alpha p + omega s; r = s - omega t */
        for (uint64_t i = lo; i < hi; i++) {
            c->x[i] += c->a * c->u[i] + c->b * c->v[i];
            c->y[i] = c->v[i] - c->b * c->w[i];
        }
        break;
    case 3: /* x += alpha p; r -= alpha q */
        for (uint64_t i = lo; i < hi; i++) {
            c->x[i] += c->a * c->u[i];
            c->y[i] -= c->a * c->v[i];
        }
        break;
    case 4: /* p = r + beta p */
        for (uint64_t i = lo; i < hi; i++) c->x[i] = c->u[i] + c->a * c->x[i];
        break;
    }
}

static void vec_op(uint64_t n, axpy_ctx c) { par_for(n, g_threads <= 1 ? 1 : 4 * g_threads, axpy_range, &c); }

/* KSPBCGS with PCNONE from a zero guess (the reference's KSP for momentum and
 * scalars, FlowSolver.hpp:513-519; solve at FlowSolver.inl:1341-1375). */
static int solve_bicgstab(const mco_solver *s, const double *val, const double *b, double *x, double rtol)
{
    const uint64_t n = s->N;
    double *r = (double *)malloc(n * sizeof(double)), *r0 = (double *)malloc(n * sizeof(double));
    double *p = (double *)calloc(n, sizeof(double)), *v = (double *)calloc(n, sizeof(double));
    double *sv = (double *)malloc(n * sizeof(double)), *t = (double *)malloc(n * sizeof(double));
    memcpy(r, b, n * sizeof(double));
    memcpy(r0, b, n * sizeof(double));
    for (uint64_t i = 0; i < n; i++) x[i] = 0.0;
    const double bnorm = sqrt(dotn(b, b, n));
    int its = 0;
    if (bnorm != 0.0) {
        double rho = 1.0, alpha = 1.0, omega = 1.0;
        its = -s->prm.max_iters;
        for (int k = 1; k <= s->prm.max_iters; k++) {
            const double rho_new = dotn(r0, r, n);
            if (rho_new == 0.0) { its = -k; break; }
            const double beta = (rho_new / rho) * (alpha / omega);
            vec_op(n, (axpy_ctx){0, beta, omega, p, NULL, NULL, r, v, NULL});
            spmv(s, val, p, v);
            alpha = rho_new / dotn(r0, v, n);
            vec_op(n, (axpy_ctx){1, alpha, 0.0, sv, NULL, NULL, r, v, NULL});
            spmv(s, val, sv, t);
            const double tt = dotn(t, t, n);
            omega = (tt != 0.0) ? dotn(t, sv, n) / tt : 0.0;
            vec_op(n, (axpy_ctx){2, alpha, omega, x, r, NULL, p, sv, t});
            rho = rho_new;
            const double rn = sqrt(dotn(r, r, n));
            if (rn <= rtol * bnorm) { its = k; break; }
            if (omega == 0.0) { its = -k; break; }
        }
    }
    free(r); free(r0); free(p); free(v); free(sv); free(t);
    return its;
}

/* The pressure-correction KSP (FGMRES + GAMG in the reference,
 * FlowSolver.hpp:521-527) restated as conjugate gradients on the singular
 * symmetric system with mean-zero projection of the right-hand side and of
 * the solution.  abs_floor (>= 0) is an absolute residual floor. */
static int solve_cg_projected(const mco_solver *s, const double *val, const double *b_in, double *x, double rtol,
                              double abs_floor, double *bnorm_out)
{
    const uint64_t n = s->N;
    double *b = (double *)malloc(n * sizeof(double)), *r = (double *)malloc(n * sizeof(double));
    double *p = (double *)malloc(n * sizeof(double)), *q = (double *)malloc(n * sizeof(double));
    memcpy(b, b_in, n * sizeof(double));
    project_mean_zero(b, n);
    for (uint64_t i = 0; i < n; i++) x[i] = 0.0;
    memcpy(r, b, n * sizeof(double));
    memcpy(p, b, n * sizeof(double));
    double rr = dotn(r, r, n);
    const double bnorm = sqrt(rr);
    if (bnorm_out) *bnorm_out = bnorm;
    const double tol = smax(rtol * bnorm, abs_floor);
    int k = 0;
    if (bnorm != 0.0 && bnorm > abs_floor) {
        for (k = 1; k <= s->prm.max_iters; k++) {
            spmv(s, val, p, q);
            const double alpha = rr / dotn(p, q, n);
            vec_op(n, (axpy_ctx){3, alpha, 0.0, x, r, NULL, p, q, NULL});
            const double rr_new = dotn(r, r, n);
            if (sqrt(rr_new) <= tol) break;
            const double beta = rr_new / rr;
            rr = rr_new;
            vec_op(n, (axpy_ctx){4, beta, 0.0, p, NULL, NULL, r, NULL, NULL});
        }
        project_mean_zero(x, n);
        if (k > s->prm.max_iters) k = -s->prm.max_iters;
    }
    free(b); free(r); free(p); free(q);
    return k;
}

/* ------------------------------------------------------------ construction */

/* FlowSolver constructor (FlowSolver.hpp:147-539) for one rank: face geometry
 * (:253-294 internal, :349-397 boundary), cell data (:302-347), boundary slot
 * values and inlet effective viscosity (:403-485). */
mco_solver *mco_create(const mco_mesh *m, const mco_params *prm)
{
    mco_solver *s = (mco_solver *)calloc(1, sizeof(mco_solver));
    s->prm = *prm;
    const uint64_t N = m->cells, F = m->faces;
    s->N = N; s->F = F; s->P = m->points;
    s->faces = m->face_cells;
    s->cell_faces = m->cell_faces;
    s->cc = m->cell_centers;
    s->cell_nbrs = m->cell_neighbours;
    memcpy(s->btype, m->boundary_types, sizeof(s->btype));
    s->farea = (double *)calloc(F, sizeof(double));
    s->flam = (double *)calloc(F, sizeof(double));
    s->frl = (double *)calloc(F, sizeof(double));
    s->fnorm = (double *)calloc(3 * F, sizeof(double));
    s->fcen = (double *)calloc(3 * F, sizeof(double));
    s->vol = (double *)calloc(N, sizeof(double));
    s->rho = (double *)calloc(N, sizeof(double));
    for (int k = 0; k < MCO_NFIELDS; k++) s->phi[k] = (double *)calloc(N + 6, sizeof(double));
    const int gfields[12] = {MCO_U, MCO_V, MCO_W, MCO_P, MCO_PP, MCO_TEM,
                             MCO_TE, MCO_ED, MCO_FUL, MCO_PRO, MCO_VARF, MCO_VARP};
    for (int k = 0; k < (prm->scalars ? 12 : 6); k++) s->grad[gfields[k]] = (double *)calloc(3 * N, sizeof(double));
    s->AU = (double *)calloc(N + 6, sizeof(double));
    s->AV = (double *)calloc(N + 6, sizeof(double));
    s->AW = (double *)calloc(N + 6, sizeof(double));
    s->SU = (double *)calloc(N + 6, sizeof(double));
    s->SV = (double *)calloc(N + 6, sizeof(double));
    s->SW = (double *)calloc(N + 6, sizeof(double));
    s->ff = (double *)calloc(2 * F, sizeof(double));
    s->mdot = (double *)calloc(F, sizeof(double));
    s->src = (double *)calloc(5 * N, sizeof(double));
    build_pattern(s);

    const double *pts = m->points_xyz;
    for (uint64_t f = 0; f < F; f++) { /* internal faces, :253-294 */
        const uint64_t c0 = s->faces[2 * f], c1 = s->faces[2 * f + 1];
        if (c1 >= N) continue;
        uint64_t ids[4];
        int cnt = 0;
        for (int n0 = 0; n0 < 8; n0++)
            for (int n1 = 0; n1 < 8; n1++)
                if (m->cell_nodes[8 * c0 + n0] == m->cell_nodes[8 * c1 + n1]) ids[cnt++] = m->cell_nodes[8 * c0 + n0];
        if (cnt != 4) { mco_destroy(s); return NULL; }
        const v3 n0 = ld3(pts, ids[0]), n1 = ld3(pts, ids[1]), n2 = ld3(pts, ids[2]), n3 = ld3(pts, ids[3]);
        const v3 d01 = vsub(ld3(s->cc, c1), ld3(s->cc, c0));
        s->farea[f] = vmag(vsub(n2, n0)) * vmag(vsub(n1, n0));
        v3 fc = vadd(vadd(vadd(n0, n1), n2), n3);
        fc = vdiv(fc, 4.0);
        st3(s->fcen, f, fc);
        s->flam[f] = vmag(vsub(fc, ld3(s->cc, c0))) / vmag(d01);
        v3 nrm = vcross(vsub(n2, n0), vsub(n1, n0));
        if (vdot(nrm, vsub(ld3(s->cc, c1), ld3(s->cc, c0))) < 0) nrm = vscale(nrm, -1.);
        st3(s->fnorm, f, nrm);
        s->frl[f] = s->farea[f] / vmag(d01) / vcos(nrm, d01);
        s->mdot[f] = 0.0;
    }
    s->eff_visc = prm->viscosity;
    for (uint64_t c = 0; c < N; c++) { /* cell loop, :302-398 */
        const uint64_t *cn = m->cell_nodes + 8 * c;
        s->rho[c] = prm->density;
        const double width = vmag(vsub(ld3(pts, cn[VB]), ld3(pts, cn[VA])));
        const double height = vmag(vsub(ld3(pts, cn[VC]), ld3(pts, cn[VA])));
        const double length = vmag(vsub(ld3(pts, cn[VE]), ld3(pts, cn[VA])));
        s->vol[c] = width * height * length;
        for (int f = 0; f < 6; f++) {
            if (m->cell_neighbours[6 * c + f] < N) continue;
            const uint64_t face = m->cell_faces[6 * c + f];
            const v3 n0 = ld3(pts, cn[face_vertex_map[f][0]]), n1 = ld3(pts, cn[face_vertex_map[f][1]]);
            const v3 n2 = ld3(pts, cn[face_vertex_map[f][2]]), n3 = ld3(pts, cn[face_vertex_map[f][3]]);
            s->flam[face] = 1.0;
            s->farea[face] = vmag(vsub(n2, n0)) * vmag(vsub(n1, n0));
            const v3 fc = vdiv(vadd(vadd(vadd(n0, n1), n2), n3), 4.0);
            st3(s->fcen, face, fc);
            v3 nrm = vcross(vsub(n2, n0), vsub(n1, n0));
            /* every boundary type orients the normal outwards (:370-391) */
            if (vdot(nrm, vsub(ld3(s->cc, c), fc)) > 0) nrm = vscale(nrm, -1.);
            st3(s->fnorm, face, nrm);
            s->mdot[face] = 0.0;
            const v3 dcf = vsub(fc, ld3(s->cc, c));
            s->frl[face] = s->farea[face] / vmag(dcf) / vcos(nrm, dcf);
        }
        /* initial interior state, :315-327 */
        s->phi[MCO_U][c] = prm->inlet_u;
        s->phi[MCO_V][c] = 0.0;
        s->phi[MCO_W][c] = 0.0;
        s->phi[MCO_P][c] = prm->pressure0;
        s->phi[MCO_PP][c] = 0.0;
        s->phi[MCO_TE][c] = 0.0001;
        s->phi[MCO_ED][c] = 0.0;
        s->phi[MCO_TEM][c] = prm->temperature0;
        s->phi[MCO_FUL][c] = 0.1;
        s->phi[MCO_PRO][c] = 0.001;
        s->phi[MCO_VARF][c] = 0.1;
        s->phi[MCO_VARP][c] = 0.001;
    }
    /* boundary slots and inlet viscosity, :403-485 */
    const double velmag2 = pow(prm->inlet_u, 2) + pow(0.0, 2) + pow(0.0, 2);
    s->inlet_eff_visc = s->eff_visc + 1.2 * 0.09 * (3.0 / 2.0 * ((0.1 * 0.1) * velmag2)) /
                                          ((pow(0.09, 0.75) * pow((3.0 / 2.0 * ((0.1 * 0.1) * velmag2)), 1.5)) + 0.00000000000000000001);
    for (int b = 0; b < 6; b++) {
        const uint64_t i = N + (uint64_t)b;
        const int t = (int)s->btype[b];
        s->phi[MCO_U][i] = (t == INLET || t == OUTLET) ? prm->inlet_u : 0.0;
        s->phi[MCO_V][i] = 0.0;
        s->phi[MCO_W][i] = 0.0;
        s->phi[MCO_P][i] = prm->pressure0;
        s->phi[MCO_PP][i] = 0.0;
        s->phi[MCO_TEM][i] = prm->temperature0;
        /* the other scalars: defaults, then per boundary type */
        double te = 0.0001, ed = 0.0, ful = 0.1, pro = 0.001, varf = 0.1, varp = 0.001;
        if (t == INLET) {
            te = 3.0 / 2.0 * ((0.1 * 0.1) * velmag2);
            ed = pow(0.09, 0.75) * pow(te, 1.5);
            ful = 0.1; pro = 0.0; varf = 0.1; varp = 0.0;
        } else if (t == WALL) {
            ful = 0.0; pro = 0.0; varf = 0.0; varp = 0.0;
        }
        s->phi[MCO_TE][i] = te;
        s->phi[MCO_ED][i] = ed;
        s->phi[MCO_TP][i] = 0.0;
        s->phi[MCO_FUL][i] = ful;
        s->phi[MCO_PRO][i] = pro;
        s->phi[MCO_VARF][i] = varf;
        s->phi[MCO_VARP][i] = varp;
    }
    s->first_pressure = 1;
    return s;
}

void mco_destroy(mco_solver *s)
{
    if (!s) return;
    free(s->farea); free(s->flam); free(s->frl); free(s->fnorm); free(s->fcen);
    free(s->vol); free(s->rho);
    for (int k = 0; k < MCO_NFIELDS; k++) { free(s->phi[k]); free(s->grad[k]); }
    free(s->AU); free(s->AV); free(s->AW); free(s->SU); free(s->SV); free(s->SW);
    free(s->ff); free(s->mdot); free(s->src);
    free(s->rp); free(s->col); free(s->valA); free(s->valP); free(s->bA); free(s->bP);
    free(s);
}

/* --------------------------------------------------------------- accessors */

uint64_t mco_phi_length(const mco_solver *s) { return s->N + 6; }

int mco_set_field(mco_solver *s, int which, const double *vals)
{
    if (which < 0 || which >= MCO_NFIELDS) return -1;
    memcpy(s->phi[which], vals, (s->N + 6) * sizeof(double));
    return 0;
}

int mco_get_field(const mco_solver *s, int which, double *out)
{
    if (which < 0 || which >= MCO_NFIELDS) return -1;
    memcpy(out, s->phi[which], (s->N + 6) * sizeof(double));
    return 0;
}

int mco_get_grad(const mco_solver *s, int which, double *out)
{
    if (which < 0 || which >= MCO_NFIELDS || !s->grad[which]) return -1;
    memcpy(out, s->grad[which], 3 * s->N * sizeof(double));
    return 0;
}

int mco_get_cell_array(const mco_solver *s, int which, double *out)
{
    const double *a[8] = {s->AU, s->AV, s->AW, s->SU, s->SV, s->SW, s->vol, s->rho};
    if (which < 0 || which >= 8) return -1;
    memcpy(out, a[which], s->N * sizeof(double));
    return 0;
}

int mco_get_face_array(const mco_solver *s, int which, double *out)
{
    const uint64_t F = s->F;
    switch (which) {
    case 0: memcpy(out, s->mdot, F * sizeof(double)); return 0;
    case 1: memcpy(out, s->farea, F * sizeof(double)); return 0;
    case 2: memcpy(out, s->flam, F * sizeof(double)); return 0;
    case 3: memcpy(out, s->frl, F * sizeof(double)); return 0;
    case 4: memcpy(out, s->ff, 2 * F * sizeof(double)); return 0;
    case 5: memcpy(out, s->fnorm, 3 * F * sizeof(double)); return 0;
    case 6: memcpy(out, s->fcen, 3 * F * sizeof(double)); return 0;
    default: return -1;
    }
}

int mco_set_sources(mco_solver *s, const double *terms)
{
    memcpy(s->src, terms, 5 * s->N * sizeof(double));
    s->sources_set = 1;
    return 0;
}

int mco_get_csr(const mco_solver *s, int which, int *n, int *nnz, int *row_ptr, int *col, double *val)
{
    *n = (int)s->N;
    *nnz = s->nnz;
    if (row_ptr) memcpy(row_ptr, s->rp, (s->N + 1) * sizeof(int));
    if (col) memcpy(col, s->col, (size_t)s->nnz * sizeof(int));
    if (val) memcpy(val, which == 0 ? s->valA : s->valP, (size_t)s->nnz * sizeof(double));
    return 0;
}

int mco_get_rhs(const mco_solver *s, int which, double *out)
{
    memcpy(out, which == 0 ? s->bA : s->bP, s->N * sizeof(double));
    return 0;
}

void mco_get_stats(const mco_solver *s, mco_stats *out) { *out = s->stats; }
double mco_inlet_effective_viscosity(const mco_solver *s) { return s->inlet_eff_visc; }

/* --------------------------------------------------------------- gradients */

/* solve (FlowSolver.inl:895-915): Cramer's rule, det == 0 gives zero. */
static void solve3(double A[3][3], const double *b, double *out)
{
    const double det = (A[0][0] * (A[1][1] * A[2][2] - A[2][1] * A[1][2])) -
                       (A[0][1] * (A[1][0] * A[2][2] - A[2][0] * A[1][2])) +
                       (A[0][2] * (A[1][0] * A[2][1] - A[2][0] * A[1][1]));
    double invdet = 0.0;
    if (det != 0.0) invdet = 1 / det;
    out[0] = (b[0] * invdet * (A[1][1] * A[2][2] - A[2][1] * A[1][2])) +
             (b[1] * invdet * (A[2][1] * A[0][2] - A[0][1] * A[2][2])) +
             (b[2] * invdet * (A[0][1] * A[1][2] - A[1][1] * A[0][2]));
    out[1] = (b[0] * invdet * (A[1][2] * A[2][0] - A[1][0] * A[2][2])) +
             (b[1] * invdet * (A[0][0] * A[2][2] - A[2][0] * A[0][2])) +
             (b[2] * invdet * (A[1][0] * A[0][2] - A[0][0] * A[1][2]));
    out[2] = (b[0] * invdet * (A[1][0] * A[2][1] - A[2][0] * A[1][1])) +
             (b[1] * invdet * (A[2][0] * A[0][1] - A[0][0] * A[2][1])) +
             (b[2] * invdet * (A[0][0] * A[1][1] - A[1][0] * A[0][1]));
}

/* Least-squares gradients of nf fields (get_phi_gradients, FlowSolver.inl:917-1063,
 * and get_phi_gradient, :738-803).  zero_bnd[k] != 0 gives dphi = 0 on
 * boundary faces (the pressure treatment, :980 and :773-776). */
static void lsq_gradients(mco_solver *s, const int *fields, const int *zero_bnd, int nf)
{
    const uint64_t N = s->N;
    for (uint64_t c = 0; c < N; c++) {
        double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        double b[8][3];
        memset(b, 0, sizeof(b));
        for (int f = 0; f < 6; f++) {
            const uint64_t face = s->cell_faces[6 * c + f];
            const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
            double dphi[8];
            v3 dX;
            if (c1 < N) {
                const double mask = (c0 == c) ? 1. : -1.;
                for (int k = 0; k < nf; k++) dphi[k] = mask * (s->phi[fields[k]][c1] - s->phi[fields[k]][c0]);
                dX = vscale(vsub(ld3(s->cc, c1), ld3(s->cc, c0)), mask);
            } else {
                const uint64_t bc = c1 - N;
                for (int k = 0; k < nf; k++) dphi[k] = zero_bnd[k] ? 0.0 : s->phi[fields[k]][N + bc] - s->phi[fields[k]][c0];
                dX = vsub(ld3(s->fcen, face), ld3(s->cc, c0));
            }
            A[0][0] += (dX.x * dX.x);
            A[1][0] += (dX.x * dX.y);
            A[2][0] += (dX.x * dX.z);
            A[0][1] += (dX.y * dX.x);
            A[1][1] += (dX.y * dX.y);
            A[2][1] += (dX.y * dX.z);
            A[0][2] += (dX.z * dX.x);
            A[1][2] += (dX.z * dX.y);
            A[2][2] += (dX.z * dX.z);
            for (int k = 0; k < nf; k++) {
                b[k][0] += (dX.x * dphi[k]);
                b[k][1] += (dX.y * dphi[k]);
                b[k][2] += (dX.z * dphi[k]);
            }
        }
        for (int k = 0; k < nf; k++) solve3(A, b[k], s->grad[fields[k]] + 3 * c);
    }
}

void mco_stage_gradients(mco_solver *s)
{
    static const int fields[5] = {MCO_U, MCO_V, MCO_W, MCO_P, MCO_TEM};
    static const int zb[5] = {0, 0, 0, 1, 0};
    lsq_gradients(s, fields, zb, 5);
    if (s->prm.scalars) {
        static const int more[6] = {MCO_TE, MCO_ED, MCO_FUL, MCO_PRO, MCO_VARF, MCO_VARP};
        static const int zb6[6] = {0, 0, 0, 0, 0, 0};
        lsq_gradients(s, more, zb6, 6);
    }
}

static void single_gradient_pressure(mco_solver *s, int field)
{
    const int f[1] = {field};
    const int zb[1] = {1};
    lsq_gradients(s, f, zb, 1);
}

/* ---------------------------------------------------------------- momentum */

/* precomp_AU (FlowSolver.inl:1065-1104) */
static void precomp_AU(mco_solver *s)
{
    const uint64_t N = s->N;
    for (uint64_t i = 0; i < N; i++) s->AU[i] = 0.0;
    for (uint64_t face = 0; face < s->F; face++) {
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        if (c1 < N) continue;
        const int t = (int)s->btype[c1 - N];
        if (t == INLET || t == OUTLET) {
            const double VisFace = s->eff_visc * s->frl[face];
            const double f = -VisFace + smin(s->mdot[face], 0.0);
            s->AU[c0] = s->AU[c0] - f;
        }
    }
    const double rdelta = 1.0 / s->prm.delta;
    for (uint64_t i = 0; i < N; i++) {
        const double f = s->rho[i] * s->vol[i] * rdelta;
        s->AU[i] += f;
    }
}

static void calculate_mass_flux(mco_solver *s);

/* set_up_field (FlowSolver.inl:1106-1113) */
void mco_stage_set_up_field(mco_solver *s)
{
    precomp_AU(s);
    calculate_mass_flux(s);
}

/* calculate_flux_UVW (FlowSolver.inl:1377-1653) */
static void calculate_flux_UVW(mco_solver *s)
{
    const uint64_t N = s->N;
    const double GammaBlend = 0.0;
    const double mu = s->eff_visc;
    double *U = s->phi[MCO_U], *V = s->phi[MCO_V], *W = s->phi[MCO_W];
    const double *gU = s->grad[MCO_U], *gV = s->grad[MCO_V], *gW = s->grad[MCO_W];
    for (uint64_t face = 0; face < s->F; face++) {
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        const v3 S = ld3(s->fnorm, face);
        if (c1 < N) {
            const double lambda0 = s->flam[face];
            const double lambda1 = 1.0 - lambda0;
            const v3 dU = vadd(vscale(ld3(gU, c0), lambda0), vscale(ld3(gU, c1), lambda1));
            const v3 dV = vadd(vscale(ld3(gV, c0), lambda0), vscale(ld3(gV, c1), lambda1));
            const v3 dW = vadd(vscale(ld3(gW, c0), lambda0), vscale(ld3(gW, c1), lambda1));
            const double Visac = mu * lambda0 + mu * lambda1;
            const double VisFace = Visac * s->frl[face];
            const v3 Xpn = vsub(ld3(s->cc, c1), ld3(s->cc, c0));
            const double md = s->mdot[face];
            double UFace, VFace, WFace;
            if (md >= 0.0) { UFace = U[c0]; VFace = V[c0]; WFace = W[c0]; }
            else { UFace = U[c1]; VFace = V[c1]; WFace = W[c1]; }
            const double fuce = md * UFace, fvce = md * VFace, fwce = md * WFace;
            const double fude = Visac * ((dU.x + dU.x) * S.x + (dU.y + dV.x) * S.y + (dU.z + dW.x) * S.z);
            const double fvde = Visac * ((dU.y + dV.x) * S.x + (dV.y + dV.y) * S.y + (dV.z + dW.y) * S.z);
            const double fwde = Visac * ((dU.z + dW.x) * S.x + (dW.y + dV.z) * S.y + (dW.z + dW.z) * S.z);
            const double fmin = smin(md, 0.0), fmax = smax(md, 0.0);
            const double fuci = fmin * U[c0] + fmax * U[c1];
            const double fvci = fmin * V[c0] + fmax * V[c1];
            const double fwci = fmin * W[c0] + fmax * W[c1];
            const double fudi = VisFace * vdot(dU, Xpn);
            const double fvdi = VisFace * vdot(dV, Xpn);
            const double fwdi = VisFace * vdot(dW, Xpn);
            s->ff[2 * face] = -VisFace - smax(md, 0.0);
            s->ff[2 * face + 1] = -VisFace + smin(md, 0.0);
            const double bu = GammaBlend * (fuce - fuci);
            const double bv = GammaBlend * (fvce - fvci);
            const double bw = GammaBlend * (fwce - fwci);
            s->SU[c0] = s->SU[c0] - bu + fude - fudi;
            s->SV[c0] = s->SV[c0] - bv + fvde - fvdi;
            s->SW[c0] = s->SW[c0] - bw + fwde - fwdi;
            s->SU[c1] = s->SU[c1] + bu - fude + fudi;
            s->SV[c1] = s->SV[c1] + bv - fvde + fvdi;
            s->SW[c1] = s->SW[c1] + bw - fwde + fwdi;
        } else {
            const uint64_t bc = c1 - N;
            const int t = (int)s->btype[bc];
            if (t == INLET || t == OUTLET) {
                const v3 dU = ld3(gU, c0), dV = ld3(gV, c0), dW = ld3(gW, c0);
                double UFace, VFace, WFace, Visac;
                if (t == INLET) { UFace = s->prm.inlet_u; VFace = 0.0; WFace = 0.0; Visac = s->inlet_eff_visc; }
                else { UFace = U[c0]; VFace = V[c0]; WFace = W[c0]; Visac = mu; }
                const v3 Xpn = vsub(ld3(s->fcen, face), ld3(s->cc, c0));
                const double VisFace = Visac * s->frl[face];
                const double fude = Visac * ((dU.x + dU.x) * S.x + (dU.y + dV.x) * S.y + (dU.z + dW.x) * S.z);
                const double fvde = Visac * ((dU.y + dV.x) * S.x + (dV.y + dV.y) * S.y + (dV.z + dW.y) * S.z);
                const double fwde = Visac * ((dU.z + dW.x) * S.x + (dW.y + dV.z) * S.y + (dW.z + dW.z) * S.z);
                const double fudi = VisFace * vdot(dU, Xpn);
                const double fvdi = VisFace * vdot(dV, Xpn);
                const double fwdi = VisFace * vdot(dW, Xpn);
                if (t == OUTLET && s->mdot[face] < 0.0) s->mdot[face] = 1e-15; /* :1576-1580 */
                const double f = -VisFace + smin(s->mdot[face], 0.0);
                s->AU[c0] = s->AU[c0] - f;
                s->SU[c0] = s->SU[c0] - f * UFace + fude - fudi;
                U[N + bc] = UFace;
                s->AV[c0] = s->AV[c0] - f;
                s->SV[c0] = s->SV[c0] - f * VFace + fvde - fvdi;
                V[N + bc] = VFace;
                s->AW[c0] = s->AW[c0] - f;
                s->SW[c0] = s->SW[c0] - f * WFace + fwde - fwdi;
                W[N + bc] = WFace;
            } else if (t == WALL) {
                const double Visac = mu;
                const v3 Xpn = vsub(ld3(s->fcen, face), ld3(s->cc, c0));
                const double coef = Visac * s->frl[face];
                const v3 Up = mk(U[c0] - 0., V[c0] - 0., W[c0] - 0.);
                const double dp = vdot(Up, vnorm(S));
                const v3 Ut = vsub(Up, vscale(vnorm(S), dp));
                const double Uvel = fabs(Ut.x) + fabs(Ut.y) + fabs(Ut.z);
                v3 force;
                if (Uvel > 0.0) {
                    const double distance = vmag(Xpn);
                    force = vdiv(vscale(Ut, s->farea[face] * Visac), distance);
                } else {
                    force = mk(0.0, 0.0, 0.0);
                }
                s->AU[c0] = s->AU[c0] + coef;
                s->AV[c0] = s->AV[c0] + coef;
                s->AW[c0] = s->AW[c0] + coef;
                s->SU[c0] = s->SU[c0] + coef * U[c0] - force.x;
                s->SV[c0] = s->SV[c0] + coef * V[c0] - force.y;
                s->SW[c0] = s->SW[c0] + coef * W[c0] - force.z;
                U[N + bc] = 0.;
                V[N + bc] = 0.;
                W[N + bc] = 0.;
            }
        }
    }
}

/* setup_sparse_matrix (FlowSolver.inl:1186-1297) into the matrix A / b. */
static void setup_sparse_matrix(mco_solver *s, double URF, double *Aphi, const double *phi, double *Sphi)
{
    const uint64_t N = s->N;
    const double RURF = 1. / URF;
    memset(s->valA, 0, (size_t)s->nnz * sizeof(double));
    memset(s->bA, 0, N * sizeof(double));
    for (uint64_t face = 0; face < s->F; face++) {
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        if (c1 >= N) continue;
        mat_set(s, s->valA, c0, c1, s->ff[2 * face + 1]);
        mat_set(s, s->valA, c1, c0, s->ff[2 * face]);
        Aphi[c0] -= s->ff[2 * face + 1];
        Aphi[c1] -= s->ff[2 * face];
    }
    for (uint64_t i = 0; i < N; i++) {
        Aphi[i] *= RURF;
        Sphi[i] = Sphi[i] + (1.0 - URF) * Aphi[i] * phi[i];
        mat_set(s, s->valA, i, i, Aphi[i]);
        s->bA[i] = Sphi[i];
    }
}

/* update_sparse_matrix (FlowSolver.inl:1299-1339): new diagonal and b only. */
static void update_sparse_matrix(mco_solver *s, double URF, double *Aphi, const double *phi, double *Sphi)
{
    const uint64_t N = s->N;
    const double RURF = 1. / URF;
    for (uint64_t face = 0; face < s->F; face++) {
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        if (c1 >= N) continue;
        Aphi[c0] -= s->ff[2 * face + 1];
        Aphi[c1] -= s->ff[2 * face];
    }
    for (uint64_t i = 0; i < N; i++) {
        Aphi[i] *= RURF;
        Sphi[i] = Sphi[i] + (1.0 - URF) * Aphi[i] * phi[i];
        mat_set(s, s->valA, i, i, Aphi[i]);
        s->bA[i] = Sphi[i];
    }
}

/* solve_sparse_matrix (FlowSolver.inl:1341-1375) */
static int solve_sparse_matrix(mco_solver *s, double *phi)
{
    return solve_bicgstab(s, s->valA, s->bA, phi, s->prm.u_rtol);
}

/* calculate_UVW (FlowSolver.inl:1655-1810); simple mode adds the particle
 * momentum the reference leaves commented out (:1723-1729). */
int mco_stage_calculate_uvw(mco_solver *s)
{
    const uint64_t N = s->N;
    for (uint64_t i = 0; i < N; i++) {
        s->AU[i] = 0.0; s->AV[i] = 0.0; s->AW[i] = 0.0;
        s->SU[i] = 0.0; s->SV[i] = 0.0; s->SW[i] = 0.0;
    }
    calculate_flux_UVW(s);
    const double *T = s->phi[MCO_TEM];
    for (uint64_t i = 0; i < N; i++) { /* buoyancy, :1689-1697 */
        const double BodyForce = -0.001 * s->rho[i] * s->vol[i] * (T[i] - s->prm.temperature0);
        const double gravity[3] = {0.0, -9.81, 0.0};
        s->SU[i] += gravity[0] * BodyForce;
        s->SV[i] += gravity[1] * BodyForce;
        s->SW[i] += gravity[2] * BodyForce;
    }
    const double *gP = s->grad[MCO_P];
    for (uint64_t i = 0; i < N; i++) { /* pressure force, :1700-1705 */
        s->SU[i] -= gP[3 * i] * s->vol[i];
        s->SV[i] -= gP[3 * i + 1] * s->vol[i];
        s->SW[i] -= gP[3 * i + 2] * s->vol[i];
    }
    const double rdelta = 1.0 / s->prm.delta;
    double *U = s->phi[MCO_U], *V = s->phi[MCO_V], *W = s->phi[MCO_W];
    for (uint64_t i = 0; i < N; i++) { /* transient, :1708-1721 */
        const double f = s->rho[i] * s->vol[i] * rdelta;
        s->SU[i] += f * U[i];
        s->SV[i] += f * V[i];
        s->SW[i] += f * W[i];
        s->AU[i] += f;
        s->AV[i] += f;
        s->AW[i] += f;
    }
    if (s->prm.mode == MCO_MODE_SIMPLE)
        for (uint64_t i = 0; i < N; i++) {
            s->SU[i] += s->src[5 * i];
            s->SV[i] += s->src[5 * i + 1];
            s->SW[i] += s->src[5 * i + 2];
        }
    const double urf = s->prm.urf_momentum;
    int bad = 0;
    setup_sparse_matrix(s, urf, s->AU, U, s->SU);
    s->stats.momentum_iters[0] = solve_sparse_matrix(s, U);
    update_sparse_matrix(s, urf, s->AV, V, s->SV);
    s->stats.momentum_iters[1] = solve_sparse_matrix(s, V);
    update_sparse_matrix(s, urf, s->AW, W, s->SW);
    s->stats.momentum_iters[2] = solve_sparse_matrix(s, W);
    for (int k = 0; k < 3; k++) bad |= s->stats.momentum_iters[k] < 0;
    return bad ? -1 : 0;
}

/* ---------------------------------------------------------------- pressure */

/* update_mass_flux (FlowSolver.inl:1812-1878) */
static void update_mass_flux(mco_solver *s)
{
    const uint64_t N = s->N;
    const double *gPP = s->grad[MCO_PP];
    for (uint64_t face = 0; face < s->F; face++) {
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        if (c1 >= N) continue;
        const v3 fc = ld3(s->fcen, face), S = ld3(s->fnorm, face);
        const v3 x0 = ld3(s->cc, c0), x1 = ld3(s->cc, c1);
        const v3 Xpac = vsub(fc, vscale(vnorm(S), vdot(vsub(fc, x0), vnorm(S))));
        const v3 Xnac = vsub(fc, vscale(vnorm(S), vdot(vsub(fc, x1), vnorm(S))));
        v3 Xn = vsub(Xnac, x1);
        v3 Xp = vsub(Xpac, x0);
        if (fabs(Xn.x) < 0.0000000000000003) Xn.x = 0.0;
        if (fabs(Xn.y) < 0.0000000000000003) Xn.y = 0.0;
        if (fabs(Xn.z) < 0.0000000000000003) Xn.z = 0.0;
        if (fabs(Xp.x) < 0.0000000000000003) Xp.x = 0.0;
        if (fabs(Xp.y) < 0.0000000000000003) Xp.y = 0.0;
        if (fabs(Xp.z) < 0.0000000000000003) Xp.z = 0.0;
        const double fact = s->ff[2 * face];
        const double dpx = gPP[3 * c1] * Xn.x - gPP[3 * c0] * Xp.x;
        const double dpy = gPP[3 * c1 + 1] * Xn.y - gPP[3 * c0 + 1] * Xp.y;
        const double dpz = gPP[3 * c1 + 2] * Xn.z - gPP[3 * c0 + 2] * Xp.z;
        const double fc_ = fact * (dpx + dpy + dpz) * s->prm.flux_corr;
        s->mdot[face] += fc_;
        s->SU[c0] -= fc_;
        s->SU[c1] += fc_;
    }
}

/* calculate_mass_flux (FlowSolver.inl:1880-2104).  Simple mode: zero-gradient
 * outlet flux from the owner cell velocity, outlet fluxes scaled so that the
 * boundary balance matches the particle mass source, and the mass source
 * added to the continuity right-hand side. */
static void calculate_mass_flux(mco_solver *s)
{
    const uint64_t N = s->N;
    const int simple = s->prm.mode == MCO_MODE_SIMPLE;
    const double *U = s->phi[MCO_U], *V = s->phi[MCO_V], *W = s->phi[MCO_W], *P = s->phi[MCO_P];
    const double *gU = s->grad[MCO_U], *gV = s->grad[MCO_V], *gW = s->grad[MCO_W], *gP = s->grad[MCO_P];
    for (uint64_t face = 0; face < s->F; face++) {
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        const v3 S = ld3(s->fnorm, face);
        if (c1 < N) {
            const double lambda0 = s->flam[face];
            const double lambda1 = 1.0 - lambda0;
            const v3 dU = vadd(vscale(ld3(gU, c0), lambda0), vscale(ld3(gU, c1), lambda1));
            const v3 dV = vadd(vscale(ld3(gV, c0), lambda0), vscale(ld3(gV, c1), lambda1));
            const v3 dW = vadd(vscale(ld3(gW, c0), lambda0), vscale(ld3(gW, c1), lambda1));
            const v3 x0 = ld3(s->cc, c0), x1 = ld3(s->cc, c1), fc = ld3(s->fcen, face);
            const v3 Xac = vadd(vscale(x1, lambda1), vscale(x0, lambda0));
            const v3 delta = vsub(fc, Xac);
            const double UFace = U[c1] * lambda1 + U[c0] * lambda0 + vdot(dU, delta);
            const double VFace = V[c1] * lambda1 + V[c0] * lambda0 + vdot(dV, delta);
            const double WFace = W[c1] * lambda1 + W[c0] * lambda0 + vdot(dW, delta);
            const double densityf = s->rho[c0] * lambda0 + s->rho[c1] * lambda1;
            s->mdot[face] = densityf * (UFace * S.x + VFace * S.y + WFace * S.z);
            const v3 Xpac = vsub(fc, vscale(vnorm(S), vdot(vsub(fc, x0), vnorm(S))));
            const v3 Xnac = vsub(fc, vscale(vnorm(S), vdot(vsub(fc, x1), vnorm(S))));
            const v3 delp = vsub(Xpac, x0);
            const v3 deln = vsub(Xnac, x1);
            const double cell0_P = P[c0] + vdot(ld3(gP, c0), delp);
            const double cell1_P = P[c1] + vdot(ld3(gP, c1), deln);
            const v3 Xpn = vsub(Xnac, Xpac);
            const v3 Xpn2 = vsub(x1, x0);
            const double ApV0 = (s->AU[c0] != 0.0) ? 1.0 / s->AU[c0] : 0.0;
            const double ApV1 = (s->AU[c1] != 0.0) ? 1.0 / s->AU[c1] : 0.0;
            double ApV = s->rho[c0] * ApV0 * lambda0 + s->rho[c1] * ApV1 * lambda1;
            const double volume_avg = s->vol[c0] * lambda0 + s->vol[c1] * lambda1;
            ApV = ApV * s->farea[face] * volume_avg / vdot(Xpn2, vnorm(S));
            const double dpx = (gP[3 * c1] * lambda1 + gP[3 * c0] * lambda0) * Xpn.x;
            const double dpy = (gP[3 * c1 + 1] * lambda1 + gP[3 * c0 + 1] * lambda0) * Xpn.y;
            const double dpz = (gP[3 * c1 + 2] * lambda1 + gP[3 * c0 + 2] * lambda0) * Xpn.z;
            s->ff[2 * face] = -ApV;
            s->ff[2 * face + 1] = -ApV;
            s->mdot[face] -= ApV * ((cell1_P - cell0_P) - dpx - dpy - dpz);
        } else {
            const int t = (int)s->btype[c1 - N];
            if (t == INLET) {
                const v3 vin = mk(s->prm.inlet_u, 0.0, 0.0);
                const double Din = s->prm.density;
                s->mdot[face] = Din * vdot(vin, S);
                s->SU[c0] = s->SU[c0] - s->mdot[face];
            } else if (t == OUTLET) {
                const v3 vout = simple ? mk(U[c0], V[c0], W[c0]) : mk(s->prm.inlet_u, 0.0, 0.0);
                const double Din = s->prm.density;
                s->mdot[face] = Din * vdot(vout, S);
                if (s->mdot[face] < 0.0) { /* :1989-2000 (TE/ED slots are not restated) */
                    s->mdot[face] = 1e-15;
                    s->phi[MCO_TEM][c1] = s->phi[MCO_TEM][c0];
                }
            } else if (t == WALL) {
                s->mdot[face] = 0.0;
            }
        }
    }
    double FlowOut = 0.0, FlowIn = 0.0, areaout = 0.0;
    for (uint64_t face = 0; face < s->F; face++) { /* :2014-2030 */
        const uint64_t c1 = s->faces[2 * face + 1];
        if (c1 < N) continue;
        const int t = (int)s->btype[c1 - N];
        if (t == INLET) FlowIn += s->mdot[face];
        else if (t == OUTLET) { FlowOut += s->mdot[face]; areaout += s->farea[face]; }
    }
    double msrc = 0.0;
    if (simple)
        for (uint64_t i = 0; i < N; i++) msrc += s->src[5 * i + 4];
    if (FlowOut < 0.0000000001) { /* :2049-2079 */
        const double ratearea = -FlowIn / areaout;
        FlowOut = 0.0;
        for (uint64_t face = 0; face < s->F; face++) {
            const uint64_t c1 = s->faces[2 * face + 1];
            if (c1 < N) continue;
            const uint64_t bc = c1 - N;
            if ((int)s->btype[bc] == OUTLET) {
                s->mdot[face] = ratearea * s->farea[face];
                s->phi[MCO_U][N + bc] = s->prm.inlet_u;
                s->phi[MCO_V][N + bc] = 0.0;
                s->phi[MCO_W][N + bc] = 0.0;
                FlowOut += s->mdot[face];
            }
        }
    } else if (simple) {
        const double fact = (msrc - FlowIn) / FlowOut;
        for (uint64_t face = 0; face < s->F; face++) {
            const uint64_t c1 = s->faces[2 * face + 1];
            if (c1 < N || (int)s->btype[c1 - N] != OUTLET) continue;
            s->mdot[face] *= fact;
        }
    }
    for (uint64_t face = 0; face < s->F; face++) { /* :2084-2103 */
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        if (c1 < N || (int)s->btype[c1 - N] != OUTLET) continue;
        s->SU[c0] -= s->mdot[face];
    }
    if (simple)
        for (uint64_t i = 0; i < N; i++) s->SU[i] += s->src[5 * i + 4];
}

/* setup_pressure_matrix (FlowSolver.inl:2106-2201): into Pressure_A while
 * first_pressure, otherwise into A (compat).  Simple mode always writes the
 * pressure-correction system. */
static void setup_pressure_matrix(mco_solver *s)
{
    const uint64_t N = s->N;
    const int to_pressure = s->first_pressure || s->prm.mode == MCO_MODE_SIMPLE;
    double *val = to_pressure ? s->valP : s->valA;
    memset(val, 0, (size_t)s->nnz * sizeof(double));
    for (uint64_t face = 0; face < s->F; face++) {
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        if (c1 >= N) continue;
        mat_set(s, val, c0, c1, s->ff[2 * face + 1]);
        mat_set(s, val, c1, c0, s->ff[2 * face]);
        s->SU[c0] -= s->mdot[face];
        s->SU[c1] += s->mdot[face];
        s->AV[c0] -= s->ff[2 * face + 1];
        s->AV[c1] -= s->ff[2 * face];
    }
    for (uint64_t i = 0; i < N; i++) mat_set(s, val, i, i, s->AV[i]);
}

/* solve_pressure_matrix (FlowSolver.inl:2203-2273): the right-hand side goes
 * to Pressure_b only while first_pressure; the solve always uses Pressure_A
 * and Pressure_b (compat).  Simple mode loads the current S_U every time. */
static int solve_pressure_matrix(mco_solver *s, int loop_num)
{
    const uint64_t N = s->N;
    const int simple = s->prm.mode == MCO_MODE_SIMPLE;
    if (s->first_pressure || simple) memcpy(s->bP, s->SU, N * sizeof(double));
    else memcpy(s->bA, s->SU, N * sizeof(double));
    double bnorm = 0.0;
    const double floor = (simple && loop_num > 1) ? s->prm.p_rtol * s->p_bnorm_ref : 0.0;
    const int its = solve_cg_projected(s, s->valP, s->bP, s->phi[MCO_PP], s->prm.p_rtol, floor, &bnorm);
    if (loop_num == 1) s->p_bnorm_ref = bnorm;
    s->stats.pressure_solves++;
    s->stats.pressure_iters_total += its < 0 ? -its : its;
    if (loop_num == 1) s->stats.pressure_iters_first = its;
    return its;
}

/* Update_P_at_boundaries (FlowSolver.inl:2275-2290) */
static void update_P_at_boundaries(mco_solver *s, double *phi)
{
    for (uint64_t face = 0; face < s->F; face++) {
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        if (c1 < s->N) continue;
        phi[c1] = phi[c0]; /* c1 = N + boundary cell */
    }
}

/* update_P (FlowSolver.inl:2292-2315) */
static void update_P(mco_solver *s, double *phi, const double *grad)
{
    for (uint64_t face = 0; face < s->F; face++) {
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        if (c1 < s->N) continue;
        if ((int)s->btype[c1 - s->N] == OUTLET) phi[c1] = phi[c0];
        else {
            const v3 ds = vsub(ld3(s->fcen, face), ld3(s->cc, c0));
            phi[c1] = phi[c0] + vdot(ld3(grad, c0), ds);
        }
    }
}

/* calculate_pressure (FlowSolver.inl:2317-2514) */
int mco_stage_calculate_pressure(mco_solver *s)
{
    const uint64_t N = s->N;
    const int simple = s->prm.mode == MCO_MODE_SIMPLE;
    int Loop_num = 0, cont = 1, bad = 0;
    double pc_max = 0, pc_ref = 0;
    for (uint64_t i = 0; i < N; i++) { s->AV[i] = 0.0; s->SU[i] = 0.0; }
    for (uint64_t f = 0; f < s->F; f++) { s->mdot[f] = 0.0; s->ff[2 * f] = 0.0; s->ff[2 * f + 1] = 0.0; }
    calculate_mass_flux(s);
    setup_pressure_matrix(s);
    double *PP = s->phi[MCO_PP], *P = s->phi[MCO_P];
    double *U = s->phi[MCO_U], *V = s->phi[MCO_V], *W = s->phi[MCO_W];
    const double *gPP = s->grad[MCO_PP];
    while (cont) {
        Loop_num++;
        if (solve_pressure_matrix(s, Loop_num) < 0) bad = 1;
        pc_max = PP[0];
        for (uint64_t i = 1; i < N; i++)
            if (fabs(PP[i]) > pc_max) pc_max = fabs(PP[i]);
        if (Loop_num == 1) { pc_ref = pc_max; s->stats.pressure_correction_max_first = pc_max; }
        update_P_at_boundaries(s, PP);
        single_gradient_pressure(s, MCO_PP);
        for (uint64_t face = 0; face < s->F; face++) {
            const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
            if (c1 >= N) continue;
            s->mdot[face] += (s->ff[2 * face] * (PP[c1] - PP[c0]));
        }
        for (uint64_t c = 0; c < N; c++) {
            const double Ar = (s->AU[c] != 0.0) ? 1.0 / s->AU[c] : 0.0;
            const double fact = s->vol[c] * Ar;
            if (simple) {
                P[c] += s->prm.urf_pressure * PP[c];
                U[c] -= gPP[3 * c] * fact;
                V[c] -= gPP[3 * c + 1] * fact;
                W[c] -= gPP[3 * c + 2] * fact;
            } else if (s->first_pressure) {
                P[c] += s->prm.urf_pressure * PP[c];
                U[c] -= gPP[3 * c] * fact;
                V[c] -= gPP[3 * c + 1] * fact;
                W[c] -= gPP[3 * c + 2] * fact;
                s->first_pressure = 0;
            }
        }
        for (uint64_t i = 0; i < N; i++) s->SU[i] = 0.0;
        update_mass_flux(s);
        for (uint64_t i = 0; i < N + 6; i++) PP[i] = 0.0;
        if (Loop_num >= 4 || pc_max <= 0.25 * pc_ref) cont = 0;
    }
    update_P_at_boundaries(s, P);
    single_gradient_pressure(s, MCO_P);
    update_P(s, P, s->grad[MCO_P]);
    return bad ? -1 : 0;
}

/* --------------------------------------------------------- scalar transports */

/* Scalar types of Scalar_solve (utils.hpp:31-37). */
enum { SC_TERBTE = 0, SC_TERBED = 1, SC_TEMP = 2, SC_FUEL = 3, SC_PROG = 4, SC_VARFU = 5, SC_VARPR = 6 };

static int scalar_type_of_field(int field)
{
    switch (field) {
    case MCO_TE: return SC_TERBTE;
    case MCO_ED: return SC_TERBED;
    case MCO_TEM: return SC_TEMP;
    case MCO_FUL: return SC_FUEL;
    case MCO_PRO: return SC_PROG;
    case MCO_VARF: return SC_VARFU;
    case MCO_VARP: return SC_VARPR;
    default: return -1;
    }
}

/* Effective diffusivity of a scalar from Visac = (face viscosity - mu)
 * (FluxScalar, FlowSolver.inl:2543-2561, repeated at :2663-2681 and :2703-2721). */
static double scalar_visac(int type, double mu, double Visac)
{
    if (type == SC_TEMP) return (mu + Visac / 0.9) / 0.6905;
    if (type == SC_TERBTE) return mu + Visac;
    if (type == SC_TERBED) return mu + Visac / 1.219;
    return (mu + Visac / 0.9) / 0.9;
}

/* Inlet value of a scalar (FluxScalar, FlowSolver.inl:2625-2659). */
static double scalar_inlet(const mco_solver *s, int type)
{
    const double velmag2 = pow(s->prm.inlet_u, 2) + pow(0.0, 2) + pow(0.0, 2);
    switch (type) {
    case SC_TEMP: return s->prm.temperature0;
    case SC_TERBTE: return 3.0 / 2.0 * ((0.1 * 0.1) * velmag2);
    case SC_TERBED: return pow(0.09, 0.75) * pow((3.0 / 2.0 * ((0.1 * 0.1) * velmag2)), 1.5);
    case SC_FUEL: return 0.1;
    case SC_VARFU: return 0.1;
    default: return 0.0; /* PROG, VARPR */
    }
}

/* FluxScalar (FlowSolver.inl:2516-2744): implicit upwind convection and
 * diffusion into face_fields, explicit diffusion into S_phi.U, boundary
 * values and inlet coefficients into A_phi.V. */
static void flux_scalar(mco_solver *s, int type, double *phi, const double *g)
{
    const uint64_t N = s->N;
    const double mu = s->eff_visc;
    const double GammaBlend = 0.0;
    for (uint64_t face = 0; face < s->F; face++) {
        const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
        const v3 S = ld3(s->fnorm, face);
        const double md = s->mdot[face];
        if (c1 < N) {
            const double lambda0 = s->flam[face];
            const double lambda1 = 1.0 - lambda0;
            double Visac = mu * lambda0 + mu * lambda1;
            Visac -= mu;
            Visac = scalar_visac(type, mu, Visac);
            const v3 dPhi = vadd(vscale(ld3(g, c0), lambda0), vscale(ld3(g, c1), lambda1));
            const v3 Xpn = vsub(ld3(s->cc, c1), ld3(s->cc, c0));
            const double VisFace = Visac * s->frl[face];
            const double PhiFace = (md >= 0.0) ? phi[c0] : phi[c1];
            const double fce = md * PhiFace;
            const double fde1 = Visac * vdot(dPhi, S);
            const double fci = smin(md, 0.0) * phi[c0] + smax(md, 0.0) * phi[c1];
            const double fdi = VisFace * vdot(dPhi, Xpn);
            s->ff[2 * face] = -VisFace - smax(md, 0.0);
            s->ff[2 * face + 1] = -VisFace + smin(md, 0.0);
            const double blend = GammaBlend * (fce - fci);
            s->SU[c0] = s->SU[c0] - blend + fde1 - fdi;
            s->SU[c1] = s->SU[c1] + blend - fde1 + fdi;
        } else {
            const uint64_t bc = c1 - N;
            const int t = (int)s->btype[bc];
            const v3 dPhi = ld3(g, c0);
            const v3 Xpn = vsub(ld3(s->fcen, face), ld3(s->cc, c0));
            if (t == INLET) {
                const double PhiFace = scalar_inlet(s, type);
                double Visac = s->inlet_eff_visc;
                Visac -= mu;
                Visac = scalar_visac(type, mu, Visac);
                const double VisFace = Visac * s->frl[face];
                const double fde = Visac * vdot(dPhi, S);
                const double fdi = VisFace * vdot(dPhi, Xpn);
                const double f = -VisFace + smin(md, 0.0);
                s->AV[c0] = s->AV[c0] - f;
                s->SU[c0] = s->SU[c0] - f * PhiFace + fde - fdi;
                phi[N + bc] = PhiFace;
            } else if (t == OUTLET) {
                double Visac = mu;
                Visac -= mu;
                Visac = scalar_visac(type, mu, Visac);
                const double PhiFace = phi[c0] + vdot(dPhi, Xpn);
                const double VisFace = Visac * s->frl[face];
                const double fde = Visac * vdot(dPhi, S);
                const double fdi = VisFace * vdot(dPhi, Xpn);
                s->SU[c0] = s->SU[c0] + fde - fdi;
                phi[N + bc] = PhiFace;
            } else if (t == WALL) {
                /* the reference's condition (type != TERBTE or type != TERBED) always holds */
                phi[N + bc] = phi[c0];
            }
        }
    }
}

/* solveTurbulenceModels (FlowSolver.inl:2746-2883): k production and
 * dissipation with the wall-function production at wall cells (TERBTE);
 * epsilon sources and the fixed wall-cell dissipation, whose rows are
 * decoupled by zeroing their side of face_fields (TERBED). */
static void solve_turbulence(mco_solver *s, int type)
{
    const uint64_t N = s->N;
    const double mu = s->eff_visc;
    double *TE = s->phi[MCO_TE], *ED = s->phi[MCO_ED], *TP = s->phi[MCO_TP];
    const double Cmu = 0.09;
    const double Cmu75 = pow(Cmu, 0.75);
    if (type == SC_TERBTE) {
        const double *gU = s->grad[MCO_U], *gV = s->grad[MCO_V], *gW = s->grad[MCO_W];
        for (uint64_t i = 0; i < N; i++) {
            const v3 dU = ld3(gU, i), dV = ld3(gV, i), dW = ld3(gW, i);
            const double s1 = (dU.x + dU.x) * dU.x + (dU.y + dV.x) * dU.y + (dU.z + dW.x) * dU.z;
            const double s2 = (dV.x + dU.y) * dV.x + (dV.y + dV.y) * dV.y + (dV.z + dW.y) * dV.z;
            const double s3 = (dW.x + dU.z) * dW.x + (dW.y + dV.z) * dW.y + (dW.z + dW.z) * dW.z;
            const double VisT = mu - mu;
            const double Pk = VisT * (s1 + s2 + s3);
            TP[i] = Pk;
            const double Dis = s->rho[i] * ED[i];
            s->SU[i] = s->SU[i] + TP[i] * s->vol[i];
            s->AV[i] = s->AV[i] + Dis / (TE[i] + 0.000000000000000001) * s->vol[i];
        }
        for (uint64_t face = 0; face < s->F; face++) {
            const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
            if (c1 < N) continue;
            const uint64_t bc = c1 - N;
            if ((int)s->btype[bc] != WALL) continue;
            s->SU[c0] = s->SU[c0] - TP[c0] * s->vol[c0];
            const double Visc = mu;
            const v3 Xpn = vsub(ld3(s->fcen, face), ld3(s->cc, c0));
            const v3 Up = mk(s->phi[MCO_U][c0] - 0., s->phi[MCO_V][c0] - 0., s->phi[MCO_W][c0] - 0.);
            const v3 nrm = vnorm(ld3(s->fnorm, face));
            const double dp = vdot(Up, nrm);
            const v3 Ut = vsub(Up, vscale(nrm, dp));
            const double Uvel = sqrt(vdot(Ut, Ut));
            const double distance_to_face = vmag(Xpn);
            const double rkapdn = 1.0 / (0.419 * distance_to_face);
            const double Tau_w = Visc * Uvel / distance_to_face;
            const double Utau = sqrt(Tau_w / s->rho[c0]);
            TP[c0] = Tau_w * Utau * rkapdn;
            TE[N + bc] = TE[c0];
            s->SU[c0] = s->SU[c0] + TP[c0] * s->vol[c0];
            const double DisP = Cmu75 * sqrt(TE[c0]) * rkapdn;
            s->AV[c0] = s->AV[c0] + s->rho[c0] * DisP * s->vol[c0];
        }
    } else if (type == SC_TERBED) {
        for (uint64_t i = 0; i < N; i++) {
            const double fact = ED[i] / (TE[i] + 0.000000000000000001) * s->vol[i];
            s->SU[i] = s->SU[i] + 1.44 * fact * TP[i];
            s->AV[i] = s->AV[i] + 1.92 * fact * s->rho[i];
        }
        for (uint64_t face = 0; face < s->F; face++) {
            const uint64_t c0 = s->faces[2 * face], c1 = s->faces[2 * face + 1];
            if (c1 < N) continue;
            const uint64_t bc = c1 - N;
            if ((int)s->btype[bc] != WALL) continue;
            const double turb = TE[c0];
            const double distance = vmag(vsub(ld3(s->fcen, face), ld3(s->cc, c0)));
            const double Dis = Cmu75 * pow(turb, 1.5) / (distance * 0.419);
            for (int j = 0; j < 6; j++) {
                const uint64_t nf = s->cell_faces[6 * c0 + j];
                const uint64_t a = s->faces[2 * nf], b = s->faces[2 * nf + 1];
                if (a < N && b < N) {
                    if (a == c0) s->ff[2 * nf + 1] = 0.0;
                    else if (b == c0) s->ff[2 * nf] = 0.0;
                }
            }
            ED[c0] = Dis;
            s->SU[c0] = Dis;
            s->AV[c0] = 1;
            ED[N + bc] = ED[c0];
        }
    }
}

/* Scalar_solve (FlowSolver.inl:2885-3076) for one scalar: fluxes, the
 * unsteady term, turbulence sources, the system with its under-relaxation,
 * BiCGStab, and for k and epsilon the replacement of negative values by the
 * mean of the internal neighbours (:2956-2985).  Simple mode adds the
 * particle energy to T (left commented out in the reference, :2919-2925). */
int mco_stage_scalar(mco_solver *s, int field)
{
    const int type = scalar_type_of_field(field);
    if (type < 0 || !s->grad[field]) return -1;
    const uint64_t N = s->N;
    double *phi = s->phi[field];
    for (uint64_t i = 0; i < N; i++) { s->AV[i] = 0.0; s->SU[i] = 0.0; }
    flux_scalar(s, type, phi, s->grad[field]);
    const double rdelta = 1.0 / s->prm.delta;
    for (uint64_t i = 0; i < N; i++) {
        const double f = s->rho[i] * s->vol[i] * rdelta;
        s->SU[i] += f * phi[i];
        s->AV[i] += f;
    }
    if (type == SC_TEMP && s->prm.mode == MCO_MODE_SIMPLE)
        for (uint64_t i = 0; i < N; i++) s->SU[i] += s->src[5 * i + 3];
    if (type == SC_TERBTE || type == SC_TERBED) solve_turbulence(s, type);
    double underrelax;
    if (type == SC_TERBTE || type == SC_TERBED) underrelax = 0.5;
    else if (type == SC_TEMP) underrelax = s->prm.urf_temperature;
    else underrelax = 0.95;
    setup_sparse_matrix(s, underrelax, s->AV, phi, s->SU);
    const int its = solve_sparse_matrix(s, phi);
    if (type == SC_TERBTE || type == SC_TERBED) {
        for (uint64_t i = 0; i < N; i++) {
            int count = 0;
            double phisum = 0.0;
            if (phi[i] < 0.0) {
                for (int j = 0; j < 6; j++) {
                    const uint64_t nb = s->cell_nbrs[6 * i + j];
                    if (nb < N) {
                        count++;
                        phisum += phi[nb];
                    }
                }
                phisum = (phisum / count);
                phi[i] = smax(phisum, 0.000000000001);
            }
        }
    }
    if (type == SC_TEMP) s->stats.temperature_iters = its;
    else s->stats.scalar_iters[type < SC_TEMP ? type : type - 1] = its;
    return its < 0 ? -1 : 0;
}

int mco_stage_scalar_temperature(mco_solver *s) { return mco_stage_scalar(s, MCO_TEM); }

/* ---------------------------------------------------------------- the pass */

static double mass_imbalance(const mco_solver *s)
{
    const uint64_t N = s->N;
    double *div = (double *)calloc(N, sizeof(double));
    for (uint64_t f = 0; f < s->F; f++) {
        const uint64_t c0 = s->faces[2 * f], c1 = s->faces[2 * f + 1];
        div[c0] += s->mdot[f];
        if (c1 < N) div[c1] -= s->mdot[f];
    }
    double m = 0.0;
    for (uint64_t i = 0; i < N; i++) {
        const double r = fabs(div[i] - (s->prm.mode == MCO_MODE_SIMPLE ? s->src[5 * i + 4] : 0.0));
        if (r > m) m = r;
    }
    free(div);
    return m;
}

/* One iteration of the loop in FlowSolver::timestep (FlowSolver.inl:3188-3268):
 * the coupled fields, and with params.scalars the other six scalar transports
 * in the reference's order.  The FGM lookup (:1138-1184) is not restated: it
 * only writes S_phi.U, which every later stage zeroes before use. */
int mco_pass(mco_solver *s)
{
    const int i = s->pass_in_step;
    memset(&s->stats, 0, sizeof(s->stats));
    mco_stage_gradients(s);
    if (s->timestep_count == 0 && i == 0) mco_stage_set_up_field(s);
    int rc = 0;
    rc |= mco_stage_calculate_uvw(s);
    rc |= mco_stage_calculate_pressure(s);
    if (s->prm.scalars) {
        static const int order[7] = {MCO_TE, MCO_ED, MCO_TEM, MCO_FUL, MCO_PRO, MCO_VARF, MCO_VARP};
        for (int k = 0; k < 7; k++) rc |= mco_stage_scalar(s, order[k]);
    } else {
        rc |= mco_stage_scalar_temperature(s);
    }
    s->stats.mass_imbalance = mass_imbalance(s);
    s->pass_in_step++;
    if (s->pass_in_step == 3) {
        s->pass_in_step = 0;
        s->timestep_count++;
    }
    return rc;
}
