// Implementation of the single-rank MPI type table and the sequential PETSc
// subset declared in petscksp.h.  Test infrastructure only (see petscksp.h for
// the solver semantics this file defines).
#include "petscksp.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>

MPI_Comm PETSC_COMM_WORLD = MPI_COMM_WORLD;

// ---------------------------------------------------------------- MPI types
static std::vector<int> g_type_sizes;

extern "C" int mcshim_type_size(MPI_Datatype t)
{
    switch (t) {
    case 1: return 1;
    case 4: return 4;
    case 5: return 4;
    case 8: return 8;
    case 9: return 8;
    case 10: return 8;
    default: break;
    }
    if (t >= 100 && (size_t)(t - 100) < g_type_sizes.size()) return g_type_sizes[t - 100];
    return 0;
}

extern "C" MPI_Datatype mcshim_type_register(int bytes)
{
    g_type_sizes.push_back(bytes);
    return (MPI_Datatype)(100 + (int)g_type_sizes.size() - 1);
}

// ------------------------------------------------- staged point-to-point
// Messages from fake particle ranks for update_flow_field: per rank, tag 0
// carries uint64 cell indexes and tag 2 the particle_aos rows.  Sends are
// recorded as (destination, tag, bytes).
struct StagedRank {
    int rank;
    std::vector<char> part[3];
    bool probed = false;
};
static std::vector<StagedRank> g_staged;
struct SentMessage {
    int dst, tag;
    std::vector<char> data;
};
static std::vector<SentMessage> g_outbox;

extern "C" void mcshim_inject_reset()
{
    g_staged.clear();
    g_outbox.clear();
}

extern "C" void mcshim_inject_rank(int rank, long n, const uint64_t *cells, const double *aos, int aos_doubles)
{
    StagedRank r;
    r.rank = rank;
    r.part[0].assign((const char *)cells, (const char *)cells + n * sizeof(uint64_t));
    r.part[2].assign((const char *)aos, (const char *)aos + n * aos_doubles * sizeof(double));
    g_staged.push_back(r);
}

extern "C" int mcshim_iprobe(int *flag, MPI_Status *st)
{
    *flag = 0;
    for (StagedRank &r : g_staged) {
        if (r.probed) continue;
        r.probed = true;
        *flag = 1;
        if (st) {
            st->MPI_SOURCE = r.rank;
            st->MPI_TAG = 0;
            st->_ucount = r.part[0].size();
        }
        return 0;
    }
    return 0;
}

extern "C" int mcshim_irecv(void *buf, size_t bytes, int src, int tag)
{
    for (StagedRank &r : g_staged) {
        if (r.rank != src || (tag != 0 && tag != 2) || r.part[tag].size() < bytes) continue;
        std::memcpy(buf, r.part[tag].data(), bytes);
        return 0;
    }
    std::fprintf(stderr, "mpi shim: no staged message from %d with tag %d\n", src, tag);
    std::abort();
}

extern "C" int mcshim_isend(const void *buf, size_t bytes, int dst, int tag)
{
    SentMessage m{dst, tag, std::vector<char>((const char *)buf, (const char *)buf + bytes)};
    g_outbox.push_back(std::move(m));
    return 0;
}

extern "C" long mcshim_outbox_count() { return (long)g_outbox.size(); }

// Message i of the outbox: destination, tag and size; copies the bytes when out is given.
extern "C" long mcshim_outbox_get(long i, int *dst, int *tag, void *out)
{
    if (i < 0 || (size_t)i >= g_outbox.size()) return -1;
    const SentMessage &m = g_outbox[i];
    *dst = m.dst;
    *tag = m.tag;
    if (out) std::memcpy(out, m.data.data(), m.data.size());
    return (long)m.data.size();
}

// ---------------------------------------------------------------- PETSc
struct mcshim_Mat {
    PetscInt n = 0;
    std::vector<std::map<PetscInt, double>> rows;
};
struct mcshim_Vec {
    std::vector<double> v;
};
struct mcshim_PC {
    std::string type = PCNONE;
};
struct mcshim_KSP {
    std::string type = KSPBCGS;
    mcshim_PC pc;
    Mat A = nullptr;
    int reason = 0;
    int iters = 0;
};

static double g_bcgs_rtol = 1e-13;
static double g_cg_rtol = 1e-13;
static int g_max_iters = 100000;
static int g_last_iters = 0;
static double g_last_relres = 0.0;
static int g_last_kind = -1;
static long g_count_bcgs = 0, g_count_cg = 0;

extern "C" void mcshim_set_tolerances(double bcgs_rtol, double cg_rtol, int max_iters)
{
    g_bcgs_rtol = bcgs_rtol;
    g_cg_rtol = cg_rtol;
    g_max_iters = max_iters;
}
extern "C" void mcshim_last_solve(int *iters, double *rel_residual, int *kind)
{
    *iters = g_last_iters;
    *rel_residual = g_last_relres;
    *kind = g_last_kind;
}
extern "C" void mcshim_solve_counts(long *bcgs, long *cg)
{
    *bcgs = g_count_bcgs;
    *cg = g_count_cg;
}

PetscErrorCode PetscInitialize(int *, char ***, const char *, const char *) { return 0; }
PetscErrorCode PetscFinalize(void) { return 0; }

PetscErrorCode MatCreate(MPI_Comm, Mat *A) { *A = new mcshim_Mat(); return 0; }
PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt, PetscInt, PetscInt)
{
    A->n = m;
    A->rows.assign((size_t)m, {});
    return 0;
}
PetscErrorCode MatSetFromOptions(Mat) { return 0; }
PetscErrorCode MatSeqAIJSetPreallocation(Mat, PetscInt, const PetscInt[]) { return 0; }
PetscErrorCode MatMPIAIJSetPreallocation(Mat, PetscInt, const PetscInt[], PetscInt, const PetscInt[]) { return 0; }
PetscErrorCode MatSetUp(Mat) { return 0; }
PetscErrorCode MatDuplicate(Mat A, MatDuplicateOption op, Mat *B)
{
    Mat C = new mcshim_Mat(*A);
    if (op == MAT_DO_NOT_COPY_VALUES)
        for (auto &row : C->rows)
            for (auto &kv : row) kv.second = 0.0;
    *B = C;
    return 0;
}
PetscErrorCode MatZeroEntries(Mat A)
{
    for (auto &row : A->rows)
        for (auto &kv : row) kv.second = 0.0;
    return 0;
}
PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode mode)
{
    if (i < 0 || i >= A->n || j < 0 || j >= A->n) {
        fprintf(stderr, "mcshim: MatSetValue(%d,%d) outside %d x %d\n", i, j, A->n, A->n);
        abort();
    }
    if (mode == ADD_VALUES)
        A->rows[(size_t)i][j] += v;
    else
        A->rows[(size_t)i][j] = v;
    return 0;
}
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatGetOwnershipRange(Mat A, PetscInt *first, PetscInt *last)
{
    *first = 0;
    *last = A->n;
    return 0;
}
PetscErrorCode MatDestroy(Mat *A) { delete *A; *A = nullptr; return 0; }

PetscErrorCode VecCreate(MPI_Comm, Vec *v) { *v = new mcshim_Vec(); return 0; }
PetscErrorCode VecSetSizes(Vec v, PetscInt n, PetscInt) { v->v.assign((size_t)n, 0.0); return 0; }
PetscErrorCode VecSetFromOptions(Vec) { return 0; }
PetscErrorCode VecDuplicate(Vec v, Vec *w) { *w = new mcshim_Vec(); (*w)->v.assign(v->v.size(), 0.0); return 0; }
PetscErrorCode VecZeroEntries(Vec v) { std::fill(v->v.begin(), v->v.end(), 0.0); return 0; }
PetscErrorCode VecSetValue(Vec v, PetscInt i, PetscScalar x, InsertMode mode)
{
    if (i < 0 || (size_t)i >= v->v.size()) abort();
    if (mode == ADD_VALUES)
        v->v[(size_t)i] += x;
    else
        v->v[(size_t)i] = x;
    return 0;
}
PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
PetscErrorCode VecGetValues(Vec v, PetscInt n, const PetscInt idx[], PetscScalar y[])
{
    for (PetscInt i = 0; i < n; i++) y[i] = v->v[(size_t)idx[i]];
    return 0;
}
PetscErrorCode VecDestroy(Vec *v) { delete *v; *v = nullptr; return 0; }

PetscErrorCode KSPCreate(MPI_Comm, KSP *ksp) { *ksp = new mcshim_KSP(); return 0; }
PetscErrorCode KSPSetType(KSP ksp, KSPType type) { ksp->type = type; return 0; }
PetscErrorCode KSPGetPC(KSP ksp, PC *pc) { *pc = &ksp->pc; return 0; }
PetscErrorCode PCSetType(PC pc, PCType type) { pc->type = type; return 0; }
PetscErrorCode KSPSetPC(KSP ksp, PC pc)
{
    if (pc != &ksp->pc) ksp->pc = *pc;
    return 0;
}
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat) { ksp->A = A; return 0; }
PetscErrorCode KSPSetFromOptions(KSP) { return 0; }
PetscErrorCode KSPGetConvergedReason(KSP ksp, KSPConvergedReason *r) { *r = ksp->reason; return 0; }
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt *its) { *its = ksp->iters; return 0; }
PetscErrorCode KSPDestroy(KSP *ksp) { delete *ksp; *ksp = nullptr; return 0; }

namespace {

struct Csr {
    PetscInt n = 0;
    std::vector<PetscInt> rp, col;
    std::vector<double> val;
};

Csr to_csr(const mcshim_Mat *A)
{
    Csr c;
    c.n = A->n;
    c.rp.assign((size_t)A->n + 1, 0);
    for (PetscInt i = 0; i < A->n; i++) {
        for (const auto &kv : A->rows[(size_t)i]) {
            c.col.push_back(kv.first);
            c.val.push_back(kv.second);
        }
        c.rp[(size_t)i + 1] = (PetscInt)c.col.size();
    }
    return c;
}

void spmv(const Csr &A, const std::vector<double> &x, std::vector<double> &y)
{
    for (PetscInt i = 0; i < A.n; i++) {
        double s = 0.0;
        for (PetscInt k = A.rp[(size_t)i]; k < A.rp[(size_t)i + 1]; k++) s += A.val[(size_t)k] * x[(size_t)A.col[(size_t)k]];
        y[(size_t)i] = s;
    }
}

double dot(const std::vector<double> &a, const std::vector<double> &b)
{
    double s = 0.0;
    for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
    return s;
}

void project_mean_zero(std::vector<double> &v)
{
    double s = 0.0;
    for (double x : v) s += x;
    const double m = s / (double)v.size();
    for (double &x : v) x -= m;
}

// Unpreconditioned BiCGStab from x = 0, residual checked after each full step.
int bicgstab(const Csr &A, const std::vector<double> &b, std::vector<double> &x, double rtol, int max_iters, double *relres)
{
    const size_t n = b.size();
    x.assign(n, 0.0);
    std::vector<double> r(b), r0(b), p(n, 0.0), v(n, 0.0), s(n), t(n);
    const double bnorm = std::sqrt(dot(b, b));
    *relres = 0.0;
    if (bnorm == 0.0) return 0;
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    for (int k = 1; k <= max_iters; k++) {
        const double rho_new = dot(r0, r);
        if (rho_new == 0.0) { *relres = std::sqrt(dot(r, r)) / bnorm; return -k; }
        const double beta = (rho_new / rho) * (alpha / omega);
        for (size_t i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        spmv(A, p, v);
        alpha = rho_new / dot(r0, v);
        for (size_t i = 0; i < n; i++) s[i] = r[i] - alpha * v[i];
        spmv(A, s, t);
        const double tt = dot(t, t);
        omega = (tt != 0.0) ? dot(t, s) / tt : 0.0;
        for (size_t i = 0; i < n; i++) {
            x[i] += alpha * p[i] + omega * s[i];
            r[i] = s[i] - omega * t[i];
        }
        rho = rho_new;
        const double rn = std::sqrt(dot(r, r));
        *relres = rn / bnorm;
        if (rn <= rtol * bnorm) return k;
        if (omega == 0.0) return -k;
    }
    return -max_iters;
}

// Conjugate gradients on the singular symmetric system, mean-zero projected.
int cg_projected(const Csr &A, const std::vector<double> &b_in, std::vector<double> &x, double rtol, int max_iters, double *relres)
{
    const size_t n = b_in.size();
    std::vector<double> b(b_in);
    project_mean_zero(b);
    x.assign(n, 0.0);
    std::vector<double> r(b), p(b), q(n);
    double rr = dot(r, r);
    const double bnorm = std::sqrt(rr);
    *relres = 0.0;
    if (bnorm == 0.0) return 0;
    int k = 1;
    for (; k <= max_iters; k++) {
        spmv(A, p, q);
        const double alpha = rr / dot(p, q);
        for (size_t i = 0; i < n; i++) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
        }
        const double rr_new = dot(r, r);
        *relres = std::sqrt(rr_new) / bnorm;
        if (std::sqrt(rr_new) <= rtol * bnorm) break;
        const double beta = rr_new / rr;
        rr = rr_new;
        for (size_t i = 0; i < n; i++) p[i] = r[i] + beta * p[i];
    }
    project_mean_zero(x);
    return k > max_iters ? -max_iters : k;
}

} // namespace

PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x)
{
    const Csr A = to_csr(ksp->A);
    double relres = 0.0;
    int its;
    if (ksp->type == KSPBCGS) {
        its = bicgstab(A, b->v, x->v, g_bcgs_rtol, g_max_iters, &relres);
        g_last_kind = 0;
        g_count_bcgs++;
    } else {
        its = cg_projected(A, b->v, x->v, g_cg_rtol, g_max_iters, &relres);
        g_last_kind = 1;
        g_count_cg++;
    }
    ksp->iters = its < 0 ? -its : its;
    ksp->reason = its < 0 ? -3 : 2;
    g_last_iters = ksp->iters;
    g_last_relres = relres;
    return 0;
}

extern "C" void mcshim_mat_csr(Mat A, PetscInt *n, PetscInt *nnz, PetscInt *row_ptr, PetscInt *col, double *val)
{
    const Csr c = to_csr(A);
    *n = c.n;
    *nnz = (PetscInt)c.col.size();
    if (row_ptr) std::memcpy(row_ptr, c.rp.data(), c.rp.size() * sizeof(PetscInt));
    if (col) std::memcpy(col, c.col.data(), c.col.size() * sizeof(PetscInt));
    if (val) std::memcpy(val, c.val.data(), c.val.size() * sizeof(double));
}

extern "C" void mcshim_vec_values(Vec v, PetscInt *n, double *out)
{
    *n = (PetscInt)v->v.size();
    if (out) std::memcpy(out, v->v.data(), v->v.size() * sizeof(double));
}
