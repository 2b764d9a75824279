/*
 * CPU restatement of miniCOMBUST's flow-solver SIMPLE pass (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this library, and only as the checker
 * or the timed CPU baseline, never as the thing measured or shipped.
 *
 * It restates, function by function, the reference CPU FlowSolver
 * (include/flow/FlowSolver.{hpp,inl}) and mesh builder
 * (src/examples/mesh_examples.cpp): the fields the SIMPLE pass couples (u, v,
 * w, p, the pressure correction and T) and, with params.scalars, the other
 * scalar transports (k, epsilon, mixture fraction, progress variable and the
 * two variances).  Each function in mc_oracle.c
 * cites the reference lines it follows.  Two modes:
 *
 *   MCO_MODE_COMPAT  the reference's control flow, constants and quirks
 *                    (stale pressure-correction system after the first solve,
 *                    cell-0-only correction, fixed outlet flux, no particle
 *                    sources).  With the same solver tolerances it matches the
 *                    reference compiled from its sources bit for bit.
 *   MCO_MODE_SIMPLE  the corrected SIMPLE pass used for the benchmark physics:
 *                    fresh pressure-correction system each corrector,
 *                    corrections applied to every cell with the pressure
 *                    under-relaxation, zero-gradient outlet with a global mass
 *                    balance, particle momentum/energy/mass sources.
 *
 * Linear solves (the reference's PETSc KSP): unpreconditioned BiCGStab for the
 * momentum and temperature systems, conjugate gradients with mean-zero
 * projection for the singular pressure-correction system, both from a zero
 * initial guess, stopping on ||r||_2 <= rtol ||b||_2.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { MCO_MODE_COMPAT = 0, MCO_MODE_SIMPLE = 1 };

/* Field indices follow phi_vector<T> (utils.hpp:158-174). */
enum {
    MCO_U = 0, MCO_V = 1, MCO_W = 2, MCO_P = 3, MCO_PP = 4, MCO_TE = 5, MCO_ED = 6,
    MCO_TP = 7, MCO_TEM = 8, MCO_FUL = 9, MCO_PRO = 10, MCO_VARF = 11, MCO_VARP = 12,
    MCO_NFIELDS = 13
};

typedef struct mco_params {
    int mode;
    double delta;          /* time step (minicombust.cpp:120) */
    double density;        /* FlowSolver.hpp:342 */
    double viscosity;      /* FlowSolver.hpp:296 */
    double inlet_u;        /* Mesh.hpp:114 (x component; y, z are 0) */
    double pressure0;      /* Mesh.hpp:115 */
    double temperature0;   /* Mesh.hpp:116: initial, inlet and buoyancy reference T */
    double urf_momentum;   /* FlowSolver.inl:1731 */
    double urf_pressure;   /* FlowSolver.inl:2425 */
    double urf_temperature;/* FlowSolver.inl:2939-2946 */
    double flux_corr;      /* FlowSolver.inl:1871 */
    double u_rtol;         /* momentum and temperature BiCGStab tolerance */
    double p_rtol;         /* pressure-correction CG tolerance */
    int max_iters;
    int scalars;           /* 1: also the six other scalar transports (TE, ED, FUL, PRO, VARF, VARP) */
} mco_params;

typedef struct mco_mesh {
    uint64_t ex, ey, ez;          /* elements per dimension */
    uint64_t cells, faces, points;
    double *points_xyz;           /* [points][3] */
    uint64_t *cell_nodes;         /* [cells][8], vertex order A..H */
    uint64_t *face_cells;         /* [faces][2] = {cell0, cell1}; cell1 >= cells is boundary cells + dir */
    uint64_t *cell_faces;         /* [cells][6] FRONT, BACK, LEFT, RIGHT, DOWN, UP */
    uint64_t *cell_neighbours;    /* [cells][6], UINT64_MAX on the domain boundary */
    double *cell_centers;         /* [cells][3] */
    uint64_t boundary_types[6];   /* 1 WALL, 2 INLET, 3 OUTLET */
} mco_mesh;

typedef struct mco_solver mco_solver;

void mco_default_params(mco_params *p, int mode);

/* Host threads of the linear solves (default 1).  With 1 every sum runs in
 * index order, which is what the pinning against the reference needs; more
 * threads split the vector loops and sum dot products in fixed chunks (for
 * large checks, where the result only has to meet a tolerance). */
void mco_set_threads(int n);

/* load_mesh for one flow rank (mesh_examples.cpp:120-571). */
int mco_mesh_box(uint64_t ex, uint64_t ey, uint64_t ez, double lx, double ly, double lz, mco_mesh *m);
void mco_mesh_free(mco_mesh *m);

mco_solver *mco_create(const mco_mesh *m, const mco_params *p);
void mco_destroy(mco_solver *s);

uint64_t mco_phi_length(const mco_solver *s); /* cells + 6 boundary slots */
int mco_set_field(mco_solver *s, int which, const double *vals);   /* length phi_length */
int mco_get_field(const mco_solver *s, int which, double *out);    /* length phi_length */
int mco_get_grad(const mco_solver *s, int which, double *out);     /* [cells][3]; U,V,W,P,PP,TEM */
/* which: 0..2 A_phi.U/V/W, 3..5 S_phi.U/V/W, 6 volumes, 7 densities */
int mco_get_cell_array(const mco_solver *s, int which, double *out);
/* which: 0 mass flux, 1 area, 2 lambda, 3 rlencos, 4 face_fields (2/face), 5 normals, 6 centres */
int mco_get_face_array(const mco_solver *s, int which, double *out);
/* particle_aos per cell: {momentum.x, momentum.y, momentum.z, energy, fuel(mass)} */
int mco_set_sources(mco_solver *s, const double *terms);
/* which: 0 momentum/scalar matrix A, 1 pressure-correction matrix.  row_ptr[n+1], col/val[nnz]. */
int mco_get_csr(const mco_solver *s, int which, int *n, int *nnz, int *row_ptr, int *col, double *val);
/* which: 0 b, 1 pressure-correction right-hand side */
int mco_get_rhs(const mco_solver *s, int which, double *out);

/* One SIMPLE pass (FlowSolver.inl:3188-3268 for u, v, w, p, T). */
int mco_pass(mco_solver *s);
/* Stages, callable one at a time. */
void mco_stage_gradients(mco_solver *s);
void mco_stage_set_up_field(mco_solver *s);
int mco_stage_calculate_uvw(mco_solver *s);
int mco_stage_calculate_pressure(mco_solver *s);
int mco_stage_scalar_temperature(mco_solver *s);
/* Scalar_solve for one scalar field: MCO_TE, MCO_ED, MCO_TEM, MCO_FUL, MCO_PRO,
 * MCO_VARF or MCO_VARP (the six other than MCO_TEM need params.scalars). */
int mco_stage_scalar(mco_solver *s, int field);

typedef struct mco_stats {
    int momentum_iters[3];
    int temperature_iters;
    int pressure_solves;
    int pressure_iters_total;
    int pressure_iters_first;
    double pressure_correction_max_first;
    double mass_imbalance;        /* ||div(mdot) - sources||_inf after the pass */
    int scalar_iters[6];          /* TE, ED, FUL, PRO, VARF, VARP */
} mco_stats;
void mco_get_stats(const mco_solver *s, mco_stats *out);
double mco_inlet_effective_viscosity(const mco_solver *s);

#ifdef __cplusplus
}
#endif
