// Declarations and argument blocks of the SIMPLE-pass assembly kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mc_internal.h"

namespace mcb {

// Device view of the mesh passed to kernels by value.
struct MeshArgs {
    int F;
    const int *fc0, *fc1, *sface;
    // Both cells of a cell's faces without reading them through the face
    // index: col[k][c] is the other cell of face sface[k][c] (c itself on a
    // boundary face) and bit k of own[c] is set when c is that face's cell0.
    const int *col;
    const uint8_t *own;
    const double *area, *lam, *rl, *Sx, *Sy, *Sz, *xf, *yf, *zf;
    const double *xc, *yc, *zc, *vol, *rho;
    const int *outlet_faces;
    int n_outlet;
};

// Storage of the FP64 momentum, temperature and scalar rows for the solvers.
// code null: slot order (slot k = the k-th face of the cell in reference
// order).  Otherwise by direction: the value of slot k goes to position
// (pos >> 3d) & 7 of the row, d = (code[c] >> 3k) & 7 its direction (7: no
// value), 0 where the row has no neighbour that way; the solvers then read no
// column data.  The positions follow the order in which the directions occur
// in every row's slots, so each row sums its nonzero terms in slot order.
struct RowStore {
    const uint32_t *code = nullptr;
    uint32_t pos = 0;
};

// FP32 copy of assembled rows (refined path): scaled by 1 / diag, by direction.
struct Fp32Rows {
    float *d32 = nullptr;        // null: no copy
    float *o32 = nullptr;        // [6][N]
    const uint32_t *code = nullptr;  // null: slot order
    int scale_rows = 1;          // divide the row by its diagonal
};

template <int NF>
struct GradArgs {
    const double *phi[NF];
    double *gx[NF], *gy[NF], *gz[NF];
    unsigned zero_boundary;  // bit k: dphi = 0 on boundary faces for field k
};

struct MomentumArgs {
    double *U, *V, *W;          // interior read, boundary slots written
    const double *T;
    const double *gU[3], *gV[3], *gW[3], *gP[3];
    double *mdot;               // outlet clamp write (:1576-1580)
    const double *src;          // [5][N] particle terms or null
    double *off;                // [6][N]
    double *AU;                 // diagonal after under-relaxation (A_phi.U)
    double *b;                  // [3][N]
    RowStore store;
    Fp32Rows f32;
};

struct ScalarArgs {
    double *phi;                // T: interior read, boundary slots written
    const double *g[3];
    const double *mdot;
    const double *src;
    double *off, *diag, *b;
    // temperature kernel: the pass's mass imbalance max |div(mdot) - mass source|
    // into *imbalance, which must be zero before the launch (null: not computed)
    double *imbalance;
    RowStore store;
    Fp32Rows f32;               // temperature kernel only
};

// Extra inputs of the k and epsilon transports (solveTurbulenceModels).
struct TurbArgs {
    const double *U, *V, *W;
    const double *gU[3], *gV[3], *gW[3];
    const double *TE, *ED;      // k and epsilon (the one being assembled is also ScalarArgs::phi)
    double *TP;                 // turbulent production: written by k, read by epsilon
};

// Replacement of negative k / epsilon values after their solve.
struct ClipArgs {
    double *phi;
    const int *nbr;             // [6][N]
    const int *key;             // caller's id of each cell (null: identity)
    const int *o2n;             // caller's id -> cell (null: identity)
    int *list;                  // [cap] negative cells
    unsigned int *count;        // zero before the first launch; reset by k_scalar_clip
    int cap;
};

struct MassFluxArgs {
    const double *U, *V, *W, *P, *AU;
    const double *gU[3], *gV[3], *gW[3], *gP[3];
    double *mdot, *ff0, *ff1;
    double *partials;
    unsigned int *counter;
    FluxBalance *balance;
    double mass_source_total;
    const double *mass_source_dev;  // non-null: the total is read here instead (device-resident sources)
};

struct PressureRowArgs {
    const double *mdot, *ff0, *ff1, *src;
    double *off, *diag, *b;
    Fp32Rows f32;               // the FP32 level 0 of the AMG hierarchy (refined path)
    // the FP64 copy the solvers read, stored by direction (by the direction
    // codes `code`): all six directions, or with dir64_sym the half form of
    // a symmetric matrix (DirCodes::sym); null: none
    double *dir64;
    int dir64_sym;
    const uint32_t *code;
    double *diag_max;           // max |diag| (zero before the launch); null: not formed
};

// The by-direction FP64 copy of a matrix stored by slot with direction
// codes: out[d N + i] = off[k][i] for the slot k of direction d (0 where the
// row has none), or with sym (DirCodes::sym) only d = 1, 3, 5 into
// out[(d >> 1) N + i].
__global__ void k_dir_rows64(int N, const double *off, const uint32_t *code, double *out, int sym);

struct CorrectArgs {
    double *PP, *P, *U, *V, *W;
    const double *AU;
    const double *gPP[3];
    const double *ff0;
    double *mdot, *fcorr;
    double *next_rhs;           // null: do not build the next corrector's right-hand side
};

// The gradient kernel is a template; it is launched from its own translation
// unit (a template kernel launched elsewhere without relocatable device code
// would register a stub with no device code).
void launch_lsq_gradients5(cudaStream_t s, int N, const int *nbr, const int *fc1, const double *xc,
                           const double *yc, const double *zc, const double *xf, const double *yf, const double *zf,
                           const GradArgs<5> &a);
void launch_lsq_gradients1(cudaStream_t s, int N, const int *nbr, const int *fc1, const double *xc,
                           const double *yc, const double *zc, const double *xf, const double *yf, const double *zf,
                           const GradArgs<1> &a);
__global__ void k_precomp_au(Physics ph, MeshArgs m, const double *mdot, double *AU);
__global__ void k_momentum_assemble(Physics ph, MeshArgs m, MomentumArgs a);
__global__ void k_temperature_assemble(Physics ph, MeshArgs m, ScalarArgs a);
// FluxScalar + Scalar_solve assembly of one of TE, ED, FUL, PRO, VARF, VARP
// (type = SC_*), with the k-epsilon sources for TE and ED.
void launch_scalar_assemble(cudaStream_t s, int type, const Physics &ph, const MeshArgs &m, const ScalarArgs &a,
                            const TurbArgs &t);
void launch_lsq_gradients6(cudaStream_t s, int N, const int *nbr, const int *fc1, const double *xc,
                           const double *yc, const double *zc, const double *xf, const double *yf, const double *zf,
                           const GradArgs<6> &a);
// Negative k / epsilon values after the solve (FlowSolver.inl:2956-2985):
// list them, then replace them one at a time in the caller's cell order.
__global__ void k_scalar_negatives(int N, ClipArgs a);
__global__ void k_scalar_clip(int N, ClipArgs a);
__global__ void k_mass_flux(Physics ph, MeshArgs m, MassFluxArgs a);
__global__ void k_outlet_fix(Physics ph, MeshArgs m, double *mdot, double *U, double *V, double *W,
                             const FluxBalance *bal);
__global__ void k_pressure_rows(Physics ph, MeshArgs m, PressureRowArgs a);
__global__ void k_pp_correct_faces(Physics ph, MeshArgs m, CorrectArgs a);
__global__ void k_pp_correct_cells(Physics ph, MeshArgs m, CorrectArgs a, int correct_all, int correct_cell0);
__global__ void k_update_p_boundary(Physics ph, MeshArgs m, double *P, double *gPx, double *gPy, double *gPz,
                                    const int *nbr);
__global__ void k_pp_max(int N, int cell0, const double *PP, double *partials, unsigned int *counter, double *out);
// Sum of x[0..n) into *out, deterministic (per-block partials, last block reduces in order).
__global__ void k_sum(int n, const double *x, double *partials, unsigned int *counter, double *out);


} // namespace mcb
