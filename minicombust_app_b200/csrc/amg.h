// Aggregation AMG for the pressure-correction system.
//
// Hierarchy (built once per mesh on the host, from the matrix graph only):
// level 0 is the pressure-correction matrix (7-point ELL); each coarser level
// groups up to 2 x 2 x 2 cells of the level below into one aggregate, found
// by walking the cells' directional neighbours (+x, +y, +z from the first
// unaggregated cell), so that on a box every coarse level is again a 7-point
// box operator.  Coarse matrices are Galerkin products A_c = P^T A P with the
// piecewise-constant prolongation P; their values are recomputed on the GPU
// whenever the fine values change, by summing precomputed lists of fine
// entries (a gather, deterministic).  The coarsest level (<= 128 rows) is
// solved exactly with the explicit inverse of A_c + sigma 1 1^T, which for
// the singular pure-Neumann system gives the minimum-norm solution of a
// consistent right-hand side.
//
// Preconditioner: one symmetric V-cycle -- nu damped-Jacobi sweeps before and
// after the coarse correction (scaled by alpha) on every level -- so PCG
// sees a fixed symmetric operator.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "krylov.cuh"

namespace mcb {

constexpr int AMG_MAX_LEVELS = 16;
constexpr int AMG_COARSEST_MAX = 128;
// Levels with at most this many rows (down to the coarsest) run as one
// single-block kernel per V-cycle; at most AMG_FUSED_LEVELS of them.
constexpr int AMG_FUSE_MAX_ROWS = 1024;
constexpr int AMG_FUSED_LEVELS = 6;
constexpr int AMG_MAX_SWEEPS = 8;

// Device view of one level; T is the storage type of values and vectors.
template <typename T>
struct AmgLevelT {
    int n;          // rows
    int k;          // off-diagonal slots (ELL width)
    T *diag;        // [n]
    T *off;         // [k][n]
    const int *col; // [k][n], unused slots point at their own row
    DirCodes dc;    // level 0 of a structured box: columns from direction codes (k = 6)
    // restriction to the next level: members of coarse row I are mlist[mptr[I] .. mptr[I+1])
    const int *agg;   // [n] aggregate (next-level row) of each row
    const int *mptr;  // [n_next + 1]
    const int *mlist; // [n]
    // Galerkin lists building THIS level's values from the level below:
    // entry e = row * (k + 1) + slot (slot 0 = diagonal, s + 1 = off slot s)
    // sums fine values gidx[gptr[e] .. gptr[e+1]) (fine diag id < n_fine,
    // fine off id = n_fine + s * n_fine + row).
    const int *gptr;
    const int *gidx;
    T *r;           // right-hand side of the level
    T *e[2];        // ping-pong iterates
    // FP32 level 0 stored by direction: its off-diagonal values also in FP16,
    // times scale16[0] (a power of two chosen each time the values change);
    // the sweeps and the restriction of the V-cycle read these (and multiply
    // by scale16[1] = 1 / scale16[0]), the PCG product keeps the FP32 values.
    // Null: every kernel reads off.
    __half *off16 = nullptr;
    float *scale16 = nullptr;
};
using AmgLevel = AmgLevelT<double>;

struct AmgHierarchy {
    int levels = 0;
    AmgLevelT<double> lv[AMG_MAX_LEVELS];    // FP64 values (level 0 = the pressure-correction matrix)
    // level 0 with its values in slot order: the source of the Galerkin
    // lists of level 1 and of the FP32 level 0 (lv[0] itself may be the
    // half-form copy, DirCodes::sym)
    AmgLevelT<double> g0;
    AmgLevelT<float> lv32[AMG_MAX_LEVELS];   // FP32 values, when the refined FP32 path is enabled
    bool has32 = false;
    double *dense = nullptr;       // coarsest inverse [n][n] (row-major, exactly symmetric), FP64
    double *dense_next = nullptr;  // the inverse being formed for the next pass (lagged setup)
    int sweeps = 2;
    double omega = 0.6667;
    double omega_sweep[AMG_MAX_SWEEPS] = {};  // damping of sweep k before the coarse correction (reversed after)
    double alpha = 1.0;
    int fused_from = 0;   // first level of the single-block coarse cycle (set by amg_plan_fused)
};

// Damping of each sweep: amg_omega for every sweep (ratio 0), or the
// reciprocal Chebyshev roots on [2 / ratio, 2] (ratio > 1).
void amg_set_damping(AmgHierarchy &H, double ratio);

// Choose the levels that the single-block coarse cycle takes over.
void amg_plan_fused(AmgHierarchy &H);

// Host-side construction of the pattern data.  Inputs: level-0 ELL columns
// (col0[6][N], boundary slots = own row) and directional neighbours dn0[6][N]
// in cell_faces slot order (FRONT -z, BACK +z, LEFT -x, RIGHT +x, DOWN -y,
// UP +y; -1 on the boundary).
struct AmgHostLevel {
    int n = 0, k = 0;
    std::vector<int> col;               // [k][n]
    std::vector<int> agg, mptr, mlist;  // restriction to the next level
    std::vector<int> gptr, gidx;        // Galerkin lists for this level (levels >= 1)
    // Levels >= 1 whose rows all reach their neighbours through six fixed
    // offsets (the coarse levels of a structured box): slot s holds the
    // neighbour at row + doff[s] (offsets ascending, the same order as sorted
    // columns), with value 0 and column = row where the row has none.
    int dia = 0;
    int doff[6] = {0, 0, 0, 0, 0, 0};
};

int amg_build_host(int N, const std::vector<int> &col0, const std::vector<int> &dn0, std::vector<AmgHostLevel> &out,
                   std::string &err);

// Device work, all asynchronous on stream s.
// Galerkin values of levels 1..L-1 for the FP64 (T = double) or the FP32
// (T = float; level 0 rounded from FP64 first, unless the pressure kernel
// has just written it: level0_ready) hierarchy, and the FP16 copy of the
// FP32 level 0 where there is one, scaled by max |diag| in *dmax (formed by
// the pressure kernel with level0_ready, else here through partials and
// counter).
template <typename T>
void amg_setup_levels(cudaStream_t s, const AmgHierarchy &H, bool level0_ready, double *partials,
                      unsigned int *counter, double *dmax);
// Explicit inverse of the coarsest level's current values into `out`
// (n x n FP64); reads only the coarsest level.
template <typename T>
void amg_coarsest_inverse(cudaStream_t s, const AmgHierarchy &H, double *out);
// z = V-cycle(r0) on level 0; z goes to zp[i].x (the PCG interleaved buffer)
// and r0 . z (FP64 sum) into the PCG state.  Kernels are no-ops once
// st->done is set.
struct PcgState;
template <typename T>
void amg_vcycle(cudaStream_t s, const AmgHierarchy &H, const T *r0, void *zp_out, PcgState *st, double *partials,
                unsigned int *counter, int is_init);
int amg_kernels_per_vcycle(const AmgHierarchy &H, bool fp32);

} // namespace mcb
