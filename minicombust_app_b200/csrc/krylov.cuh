// Krylov solvers on 7-point ELL matrices, all state on the device.
//
// Each iteration is two (PCG) or three (BiCGStab) fused kernels: the vector
// update whose result a sparse product needs at neighbouring rows is
// recomputed on the fly for those rows, so no kernel waits for another
// grid-wide update.  Scalars (alpha, beta, omega, norms) are produced by the
// last block of each kernel from per-block partials in a fixed order, so the
// solves are deterministic.  Converged solves turn later launches into no-ops;
// the host polls a small status block between batches of iterations.
#pragma once

#include <stdint.h>

#include <cuda_runtime.h>

namespace mcb {

// Paired vector type for the interleaved (z, p) buffers.
template <typename T>
struct Pair;
template <>
struct Pair<double> {
    using type = double2;
};
template <>
struct Pair<float> {
    using type = float2;
};

// Columns of the 7-point rows in direction-code form: on a structured box in
// x-fastest order the neighbour through direction d is always row + doff[d],
// so a row's six columns fit one 32-bit word (3 bits per slot: the direction
// 0..5 of the slot, or 7 for an unused slot).  Kernels then read 4 bytes per
// row instead of 24.
// Most rows (all interior cells) share one code word, `canon`, whose
// per-slot offsets are kept ready in coff.
// `dia` marks a copy of the values stored by direction instead of by slot
// (slot d = direction d, zero where the row has no neighbour that way): its
// columns are row + doff[d] (clamped into [0, N), where the value is 0), so
// the kernels read no column data at all.
// `sym` (with `dia`) marks the copy of a symmetric matrix that keeps only
// the couplings of the directions with positive offsets (d = 1, 3, 5 in slot
// d >> 1): the coupling of row i in direction d - 1 is the one row
// i + doff[d - 1] keeps for direction d (A_ij = A_ji), and 0 where that row
// index is below 0.  A row with no neighbour in direction d - 1 reads the
// stored 0 of the row before it on the x-line, y-column or z-column edge.
// Half the off-diagonal bytes.
struct DirCodes {
    const uint32_t *code = nullptr;  // [N]; nullptr: use the column list
    int doff[6] = {0, 0, 0, 0, 0, 0};
    uint32_t canon = 0;
    int coff[6] = {0, 0, 0, 0, 0, 0};
    int dia = 0;
    int sym = 0;
};

// The same codes for a copy of the values in direction order (see `dia`).
inline DirCodes by_direction(DirCodes dc)
{
    dc.dia = dc.code ? 1 : 0;
    dc.sym = 0;
    return dc;
}

// A symmetric matrix's copy in the half form (see `sym`): needs codes whose
// even directions are the negatives of the odd ones.
inline bool sym_applies(const DirCodes &dc)
{
    if (!dc.code) return false;
    for (int j = 0; j < 3; j++)
        if (!(dc.doff[2 * j] < 0 && dc.doff[2 * j] == -dc.doff[2 * j + 1])) return false;
    return true;
}
inline DirCodes by_direction_sym(DirCodes dc)
{
    dc = by_direction(dc);
    dc.sym = dc.dia;
    return dc;
}

// Value of slot k of row i (its column ck from row_cols / with_row_cols).
// Only FP64 copies come in the half form (the FP32 kernels compile without
// it: the extra path cost them registers and time).
template <typename T>
__device__ __forceinline__ T ell_val(const DirCodes &dc, const T *__restrict__ off, int N, int i, int k, int ck)
{
    if (sizeof(T) == sizeof(float) || !dc.sym) return off[(size_t)k * N + i];
    const size_t j = (size_t)(k >> 1) * N;
    if (k & 1) return off[j + i];
    return (i + dc.doff[k] >= 0) ? off[j + ck] : (T)0;
}

__device__ __forceinline__ void dia_cols(const DirCodes &dc, int N, int i, int (&c)[6])
{
#pragma unroll
    for (int k = 0; k < 6; k++) c[k] = min(max(i + dc.doff[k], 0), N - 1);
}

// Column of each slot of row i (the row itself for an unused slot).
// Columns of a row from its code word (six 3-bit direction indices).
__device__ __forceinline__ void decode_cols(const DirCodes &dc, uint32_t cw, int i, int (&c)[6])
{
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const unsigned d = (cw >> (3 * k)) & 7u;
        int o = 0;
#pragma unroll
        for (int q = 0; q < 6; q++) o = (d == (unsigned)q) ? dc.doff[q] : o;
        c[k] = i + o;
    }
}

__device__ __forceinline__ void row_cols(const DirCodes &dc, const int *__restrict__ col, int N, int i, int (&c)[6])
{
    if (dc.dia) {
        dia_cols(dc, N, i, c);
    } else if (dc.code) {
        const uint32_t cw = dc.code[i];
        if (cw == dc.canon) {
#pragma unroll
            for (int k = 0; k < 6; k++) c[k] = i + dc.coff[k];
        } else {
            decode_cols(dc, cw, i, c);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 6; k++) c[k] = col[(size_t)k * N + i];
    }
}

// Evaluate f(columns) for row i.  With direction codes f first runs on the
// canonical columns (clamped into [0, N)) while the row's code word is still
// in flight, so its neighbour loads do not wait for the code; only rows whose
// code differs (the boundary rows of a box) run f again with their decoded
// columns.  f must have no side effects; its result for a canonical row is
// the same as with the columns of row_cols.
template <typename F>
__device__ __forceinline__ auto with_row_cols(const DirCodes &dc, const int *__restrict__ col, int N, int i, F &&f)
{
    int c[6];
    if (dc.dia) {
        dia_cols(dc, N, i, c);
        return f(c);
    }
    if (dc.code) {
        const uint32_t cw = dc.code[i];
#pragma unroll
        for (int k = 0; k < 6; k++) c[k] = min(max(i + dc.coff[k], 0), N - 1);
        auto r = f(c);
        if (cw != dc.canon) {
            decode_cols(dc, cw, i, c);
            r = f(c);
        }
        return r;
    }
#pragma unroll
    for (int k = 0; k < 6; k++) c[k] = col[(size_t)k * N + i];
    return f(c);
}

// FP32 values of row i; with codes in direction order (slot d = direction d,
// zero for a direction the row lacks), else in the original slot order.
__device__ __forceinline__ void round_row_by_direction(const double *__restrict__ off, const uint32_t *__restrict__ code,
                                                       int N, int i, float (&o)[6], double scale = 1.0)
{
    if (code) {
        const uint32_t cw = code[i];
#pragma unroll
        for (int d = 0; d < 6; d++) o[d] = 0.f;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const unsigned d = (cw >> (3 * k)) & 7u;
            const float v = (float)(off[(size_t)k * N + i] * scale);
#pragma unroll
            for (int q = 0; q < 6; q++) o[q] = (d == (unsigned)q) ? v : o[q];
        }
    } else {
#pragma unroll
        for (int k = 0; k < 6; k++) o[k] = (float)(off[(size_t)k * N + i] * scale);
    }
}

// Row scaling of the FP32 inner BiCGStab systems (Jacobi preconditioning
// from the left): 1 / diag, or 1 for a row without a diagonal.
__device__ __forceinline__ double row_scale(const double *__restrict__ diag, int i)
{
    const double d = diag[i];
    return d != 0.0 ? 1.0 / d : 1.0;
}

// 7-point system in ELL form; T is the storage type of the values.
template <typename T>
struct EllT {
    int N;
    const T *diag;
    const T *off;   // [6][N]
    const int *col; // [6][N]
    DirCodes dc{};
};
using Ell = EllT<double>;

template <typename T>
__device__ __forceinline__ void row_cols(const EllT<T> &A, int i, int (&c)[6])
{
    row_cols(A.dc, A.col, A.N, i, c);
}

struct PcgState {
    double rz, rz_old, alpha, pq, rr, bb, tol2, mean, xmean;
    int iter, done, status, max_iters;
};

template <int R>
struct BicgState {
    double rho[R], rho_new[R], alpha[R], omega[R], bb[R], rr[R], tol2[R];
    int iter[R], done[R], status[R];
    int all_done, max_iters;
};

// zp[k][i] = (z_i, p_i): the preconditioned residual and the search
// direction interleaved, so that a neighbour costs one 16-byte gather.
// Iteration k reads zp[k & 1] and writes p into zp[(k & 1) ^ 1], where the
// next z is then stored.
// Storage type T (double, or float for the inner solve of the refined
// pressure path); dot products and the scalars in PcgState stay FP64.
template <typename T>
struct PcgVectorsT {
    T *x, *r, *q;
    typename Pair<T>::type *zp[2];
    const T *b;
    double *partials;
    unsigned int *counter;
    PcgState *st;
};
using PcgVectors = PcgVectorsT<double>;

// Storage type T (double, or float for the inner solves of the refined
// path); dot products and the scalars in BicgState stay FP64.
template <typename T, int R>
struct BicgVectorsT {
    T *x[R];
    const T *b;          // [R][N]
    T *r, *r0, *p[2], *v[2], *s, *t;  // each [R][N]
    double *partials;
    unsigned int *counter;
    BicgState<R> *st;
};
template <int R>
using BicgVectors = BicgVectorsT<double, R>;

// FP64 iterative refinement around FP32 BiCGStab solves of R systems with
// one matrix (momentum: R = 3; temperature: R = 1): x (FP64) starts at zero,
// r = b - A x in FP64, r32 = (float) r feeds the inner solve of A32 e = r32,
// x += e; each system stops when ||r_j|| <= rtol ||b_j||.
template <int R>
struct BirState {
    double bb[R], rr[R], tol2[R];
    int done[R], status[R];
    int iter, all_done, max_outer, pad;
};
template <int R>
struct BirVectors {
    double *x[R];
    const double *b;     // [R][N]
    float *r32;          // [R][N]
    const float *e;      // [R][N] inner solution
    double *partials;
    unsigned int *counter;
    BirState<R> *st;
};

// x-line sweeps: the inner solver of the refined momentum and temperature
// systems (FP32, row-scaled, values by direction) on a structured box whose
// cells run x-fastest along whole lines.  The splitting keeps, per x-line,
// the diagonal and the -x couplings (a first-order recurrence along the
// line); the other couplings act through the previous iterate.
struct LineSystem {
    int N = 0;
    int ex = 0;        // cells per x-line (the line length, <= 1024)
    int P = 0;         // unused (kept 0)
    int dxm = 0, dxp = 0;      // by-direction slots of the -x and +x couplings
    int yz[4] = {0, 0, 0, 0};  // the other four slots
    int yzoff[4] = {0, 0, 0, 0};
    const float *d = nullptr;   // diagonal [N]
    const float *off = nullptr; // [6][N] by direction
};
// One sweep step for R right-hand sides [R][N]: with first set, M e_new = r;
// otherwise M e_new = r - (M - A) e_prev.  With add set (the last step of an
// inner solve) the step's result is added to the FP64 solutions add->x of
// the systems still open instead of being stored (e_new unused): the
// refinement update x += e without a kernel of its own.
template <int R>
void line_step(cudaStream_t s, const LineSystem &L, const float *r, const float *e_prev, float *e_new, int first,
               const BirVectors<R> *add = nullptr);

enum { KRYLOV_OK = 0, KRYLOV_NOT_CONVERGED = 1, KRYLOV_NONFINITE = 2 };

// Grid size used by the Krylov kernels for N rows.
int krylov_grid(int N);

// Programmatic dependent launch: a kernel started with pdl_launch may be
// scheduled while its stream predecessor drains; pdl_wait (its first
// statement) blocks until the predecessor has completed and its memory is
// visible.  In a kernel launched the ordinary way pdl_wait returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

bool pdl_enabled();  // MC_PDL=0 launches every kernel the ordinary way

template <typename... KArgs, typename... Args>
inline void pdl_launch(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args &&...args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, static_cast<Args &&>(args)...);
}

// Single-kernel launchers (asynchronous on stream).  PCG uses Jacobi
// preconditioning; with project != 0 the right-hand side and the solution are
// projected onto mean zero (the singular pure-Neumann pressure-correction
// system).  Ping-pong buffers: iteration k reads p[k & 1] and writes p[(k & 1) ^ 1].
void pcg_mean(cudaStream_t s, const Ell &A, const PcgVectors &v);
void pcg_init(cudaStream_t s, const Ell &A, const PcgVectors &v, double rtol, double abs_floor, int max_iters,
              int use_x0, int project);
template <typename T>
void pcg_iter1(cudaStream_t s, const EllT<T> &A, const PcgVectorsT<T> &v, int pin);
void pcg_iter2(cudaStream_t s, const Ell &A, const PcgVectors &v, int pnew);
// AMG-preconditioned variant: init without z, update without z (amg.cu
// computes z and r . z after each update).
template <typename T>
void pcg_init_amg(cudaStream_t s, const EllT<T> &A, const PcgVectorsT<T> &v, double rtol, double abs_floor,
                  int max_iters, int project, int use_x0 = 0);
template <typename T>
void pcg_iter2_amg(cudaStream_t s, const EllT<T> &A, const PcgVectorsT<T> &v, int pnew);
// FP64 iterative refinement around an FP32 inner solve: the state's mean
// (from pcg_mean) defines b' = b - mean; ir_init sets x = 0, r = b', r32 =
// (float) r and the tolerance (or applies a guess, IrGuess); ir_residual
// recomputes the FP64 true residual, its norm, r32, and the convergence flag
// (with e given, of x + e, which it stores in xout != x: the update x += e
// and the residual in one pass).  r may be null in both.
// Initial guess of the pressure correction from up to two candidates xa, xb
// (a null candidate is skipped): the combination x0 = alpha xa + beta xb
// that minimises ||b' - A x0|| (b' = b - st->mean).  Zero lies in the span,
// so the guess never starts from a larger residual than the zero guess; if
// rounding says otherwise the zero guess is used.  rr[] are the residuals of
// the single candidates, rc that of the combination.
struct GuessState {
    double bb, rr[2], coef[2], rc;
    int choice;      // -1 zero, 2 combination
    int net_status;  // copy of the network's status (nonzero: its prediction was zeroed)
};
// The guess applied by ir_init itself: x0 = alpha xa + beta xb (coefficients
// in *gs) and r = b' - (alpha u + beta w) with u = A xa, w = A xb as
// guess_residuals stored them.  gs null: not used.
struct IrGuess {
    const GuessState *gs = nullptr;
    const double *xa = nullptr, *xb = nullptr, *u = nullptr, *w = nullptr;
};
void ir_init(cudaStream_t s, const Ell &A, const double *b, double *x, double *r, float *r32, PcgState *st,
             double *partials, unsigned int *counter, double rtol, double abs_floor, int max_outer, int use_x0 = 0,
             const IrGuess &g = IrGuess{});
// uo, wo (optional): A xa and A xb are also stored there.
void guess_residuals(cudaStream_t s, const Ell &A, const double *b, const PcgState *st, const double *xa,
                     const double *xb, GuessState *gs, double *partials, unsigned int *counter,
                     double *uo = nullptr, double *wo = nullptr);
void guess_apply(cudaStream_t s, int N, double *x, const double *xa, const double *xb, const GuessState *gs);
void ir_residual(cudaStream_t s, const Ell &A, const double *b, const double *x, double *r, float *r32, PcgState *st,
                 double *partials, unsigned int *counter, const float *e = nullptr, double *xout = nullptr);
void pcg_xmean(cudaStream_t s, int N, const PcgVectors &v);
void pcg_sub_xmean(cudaStream_t s, int N, const PcgVectors &v);

template <typename T, int R>
void bicg_init_t(cudaStream_t s, const EllT<T> &A, const BicgVectorsT<T, R> &v, double rtol, int max_iters);
template <typename T, int R>
void bicg_1_t(cudaStream_t s, const EllT<T> &A, const BicgVectorsT<T, R> &v, int pin);
template <typename T, int R>
void bicg_2_t(cudaStream_t s, const EllT<T> &A, const BicgVectorsT<T, R> &v, int vnew);
template <typename T, int R>
void bicg_3_t(cudaStream_t s, const EllT<T> &A, const BicgVectorsT<T, R> &v, int pnew);
template <int R>
void bir_init(cudaStream_t s, const Ell &A, const BirVectors<R> &v, double rtol, int max_outer);
template <int R>
void bir_add(cudaStream_t s, int N, const BirVectors<R> &v);
template <int R>
void bir_residual(cudaStream_t s, const Ell &A, const BirVectors<R> &v);
// FP32 copy of a 7-point matrix's rows scaled by 1 / diag (the inner systems
// of the refined BiCGStab solves), by direction when `code` is given (see
// DirCodes::dia), else in slot order.
void round_ell(cudaStream_t s, int N, const double *diag, const double *off, const uint32_t *code, float *diag32,
               float *off32);

template <int R>
void bicg_init(cudaStream_t s, const Ell &A, const BicgVectors<R> &v, double rtol, int max_iters);
template <int R>
void bicg_1(cudaStream_t s, const Ell &A, const BicgVectors<R> &v, int pin);
template <int R>
void bicg_2(cudaStream_t s, const Ell &A, const BicgVectors<R> &v, int vnew);
template <int R>
void bicg_3(cudaStream_t s, const Ell &A, const BicgVectors<R> &v, int pnew);

// Kernels launched per iteration (for launch accounting).
constexpr int PCG_KERNELS_PER_ITER = 2;
constexpr int BICG_KERNELS_PER_ITER = 3;

} // namespace mcb
