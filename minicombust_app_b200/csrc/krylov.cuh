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

#include <cuda_runtime.h>

namespace mcb {

struct Ell {
    int N;
    const double *diag;
    const double *off;  // [6][N]
    const int *col;     // [6][N]
};

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
struct PcgVectors {
    double *x, *r, *q;
    double2 *zp[2];
    const double *b;
    double *partials;
    unsigned int *counter;
    PcgState *st;
};

template <int R>
struct BicgVectors {
    double *x[R];
    const double *b;          // [R][N]
    double *r, *r0, *p[2], *v[2], *s, *t;  // each [R][N]
    double *partials;
    unsigned int *counter;
    BicgState<R> *st;
};

enum { KRYLOV_OK = 0, KRYLOV_NOT_CONVERGED = 1, KRYLOV_NONFINITE = 2 };

// Grid size used by the Krylov kernels for N rows.
int krylov_grid(int N);

// Single-kernel launchers (asynchronous on stream).  PCG uses Jacobi
// preconditioning; with project != 0 the right-hand side and the solution are
// projected onto mean zero (the singular pure-Neumann pressure-correction
// system).  Ping-pong buffers: iteration k reads p[k & 1] and writes p[(k & 1) ^ 1].
void pcg_mean(cudaStream_t s, const Ell &A, const PcgVectors &v);
void pcg_init(cudaStream_t s, const Ell &A, const PcgVectors &v, double rtol, double abs_floor, int max_iters,
              int use_x0, int project);
void pcg_iter1(cudaStream_t s, const Ell &A, const PcgVectors &v, int pin);
void pcg_iter2(cudaStream_t s, const Ell &A, const PcgVectors &v, int pnew);
// AMG-preconditioned variant: init without z, update without z (amg.cu
// computes z and r . z after each update).
void pcg_init_amg(cudaStream_t s, const Ell &A, const PcgVectors &v, double rtol, double abs_floor, int max_iters,
                  int project);
void pcg_iter2_amg(cudaStream_t s, const Ell &A, const PcgVectors &v, int pnew);
void pcg_xmean(cudaStream_t s, int N, const PcgVectors &v);
void pcg_sub_xmean(cudaStream_t s, int N, const PcgVectors &v);

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
