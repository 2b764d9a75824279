// Krylov solvers (see krylov.cuh).  FP64 throughout; bandwidth bound: an
// iteration streams the 7-point matrix (12 bytes per entry) and a handful of
// vectors.
#include "krylov.cuh"

#include <algorithm>
#include <cstdlib>

#include "mc_reduce.cuh"

// Resident blocks per SM the grid-stride Krylov kernels are sized for.
#ifndef MCB_KRYLOV_BLOCKS_PER_SM
#define MCB_KRYLOV_BLOCKS_PER_SM 8
#endif

namespace mcb {

bool pdl_enabled()
{
    static int v = -1;
    if (v < 0) {
        const char *e = std::getenv("MC_PDL");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}


namespace {

__device__ __forceinline__ bool finite(double x) { return isfinite(x); }

} // namespace

int krylov_grid(int N)
{
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const int need = (N + MCB_THREADS - 1) / MCB_THREADS;
    return std::max(1, std::min(need, sms * MCB_KRYLOV_BLOCKS_PER_SM));
}

// ---------------------------------------------------------------------- PCG

__global__ void __launch_bounds__(MCB_THREADS) k_pcg_mean(int N, const double *__restrict__ b, PcgVectors v)
{
    __shared__ double sh[1][MCB_THREADS];
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) acc[0] += b[i];
    if (publish_partials<1>(acc, v.partials, v.counter, sh)) {
        double tot[1];
        reduce_partials<1>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) v.st->mean = tot[0] / (double)N;
    }
}

__global__ void __launch_bounds__(MCB_THREADS) k_pcg_init(Ell A, PcgVectors v, double rtol, double abs_floor,
                                                          int max_iters, int use_x0, int project)
{
    __shared__ double sh[3][MCB_THREADS];
    const int N = A.N;
    const double mean = project ? v.st->mean : 0.0;
    double acc[3] = {0.0, 0.0, 0.0};  // b.b, r.z, r.r
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double bi = v.b[i] - mean;
        double ri = bi;
        if (use_x0) {
            double ax = A.diag[i] * v.x[i];
            int c_[6];
            row_cols(A, i, c_);
#pragma unroll
            for (int k = 0; k < 6; k++) ax += ell_val(A.dc, A.off, N, i, k, c_[k]) * v.x[c_[k]];
            ri = bi - ax;
        } else {
            v.x[i] = 0.0;
        }
        const double di = A.diag[i];
        const double zi = (di != 0.0) ? ri / di : ri;  // a zero row (isolated cell) is left unpreconditioned
        v.r[i] = ri;
        v.zp[0][i] = make_double2(zi, 0.0);
        v.zp[1][i] = make_double2(0.0, 0.0);
        acc[0] += bi * bi;
        acc[1] += ri * zi;
        acc[2] += ri * ri;
    }
    if (publish_partials<3>(acc, v.partials, v.counter, sh)) {
        double tot[3];
        reduce_partials<3>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            PcgState *st = v.st;
            st->bb = tot[0];
            st->rz = tot[1];
            st->rz_old = 1.0;
            st->rr = tot[2];
            const double t = fmax(rtol * sqrt(tot[0]), abs_floor);
            st->tol2 = t * t;
            st->iter = 0;
            st->max_iters = max_iters;
            st->status = KRYLOV_OK;
            st->done = (tot[0] == 0.0 || tot[2] <= st->tol2) ? 1 : 0;
            if (!finite(tot[0]) || !finite(tot[1])) {
                st->done = 1;
                st->status = KRYLOV_NONFINITE;
            }
        }
    }
}

// p_new = z + beta p_old (own row and, on the fly, neighbour rows); q = A p_new.
// Two rows per thread are kept in flight so that their gathers overlap.
template <typename T>
__global__ void __launch_bounds__(MCB_THREADS) k_pcg_iter1(EllT<T> A, PcgVectorsT<T> v,
                                                           const typename Pair<T>::type *__restrict__ X,
                                                           typename Pair<T>::type *__restrict__ Y)
{
    pdl_wait();
    using T2 = typename Pair<T>::type;
    __shared__ double sh[1][MCB_THREADS];
    const PcgState *st = v.st;
    if (st->done) return;
    const int N = A.N;
    const double beta = (st->iter == 0) ? 0.0 : st->rz / st->rz_old;
    const int stride = gridDim.x * blockDim.x;
    double acc[1] = {0.0};
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < N; i0 += 2 * stride) {
        const int i1 = i0 + stride;
        const bool has1 = i1 < N;
        const int j1 = has1 ? i1 : i0;
        const T2 sa = X[i0], sb = X[j1];
        const T bt = (T)beta;
        const T pa = sa.x + bt * sa.y, pb = sb.x + bt * sb.y;
        auto apply = [&](int i, T p) {
            return with_row_cols(A.dc, A.col, N, i, [&](const int(&c)[6]) {
                T q = A.diag[i] * p;
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    const T2 g = X[c[k]];
                    q += ell_val(A.dc, A.off, N, i, k, c[k]) * (g.x + bt * g.y);
                }
                return q;
            });
        };
        const T qa = apply(i0, pa), qb = apply(j1, pb);
        Y[i0].y = pa;
        v.q[i0] = qa;
        acc[0] += (double)pa * (double)qa;
        if (has1) {
            Y[i1].y = pb;
            v.q[i1] = qb;
            acc[0] += (double)pb * (double)qb;
        }
    }
    if (publish_partials<1>(acc, v.partials, v.counter, sh)) {
        double tot[1];
        reduce_partials<1>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            PcgState *s = v.st;
            s->pq = tot[0];
            s->alpha = s->rz / tot[0];
            if (!finite(s->alpha)) {
                s->done = 1;
                s->status = KRYLOV_NONFINITE;
            }
        }
    }
}

// x += alpha p; r -= alpha q; z = r / diag; convergence on ||r||.
__global__ void __launch_bounds__(MCB_THREADS) k_pcg_iter2(Ell A, PcgVectors v, double2 *__restrict__ Y)
{
    pdl_wait();
    __shared__ double sh[2][MCB_THREADS];
    const PcgState *st = v.st;
    if (st->done) return;
    const int N = A.N;
    const double alpha = st->alpha;
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double p = Y[i].y;
        v.x[i] += alpha * p;
        const double ri = v.r[i] - alpha * v.q[i];
        const double di = A.diag[i];
        const double zi = (di != 0.0) ? ri / di : ri;  // a zero row (isolated cell) is left unpreconditioned
        v.r[i] = ri;
        Y[i].x = zi;
        acc[0] += ri * zi;
        acc[1] += ri * ri;
    }
    if (publish_partials<2>(acc, v.partials, v.counter, sh)) {
        double tot[2];
        reduce_partials<2>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            PcgState *s = v.st;
            s->rz_old = s->rz;
            s->rz = tot[0];
            s->rr = tot[1];
            s->iter += 1;
            if (!finite(tot[0]) || !finite(tot[1])) {
                s->done = 1;
                s->status = KRYLOV_NONFINITE;
            } else if (tot[1] <= s->tol2) {
                s->done = 1;
            } else if (s->iter >= s->max_iters) {
                s->done = 1;
                s->status = KRYLOV_NOT_CONVERGED;
            }
        }
    }
}

// Initialisation for the AMG-preconditioned PCG: r = b - mean(b), x = 0;
// z comes from the first V-cycle (amg.cu), which also sets r . z.
template <typename T>
__global__ void __launch_bounds__(MCB_THREADS) k_pcg_init_amg(EllT<T> A, PcgVectorsT<T> v, double rtol,
                                                              double abs_floor, int max_iters, int project,
                                                              int use_x0)
{
    using T2 = typename Pair<T>::type;
    __shared__ double sh[2][MCB_THREADS];
    const int N = A.N;
    const double mean = project ? v.st->mean : 0.0;
    double acc[2] = {0.0, 0.0};  // b.b, r.r
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const T bi = (T)((double)v.b[i] - mean);
        T ri = bi;
        if (use_x0) {
            T ax = A.diag[i] * v.x[i];
            int c_[6];
            row_cols(A, i, c_);
#pragma unroll
            for (int k = 0; k < 6; k++) ax += ell_val(A.dc, A.off, N, i, k, c_[k]) * v.x[c_[k]];
            ri = bi - ax;
        } else {
            v.x[i] = (T)0;
        }
        v.r[i] = ri;
        v.zp[0][i] = T2{(T)0, (T)0};
        v.zp[1][i] = T2{(T)0, (T)0};
        acc[0] += (double)bi * (double)bi;
        acc[1] += (double)ri * (double)ri;
    }
    if (publish_partials<2>(acc, v.partials, v.counter, sh)) {
        double tot[2];
        reduce_partials<2>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            PcgState *st = v.st;
            st->bb = tot[0];
            st->rr = tot[1];
            st->rz = 0.0;
            st->rz_old = 1.0;
            const double t = fmax(rtol * sqrt(tot[0]), abs_floor);
            st->tol2 = t * t;
            st->iter = 0;
            st->max_iters = max_iters;
            st->status = KRYLOV_OK;
            st->done = (tot[0] == 0.0 || tot[1] <= st->tol2) ? 1 : 0;
            if (!finite(tot[0])) {
                st->done = 1;
                st->status = KRYLOV_NONFINITE;
            }
        }
    }
}

// x += alpha p; r -= alpha q; convergence on ||r||.  z follows from the V-cycle.
template <typename T>
__global__ void __launch_bounds__(MCB_THREADS) k_pcg_iter2_amg(EllT<T> A, PcgVectorsT<T> v,
                                                               const typename Pair<T>::type *__restrict__ Y)
{
    pdl_wait();
    __shared__ double sh[1][MCB_THREADS];
    const PcgState *st = v.st;
    if (st->done) return;
    const int N = A.N;
    const T alpha = (T)st->alpha;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        v.x[i] += alpha * Y[i].y;
        const T ri = v.r[i] - alpha * v.q[i];
        v.r[i] = ri;
        acc[0] += (double)ri * (double)ri;
    }
    if (publish_partials<1>(acc, v.partials, v.counter, sh)) {
        double tot[1];
        reduce_partials<1>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            PcgState *s = v.st;
            s->rr = tot[0];
            s->iter += 1;
            if (!finite(tot[0])) {
                s->done = 1;
                s->status = KRYLOV_NONFINITE;
            } else if (tot[0] <= s->tol2) {
                s->done = 1;
            } else if (s->iter >= s->max_iters) {
                s->done = 1;
                s->status = KRYLOV_NOT_CONVERGED;
            }
        }
    }
}

// ------------------------------------------------ FP64 iterative refinement
// Outer loop of the FP32-refined pressure solve: FP64 solution, FP64 true
// residual r = b' - A x with b' = b - mean(b), FP64 norms; each inner FP32
// solve gets r rounded to FP32 as its right-hand side.

// (A x)_i of the FP64 system.
__device__ __forceinline__ double ell_row(const Ell &A, const double *__restrict__ x, int i)
{
    return with_row_cols(A.dc, A.col, A.N, i, [&](const int(&c)[6]) {
        double ax = A.diag[i] * x[i];
#pragma unroll
        for (int k = 0; k < 6; k++) ax += ell_val(A.dc, A.off, A.N, i, k, c[k]) * x[c[k]];
        return ax;
    });
}

// (A xa)_i and (A xb)_i in one pass over the row (a null vector gives 0).
struct RowPair {
    double u, w;
};
__device__ __forceinline__ RowPair ell_row2(const Ell &A, const double *__restrict__ xa, const double *__restrict__ xb,
                                            int i)
{
    return with_row_cols(A.dc, A.col, A.N, i, [&](const int(&c)[6]) {
        RowPair o{xa ? A.diag[i] * xa[i] : 0.0, xb ? A.diag[i] * xb[i] : 0.0};
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const double a = ell_val(A.dc, A.off, A.N, i, k, c[k]);
            if (xa) o.u += a * xa[c[k]];
            if (xb) o.w += a * xb[c[k]];
        }
        return o;
    });
}

__global__ void __launch_bounds__(MCB_THREADS) k_ir_init(Ell A, const double *__restrict__ b, double *__restrict__ x,
                                                         double *__restrict__ r, float *__restrict__ r32, PcgState *st,
                                                         double *partials, unsigned int *counter, double rtol,
                                                         double abs_floor, int max_outer, int use_x0,
                                                         IrGuess g)
{
    __shared__ double sh[2][MCB_THREADS];
    const int N = A.N;
    const double mean = st->mean;
    // the guess's combination (see GuessState), applied here
    const double al = g.gs ? g.gs->coef[0] : 0.0, be = g.gs ? g.gs->coef[1] : 0.0;
    const bool ua = g.gs && g.xa && al != 0.0, ub = g.gs && g.xb && be != 0.0;
    double acc[2] = {0.0, 0.0};  // b'.b', r.r
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double bi = b[i] - mean;
        double ri = bi;
        if (g.gs) {
            x[i] = (ua ? al * g.xa[i] : 0.0) + (ub ? be * g.xb[i] : 0.0);
            ri = bi - ((ua ? al * g.u[i] : 0.0) + (ub ? be * g.w[i] : 0.0));
        } else if (use_x0) {
            ri = bi - ell_row(A, x, i);
        } else {
            x[i] = 0.0;
        }
        if (r) r[i] = ri;
        r32[i] = (float)ri;
        acc[0] += bi * bi;
        acc[1] += ri * ri;
    }
    if (publish_partials<2>(acc, partials, counter, sh)) {
        double tot[2];
        reduce_partials<2>(tot, partials, counter, sh);
        if (threadIdx.x == 0) {
            st->bb = tot[0];
            st->rr = tot[1];
            const double t = fmax(rtol * sqrt(tot[0]), abs_floor);
            st->tol2 = t * t;
            st->iter = 0;
            st->max_iters = max_outer;
            st->status = KRYLOV_OK;
            st->done = (tot[0] == 0.0 || tot[1] <= st->tol2) ? 1 : 0;
            if (!finite(tot[0]) || !finite(tot[1])) {
                st->done = 1;
                st->status = KRYLOV_NONFINITE;
            }
        }
    }
}


// Dot products of b' = b - mean, u = A xa and w = A xb; the last block
// solves the 2 x 2 least-squares problem min ||b' - alpha u - beta w||
// (1 x 1 when a candidate is absent or the two are colinear).
__global__ void __launch_bounds__(MCB_THREADS) k_guess_residuals(Ell A, const double *__restrict__ b,
                                                                 const PcgState *__restrict__ st,
                                                                 const double *__restrict__ xa,
                                                                 const double *__restrict__ xb, GuessState *gs,
                                                                 double *partials, unsigned int *counter,
                                                                 double *__restrict__ uo, double *__restrict__ wo)
{
    __shared__ double sh[6][MCB_THREADS];
    const int N = A.N;
    const double mean = st->mean;
    // bb, bu, bw, uu, uw, ww
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double bi = b[i] - mean;
        const RowPair uw = ell_row2(A, xa, xb, i);
        const double u = uw.u, w = uw.w;
        if (uo && xa) uo[i] = u;
        if (wo && xb) wo[i] = w;
        acc[0] += bi * bi;
        acc[1] += bi * u;
        acc[2] += bi * w;
        acc[3] += u * u;
        acc[4] += u * w;
        acc[5] += w * w;
    }
    if (publish_partials<6>(acc, partials, counter, sh)) {
        double t[6];
        reduce_partials<6>(t, partials, counter, sh);
        if (threadIdx.x == 0) {
            const double bb = t[0], bu = t[1], bw = t[2], uu = t[3], uw = t[4], ww = t[5];
            gs->bb = bb;
            gs->rr[0] = xa ? fmax(bb - 2.0 * bu + uu, 0.0) : -1.0;
            gs->rr[1] = xb ? fmax(bb - 2.0 * bw + ww, 0.0) : -1.0;
            double al = 0.0, be = 0.0;
            const bool ha = xa && uu > 0 && finite(uu), hb = xb && ww > 0 && finite(ww);
            const double det = uu * ww - uw * uw;
            if (ha && hb && det > 1e-12 * uu * ww) {
                al = (bu * ww - bw * uw) / det;
                be = (bw * uu - bu * uw) / det;
            } else if (hb) {
                be = bw / ww;
            } else if (ha) {
                al = bu / uu;
            }
            // residual of the combination: bb - 2 (al bu + be bw) + |al u + be w|^2
            double rc = bb - 2.0 * (al * bu + be * bw) + (al * al * uu + 2.0 * al * be * uw + be * be * ww);
            int choice = 2;
            if (!finite(rc) || !(rc < bb) || !finite(al) || !finite(be)) {
                choice = -1;
                al = be = 0.0;
                rc = bb;
            }
            gs->coef[0] = al;
            gs->coef[1] = be;
            gs->rc = fmax(rc, 0.0);
            gs->choice = choice;
        }
    }
}

// x = alpha xa + beta xb (zero for choice -1).
__global__ void __launch_bounds__(MCB_THREADS) k_guess_apply(int N, double *__restrict__ x,
                                                             const double *__restrict__ xa,
                                                             const double *__restrict__ xb,
                                                             const GuessState *__restrict__ gs)
{
    const double al = gs->coef[0], be = gs->coef[1];
    const bool ua = xa && al != 0.0, ub = xb && be != 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        x[i] = (ua ? al * xa[i] : 0.0) + (ub ? be * xb[i] : 0.0);
}

// With e set: the update x' = x + e (the inner solution) in the same pass,
// evaluated at each row where the product needs it and stored in xout (not
// in x, which neighbouring rows still read); without e, x' = x.  r may be
// null (the FP64 residual is then not stored).
__global__ void __launch_bounds__(MCB_THREADS) k_ir_residual(Ell A, const double *__restrict__ b,
                                                             const double *__restrict__ x, const float *__restrict__ e,
                                                             double *__restrict__ xout, double *__restrict__ r,
                                                             float *__restrict__ r32, PcgState *st, double *partials,
                                                             unsigned int *counter)
{
    pdl_wait();
    __shared__ double sh[1][MCB_THREADS];
    const int N = A.N;
    if (st->done) {  // nothing to add: xout still has to hold the solution
        if (e)
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) xout[i] = x[i];
        return;
    }
    const double mean = st->mean;
    double acc[1] = {0.0};
    auto xv = [&](int j) { return e ? x[j] + (double)e[j] : x[j]; };
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double xi = xv(i);
        const double ax = with_row_cols(A.dc, A.col, N, i, [&](const int(&c)[6]) {
            double s = A.diag[i] * xi;
#pragma unroll
            for (int k = 0; k < 6; k++) s += ell_val(A.dc, A.off, N, i, k, c[k]) * xv(c[k]);
            return s;
        });
        if (e) xout[i] = xi;
        const double ri = (b[i] - mean) - ax;
        if (r) r[i] = ri;
        r32[i] = (float)ri;
        acc[0] += ri * ri;
    }
    if (publish_partials<1>(acc, partials, counter, sh)) {
        double tot[1];
        reduce_partials<1>(tot, partials, counter, sh);
        if (threadIdx.x == 0) {
            st->rr = tot[0];
            st->iter += 1;
            if (!finite(tot[0])) {
                st->done = 1;
                st->status = KRYLOV_NONFINITE;
            } else if (tot[0] <= st->tol2) {
                st->done = 1;
            } else if (st->iter >= st->max_iters) {
                st->done = 1;
                st->status = KRYLOV_NOT_CONVERGED;
            }
        }
    }
}

__global__ void __launch_bounds__(MCB_THREADS) k_pcg_xmean(int N, PcgVectors v)
{
    __shared__ double sh[1][MCB_THREADS];
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) acc[0] += v.x[i];
    if (publish_partials<1>(acc, v.partials, v.counter, sh)) {
        double tot[1];
        reduce_partials<1>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) v.st->xmean = tot[0] / (double)N;
    }
}

__global__ void __launch_bounds__(MCB_THREADS) k_pcg_sub_xmean(int N, PcgVectors v)
{
    const double m = v.st->xmean;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) v.x[i] -= m;
}

void pcg_mean(cudaStream_t s, const Ell &A, const PcgVectors &v)
{
    k_pcg_mean<<<krylov_grid(A.N), MCB_THREADS, 0, s>>>(A.N, v.b, v);
}
void pcg_init(cudaStream_t s, const Ell &A, const PcgVectors &v, double rtol, double abs_floor, int max_iters,
              int use_x0, int project)
{
    k_pcg_init<<<krylov_grid(A.N), MCB_THREADS, 0, s>>>(A, v, rtol, abs_floor, max_iters, use_x0, project);
}
template <typename T>
void pcg_iter1(cudaStream_t s, const EllT<T> &A, const PcgVectorsT<T> &v, int pin)
{
    pdl_launch(k_pcg_iter1<T>, krylov_grid(A.N), MCB_THREADS, 0, s, A, v, v.zp[pin], v.zp[pin ^ 1]);
}
void pcg_iter2(cudaStream_t s, const Ell &A, const PcgVectors &v, int pnew)
{
    k_pcg_iter2<<<krylov_grid(A.N), MCB_THREADS, 0, s>>>(A, v, v.zp[pnew]);
}
template <typename T>
void pcg_init_amg(cudaStream_t s, const EllT<T> &A, const PcgVectorsT<T> &v, double rtol, double abs_floor,
                  int max_iters, int project, int use_x0)
{
    k_pcg_init_amg<T><<<krylov_grid(A.N), MCB_THREADS, 0, s>>>(A, v, rtol, abs_floor, max_iters, project, use_x0);
}
template <typename T>
void pcg_iter2_amg(cudaStream_t s, const EllT<T> &A, const PcgVectorsT<T> &v, int pnew)
{
    pdl_launch(k_pcg_iter2_amg<T>, krylov_grid(A.N), MCB_THREADS, 0, s, A, v, v.zp[pnew]);
}
#define MCB_INSTANTIATE_PCG(T)                                                                                  \
    template void pcg_iter1<T>(cudaStream_t, const EllT<T> &, const PcgVectorsT<T> &, int);                   \
    template void pcg_init_amg<T>(cudaStream_t, const EllT<T> &, const PcgVectorsT<T> &, double, double, int, \
                                  int, int);                                                                  \
    template void pcg_iter2_amg<T>(cudaStream_t, const EllT<T> &, const PcgVectorsT<T> &, int);
MCB_INSTANTIATE_PCG(double)
MCB_INSTANTIATE_PCG(float)
void ir_init(cudaStream_t s, const Ell &A, const double *b, double *x, double *r, float *r32, PcgState *st,
             double *partials, unsigned int *counter, double rtol, double abs_floor, int max_outer, int use_x0,
             const IrGuess &g)
{
    k_ir_init<<<krylov_grid(A.N), MCB_THREADS, 0, s>>>(A, b, x, r, r32, st, partials, counter, rtol, abs_floor,
                                                       max_outer, use_x0, g);
}
void guess_residuals(cudaStream_t s, const Ell &A, const double *b, const PcgState *st, const double *xa,
                     const double *xb, GuessState *gs, double *partials, unsigned int *counter, double *uo,
                     double *wo)
{
    k_guess_residuals<<<krylov_grid(A.N), MCB_THREADS, 0, s>>>(A, b, st, xa, xb, gs, partials, counter, uo, wo);
}
void guess_apply(cudaStream_t s, int N, double *x, const double *xa, const double *xb, const GuessState *gs)
{
    k_guess_apply<<<krylov_grid(N), MCB_THREADS, 0, s>>>(N, x, xa, xb, gs);
}
void ir_residual(cudaStream_t s, const Ell &A, const double *b, const double *x, double *r, float *r32, PcgState *st,
                 double *partials, unsigned int *counter, const float *e, double *xout)
{
    k_ir_residual<<<krylov_grid(A.N), MCB_THREADS, 0, s>>>(A, b, x, e, xout, r, r32, st, partials, counter);
}
void pcg_xmean(cudaStream_t s, int N, const PcgVectors &v) { k_pcg_xmean<<<krylov_grid(N), MCB_THREADS, 0, s>>>(N, v); }
void pcg_sub_xmean(cudaStream_t s, int N, const PcgVectors &v)
{
    k_pcg_sub_xmean<<<krylov_grid(N), MCB_THREADS, 0, s>>>(N, v);
}

// ----------------------------------------------------------------- BiCGStab
//
// Templated on the storage type T; the scalars of an iteration are cast to
// T once, so T = double is the plain FP64 solver and T = float keeps every
// vector and matrix access in FP32 (dot products accumulate in FP64).

template <typename T, int R>
__global__ void __launch_bounds__(MCB_THREADS) k_bicg_init(EllT<T> A, BicgVectorsT<T, R> v, double rtol,
                                                           int max_iters)
{
    __shared__ double sh[R][MCB_THREADS];
    const int N = A.N;
    double acc[R];
#pragma unroll
    for (int j = 0; j < R; j++) acc[j] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int j = 0; j < R; j++) {
            const size_t o = (size_t)j * N + i;
            const T bi = v.b[o];
            v.x[j][i] = (T)0;
            v.r[o] = bi;
            v.r0[o] = bi;
            v.p[0][o] = (T)0;
            v.p[1][o] = (T)0;
            v.v[0][o] = (T)0;
            v.v[1][o] = (T)0;
            acc[j] += (double)bi * (double)bi;
        }
    }
    if (publish_partials<R>(acc, v.partials, v.counter, sh)) {
        double tot[R];
        reduce_partials<R>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            BicgState<R> *st = v.st;
            int all = 1;
            for (int j = 0; j < R; j++) {
                st->bb[j] = tot[j];
                st->rr[j] = tot[j];
                st->rho_new[j] = tot[j];
                st->rho[j] = 1.0;
                st->alpha[j] = 1.0;
                st->omega[j] = 1.0;
                st->tol2[j] = rtol * rtol * tot[j];
                st->iter[j] = 0;
                st->status[j] = finite(tot[j]) ? KRYLOV_OK : KRYLOV_NONFINITE;
                st->done[j] = (tot[j] == 0.0 || !finite(tot[j])) ? 1 : 0;
                all &= st->done[j];
            }
            st->all_done = all;
            st->max_iters = max_iters;
        }
    }
}

// Row blocks and right-hand sides of a BiCGStab launch: fused (every block
// works on all R systems) or split (block b works on system b % R of row
// block b / R; the R blocks of a row block run together, so the matrix is
// read from L2 R - 1 times out of R).  The split form keeps one system's state
// per thread and runs at full occupancy; it is used for the FP32 inner solves.
template <int R, bool SPLIT>
struct BicgBlocks {
    int j0, j1, b, nb;
    __device__ BicgBlocks()
    {
        if (SPLIT) {
            j0 = blockIdx.x % R;
            j1 = j0 + 1;
            b = blockIdx.x / R;
            nb = gridDim.x / R;
        } else {
            j0 = 0;
            j1 = R;
            b = blockIdx.x;
            nb = gridDim.x;
        }
    }
};

template <typename P, int R>
__device__ __forceinline__ P pick(P const (&a)[R], int j)
{
    P r = a[0];
#pragma unroll
    for (int q = 1; q < R; q++) r = (j == q) ? a[q] : r;
    return r;
}

// p_new = r + beta (p_old - omega v_old); v_new = A p_new.
template <typename T, int R, bool SPLIT>
__global__ void __launch_bounds__(MCB_THREADS, SPLIT ? 8 : 4) k_bicg_1(EllT<T> A, BicgVectorsT<T, R> v, const T *__restrict__ po,
                                                        const T *__restrict__ vo, T *__restrict__ pn,
                                                        T *__restrict__ vn)
{
    pdl_wait();
    __shared__ double sh[R][MCB_THREADS];
    const BicgState<R> *st = v.st;
    if (st->all_done) return;
    const int N = A.N;
    const BicgBlocks<R, SPLIT> bb;
    double acc[R];
#pragma unroll
    for (int j = 0; j < R; j++) acc[j] = 0.0;
    if (SPLIT) {
        const int j = bb.j0;
        if (!st->done[j]) {
            const T beta = (T)((st->rho_new[j] / st->rho[j]) * (st->alpha[j] / st->omega[j]));
            const T omega = (T)st->omega[j];
            const size_t base = (size_t)j * N;
            double a = 0.0;
            for (int i = bb.b * blockDim.x + threadIdx.x; i < N; i += bb.nb * blockDim.x) {
                int colk[6];
                row_cols(A, i, colk);
                const T pi = v.r[base + i] + beta * (po[base + i] - omega * vo[base + i]);
                T vi = A.diag[i] * pi;
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    const size_t q = base + colk[k];
                    vi += A.off[(size_t)k * N + i] * (v.r[q] + beta * (po[q] - omega * vo[q]));
                }
                pn[base + i] = pi;
                vn[base + i] = vi;
                a += (double)v.r0[base + i] * (double)vi;
            }
#pragma unroll
            for (int q = 0; q < R; q++) acc[q] = (q == j) ? a : 0.0;
        }
    } else {
        T beta[R], omega[R];
        bool act[R];
#pragma unroll
        for (int j = 0; j < R; j++) {
            act[j] = !st->done[j];
            beta[j] = (T)((st->rho_new[j] / st->rho[j]) * (st->alpha[j] / st->omega[j]));
            omega[j] = (T)st->omega[j];
        }
        for (int i = bb.b * blockDim.x + threadIdx.x; i < N; i += bb.nb * blockDim.x) {
            const T d = A.diag[i];
            T offk[6];
            int colk[6];
            row_cols(A, i, colk);
#pragma unroll
            for (int k = 0; k < 6; k++) offk[k] = A.off[(size_t)k * N + i];
#pragma unroll
            for (int j = 0; j < R; j++) {
                if (!act[j]) continue;
                const size_t base = (size_t)j * N;
                const T pi = v.r[base + i] + beta[j] * (po[base + i] - omega[j] * vo[base + i]);
                T vi = d * pi;
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    const size_t q = base + colk[k];
                    vi += offk[k] * (v.r[q] + beta[j] * (po[q] - omega[j] * vo[q]));
                }
                pn[base + i] = pi;
                vn[base + i] = vi;
                acc[j] += (double)v.r0[base + i] * (double)vi;
            }
        }
    }
    if (publish_partials<R>(acc, v.partials, v.counter, sh)) {
        double tot[R];
        reduce_partials<R>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            BicgState<R> *s = v.st;
            for (int j = 0; j < R; j++) {
                if (s->done[j]) continue;
                s->alpha[j] = s->rho_new[j] / tot[j];
                if (!finite(s->alpha[j])) {
                    s->done[j] = 1;
                    s->status[j] = KRYLOV_NONFINITE;
                }
            }
        }
    }
}

// s = r - alpha v; t = A s.
template <typename T, int R, bool SPLIT>
__global__ void __launch_bounds__(MCB_THREADS, SPLIT ? 8 : 4) k_bicg_2(EllT<T> A, BicgVectorsT<T, R> v, const T *__restrict__ vv)
{
    pdl_wait();
    __shared__ double sh[2 * R][MCB_THREADS];
    const BicgState<R> *st = v.st;
    if (st->all_done) return;
    const int N = A.N;
    const BicgBlocks<R, SPLIT> bb;
    double acc[2 * R];
#pragma unroll
    for (int j = 0; j < 2 * R; j++) acc[j] = 0.0;
    if (SPLIT) {
        const int j = bb.j0;
        if (!st->done[j]) {
            const T alpha = (T)st->alpha[j];
            const size_t base = (size_t)j * N;
            double ts = 0.0, tt = 0.0;
            for (int i = bb.b * blockDim.x + threadIdx.x; i < N; i += bb.nb * blockDim.x) {
                int colk[6];
                row_cols(A, i, colk);
                const T si = v.r[base + i] - alpha * vv[base + i];
                T ti = A.diag[i] * si;
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    const size_t q = base + colk[k];
                    ti += A.off[(size_t)k * N + i] * (v.r[q] - alpha * vv[q]);
                }
                v.s[base + i] = si;
                v.t[base + i] = ti;
                ts += (double)ti * (double)si;
                tt += (double)ti * (double)ti;
            }
#pragma unroll
            for (int q = 0; q < R; q++) {
                acc[2 * q] = (q == j) ? ts : 0.0;
                acc[2 * q + 1] = (q == j) ? tt : 0.0;
            }
        }
    } else {
        T alpha[R];
        bool act[R];
#pragma unroll
        for (int j = 0; j < R; j++) {
            act[j] = !st->done[j];
            alpha[j] = (T)st->alpha[j];
        }
        for (int i = bb.b * blockDim.x + threadIdx.x; i < N; i += bb.nb * blockDim.x) {
            const T d = A.diag[i];
            T offk[6];
            int colk[6];
            row_cols(A, i, colk);
#pragma unroll
            for (int k = 0; k < 6; k++) offk[k] = A.off[(size_t)k * N + i];
#pragma unroll
            for (int j = 0; j < R; j++) {
                if (!act[j]) continue;
                const size_t base = (size_t)j * N;
                const T si = v.r[base + i] - alpha[j] * vv[base + i];
                T ti = d * si;
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    const size_t q = base + colk[k];
                    ti += offk[k] * (v.r[q] - alpha[j] * vv[q]);
                }
                v.s[base + i] = si;
                v.t[base + i] = ti;
                acc[2 * j] += (double)ti * (double)si;
                acc[2 * j + 1] += (double)ti * (double)ti;
            }
        }
    }
    if (publish_partials<2 * R>(acc, v.partials, v.counter, sh)) {
        double tot[2 * R];
        reduce_partials<2 * R>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            BicgState<R> *s = v.st;
            for (int j = 0; j < R; j++) {
                if (s->done[j]) continue;
                const double tt = tot[2 * j + 1];
                s->omega[j] = (tt != 0.0) ? tot[2 * j] / tt : 0.0;
            }
        }
    }
}

// x += alpha p + omega s; r = s - omega t; convergence on ||r||.
template <typename T, int R, bool SPLIT>
__global__ void __launch_bounds__(MCB_THREADS, SPLIT ? 8 : 1) k_bicg_3(EllT<T> A, BicgVectorsT<T, R> v, const T *__restrict__ p)
{
    pdl_wait();
    __shared__ double sh[2 * R][MCB_THREADS];
    const BicgState<R> *st = v.st;
    if (st->all_done) return;
    const int N = A.N;
    const BicgBlocks<R, SPLIT> bb;
    double acc[2 * R];
#pragma unroll
    for (int j = 0; j < 2 * R; j++) acc[j] = 0.0;
    if (SPLIT) {
        const int j = bb.j0;
        if (!st->done[j]) {
            const T alpha = (T)st->alpha[j], omega = (T)st->omega[j];
            T *x = pick(v.x, j);
            const size_t base = (size_t)j * N;
            double rr0 = 0.0, rr = 0.0;
            for (int i = bb.b * blockDim.x + threadIdx.x; i < N; i += bb.nb * blockDim.x) {
                const size_t o = base + i;
                const T si = v.s[o];
                x[i] += alpha * p[o] + omega * si;
                const T ri = si - omega * v.t[o];
                v.r[o] = ri;
                rr0 += (double)v.r0[o] * (double)ri;
                rr += (double)ri * (double)ri;
            }
#pragma unroll
            for (int q = 0; q < R; q++) {
                acc[2 * q] = (q == j) ? rr0 : 0.0;
                acc[2 * q + 1] = (q == j) ? rr : 0.0;
            }
        }
    } else {
        T alpha[R], omega[R];
        bool act[R];
#pragma unroll
        for (int j = 0; j < R; j++) {
            act[j] = !st->done[j];
            alpha[j] = (T)st->alpha[j];
            omega[j] = (T)st->omega[j];
        }
        for (int i = bb.b * blockDim.x + threadIdx.x; i < N; i += bb.nb * blockDim.x) {
#pragma unroll
            for (int j = 0; j < R; j++) {
                if (!act[j]) continue;
                const size_t o = (size_t)j * N + i;
                const T si = v.s[o];
                v.x[j][i] += alpha[j] * p[o] + omega[j] * si;
                const T ri = si - omega[j] * v.t[o];
                v.r[o] = ri;
                acc[2 * j] += (double)v.r0[o] * (double)ri;
                acc[2 * j + 1] += (double)ri * (double)ri;
            }
        }
    }
    if (publish_partials<2 * R>(acc, v.partials, v.counter, sh)) {
        double tot[2 * R];
        reduce_partials<2 * R>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            BicgState<R> *s = v.st;
            int all = 1;
            for (int j = 0; j < R; j++) {
                if (!s->done[j]) {
                    s->rho[j] = s->rho_new[j];
                    s->rho_new[j] = tot[2 * j];
                    s->rr[j] = tot[2 * j + 1];
                    s->iter[j] += 1;
                    if (!finite(tot[2 * j]) || !finite(tot[2 * j + 1])) {
                        s->done[j] = 1;
                        s->status[j] = KRYLOV_NONFINITE;
                    } else if (tot[2 * j + 1] <= s->tol2[j]) {
                        s->done[j] = 1;
                    } else if (s->omega[j] == 0.0 || tot[2 * j] == 0.0 || s->iter[j] >= s->max_iters) {
                        s->done[j] = 1;
                        s->status[j] = KRYLOV_NOT_CONVERGED;
                    }
                }
                all &= s->done[j];
            }
            s->all_done = all;
        }
    }
}

// Refinement: x = 0, r32 = (float) D^-1 b (the inner FP32 systems are the
// rows of A scaled by 1 / diag, see k_round_ell), norms and tolerances.
template <int R>
__global__ void __launch_bounds__(MCB_THREADS) k_bir_init(Ell A, BirVectors<R> v, double rtol, int max_outer)
{
    __shared__ double sh[R][MCB_THREADS];
    const int N = A.N;
    double acc[R];
#pragma unroll
    for (int j = 0; j < R; j++) acc[j] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int j = 0; j < R; j++) {
            const double bi = v.b[(size_t)j * N + i];
            v.x[j][i] = 0.0;
            v.r32[(size_t)j * N + i] = (float)(bi * row_scale(A.diag, i));
            acc[j] += bi * bi;
        }
    }
    if (publish_partials<R>(acc, v.partials, v.counter, sh)) {
        double tot[R];
        reduce_partials<R>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            BirState<R> *st = v.st;
            int all = 1;
            for (int j = 0; j < R; j++) {
                st->bb[j] = tot[j];
                st->rr[j] = tot[j];
                st->tol2[j] = rtol * rtol * tot[j];
                st->status[j] = finite(tot[j]) ? KRYLOV_OK : KRYLOV_NONFINITE;
                st->done[j] = (tot[j] == 0.0 || !finite(tot[j])) ? 1 : 0;
                all &= st->done[j];
            }
            st->iter = 0;
            st->all_done = all;
            st->max_outer = max_outer;
        }
    }
}

// x_j += e_j for the systems still open.
template <int R>
__global__ void __launch_bounds__(MCB_THREADS) k_bir_add(int N, BirVectors<R> v)
{
    const BirState<R> *st = v.st;
    if (st->all_done) return;
    bool act[R];
#pragma unroll
    for (int j = 0; j < R; j++) act[j] = !st->done[j];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int j = 0; j < R; j++)
            if (act[j]) v.x[j][i] += (double)v.e[(size_t)j * N + i];
}

// r = b - A x in FP64, r32 = (float) r (zero for closed systems), norms and
// convergence.
template <int R>
__global__ void __launch_bounds__(MCB_THREADS) k_bir_residual(Ell A, BirVectors<R> v)
{
    __shared__ double sh[R][MCB_THREADS];
    BirState<R> *st = v.st;
    if (st->all_done) return;
    const int N = A.N;
    bool act[R];
#pragma unroll
    for (int j = 0; j < R; j++) act[j] = !st->done[j];
    double acc[R];
#pragma unroll
    for (int j = 0; j < R; j++) acc[j] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double d = A.diag[i];
        double offk[6];
        int colk[6];
        row_cols(A, i, colk);
#pragma unroll
        for (int k = 0; k < 6; k++) offk[k] = A.off[(size_t)k * N + i];
#pragma unroll
        for (int j = 0; j < R; j++) {
            const size_t o = (size_t)j * N + i;
            if (!act[j]) {
                v.r32[o] = 0.f;
                continue;
            }
            const double *x = v.x[j];
            double ax = d * x[i];
#pragma unroll
            for (int k = 0; k < 6; k++) ax += offk[k] * x[colk[k]];
            const double ri = v.b[o] - ax;
            v.r32[o] = (float)(ri * (d != 0.0 ? 1.0 / d : 1.0));  // the row-scaled inner system
            acc[j] += ri * ri;
        }
    }
    if (publish_partials<R>(acc, v.partials, v.counter, sh)) {
        double tot[R];
        reduce_partials<R>(tot, v.partials, v.counter, sh);
        if (threadIdx.x == 0) {
            int all = 1;
            st->iter += 1;
            for (int j = 0; j < R; j++) {
                if (!st->done[j]) {
                    st->rr[j] = tot[j];
                    if (!finite(tot[j])) {
                        st->done[j] = 1;
                        st->status[j] = KRYLOV_NONFINITE;
                    } else if (tot[j] <= st->tol2[j]) {
                        st->done[j] = 1;
                    } else if (st->iter >= st->max_outer) {
                        st->done[j] = 1;
                        st->status[j] = KRYLOV_NOT_CONVERGED;
                    }
                }
                all &= st->done[j];
            }
            st->all_done = all;
        }
    }
}

__global__ void __launch_bounds__(MCB_THREADS) k_round_ell(int N, const double *__restrict__ diag,
                                                           const double *__restrict__ off, const uint32_t *__restrict__ code,
                                                           float *__restrict__ d32, float *__restrict__ o32)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const double sc = row_scale(diag, i);
        d32[i] = (float)(diag[i] * sc);
        float o[6];
        round_row_by_direction(off, code, N, i, o, sc);
#pragma unroll
        for (int k = 0; k < 6; k++) o32[(size_t)k * N + i] = o[k];
    }
}

template <typename T, int R>
void bicg_init_t(cudaStream_t s, const EllT<T> &A, const BicgVectorsT<T, R> &v, double rtol, int max_iters)
{
    k_bicg_init<T, R><<<krylov_grid(A.N), MCB_THREADS, 0, s>>>(A, v, rtol, max_iters);
}
// The first product and the update run in the split form (one block range
// per right-hand side; with one right-hand side the split form is the fused
// one with the register cap of full occupancy): 32 registers, 8 blocks of
// 256 per SM.  The update is a streaming kernel that the 70-register fused
// FP64 form held to 3 blocks per SM and 31 % of the DRAM bandwidth (same-box
// A/B at 2 x 128^3, plain pass: update 2.36 -> 1.42 ms, first product 2.77
// -> 2.65 ms).
template <typename T, int R>
constexpr bool bicg_split() { return true; }

template <typename T, int R>
void bicg_1_t(cudaStream_t s, const EllT<T> &A, const BicgVectorsT<T, R> &v, int pin)
{
    constexpr bool S = bicg_split<T, R>();
    pdl_launch(k_bicg_1<T, R, S>, krylov_grid(A.N) * (S ? R : 1), MCB_THREADS, 0, s, A, v, v.p[pin], v.v[pin],
               v.p[pin ^ 1], v.v[pin ^ 1]);
}
// The second product gathers two vectors per right-hand side: one pass over
// the matrix for all of them is faster than the split form here (which a
// single right-hand side uses, for its occupancy).
template <typename T, int R>
void bicg_2_t(cudaStream_t s, const EllT<T> &A, const BicgVectorsT<T, R> &v, int vnew)
{
    constexpr bool S = R == 1;
    pdl_launch(k_bicg_2<T, R, S>, krylov_grid(A.N), MCB_THREADS, 0, s, A, v, v.v[vnew]);
}
template <typename T, int R>
void bicg_3_t(cudaStream_t s, const EllT<T> &A, const BicgVectorsT<T, R> &v, int pnew)
{
    constexpr bool S = bicg_split<T, R>();
    pdl_launch(k_bicg_3<T, R, S>, krylov_grid(A.N) * (S ? R : 1), MCB_THREADS, 0, s, A, v, v.p[pnew]);
}
template <int R>
void bicg_init(cudaStream_t s, const Ell &A, const BicgVectors<R> &v, double rtol, int max_iters)
{
    bicg_init_t<double, R>(s, A, v, rtol, max_iters);
}
template <int R>
void bicg_1(cudaStream_t s, const Ell &A, const BicgVectors<R> &v, int pin)
{
    bicg_1_t<double, R>(s, A, v, pin);
}
template <int R>
void bicg_2(cudaStream_t s, const Ell &A, const BicgVectors<R> &v, int vnew)
{
    bicg_2_t<double, R>(s, A, v, vnew);
}
template <int R>
void bicg_3(cudaStream_t s, const Ell &A, const BicgVectors<R> &v, int pnew)
{
    bicg_3_t<double, R>(s, A, v, pnew);
}
template <int R>
void bir_init(cudaStream_t s, const Ell &A, const BirVectors<R> &v, double rtol, int max_outer)
{
    k_bir_init<R><<<krylov_grid(A.N), MCB_THREADS, 0, s>>>(A, v, rtol, max_outer);
}
template <int R>
void bir_add(cudaStream_t s, int N, const BirVectors<R> &v)
{
    k_bir_add<R><<<krylov_grid(N), MCB_THREADS, 0, s>>>(N, v);
}
template <int R>
void bir_residual(cudaStream_t s, const Ell &A, const BirVectors<R> &v)
{
    k_bir_residual<R><<<krylov_grid(A.N), MCB_THREADS, 0, s>>>(A, v);
}
// ------------------------------------------------------- x-line sweeps
//
// Splitting A = M - (M - A) with M the diagonal and the -x couplings of each
// x-line (a lower bidiagonal block per line: the upwind direction of the
// x-directed flow): one step solves M e_new = r - (M - A) e_prev, i.e. the
// +x, y and z couplings of the previous iterate go to the right-hand side
// and each line is a first-order recurrence e_k = (rhs_k - a_k e_{k-1}) / b_k.
// A is an M-matrix (positive diagonal, non-positive couplings, diagonally
// dominant through the transient term), so this is a regular splitting and
// the iteration converges; with convection along +x the neglected couplings
// are small and each step reduces the residual by orders of magnitude.
//
// One warp per line.  First every cell's affine map e_k = p_k + q_k e_{k-1}
// is formed from coalesced loads (32 consecutive cells per step, all of the
// line's loads independent, so they overlap) and kept in shared memory; then
// the warp walks the line in chunks of 32: a warp scan (shuffles) composes
// the chunk's maps, the value entering the chunk is applied, and the chunk's
// last value is carried into the next chunk.
template <int R>
struct LineAdd {
    double *x[R];
    const BirState<R> *st = nullptr;  // null: store e_new
};

template <int R>
__global__ void __launch_bounds__(256, R == 1 ? 8 : 6) k_line_sweep(LineSystem L, const float *__restrict__ r,
                                                    const float *__restrict__ ep, float *__restrict__ en, int first,
                                                    LineAdd<R> add)
{
    extern __shared__ float sline[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int line = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int N = L.N, ex = L.ex;
    if (line >= N / ex) return;
    float *sq = sline + (size_t)warp * ex * (R + 1);  // q[ex], then p[R][ex]
    float *sp = sq + ex;
    const size_t base = (size_t)line * ex;
#pragma unroll 1
    for (int c = lane; c < ex; c += 32) {
        const size_t i = base + c;
        const float a = L.off[(size_t)L.dxm * N + i];
        const float b = L.d[i];
        float rhs[R];
#pragma unroll
        for (int j = 0; j < R; j++) rhs[j] = r[(size_t)j * N + i];
        if (!first) {
            if (c + 1 < ex) {
                const float o = L.off[(size_t)L.dxp * N + i];
#pragma unroll
                for (int j = 0; j < R; j++) rhs[j] -= o * ep[(size_t)j * N + i + 1];
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const float o = L.off[(size_t)L.yz[u] * N + i];
                const long nb = min(max((long)i + L.yzoff[u], 0L), (long)N - 1);
#pragma unroll
                for (int j = 0; j < R; j++) rhs[j] -= o * ep[(size_t)j * N + nb];
            }
        }
        const float rb = 1.f / b;
        sq[c] = -a * rb;
#pragma unroll
        for (int j = 0; j < R; j++) sp[j * ex + c] = rhs[j] * rb;
    }
    __syncwarp();
    bool act[R];
#pragma unroll
    for (int j = 0; j < R; j++) act[j] = add.st && !add.st->done[j];
    float carry[R];
#pragma unroll
    for (int j = 0; j < R; j++) carry[j] = 0.f;
    for (int c0 = 0; c0 < ex; c0 += 32) {
        const int c = c0 + lane;
        float p[R], q = 1.f;
#pragma unroll
        for (int j = 0; j < R; j++) p[j] = 0.f;
        if (c < ex) {
            q = sq[c];
#pragma unroll
            for (int j = 0; j < R; j++) p[j] = sp[j * ex + c];
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            float pu[R];
#pragma unroll
            for (int j = 0; j < R; j++) pu[j] = __shfl_up_sync(0xffffffffu, p[j], off);
            const float qu = __shfl_up_sync(0xffffffffu, q, off);
            if (lane >= off) {
#pragma unroll
                for (int j = 0; j < R; j++) p[j] = p[j] + q * pu[j];
                q = q * qu;
            }
        }
#pragma unroll
        for (int j = 0; j < R; j++) {
            const float x = p[j] + q * carry[j];
            if (c < ex) {
                if (!add.st)
                    en[(size_t)j * N + base + c] = x;
                else if (act[j])
                    add.x[j][base + c] += (double)x;
            }
            carry[j] = __shfl_sync(0xffffffffu, x, 31);
        }
    }
}

template <int R>
void line_step(cudaStream_t s, const LineSystem &L, const float *r, const float *e_prev, float *e_new, int first,
               const BirVectors<R> *add)
{
    LineAdd<R> la{};
    if (add) {
        for (int j = 0; j < R; j++) la.x[j] = add->x[j];
        la.st = add->st;
    }
    const int lines = L.N / L.ex;
    const size_t per_warp = (size_t)L.ex * (R + 1) * sizeof(float);
    int warps = 8;
    while (warps > 1 && warps * per_warp > 48 * 1024) warps >>= 1;
    const int threads = 32 * warps;
    const int grid = (lines + warps - 1) / warps;
    k_line_sweep<R><<<grid, threads, warps * per_warp, s>>>(L, r, e_prev, e_new, first, la);
}
template void line_step<1>(cudaStream_t, const LineSystem &, const float *, const float *, float *, int,
                           const BirVectors<1> *);
template void line_step<3>(cudaStream_t, const LineSystem &, const float *, const float *, float *, int,
                           const BirVectors<3> *);

void round_ell(cudaStream_t s, int N, const double *diag, const double *off, const uint32_t *code, float *diag32,
               float *off32)
{
    k_round_ell<<<krylov_grid(N), MCB_THREADS, 0, s>>>(N, diag, off, code, diag32, off32);
}

#define MCB_INSTANTIATE_BICG_T(T, R)                                                                          \
    template void bicg_init_t<T, R>(cudaStream_t, const EllT<T> &, const BicgVectorsT<T, R> &, double, int); \
    template void bicg_1_t<T, R>(cudaStream_t, const EllT<T> &, const BicgVectorsT<T, R> &, int);            \
    template void bicg_2_t<T, R>(cudaStream_t, const EllT<T> &, const BicgVectorsT<T, R> &, int);            \
    template void bicg_3_t<T, R>(cudaStream_t, const EllT<T> &, const BicgVectorsT<T, R> &, int);
MCB_INSTANTIATE_BICG_T(double, 1)
MCB_INSTANTIATE_BICG_T(double, 3)
MCB_INSTANTIATE_BICG_T(float, 1)
MCB_INSTANTIATE_BICG_T(float, 3)

#define MCB_INSTANTIATE_BICG(R)                                                                  \
    template void bicg_init<R>(cudaStream_t, const Ell &, const BicgVectors<R> &, double, int); \
    template void bicg_1<R>(cudaStream_t, const Ell &, const BicgVectors<R> &, int);            \
    template void bicg_2<R>(cudaStream_t, const Ell &, const BicgVectors<R> &, int);            \
    template void bicg_3<R>(cudaStream_t, const Ell &, const BicgVectors<R> &, int);            \
    template void bir_init<R>(cudaStream_t, const Ell &, const BirVectors<R> &, double, int);   \
    template void bir_add<R>(cudaStream_t, int, const BirVectors<R> &);                          \
    template void bir_residual<R>(cudaStream_t, const Ell &, const BirVectors<R> &);
MCB_INSTANTIATE_BICG(1)
MCB_INSTANTIATE_BICG(3)

} // namespace mcb
