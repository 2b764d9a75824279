// Aggregation AMG for the pressure-correction system (see amg.h).
#include "amg.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "krylov.cuh"
#include "mc_reduce.cuh"

namespace mcb {

// ---------------------------------------------------------------- host setup

int amg_build_host(int N, const std::vector<int> &col0, const std::vector<int> &dn0, std::vector<AmgHostLevel> &out,
                   std::string &err)
{
    out.clear();
    AmgHostLevel L0;
    L0.n = N;
    L0.k = 6;
    L0.col = col0;
    out.push_back(std::move(L0));
    std::vector<int> dn = dn0;  // directional neighbours of the current level [6][n]
    for (int guard = 0; guard < AMG_MAX_LEVELS; guard++) {
        AmgHostLevel &cur = out.back();
        const int n = cur.n;
        if (n <= AMG_COARSEST_MAX) return 0;
        if ((int)out.size() == AMG_MAX_LEVELS) break;
        auto nb = [&](int d, int c) { return c < 0 ? -1 : dn[(size_t)d * n + c]; };
        // 2 x 2 x 2 aggregates anchored at the first unaggregated cell.  Per
        // axis the aggregate extends to the + side (x: slot 3, y: 5, z: 1)
        // when that neighbour is free, else to the - side (2, 4, 0), so the
        // blocks stay whole in any cell order (in x-fastest order the + side
        // is always free).
        std::vector<int> agg(n, -1), anchor;
        int nagg = 0;
        auto side = [&](int plus, int minus, int c) {
            const int a = nb(plus, c);
            if (a >= 0 && agg[a] < 0) return plus;
            const int b = nb(minus, c);
            return (b >= 0 && agg[b] < 0) ? minus : plus;
        };
        for (int c = 0; c < n; c++) {
            if (agg[c] >= 0) continue;
            const int A = nagg++;
            anchor.push_back(c);
            agg[c] = A;
            const int dx = side(3, 2, c), dy = side(5, 4, c), dz = side(1, 0, c);
            const int x1 = nb(dx, c), y1 = nb(dy, c), z1 = nb(dz, c);
            const int xy = x1 >= 0 ? nb(dy, x1) : nb(dx, y1);
            const int xz = x1 >= 0 ? nb(dz, x1) : nb(dx, z1);
            const int yz = y1 >= 0 ? nb(dz, y1) : nb(dy, z1);
            const int xyz = xy >= 0 ? nb(dz, xy) : (xz >= 0 ? nb(dy, xz) : nb(dx, yz));
            for (int cand : {x1, y1, xy, z1, xz, yz, xyz})
                if (cand >= 0 && agg[cand] < 0) agg[cand] = A;
        }
        if (nagg * 2 > n) {
            err = "AMG aggregation stalled (mesh without directional neighbours)";
            return -1;
        }
        cur.agg = agg;
        cur.mptr.assign(nagg + 1, 0);
        for (int c = 0; c < n; c++) cur.mptr[agg[c] + 1]++;
        for (int a = 0; a < nagg; a++) cur.mptr[a + 1] += cur.mptr[a];
        cur.mlist.assign(n, 0);
        {
            std::vector<int> fill(cur.mptr.begin(), cur.mptr.end() - 1);
            for (int c = 0; c < n; c++) cur.mlist[fill[agg[c]]++] = c;
        }
        // coarse directional neighbours: walk from the anchor until leaving the aggregate
        std::vector<int> dnc((size_t)6 * nagg, -1);
        for (int A = 0; A < nagg; A++)
            for (int d = 0; d < 6; d++) {
                int c = nb(d, anchor[A]);
                for (int steps = 0; c >= 0 && agg[c] == A && steps < 4; steps++) c = nb(d, c);
                dnc[(size_t)d * nagg + A] = (c >= 0 && agg[c] != A) ? agg[c] : -1;
            }
        // coarse pattern (sorted columns) and Galerkin lists
        AmgHostLevel nxt;
        nxt.n = nagg;
        std::vector<std::vector<int>> cols(nagg);
        int kmax = 0;
        for (int A = 0; A < nagg; A++) {
            std::vector<int> &cs = cols[A];
            for (int t = cur.mptr[A]; t < cur.mptr[A + 1]; t++) {
                const int i = cur.mlist[t];
                for (int s = 0; s < cur.k; s++) {
                    const int j = cur.col[(size_t)s * n + i];
                    if (j == i) continue;
                    const int J = agg[j];
                    if (J != A && std::find(cs.begin(), cs.end(), J) == cs.end()) cs.push_back(J);
                }
            }
            std::sort(cs.begin(), cs.end());
            kmax = std::max(kmax, (int)cs.size());
        }
        // Direction order: when every coarse neighbour of every aggregate is
        // its directional neighbour at a fixed offset per direction (six
        // distinct offsets), slot s is the direction with the s-th smallest
        // offset, so the kernels compute columns instead of reading them.
        int dir_off[6];
        bool dia = nagg > 1;
        for (int d = 0; d < 6 && dia; d++) {
            bool seen = false;
            for (int A = 0; A < nagg && dia; A++) {
                const int J = dnc[(size_t)d * nagg + A];
                if (J < 0) continue;
                if (!seen) dir_off[d] = J - A, seen = true;
                else if (J - A != dir_off[d]) dia = false;
            }
            dia = dia && seen && dir_off[d] != 0;
        }
        int slot_dir[6] = {0, 1, 2, 3, 4, 5};
        if (dia) {
            std::sort(slot_dir, slot_dir + 6, [&](int a, int b) { return dir_off[a] < dir_off[b]; });
            for (int s = 0; s + 1 < 6 && dia; s++) dia = dir_off[slot_dir[s]] != dir_off[slot_dir[s + 1]];
        }
        for (int A = 0; A < nagg && dia; A++) {
            int present = 0;
            for (int d = 0; d < 6; d++) present += dnc[(size_t)d * nagg + A] >= 0;
            dia = present == (int)cols[A].size();
            for (int J : cols[A]) {
                bool found = false;
                for (int d = 0; d < 6; d++) found = found || dnc[(size_t)d * nagg + A] == J;
                dia = dia && found;
            }
        }
        nxt.k = dia ? 6 : std::max(kmax, 1);
        const int kc = nxt.k;
        nxt.col.assign((size_t)kc * nagg, 0);
        if (dia) {
            nxt.dia = 1;
            for (int s = 0; s < 6; s++) nxt.doff[s] = dir_off[slot_dir[s]];
            for (int A = 0; A < nagg; A++)
                for (int s = 0; s < 6; s++) {
                    const int J = dnc[(size_t)slot_dir[s] * nagg + A];
                    nxt.col[(size_t)s * nagg + A] = J >= 0 ? J : A;
                }
        } else {
            for (int A = 0; A < nagg; A++)
                for (int s = 0; s < kc; s++) nxt.col[(size_t)s * nagg + A] = s < (int)cols[A].size() ? cols[A][s] : A;
        }
        auto slot_in = [&](int A, int J) {
            if (dia) {
                for (int s = 0; s < 6; s++)
                    if (nxt.col[(size_t)s * nagg + A] == J) return 1 + s;
                return 0;  // not reached: every coarse column is a directional neighbour
            }
            return 1 + (int)(std::lower_bound(cols[A].begin(), cols[A].end(), J) - cols[A].begin());
        };
        std::vector<int> count((size_t)nagg * (kc + 1) + 1, 0);
        struct Contrib { int entry, id; };
        std::vector<Contrib> contrib;
        contrib.reserve((size_t)n * 7);
        for (int A = 0; A < nagg; A++) {
            for (int t = cur.mptr[A]; t < cur.mptr[A + 1]; t++) {
                const int i = cur.mlist[t];
                contrib.push_back({A * (kc + 1), i});
                for (int s = 0; s < cur.k; s++) {
                    const int j = cur.col[(size_t)s * n + i];
                    if (j == i) continue;
                    const int J = agg[j];
                    int slot = 0;
                    if (J != A) slot = slot_in(A, J);
                    contrib.push_back({A * (kc + 1) + slot, n + s * n + i});
                }
            }
        }
        for (const Contrib &c : contrib) count[c.entry + 1]++;
        for (size_t e = 0; e + 1 < count.size(); e++) count[e + 1] += count[e];
        nxt.gptr = count;
        nxt.gidx.assign(contrib.size(), 0);
        {
            std::vector<int> fill(count.begin(), count.end() - 1);
            for (const Contrib &c : contrib) nxt.gidx[fill[c.entry]++] = c.id;
        }
        dn.swap(dnc);
        out.push_back(std::move(nxt));
    }
    err = "AMG hierarchy did not reach the coarsest size";
    return -1;
}

// ------------------------------------------------------------------ kernels

namespace {

// (A v)_i where v(j) yields the vector's value at row j (a stored vector, or
// one evaluated where it is needed).
template <bool H = false, typename T, typename V>
__device__ __forceinline__ T row_apply_v(const AmgLevelT<T> &L, int i, V &&v)
{
    const T s0 = L.diag[i] * v(i);
    if constexpr (H) {  // FP16 off-diagonal values by direction (FP32 level 0)
        int c[6];
        dia_cols(L.dc, L.n, i, c);
        T t = (T)0;
#pragma unroll
        for (int q = 0; q < 6; q++) t += (T)__half2float(L.off16[(size_t)q * L.n + i]) * v(c[q]);
        return s0 + t * (T)__ldg(L.scale16 + 1);
    }
    if (L.dc.code || L.dc.dia) {
        return with_row_cols(L.dc, L.col, L.n, i, [&](const int(&c)[6]) {
            T s = s0;
#pragma unroll
            for (int q = 0; q < 6; q++) s += ell_val(L.dc, L.off, L.n, i, q, c[q]) * v(c[q]);
            return s;
        });
    }
    T s = s0;
    for (int q = 0; q < L.k; q++) s += L.off[(size_t)q * L.n + i] * v(L.col[(size_t)q * L.n + i]);
    return s;
}

template <bool H = false, typename T>
__device__ __forceinline__ T row_apply(const AmgLevelT<T> &L, int i, const T *__restrict__ e)
{
    return row_apply_v<H>(L, i, [&](int j) { return e[j]; });
}

template <typename T>
__device__ __forceinline__ T inv_or_zero(T d)
{
    return d != (T)0 ? (T)1 / d : (T)0;
}

} // namespace

// FP32 copy of the level-0 values (in direction order when the level has
// direction codes).
__global__ void k_amg_round_level0(int n, const double *__restrict__ diag, const double *__restrict__ off,
                                   const uint32_t *__restrict__ code, float *__restrict__ diag32,
                                   float *__restrict__ off32)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    diag32[i] = (float)diag[i];
    float o[6];
    round_row_by_direction(off, code, n, i, o);
#pragma unroll
    for (int q = 0; q < 6; q++) off32[(size_t)q * n + i] = o[q];
}

// max |diag| of the FP32 level 0 into *dmax (when the pressure-row kernel
// has not formed it).
__global__ void __launch_bounds__(MCB_THREADS) k_amg_half_max(int n, const float *__restrict__ diag, double *dmax,
                                                              double *partials, unsigned int *counter)
{
    __shared__ double sh[1][MCB_THREADS];
    double m[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m[0] = fmax(m[0], (double)fabsf(diag[i]));
    if (publish_partials<1, true>(m, partials, counter, sh)) {
        double tot[1];
        reduce_partials<1, true>(tot, partials, counter, sh);
        if (threadIdx.x == 0) *dmax = tot[0];
    }
}

// FP16 copy of the FP32 level-0 off-diagonal values (by direction), times
// the power of two 2^(14 - e) with max |diag| = *dmax < 2^e, saturated at
// the largest finite FP16 value.  The rows are weakly diagonally dominant,
// so every scaled value is below 2^14 (FP16 reaches 65504) and values down
// to 2^-28 of the largest diagonal stay normal FP16 numbers.  The scale and
// its reciprocal go to scale16[0..1] for the V-cycle.
__global__ void __launch_bounds__(MCB_THREADS) k_amg_half_level0(int n, const float *__restrict__ off,
                                                                 const double *__restrict__ dmax,
                                                                 float *__restrict__ scale16,
                                                                 __half *__restrict__ off16)
{
    const double d = *dmax;
    int e = 0;
    if (d > 0.0 && isfinite(d)) frexp(d, &e);
    e = max(-100, min(100, e));
    const float sc = ldexpf(1.f, 14 - e);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scale16[0] = sc;
        scale16[1] = ldexpf(1.f, e - 14);
    }
    auto h = [&](float v) { return __float2half_rn(fminf(fmaxf(v * sc, -65504.f), 65504.f)); };
    const size_t total = (size_t)6 * n, quads = total / 4;  // both arrays 256-byte aligned
    const float4 *o4 = reinterpret_cast<const float4 *>(off);
    uint2 *h4 = reinterpret_cast<uint2 *>(off16);
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < quads; t += (size_t)gridDim.x * blockDim.x) {
        const float4 v = o4[t];
        const __half2 a = __halves2half2(h(v.x), h(v.y)), b = __halves2half2(h(v.z), h(v.w));
        uint2 u;
        memcpy(&u.x, &a, 4);
        memcpy(&u.y, &b, 4);
        h4[t] = u;
    }
    for (size_t t = 4 * quads + (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (size_t)gridDim.x * blockDim.x)
        off16[t] = h(off[t]);
}

// Coarse values as sums of fine values (the Galerkin lists index the fine
// level's slot-ordered values: level 1 of the FP32 hierarchy is summed from
// the FP64 level 0).
template <typename TF, typename T>
__global__ void k_amg_galerkin(AmgLevelT<TF> fine, AmgLevelT<T> coarse)
{
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= coarse.n) return;
    const int kc = coarse.k;
    for (int slot = 0; slot <= kc; slot++) {
        const int e = I * (kc + 1) + slot;
        double s = 0.0;
        for (int t = coarse.gptr[e]; t < coarse.gptr[e + 1]; t++) {
            const int id = coarse.gidx[t];
            s += (double)((id < fine.n) ? fine.diag[id] : fine.off[id - fine.n]);
        }
        if (slot == 0)
            coarse.diag[I] = (T)s;
        else
            coarse.off[(size_t)(slot - 1) * coarse.n + I] = (T)s;
    }
}

// Explicit inverse of A + sigma 1 1^T (sigma = mean diagonal / n) on the
// coarsest level, one block of DENSE_THREADS, FP64 in shared memory, by
// Gauss-Jordan elimination; symmetrised exactly and stored row-major in
// `dense` for the V-cycle's solve.
constexpr int DENSE_THREADS = 1024;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__global__ void __launch_bounds__(DENSE_THREADS) k_amg_dense_factor(AmgLevelT<T> L, double *dense)
{
    extern __shared__ double A[];
    // A: [n][ld] in shared memory, ld = n + 1 so that column accesses spread over the banks
    const int n = L.n, ld = n + 1, t = threadIdx.x, lane = t & 31, warp = t >> 5, nwarps = blockDim.x >> 5;
    __shared__ double sigma, wsum[DENSE_THREADS / 32];
    {
        double s = warp_sum(t < n ? (double)L.diag[t] : 0.0);
        if (lane == 0) wsum[warp] = s;
        __syncthreads();
        if (t == 0) {
            double tot = 0.0;
            for (int w = 0; w < nwarps; w++) tot += wsum[w];
            sigma = (tot / n) / n;
        }
        __syncthreads();
    }
    for (int idx = t; idx < n * ld; idx += blockDim.x) A[idx] = sigma;
    __syncthreads();
    if (t < n) {
        A[t * ld + t] += (double)L.diag[t];
        for (int q = 0; q < L.k; q++) {
            const int j = L.col[(size_t)q * n + t];
            if (j != t) A[t * ld + j] += (double)L.off[(size_t)q * n + t];
        }
    }
    __syncthreads();
    // In-place Gauss-Jordan inversion (no pivoting: the matrix is symmetric
    // positive definite).  Step k: the pivot row, with the identity's column k
    // in place of column k, divided by the pivot; every other row minus its
    // old column-k entry times that row.  Two barriers per step; thread t
    // owns column t % n of rows t / n, t / n + rows_per_pass, ...
    __shared__ double rk[AMG_COARSEST_MAX], ck[AMG_COARSEST_MAX];
    const int rpp = blockDim.x / n, jc = t % n, i0 = t / n;
    for (int k = 0; k < n; k++) {
        const double p = A[k * ld + k];
        const double pinv = p != 0.0 ? 1.0 / p : 0.0;
        if (t < n) {
            rk[t] = (t == k ? 1.0 : A[k * ld + t]) * pinv;
            ck[t] = A[t * ld + k];
        }
        __syncthreads();
        if (i0 < rpp) {
            const double r = rk[jc];
            for (int i = i0; i < n; i += rpp)
                A[i * ld + jc] = i == k ? r : (jc == k ? 0.0 : A[i * ld + jc]) - ck[i] * r;
        }
        __syncthreads();
    }
    // exactly symmetric result: both triangles take the same average
    for (int idx = t; idx < n * n; idx += blockDim.x) {
        const int i = idx / n, j = idx - i * n;
        dense[idx] = 0.5 * (A[i * ld + j] + A[j * ld + i]);
    }
}

// e = (A + sigma 1 1^T)^{-1} r on the coarsest level is one dense product
// with the symmetric inverse formed at setup (k_amg_coarse_cycle): each row
// is split over DENSE_SOLVE_PARTS threads (the reads dense[j][row] are
// coalesced across threads) and the parts are summed in a fixed order.
constexpr int DENSE_SOLVE_PARTS = 8;

template <typename T>
__global__ void k_amg_smooth_first(AmgLevelT<T> L, T omega, T *__restrict__ e, const PcgState *st)
{
    pdl_wait();
    if (st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    e[i] = omega * L.r[i] * inv_or_zero(L.diag[i]);
}

// The first two sweeps from e = 0 in one pass: e1 = e0 + omega D^-1 (r - A e0)
// with e0 = omega D^-1 r evaluated at each row where it is needed.
template <typename T, bool H = false>
__global__ void k_amg_smooth_first2(AmgLevelT<T> L, T omega, T omega2, T *__restrict__ eout, const PcgState *st)
{
    pdl_wait();
    if (st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    auto e0 = [&](int j) { return omega * L.r[j] * inv_or_zero(L.diag[j]); };
    eout[i] = e0(i) + omega2 * (L.r[i] - row_apply_v<H>(L, i, e0)) * inv_or_zero(L.diag[i]);
}

// Prolongation and the first post-smoothing sweep in one pass: the
// corrected iterate e + alpha ec[agg] is evaluated at each row where the
// sweep needs it and not stored.
// The FP32 forms of this kernel, the restriction and the last sweep are held
// to 32 registers (8 blocks of 256 per SM: full occupancy); 0 leaves the FP64
// forms to the compiler.
template <typename T, bool H = false>
__global__ void __launch_bounds__(MCB_THREADS, sizeof(T) == 4 ? 8 : 0)
    k_amg_prolong_jacobi(AmgLevelT<T> L, T omega, T alpha, const T *__restrict__ ec,
                                     const T *__restrict__ e, T *__restrict__ eout, const PcgState *st)
{
    pdl_wait();
    if (st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    auto ein = [&](int j) { return e[j] + alpha * ec[L.agg[j]]; };
    eout[i] = ein(i) + omega * (L.r[i] - row_apply_v<H>(L, i, ein)) * inv_or_zero(L.diag[i]);
}

template <typename T, bool H = false>
__global__ void k_amg_jacobi(AmgLevelT<T> L, T omega, const T *__restrict__ ein, T *__restrict__ eout,
                             const PcgState *st)
{
    pdl_wait();
    if (st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    eout[i] = ein[i] + omega * (L.r[i] - row_apply<H>(L, i, ein)) * inv_or_zero(L.diag[i]);
}

// Residual of the fine rows of coarse row I, summed: 8 lanes per coarse
// row (an aggregate has at most 8 rows; larger ones loop), each lane one
// fine row, then a fixed-order shuffle sum.  Every lane of the warp must call.
template <bool H, typename T>
__device__ __forceinline__ void restrict_row8(const AmgLevelT<T> &fine, const AmgLevelT<T> &coarse,
                                              const T *__restrict__ e, int I, int m)
{
    T s = (T)0;
    if (I < coarse.n)
        for (int t = fine.mptr[I] + m; t < fine.mptr[I + 1]; t += 8) {
            const int i = fine.mlist[t];
            s += fine.r[i] - row_apply<H>(fine, i, e);
        }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    if (I < coarse.n && m == 0) coarse.r[I] = s;
}

template <typename T, bool H = false>
__global__ void __launch_bounds__(MCB_THREADS, sizeof(T) == 4 ? 8 : 0)
    k_amg_restrict(AmgLevelT<T> fine, AmgLevelT<T> coarse, const T *__restrict__ e, const PcgState *st)
{
    pdl_wait();
    if (st->done) return;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    restrict_row8<H>(fine, coarse, e, g >> 3, g & 7);
}

template <typename T>
__global__ void k_amg_prolong(AmgLevelT<T> fine, T alpha, const T *__restrict__ ec, T *__restrict__ e,
                              const PcgState *st)
{
    pdl_wait();
    if (st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= fine.n) return;
    e[i] += alpha * ec[fine.agg[i]];
}

// Last post-smoothing sweep on level 0: z into zp[i].x and the PCG's r . z (FP64 sum).
template <typename T, bool H = false>
__global__ void __launch_bounds__(MCB_THREADS, sizeof(T) == 4 ? 8 : 0) k_amg_final(AmgLevelT<T> L, T omega, const T *__restrict__ ein,
                                                           typename Pair<T>::type *__restrict__ zp, PcgState *st,
                                                           double *partials, unsigned int *counter, int is_init)
{
    pdl_wait();
    __shared__ double sh[1][MCB_THREADS];
    if (st->done) return;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.n; i += gridDim.x * blockDim.x) {
        const T z = ein[i] + omega * (L.r[i] - row_apply<H>(L, i, ein)) * inv_or_zero(L.diag[i]);
        zp[i].x = z;
        acc[0] += (double)L.r[i] * (double)z;
    }
    if (publish_partials<1>(acc, partials, counter, sh)) {
        double tot[1];
        reduce_partials<1>(tot, partials, counter, sh);
        if (threadIdx.x == 0) {
            st->rz_old = is_init ? 1.0 : st->rz;
            st->rz = tot[0];
            if (!isfinite(tot[0])) {
                st->done = 1;
                st->status = KRYLOV_NONFINITE;
            }
        }
    }
}

// The coarse end of the V-cycle in one block: levels fused_from .. L-1
// (each at most AMG_FUSE_MAX_ROWS rows), with __syncthreads between the
// steps instead of kernel boundaries.  Same steps, order and sweeps as the
// per-level kernels: on every level but the last, nu damped-Jacobi sweeps
// (the first from e = 0) and the restriction of the residual; the dense
// solve; then, back up, prolongation (scaled by alpha) and nu sweeps.  The
// result on the first fused level ends in e[(2 nu - 1) & 1] (or e[0] when
// the coarsest level is the only one).
template <typename T>
struct AmgCoarse {
    AmgLevelT<T> lv[AMG_FUSED_LEVELS];
    int nl;
    T w[AMG_MAX_SWEEPS];  // damping of sweep k before the coarse correction (reversed after)
};

constexpr int AMG_FUSED_THREADS = AMG_COARSEST_MAX * DENSE_SOLVE_PARTS;  // 1024

template <typename T>
__global__ void __launch_bounds__(AMG_FUSED_THREADS)
    k_amg_coarse_cycle(const __grid_constant__ AmgCoarse<T> C, const double *__restrict__ dense, T alpha,
                       int sweeps, const PcgState *st)
{
    pdl_wait();
    if (st->done) return;
    __shared__ double rs[AMG_COARSEST_MAX];
    __shared__ double part[DENSE_SOLVE_PARTS][AMG_COARSEST_MAX];
    const int t = threadIdx.x, nt = blockDim.x;
    const int c_pre = (sweeps - 1) & 1;
    for (int l = 0; l + 1 < C.nl; l++) {
        const AmgLevelT<T> &L = C.lv[l];
        for (int i = t; i < L.n; i += nt) L.e[0][i] = C.w[0] * L.r[i] * inv_or_zero(L.diag[i]);
        __syncthreads();
        int c = 0;
        for (int sw = 1; sw < sweeps; sw++) {
            const T *ein = L.e[c];
            T *eout = L.e[c ^ 1];
            const T omega = C.w[sw];
            for (int i = t; i < L.n; i += nt)
                eout[i] = ein[i] + omega * (L.r[i] - row_apply(L, i, ein)) * inv_or_zero(L.diag[i]);
            c ^= 1;
            __syncthreads();
        }
        const AmgLevelT<T> &Cl = C.lv[l + 1];
        for (int g = t; g < ((Cl.n + 3) & ~3) * 8; g += nt) restrict_row8<false>(L, Cl, L.e[c], g >> 3, g & 7);
        __syncthreads();
    }
    {  // dense solve on the coarsest level
        const AmgLevelT<T> &L = C.lv[C.nl - 1];
        const int n = L.n, row = t % AMG_COARSEST_MAX, q = t / AMG_COARSEST_MAX;
        if (t < n) rs[t] = (double)L.r[t];
        __syncthreads();
        const int chunk = (n + DENSE_SOLVE_PARTS - 1) / DENSE_SOLVE_PARTS;
        double y = 0.0;
        if (row < n)
            for (int j = q * chunk; j < min(n, (q + 1) * chunk); j++) y += dense[(size_t)j * n + row] * rs[j];
        part[q][row] = y;
        __syncthreads();
        if (t < n) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < DENSE_SOLVE_PARTS; k++) s += part[k][t];
            L.e[0][t] = (T)s;
        }
        __syncthreads();
    }
    int c_up = 0;  // buffer of the coarser level's result
    for (int l = C.nl - 2; l >= 0; l--) {
        const AmgLevelT<T> &L = C.lv[l];
        const T *ec = C.lv[l + 1].e[c_up];
        int c = c_pre;
        for (int i = t; i < L.n; i += nt) L.e[c][i] += alpha * ec[L.agg[i]];
        __syncthreads();
        for (int sw = 1; sw <= sweeps; sw++) {
            const T *ein = L.e[c];
            T *eout = L.e[c ^ 1];
            const T omega = C.w[sweeps - sw];
            for (int i = t; i < L.n; i += nt)
                eout[i] = ein[i] + omega * (L.r[i] - row_apply(L, i, ein)) * inv_or_zero(L.diag[i]);
            c ^= 1;
            __syncthreads();
        }
        c_up = c;
    }
}

// ------------------------------------------------------------------ drivers

namespace {
inline int blocks(int n) { return std::max(1, (n + MCB_THREADS - 1) / MCB_THREADS); }
inline int blocks8(int n) { return std::max(1, (8 * n + MCB_THREADS - 1) / MCB_THREADS); }  // 8 threads per row
inline size_t dense_smem(int n) { return (size_t)n * (n + 1) * sizeof(double); }

template <typename T>
const AmgLevelT<T> *levels_of(const AmgHierarchy &H);
template <>
const AmgLevelT<double> *levels_of<double>(const AmgHierarchy &H) { return H.lv; }
template <>
const AmgLevelT<float> *levels_of<float>(const AmgHierarchy &H) { return H.lv32; }

template <typename T>
void set_dense_attributes()
{
    static bool done = false;
    if (done) return;
    cudaFuncSetAttribute(k_amg_dense_factor<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)dense_smem(AMG_COARSEST_MAX));
    done = true;
}
} // namespace

template <typename T>
void amg_setup_levels(cudaStream_t s, const AmgHierarchy &H, bool level0_ready, double *partials,
                      unsigned int *counter, double *dmax)
{
    const AmgLevelT<T> *lv = levels_of<T>(H);
    if (sizeof(T) == sizeof(float) && !level0_ready)
        k_amg_round_level0<<<blocks(H.g0.n), MCB_THREADS, 0, s>>>(H.g0.n, H.g0.diag, H.g0.off,
                                                                  lv[0].dc.dia ? H.g0.dc.code : nullptr,
                                                                  (float *)lv[0].diag, (float *)lv[0].off);
    if (sizeof(T) == sizeof(float) && lv[0].off16) {
        const int n = lv[0].n;
        if (!level0_ready)
            k_amg_half_max<<<krylov_grid(n), MCB_THREADS, 0, s>>>(n, (const float *)lv[0].diag, dmax, partials,
                                                                   counter);
        k_amg_half_level0<<<krylov_grid(n), MCB_THREADS, 0, s>>>(n, (const float *)lv[0].off, dmax, lv[0].scale16,
                                                                 lv[0].off16);
    }
    if (H.levels > 1) k_amg_galerkin<double, T><<<blocks(lv[1].n), MCB_THREADS, 0, s>>>(H.g0, lv[1]);
    for (int l = 2; l < H.levels; l++)
        k_amg_galerkin<T, T><<<blocks(lv[l].n), MCB_THREADS, 0, s>>>(lv[l - 1], lv[l]);
}

template <typename T>
void amg_coarsest_inverse(cudaStream_t s, const AmgHierarchy &H, double *out)
{
    set_dense_attributes<T>();
    const AmgLevelT<T> &C = levels_of<T>(H)[H.levels - 1];
    k_amg_dense_factor<T><<<1, DENSE_THREADS, dense_smem(C.n), s>>>(C, out);
}

void amg_set_damping(AmgHierarchy &H, double ratio)
{
    for (int k = 0; k < AMG_MAX_SWEEPS; k++) H.omega_sweep[k] = H.omega;
    if (!(ratio > 1.0)) return;
    // Chebyshev smoothing as damped-Jacobi sweeps: with sweep k damping by
    // 1 / lambda_k, lambda_k the roots of the degree-nu Chebyshev polynomial
    // on [b / ratio, b], nu sweeps apply that polynomial of D^-1 A, the one of
    // least maximum on the interval.  b = 2 bounds the spectrum of D^-1 A for
    // every level (Gershgorin: the rows are weakly diagonally dominant, and
    // the Galerkin products of piecewise-constant aggregation keep them so).
    const double b = 2.0, a = b / ratio, pi = 3.14159265358979323846;
    for (int k = 0; k < H.sweeps; k++)
        H.omega_sweep[k] = 1.0 / (0.5 * (b + a) + 0.5 * (b - a) * std::cos((2 * k + 1) * pi / (2 * H.sweeps)));
}

void amg_plan_fused(AmgHierarchy &H)
{
    int f = H.levels - 1;
    while (f > 1 && H.lv[f - 1].n <= AMG_FUSE_MAX_ROWS && H.levels - (f - 1) <= AMG_FUSED_LEVELS) f--;
    H.fused_from = f;
}

// FP32 V-cycles with nu >= 2 run the first two sweeps before the coarse
// correction, and the prolongation with the first sweep after it, as single
// kernels (in FP64 the extra gathers of the evaluated iterate cost more than
// the saved passes).
bool amg_paired_sweeps(const AmgHierarchy &H, bool fp32) { return fp32 && H.sweeps >= 2; }

// Per level above the fused ones: nu sweeps before and after the coarse
// correction and the restriction.
int amg_kernels_per_vcycle(const AmgHierarchy &H, bool fp32)
{
    return H.fused_from * (2 * H.sweeps + (amg_paired_sweeps(H, fp32) ? 0 : 2)) + 1;
}

template <typename T>
void amg_vcycle(cudaStream_t s, const AmgHierarchy &H, const T *r0, void *zp_out_v, PcgState *st, double *partials,
                unsigned int *counter, int is_init)
{
    using T2 = typename Pair<T>::type;
    T2 *zp_out = (T2 *)zp_out_v;
    const int L = H.levels, F = H.fused_from;
    const T alpha = (T)H.alpha;
    auto w = [&](int k) { return (T)H.omega_sweep[k]; };  // sweep k before the coarse correction
    int cur[AMG_MAX_LEVELS] = {0};
    AmgLevelT<T> lv[AMG_MAX_LEVELS];
    const AmgLevelT<T> *src = levels_of<T>(H);
    for (int l = 0; l < L; l++) lv[l] = src[l];
    lv[0].r = const_cast<T *>(r0);
    const bool pair = amg_paired_sweeps(H, sizeof(T) == sizeof(float));
    const dim3 nt(MCB_THREADS);
    // level 0 with FP16 off-diagonal values: the kernels' H forms
    const bool h0 = sizeof(T) == sizeof(float) && lv[0].off16;
    for (int l = 0; l < F; l++) {
        const AmgLevelT<T> &V = lv[l];
        const dim3 g(blocks(V.n));
        const bool hv = h0 && l == 0;
        int c = 0, sw = 1;
        if (pair) {
            pdl_launch(hv ? k_amg_smooth_first2<T, true> : k_amg_smooth_first2<T, false>, g, nt, 0, s, V, w(0), w(1),
                       V.e[1], st);
            c = 1;
            sw = 2;
        } else {
            pdl_launch(k_amg_smooth_first<T>, g, nt, 0, s, V, w(0), V.e[0], st);
        }
        for (; sw < H.sweeps; sw++) {
            pdl_launch(hv ? k_amg_jacobi<T, true> : k_amg_jacobi<T, false>, g, nt, 0, s, V, w(sw), V.e[c], V.e[c ^ 1],
                       st);
            c ^= 1;
        }
        cur[l] = c;
        pdl_launch(hv ? k_amg_restrict<T, true> : k_amg_restrict<T, false>, dim3(blocks8(lv[l + 1].n)), nt, 0, s, V,
                   lv[l + 1], V.e[c], st);
    }
    AmgCoarse<T> C;
    C.nl = L - F;
    for (int q = 0; q < C.nl; q++) C.lv[q] = lv[F + q];
    for (int k = 0; k < AMG_MAX_SWEEPS; k++) C.w[k] = w(k);
    pdl_launch(k_amg_coarse_cycle<T>, dim3(1), dim3(AMG_FUSED_THREADS), 0, s, C, H.dense, alpha, H.sweeps, st);
    cur[F] = (F < L - 1) ? (2 * H.sweeps - 1) & 1 : 0;
    for (int l = F - 1; l >= 0; l--) {
        const AmgLevelT<T> &V = lv[l];
        const dim3 g(blocks(V.n));
        const bool hv = h0 && l == 0;
        const T *ec = lv[l + 1].e[cur[l + 1]];
        int c = cur[l], sw = 1;
        if (pair) {
            pdl_launch(hv ? k_amg_prolong_jacobi<T, true> : k_amg_prolong_jacobi<T, false>, g, nt, 0, s, V,
                       w(H.sweeps - 1), alpha, ec, V.e[c], V.e[c ^ 1], st);
            c ^= 1;
            sw = 2;
        } else {
            pdl_launch(k_amg_prolong<T>, g, nt, 0, s, V, alpha, ec, V.e[c], st);
        }
        for (; sw <= H.sweeps; sw++) {
            if (l == 0 && sw == H.sweeps) {
                pdl_launch(hv ? k_amg_final<T, true> : k_amg_final<T, false>, dim3(krylov_grid(V.n)), nt, 0, s, V,
                           w(H.sweeps - sw), V.e[c], zp_out, st, partials, counter, is_init);
            } else {
                pdl_launch(hv ? k_amg_jacobi<T, true> : k_amg_jacobi<T, false>, g, nt, 0, s, V, w(H.sweeps - sw),
                           V.e[c], V.e[c ^ 1], st);
                c ^= 1;
            }
        }
        cur[l] = c;
    }
}

template void amg_setup_levels<double>(cudaStream_t, const AmgHierarchy &, bool, double *, unsigned int *, double *);
template void amg_setup_levels<float>(cudaStream_t, const AmgHierarchy &, bool, double *, unsigned int *, double *);
template void amg_coarsest_inverse<double>(cudaStream_t, const AmgHierarchy &, double *);
template void amg_coarsest_inverse<float>(cudaStream_t, const AmgHierarchy &, double *);
template void amg_vcycle<double>(cudaStream_t, const AmgHierarchy &, const double *, void *, PcgState *, double *,
                                 unsigned int *, int);
template void amg_vcycle<float>(cudaStream_t, const AmgHierarchy &, const float *, void *, PcgState *, double *,
                                unsigned int *, int);

} // namespace mcb
