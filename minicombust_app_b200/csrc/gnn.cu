// Learned initial guess: forward, backward and Adam kernels (see gnn.cuh).
//
// Inference on a graph in offset form runs each layer as one tcgen05 kernel
// (gnn_umma.cu).  The other dense products -- training, the general-graph
// layer, encoder and decoder -- are block-level GEMMs over a tile of 128
// cells with mma.sync.m16n8k16 (BF16 operands from shared memory, FP32
// accumulators); with K = 32 or 64 and N = 32 they are bound by the
// activation traffic, not by the products.  Weight gradients are per-block
// partial GEMMs (cells as the reduction dimension) summed afterwards in block
// order, so training is deterministic.
#include "gnn.cuh"

#include <algorithm>
#include <cmath>

#include "mc_reduce.cuh"

namespace mcb {

namespace {

using bf16 = __nv_bfloat16;
using bf162 = __nv_bfloat162;

constexpr int LDH = GNN_H + 8;        // row stride (elements) of [cell][32] tiles
constexpr int LDT = GNN_TILE + 8;     // row stride of transposed [channel][cell] tiles
constexpr unsigned FULL = 0xffffffffu;

int gnn_blocks(int n) { return (n + GNN_TILE - 1) / GNN_TILE; }

// Multiprocessors of the current device (persistent launches: one block each).
int sm_count()
{
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    return n;
}
int reduce_grid(int n) { return std::max(1, std::min((n + MCB_THREADS - 1) / MCB_THREADS, 148 * 4)); }

__device__ __forceinline__ uint32_t ld32(const bf16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// acc[MT][NT] += A[16 MT rows][16 KS] . W[8 NT rows][16 KS]^T for one warp.
// A and W are row-major BF16 tiles in shared memory (strides lda, ldw, even).
// Accumulator layout (m16n8): acc[.][.][0..1] = row g, cols 2t, 2t+1;
// acc[.][.][2..3] = row g + 8; g = lane / 4, t = lane % 4.
template <int MT, int NT, int KS>
__device__ __forceinline__ void warp_gemm(float (&acc)[MT][NT][4], const bf16 *A, int lda, const bf16 *W, int ldw,
                                          int lane)
{
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int ks = 0; ks < KS; ks++) {
        uint32_t a[MT][4], b[NT][2];
#pragma unroll
        for (int mt = 0; mt < MT; mt++) {
            const bf16 *p = A + (mt * 16 + g) * lda + ks * 16 + 2 * t;
            a[mt][0] = ld32(p);
            a[mt][1] = ld32(p + 8 * lda);
            a[mt][2] = ld32(p + 8);
            a[mt][3] = ld32(p + 8 * lda + 8);
        }
#pragma unroll
        for (int nt = 0; nt < NT; nt++) {
            const bf16 *q = W + (nt * 8 + g) * ldw + ks * 16 + 2 * t;
            b[nt][0] = ld32(q);
            b[nt][1] = ld32(q + 8);
        }
#pragma unroll
        for (int mt = 0; mt < MT; mt++)
#pragma unroll
            for (int nt = 0; nt < NT; nt++) mma_bf16(acc[mt][nt], a[mt], b[nt]);
    }
}

// Four 8x8 BF16 matrices from shared memory in the mma.m16n8k16 fragment
// layout (lanes 8m .. 8m + 7 give the row addresses of matrix m).
__device__ __forceinline__ void ldm_x4(uint32_t (&r)[4], const bf16 *p)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

// acc (16 rows x 32 columns) += A[16][16 KS] . W[32][16 KS]^T for one warp,
// A and W row-major BF16 in shared memory (row strides multiples of 8).
template <int KS>
__device__ __forceinline__ void warp_gemm16x32(float (&acc)[1][4][4], const bf16 *A, int lda, const bf16 *W, int ldw,
                                               int lane)
{
#pragma unroll
    for (int ks = 0; ks < KS; ks++) {
        uint32_t a[4];
        ldm_x4(a, A + (lane & 15) * lda + ks * 16 + (lane >> 4) * 8);
#pragma unroll
        for (int np = 0; np < 2; np++) {
            uint32_t b[4];
            ldm_x4(b, W + (np * 16 + (lane & 7) + ((lane >> 4) << 3)) * ldw + ks * 16 + ((lane >> 3) & 1) * 8);
            const uint32_t b0[2] = {b[0], b[1]}, b1[2] = {b[2], b[3]};
            mma_bf16(acc[0][2 * np], a, b0);
            mma_bf16(acc[0][2 * np + 1], a, b1);
        }
    }
}

// B fragments of a [32][16 KS] row-major tile (W-form) for warp_gemm16x32r:
// fr[ks][np] holds n-tiles 2 np, 2 np + 1 of k-step ks.
template <int KS>
__device__ __forceinline__ void load_bfrags(uint32_t (&fr)[KS][2][4], const bf16 *W, int ldw, int lane)
{
#pragma unroll
    for (int ks = 0; ks < KS; ks++)
#pragma unroll
        for (int np = 0; np < 2; np++)
            ldm_x4(fr[ks][np], W + (np * 16 + (lane & 7) + ((lane >> 4) << 3)) * ldw + ks * 16 + ((lane >> 3) & 1) * 8);
}

// acc (16 x 32) += A[16][16 KS] . W^T with W's fragments in registers.
template <int KS>
__device__ __forceinline__ void warp_gemm16x32r(float (&acc)[1][4][4], const bf16 *A, int lda,
                                                const uint32_t (&fr)[KS][2][4], int lane)
{
#pragma unroll
    for (int ks = 0; ks < KS; ks++) {
        uint32_t a[4];
        ldm_x4(a, A + (lane & 15) * lda + ks * 16 + (lane >> 4) * 8);
#pragma unroll
        for (int np = 0; np < 2; np++) {
            const uint32_t b0[2] = {fr[ks][np][0], fr[ks][np][1]}, b1[2] = {fr[ks][np][2], fr[ks][np][3]};
            mma_bf16(acc[0][2 * np], a, b0);
            mma_bf16(acc[0][2 * np + 1], a, b1);
        }
    }
}

template <int MT, int NT>
__device__ __forceinline__ void zero(float (&acc)[MT][NT][4])
{
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int nt = 0; nt < NT; nt++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[mt][nt][e] = 0.f;
}

template <typename T>
__device__ __forceinline__ float ldf(const T *p, int i)
{
    return (float)p[i];
}

// Per-lane staging of a warp's 32 cells: lane t holds the inputs of cell
// base + t; shuffles broadcast them inside the per-cell loops.
struct CellFeat {
    float b, d, p, v;
};

template <typename T>
__device__ __forceinline__ CellFeat load_features(const GnnGraph &g, const GnnInput<T> &in, const GnnScales &sc, int i)
{
    CellFeat f{0.f, 0.f, 0.f, 0.f};
    if (i < g.n) {
        f.b = (float)(((double)in.b[i] - sc.shift) * sc.rb);
        f.d = (float)((double)in.diag[i] * sc.rd);
        f.p = in.prev ? (float)((double)in.prev[i] * sc.rx) : 0.f;
        f.v = g.vhat[i];
    }
    return f;
}

// Per-warp column sums of per-lane values `v` (lane = channel) are exact
// already; this helper sums one value per (warp, channel) across the block
// in warp order.  red: [4][32] shared.
__device__ __forceinline__ float block_channel_sum(float v, float (*red)[GNN_H], int warp, int lane)
{
    __syncthreads();
    red[warp][lane] = v;
    __syncthreads();
    float s = 0.f;
    if (warp == 0) s = ((red[0][lane] + red[1][lane]) + red[2][lane]) + red[3][lane];
    return s;
}

// Sum over the 8 row-groups (g) of an accumulator column pair held by lanes
// with the same t; valid in lanes with g == 0.
__device__ __forceinline__ float sum_over_g(float v)
{
    v += __shfl_xor_sync(FULL, v, 4);
    v += __shfl_xor_sync(FULL, v, 8);
    v += __shfl_xor_sync(FULL, v, 16);
    return v;
}

// ------------------------------------------------------------------ kernels

template <typename T>
__global__ void __launch_bounds__(MCB_THREADS) k_gnn_scales(int n, GnnInput<T> in, double *partials,
                                                            unsigned int *counter, GnnScales *out)
{
    __shared__ double sh[2][MCB_THREADS];
    const double shift = in.shift ? *in.shift : 0.0;
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double b = (double)in.b[i] - shift;
        acc[0] += b * b;
        acc[1] += (double)in.diag[i];
    }
    if (publish_partials<2>(acc, partials, counter, sh)) {
        double tot[2];
        reduce_partials<2>(tot, partials, counter, sh);
        if (threadIdx.x == 0) {
            GnnScales s;
            s.shift = shift;
            s.sb = sqrt(tot[0] / n);
            s.sd = tot[1] / n;
            s.sx = (s.sd > 0 && isfinite(s.sb)) ? s.sb / s.sd : 0.0;
            if (!(s.sb > 0) || !(s.sx > 0) || !isfinite(s.sx)) s.sb = s.sd = s.sx = 0.0;
            s.rb = s.sb > 0 ? 1.0 / s.sb : 0.0;
            s.rd = s.sd > 0 ? 1.0 / s.sd : 0.0;
            s.rx = s.sx > 0 ? 1.0 / s.sx : 0.0;
            *out = s;
        }
    }
}

// Eight consecutive BF16 channels as one 16-byte word.
union Chunk8 {
    uint4 u;
    bf162 h[4];
};

// h0 = relu(We x + ce).  Thread = cell: one feature load, 32 channels from
// the weights in shared memory, four 16-byte stores.
template <typename T>
__global__ void __launch_bounds__(GNN_TILE) k_gnn_encode(GnnGraph g, GnnInput<T> in, const float *__restrict__ p,
                                                         const GnnScales *__restrict__ scp, bf16 *__restrict__ hout)
{
    __shared__ float sw[GNN_H * (GNN_IN + 1)];
    for (int e = threadIdx.x; e < GNN_H * (GNN_IN + 1); e += GNN_TILE) sw[e] = p[GP_WE + e];  // We then ce
    __syncthreads();
    const int i = blockIdx.x * GNN_TILE + threadIdx.x;
    if (i >= g.n) return;
    const CellFeat x = load_features(g, in, *scp, i);
#pragma unroll
    for (int c4 = 0; c4 < 4; c4++) {
        Chunk8 o;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            float z[2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int c = c4 * 8 + 2 * q + e;
                const float *w = sw + c * GNN_IN;
                z[e] = fmaxf(w[0] * x.b + w[1] * x.d + w[2] * x.p + w[3] * x.v + sw[GNN_H * GNN_IN + c], 0.f);
            }
            o.h[q] = __floats2bfloat162_rn(z[0], z[1]);
        }
        *reinterpret_cast<uint4 *>(hout + (size_t)i * GNN_H + c4 * 8) = o.u;
    }
}

// Gather of one cell's message for channel `lane` (h is [n][H] BF16).
struct SlotCache {
    int col[6];
    uint32_t edge[6];
};

__device__ __forceinline__ SlotCache load_slots(const GnnGraph &g, int i)
{
    SlotCache s;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        s.col[k] = i < g.n ? g.col[(size_t)k * g.n + i] : -1;
        s.edge[k] = i < g.n ? *reinterpret_cast<const uint32_t *>(g.edge + (size_t)k * g.n + i) : 0u;
    }
    return s;
}

__device__ __forceinline__ float2 edge_of(uint32_t bits)
{
    bf162 e;
    *reinterpret_cast<uint32_t *>(&e) = bits;
    return __bfloat1622float2(e);
}

// Asynchronous 16-byte global -> shared copy; src_bytes = 0 writes zeros.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Shared memory of k_gnn_layer (bytes): own rows [128][LDH] (a GEMM operand),
// the six neighbour rows [6][128][32] (zeros where a slot has no neighbour;
// later reused for relu(W1 u + c1) and h'), messages [128][LDH].
constexpr size_t LAYER_SMEM_H = sizeof(bf16) * GNN_TILE * LDH;
constexpr size_t LAYER_SMEM_N = sizeof(bf16) * 6 * GNN_TILE * GNN_H;
constexpr size_t LAYER_SMEM = 2 * LAYER_SMEM_H + LAYER_SMEM_N;

// One message-passing layer on a tile of 128 cells, 256 threads; TRAIN also
// stores relu(W1 u + c1).  Thread (row r, chunk c) handles rows r, r + 64
// and channels 8c .. 8c + 7; all 14 row copies of a thread are in flight
// together.  Warp w owns rows 16w .. 16w + 15 in the products.  The weight
// fragments are read through L1 (the same 6 KB for every block).
constexpr int LAYER_THREADS = 2 * GNN_TILE;

template <bool TRAIN>
__global__ void __launch_bounds__(LAYER_THREADS) k_gnn_layer(GnnGraph g, const float *__restrict__ pl,
                                                             const bf16 *__restrict__ pkl,
                                                             const bf16 *__restrict__ hin, bf16 *__restrict__ hout,
                                                             bf16 *__restrict__ asave)
{
    extern __shared__ __align__(16) unsigned char smem[];
    bf16 *sH = reinterpret_cast<bf16 *>(smem);
    bf16 *sN = reinterpret_cast<bf16 *>(smem + LAYER_SMEM_H);
    bf16 *sM = reinterpret_cast<bf16 *>(smem + LAYER_SMEM_H + LAYER_SMEM_N);
    bf16 *sA = sN;  // after the messages are formed
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int c4 = tid & 3, r0 = tid >> 2;
    const int n = g.n, base = blockIdx.x * GNN_TILE;
    // 1. stage own and neighbour rows
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int r = r0 + 64 * q, i = base + r;
        const bool in = i < n;
        cp_async16(sH + r * LDH + c4 * 8, hin + (size_t)(in ? i : 0) * GNN_H + c4 * 8, in ? 16 : 0);
        const unsigned mk = (in && g.affine) ? g.mask[i] : 0u;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            int j;
            bool ok;
            if (g.affine) {
                ok = (mk >> k) & 1u;
                j = ok ? i + g.doff[k] : 0;
            } else {
                j = in ? g.col[(size_t)k * n + i] : 0;
                ok = in && j != i;
                j = ok ? j : 0;
            }
            cp_async16(sN + (k * GNN_TILE + r) * GNN_H + c4 * 8, hin + (size_t)j * GNN_H + c4 * 8, ok ? 16 : 0);
        }
    }
    // gates while the copies are in flight
    float wg0[8], wg1[8], cg[8];
#pragma unroll
    for (int c = 0; c < 8; c++) {
        wg0[c] = pl[GPL_WG + 2 * (c4 * 8 + c)];
        wg1[c] = pl[GPL_WG + 2 * (c4 * 8 + c) + 1];
        cg[c] = pl[GPL_CG + c4 * 8 + c];
    }
    cp_async_wait_all();
    __syncthreads();
    // 2. messages (rows with no neighbour in a slot were staged as zeros)
    if (g.affine) {
        float gate[6][8];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const float2 e = edge_of(g.ebits[k]);
#pragma unroll
            for (int c = 0; c < 8; c++) gate[k][c] = wg0[c] * e.x + wg1[c] * e.y + cg[c];
        }
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int r = r0 + 64 * q;
            float m[8];
#pragma unroll
            for (int c = 0; c < 8; c++) m[c] = 0.f;
#pragma unroll
            for (int k = 0; k < 6; k++) {
                Chunk8 v;
                v.u = *reinterpret_cast<const uint4 *>(sN + (k * GNN_TILE + r) * GNN_H + c4 * 8);
#pragma unroll
                for (int q2 = 0; q2 < 4; q2++) {
                    const float2 h = __bfloat1622float2(v.h[q2]);
                    m[2 * q2] += gate[k][2 * q2] * h.x;
                    m[2 * q2 + 1] += gate[k][2 * q2 + 1] * h.y;
                }
            }
            Chunk8 mo;
#pragma unroll
            for (int q2 = 0; q2 < 4; q2++) mo.h[q2] = __floats2bfloat162_rn(m[2 * q2], m[2 * q2 + 1]);
            *reinterpret_cast<uint4 *>(sM + r * LDH + c4 * 8) = mo.u;
        }
    } else {
        // m = wg0 (.) sum e.x h_j + wg1 (.) sum e.y h_j + cg (.) sum h_j
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int r = r0 + 64 * q, i = base + r;
            float s0[8], s1[8], s2[8];
#pragma unroll
            for (int c = 0; c < 8; c++) s0[c] = s1[c] = s2[c] = 0.f;
#pragma unroll
            for (int k = 0; k < 6; k++) {
                Chunk8 v;
                v.u = *reinterpret_cast<const uint4 *>(sN + (k * GNN_TILE + r) * GNN_H + c4 * 8);
                const float2 e =
                    edge_of(i < n ? *reinterpret_cast<const uint32_t *>(g.edge + (size_t)k * n + i) : 0u);
#pragma unroll
                for (int q2 = 0; q2 < 4; q2++) {
                    const float2 h = __bfloat1622float2(v.h[q2]);
                    s0[2 * q2] += e.x * h.x;
                    s0[2 * q2 + 1] += e.x * h.y;
                    s1[2 * q2] += e.y * h.x;
                    s1[2 * q2 + 1] += e.y * h.y;
                    s2[2 * q2] += h.x;
                    s2[2 * q2 + 1] += h.y;
                }
            }
            Chunk8 mo;
#pragma unroll
            for (int q2 = 0; q2 < 4; q2++) {
                const int c = 2 * q2;
                mo.h[q2] = __floats2bfloat162_rn(wg0[c] * s0[c] + wg1[c] * s1[c] + cg[c] * s2[c],
                                                 wg0[c + 1] * s0[c + 1] + wg1[c + 1] * s1[c + 1] + cg[c + 1] * s2[c + 1]);
            }
            *reinterpret_cast<uint4 *>(sM + r * LDH + c4 * 8) = mo.u;
        }
    }
    __syncthreads();
    // 3. z = W1 [h; m] + c1 on the warp's 16 rows
    const int gq = lane >> 2, tq = lane & 3;
    float b1[4][2], b2[4][2];
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
            b1[nt][e] = pl[GPL_C1 + nt * 8 + 2 * tq + e];
            b2[nt][e] = pl[GPL_C2 + nt * 8 + 2 * tq + e];
        }
    float acc[1][4][4];
    zero(acc);
    warp_gemm<1, 4, 2>(acc, sH + warp * 16 * LDH, LDH, pkl + GKL_W1, 2 * GNN_H, lane);
    warp_gemm<1, 4, 2>(acc, sM + warp * 16 * LDH, LDH, pkl + GKL_W1 + GNN_H, 2 * GNN_H, lane);
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
        for (int hf = 0; hf < 2; hf++) {
            const int row = warp * 16 + gq + 8 * hf, col = nt * 8 + 2 * tq;
            const bf162 v = __floats2bfloat162_rn(fmaxf(acc[0][nt][2 * hf] + b1[nt][0], 0.f),
                                                  fmaxf(acc[0][nt][2 * hf + 1] + b1[nt][1], 0.f));
            *reinterpret_cast<bf162 *>(sA + row * LDH + col) = v;
            if (TRAIN && base + row < n) *reinterpret_cast<bf162 *>(asave + (size_t)(base + row) * GNN_H + col) = v;
        }
    __syncwarp();
    // 4. h' = h + W2 a + c2
    zero(acc);
    warp_gemm<1, 4, 2>(acc, sA + warp * 16 * LDH, LDH, pkl + GKL_W2, GNN_H, lane);
    __syncwarp();  // the warp's reads of sA are done; its rows now take h'
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
        for (int hf = 0; hf < 2; hf++) {
            const int row = warp * 16 + gq + 8 * hf, col = nt * 8 + 2 * tq;
            const float2 hv = __bfloat1622float2(*reinterpret_cast<const bf162 *>(sH + row * LDH + col));
            *reinterpret_cast<bf162 *>(sA + row * LDH + col) = __floats2bfloat162_rn(
                hv.x + (acc[0][nt][2 * hf] + b2[nt][0]), hv.y + (acc[0][nt][2 * hf + 1] + b2[nt][1]));
        }
    __syncwarp();
    // 5. coalesced store of the warp's 16 rows: 4 lanes per 64-byte row
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int row = warp * 16 + (lane >> 2) + 8 * q, i = base + row;
        if (i < n)
            *reinterpret_cast<uint4 *>(hout + (size_t)i * GNN_H + (lane & 3) * 8) =
                *reinterpret_cast<const uint4 *>(sA + row * LDH + (lane & 3) * 8);
    }
}

// Offset-form weights of every layer: slot 0 = W1 columns of h_i, slot 1 + k
// = W1 columns of m with each input channel c scaled by the gate of
// direction k, g_k[c] = Wg[c] . e_k + cg[c].  Row-major [out][in] per slot.
__global__ void k_gnn_fold(const float *__restrict__ p, GnnGraph g, bf16 *__restrict__ fold)
{
    constexpr int PER_LAYER = 7 * GNN_H * GNN_H;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < GNN_L * PER_LAYER; e += gridDim.x * blockDim.x) {
        const int l = e / PER_LAYER, r = e % PER_LAYER;
        const int k = r / (GNN_H * GNN_H), o = (r / GNN_H) % GNN_H, c = r % GNN_H;
        const float *pl = p + GP_LAYER0 + l * GPL_SIZE;
        float v;
        if (k == 0) {
            v = pl[GPL_W1 + o * 2 * GNN_H + c];
        } else {
            const float2 ek = edge_of(g.ebits[k - 1]);
            const float gate = pl[GPL_WG + 2 * c] * ek.x + pl[GPL_WG + 2 * c + 1] * ek.y + pl[GPL_CG + c];
            v = pl[GPL_W1 + o * 2 * GNN_H + GNN_H + c] * gate;
        }
        fold[e] = __float2bfloat16(v);
    }
}

// Shared memory of k_gnn_layer_fold: the layer's weights -- the seven folded
// W1 slots [7][32][LDH] and W2 [32][LDH] -- then two buffers of seven row
// tiles [7][128][LDH] (the cells' own rows and their neighbours through the
// six directions, zeros on the boundary).
constexpr size_t FOLD_SMEM_W = sizeof(bf16) * 8 * GNN_H * LDH;
constexpr size_t FOLD_SMEM_T = sizeof(bf16) * 7 * GNN_TILE * LDH;
constexpr size_t FOLD_SMEM = FOLD_SMEM_W + 2 * FOLD_SMEM_T;

// Mask bytes of this thread's two rows of a tile (0 beyond the last cell).
__device__ __forceinline__ void load_fold_masks(const GnnGraph &g, int base, unsigned (&mk)[2])
{
    const int r0 = threadIdx.x >> 2;
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int i = base + r0 + 64 * q;
        mk[q] = i < g.n ? g.mask[i] : 0u;
    }
}

// Asynchronous copies of one tile's seven row tiles (thread = chunk of 8
// channels x rows r, r + 64), with the rows' masks already in registers.
__device__ __forceinline__ void stage_fold_tile(const GnnGraph &g, const bf16 *__restrict__ hin, bf16 *sT, int base,
                                                const unsigned (&mks)[2])
{
    const int c4 = threadIdx.x & 3, r0 = threadIdx.x >> 2, n = g.n;
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int r = r0 + 64 * q, i = base + r;
        const bool in = i < n;
        cp_async16(sT + r * LDH + c4 * 8, hin + (size_t)(in ? i : 0) * GNN_H + c4 * 8, in ? 16 : 0);
        const unsigned mk = mks[q];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const bool ok = (mk >> k) & 1u;
            const int j = ok ? i + g.doff[k] : 0;
            cp_async16(sT + ((1 + k) * GNN_TILE + r) * LDH + c4 * 8, hin + (size_t)j * GNN_H + c4 * 8, ok ? 16 : 0);
        }
    }
}

// One message-passing layer on a graph in offset form (inference),
// persistent: one block per SM keeps the weights, prefetches the next tile
// while computing the current one.  Per tile: z = sum_k T_k Wf_k^T over the
// seven staged tiles, a = relu(z + c1), h' = h + W2 a + c2; warp w owns rows
// 16w .. 16w + 15.
__global__ void __launch_bounds__(LAYER_THREADS, 1) k_gnn_layer_fold(GnnGraph g, const float *__restrict__ pl,
                                                                     const bf16 *__restrict__ wf,
                                                                     const bf16 *__restrict__ pkl,
                                                                     const bf16 *__restrict__ hin,
                                                                     bf16 *__restrict__ hout, int ntiles)
{
    extern __shared__ __align__(16) unsigned char smem[];
    bf16 *sW = reinterpret_cast<bf16 *>(smem);  // [8][32][LDH]: 7 folded W1 slots, W2
    auto tile_buf = [&](int b) { return reinterpret_cast<bf16 *>(smem + FOLD_SMEM_W + (size_t)b * FOLD_SMEM_T); };
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = g.n;
#pragma unroll
    for (int q = 0; q < 4; q++) {  // 8 x 32 weight rows of 64 bytes, 4 chunks per thread
        const int e = tid + LAYER_THREADS * q, row = e >> 2, part = e & 3;
        const bf16 *src = row < 7 * GNN_H ? wf + (size_t)row * GNN_H : pkl + GKL_W2 + (size_t)(row - 7 * GNN_H) * GNN_H;
        cp_async16(sW + row * LDH + part * 8, src + part * 8, 16);
    }
    int tile = blockIdx.x;
    unsigned mk[2];
    load_fold_masks(g, tile * GNN_TILE, mk);
    if (tile < ntiles) stage_fold_tile(g, hin, tile_buf(0), tile * GNN_TILE, mk);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    load_fold_masks(g, (tile + gridDim.x) * GNN_TILE, mk);  // one tile ahead of the copies
    // the layer's weight fragments stay in registers for the whole launch
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    uint32_t w1f[7][2][2][4], w2f[2][2][4];
#pragma unroll
    for (int k = 0; k < 7; k++) load_bfrags<2>(w1f[k], sW + k * GNN_H * LDH, LDH, lane);
    load_bfrags<2>(w2f, sW + 7 * GNN_H * LDH, LDH, lane);
    const int gq = lane >> 2, tq = lane & 3;
    float b1[4][2], b2[4][2];
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
            b1[nt][e] = pl[GPL_C1 + nt * 8 + 2 * tq + e];
            b2[nt][e] = pl[GPL_C2 + nt * 8 + 2 * tq + e];
        }
    for (int buf = 0; tile < ntiles; tile += gridDim.x, buf ^= 1) {
        const int next = tile + gridDim.x;
        if (next < ntiles) stage_fold_tile(g, hin, tile_buf(buf ^ 1), next * GNN_TILE, mk);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        load_fold_masks(g, (next + gridDim.x) * GNN_TILE, mk);  // lands while this tile computes
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this tile (and the weights) landed
        __syncthreads();
        bf16 *sT = tile_buf(buf);
        const int base = tile * GNN_TILE;
        float acc[1][4][4], acc2[1][4][4];  // even and odd slots: two independent accumulation chains
        zero(acc);
        zero(acc2);
#pragma unroll
        for (int k = 0; k < 7; k += 2) warp_gemm16x32r<2>(acc, sT + (k * GNN_TILE + warp * 16) * LDH, LDH, w1f[k], lane);
#pragma unroll
        for (int k = 1; k < 7; k += 2) warp_gemm16x32r<2>(acc2, sT + (k * GNN_TILE + warp * 16) * LDH, LDH, w1f[k], lane);
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[0][nt][e] += acc2[0][nt][e];
        __syncwarp();  // the warp's reads of its rows are done; tile 1 rows now take a, then h'
        bf16 *sA = sT + GNN_TILE * LDH;
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int hf = 0; hf < 2; hf++) {
                const int row = warp * 16 + gq + 8 * hf, col = nt * 8 + 2 * tq;
                *reinterpret_cast<bf162 *>(sA + row * LDH + col) =
                    __floats2bfloat162_rn(fmaxf(acc[0][nt][2 * hf] + b1[nt][0], 0.f),
                                          fmaxf(acc[0][nt][2 * hf + 1] + b1[nt][1], 0.f));
            }
        __syncwarp();
        zero(acc);
        warp_gemm16x32r<2>(acc, sA + warp * 16 * LDH, LDH, w2f, lane);
        __syncwarp();
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int hf = 0; hf < 2; hf++) {
                const int row = warp * 16 + gq + 8 * hf, col = nt * 8 + 2 * tq;
                const float2 hv = __bfloat1622float2(*reinterpret_cast<const bf162 *>(sT + row * LDH + col));
                *reinterpret_cast<bf162 *>(sA + row * LDH + col) = __floats2bfloat162_rn(
                    hv.x + (acc[0][nt][2 * hf] + b2[nt][0]), hv.y + (acc[0][nt][2 * hf + 1] + b2[nt][1]));
            }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int row = warp * 16 + (lane >> 2) + 8 * q, i = base + row;
            if (i < n)
                *reinterpret_cast<uint4 *>(hout + (size_t)i * GNN_H + (lane & 3) * 8) =
                    *reinterpret_cast<const uint4 *>(sA + row * LDH + (lane & 3) * 8);
        }
        __syncthreads();  // every warp is done with this buffer before it is refilled
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Load a [128][32] BF16 tile of rows base.. into shared memory (row stride LDH).
__device__ __forceinline__ void load_tile(bf16 *s, const bf16 *__restrict__ h, int base, int n)
{
    for (int e = threadIdx.x; e < GNN_TILE * 4; e += GNN_TILE) {
        const int row = e >> 2, part = e & 3, i = base + row;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (i < n) v = *reinterpret_cast<const uint4 *>(h + (size_t)i * GNN_H + part * 8);
        *reinterpret_cast<uint4 *>(s + row * LDH + part * 8) = v;
    }
}

// y = wo . relu(Wd h + cd) + co; x0 = s_x y.
template <bool TRAIN>
__global__ void __launch_bounds__(GNN_TILE) k_gnn_decode(GnnGraph g, const float *__restrict__ pd,
                                                         const bf16 *__restrict__ pkd, const bf16 *__restrict__ hin,
                                                         const GnnScales *__restrict__ scp, float *__restrict__ y,
                                                         double *__restrict__ x0, bf16 *__restrict__ qsave,
                                                         const int *__restrict__ status)
{
    __shared__ __align__(16) bf16 sH[GNN_TILE * LDH];
    __shared__ __align__(16) bf16 sW[GNN_H * LDH];
    __shared__ float sCD[GNN_H], sWO[GNN_H];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = g.n, ntiles = (n + GNN_TILE - 1) / GNN_TILE;
    for (int e = tid; e < GNN_H * GNN_H; e += GNN_TILE) sW[(e >> 5) * LDH + (e & 31)] = pkd[e];
    if (tid < GNN_H) {
        sCD[tid] = pd[GPD_CD + tid];
        sWO[tid] = pd[GPD_WO + tid];
    }
    const float co = pd[GPD_CO];
    const double sx = scp->sx;
    const bool zeroed = *status != 0;
    const int gq = lane >> 2, tq = lane & 3;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {  // the block's tiles share its weights
        const int base = tile * GNN_TILE;
        __syncthreads();  // the previous tile's reads of sH are done
        load_tile(sH, hin, base, n);
        __syncthreads();
        float acc[2][4][4];
        zero(acc);
        warp_gemm<2, 4, 2>(acc, sH + warp * 32 * LDH, LDH, sW, LDH, lane);
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int hf = 0; hf < 2; hf++) {
                const int row = warp * 32 + mt * 16 + gq + 8 * hf, i = base + row;
                float s = 0.f;
#pragma unroll
                for (int nt = 0; nt < 4; nt++) {
                    const int col = nt * 8 + 2 * tq;
                    const float q0 = fmaxf(acc[mt][nt][2 * hf] + sCD[col], 0.f);
                    const float q1 = fmaxf(acc[mt][nt][2 * hf + 1] + sCD[col + 1], 0.f);
                    const bf162 qv = __floats2bfloat162_rn(q0, q1);
                    const float2 qr = __bfloat1622float2(qv);
                    s += sWO[col] * qr.x + sWO[col + 1] * qr.y;
                    if (TRAIN && i < n) *reinterpret_cast<bf162 *>(qsave + (size_t)i * GNN_H + col) = qv;
                }
                s += __shfl_xor_sync(FULL, s, 1);
                s += __shfl_xor_sync(FULL, s, 2);
                if (tq == 0 && i < n) {
                    const float yi = zeroed ? 0.f : s + co;
                    y[i] = yi;
                    if (x0) x0[i] = sx * (double)yi;
                }
            }
    }
}

// After the tcgen05 layers, whose last one writes the prediction: a pipeline
// wait that ran out (status set) leaves tiles unwritten, so the prediction
// is zero then, as k_gnn_decode writes it.
__global__ void __launch_bounds__(MCB_THREADS) k_gnn_zero_on_fail(int n, const int *__restrict__ status,
                                                                  float *__restrict__ y, double *__restrict__ x0)
{
    if (*status == 0) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        y[i] = 0.f;
        if (x0) x0[i] = 0.0;
    }
}

// ---------------------------------------------------------------- training

// Mean of (y - t / s_x) over the cells.
__global__ void __launch_bounds__(MCB_THREADS) k_gnn_loss_mean(int n, const float *__restrict__ y,
                                                               const float *__restrict__ t,
                                                               const GnnScales *__restrict__ scp, double *partials,
                                                               unsigned int *counter, double *loss)
{
    __shared__ double sh[1][MCB_THREADS];
    const double sx = scp->sx, rx = sx > 0 ? 1.0 / sx : 0.0;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc[0] += (double)y[i] - (double)t[i] * rx;
    if (publish_partials<1>(acc, partials, counter, sh)) {
        double tot[1];
        reduce_partials<1>(tot, partials, counter, sh);
        if (threadIdx.x == 0) loss[0] = tot[0] / n;
    }
}

// dy = 2 weight (y - t / s_x - mean) / n; loss = mean of the squares.
__global__ void __launch_bounds__(MCB_THREADS) k_gnn_loss_grad(int n, const float *__restrict__ y,
                                                               const float *__restrict__ t,
                                                               const GnnScales *__restrict__ scp, float weight,
                                                               float *__restrict__ dy, double *partials,
                                                               unsigned int *counter, double *loss)
{
    __shared__ double sh[1][MCB_THREADS];
    const double sx = scp->sx, rx = sx > 0 ? 1.0 / sx : 0.0, mu = loss[0];
    const double k = 2.0 * (double)weight / n;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double d = (double)y[i] - (double)t[i] * rx - mu;
        dy[i] = (float)(k * d);
        acc[0] += d * d;
    }
    if (publish_partials<1>(acc, partials, counter, sh)) {
        double tot[1];
        reduce_partials<1>(tot, partials, counter, sh);
        if (threadIdx.x == 0) loss[1] = tot[0] / n;
    }
}

// Decoder backward: dh = Wd^T dq with dq = dy wo (.) [q > 0]; partial
// gradients of Wd, cd, wo, co.
__global__ void __launch_bounds__(GNN_TILE) k_gnn_decode_bwd(GnnGraph g, const float *__restrict__ pd,
                                                             const bf16 *__restrict__ pkd,
                                                             const bf16 *__restrict__ hin,
                                                             const bf16 *__restrict__ q, const float *__restrict__ dy,
                                                             float *__restrict__ dh, float *__restrict__ gpart)
{
    __shared__ __align__(16) bf16 sDQ[GNN_TILE * LDH];
    __shared__ __align__(16) bf16 sDQT[GNN_H * LDT];
    __shared__ __align__(16) bf16 sHT[GNN_H * LDT];
    __shared__ __align__(16) bf16 sWT[GNN_H * LDH];
    __shared__ float red[4][GNN_H];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = g.n, base = blockIdx.x * GNN_TILE;
    for (int e = tid; e < GNN_H * GNN_H; e += GNN_TILE) sWT[(e & 31) * LDH + (e >> 5)] = pkd[e];  // [in][out]
    const float wo = pd[GPD_WO + lane];
    float s_dcd = 0.f, s_dwo = 0.f, s_dco = 0.f;
    for (int r = 0; r < 32; r++) {
        const int row = warp * 32 + r, i = base + row;
        float dq = 0.f;
        bf16 hv = __float2bfloat16(0.f);
        if (i < n) {
            const float qi = __bfloat162float(q[(size_t)i * GNN_H + lane]), d = dy[i];
            dq = qi > 0.f ? d * wo : 0.f;
            s_dwo += d * qi;
            s_dco += d;
            hv = hin[(size_t)i * GNN_H + lane];
        }
        s_dcd += dq;
        const bf16 dqb = __float2bfloat16(dq);
        sDQ[row * LDH + lane] = dqb;
        sDQT[lane * LDT + row] = dqb;
        sHT[lane * LDT + row] = hv;
    }
    __syncthreads();
    const int gq = lane >> 2, tq = lane & 3;
    {
        float acc[2][4][4];
        zero(acc);
        warp_gemm<2, 4, 2>(acc, sDQ + warp * 32 * LDH, LDH, sWT, LDH, lane);
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
#pragma unroll
                for (int hf = 0; hf < 2; hf++) {
                    const int row = warp * 32 + mt * 16 + gq + 8 * hf, col = nt * 8 + 2 * tq, i = base + row;
                    if (i < n)
                        *reinterpret_cast<float2 *>(dh + (size_t)i * GNN_H + col) =
                            make_float2(acc[mt][nt][2 * hf], acc[mt][nt][2 * hf + 1]);
                }
    }
    float *gp = gpart + (size_t)blockIdx.x * GNN_NPARAM + GP_DEC;
    {
        // dWd[o][in] = sum_cells dq[cell][o] h[cell][in]: warp -> (m-tile warp / 2, n-tiles 2 (warp % 2) ..)
        float acc[1][2][4];
        zero(acc);
        const int mt0 = warp >> 1, nt0 = (warp & 1) * 2;
        warp_gemm<1, 2, 8>(acc, sDQT + mt0 * 16 * LDT, LDT, sHT + nt0 * 8 * LDT, LDT, lane);
#pragma unroll
        for (int nt = 0; nt < 2; nt++)
#pragma unroll
            for (int hf = 0; hf < 2; hf++) {
                const int o = mt0 * 16 + gq + 8 * hf, in = (nt0 + nt) * 8 + 2 * tq;
                gp[GPD_WD + o * GNN_H + in] = acc[0][nt][2 * hf];
                gp[GPD_WD + o * GNN_H + in + 1] = acc[0][nt][2 * hf + 1];
            }
    }
    const float t_dcd = block_channel_sum(s_dcd, red, warp, lane);
    if (warp == 0) gp[GPD_CD + lane] = t_dcd;
    const float t_dwo = block_channel_sum(s_dwo, red, warp, lane);
    if (warp == 0) gp[GPD_WO + lane] = t_dwo;
    const float t_dco = block_channel_sum(lane == 0 ? s_dco : 0.f, red, warp, lane);
    if (warp == 0 && lane == 0) gp[GPD_CO] = t_dco;
}

// Layer backward, dense part.  In: dho = dL/dh' (FP32), the layer input h and
// the saved activation a.  Out: dhs = dL/dh through the residual and the
// self half of u; dm = dL/dm; partial gradients of W1, c1, W2, c2.
constexpr size_t BWD_SMEM = sizeof(bf16) * ((size_t)2 * GNN_H * LDT      // sUT
                                            + (size_t)GNN_TILE * LDH     // sDH
                                            + (size_t)GNN_H * LDT        // sDHT
                                            + (size_t)GNN_H * LDT        // sAT
                                            + (size_t)GNN_TILE * LDH     // sDZ
                                            + (size_t)GNN_H * LDT        // sDZT
                                            + (size_t)GNN_H * LDH        // sW2T
                                            + (size_t)2 * GNN_H * LDH)   // sW1T
                            + sizeof(float) * 4 * GNN_H;

__global__ void __launch_bounds__(GNN_TILE) k_gnn_layer_bwd_mlp(GnnGraph g, const float *__restrict__ pl,
                                                                const bf16 *__restrict__ pkl,
                                                                const bf16 *__restrict__ hin,
                                                                const bf16 *__restrict__ a,
                                                                const float *__restrict__ dho,
                                                                float *__restrict__ dhs, float *__restrict__ dm,
                                                                float *__restrict__ gpart)
{
    extern __shared__ __align__(16) unsigned char smem[];
    bf16 *sUT = reinterpret_cast<bf16 *>(smem);
    bf16 *sDH = sUT + 2 * GNN_H * LDT;
    bf16 *sDHT = sDH + GNN_TILE * LDH;
    bf16 *sAT = sDHT + GNN_H * LDT;
    bf16 *sDZ = sAT + GNN_H * LDT;
    bf16 *sDZT = sDZ + GNN_TILE * LDH;
    bf16 *sW2T = sDZT + GNN_H * LDT;
    bf16 *sW1T = sW2T + GNN_H * LDH;
    float(*red)[GNN_H] = reinterpret_cast<float(*)[GNN_H]>(sW1T + 2 * GNN_H * LDH);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = g.n, base = blockIdx.x * GNN_TILE;
    for (int e = tid; e < GNN_H * GNN_H; e += GNN_TILE) sW2T[(e & 31) * LDH + (e >> 5)] = pkl[GKL_W2 + e];
    for (int e = tid; e < GNN_H * 2 * GNN_H; e += GNN_TILE) sW1T[(e & 63) * LDH + (e >> 6)] = pkl[GKL_W1 + e];
    float s_dc2 = 0.f;
    {
        const float wg0 = pl[GPL_WG + 2 * lane], wg1 = pl[GPL_WG + 2 * lane + 1], cg = pl[GPL_CG + lane];
        const SlotCache mine = load_slots(g, base + warp * 32 + lane);
        for (int r = 0; r < 32; r++) {
            const int row = warp * 32 + r, i = base + row;
            bf16 hi = __float2bfloat16(0.f), ai = hi;
            float m = 0.f, d = 0.f;
            if (i < n) {
                hi = hin[(size_t)i * GNN_H + lane];
                ai = a[(size_t)i * GNN_H + lane];
                d = dho[(size_t)i * GNN_H + lane];
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    const int j = __shfl_sync(FULL, mine.col[k], r);
                    const float2 e = edge_of(__shfl_sync(FULL, mine.edge[k], r));
                    if (j != i) m += (wg0 * e.x + wg1 * e.y + cg) * __bfloat162float(hin[(size_t)j * GNN_H + lane]);
                }
            }
            s_dc2 += d;
            sUT[lane * LDT + row] = hi;
            sUT[(GNN_H + lane) * LDT + row] = __float2bfloat16(m);
            sAT[lane * LDT + row] = ai;
            const bf16 db = __float2bfloat16(d);
            sDH[row * LDH + lane] = db;
            sDHT[lane * LDT + row] = db;
        }
    }
    __syncthreads();
    const int gq = lane >> 2, tq = lane & 3;
    float dc1[4][2];
    {
        float acc[2][4][4];
        zero(acc);
        warp_gemm<2, 4, 2>(acc, sDH + warp * 32 * LDH, LDH, sW2T, LDH, lane);
#pragma unroll
        for (int nt = 0; nt < 4; nt++) dc1[nt][0] = dc1[nt][1] = 0.f;
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
#pragma unroll
                for (int hf = 0; hf < 2; hf++) {
                    const int row = warp * 32 + mt * 16 + gq + 8 * hf, col = nt * 8 + 2 * tq;
                    const float a0 = __bfloat162float(sAT[col * LDT + row]);
                    const float a1 = __bfloat162float(sAT[(col + 1) * LDT + row]);
                    const float z0 = a0 > 0.f ? acc[mt][nt][2 * hf] : 0.f;
                    const float z1 = a1 > 0.f ? acc[mt][nt][2 * hf + 1] : 0.f;
                    dc1[nt][0] += z0;
                    dc1[nt][1] += z1;
                    const bf162 zb = __floats2bfloat162_rn(z0, z1);
                    *reinterpret_cast<bf162 *>(sDZ + row * LDH + col) = zb;
                    sDZT[col * LDT + row] = zb.x;
                    sDZT[(col + 1) * LDT + row] = zb.y;
                }
    }
    __syncthreads();
    {
        float acc[2][8][4];
        zero(acc);
        warp_gemm<2, 8, 2>(acc, sDZ + warp * 32 * LDH, LDH, sW1T, LDH, lane);
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int nt = 0; nt < 8; nt++)
#pragma unroll
                for (int hf = 0; hf < 2; hf++) {
                    const int row = warp * 32 + mt * 16 + gq + 8 * hf, col = nt * 8 + 2 * tq, i = base + row;
                    if (i >= n) continue;
                    if (nt < 4) {
                        const float2 d = *reinterpret_cast<const float2 *>(dho + (size_t)i * GNN_H + col);
                        *reinterpret_cast<float2 *>(dhs + (size_t)i * GNN_H + col) =
                            make_float2(d.x + acc[mt][nt][2 * hf], d.y + acc[mt][nt][2 * hf + 1]);
                    } else {
                        *reinterpret_cast<float2 *>(dm + (size_t)i * GNN_H + col - GNN_H) =
                            make_float2(acc[mt][nt][2 * hf], acc[mt][nt][2 * hf + 1]);
                    }
                }
    }
    float *gp = gpart + (size_t)blockIdx.x * GNN_NPARAM;
    {
        // dW2[o][in] = sum_cells dh'[cell][o] a[cell][in]
        float acc[1][2][4];
        zero(acc);
        const int mt0 = warp >> 1, nt0 = (warp & 1) * 2;
        warp_gemm<1, 2, 8>(acc, sDHT + mt0 * 16 * LDT, LDT, sAT + nt0 * 8 * LDT, LDT, lane);
#pragma unroll
        for (int nt = 0; nt < 2; nt++)
#pragma unroll
            for (int hf = 0; hf < 2; hf++) {
                const int o = mt0 * 16 + gq + 8 * hf, in = (nt0 + nt) * 8 + 2 * tq;
                gp[GPL_W2 + o * GNN_H + in] = acc[0][nt][2 * hf];
                gp[GPL_W2 + o * GNN_H + in + 1] = acc[0][nt][2 * hf + 1];
            }
    }
    {
        // dW1[o][k] = sum_cells dz[cell][o] u[cell][k]
        float acc[1][4][4];
        zero(acc);
        const int mt0 = warp >> 1, nt0 = (warp & 1) * 4;
        warp_gemm<1, 4, 8>(acc, sDZT + mt0 * 16 * LDT, LDT, sUT + nt0 * 8 * LDT, LDT, lane);
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int hf = 0; hf < 2; hf++) {
                const int o = mt0 * 16 + gq + 8 * hf, k = (nt0 + nt) * 8 + 2 * tq;
                gp[GPL_W1 + o * 2 * GNN_H + k] = acc[0][nt][2 * hf];
                gp[GPL_W1 + o * 2 * GNN_H + k + 1] = acc[0][nt][2 * hf + 1];
            }
    }
    // dc1: per-thread column sums -> over g lanes -> over warps
    __syncthreads();
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const float v = sum_over_g(dc1[nt][e]);
            if (gq == 0) red[warp][nt * 8 + 2 * tq + e] = v;
        }
    __syncthreads();
    if (warp == 0) gp[GPL_C1 + lane] = ((red[0][lane] + red[1][lane]) + red[2][lane]) + red[3][lane];
    const float t_dc2 = block_channel_sum(s_dc2, red, warp, lane);
    if (warp == 0) gp[GPL_C2 + lane] = t_dc2;
}

// Layer backward, message part: dh_in_j = dhs_j + sum over j's internal
// slots of g (.) dm_other; partial gradients of Wg, cg.
__global__ void __launch_bounds__(GNN_TILE) k_gnn_layer_bwd_msg(GnnGraph g, const float *__restrict__ pl,
                                                                const bf16 *__restrict__ hin,
                                                                const float *__restrict__ dhs,
                                                                const float *__restrict__ dm,
                                                                float *__restrict__ dhi, float *__restrict__ gpart)
{
    __shared__ float red[4][GNN_H];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = g.n, base = blockIdx.x * GNN_TILE;
    const float wg0 = pl[GPL_WG + 2 * lane], wg1 = pl[GPL_WG + 2 * lane + 1], cg = pl[GPL_CG + lane];
    const SlotCache mine = load_slots(g, base + warp * 32 + lane);
    float s0 = 0.f, s1 = 0.f, sc = 0.f;
    for (int r = 0; r < 32; r++) {
        const int i = base + warp * 32 + r;
        if (i >= n) break;
        const float dmi = dm[(size_t)i * GNN_H + lane];
        float acc = dhs[(size_t)i * GNN_H + lane];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const int j = __shfl_sync(FULL, mine.col[k], r);
            const float2 e = edge_of(__shfl_sync(FULL, mine.edge[k], r));
            if (j != i) {
                acc += (wg0 * e.x + wg1 * e.y + cg) * dm[(size_t)j * GNN_H + lane];
                const float t = dmi * __bfloat162float(hin[(size_t)j * GNN_H + lane]);
                s0 += t * e.x;
                s1 += t * e.y;
                sc += t;
            }
        }
        dhi[(size_t)i * GNN_H + lane] = acc;
    }
    float *gp = gpart + (size_t)blockIdx.x * GNN_NPARAM;
    const float t0 = block_channel_sum(s0, red, warp, lane);
    if (warp == 0) gp[GPL_WG + 2 * lane] = t0;
    const float t1 = block_channel_sum(s1, red, warp, lane);
    if (warp == 0) gp[GPL_WG + 2 * lane + 1] = t1;
    const float tc = block_channel_sum(sc, red, warp, lane);
    if (warp == 0) gp[GPL_CG + lane] = tc;
}

// Encoder backward: partial gradients of We, ce.
__global__ void __launch_bounds__(GNN_TILE) k_gnn_encode_bwd(GnnGraph g, GnnInput<float> in,
                                                             const GnnScales *__restrict__ scp,
                                                             const bf16 *__restrict__ h0,
                                                             const float *__restrict__ dh0,
                                                             float *__restrict__ gpart)
{
    __shared__ float red[4][GNN_H];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int base = blockIdx.x * GNN_TILE + warp * 32;
    const GnnScales sc = *scp;
    const CellFeat mine = load_features(g, in, sc, base + lane);
    float s[GNN_IN + 1] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int r = 0; r < 32; r++) {
        const float xb = __shfl_sync(FULL, mine.b, r), xd = __shfl_sync(FULL, mine.d, r);
        const float xp = __shfl_sync(FULL, mine.p, r), xv = __shfl_sync(FULL, mine.v, r);
        const int i = base + r;
        if (i >= g.n) break;
        const float h = __bfloat162float(h0[(size_t)i * GNN_H + lane]);
        const float dz = h > 0.f ? dh0[(size_t)i * GNN_H + lane] : 0.f;
        s[0] += dz * xb;
        s[1] += dz * xd;
        s[2] += dz * xp;
        s[3] += dz * xv;
        s[4] += dz;
    }
    float *gp = gpart + (size_t)blockIdx.x * GNN_NPARAM;
    for (int f = 0; f < GNN_IN; f++) {
        const float t = block_channel_sum(s[f], red, warp, lane);
        if (warp == 0) gp[GP_WE + lane * GNN_IN + f] = t;
    }
    const float t = block_channel_sum(s[4], red, warp, lane);
    if (warp == 0) gp[GP_CE + lane] = t;
}

// grad[p] += sum over blocks of gpart[block][p], in block order.
__global__ void k_gnn_reduce(int nblocks, const float *__restrict__ gpart, float *__restrict__ grad)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < GNN_NPARAM; p += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int b = 0; b < nblocks; b++) s += gpart[(size_t)b * GNN_NPARAM + p];
        grad[p] += s;
    }
}

__global__ void k_gnn_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                           float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < GNN_NPARAM; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void k_gnn_pack(const float *__restrict__ p, bf16 *__restrict__ pk)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < GNN_NPACK; e += gridDim.x * blockDim.x) {
        float v;
        if (e < GK_WD) {
            const int l = e / GKL_SIZE, r = e % GKL_SIZE;
            v = r < GKL_W2 ? p[GP_LAYER0 + l * GPL_SIZE + GPL_W1 + r] : p[GP_LAYER0 + l * GPL_SIZE + GPL_W2 + r - GKL_W2];
        } else {
            v = p[GP_DEC + GPD_WD + e - GK_WD];
        }
        pk[e] = __float2bfloat16(v);
    }
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

} // namespace

// ------------------------------------------------------------------ host API

size_t gnn_work_bytes(int n, bool train)
{
    GnnWork w;
    gnn_work_carve(w, nullptr, n, train);
    return (size_t)(reinterpret_cast<uintptr_t>(w.loss) + align256(2 * sizeof(double)));
}

void gnn_work_carve(GnnWork &w, char *base, int n, bool train)
{
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char *p = base + off;
        off += align256(bytes);
        return p;
    };
    w.n = n;
    w.nblocks = gnn_blocks(n);
    w.train = train;
    const size_t hb = (size_t)n * GNN_H * sizeof(bf16), fb = (size_t)n * GNN_H * sizeof(float);
    const int nh = train ? GNN_L + 1 : 2;
    for (int l = 0; l <= GNN_L; l++) w.h[l] = l < nh ? reinterpret_cast<bf16 *>(take(hb)) : nullptr;
    for (int l = 0; l < GNN_L; l++) w.a[l] = train ? reinterpret_cast<bf16 *>(take(hb)) : nullptr;
    w.q = train ? reinterpret_cast<bf16 *>(take(hb)) : nullptr;
    w.y = reinterpret_cast<float *>(take((size_t)n * sizeof(float)));
    w.fold = reinterpret_cast<bf16 *>(take((size_t)GNN_L * 7 * GNN_H * GNN_H * sizeof(bf16)));
    w.dh[0] = train ? reinterpret_cast<float *>(take(fb)) : nullptr;
    w.dh[1] = train ? reinterpret_cast<float *>(take(fb)) : nullptr;
    w.dm = train ? reinterpret_cast<float *>(take(fb)) : nullptr;
    w.dy = train ? reinterpret_cast<float *>(take((size_t)n * sizeof(float))) : nullptr;
    w.gpart = train ? reinterpret_cast<float *>(take((size_t)w.nblocks * GNN_NPARAM * sizeof(float))) : nullptr;
    w.partials = reinterpret_cast<double *>(take((size_t)reduce_grid(n) * 2 * sizeof(double)));
    w.counter = reinterpret_cast<unsigned int *>(take(256));
    w.scales = reinterpret_cast<GnnScales *>(take(sizeof(GnnScales)));
    w.status = reinterpret_cast<int *>(take(sizeof(int)));
    w.loss = reinterpret_cast<double *>(base + off);
}

void gnn_init_params(float *p, uint64_t seed)
{
    uint64_t state = seed;
    auto next = [&]() {  // splitmix64
        uint64_t z = (state += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
    };
    auto fill = [&](int off, int count, int fan_in, double gain) {
        const double a = gain * std::sqrt(6.0 / fan_in);
        for (int i = 0; i < count; i++) p[off + i] = (float)((2.0 * next() - 1.0) * a);
    };
    for (int i = 0; i < GNN_NPARAM; i++) p[i] = 0.f;
    fill(GP_WE, GNN_H * GNN_IN, GNN_IN, 1.0);
    for (int l = 0; l < GNN_L; l++) {
        const int b = GP_LAYER0 + l * GPL_SIZE;
        fill(b + GPL_WG, GNN_H * 2, 2, 0.5);
        for (int c = 0; c < GNN_H; c++) p[b + GPL_CG + c] = 1.0f / 6.0f;
        fill(b + GPL_W1, GNN_H * 2 * GNN_H, 2 * GNN_H, 1.0);
        fill(b + GPL_W2, GNN_H * GNN_H, GNN_H, 0.2);
    }
    fill(GP_DEC + GPD_WD, GNN_H * GNN_H, GNN_H, 1.0);
    fill(GP_DEC + GPD_WO, GNN_H, GNN_H, 0.5);
}

void gnn_pack(cudaStream_t s, const float *p, bf16 *pk) { k_gnn_pack<<<32, 256, 0, s>>>(p, pk); }

// train: keep every layer's input and relu(W1 u + c1) for the backward pass
// (needs a work area carved with train = true); inference ping-pongs h[0],
// h[1] and uses the offset-form weights where the graph allows.
template <typename T>
static void forward_impl(cudaStream_t s, const GnnGraph &g, const GnnInput<T> &in, const float *p, const bf16 *pk,
                         GnnWork &w, double *x0, bool train, int parts = GNN_FWD_ALL)
{
    const int nb = gnn_blocks(g.n);
    const bool folded = !train && g.affine;
    const GnnLayerPath path = gnn_layer_path();
    GnnTmaMap maps[2];
    const bool umma = folded && path != GnnLayerPath::Mma && gnn_umma_map(&maps[0], w.h[0], g.n) &&
                      gnn_umma_map(&maps[1], w.h[1], g.n) && gnn_umma_ready();
    if (parts & GNN_FWD_BEGIN) {
        cudaMemsetAsync(w.status, 0, sizeof(int), s);
        if (folded && !umma && path == GnnLayerPath::UmmaRequired) cudaMemsetAsync(w.status, 0x7f, sizeof(int), s);
        k_gnn_scales<T><<<reduce_grid(g.n), MCB_THREADS, 0, s>>>(g.n, in, w.partials, w.counter, w.scales);
        k_gnn_encode<T><<<nb, GNN_TILE, 0, s>>>(g, in, p, w.scales, w.h[0]);
        if (folded) k_gnn_fold<<<(GNN_L * 7 * GNN_H * GNN_H + 255) / 256, 256, 0, s>>>(p, g, w.fold);
    }
    if (folded) {
        cudaFuncSetAttribute(k_gnn_layer_fold, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FOLD_SMEM);
    } else {
        cudaFuncSetAttribute(k_gnn_layer<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LAYER_SMEM);
        cudaFuncSetAttribute(k_gnn_layer<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LAYER_SMEM);
    }
    // the tcgen05 path runs the decoder inside the last layer
    const GnnUmmaDecode dec{pk + GK_WD, p + GP_DEC, w.scales, w.y, x0};
    for (int l = 0; (parts & GNN_FWD_LAYERS) && l < GNN_L; l++) {
        const float *pl = p + GP_LAYER0 + l * GPL_SIZE;
        const bf16 *pkl = pk + GK_LAYER0 + l * GKL_SIZE;
        if (train)
            k_gnn_layer<true><<<nb, LAYER_THREADS, LAYER_SMEM, s>>>(g, pl, pkl, w.h[l], w.h[l + 1], w.a[l]);
        else if (folded) {
            const bf16 *wf = w.fold + (size_t)l * 7 * GNN_H * GNN_H;
            if (umma)
                gnn_layer_umma(s, g, maps[l & 1], pl, wf, pkl, w.h[l & 1], w.h[(l + 1) & 1], w.status, sm_count(),
                               l == GNN_L - 1 ? &dec : nullptr);
            else
                k_gnn_layer_fold<<<std::min(nb, sm_count()), LAYER_THREADS, FOLD_SMEM, s>>>(
                    g, pl, wf, pkl, w.h[l & 1], w.h[(l + 1) & 1], nb);
        } else
            k_gnn_layer<false><<<nb, LAYER_THREADS, LAYER_SMEM, s>>>(g, pl, pkl, w.h[l & 1], w.h[(l + 1) & 1], nullptr);
    }
    if (!(parts & GNN_FWD_END)) return;
    if (umma) {
        k_gnn_zero_on_fail<<<reduce_grid(g.n), MCB_THREADS, 0, s>>>(g.n, w.status, w.y, x0);
        return;
    }
    const bf16 *hl = train ? w.h[GNN_L] : w.h[GNN_L & 1];
    const int gd = std::min(nb, 16 * sm_count());  // the decoder loops over tiles
    if (train)
        k_gnn_decode<true><<<gd, GNN_TILE, 0, s>>>(g, p + GP_DEC, pk + GK_WD, hl, w.scales, w.y, x0, w.q, w.status);
    else
        k_gnn_decode<false><<<gd, GNN_TILE, 0, s>>>(g, p + GP_DEC, pk + GK_WD, hl, w.scales, w.y, x0, nullptr,
                                                    w.status);
}

template <typename T>
void gnn_forward(cudaStream_t s, const GnnGraph &g, const GnnInput<T> &in, const float *p, const bf16 *pk, GnnWork &w,
                 double *x0, int parts)
{
    forward_impl<T>(s, g, in, p, pk, w, x0, false, parts);
}
template void gnn_forward<double>(cudaStream_t, const GnnGraph &, const GnnInput<double> &, const float *,
                                  const bf16 *, GnnWork &, double *, int);
template void gnn_forward<float>(cudaStream_t, const GnnGraph &, const GnnInput<float> &, const float *, const bf16 *,
                                 GnnWork &, double *, int);

int gnn_forward_launches() { return 4 + GNN_L; }

void gnn_loss_backward(cudaStream_t s, const GnnGraph &g, const GnnInput<float> &in, const float *target,
                       const float *p, const bf16 *pk, GnnWork &w, float *grad, float weight)
{
    cudaFuncSetAttribute(k_gnn_layer_bwd_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BWD_SMEM);
    const int nb = gnn_blocks(g.n), rg = reduce_grid(g.n);
    forward_impl<float>(s, g, in, p, pk, w, nullptr, true);
    k_gnn_loss_mean<<<rg, MCB_THREADS, 0, s>>>(g.n, w.y, target, w.scales, w.partials, w.counter, w.loss);
    k_gnn_loss_grad<<<rg, MCB_THREADS, 0, s>>>(g.n, w.y, target, w.scales, weight, w.dy, w.partials, w.counter,
                                               w.loss);
    k_gnn_decode_bwd<<<nb, GNN_TILE, 0, s>>>(g, p + GP_DEC, pk + GK_WD, w.h[GNN_L], w.q, w.dy, w.dh[0], w.gpart);
    int cur = 0;  // w.dh[cur] = dL/d(output of layer l)
    for (int l = GNN_L - 1; l >= 0; l--) {
        const float *pl = p + GP_LAYER0 + l * GPL_SIZE;
        const bf16 *pkl = pk + GK_LAYER0 + l * GKL_SIZE;
        float *gpl = w.gpart + GP_LAYER0 + l * GPL_SIZE;
        k_gnn_layer_bwd_mlp<<<nb, GNN_TILE, BWD_SMEM, s>>>(g, pl, pkl, w.h[l], w.a[l], w.dh[cur], w.dh[cur ^ 1], w.dm,
                                                           gpl);
        k_gnn_layer_bwd_msg<<<nb, GNN_TILE, 0, s>>>(g, pl, w.h[l], w.dh[cur ^ 1], w.dm, w.dh[cur], gpl);
    }
    k_gnn_encode_bwd<<<nb, GNN_TILE, 0, s>>>(g, in, w.scales, w.h[0], w.dh[cur], w.gpart);
    k_gnn_reduce<<<(GNN_NPARAM + 255) / 256, 256, 0, s>>>(nb, w.gpart, grad);
}

void gnn_adam(cudaStream_t s, float *p, const float *grad, float *m, float *v, float lr, float b1, float b2, float eps,
              int t)
{
    const float c1 = 1.f - std::pow(b1, (float)t), c2 = 1.f - std::pow(b2, (float)t);
    k_gnn_adam<<<(GNN_NPARAM + 255) / 256, 256, 0, s>>>(p, grad, m, v, lr, b1, b2, eps, c1, c2);
}

} // namespace mcb
