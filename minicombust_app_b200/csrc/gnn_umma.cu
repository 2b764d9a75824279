// Message-passing layer of the learned guess on the fifth-generation tensor
// cores (inference, graph in offset form).
//
// Per tile of 128 cells the layer is two products with the accumulators in
// TMEM:
//   D1 = U . W1f^T      U = [h_i | h_{i+d_1} | ... | h_{i+d_6}]  (128 x 224)
//   a  = relu(D1 + c1)                                         (BF16)
//   D2 = a . W2^T,      h'_i = h_i + (D2 + c2)                 (BF16)
// where W1f holds the folded gates (see k_gnn_fold).  The seven 128-row
// slices of U are contiguous row ranges of h (offset form), so each is one
// 2-D TMA tile load (8 KB, 128 rows x 64 B) with the 64-byte swizzle, which is
// the K-major operand layout of the MMA for 64-byte rows (8-row groups 512 B
// apart, a K = 16 step 32 bytes into the row); rows outside [0, n) read
// zeros, and rows of directions a cell does not have (mask bit clear) are
// zeroed in shared memory before the MMA is issued.
//
// Warp roles (one persistent block per SM):
//   warps 0-11  three epilogue groups of four warps; group g owns the tiles
//               j = g, g + 3, ... of the block, their copy stage g and
//               their TMEM columns (so each barrier's phases are consumed in
//               order); thread r of a group is row r of the tile and TMEM
//               lane r (warp w reads lanes 32 (w % 4) ..)
//   warp 12     TMA producer (one thread)
//   warp 13     TMEM allocation and the MMA issue (one elected thread)
//   warps 14-17 masking: thread r zeroes the missing-direction rows of row r
//               of each tile as soon as its copies land
// The MMA thread issues whichever product is ready -- the first product of
// a tile once its slices are masked and its group has read the previous
// first product out of TMEM, the second once the group has written the
// a-tile.  A stage is refilled as soon as its first product completes, so
// the copies run ahead of the epilogues instead of waiting for them, and
// the copies, the tensor core and three tiles' epilogues overlap.  Every
// wait is bounded: on
// a time-out the block records a status, drains its copies and MMAs, frees
// its TMEM and returns, and the decoder then writes a zero prediction.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "gnn.cuh"
#include "sm100.cuh"

namespace mcb {

namespace {

using bf16 = __nv_bfloat16;
using namespace sm100;

constexpr int UM_STAGES = 3;
constexpr int UM_SLICE = GNN_TILE * GNN_H * 2;      // 8192 B: 128 rows x 64 B
constexpr int UM_STAGE = 7 * UM_SLICE;              // 57344 B
constexpr int UM_B1 = 7 * GNN_H * GNN_H * 2;        // 14336 B: 28 K-groups of 32 rows x 16 B
constexpr int UM_B2 = GNN_H * GNN_H * 2;            // 2048 B
constexpr int UM_A1 = GNN_TILE * GNN_H * 2;         // 8192 B per epilogue group
constexpr int UM_GROUPS = 3;  // one copy stage per group
constexpr int UM_THREADS = 128 * UM_GROUPS + 64 + 128;
// TMEM columns of a group: D1 and D2 (and for the last layer D3 of the
// decoder), 32 columns each, at 128-column group strides; a power of two
constexpr uint32_t UM_TMEM_COLS = 512;
constexpr uint32_t UM_GROUP_COLS = 128;
constexpr int WARP_TMA = 4 * UM_GROUPS, WARP_MMA = 4 * UM_GROUPS + 1, WARP_MASK = 4 * UM_GROUPS + 2;

constexpr int OFF_STAGE = 0;
constexpr int OFF_B1 = OFF_STAGE + UM_STAGES * UM_STAGE;
constexpr int OFF_B2 = OFF_B1 + UM_B1;
constexpr int OFF_B3 = OFF_B2 + UM_B2;                // the decoder's Wd (last layer)
constexpr int OFF_A1 = OFF_B3 + UM_B2;
constexpr int OFF_BIAS = OFF_A1 + UM_GROUPS * UM_A1;  // c1, c2, cd, wo
constexpr int OFF_BAR = OFF_BIAS + 4 * GNN_H * 4;
// barriers: full[3], masked[3], empty[3], d1full[3], a1full[3], d2full[3],
// d1free[3], hfull[3], d3full[3], fin
constexpr int NBAR = 3 * UM_STAGES + 6 * UM_GROUPS + 1;
constexpr int OFF_MISC = OFF_BAR + NBAR * 8;
constexpr int UM_SMEM_USED = OFF_MISC + 16;
constexpr int UM_SMEM = UM_SMEM_USED + 1024;        // slack for the 1024-byte alignment of the base

constexpr uint32_t WAIT_LIMIT = 1u << 22;
constexpr unsigned FULL = 0xffffffffu;

static_assert(UM_SMEM <= 227 * 1024, "shared memory of the tensor-core layer");
static_assert(UM_STAGES == UM_GROUPS && UM_GROUP_COLS * UM_GROUPS <= UM_TMEM_COLS, "stage and TMEM set per group");
static_assert(OFF_B1 % 1024 == 0 && OFF_A1 % 1024 == 0, "operand alignment");

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    uint32_t u;
    memcpy(&u, &v, 4);
    return u;
}

__device__ __forceinline__ float2 unpack_bf16(uint32_t u)
{
    __nv_bfloat162 v;
    memcpy(&v, &u, 4);
    return __bfloat1622float2(v);
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

struct UmmaBars {
    uint32_t base;
    __device__ uint32_t full(int s) const { return base + 8 * s; }
    __device__ uint32_t masked(int s) const { return base + 8 * (UM_STAGES + s); }
    __device__ uint32_t empty(int s) const { return base + 8 * (2 * UM_STAGES + s); }
    __device__ uint32_t d1full(int g) const { return base + 8 * (3 * UM_STAGES + g); }
    __device__ uint32_t a1full(int g) const { return base + 8 * (3 * UM_STAGES + UM_GROUPS + g); }
    __device__ uint32_t d2full(int g) const { return base + 8 * (3 * UM_STAGES + 2 * UM_GROUPS + g); }
    __device__ uint32_t d1free(int g) const { return base + 8 * (3 * UM_STAGES + 3 * UM_GROUPS + g); }
    __device__ uint32_t hfull(int g) const { return base + 8 * (3 * UM_STAGES + 4 * UM_GROUPS + g); }
    __device__ uint32_t d3full(int g) const { return base + 8 * (3 * UM_STAGES + 5 * UM_GROUPS + g); }
    __device__ uint32_t fin() const { return base + 8 * (3 * UM_STAGES + 6 * UM_GROUPS); }
};

// The decoder fused into the last layer (LAST): y = wo . relu(Wd h' + cd) + co
// and x0 = s_x y, with D3 = h' Wd^T a third product per tile (h' in BF16, as
// the layer stores it for k_gnn_decode).
struct UmmaDecode {
    const bf16 *pkd;     // Wd, BF16 [32][32]
    const float *pd;     // the decoder's FP32 parameters (cd, wo, co)
    const GnnScales *scales;
    float *y;
    double *x0;          // may be null
};

template <bool LAST>
__global__ void __launch_bounds__(UM_THREADS, 1)
    k_gnn_layer_umma(const __grid_constant__ CUtensorMap tmap, GnnGraph g, const float *__restrict__ pl,
                     const bf16 *__restrict__ wf, const bf16 *__restrict__ pkl, const bf16 *__restrict__ hin,
                     bf16 *__restrict__ hout, int ntiles, int *status, uint32_t wait_polls, UmmaDecode dec)
{
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t sbase = (raw + 1023u) & ~1023u;
    unsigned char *sgen = smem_raw + (sbase - raw);
    float *sC1 = reinterpret_cast<float *>(sgen + OFF_BIAS);
    float *sC2 = sC1 + GNN_H;
    float *sCD = sC2 + GNN_H;
    float *sWO = sCD + GNN_H;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(sgen + OFF_MISC);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sgen + OFF_MISC + 4);
    const UmmaBars bars{sbase + OFF_BAR};
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        for (int s = 0; s < UM_STAGES; s++) {
            mbar_init(bars.full(s), 1);
            mbar_init(bars.masked(s), 128);
            mbar_init(bars.empty(s), 1);
        }
        for (int q = 0; q < UM_GROUPS; q++) {
            mbar_init(bars.d1full(q), 1);
            mbar_init(bars.a1full(q), 128);
            mbar_init(bars.d2full(q), 1);
            mbar_init(bars.d1free(q), 128);
            mbar_init(bars.hfull(q), 128);
            mbar_init(bars.d3full(q), 1);
        }
        mbar_init(bars.fin(), 1);
        *abort_flag = 0;
        mbar_fence_init();
    }
    if (warp == WARP_MMA) {
        tmem_alloc(smem_u32(tmem_slot), UM_TMEM_COLS);
        tmem_relinquish();
    }
    // B operands, K-major without swizzle: element (n, k) at
    // (k / 8) * 512 + n * 16 + (k % 8) * 2 -- core matrices of 8 rows x 16 B,
    // 8-row groups 128 B apart, K groups 512 B apart.
    for (int e = tid; e < (LAST ? 9 : 8) * GNN_H * 4; e += UM_THREADS) {
        const int slot = e >> 7, rem = e & 127, n = rem >> 2, c = rem & 3;
        const uint4 v = slot < 7  ? *reinterpret_cast<const uint4 *>(wf + ((size_t)slot * GNN_H + n) * GNN_H + c * 8)
                        : slot == 7 ? *reinterpret_cast<const uint4 *>(pkl + GKL_W2 + n * GNN_H + c * 8)
                                    : *reinterpret_cast<const uint4 *>(dec.pkd + n * GNN_H + c * 8);
        const uint32_t dst = slot < 7  ? sbase + OFF_B1 + (slot * 4 + c) * 512 + n * 16
                             : slot == 7 ? sbase + OFF_B2 + c * 512 + n * 16
                                         : sbase + OFF_B3 + c * 512 + n * 16;
        st_shared_v4(dst, v.x, v.y, v.z, v.w);
    }
    if (tid < GNN_H) {
        sC1[tid] = pl[GPL_C1 + tid];
        sC2[tid] = pl[GPL_C2 + tid];
        if (LAST) {
            sCD[tid] = dec.pd[GPD_CD + tid];
            sWO[tid] = dec.pd[GPD_WO + tid];
        }
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    auto fail = [&](int code) {
        *abort_flag = 1;
        atomicExch(status, code);
    };

    if (warp == WARP_TMA) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            tma_prefetch_desc(&tmap);
            int issued = 0;
            for (int j = 0;; j++) {
                const int tile = blockIdx.x + j * gridDim.x;
                if (tile >= ntiles) break;
                const int s = j % UM_STAGES;
                if (j >= UM_STAGES && !mbar_wait(bars.empty(s), ((j / UM_STAGES) - 1) & 1, abort_flag, wait_polls)) {
                    fail(1);
                    break;
                }
                mbar_arrive_expect_tx(bars.full(s), UM_STAGE);
                const int y0 = tile * GNN_TILE;
                const uint32_t dst = sbase + OFF_STAGE + s * UM_STAGE;
                tma_load_2d(dst, &tmap, bars.full(s), 0, y0);
#pragma unroll
                for (int k = 0; k < 6; k++) tma_load_2d(dst + (1 + k) * UM_SLICE, &tmap, bars.full(s), 0, y0 + g.doff[k]);
                issued = j + 1;
            }
            // every copy this block started lands before the block exits
            for (int s = 0; s < UM_STAGES; s++) {
                int jl = -1;
                for (int j = s; j < issued; j += UM_STAGES) jl = j;
                if (jl >= 0 && !mbar_wait(bars.full(s), (jl / UM_STAGES) & 1, nullptr, WAIT_LIMIT)) fail(2);
            }
        }
    } else if (warp == WARP_MMA) {
        // ---------------------------------------------------------- MMA issue
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16_f32(GNN_TILE, GNN_H);
            const int nj = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
            int j1 = 0, j2 = 0, j3 = 0;  // next tile of the first / second / decoder product
            uint32_t idle = 0;
            while (LAST ? j3 < nj : j2 < nj) {
                bool progressed = false;
                if (j1 < nj && mbar_test_wait(bars.masked(j1 % UM_STAGES), (j1 / UM_STAGES) & 1) &&
                    (j1 < UM_GROUPS || mbar_test_wait(bars.d1free(j1 % UM_GROUPS), ((j1 / UM_GROUPS) - 1) & 1))) {
                    tc_fence_after();
                    const int s = j1 % UM_STAGES, q = j1 % UM_GROUPS;
                    const uint32_t a0 = sbase + OFF_STAGE + s * UM_STAGE;
#pragma unroll
                    for (int ks = 0; ks < 14; ks++) {
                        const uint64_t ad = smem_desc(a0 + (ks >> 1) * UM_SLICE + (ks & 1) * 32, 16, 512,
                                                      DESC_SWIZZLE_64B);
                        const uint64_t bd = smem_desc(sbase + OFF_B1 + ks * 1024, 512, 128, DESC_SWIZZLE_NONE);
                        umma_f16(tmem + q * UM_GROUP_COLS, ad, bd, idesc, ks > 0);
                    }
                    umma_commit(bars.empty(s));
                    umma_commit(bars.d1full(q));
                    j1++;
                    progressed = true;
                }
                if (j2 < j1 && mbar_test_wait(bars.a1full(j2 % UM_GROUPS), (j2 / UM_GROUPS) & 1)) {
                    tc_fence_after();
                    const int q = j2 % UM_GROUPS;
#pragma unroll
                    for (int ks = 0; ks < 2; ks++) {
                        const uint64_t ad = smem_desc(sbase + OFF_A1 + q * UM_A1 + ks * 4096, 2048, 128, DESC_SWIZZLE_NONE);
                        const uint64_t bd = smem_desc(sbase + OFF_B2 + ks * 1024, 512, 128, DESC_SWIZZLE_NONE);
                        umma_f16(tmem + q * UM_GROUP_COLS + 32, ad, bd, idesc, ks > 0);
                    }
                    umma_commit(bars.d2full(q));
                    j2++;
                    progressed = true;
                }
                if (LAST && j3 < j2 && mbar_test_wait(bars.hfull(j3 % UM_GROUPS), (j3 / UM_GROUPS) & 1)) {
                    tc_fence_after();
                    const int q = j3 % UM_GROUPS;
#pragma unroll
                    for (int ks = 0; ks < 2; ks++) {  // h' of the tile, in the group's a-tile
                        const uint64_t ad = smem_desc(sbase + OFF_A1 + q * UM_A1 + ks * 4096, 2048, 128, DESC_SWIZZLE_NONE);
                        const uint64_t bd = smem_desc(sbase + OFF_B3 + ks * 1024, 512, 128, DESC_SWIZZLE_NONE);
                        umma_f16(tmem + q * UM_GROUP_COLS + 64, ad, bd, idesc, ks > 0);
                    }
                    umma_commit(bars.d3full(q));
                    j3++;
                    progressed = true;
                }
                if (progressed) {
                    idle = 0;
                } else if (++idle > 16u * wait_polls || *abort_flag) {  // test_wait does not suspend
                    fail(3);
                    break;
                }
            }
            // every MMA this thread issued completes before TMEM is freed
            umma_commit(bars.fin());
            if (!mbar_wait(bars.fin(), 0, nullptr, WAIT_LIMIT)) fail(5);
        }
    } else if (warp >= WARP_MASK) {
        // ---------------------------------------------------------- masking
        const int r = tid - 32 * WARP_MASK;  // row of the tile
        for (int j = 0;; j++) {
            const int tile = blockIdx.x + j * gridDim.x;
            if (tile >= ntiles) break;
            const int s = j % UM_STAGES, i = tile * GNN_TILE + r;
            const unsigned mk = i < g.n ? g.mask[i] : 0u;
            const bool ok = mbar_wait(bars.full(s), (j / UM_STAGES) & 1, abort_flag, wait_polls);
            if (!__all_sync(FULL, ok)) {
                fail(6);
                break;
            }
            // rows of directions this cell does not have read zeros
            const uint32_t row0 = sbase + OFF_STAGE + s * UM_STAGE + r * 64;  // the swizzle stays inside a row
#pragma unroll
            for (int k = 0; k < 6; k++)
                if (!((mk >> k) & 1u)) {
                    const uint32_t a = row0 + (1 + k) * UM_SLICE;
#pragma unroll
                    for (int c = 0; c < 4; c++) st_shared_v4(a + 16 * c, 0u, 0u, 0u, 0u);
                }
            if (mk != 0x3fu) fence_proxy_async_smem();  // only a thread that wrote zeros has to order them
            mbar_arrive(bars.masked(s));
        }
    } else {
        // ---------------------------------------------------------- epilogue
        const int q = warp >> 2, r = tid & 127;  // group, row
        const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
        const uint32_t a1 = sbase + OFF_A1 + q * UM_A1 + r * 16;
        for (int j = q;; j += UM_GROUPS) {
            const int tile = blockIdx.x + j * gridDim.x;
            if (tile >= ntiles) break;
            const int i = tile * GNN_TILE + r;
            const bool in = i < g.n;
            uint4 hv[4];
#pragma unroll
            for (int c = 0; c < 4; c++)
                hv[c] = in ? __ldg(reinterpret_cast<const uint4 *>(hin + (size_t)i * GNN_H) + c) : make_uint4(0, 0, 0, 0);

            // a = relu(D1 + c1) into the group's K-major a-tile; D1 is
            // released for the group's next tile as soon as it is read
            bool ok = mbar_wait(bars.d1full(q), (j / UM_GROUPS) & 1, abort_flag, wait_polls);
            if (!__all_sync(FULL, ok)) {
                fail(7);
                break;
            }
            tc_fence_after();
            uint32_t v[32];
            tmem_ld32(tmem + q * UM_GROUP_COLS + lane_base, v);
            tc_fence_before();
            mbar_arrive(bars.d1free(q));
#pragma unroll
            for (int c = 0; c < 4; c++) {
                uint32_t pk[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int col = 8 * c + 2 * e;
                    pk[e] = pack_bf16(fmaxf(__uint_as_float(v[col]) + sC1[col], 0.f),
                                      fmaxf(__uint_as_float(v[col + 1]) + sC1[col + 1], 0.f));
                }
                st_shared_v4(a1 + c * 2048, pk[0], pk[1], pk[2], pk[3]);
            }
            fence_proxy_async_smem();
            tc_fence_before();
            mbar_arrive(bars.a1full(q));

            // h' = h + (D2 + c2)
            ok = mbar_wait(bars.d2full(q), (j / UM_GROUPS) & 1, abort_flag, wait_polls);
            if (!__all_sync(FULL, ok)) {
                fail(8);
                break;
            }
            tc_fence_after();
            tmem_ld32(tmem + q * UM_GROUP_COLS + 32 + lane_base, v);
            tc_fence_before();
            uint32_t o[4][4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const uint32_t hw[4] = {hv[c].x, hv[c].y, hv[c].z, hv[c].w};
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int col = 8 * c + 2 * e;
                    const float2 h2 = unpack_bf16(hw[e]);
                    o[c][e] = pack_bf16(h2.x + (__uint_as_float(v[col]) + sC2[col]),
                                        h2.y + (__uint_as_float(v[col + 1]) + sC2[col + 1]));
                }
            }
            if (!LAST) {
                if (in) {
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        *reinterpret_cast<uint4 *>(hout + (size_t)i * GNN_H + c * 8) =
                            make_uint4(o[c][0], o[c][1], o[c][2], o[c][3]);
                }
                continue;
            }
            // the decoder: h' (rows outside the mesh are zeros) into the
            // group's a-tile, whose second product has completed
#pragma unroll
            for (int c = 0; c < 4; c++)
                st_shared_v4(a1 + c * 2048, in ? o[c][0] : 0u, in ? o[c][1] : 0u, in ? o[c][2] : 0u, in ? o[c][3] : 0u);
            fence_proxy_async_smem();
            tc_fence_before();
            mbar_arrive(bars.hfull(q));
            ok = mbar_wait(bars.d3full(q), (j / UM_GROUPS) & 1, abort_flag, wait_polls);
            if (!__all_sync(FULL, ok)) {
                fail(9);
                break;
            }
            tc_fence_after();
            tmem_ld32(tmem + q * UM_GROUP_COLS + 64 + lane_base, v);
            tc_fence_before();
            float ys = 0.f;
#pragma unroll
            for (int col = 0; col < GNN_H; col += 2) {  // q = relu(Wd h' + cd), rounded to BF16 as stored
                const float2 qr = unpack_bf16(pack_bf16(fmaxf(__uint_as_float(v[col]) + sCD[col], 0.f),
                                                        fmaxf(__uint_as_float(v[col + 1]) + sCD[col + 1], 0.f)));
                ys += sWO[col] * qr.x + sWO[col + 1] * qr.y;
            }
            if (in) {
                const float yi = ys + dec.pd[GPD_CO];
                dec.y[i] = yi;
                if (dec.x0) dec.x0[i] = dec.scales->sx * (double)yi;
            }
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp == WARP_MMA) {
        tc_fence_after();
        tmem_dealloc(tmem, UM_TMEM_COLS);
    }
}

} // namespace

// Polls of the layer's pipeline waits before it gives up (the waits that
// drain copies and products in flight before the block exits keep the full
// bound).  MC_GNN_WAIT_POLLS overrides the bound, read at every launch, so a
// test can make the pipeline waits run out (0: the first wait fails) and then
// restore it on the same handle.
static uint32_t wait_polls()
{
    const char *v = std::getenv("MC_GNN_WAIT_POLLS");
    if (v && *v) {
        const long n = std::strtol(v, nullptr, 10);
        if (n >= 0 && n < (long)WAIT_LIMIT) return (uint32_t)n;
    }
    return WAIT_LIMIT;
}

GnnLayerPath gnn_layer_path()
{
    const char *v = std::getenv("MC_GNN_LAYER");
    if (v && std::strcmp(v, "mma") == 0) return GnnLayerPath::Mma;
    if (v && std::strcmp(v, "umma") == 0) return GnnLayerPath::UmmaRequired;
    return GnnLayerPath::Umma;
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

} // namespace

bool gnn_umma_map(GnnTmaMap *m, const bf16 *h, int n)
{
    static_assert(sizeof(GnnTmaMap) == sizeof(CUtensorMap), "tensor map size");
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || n <= 0 || (reinterpret_cast<uintptr_t>(h) & 15u)) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)GNN_H, (cuuint64_t)n};
    const cuuint64_t strides[1] = {(cuuint64_t)GNN_H * sizeof(bf16)};
    const cuuint32_t box[2] = {(cuuint32_t)GNN_H, (cuuint32_t)GNN_TILE};
    const cuuint32_t estr[2] = {1, 1};
    CUtensorMap t;
    if (fn(&t, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(h), dims, strides, box, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    std::memcpy(m->raw, &t, sizeof(t));
    return true;
}

bool gnn_umma_ready()
{
    static int state = 0;  // 0 unknown, 1 ready, -1 failed
    if (state == 0)
        state = (cudaFuncSetAttribute(k_gnn_layer_umma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, UM_SMEM) ==
                     cudaSuccess &&
                 cudaFuncSetAttribute(k_gnn_layer_umma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, UM_SMEM) ==
                     cudaSuccess)
                    ? 1
                    : -1;
    return state > 0;
}

void gnn_layer_umma(cudaStream_t s, const GnnGraph &g, const GnnTmaMap &map, const float *pl, const bf16 *wf,
                    const bf16 *pkl, const bf16 *hin, bf16 *hout, int *status, int grid, const GnnUmmaDecode *dec)
{
    CUtensorMap t;
    std::memcpy(&t, map.raw, sizeof(t));
    const int ntiles = (g.n + GNN_TILE - 1) / GNN_TILE;
    const int blocks = std::max(1, std::min(grid, ntiles));
    if (dec) {
        const UmmaDecode d{dec->pkd, dec->pd, dec->scales, dec->y, dec->x0};
        k_gnn_layer_umma<true><<<blocks, UM_THREADS, UM_SMEM, s>>>(t, g, pl, wf, pkl, hin, hout, ntiles, status,
                                                                  wait_polls(), d);
    } else {
        k_gnn_layer_umma<false><<<blocks, UM_THREADS, UM_SMEM, s>>>(t, g, pl, wf, pkl, hin, hout, ntiles, status,
                                                                   wait_polls(), UmmaDecode{});
    }
}

} // namespace mcb
