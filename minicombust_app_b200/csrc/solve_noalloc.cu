// Allocation-free variant of the single-system BiCGStab solve.
//
// The handle-based solver keeps its Krylov vectors, block partials and status
// block in the handle's cudaMalloc arena.  This entry point runs the same
// kernels (k_bicg_init/1/2/3 with one right-hand side, as in the temperature
// stage) on a system the caller owns, with every scratch byte taken from the
// file-scope array below instead.  It exists for callers that must not
// allocate device memory: hosts that reserve all device memory for their own
// pool or fixed budget at start-up (a library cudaMalloc would then fail, or
// take memory the host has promised elsewhere), and callers inside a
// time-critical loop, where cudaMalloc/cudaFree can synchronise the device and
// stall their other streams.
//
// Limits and sharing:
//   - at most MC_SOLVE_NOALLOC_MAX_ROWS rows; the array holds 8 vectors of that
//     length plus partials and status, about 16 MB, on every device that
//     loads the library, until the process exits;
//   - every call uses the same array: calls that overlap on the GPU (on
//     different streams or host threads) race; the status counter is cleared
//     at the start of each call, and every vector is initialised by the solve;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current).
#include <cuda_runtime.h>

#include <mutex>

#include "krylov.cuh"
#include "mc_reduce.cuh"
#include "minicombust_flow.h"

namespace {

constexpr int kMaxRows = MC_SOLVE_NOALLOC_MAX_ROWS;
constexpr int kVectors = 8;                       // r, r0, p[2], v[2], s, t
// The Krylov kernels run MCB_THREADS threads per block and at most one block
// per MCB_THREADS rows (krylov_grid), so kMaxRows rows need at most kMaxBlocks
// blocks; the single-system BiCGStab kernels publish at most 2 partials per
// block (publish_partials<2 * R>, R = 1).  The call also checks krylov_grid(n)
// against kMaxBlocks at run time.
constexpr int kMaxBlocks = (kMaxRows + MCB_THREADS - 1) / MCB_THREADS;
constexpr int kPartialsPerBlock = 8;
static_assert(MCB_THREADS == 256, "scratch partitioning assumes 256-thread Krylov blocks");
static_assert(kPartialsPerBlock >= 2, "BiCGStab with one right-hand side publishes 2 partials per block");
constexpr size_t kStatusDoubles = 64;             // counter (first 8 bytes) + BicgState<1>
constexpr size_t kScratchDoubles =
    (size_t)kVectors * kMaxRows + (size_t)kMaxBlocks * kPartialsPerBlock + kStatusDoubles;

static_assert(sizeof(mcb::BicgState<1>) + 8 <= kStatusDoubles * sizeof(double), "status block too small");

static __device__ __align__(256) double g_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double *g_scratch_addr[kMaxDevices] = {nullptr};

int scratch_for_current_device(double **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MC_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return MC_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) return MC_ERR_CUDA;
        g_scratch_addr[dev] = (double *)p;
    }
    *out = g_scratch_addr[dev];
    return MC_OK;
}

} // namespace

extern "C" int mc_solve_bicgstab_noalloc(int n, const double *diag, const double *off, const int *col,
                                         const double *b, double *x, double rtol, int max_iters, void *stream,
                                         int *iterations)
{
    if (n <= 0 || n > kMaxRows) return MC_ERR_ARG;  // larger systems need the handle-based solver
    if (!diag || !off || !col || !b || !x || !(rtol > 0.0) || max_iters <= 0) return MC_ERR_ARG;
    if (mcb::krylov_grid(n) > kMaxBlocks) return MC_ERR_UNSUPPORTED;  // partials would not fit
    double *base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc != MC_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;

    mcb::BicgVectors<1> v{};
    v.x[0] = x;
    v.b = b;
    v.r = base;
    v.r0 = base + (size_t)1 * kMaxRows;
    v.p[0] = base + (size_t)2 * kMaxRows;
    v.p[1] = base + (size_t)3 * kMaxRows;
    v.v[0] = base + (size_t)4 * kMaxRows;
    v.v[1] = base + (size_t)5 * kMaxRows;
    v.s = base + (size_t)6 * kMaxRows;
    v.t = base + (size_t)7 * kMaxRows;
    v.partials = base + (size_t)kVectors * kMaxRows;
    double *status = v.partials + (size_t)kMaxBlocks * kPartialsPerBlock;
    v.counter = (unsigned int *)status;
    v.st = (mcb::BicgState<1> *)(status + 1);

    // The counter must start at zero; a previous call leaves it at zero unless
    // it was interrupted, so clear it (and the status) every time.
    if (cudaMemsetAsync(status, 0, kStatusDoubles * sizeof(double), s) != cudaSuccess) return MC_ERR_CUDA;
    const mcb::Ell A{n, diag, off, col};
    mcb::bicg_init<1>(s, A, v, rtol, max_iters);
    if (cudaGetLastError() != cudaSuccess) return MC_ERR_CUDA;

    constexpr int kBatch = 8;  // iterations between status reads (even: ping-pong buffers)
    mcb::BicgState<1> hs{};
    const long max_batches = max_iters / kBatch + 2;
    for (long batch = 0;; batch++) {
        if (cudaMemcpyAsync(&hs, v.st, sizeof(hs), cudaMemcpyDeviceToHost, s) != cudaSuccess) return MC_ERR_CUDA;
        if (cudaStreamSynchronize(s) != cudaSuccess) return MC_ERR_CUDA;
        if (hs.all_done) break;
        if (batch > max_batches) return MC_ERR_NOT_CONVERGED;
        for (int it = 0; it < kBatch; it++) {
            const int pin = it & 1;
            mcb::bicg_1<1>(s, A, v, pin);
            mcb::bicg_2<1>(s, A, v, pin ^ 1);
            mcb::bicg_3<1>(s, A, v, pin ^ 1);
        }
        if (cudaGetLastError() != cudaSuccess) return MC_ERR_CUDA;
    }
    if (iterations) *iterations = hs.iter[0];
    if (hs.status[0] == mcb::KRYLOV_NONFINITE) return MC_ERR_NONFINITE;
    if (hs.status[0] != mcb::KRYLOV_OK) return MC_ERR_NOT_CONVERGED;
    return MC_OK;
}
