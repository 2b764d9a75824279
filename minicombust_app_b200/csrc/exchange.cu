// Flow/particle exchange kernels (exchange.cuh).  Built with -fmad=false so
// that the node interpolation evaluates the reference's expressions as
// written (FlowSolver.inl:428-494).
#include "exchange.cuh"

#include <algorithm>

namespace mcb {

namespace {

constexpr int kSortBlock = 1024;            // threads per sort block
constexpr int kSortTile = 2 * kSortBlock;   // keys per shared-memory tile

__global__ void __launch_bounds__(256) k_particle_keys(int n, int n2, const int *__restrict__ cells,
                                                       uint64_t *__restrict__ keys)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x)
        keys[i] = i < n ? (((uint64_t)(uint32_t)cells[i]) << 32) | (uint64_t)(uint32_t)i : ~0ull;
}

__device__ __forceinline__ void cmp_swap(uint64_t &a, uint64_t &b, bool up)
{
    if ((a > b) == up) {
        const uint64_t t = a;
        a = b;
        b = t;
    }
}

// Bitonic sort of each tile of kSortTile keys (all stages k <= kSortTile).
__global__ void __launch_bounds__(kSortBlock) k_sort_tiles(uint64_t *__restrict__ keys)
{
    __shared__ uint64_t sh[kSortTile];
    const size_t base = (size_t)blockIdx.x * kSortTile;
    sh[threadIdx.x] = keys[base + threadIdx.x];
    sh[threadIdx.x + kSortBlock] = keys[base + threadIdx.x + kSortBlock];
    __syncthreads();
    for (int k = 2; k <= kSortTile; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int t = threadIdx.x;
            const int i = 2 * j * (t / j) + (t % j);  // lower index of this thread's pair
            const bool up = (((base + i) & k) == 0);
            cmp_swap(sh[i], sh[i + j], up);
            __syncthreads();
        }
    }
    keys[base + threadIdx.x] = sh[threadIdx.x];
    keys[base + threadIdx.x + kSortBlock] = sh[threadIdx.x + kSortBlock];
}

// The steps j < kSortTile of merge stage k, inside each tile.
__global__ void __launch_bounds__(kSortBlock) k_merge_tiles(uint64_t *__restrict__ keys, int k)
{
    __shared__ uint64_t sh[kSortTile];
    const size_t base = (size_t)blockIdx.x * kSortTile;
    sh[threadIdx.x] = keys[base + threadIdx.x];
    sh[threadIdx.x + kSortBlock] = keys[base + threadIdx.x + kSortBlock];
    __syncthreads();
    for (int j = kSortTile >> 1; j > 0; j >>= 1) {
        const int t = threadIdx.x;
        const int i = 2 * j * (t / j) + (t % j);
        const bool up = (((base + i) & (size_t)k) == 0);
        cmp_swap(sh[i], sh[i + j], up);
        __syncthreads();
    }
    keys[base + threadIdx.x] = sh[threadIdx.x];
    keys[base + threadIdx.x + kSortBlock] = sh[threadIdx.x + kSortBlock];
}

// One step (k, j >= kSortTile) of the merge network across tiles.
__global__ void __launch_bounds__(256) k_merge_global(uint64_t *__restrict__ keys, int n2, int k, int j)
{
    const int half = n2 >> 1;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < half; t += gridDim.x * blockDim.x) {
        const int i = 2 * j * (t / j) + (t % j);
        const bool up = ((i & k) == 0);
        uint64_t a = keys[i], b = keys[i + j];
        if ((a > b) == up) {
            keys[i] = b;
            keys[i + j] = a;
        }
    }
}

// One thread per sorted position that starts a cell's run: the run's rows
// summed in order, starting from zero (the reference zeroes particle_terms
// and adds row by row, FlowSolver.inl:507, 699-704).
__global__ void __launch_bounds__(256) k_particle_sums(int n, const uint64_t *__restrict__ keys,
                                                       const double *__restrict__ rows, const int *__restrict__ o2n,
                                                       int N, double *__restrict__ src)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t cell = (uint32_t)(keys[i] >> 32);
        if (i > 0 && (uint32_t)(keys[i - 1] >> 32) == cell) continue;
        double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int j = i; j < n && (uint32_t)(keys[j] >> 32) == cell; j++) {
            const size_t r = (size_t)(uint32_t)(keys[j] & 0xffffffffu);
#pragma unroll
            for (int k = 0; k < 5; k++) s[k] += rows[5 * r + k];
        }
        const int c = o2n ? o2n[cell] : (int)cell;
#pragma unroll
        for (int k = 0; k < 5; k++) src[(size_t)k * N + c] = s[k];
    }
}

__global__ void __launch_bounds__(256) k_mark_nodes(int n, const int *__restrict__ req,
                                                    const int *__restrict__ cell_nodes, unsigned char *__restrict__ flag)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t c = (size_t)req[i];
#pragma unroll
        for (int v = 0; v < 8; v++) flag[cell_nodes[8 * c + v]] = 1;
    }
}

__global__ void __launch_bounds__(1024) k_count_flags(int P, const unsigned char *__restrict__ flag, int *counts)
{
    const int i = blockIdx.x * 1024 + threadIdx.x;
    const int f = (i < P && flag[i]) ? 1 : 0;
    const int c = __syncthreads_count(f);
    if (threadIdx.x == 0) counts[blockIdx.x] = c;
}

// Exclusive scan of the block counts in place (one block), total in *count.
__global__ void __launch_bounds__(1024) k_scan_counts(int nb, int *counts, int *count)
{
    __shared__ int sh[1024];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? counts[i] : 0;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            const int t = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < nb) counts[i] = carry + sh[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += sh[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = carry;
}

// Flagged node ids written in ascending order; the flags are cleared.
__global__ void __launch_bounds__(1024) k_scatter_flags(int P, unsigned char *__restrict__ flag,
                                                        const int *__restrict__ offsets, int *__restrict__ nodes)
{
    __shared__ int warp_base[32];
    const int i = blockIdx.x * 1024 + threadIdx.x;
    const bool f = i < P && flag[i];
    const unsigned ballot = __ballot_sync(0xffffffffu, f);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_base[warp] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int w = 0; w < 32; w++) {
            const int c = warp_base[w];
            warp_base[w] = acc;
            acc += c;
        }
    }
    __syncthreads();
    if (f) {
        nodes[offsets[blockIdx.x] + warp_base[warp] + __popc(ballot & ((1u << lane) - 1u))] = i;
        flag[i] = 0;
    }
}

// interpolate_to_nodes (FlowSolver.inl:428-494) for one node: the share of
// the reference gas state for the missing cells (get_neighbour_cells,
// :323-334), then each cell around the node, in ascending cell id.
__global__ void __launch_bounds__(256) k_node_values(int n, const int *__restrict__ nodes, NodeArgs a,
                                                     double *__restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int node = nodes[i];
        const int b = a.pc_off[node], e = a.pc_off[node + 1];
        const double node_neighbours = 8;
        const double boundary_neighbours = node_neighbours - (double)(e - b);
        const double share = boundary_neighbours / node_neighbours;
        double vx = a.u_ref * share, vy = 0.0 * share, vz = 0.0 * share;
        double pr = a.p_ref * share, te = a.t_ref * share;
        const double x = a.px[node], y = a.py[node], z = a.pz[node];
        for (int k = b; k < e; k++) {
            const int c = a.pc_cells[k];
            const double dx = x - a.xc[c], dy = y - a.yc[c], dz = z - a.zc[c];
            te += (a.T[c] + (a.gT[0][c] * dx + a.gT[1][c] * dy + a.gT[2][c] * dz)) / node_neighbours;
            pr += (a.P[c] + (a.gP[0][c] * dx + a.gP[1][c] * dy + a.gP[2][c] * dz)) / node_neighbours;
            vx += (a.U[c] + (a.gU[0][c] * dx + a.gU[1][c] * dy + a.gU[2][c] * dz)) / node_neighbours;
            vy += (a.V[c] + (a.gV[0][c] * dx + a.gV[1][c] * dy + a.gV[2][c] * dz)) / node_neighbours;
            vz += (a.W[c] + (a.gW[0][c] * dx + a.gW[1][c] * dy + a.gW[2][c] * dz)) / node_neighbours;
        }
        double *o = out + 5 * (size_t)i;
        o[0] = vx;
        o[1] = vy;
        o[2] = vz;
        o[3] = pr;
        o[4] = te;
    }
}

inline int grid_for(long n, int threads) { return (int)std::min<long>(4096, std::max<long>(1, (n + threads - 1) / threads)); }

} // namespace

void particle_keys(cudaStream_t s, int n, int n2, const int *cells, uint64_t *keys)
{
    k_particle_keys<<<grid_for(n2, 256), 256, 0, s>>>(n, n2, cells, keys);
}

void sort_keys(cudaStream_t s, uint64_t *keys, int n2)
{
    const int tiles = n2 / kSortTile;
    k_sort_tiles<<<tiles, kSortBlock, 0, s>>>(keys);
    for (int k = 2 * kSortTile; k <= n2; k <<= 1) {
        for (int j = k >> 1; j >= kSortTile; j >>= 1) k_merge_global<<<grid_for(n2 / 2, 256), 256, 0, s>>>(keys, n2, k, j);
        k_merge_tiles<<<tiles, kSortBlock, 0, s>>>(keys, k);
    }
}

void particle_sums(cudaStream_t s, int n, const uint64_t *keys, const double *rows, const int *o2n, int N, double *src)
{
    k_particle_sums<<<grid_for(n, 256), 256, 0, s>>>(n, keys, rows, o2n, N, src);
}

void mark_nodes(cudaStream_t s, int n_req, const int *req, const int *cell_nodes, unsigned char *flag)
{
    k_mark_nodes<<<grid_for(n_req, 256), 256, 0, s>>>(n_req, req, cell_nodes, flag);
}

void compact_nodes(cudaStream_t s, int P, unsigned char *flag, int *block_counts, int *nodes, int *count)
{
    const int nb = (P + 1023) / 1024;
    k_count_flags<<<nb, 1024, 0, s>>>(P, flag, block_counts);
    k_scan_counts<<<1, 1024, 0, s>>>(nb, block_counts, count);
    k_scatter_flags<<<nb, 1024, 0, s>>>(P, flag, block_counts, nodes);
}

void node_values(cudaStream_t s, int n, const int *nodes, const NodeArgs &a, double *out)
{
    k_node_values<<<grid_for(n, 256), 256, 0, s>>>(n, nodes, a, out);
}

} // namespace mcb
