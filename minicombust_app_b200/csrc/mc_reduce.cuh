// Deterministic grid reductions without atomics on data: each block writes
// its partial sums, the last block to arrive (one atomicAdd on a counter, no
// waiting) reduces the partials in a fixed order and publishes the result.
// Block size is fixed at MCB_THREADS.
#pragma once

#include <cuda_runtime.h>

#define MCB_THREADS 256

namespace mcb {

// Sum of one value per thread across the block; result valid in thread 0.
template <int K>
__device__ inline void block_sum(double (&v)[K], double (*sh)[MCB_THREADS])
{
    __syncthreads();  // sh may still be read from a previous reduction
#pragma unroll
    for (int k = 0; k < K; k++) sh[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int s = MCB_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
#pragma unroll
            for (int k = 0; k < K; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = sh[k][0];
}

template <int K>
__device__ inline void block_max(double (&v)[K], double (*sh)[MCB_THREADS])
{
    __syncthreads();  // sh may still be read from a previous reduction
#pragma unroll
    for (int k = 0; k < K; k++) sh[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int s = MCB_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
#pragma unroll
            for (int k = 0; k < K; k++) sh[k][threadIdx.x] = fmax(sh[k][threadIdx.x], sh[k][threadIdx.x + s]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = sh[k][0];
}

// Reduce the threads' values across the block, publish the block's K
// partials and report whether this block is the last to arrive.
// partials: [gridDim.x][K]; counter must be zero before the launch and is
// reset by the last block.
template <int K, bool MAX = false>
__device__ inline bool publish_partials(const double (&v)[K], double *partials, unsigned int *counter,
                                        double (*sh)[MCB_THREADS])
{
    __shared__ bool am_last;
    double b[K];
#pragma unroll
    for (int k = 0; k < K; k++) b[k] = v[k];
    if (MAX)
        block_max<K>(b, sh);
    else
        block_sum<K>(b, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) partials[(size_t)blockIdx.x * K + k] = b[k];
        __threadfence();
        const unsigned int prev = atomicAdd(counter, 1u);
        am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    return am_last;
}

// In the last block: reduce the partials of all blocks (fixed order: thread
// t takes blocks t, t+256, ..., then a fixed tree).  Result in thread 0.
template <int K, bool MAX = false>
__device__ inline void reduce_partials(double (&out)[K], const double *partials, unsigned int *counter,
                                       double (*sh)[MCB_THREADS])
{
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = MAX ? -1.0e308 : 0.0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += MCB_THREADS) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            const double p = __ldcg(partials + (size_t)b * K + k);
            acc[k] = MAX ? fmax(acc[k], p) : acc[k] + p;
        }
    }
    if (MAX)
        block_max<K>(acc, sh);
    else
        block_sum<K>(acc, sh);
#pragma unroll
    for (int k = 0; k < K; k++) out[k] = acc[k];
    if (threadIdx.x == 0) *counter = 0u;
}

} // namespace mcb
