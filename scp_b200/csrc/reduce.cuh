// reduce.cuh -- deterministic FP64 block reductions.
//
// Every reduction in the library is two-level with a fixed shape: each CTA of
// a fixed-size grid folds its grid-stride share of sites in a fixed order,
// then a warp-shuffle tree and a fixed cross-warp order produce one partial
// per CTA, and a single finishing CTA folds the partials in index order.  The
// result is bitwise reproducible from run to run and independent of timing
// (the reference GPU code uses atomicAdd on doubles, sfa/sim/scp_sim.cu:2051-2087,
// whose summation order varies between runs).
#pragma once
#include "common.cuh"

namespace scp {

constexpr int kRedThreads = 256;
constexpr int kRedMaxBlocks = 1184;   // 8 x 148 SMs

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Fold NS sums and NM maxima held per thread into one partial per CTA at
// part[blockIdx.x * (NS+NM) + q].  scratch: shared array of (NS+NM)*32 doubles.
template <int NS, int NM>
__device__ __forceinline__ void block_fold(const double (&sums)[NS > 0 ? NS : 1],
                                           const double (&maxs)[NM > 0 ? NM : 1],
                                           double *scratch, double *part) {
    constexpr int NQ = NS + NM;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NS; q++) {
        double v = warp_sum(sums[q]);
        if (lane == 0) scratch[q * 32 + wid] = v;
    }
#pragma unroll
    for (int q = 0; q < NM; q++) {
        double v = warp_max(maxs[q]);
        if (lane == 0) scratch[(NS + q) * 32 + wid] = v;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NQ; q += blockDim.x) {
        double acc = scratch[q * 32];
        for (int w = 1; w < nw; w++)
            acc = (q < NS) ? acc + scratch[q * 32 + w] : fmax(acc, scratch[q * 32 + w]);
        part[(size_t)blockIdx.x * NQ + q] = acc;
    }
    __syncthreads();
}

// One warp per slot folds nb partials in index order into out[q].
template <int NS, int NM>
__global__ void fold_partials_kernel(const double *part, int nb, double *out) {
    constexpr int NQ = NS + NM;
    const int lane = threadIdx.x & 31;
    for (int q = threadIdx.x >> 5; q < NQ; q += blockDim.x >> 5) {
        const bool is_max = q >= NS;
        double acc = is_max ? -INFINITY : 0.0;
        for (int b = lane; b < nb; b += 32) {
            const double v = part[(size_t)b * NQ + q];
            acc = is_max ? fmax(acc, v) : acc + v;
        }
        acc = is_max ? warp_max(acc) : warp_sum(acc);
        if (lane == 0) out[q] = acc;
    }
}

// The same fold as fold_partials_kernel, run by the last CTA of a grid to
// finish (threads of one CTA, one warp per slot): the result is bit for bit
// the one fold_partials_kernel gives.  part is read through L2 (__ldcg) since
// it was written by other CTAs during this launch.
template <int NS, int NM>
__device__ __forceinline__ void fold_partials_block(const double *part, int nb, double *out) {
    constexpr int NQ = NS + NM;
    const int lane = threadIdx.x & 31;
    for (int q = threadIdx.x >> 5; q < NQ; q += blockDim.x >> 5) {
        const bool is_max = q >= NS;
        double acc = is_max ? -INFINITY : 0.0;
        for (int b = lane; b < nb; b += 32) {
            const double v = __ldcg(part + (size_t)b * NQ + q);
            acc = is_max ? fmax(acc, v) : acc + v;
        }
        acc = is_max ? warp_max(acc) : warp_sum(acc);
        if (lane == 0) out[q] = acc;
    }
}

// After block_fold: true in exactly one CTA, the last to finish, once every
// CTA's partial is visible to it.  count is reset by that CTA for the next
// launch.  No CTA waits for another.
__device__ __forceinline__ bool last_block_done(unsigned *count) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(count, 1u);
        last = (t == gridDim.x - 1);
        if (last) *count = 0;
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

inline int red_blocks(long long n3) {
    long long b = (n3 + kRedThreads - 1) / kRedThreads;
    return (int)(b < kRedMaxBlocks ? (b < 1 ? 1 : b) : kRedMaxBlocks);
}

}  // namespace scp
