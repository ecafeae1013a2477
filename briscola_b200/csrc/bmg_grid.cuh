// bmg_grid.cuh -- how the cell kernels map their grids onto the bricks of
// a level (grid z walks the planes of brick 0, then brick 1, ...), block
// shapes, and the block reductions of the norm kernels.
#pragma once

#include "bmg_internal.h"

namespace bmg {

// brick of grid plane z and the plane index inside it
template <typename T>
__device__ __forceinline__ int brick_of(const Bricks<T>& B, int z, int& i) {
    int b = 0;
    while (b + 1 < B.nb && z >= B.z0[b + 1]) ++b;
    i = z - B.z0[b];
    return b;
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
    // NT threads in a block of any shape; the result is valid in thread 0
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31, warp = tid >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    v = 0.0;
    if (warp == 0) {
        v = lane < NT / 32 ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

constexpr int kFinalThreads = 1024;  // one-block kernels that add per-block partials

// sum of n per-block partials by one block of NT threads: four independent
// accumulators per thread keep many loads in flight; the assignment and the
// order are fixed, so the result is reproducible
template <int NT>
__device__ __forceinline__ double sum_partials(const double* __restrict__ p, long n, double* sh) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    long q = threadIdx.x;
    for (; q + 3 * NT < n; q += 4 * NT) {
        a0 += p[q];
        a1 += p[q + NT];
        a2 += p[q + 2 * NT];
        a3 += p[q + 3 * NT];
    }
    for (; q < n; q += NT) a0 += p[q];
    return block_sum<NT>((a0 + a1) + (a2 + a3), sh);
}

__device__ __forceinline__ long block_id() {
    return ((long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
}

inline dim3 block_for(int n2) {
    // k extent on lanes; small rows give the spare lanes to j
    if (n2 >= 64) return dim3(64, 4, 1);
    if (n2 >= 32) return dim3(32, 8, 1);
    if (n2 >= 16) return dim3(16, 16, 1);
    return dim3(8, 32, 1);
}

template <typename T>
inline dim3 grid_for(const Bricks<T>& B, int nk, dim3 blk) {
    return dim3((nk + blk.x - 1) / blk.x, (B.max1 + blk.y - 1) / blk.y, B.z0[B.nb]);
}

}  // namespace bmg
