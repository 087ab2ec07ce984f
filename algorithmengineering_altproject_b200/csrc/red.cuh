// Deterministic block / grid reductions in the canonical order described in t3d_common.cuh.
#pragma once
#include "t3d_common.cuh"

namespace t3d {

__device__ __forceinline__ double warp_fold(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

__device__ __forceinline__ float warp_fold_max(float v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, off));
    return v;
}

// Sum of one value per thread of the block; valid in every lane of warp 0.
// `sh` must hold 32 doubles.  Contains __syncthreads: call from all threads.
__device__ __forceinline__ double block_fold(double v, double* sh) {
    v = warp_fold(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = (l < (int)(blockDim.x >> 5)) ? sh[l] : 0.0;
        t = warp_fold(t);
    }
    __syncthreads();
    return t;
}

// Publishes the block's partial; the last block to arrive folds all partials (threads stride over
// them in index order, then block_fold) and returns true with *total valid in warp 0.
// Resets the arrival counter for the next use of the slot.
__device__ __forceinline__ bool grid_fold(double v, RedSlot slot, double* sh, double* total) {
    __shared__ int am_last;
    const double b = block_fold(v, sh);
    if (threadIdx.x == 0) {
        slot.partial[blockIdx.x] = b;
        __threadfence();
        const unsigned int t = atomicAdd(slot.counter, 1u);
        am_last = (t == gridDim.x - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s = s + __ldcg(slot.partial + i);
    *total = block_fold(s, sh);
    if (threadIdx.x == 0) *slot.counter = 0u;
    return true;
}

}  // namespace t3d
