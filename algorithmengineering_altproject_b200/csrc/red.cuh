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

// A block of one logical launch: its index and the launch's block count.  A plain launch passes
// (blockIdx.x, gridDim.x); a batched launch runs the logical launches of many instances as one persistent
// grid, each real block taking (instance, virtual block) items, and passes the item's index and its
// instance's block count, so every instance computes exactly what its own launch would.
struct VB {
    int b, n;
};
__device__ __forceinline__ VB vb_real() { return VB{(int)blockIdx.x, (int)gridDim.x}; }

// Publishes the block's partial; the last block to arrive folds all partials (threads stride over
// them in index order, then block_fold) and returns true with *total valid in warp 0.
// Resets the arrival counter for the next use of the slot.
__device__ __forceinline__ bool grid_fold(double v, RedSlot slot, double* sh, double* total, VB vb) {
    __shared__ int am_last;
    const double b = block_fold(v, sh);
    if (threadIdx.x == 0) {
        slot.partial[vb.b] = b;
        __threadfence();
        const unsigned int t = atomicAdd(slot.counter, 1u);
        am_last = (t == (unsigned)vb.n - 1u) ? 1 : 0;
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < vb.n; i += blockDim.x) s = s + __ldcg(slot.partial + i);
    *total = block_fold(s, sh);
    if (threadIdx.x == 0) *slot.counter = 0u;
    return true;
}
__device__ __forceinline__ bool grid_fold(double v, RedSlot slot, double* sh, double* total) {
    return grid_fold(v, slot, sh, total, vb_real());
}

// Instance of virtual block v in a batched launch: vstart[0..n] is the prefix sum of the instances' block
// counts (vstart[0] = 0).  Binary search; every thread of the block computes the same result.
__device__ __forceinline__ int batch_instance(const int* __restrict__ vstart, int n, int v) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(vstart + mid) <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// A persistent grid walks the (instance, logical block) list of the active instances (act, kernels.hpp):
// logical block v is block v - vs[k] of the k-th active instance, k = batch_instance(vs, n, v), in a launch of
// vs[k+1] - vs[k] blocks.  The body runs as in that instance's own launch; the barrier between items keeps
// shared scratch from being overwritten early.
template <class A, class F>
__device__ __forceinline__ void batch_walk(const A* __restrict__ a, const int* __restrict__ act, int N, F&& f) {
    const int n = __ldg(act);
    const int* __restrict__ pos = act + 1;
    const int* __restrict__ vs = act + 1 + N;
    const int total = __ldg(vs + n);
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
        const int k = batch_instance(vs, n, v);
        const int v0 = __ldg(vs + k);
        f(a[__ldg(pos + k)], VB{v - v0, __ldg(vs + k + 1) - v0});
        __syncthreads();
    }
}

}  // namespace t3d
