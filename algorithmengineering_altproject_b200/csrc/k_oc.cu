// Optimality-criteria update (driver.cpp:160-189): dc scaling, the lambda bisection with its volume
// sum, change and sharpness.  Two summation orders are provided:
//   fp64_sum = 1  canonical deterministic FP64 sums over cells (the throughput path);
//   fp64_sum = 0  the float summation order of the reference build's vectorised std::accumulate over
//                 the Morton-ordered element vector (8 lane sums, folded, remainder), which keeps the
//                 bisection bit-identical to the reference.
#include "kernels.hpp"
#include "red.cuh"

namespace t3d {

namespace {

// dc = dcf / max(1e-3, x) (driver.cpp:166)
__global__ void k_dc_scale(Grid g, const uint8_t* __restrict__ solid, const float* __restrict__ dcf,
                           const float* __restrict__ x, float* __restrict__ dc) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.NE || !solid[i]) return;
    const float xv = x[i];
    dc[i] = dcf[i] / (1.0e-3f < xv ? xv : 1.0e-3f);
}

__global__ void k_oc_init(OcState* st) {
    st->l1 = 0.0f;
    st->l2 = 1e9f;
    st->lmid = 0.0f;
    st->vol = 0.0f;
    st->passes = 0;
    st->done = 0;
}

// xnew = max(1e-3, clamp(clamp(x*sqrt(max(1e-30,-dc*(2/(l1+l2)))), x-0.2, x+0.2), 0, 1))
// (driver.cpp:174-180; -dc/lmid is evaluated as -dc*(2/(l1+l2)) as in the reference build)
__device__ __forceinline__ float oc_candidate(float xv, float d, float rl) {
    float q = -(d * rl);
    if (q < 1e-30f) q = 1e-30f;
    const float val = sqrtf(q);
    const float lo = xv - 0.2f, hi = xv + 0.2f;
    float xe = xv * val;
    xe = xe < lo ? lo : (hi < xe ? hi : xe);
    xe = xe < 0.0f ? 0.0f : (1.0f < xe ? 1.0f : xe);
    return 1.0e-3f < xe ? xe : 1.0e-3f;
}

__device__ __forceinline__ bool oc_continue(const OcState* st) {
    const float l1 = st->l1, l2 = st->l2;
    return (double)((l2 - l1) / (l1 + l2)) > 1e-6;
}

__global__ void __launch_bounds__(RED_THREADS) k_oc_pass(Grid g, const uint8_t* __restrict__ solid,
                                                         const float* __restrict__ x, const float* __restrict__ dc,
                                                         float* __restrict__ xnew, OcState* st, int fp64_sum,
                                                         float V0, int64_t ne, RedSlot red) {
    __shared__ double sh[32];
    if (st->done) return;
    if (!oc_continue(st)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->done = 1;
        return;
    }
    const float l1 = st->l1, l2 = st->l2;
    const float lmid = 0.5f * (l1 + l2);
    const float rl = 2.0f / (l1 + l2);
    const int ncell = g.nx * g.ny * g.nz;
    double part = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ncell; k += gridDim.x * blockDim.x) {
        const int cx = k % g.nx, cy = (k / g.nx) % g.ny, cz = k / (g.nx * g.ny);
        const int64_t ci = g.cell(cx, cy, cz);
        const uint8_t sc = solid[ci];
        if (!sc) continue;
        // passive solid elements of an external model (solid = 2) stay at 1 (TOP3D_XL.m:152,166)
        const float xn = sc == 2 ? 1.0f : oc_candidate(x[ci], dc[ci], rl);
        xnew[ci] = xn;
        part = part + (double)xn;
    }
    if (!fp64_sum) return;
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) {
        const float vol = (float)tot / (float)ne;
        st->vol = vol;
        st->lmid = lmid;
        if (vol - V0 > 0) st->l1 = lmid;
        else st->l2 = lmid;
        st->passes = st->passes + 1;
    }
}

// Reference-build float sum of t over the Morton-ordered elements (see the oracle's vec8_sum):
// 8 lane sums over 8*floor(n/8) values, folded ((l0+l4)+(l2+l6)) + ((l1+l5)+(l3+l7)); 4..7 remaining
// values added lane-wise to (l0+l4, ..) and folded (m1+m3)+(m0+m2); last 0..3 added in sequence.
// Run by one warp: lanes 0..7 own the lane sums.
template <class T>
__device__ float vec8_sum_warp(int64_t n, const int32_t* __restrict__ perm, T value) {
    const int lane = threadIdx.x & 31;
    const int64_t nb = n >= 8 ? n / 8 : 0;
    float l = 0.0f;
    if (lane < 8) {
        int64_t b = 0;
        for (; b + 4 <= nb; b += 4) {
            const float v0 = value(perm[8 * b + lane]);
            const float v1 = value(perm[8 * (b + 1) + lane]);
            const float v2 = value(perm[8 * (b + 2) + lane]);
            const float v3 = value(perm[8 * (b + 3) + lane]);
            l = l + v0;
            l = l + v1;
            l = l + v2;
            l = l + v3;
        }
        for (; b < nb; ++b) l = l + value(perm[8 * b + lane]);
    }
    // h_j = l_{j+4} + l_j for j < 4
    const float up = __shfl_down_sync(0xffffffffu, l, 4);
    float h = (lane < 4) ? (nb > 0 ? up + l : 0.0f) : 0.0f;
    const float h0 = __shfl_sync(0xffffffffu, h, 0), h1 = __shfl_sync(0xffffffffu, h, 1);
    const float h2 = __shfl_sync(0xffffffffu, h, 2), h3 = __shfl_sync(0xffffffffu, h, 3);
    float s = nb > 0 ? (h1 + h3) + (h0 + h2) : 0.0f;
    int64_t i = 8 * nb;
    if (n - i >= 4) {
        const float m0 = h0 + value(perm[i]), m1 = h1 + value(perm[i + 1]);
        const float m2 = h2 + value(perm[i + 2]), m3 = h3 + value(perm[i + 3]);
        s = (m1 + m3) + (m0 + m2);
        i += 4;
    }
    for (; i < n; ++i) s = s + value(perm[i]);
    return s;
}

__global__ void k_oc_vec8_vol(int64_t ne, const int32_t* __restrict__ perm, const float* __restrict__ xnew,
                              OcState* st, float V0) {
    if (st->done) return;
    const float l1 = st->l1, l2 = st->l2;
    const float lmid = 0.5f * (l1 + l2);
    const float s = vec8_sum_warp(ne, perm, [&](int32_t c) { return xnew[c]; });
    if (threadIdx.x == 0) {
        const float vol = s * (1.0f / (float)ne);
        st->vol = vol;
        st->lmid = lmid;
        if (vol - V0 > 0) st->l1 = lmid;
        else st->l2 = lmid;
        st->passes = st->passes + 1;
    }
}

__global__ void k_oc_vec8_stats(int64_t ne, const int32_t* __restrict__ perm, const float* __restrict__ x,
                                OcState* st) {
    const float sv = vec8_sum_warp(ne, perm, [&](int32_t c) { return x[c]; });
    const float sp = vec8_sum_warp(ne, perm, [&](int32_t c) { const float v = x[c]; return v * (1.0f - v); });
    if (threadIdx.x == 0) {
        st->volfrac = sv / (float)ne;
        st->sharp = 4.0f * sp / (float)ne;
    }
}

// change = max|xnew-x| (order-free), x = xnew; FP64 sums of x and x(1-x) for the fp64 path
__global__ void __launch_bounds__(RED_THREADS) k_oc_finish(Grid g, const uint8_t* __restrict__ solid,
                                                           float* __restrict__ x, const float* __restrict__ xnew,
                                                           OcState* st, int fp64_sum, int64_t ne, RedSlot r1,
                                                           RedSlot r2) {
    __shared__ double sh[32];
    __shared__ float shm[32];
    const int ncell = g.nx * g.ny * g.nz;
    float ch = 0.0f;
    double sv = 0.0, sp = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ncell; k += gridDim.x * blockDim.x) {
        const int cx = k % g.nx, cy = (k / g.nx) % g.ny, cz = k / (g.nx * g.ny);
        const int64_t ci = g.cell(cx, cy, cz);
        if (!solid[ci]) continue;
        const float xn = xnew[ci];
        ch = fmaxf(ch, fabsf(xn - x[ci]));
        x[ci] = xn;
        sv = sv + (double)xn;
        sp = sp + (double)(xn * (1.0f - xn));
    }
    // max-reduction: order does not matter; non-negative floats compare as their bit patterns
    ch = warp_fold_max(ch);
    if ((threadIdx.x & 31) == 0) shm[threadIdx.x >> 5] = ch;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, shm[w]);
        atomicMax(reinterpret_cast<int*>(&st->change), __float_as_int(m));
    }
    if (!fp64_sum) return;
    double tv, tp;
    if (grid_fold(sv, r1, sh, &tv) && threadIdx.x == 0) st->volfrac = (float)tv / (float)ne;
    __syncthreads();
    if (grid_fold(sp, r2, sh, &tp) && threadIdx.x == 0) st->sharp = 4.0f * (float)tp / (float)ne;
}

__global__ void k_oc_reset_change(OcState* st) { st->change = 0.0f; }

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void launch_dc_scale(const Grid& g, const uint8_t* solid, const float* dcf, const float* x, float* dc,
                     cudaStream_t s) {
    k_dc_scale<<<blocks_for(g.NE, 256), 256, 0, s>>>(g, solid, dcf, x, dc);
}
void launch_oc_init(OcState* st, cudaStream_t s) { k_oc_init<<<1, 1, 0, s>>>(st); }
void launch_oc_pass(const Grid& g, const uint8_t* solid, const float* x, const float* dc, float* xnew, OcState* st,
                    int fp64_sum, float V0, int64_t ne, RedSlot red, cudaStream_t s) {
    k_oc_pass<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, solid, x, dc, xnew, st, fp64_sum, V0, ne, red);
}
void launch_oc_vec8_vol(int64_t ne, const int32_t* morton_cells, const float* xnew, OcState* st, float V0,
                        cudaStream_t s) {
    k_oc_vec8_vol<<<1, 32, 0, s>>>(ne, morton_cells, xnew, st, V0);
}
void launch_oc_finish(const Grid& g, const uint8_t* solid, float* x, const float* xnew, OcState* st, int fp64_sum,
                      int64_t ne, RedSlot r1, RedSlot r2, cudaStream_t s) {
    k_oc_reset_change<<<1, 1, 0, s>>>(st);
    k_oc_finish<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, solid, x, xnew, st, fp64_sum, ne, r1, r2);
}
void launch_oc_vec8_stats(int64_t ne, const int32_t* morton_cells, const float* x, OcState* st, cudaStream_t s) {
    k_oc_vec8_stats<<<1, 32, 0, s>>>(ne, morton_cells, x, st);
}

}  // namespace t3d
