// Mixed-precision solve: FP32 storage and arithmetic for the inner MG-preconditioned PCG (matvec,
// smoother, transfers, vector updates) inside an FP64 defect-correction loop.  FP64 is kept for the
// inner products and alpha/beta (device scalars), the true-residual recompute b - K64 u64 (the FP64
// matvec), the coarsest-level factor and solve, and the accumulation u64 += d32.  Same algorithm as
// the FP64 path (solver.cpp:87-217, preconditioner.cpp:88-265); only the storage precision differs.
#include <algorithm>

#include "kernels.hpp"
#include "red.cuh"

namespace t3d {

namespace {

__device__ __forceinline__ void node_ijk(const Grid& g, int n, int& ix, int& iy, int& iz) {
    ix = n % g.nnx;
    const int t = n / g.nnx;
    iy = t % g.nny;
    iz = t / g.nny;
}

__device__ __forceinline__ float hatf(int i, int s) {   // 1 - |i-(s-1)|/s, exact in binary for s = 2, 4
    return 1.0f - fabsf((float)(i - (s - 1))) * (1.0f / s);
}

// Row remaps between the unpadded FP64 layouts and the pitched FP32 images: `rows` rows of `len` values
// at pitch `sp` in the source and `dp` in the destination.  Pads of an FP32 destination are written zero.
template <class A, class B>
__global__ void k_rows_convert(int64_t rows, int len, int sp, int dp, const A* __restrict__ a, B* __restrict__ b) {
    const int w = dp > len ? dp : len;   // FP32 destinations cover their pads
    const int64_t total = rows * w;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / w;
        const int i = (int)(t - row * w);
        if (i < len) b[row * dp + i] = (B)a[row * sp + i];
        else if (i < dp) b[row * dp + i] = (B)0;
    }
}

// FP32 image of a level diagonal as the reciprocal 1 / max(1e-30, D) used by the FP32 smoother
__global__ void k_recip_diag32(int64_t rows, int len, int pitch, const double* __restrict__ d, float* __restrict__ rd) {
    const int64_t total = rows * pitch;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / pitch;
        const int i = (int)(t - row * pitch);
        const double v = i < len ? d[row * len + i] : 1.0;
        rd[t] = i < len ? (float)(1.0 / (1.0e-30 < v ? v : 1.0e-30)) : 0.0f;
    }
}

// r64 = b - A u64; r32 = (float)r64 (pitched, pads zero); d32 = 0; |r64|^2 into *rn2 (FP64)
__global__ void __launch_bounds__(RED_THREADS) k_mixed_residual(Grid g, const double* __restrict__ b,
                                                                const double* __restrict__ Au,
                                                                float* __restrict__ r32, float* __restrict__ d32,
                                                                RedSlot red, double* __restrict__ rn2) {
    __shared__ double sh[32];
    const int64_t total = 3 * g.NNp;
    double part = 0.0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / g.px;
        const int i = (int)(t - row * g.px);
        float rv32 = 0.0f;
        if (i < g.nnx) {
            const int64_t k = row * g.nnx + i;
            const double rv = b[k] - Au[k];
            rv32 = (float)rv;
            part = fma(rv, rv, part);
        }
        r32[t] = rv32;
        d32[t] = 0.0f;
    }
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) *rn2 = tot;
}

// u64 += d32 (d32 pitched)
__global__ void k_mixed_accumulate(Grid g, double* __restrict__ u, const float* __restrict__ d) {
    const int64_t total = 3 * g.NN;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = k / g.nnx;
        const int i = (int)(k - row * g.nnx);
        u[k] = u[k] + (double)d[row * g.px + i];
    }
}

// ---------------------------------------------------------------- K(E) p in FP32
// Node-centric gather in the colour order of the FP64 kernel; Ke rows read from shared memory as
// float4; FP32 FMA chains; p.Ap folded in FP64.
__global__ void __launch_bounds__(RED_THREADS) k_matvec32(Grid g, const float* __restrict__ Keg,
                                                          const float* __restrict__ E,
                                                          const uint8_t* __restrict__ mask,
                                                          const float* __restrict__ u, float* __restrict__ y,
                                                          RedSlot dot, PcgScalars* S, int mark) {
    __shared__ __align__(16) float Ke[576];
    __shared__ double sh[32];
    if (S != nullptr && mark && blockIdx.x == 0 && threadIdx.x == 0) S->xit = S->it;   // the PCG product
    if (S != nullptr && S->done) return;
    for (int i = threadIdx.x; i < 576; i += blockDim.x) Ke[i] = Keg[i];
    __syncthreads();
    const int NN = (int)g.NN, NP = (int)g.NNp;
    const float* __restrict__ u0 = u;
    const float* __restrict__ u1 = u + NP;
    const float* __restrict__ u2 = u + 2 * (int64_t)NP;
    double part = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x) {
        int ix, iy, iz;
        node_ijk(g, n, ix, iy, iz);
        const int np = (int)g.pnode(ix, iy, iz);
        float y0 = 0.0f, y1 = 0.0f, y2 = 0.0f;
#pragma unroll 1
        for (int col = 0; col < 8; ++col) {
            const int cx = (((ix - 1) & 1) == (col & 1)) ? ix - 1 : ix;
            const int cy = (((g.ny - iy) & 1) == ((col >> 1) & 1)) ? iy - 1 : iy;
            const int cz = (((iz - 1) & 1) == ((col >> 2) & 1)) ? iz - 1 : iz;
            const float Ee = E[g.pcell(cx, cy, cz)];
            if (Ee <= 1.0e-16f) continue;
            const int a = corner_of(ix - cx, iy - cy, iz - cz);
            float ue[24];
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const int m = (int)g.pnode(cx + corner_dx(b), cy + corner_dy(b), cz + corner_dz(b));
                ue[3 * b + 0] = u0[m];
                ue[3 * b + 1] = u1[m];
                ue[3 * b + 2] = u2[m];
            }
            const float4* K0 = reinterpret_cast<const float4*>(Ke + (3 * a) * 24);
            float f0 = 0.0f, f1 = 0.0f, f2 = 0.0f;
#pragma unroll
            for (int j = 0; j < 24; j += 4) {
                const float4 k0 = K0[j / 4], k1 = K0[6 + j / 4], k2 = K0[12 + j / 4];
                f0 = fmaf(k0.x, ue[j], f0); f0 = fmaf(k0.y, ue[j + 1], f0);
                f0 = fmaf(k0.z, ue[j + 2], f0); f0 = fmaf(k0.w, ue[j + 3], f0);
                f1 = fmaf(k1.x, ue[j], f1); f1 = fmaf(k1.y, ue[j + 1], f1);
                f1 = fmaf(k1.z, ue[j + 2], f1); f1 = fmaf(k1.w, ue[j + 3], f1);
                f2 = fmaf(k2.x, ue[j], f2); f2 = fmaf(k2.y, ue[j + 1], f2);
                f2 = fmaf(k2.z, ue[j + 2], f2); f2 = fmaf(k2.w, ue[j + 3], f2);
            }
            y0 = fmaf(f0, Ee, y0);
            y1 = fmaf(f1, Ee, y1);
            y2 = fmaf(f2, Ee, y2);
        }
        const int mk = mask[n];
        if (mk & 1) y0 = 0.0f;
        if (mk & 2) y1 = 0.0f;
        if (mk & 4) y2 = 0.0f;
        y[np] = y0;
        y[NP + np] = y1;
        y[2 * (int64_t)NP + np] = y2;
        if (dot.partial) {
            part = fma((double)u0[np], (double)y0, part);
            part = fma((double)u1[np], (double)y1, part);
            part = fma((double)u2[np], (double)y2, part);
        }
    }
    if (dot.partial) {
        double tot;
        if (grid_fold(part, dot, sh, &tot) && threadIdx.x == 0) S->denom = tot;
    }
}

// ---------------------------------------------------------------- V-cycle in FP32
// Kernel bodies take the logical block (VB) so that the batched launches below run them unchanged.
__device__ __forceinline__ void restrict_x32(VB vb, const MgLevel32& Lc, const MgLevel32& Lf,
                                             const float* __restrict__ rf, float* __restrict__ a1,
                                             const PcgScalars* S) {
    if (S->done) return;
    const int cnx = Lc.nx + 1, fnx = Lf.nx + 1, fny = Lf.ny + 1, fnz = Lf.nz + 1;
    const int64_t total = (int64_t)fnz * fny * cnx;
    const int64_t t = (int64_t)vb.b * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int cx = (int)(t % cnx);
    const int64_t row = t / cnx;
    const int s = Lc.span, ws = 2 * s - 1;
    const int64_t fNN = Lf.cs;
    const float* __restrict__ src = rf + row * Lf.pitch;
    float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
    for (int ix = 0; ix < ws; ++ix) {
        const int fx = cx * s + ix - (s - 1);
        if (fx < 0 || fx >= fnx) continue;
        const float w = hatf(ix, s);
        v0 = fmaf(w, src[fx], v0);
        v1 = fmaf(w, src[fNN + fx], v1);
        v2 = fmaf(w, src[2 * fNN + fx], v2);
    }
    a1[t] = v0;
    a1[total + t] = v1;
    a1[2 * total + t] = v2;
}
__global__ void k_restrict_x32(MgLevel32 Lc, MgLevel32 Lf, const float* __restrict__ rf, float* __restrict__ a1,
                               const PcgScalars* S) {
    restrict_x32(vb_real(), Lc, Lf, rf, a1, S);
}

// Sum of the in-range hat weights of the window of coarse index c (span SP) over n fine points.
template <int SP>
__device__ __forceinline__ float hat_sum(int c, int n) {
    float sw = 0.0f;
#pragma unroll
    for (int i = 0; i < 2 * SP - 1; ++i) {
        const int f = c * SP + i - (SP - 1);
        if (f >= 0 && f < n) sw += hatf(i, SP);
    }
    return sw;
}

// y and z window sums of the x-pass result a1[fz][fy][cx] in one pass, normalised by the summed in-range
// weights and masked (the k_restrict_y32 + k_restrict_z32 pair fused; one thread per coarse node).
template <int SP>
__device__ __forceinline__ void restrict_yz32(VB vb, const MgLevel32& Lc, const MgLevel32& Lf,
                                              const float* __restrict__ a1, float* __restrict__ rc,
                                              const PcgScalars* S, int normalize) {
    if (S->done) return;
    constexpr int WS = 2 * SP - 1;
    const int n = vb.b * blockDim.x + threadIdx.x;
    if (n >= Lc.nn) return;
    const int cnx = Lc.nx + 1, cny = Lc.ny + 1;
    const int fnx = Lf.nx + 1, fny = Lf.ny + 1, fnz = Lf.nz + 1;
    const int cx = n % cnx, cy = (n / cnx) % cny, cz = n / (cnx * cny);
    const int total1 = fnz * fny * cnx;
    float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
#pragma unroll
    for (int iz = 0; iz < WS; ++iz) {
        const int fz = cz * SP + iz - (SP - 1);
        if (fz < 0 || fz >= fnz) continue;
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
#pragma unroll
        for (int iy = 0; iy < WS; ++iy) {
            const int fy = cy * SP + iy - (SP - 1);
            if (fy < 0 || fy >= fny) continue;
            const float w = hatf(iy, SP);
            const int i = (fz * fny + fy) * cnx + cx;
            s0 = fmaf(w, a1[i], s0);
            s1 = fmaf(w, a1[total1 + i], s1);
            s2 = fmaf(w, a1[2 * total1 + i], s2);
        }
        const float w = hatf(iz, SP);
        v0 = fmaf(w, s0, v0);
        v1 = fmaf(w, s1, v1);
        v2 = fmaf(w, s2, v2);
    }
    // normalised average (transfers.cpp:520-528) or, for the Standard cycle, the transposed prolongation
    const float iw = normalize ? 1.0f / (hat_sum<SP>(cz, fnz) * hat_sum<SP>(cy, fny) * hat_sum<SP>(cx, fnx)) : 1.0f;
    const int m = Lc.mask[n];
    rc[n] = (m & 1) ? 0.0f : v0 * iw;
    rc[Lc.nn + n] = (m & 2) ? 0.0f : v1 * iw;
    rc[2 * Lc.nn + n] = (m & 4) ? 0.0f : v2 * iw;
}
template <int SP>
__global__ void __launch_bounds__(256) k_restrict_yz32(MgLevel32 Lc, MgLevel32 Lf, const float* __restrict__ a1,
                                                       float* __restrict__ rc, const PcgScalars* S, int normalize) {
    restrict_yz32<SP>(vb_real(), Lc, Lf, a1, rc, S, normalize);
}

// The whole 3D window of the fine residual in one pass (levels small enough to sit in L2).
template <int SP>
__device__ __forceinline__ void restrict_xyz32(VB vb, const MgLevel32& Lc, const MgLevel32& Lf,
                                               const float* __restrict__ rf, float* __restrict__ rc,
                                               const PcgScalars* S, int normalize) {
    if (S->done) return;
    constexpr int WS = 2 * SP - 1;
    const int n = vb.b * blockDim.x + threadIdx.x;
    if (n >= Lc.nn) return;
    const int cnx = Lc.nx + 1, cny = Lc.ny + 1;
    const int fnx = Lf.nx + 1, fny = Lf.ny + 1, fnz = Lf.nz + 1;
    const int cx = n % cnx, cy = (n / cnx) % cny, cz = n / (cnx * cny);
    const int fNN = (int)Lf.cs;
    float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
#pragma unroll
    for (int iz = 0; iz < WS; ++iz) {
        const int fz = cz * SP + iz - (SP - 1);
        if (fz < 0 || fz >= fnz) continue;
        float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f;
#pragma unroll
        for (int iy = 0; iy < WS; ++iy) {
            const int fy = cy * SP + iy - (SP - 1);
            if (fy < 0 || fy >= fny) continue;
            const float* __restrict__ src = rf + (fz * fny + fy) * Lf.pitch;
            float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
#pragma unroll
            for (int ix = 0; ix < WS; ++ix) {
                const int fx = cx * SP + ix - (SP - 1);
                if (fx < 0 || fx >= fnx) continue;
                const float w = hatf(ix, SP);
                s0 = fmaf(w, src[fx], s0);
                s1 = fmaf(w, src[fNN + fx], s1);
                s2 = fmaf(w, src[2 * fNN + fx], s2);
            }
            const float w = hatf(iy, SP);
            t0 = fmaf(w, s0, t0);
            t1 = fmaf(w, s1, t1);
            t2 = fmaf(w, s2, t2);
        }
        const float w = hatf(iz, SP);
        v0 = fmaf(w, t0, v0);
        v1 = fmaf(w, t1, v1);
        v2 = fmaf(w, t2, v2);
    }
    // normalised average (transfers.cpp:520-528) or, for the Standard cycle, the transposed prolongation
    const float iw = normalize ? 1.0f / (hat_sum<SP>(cz, fnz) * hat_sum<SP>(cy, fny) * hat_sum<SP>(cx, fnx)) : 1.0f;
    const int m = Lc.mask[n];
    rc[n] = (m & 1) ? 0.0f : v0 * iw;
    rc[Lc.nn + n] = (m & 2) ? 0.0f : v1 * iw;
    rc[2 * Lc.nn + n] = (m & 4) ? 0.0f : v2 * iw;
}
template <int SP>
__global__ void __launch_bounds__(256) k_restrict_xyz32(MgLevel32 Lc, MgLevel32 Lf, const float* __restrict__ rf,
                                                        float* __restrict__ rc, const PcgScalars* S, int normalize) {
    restrict_xyz32<SP>(vb_real(), Lc, Lf, rf, rc, S, normalize);
}

// Trilinear prolongation at fine node (fx,fy,fz) from the coarse cell fx >> sh (span 1 << sh), clamped to the
// last coarse cell (transfers.cpp:396-408).
__device__ __forceinline__ void prolong_node32(const MgLevel32& Lc, const float* __restrict__ xc, int fx, int fy,
                                               int fz, int sh, float P[3]) {
    const int s = 1 << sh;
    const int cny = Lc.ny + 1;
    int cx = fx >> sh, cy = fy >> sh, cz = fz >> sh;
    int rx = fx & (s - 1), ry = fy & (s - 1), rz = fz & (s - 1);
    if (cx >= Lc.nx) { cx = Lc.nx - 1; rx = s; }
    if (cy >= Lc.ny) { cy = Lc.ny - 1; ry = s; }
    if (cz >= Lc.nz) { cz = Lc.nz - 1; rz = s; }
    const float inv = 1.0f / (float)s;   // exact: s is a power of two
    const float wx1 = rx * inv, wx0 = 1.0f - wx1;
    const float wy1 = ry * inv, wy0 = 1.0f - wy1;
    const float wz1 = rz * inv, wz0 = 1.0f - wz1;
    const int b = (cz * cny + cy) * Lc.pitch + cx;
    const int pz = Lc.pitch * cny;
    const int cnx_ = Lc.pitch;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float* X = xc + c * Lc.cs;
        const float lo = fmaf(wy1, fmaf(wx1, X[b + cnx_ + 1], wx0 * X[b + cnx_]), wy0 * fmaf(wx1, X[b + 1], wx0 * X[b]));
        const float hi = fmaf(wy1, fmaf(wx1, X[b + pz + cnx_ + 1], wx0 * X[b + pz + cnx_]),
                              wy0 * fmaf(wx1, X[b + pz + 1], wx0 * X[b + pz]));
        P[c] = fmaf(wz1, hi, wz0 * lo);
    }
}

__device__ __forceinline__ void prolong_smooth32(VB vb, const MgLevel32& Lc, const MgLevel32& Lf,
                                                 const float* __restrict__ xc, const float* __restrict__ rf,
                                                 float* __restrict__ xf, float w, const PcgScalars* S) {
    if (S->done) return;
    const int n = vb.b * blockDim.x + threadIdx.x;
    if (n >= Lf.nn) return;
    const int fnx = Lf.nx + 1, fny = Lf.ny + 1;
    const int fx = n % fnx, fy = (n / fnx) % fny, fz = n / (fnx * fny);
    float P[3];
    prolong_node32(Lc, xc, fx, fy, fz, __ffs(Lc.span) - 1, P);
    const int m = Lf.mask[n];
    const int64_t np = (int64_t)(n / fnx) * Lf.pitch + fx;
    for (int c = 0; c < 3; ++c) {
        const float t = (w * rf[c * Lf.cs + np]) * Lf.diag[c * Lf.cs + np];
        xf[c * Lf.cs + np] = ((m >> c) & 1) ? 0.0f : (t + P[c]) + t;
    }
}
__global__ void k_prolong_smooth32(MgLevel32 Lc, MgLevel32 Lf, const float* __restrict__ xc,
                                   const float* __restrict__ rf, float* __restrict__ xf, float w,
                                   const PcgScalars* S) {
    prolong_smooth32(vb_real(), Lc, Lf, xc, rf, xf, w, S);
}

// Finest-level prolongation + smoothing + r.z.  Each lane takes a run of SP consecutive fine nodes of one
// row that share one coarse cell in x (fine x = SP * j + k): the 8 coarse corners are gathered once and
// interpolated in y and z once per run; each node then only interpolates in x.  The last node of a row
// (fine x = nx, clamped to the last coarse cell with weight 1) is its own run.
template <int SP>
__device__ __forceinline__ void prolong_smooth0_32(VB vb, const MgLevel32& Lc, const MgLevel32& Lf,
                                                   const float* __restrict__ xc, const float* __restrict__ r,
                                                   float* __restrict__ z, float w, RedSlot dot, PcgScalars* S,
                                                   double* sh) {
    if (S->done) return;
    const int CS = (int)Lf.cs;
    const int fnx = Lf.nx + 1, fny = Lf.ny + 1;
    const int cnx = Lc.pitch, cny = Lc.ny + 1, cnn = (int)Lc.cs;
    const int runs = Lf.nx / SP + 1;                 // runs per row (the last one is the single node x = nx)
    const int chunks = (runs + 31) >> 5;
    const int items = chunks * fny * (Lf.nz + 1);
    const int lane = threadIdx.x & 31;
    const int nw = (vb.n * blockDim.x) >> 5;
    constexpr float inv = 1.0f / (float)SP;          // exact: SP is a power of two
    double part = 0.0;
    for (int it = (vb.b * blockDim.x + threadIdx.x) >> 5; it < items; it += nw) {
        const int row = it / chunks;
        const int j = (it - row * chunks) * 32 + lane;
        if (j >= runs) continue;
        const int fz = row / fny, fy = row - fz * fny;
        int cx = j, cy = fy / SP, cz = fz / SP;
        int ry = fy - cy * SP, rz = fz - cz * SP;
        const bool last = cx >= Lc.nx;               // fine x = nx: weight 1 on the last coarse node
        if (last) cx = Lc.nx - 1;
        if (cy >= Lc.ny) { cy = Lc.ny - 1; ry = SP; }
        if (cz >= Lc.nz) { cz = Lc.nz - 1; rz = SP; }
        const float wy1 = ry * inv, wy0 = 1.0f - wy1, wz1 = rz * inv, wz0 = 1.0f - wz1;
        const int b = (cz * cny + cy) * cnx + cx, pz = cnx * cny;
        float L[3], R[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float* X = xc + c * cnn;
            const float x00 = X[b], x10 = X[b + 1], x01 = X[b + cnx], x11 = X[b + cnx + 1];
            const float y00 = X[b + pz], y10 = X[b + pz + 1], y01 = X[b + pz + cnx], y11 = X[b + pz + cnx + 1];
            L[c] = fmaf(wz1, fmaf(wy1, y01, wy0 * y00), wz0 * fmaf(wy1, x01, wy0 * x00));
            R[c] = fmaf(wz1, fmaf(wy1, y11, wy0 * y10), wz0 * fmaf(wy1, x11, wy0 * x10));
        }
        const int nb = row * fnx + SP * j, npb = row * Lf.pitch + SP * j;
        const int nk = last ? 1 : SP;
#pragma unroll
        for (int k = 0; k < SP; ++k) {
            if (k >= nk) break;
            const int n = nb + k, np = npb + k;
            const float wx1 = last ? 1.0f : k * inv, wx0 = 1.0f - wx1;
            const int m = Lf.mask[n];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float rv = r[c * CS + np];
                const float t = (w * rv) * Lf.diag[c * CS + np];
                const float P = fmaf(wx1, R[c], wx0 * L[c]);
                const float zv = ((m >> c) & 1) ? 0.0f : (t + P) + t;
                z[c * CS + np] = zv;
                part = fma((double)rv, (double)zv, part);
            }
        }
    }
    double tot;
    if (grid_fold(part, dot, sh, &tot, vb) && threadIdx.x == 0) {
        if (S->first) {
            S->rz = tot;
            S->first = 0;
        } else {
            const double rz = S->rz;
            S->beta = tot / (1.0e-30 < rz ? rz : 1.0e-30);
            S->rz = tot;
        }
    }
}
template <int SP>
__global__ void __launch_bounds__(RED_THREADS) k_prolong_smooth0_32(MgLevel32 Lc, MgLevel32 Lf,
                                                                    const float* __restrict__ xc,
                                                                    const float* __restrict__ r,
                                                                    float* __restrict__ z, float w, RedSlot dot,
                                                                    PcgScalars* S) {
    __shared__ double sh[32];
    prolong_smooth0_32<SP>(vb_real(), Lc, Lf, xc, r, z, w, dot, S, sh);
}

// coarsest level: FP64 inverse applied to the FP32 residual in FP64, or the Jacobi fallback.  Dense form: a block
// of COARSE_THREADS computes 32 outputs, its warps splitting the inner index into contiguous ranges (loads of X
// coalesced across the 32 outputs), then warp 0 adds the warps' partial sums in warp order.
constexpr int COARSE_THREADS = 256, COARSE_WARPS = COARSE_THREADS / 32;
__host__ __device__ inline int coarse_blocks(int N, int64_t nn) {
    return N > 0 ? (N + 31) / 32 : (int)(nn + COARSE_THREADS - 1) / COARSE_THREADS;
}
__device__ __forceinline__ void coarse_solve32(VB vb, const MgLevel32& L, const double* __restrict__ X, int N,
                                               const int* __restrict__ status, const PcgScalars* S, double* rs,
                                               double* part) {
    if (S->done) return;
    const int64_t nn = L.nn;
    if (N == 0 || *status != 1) {
        for (int64_t n = (int64_t)vb.b * blockDim.x + threadIdx.x; n < nn; n += (int64_t)vb.n * blockDim.x) {
            const int m = L.mask[n];
            for (int c = 0; c < 3; ++c)
                L.x[c * nn + n] = ((m >> c) & 1) ? 0.0f : L.r[c * nn + n] * L.diag[c * nn + n];
        }
        return;
    }
    for (int j = threadIdx.x; j < N; j += blockDim.x) rs[j] = (double)L.r[(j % 3) * nn + j / 3];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = vb.b * 32 + lane;
    const int per = (N + COARSE_WARPS - 1) / COARSE_WARPS, j0 = w * per, j1 = min(N, j0 + per);
    double acc = 0.0;
    if (i < N)
        for (int j = j0; j < j1; ++j) acc = fma(X[(int64_t)j * N + i], rs[j], acc);
    part[w * 32 + lane] = acc;
    __syncthreads();
    if (w == 0 && i < N) {
        double t = 0.0;
        for (int k = 0; k < COARSE_WARPS; ++k) t += part[k * 32 + lane];
        const int ni = i / 3, ci = i % 3;
        L.x[ci * nn + ni] = ((L.mask[ni] >> ci) & 1) ? 0.0f : (float)t;
    }
}
__global__ void __launch_bounds__(COARSE_THREADS) k_coarse_solve32(MgLevel32 L, const double* __restrict__ X, int N,
                                                                   const int* __restrict__ status, const PcgScalars* S) {
    extern __shared__ double rs[];
    coarse_solve32(vb_real(), L, X, N, status, S, rs, rs + (N > 0 ? N : 0));
}

// ---------------------------------------------------------------- PCG vector steps in FP32
// r -= alpha Ap and |r|^2 (alpha = r.z / p.Ap of this iteration, stored for the direction kernel, which
// applies x += alpha p while it reads p anyway)
__device__ __forceinline__ void pcg_update32(VB vb, int64_t NNp, float* __restrict__ r, const float* __restrict__ Ap,
                                             RedSlot red, PcgScalars* S, double* sh) {
    if (S->done) return;
    const double den = S->denom;
    // breakdown of the FP32 recurrence (p.Ap <= 0 or r.z <= 0, e.g. an indefinite preconditioner): stop this
    // inner solve before the step; the FP64 outer loop restarts from the true residual.  Every block reads the
    // same scalars, so they all take the same branch.
    if (!(den > 0.0) || !(S->rz > 0.0)) {
        if (vb.b == 0 && threadIdx.x == 0) {
            S->alpha = 0.0f;
            S->done = 1;
            S->result = S->it;
        }
        return;
    }
    const float alpha = (float)(S->rz / den);
    if (vb.b == 0 && threadIdx.x == 0) S->alpha = alpha;
    // the three component planes are contiguous: one flat vector of 3 NNp floats (pads stay zero), 16-byte
    // accesses (cudaMalloc bases are 256-byte aligned; NNp is a multiple of 4)
    const int n3 = (int)(3 * NNp), n4 = n3 >> 2;
    const int stride = vb.n * blockDim.x;
    float4* __restrict__ r4 = reinterpret_cast<float4*>(r);
    const float4* __restrict__ a4 = reinterpret_cast<const float4*>(Ap);
    double part = 0.0;
    for (int i = vb.b * blockDim.x + threadIdx.x; i < n4; i += stride) {
        const float4 av = a4[i];
        float4 rv = r4[i];
        rv.x = fmaf(-alpha, av.x, rv.x); rv.y = fmaf(-alpha, av.y, rv.y);
        rv.z = fmaf(-alpha, av.z, rv.z); rv.w = fmaf(-alpha, av.w, rv.w);
        r4[i] = rv;
        part += (double)fmaf(rv.w, rv.w, fmaf(rv.z, rv.z, fmaf(rv.y, rv.y, rv.x * rv.x)));
    }
    for (int i = 4 * n4 + vb.b * blockDim.x + threadIdx.x; i < n3; i += stride) {
        const float rv = fmaf(-alpha, Ap[i], r[i]);
        r[i] = rv;
        part = fma((double)rv, (double)rv, part);
    }
    double tot;
    if (grid_fold(part, red, sh, &tot, vb) && threadIdx.x == 0) {
        S->rnorm2 = tot;
        S->it = S->it + 1;
        if (sqrt(tot) < S->stop) {
            S->done = 1;
            S->result = S->it;
        } else if (S->maxit > 0 && S->it >= S->maxit) {   // iteration budget of this inner solve spent
            S->done = 1;
        }
    }
}
__global__ void __launch_bounds__(RED_THREADS) k_pcg_update32(Grid g, float* __restrict__ r,
                                                              const float* __restrict__ Ap, RedSlot red,
                                                              PcgScalars* S) {
    __shared__ double sh[32];
    pcg_update32(vb_real(), g.NNp, r, Ap, red, S, sh);
}

// x += alpha p_old and, unless the update just converged, p = z + beta p_old.  Once converged, the
// step is applied by the first launch only (xit == it afterwards).
__device__ __forceinline__ void pcg_direction32(VB vb, int64_t NNp, const float* __restrict__ z, float* __restrict__ p,
                                                float* __restrict__ x, const PcgScalars* S) {
    if (S->xit == S->it) return;
    const bool move = !S->done;
    const float beta = (float)S->beta, alpha = S->alpha;
    const int n3 = (int)(3 * NNp), n4 = n3 >> 2;
    const int stride = vb.n * blockDim.x;
    float4* __restrict__ p4 = reinterpret_cast<float4*>(p);
    float4* __restrict__ x4 = reinterpret_cast<float4*>(x);
    const float4* __restrict__ z4 = reinterpret_cast<const float4*>(z);
    for (int i = vb.b * blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 pv = p4[i], xv = x4[i];
        xv.x = fmaf(alpha, pv.x, xv.x); xv.y = fmaf(alpha, pv.y, xv.y);
        xv.z = fmaf(alpha, pv.z, xv.z); xv.w = fmaf(alpha, pv.w, xv.w);
        x4[i] = xv;
        if (move) {
            const float4 zv = z4[i];
            pv.x = fmaf(beta, pv.x, zv.x); pv.y = fmaf(beta, pv.y, zv.y);
            pv.z = fmaf(beta, pv.z, zv.z); pv.w = fmaf(beta, pv.w, zv.w);
            p4[i] = pv;
        }
    }
    for (int i = 4 * n4 + vb.b * blockDim.x + threadIdx.x; i < n3; i += stride) {
        const float pv = p[i];
        x[i] = fmaf(alpha, pv, x[i]);
        if (move) p[i] = fmaf(beta, pv, z[i]);
    }
}
__global__ void k_pcg_direction32(Grid g, const float* __restrict__ z, float* __restrict__ p,
                                  float* __restrict__ x, PcgScalars* S) {
    pcg_direction32(vb_real(), g.NNp, z, p, x, S);
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// ---------------------------------------------------------------- batched launches
// one thread per launch list: the positions of its instances still iterating and their block prefix sums
__global__ void k_batch_compact(const BatchCompact* __restrict__ jobs, int njobs) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const BatchCompact J = jobs[j];
    int n = 0, acc = 0;
    J.act[1 + J.N] = 0;
    for (int p = 0; p < J.N; ++p) {
        if (J.S[p]->done) continue;
        J.act[1 + n] = p;
        acc += J.blocks[p];
        ++n;
        J.act[1 + J.N + n] = acc;
    }
    J.act[0] = n;
}

__global__ void __launch_bounds__(RED_THREADS) k_batch_update32(const BatchUpdate* __restrict__ a,
                                                                const int* __restrict__ act, int N) {
    __shared__ double sh[32];
    batch_walk(a, act, N, [&](const BatchUpdate& A, VB vb) { pcg_update32(vb, A.NNp, A.r, A.Ap, A.red, A.S, sh); });
}

__global__ void __launch_bounds__(RED_THREADS) k_batch_direction32(const BatchDirection* __restrict__ a,
                                                                   const int* __restrict__ act, int N) {
    batch_walk(a, act, N, [&](const BatchDirection& A, VB vb) { pcg_direction32(vb, A.NNp, A.z, A.p, A.x, A.S); });
}

// stage 0: span-4 transitions run their x pass, span-2 ones their whole window; stage 1: the span-4 y-z pass
__global__ void __launch_bounds__(256) k_batch_restrict32(const BatchRestrict* __restrict__ a,
                                                          const int* __restrict__ act, int N, int stage) {
    batch_walk(a, act, N, [&](const BatchRestrict& A, VB vb) {
        const MgLevel32 Lc = A.Lc, Lf = A.Lf;
        if (Lc.span == 4) {
            if (stage == 0) restrict_x32(vb, Lc, Lf, A.rf, A.a1, A.S);
            else restrict_yz32<4>(vb, Lc, Lf, A.a1, A.rc, A.S, A.normalize);
        } else {
            restrict_xyz32<2>(vb, Lc, Lf, A.rf, A.rc, A.S, A.normalize);
        }
    });
}

__global__ void __launch_bounds__(256) k_batch_prolong32(const BatchProlong* __restrict__ a,
                                                         const int* __restrict__ act, int N) {
    batch_walk(a, act, N, [&](const BatchProlong& A, VB vb) {
        const MgLevel32 Lc = A.Lc, Lf = A.Lf;
        prolong_smooth32(vb, Lc, Lf, Lc.x, Lf.r, Lf.x, A.w, A.S);
    });
}

__global__ void __launch_bounds__(RED_THREADS) k_batch_prolong0_32(const BatchProlong0* __restrict__ a,
                                                                   const int* __restrict__ act, int N) {
    __shared__ double sh[32];
    batch_walk(a, act, N, [&](const BatchProlong0& A, VB vb) {
        const MgLevel32 Lc = A.Lc, Lf = A.Lf;
        if (Lc.span == 4) prolong_smooth0_32<4>(vb, Lc, Lf, Lc.x, A.r, A.z, A.w, A.dot, A.S, sh);
        else prolong_smooth0_32<2>(vb, Lc, Lf, Lc.x, A.r, A.z, A.w, A.dot, A.S, sh);
    });
}

__global__ void __launch_bounds__(COARSE_THREADS) k_batch_coarse32(const BatchCoarse* __restrict__ a,
                                                                   const int* __restrict__ act, int N, int max_n) {
    extern __shared__ double rs[];
    batch_walk(a, act, N, [&](const BatchCoarse& A, VB vb) {
        const MgLevel32 L = A.L;
        coarse_solve32(vb, L, A.X, A.N, A.status, A.S, rs, rs + max_n);
    });
}

// the instances' done flags gathered into one array (one copy to the host per poll)
__global__ void k_batch_flags(PcgScalars* const* __restrict__ S, int n, int* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = S[i]->done;
}

// persistent grid of the batched launches: 8 resident blocks per SM of B200 (148 SMs), fewer for short lists
constexpr int BATCH_GRID = 8 * 148;

}  // namespace

int batch_blocks_update() { return RED_BLOCKS; }
int batch_blocks_prolong0() { return RED_BLOCKS; }
int batch_blocks_restrict(const BatchRestrict& a, int stage) {
    const MgLevel32& Lc = a.Lc;
    const MgLevel32& Lf = a.Lf;
    if (Lc.span == 4) {
        if (stage == 0) return (int)blocks_for((int64_t)(Lf.nz + 1) * (Lf.ny + 1) * (Lc.nx + 1), 256);
        return (int)blocks_for(Lc.nn, 256);
    }
    return stage == 0 ? (int)blocks_for(Lc.nn, 256) : 0;
}
int batch_blocks_prolong(const BatchProlong& a) { return (int)blocks_for(a.Lf.nn, 256); }
int batch_blocks_coarse(const BatchCoarse& a) { return std::max(1, coarse_blocks(a.N, a.L.nn)); }
void launch_batch_flags(PcgScalars* const* S, int n, int* out, cudaStream_t s) {
    k_batch_flags<<<1, 256, 0, s>>>(S, n, out);
}
void launch_batch_compact(const BatchCompact* jobs, int njobs, cudaStream_t s) {
    k_batch_compact<<<(njobs + 31) / 32, 32, 0, s>>>(jobs, njobs);
}
void launch_batch_update32(const BatchUpdate* a, const int* act, int N, cudaStream_t s) {
    k_batch_update32<<<BATCH_GRID, RED_THREADS, 0, s>>>(a, act, N);
}
void launch_batch_direction32(const BatchDirection* a, const int* act, int N, cudaStream_t s) {
    k_batch_direction32<<<BATCH_GRID, RED_THREADS, 0, s>>>(a, act, N);
}
void launch_batch_restrict32(const BatchRestrict* a, const int* act, int N, int stage, cudaStream_t s) {
    k_batch_restrict32<<<BATCH_GRID, 256, 0, s>>>(a, act, N, stage);
}
void launch_batch_prolong32(const BatchProlong* a, const int* act, int N, cudaStream_t s) {
    k_batch_prolong32<<<BATCH_GRID, 256, 0, s>>>(a, act, N);
}
void launch_batch_prolong0_32(const BatchProlong0* a, const int* act, int N, cudaStream_t s) {
    k_batch_prolong0_32<<<BATCH_GRID, RED_THREADS, 0, s>>>(a, act, N);
}
void launch_batch_coarse32(const BatchCoarse* a, const int* act, int N, int max_n, cudaStream_t s) {
    const int mn = max_n > 0 ? max_n : 0;
    k_batch_coarse32<<<BATCH_GRID, COARSE_THREADS, (size_t)(mn + 32 * COARSE_WARPS) * sizeof(double), s>>>(a, act, N,
                                                                                                           mn);
}

void launch_nodes_to32(const Grid& g, const double* a, float* b, cudaStream_t s) {
    k_rows_convert<double, float><<<RED_BLOCKS, 256, 0, s>>>(3 * (int64_t)g.nny * g.nnz, g.nnx, g.nnx, g.px, a, b);
}
void launch_nodes_from32(const Grid& g, const float* a, double* b, cudaStream_t s) {
    k_rows_convert<float, double><<<RED_BLOCKS, 256, 0, s>>>(3 * (int64_t)g.nny * g.nnz, g.nnx, g.px, g.nnx, a, b);
}
void launch_cells_to32(const Grid& g, const double* a, float* b, cudaStream_t s) {
    k_rows_convert<double, float><<<RED_BLOCKS, 256, 0, s>>>((int64_t)g.ey * g.ez, g.ex, g.ex, g.pex, a, b);
}
void launch_mixed_residual(const Grid& g, const double* b, const double* Au, float* r32, float* d32, RedSlot red,
                           double* rn2, cudaStream_t s) {
    k_mixed_residual<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, b, Au, r32, d32, red, rn2);
}
void launch_mixed_accumulate(const Grid& g, double* u, const float* d, cudaStream_t s) {
    k_mixed_accumulate<<<RED_BLOCKS, 256, 0, s>>>(g, u, d);
}
void launch_recip_diag32(int64_t rows, int len, int pitch, const double* d, float* rd, cudaStream_t s) {
    k_recip_diag32<<<RED_BLOCKS, 256, 0, s>>>(rows, len, pitch, d, rd);
}

void launch_matvec32(const Grid& g, const float* Ke, const float* E, const uint8_t* mask, const float* u, float* y,
                     RedSlot dot, PcgScalars* S, int mark, cudaStream_t s) {
    k_matvec32<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, Ke, E, mask, u, y, dot, S, mark);
}
// x pass then a fused y-z pass on the finest transition (span 4); one fused x-y-z pass on the
// coarser ones (span 2), whose fine residual sits in L2.
void launch_restrict32(const MgLevel32& Lc, const MgLevel32& Lf, const float* rf, float* rc, float* a1,
                       const PcgScalars* S, cudaStream_t s, bool normalize) {
    const int64_t n1 = (int64_t)(Lf.nz + 1) * (Lf.ny + 1) * (Lc.nx + 1);
    if (Lc.span == 4) {
        k_restrict_x32<<<blocks_for(n1, 256), 256, 0, s>>>(Lc, Lf, rf, a1, S);
        k_restrict_yz32<4><<<blocks_for(Lc.nn, 256), 256, 0, s>>>(Lc, Lf, a1, rc, S, normalize ? 1 : 0);
    } else {
        k_restrict_xyz32<2><<<blocks_for(Lc.nn, 256), 256, 0, s>>>(Lc, Lf, rf, rc, S, normalize ? 1 : 0);
    }
}
void launch_rows_to32(int64_t rows, int len, const double* a, float* b, cudaStream_t s) {
    k_rows_convert<double, float><<<RED_BLOCKS, 256, 0, s>>>(rows, len, len, len, a, b);
}
void launch_prolong_smooth32(const MgLevel32& Lc, const MgLevel32& Lf, const float* xc, const float* rf, float* xf,
                             float w, const PcgScalars* S, cudaStream_t s) {
    k_prolong_smooth32<<<blocks_for(Lf.nn, 256), 256, 0, s>>>(Lc, Lf, xc, rf, xf, w, S);
}
void launch_prolong_smooth0_32(const MgLevel32& Lc, const MgLevel32& Lf, const float* xc, const float* r, float* z,
                               float w, RedSlot dot, PcgScalars* S, cudaStream_t s) {
    if (Lc.span == 4) k_prolong_smooth0_32<4><<<RED_BLOCKS, RED_THREADS, 0, s>>>(Lc, Lf, xc, r, z, w, dot, S);
    else k_prolong_smooth0_32<2><<<RED_BLOCKS, RED_THREADS, 0, s>>>(Lc, Lf, xc, r, z, w, dot, S);
}
void launch_coarse_solve32(const MgLevel32& L, const double* X, int N, const int* status, const PcgScalars* S,
                           cudaStream_t s) {
    const unsigned blocks = (unsigned)std::max(1, coarse_blocks(N, L.nn));
    k_coarse_solve32<<<blocks, COARSE_THREADS, (size_t)((N > 0 ? N : 0) + 32 * COARSE_WARPS) * sizeof(double), s>>>(
        L, X, N, status, S);
}
void launch_pcg_update32(const Grid& g, float* x, float* r, const float* p, const float* Ap, RedSlot red,
                         PcgScalars* S, cudaStream_t s) {
    (void)x;
    (void)p;
    k_pcg_update32<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, r, Ap, red, S);
}
void launch_pcg_direction32(const Grid& g, const float* z, float* p, float* x, PcgScalars* S, cudaStream_t s) {
    k_pcg_direction32<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, z, p, x, S);
}

}  // namespace t3d
