// K(E) p in FP32, modal form, with the node planes staged by the Tensor Memory Accelerator.
//
// Same per-element arithmetic as k_matvec32_modal (packed FP32x2 form), so the two kernels give
// bit-identical results; what changes is how a tile's footprint reaches shared memory:
//   * one elected thread issues, per node plane, ONE 4-D bulk tensor copy of the tile's node rows for all
//     three components (box RW x (BY+1) x 1 x 3 of the pitched FP32 displacement image) and ONE 3-D copy of
//     the moduli of the element layer below the plane (box RW x BY x 1 of the pitched FP32 moduli), both
//     completing on the plane's mbarrier (expect-tx of the box bytes);
//   * the rows start at x rounded down to a multiple of 4 (16-byte TMA coordinate rule); the kernel reads
//     from the remainder on: node x = X0-1+i sits at column sx + i of its smem row, sx = (X0-1) & 3;
//   * boxes that reach outside the grid (x = -1, y = -1, z = -1 or z = nnz) read zeros (TMA fill), which
//     is what the cp.async kernel's predicated copies produced;
//   * the other threads only wait on the mbarrier: no per-thread copy instructions and no L1 traffic for
//     the loads.
// The tensor maps cover this GPU's own memory only and no copy uses cluster multicast.
//
// Ring: STAGES slots {u box, E box} with one mbarrier each; a slot is reused once every thread has passed
// the per-plane __syncthreads that follows its last read.  mbarrier waits are bounded: after
// TMA_WAIT_LIMIT polls a thread records the failure in *err and continues (garbage, never a hang); the
// host checks *err after the solve.
#pragma once
#include <cuda.h>

#include "kernels.hpp"
#include "modal.cuh"
#include "red.cuh"

namespace t3d {

namespace {

constexpr long long TMA_WAIT_LIMIT = 1ll << 24;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false (and *err set) when the barrier's phase did not complete within the limit.  Once any
// thread has given up (err set, or `failed` in this thread) waits return at once, so a kernel whose copies
// never land still ends promptly.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, int* err, bool& failed) {
    if (failed) return false;
    for (long long k = 0; k < TMA_WAIT_LIMIT; ++k) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((k & 1023) == 1023 && *(volatile int*)err) {
            failed = true;
            return false;
        }
    }
    atomicExch(err, 1);
    failed = true;
    return false;
}
__device__ __forceinline__ void tma_load_4d(unsigned dst, const CUtensorMap* map, int x, int y, int z, int c,
                                            unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(c), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap* map, int x, int y, int z, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

}  // namespace

// Shared memory of one CTA: STAGES slots of {u box [3][PY][RW], E box [BY][RW]} (each rounded up to 128
// bytes, the TMA destination alignment), the corner-exchange buffers and the mbarriers.
template <int BX, int BY, int STAGES>
struct TmaSmem {
    static constexpr int RW = (BX + 1 + 3 + 3) / 4 * 4;   // footprint row + up to 3 leading values, x4
    static constexpr int PY = BY + 1;
    static constexpr int UF = (3 * PY * RW + 31) / 32 * 32;   // floats per u slot (128-byte multiple)
    static constexpr int EF = (BY * RW + 31) / 32 * 32;
    static constexpr unsigned UBYTES = 3u * PY * RW * 4u, EBYTES = (unsigned)BY * RW * 4u;
    float u[STAGES][UF];
    float e[STAGES][EF];
    float4 outc[2][3][BY][BX];
    double sh[32];
    unsigned long long bar[STAGES];
};

// Epilogue of an owned node (K x at the node in y0..y2, x's own values in h):
//   MODE 0  the PCG's K(E)p: y = K x (fixed DOFs 0); with dot.partial, x.(K x) folded into S->denom;
//   MODE 1  the Standard V-cycle's residual: y = r - K x (fixed DOFs 0);
//   MODE 2  the Standard V-cycle's correction: y = x + omega (r - K x) / D (rd = 1/D; fixed DOFs 0) written to a
//           buffer other than x, with r.y folded into S (rz, or beta and rz, as the V-cycle's r.z).
// The CTA's shared memory, 128-byte aligned (the launch adds 128 bytes of slack for the shift).
template <class SM>
__device__ __forceinline__ SM& tma_smem() {
    extern __shared__ __align__(128) unsigned char tma_smem_raw[];
    return *reinterpret_cast<SM*>(tma_smem_raw + ((128u - (smem_u32(tma_smem_raw) & 127u)) & 127u));
}
template <class SM, int STAGES>
__device__ __forceinline__ void tma_ring_init(SM& sm) {
    if (threadIdx.x == 0) {
        for (int k = 0; k < STAGES; ++k) mbar_init(smem_u32(&sm.bar[k]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
}
__device__ __forceinline__ void tma_prefetch_maps(const CUtensorMap* umap, const CUtensorMap* emap) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(umap) : "memory");
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(emap) : "memory");
}

// One logical block (vb) of the product: work items vb.b, vb.b + vb.n, ... of the tiling t.  gp (planes this
// CTA has consumed: ring slot and mbarrier phase) and failed (a wait of this thread gave up) carry over from
// one call to the next in the same CTA.
template <int BX, int BY, int STAGES, int MODE>
__device__ __forceinline__ void tma_matvec_body(TmaSmem<BX, BY, STAGES>& sm, const CUtensorMap* umap,
                                                const CUtensorMap* emap, const Grid& g, const ModalKe& kh,
                                                const ModalTiling& t, const uint8_t* __restrict__ mask,
                                                float* __restrict__ y, RedSlot dot, PcgScalars* S, int mark, int* err,
                                                const float* __restrict__ rv, const float* __restrict__ rd,
                                                float omega, VB vb, unsigned& gp, bool& failed) {
    using SM = TmaSmem<BX, BY, STAGES>;
    constexpr int RW = SM::RW, PY = SM::PY;
    static_assert(STAGES >= 2, "ring needs two slots at least");
    // mark: the PCG product (not an operator inside the V-cycle) records that the last alpha is in x
    if (S != nullptr && mark && vb.b == 0 && threadIdx.x == 0) S->xit = S->it;
    if (S != nullptr && S->done) return;
    const int tx = threadIdx.x % BX, ty = threadIdx.x / BX;
    const bool producer = threadIdx.x == 0;
    const int64_t NXY = (int64_t)g.px * g.nny, MXY = (int64_t)g.nnx * g.nny;
    double part = 0.0;
    for (int w = vb.b; w < t.items; w += vb.n) {
        const int itx = w % t.tiles_x;
        const int rest = w / t.tiles_x;
        const int ity = rest % t.tiles_y;
        const int Z0 = (rest / t.tiles_y) * t.slab;
        const int Z1 = min(Z0 + t.slab, g.nnz);
        const int X0 = itx * (BX - 1), Y0 = ity * (BY - 1);
        const int cx = X0 - 1 + tx, cy = Y0 - 1 + ty;            // element column and own node
        const int xu = (X0 - 1) & ~3, sx = (X0 - 1) - xu;        // node box x start (16-byte aligned), shift
        const int xe = X0 & ~3, se = X0 - xe;                    // cell box: cell x = cx + 1
        const bool owner = tx > 0 && ty > 0 && cx < g.nnx && cy < g.nny;
        const int nplanes = Z1 - Z0 + 2;                          // node planes Z0-1 .. Z1
        auto issue = [&](int k) {                                 // plane Z0-1+k into ring slot (gp + k) % STAGES
            const int q = Z0 - 1 + k;
            const int s = (int)((gp + (unsigned)k) % STAGES);
            const unsigned bar = smem_u32(&sm.bar[s]);
            mbar_expect_tx(bar, SM::UBYTES + SM::EBYTES);
            tma_load_4d(smem_u32(&sm.u[s][0]), umap, xu, Y0 - 1, q, 0, bar);
            tma_load_3d(smem_u32(&sm.e[s][0]), emap, xe, Y0, q, bar);   // layer q-1: cells z = q
        };
        __syncthreads();                                          // the previous item's readers are done
        if (producer)
            for (int k = 0; k < STAGES - 1 && k < nplanes; ++k) issue(k);
        Modes2 bot2{0.f, 0.f, 0.f, 0.f}, acc2{0.f, 0.f, 0.f, 0.f};   // component 2
        const float2 z2 = make_float2(0.f, 0.f);
        Modes2x2 bot01{z2, z2, z2, z2}, acc01{z2, z2, z2, z2};   // components 0 and 1
        float4 h1 = make_float4(0.f, 0.f, 0.f, 0.f), h2 = h1;     // own node values of planes pz-1, pz-2
        float k0 = 0.f, k1 = 0.f, k2 = 0.f;                      // own element's corner (0,0) of plane pz-2
        int mk_next = 0;                                         // mask byte of plane pz-1
        const int node_off = owner ? cy * g.px + cx : 0;
        const int mask_off = owner ? cy * g.nnx + cx : 0;
        const int ubase = ty * RW + sx + tx, ebase = ty * RW + se + tx;
        constexpr int CS = PY * RW;                              // component stride in the u box
#pragma unroll 1
        for (int it = 0; it <= nplanes; ++it) {
            const int pz = Z0 - 1 + it;
            const int s = (int)((gp + (unsigned)it) % STAGES);
            if (it < nplanes) mbar_wait(smem_u32(&sm.bar[s]), ((gp + (unsigned)it) / STAGES) & 1u, err, failed);
            __syncthreads();                 // plane pz landed; the corners of plane pz-2 are visible
            if (producer && it + STAGES - 1 < nplanes) issue(it + STAGES - 1);
            if (owner && pz - 2 >= Z0) {     // plane pz-2: own corner + 3 neighbours, fixed order
                const int pb = (it - 1) & 1;
                const float4 s1 = sm.outc[pb][0][ty][tx - 1], s2 = sm.outc[pb][1][ty - 1][tx],
                             s3 = sm.outc[pb][2][ty - 1][tx - 1];
                float y0 = ((k0 + s1.x) + s2.x) + s3.x;
                float y1 = ((k1 + s1.y) + s2.y) + s3.y;
                float y2 = ((k2 + s1.z) + s2.z) + s3.z;
                const int n = node_off + (pz - 2) * (int)NXY;
                const int NP = (int)g.NNp;
                if (MODE == 1) {
                    y0 = rv[n] - y0;
                    y1 = rv[NP + n] - y1;
                    y2 = rv[2 * NP + n] - y2;
                } else if (MODE == 2) {
                    const float r0 = rv[n], r1 = rv[NP + n], r2 = rv[2 * NP + n];
                    y0 = h2.x + (omega * (r0 - y0)) * rd[n];
                    y1 = h2.y + (omega * (r1 - y1)) * rd[NP + n];
                    y2 = h2.z + (omega * (r2 - y2)) * rd[2 * NP + n];
                    if (mk_next & 1) y0 = 0.f;
                    if (mk_next & 2) y1 = 0.f;
                    if (mk_next & 4) y2 = 0.f;
                    part += (double)fmaf(r2, y2, fmaf(r1, y1, r0 * y0));
                }
                if (mk_next & 1) y0 = 0.f;
                if (mk_next & 2) y1 = 0.f;
                if (mk_next & 4) y2 = 0.f;
                y[n] = y0;
                y[NP + n] = y1;
                y[2 * NP + n] = y2;
                if (MODE == 0 && dot.partial)   // the node's 3 FP32 products summed in FP32, accumulated in FP64
                    part += (double)fmaf(h2.z, y2, fmaf(h2.y, y1, h2.x * y0));
            }
            if (owner && pz - 1 >= Z0 && pz - 1 < Z1) mk_next = mask[mask_off + (pz - 1) * (int)MXY];
            if (it < nplanes) {
                const float* U = sm.u[s] + ubase;
                const float4 a = make_float4(U[0], U[CS], U[2 * CS], 0.f);
                const float4 b = make_float4(U[1], U[CS + 1], U[2 * CS + 1], 0.f);
                const float4 c = make_float4(U[RW], U[CS + RW], U[2 * CS + RW], 0.f);
                const float4 d = make_float4(U[RW + 1], U[CS + RW + 1], U[2 * CS + RW + 1], 0.f);
                const Modes2x2 top01 = fwd2x2(make_float2(a.x, a.y), make_float2(b.x, b.y), make_float2(c.x, c.y),
                                              make_float2(d.x, d.y));
                const Modes2 top2 = fwd2(a.z, b.z, c.z, d.z);
                if (it >= 1) {               // element layer pz-1 between planes pz-1 (bot) and pz (top)
                    const float Ee = sm.e[s][ebase];
                    const float2 E2 = make_float2(Ee, Ee);
                    float2 cm01[8];
                    cm01[0] = z2;
                    cm01[1] = mul2(E2, add2(top01.m10, bot01.m10));
                    cm01[2] = mul2(E2, add2(top01.m01, bot01.m01));
                    cm01[3] = mul2(E2, add2(top01.m11, bot01.m11));
                    cm01[4] = mul2(E2, sub2(top01.m00, bot01.m00));
                    cm01[5] = mul2(E2, sub2(top01.m10, bot01.m10));
                    cm01[6] = mul2(E2, sub2(top01.m01, bot01.m01));
                    cm01[7] = mul2(E2, sub2(top01.m11, bot01.m11));
                    float cm[24];
#pragma unroll
                    for (int m = 0; m < 8; ++m) {
                        cm[m] = cm01[m].x;
                        cm[8 + m] = cm01[m].y;
                    }
                    cm[16] = 0.f;
                    cm[17] = Ee * (top2.m10 + bot2.m10);
                    cm[18] = Ee * (top2.m01 + bot2.m01);
                    cm[19] = Ee * (top2.m11 + bot2.m11);
                    cm[20] = Ee * (top2.m00 - bot2.m00);
                    cm[21] = Ee * (top2.m10 - bot2.m10);
                    cm[22] = Ee * (top2.m01 - bot2.m01);
                    cm[23] = Ee * (top2.m11 - bot2.m11);
                    float yh[24];
#pragma unroll
                    for (int i = 0; i < 24; ++i) yh[i] = 0.f;
                    {
                        int e = 0;
#define T3D_KH_FMA(dd, ss) yh[dd] = fmaf(kh.v[e++], cm[ss], yh[dd]);
                        T3D_KH_PATTERN(T3D_KH_FMA)
#undef T3D_KH_FMA
                    }
                    float2 q01[8];
#pragma unroll
                    for (int m = 0; m < 8; ++m) q01[m] = make_float2(yh[m], yh[8 + m]);
                    const Modes2x2 fin01{sub2(acc01.m00, q01[4]), add2(acc01.m10, sub2(q01[1], q01[5])),
                                         add2(acc01.m01, sub2(q01[2], q01[6])), add2(acc01.m11, sub2(q01[3], q01[7]))};
                    acc01 = Modes2x2{q01[4], add2(q01[1], q01[5]), add2(q01[2], q01[6]), add2(q01[3], q01[7])};
                    const float* r = yh + 16;
                    const Modes2 fin2{acc2.m00 - r[4], acc2.m10 + (r[1] - r[5]), acc2.m01 + (r[2] - r[6]),
                                      acc2.m11 + (r[3] - r[7])};
                    acc2 = Modes2{r[4], r[1] + r[5], r[2] + r[6], r[3] + r[7]};
                    float2 w00, w10, w01, w11;
                    inv2x2(fin01, w00, w10, w01, w11);
                    float v200, v210, v201, v211;
                    inv2(fin2, v200, v210, v201, v211);
                    if (it >= 2) {
                        k0 = w00.x;
                        k1 = w00.y;
                        k2 = v200;
                        const int pb = it & 1;
                        sm.outc[pb][0][ty][tx] = make_float4(w10.x, w10.y, v210, 0.f);
                        sm.outc[pb][1][ty][tx] = make_float4(w01.x, w01.y, v201, 0.f);
                        sm.outc[pb][2][ty][tx] = make_float4(w11.x, w11.y, v211, 0.f);
                    }
                }
                bot01 = top01;
                bot2 = top2;
                h2 = h1;
                h1 = a;
            }
        }
        gp += (unsigned)nplanes;
    }
    if (MODE == 0 && dot.partial) {
        double tot;
        if (grid_fold(part, dot, sm.sh, &tot, vb) && threadIdx.x == 0) S->denom = tot;
    }
    if (MODE == 2) {
        double tot;
        if (grid_fold(part, dot, sm.sh, &tot, vb) && threadIdx.x == 0) {
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
}

template <int BX, int BY, int MINB, int STAGES, int MODE = 0>
__global__ void __launch_bounds__(BX * BY, MINB)
    k_matvec32_tma(const __grid_constant__ CUtensorMap umap, const __grid_constant__ CUtensorMap emap, Grid g,
                   ModalKe kh, ModalTiling t, const uint8_t* __restrict__ mask, float* __restrict__ y, RedSlot dot,
                   PcgScalars* S, int mark, int* err, const float* __restrict__ rv, const float* __restrict__ rd,
                   float omega) {
    using SM = TmaSmem<BX, BY, STAGES>;
    SM& sm = tma_smem<SM>();
    tma_ring_init<SM, STAGES>(sm);
    if (threadIdx.x == 0) tma_prefetch_maps(&umap, &emap);
    __syncthreads();
    unsigned gp = 0;
    bool failed = false;
    tma_matvec_body<BX, BY, STAGES, MODE>(sm, &umap, &emap, g, kh, t, mask, y, dot, S, mark, err, rv, rd, omega,
                                          vb_real(), gp, failed);
}

// Batched K(E)u (MODE 0 the PCG product with the p.Ap fold; 1, 2 the Standard cycle's fused residual and
// correction): many instances in one persistent launch.  The work
// list is (active instance, logical block) (act, kernels.hpp): each logical block runs its instance's own
// tiling, reduction slot and scalars, so each instance's result is the one its own launch gives.  The tensor maps sit in global memory, one pair per instance, written by the host
// before the launch; they cover this GPU's own buffers and no copy uses cluster multicast.  Instances whose
// inner solve has converged (S->done) skip their blocks: the per-instance convergence mask.
template <int BX, int BY, int MINB, int STAGES, int MODE = 0>
__global__ void __launch_bounds__(BX * BY, MINB)
    k_matvec32_tma_batched(const BatchMatvec* __restrict__ a, const int* __restrict__ act, int N, ModalKe kh,
                           int* err) {
    using SM = TmaSmem<BX, BY, STAGES>;
    SM& sm = tma_smem<SM>();
    tma_ring_init<SM, STAGES>(sm);
    __syncthreads();
    unsigned gp = 0;
    bool failed = false;
    const int n = __ldg(act);                      // the active instances (layout: kernels.hpp)
    const int* __restrict__ pos = act + 1;
    const int* __restrict__ vs = act + 1 + N;
    const int total = __ldg(vs + n);
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
        const int k = batch_instance(vs, n, v);
        const BatchMatvec& A = a[__ldg(pos + k)];
        const int v0 = __ldg(vs + k);
        const Grid g = A.g;
        const ModalTiling t = A.t;
        if (threadIdx.x == 0) tma_prefetch_maps(A.umap, A.emap);
        tma_matvec_body<BX, BY, STAGES, MODE>(sm, A.umap, A.emap, g, kh, t, A.mask, A.y, A.dot, A.S, MODE == 0 ? 1 : 0,
                                              err, A.rv, A.rd, A.omega, VB{v - v0, __ldg(vs + k + 1) - v0}, gp,
                                              failed);
        __syncthreads();
    }
}

}  // namespace t3d
