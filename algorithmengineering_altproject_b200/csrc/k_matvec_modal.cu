// K(E) p in FP32 through the modal (corner-Hadamard) form of the hex8 stiffness.
//
// The 8 corner values of one displacement component inside a voxel are mapped to the coefficients of
// the tensor-product basis {1, x, y, xy, z, xz, yz, xyz} on [-1,1]^3 by a Hadamard transform (adds
// and subtracts only).  Because that basis is L2-orthogonal on the cube and the element is an
// axis-aligned cube with an isotropic material, the 24x24 element stiffness (fea.cpp:117-179) becomes
// block diagonal with only 45 nonzeros (rigid translations have no energy; normal strains couple in one
// 3x3 block; shears, bilinear and trilinear modes in 2x2 / 3x3 / 1x1 blocks).  The values are taken from
// the context's own Ke (Kh = T^T Ke T / 64, checked on the host to vanish off this pattern), so the
// operator is the reference's Ke * u_e up to FP32 rounding: per element
//     y_e = E_e * T (Kh (T^T u_e))
// costs about 180 flops instead of 1152.
//
// Data flow (one CTA of BX x BY threads per tile; threads = element columns):
//   * a tile owns the nodes x in [X0, X0+BX-1), y in [Y0, Y0+BY-1) of a slab of node planes
//     z in [Z0, Z1); its element footprint is cx in [X0-1, X0+BX-1), cy in [Y0-1, Y0+BY-1);
//   * it marches up the slab: each node plane (BX+1)x(BY+1) is read once from HBM (coalesced, into
//     registers one plane ahead, then into shared memory); the x-y Hadamard stage of a plane is kept in
//     registers and reused by the element layers below and above it;
//   * the contributions of the layer below and above a node plane are summed in modal x-y form, then
//     transformed back to corners and exchanged through shared memory so that each owned node adds its
//     4 element columns in a fixed order (deterministic, no atomics);
//   * fixed DOFs are zeroed by the node mask (their inputs are exact zeros); p.Ap is folded in FP64.
// Work items (tile, slab) are walked by a persistent grid in x-fastest order so that concurrent CTAs
// share their halo planes through L2.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

#include "k_matvec_tma.cuh"
#include "kernels.hpp"
#include "modal.cuh"
#include "red.cuh"
#include "t3d_b200.h"

namespace t3d {

namespace {

__device__ __forceinline__ void cp_async4(unsigned s, const float* gsrc, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc), "r"(valid ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

}  // namespace

// Shared-memory layout of one CTA (dynamic): STAGES ring slots of {node plane footprint, moduli of
// the element layer below it}, then two corner-exchange buffers.
template <int BX, int BY, int STAGES>
struct ModalSmem {
    static constexpr int PX = BX + 1, PY = BY + 1;
    float4 plane[STAGES][PY][PX];   // (c0, c1, c2, -) of each footprint node
    float emod[STAGES][BY][BX];     // E of element column (tx, ty) in the layer below the plane
    float4 outc[2][3][BY][BX];      // corners (1,0), (0,1), (1,1) of each element column, by plane parity
    double sh[32];
};

template <int BX, int BY, int MINB, int STAGES, int PACK>
__global__ void __launch_bounds__(BX * BY, MINB)
    k_matvec32_modal(Grid g, ModalKe kh, ModalTiling t, const float* __restrict__ E,
                     const uint8_t* __restrict__ mask, const float* __restrict__ u, float* __restrict__ y,
                     RedSlot dot, PcgScalars* S, int mark) {
    constexpr int PX = BX + 1, PY = BY + 1;
    static_assert(PY <= BX, "the footprint column is loaded by one row of BX threads");
    static_assert(STAGES >= 2, "ring needs two slots at least");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ModalSmem<BX, BY, STAGES>& sm = *reinterpret_cast<ModalSmem<BX, BY, STAGES>*>(smem_raw);
    // mark: the PCG product (not an operator inside the V-cycle) records that the last alpha is in x
    if (S != nullptr && mark && blockIdx.x == 0 && threadIdx.x == 0) S->xit = S->it;
    if (S != nullptr && S->done) return;
    const int tx = threadIdx.x % BX, ty = threadIdx.x / BX;
    // FP32 images are pitched (rows of g.px nodes, g.pex cells); the node mask is not
    const int64_t NN = g.NNp, NXY = (int64_t)g.px * g.nny, EXY = (int64_t)g.pex * g.ey;
    const int64_t MXY = (int64_t)g.nnx * g.nny;
    // besides its own node, thread row 0 loads the footprint's last row, thread row 1 its last column
    const int ex_kind = (ty == 0) ? 1 : ((ty == 1 && tx < PY) ? 2 : 0);
    double part = 0.0;
    for (int w = blockIdx.x; w < t.items; w += gridDim.x) {
        const int itx = w % t.tiles_x;
        const int rest = w / t.tiles_x;
        const int ity = rest % t.tiles_y;
        const int Z0 = (rest / t.tiles_y) * t.slab;
        const int Z1 = min(Z0 + t.slab, g.nnz);
        const int X0 = itx * (BX - 1), Y0 = ity * (BY - 1);
        const int cx = X0 - 1 + tx, cy = Y0 - 1 + ty;           // element column and own node
        const int exx = ex_kind == 1 ? cx : X0 - 1 + BX;
        const int exy = ex_kind == 1 ? Y0 - 1 + BY : Y0 - 1 + tx;
        const bool own_xy = cx >= 0 && cy >= 0 && cx < g.nnx && cy < g.nny;
        const bool ext_xy = ex_kind != 0 && exx >= 0 && exy >= 0 && exx < g.nnx && exy < g.nny;
        const bool e_in = cx <= g.nx && cy <= g.ny;             // cell array covers cx, cy in [-1, n]
        const bool owner = tx > 0 && ty > 0 && own_xy;
        // plane-0 offsets (32-bit: 3 NN < 2^31); plane q adds q * NXY (nodes) or q * EXY (the layer
        // below plane q is q-1)
        const int own_off = own_xy ? cy * g.px + cx : 0;
        const int ext_off = ext_xy ? exy * g.px + exx : 0;
        const int e_off = e_in ? (int)g.pcell(cx, cy, -1) : 0;
        const unsigned own_s = (unsigned)__cvta_generic_to_shared(&sm.plane[0][ty][tx].x);
        const unsigned ext_s = (unsigned)__cvta_generic_to_shared(
            ex_kind == 1 ? &sm.plane[0][BY][tx].x : &sm.plane[0][min(tx, PY - 1)][BX].x);
        const unsigned e_s = (unsigned)__cvta_generic_to_shared(&sm.emod[0][ty][tx]);
        const int nplanes = Z1 - Z0 + 2;                         // node planes Z0-1 .. Z1
        auto issue = [&](int k) {                                // plane Z0-1+k into ring slot k % STAGES
            const int q = Z0 - 1 + k, s = k % STAGES;
            const bool vz = q >= 0 && q < g.nnz;
            const int on = q * (int)NXY;
            const bool vo = own_xy && vz, ve = ext_xy && vz;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                cp_async4(own_s + s * (PY * PX * 16) + 4 * c, u + (vo ? own_off + on + c * (int)NN : 0), vo);
                if (ex_kind)
                    cp_async4(ext_s + s * (PY * PX * 16) + 4 * c, u + (ve ? ext_off + on + c * (int)NN : 0), ve);
            }
            const bool vm = e_in && q >= 0;
            cp_async4(e_s + s * (BY * BX * 4), E + (vm ? e_off + q * (int)EXY : 0), vm);
        };
        __syncthreads();                                         // the previous item's readers are done
#pragma unroll
        for (int k = 0; k < STAGES - 1; ++k) {
            if (k < nplanes) issue(k);
            cp_async_commit();
        }
        Modes2 bot[3], acc[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) acc[k] = bot[k] = Modes2{0.f, 0.f, 0.f, 0.f};
        const float2 z2 = make_float2(0.f, 0.f);
        Modes2x2 bot01{z2, z2, z2, z2}, acc01{z2, z2, z2, z2};   // PACK: components 0 and 1 (bot/acc[2] = comp 2)
        float4 h1 = make_float4(0.f, 0.f, 0.f, 0.f), h2 = h1;     // own node values of planes pz-1, pz-2
        float k0 = 0.f, k1 = 0.f, k2 = 0.f;                      // own element's corner (0,0) of plane pz-2
        int mk_next = 0;                                         // mask byte of plane pz-1
        const int node_off = owner ? cy * g.px + cx : 0;
        const int mask_off = owner ? cy * g.nnx + cx : 0;
#pragma unroll 2
        for (int it = 0; it <= nplanes; ++it) {
            const int pz = Z0 - 1 + it;
            cp_async_wait<STAGES - 2>();
            __syncthreads();                 // plane pz and the corners of plane pz-2 are visible
            if (it + STAGES - 1 < nplanes) issue(it + STAGES - 1);
            cp_async_commit();
            if (owner && pz - 2 >= Z0) {     // plane pz-2: own corner + 3 neighbours, fixed order
                const int pb = (it - 1) & 1;
                const float4 s1 = sm.outc[pb][0][ty][tx - 1], s2 = sm.outc[pb][1][ty - 1][tx],
                             s3 = sm.outc[pb][2][ty - 1][tx - 1];
                float y0 = ((k0 + s1.x) + s2.x) + s3.x;
                float y1 = ((k1 + s1.y) + s2.y) + s3.y;
                float y2 = ((k2 + s1.z) + s2.z) + s3.z;
                if (mk_next & 1) y0 = 0.f;
                if (mk_next & 2) y1 = 0.f;
                if (mk_next & 4) y2 = 0.f;
                const int n = node_off + (pz - 2) * (int)NXY;
                y[n] = y0;
                y[(int)NN + n] = y1;
                y[2 * (int)NN + n] = y2;
                if (dot.partial)   // the node's 3 FP32 products summed in FP32, accumulated in FP64
                    part += (double)fmaf(h2.z, y2, fmaf(h2.y, y1, h2.x * y0));
            }
            if (owner && pz - 1 >= Z0 && pz - 1 < Z1) mk_next = mask[mask_off + (pz - 1) * (int)MXY];
            if (!PACK && it < nplanes) {
                const int s = it % STAGES;
                const float4 a = sm.plane[s][ty][tx], b = sm.plane[s][ty][tx + 1], c = sm.plane[s][ty + 1][tx],
                             d = sm.plane[s][ty + 1][tx + 1];
                Modes2 top[3];
                top[0] = fwd2(a.x, b.x, c.x, d.x);
                top[1] = fwd2(a.y, b.y, c.y, d.y);
                top[2] = fwd2(a.z, b.z, c.z, d.z);
                if (it >= 1) {               // element layer pz-1 between planes pz-1 (bot) and pz (top)
                    const float Ee = sm.emod[s][ty][tx];
                    float cm[24];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        cm[8 * q + 0] = 0.f;
                        cm[8 * q + 1] = Ee * (top[q].m10 + bot[q].m10);
                        cm[8 * q + 2] = Ee * (top[q].m01 + bot[q].m01);
                        cm[8 * q + 3] = Ee * (top[q].m11 + bot[q].m11);
                        cm[8 * q + 4] = Ee * (top[q].m00 - bot[q].m00);
                        cm[8 * q + 5] = Ee * (top[q].m10 - bot[q].m10);
                        cm[8 * q + 6] = Ee * (top[q].m01 - bot[q].m01);
                        cm[8 * q + 7] = Ee * (top[q].m11 - bot[q].m11);
                    }
                    float yh[24];
#pragma unroll
                    for (int i = 0; i < 24; ++i) yh[i] = 0.f;
                    {
                        int e = 0;
#define T3D_KH_FMA(dd, ss) yh[dd] = fmaf(kh.v[e++], cm[ss], yh[dd]);
                        T3D_KH_PATTERN(T3D_KH_FMA)
#undef T3D_KH_FMA
                    }
                    float v[3][4];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        const float* r = yh + 8 * q;
                        const Modes2 fin{acc[q].m00 - r[4], acc[q].m10 + (r[1] - r[5]), acc[q].m01 + (r[2] - r[6]),
                                         acc[q].m11 + (r[3] - r[7])};                         // plane pz-1 complete
                        acc[q] = Modes2{r[4], r[1] + r[5], r[2] + r[6], r[3] + r[7]};        // onto plane pz
                        inv2(fin, v[q][0], v[q][1], v[q][2], v[q][3]);
                    }
                    if (it >= 2) {           // plane pz-1 >= Z0 is owned: publish the 3 foreign corners
                        k0 = v[0][0];
                        k1 = v[1][0];
                        k2 = v[2][0];
                        const int pb = it & 1;
                        sm.outc[pb][0][ty][tx] = make_float4(v[0][1], v[1][1], v[2][1], 0.f);
                        sm.outc[pb][1][ty][tx] = make_float4(v[0][2], v[1][2], v[2][2], 0.f);
                        sm.outc[pb][2][ty][tx] = make_float4(v[0][3], v[1][3], v[2][3], 0.f);
                    }
                }
#pragma unroll
                for (int q = 0; q < 3; ++q) bot[q] = top[q];
                h2 = h1;
                h1 = a;
            }
            if (PACK && it < nplanes) {      // same layer arithmetic, components 0 and 1 packed
                const int s = it % STAGES;
                const float4 a = sm.plane[s][ty][tx], b = sm.plane[s][ty][tx + 1], c = sm.plane[s][ty + 1][tx],
                             d = sm.plane[s][ty + 1][tx + 1];
                const Modes2x2 top01 = fwd2x2(make_float2(a.x, a.y), make_float2(b.x, b.y), make_float2(c.x, c.y),
                                              make_float2(d.x, d.y));
                const Modes2 top2 = fwd2(a.z, b.z, c.z, d.z);
                if (it >= 1) {
                    const float Ee = sm.emod[s][ty][tx];
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
                    cm[17] = Ee * (top2.m10 + bot[2].m10);
                    cm[18] = Ee * (top2.m01 + bot[2].m01);
                    cm[19] = Ee * (top2.m11 + bot[2].m11);
                    cm[20] = Ee * (top2.m00 - bot[2].m00);
                    cm[21] = Ee * (top2.m10 - bot[2].m10);
                    cm[22] = Ee * (top2.m01 - bot[2].m01);
                    cm[23] = Ee * (top2.m11 - bot[2].m11);
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
                    const Modes2 fin2{acc[2].m00 - r[4], acc[2].m10 + (r[1] - r[5]), acc[2].m01 + (r[2] - r[6]),
                                      acc[2].m11 + (r[3] - r[7])};
                    acc[2] = Modes2{r[4], r[1] + r[5], r[2] + r[6], r[3] + r[7]};
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
                bot[2] = top2;
                h2 = h1;
                h1 = a;
            }
        }
        cp_async_wait<0>();
    }
    if (dot.partial) {
        double tot;
        if (grid_fold(part, dot, sm.sh, &tot) && threadIdx.x == 0) S->denom = tot;
    }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// Tensor maps of the pitched FP32 displacement image u (x, y, z, component; box rw x py x 1 x 3) and moduli
// E (x, y, z; box rw x by x 1).  Strides are multiples of 16 bytes because the rows are pitched; elements
// outside the arrays read as zero.
bool modal_tensor_maps(const Grid& g, const float* u, const float* E, int rw, int py, int by, CUtensorMap* um,
                       CUtensorMap* em) {
    const EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    const cuuint64_t ud[4] = {(cuuint64_t)g.px, (cuuint64_t)g.nny, (cuuint64_t)g.nnz, 3};
    const cuuint64_t us[3] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.px * g.nny * 4, (cuuint64_t)g.NNp * 4};
    const cuuint32_t ub[4] = {(cuuint32_t)rw, (cuuint32_t)py, 1, 3};
    const cuuint32_t one[4] = {1, 1, 1, 1};
    if (fn(um, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(u), ud, us, ub, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS)
        return false;
    const cuuint64_t ed[3] = {(cuuint64_t)g.pex, (cuuint64_t)g.ey, (cuuint64_t)g.ez};
    const cuuint64_t es[2] = {(cuuint64_t)g.pex * 4, (cuuint64_t)g.pex * g.ey * 4};
    const cuuint32_t eb[3] = {(cuuint32_t)rw, (cuuint32_t)by, 1};
    return fn(em, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(E), ed, es, eb, one,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tile shapes the autotuner chooses from: CTA of BX x BY element columns, MINB CTAs per SM, ring depth;
// planes staged by per-thread cp.async (ModalShape) or by the Tensor Memory Accelerator (TmaShape).
// launch() returns false when the shape cannot run on these buffers (no tensor map could be made).
template <int BX, int BY, int MINB, int ST, int PACK = 0>
struct ModalShape {
    static constexpr int bx = BX, by = BY, stages = ST, packed = PACK, tma = 0;
    static constexpr size_t smem = sizeof(ModalSmem<BX, BY, ST>);
    static const void* fn() { return reinterpret_cast<const void*>(k_matvec32_modal<BX, BY, MINB, ST, PACK>); }
    static bool launch(const Grid& g, const ModalKe& kh, const ModalTiling& t, const float* E, const uint8_t* mask,
                       const float* u, float* y, RedSlot dot, PcgScalars* S, int mark, int* err, cudaStream_t s) {
        (void)err;
        k_matvec32_modal<BX, BY, MINB, ST, PACK><<<t.grid, BX * BY, smem, s>>>(g, kh, t, E, mask, u, y, dot, S, mark);
        return true;
    }
};
template <int BX, int BY, int MINB, int ST>
struct TmaShape {
    using SM = TmaSmem<BX, BY, ST>;
    static constexpr int bx = BX, by = BY, stages = ST, packed = 1, tma = 1;
    static constexpr size_t smem = sizeof(SM) + 128;   // + slack for the 128-byte alignment of the ring
    static const void* fn() { return reinterpret_cast<const void*>(k_matvec32_tma<BX, BY, MINB, ST>); }
    static const void* fn_batched(int mode) {
        return mode == 0   ? reinterpret_cast<const void*>(k_matvec32_tma_batched<BX, BY, MINB, ST, 0>)
               : mode == 1 ? reinterpret_cast<const void*>(k_matvec32_tma_batched<BX, BY, MINB, ST, 1>)
                           : reinterpret_cast<const void*>(k_matvec32_tma_batched<BX, BY, MINB, ST, 2>);
    }
    static bool maps(const Grid& g, const float* u, const float* E, CUtensorMap* um, CUtensorMap* em) {
        return modal_tensor_maps(g, u, E, SM::RW, SM::PY, BY, um, em);
    }
    static void batched(int mode, const BatchMatvec* a, const int* act, int N, const ModalKe& kh, int grid, int* err,
                        cudaStream_t s) {
        if (mode == 0) k_matvec32_tma_batched<BX, BY, MINB, ST, 0><<<grid, BX * BY, smem, s>>>(a, act, N, kh, err);
        else if (mode == 1) k_matvec32_tma_batched<BX, BY, MINB, ST, 1><<<grid, BX * BY, smem, s>>>(a, act, N, kh, err);
        else k_matvec32_tma_batched<BX, BY, MINB, ST, 2><<<grid, BX * BY, smem, s>>>(a, act, N, kh, err);
    }
    static bool launch(const Grid& g, const ModalKe& kh, const ModalTiling& t, const float* E, const uint8_t* mask,
                       const float* u, float* y, RedSlot dot, PcgScalars* S, int mark, int* err, cudaStream_t s) {
        CUtensorMap um, em;
        if (!modal_tensor_maps(g, u, E, SM::RW, SM::PY, BY, &um, &em)) return false;
        k_matvec32_tma<BX, BY, MINB, ST, 0><<<t.grid, BX * BY, smem, s>>>(um, em, g, kh, t, mask, y, dot, S, mark, err,
                                                                         nullptr, nullptr, 0.0f);
        return true;
    }
    static const void* fn_mode(int mode) {
        return mode == 1 ? reinterpret_cast<const void*>(k_matvec32_tma<BX, BY, MINB, ST, 1>)
                         : reinterpret_cast<const void*>(k_matvec32_tma<BX, BY, MINB, ST, 2>);
    }
    static bool fused(int mode, const Grid& g, const ModalKe& kh, const ModalTiling& t, const float* E,
                      const uint8_t* mask, const float* u, float* y, const float* r, const float* rd, float w,
                      RedSlot dot, PcgScalars* S, int* err, cudaStream_t s) {
        CUtensorMap um, em;
        if (!modal_tensor_maps(g, u, E, SM::RW, SM::PY, BY, &um, &em)) return false;
        if (mode == 1)
            k_matvec32_tma<BX, BY, MINB, ST, 1><<<t.grid, BX * BY, smem, s>>>(um, em, g, kh, t, mask, y, dot, S, 0, err,
                                                                             r, rd, w);
        else
            k_matvec32_tma<BX, BY, MINB, ST, 2><<<t.grid, BX * BY, smem, s>>>(um, em, g, kh, t, mask, y, dot, S, 0, err,
                                                                             r, rd, w);
        return true;
    }
};
struct ModalVariant {
    int bx, by, stages, packed, tma;
    size_t smem;
    const void* (*fn)();
    bool (*launch)(const Grid&, const ModalKe&, const ModalTiling&, const float*, const uint8_t*, const float*,
                   float*, RedSlot, PcgScalars*, int, int*, cudaStream_t);
    // the fused Standard-cycle epilogues (TMA shapes only)
    const void* (*fn_mode)(int);
    bool (*fused)(int, const Grid&, const ModalKe&, const ModalTiling&, const float*, const uint8_t*, const float*,
                  float*, const float*, const float*, float, RedSlot, PcgScalars*, int*, cudaStream_t);
    // the batched PCG product over many instances (TMA shapes only)
    const void* (*fn_batched)(int);
    bool (*maps)(const Grid&, const float*, const float*, CUtensorMap*, CUtensorMap*);
    void (*batched)(int, const BatchMatvec*, const int*, int, const ModalKe&, int, int*, cudaStream_t);
};
template <class V>
constexpr ModalVariant variant_of() {
    if constexpr (V::tma)
        return ModalVariant{V::bx, V::by, V::stages, V::packed, V::tma, V::smem, &V::fn, &V::launch, &V::fn_mode,
                            &V::fused, &V::fn_batched, &V::maps, &V::batched};
    else
        return ModalVariant{V::bx, V::by, V::stages, V::packed, V::tma, V::smem, &V::fn, &V::launch, nullptr, nullptr,
                            nullptr, nullptr, nullptr};
}
const ModalVariant MODAL_VARIANTS[] = {
    variant_of<ModalShape<32, 8, 2, 4, 1>>(),   // variant 0: the fallback of a TMA shape without tensor maps
    variant_of<ModalShape<32, 8, 2, 4>>(),
    variant_of<ModalShape<32, 8, 2, 3>>(),
    variant_of<ModalShape<32, 8, 3, 3>>(),
    variant_of<ModalShape<32, 16, 2, 3>>(),
    variant_of<ModalShape<32, 16, 1, 4>>(),
    variant_of<TmaShape<32, 8, 2, 4>>(),
    variant_of<TmaShape<32, 8, 3, 3>>(),
    variant_of<TmaShape<32, 16, 1, 4>>(),
    variant_of<TmaShape<32, 16, 2, 3>>(),
};
constexpr int MODAL_NVARIANTS = sizeof(MODAL_VARIANTS) / sizeof(MODAL_VARIANTS[0]);
constexpr int MODAL_SLAB_MIN = 8;

// corner a of the reference's local order at grid offset (corner_dx, corner_dy, corner_dz)(a);
// T8[a][m] = s_x^i s_y^j s_z^k with s = 2 d - 1 and mode m = i + 2 j + 4 k
bool modal_ke_from(const double* Ke, ModalKe* out, double* off) {
    double T8[8][8];
    for (int a = 0; a < 8; ++a) {
        const int s[3] = {2 * corner_dx(a) - 1, 2 * corner_dy(a) - 1, 2 * corner_dz(a) - 1};
        for (int m = 0; m < 8; ++m)
            T8[a][m] = (double)((m & 1 ? s[0] : 1) * (m & 2 ? s[1] : 1) * (m & 4 ? s[2] : 1));
    }
    // Kh[(c,m)][(e,n)] = sum_{a,b} T8[a][m] Ke[3a+c][3b+e] T8[b][n] / 64, index comp*8 + mode
    // (local: contexts may be created concurrently from several host threads)
    double Kh[24][24];
    double mx = 0.0;
    for (int c = 0; c < 3; ++c)
        for (int m = 0; m < 8; ++m)
            for (int e = 0; e < 3; ++e)
                for (int n = 0; n < 8; ++n) {
                    double acc = 0.0;
                    for (int a = 0; a < 8; ++a)
                        for (int b = 0; b < 8; ++b) acc += T8[a][m] * Ke[(3 * a + c) * 24 + 3 * b + e] * T8[b][n];
                    Kh[c * 8 + m][e * 8 + n] = acc / 64.0;
                    mx = std::fmax(mx, std::fabs(acc / 64.0));
                }
    bool in[24][24] = {};
    for (int k = 0; k < 45; ++k) {
        in[KH_PATTERN_HOST[k].dst][KH_PATTERN_HOST[k].src] = true;
        out->v[k] = (float)Kh[KH_PATTERN_HOST[k].dst][KH_PATTERN_HOST[k].src];
    }
    double worst = 0.0;
    for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j)
            if (!in[i][j]) worst = std::fmax(worst, std::fabs(Kh[i][j]));
    *off = mx > 0.0 ? worst / mx : 1.0;
    return mx > 0.0 && *off <= 1e-10;
}

void modal_variant_desc(int variant, int out[4]) {
    const ModalVariant& v = MODAL_VARIANTS[variant < 0 || variant >= MODAL_NVARIANTS ? 0 : variant];
    out[0] = v.bx;
    out[1] = v.by;
    out[2] = v.stages;
    out[3] = v.tma ? 2 : v.packed;
}

int modal_tiling(const Grid& g, int dev, int variant, ModalTiling* t) {
    if (variant < 0 || variant >= MODAL_NVARIANTS) return set_error(T3D_ERR_INVALID, "bad modal tile variant");
    const ModalVariant& v = MODAL_VARIANTS[variant];
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaDeviceGetAttribute", __FILE__, __LINE__);
    e = cudaFuncSetAttribute(v.fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaFuncSetAttribute", __FILE__, __LINE__);
    for (int mode = 1; v.fn_mode && mode <= 2; ++mode) {
        e = cudaFuncSetAttribute(v.fn_mode(mode), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem);
        if (e != cudaSuccess) return set_cuda_error(e, "cudaFuncSetAttribute", __FILE__, __LINE__);
    }
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn(), v.bx * v.by, v.smem);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor", __FILE__, __LINE__);
    const int resident = std::max(1, std::min(sms * std::max(per_sm, 1), RED_BLOCKS));
    t->variant = variant;
    t->tiles_x = (g.nnx + v.bx - 2) / (v.bx - 1);
    t->tiles_y = (g.nny + v.by - 2) / (v.by - 1);
    const int tiles = t->tiles_x * t->tiles_y;
    // slabs: enough work items for about 8 waves of the resident CTAs, slabs of at least 8 planes
    int slabs = std::max(1, (8 * resident + tiles - 1) / tiles);
    slabs = std::min(slabs, std::max(1, g.nnz / MODAL_SLAB_MIN));
    t->slab = (g.nnz + slabs - 1) / slabs;
    t->slabs = (g.nnz + t->slab - 1) / t->slab;
    t->items = tiles * t->slabs;
    t->grid = std::min(resident, t->items);
    return 0;
}

// The choice is cached per (device, grid) for the life of the process, so that every context of one grid
// size uses the same tile shape: results then do not depend on which contexts ran before or beside it
// (the shape fixes the block order of the FP64 p.Ap partial sums).
int modal_autotune(const Grid& g, int dev, const ModalKe& kh, const float* E, const uint8_t* mask, const float* u,
                   float* y, int* err, cudaStream_t s, ModalTiling* best) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int>, ModalTiling> cache;
    const auto key = std::make_tuple(dev, g.nx, g.ny, g.nz);
    std::lock_guard<std::mutex> lock(mu);
    const auto hit = cache.find(key);
    if (hit != cache.end()) {
        *best = hit->second;
        return modal_tiling(g, dev, best->variant, best);   // sets the shared-memory attribute on this device
    }
    cudaEvent_t e0, e1;
    cudaError_t e = cudaEventCreate(&e0);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaEventCreate", __FILE__, __LINE__);
    e = cudaEventCreate(&e1);
    if (e != cudaSuccess) {
        cudaEventDestroy(e0);
        return set_cuda_error(e, "cudaEventCreate", __FILE__, __LINE__);
    }
    float best_ms = 0.f;
    int rc = 0;
    bool have = false;
    for (int v = 0; v < MODAL_NVARIANTS && rc == 0; ++v) {
        ModalTiling t{};
        if ((rc = modal_tiling(g, dev, v, &t)) != 0) break;
        const RedSlot none{nullptr, nullptr};
        if (!MODAL_VARIANTS[v].launch(g, kh, t, E, mask, u, y, none, nullptr, 0, err, s)) continue;   // warm-up
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3; ++r) MODAL_VARIANTS[v].launch(g, kh, t, E, mask, u, y, none, nullptr, 0, err, s);
        cudaEventRecord(e1, s);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) {
            rc = set_cuda_error(e, "modal autotune", __FILE__, __LINE__);
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (!have || ms < best_ms) {
            best_ms = ms;
            *best = t;
            have = true;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == 0) cache[key] = *best;
    return rc;
}

bool modal_fused_available(const ModalTiling& t) {
    return t.variant >= 0 && t.variant < MODAL_NVARIANTS && MODAL_VARIANTS[t.variant].fused != nullptr;
}

bool launch_matvec32_fused(int mode, const Grid& g, const ModalKe& kh, const ModalTiling& t, const float* E,
                           const uint8_t* mask, const float* u, float* y, const float* r, const float* rd, float w,
                           RedSlot dot, PcgScalars* S, int* err, cudaStream_t s) {
    const ModalVariant& v = MODAL_VARIANTS[t.variant];
    return v.fused != nullptr && v.fused(mode, g, kh, t, E, mask, u, y, r, rd, w, dot, S, err, s);
}

bool modal_batched_available(int variant) {
    return variant >= 0 && variant < MODAL_NVARIANTS && MODAL_VARIANTS[variant].batched != nullptr;
}

// resident CTAs of the batched kernel on this device (its persistent grid); sets its shared-memory size
int modal_batched_grid(int variant, int dev, int* grid) {
    if (!modal_batched_available(variant)) return set_error(T3D_ERR_INVALID, "tile shape has no batched form");
    const ModalVariant& v = MODAL_VARIANTS[variant];
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaDeviceGetAttribute", __FILE__, __LINE__);
    for (int mode = 0; mode <= 2; ++mode) {
        e = cudaFuncSetAttribute(v.fn_batched(mode), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem);
        if (e != cudaSuccess) return set_cuda_error(e, "cudaFuncSetAttribute", __FILE__, __LINE__);
    }
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn_batched(0), v.bx * v.by, v.smem);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor", __FILE__, __LINE__);
    *grid = std::max(1, sms * std::max(per_sm, 1));
    return T3D_OK;
}

bool modal_tensor_maps_for(int variant, const Grid& g, const float* u, const float* E, CUtensorMap* umap,
                           CUtensorMap* emap) {
    return modal_batched_available(variant) && MODAL_VARIANTS[variant].maps(g, u, E, umap, emap);
}

bool launch_batch_matvec32(int variant, int mode, const BatchMatvec* a, const int* act, int N, const ModalKe& kh,
                           int grid, int* err, cudaStream_t s) {
    if (!modal_batched_available(variant) || N <= 0) return false;
    MODAL_VARIANTS[variant].batched(mode, a, act, N, kh, grid, err, s);
    return true;
}

void launch_matvec32_modal(const Grid& g, const ModalKe& kh, const ModalTiling& t, const float* E,
                           const uint8_t* mask, const float* u, float* y, RedSlot dot, PcgScalars* S, int mark,
                           int* err, cudaStream_t s) {
    if (MODAL_VARIANTS[t.variant].launch(g, kh, t, E, mask, u, y, dot, S, mark, err, s)) return;
    // no tensor map for these buffers: the cp.async form of the same arithmetic (bit-identical results)
    ModalTiling t0 = t;
    int dev = 0;
    cudaGetDevice(&dev);
    modal_tiling(g, dev, 0, &t0);
    MODAL_VARIANTS[0].launch(g, kh, t0, E, mask, u, y, dot, S, mark, err, s);
}

}  // namespace t3d
