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
#include <algorithm>
#include <cmath>

#include "kernels.hpp"
#include "red.cuh"

namespace t3d {

namespace {

// modal index = component * 8 + mode, mode bit 0 = x, bit 1 = y, bit 2 = z (constant mode 0 unused)
// X(dst, src) for each of the 45 nonzeros, in the order of ModalKe::v
#define T3D_KH_PATTERN(X)                                                                          \
    /* normal strains: (0,x) (1,y) (2,z) */                                                        \
    X(1, 1) X(1, 10) X(1, 20) X(10, 1) X(10, 10) X(10, 20) X(20, 1) X(20, 10) X(20, 20)            \
    /* shears xy, xz, yz */                                                                        \
    X(9, 9) X(9, 2) X(2, 9) X(2, 2) X(17, 17) X(17, 4) X(4, 17) X(4, 4)                            \
    X(18, 18) X(18, 12) X(12, 18) X(12, 12)                                                        \
    /* bilinear pairs */                                                                           \
    X(3, 3) X(3, 22) X(22, 3) X(22, 22) X(11, 11) X(11, 21) X(21, 11) X(21, 21)                    \
    X(5, 5) X(5, 14) X(14, 5) X(14, 14)                                                            \
    /* bilinear triple (2,xy) (1,xz) (0,yz) */                                                     \
    X(19, 19) X(19, 13) X(19, 6) X(13, 19) X(13, 13) X(13, 6) X(6, 19) X(6, 13) X(6, 6)            \
    /* trilinear */                                                                                \
    X(7, 7) X(15, 15) X(23, 23)

struct KhEntry {
    int dst, src;
};
#define T3D_KH_ENTRY(d, s) {d, s},
constexpr KhEntry KH_PATTERN_HOST[45] = {T3D_KH_PATTERN(T3D_KH_ENTRY)};
#undef T3D_KH_ENTRY

// x-y Hadamard stage of one component on one node plane: corners (dx,dy) -> modes (i,j)
struct Modes2 {
    float m00, m10, m01, m11;
};

__device__ __forceinline__ Modes2 fwd2(float u00, float u10, float u01, float u11) {
    const float s0 = u00 + u10, d0 = u10 - u00, s1 = u01 + u11, d1 = u11 - u01;
    return Modes2{s0 + s1, d0 + d1, s1 - s0, d1 - d0};
}

// inverse x-y stage: modes (i,j) -> corner values (dx,dy) = sum s_x^i s_y^j w_ij
__device__ __forceinline__ void inv2(const Modes2& w, float& v00, float& v10, float& v01, float& v11) {
    const float p = w.m00 - w.m01, q = w.m10 - w.m11, pp = w.m00 + w.m01, qq = w.m10 + w.m11;
    v00 = p - q;
    v10 = p + q;
    v01 = pp - qq;
    v11 = pp + qq;
}

__device__ __forceinline__ float4 ld_node(const float* __restrict__ u0, const float* __restrict__ u1,
                                          const float* __restrict__ u2, const Grid& g, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= g.nnx || y >= g.nny || z >= g.nnz) return make_float4(0.f, 0.f, 0.f, 0.f);
    const int64_t n = g.node(x, y, z);
    return make_float4(__ldg(u0 + n), __ldg(u1 + n), __ldg(u2 + n), 0.f);
}

}  // namespace

template <int BX, int BY, int MINB>
__global__ void __launch_bounds__(BX * BY, MINB)
    k_matvec32_modal(Grid g, ModalKe kh, ModalTiling t, const float* __restrict__ E,
                     const uint8_t* __restrict__ mask, const float* __restrict__ u, float* __restrict__ y,
                     RedSlot dot, PcgScalars* S) {
    constexpr int PX = BX + 1, PY = BY + 1;
    static_assert(PY <= BX, "the footprint column is loaded by one warp-row of BX threads");
    __shared__ float4 plane[PY][PX];        // node plane footprint (c0, c1, c2, -)
    __shared__ float4 outc[4][BY][BX];      // corner (dx + 2 dy) contributions of each element column
    __shared__ double sh[32];
    if (S != nullptr && S->done) return;
    const int tx = threadIdx.x % BX, ty = threadIdx.x / BX;
    const int64_t NN = g.NN;
    const float* __restrict__ u0 = u;
    const float* __restrict__ u1 = u + NN;
    const float* __restrict__ u2 = u + 2 * NN;
    // besides its own node, thread row 0 loads the footprint's last row, thread row 1 its last column
    const int ex_kind = (ty == 0) ? 1 : ((ty == 1 && tx < PY) ? 2 : 0);
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
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
        const bool owner = tx > 0 && ty > 0 && cx < g.nnx && cy < g.nny;
        const bool e_in = cx <= g.nx && cy <= g.ny;             // inside the cell array (ghost ring included)
        float4 own = ld_node(u0, u1, u2, g, cx, cy, Z0 - 1);
        float4 ext = ex_kind ? ld_node(u0, u1, u2, g, exx, exy, Z0 - 1) : zero4;
        float4 own_prev = zero4;
        Modes2 bot[3], acc[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) acc[k] = Modes2{0.f, 0.f, 0.f, 0.f};
        for (int pz = Z0 - 1; pz <= Z1; ++pz) {
            plane[ty][tx] = own;
            if (ex_kind == 1) plane[BY][tx] = ext;
            else if (ex_kind == 2) plane[tx][BX] = ext;
            const float4 cur = own;
            if (pz < Z1) {   // next plane into registers while this one is used
                own = ld_node(u0, u1, u2, g, cx, cy, pz + 1);
                if (ex_kind) ext = ld_node(u0, u1, u2, g, exx, exy, pz + 1);
            }
            __syncthreads();
            const float4 a = plane[ty][tx], b = plane[ty][tx + 1], c = plane[ty + 1][tx], d = plane[ty + 1][tx + 1];
            Modes2 top[3];
            top[0] = fwd2(a.x, b.x, c.x, d.x);
            top[1] = fwd2(a.y, b.y, c.y, d.y);
            top[2] = fwd2(a.z, b.z, c.z, d.z);
            const bool emit = pz - 1 >= Z0;                    // plane pz-1 is owned and now complete
            if (pz >= Z0) {                                    // element layer cz = pz-1
                const float Ee = e_in ? __ldg(E + g.cell(cx, cy, pz - 1)) : 0.f;
                float cm[24];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    cm[8 * k + 0] = 0.f;
                    cm[8 * k + 1] = Ee * (top[k].m10 + bot[k].m10);
                    cm[8 * k + 2] = Ee * (top[k].m01 + bot[k].m01);
                    cm[8 * k + 3] = Ee * (top[k].m11 + bot[k].m11);
                    cm[8 * k + 4] = Ee * (top[k].m00 - bot[k].m00);
                    cm[8 * k + 5] = Ee * (top[k].m10 - bot[k].m10);
                    cm[8 * k + 6] = Ee * (top[k].m01 - bot[k].m01);
                    cm[8 * k + 7] = Ee * (top[k].m11 - bot[k].m11);
                }
                float yh[24];
#pragma unroll
                for (int i = 0; i < 24; ++i) yh[i] = 0.f;
                {
                    int e = 0;
#define T3D_KH_FMA(d, s) yh[d] = fmaf(kh.v[e++], cm[s], yh[d]);
                    T3D_KH_PATTERN(T3D_KH_FMA)
#undef T3D_KH_FMA
                }
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float* q = yh + 8 * k;
                    const Modes2 tb{-q[4], q[1] - q[5], q[2] - q[6], q[3] - q[7]};   // onto plane pz-1
                    const Modes2 tt{q[4], q[1] + q[5], q[2] + q[6], q[3] + q[7]};    // onto plane pz
                    const Modes2 fin{acc[k].m00 + tb.m00, acc[k].m10 + tb.m10, acc[k].m01 + tb.m01,
                                     acc[k].m11 + tb.m11};
                    acc[k] = tt;
                    bot[k] = fin;   // reuse as the finished plane pz-1 (bot is replaced by top below)
                }
                if (emit) {
                    float v[3][4];
#pragma unroll
                    for (int k = 0; k < 3; ++k) inv2(bot[k], v[k][0], v[k][1], v[k][2], v[k][3]);
#pragma unroll
                    for (int q = 0; q < 4; ++q) outc[q][ty][tx] = make_float4(v[0][q], v[1][q], v[2][q], 0.f);
                }
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) bot[k] = top[k];
            __syncthreads();
            if (emit && owner) {
                const float4 s0 = outc[0][ty][tx], s1 = outc[1][ty][tx - 1], s2 = outc[2][ty - 1][tx],
                             s3 = outc[3][ty - 1][tx - 1];
                float y0 = ((s0.x + s1.x) + s2.x) + s3.x;
                float y1 = ((s0.y + s1.y) + s2.y) + s3.y;
                float y2 = ((s0.z + s1.z) + s2.z) + s3.z;
                const int64_t n = g.node(cx, cy, pz - 1);
                const int mk = mask[n];
                if (mk & 1) y0 = 0.f;
                if (mk & 2) y1 = 0.f;
                if (mk & 4) y2 = 0.f;
                y[n] = y0;
                y[NN + n] = y1;
                y[2 * NN + n] = y2;
                if (dot.partial) {
                    part = fma((double)own_prev.x, (double)y0, part);
                    part = fma((double)own_prev.y, (double)y1, part);
                    part = fma((double)own_prev.z, (double)y2, part);
                }
            }
            own_prev = cur;
        }
    }
    if (dot.partial) {
        double tot;
        if (grid_fold(part, dot, sh, &tot) && threadIdx.x == 0) S->denom = tot;
    }
}

constexpr int MODAL_BX = 32, MODAL_BY = 16, MODAL_MINB = 2;
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
    static double Kh[24][24];
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

int modal_tiling(const Grid& g, int dev, ModalTiling* t) {
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaDeviceGetAttribute", __FILE__, __LINE__);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_matvec32_modal<MODAL_BX, MODAL_BY, MODAL_MINB>, MODAL_BX * MODAL_BY, 0);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor", __FILE__, __LINE__);
    const int resident = std::max(1, std::min(sms * std::max(per_sm, 1), RED_BLOCKS));
    t->tiles_x = (g.nnx + MODAL_BX - 2) / (MODAL_BX - 1);
    t->tiles_y = (g.nny + MODAL_BY - 2) / (MODAL_BY - 1);
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

void launch_matvec32_modal(const Grid& g, const ModalKe& kh, const ModalTiling& t, const float* E,
                           const uint8_t* mask, const float* u, float* y, RedSlot dot, PcgScalars* S,
                           cudaStream_t s) {
    k_matvec32_modal<MODAL_BX, MODAL_BY, MODAL_MINB>
        <<<t.grid, MODAL_BX * MODAL_BY, 0, s>>>(g, kh, t, E, mask, u, y, dot, S);
}

}  // namespace t3d
