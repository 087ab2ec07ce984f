// K(E) u in FP64, element-streaming, bit-identical to the node-centric k_matvec64 (and so to the oracle).
//
// k_matvec64 gathers, for every node, the 24 values of each of its 8 elements (192 loads per node) and
// runs the 24-term FMA chain of the node's 3 rows of Ke; that form is L1-bound.  Here each element's 24
// values are gathered once and all 8 x 3 chains of the element are run in the same operation order
// (f = fma(Ke[row][j], u_e[j], f), j = 0..23); each node then adds its 8 element contributions in the
// reference's colour order (colour = ex&1 | (ey&1)<<1 | (ez&1)<<2, fea.cpp:300), y = fma(f, E, y),
// skipping E <= 1e-16, exactly as k_matvec64 does.  Only the place where each chain runs changes.
//
// Streaming: a CTA of BX x BY threads (one element column each) owns a (BX-1) x (BY-1) tile of node
// columns and marches up a slab of node planes; node planes come through a 3-slot cp.async ring in
// shared memory (the plane below stays in the ring while the plane above arrives).  Per element layer
// the chains' results for the bottom and top corners go to shared memory; each owned node folds its 4
// same-layer elements in colour order and carries the other layer's part to the next plane (a partial
// sum when that layer comes first in the node's colour order, the 4 raw triples otherwise).
// Coefficients: a DFMA whose coefficient is a constant-bank operand issues at about half the rate of
// one with register operands only, and a shared-memory broadcast of FP64 coefficients costs more than
// the DFMAs it feeds.  The built-in Ke has only KE_ND distinct magnitudes (ke_pattern.inc), so for it
// (PAT) they sit in registers and each coefficient is +-D[ke_idx(i)] (negation is an exact operand
// modifier); the 24 rows of a column run in ke_row_order so that consecutive DFMAs share a coefficient
// register.  Any other Ke (t3d_set_ke) is passed by value and read from the constant bank.
// p.Ap is not fused: the caller folds it in the canonical order.
#include <algorithm>
#include <cmath>

#include "kernels.hpp"
#include "ke_pattern.inc"
#include "red.cuh"
#include "t3d_b200.h"

namespace t3d {

namespace {

__device__ __forceinline__ void cp_async8(unsigned s, const double* gsrc, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }


static_assert(KE_ND <= KE_MAX_DISTINCT, "distinct-magnitude buffer too small");

constexpr int S64_BX = 32;
constexpr int S64_BY = 8;
constexpr int S64_SLAB_MIN = 16;   // planes per slab at least (the slab's first element layer is computed twice)

// Shared-memory layout of one CTA, in doubles.
struct S64 {
    static constexpr int BX = S64_BX, BY = S64_BY, PX = BX + 1, PY = BY + 1, NT = BX * BY;
    static constexpr int PLANE = 0;                     // [3 ring slots][3 components][PY][PX]
    static constexpr int PLANE_SZ = 3 * PY * PX;
    static constexpr int EMOD = PLANE + 3 * PLANE_SZ;   // [3 ring slots][BY][BX]: E of one element layer
    static constexpr int FB = EMOD + 3 * NT;            // [12][BY][BX]: rows 3a+r, corners a = 0..3
    static constexpr int FT = FB + 12 * NT;             // [2 layer parity][12][BY][BX]: rows 3(a-4)+r, a = 4..7
    static constexpr int TOTAL = FT + 24 * NT;
    static constexpr size_t BYTES = TOTAL * sizeof(double);
};

__device__ __forceinline__ unsigned smem_addr(const double* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

// footprint of node plane iz, (PX x PY) nodes from (X0-1, Y0-1), 3 components, zero outside the grid
__device__ __forceinline__ void load_plane(const Grid& g, const double* __restrict__ u, int X0, int Y0, int iz,
                                           double* dst) {
    constexpr int AREA = S64::PY * S64::PX;
    const bool zok = iz >= 0 && iz < g.nnz;
    for (int i = threadIdx.x; i < 3 * AREA; i += S64::NT) {
        const int c = i / AREA, rem = i - c * AREA, py = rem / S64::PX, px = rem - py * S64::PX;
        const int ix = X0 - 1 + px, iy = Y0 - 1 + py;
        const bool ok = zok && ix >= 0 && ix < g.nnx && iy >= 0 && iy < g.nny;
        const double* src = ok ? u + c * g.NN + g.node(ix, iy, iz) : u;
        cp_async8(smem_addr(dst + i), src, ok);
    }
}

// E of element layer cz over the tile's BX x BY element columns from cell (X0-1, Y0-1); cells beyond
// the ghost ring read as 0 (they are skipped like the ghosts)
__device__ __forceinline__ void load_emod(const Grid& g, const double* __restrict__ E, int X0, int Y0, int cz,
                                          double* dst) {
    const int tx = threadIdx.x % S64::BX, ty = threadIdx.x / S64::BX;
    const int cx = X0 - 1 + tx, cy = Y0 - 1 + ty;
    const bool ok = cx <= g.nx && cy <= g.ny;
    cp_async8(smem_addr(dst + threadIdx.x), ok ? E + g.cell(cx, cy, cz) : E, ok);
}

template <bool PAT>
__global__ void __launch_bounds__(S64::NT, 2) k_matvec64_stream(Grid g, Stream64Tiling t, const Ke64 ke,
                                                                const double* __restrict__ Kd,
                                                                const double* __restrict__ E,
                                                                const uint8_t* __restrict__ mask,
                                                                const double* __restrict__ u,
                                                                double* __restrict__ y, const PcgScalars* S) {
    extern __shared__ __align__(16) double sm[];
    if (S != nullptr && S->done) return;
    constexpr int BX = S64::BX, BY = S64::BY, NT = S64::NT, PX = S64::PX, AREA = S64::PY * S64::PX;
    double* Fb = sm + S64::FB;
    const int tx = threadIdx.x % BX, ty = threadIdx.x / BX;
    const int64_t NN = g.NN;
    double D[PAT ? KE_ND : 1];   // PAT: the distinct magnitudes of Ke, loaded once into registers
#pragma unroll
    for (int d = 0; d < (PAT ? KE_ND : 1); ++d) D[d] = PAT ? __ldg(Kd + d) : 0.0;

    for (int w = blockIdx.x; w < t.items; w += gridDim.x) {
        const int tix = w % t.tiles_x, rest = w / t.tiles_x;
        const int tiy = rest % t.tiles_y, sl = rest / t.tiles_y;
        const int X0 = tix * (BX - 1), Y0 = tiy * (BY - 1);
        const int Z0 = sl * t.slab, Z1 = min(Z0 + t.slab, g.nnz);
        const int nlay = Z1 - Z0 + 1;   // element layers Z0-1 .. Z1-1
        __syncthreads();                // the previous item's owners are done with the rings
        load_plane(g, u, X0, Y0, Z0 - 1, sm + S64::PLANE);
        load_plane(g, u, X0, Y0, Z0, sm + S64::PLANE + S64::PLANE_SZ);
        load_emod(g, E, X0, Y0, Z0 - 1, sm + S64::EMOD);
        cp_commit();
#pragma unroll 1
        for (int k = 0; k < nlay; ++k) {
            const int cz = Z0 - 1 + k;   // element layer between node planes cz and cz+1
            cp_wait0();
            __syncthreads();
            if (k + 1 < nlay) {          // node plane cz+2 and the E of layer cz+1 for the next step
                load_plane(g, u, X0, Y0, cz + 2, sm + S64::PLANE + ((k + 2) % 3) * S64::PLANE_SZ);
                load_emod(g, E, X0, Y0, cz + 1, sm + S64::EMOD + ((k + 1) % 3) * NT);
            }
            cp_commit();
            // ---- element (tx, ty) of layer cz: the 24 FMA chains f_row = fma(Ke[row][j], u_e[j], f_row), j = 0..23
            double* Ft = sm + S64::FT + (k & 1) * 12 * NT;
            const double Ee = sm[S64::EMOD + (k % 3) * NT + threadIdx.x];
            if (PAT && !(Ee <= 1.0e-16)) {   // the owners skip exactly the elements skipped here
                const double* Pb = sm + S64::PLANE + (k % 3) * S64::PLANE_SZ;
                const double* Pt = sm + S64::PLANE + ((k + 1) % 3) * S64::PLANE_SZ;
                double f[24];
#pragma unroll
                for (int q = 0; q < 24; ++q) f[q] = 0.0;
#pragma unroll
                for (int j = 0; j < 24; ++j) {
                    const int a = j / 3, c = j % 3;
                    const double uj = (a < 4 ? Pb : Pt)[c * AREA + (ty + corner_dy(a)) * PX + tx + corner_dx(a)];
#pragma unroll
                    for (int r = 0; r < 24; ++r) {
                        const int q = ke_row_order(24 * j + r), i = 24 * q + j;
                        f[q] = fma(ke_neg(i) ? -D[ke_idx(i)] : D[ke_idx(i)], uj, f[q]);
                    }
                }
#pragma unroll
                for (int q = 0; q < 12; ++q) Fb[q * NT + threadIdx.x] = f[q];
#pragma unroll
                for (int q = 0; q < 12; ++q) Ft[q * NT + threadIdx.x] = f[12 + q];
            } else if (!PAT && !(Ee <= 1.0e-16)) {   // any Ke: two halves of 12 rows, coefficients from the constant bank
                const double* Pb = sm + S64::PLANE + (k % 3) * S64::PLANE_SZ;
                const double* Pt = sm + S64::PLANE + ((k + 1) % 3) * S64::PLANE_SZ;
                double ue[24];
#pragma unroll
                for (int a = 0; a < 8; ++a) {
                    const double* P = a < 4 ? Pb : Pt;
                    const int o = (ty + corner_dy(a)) * PX + tx + corner_dx(a);
#pragma unroll
                    for (int c = 0; c < 3; ++c) ue[3 * a + c] = P[c * AREA + o];
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    double f[12];
#pragma unroll
                    for (int q = 0; q < 12; ++q) f[q] = 0.0;
#pragma unroll
                    for (int j = 0; j < 24; ++j)
#pragma unroll
                        for (int q = 0; q < 12; ++q) f[q] = fma(ke.v[(12 * h + q) * 24 + j], ue[j], f[q]);
                    double* F = h == 0 ? Fb : Ft;
#pragma unroll
                    for (int q = 0; q < 12; ++q) F[q * NT + threadIdx.x] = f[q];
                }
            }
            __syncthreads();
            // ---- owners finish node plane iz = cz: 8 elements in colour order, even element layer first
            if (k >= 1 && tx < BX - 1 && ty < BY - 1) {
                const int ix = X0 + tx, iy = Y0 + ty, iz = cz;
                if (ix < g.nnx && iy < g.nny) {
                    const double* Ebelow = sm + S64::EMOD + ((k - 1) % 3) * NT;
                    const double* Eabove = sm + S64::EMOD + (k % 3) * NT;
                    const double* Fbelow = sm + S64::FT + ((k - 1) & 1) * 12 * NT;
                    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
#pragma unroll
                    for (int col = 0; col < 8; ++col) {
                        const int sx = (((ix - 1) & 1) == (col & 1)) ? 0 : 1;   // element column tx+sx: cx = ix-1+sx
                        const int sy = (((g.ny - iy) & 1) == ((col >> 1) & 1)) ? 0 : 1;
                        const int sz = (((iz - 1) & 1) == ((col >> 2) & 1)) ? 0 : 1;   // 0: layer iz-1, 1: layer iz
                        const int e = (ty + sy) * BX + tx + sx;
                        const double Ec = sz ? Eabove[e] : Ebelow[e];
                        if (Ec <= 1.0e-16) continue;
                        const int a = corner_of(1 - sx, 1 - sy, 1 - sz);
                        const double* F = sz ? Fb + 3 * a * NT : Fbelow + 3 * (a - 4) * NT;
                        y0 = fma(F[e], Ec, y0);
                        y1 = fma(F[NT + e], Ec, y1);
                        y2 = fma(F[2 * NT + e], Ec, y2);
                    }
                    const int64_t n = g.node(ix, iy, iz);
                    const int mk = mask[n];
                    if (mk & 1) y0 = 0.0;
                    if (mk & 2) y1 = 0.0;
                    if (mk & 4) y2 = 0.0;
                    y[n] = y0;
                    y[NN + n] = y1;
                    y[2 * NN + n] = y2;
                }
            }
        }
    }
    cp_wait0();
}

// p.Ap in the canonical order of k_dot (the fused dot of the node-centric kernel), skipped once S->done
__global__ void __launch_bounds__(RED_THREADS) k_dot_pcg(Grid g, const double* __restrict__ a,
                                                         const double* __restrict__ b, RedSlot red, PcgScalars* S) {
    __shared__ double sh[32];
    if (S->done) return;
    const int NN = (int)g.NN;
    double part = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c) part = part + a[c * (int64_t)NN + n] * b[c * (int64_t)NN + n];
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) S->denom = tot;
}

}  // namespace

bool ke_pattern_magnitudes(const double* Ke, double* D) {
    for (int d = 0; d < KE_ND; ++d) D[d] = std::fabs(Ke[ke_first(d)]);
    for (int i = 0; i < 576; ++i)
        if (Ke[i] != (ke_neg(i) ? -D[ke_idx(i)] : D[ke_idx(i)])) return false;
    return true;
}

int stream64_tiling(const Grid& g, int dev, Stream64Tiling* t) {
    int per_sm = 1 << 30, sms = 0;
    for (auto fn : {k_matvec64_stream<true>, k_matvec64_stream<false>}) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S64::BYTES);
        if (e != cudaSuccess) return set_cuda_error(e, "cudaFuncSetAttribute", __FILE__, __LINE__);
        int n = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, S64::NT, S64::BYTES);
        if (e != cudaSuccess)
            return set_cuda_error(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor", __FILE__, __LINE__);
        per_sm = std::min(per_sm, n);
    }
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaDeviceGetAttribute", __FILE__, __LINE__);
    if (per_sm < 1) return set_error(T3D_ERR_CUDA, "FP64 streaming K(E)u does not fit on an SM");
    const int resident = per_sm * sms;
    t->tiles_x = (g.nnx + S64::BX - 2) / (S64::BX - 1);
    t->tiles_y = (g.nny + S64::BY - 2) / (S64::BY - 1);
    const int tiles = t->tiles_x * t->tiles_y;
    // slabs: about 8 waves of the resident CTAs, slabs of at least S64_SLAB_MIN planes
    int slabs = std::max(1, (8 * resident + tiles - 1) / tiles);
    slabs = std::min(slabs, std::max(1, g.nnz / S64_SLAB_MIN));
    t->slab = (g.nnz + slabs - 1) / slabs;
    t->slabs = (g.nnz + t->slab - 1) / t->slab;
    t->items = tiles * t->slabs;
    t->grid = std::min(resident, t->items);
    return T3D_OK;
}

void launch_matvec64_stream(const Grid& g, const Stream64Tiling& t, const double* Ke_host, const double* Kd,
                            const double* E, const uint8_t* mask, const double* u, double* y, const PcgScalars* S,
                            cudaStream_t s) {
    if (Kd) {   // the by-value Ke is not read in this form
        static const Ke64 unused{};
        k_matvec64_stream<true><<<t.grid, S64::NT, S64::BYTES, s>>>(g, t, unused, Kd, E, mask, u, y, S);
        return;
    }
    Ke64 ke;
    for (int i = 0; i < 576; ++i) ke.v[i] = Ke_host[i];
    k_matvec64_stream<false><<<t.grid, S64::NT, S64::BYTES, s>>>(g, t, ke, nullptr, E, mask, u, y, S);
}

void launch_dot_pcg(const Grid& g, const double* p, const double* Ap, RedSlot red, PcgScalars* S, cudaStream_t s) {
    k_dot_pcg<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, p, Ap, red, S);
}

}  // namespace t3d
