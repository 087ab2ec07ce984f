// PDE (Helmholtz) filter kernels (filter.cpp:9-275): element->node load, the 8x8-kernel node
// operator, its Jacobi-PCG steps on device scalars, node->element average.
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

// Priority of a dimension in the Morton order of the 2x2x2 cells around a node: the highest bit in
// which the two candidate coordinates differ (= trailing zeros of the larger one), interleaved as
// 3*bit + {2 for x, 1 for y, 0 for z} (fea.cpp:61-67).  Larger coordinate = "upper" bit 1.
__device__ __forceinline__ int morton_priority(int upper, int offset) {
    return upper > 0 ? 3 * (__ffs(upper) - 1) + offset : -1;
}

// Visits the (up to 8) solid cells around node (ix,iy,iz) in increasing Morton key of their
// reference element coordinates (ex,ey,ez) = (cx, ny-1-cy, cz); f(cell_index, corner) is called
// for each.  This is the order in which the reference's element loops add into a node
// (filter.cpp:66-68, 177-182).
template <class F>
__device__ __forceinline__ void for_cells_morton(const Grid& g, const uint8_t* __restrict__ solid, int ix, int iy,
                                                 int iz, F f) {
    // upper coordinates: ex = ix (cell cx=ix), ey = ny-iy (cell cy=iy-1), ez = iz (cell cz=iz)
    const int px = morton_priority(ix, 2), py = morton_priority(g.ny - iy, 1), pz = morton_priority(iz, 0);
    int d[3] = {0, 1, 2};
    int p[3] = {px, py, pz};
    // sort dims by descending priority (priorities of distinct dims never tie)
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2 - a; ++b)
            if (p[b] < p[b + 1]) {
                int t = p[b]; p[b] = p[b + 1]; p[b + 1] = t;
                t = d[b]; d[b] = d[b + 1]; d[b + 1] = t;
            }
    for (int k = 0; k < 8; ++k) {
        int up[3];
        up[d[0]] = (k >> 2) & 1;
        up[d[1]] = (k >> 1) & 1;
        up[d[2]] = k & 1;
        const int cx = up[0] ? ix : ix - 1;
        const int cy = up[1] ? iy - 1 : iy;
        const int cz = up[2] ? iz : iz - 1;
        const int64_t ci = g.cell(cx, cy, cz);
        if (!solid[ci]) continue;
        f(ci, corner_of(ix - cx, iy - cy, iz - cz));
    }
}

// inverse row-sum preconditioner (filter.cpp:56-70)
__global__ void k_filter_diag(Grid g, const uint8_t* __restrict__ solid, const double* __restrict__ kf,
                              double* __restrict__ fdiag) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.NN) return;
    int ix, iy, iz;
    node_ijk(g, n, ix, iy, iz);
    double v = 0.0;
    for_cells_morton(g, solid, ix, iy, iz, [&](int64_t, int a) { v = v + kf[64 + a]; });
    fdiag[n] = v > 0 ? 1.0 / v : 1.0;
}

// rhs_n = sum over elements (Morton order) of (double)src_e * 1/8 (filter.cpp:177-182)
__global__ void k_filter_rhs(Grid g, const uint8_t* __restrict__ solid, const float* __restrict__ src,
                             double* __restrict__ rhs) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.NN) return;
    int ix, iy, iz;
    node_ijk(g, n, ix, iy, iz);
    double v = 0.0;
    for_cells_morton(g, solid, ix, iy, iz, [&](int64_t ci, int) { v = v + (double)src[ci] * (1.0 / 8.0); });
    rhs[n] = v;
}

// |rhs|, |rhs-lastRhs| and the warm-start decision (filter.cpp:185-199)
__global__ void __launch_bounds__(RED_THREADS) k_filter_norms(Grid g, const double* __restrict__ rhs,
                                                              const double* __restrict__ last, RedSlot r1,
                                                              RedSlot r2, FilterScalars* F) {
    __shared__ double sh[32];
    const int NN = (int)g.NN;
    double a = 0.0, b = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x) {
        const double v = rhs[n], d = v - last[n];
        a = a + v * v;
        b = b + d * d;
    }
    double ta, tb;
    const bool la = grid_fold(a, r1, sh, &ta);
    if (la && threadIdx.x == 0) F->nr2 = ta;
    __syncthreads();
    const bool lb = grid_fold(b, r2, sh, &tb);
    if (lb && threadIdx.x == 0) F->df2 = tb;
    (void)la;
}

__global__ void k_filter_x0(Grid g, const double* __restrict__ lastx, double* __restrict__ x,
                            const FilterScalars* F) {
    const double nr = sqrt(F->nr2), df = sqrt(F->df2);
    const bool warm = (nr > 0.0) && (df / (1.0e-30 < nr ? nr : 1.0e-30) < 1000.0);
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.NN; n += gridDim.x * blockDim.x)
        x[n] = warm ? lastx[n] : 0.0;
}

// y = K_F x, node gather in colour order (filter.cpp:77-173); optional p.Ap into F->den
__global__ void __launch_bounds__(RED_THREADS) k_filter_matvec(Grid g, const uint8_t* __restrict__ solid,
                                                               const double* __restrict__ kf,
                                                               const double* __restrict__ x,
                                                               double* __restrict__ y, RedSlot dot,
                                                               FilterScalars* F) {
    __shared__ double K[64];
    __shared__ double sh[32];
    if (dot.partial && F->done) return;
    if (threadIdx.x < 64) K[threadIdx.x] = kf[threadIdx.x];
    __syncthreads();
    const int NN = (int)g.NN;
    double part = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x) {
        int ix, iy, iz;
        node_ijk(g, n, ix, iy, iz);
        double acc = 0.0;
        for (int col = 0; col < 8; ++col) {
            const int cx = (((ix - 1) & 1) == (col & 1)) ? ix - 1 : ix;
            const int cy = (((g.ny - iy) & 1) == ((col >> 1) & 1)) ? iy - 1 : iy;
            const int cz = (((iz - 1) & 1) == ((col >> 2) & 1)) ? iz - 1 : iz;
            if (!solid[g.cell(cx, cy, cz)]) continue;
            const int a = corner_of(ix - cx, iy - cy, iz - cz);
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 8; ++j)
                s = s + K[a * 8 + j] * x[g.node(cx + corner_dx(j), cy + corner_dy(j), cz + corner_dz(j))];
            acc = acc + s;
        }
        y[n] = acc;
        if (dot.partial) part = part + x[n] * acc;
    }
    if (dot.partial) {
        double tot;
        if (grid_fold(part, dot, sh, &tot) && threadIdx.x == 0) F->den = tot;
    }
}

// r = rhs - A x0; z = D r; rz = r.z (0 -> 1); p = z; early exit when |r| < 1e-2 (filter.cpp:200-239)
__global__ void __launch_bounds__(RED_THREADS) k_filter_r0(Grid g, const double* __restrict__ rhs,
                                                           const double* __restrict__ Ax,
                                                           const double* __restrict__ fdiag, double* __restrict__ r,
                                                           double* __restrict__ z, double* __restrict__ p, RedSlot r1,
                                                           RedSlot r2, FilterScalars* F) {
    __shared__ double sh[32];
    const int NN = (int)g.NN;
    double a = 0.0, b = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x) {
        const double rv = rhs[n] - Ax[n];
        r[n] = rv;
        const double zv = fdiag[n] * rv;
        z[n] = zv;
        p[n] = zv;
        a = a + rv * zv;
        b = b + rv * rv;
    }
    double ta, tb;
    if (grid_fold(a, r1, sh, &ta) && threadIdx.x == 0) F->rz = (ta == 0) ? 1.0 : ta;
    __syncthreads();
    if (grid_fold(b, r2, sh, &tb) && threadIdx.x == 0) {
        F->done = (sqrt(tb) < 1.0e-2) ? 1 : 0;
        F->it = 0;
    }
}

// x += alpha p; r -= alpha Ap; stop when |r| < 1e-3 (filter.cpp:241-250)
__global__ void __launch_bounds__(RED_THREADS) k_filter_update(Grid g, double* __restrict__ x, double* __restrict__ r,
                                                               const double* __restrict__ p,
                                                               const double* __restrict__ Ap, RedSlot red,
                                                               FilterScalars* F) {
    __shared__ double sh[32];
    if (F->done) return;
    const double den = F->den;
    const double alpha = F->rz / (1.0e-30 < den ? den : 1.0e-30);
    const int NN = (int)g.NN;
    double part = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x) {
        x[n] = x[n] + alpha * p[n];
        const double rv = r[n] - alpha * Ap[n];
        r[n] = rv;
        part = part + rv * rv;
    }
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) {
        F->it = F->it + 1;
        if (sqrt(tot) < 1e-3) F->done = 1;
    }
}

// z = D r; rz_new = r.z; beta = rz_new/max(1e-30,rz) (filter.cpp:251-264)
__global__ void __launch_bounds__(RED_THREADS) k_filter_precond(Grid g, const double* __restrict__ r,
                                                                const double* __restrict__ fdiag,
                                                                double* __restrict__ z, RedSlot red,
                                                                FilterScalars* F) {
    __shared__ double sh[32];
    if (F->done) return;
    const int NN = (int)g.NN;
    double part = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x) {
        const double rv = r[n];
        const double zv = fdiag[n] * rv;
        z[n] = zv;
        part = part + rv * zv;
    }
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) {
        const double rz = F->rz;
        F->beta = tot / (1.0e-30 < rz ? rz : 1.0e-30);
        F->rz = tot;
    }
}

__global__ void k_filter_direction(Grid g, const double* __restrict__ z, double* __restrict__ p,
                                   const FilterScalars* F) {
    if (F->done) return;
    const double beta = F->beta;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.NN; n += gridDim.x * blockDim.x)
        p[n] = z[n] + beta * p[n];
}

// dst_e = (float)(sum_a x[node_a] * 1/8), corners in reference order (filter.cpp:267-271)
__global__ void k_filter_to_cells(Grid g, const uint8_t* __restrict__ solid, const double* __restrict__ x,
                                  float* __restrict__ dst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.nx * g.ny * g.nz) return;
    const int cx = k % g.nx, cy = (k / g.nx) % g.ny, cz = k / (g.nx * g.ny);
    const int64_t ci = g.cell(cx, cy, cz);
    if (!solid[ci]) return;
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) s = s + x[g.node(cx + corner_dx(a), cy + corner_dy(a), cz + corner_dz(a))];
    dst[ci] = (float)(s * (1.0 / 8.0));
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void launch_filter_diag(const Grid& g, const uint8_t* solid, const double* kf, double* fdiag, cudaStream_t s) {
    k_filter_diag<<<blocks_for(g.NN, 256), 256, 0, s>>>(g, solid, kf, fdiag);
}
void launch_filter_rhs(const Grid& g, const uint8_t* solid, const float* src, double* rhs, cudaStream_t s) {
    k_filter_rhs<<<blocks_for(g.NN, 256), 256, 0, s>>>(g, solid, src, rhs);
}
void launch_filter_norms(const Grid& g, const double* rhs, const double* lastrhs, RedSlot r1, RedSlot r2,
                         FilterScalars* F, cudaStream_t s) {
    k_filter_norms<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, rhs, lastrhs, r1, r2, F);
}
void launch_filter_x0(const Grid& g, const double* lastx, double* x, const FilterScalars* F, cudaStream_t s) {
    k_filter_x0<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, lastx, x, F);
}
void launch_filter_matvec(const Grid& g, const uint8_t* solid, const double* kf, const double* x, double* y,
                          RedSlot dot, FilterScalars* F, cudaStream_t s) {
    k_filter_matvec<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, solid, kf, x, y, dot, F);
}
void launch_filter_r0(const Grid& g, const double* rhs, const double* Ax, const double* fdiag, double* r, double* z,
                      double* p, RedSlot r1, RedSlot r2, FilterScalars* F, cudaStream_t s) {
    k_filter_r0<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, rhs, Ax, fdiag, r, z, p, r1, r2, F);
}
void launch_filter_update(const Grid& g, double* x, double* r, const double* p, const double* Ap, RedSlot red,
                          FilterScalars* F, cudaStream_t s) {
    k_filter_update<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, x, r, p, Ap, red, F);
}
void launch_filter_precond(const Grid& g, const double* r, const double* fdiag, double* z, RedSlot red,
                           FilterScalars* F, cudaStream_t s) {
    k_filter_precond<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, r, fdiag, z, red, F);
}
void launch_filter_direction(const Grid& g, const double* z, double* p, const FilterScalars* F, cudaStream_t s) {
    k_filter_direction<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, z, p, F);
}
void launch_filter_to_cells(const Grid& g, const uint8_t* solid, const double* x, float* dst, cudaStream_t s) {
    k_filter_to_cells<<<blocks_for((int64_t)g.nx * g.ny * g.nz, 256), 256, 0, s>>>(g, solid, x, dst);
}

}  // namespace t3d
