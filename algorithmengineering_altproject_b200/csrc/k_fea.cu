// FEA kernels: model set-up, the matrix-free hex8 K(E)u product, compliance, SIMP moduli and
// sensitivities, and the layout conversions used at the C-ABI boundary.
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

// ------------------------------------------------------------------ set-up (fea.cpp:181-447)
__global__ void k_setup_cells(Grid g, Cuboid c, VoidSet v, uint8_t* solid) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.NE) return;
    const int gx = (int)(i % g.ex);
    const int gy = (int)((i / g.ex) % g.ey);
    const int gz = (int)(i / ((int64_t)g.ex * g.ey));
    const int cx = gx - 1, cy = gy - 1, cz = gz - 1;
    uint8_t s = 0;
    if (cx >= 0 && cx < g.nx && cy >= 0 && cy < g.ny && cz >= 0 && cz < g.nz)
        s = (cx < c.nelx && cy >= g.ny - c.nely && cz < c.nelz && !in_void(v, cx, g.ny - 1 - cy, cz)) ? 1 : 0;
    solid[i] = s;
}

// fixed = x=0 face (fea.cpp:374-385; fix_x0 = 0 for external models, whose fixations come from a list)
// or node touched by no solid element (fea.cpp:406-417)
__global__ void k_setup_mask0(Grid g, const uint8_t* __restrict__ solid, int fix_x0, uint8_t* __restrict__ mask) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.NN) return;
    int ix, iy, iz;
    node_ijk(g, n, ix, iy, iz);
    int used = 0;
    for (int dz = -1; dz <= 0; ++dz)
        for (int dy = -1; dy <= 0; ++dy)
            for (int dx = -1; dx <= 0; ++dx) used |= solid[g.cell(ix + dx, iy + dy, iz + dz)];
    mask[n] = ((fix_x0 && ix == 0) || !used) ? 7 : 0;
}

// listed fixations of an external model (TOP3D_XL.m:529-534): OR the DOF bits into distinct nodes
__global__ void k_setup_fix_list(int n, const int32_t* __restrict__ node, const uint8_t* __restrict__ bits,
                                 uint8_t* __restrict__ mask) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) mask[node[i]] |= bits[i];
}

// weighted element compliance of several load cases (TOP3D_XL.m:621): acc = w ce (first case), acc + w ce
__global__ void k_cells_axpy(int64_t n, int first, double w, const double* __restrict__ ce, double* __restrict__ acc) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double t = w * ce[i];
    acc[i] = first ? t : acc[i] + t;
}

// listed loads of an external model (TOP3D_XL.m:536-545) on distinct nodes, dropped on fixed DOFs
__global__ void k_setup_load_list(Grid g, int n, const int32_t* __restrict__ node, const double* __restrict__ f,
                                  const uint8_t* __restrict__ mask, double* __restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t m = node[i];
    for (int c = 0; c < 3; ++c)
        if (!((mask[m] >> c) & 1)) b[c * g.NN + m] = f[3 * i + c];
}

// -Z load slab on ix = ix_load, iz <= iz_max, all iy (fea.cpp:388-403), dropped on fixed DOFs
__global__ void k_setup_load(Grid g, int ix_load, int iz_max, double fz, const uint8_t* __restrict__ mask,
                             double* __restrict__ bz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (iz_max + 1) * g.nny) return;
    const int iy = i % g.nny, iz = i / g.nny;
    const int64_t n = g.node(ix_load, iy, iz);
    if (!(mask[n] & 4)) bz[n] = fz;
}

// force f on component comp of every free node in a box of nodes (load cases beyond the reference's)
__global__ void k_setup_box_load(Grid g, int x0, int x1, int y0, int y1, int z0, int z1, int comp, double f,
                                 const uint8_t* __restrict__ mask, double* __restrict__ b) {
    const int nx = x1 - x0 + 1, ny = y1 - y0 + 1, nz = z1 - z0 + 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx * ny * nz) return;
    const int64_t n = g.node(x0 + i % nx, y0 + (i / nx) % ny, z0 + i / (nx * ny));
    if (!((mask[n] >> comp) & 1)) b[comp * g.NN + n] += f;
}

// ------------------------------------------------------------------ K(E) u  (fea.cpp:692-837)
// Node-centric gather.  For each node the 8 incident elements are visited in the reference's colour
// order (colour = ex&1 | (ey&1)<<1 | (ez&1)<<2, fea.cpp:300), each contributing its 3 rows of
// Ke*u_e as an FMA chain over the 24 columns, scaled by E with one more FMA.  That is the exact
// operation sequence of the colour-serialised scatter of the reference (and of the oracle), so the
// result is bit-identical to it.  Elements with E <= 1e-16 (and empty/ghost cells, E = 0) are skipped.
// With dot.partial set, p.Ap is accumulated in the canonical reduction order into S->denom.
__global__ void __launch_bounds__(RED_THREADS) k_matvec64(Grid g, const double* __restrict__ Keg,
                                                          const double* __restrict__ E,
                                                          const uint8_t* __restrict__ mask,
                                                          const double* __restrict__ u, double* __restrict__ y,
                                                          RedSlot dot, PcgScalars* S) {
    __shared__ __align__(16) double Ke[576];
    __shared__ double sh[32];
    if (S != nullptr && S->done) return;
    for (int i = threadIdx.x; i < 576; i += blockDim.x) Ke[i] = Keg[i];
    __syncthreads();
    const int NN = (int)g.NN;
    const double* __restrict__ u0 = u;
    const double* __restrict__ u1 = u + NN;
    const double* __restrict__ u2 = u + 2 * (int64_t)NN;
    double part = 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += stride) {
        int ix, iy, iz;
        node_ijk(g, n, ix, iy, iz);
        double y0 = 0.0, y1 = 0.0, y2 = 0.0;
#pragma unroll 1
        for (int col = 0; col < 8; ++col) {
            const int cx = (((ix - 1) & 1) == (col & 1)) ? ix - 1 : ix;
            const int cy = (((g.ny - iy) & 1) == ((col >> 1) & 1)) ? iy - 1 : iy;
            const int cz = (((iz - 1) & 1) == ((col >> 2) & 1)) ? iz - 1 : iz;
            const double Ee = E[g.cell(cx, cy, cz)];
            if (Ee <= 1.0e-16) continue;
            const int a = corner_of(ix - cx, iy - cy, iz - cz);
            double ue[24];
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const int m = (int)g.node(cx + corner_dx(b), cy + corner_dy(b), cz + corner_dz(b));
                ue[3 * b + 0] = u0[m];
                ue[3 * b + 1] = u1[m];
                ue[3 * b + 2] = u2[m];
            }
            const double2* K0 = reinterpret_cast<const double2*>(Ke + (3 * a) * 24);
            double f0 = 0.0, f1 = 0.0, f2 = 0.0;
#pragma unroll
            for (int j = 0; j < 24; j += 2) {
                const double2 k0 = K0[j / 2], k1 = K0[12 + j / 2], k2 = K0[24 + j / 2];
                f0 = fma(k0.x, ue[j], f0);
                f0 = fma(k0.y, ue[j + 1], f0);
                f1 = fma(k1.x, ue[j], f1);
                f1 = fma(k1.y, ue[j + 1], f1);
                f2 = fma(k2.x, ue[j], f2);
                f2 = fma(k2.y, ue[j + 1], f2);
            }
            y0 = fma(f0, Ee, y0);
            y1 = fma(f1, Ee, y1);
            y2 = fma(f2, Ee, y2);
        }
        const int mk = mask[n];
        if (mk & 1) y0 = 0.0;
        if (mk & 2) y1 = 0.0;
        if (mk & 4) y2 = 0.0;
        y[n] = y0;
        y[NN + n] = y1;
        y[2 * (int64_t)NN + n] = y2;
        if (dot.partial) {
            part = part + u0[n] * y0;
            part = part + u1[n] * y1;
            part = part + u2[n] * y2;
        }
    }
    if (dot.partial) {
        double tot;
        if (grid_fold(part, dot, sh, &tot) && threadIdx.x == 0) S->denom = tot;
    }
}

// ------------------------------------------------------------------ compliance (fea.cpp:587-677)
// ce = ue' Ke ue per solid element (0 when E <= 1e-16); C = sum E*ce in canonical order over cells
// (cell index k = (cz*ny + cy)*nx + cx).
__global__ void __launch_bounds__(RED_THREADS) k_compliance64(Grid g, const double* __restrict__ Keg,
                                                              const double* __restrict__ E,
                                                              const double* __restrict__ u,
                                                              double* __restrict__ ce, RedSlot red,
                                                              double* __restrict__ C) {
    __shared__ double Ke[576];
    __shared__ double sh[32];
    for (int i = threadIdx.x; i < 576; i += blockDim.x) Ke[i] = Keg[i];
    __syncthreads();
    const int NN = (int)g.NN;
    const int ncell = g.nx * g.ny * g.nz;
    double part = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ncell; k += gridDim.x * blockDim.x) {
        const int cx = k % g.nx, cy = (k / g.nx) % g.ny, cz = k / (g.nx * g.ny);
        const int64_t ci = g.cell(cx, cy, cz);
        const double Ee = E[ci];
        if (Ee <= 1.0e-16) {
            ce[ci] = 0.0;
            continue;
        }
        double ue[24];
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const int m = (int)g.node(cx + corner_dx(b), cy + corner_dy(b), cz + corner_dz(b));
            ue[3 * b + 0] = u[m];
            ue[3 * b + 1] = u[NN + m];
            ue[3 * b + 2] = u[2 * (int64_t)NN + m];
        }
        double s = 0.0;
#pragma unroll 4
        for (int i = 0; i < 24; ++i) {
            double row = 0.0;
#pragma unroll
            for (int j = 0; j < 24; ++j) row = row + Ke[i * 24 + j] * ue[j];
            s = s + ue[i] * row;
        }
        ce[ci] = s;
        part = part + Ee * s;
    }
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) *C = tot;
}

// printed objective Cdisp = (sum E*(ce*(1/Csolid)))*Csolid (driver.cpp:144-150)
__global__ void __launch_bounds__(RED_THREADS) k_objective(Grid g, const double* __restrict__ E,
                                                           const double* __restrict__ ce,
                                                           const double* __restrict__ Csolid, RedSlot red,
                                                           double* __restrict__ obj) {
    __shared__ double sh[32];
    const double cs = *Csolid;
    const double rc = 1.0 / cs;
    const int ncell = g.nx * g.ny * g.nz;
    double part = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ncell; k += gridDim.x * blockDim.x) {
        const int cx = k % g.nx, cy = (k / g.nx) % g.ny, cz = k / (g.nx * g.ny);
        const int64_t ci = g.cell(cx, cy, cz);
        const double Ee = E[ci];
        if (Ee == 0.0) continue;
        part = part + Ee * (ce[ci] * rc);
    }
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) *obj = cs > 0 ? tot * cs : tot;
}

// x^p rounded once to float (integer p by repeated double multiplication)
__device__ __forceinline__ float pow_rounded(float x, float p) {
    const double xd = (double)x;
    if (p == 3.0f) return (float)(xd * xd * xd);
    if (p == 2.0f) return (float)(xd * xd);
    if (p == 1.0f) return x;
    return (float)pow(xd, (double)p);
}

__device__ __forceinline__ float clamp01(float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); }

// SIMP modulus E = fma(rho^p, E0-Emin, Emin) in float (driver.cpp:117-121)
__global__ void k_simp(Grid g, const uint8_t* __restrict__ solid, const float* __restrict__ x, float E0, float Emin,
                       float penal, double* __restrict__ E) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.NE) return;
    if (!solid[i]) { E[i] = 0.0; return; }
    const float pw = pow_rounded(clamp01(x[i]), penal);
    E[i] = (double)__fmaf_rn(pw, E0 - Emin, Emin);
}

// dc = ceNorm*(rho^(p-1)*((Emin-E0)*p)), ceNorm = (float)(ce*(1/Csolid)); xdc = x*dc (driver.cpp:151-162)
__global__ void k_sens(Grid g, const uint8_t* __restrict__ solid, const float* __restrict__ x,
                       const double* __restrict__ ce, const double* __restrict__ Csolid, float E0, float Emin,
                       float penal, float* __restrict__ dc, float* __restrict__ xdc) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.NE) return;
    if (!solid[i]) { dc[i] = 0.0f; xdc[i] = 0.0f; return; }
    const double cs = *Csolid;
    const float pw = pow_rounded(clamp01(x[i]), penal - 1.0f);
    const float K = (Emin - E0) * penal;
    const float cn = cs > 0 ? (float)(ce[i] * (1.0 / cs)) : (float)ce[i];
    const float d = cn * (pw * K);
    dc[i] = d;
    xdc[i] = x[i] * d;
}

// ------------------------------------------------------------------ MG fine diagonal (diagonal.cpp:11-53, 140-147)
__global__ void k_diag0(Grid g, const double* __restrict__ Keg, const double* __restrict__ E,
                        const uint8_t* __restrict__ mask, double* __restrict__ diag) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.NN) return;
    int ix, iy, iz;
    node_ijk(g, n, ix, iy, iz);
    double d[3] = {0.0, 0.0, 0.0};
    for (int col = 0; col < 8; ++col) {
        const int cx = (((ix - 1) & 1) == (col & 1)) ? ix - 1 : ix;
        const int cy = (((g.ny - iy) & 1) == ((col >> 1) & 1)) ? iy - 1 : iy;
        const int cz = (((iz - 1) & 1) == ((col >> 2) & 1)) ? iz - 1 : iz;
        const double Ee = E[g.cell(cx, cy, cz)];
        const int a = corner_of(ix - cx, iy - cy, iz - cz);
        for (int c = 0; c < 3; ++c) {
            const int l = 3 * a + c;
            d[c] = d[c] + Keg[l * 24 + l] * Ee;
        }
    }
    const int mk = mask[n];
    for (int c = 0; c < 3; ++c) {
        double v = d[c];
        if (!(v > 0.0)) v = 1.0;
        if (mk & (1 << c)) v = 1.0;
        diag[c * g.NN + n] = v;
    }
}

// ------------------------------------------------------------------ canonical node reductions
__global__ void __launch_bounds__(RED_THREADS) k_dot(Grid g, int ncomp, const double* __restrict__ a,
                                                     const double* __restrict__ b, RedSlot red,
                                                     double* __restrict__ out) {
    __shared__ double sh[32];
    const int NN = (int)g.NN;
    double part = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x)
        for (int c = 0; c < ncomp; ++c) part = part + a[c * (int64_t)NN + n] * b[c * (int64_t)NN + n];
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) *out = tot;
}

// ---------------------------------------------------------------- layout conversions
__global__ void k_scatter_free(int64_t nf, const int32_t* __restrict__ fd, const double* __restrict__ v, int64_t NN,
                               double* __restrict__ grid) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    const int32_t d = fd[i];
    grid[(int64_t)(d % 3) * NN + d / 3] = v[i];
}
__global__ void k_gather_free(int64_t nf, const int32_t* __restrict__ fd, const double* __restrict__ grid, int64_t NN,
                              double* __restrict__ v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    const int32_t d = fd[i];
    v[i] = grid[(int64_t)(d % 3) * NN + d / 3];
}
template <class T>
__global__ void k_cells_from(int64_t ne, const int32_t* __restrict__ cell_of, const T* __restrict__ v,
                             T* __restrict__ cells) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ne) cells[cell_of[i]] = v[i];
}
template <class T>
__global__ void k_cells_to(int64_t ne, const int32_t* __restrict__ cell_of, const T* __restrict__ cells,
                           T* __restrict__ v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ne) v[i] = cells[cell_of[i]];
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void launch_setup_cells(const Grid& g, Cuboid c, const VoidSet& v, uint8_t* solid, cudaStream_t s) {
    k_setup_cells<<<blocks_for(g.NE, 256), 256, 0, s>>>(g, c, v, solid);
}
void launch_setup_box_load(const Grid& g, int x0, int x1, int y0, int y1, int z0, int z1, int comp, double f,
                           const uint8_t* mask, double* b, cudaStream_t s) {
    const int n = (x1 - x0 + 1) * (y1 - y0 + 1) * (z1 - z0 + 1);
    k_setup_box_load<<<blocks_for(n, 256), 256, 0, s>>>(g, x0, x1, y0, y1, z0, z1, comp, f, mask, b);
}
void launch_setup_mask0(const Grid& g, const uint8_t* solid, int fix_x0, uint8_t* mask, cudaStream_t s) {
    k_setup_mask0<<<blocks_for(g.NN, 256), 256, 0, s>>>(g, solid, fix_x0, mask);
}
void launch_cells_axpy(int64_t n, int first, double w, const double* ce, double* acc, cudaStream_t s) {
    k_cells_axpy<<<blocks_for(n, 256), 256, 0, s>>>(n, first, w, ce, acc);
}
void launch_setup_fix_list(int n, const int32_t* node, const uint8_t* bits, uint8_t* mask, cudaStream_t s) {
    if (n > 0) k_setup_fix_list<<<blocks_for(n, 256), 256, 0, s>>>(n, node, bits, mask);
}
void launch_setup_load_list(const Grid& g, int n, const int32_t* node, const double* f, const uint8_t* mask, double* b,
                            cudaStream_t s) {
    if (n > 0) k_setup_load_list<<<blocks_for(n, 256), 256, 0, s>>>(g, n, node, f, mask, b);
}
void launch_setup_load(const Grid& g, int ix_load, int iz_max, double fz, const uint8_t* mask, double* b,
                       cudaStream_t s) {
    const int n = (iz_max + 1) * g.nny;
    k_setup_load<<<blocks_for(n, 256), 256, 0, s>>>(g, ix_load, iz_max, fz, mask, b + 2 * g.NN);
}
void launch_matvec64(const Grid& g, const double* Ke, const double* E, const uint8_t* mask, const double* u,
                     double* y, RedSlot dot, PcgScalars* S, cudaStream_t s) {
    k_matvec64<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, Ke, E, mask, u, y, dot, S);
}
void launch_compliance64(const Grid& g, const double* Ke, const double* E, const double* u, double* ce,
                         RedSlot red, double* C, cudaStream_t s) {
    k_compliance64<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, Ke, E, u, ce, red, C);
}
void launch_objective(const Grid& g, const double* E, const double* ce, const double* Csolid, RedSlot red,
                      double* obj, cudaStream_t s) {
    k_objective<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, E, ce, Csolid, red, obj);
}
void launch_simp(const Grid& g, const uint8_t* solid, const float* x, float E0, float Emin, float penal, double* E,
                 cudaStream_t s) {
    k_simp<<<blocks_for(g.NE, 256), 256, 0, s>>>(g, solid, x, E0, Emin, penal, E);
}
void launch_sens(const Grid& g, const uint8_t* solid, const float* x, const double* ce, const double* Csolid,
                 float E0, float Emin, float penal, float* dc, float* xdc, cudaStream_t s) {
    k_sens<<<blocks_for(g.NE, 256), 256, 0, s>>>(g, solid, x, ce, Csolid, E0, Emin, penal, dc, xdc);
}
void launch_diag0(const Grid& g, const double* Ke, const double* E, const uint8_t* mask, double* diag,
                  cudaStream_t s) {
    k_diag0<<<blocks_for(g.NN, 256), 256, 0, s>>>(g, Ke, E, mask, diag);
}
void launch_dot(const Grid& g, int ncomp, const double* a, const double* b, RedSlot red, double* out, cudaStream_t s) {
    k_dot<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, ncomp, a, b, red, out);
}
void launch_scatter_free(int64_t nf, const int32_t* free_dofs, const double* vfree, int64_t NN, double* grid,
                         cudaStream_t s) {
    k_scatter_free<<<blocks_for(nf, 256), 256, 0, s>>>(nf, free_dofs, vfree, NN, grid);
}
void launch_gather_free(int64_t nf, const int32_t* free_dofs, const double* grid, int64_t NN, double* vfree,
                        cudaStream_t s) {
    k_gather_free<<<blocks_for(nf, 256), 256, 0, s>>>(nf, free_dofs, grid, NN, vfree);
}
void launch_cells_from_morton_f64(int64_t ne, const int32_t* cell_of, const double* v, double* cells, cudaStream_t s) {
    k_cells_from<double><<<blocks_for(ne, 256), 256, 0, s>>>(ne, cell_of, v, cells);
}
void launch_cells_to_morton_f64(int64_t ne, const int32_t* cell_of, const double* cells, double* v, cudaStream_t s) {
    k_cells_to<double><<<blocks_for(ne, 256), 256, 0, s>>>(ne, cell_of, cells, v);
}
void launch_cells_from_morton_f32(int64_t ne, const int32_t* cell_of, const float* v, float* cells, cudaStream_t s) {
    k_cells_from<float><<<blocks_for(ne, 256), 256, 0, s>>>(ne, cell_of, v, cells);
}
void launch_cells_to_morton_f32(int64_t ne, const int32_t* cell_of, const float* cells, float* v, cudaStream_t s) {
    k_cells_to<float><<<blocks_for(ne, 256), 256, 0, s>>>(ne, cell_of, cells, v);
}

}  // namespace t3d
