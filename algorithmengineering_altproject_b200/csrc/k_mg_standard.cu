// The 'Standard' V-cycle option (the MATLAB original's typeVcycle_ = 'Standard', TOP3D_XL.m:772-807):
// Jacobi smoothing with the true residual on every level, Galerkin coarse operators, restriction = the
// transpose of the trilinear prolongation, so the cycle is symmetric and PCG can use it.
//
//   down, l = 0..L-2:  x_l = w r_l / D_l;  r_{l+1} = P^T (r_l - K_l x_l)
//   coarsest:          x_L = K_L^{-1} r_L  (dense Cholesky, or Jacobi when too large)
//   up,   l = L-2..0:  x_l += P x_{l+1};  x_l += w (r_l - K_l x_l) / D_l
//
// K_0 = K(E); K_l = P~^T K_{l-1} P~ with P~ = M_{l-1} P M_l (M = the levels' free-DOF masks), stored as one
// 24x24 matrix per coarse element (local DOF 3a+c, grid corner order); D_l = diag(K_l), fixed or
// non-positive entries -> 1.  Level-1 element matrices are sums of E_c G_pos over the s^3 children, with
// G_pos = W_pos^T Ke W_pos precomputed per child position (W_pos: trilinear weights of the child's corners);
// children touching a fixed DOF take the masked product explicitly.  All FP64, deterministic orders.
// The assembly keeps element matrices element-major (576 consecutive entries per element); the level products
// read an entry-major copy (kel_index: entry k of element e at k * ne + e), in which threads working on
// consecutive nodes read consecutive addresses.
#include "kernels.hpp"
#include "red.cuh"

namespace t3d {

namespace {

// weight of coarse corner A at fine offset (fx, fy, fz) in [0, s]^3 of a span-s coarse element
__device__ __forceinline__ double tri_w(int s, int fx, int fy, int fz, int A) {
    const double is = 1.0 / s;   // s is 2 or 4: exact
    const double wx = corner_dx(A) ? fx * is : (s - fx) * is;
    const double wy = corner_dy(A) ? fy * is : (s - fy) * is;
    const double wz = corner_dz(A) ? fz * is : (s - fz) * is;
    return wx * wy * wz;
}

__device__ __forceinline__ int lnode(const MgLevel& L, int x, int y, int z) {
    return (z * (L.ny + 1) + y) * (L.nx + 1) + x;
}

// level-1 element matrices from the finest grid: one CTA (576 threads, thread = entry (P, Q)) per GB
// consecutive coarse elements (cz*ny1 + cy)*nx1 + cx, so that each G_pos entry is read once per batch;
// children are summed in position order, masked ones by the explicit product
constexpr int GB = 16;

__global__ void __launch_bounds__(576, 1) k_galerkin_fine(Grid g, MgLevel L1, int s, const double* __restrict__ E,
                                                       const uint8_t* __restrict__ mask0,
                                                       const double* __restrict__ Gpos,
                                                       const double* __restrict__ Keg, double* __restrict__ Kel) {
    __shared__ __align__(16) double Ec[64][GB];   // child moduli by position (0: skipped), s^3 <= 64
    __shared__ uint8_t cmk[GB][64][8];            // child corner masks
    __shared__ uint8_t anym[GB][64];              // child touches a fixed DOF
    __shared__ uint8_t cmask[GB][8];              // coarse corner masks
    __shared__ uint8_t nm[GB][125];               // masks of each coarse element's (s+1)^3 fine nodes (s <= 4)
    __shared__ double wt[125][8];                 // tri_w(s, fx, fy, fz, A) at fine offsets 0..s: the same values
    __shared__ double kg[576];                    // the fine element stiffness
    __shared__ double us[576];                    // a masked child's inner sums u(a; r, B, q)
    __shared__ int masked;                        // some child of the batch touches a fixed DOF
    const int ne1 = L1.nx * L1.ny * L1.nz, ns = s * s * s, s1 = s + 1, nr = s1 * s1 * s1;
    const int e0 = blockIdx.x * GB;
    if (threadIdx.x == 0) masked = 0;
    for (int q = threadIdx.x; q < GB * nr; q += blockDim.x) {   // each node mask loaded once per block
        const int b = q / nr, o = q % nr, ce = e0 + b;
        uint8_t m = 0;
        if (ce < ne1) {
            const int cx = ce % L1.nx, cy = (ce / L1.nx) % L1.ny, cz = ce / (L1.nx * L1.ny);
            m = mask0[g.node(cx * s + o % s1, cy * s + (o / s1) % s1, cz * s + o / (s1 * s1))];
        }
        nm[b][o] = m;
    }
    for (int t = threadIdx.x; t < nr * 8; t += blockDim.x) {
        const int o = t / 8;
        wt[o][t % 8] = tri_w(s, o % s1, (o / s1) % s1, o / (s1 * s1), t % 8);
    }
    kg[threadIdx.x] = Keg[threadIdx.x];
    __syncthreads();
    for (int q = threadIdx.x; q < GB * ns; q += blockDim.x) {
        const int b = q / ns, p = q % ns, ce = e0 + b;
        double Ee = 0.0;
        uint8_t any = 0;
        if (ce < ne1) {
            const int cx = ce % L1.nx, cy = (ce / L1.nx) % L1.ny, cz = ce / (L1.nx * L1.ny);
            const int i = p % s, j = (p / s) % s, k = p / (s * s);
            const int fx = cx * s + i, fy = cy * s + j, fz = cz * s + k;
            const double e = E[g.cell(fx, fy, fz)];
            Ee = e <= 1.0e-16 ? 0.0 : e;   // K(E) skips these elements
            for (int a = 0; a < 8; ++a) {
                const uint8_t m = nm[b][((k + corner_dz(a)) * s1 + j + corner_dy(a)) * s1 + i + corner_dx(a)];
                cmk[b][p][a] = m;
                any |= m;
            }
        }
        Ec[p][b] = Ee;
        anym[b][p] = any;
        if (any && Ee != 0.0) masked = 1;
    }
    for (int q = threadIdx.x; q < GB * 8; q += blockDim.x) {
        const int b = q / 8, A = q % 8, ce = e0 + b;
        uint8_t m = 0;
        if (ce < ne1) {
            const int cx = ce % L1.nx, cy = (ce / L1.nx) % L1.ny, cz = ce / (L1.nx * L1.ny);
            m = L1.mask[lnode(L1, cx + corner_dx(A), cy + corner_dy(A), cz + corner_dz(A))];
        }
        cmask[b][A] = m;
    }
    __syncthreads();
    const int P = threadIdx.x / 24, Q = threadIdx.x % 24;
    const int A = P / 3, r = P % 3, B = Q / 3, q = Q % 3;
    const double* __restrict__ gcol = Gpos + threadIdx.x;
    double acc[GB];
#pragma unroll
    for (int b = 0; b < GB; ++b) acc[b] = 0.0;
    if (!masked) {
        // Every child is plain: acc_b += E_bp G_p[t] for all b in position order.  A skipped child (E_bp = 0)
        // adds +-0, which leaves acc unchanged (acc starts at +0 and a sum never turns into -0), so the sums are
        // those of the per-child test below.  The next four children's G_pos entries load while four are summed.
        double gn[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) gn[v] = gcol[v * 576];   // ns = s^3 is 8 or 64
        for (int p0 = 0; p0 < ns; p0 += 4) {
            double gc[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) gc[v] = gn[v];
            if (p0 + 4 < ns) {
#pragma unroll
                for (int v = 0; v < 4; ++v) gn[v] = gcol[(p0 + 4 + v) * 576];
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const double2* e2 = reinterpret_cast<const double2*>(&Ec[p0 + v][0]);
#pragma unroll
                for (int h = 0; h < GB / 2; ++h) {
                    const double2 e = e2[h];
                    acc[2 * h] = acc[2 * h] + e.x * gc[v];
                    acc[2 * h + 1] = acc[2 * h + 1] + e.y * gc[v];
                }
            }
        }
    } else {
        for (int p = 0; p < ns; ++p) {
            const double gp = gcol[p * 576];
            const int i = p % s, j = (p / s) % s, k = p / (s * s);
#pragma unroll
            for (int b = 0; b < GB; ++b) {
                const double Ee = Ec[p][b];
                if (Ee == 0.0) continue;
                if (!anym[b][p]) {
                    acc[b] = acc[b] + Ee * gp;
                } else {   // sum_{a,c} w_aA w_cB M_ar M_cq E Ke[3a+r][3c+q]
                    // the inner sums u(a; r, B, q) = sum_c w_cB M_cq Ke[3a+r][3c+q] do not depend on A: thread
                    // (3a+r, Q) forms its own once into us, and the outer sum over a reads them (the same terms in
                    // the same order as summing u inside the loop over a).  The branch is the same for the block.
                    double u = 0.0;
                    for (int c = 0; c < 8; ++c) {
                        if ((cmk[b][p][c] >> q) & 1) continue;
                        const double wc = wt[((k + corner_dz(c)) * s1 + j + corner_dy(c)) * s1 + i + corner_dx(c)][B];
                        u = u + wc * kg[(3 * A + r) * 24 + 3 * c + q];
                    }
                    us[threadIdx.x] = u;
                    __syncthreads();
                    double t = 0.0;
                    for (int a = 0; a < 8; ++a) {
                        if ((cmk[b][p][a] >> r) & 1) continue;
                        const double wa = wt[((k + corner_dz(a)) * s1 + j + corner_dy(a)) * s1 + i + corner_dx(a)][A];
                        t = t + wa * us[(3 * a + r) * 24 + Q];
                    }
                    acc[b] = acc[b] + Ee * t;
                    __syncthreads();   // us is rewritten by the next masked child
                }
            }
        }
    }
#pragma unroll
    for (int b = 0; b < GB; ++b) {
        const int ce = e0 + b;
        if (ce >= ne1) continue;
        double v = acc[b];
        if (((cmask[b][A] >> r) & 1) || ((cmask[b][B] >> q) & 1)) v = 0.0;
        Kel[(int64_t)ce * 576 + threadIdx.x] = v;
    }
}

// level-l element matrices from level l-1's (already masked): sum over the s^3 children of W^T K_c W
__global__ void __launch_bounds__(576) k_galerkin_coarse(MgLevel Lf, MgLevel Lc, const double* __restrict__ Kf,
                                                         double* __restrict__ Kc) {
    __shared__ int cmask[8];
    __shared__ double wt[125][8];   // tri_w(s, fx, fy, fz, A) at fine offsets 0..s (s <= 4), the same values
    __shared__ double kf[576];      // the current child's element matrix
    __shared__ double us[576];      // its inner sums u(a; r, B, q), entry (3a+r)*24 + 3B+q
    const int s = Lc.span, s1 = s + 1;
    const int ce = blockIdx.x;
    const int cx = ce % Lc.nx, cy = (ce / Lc.nx) % Lc.ny, cz = ce / (Lc.nx * Lc.ny);
    const int P = threadIdx.x / 24, Q = threadIdx.x % 24;
    const int A = P / 3, r = P % 3, B = Q / 3, q = Q % 3;
    if (threadIdx.x < 8)
        cmask[threadIdx.x] = Lc.mask[lnode(Lc, cx + corner_dx(threadIdx.x), cy + corner_dy(threadIdx.x),
                                           cz + corner_dz(threadIdx.x))];
    for (int t = threadIdx.x; t < s1 * s1 * s1 * 8; t += blockDim.x) {
        const int o = t / 8;
        wt[o][t % 8] = tri_w(s, o % s1, (o / s1) % s1, o / (s1 * s1), t % 8);
    }
    // t = sum_a w_aA u(a; r, B, q) with u(a; r, B, q) = sum_b w_bB K_c[3a+r][3b+q]: u does not depend on A, so
    // thread (3a+r, Q) forms its own once per child into us and the sum over a reads them -- the same terms in
    // the same order as summing u inside the loop over a.  The next child's matrix entry loads meanwhile.
    const int ns = s * s * s;
    auto child = [&](int p) {
        const int i = p % s, j = (p / s) % s, k = p / (s * s);
        return ((int64_t)((cz * s + k) * Lf.ny + cy * s + j) * Lf.nx + cx * s + i) * 576 + threadIdx.x;
    };
    double knext = Kf[child(0)];
    double acc = 0.0;
    for (int p = 0; p < ns; ++p) {
        const int i = p % s, j = (p / s) % s, k = p / (s * s);
        kf[threadIdx.x] = knext;
        __syncthreads();   // kf is complete (and the weights ready)
        if (p + 1 < ns) knext = Kf[child(p + 1)];
        double u = 0.0;
        for (int b = 0; b < 8; ++b) {
            const double wb = wt[(k + corner_dz(b)) * s1 * s1 + (j + corner_dy(b)) * s1 + i + corner_dx(b)][B];
            u = u + wb * kf[(3 * A + r) * 24 + 3 * b + q];
        }
        us[threadIdx.x] = u;
        __syncthreads();   // us is complete
        double t = 0.0;
        for (int a = 0; a < 8; ++a) {
            const double wa = wt[(k + corner_dz(a)) * s1 * s1 + (j + corner_dy(a)) * s1 + i + corner_dx(a)][A];
            t = t + wa * us[(3 * a + r) * 24 + Q];
        }
        acc = acc + t;
        __syncthreads();   // kf and us are rewritten by the next child
    }
    if (((cmask[A] >> r) & 1) || ((cmask[B] >> q) & 1)) acc = 0.0;
    Kc[(int64_t)ce * 576 + threadIdx.x] = acc;
}

// D = diag of the assembled level operator; fixed or non-positive -> 1
__global__ void k_level_diag(MgLevel L, const double* __restrict__ Kel) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nn) return;
    const int nnx = L.nx + 1, nny = L.ny + 1;
    const int x = n % nnx, y = (n / nnx) % nny, z = n / (nnx * nny);
    const int m = L.mask[n];
    for (int c = 0; c < 3; ++c) {
        double d = 0.0;
        for (int dz = 0; dz <= 1; ++dz)
            for (int dy = 0; dy <= 1; ++dy)
                for (int dx = 0; dx <= 1; ++dx) {
                    const int ex = x - dx, ey = y - dy, ez = z - dz;
                    if (ex < 0 || ey < 0 || ez < 0 || ex >= L.nx || ey >= L.ny || ez >= L.nz) continue;
                    const int a = corner_of(dx, dy, dz), e = (ez * L.ny + ey) * L.nx + ex;
                    d = d + Kel[(int64_t)e * 576 + (3 * a + c) * 24 + 3 * a + c];
                }
        L.diag[c * L.nn + n] = (((m >> c) & 1) || !(d > 0.0)) ? 1.0 : d;
    }
}

// y = K_l x from the entry-major element matrices KelT (node-centric gather), fixed DOFs 0
__global__ void k_level_matvec(MgLevel L, const double* __restrict__ Kel, const double* __restrict__ x,
                               double* __restrict__ y, const PcgScalars* S) {
    if (S != nullptr && S->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nn) return;
    const int nnx = L.nx + 1, nny = L.ny + 1;
    const int X = n % nnx, Y = (n / nnx) % nny, Z = n / (nnx * nny);
    const int64_t ne = (int64_t)L.nx * L.ny * L.nz;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int dz = 0; dz <= 1; ++dz)
        for (int dy = 0; dy <= 1; ++dy)
            for (int dx = 0; dx <= 1; ++dx) {
                const int ex = X - dx, ey = Y - dy, ez = Z - dz;
                if (ex < 0 || ey < 0 || ez < 0 || ex >= L.nx || ey >= L.ny || ez >= L.nz) continue;
                const int a = corner_of(dx, dy, dz);
                const double* K = Kel + ((ez * L.ny + ey) * L.nx + ex);   // entry k at K[k * ne]
                for (int b = 0; b < 8; ++b) {
                    const int m = lnode(L, ex + corner_dx(b), ey + corner_dy(b), ez + corner_dz(b));
                    for (int c = 0; c < 3; ++c) {
                        const double xv = x[c * L.nn + m];
                        for (int r = 0; r < 3; ++r) acc[r] = acc[r] + K[((3 * a + r) * 24 + 3 * b + c) * ne] * xv;
                    }
                }
            }
    const int mk = L.mask[n];
    for (int r = 0; r < 3; ++r) y[r * L.nn + n] = ((mk >> r) & 1) ? 0.0 : acc[r];
}

__device__ __forceinline__ double inv_diag(const MgLevel& L, int c, int n) {
    const double d = L.diag[c * L.nn + n];
    return 1.0 / (1.0e-30 < d ? d : 1.0e-30);
}

// x = w r / D
__global__ void k_jacobi_init(MgLevel L, const double* __restrict__ r, double* __restrict__ x, double w,
                              const PcgScalars* S) {
    if (S != nullptr && S->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nn) return;
    const int m = L.mask[n];
    for (int c = 0; c < 3; ++c)
        x[c * L.nn + n] = ((m >> c) & 1) ? 0.0 : (w * r[c * L.nn + n]) * inv_diag(L, c, n);
}

// d = r - Kx (in place on Kx)
__global__ void k_residual(MgLevel L, const double* __restrict__ r, double* __restrict__ kx, const PcgScalars* S) {
    if (S != nullptr && S->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nn) return;
    const int m = L.mask[n];
    for (int c = 0; c < 3; ++c) kx[c * L.nn + n] = ((m >> c) & 1) ? 0.0 : r[c * L.nn + n] - kx[c * L.nn + n];
}

// x += w (r - Kx) / D
__global__ void k_jacobi_correct(MgLevel L, const double* __restrict__ r, const double* __restrict__ kx,
                                 double* __restrict__ x, double w, const PcgScalars* S) {
    if (S != nullptr && S->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nn) return;
    const int m = L.mask[n];
    for (int c = 0; c < 3; ++c) {
        const int64_t i = c * L.nn + n;
        x[i] = ((m >> c) & 1) ? 0.0 : x[i] + (w * (r[i] - kx[i])) * inv_diag(L, c, n);
    }
}

// xf += P xc (trilinear from the coarse cell floor(f/s), clamped to the last cell), fixed DOFs 0
__global__ void k_prolong_add(MgLevel Lc, MgLevel Lf, const double* __restrict__ xc, double* __restrict__ xf,
                              const PcgScalars* S) {
    if (S != nullptr && S->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Lf.nn) return;
    const int s = Lc.span;
    const int fnx = Lf.nx + 1, fny = Lf.ny + 1;
    const int fx = n % fnx, fy = (n / fnx) % fny, fz = n / (fnx * fny);
    int cx = fx / s, cy = fy / s, cz = fz / s;
    if (cx >= Lc.nx) cx = Lc.nx - 1;
    if (cy >= Lc.ny) cy = Lc.ny - 1;
    if (cz >= Lc.nz) cz = Lc.nz - 1;
    const int m = Lf.mask[n];
    for (int c = 0; c < 3; ++c) {
        double p = 0.0;
        for (int A = 0; A < 8; ++A)
            p = p + tri_w(s, fx - cx * s, fy - cy * s, fz - cz * s, A) *
                        xc[c * Lc.nn + lnode(Lc, cx + corner_dx(A), cy + corner_dy(A), cz + corner_dz(A))];
        const int64_t i = c * Lf.nn + n;
        xf[i] = ((m >> c) & 1) ? 0.0 : xf[i] + p;
    }
}

// r.z in the canonical order; the last block sets rz (first use) or beta = rz_new/max(1e-30,rz), rz = rz_new
__global__ void __launch_bounds__(RED_THREADS) k_dot_rz(int64_t NN, const double* __restrict__ r,
                                                        const double* __restrict__ z, RedSlot red, PcgScalars* S) {
    __shared__ double sh[32];
    if (S->done) return;
    double part = 0.0;
    for (int64_t n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += (int64_t)gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c) part = part + r[c * NN + n] * z[c * NN + n];
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) {
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

// element matrices of a level in the coarsest assembly's layout: cel = (cz*nx + cx)*ny + (ny-1-cy)
__global__ void k_to_coarse_layout(MgLevel L, const double* __restrict__ Kel, double* __restrict__ Kce) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ne = (int64_t)L.nx * L.ny * L.nz;
    if (t >= ne * 576) return;
    const int e = (int)(t / 576), k = (int)(t % 576);
    const int cx = e % L.nx, cy = (e / L.nx) % L.ny, cz = e / (L.nx * L.ny);
    const int cel = (cz * L.nx + cx) * L.ny + (L.ny - 1 - cy);
    Kce[(int64_t)cel * 576 + k] = Kel[t];
}

// element-major -> entry-major (dst[k * ne + e] = src[e * 576 + k]) through 32 x 32 shared-memory tiles, with
// the FP32 image written instead when B is float
template <class B>
__global__ void k_kel_transpose(int64_t ne, const double* __restrict__ src, B* __restrict__ dst) {
    __shared__ double tile[32][33];
    const int64_t e0 = (int64_t)blockIdx.x * 32;
    const int k0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {   // rows = elements, columns = entries (coalesced in k)
        const int64_t e = e0 + j;
        const int k = k0 + threadIdx.x;
        tile[j][threadIdx.x] = (e < ne && k < 576) ? src[e * 576 + k] : 0.0;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {   // rows = entries, columns = elements (coalesced in e)
        const int k = k0 + j;
        const int64_t e = e0 + threadIdx.x;
        if (e < ne && k < 576) dst[(int64_t)k * ne + e] = (B)tile[threadIdx.x][j];
    }
}

inline unsigned blocks_of(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void launch_kel_transpose(int64_t ne, const double* Kel, double* KelT, cudaStream_t s) {
    k_kel_transpose<double><<<dim3((unsigned)((ne + 31) / 32), 18), dim3(32, 8), 0, s>>>(ne, Kel, KelT);
}
void launch_kel_transpose32(int64_t ne, const double* Kel, float* KelT32, cudaStream_t s) {
    k_kel_transpose<float><<<dim3((unsigned)((ne + 31) / 32), 18), dim3(32, 8), 0, s>>>(ne, Kel, KelT32);
}

void galerkin_positions(int s, const double* Ke, double* G) {
    for (int k = 0; k < s; ++k)
        for (int j = 0; j < s; ++j)
            for (int i = 0; i < s; ++i) {
                double w[8][8];   // w[a][A]: child corner a -> coarse corner A
                for (int a = 0; a < 8; ++a)
                    for (int A = 0; A < 8; ++A) {
                        const int fx = i + corner_dx(a), fy = j + corner_dy(a), fz = k + corner_dz(a);
                        const double wx = corner_dx(A) ? (double)fx / s : (double)(s - fx) / s;
                        const double wy = corner_dy(A) ? (double)fy / s : (double)(s - fy) / s;
                        const double wz = corner_dz(A) ? (double)fz / s : (double)(s - fz) / s;
                        w[a][A] = wx * wy * wz;
                    }
                double* Gp = G + ((k * s + j) * s + i) * 576;
                for (int P = 0; P < 24; ++P)
                    for (int Q = 0; Q < 24; ++Q) {
                        const int A = P / 3, r = P % 3, B = Q / 3, q = Q % 3;
                        double t = 0.0;
                        for (int a = 0; a < 8; ++a) {
                            double u = 0.0;
                            for (int b = 0; b < 8; ++b) u = u + w[b][B] * Ke[(3 * a + r) * 24 + 3 * b + q];
                            t = t + w[a][A] * u;
                        }
                        Gp[P * 24 + Q] = t;
                    }
            }
}

void launch_galerkin_fine(const Grid& g, const MgLevel& L1, const double* E, const uint8_t* mask0, const double* Gpos,
                          const double* Ke, double* Kel, cudaStream_t s) {
    k_galerkin_fine<<<blocks_of((int64_t)L1.nx * L1.ny * L1.nz, GB), 576, 0, s>>>(g, L1, L1.span, E, mask0, Gpos, Ke,
                                                                              Kel);
}
void launch_galerkin_coarse(const MgLevel& Lf, const MgLevel& Lc, const double* Kf, double* Kc, cudaStream_t s) {
    k_galerkin_coarse<<<Lc.nx * Lc.ny * Lc.nz, 576, 0, s>>>(Lf, Lc, Kf, Kc);
}
void launch_level_diag(const MgLevel& L, const double* Kel, cudaStream_t s) {
    k_level_diag<<<blocks_of(L.nn, 256), 256, 0, s>>>(L, Kel);
}
void launch_level_matvec(const MgLevel& L, const double* Kel, const double* x, double* y, const PcgScalars* S,
                         cudaStream_t s) {
    k_level_matvec<<<blocks_of(L.nn, 128), 128, 0, s>>>(L, Kel, x, y, S);
}
void launch_jacobi_init(const MgLevel& L, const double* r, double* x, double w, const PcgScalars* S, cudaStream_t s) {
    k_jacobi_init<<<blocks_of(L.nn, 256), 256, 0, s>>>(L, r, x, w, S);
}
void launch_residual(const MgLevel& L, const double* r, double* kx, const PcgScalars* S, cudaStream_t s) {
    k_residual<<<blocks_of(L.nn, 256), 256, 0, s>>>(L, r, kx, S);
}
void launch_jacobi_correct(const MgLevel& L, const double* r, const double* kx, double* x, double w,
                           const PcgScalars* S, cudaStream_t s) {
    k_jacobi_correct<<<blocks_of(L.nn, 256), 256, 0, s>>>(L, r, kx, x, w, S);
}
void launch_prolong_add(const MgLevel& Lc, const MgLevel& Lf, const double* xc, double* xf, const PcgScalars* S,
                        cudaStream_t s) {
    k_prolong_add<<<blocks_of(Lf.nn, 256), 256, 0, s>>>(Lc, Lf, xc, xf, S);
}
void launch_dot_rz(int64_t NN, const double* r, const double* z, RedSlot red, PcgScalars* S, cudaStream_t s) {
    k_dot_rz<<<RED_BLOCKS, RED_THREADS, 0, s>>>(NN, r, z, red, S);
}
void launch_to_coarse_layout(const MgLevel& L, const double* Kel, double* Kce, cudaStream_t s) {
    k_to_coarse_layout<<<blocks_of((int64_t)L.nx * L.ny * L.nz * 576, 256), 256, 0, s>>>(L, Kel, Kce);
}

}  // namespace t3d
