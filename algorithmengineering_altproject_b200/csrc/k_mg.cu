// Geometric-multigrid kernels: BC masks per level, Jacobi diagonals, restriction, prolongation
// fused with the additive smoother, the coarsest dense Galerkin matrix, its Cholesky factor and
// the coarsest triangular solves.  Every kernel mirrors the reference's arithmetic order
// (transfers.cpp, diagonal.cpp, coarsest.cpp, preconditioner.cpp) operation for operation.
#include "kernels.hpp"
#include "red.cuh"

#include <algorithm>

namespace t3d {

namespace {

struct LevelIdx {
    int nnx, nny, nnz;
    __device__ LevelIdx(const MgLevel& L) : nnx(L.nx + 1), nny(L.ny + 1), nnz(L.nz + 1) {}
    __device__ int node(int x, int y, int z) const { return (z * nny + y) * nnx + x; }
};

__device__ __forceinline__ double hat(int i, int s) {   // 1 - |i-(s-1)|/s  (transfers.cpp:123-126)
    return 1.0 - fabs((double)(i - (s - 1))) * (1.0 / s);
}

// trilinear weight of coarse corner a at sub-node (ix,iy,iz) of a span-s element (hierarchy.cpp:13-42)
__device__ __forceinline__ double corner_weight(int s, int ix, int iy, int iz, int a) {
    const double xi = -1.0 + 2.0 * ((double)ix / (double)s);
    const double eta = -1.0 + 2.0 * ((double)iy / (double)s);
    const double zeta = -1.0 + 2.0 * ((double)iz / (double)s);
    const double sx = (a == 1 || a == 2 || a == 5 || a == 6) ? 1.0 : -1.0;
    const double sy = (a == 2 || a == 3 || a == 6 || a == 7) ? 1.0 : -1.0;
    const double sz = a >= 4 ? 1.0 : -1.0;
    return 0.125 * (1.0 + sx * xi) * (1.0 + sy * eta) * (1.0 + sz * zeta);
}

// ------------------------------------------------------------------ masks (masks.cpp:11-37)
// coarse bit c = normalised restriction (valSum/wSum form) of the fine 0/1 field > 0.5
__global__ void k_mask_restrict(MgLevel Lc, MgLevel Lf) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Lc.nn) return;
    const LevelIdx C(Lc), F(Lf);
    const int cx = n % C.nnx, cy = (n / C.nnx) % C.nny, cz = n / (C.nnx * C.nny);
    const int s = Lc.span, ws = 2 * s - 1;
    double v[3] = {0, 0, 0}, wsum = 0.0;
    for (int iz = 0; iz < ws; ++iz) {
        const int fz = cz * s + iz - (s - 1);
        if (fz < 0 || fz >= F.nnz) continue;
        for (int iy = 0; iy < ws; ++iy) {
            const int fy = cy * s + iy - (s - 1);
            if (fy < 0 || fy >= F.nny) continue;
            const double wzy = hat(iz, s) * hat(iy, s);
            for (int ix = 0; ix < ws; ++ix) {
                const int fx = cx * s + ix - (s - 1);
                if (fx < 0 || fx >= F.nnx) continue;
                const double w = wzy * hat(ix, s);
                const int m = Lf.mask[F.node(fx, fy, fz)];
                for (int c = 0; c < 3; ++c) v[c] = v[c] + ((m >> c) & 1 ? 1.0 : 0.0) * w;
                wsum = wsum + w;
            }
        }
    }
    int out = 0;
    for (int c = 0; c < 3; ++c) {
        const double r = wsum > 1e-12 ? v[c] / wsum : 0.0;
        if (r > 0.5) out |= 1 << c;
    }
    Lc.mask[n] = (uint8_t)out;
}

// ------------------------------------------------------------------ coarse diagonal (diagonal.cpp:66-138)
// Gather per coarse DOF: incident coarse elements in colour order, their (s+1)^3 sub-nodes in
// (iz,iy,ix) order, weight W_a^2, skipping fixed coarse or fine DOFs.
__global__ void k_diag_coarsen(MgLevel Lc, MgLevel Lf) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Lc.nn) return;
    const LevelIdx C(Lc), F(Lf);
    const int X = n % C.nnx, Y = (n / C.nnx) % C.nny, Z = n / (C.nnx * C.nny);
    const int s = Lc.span;
    const int cm = Lc.mask[n];
    const int64_t fNN = Lf.nn;
    double dc[3] = {0, 0, 0}, ws[3] = {0, 0, 0};
    for (int col = 0; col < 8; ++col) {
        const int ccx = (((X - 1) & 1) == (col & 1)) ? X - 1 : X;
        const int ccy = (((Lc.ny - Y) & 1) == ((col >> 1) & 1)) ? Y - 1 : Y;
        const int ccz = (((Z - 1) & 1) == ((col >> 2) & 1)) ? Z - 1 : Z;
        if (ccx < 0 || ccx >= Lc.nx || ccy < 0 || ccy >= Lc.ny || ccz < 0 || ccz >= Lc.nz) continue;
        const int a = corner_of(X - ccx, Y - ccy, Z - ccz);
        const int fx0 = ccx * s, fy0 = (ccy + 1) * s, fz0 = ccz * s;
        for (int iz = 0; iz <= s; ++iz)
            for (int iy = 0; iy <= s; ++iy)
                for (int ix = 0; ix <= s; ++ix) {
                    const int fn = F.node(fx0 + ix, fy0 - iy, fz0 + iz);
                    const double w = corner_weight(s, ix, iy, iz, a);
                    const double w2 = w * w;
                    const int fm = Lf.mask[fn];
                    for (int c = 0; c < 3; ++c) {
                        if (((cm >> c) & 1) || ((fm >> c) & 1)) continue;
                        dc[c] = dc[c] + w2 * Lf.diag[c * fNN + fn];
                        ws[c] = ws[c] + w2;
                    }
                }
    }
    for (int c = 0; c < 3; ++c) {
        double v;
        if ((cm >> c) & 1) v = 1.0;
        else if (ws[c] > 0) {
            v = dc[c] / ws[c];
            if (!(v > 0.0)) v = 1.0;
        } else v = 1.0;
        Lc.diag[c * Lc.nn + n] = v;
    }
}

// ------------------------------------------------------------------ restriction (transfers.cpp:449-533)
// The normalised hat-weighted window average, evaluated separably in three passes (x sums for each
// fine (z,y) row, then y, then z; each sum in increasing index order from 0; weight sum = product
// of the exact 1D sums), then scaled by 1/wSum and masked (preconditioner.cpp:183-191).  The CPU
// oracle's canonical mode evaluates the same order.
__global__ void k_restrict_x(MgLevel Lc, MgLevel Lf, const double* __restrict__ rf, double* __restrict__ a1,
                             const PcgScalars* S) {
    if (S != nullptr && S->done) return;
    const int cnx = Lc.nx + 1, fnx = Lf.nx + 1, fny = Lf.ny + 1, fnz = Lf.nz + 1;
    const int64_t total = (int64_t)fnz * fny * cnx;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int cx = (int)(t % cnx);
    const int64_t row = t / cnx;   // fz*fny + fy
    const int s = Lc.span, ws = 2 * s - 1;
    const int64_t fNN = Lf.nn;
    const double* __restrict__ src = rf + row * fnx;
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
    for (int ix = 0; ix < ws; ++ix) {
        const int fx = cx * s + ix - (s - 1);
        if (fx < 0 || fx >= fnx) continue;
        const double w = hat(ix, s);
        v0 = v0 + w * src[fx];
        v1 = v1 + w * src[fNN + fx];
        v2 = v2 + w * src[2 * fNN + fx];
    }
    a1[t] = v0;
    a1[total + t] = v1;
    a1[2 * total + t] = v2;
}

__global__ void k_restrict_y(MgLevel Lc, MgLevel Lf, const double* __restrict__ a1, double* __restrict__ a2,
                             const PcgScalars* S) {
    if (S != nullptr && S->done) return;
    const int cnx = Lc.nx + 1, cny = Lc.ny + 1, fny = Lf.ny + 1, fnz = Lf.nz + 1;
    const int64_t total = (int64_t)fnz * cny * cnx, total1 = (int64_t)fnz * fny * cnx;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int cx = (int)(t % cnx);
    const int cy = (int)((t / cnx) % cny);
    const int fz = (int)(t / ((int64_t)cnx * cny));
    const int s = Lc.span, ws = 2 * s - 1;
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
    for (int iy = 0; iy < ws; ++iy) {
        const int fy = cy * s + iy - (s - 1);
        if (fy < 0 || fy >= fny) continue;
        const double w = hat(iy, s);
        const int64_t i = ((int64_t)fz * fny + fy) * cnx + cx;
        v0 = v0 + w * a1[i];
        v1 = v1 + w * a1[total1 + i];
        v2 = v2 + w * a1[2 * total1 + i];
    }
    a2[t] = v0;
    a2[total + t] = v1;
    a2[2 * total + t] = v2;
}

// normalize = 0: the plain hat-weighted sum, i.e. the transpose of the trilinear prolongation (the
// 'Standard' V-cycle option)
__global__ void k_restrict_z(MgLevel Lc, MgLevel Lf, const double* __restrict__ a2, double* __restrict__ rc,
                             const PcgScalars* S, int normalize) {
    if (S != nullptr && S->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Lc.nn) return;
    const int cnx = Lc.nx + 1, cny = Lc.ny + 1;
    const int fnx = Lf.nx + 1, fny = Lf.ny + 1, fnz = Lf.nz + 1;
    const int cx = n % cnx, cy = (n / cnx) % cny, cz = n / (cnx * cny);
    const int s = Lc.span, ws = 2 * s - 1;
    const int64_t total2 = (int64_t)fnz * cny * cnx;
    double swx = 0.0, swy = 0.0, swz = 0.0;
    for (int i = 0; i < ws; ++i) {
        const int fx = cx * s + i - (s - 1), fy = cy * s + i - (s - 1);
        if (fx >= 0 && fx < fnx) swx = swx + hat(i, s);
        if (fy >= 0 && fy < fny) swy = swy + hat(i, s);
    }
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
    for (int iz = 0; iz < ws; ++iz) {
        const int fz = cz * s + iz - (s - 1);
        if (fz < 0 || fz >= fnz) continue;
        swz = swz + hat(iz, s);
        const double w = hat(iz, s);
        const int64_t i = ((int64_t)fz * cny + cy) * cnx + cx;
        v0 = v0 + w * a2[i];
        v1 = v1 + w * a2[total2 + i];
        v2 = v2 + w * a2[2 * total2 + i];
    }
    const double wsum = swz * swy * swx;
    double o0 = 0.0, o1 = 0.0, o2 = 0.0;
    if (!normalize) {
        o0 = v0;
        o1 = v1;
        o2 = v2;
    } else if (wsum > 1e-12) {
        const double iw = 1.0 / wsum;
        o0 = v0 * iw;
        o1 = v1 * iw;
        o2 = v2 * iw;
    }
    const int m = Lc.mask[n];
    rc[n] = (m & 1) ? 0.0 : o0;
    rc[Lc.nn + n] = (m & 2) ? 0.0 : o1;
    rc[2 * Lc.nn + n] = (m & 4) ? 0.0 : o2;
}

// coarsest Jacobi fallback x = r/max(1e-30,D) without weight, masked (preconditioner.cpp:199-227)
__global__ void k_coarse_jacobi(MgLevel L, const PcgScalars* S) {
    if (S != nullptr && S->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nn) return;
    const int m = L.mask[n];
    for (int c = 0; c < 3; ++c) {
        const double d = L.diag[c * L.nn + n];
        const double dd = 1.0e-30 < d ? d : 1.0e-30;
        L.x[c * L.nn + n] = ((m >> c) & 1) ? 0.0 : L.r[c * L.nn + n] / dd;
    }
}

// trilinear prolongation from the coarse cell floor(f/s), clamped to the last cell
// (transfers.cpp:378-445), then x = ((w r/D) + P x_c) + (w r/D), 0 on fixed DOFs
// (preconditioner.cpp:163-173, 230-253).
__device__ __forceinline__ void prolong_node(const MgLevel& Lc, int s, const double* __restrict__ xc, int fx, int fy,
                                             int fz, double P[3]) {
    const int cnx = Lc.nx + 1, cny = Lc.ny + 1;
    int cx = fx / s, cy = fy / s, cz = fz / s;
    int rx = fx % s, ry = fy % s, rz = fz % s;
    if (cx >= Lc.nx) { cx = Lc.nx - 1; rx = s; }
    if (cy >= Lc.ny) { cy = Lc.ny - 1; ry = s; }
    if (cz >= Lc.nz) { cz = Lc.nz - 1; rz = s; }
    const double inv = 1.0 / s;
    const double wx1 = rx * inv, wx0 = 1.0 - wx1;
    const double wy1 = ry * inv, wy0 = 1.0 - wy1;
    const double wz1 = rz * inv, wz0 = 1.0 - wz1;
    const int b = (cz * cny + cy) * cnx + cx;
    const int pz = cnx * cny;
    const int n000 = b, n100 = b + 1, n010 = b + cnx, n110 = b + cnx + 1;
    for (int c = 0; c < 3; ++c) {
        const double* X = xc + c * Lc.nn;
        P[c] = X[n000] * wx0 * wy0 * wz0 + X[n100] * wx1 * wy0 * wz0 + X[n010] * wx0 * wy1 * wz0 +
               X[n110] * wx1 * wy1 * wz0 + X[n000 + pz] * wx0 * wy0 * wz1 + X[n100 + pz] * wx1 * wy0 * wz1 +
               X[n010 + pz] * wx0 * wy1 * wz1 + X[n110 + pz] * wx1 * wy1 * wz1;
    }
}

__global__ void k_prolong_smooth(MgLevel Lc, MgLevel Lf, const double* __restrict__ xc,
                                 const double* __restrict__ rf, double* __restrict__ xf, double w,
                                 const PcgScalars* S) {
    if (S != nullptr && S->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Lf.nn) return;
    const int fnx = Lf.nx + 1, fny = Lf.ny + 1;
    const int fx = n % fnx, fy = (n / fnx) % fny, fz = n / (fnx * fny);
    double P[3];
    prolong_node(Lc, Lc.span, xc, fx, fy, fz, P);
    const int m = Lf.mask[n];
    for (int c = 0; c < 3; ++c) {
        const double d = Lf.diag[c * Lf.nn + n];
        const double dd = 1.0e-30 < d ? d : 1.0e-30;
        const double t = w * rf[c * Lf.nn + n] / dd;
        xf[c * Lf.nn + n] = ((m >> c) & 1) ? 0.0 : (t + P[c]) + t;
    }
}

// level 0: writes z and forms r.z in the canonical order; the last block sets rz (first use) or
// beta = rz_new/max(1e-30,rz), rz = rz_new (solver.cpp:186-198)
__global__ void __launch_bounds__(RED_THREADS) k_prolong_smooth0(MgLevel Lc, MgLevel Lf, const double* __restrict__ xc,
                                                                 const double* __restrict__ r, double* __restrict__ z,
                                                                 double w, RedSlot dot, PcgScalars* S) {
    __shared__ double sh[32];
    if (S->done) return;
    const int NN = (int)Lf.nn;
    const int fnx = Lf.nx + 1, fny = Lf.ny + 1;
    double part = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x) {
        const int fx = n % fnx, fy = (n / fnx) % fny, fz = n / (fnx * fny);
        double P[3];
        prolong_node(Lc, Lc.span, xc, fx, fy, fz, P);
        const int m = Lf.mask[n];
        for (int c = 0; c < 3; ++c) {
            const double d = Lf.diag[c * (int64_t)NN + n];
            const double dd = 1.0e-30 < d ? d : 1.0e-30;
            const double rv = r[c * (int64_t)NN + n];
            const double t = w * rv / dd;
            const double zv = ((m >> c) & 1) ? 0.0 : (t + P[c]) + t;
            z[c * (int64_t)NN + n] = zv;
            part = part + rv * zv;
        }
    }
    double tot;
    if (grid_fold(part, dot, sh, &tot) && threadIdx.x == 0) {
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

// ------------------------------------------------------------------ coarsest Galerkin (coarsest.cpp:138-323)
// One CTA (576 threads, thread = entry (i,j)) per coarse element.  The s^3 finest-grid sub-elements
// at the corner-sampled positions contribute T'(Kf T); Kf = Ke with modulus max(Emin,E) of the
// y-mirrored cell, with fixed DOFs' rows/cols replaced by identity when the sub-element touches any.
__global__ void __launch_bounds__(576) k_coarse_element(Grid g0, MgLevel Lc, int s, const uint8_t* __restrict__ mask0,
                                                        const double* __restrict__ E, const double* __restrict__ Keg,
                                                        double emin, double* __restrict__ Kce) {
    __shared__ double T[576], Kf[576], M[576];
    __shared__ int fmask[8];
    const int cel = blockIdx.x;   // (cez*nxc + cex)*nyc + cey
    const int nyc = Lc.ny, nxc = Lc.nx;
    const int cey = cel % nyc, cex = (cel / nyc) % nxc, cez = cel / (nyc * nxc);
    const int i = threadIdx.x / 24, j = threadIdx.x % 24;
    double acc_e = 0.0;
    for (int iz = 0; iz < s; ++iz)
        for (int iy = 0; iy < s; ++iy)
            for (int ix = 0; ix < s; ++ix) {
                const int fex = cex * s + ix, fey = (nyc - cey) * s - iy - 1, fez = cez * s + iz;
                double Ee = E[g0.cell(fex, g0.ny - 1 - fey, fez)];
                Ee = emin < Ee ? Ee : emin;
                if (threadIdx.x < 8) {
                    const int v = threadIdx.x;
                    fmask[v] = mask0[g0.node(fex + corner_dx(v), fey + corner_dy(v), fez + corner_dz(v))];
                }
                __syncthreads();
                int masked = 0;
                for (int v = 0; v < 8; ++v) masked |= fmask[v];
                {
                    // T[(3v+d), (3a+d)] = W_a at sub-node (ix+vx, iy+vy, iz+vz)
                    const int v = i / 3, d = i % 3, a = j / 3, e = j % 3;
                    const int vx = corner_dx(v), vy = 1 - corner_dy(v), vz = corner_dz(v);
                    T[threadIdx.x] = (d == e) ? corner_weight(s, ix + vx, iy + vy, iz + vz, a) : 0.0;
                    double k = masked ? Ee * Keg[threadIdx.x] : Keg[threadIdx.x];
                    if (masked) {
                        const int vi = i / 3, di = i % 3, vj = j / 3, dj = j % 3;
                        const int fi = (fmask[vi] >> di) & 1, fj = (fmask[vj] >> dj) & 1;
                        if (fi || fj) k = (i == j) ? 1.0 : 0.0;
                    }
                    Kf[threadIdx.x] = k;
                }
                __syncthreads();
                double m = 0.0;
                for (int k = 0; k < 24; ++k) m = m + Kf[i * 24 + k] * T[k * 24 + j];
                M[threadIdx.x] = m;
                __syncthreads();
                double acc = 0.0;
                for (int k = 0; k < 24; ++k) acc = acc + T[k * 24 + i] * M[k * 24 + j];
                acc_e = acc_e + (masked ? acc : Ee * acc);
                __syncthreads();
            }
    Kce[(int64_t)cel * 576 + threadIdx.x] = acc_e;
}

// Kc (row-major N x N, N = 3*coarse nodes, DOF 3n+c): lower-triangle sums over coarse elements in
// (cez, cex, cey) order, upper triangle 0, coarsest BC rows/cols -> identity (preconditioner.cpp:65-73)
__global__ void k_coarse_assemble(MgLevel Lc, const double* __restrict__ Kce, double* __restrict__ Kc) {
    const int N = 3 * (int)Lc.nn;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)N * N) return;
    const int gi = (int)(t / N), gj = (int)(t % N);
    const int nnx = Lc.nx + 1, nny = Lc.ny + 1;
    const int ni = gi / 3, ci = gi % 3, nj = gj / 3, cj = gj % 3;
    double v = 0.0;
    if (gi >= gj) {
        const int Xi = ni % nnx, Yi = (ni / nnx) % nny, Zi = ni / (nnx * nny);
        const int Xj = nj % nnx, Yj = (nj / nnx) % nny, Zj = nj / (nnx * nny);
        for (int ccz = Zi - 1; ccz <= Zi; ++ccz)
            for (int ccx = Xi - 1; ccx <= Xi; ++ccx)
                for (int ccy = Yi; ccy >= Yi - 1; --ccy) {   // cey = nyc-1-ccy ascending
                    if (ccx < 0 || ccx >= Lc.nx || ccy < 0 || ccy >= Lc.ny || ccz < 0 || ccz >= Lc.nz) continue;
                    const int dxj = Xj - ccx, dyj = Yj - ccy, dzj = Zj - ccz;
                    if (dxj < 0 || dxj > 1 || dyj < 0 || dyj > 1 || dzj < 0 || dzj > 1) continue;
                    const int ai = corner_of(Xi - ccx, Yi - ccy, Zi - ccz), aj = corner_of(dxj, dyj, dzj);
                    const int cel = (ccz * Lc.nx + ccx) * Lc.ny + (Lc.ny - 1 - ccy);
                    v = v + Kce[(int64_t)cel * 576 + (3 * ai + ci) * 24 + (3 * aj + cj)];
                }
    }
    const int mi = (Lc.mask[ni] >> ci) & 1, mj = (Lc.mask[nj] >> cj) & 1;
    if (mi || mj) v = (gi == gj) ? 1.0 : 0.0;
    Kc[t] = v;
}

// Cholesky of the lower triangle with the row-oriented sums of coarsest.cpp:13-35:
// L_ij = (A_ij - sum_{k<j} L_ik L_jk) / L_jj, L_jj = sqrt(A_jj - sum_{k<j} L_jk^2), sums in k order.
// Factor column j is LT[j*N + i] = L_ij.  Blocked right-looking: when column j is reached, LT holds in its rows
// i >= j the entry A_ij minus the products L_ik L_jk of the earlier columns, subtracted one at a time in
// increasing k -- the very sequence of the left-looking sum s = A_ij - L_i0 L_j0 - L_i1 L_j1 - ...
// (coarsest.cpp:24-58), so the factor is the same bit for bit.  Panels of CHOL_NB columns are factored by one
// CTA in shared memory; the panel's products are then subtracted from all later columns, in increasing k, by
// a grid of 32x32 tiles.  *status = 1 on success, 0 if not SPD (a non-positive pivot).
constexpr int CHOL_NB = 32;                  // panel width
constexpr int CHOL_SMEM_DOUBLES = 25600;     // panel bound: CHOL_NB x N doubles for N <= 800 (200 KB)
constexpr int CHOL_TILE = 32;

// LT = the lower triangle of A, transposed (column j contiguous); *status = 1
__global__ void k_chol_init(const double* __restrict__ A, double* __restrict__ LT, int N, int* status) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) *status = 1;
    if (t >= (int64_t)N * N) return;
    const int jj = (int)(t / N), ii = (int)(t % N);   // LT[jj][ii] = A[ii][jj] (lower)
    LT[t] = ii >= jj ? A[(int64_t)ii * N + jj] : 0.0;
}

// columns [k0, k1) of the factor, rows [k0, N): pan[c * R + o] = LT[(k0 + c) * N + k0 + o], R = N - k0
__global__ void __launch_bounds__(1024) k_chol_panel(double* __restrict__ LT, int N, int k0, int k1, int* status) {
    extern __shared__ double pan[];
    __shared__ int fail;
    if (*status == 0) return;   // an earlier panel failed (the same value for every thread)
    const int R = N - k0, W = k1 - k0;
    for (int t = threadIdx.x; t < W * R; t += blockDim.x) {
        const int c = t / R, o = t - c * R;
        pan[t] = LT[(int64_t)(k0 + c) * N + k0 + o];
    }
    if (threadIdx.x == 0) fail = 0;
    __syncthreads();
    for (int c = 0; c < W; ++c) {
        double* col = pan + c * R;   // column j = k0 + c; its row i at col[i - k0]
        if (threadIdx.x == 0) {
            const double s = col[c];
            if (s <= 0.0) fail = 1;
            else col[c] = sqrt(s);
        }
        __syncthreads();
        if (fail) break;
        const double ljj = col[c];
        for (int o = c + 1 + threadIdx.x; o < R; o += blockDim.x) col[o] = col[o] / ljj;
        __syncthreads();
        // the panel's later columns m = k0 + d, rows i >= m: subtract L_ij L_mj
        const int rest = W - c - 1;
        for (int t = threadIdx.x; t < rest * R; t += blockDim.x) {
            const int d = c + 1 + t / R, o = t % R;
            if (o >= d) pan[d * R + o] = pan[d * R + o] - col[o] * col[d];
        }
        __syncthreads();
    }
    if (fail) {
        if (threadIdx.x == 0) *status = 0;
        return;
    }
    for (int t = threadIdx.x; t < W * R; t += blockDim.x) {
        const int c = t / R, o = t - c * R;
        LT[(int64_t)(k0 + c) * N + k0 + o] = pan[t];
    }
}

// columns m >= k1, rows i >= m: subtract L_ij L_mj for the panel's columns j = k0..k1-1 in increasing j.
// Block t is the lower-triangular tile (bm <= bi) of 32 columns m and 32 rows i.
__global__ void __launch_bounds__(256) k_chol_trailing(double* __restrict__ LT, int N, int k0, int k1,
                                                       const int* status) {
    __shared__ double Pm[CHOL_NB][CHOL_TILE], Pi[CHOL_NB][CHOL_TILE];
    if (*status == 0) return;
    const int t = blockIdx.x;
    int bi = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
    while (bi * (bi + 1) / 2 > t) --bi;
    const int bm = t - bi * (bi + 1) / 2;
    const int m0 = k1 + bm * CHOL_TILE, i0 = k1 + bi * CHOL_TILE, W = k1 - k0;
    for (int q = threadIdx.x; q < W * CHOL_TILE; q += blockDim.x) {
        const int c = q / CHOL_TILE, x = q % CHOL_TILE;
        const double* Lj = LT + (int64_t)(k0 + c) * N;
        Pm[c][x] = m0 + x < N ? Lj[m0 + x] : 0.0;
        Pi[c][x] = i0 + x < N ? Lj[i0 + x] : 0.0;
    }
    __syncthreads();
    const int x = threadIdx.x % CHOL_TILE, y = threadIdx.x / CHOL_TILE;
    const int i = i0 + x;
    for (int u = y; u < CHOL_TILE; u += blockDim.x / CHOL_TILE) {
        const int m = m0 + u;
        if (m >= N || i >= N || i < m) continue;
        double* w = LT + (int64_t)m * N + i;
        double v = *w;
        for (int c = 0; c < W; ++c) v = v - Pi[c][x] * Pm[c][u];
        *w = v;
    }
}

// Lrow = the factor by rows (Lrow[i*N + j] = L_ij, 0 above the diagonal), written only on success
__global__ void k_chol_rows(const double* __restrict__ LT, double* __restrict__ Lrow, int N, const int* status) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)N * N || *status == 0) return;
    const int ii = (int)(t / N), jj = (int)(t % N);
    Lrow[t] = jj <= ii ? LT[(int64_t)jj * N + ii] : 0.0;
}

// Coarsest inverse for the canonical coarsest solve: column j of X = L'^-1 L^-1 e_j (coarsest.cpp:92-122),
// stored contiguously (X[j*N + i]).  A warp per column, both substitutions column-oriented: when x_k is final
// every row below takes its term L_ik x_k, so each row's running value receives its terms in increasing k
// (forward) and decreasing i (backward) and is divided last -- the order of the row-oriented sums, bit for bit.
// Rows above j are skipped in the forward pass: their values stay +0 and leave the others unchanged (each
// running value there is +0 or 1, never -0).  The warp's lanes split the rows; the factor is read by columns
// (LT) in the forward pass and by rows (Lrow) in the backward one, both coalesced.
constexpr int INV_WARPS = 8;   // columns per block
constexpr int INV_MAX_N = 1000;   // the largest dense coarsest system (NlimitDofs)
__global__ void __launch_bounds__(INV_WARPS * 32) k_coarse_inverse(const double* __restrict__ LT,
                                                                   const double* __restrict__ Lrow, int N,
                                                                   const int* __restrict__ status,
                                                                   double* __restrict__ X) {
    extern __shared__ double xs_all[];   // [INV_WARPS][N]
    if (*status != 1) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int j = blockIdx.x * INV_WARPS + w;
    if (j >= N) return;   // the whole warp (no block barrier below)
    double* xs = xs_all + (int64_t)w * N;
    for (int i = lane; i < N; i += 32) xs[i] = (i == j) ? 1.0 : 0.0;
    __syncwarp();
    for (int k = j; k < N; ++k) {
        const double xk = xs[k] / Lrow[(int64_t)k * N + k];
        __syncwarp();
        if (lane == (k & 31)) xs[k] = xk;
        const double* __restrict__ Lk = LT + (int64_t)k * N;   // column k: L_ik at Lk[i]
        for (int i = k + 1 + lane; i < N; i += 32) xs[i] = xs[i] - Lk[i] * xk;
        __syncwarp();
    }
    for (int i = N - 1; i >= 0; --i) {
        const double* __restrict__ Li = Lrow + (int64_t)i * N;
        const double xi = xs[i] / Li[i];
        __syncwarp();
        if (lane == (i & 31)) xs[i] = xi;
        for (int k = lane; k < i; k += 32) xs[k] = xs[k] - Li[k] * xi;
        __syncwarp();
    }
    for (int i = lane; i < N; i += 32) X[(int64_t)j * N + i] = xs[i];
}

// Coarsest solve x_i = sum_j X[i][j] r_j (sequential in j) when the factorisation succeeded, else
// the Jacobi fallback x = r/max(1e-30,D) (preconditioner.cpp:195-215); masked (:217-227).
__global__ void __launch_bounds__(128) k_coarse_solve(MgLevel L, const double* __restrict__ X, int N,
                                                      const int* __restrict__ status, const PcgScalars* S) {
    extern __shared__ double rs[];
    if (S != nullptr && S->done) return;
    const int64_t nn = L.nn;
    if (*status != 1) {
        for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
            const int m = L.mask[n];
            for (int c = 0; c < 3; ++c) {
                const double d = L.diag[c * nn + n];
                const double dd = 1.0e-30 < d ? d : 1.0e-30;
                L.x[c * nn + n] = ((m >> c) & 1) ? 0.0 : L.r[c * nn + n] / dd;
            }
        }
        return;
    }
    for (int j = threadIdx.x; j < N; j += blockDim.x) rs[j] = L.r[(j % 3) * nn + j / 3];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double acc = 0.0;
    for (int j = 0; j < N; ++j) acc = acc + X[(int64_t)j * N + i] * rs[j];
    const int ni = i / 3, ci = i % 3;
    L.x[ci * nn + ni] = ((L.mask[ni] >> ci) & 1) ? 0.0 : acc;
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void launch_mask_restrict(const MgLevel& Lc, const MgLevel& Lf, cudaStream_t s) {
    k_mask_restrict<<<blocks_for(Lc.nn, 128), 128, 0, s>>>(Lc, Lf);
}
void launch_diag_coarsen(const MgLevel& Lc, const MgLevel& Lf, cudaStream_t s) {
    k_diag_coarsen<<<blocks_for(Lc.nn, 128), 128, 0, s>>>(Lc, Lf);
}
void launch_restrict(const MgLevel& Lc, const MgLevel& Lf, const double* rf, double* rc, double* a1, double* a2,
                     const PcgScalars* S, cudaStream_t s, bool normalize) {
    const int64_t n1 = (int64_t)(Lf.nz + 1) * (Lf.ny + 1) * (Lc.nx + 1);
    const int64_t n2 = (int64_t)(Lf.nz + 1) * (Lc.ny + 1) * (Lc.nx + 1);
    k_restrict_x<<<blocks_for(n1, 256), 256, 0, s>>>(Lc, Lf, rf, a1, S);
    k_restrict_y<<<blocks_for(n2, 256), 256, 0, s>>>(Lc, Lf, a1, a2, S);
    k_restrict_z<<<blocks_for(Lc.nn, 128), 128, 0, s>>>(Lc, Lf, a2, rc, S, normalize ? 1 : 0);
}
void launch_coarse_jacobi(const MgLevel& L, const PcgScalars* S, cudaStream_t s) {
    k_coarse_jacobi<<<blocks_for(L.nn, 128), 128, 0, s>>>(L, S);
}
void launch_prolong_smooth(const MgLevel& Lc, const MgLevel& Lf, const double* xc, const double* rf, double* xf,
                           double weight, const PcgScalars* S, cudaStream_t s) {
    k_prolong_smooth<<<blocks_for(Lf.nn, 256), 256, 0, s>>>(Lc, Lf, xc, rf, xf, weight, S);
}
void launch_prolong_smooth0(const MgLevel& Lc, const MgLevel& Lf, const double* xc, const double* r, double* z,
                            double weight, RedSlot dot, PcgScalars* S, cudaStream_t s) {
    k_prolong_smooth0<<<RED_BLOCKS, RED_THREADS, 0, s>>>(Lc, Lf, xc, r, z, weight, dot, S);
}
void launch_coarse_element_matrices(const Grid& g0, const MgLevel& Lc, int span, const uint8_t* mask0, const double* E,
                                    const double* Ke, double emin, double* Kce, cudaStream_t s) {
    const int ncel = Lc.nx * Lc.ny * Lc.nz;
    k_coarse_element<<<ncel, 576, 0, s>>>(g0, Lc, span, mask0, E, Ke, emin, Kce);
}
void launch_coarse_assemble(const MgLevel& Lc, const double* Kce, double* Kc, cudaStream_t s) {
    const int64_t N = 3 * Lc.nn;
    k_coarse_assemble<<<blocks_for(N * N, 256), 256, 0, s>>>(Lc, Kce, Kc);
}
int launch_cholesky(const double* A, double* LT, double* Lrow, int N, int* status, cudaStream_t s) {
    const int64_t NN = (int64_t)N * N;
    k_chol_init<<<std::max(1u, blocks_for(NN, 256)), 256, 0, s>>>(A, LT, N, status);
    int launches = 1;
    if (N <= 0) return launches;
    const int nb = std::max(1, std::min(CHOL_NB, CHOL_SMEM_DOUBLES / N));
    // the attribute is per function, not per launch: always the bound, so that contexts set up concurrently
    // from several host threads never lower it under another thread's launch
    cudaFuncSetAttribute(k_chol_panel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(CHOL_SMEM_DOUBLES * sizeof(double)));
    for (int k0 = 0; k0 < N; k0 += nb) {
        const int k1 = std::min(k0 + nb, N);
        k_chol_panel<<<1, 1024, (size_t)(k1 - k0) * (N - k0) * sizeof(double), s>>>(LT, N, k0, k1, status);
        const int T = (N - k1 + CHOL_TILE - 1) / CHOL_TILE;
        if (T > 0) k_chol_trailing<<<T * (T + 1) / 2, 256, 0, s>>>(LT, N, k0, k1, status);
        launches += T > 0 ? 2 : 1;
    }
    k_chol_rows<<<blocks_for(NN, 256), 256, 0, s>>>(LT, Lrow, N, status);
    return launches + 1;
}
void launch_coarse_inverse(const double* LT, const double* Lrow, int N, const int* status, double* X,
                           cudaStream_t s) {
    const size_t smem = (size_t)N * INV_WARPS * sizeof(double);   // N <= 1000: at most 64 KB
    // the attribute is per function, not per launch: always the bound for the largest N, so that contexts set
    // up concurrently from several host threads never lower it under another thread's launch
    cudaFuncSetAttribute(k_coarse_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(INV_MAX_N * INV_WARPS * sizeof(double)));
    k_coarse_inverse<<<blocks_for(N, INV_WARPS), INV_WARPS * 32, smem, s>>>(LT, Lrow, N, status, X);
}
void launch_coarse_solve(const MgLevel& L, const double* X, int N, const int* status, const PcgScalars* S,
                         cudaStream_t s) {
    const int64_t work = N > 0 ? N : L.nn;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, (work + 127) / 128);
    k_coarse_solve<<<blocks, 128, (size_t)std::max(N, 1) * sizeof(double), s>>>(L, X, N, status, S);
}

}  // namespace t3d
