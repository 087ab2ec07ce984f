// The 'Standard' V-cycle (TOP3D_XL.m:772-807; FP64 form and derivation in k_mg_standard.cu) in FP32 for the
// mixed-precision inner solve:
//
//   down, l = 0..L-2:  x_l = w r_l / D_l;  r_{l+1} = P^T (r_l - K_l x_l)
//   coarsest:          x_L = K_L^{-1} r_L  (the FP64 inverse of the Galerkin coarsest matrix)
//   up,   l = L-2..0:  x_l += P x_{l+1};  x_l += w (r_l - K_l x_l) / D_l
//
// FP32 storage and arithmetic: the level vectors, the reciprocal diagonals 1/D_l, the Galerkin element
// matrices of the coarse levels (FP32 images of the FP64 set-up), and K_0 = the modal FP32 K(E) of the moduli
// the hierarchy was built from.  Level 0's vectors are pitched (Grid::px rows, MgLevel32::pitch/cs); the
// coarse levels' are not.  Every kernel skips its work once S->done (the inner PCG converged).
#include <type_traits>

#include "kernels.hpp"
#include "red.cuh"

namespace t3d {

namespace {

__device__ __forceinline__ float tri_wf(int s, int fx, int fy, int fz, int A) {
    const float is = 1.0f / (float)s;   // s is 2 or 4: exact
    const float wx = corner_dx(A) ? fx * is : (s - fx) * is;
    const float wy = corner_dy(A) ? fy * is : (s - fy) * is;
    const float wz = corner_dz(A) ? fz * is : (s - fz) * is;
    return wx * wy * wz;
}

// node n (unpadded, the mask's index) of level L -> index into its (possibly pitched) vectors
__device__ __forceinline__ int64_t vidx(const MgLevel32& L, int64_t n) {
    const int nnx = L.nx + 1;
    return (n / nnx) * L.pitch + n % nnx;
}

template <class V>
__device__ __forceinline__ float& lane_of(V& v, int k) {
    return reinterpret_cast<float*>(&v)[k];
}
template <class V>
__device__ __forceinline__ float lane_of(const V& v, int k) {
    return reinterpret_cast<const float*>(&v)[k];
}

// x = w r / D on the pitched finest level: 4 consecutive row entries per thread (16-byte loads and stores of the
// pitched vectors; the row's pads past x = nx stay zero).  Same arithmetic per DOF as the generic loop.
__device__ __forceinline__ void jacobi_init0_32(VB vb, const MgLevel32& L, const float* __restrict__ r,
                                               float* __restrict__ x, float w) {
    const int fnx = L.nx + 1, q4 = L.pitch >> 2;
    const int64_t rows = (int64_t)(L.ny + 1) * (L.nz + 1), per_c = rows * q4;
    for (int64_t t = (int64_t)vb.b * blockDim.x + threadIdx.x; t < 3 * per_c; t += (int64_t)vb.n * blockDim.x) {
        const int c = (int)(t / per_c);
        const int64_t rt = t - c * per_c, row = rt / q4;
        const int x0 = 4 * (int)(rt - row * q4);
        const int64_t i = c * L.cs + row * L.pitch + x0;
        const float4 rv = *reinterpret_cast<const float4*>(r + i), dv = *reinterpret_cast<const float4*>(L.diag + i);
        float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
        const uint8_t* mk = L.mask + row * fnx;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int fx = x0 + k;
            if (fx < fnx && !((mk[fx] >> c) & 1)) lane_of(o, k) = (w * lane_of(rv, k)) * lane_of(dv, k);
        }
        *reinterpret_cast<float4*>(x + i) = o;
    }
}

// xo = xi + P xc on the pitched finest level.  A thread takes a run of SP consecutive fine nodes of one row that
// share one coarse cell (fine x = SP j + k; the row's last node, x = nx, clamped to the last coarse cell, is a run
// of its own): the cell's 8 corners are loaded once for the run and its nodes move as one SP-wide vector.
// Consecutive threads take consecutive runs across row ends.  Same weights and accumulation order per node as
// the generic loop of prolong_add32.
template <int SP>
__device__ __forceinline__ void prolong_add0_32(VB vb, const MgLevel32& Lc, const MgLevel32& Lf,
                                                const float* __restrict__ xc, const float* xi, float* xo) {
    using V = typename std::conditional<SP == 4, float4, float2>::type;
    const int fnx = Lf.nx + 1, fny = Lf.ny + 1, cnx = Lc.nx + 1, cny = Lc.ny + 1;
    const int runs = Lc.nx + 1;   // Lf.nx = SP Lc.nx: Lc.nx runs of SP nodes and the last node
    const int64_t total = (int64_t)runs * fny * (Lf.nz + 1);
    for (int64_t t = (int64_t)vb.b * blockDim.x + threadIdx.x; t < total; t += (int64_t)vb.n * blockDim.x) {
        const int64_t row = t / runs;
        const int j = (int)(t - row * runs);
        const int fz = (int)(row / fny), fy = (int)(row - (int64_t)fz * fny);
        const bool last = j == Lc.nx;
        const int cx = last ? Lc.nx - 1 : j;
        int cy = fy / SP, cz = fz / SP;
        if (cy >= Lc.ny) cy = Lc.ny - 1;
        if (cz >= Lc.nz) cz = Lc.nz - 1;
        // the run's fine rows are loaded first, so that their HBM reads and the coarse corners' L2 reads are in
        // flight together (xo may be xi: every read of the run precedes its writes, as before)
        const int64_t rb = row * Lf.pitch + SP * j;
        V v[3];
        if (!last) {
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] = *reinterpret_cast<const V*>(xi + c * Lf.cs + rb);
        }
        float X[3][8];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int A = 0; A < 8; ++A)
                X[c][A] = xc[c * Lc.cs + ((int64_t)(cz + corner_dz(A)) * cny + cy + corner_dy(A)) * cnx + cx +
                             corner_dx(A)];
        // the weights tri_wf(...) = w_x w_y w_z are products of multiples of 1/SP (SP = 2, 4): exact in any
        // order, so w_y w_z is formed once per run and w_x per node, giving the same values bit for bit
        constexpr float is = 1.0f / (float)SP;
        const int ry = fy - cy * SP, rz = fz - cz * SP;
        float wyz[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            wyz[q] = ((q & 1) ? ry * is : (SP - ry) * is) * ((q & 2) ? rz * is : (SP - rz) * is);
        const uint8_t* mk = Lf.mask + row * fnx;
        if (last) {   // x = nx: one node, all weight on the cell's upper x corners
            const int fx = Lf.nx, m = mk[fx];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float p = 0.0f;
#pragma unroll
                for (int A = 0; A < 8; ++A)
                    p = fmaf((corner_dx(A) ? 1.0f : 0.0f) * wyz[corner_dy(A) + 2 * corner_dz(A)], X[c][A], p);
                const int64_t i = c * Lf.cs + row * Lf.pitch + fx;
                xo[i] = ((m >> c) & 1) ? 0.0f : xi[i] + p;
            }
            continue;
        }
        int m[SP];
        float w[SP][8];
#pragma unroll
        for (int k = 0; k < SP; ++k) {
            m[k] = mk[SP * j + k];
#pragma unroll
            for (int A = 0; A < 8; ++A)
                w[k][A] = (corner_dx(A) ? k * is : (SP - k) * is) * wyz[corner_dy(A) + 2 * corner_dz(A)];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            V o;
#pragma unroll
            for (int k = 0; k < SP; ++k) {
                float p = 0.0f;
#pragma unroll
                for (int A = 0; A < 8; ++A) p = fmaf(w[k][A], X[c][A], p);
                lane_of(o, k) = ((m[k] >> c) & 1) ? 0.0f : lane_of(v[c], k) + p;
            }
            *reinterpret_cast<V*>(xo + c * Lf.cs + rb) = o;
        }
    }
}

// x = w r / D
// (kernel bodies take the logical block VB, so that the batched launches below run them unchanged)
__device__ __forceinline__ void jacobi_init32(VB vb, const MgLevel32& L, const float* __restrict__ r,
                                              float* __restrict__ x, float w, const PcgScalars* S) {
    if (S->done) return;
    if (L.pitch != L.nx + 1) {   // the pitched finest level
        jacobi_init0_32(vb, L, r, x, w);
        return;
    }
    for (int64_t n = (int64_t)vb.b * blockDim.x + threadIdx.x; n < L.nn; n += (int64_t)vb.n * blockDim.x) {
        const int m = L.mask[n];
        const int64_t v = vidx(L, n);
        for (int c = 0; c < 3; ++c) {
            const int64_t i = c * L.cs + v;
            x[i] = ((m >> c) & 1) ? 0.0f : (w * r[i]) * L.diag[i];
        }
    }
}

__global__ void k_jacobi_init32(MgLevel32 L, const float* __restrict__ r, float* __restrict__ x, float w,
                                const PcgScalars* S) {
    jacobi_init32(vb_real(), L, r, x, w, S);
}

// kx <- r - kx
__device__ __forceinline__ void residual32(VB vb, const MgLevel32& L, const float* __restrict__ r,
                                           float* __restrict__ kx, const PcgScalars* S) {
    if (S->done) return;
    for (int64_t n = (int64_t)vb.b * blockDim.x + threadIdx.x; n < L.nn; n += (int64_t)vb.n * blockDim.x) {
        const int m = L.mask[n];
        const int64_t v = vidx(L, n);
        for (int c = 0; c < 3; ++c) {
            const int64_t i = c * L.cs + v;
            kx[i] = ((m >> c) & 1) ? 0.0f : r[i] - kx[i];
        }
    }
}

__global__ void k_residual32(MgLevel32 L, const float* __restrict__ r, float* __restrict__ kx, const PcgScalars* S) {
    residual32(vb_real(), L, r, kx, S);
}

// x += w (r - kx) / D
__device__ __forceinline__ void jacobi_correct32(VB vb, const MgLevel32& L, const float* __restrict__ r,
                                                 const float* __restrict__ kx, float* __restrict__ x, float w,
                                                 const PcgScalars* S) {
    if (S->done) return;
    for (int64_t n = (int64_t)vb.b * blockDim.x + threadIdx.x; n < L.nn; n += (int64_t)vb.n * blockDim.x) {
        const int m = L.mask[n];
        const int64_t v = vidx(L, n);
        for (int c = 0; c < 3; ++c) {
            const int64_t i = c * L.cs + v;
            x[i] = ((m >> c) & 1) ? 0.0f : x[i] + (w * (r[i] - kx[i])) * L.diag[i];
        }
    }
}

__global__ void k_jacobi_correct32(MgLevel32 L, const float* __restrict__ r, const float* __restrict__ kx,
                                   float* __restrict__ x, float w, const PcgScalars* S) {
    jacobi_correct32(vb_real(), L, r, kx, x, w, S);
}

// xo = xi + P xc (trilinear from the coarse cell floor(f/s), clamped to the last cell), fixed DOFs 0; xo may be xi
__device__ __forceinline__ void prolong_add32(VB vb, const MgLevel32& Lc, const MgLevel32& Lf,
                                              const float* __restrict__ xc, const float* xi, float* xo,
                                              const PcgScalars* S) {
    if (S->done) return;
    if (Lf.pitch != Lf.nx + 1 && (Lc.span == 2 || Lc.span == 4) && Lf.nx == Lc.span * Lc.nx) {   // pitched level 0
        if (Lc.span == 4) prolong_add0_32<4>(vb, Lc, Lf, xc, xi, xo);
        else prolong_add0_32<2>(vb, Lc, Lf, xc, xi, xo);
        return;
    }
    const int s = Lc.span;
    const int fnx = Lf.nx + 1, fny = Lf.ny + 1, cnx = Lc.nx + 1, cny = Lc.ny + 1;
    for (int64_t n = (int64_t)vb.b * blockDim.x + threadIdx.x; n < Lf.nn; n += (int64_t)vb.n * blockDim.x) {
        const int fx = (int)(n % fnx), fy = (int)((n / fnx) % fny), fz = (int)(n / ((int64_t)fnx * fny));
        int cx = fx / s, cy = fy / s, cz = fz / s;
        if (cx >= Lc.nx) cx = Lc.nx - 1;
        if (cy >= Lc.ny) cy = Lc.ny - 1;
        if (cz >= Lc.nz) cz = Lc.nz - 1;
        const int m = Lf.mask[n];
        const int64_t v = vidx(Lf, n);
        for (int c = 0; c < 3; ++c) {
            float p = 0.0f;
            for (int A = 0; A < 8; ++A)
                p = fmaf(tri_wf(s, fx - cx * s, fy - cy * s, fz - cz * s, A),
                         xc[c * Lc.cs + ((int64_t)(cz + corner_dz(A)) * cny + cy + corner_dy(A)) * cnx + cx + corner_dx(A)],
                         p);
            const int64_t i = c * Lf.cs + v;
            xo[i] = ((m >> c) & 1) ? 0.0f : xi[i] + p;
        }
    }
}
__global__ void k_prolong_add32(MgLevel32 Lc, MgLevel32 Lf, const float* __restrict__ xc, const float* xi, float* xo,
                                const PcgScalars* S) {
    prolong_add32(vb_real(), Lc, Lf, xc, xi, xo, S);
}

// packed position of entry (i, j) of a symmetric 24x24 matrix: the upper triangle row by row, 300 entries
__host__ __device__ constexpr int sym_pack(int i, int j) {
    return i <= j ? i * 24 - i * (i - 1) / 2 + (j - i) : j * 24 - j * (j - 1) / 2 + (i - j);
}
constexpr int SYM_N = 300;

// y = K_l x from the FP32 element matrices of a coarse level, stored symmetric-packed and entry-major (entry p of
// element e at p * ne + e; the Galerkin operators P^T K P are symmetric).  Node-centric gather: each node reads
// the three rows of its corner in the 8 element matrices around it (all loops unrolled, so the packed positions
// are constants); consecutive nodes read consecutive addresses.  Fixed DOFs 0.
__device__ __forceinline__ void level_matvec32(VB vb, const MgLevel32& L, const float* __restrict__ Kel,
                                               const float* __restrict__ x, float* __restrict__ y,
                                               const PcgScalars* S) {
    if (S->done) return;
    const int nnx = L.nx + 1, nny = L.ny + 1;
    const int64_t ne = (int64_t)L.nx * L.ny * L.nz;
    for (int64_t n = (int64_t)vb.b * blockDim.x + threadIdx.x; n < L.nn; n += (int64_t)vb.n * blockDim.x) {
        const int X = (int)(n % nnx), Y = (int)((n / nnx) % nny), Z = (int)(n / ((int64_t)nnx * nny));
        float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f;
#pragma unroll
        for (int dz = 0; dz <= 1; ++dz)
#pragma unroll
            for (int dy = 0; dy <= 1; ++dy)
#pragma unroll
                for (int dx = 0; dx <= 1; ++dx) {
                    const int ex = X - dx, ey = Y - dy, ez = Z - dz;
                    if (ex < 0 || ey < 0 || ez < 0 || ex >= L.nx || ey >= L.ny || ez >= L.nz) continue;
                    const int a = corner_of(dx, dy, dz);
                    const float* K = Kel + ((int64_t)(ez * L.ny + ey) * L.nx + ex);
#pragma unroll
                    for (int b = 0; b < 8; ++b) {
                        const int64_t m = ((int64_t)(ez + corner_dz(b)) * nny + ey + corner_dy(b)) * nnx + ex + corner_dx(b);
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const float xv = x[c * L.cs + m];
                            acc0 = fmaf(K[sym_pack(3 * a, 3 * b + c) * ne], xv, acc0);
                            acc1 = fmaf(K[sym_pack(3 * a + 1, 3 * b + c) * ne], xv, acc1);
                            acc2 = fmaf(K[sym_pack(3 * a + 2, 3 * b + c) * ne], xv, acc2);
                        }
                    }
                }
        const int mk = L.mask[n];
        y[n] = (mk & 1) ? 0.0f : acc0;
        y[L.cs + n] = (mk & 2) ? 0.0f : acc1;
        y[2 * L.cs + n] = (mk & 4) ? 0.0f : acc2;
    }
}
__global__ void k_level_matvec32(MgLevel32 L, const float* __restrict__ Kel, const float* __restrict__ x,
                                 float* __restrict__ y, const PcgScalars* S) {
    level_matvec32(vb_real(), L, Kel, x, y, S);
}

// FP32 symmetric-packed, entry-major image of element-major FP64 element matrices (the upper triangle):
// dst[p * ne + e] = src[e * 576 + 24 i + j], (i, j) the p-th upper-triangle entry
__global__ void k_kel_pack32(int64_t ne, const double* __restrict__ src, float* __restrict__ dst) {
    __shared__ short ij[SYM_N];
    for (int p = threadIdx.x + threadIdx.y * 32; p < SYM_N; p += 32 * blockDim.y) {
        int i = 0, q = p;
        while (q >= 24 - i) {
            q -= 24 - i;
            ++i;
        }
        ij[p] = (short)(i * 24 + i + q);
    }
    __syncthreads();
    const int64_t e = (int64_t)blockIdx.x * 32 + threadIdx.x;
    if (e >= ne) return;
    for (int p = threadIdx.y; p < SYM_N; p += blockDim.y) dst[(int64_t)p * ne + e] = (float)src[e * 576 + ij[p]];
}

// r.z over pitched FP32 vectors (pads zero), accumulated in FP64; the last block sets rz (first use) or
// beta = rz_new / max(1e-30, rz), rz = rz_new
__global__ void __launch_bounds__(RED_THREADS) k_dot_rz32(int64_t n3, const float* __restrict__ r,
                                                          const float* __restrict__ z, RedSlot red, PcgScalars* S) {
    __shared__ double sh[32];
    if (S->done) return;
    const int64_t n4 = n3 >> 2;
    const float4* r4 = reinterpret_cast<const float4*>(r);
    const float4* z4 = reinterpret_cast<const float4*>(z);
    double part = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 a = r4[i], b = z4[i];
        part += (double)fmaf(a.w, b.w, fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)));
    }
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

inline unsigned blocks_of(int64_t n, int t) {
    const int64_t b = (n + t - 1) / t;
    return (unsigned)(b < 8 * RED_BLOCKS ? (b > 0 ? b : 1) : 8 * RED_BLOCKS);
}

// ---------------------------------------------------------------- batched launches (persistent grids)
__global__ void __launch_bounds__(256) k_batch_level_op32(const BatchLevelOp* __restrict__ a,
                                                          const int* __restrict__ act, int N, int op) {
    batch_walk(a, act, N, [&](const BatchLevelOp& A, VB vb) {
        const MgLevel32 L = A.L;
        if (op == 0) jacobi_init32(vb, L, A.r, A.x, A.w, A.S);
        else if (op == 1) residual32(vb, L, A.r, A.kx, A.S);
        else jacobi_correct32(vb, L, A.r, A.kx, A.x, A.w, A.S);
    });
}
__global__ void __launch_bounds__(256) k_batch_prolong_add32(const BatchProlongAdd* __restrict__ a,
                                                             const int* __restrict__ act, int N) {
    batch_walk(a, act, N, [&](const BatchProlongAdd& A, VB vb) {
        const MgLevel32 Lc = A.Lc, Lf = A.Lf;
        prolong_add32(vb, Lc, Lf, A.xc, A.xi, A.xo, A.S);
    });
}
__global__ void __launch_bounds__(128) k_batch_level_matvec32(const BatchLevelMatvec* __restrict__ a,
                                                              const int* __restrict__ act, int N) {
    batch_walk(a, act, N, [&](const BatchLevelMatvec& A, VB vb) {
        const MgLevel32 L = A.L;
        level_matvec32(vb, L, A.Kel, A.x, A.y, A.S);
    });
}
constexpr int BATCH_GRID256 = 8 * 148, BATCH_GRID128 = 16 * 148;

}  // namespace

int batch_blocks_level_op(const BatchLevelOp& a) { return (int)blocks_of(a.L.nn, 256); }
int batch_blocks_prolong_add(const BatchProlongAdd& a) { return (int)blocks_of(a.Lf.nn, 256); }
int batch_blocks_level_matvec(const BatchLevelMatvec& a) { return (int)blocks_of(a.L.nn, 128); }
void launch_batch_level_op32(const BatchLevelOp* a, const int* act, int N, int op, cudaStream_t s) {
    k_batch_level_op32<<<BATCH_GRID256, 256, 0, s>>>(a, act, N, op);
}
void launch_batch_prolong_add32(const BatchProlongAdd* a, const int* act, int N, cudaStream_t s) {
    k_batch_prolong_add32<<<BATCH_GRID256, 256, 0, s>>>(a, act, N);
}
void launch_batch_level_matvec32(const BatchLevelMatvec* a, const int* act, int N, cudaStream_t s) {
    k_batch_level_matvec32<<<BATCH_GRID128, 128, 0, s>>>(a, act, N);
}

void launch_jacobi_init32(const MgLevel32& L, const float* r, float* x, float w, const PcgScalars* S, cudaStream_t s) {
    k_jacobi_init32<<<blocks_of(L.nn, 256), 256, 0, s>>>(L, r, x, w, S);
}
void launch_residual32(const MgLevel32& L, const float* r, float* kx, const PcgScalars* S, cudaStream_t s) {
    k_residual32<<<blocks_of(L.nn, 256), 256, 0, s>>>(L, r, kx, S);
}
void launch_jacobi_correct32(const MgLevel32& L, const float* r, const float* kx, float* x, float w,
                             const PcgScalars* S, cudaStream_t s) {
    k_jacobi_correct32<<<blocks_of(L.nn, 256), 256, 0, s>>>(L, r, kx, x, w, S);
}
void launch_prolong_add32(const MgLevel32& Lc, const MgLevel32& Lf, const float* xc, const float* xi, float* xo,
                          const PcgScalars* S, cudaStream_t s) {
    k_prolong_add32<<<blocks_of(Lf.nn, 256), 256, 0, s>>>(Lc, Lf, xc, xi, xo, S);
}
void launch_level_matvec32(const MgLevel32& L, const float* Kel, const float* x, float* y, const PcgScalars* S,
                           cudaStream_t s) {
    k_level_matvec32<<<blocks_of(L.nn, 128), 128, 0, s>>>(L, Kel, x, y, S);
}
void launch_kel_pack32(int64_t ne, const double* Kel, float* KelP32, cudaStream_t s) {
    k_kel_pack32<<<(unsigned)((ne + 31) / 32), dim3(32, 8), 0, s>>>(ne, Kel, KelP32);
}
void launch_dot_rz32(int64_t n3, const float* r, const float* z, RedSlot red, PcgScalars* S, cudaStream_t s) {
    k_dot_rz32<<<RED_BLOCKS, RED_THREADS, 0, s>>>(n3, r, z, red, S);
}

}  // namespace t3d
