// PCG vector steps of PCG_free (solver.cpp:87-217) on device-resident scalars.
// Each kernel returns at once when the solve has converged (S->done), so a fixed sequence of
// iterations can be queued (or replayed from a CUDA graph) without host round trips.
#include "kernels.hpp"
#include "red.cuh"

namespace t3d {

namespace {

// r = b - A x and b.b; initialises the scalars (solver.cpp:111-149)
__global__ void __launch_bounds__(RED_THREADS) k_pcg_init(Grid g, const double* __restrict__ b,
                                                          const double* __restrict__ Ax, double* __restrict__ r,
                                                          RedSlot red, PcgScalars* S, double tol) {
    __shared__ double sh[32];
    const int NN = (int)g.NN;
    double part = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c) {
            const int64_t i = c * (int64_t)NN + n;
            const double bv = b[i];
            r[i] = bv - Ax[i];
            part = part + bv * bv;
        }
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) {
        const double nb = sqrt(tot);
        S->bnorm2 = tot;
        S->stop = (1.0e-30 < nb ? nb : 1.0e-30) * tol;
        S->tol = tol;
        S->it = 0;
        S->done = 0;
        S->result = 0;
        S->first = 1;
    }
}

// x += alpha p; r -= alpha Ap; |r|^2; convergence (solver.cpp:171-184)
__global__ void __launch_bounds__(RED_THREADS) k_pcg_update(Grid g, double* __restrict__ x, double* __restrict__ r,
                                                            const double* __restrict__ p,
                                                            const double* __restrict__ Ap, RedSlot red,
                                                            PcgScalars* S) {
    __shared__ double sh[32];
    if (S->done) return;
    const double den = S->denom;
    const double alpha = S->rz / (1.0e-30 < den ? den : 1.0e-30);
    const int NN = (int)g.NN;
    double part = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c) {
            const int64_t i = c * (int64_t)NN + n;
            x[i] = x[i] + alpha * p[i];
            const double rv = r[i] - alpha * Ap[i];
            r[i] = rv;
            part = part + rv * rv;
        }
    double tot;
    if (grid_fold(part, red, sh, &tot) && threadIdx.x == 0) {
        S->rnorm2 = tot;
        S->it = S->it + 1;
        if (sqrt(tot) < S->stop) {
            S->done = 1;
            S->result = S->it;
        }
    }
}

// p = z + beta p (solver.cpp:200-204)
__global__ void k_pcg_direction(Grid g, const double* __restrict__ z, double* __restrict__ p, PcgScalars* S) {
    if (S->done) return;
    const double beta = S->beta;
    const int64_t n3 = 3 * g.NN;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

}  // namespace

void launch_pcg_init(const Grid& g, const double* b, const double* Ax, double* r, RedSlot red, PcgScalars* S,
                     double tol, cudaStream_t s) {
    k_pcg_init<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, b, Ax, r, red, S, tol);
}
void launch_pcg_start(const Grid& g, const double* z, double* p, cudaStream_t s) {
    cudaMemcpyAsync(p, z, 3 * g.NN * sizeof(double), cudaMemcpyDeviceToDevice, s);
}
void launch_pcg_update(const Grid& g, double* x, double* r, const double* p, const double* Ap, RedSlot red,
                       PcgScalars* S, cudaStream_t s) {
    k_pcg_update<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, x, r, p, Ap, red, S);
}
void launch_pcg_direction(const Grid& g, const double* z, double* p, PcgScalars* S, cudaStream_t s) {
    k_pcg_direction<<<RED_BLOCKS, RED_THREADS, 0, s>>>(g, z, p, S);
}

}  // namespace t3d
