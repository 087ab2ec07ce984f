// Allocation-free compliance entry point.
//
// Some callers cannot allocate device memory when they call into this library: code that runs
// inside a host framework which owns the whole device heap (a plugin whose host pre-reserves
// memory pools and forbids cudaMalloc behind its back), real-time or serving loops that must not
// hit the allocator (cudaMalloc can synchronise the device and stall every stream), or callers that
// hold their own buffers and want no hidden context at all.  For them t3d_compliance_noalloc takes
// every input and output as a device pointer and keeps its only scratch -- the per-block partial
// sums of the compliance reduction and their arrival counter -- in the file-scope array below.
//
// That array belongs to the library image: every GPU that loads the library holds it
// (NOALLOC_MAX_BLOCKS+1 doubles, 512 KiB) until the process exits.  Its size bounds the grid:
// one partial per 256 cells, so at most NOALLOC_MAX_BLOCKS*256 padded cells per call.
// All calls share the array, so calls that overlap on the GPU (two streams, or two host threads on
// the same device) race on it; callers must serialise them.
#include "t3d_b200.h"
#include "kernels.hpp"
#include "red.cuh"

#include <atomic>
#include <cstdint>
#include <string>

namespace t3d {

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_MAX_BLOCKS = 65536;
constexpr int NOALLOC_MAX_DEVICES = 64;

// partials[0 .. NOALLOC_MAX_BLOCKS-1], then the arrival counter (as the first 4 bytes of the last slot)
static __device__ __align__(256) double g_scratch[NOALLOC_MAX_BLOCKS + 1];

// device address of g_scratch per device ordinal, filled by the first call on each device.  Atomic slots:
// host threads may make their first calls concurrently (each stores the same address).  The address is the
// one in the device's primary context, the context the CUDA runtime makes current.
std::atomic<double*> g_scratch_addr[NOALLOC_MAX_DEVICES];

struct KeArg {
    double k[576];
};

// ce_e = ue' Ke ue for solid cells (0 when E <= 1e-16) with the arithmetic of k_compliance64, one
// thread per cell in canonical cell order; C = sum E*ce folded per block, then by the last block.
__global__ void __launch_bounds__(NOALLOC_THREADS) k_compliance_noalloc(Grid g, const __grid_constant__ KeArg K,
                                                                        const double* __restrict__ E,
                                                                        const double* __restrict__ u,
                                                                        double* __restrict__ ce, double* scratch,
                                                                        double* __restrict__ C) {
    __shared__ double Ke[576];
    __shared__ double sh[32];
    for (int i = threadIdx.x; i < 576; i += blockDim.x) Ke[i] = K.k[i];
    __syncthreads();
    const int NN = (int)g.NN;
    const int ncell = g.nx * g.ny * g.nz;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double part = 0.0;
    if (k < ncell) {
        const int cx = k % g.nx, cy = (k / g.nx) % g.ny, cz = k / (g.nx * g.ny);
        const int64_t ci = g.cell(cx, cy, cz);
        const double Ee = E[ci];
        if (Ee <= 1.0e-16) {
            ce[ci] = 0.0;
        } else {
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
            part = Ee * s;
        }
    }
    RedSlot slot{scratch, reinterpret_cast<unsigned int*>(scratch + NOALLOC_MAX_BLOCKS)};
    double tot;
    if (grid_fold(part, slot, sh, &tot) && threadIdx.x == 0) *C = tot;
}

// once per device, with that device current: the device address of the scratch array
int scratch_for_current_device(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDevice", __FILE__, __LINE__);
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return set_error(T3D_ERR_UNSUPPORTED, "device ordinal too large");
    double* addr = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!addr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return set_cuda_error(e, "cudaGetSymbolAddress(g_scratch)", __FILE__, __LINE__);
        addr = static_cast<double*>(p);
        g_scratch_addr[dev].store(addr, std::memory_order_release);
    }
    *out = addr;
    return T3D_OK;
}

}  // namespace

}  // namespace t3d

extern "C" int t3d_compliance_noalloc(int nely, int nelx, int nelz, const double* ke576, const double* d_E,
                                      const double* d_u, double* d_ce, double* d_C, void* stream) {
    using namespace t3d;
    if (nely <= 0 || nelx <= 0 || nelz <= 0) return set_error(T3D_ERR_INVALID, "element counts must be positive");
    if (!ke576 || !d_E || !d_u || !d_ce || !d_C) return set_error(T3D_ERR_INVALID, "null argument");
    // padded grid of the reference (padding.hpp:23-53), as in t3d_create
    uint64_t nvox = (uint64_t)nelx * nely * nelz;
    int L = 0;
    while (nvox >= 50000u) { ++L; nvox = (nvox + 4u) / 8u; }
    if (L < 3) L = 3;
    const int step = 1 << L;
    const int nx = (nelx + step - 1) / step * step, ny = (nely + step - 1) / step * step,
              nz = (nelz + step - 1) / step * step;
    const int64_t ncell = (int64_t)nx * ny * nz;
    const int64_t blocks = (ncell + NOALLOC_THREADS - 1) / NOALLOC_THREADS;
    if (blocks > NOALLOC_MAX_BLOCKS)
        return set_error(T3D_ERR_UNSUPPORTED,
                         "grid too large for the allocation-free path: " + std::to_string(ncell) +
                             " padded cells, at most " + std::to_string((int64_t)NOALLOC_MAX_BLOCKS * NOALLOC_THREADS));
    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != T3D_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the arrival counter must start at zero (the last block also resets it)
    cudaError_t e = cudaMemsetAsync(scratch + NOALLOC_MAX_BLOCKS, 0, sizeof(double), s);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaMemsetAsync(counter)", __FILE__, __LINE__);
    KeArg K;
    for (int i = 0; i < 576; ++i) K.k[i] = ke576[i];
    const Grid g = make_grid(nx, ny, nz);
    k_compliance_noalloc<<<(unsigned)blocks, NOALLOC_THREADS, 0, s>>>(g, K, d_E, d_u, d_ce, scratch, d_C);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error(e, "k_compliance_noalloc launch", __FILE__, __LINE__);
    return T3D_OK;
}
