// Shared device/host definitions of the B200 topology-optimisation library.
//
// Data layout in HBM (all arrays device-resident for the life of a context):
//   node vectors   3 SoA planes of (nnx*nny*nnz) values, node n = (iz*nny + iy)*nnx + ix
//                  (lexicographic, the reference's node numbering fea.cpp:253-255);
//                  component c of node n at [c*NN + n].  Fixed DOFs hold exact zeros.
//   cell arrays    (nx+2)*(ny+2)*(nz+2) values with a zero ghost ring; cell (cx,cy,cz) at
//                  ((cz+1)*(ny+2) + cy+1)*(nx+2) + cx+1.  Cell (cx,cy,cz) is the reference element
//                  (ex,ey,ez) = (cx, ny-1-cy, cz) (fea.cpp:222).  Non-solid cells hold E = 0.
//   node masks     one byte per node, bit c = DOF c fixed.
//   FP32 images    the mixed-precision inner solve keeps its finest-level node vectors and moduli with
//                  rows padded to a multiple of 4 values (pitch px for nodes, pex for cells; the pads
//                  hold zeros), so that every row starts on a 16-byte boundary: TMA tensor maps need
//                  16-byte row strides, and 257 nodes per row (1028 bytes) is not one.
//
// Every floating-point kernel is compiled with -fmad=false; fused multiply-adds are written out
// with fma() where the algorithm uses them, so the CPU oracle can mirror each operation.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace t3d {

// Canonical deterministic reduction geometry: grid-stride loops over nodes with exactly
// RED_BLOCKS x RED_THREADS threads; per-thread sequential partials (components 0,1,2 of each node
// in turn), xor-butterfly inside each warp, the 8 warp sums folded the same way by warp 0, and the
// RED_BLOCKS block partials folded by the last block to finish (threads stride over the partials,
// then the same two-level butterfly).  The result depends only on the vector length.
constexpr int RED_BLOCKS = 1184;   // 8 x 148 SMs
constexpr int RED_THREADS = 256;

// Reference local corner order (fea.cpp:257-264): corner a of the element in cell (cx,cy,cz) sits at
// node (cx+CX[a], cy+CY[a], cz+CZ[a]).
__host__ __device__ constexpr int corner_dx(int a) { return (a == 1 || a == 2 || a == 5 || a == 6) ? 1 : 0; }
__host__ __device__ constexpr int corner_dy(int a) { return (a == 0 || a == 1 || a == 4 || a == 5) ? 1 : 0; }
__host__ __device__ constexpr int corner_dz(int a) { return a >= 4 ? 1 : 0; }
// inverse: node offset (dx,dy,dz) inside the cell -> corner a
__host__ __device__ constexpr int corner_of(int dx, int dy, int dz) {
    return dz * 4 + (dy ? (dx ? 1 : 0) : (dx ? 2 : 3));
}

struct Grid {
    int nx, ny, nz;      // elements (padded)
    int nnx, nny, nnz;   // nodes
    int64_t NN;          // nodes per plane
    int ex, ey, ez;      // cell-array dims with ghost ring (nx+2, ...)
    int64_t NE;          // cell-array length
    int px;              // FP32 node row pitch: nnx rounded up to a multiple of 4
    int64_t NNp;         // px * nny * nnz: one component plane of an FP32 node vector
    int pex;             // FP32 cell row pitch: ex rounded up to a multiple of 4
    int64_t NEp;         // pex * ey * ez

    __host__ __device__ int64_t node(int ix, int iy, int iz) const {
        return ((int64_t)iz * nny + iy) * nnx + ix;
    }
    __host__ __device__ int64_t cell(int cx, int cy, int cz) const {
        return ((int64_t)(cz + 1) * ey + (cy + 1)) * ex + (cx + 1);
    }
    __host__ __device__ int64_t pnode(int ix, int iy, int iz) const {   // FP32 node vectors
        return ((int64_t)iz * nny + iy) * px + ix;
    }
    __host__ __device__ int64_t pcell(int cx, int cy, int cz) const {   // FP32 moduli
        return ((int64_t)(cz + 1) * ey + (cy + 1)) * pex + (cx + 1);
    }
};

inline Grid make_grid(int nx, int ny, int nz) {
    Grid g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.nnx = nx + 1; g.nny = ny + 1; g.nnz = nz + 1;
    g.NN = (int64_t)g.nnx * g.nny * g.nnz;
    g.ex = nx + 2; g.ey = ny + 2; g.ez = nz + 2;
    g.NE = (int64_t)g.ex * g.ey * g.ez;
    g.px = (g.nnx + 3) / 4 * 4;
    g.NNp = (int64_t)g.px * g.nny * g.nnz;
    g.pex = (g.ex + 3) / 4 * 4;
    g.NEp = (int64_t)g.pex * g.ey * g.ez;
    return g;
}

// Scalars of one PCG solve, resident on the device so that iterations need no host round trip.
struct PcgScalars {
    double rz;        // r.z of the current search direction
    double denom;     // p.Ap
    double rnorm2;    // r.r after the update
    double stop;      // max(1e-30,|b|)*tol
    double bnorm2;    // b.b
    double beta;
    double tol;
    int it;           // iterations completed
    int done;         // 1 once |r| < stop
    int result;       // PCG_free return value (solver.cpp:184,216)
    int first;        // 1 while the initial r.z is being formed
    // FP32 inner solve only: the direction kernel applies x += alpha p_old; xit = the iteration whose
    // alpha is already in x (set by the next K(E)p launch), so a converged step is applied exactly once
    int xit;
    float alpha;      // alpha of iteration `it`, stored by the update kernel
    int maxit;        // FP32 inner solve: done once `it` reaches it (0: no cap); the FP64 path ignores it
};

// Reduction scratch: RED_BLOCKS partials + arrival counter per reduction slot.
struct RedSlot {
    double* partial;
    unsigned int* counter;
};

}  // namespace t3d

#define T3D_CUDA_OK(call)                                                       \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) return t3d::set_cuda_error(e_, #call, __FILE__, __LINE__); \
    } while (0)
