// Host-side launchers of the B200 kernels.  All launches go to the given stream; none allocates.
#pragma once
#include <cuda.h>

#include <string>

#include "t3d_common.cuh"

namespace t3d {

struct Cuboid {          // solid region of the padded grid (fea.cpp:204-215)
    int nelx, nely, nelz;
};

// Passive-void ellipsoids removed from the cuboid (absent voxels, like the padding of fea.cpp:204-215):
// element (ex, ey, ez) in the reference's element coordinates is void when its centre lies inside.
constexpr int MAX_VOIDS = 4;
struct VoidSet {
    int n;
    double c[MAX_VOIDS][3];   // centres (element units)
    double r[MAX_VOIDS][3];   // radii (element units, > 0)
};
__host__ __device__ inline bool in_void(const VoidSet& v, int ex, int ey, int ez) {
    for (int k = 0; k < v.n; ++k) {
        const double dx = (ex + 0.5 - v.c[k][0]) / v.r[k][0];
        const double dy = (ey + 0.5 - v.c[k][1]) / v.r[k][1];
        const double dz = (ez + 0.5 - v.c[k][2]) / v.r[k][2];
        if (dx * dx + dy * dy + dz * dz <= 1.0) return true;
    }
    return false;
}

int set_cuda_error(cudaError_t e, const char* what, const char* file, int line);
int set_error(int code, const std::string& msg);

struct MgLevel {         // one structured multigrid level (hierarchy.cpp:45-81)
    int nx, ny, nz, span;
    int64_t nn;          // nodes
    double* r;           // 3 SoA planes (level 0: not used, the PCG vectors are passed directly)
    double* x;
    double* diag;        // 3 SoA planes
    uint8_t* mask;       // per node, bit c = fixed
};

struct MgLevel32 {       // FP32 copy of a level's vectors for the mixed-precision inner solve
    int nx, ny, nz, span;
    int64_t nn;           // nodes (the mask's length)
    int pitch;            // row pitch of the vectors: the grid's px on the finest level, nx + 1 on the others
    int64_t cs;           // component stride of the vectors: pitch * (ny + 1) * (nz + 1)
    float* r;
    float* x;
    float* diag;          // reciprocal diagonal 1 / max(1e-30, D) in FP32
    const uint8_t* mask;  // shared with the FP64 level (unpadded, nn bytes)
};

// ---- model set-up (fea.cpp:181-447)
void launch_setup_cells(const Grid& g, Cuboid c, const VoidSet& v, uint8_t* solid, cudaStream_t s);
// fix_x0: the reference's x = 0 face fixation (0 for external models with listed fixations)
void launch_setup_mask0(const Grid& g, const uint8_t* solid, int fix_x0, uint8_t* mask, cudaStream_t s);
// listed fixations / loads on distinct grid nodes (external models); loads are dropped on fixed DOFs
// acc = w ce (first) or acc + w ce over n cells: the weighted compliance of several load cases
void launch_cells_axpy(int64_t n, int first, double w, const double* ce, double* acc, cudaStream_t s);
void launch_setup_fix_list(int n, const int32_t* node, const uint8_t* bits, uint8_t* mask, cudaStream_t s);
void launch_setup_load_list(const Grid& g, int n, const int32_t* node, const double* f, const uint8_t* mask, double* b,
                            cudaStream_t s);
void launch_setup_load(const Grid& g, int ix_load, int iz_max, double fz, const uint8_t* mask, double* b,
                       cudaStream_t s);
// force f (component comp) on every free DOF of the node box [x0,x1]x[y0,y1]x[z0,z1] (grid coordinates)
void launch_setup_box_load(const Grid& g, int x0, int x1, int y0, int y1, int z0, int z1, int comp, double f,
                           const uint8_t* mask, double* b, cudaStream_t s);

// ---- FEA operators
// Ke: device pointer to the 576 stiffness coefficients
void launch_matvec64(const Grid& g, const double* Ke, const double* E, const uint8_t* mask, const double* u,
                     double* y, RedSlot dot, PcgScalars* S, cudaStream_t s);
// Element-streaming form of the same product (bit-identical; no fused dot).  The tiling is fixed per
// grid and device: stream64_tiling also sets the kernel's shared-memory attribute on the current device.
struct Stream64Tiling {   // persistent walk over (x tile, y tile, z slab) work items
    int tiles_x, tiles_y, slabs, slab, items, grid;
};
struct Ke64 {             // Ke by value (576 doubles, row-major): a kernel parameter, read from the constant bank
    double v[576];
};
constexpr int KE_MAX_DISTINCT = 32;   // room for the distinct-magnitude list of the built-in Ke
// true when Ke has the coefficient pattern of the built-in hex8 Ke; D[0..KE_MAX_DISTINCT) receives its
// distinct magnitudes (the streaming kernel's register-operand form)
bool ke_pattern_magnitudes(const double* Ke, double* D);
int stream64_tiling(const Grid& g, int dev, Stream64Tiling* t);
// Kd: device copy of the magnitudes when Ke has the built-in pattern, else nullptr; then Ke_host (the
// context's host copy of Ke) is copied into the launch (and into a graph that captures it)
void launch_matvec64_stream(const Grid& g, const Stream64Tiling& t, const double* Ke_host, const double* Kd,
                            const double* E, const uint8_t* mask, const double* u, double* y, const PcgScalars* S,
                            cudaStream_t s);
// S->denom = p.Ap (3 components) in the canonical reduction order, unless S->done
void launch_dot_pcg(const Grid& g, const double* p, const double* Ap, RedSlot red, PcgScalars* S, cudaStream_t s);
void launch_compliance64(const Grid& g, const double* Ke, const double* E, const double* u, double* ce,
                         RedSlot red, double* C, cudaStream_t s);
void launch_simp(const Grid& g, const uint8_t* solid, const float* x, float E0, float Emin, float penal, double* E,
                 cudaStream_t s);
void launch_sens(const Grid& g, const uint8_t* solid, const float* x, const double* ce, const double* Csolid,
                 float E0, float Emin, float penal, float* dc, float* xdc, cudaStream_t s);
void launch_objective(const Grid& g, const double* E, const double* ce, const double* Csolid, RedSlot red,
                      double* obj, cudaStream_t s);

// ---- multigrid (hierarchy.cpp, masks.cpp, diagonal.cpp, transfers.cpp, coarsest.cpp, preconditioner.cpp)
void launch_diag0(const Grid& g, const double* Ke, const double* E, const uint8_t* mask, double* diag,
                  cudaStream_t s);
void launch_mask_restrict(const MgLevel& Lc, const MgLevel& Lf, cudaStream_t s);
void launch_diag_coarsen(const MgLevel& Lc, const MgLevel& Lf, cudaStream_t s);
// separable restriction; a1, a2: pass buffers of 3*(fnz*fny*cnx) and 3*(fnz*cny*cnx) doubles
// normalize = false: the transpose of the trilinear prolongation (no division by the weight sum)
void launch_restrict(const MgLevel& Lc, const MgLevel& Lf, const double* rf, double* rc, double* a1, double* a2,
                     const PcgScalars* S, cudaStream_t s, bool normalize = true);
void launch_coarse_jacobi(const MgLevel& L, const PcgScalars* S, cudaStream_t s);
void launch_prolong_smooth(const MgLevel& Lc, const MgLevel& Lf, const double* xc, const double* rf, double* xf,
                           double weight, const PcgScalars* S, cudaStream_t s);
void launch_prolong_smooth0(const MgLevel& Lc, const MgLevel& Lf, const double* xc, const double* r, double* z,
                            double weight, RedSlot dot, PcgScalars* S, cudaStream_t s);
// coarsest dense Galerkin matrix, Cholesky factor and triangular solves (coarsest.cpp, preconditioner.cpp:47-78)
// span: fine elements per coarse element edge that are sampled (the coarsest level's own span in the
// reference's assembly; the product of all spans for the full Galerkin operator)
void launch_coarse_element_matrices(const Grid& g0, const MgLevel& Lc, int span, const uint8_t* mask0, const double* E,
                                    const double* Ke, double emin, double* Kce, cudaStream_t s);
void launch_coarse_assemble(const MgLevel& Lc, const double* Kce, double* Kc, cudaStream_t s);
// returns the number of kernels it launched
int launch_cholesky(const double* A, double* LT, double* Lrow, int N, int* status, cudaStream_t s);
// canonical coarsest solve: inverse columns from the factor, then x = X r (Jacobi fallback when
// *status != 1, preconditioner.cpp:76-77, 195-215)
void launch_coarse_inverse(const double* LT, const double* Lrow, int N, const int* status, double* X,
                           cudaStream_t s);
void launch_coarse_solve(const MgLevel& L, const double* X, int N, const int* status, const PcgScalars* S,
                         cudaStream_t s);

// ---- 'Standard' V-cycle option (TOP3D_XL.m:772-807): Galerkin element matrices per level, smoothing with
// the true residual; FP64.  The assembly stores element matrices element-major (576 entries per element,
// row-major 24x24, local DOF 3a+c); the level products read an entry-major copy, entry k of element e of a
// level with ne elements at kel_index(e, k, ne) = k * ne + e.
__host__ __device__ inline int64_t kel_index(int64_t e, int k, int64_t ne) { return (int64_t)k * ne + e; }
void launch_kel_transpose(int64_t ne, const double* Kel, double* KelT, cudaStream_t s);
void launch_kel_transpose32(int64_t ne, const double* Kel, float* KelT32, cudaStream_t s);
// G[pos][576] = W_pos^T Ke W_pos for the s^3 child positions of a span-s coarse element (host)
void galerkin_positions(int s, const double* Ke, double* G);
void launch_galerkin_fine(const Grid& g, const MgLevel& L1, const double* E, const uint8_t* mask0, const double* Gpos,
                          const double* Ke, double* Kel, cudaStream_t s);
void launch_galerkin_coarse(const MgLevel& Lf, const MgLevel& Lc, const double* Kf, double* Kc, cudaStream_t s);
void launch_level_diag(const MgLevel& L, const double* Kel, cudaStream_t s);
// KelT: the level's entry-major element matrices
void launch_level_matvec(const MgLevel& L, const double* KelT, const double* x, double* y, const PcgScalars* S,
                         cudaStream_t s);
void launch_jacobi_init(const MgLevel& L, const double* r, double* x, double w, const PcgScalars* S, cudaStream_t s);
void launch_residual(const MgLevel& L, const double* r, double* kx, const PcgScalars* S, cudaStream_t s);
void launch_jacobi_correct(const MgLevel& L, const double* r, const double* kx, double* x, double w,
                           const PcgScalars* S, cudaStream_t s);
void launch_prolong_add(const MgLevel& Lc, const MgLevel& Lf, const double* xc, double* xf, const PcgScalars* S,
                        cudaStream_t s);
void launch_dot_rz(int64_t NN, const double* r, const double* z, RedSlot red, PcgScalars* S, cudaStream_t s);
void launch_to_coarse_layout(const MgLevel& L, const double* Kel, double* Kce, cudaStream_t s);

// ---- PCG vector steps (solver.cpp:87-217)
void launch_pcg_init(const Grid& g, const double* b, const double* Ax, double* r, RedSlot red, PcgScalars* S,
                     double tol, cudaStream_t s);
void launch_pcg_start(const Grid& g, const double* z, double* p, cudaStream_t s);
void launch_pcg_update(const Grid& g, double* x, double* r, const double* p, const double* Ap, RedSlot red,
                       PcgScalars* S, cudaStream_t s);
void launch_pcg_direction(const Grid& g, const double* z, double* p, PcgScalars* S, cudaStream_t s);

// ---- PDE filter (filter.cpp)
struct FilterScalars {
    double nr2, df2;          // |rhs|^2, |rhs - lastRhs|^2
    double rz, den, beta;
    int warm, done, it, pad;
};
// kf: 64 kernel entries followed by the 8 row sums (filter.cpp:53-70)
void launch_filter_diag(const Grid& g, const uint8_t* solid, const double* kf, double* fdiag, cudaStream_t s);
void launch_filter_rhs(const Grid& g, const uint8_t* solid, const float* src, double* rhs, cudaStream_t s);
void launch_filter_norms(const Grid& g, const double* rhs, const double* lastrhs, RedSlot r1, RedSlot r2,
                         FilterScalars* F, cudaStream_t s);
void launch_filter_x0(const Grid& g, const double* lastx, double* x, const FilterScalars* F, cudaStream_t s);
void launch_filter_matvec(const Grid& g, const uint8_t* solid, const double* kf, const double* x, double* y,
                          RedSlot dot, FilterScalars* F, cudaStream_t s);
void launch_filter_r0(const Grid& g, const double* rhs, const double* Ax, const double* fdiag, double* r, double* z,
                      double* p, RedSlot r1, RedSlot r2, FilterScalars* F, cudaStream_t s);
void launch_filter_update(const Grid& g, double* x, double* r, const double* p, const double* Ap, RedSlot red,
                          FilterScalars* F, cudaStream_t s);
void launch_filter_precond(const Grid& g, const double* r, const double* fdiag, double* z, RedSlot red,
                           FilterScalars* F, cudaStream_t s);
void launch_filter_direction(const Grid& g, const double* z, double* p, const FilterScalars* F, cudaStream_t s);
void launch_filter_to_cells(const Grid& g, const uint8_t* solid, const double* x, float* dst, cudaStream_t s);

// ---- generic canonical reductions over node arrays (ncomp SoA planes of NN values)
void launch_dot(const Grid& g, int ncomp, const double* a, const double* b, RedSlot red, double* out, cudaStream_t s);
void launch_diffnorm(const Grid& g, const double* a, const double* b, RedSlot red, double* out_a2, double* out_d2,
                     cudaStream_t s);

// ---- layout conversion between the reference's layouts and the device grid
void launch_scatter_free(int64_t nf, const int32_t* free_dofs, const double* vfree, int64_t NN, double* grid,
                         cudaStream_t s);
void launch_gather_free(int64_t nf, const int32_t* free_dofs, const double* grid, int64_t NN, double* vfree,
                        cudaStream_t s);
void launch_cells_from_morton_f64(int64_t ne, const int32_t* cell_of, const double* v, double* cells, cudaStream_t s);
void launch_cells_to_morton_f64(int64_t ne, const int32_t* cell_of, const double* cells, double* v, cudaStream_t s);
void launch_cells_from_morton_f32(int64_t ne, const int32_t* cell_of, const float* v, float* cells, cudaStream_t s);
void launch_cells_to_morton_f32(int64_t ne, const int32_t* cell_of, const float* cells, float* v, cudaStream_t s);

// ---- OC (driver.cpp:160-189)
struct OcState {
    float l1, l2, lmid, vol;
    float change, sharp, volfrac, pad;
    int passes, done, pad1, pad2;
};
void launch_dc_scale(const Grid& g, const uint8_t* solid, const float* dcf, const float* x, float* dc,
                     cudaStream_t s);
void launch_oc_init(OcState* st, cudaStream_t s);
// one bisection pass: xnew for lmid; fp64_sum: canonical FP64 volume sum + l1/l2 update in the same kernel
void launch_oc_pass(const Grid& g, const uint8_t* solid, const float* x, const float* dc, float* xnew, OcState* st,
                    int fp64_sum, float V0, int64_t ne, RedSlot red, cudaStream_t s);
// reference-order volume sum (8-lane vectorised std::accumulate over Morton order) + l1/l2 update
void launch_oc_vec8_vol(int64_t ne, const int32_t* morton_cells, const float* xnew, OcState* st, float V0,
                        cudaStream_t s);
// change = max|xnew-x|, x = xnew; fp64_sum: sharpness and volume fraction by canonical FP64 sums
void launch_oc_finish(const Grid& g, const uint8_t* solid, float* x, const float* xnew, OcState* st, int fp64_sum,
                      int64_t ne, RedSlot r1, RedSlot r2, cudaStream_t s);
// reference-order sharpness and volume fraction
void launch_oc_vec8_stats(int64_t ne, const int32_t* morton_cells, const float* x, OcState* st, cudaStream_t s);

// ---- mixed precision (k_mixed.cu)
// FP64 node vector (3 planes, rows of nnx) -> FP32 image (rows of px, pads zero), and back
void launch_nodes_to32(const Grid& g, const double* a, float* b, cudaStream_t s);
void launch_nodes_from32(const Grid& g, const float* a, double* b, cudaStream_t s);
// FP64 moduli (cells, rows of ex) -> FP32 image (rows of pex, pads zero)
void launch_cells_to32(const Grid& g, const double* a, float* b, cudaStream_t s);
// reciprocal FP32 diagonal 1 / max(1e-30, D) of a level: rows of `len` values (3 planes) -> rows of `pitch`
void launch_recip_diag32(int64_t rows, int len, int pitch, const double* d, float* rd, cudaStream_t s);
void launch_mixed_residual(const Grid& g, const double* b, const double* Au, float* r32, float* d32, RedSlot red,
                           double* rn2, cudaStream_t s);
void launch_mixed_accumulate(const Grid& g, double* u, const float* d, cudaStream_t s);
// mark = 1 for the PCG's own K(E)p (records S->xit), 0 for the operator inside the Standard V-cycle
void launch_matvec32(const Grid& g, const float* Ke, const float* E, const uint8_t* mask, const float* u, float* y,
                     RedSlot dot, PcgScalars* S, int mark, cudaStream_t s);
// rc = normalised restriction of rf (normalize = false: the transposed prolongation); a1 holds the x-pass
// result on span-4 transitions
void launch_restrict32(const MgLevel32& Lc, const MgLevel32& Lf, const float* rf, float* rc, float* a1,
                       const PcgScalars* S, cudaStream_t s, bool normalize = true);
// FP32 image of `rows` rows of `len` doubles (same layout)
void launch_rows_to32(int64_t rows, int len, const double* a, float* b, cudaStream_t s);
// ---- the Standard V-cycle in FP32 (k_mg_standard32.cu)
void launch_jacobi_init32(const MgLevel32& L, const float* r, float* x, float w, const PcgScalars* S, cudaStream_t s);
void launch_residual32(const MgLevel32& L, const float* r, float* kx, const PcgScalars* S, cudaStream_t s);
void launch_jacobi_correct32(const MgLevel32& L, const float* r, const float* kx, float* x, float w,
                             const PcgScalars* S, cudaStream_t s);
// xo = xi + P xc (fixed DOFs 0); xo may be xi
void launch_prolong_add32(const MgLevel32& Lc, const MgLevel32& Lf, const float* xc, const float* xi, float* xo,
                          const PcgScalars* S, cudaStream_t s);
// KelP32: the level's element matrices as FP32, symmetric-packed (300 upper-triangle entries), entry-major
void launch_level_matvec32(const MgLevel32& L, const float* KelP32, const float* x, float* y, const PcgScalars* S,
                           cudaStream_t s);
void launch_kel_pack32(int64_t ne, const double* Kel, float* KelP32, cudaStream_t s);
void launch_dot_rz32(int64_t n3, const float* r, const float* z, RedSlot red, PcgScalars* S, cudaStream_t s);
void launch_prolong_smooth32(const MgLevel32& Lc, const MgLevel32& Lf, const float* xc, const float* rf, float* xf,
                             float w, const PcgScalars* S, cudaStream_t s);
void launch_prolong_smooth0_32(const MgLevel32& Lc, const MgLevel32& Lf, const float* xc, const float* r, float* z,
                               float w, RedSlot dot, PcgScalars* S, cudaStream_t s);
void launch_coarse_solve32(const MgLevel32& L, const double* X, int N, const int* status, const PcgScalars* S,
                           cudaStream_t s);
void launch_pcg_update32(const Grid& g, float* x, float* r, const float* p, const float* Ap, RedSlot red,
                         PcgScalars* S, cudaStream_t s);
// p = z + beta p and the deferred x += alpha p of the same iteration (see PcgScalars::xit)
void launch_pcg_direction32(const Grid& g, const float* z, float* p, float* x, PcgScalars* S, cudaStream_t s);

// ---- FP32 K(E)p through the modal form of Ke (k_matvec_modal.cu)
struct ModalKe {         // the 45 nonzeros of T^T Ke T / 64 in the fixed block pattern
    float v[45];
};
struct ModalTiling {     // persistent walk over (x tile, y tile, z slab) work items
    int tiles_x, tiles_y, slabs, slab, items, grid, variant;
};
// Projects Ke (576 doubles, row-major, local DOF 3a+c) onto the modal pattern.  Returns false when Ke
// has entries off the pattern (relative size above 1e-10), i.e. it is not the stiffness of an
// axis-aligned cubic isotropic voxel; *off receives the largest relative off-pattern entry.
bool modal_ke_from(const double* Ke, ModalKe* out, double* off);
// (threads in x, threads in y, ring slots, packed FP32x2) of tile shape `variant`
void modal_variant_desc(int variant, int out[4]);
// Tiling and persistent grid size of tile shape `variant` on device `dev` (grid <= RED_BLOCKS).
int modal_tiling(const Grid& g, int dev, int variant, ModalTiling* t);
// Times every tile shape on the given buffers (3 launches each, stream-ordered, CUDA events) and returns
// the fastest one's tiling.  y is overwritten.
// err: device int set to 1 by a TMA-staged shape whose mbarrier wait gave up (never expected; checked by the host)
int modal_autotune(const Grid& g, int dev, const ModalKe& kh, const float* E, const uint8_t* mask, const float* u,
                   float* y, int* err, cudaStream_t s, ModalTiling* best);
void launch_matvec32_modal(const Grid& g, const ModalKe& kh, const ModalTiling& t, const float* E,
                           const uint8_t* mask, const float* u, float* y, RedSlot dot, PcgScalars* S, int mark,
                           int* err, cudaStream_t s);

// The Standard V-cycle's level-0 operator with its elementwise step fused into the epilogue (TMA tile shapes only;
// false when the tiling's shape has no fused form, then nothing was launched):
//   mode 1: y = r - K(E)u;  mode 2: y = u + w (r - K(E)u) rd (rd = 1/D; y must not alias u), r.y -> S (rz / beta)
bool modal_fused_available(const ModalTiling& t);
bool launch_matvec32_fused(int mode, const Grid& g, const ModalKe& kh, const ModalTiling& t, const float* E,
                           const uint8_t* mask, const float* u, float* y, const float* r, const float* rd, float w,
                           RedSlot dot, PcgScalars* S, int* err, cudaStream_t s);

// ---- batched launches (batch.cu): one persistent launch runs the logical launches of many instances of
// uneven size.  Each takes a device array of the N instances' arguments and `act`, the instances still
// iterating: act[0] = their count n, act[1 .. n] their positions in the argument array, act[1+N .. 1+N+n]
// the prefix sum of their logical block counts (an instance's count is the grid of its own launch, so its
// arithmetic and reduction order are those of that launch).  launch_batch_compact rebuilds `act` from the
// instances' done flags between iterations; instances that finish inside an iteration skip their blocks there
// (S->done), as their own launches would.
struct BatchMatvec {      // K(E)u in the TMA tile shapes (maps in global memory) with the epilogue of `mode`:
    Grid g;               // 0 the PCG product with p.Ap; 1 / 2 the Standard cycle's fused residual / correction
    ModalTiling t;        // (launch_matvec32_fused)
    const uint8_t* mask;
    float* y;
    RedSlot dot;
    PcgScalars* S;
    const CUtensorMap* umap;
    const CUtensorMap* emap;
    const float* rv;      // modes 1, 2: r
    const float* rd;      // mode 2: 1/D
    float omega;          // mode 2: Jacobi weight
};
struct BatchUpdate {      // r -= alpha Ap with |r|^2
    int64_t NNp;
    float* r;
    const float* Ap;
    RedSlot red;
    PcgScalars* S;
};
struct BatchDirection {   // x += alpha p, p = z + beta p
    int64_t NNp;
    const float* z;
    float* p;
    float* x;
    PcgScalars* S;
};
struct BatchRestrict {    // restriction Lf -> Lc: span 4 x pass rf -> a1 then y-z pass a1 -> rc; span 2 rf -> rc
    MgLevel32 Lc, Lf;
    const float* rf;
    float* a1;
    float* rc;
    PcgScalars* S;
    int normalize;        // 1: the Adapted cycle's weighted average; 0: the Standard cycle's P^T
};
struct BatchProlong {     // prolongation + smoothing on a level above the finest
    MgLevel32 Lc, Lf;
    float w;
    PcgScalars* S;
};
struct BatchProlong0 {    // finest-level prolongation + smoothing with r.z
    MgLevel32 Lc, Lf;
    const float* r;
    float* z;
    float w;
    RedSlot dot;
    PcgScalars* S;
};
struct BatchCoarse {      // coarsest-level solve
    MgLevel32 L;
    const double* X;
    int N;
    const int* status;
    PcgScalars* S;
};
// the Standard V-cycle's level steps (FP32): op 0 x = w r / D, op 1 kx <- r - kx, op 2 x += w (r - kx) / D
struct BatchLevelOp {
    MgLevel32 L;
    const float* r;
    float* kx;
    float* x;
    float w;
    PcgScalars* S;
};
struct BatchProlongAdd {  // xo = xi + P xc
    MgLevel32 Lc, Lf;
    const float* xc;
    const float* xi;
    float* xo;
    PcgScalars* S;
};
struct BatchLevelMatvec { // y = K_l x from the level's FP32 element matrices
    MgLevel32 L;
    const float* Kel;
    const float* x;
    float* y;
    PcgScalars* S;
};
int batch_blocks_level_op(const BatchLevelOp& a);
int batch_blocks_prolong_add(const BatchProlongAdd& a);
int batch_blocks_level_matvec(const BatchLevelMatvec& a);
void launch_batch_level_op32(const BatchLevelOp* a, const int* act, int N, int op, cudaStream_t s);
void launch_batch_prolong_add32(const BatchProlongAdd* a, const int* act, int N, cudaStream_t s);
void launch_batch_level_matvec32(const BatchLevelMatvec* a, const int* act, int N, cudaStream_t s);

struct BatchCompact {     // one launch list's compaction: act from the done flags of its N instances
    PcgScalars* const* S;   // per position
    const int* blocks;      // per position
    int N;
    int* act;
};
// logical block counts of one instance's own launches
int batch_blocks_update();
int batch_blocks_restrict(const BatchRestrict& a, int stage);   // stage 0: x or x-y-z pass, 1: y-z pass (0 if none)
int batch_blocks_prolong(const BatchProlong& a);
int batch_blocks_prolong0();
int batch_blocks_coarse(const BatchCoarse& a);
// the launches (a, act on the device; N instances in the list)
void launch_batch_flags(PcgScalars* const* S, int n, int* out, cudaStream_t s);   // out[i] = S[i]->done
void launch_batch_compact(const BatchCompact* jobs, int njobs, cudaStream_t s);
void launch_batch_update32(const BatchUpdate* a, const int* act, int N, cudaStream_t s);
void launch_batch_direction32(const BatchDirection* a, const int* act, int N, cudaStream_t s);
void launch_batch_restrict32(const BatchRestrict* a, const int* act, int N, int stage, cudaStream_t s);
void launch_batch_prolong32(const BatchProlong* a, const int* act, int N, cudaStream_t s);
void launch_batch_prolong0_32(const BatchProlong0* a, const int* act, int N, cudaStream_t s);
void launch_batch_coarse32(const BatchCoarse* a, const int* act, int N, int max_n, cudaStream_t s);
// the batched PCG product: variant = the members' common TMA tile shape; false when it has no batched form
bool modal_batched_available(int variant);
int modal_batched_grid(int variant, int dev, int* grid);
bool launch_batch_matvec32(int variant, int mode, const BatchMatvec* a, const int* act, int N, const ModalKe& kh,
                           int grid, int* err, cudaStream_t s);
// the tensor maps of one instance's PCG product (p and E images); false when they cannot be encoded
bool modal_tensor_maps_for(int variant, const Grid& g, const float* u, const float* E, CUtensorMap* umap,
                           CUtensorMap* emap);

// ---- surface export (k_stl.cu, io.cpp:80-87)
int stl_chunks(const Grid& g);
// per-chunk face counts scanned in place: bsum[i] = faces before chunk i, bsum[chunks] = total faces
// (bsum holds stl_chunks(g) + 1 entries)
void launch_stl_count(const Grid& g, const float* density_cells, float iso, unsigned* bsum, cudaStream_t s);
// the STL records (50 bytes per triangle, 2 triangles per face) at their final offsets
void launch_stl_write(const Grid& g, const float* density_cells, float iso, const unsigned* boff, uint16_t* body,
                      cudaStream_t s);

}  // namespace t3d
