// Internal host runtime shared by context.cu (one design per context) and batch.cu (many designs per
// launch): the context of one design and the pieces of its design iteration that the batched path reuses.
#pragma once
#include "t3d_b200.h"
#include "kernels.hpp"
#include "topvoxel.hpp"

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

namespace t3d {

#define CHECK(call)                       \
    do {                                  \
        int rc_ = (call);                 \
        if (rc_ != T3D_OK) return rc_;    \
    } while (0)

// One device allocation carved into the buffers of several contexts (bump allocation, 256-byte aligned).
struct Arena {
    char* base = nullptr;
    size_t size = 0, used = 0;
};

// ------------------------------------------------------------------ context
struct Context {
    t3d_params prm{};
    Grid g{};
    Cuboid cub{};
    VoidSet voids{};            // passive-void ellipsoids (absent voxels)
    int load_case = T3D_LOAD_TIP_LINE;
    int dev = 0;
    cudaStream_t st = nullptr;
    int nlev = 0;
    MgLevel lv[8]{};
    int Nc = 0;                 // dense coarsest size (0: Jacobi coarsest)
    int64_t ne = 0;             // solid elements
    size_t bytes = 0;
    std::vector<void*> allocs;

    double* Ke = nullptr;       // 576
    double* kf = nullptr;       // 72
    double Ke_h[576];
    uint8_t* solid = nullptr;   // cells
    uint8_t* mask0 = nullptr;   // nodes
    double *E = nullptr, *ce = nullptr;                       // cells
    float *x = nullptr, *xnew = nullptr, *dc = nullptr, *xdc = nullptr, *dcf = nullptr;   // cells
    double *b = nullptr, *u = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr;  // 3 NN
    PcgScalars* S = nullptr;
    FilterScalars* FS = nullptr;
    OcState* OC = nullptr;
    double* scal = nullptr;     // [0] C, [1] Csolid, [2] objective
    bool mv64_stream = false;   // FP64 K(E)u by the element-streaming kernel (else node-centric)
    Stream64Tiling st64{};
    std::shared_ptr<const VoxelModel> vox;   // external (TopVoxel) model, else the built-in cuboid
    // several load cases (external models): per-case loads and warm starts, weighted element compliance
    int ncases = 1;
    double *b_cases = nullptr, *u_cases = nullptr, *ce_acc = nullptr, *one = nullptr;
    // 'Standard' V-cycle option: Galerkin element matrices per level (l >= 1), child-position products of
    // Ke for level 1, and one scratch vector per level
    bool standard = false;
    double* E_mg = nullptr;     // the moduli the hierarchy was built from (the cycle's level-0 operator)
    double* Kel[8]{};           // element-major (assembly)
    double* KelT[8]{};          // entry-major copies read by the level products
    double* Gpos = nullptr;
    double* vtmp[8]{};
    bool ke_pat = false;        // Ke has the built-in coefficient pattern: its magnitudes are in Kd
    double* Kd = nullptr;       // [KE_MAX_DISTINCT]
    RedSlot slot[4]{};
    double *Kce = nullptr, *Kc = nullptr, *LT = nullptr, *Lrow = nullptr, *Xc = nullptr;
    double* ra1[8]{};           // separable-restriction pass buffers per level transition
    double* ra2[8]{};
    int* chol_status = nullptr;
    double *frhs = nullptr, *fx = nullptr, *fr = nullptr, *fz = nullptr, *fp = nullptr, *fAp = nullptr,
           *flastx = nullptr, *flastrhs = nullptr, *fdiag = nullptr;
    // mixed precision (T3D_MIXED): FP32 inner-solve state
    bool mixed = false;
    float* Ke32 = nullptr;
    ModalKe kh{};               // modal form of Ke for the FP32 K(E)p (valid when `modal`)
    ModalTiling mt{};
    bool modal = false;
    double modal_off = 0.0;     // largest relative off-pattern entry of T^T Ke T
    float* E32 = nullptr;
    float *r32 = nullptr, *d32 = nullptr, *z32 = nullptr, *p32 = nullptr, *Ap32 = nullptr;
    MgLevel32 lv32[8]{};
    float* ra1_32[8]{};         // x-pass buffer of the FP32 restriction (its y and z passes are fused)
    // the Standard V-cycle in FP32: element-matrix images and scratch per coarse level, level-0 moduli image
    float* Kel32[8]{};
    float* vtmp32[8]{};
    float* E_mg32 = nullptr;
    PcgScalars* S32 = nullptr;
    int* tma_err = nullptr;     // set by a TMA-staged K(E)p whose mbarrier wait gave up (checked after solves)
    cudaGraphExec_t pcg32_graph = nullptr;
    int64_t pcg32_graph_launches = 0;
    int last_outer = 0;
    // lazily built maps between the reference's layouts and the grid
    int32_t* morton = nullptr;          // [ne] cell index of the k-th element in Morton order
    std::vector<int32_t> morton_h;
    int32_t* free_d = nullptr;
    std::vector<int32_t> free_h;
    double* stage = nullptr;            // staging buffer for host<->device conversions
    size_t stage_n = 0;
    // pinned host mirror of small device state
    PcgScalars* S_h = nullptr;
    OcState* OC_h = nullptr;
    FilterScalars* FS_h = nullptr;
    double* scal_h = nullptr;
    int* flag_h = nullptr;              // two done-flag slots for pipelined polling
    // CUDA graph of a chunk of PCG iterations
    cudaGraphExec_t pcg_graph = nullptr;
    int pcg_graph_len = 0;
    bool use_graph = true;
    // design state
    bool mg_ready = false;
    bool design_ready = false;
    float V0 = 0.0f;
    int loop = 0;
    cudaEvent_t ev[8]{};
    int64_t launches = 0;   // kernels launched (graph replays counted per node)

    // device memory: carved from `arena` while one is attached and has room, else cudaMalloc'd (and freed
    // with the context); carved counts both, each rounded up to 256 bytes (the size an arena needs)
    Arena* arena = nullptr;
    size_t carved = 0;
    template <class T>
    int alloc(T** ptr, size_t n) {
        void* q = nullptr;
        const size_t nb = std::max<size_t>(n, 1) * sizeof(T);
        const size_t nr = (nb + 255) / 256 * 256;
        carved += nr;
        bytes += nb;
        if (arena && arena->used + nr <= arena->size) {
            q = arena->base + arena->used;
            arena->used += nr;
            *ptr = static_cast<T*>(q);
            return T3D_OK;
        }
        cudaError_t e = cudaMalloc(&q, nb);
        if (e != cudaSuccess) return set_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
        allocs.push_back(q);
        *ptr = static_cast<T*>(q);
        return T3D_OK;
    }

    ~Context() {
        if (pcg_graph) cudaGraphExecDestroy(pcg_graph);
        if (pcg32_graph) cudaGraphExecDestroy(pcg32_graph);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (void* q : allocs) cudaFree(q);
        if (S_h) cudaFreeHost(S_h);
        if (OC_h) cudaFreeHost(OC_h);
        if (FS_h) cudaFreeHost(FS_h);
        if (scal_h) cudaFreeHost(scal_h);
        if (flag_h) cudaFreeHost(flag_h);
        if (st) cudaStreamDestroy(st);
    }
};

int launch_check(const char* what);
int sync(Context* c);
int check_tma(Context* c);
int create(int nely, int nelx, int nelz, const t3d_params* prm, const t3d_problem* pb, Context* c);
int ensure_morton(Context* c);
// y = K(E) u in FP64 on c->E; returns the number of kernels launched
int matvec64(Context* c, const double* u, double* y, RedSlot dot, PcgScalars* S);
int design_init(Context* c, float V0, double* Csolid);
// a design iteration without its solve: design_pre (loop count, SIMP, MG rebuild when due) ... the solve of
// K(E) u = b with the compliance into c->scal[0] ... design_post (objective, sensitivities, filter, OC, record)
int design_pre(Context* c);
int design_post(Context* c, int pcg_iters, t3d_iter_record* rec);
// z = M r: one FP32 V-cycle of the mixed-precision inner solve (either cycle) on c->st
int member_vcycle32(Context* c, const float* r, float* z, PcgScalars* S, RedSlot dot);

}  // namespace t3d

struct t3d_context : public t3d::Context {};
