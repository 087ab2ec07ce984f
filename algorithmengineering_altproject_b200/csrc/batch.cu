// Batched designs: many designs of uneven grid size advance together, one launch per kernel of the inner
// PCG iteration for all of them.
//
// Layout.  The members' buffers are carved from one device arena (sized by a first, counting creation of each
// member).  Each member keeps its own context -- grid, MG hierarchy, FP32/FP64 vectors, reduction slots and
// scalars -- so everything outside the inner solve runs per member on the member's stream, in parallel host
// threads (SIMP, MG rebuild, compliance, sensitivities, filter, OC).
//
// Work list.  Every kernel of the FP32 MG-PCG iteration is one persistent launch over (instance, logical
// block) items (kernels.hpp, "batched launches"): logical block v of instance i is block v - vstart[i] of
// the launch the member would make alone, so each member's arithmetic and reduction order are those of its
// own launch and its results are identical to a solo run with the same parameters.  Members whose inner
// solve has converged or spent its budget (S->done, set on the device) skip their items: the per-instance
// convergence mask.  BATCH_CHUNK iterations are captured once in a CUDA graph and replayed; the host polls
// the members' done flags (gathered into one array) after each replay.
//
// The FP64 defect-correction loop around the inner solve (mixed_solve in context.cu) is run for all members
// in lock step: one true-residual pass for the members still iterating, one batched inner solve, one
// accumulation, and again, each member with its own stop test and iteration budget.
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>

#include "context.hpp"

namespace t3d {

namespace {

constexpr int BATCH_CHUNK = 16;      // inner PCG iterations per graph replay
constexpr int BATCH_THREADS = 16;    // host threads of the per-member phases
constexpr int BATCH_MAX_OUTER = 64;  // defect-correction passes (as the single-design solve)

struct LaunchList {      // one batched launch: per-instance arguments and block prefix sums on the device
    void* args = nullptr;
    int* vstart = nullptr;
    int n = 0;
    int64_t blocks = 0;
};

}  // namespace

struct Batch {
    int dev = 0;
    std::vector<t3d_context*> m;
    Arena arena;
    cudaStream_t st = nullptr;
    int variant = T3D_BATCH_TILE - 1;
    int mv_grid = 0;
    ModalKe kh{};
    std::vector<void*> dallocs;
    LaunchList mv, up, dir, p0, co;
    LaunchList rs0[8], rs1[8], pr[8];
    int maxL = 0, coarse_max = 0;
    CUtensorMap* maps = nullptr;
    PcgScalars** dS = nullptr;
    int* dflags = nullptr;
    int* err = nullptr;
    int* hflags = nullptr;       // pinned
    PcgScalars* hS = nullptr;    // pinned
    double* hscal = nullptr;     // pinned
    cudaGraphExec_t graph = nullptr;
    int64_t launches = 0;
    int iter_kernels = 0;
    int64_t iter_blocks = 0;

    template <class T>
    int dalloc(T** p, size_t n) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) return set_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
        dallocs.push_back(q);
        *p = static_cast<T*>(q);
        return T3D_OK;
    }

    ~Batch() {
        cudaSetDevice(dev);
        if (st) cudaStreamSynchronize(st);
        if (graph) cudaGraphExecDestroy(graph);
        for (t3d_context* c : m) {
            if (!c) continue;
            cudaStreamSynchronize(c->st);
            delete c;
        }
        for (void* q : dallocs) cudaFree(q);
        if (arena.base) cudaFree(arena.base);
        if (hflags) cudaFreeHost(hflags);
        if (hS) cudaFreeHost(hS);
        if (hscal) cudaFreeHost(hscal);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

// uploads one launch list: args[k] with blocks[k] logical blocks each
template <class T>
int make_list(Batch* B, const std::vector<T>& a, const std::vector<int>& blocks, LaunchList* L) {
    L->n = (int)a.size();
    L->blocks = 0;
    if (L->n == 0) return T3D_OK;
    std::vector<int> vs((size_t)L->n + 1, 0);
    for (int k = 0; k < L->n; ++k) {
        if (blocks[k] <= 0) return set_error(T3D_ERR_INVALID, "batched launch with an empty instance");
        vs[k + 1] = vs[k] + blocks[k];
    }
    L->blocks = vs[L->n];
    T* da = nullptr;
    CHECK(B->dalloc(&da, a.size()));
    CHECK(B->dalloc(&L->vstart, vs.size()));
    T3D_CUDA_OK(cudaMemcpy(da, a.data(), a.size() * sizeof(T), cudaMemcpyHostToDevice));
    T3D_CUDA_OK(cudaMemcpy(L->vstart, vs.data(), vs.size() * sizeof(int), cudaMemcpyHostToDevice));
    L->args = da;
    return T3D_OK;
}

// runs f(i) for every member on up to BATCH_THREADS host threads; the first failure (with its message,
// which lives in the failing thread) is returned
template <class F>
int for_members(Batch* B, F f) {
    const int n = (int)B->m.size();
    std::vector<int> rc((size_t)n, T3D_OK);
    std::vector<std::string> msg((size_t)n);
    std::atomic<int> next{0};
    auto work = [&]() {
        cudaSetDevice(B->dev);
        for (int i; (i = next.fetch_add(1)) < n;) {
            rc[(size_t)i] = f(i);
            if (rc[(size_t)i] != T3D_OK) msg[(size_t)i] = t3d_last_error();
        }
    };
    std::vector<std::thread> th;
    for (int k = 1; k < std::min(n, BATCH_THREADS); ++k) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
    for (int i = 0; i < n; ++i)
        if (rc[(size_t)i] != T3D_OK) return set_error(rc[(size_t)i], "batch member " + std::to_string(i) + ": " + msg[(size_t)i]);
    return T3D_OK;
}

}  // namespace

// ------------------------------------------------------------------ creation
static int batch_members_check(Batch* B) {
    const t3d_context* c0 = B->m[0];
    for (size_t i = 0; i < B->m.size(); ++i) {
        const t3d_context* c = B->m[i];
        const std::string who = "batch member " + std::to_string(i) + ": ";
        if (!c->mixed) return set_error(T3D_ERR_INVALID, who + "batched designs need precision T3D_MIXED");
        if (c->standard) return set_error(T3D_ERR_INVALID, who + "batched designs use the Adapted V-cycle");
        if (c->ncases != 1) return set_error(T3D_ERR_INVALID, who + "batched designs have one load case");
        if (c->nlev < 2) return set_error(T3D_ERR_INVALID, who + "batched designs need two MG levels at least");
        if (!c->modal || c->mt.variant != B->variant)
            return set_error(T3D_ERR_INVALID, who + "the batched K(E)p needs the modal TMA tile shape");
        if (c->dev != c0->dev) return set_error(T3D_ERR_INVALID, who + "members must share one device");
        if (std::memcmp(&c->kh, &c0->kh, sizeof c->kh) != 0)
            return set_error(T3D_ERR_INVALID, who + "members must share one element stiffness (E0, nu)");
    }
    return T3D_OK;
}

// the launch lists of one batched PCG iteration (all arguments are fixed for the life of the batch: the
// members' buffers never move)
static int batch_lists(Batch* B) {
    const int n = (int)B->m.size();
    std::vector<CUtensorMap> maps(2 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        const t3d_context* c = B->m[i];
        if (!modal_tensor_maps_for(B->variant, c->g, c->p32, c->E32, &maps[2 * i], &maps[2 * i + 1]))
            return set_error(T3D_ERR_CUDA, "batch member " + std::to_string(i) + ": tensor maps could not be encoded");
    }
    CHECK(B->dalloc(&B->maps, maps.size()));
    T3D_CUDA_OK(cudaMemcpy(B->maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));

    std::vector<BatchMatvec> mv;
    std::vector<BatchUpdate> up;
    std::vector<BatchDirection> dir;
    std::vector<BatchProlong0> p0;
    std::vector<BatchCoarse> co;
    std::vector<int> bmv, bup, bdir, bp0, bco;
    std::vector<PcgScalars*> S;
    B->maxL = 0;
    B->coarse_max = 0;
    for (int i = 0; i < n; ++i) {
        t3d_context* c = B->m[i];
        mv.push_back(BatchMatvec{c->g, c->mt, c->mask0, c->Ap32, c->slot[0], c->S32, B->maps + 2 * i, B->maps + 2 * i + 1});
        bmv.push_back(c->mt.grid);
        up.push_back(BatchUpdate{c->g.NNp, c->r32, c->Ap32, c->slot[1], c->S32});
        bup.push_back(batch_blocks_update());
        dir.push_back(BatchDirection{c->g.NNp, c->z32, c->p32, c->d32, c->S32});
        bdir.push_back(batch_blocks_update());
        p0.push_back(BatchProlong0{c->lv32[1], c->lv32[0], c->r32, c->z32, c->prm.mg_weight, c->slot[2], c->S32});
        bp0.push_back(batch_blocks_prolong0());
        const BatchCoarse bc{c->lv32[c->nlev - 1], c->Xc, c->Nc, c->chol_status, c->S32};
        co.push_back(bc);
        bco.push_back(batch_blocks_coarse(bc));
        S.push_back(c->S32);
        B->maxL = std::max(B->maxL, c->nlev);
        B->coarse_max = std::max(B->coarse_max, c->Nc);
    }
    CHECK(make_list(B, mv, bmv, &B->mv));
    CHECK(make_list(B, up, bup, &B->up));
    CHECK(make_list(B, dir, bdir, &B->dir));
    CHECK(make_list(B, p0, bp0, &B->p0));
    CHECK(make_list(B, co, bco, &B->co));
    B->iter_kernels = 5;
    B->iter_blocks = B->mv.blocks + B->up.blocks + B->dir.blocks + B->p0.blocks + B->co.blocks;
    for (int l = 0; l + 1 < B->maxL; ++l) {
        std::vector<BatchRestrict> r0, r1;
        std::vector<BatchProlong> pr;
        std::vector<int> b0, b1, bp;
        for (int i = 0; i < n; ++i) {
            t3d_context* c = B->m[i];
            if (c->nlev - 1 <= l) continue;
            const BatchRestrict a{c->lv32[l + 1], c->lv32[l], l == 0 ? c->r32 : c->lv32[l].r, c->ra1_32[l],
                                  c->lv32[l + 1].r, c->S32};
            r0.push_back(a);
            b0.push_back(batch_blocks_restrict(a, 0));
            if (batch_blocks_restrict(a, 1) > 0) {
                r1.push_back(a);
                b1.push_back(batch_blocks_restrict(a, 1));
            }
            if (l >= 1) {
                const BatchProlong p{c->lv32[l + 1], c->lv32[l], c->prm.mg_weight, c->S32};
                pr.push_back(p);
                bp.push_back(batch_blocks_prolong(p));
            }
        }
        CHECK(make_list(B, r0, b0, &B->rs0[l]));
        CHECK(make_list(B, r1, b1, &B->rs1[l]));
        CHECK(make_list(B, pr, bp, &B->pr[l]));
        B->iter_kernels += (B->rs0[l].n > 0) + (B->rs1[l].n > 0) + (B->pr[l].n > 0);
        B->iter_blocks += B->rs0[l].blocks + B->rs1[l].blocks + B->pr[l].blocks;
    }
    CHECK(B->dalloc(&B->dS, S.size()));
    T3D_CUDA_OK(cudaMemcpy(B->dS, S.data(), S.size() * sizeof(PcgScalars*), cudaMemcpyHostToDevice));
    CHECK(B->dalloc(&B->dflags, (size_t)n));
    CHECK(B->dalloc(&B->err, 1));
    T3D_CUDA_OK(cudaMemset(B->err, 0, sizeof(int)));
    T3D_CUDA_OK(cudaMallocHost(&B->hflags, (size_t)n * sizeof(int)));
    T3D_CUDA_OK(cudaMallocHost(&B->hS, (size_t)n * sizeof(PcgScalars)));
    T3D_CUDA_OK(cudaMallocHost(&B->hscal, (size_t)n * sizeof(double)));
    return modal_batched_grid(B->variant, B->dev, &B->mv_grid);
}

static int batch_create(int n, const int* dims, const t3d_params* params, const t3d_problem* problems, Batch* B) {
    if (n <= 0 || !dims) return set_error(T3D_ERR_INVALID, "batch needs n > 0 members and their dims");
    std::vector<t3d_params> P((size_t)n);
    std::vector<t3d_problem> Q((size_t)n);
    for (int i = 0; i < n; ++i) {
        if (params) P[(size_t)i] = params[i];
        else {
            t3d_params_default(&P[(size_t)i]);
            P[(size_t)i].precision = T3D_MIXED;
        }
        P[(size_t)i].matvec32_tile = T3D_BATCH_TILE;
        if (problems) Q[(size_t)i] = problems[i];
        else {
            std::memset(&Q[(size_t)i], 0, sizeof(t3d_problem));
            Q[(size_t)i].load_case = T3D_LOAD_TIP_LINE;
        }
    }
    B->dev = P[0].device;
    T3D_CUDA_OK(cudaSetDevice(B->dev));
    // pass 1: the device bytes each member carves (created and released one at a time)
    size_t total = 0;
    for (int i = 0; i < n; ++i) {
        std::unique_ptr<t3d_context> t(new t3d_context());
        CHECK(create(dims[3 * i], dims[3 * i + 1], dims[3 * i + 2], &P[(size_t)i], &Q[(size_t)i], t.get()));
        total += t->carved;
    }
    // pass 2: the members inside one arena
    T3D_CUDA_OK(cudaMalloc(reinterpret_cast<void**>(&B->arena.base), total));
    B->arena.size = total;
    for (int i = 0; i < n; ++i) {
        t3d_context* c = new t3d_context();
        B->m.push_back(c);
        c->arena = &B->arena;
        const int rc = create(dims[3 * i], dims[3 * i + 1], dims[3 * i + 2], &P[(size_t)i], &Q[(size_t)i], c);
        c->arena = nullptr;
        if (rc != T3D_OK) return rc;
    }
    CHECK(batch_members_check(B));
    B->kh = B->m[0]->kh;
    B->variant = B->m[0]->mt.variant;
    T3D_CUDA_OK(cudaStreamCreateWithFlags(&B->st, cudaStreamNonBlocking));
    return batch_lists(B);
}

// ------------------------------------------------------------------ the batched inner solve
static void batch_vcycle(Batch* B) {
    for (int l = 0; l + 1 < B->maxL; ++l) {
        if (B->rs0[l].n)
            launch_batch_restrict32(static_cast<const BatchRestrict*>(B->rs0[l].args), B->rs0[l].vstart, B->rs0[l].n, 0,
                                    B->st);
        if (B->rs1[l].n)
            launch_batch_restrict32(static_cast<const BatchRestrict*>(B->rs1[l].args), B->rs1[l].vstart, B->rs1[l].n, 1,
                                    B->st);
    }
    launch_batch_coarse32(static_cast<const BatchCoarse*>(B->co.args), B->co.vstart, B->co.n, B->coarse_max, B->st);
    for (int l = B->maxL - 2; l >= 1; --l)
        if (B->pr[l].n)
            launch_batch_prolong32(static_cast<const BatchProlong*>(B->pr[l].args), B->pr[l].vstart, B->pr[l].n, B->st);
    launch_batch_prolong0_32(static_cast<const BatchProlong0*>(B->p0.args), B->p0.vstart, B->p0.n, B->st);
}

// one PCG iteration of every member (pcg32_iteration in context.cu, batched)
static void batch_iteration(Batch* B) {
    launch_batch_matvec32(B->variant, static_cast<const BatchMatvec*>(B->mv.args), B->mv.vstart, B->mv.n, B->kh,
                          B->mv_grid, B->err, B->st);
    launch_batch_update32(static_cast<const BatchUpdate*>(B->up.args), B->up.vstart, B->up.n, B->st);
    batch_vcycle(B);
    launch_batch_direction32(static_cast<const BatchDirection*>(B->dir.args), B->dir.vstart, B->dir.n, B->st);
}

static int batch_graph(Batch* B) {
    if (B->graph) return T3D_OK;
    cudaGraph_t graph;
    T3D_CUDA_OK(cudaStreamBeginCapture(B->st, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < BATCH_CHUNK; ++k) batch_iteration(B);
    T3D_CUDA_OK(cudaStreamEndCapture(B->st, &graph));
    cudaError_t e = cudaGraphInstantiate(&B->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGraphInstantiate", __FILE__, __LINE__);
    return T3D_OK;
}

// While the batch stream runs the members' solve, every member context issues its own launches there too (its
// stream is idle: the host synchronised it before); restored on exit.
struct OnBatchStream {
    Batch* B;
    std::vector<cudaStream_t> own;
    explicit OnBatchStream(Batch* b) : B(b) {
        for (t3d_context* c : B->m) {
            own.push_back(c->st);
            c->st = B->st;
        }
    }
    ~OnBatchStream() {
        for (size_t i = 0; i < B->m.size(); ++i) B->m[i]->st = own[i];
    }
};

// mixed_solve (context.cu) for every member in lock step: the FP64 true residual and stop test per member,
// the FP32 inner MG-PCG of all members still iterating in batched launches (inner target max(stop,
// 1e-5 |r64|), at most the member's remaining budget), then u64 += d32.  iters[i]: the member's inner
// iterations, or its cg_max_it when the budget ran out unconverged.
static int batch_solve(Batch* B, int* iters) {
    const int n = (int)B->m.size();
    CHECK(batch_graph(B));
    OnBatchStream on(B);
    std::vector<double> stop((size_t)n), rn((size_t)n);
    std::vector<int> budget((size_t)n), used((size_t)n, 0), outer((size_t)n, 0);
    std::vector<char> conv((size_t)n, 0), active((size_t)n, 1);
    for (int i = 0; i < n; ++i) {
        t3d_context* c = B->m[i];
        launch_cells_to32(c->g, c->E, c->E32, B->st);
        launch_dot(c->g, 3, c->b, c->b, c->slot[3], c->scal + 5, B->st);
        c->launches += 2;
        T3D_CUDA_OK(cudaMemcpyAsync(B->hscal + i, c->scal + 5, sizeof(double), cudaMemcpyDeviceToHost, B->st));
    }
    T3D_CUDA_OK(cudaStreamSynchronize(B->st));
    for (int i = 0; i < n; ++i) {
        const double nb = std::sqrt(B->hscal[i]);
        stop[(size_t)i] = (1.0e-30 < nb ? nb : 1.0e-30) * (double)B->m[i]->prm.cg_tol;
        budget[(size_t)i] = B->m[i]->prm.cg_max_it;
    }
    for (int pass = 0; pass < BATCH_MAX_OUTER; ++pass) {
        for (int i = 0; i < n; ++i) {
            if (!active[(size_t)i]) continue;
            t3d_context* c = B->m[i];
            c->launches += 1 + matvec64(c, c->u, c->Ap, RedSlot{nullptr, nullptr}, nullptr);
            launch_mixed_residual(c->g, c->b, c->Ap, c->r32, c->d32, c->slot[3], c->scal + 6, B->st);
            T3D_CUDA_OK(cudaMemcpyAsync(B->hscal + i, c->scal + 6, sizeof(double), cudaMemcpyDeviceToHost, B->st));
        }
        CHECK(launch_check("batched residual"));
        T3D_CUDA_OK(cudaStreamSynchronize(B->st));
        bool any = false;
        for (int i = 0; i < n; ++i) {
            if (!active[(size_t)i]) continue;
            rn[(size_t)i] = std::sqrt(B->hscal[i]);
            if (rn[(size_t)i] < stop[(size_t)i]) {
                conv[(size_t)i] = 1;
                active[(size_t)i] = 0;
            } else if (budget[(size_t)i] <= 0) {
                active[(size_t)i] = 0;
            } else {
                any = true;
                ++outer[(size_t)i];
            }
        }
        if (!any) break;
        // per-member inner-solve scalars; members not iterating are masked (done, nothing left to apply)
        for (int i = 0; i < n; ++i) {
            PcgScalars& h = B->hS[i];
            std::memset(&h, 0, sizeof h);
            if (active[(size_t)i]) {
                h.stop = std::max(stop[(size_t)i], 1e-5 * rn[(size_t)i]);
                h.tol = (double)B->m[i]->prm.cg_tol;
                h.first = 1;
                h.maxit = budget[(size_t)i];
            } else {
                h.done = 1;
            }
            T3D_CUDA_OK(cudaMemcpyAsync(B->m[i]->S32, &h, sizeof h, cudaMemcpyHostToDevice, B->st));
        }
        batch_vcycle(B);   // z = M r for the members iterating
        B->launches += B->iter_kernels - 3;
        for (int i = 0; i < n; ++i)
            if (active[(size_t)i]) {
                const t3d_context* c = B->m[i];
                T3D_CUDA_OK(cudaMemcpyAsync(c->p32, c->z32, 3 * c->g.NNp * sizeof(float), cudaMemcpyDeviceToDevice,
                                            B->st));
            }
        int longest = 0;
        for (int i = 0; i < n; ++i)
            if (active[(size_t)i]) longest = std::max(longest, budget[(size_t)i]);
        for (int chunk = 0;; ++chunk) {
            T3D_CUDA_OK(cudaGraphLaunch(B->graph, B->st));
            B->launches += (int64_t)BATCH_CHUNK * B->iter_kernels + 1;
            launch_batch_flags(B->dS, n, B->dflags, B->st);
            T3D_CUDA_OK(cudaMemcpyAsync(B->hflags, B->dflags, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, B->st));
            T3D_CUDA_OK(cudaStreamSynchronize(B->st));
            bool all = true;
            for (int i = 0; i < n; ++i) all = all && B->hflags[i] != 0;
            if (all) break;
            // every member stops by its own budget on the device (PcgScalars::maxit); this bound never binds
            if ((int64_t)(chunk + 1) * BATCH_CHUNK > (int64_t)longest + BATCH_CHUNK)
                return set_error(T3D_ERR_NUMERIC, "batched inner solve did not stop within its budget");
        }
        for (int i = 0; i < n; ++i) {
            if (!active[(size_t)i]) continue;
            t3d_context* c = B->m[i];
            launch_mixed_accumulate(c->g, c->u, c->d32, B->st);
            c->launches += 1;
            T3D_CUDA_OK(cudaMemcpyAsync(B->hS + i, c->S32, sizeof(PcgScalars), cudaMemcpyDeviceToHost, B->st));
        }
        T3D_CUDA_OK(cudaStreamSynchronize(B->st));
        for (int i = 0; i < n; ++i) {
            if (!active[(size_t)i]) continue;
            used[(size_t)i] += B->hS[i].it;
            budget[(size_t)i] -= B->hS[i].it;
        }
    }
    for (int i = 0; i < n; ++i) {
        iters[i] = conv[(size_t)i] ? used[(size_t)i] : B->m[i]->prm.cg_max_it;
        B->m[i]->last_outer = outer[(size_t)i];
    }
    int e = 0;
    T3D_CUDA_OK(cudaMemcpy(&e, B->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return set_error(T3D_ERR_CUDA, "batched TMA-staged K(E)p: an mbarrier wait timed out");
    return T3D_OK;
}

static int batch_design_step(Batch* B, t3d_iter_record* recs) {
    CHECK(for_members(B, [&](int i) -> int {
        t3d_context* c = B->m[i];
        CHECK(design_pre(c));
        T3D_CUDA_OK(cudaStreamSynchronize(c->st));
        return T3D_OK;
    }));
    std::vector<int> its(B->m.size(), 0);
    CHECK(batch_solve(B, its.data()));
    return for_members(B, [&](int i) -> int {
        t3d_context* c = B->m[i];
        launch_compliance64(c->g, c->Ke, c->E, c->u, c->ce, c->slot[0], c->scal + 0, c->st);
        c->launches += 1;
        return design_post(c, its[(size_t)i], recs ? recs + i : nullptr);
    });
}

}  // namespace t3d

// ====================================================================== C-ABI
struct t3d_batch : public t3d::Batch {};

extern "C" {

int t3d_batch_create(int n, const int* dims, const t3d_params* params, const t3d_problem* problems, t3d_batch** out) {
    if (!out) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    *out = nullptr;
    t3d_batch* b = new (std::nothrow) t3d_batch();
    if (!b) return t3d::set_error(T3D_ERR_OOM, "host allocation failed");
    const int rc = t3d::batch_create(n, dims, params, problems, b);
    if (rc != T3D_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return T3D_OK;
}

int t3d_batch_member(t3d_batch* b, int i, t3d_context** out) {
    if (!b || !out || i < 0 || i >= (int)b->m.size()) return t3d::set_error(T3D_ERR_INVALID, "bad batch member");
    *out = b->m[(size_t)i];
    return T3D_OK;
}

int t3d_batch_design_init(t3d_batch* b, const float* V0, double* c_solid) {
    if (!b || !V0) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    if (cudaSetDevice(b->dev) != cudaSuccess) return t3d::set_error(T3D_ERR_CUDA, "cudaSetDevice failed");
    return t3d::for_members(b, [&](int i) -> int {
        return t3d::design_init(b->m[(size_t)i], V0[i], c_solid ? c_solid + i : nullptr);
    });
}

int t3d_batch_design_step(t3d_batch* b, t3d_iter_record* recs) {
    if (!b) return t3d::set_error(T3D_ERR_INVALID, "null batch");
    if (cudaSetDevice(b->dev) != cudaSuccess) return t3d::set_error(T3D_ERR_CUDA, "cudaSetDevice failed");
    return t3d::batch_design_step(b, recs);
}

int t3d_batch_info(t3d_batch* b, int64_t* info) {
    if (!b || !info) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    int64_t member = 0;
    for (const t3d_context* c : b->m) member += c->launches;
    info[0] = (int64_t)b->arena.size;
    info[1] = (int64_t)b->m.size();
    info[2] = b->launches;
    info[3] = b->iter_kernels;
    info[4] = b->iter_blocks;
    info[5] = member;
    return T3D_OK;
}

int t3d_batch_destroy(t3d_batch* b) {
    delete b;
    return T3D_OK;
}

}  // extern "C"
