// Batched designs: many designs of uneven grid size advance together, one launch per kernel of the inner
// PCG iteration for all of them.
//
// Layout.  The members' buffers are carved from one device arena (sized by a first, counting creation of each
// member).  Each member keeps its own context -- grid, MG hierarchy, FP32/FP64 vectors, reduction slots and
// scalars -- so everything outside the inner solve runs per member on the member's stream, in parallel host
// threads (SIMP, MG rebuild, compliance, sensitivities, filter, OC).
//
// Work list.  Every kernel of the FP32 MG-PCG iteration is one persistent launch over (instance, logical
// block) items (kernels.hpp, "batched launches"): the logical blocks of an instance are the blocks of the
// launch the member would make alone, so each member's arithmetic and reduction order are those of its own
// launch and its results are identical to a solo run with the same parameters.  Per-instance convergence
// masks: a member whose inner solve has converged or spent its budget (S->done, set on the device) skips its
// items for the rest of that iteration, and a compaction kernel at the end of every iteration drops it from
// the work lists, so finished members cost nothing while the others go on.  BATCH_CHUNK iterations are
// captured once in a CUDA graph and replayed; the host polls the members' done flags (gathered into one
// array) after each replay.
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

struct LaunchList {      // one batched launch: per-instance arguments and the active-instance list on the device
    void* args = nullptr;
    int* act = nullptr;   // n, positions, block prefix sums (kernels.hpp)
    int n = 0;            // instances in the list
    int64_t blocks = 0;   // logical blocks with every instance active
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
    bool standard = false;       // the members' V-cycle (all the same): Standard, else Adapted
    LaunchList mv, up, dir, p0, co, mv1, mv2;
    LaunchList rs0[8], rs1[8], pr[8], lop[8], lmv[8], pa[8];
    int maxL = 0, coarse_max = 0;
    CUtensorMap* maps = nullptr;
    std::vector<BatchCompact> jobs;   // one per launch list
    BatchCompact* djobs = nullptr;
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
    int n_arena = 0;             // members 0 .. n_arena-1 live in the arena (created with the batch)
    bool dirty = true;           // membership changed: the launch lists and the graph are rebuilt before use

    template <class T>
    int dalloc(T** p, size_t n) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) return set_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
        dallocs.push_back(q);
        *p = static_cast<T*>(q);
        return T3D_OK;
    }

    // the launch lists, the graph and the polling buffers (rebuilt when membership changes)
    void free_lists() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        for (void* q : dallocs) cudaFree(q);
        dallocs.clear();
        if (hflags) cudaFreeHost(hflags);
        if (hS) cudaFreeHost(hS);
        if (hscal) cudaFreeHost(hscal);
        hflags = nullptr;
        hS = nullptr;
        hscal = nullptr;
        maps = nullptr;
        jobs.clear();
        djobs = nullptr;
        dS = nullptr;
        dflags = nullptr;
        err = nullptr;
        mv = up = dir = p0 = co = mv1 = mv2 = LaunchList{};
        for (int l = 0; l < 8; ++l) rs0[l] = rs1[l] = pr[l] = lop[l] = lmv[l] = pa[l] = LaunchList{};
    }

    ~Batch() {
        cudaSetDevice(dev);
        if (st) cudaStreamSynchronize(st);
        for (t3d_context* c : m) {
            if (!c) continue;
            cudaStreamSynchronize(c->st);
            delete c;
        }
        free_lists();
        if (arena.base) cudaFree(arena.base);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

// uploads one launch list: args[k] with blocks[k] logical blocks each and scalars S[k]; the active list starts
// with every instance and its compaction job is queued
template <class T>
int make_list(Batch* B, const std::vector<T>& a, const std::vector<int>& blocks, const std::vector<PcgScalars*>& S,
              LaunchList* L) {
    const int N = (int)a.size();
    L->n = N;
    L->blocks = 0;
    if (N == 0) return T3D_OK;
    std::vector<int> act(2 * (size_t)N + 2, 0);
    act[0] = N;
    for (int k = 0; k < N; ++k) {
        if (blocks[k] <= 0) return set_error(T3D_ERR_INVALID, "batched launch with an empty instance");
        act[1 + k] = k;
        act[2 + N + k] = act[1 + N + k] + blocks[k];
    }
    L->blocks = act[1 + 2 * N];
    T* da = nullptr;
    int* db = nullptr;
    PcgScalars** dS = nullptr;
    CHECK(B->dalloc(&da, a.size()));
    CHECK(B->dalloc(&L->act, act.size()));
    CHECK(B->dalloc(&db, blocks.size()));
    CHECK(B->dalloc(&dS, S.size()));
    T3D_CUDA_OK(cudaMemcpy(da, a.data(), a.size() * sizeof(T), cudaMemcpyHostToDevice));
    T3D_CUDA_OK(cudaMemcpy(L->act, act.data(), act.size() * sizeof(int), cudaMemcpyHostToDevice));
    T3D_CUDA_OK(cudaMemcpy(db, blocks.data(), blocks.size() * sizeof(int), cudaMemcpyHostToDevice));
    T3D_CUDA_OK(cudaMemcpy(dS, S.data(), S.size() * sizeof(PcgScalars*), cudaMemcpyHostToDevice));
    L->args = da;
    B->jobs.push_back(BatchCompact{dS, db, N, L->act});
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
        if (c->standard != c0->standard) return set_error(T3D_ERR_INVALID, who + "members must share one V-cycle");
        if (c->ncases != 1) return set_error(T3D_ERR_INVALID, who + "batched designs have one load case");
        if (c->nlev < 2) return set_error(T3D_ERR_INVALID, who + "batched designs need two MG levels at least");
        if (!c->modal || c->mt.variant != B->variant || !modal_fused_available(c->mt))
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
    T3D_CUDA_OK(cudaStreamSynchronize(B->st));
    B->free_lists();
    B->dirty = true;
    const int n = (int)B->m.size();
    if (n == 0) return T3D_OK;
    B->standard = B->m[0]->standard;
    // tensor maps per member: the PCG product (p, E); the Standard cycle's level-0 products (z, E_mg), (Ap, E_mg)
    const int per = B->standard ? 6 : 2;
    std::vector<CUtensorMap> maps((size_t)per * n);
    for (int i = 0; i < n; ++i) {
        const t3d_context* c = B->m[i];
        CUtensorMap* q = &maps[(size_t)per * i];
        bool ok = modal_tensor_maps_for(B->variant, c->g, c->p32, c->E32, q, q + 1);
        if (B->standard)
            ok = ok && modal_tensor_maps_for(B->variant, c->g, c->z32, c->E_mg32, q + 2, q + 3) &&
                 modal_tensor_maps_for(B->variant, c->g, c->Ap32, c->E_mg32, q + 4, q + 5);
        if (!ok) return set_error(T3D_ERR_CUDA, "batch member " + std::to_string(i) + ": tensor maps could not be encoded");
    }
    CHECK(B->dalloc(&B->maps, maps.size()));
    T3D_CUDA_OK(cudaMemcpy(B->maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));

    B->maxL = 0;
    B->coarse_max = 0;
    B->iter_kernels = 0;
    B->iter_blocks = 0;
    for (const t3d_context* c : B->m) {
        B->maxL = std::max(B->maxL, c->nlev);
        B->coarse_max = std::max(B->coarse_max, c->Nc);
    }
    // one list: the arguments f(c, i) of the members that `take` (c, i), with their block counts
    auto list = [&](LaunchList* L, auto take, auto f, auto blocks) -> int {
        using A = decltype(f(B->m[0], 0));
        std::vector<A> a;
        std::vector<int> bl;
        std::vector<PcgScalars*> S;
        for (int i = 0; i < n; ++i) {
            t3d_context* c = B->m[i];
            if (!take(c)) continue;
            a.push_back(f(c, i));
            bl.push_back(blocks(a.back()));
            S.push_back(c->S32);
        }
        CHECK(make_list(B, a, bl, S, L));
        B->iter_kernels += L->n > 0;
        B->iter_blocks += L->blocks;
        return T3D_OK;
    };
    auto all = [](const t3d_context*) { return true; };
    auto mvb = [](const BatchMatvec& a) { return a.t.grid; };
    CHECK(list(&B->mv, all, [&](t3d_context* c, int i) {
        const CUtensorMap* q = B->maps + (size_t)per * i;
        return BatchMatvec{c->g, c->mt, c->mask0, c->Ap32, c->slot[0], c->S32, q, q + 1, nullptr, nullptr, 0.f};
    }, mvb));
    CHECK(list(&B->up, all, [](t3d_context* c, int) {
        return BatchUpdate{c->g.NNp, c->r32, c->Ap32, c->slot[1], c->S32};
    }, [](const BatchUpdate&) { return batch_blocks_update(); }));
    CHECK(list(&B->dir, all, [](t3d_context* c, int) {
        return BatchDirection{c->g.NNp, c->z32, c->p32, c->d32, c->S32};
    }, [](const BatchDirection&) { return batch_blocks_update(); }));
    CHECK(list(&B->co, all, [](t3d_context* c, int) {
        return BatchCoarse{c->lv32[c->nlev - 1], c->Xc, c->Nc, c->chol_status, c->S32};
    }, [](const BatchCoarse& a) { return batch_blocks_coarse(a); }));
    const int norm = B->standard ? 0 : 1;
    for (int l = 0; l + 1 < B->maxL; ++l) {
        auto below = [l](const t3d_context* c) { return c->nlev - 1 > l; };
        auto rs = [&, l](t3d_context* c, int) {
            const float* src = B->standard ? (l == 0 ? c->Ap32 : c->vtmp32[l]) : (l == 0 ? c->r32 : c->lv32[l].r);
            return BatchRestrict{c->lv32[l + 1], c->lv32[l], src, c->ra1_32[l], c->lv32[l + 1].r, c->S32, norm};
        };
        CHECK(list(&B->rs0[l], below, rs, [](const BatchRestrict& a) { return batch_blocks_restrict(a, 0); }));
        CHECK(list(&B->rs1[l], [&, l](const t3d_context* c) {
            return c->nlev - 1 > l && c->lv32[l + 1].span == 4;
        }, rs, [](const BatchRestrict& a) { return batch_blocks_restrict(a, 1); }));
        if (!B->standard) {
            if (l >= 1)
                CHECK(list(&B->pr[l], below, [l](t3d_context* c, int) {
                    return BatchProlong{c->lv32[l + 1], c->lv32[l], c->prm.mg_weight, c->S32};
                }, [](const BatchProlong& a) { return batch_blocks_prolong(a); }));
            continue;
        }
        // the Standard cycle's level steps, level matrices and prolongations (level 0: z, r and the TMA products)
        CHECK(list(&B->lop[l], below, [l](t3d_context* c, int) {
            const MgLevel32& L = c->lv32[l];
            return l == 0 ? BatchLevelOp{L, c->r32, nullptr, c->z32, c->prm.mg_standard_weight, c->S32}
                          : BatchLevelOp{L, L.r, c->vtmp32[l], L.x, c->prm.mg_standard_weight, c->S32};
        }, [](const BatchLevelOp& a) { return batch_blocks_level_op(a); }));
        CHECK(list(&B->pa[l], below, [l](t3d_context* c, int) {
            const MgLevel32 &Lc = c->lv32[l + 1], &Lf = c->lv32[l];
            return l == 0 ? BatchProlongAdd{Lc, Lf, Lc.x, c->z32, c->Ap32, c->S32}
                          : BatchProlongAdd{Lc, Lf, Lc.x, Lf.x, Lf.x, c->S32};
        }, [](const BatchProlongAdd& a) { return batch_blocks_prolong_add(a); }));
        if (l >= 1) {
            CHECK(list(&B->lmv[l], below, [l](t3d_context* c, int) {
                return BatchLevelMatvec{c->lv32[l], c->Kel32[l], c->lv32[l].x, c->vtmp32[l], c->S32};
            }, [](const BatchLevelMatvec& a) { return batch_blocks_level_matvec(a); }));
            // each level op and level product runs twice per cycle (down and up)
            B->iter_kernels += 2;
            B->iter_blocks += B->lop[l].blocks + B->lmv[l].blocks;
        }
    }
    if (B->standard) {
        CHECK(list(&B->mv1, all, [&](t3d_context* c, int i) {
            const CUtensorMap* q = B->maps + (size_t)per * i + 2;
            return BatchMatvec{c->g, c->mt, c->mask0, c->Ap32, RedSlot{nullptr, nullptr}, c->S32, q, q + 1, c->r32,
                               nullptr, c->prm.mg_standard_weight};
        }, mvb));
        CHECK(list(&B->mv2, all, [&](t3d_context* c, int i) {
            const CUtensorMap* q = B->maps + (size_t)per * i + 4;
            return BatchMatvec{c->g, c->mt, c->mask0, c->z32, c->slot[2], c->S32, q, q + 1, c->r32, c->lv32[0].diag,
                               c->prm.mg_standard_weight};
        }, mvb));
    } else {
        CHECK(list(&B->p0, all, [](t3d_context* c, int) {
            return BatchProlong0{c->lv32[1], c->lv32[0], c->r32, c->z32, c->prm.mg_weight, c->slot[2], c->S32};
        }, [](const BatchProlong0&) { return batch_blocks_prolong0(); }));
    }
    std::vector<PcgScalars*> S;
    for (const t3d_context* c : B->m) S.push_back(c->S32);
    CHECK(B->dalloc(&B->djobs, B->jobs.size()));
    T3D_CUDA_OK(cudaMemcpy(B->djobs, B->jobs.data(), B->jobs.size() * sizeof(BatchCompact), cudaMemcpyHostToDevice));
    B->iter_kernels += 1;   // the compaction
    CHECK(B->dalloc(&B->dS, S.size()));
    T3D_CUDA_OK(cudaMemcpy(B->dS, S.data(), S.size() * sizeof(PcgScalars*), cudaMemcpyHostToDevice));
    CHECK(B->dalloc(&B->dflags, (size_t)n));
    CHECK(B->dalloc(&B->err, 1));
    T3D_CUDA_OK(cudaMemset(B->err, 0, sizeof(int)));
    T3D_CUDA_OK(cudaMallocHost(&B->hflags, (size_t)n * sizeof(int)));
    T3D_CUDA_OK(cudaMallocHost(&B->hS, (size_t)n * sizeof(PcgScalars)));
    T3D_CUDA_OK(cudaMallocHost(&B->hscal, (size_t)n * sizeof(double)));
    CHECK(modal_batched_grid(B->variant, B->dev, &B->mv_grid));
    B->dirty = false;
    return T3D_OK;
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
    B->n_arena = n;
    T3D_CUDA_OK(cudaStreamCreateWithFlags(&B->st, cudaStreamNonBlocking));
    return batch_lists(B);
}

// ------------------------------------------------------------------ the batched inner solve
template <class T>
static const T* args_of(const LaunchList& L) {
    return static_cast<const T*>(L.args);
}

static void batch_restrict(Batch* B, int l) {
    if (B->rs0[l].n) launch_batch_restrict32(args_of<BatchRestrict>(B->rs0[l]), B->rs0[l].act, B->rs0[l].n, 0, B->st);
    if (B->rs1[l].n) launch_batch_restrict32(args_of<BatchRestrict>(B->rs1[l]), B->rs1[l].act, B->rs1[l].n, 1, B->st);
}

static void batch_product(Batch* B, int mode, const LaunchList& L) {
    launch_batch_matvec32(B->variant, mode, args_of<BatchMatvec>(L), L.act, L.n, B->kh, B->mv_grid, B->err, B->st);
}

// vcycle32 (context.cu) for every member: the Adapted cycle, or the Standard one (vcycle32_standard) with its
// level-0 residual and correction fused into the TMA products
static void batch_vcycle(Batch* B) {
    if (!B->standard) {
        for (int l = 0; l + 1 < B->maxL; ++l) batch_restrict(B, l);
        launch_batch_coarse32(args_of<BatchCoarse>(B->co), B->co.act, B->co.n, B->coarse_max, B->st);
        for (int l = B->maxL - 2; l >= 1; --l)
            if (B->pr[l].n) launch_batch_prolong32(args_of<BatchProlong>(B->pr[l]), B->pr[l].act, B->pr[l].n, B->st);
        launch_batch_prolong0_32(args_of<BatchProlong0>(B->p0), B->p0.act, B->p0.n, B->st);
        return;
    }
    for (int l = 0; l + 1 < B->maxL; ++l) {
        const LaunchList& op = B->lop[l];
        launch_batch_level_op32(args_of<BatchLevelOp>(op), op.act, op.n, 0, B->st);          // x = w r / D
        if (l == 0) {
            batch_product(B, 1, B->mv1);                                                     // t = r - K x
        } else {
            const LaunchList& mv = B->lmv[l];
            launch_batch_level_matvec32(args_of<BatchLevelMatvec>(mv), mv.act, mv.n, B->st);   // t = K x
            launch_batch_level_op32(args_of<BatchLevelOp>(op), op.act, op.n, 1, B->st);      // t = r - t
        }
        batch_restrict(B, l);                                                                // r' = P^T t
    }
    launch_batch_coarse32(args_of<BatchCoarse>(B->co), B->co.act, B->co.n, B->coarse_max, B->st);
    for (int l = B->maxL - 2; l >= 1; --l) {
        const LaunchList &pa = B->pa[l], &mv = B->lmv[l], &op = B->lop[l];
        launch_batch_prolong_add32(args_of<BatchProlongAdd>(pa), pa.act, pa.n, B->st);       // x += P x'
        launch_batch_level_matvec32(args_of<BatchLevelMatvec>(mv), mv.act, mv.n, B->st);     // t = K x
        launch_batch_level_op32(args_of<BatchLevelOp>(op), op.act, op.n, 2, B->st);          // x += w (r - t) / D
    }
    launch_batch_prolong_add32(args_of<BatchProlongAdd>(B->pa[0]), B->pa[0].act, B->pa[0].n, B->st);   // T = z + P x'
    batch_product(B, 2, B->mv2);                                      // z = T + w (r - K T) / D, with r.z
}

// one PCG iteration of every member (pcg32_iteration in context.cu, batched)
static void batch_iteration(Batch* B) {
    batch_product(B, 0, B->mv);
    launch_batch_update32(args_of<BatchUpdate>(B->up), B->up.act, B->up.n, B->st);
    batch_vcycle(B);
    launch_batch_direction32(args_of<BatchDirection>(B->dir), B->dir.act, B->dir.n, B->st);
    // members whose solve ended in this iteration (their last step applied above) leave the work lists
    launch_batch_compact(B->djobs, (int)B->jobs.size(), B->st);
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
        launch_batch_compact(B->djobs, (int)B->jobs.size(), B->st);   // the members iterating in this pass
        batch_vcycle(B);   // z = M r for them
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
    if (B->m.empty()) return T3D_OK;
    if (B->dirty) CHECK(batch_lists(B));
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

int t3d_batch_open(int device, t3d_batch** out) {
    if (!out) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    *out = nullptr;
    t3d_batch* b = new (std::nothrow) t3d_batch();
    if (!b) return t3d::set_error(T3D_ERR_OOM, "host allocation failed");
    b->dev = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete b;
        return t3d::set_cuda_error(e, "t3d_batch_open", __FILE__, __LINE__);
    }
    *out = b;
    return T3D_OK;
}

int t3d_batch_adopt(t3d_batch* b, t3d_context* ctx) {
    if (!b || !ctx) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    if (!ctx->design_ready) return t3d::set_error(T3D_ERR_INVALID, "t3d_design_init not called on the context");
    for (const t3d_context* c : b->m)
        if (c == ctx) return t3d::set_error(T3D_ERR_INVALID, "context is already a batch member");
    if (cudaSetDevice(b->dev) != cudaSuccess) return t3d::set_error(T3D_ERR_CUDA, "cudaSetDevice failed");
    if (ctx->dev != b->dev) return t3d::set_error(T3D_ERR_INVALID, "context is on another device");
    b->m.push_back(ctx);
    const int rc = t3d::batch_members_check(b);
    if (rc != T3D_OK) {
        b->m.pop_back();
        return rc;
    }
    if (b->m.size() == 1) b->kh = ctx->kh;
    b->dirty = true;
    return T3D_OK;
}

int t3d_batch_release(t3d_batch* b, int i, t3d_context** out) {
    if (!b || !out || i < 0 || i >= (int)b->m.size()) return t3d::set_error(T3D_ERR_INVALID, "bad batch member");
    if (i < b->n_arena) return t3d::set_error(T3D_ERR_INVALID, "member lives in the batch arena");
    if (cudaSetDevice(b->dev) != cudaSuccess) return t3d::set_error(T3D_ERR_CUDA, "cudaSetDevice failed");
    if (cudaStreamSynchronize(b->st) != cudaSuccess) return t3d::set_error(T3D_ERR_CUDA, "batch stream failed");
    *out = b->m[(size_t)i];
    b->m.erase(b->m.begin() + i);
    b->dirty = true;
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
