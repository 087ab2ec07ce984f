// Drop-in implementation of the reference's C++ operator API over libt3d_b200's C-ABI.
//
// Compiled against the reference's own headers (cpp/include: core.hpp, fea.hpp, solver.hpp, filter.hpp,
// driver.hpp, multigrid/multigrid.hpp), this file defines the free functions those headers declare, so a
// program written against them -- the reference CLI apps/top3d_cli.cpp, unmodified -- links this library
// in place of the reference's cpp/src and runs on the GPU.  Every operator forwards to one C-ABI call:
//
//   ComputeVoxelKe                     (fea.hpp:37)            t3d_voxel_ke
//   CreateVoxelFEAmodel_Cuboid         (fea.hpp:38)            t3d_create (+ t3d_get_info / _element_map / _ke)
//   ApplyBoundaryConditions            (fea.hpp:39)            t3d_get_free_dofs, t3d_get_load
//   K_times_u_finest, both overloads   (fea.hpp:42,45)         t3d_matvec
//   ComputeCompliance                  (fea.hpp:47)            t3d_compliance
//   restrict_to_free/scatter_from_free (solver.hpp:8-9)        host index copies (the layout boundary)
//   make_jacobi_preconditioner         (solver.hpp:22)         t3d_mg_setup + t3d_mg_get_diag (level 0)
//   PCG_free                           (solver.hpp:24-27)      t3d_pcg for this library's preconditioner
//   mg::BuildMGHierarchy, build_static_once (multigrid.hpp:64-65)     t3d_get_info, t3d_mg_get_mask
//   mg::make_diagonal_preconditioner_from_static (multigrid.hpp:66-68) t3d_mg_setup; closure = t3d_vcycle
//   SetupPDEFilter / ApplyPDEFilter    (filter.hpp:17,28)      t3d_filter_setup / t3d_filter_apply
//   TOP3D_XL_GLOBAL                    (driver.hpp:4)          t3d_design_init + t3d_design_step, device-resident
//   InitialSettings                    (core.hpp:99)           the GlobalParams defaults
//
// Each reference `Problem` object is bound (by address) to one device context, created by
// CreateVoxelFEAmodel_Cuboid or on first use from pb.mesh.origRes*; a Problem whose sizes or solver
// parameters change gets a new context.  Fields of Problem that only the reference's own CPU kernels
// read (eNodMat, eDofMat, coloring, eDofFreeMat, node maps) are left empty; pb.F holds the load on the
// free DOFs (zero on fixed DOFs, which nothing on the reference's path reads).  Errors, which the
// reference does not report, are thrown as std::runtime_error with the library's message.
//
// Environment (TOP3D_XL_GLOBAL only): T3D_PRECISION=mixed selects the FP32-inner mixed-precision solve
// (default: the reference's FP64 PCG), T3D_DEVICE selects the CUDA device (default 0).
#include "core.hpp"
#include "driver.hpp"
#include "fea.hpp"
#include "filter.hpp"
#include "multigrid/multigrid.hpp"
#include "solver.hpp"
#include "t3d_b200.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

void check(int rc, const char* what) {
    if (rc != T3D_OK) throw std::runtime_error(std::string(what) + ": " + t3d_last_error());
}

int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    return (v && *v) ? std::atoi(v) : dflt;
}

// The device context behind one reference Problem, and the parameters it was created with.
struct Binding {
    t3d_context* ctx = nullptr;
    int nely = 0, nelx = 0, nelz = 0;
    t3d_params prm{};
    float filter_rmin = 0.0f;
    uint64_t mg_generation = 0;   // t3d_mg_setup calls so far: which preconditioner the context holds
    int64_t ne = 0, nn = 0, nf = 0;
    Binding() = default;
    Binding(const Binding&) = delete;
    Binding& operator=(const Binding&) = delete;
    ~Binding() {
        if (ctx) t3d_destroy(ctx);
    }
};

std::mutex g_mu;
std::map<const top3d::Problem*, std::shared_ptr<Binding>> g_bind;

t3d_params params_of(const top3d::Problem& pb, const top3d::mg::MGPrecondConfig* mg) {
    t3d_params p;
    check(t3d_params_default(&p), "t3d_params_default");
    p.E0 = pb.params.youngsModulus;
    p.Emin = pb.params.youngsModulusMin;
    p.penal = pb.params.simpPenalty;
    p.cg_tol = pb.params.cgTol;
    p.cg_max_it = pb.params.cgMaxIt;
    p.device = env_int("T3D_DEVICE", 0);
    if (mg) {
        p.mg_nondyadic = mg->nonDyadic ? 1 : 0;
        p.mg_max_levels = mg->maxLevels;
        p.mg_weight = mg->weight;
    }
    return p;
}

bool same_params(const t3d_params& a, const t3d_params& b) {
    return a.E0 == b.E0 && a.Emin == b.Emin && a.penal == b.penal && a.cg_tol == b.cg_tol &&
           a.cg_max_it == b.cg_max_it && a.device == b.device && a.mg_nondyadic == b.mg_nondyadic &&
           a.mg_max_levels == b.mg_max_levels && a.mg_weight == b.mg_weight;
}

std::shared_ptr<Binding> create_binding(const top3d::Problem& pb, int nely, int nelx, int nelz, const t3d_params& p) {
    auto b = std::make_shared<Binding>();
    check(t3d_create(nely, nelx, nelz, &p, &b->ctx), "t3d_create");
    b->nely = nely;
    b->nelx = nelx;
    b->nelz = nelz;
    b->prm = p;
    b->filter_rmin = p.filter_rmin;
    t3d_info inf;
    check(t3d_get_info(b->ctx, &inf), "t3d_get_info");
    b->ne = inf.num_elements;
    b->nn = inf.num_nodes;
    b->nf = inf.num_free;
    g_bind[&pb] = b;
    return b;
}

// The binding of pb; with `mg`, one whose multigrid parameters are those of `mg` (else the binding's own).
std::shared_ptr<Binding> binding(const top3d::Problem& pb, const top3d::mg::MGPrecondConfig* mg = nullptr) {
    const auto& m = pb.mesh;
    if (m.origResX <= 0 || m.origResY <= 0 || m.origResZ <= 0)
        throw std::runtime_error("Problem has no cuboid: call CreateVoxelFEAmodel_Cuboid first");
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_bind.find(&pb);
    if (it != g_bind.end()) {
        const auto& b = it->second;
        t3d_params want = params_of(pb, nullptr);
        want.mg_nondyadic = b->prm.mg_nondyadic;
        want.mg_max_levels = b->prm.mg_max_levels;
        want.mg_weight = b->prm.mg_weight;
        if (mg) {
            want.mg_nondyadic = mg->nonDyadic ? 1 : 0;
            want.mg_max_levels = mg->maxLevels;
            want.mg_weight = mg->weight;
        }
        if (b->nely == m.origResY && b->nelx == m.origResX && b->nelz == m.origResZ && same_params(b->prm, want))
            return b;
        const float rmin = b->filter_rmin;
        auto nb = create_binding(pb, m.origResY, m.origResX, m.origResZ, want);
        if (rmin != nb->filter_rmin) {
            check(t3d_filter_setup(nb->ctx, rmin), "t3d_filter_setup");
            nb->filter_rmin = rmin;
        }
        return nb;
    }
    return create_binding(pb, m.origResY, m.origResX, m.origResZ, params_of(pb, mg));
}

// A preconditioner made by make_diagonal_preconditioner_from_static: the V-cycle of the bound context
// with the hierarchy set up from moduli E.  When another preconditioner was set up on the same context
// since, it sets its own up again before use (the reference's closures each own their diagonals).
struct MgPreconditioner {
    std::shared_ptr<Binding> b;
    std::shared_ptr<const std::vector<double>> E;
    mutable uint64_t generation = 0;   // the set-up this closure made last
    void make_current() const {
        if (b->mg_generation == generation) return;
        check(t3d_mg_setup(b->ctx, E->data()), "t3d_mg_setup");
        generation = ++b->mg_generation;
    }
    void operator()(const std::vector<double>& r, std::vector<double>& z) const {
        make_current();
        z.resize(r.size());
        check(t3d_vcycle(b->ctx, r.data(), z.data()), "t3d_vcycle");
    }
};

void require_size(size_t got, int64_t want, const char* what) {
    if ((int64_t)got != want)
        throw std::runtime_error(std::string(what) + ": size " + std::to_string(got) + ", expected " +
                                 std::to_string(want));
}

}  // namespace

namespace top3d {

void InitialSettings(GlobalParams& out) { out = GlobalParams{}; }

std::array<double, 24 * 24> ComputeVoxelKe(double nu, double cellSize) {
    std::array<double, 24 * 24> Ke{};
    check(t3d_voxel_ke(nu, cellSize, Ke.data()), "t3d_voxel_ke");
    return Ke;
}

void CreateVoxelFEAmodel_Cuboid(Problem& pb, int nely, int nelx, int nelz) {
    std::shared_ptr<Binding> b;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        b = create_binding(pb, nely, nelx, nelz, params_of(pb, nullptr));
    }
    t3d_info inf;
    check(t3d_get_info(b->ctx, &inf), "t3d_get_info");
    auto& m = pb.mesh;
    m.resX = (int)inf.res[0];
    m.resY = (int)inf.res[1];
    m.resZ = (int)inf.res[2];
    m.origResX = nelx;
    m.origResY = nely;
    m.origResZ = nelz;
    m.numElements = (int)inf.num_elements;
    m.numNodes = (int)inf.num_nodes;
    m.numDOFs = 3 * m.numNodes;
    m.eleMapBack.resize(m.numElements);
    check(t3d_get_element_map(b->ctx, m.eleMapBack.data()), "t3d_get_element_map");
    check(t3d_get_ke(b->ctx, m.Ke.data()), "t3d_get_ke");
    pb.density.assign(m.numElements, 0.0f);
}

void ApplyBoundaryConditions(Problem& pb) {
    auto b = binding(pb);
    std::vector<int32_t> fd(b->nf);
    check(t3d_get_free_dofs(b->ctx, fd.data()), "t3d_get_free_dofs");
    pb.freeDofIndex.assign(fd.begin(), fd.end());
    pb.freeNodeIndex.resize(fd.size());
    pb.freeCompIndex.resize(fd.size());
    pb.isFreeDOF.assign((size_t)pb.mesh.numDOFs, 0);
    for (size_t i = 0; i < fd.size(); ++i) {
        pb.freeNodeIndex[i] = fd[i] / 3;
        pb.freeCompIndex[i] = fd[i] % 3;
        pb.isFreeDOF[(size_t)fd[i]] = 1;
    }
    std::vector<double> bf(b->nf);
    check(t3d_get_load(b->ctx, bf.data()), "t3d_get_load");
    for (auto* v : {&pb.F.ux, &pb.F.uy, &pb.F.uz}) v->assign((size_t)pb.mesh.numNodes, 0.0);
    scatter_from_free(pb, bf, pb.F);
}

void restrict_to_free(const Problem& pb, const DOFData& full, std::vector<double>& freev) {
    freev.resize(pb.freeDofIndex.size());
    for (size_t i = 0; i < pb.freeDofIndex.size(); ++i) {
        const int n = pb.freeDofIndex[i] / 3, c = pb.freeDofIndex[i] % 3;
        freev[i] = c == 0 ? full.ux[n] : (c == 1 ? full.uy[n] : full.uz[n]);
    }
}

void scatter_from_free(const Problem& pb, const std::vector<double>& freev, DOFData& full) {
    for (size_t i = 0; i < pb.freeDofIndex.size(); ++i) {
        const int n = pb.freeDofIndex[i] / 3, c = pb.freeDofIndex[i] % 3;
        (c == 0 ? full.ux : (c == 1 ? full.uy : full.uz))[n] = freev[i];
    }
}

void K_times_u_finest(const Problem& pb, const std::vector<double>& eleE, const std::vector<double>& uFree,
                      std::vector<double>& yFree) {
    auto b = binding(pb);
    require_size(eleE.size(), b->ne, "K_times_u_finest eleE");
    require_size(uFree.size(), b->nf, "K_times_u_finest uFree");
    yFree.resize(uFree.size());
    check(t3d_matvec(b->ctx, eleE.data(), uFree.data(), yFree.data()), "t3d_matvec");
}

void K_times_u_finest(const Problem& pb, const std::vector<double>& eleE, const std::vector<double>& uFree,
                      std::vector<double>& yFree, KTimesUWorkspace&) {
    K_times_u_finest(pb, eleE, uFree, yFree);
}

double ComputeCompliance(const Problem& pb, const std::vector<double>& eleE, const DOFData& U, std::vector<double>& ce) {
    auto b = binding(pb);
    require_size(eleE.size(), b->ne, "ComputeCompliance eleE");
    std::vector<double> u;
    restrict_to_free(pb, U, u);
    ce.resize((size_t)b->ne);
    double C = 0.0;
    check(t3d_compliance(b->ctx, eleE.data(), u.data(), ce.data(), &C), "t3d_compliance");
    return C;
}

Preconditioner make_jacobi_preconditioner(const Problem& pb, const std::vector<double>& eleE) {
    // the level-0 diagonal of the multigrid set-up is sum_e E_e Ke_ii (diagonal.cpp:11-60); restricted to
    // the free DOFs, entries <= 1e-30 become 1 (solver.cpp:65-69)
    auto b = binding(pb);
    require_size(eleE.size(), b->ne, "make_jacobi_preconditioner eleE");
    check(t3d_mg_setup(b->ctx, eleE.data()), "t3d_mg_setup");
    ++b->mg_generation;
    std::vector<double> full(3 * (size_t)b->nn);
    check(t3d_mg_get_diag(b->ctx, 0, full.data()), "t3d_mg_get_diag");
    std::vector<double> diag(pb.freeDofIndex.size());
    for (size_t i = 0; i < diag.size(); ++i) {
        const double d = full[(size_t)pb.freeDofIndex[i]];
        diag[i] = d > 1.0e-30 ? d : 1.0;
    }
    return [diag = std::move(diag)](const std::vector<double>& r, std::vector<double>& z) {
        z.resize(r.size());
        for (size_t i = 0; i < r.size(); ++i) z[i] = r[i] / diag[i];
    };
}

int PCG_free(const Problem& pb, const std::vector<double>& eleE, const std::vector<double>& bFree,
             std::vector<double>& xFree, double tol, int maxIt, const Preconditioner& M, PCGFreeWorkspace& ws) {
    auto b = binding(pb);
    require_size(bFree.size(), b->nf, "PCG_free bFree");
    if (xFree.empty()) xFree.assign(bFree.size(), 0.0);
    require_size(xFree.size(), b->nf, "PCG_free xFree");
    const MgPreconditioner* mg = M ? M.target<MgPreconditioner>() : nullptr;
    if (mg && mg->b == b) {   // the device-resident PCG with this context's V-cycle
        mg->make_current();
        int iters = 0;
        check(t3d_pcg(b->ctx, eleE.data(), bFree.data(), xFree.data(), tol, maxIt, &iters), "t3d_pcg");
        return iters;
    }
    // any other preconditioner (or none): PCG_free's iteration (solver.cpp:87-217) on the host around the
    // device K(E)p, the same recurrence and stopping test
    const size_t n = bFree.size();
    ws.r.resize(n);
    ws.z.resize(n);
    ws.p.resize(n);
    ws.Ap.resize(n);
    K_times_u_finest(pb, eleE, xFree, ws.Ap);
    for (size_t i = 0; i < n; ++i) ws.r[i] = bFree[i] - ws.Ap[i];
    if (M) M(ws.r, ws.z);
    else ws.z = ws.r;
    double rz = 0.0, nb2 = 0.0;
    for (size_t i = 0; i < n; ++i) {
        rz += ws.r[i] * ws.z[i];
        nb2 += bFree[i] * bFree[i];
    }
    ws.p = ws.z;
    const double stop = std::max(1.0e-30, std::sqrt(nb2)) * tol;
    for (int it = 0; it < maxIt; ++it) {
        K_times_u_finest(pb, eleE, ws.p, ws.Ap);
        double den = 0.0;
        for (size_t i = 0; i < n; ++i) den += ws.p[i] * ws.Ap[i];
        const double alpha = rz / std::max(1.0e-30, den);
        double rr = 0.0;
        for (size_t i = 0; i < n; ++i) {
            xFree[i] += alpha * ws.p[i];
            ws.r[i] -= alpha * ws.Ap[i];
            rr += ws.r[i] * ws.r[i];
        }
        if (std::sqrt(rr) < stop) return it + 1;
        if (M) M(ws.r, ws.z);
        else ws.z = ws.r;
        double rz_new = 0.0;
        for (size_t i = 0; i < n; ++i) rz_new += ws.r[i] * ws.z[i];
        const double beta = rz_new / std::max(1.0e-30, rz);
        rz = rz_new;
        for (size_t i = 0; i < n; ++i) ws.p[i] = ws.z[i] + beta * ws.p[i];
    }
    return maxIt;
}

namespace mg {

void BuildMGHierarchy(const Problem& pb, bool nonDyadic, MGHierarchy& H, int maxLevels) {
    MGPrecondConfig cfg;
    auto cur = binding(pb);
    cfg.weight = cur->prm.mg_weight;
    cfg.nonDyadic = nonDyadic;
    cfg.maxLevels = maxLevels;
    auto b = binding(pb, &cfg);
    t3d_info inf;
    check(t3d_get_info(b->ctx, &inf), "t3d_get_info");
    H.nonDyadic = nonDyadic;
    H.levels.assign((size_t)inf.num_levels, MGLevel{});
    for (int l = 0; l < (int)inf.num_levels; ++l) {
        MGLevel& L = H.levels[(size_t)l];
        L.resX = (int)inf.levels[l][0];
        L.resY = (int)inf.levels[l][1];
        L.resZ = (int)inf.levels[l][2];
        L.spanWidth = (int)inf.levels[l][3];
        L.numElements = L.resX * L.resY * L.resZ;
        L.numNodes = (L.resX + 1) * (L.resY + 1) * (L.resZ + 1);
        L.numDOFs = 3 * L.numNodes;
    }
}

void build_static_once(const Problem& pb, const MGPrecondConfig& cfg, MGHierarchy& H,
                       std::vector<std::vector<uint8_t>>& fixedMasks) {
    auto b = binding(pb, &cfg);
    BuildMGHierarchy(pb, cfg.nonDyadic, H, cfg.maxLevels);
    fixedMasks.assign(H.levels.size(), {});
    for (size_t l = 0; l < H.levels.size(); ++l) {
        fixedMasks[l].resize((size_t)H.levels[l].numDOFs);
        check(t3d_mg_get_mask(b->ctx, (int)l, fixedMasks[l].data()), "t3d_mg_get_mask");
    }
}

Preconditioner make_diagonal_preconditioner_from_static(const Problem& pb, const MGHierarchy&,
                                                        const std::vector<std::vector<uint8_t>>&,
                                                        const std::vector<double>& eleE, const MGPrecondConfig& cfg) {
    auto b = binding(pb, &cfg);
    require_size(eleE.size(), b->ne, "make_diagonal_preconditioner_from_static eleE");
    MgPreconditioner P;
    P.b = b;
    P.E = std::make_shared<const std::vector<double>>(eleE);
    check(t3d_mg_setup(b->ctx, eleE.data()), "t3d_mg_setup");
    P.generation = ++b->mg_generation;
    return P;
}

}  // namespace mg

PDEFilter SetupPDEFilter(const Problem& pb, float filterRadius) {
    auto b = binding(pb);
    check(t3d_filter_setup(b->ctx, filterRadius), "t3d_filter_setup");
    b->filter_rmin = filterRadius;
    PDEFilter f;
    f.diagPrecondNode.resize((size_t)b->nn);
    f.lastXNode.resize((size_t)b->nn);
    f.lastRhsNode.resize((size_t)b->nn);
    check(t3d_filter_get_state(b->ctx, f.lastXNode.data(), f.lastRhsNode.data(), f.diagPrecondNode.data()),
          "t3d_filter_get_state");
    return f;
}

void ApplyPDEFilter(const Problem& pb, PDEFilter& f, const std::vector<float>& src, std::vector<float>& dst,
                    PDEFilterWorkspace&) {
    auto b = binding(pb);
    require_size(src.size(), b->ne, "ApplyPDEFilter src");
    // the warm start travels in the PDEFilter, as in the reference (filter.cpp:175-275)
    if ((int64_t)f.lastXNode.size() == b->nn && (int64_t)f.lastRhsNode.size() == b->nn)
        check(t3d_filter_set_state(b->ctx, f.lastXNode.data(), f.lastRhsNode.data()), "t3d_filter_set_state");
    dst.resize(src.size());
    check(t3d_filter_apply(b->ctx, src.data(), dst.data()), "t3d_filter_apply");
    f.lastXNode.resize((size_t)b->nn);
    f.lastRhsNode.resize((size_t)b->nn);
    check(t3d_filter_get_state(b->ctx, f.lastXNode.data(), f.lastRhsNode.data(), nullptr), "t3d_filter_get_state");
}

// The reference driver (driver.cpp:23-280) with the whole design loop resident on the device: the same
// inputs block, solid-domain line, per-iteration "It.:" lines, summary, comments file and STL export.
void TOP3D_XL_GLOBAL(int nely, int nelx, int nelz, float V0, int nLoop, float rMin, int simulation_count) {
    const auto tAll = std::chrono::steady_clock::now();
    for (int sim = 0; sim < simulation_count; ++sim) {
        const auto tStartTotal = std::chrono::steady_clock::now();
        GlobalParams gp;
        InitialSettings(gp);
        std::cout << "\n==========================Displaying Inputs==========================\n";
        std::cout << "Simulation: " << sim << "\n";
        std::cout << std::fixed << std::setprecision(4);
        std::cout << "..............................................Volume Fraction: " << std::setw(6) << V0 << "\n";
        std::cout << "..........................................Filter Radius: " << std::setw(6) << rMin << " Cells\n";
        std::cout << std::scientific << std::setprecision(4);
        std::cout << "................................................Cell Size: " << std::setw(10) << gp.cellSize << "\n";
        std::cout << std::fixed;
        std::cout << ".................................................#CG Iterations: " << std::setw(4) << gp.cgMaxIt
                  << "\n";
        std::cout << std::scientific << std::setprecision(4);
        std::cout << "...........................................Youngs Modulus: " << std::setw(10) << gp.youngsModulus
                  << "\n";
        std::cout << "....................................Youngs Modulus (Min.): " << std::setw(10)
                  << gp.youngsModulusMin << "\n";
        std::cout << "...........................................Poissons Ratio: " << std::setw(10) << gp.poissonRatio
                  << "\n";
        std::cout << std::fixed << std::setprecision(6);

        auto tStart = std::chrono::steady_clock::now();
        t3d_params p;
        check(t3d_params_default(&p), "t3d_params_default");
        p.E0 = gp.youngsModulus;
        p.Emin = gp.youngsModulusMin;
        p.penal = gp.simpPenalty;
        p.cg_tol = gp.cgTol;
        p.cg_max_it = gp.cgMaxIt;
        p.mg_nondyadic = 1;      // driver.cpp:54
        p.mg_max_levels = 5;
        p.mg_weight = 0.6f;
        p.filter_rmin = rMin;
        p.device = env_int("T3D_DEVICE", 0);
        const char* prec = std::getenv("T3D_PRECISION");
        p.precision = (prec && std::string(prec) == "mixed") ? T3D_MIXED : T3D_FP64;
        std::cout << "Building Multigrid Hierarchy..." << std::endl;
        t3d_context* ctx = nullptr;
        check(t3d_create(nely, nelx, nelz, &p, &ctx), "t3d_create");
        std::unique_ptr<t3d_context, int (*)(t3d_context*)> own(ctx, t3d_destroy);
        t3d_info inf;
        check(t3d_get_info(ctx, &inf), "t3d_get_info");
        const float tModel = std::chrono::duration<float>(std::chrono::steady_clock::now() - tStart).count();
        std::cout << "Preparing Voxel-based FEA Model Costs " << std::setw(10) << std::setprecision(1) << tModel << "s\n";

        tStart = std::chrono::steady_clock::now();
        double Csolid = 0.0;
        check(t3d_design_init(ctx, V0, &Csolid), "t3d_design_init");
        const float tSolid = std::chrono::duration<float>(std::chrono::steady_clock::now() - tStart).count();
        std::cout << std::scientific << std::setprecision(6);
        std::cout << "Compliance of Fully Solid Domain: " << std::setw(16) << Csolid << "\n";
        std::cout << std::fixed;
        std::cout << " It.: " << std::setw(4) << 0 << " Solver Time: " << std::setw(4) << std::setprecision(0) << tSolid
                  << "s.\n\n";
        std::cout << std::setprecision(6);

        int loop = 0;
        float change = 1.0f, sharpness = 1.0f;
        float sumCG = 0.0f, sumOpt = 0.0f, sumFilter = 0.0f, sumIter = 0.0f, objFirst = 0.0f, objLast = 0.0f;
        while (loop < nLoop && change > 1e-4 && sharpness > 0.01) {
            t3d_iter_record r;
            check(t3d_design_step(ctx, &r), "t3d_design_step");
            loop = r.loop;
            change = r.change;
            sharpness = r.sharp;
            if (loop == 1) objFirst = (float)r.obj;
            objLast = (float)r.obj;
            sumCG += (float)r.t_cg;
            sumOpt += (float)r.t_opt;
            sumFilter += (float)r.t_filter;
            sumIter += (float)r.t_total;
            std::cout << std::scientific << std::setprecision(8);
            std::cout << " It.:" << std::setw(4) << loop << " Obj.:" << std::setw(16) << r.obj << " Vol.:" << std::setw(6)
                      << std::setprecision(4) << r.vol << " Sharp.:" << std::setw(6) << r.sharp << " Cons.:" << std::setw(4)
                      << std::setprecision(2) << r.cons << " Ch.:" << std::setw(4) << r.change << "\n";
            std::cout << std::fixed << std::setprecision(2);
            std::cout << " It.: " << std::setw(4) << loop << " (Time)... Total per-It.: " << std::setw(8)
                      << std::scientific << (float)r.t_total << "s;"
                      << " CG: " << std::setw(8) << (float)r.t_cg << "s;"
                      << " Opti.: " << std::setw(8) << (float)r.t_opt << "s;"
                      << " Filtering: " << std::setw(8) << (float)r.t_filter << "s.\n";
            std::cout << std::fixed;
        }
        const float tTotal = std::chrono::duration<float>(std::chrono::steady_clock::now() - tStartTotal).count();
        std::cout << "\n..........Performing Topology Optimization Costs (in total): " << std::scientific
                  << std::setprecision(4) << tTotal << "s.\n";
        std::cout << std::fixed;

        const float avg = loop > 0 ? sumIter / (float)loop : 0.0f;
        std::ostringstream s;
        s << "PARAMETERS\n"
          << "original dims: x=" << nelx << ", y=" << nely << ", z=" << nelz << "\n"
          << "padded dims: x=" << inf.res[0] << ", y=" << inf.res[1] << ", z=" << inf.res[2] << "\n"
          << "v0: " << V0 << "\n\n"
          << "SOLVING\n"
          << "iterations: " << loop << "\n"
          << "cg iterations: " << gp.cgMaxIt << "\n\n"
          << "RESULTS\n"
          << "compliance solid: " << std::scientific << std::setprecision(6) << Csolid << "\n"
          << "objective first: " << objFirst << "\n"
          << "objective last: " << objLast << "\n\n"
          << "TIME\n"
          << "total solver time: " << sumCG << "\n"
          << "time per iter: " << std::fixed << std::setprecision(4) << avg << "\n"
          << "percentage time spent on cg: " << std::setprecision(2) << (sumIter > 0 ? 100.0f * sumCG / sumIter : 0.0f)
          << "%\n"
          << "percentage time spent on optim: " << (sumIter > 0 ? 100.0f * sumOpt / sumIter : 0.0f) << "%\n"
          << "percentage time spent on filtering: " << (sumIter > 0 ? 100.0f * sumFilter / sumIter : 0.0f) << "%\n\n"
          << "DEVICE\n"
          << "GPU " << p.device << (p.precision == T3D_MIXED ? " (mixed precision)" : " (FP64)") << "\n\n"
          << "NOTES\n";
        std::cout << "\n" << s.str() << std::endl;

        // out/ next to the working directory, as the reference's io.cpp:23-46 chooses it
        namespace fs = std::filesystem;
        std::error_code ec;
        fs::path out = fs::current_path(ec) / "out";
        if (!fs::exists(out, ec) && fs::exists(fs::current_path(ec).parent_path() / "out", ec))
            out = fs::current_path(ec).parent_path() / "out";
        const std::time_t now = std::time(nullptr);
        char stamp[32];
        std::strftime(stamp, sizeof stamp, "%Y%m%d_%H%M%S", std::localtime(&now));
        std::string tag = std::string("GLOBAL_") + stamp;
        if (const char* job = std::getenv("SLURM_JOB_ID"))
            if (*job) tag += std::string("_") + job;
        fs::create_directories(out / "comments", ec);
        fs::create_directories(out / "stl", ec);
        std::ofstream((out / "comments" / (tag + ".md")).string()) << s.str();
        const std::string stl = (out / "stl" / (tag + ".stl")).string();
        int64_t ntri = 0;
        check(t3d_export_stl(ctx, nullptr, 0.3f, stl.c_str(), &ntri), "t3d_export_stl");
        std::cout << "STL file saved to: " << stl << "\n";
        std::cout << "\nDone.\n";
    }
    const float fin = std::chrono::duration<float>(std::chrono::steady_clock::now() - tAll).count();
    std::cout << "\n............Total runtime time for " << simulation_count << " simulations" << std::scientific
              << std::setprecision(4) << fin << "s.\n";
}

}  // namespace top3d
