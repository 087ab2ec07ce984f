// Test infrastructure only: a harness around the UNMODIFIED reference sources
// (natashahirt/AlgorithmEngineering_AltProject, cpp/src/*.cpp, cpp/src/multigrid/*.cpp).
//
// It is linked by oracle/Makefile into oracle/_ref/libt3d_ref.so together with the
// reference's own objects.  Nothing in the product links it; tests/, the smoke check
// and bench.py's CPU-baseline leg are its only users.
//
// Two kinds of entry points:
//  1. single-call wrappers around the reference's public operator API
//     (fea.hpp:37-47, solver.hpp:8-27, multigrid/multigrid.hpp:64-68, filter.hpp:17-28),
//     used to pin the C restatement in oracle/t3d_oracle.c and to produce golden vectors;
//  2. a capture run of the reference driver TOP3D_XL_GLOBAL (driver.cpp:23-280): the
//     driver's calls to PCG_free, ComputeCompliance, ApplyPDEFilter,
//     make_diagonal_preconditioner_from_static and export_surface_stl are routed through
//     `ld --wrap` shims below that record their inputs/outputs as raw binary files and
//     then call the real reference function.  The driver source itself is untouched.
#include "core.hpp"
#include "fea.hpp"
#include "solver.hpp"
#include "filter.hpp"
#include "driver.hpp"
#include "multigrid/multigrid.hpp"
#include "multigrid/detail/diagonal.hpp"
#include "multigrid/detail/coarsest.hpp"
#include "multigrid/detail/transfers.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <numeric>
#include <cstring>
#include <string>
#include <vector>
#include <memory>
#if defined(_OPENMP)
#include <omp.h>
#endif

using namespace top3d;

namespace {

struct RefCtx {
    Problem pb;
    // design state of ref_sample_iteration (driver.cpp:60-84 initialisation)
    std::vector<float> x;
    std::vector<double> uWarm, bFree;
    bool sampleReady = false;
    mg::MGPrecondConfig cfg;
    mg::MGHierarchy H;
    std::vector<std::vector<uint8_t>> masks;
    Preconditioner M;
    PCGFreeWorkspace pws;
    PDEFilter pf;
    PDEFilterWorkspace fws;
    bool filterReady = false;
};

template <class T>
void write_bin(const std::string& path, const T* p, size_t n) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return;
    std::fwrite(p, sizeof(T), n, f);
    std::fclose(f);
}

std::string g_capdir;
int g_pcg_calls = 0, g_cc_calls = 0, g_filt_calls = 0, g_prec_calls = 0;

std::string cap_path(const char* kind, int idx, const char* field) {
    char buf[256];
    std::snprintf(buf, sizeof buf, "%s/%s_%03d_%s.bin", g_capdir.c_str(), kind, idx, field);
    return std::string(buf);
}

}  // namespace

// ---------------------------------------------------------------- capture shims
// Symbol names are the Itanium-mangled names of the reference functions; `ld --wrap=SYM`
// sends the driver's calls to __wrap_SYM and makes __real_SYM the original.

int real_pcg(const Problem&, const std::vector<double>&, const std::vector<double>&, std::vector<double>&,
             double, int, const Preconditioner&, PCGFreeWorkspace&)
    __asm__("__real__ZN5top3d8PCG_freeERKNS_7ProblemERKSt6vectorIdSaIdEES7_RS5_diRKSt8functionIFvS7_S8_EERNS_16PCGFreeWorkspaceE");
int wrap_pcg(const Problem&, const std::vector<double>&, const std::vector<double>&, std::vector<double>&,
             double, int, const Preconditioner&, PCGFreeWorkspace&)
    __asm__("__wrap__ZN5top3d8PCG_freeERKNS_7ProblemERKSt6vectorIdSaIdEES7_RS5_diRKSt8functionIFvS7_S8_EERNS_16PCGFreeWorkspaceE");

int wrap_pcg(const Problem& pb, const std::vector<double>& E, const std::vector<double>& b,
             std::vector<double>& x, double tol, int maxIt, const Preconditioner& M, PCGFreeWorkspace& ws) {
    const int k = g_pcg_calls++;
    if (!g_capdir.empty()) {
        write_bin(cap_path("pcg", k, "E"), E.data(), E.size());
        write_bin(cap_path("pcg", k, "x0"), x.data(), x.size());
    }
    int it = real_pcg(pb, E, b, x, tol, maxIt, M, ws);
    if (!g_capdir.empty()) {
        write_bin(cap_path("pcg", k, "x1"), x.data(), x.size());
        int32_t v = it;
        write_bin(cap_path("pcg", k, "iters"), &v, 1);
    }
    return it;
}

double real_cc(const Problem&, const std::vector<double>&, const DOFData&, std::vector<double>&)
    __asm__("__real__ZN5top3d17ComputeComplianceERKNS_7ProblemERKSt6vectorIdSaIdEERKNS_7DOFDataERS5_");
double wrap_cc(const Problem&, const std::vector<double>&, const DOFData&, std::vector<double>&)
    __asm__("__wrap__ZN5top3d17ComputeComplianceERKNS_7ProblemERKSt6vectorIdSaIdEERKNS_7DOFDataERS5_");

double wrap_cc(const Problem& pb, const std::vector<double>& E, const DOFData& U, std::vector<double>& ce) {
    const int k = g_cc_calls++;
    double C = real_cc(pb, E, U, ce);
    if (!g_capdir.empty()) {
        write_bin(cap_path("cc", k, "ce"), ce.data(), ce.size());
        write_bin(cap_path("cc", k, "C"), &C, 1);
    }
    return C;
}

void real_filt(const Problem&, PDEFilter&, const std::vector<float>&, std::vector<float>&, PDEFilterWorkspace&)
    __asm__("__real__ZN5top3d14ApplyPDEFilterERKNS_7ProblemERNS_9PDEFilterERKSt6vectorIfSaIfEERS7_RNS_18PDEFilterWorkspaceE");
void wrap_filt(const Problem&, PDEFilter&, const std::vector<float>&, std::vector<float>&, PDEFilterWorkspace&)
    __asm__("__wrap__ZN5top3d14ApplyPDEFilterERKNS_7ProblemERNS_9PDEFilterERKSt6vectorIfSaIfEERS7_RNS_18PDEFilterWorkspaceE");

void wrap_filt(const Problem& pb, PDEFilter& pf, const std::vector<float>& src, std::vector<float>& dst,
               PDEFilterWorkspace& ws) {
    const int k = g_filt_calls++;
    if (!g_capdir.empty()) {
        write_bin(cap_path("filt", k, "src"), src.data(), src.size());
        write_bin(cap_path("filt", k, "lastx0"), pf.lastXNode.data(), pf.lastXNode.size());
        write_bin(cap_path("filt", k, "lastrhs0"), pf.lastRhsNode.data(), pf.lastRhsNode.size());
    }
    real_filt(pb, pf, src, dst, ws);
    if (!g_capdir.empty()) {
        write_bin(cap_path("filt", k, "dst"), dst.data(), dst.size());
    }
}

Preconditioner real_prec(const Problem&, const mg::MGHierarchy&, const std::vector<std::vector<uint8_t>>&,
                         const std::vector<double>&, const mg::MGPrecondConfig&)
    __asm__("__real__ZN5top3d2mg40make_diagonal_preconditioner_from_staticERKNS_7ProblemERKNS0_11MGHierarchyERKSt6vectorIS7_IhSaIhEESaIS9_EERKS7_IdSaIdEERKNS0_15MGPrecondConfigE");
Preconditioner wrap_prec(const Problem&, const mg::MGHierarchy&, const std::vector<std::vector<uint8_t>>&,
                         const std::vector<double>&, const mg::MGPrecondConfig&)
    __asm__("__wrap__ZN5top3d2mg40make_diagonal_preconditioner_from_staticERKNS_7ProblemERKNS0_11MGHierarchyERKSt6vectorIS7_IhSaIhEESaIS9_EERKS7_IdSaIdEERKNS0_15MGPrecondConfigE");

Preconditioner wrap_prec(const Problem& pb, const mg::MGHierarchy& H, const std::vector<std::vector<uint8_t>>& m,
                         const std::vector<double>& E, const mg::MGPrecondConfig& cfg) {
    const int k = g_prec_calls++;
    if (!g_capdir.empty()) {
        int32_t v = g_pcg_calls;  // index of the PCG call that will first use this preconditioner
        write_bin(cap_path("prec", k, "first_pcg"), &v, 1);
    }
    return real_prec(pb, H, m, E, cfg);
}

void real_stl(const Problem&, const std::vector<float>&, const std::string&, float)
    __asm__("__real__ZN5top3d18export_surface_stlERKNS_7ProblemERKSt6vectorIfSaIfEERKNSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEEf");
void wrap_stl(const Problem&, const std::vector<float>&, const std::string&, float)
    __asm__("__wrap__ZN5top3d18export_surface_stlERKNS_7ProblemERKSt6vectorIfSaIfEERKNSt7__cxx1112basic_stringIcSt11char_traitsIcESaIcEEEf");

void wrap_stl(const Problem& pb, const std::vector<float>& xPhys, const std::string& path, float iso) {
    (void)path; (void)iso;
    if (!g_capdir.empty()) write_bin(g_capdir + "/xphys_final.bin", xPhys.data(), xPhys.size());
    // the STL file itself is not written: the capture run only records the design
    (void)pb;
}

// ---------------------------------------------------------------- C entry points
extern "C" {

void ref_set_threads(int n) {
#if defined(_OPENMP)
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int ref_max_threads(void) {
#if defined(_OPENMP)
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Run the reference driver TOP3D_XL_GLOBAL once with capture into `capdir` ("" = no capture).
void ref_run_global(int nely, int nelx, int nelz, float V0, int nLoop, float rMin, const char* capdir) {
    g_capdir = capdir ? capdir : "";
    g_pcg_calls = g_cc_calls = g_filt_calls = g_prec_calls = 0;
    TOP3D_XL_GLOBAL(nely, nelx, nelz, V0, nLoop, rMin, 1);
    g_capdir.clear();
}

// Build the cuboid model exactly as the driver does (driver.cpp:47-55) with an optional
// Emin override and MG level cap.
void* ref_create(int nely, int nelx, int nelz, int maxLevels, float emin) {
    auto* c = new RefCtx();
    InitialSettings(c->pb.params);
    if (emin > 0.f) c->pb.params.youngsModulusMin = emin;
    CreateVoxelFEAmodel_Cuboid(c->pb, nely, nelx, nelz);
    ApplyBoundaryConditions(c->pb);
    c->cfg.nonDyadic = true;
    c->cfg.maxLevels = maxLevels > 0 ? maxLevels : 5;
    c->cfg.weight = 0.6f;
    mg::build_static_once(c->pb, c->cfg, c->H, c->masks);
    return c;
}

void ref_destroy(void* h) { delete static_cast<RefCtx*>(h); }

// info[0..]: resX,resY,resZ, numElements, numNodes, nFree, nLevels, then per level (resX,resY,resZ,span)
void ref_info(void* h, int64_t* info) {
    auto* c = static_cast<RefCtx*>(h);
    const auto& m = c->pb.mesh;
    info[0] = m.resX; info[1] = m.resY; info[2] = m.resZ;
    info[3] = m.numElements; info[4] = m.numNodes; info[5] = (int64_t)c->pb.freeDofIndex.size();
    info[6] = (int64_t)c->H.levels.size();
    for (size_t l = 0; l < c->H.levels.size() && l < 8; ++l) {
        info[7 + 4 * l + 0] = c->H.levels[l].resX;
        info[7 + 4 * l + 1] = c->H.levels[l].resY;
        info[7 + 4 * l + 2] = c->H.levels[l].resZ;
        info[7 + 4 * l + 3] = c->H.levels[l].spanWidth;
    }
}

void ref_ele_map_back(void* h, int32_t* out) {
    auto* c = static_cast<RefCtx*>(h);
    std::memcpy(out, c->pb.mesh.eleMapBack.data(), c->pb.mesh.eleMapBack.size() * 4);
}

void ref_free_dofs(void* h, int32_t* out) {
    auto* c = static_cast<RefCtx*>(h);
    for (size_t i = 0; i < c->pb.freeDofIndex.size(); ++i) out[i] = c->pb.freeDofIndex[i];
}

void ref_bfree(void* h, double* out) {
    auto* c = static_cast<RefCtx*>(h);
    std::vector<double> b;
    restrict_to_free(c->pb, c->pb.F, b);
    std::memcpy(out, b.data(), b.size() * 8);
}

void ref_ke(void* h, double* out) {
    auto* c = static_cast<RefCtx*>(h);
    std::memcpy(out, c->pb.mesh.Ke.data(), 576 * 8);
}

void ref_matvec(void* h, const double* E, const double* u, double* y) {
    auto* c = static_cast<RefCtx*>(h);
    const size_t ne = c->pb.mesh.numElements, nf = c->pb.freeDofIndex.size();
    std::vector<double> Ev(E, E + ne), uv(u, u + nf), yv;
    K_times_u_finest(c->pb, Ev, uv, yv);
    std::memcpy(y, yv.data(), nf * 8);
}

// make_diagonal_preconditioner_from_static for the given moduli (multigrid.hpp:66-68)
void ref_mg_build(void* h, const double* E) {
    auto* c = static_cast<RefCtx*>(h);
    std::vector<double> Ev(E, E + c->pb.mesh.numElements);
    c->M = mg::make_diagonal_preconditioner_from_static(c->pb, c->H, c->masks, Ev, c->cfg);
}

void ref_vcycle(void* h, const double* r, double* z) {
    auto* c = static_cast<RefCtx*>(h);
    const size_t nf = c->pb.freeDofIndex.size();
    std::vector<double> rv(r, r + nf), zv(nf, 0.0);
    c->M(rv, zv);
    std::memcpy(z, zv.data(), nf * 8);
}

int ref_pcg(void* h, const double* E, const double* b, double* x, double tol, int maxIt) {
    auto* c = static_cast<RefCtx*>(h);
    const size_t ne = c->pb.mesh.numElements, nf = c->pb.freeDofIndex.size();
    std::vector<double> Ev(E, E + ne), bv(b, b + nf), xv(x, x + nf);
    int it = PCG_free(c->pb, Ev, bv, xv, tol, maxIt, c->M, c->pws);
    std::memcpy(x, xv.data(), nf * 8);
    return it;
}

double ref_compliance(void* h, const double* E, const double* uFree, double* ce) {
    auto* c = static_cast<RefCtx*>(h);
    const size_t ne = c->pb.mesh.numElements, nf = c->pb.freeDofIndex.size();
    std::vector<double> Ev(E, E + ne), uv(uFree, uFree + nf), cev;
    DOFData U;
    U.ux.assign(c->pb.mesh.numNodes, 0.0);
    U.uy.assign(c->pb.mesh.numNodes, 0.0);
    U.uz.assign(c->pb.mesh.numNodes, 0.0);
    scatter_from_free(c->pb, uv, U);
    double C = ComputeCompliance(c->pb, Ev, U, cev);
    std::memcpy(ce, cev.data(), ne * 8);
    return C;
}

// Per-level Jacobi diagonals (MG_BuildDiagonals, diagonal.cpp:140-160), interleaved 3n+c.
void ref_mg_diag(void* h, const double* E, int level, double* out) {
    auto* c = static_cast<RefCtx*>(h);
    std::vector<double> Ev(E, E + c->pb.mesh.numElements);
    std::vector<std::vector<double>> d;
    mg::MG_BuildDiagonals(c->pb, c->H, c->masks, Ev, d);
    std::memcpy(out, d[level].data(), d[level].size() * 8);
}

void ref_mg_mask(void* h, int level, uint8_t* out) {
    auto* c = static_cast<RefCtx*>(h);
    std::memcpy(out, c->masks[level].data(), c->masks[level].size());
}

// Coarsest Galerkin matrix (lower triangle + BC identity rows, preconditioner.cpp:56-73),
// before factorisation.  Returns N (0 when the reference would use the Jacobi fallback).
int ref_coarse_matrix(void* h, const double* E, double* out) {
    auto* c = static_cast<RefCtx*>(h);
    const auto& Lc = c->H.levels.back();
    int N = 3 * Lc.numNodes;
    if (c->H.levels.size() == 1 || N > 1000) return 0;
    std::vector<double> Ev(E, E + c->pb.mesh.numElements), full, Kc;
    mg::EleMod_CompactToFull_Finest(c->pb, Ev, full);
    mg::MG_AssembleCoarsestDenseK_Galerkin(c->pb, c->H, full, c->masks.front(), Kc);
    for (int n = 0; n < Lc.numNodes; n++)
        for (int cc = 0; cc < 3; cc++)
            if (c->masks.back()[3 * n + cc]) {
                int d = 3 * n + cc;
                for (int j = 0; j < N; j++) { Kc[d * N + j] = 0.0; Kc[j * N + d] = 0.0; }
                Kc[d * N + d] = 1.0;
            }
    std::memcpy(out, Kc.data(), (size_t)N * N * 8);
    return N;
}

void ref_filter_setup(void* h, float rMin) {
    auto* c = static_cast<RefCtx*>(h);
    c->pf = SetupPDEFilter(c->pb, rMin);
    c->filterReady = true;
}

void ref_filter_apply(void* h, const float* src, float* dst) {
    auto* c = static_cast<RefCtx*>(h);
    const size_t ne = c->pb.mesh.numElements;
    std::vector<float> s(src, src + ne), d;
    ApplyPDEFilter(c->pb, c->pf, s, d, c->fws);
    std::memcpy(dst, d.data(), ne * 4);
}

// lastX / lastRhs warm-start state and the inverse row-sum preconditioner (numNodes each)
void ref_filter_state(void* h, double* lastx, double* lastrhs, double* diag) {
    auto* c = static_cast<RefCtx*>(h);
    const size_t nn = c->pb.mesh.numNodes;
    if (lastx) std::memcpy(lastx, c->pf.lastXNode.data(), nn * 8);
    if (lastrhs) std::memcpy(lastrhs, c->pf.lastRhsNode.data(), nn * 8);
    if (diag) std::memcpy(diag, c->pf.diagPrecondNode.data(), nn * 8);
}

void ref_filter_set_state(void* h, const double* lastx, const double* lastrhs) {
    auto* c = static_cast<RefCtx*>(h);
    const size_t nn = c->pb.mesh.numNodes;
    c->pf.lastXNode.assign(lastx, lastx + nn);
    c->pf.lastRhsNode.assign(lastrhs, lastrhs + nn);
}

// One design iteration of the reference (driver.cpp:115-189) with PCG capped at pcg_max
// iterations, for bounded CPU-baseline samples: the reference's own PCG_free, ComputeCompliance,
// make_diagonal_preconditioner_from_static and ApplyPDEFilter, with the driver's inline SIMP,
// sensitivity and OC loops restated here and compiled with the reference's flags.
// times[0..5] = seconds in SIMP, MG rebuild, PCG, compliance+sensitivities, filter, OC;
// returns the PCG iteration count.
int ref_sample_iteration(void* h, float V0, int pcg_max, int rebuild_mg, double* times) {
    auto* c = static_cast<RefCtx*>(h);
    using clk = std::chrono::steady_clock;
    auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
    const int ne = c->pb.mesh.numElements;
    if (!c->sampleReady) {
        c->x.assign(ne, V0);
        restrict_to_free(c->pb, c->pb.F, c->bFree);
        c->uWarm.assign(c->bFree.size(), 0.0);
        if (!c->filterReady) { c->pf = SetupPDEFilter(c->pb, std::sqrt(3.0f)); c->filterReady = true; }
        c->sampleReady = true;
    }
    const auto& P = c->pb.params;
    std::vector<double> E(ne), ce;
    auto t0 = clk::now();
    for (int e = 0; e < ne; e++) {
        float rho = std::clamp(c->x[e], 0.0f, 1.0f);
        float powp = static_cast<float>(std::pow(rho, P.simpPenalty));
        E[e] = P.youngsModulusMin + powp * (P.youngsModulus - P.youngsModulusMin);
    }
    auto t1 = clk::now();
    if (rebuild_mg || !c->M) c->M = mg::make_diagonal_preconditioner_from_static(c->pb, c->H, c->masks, E, c->cfg);
    auto t2 = clk::now();
    int it = PCG_free(c->pb, E, c->bFree, c->uWarm, P.cgTol, pcg_max, c->M, c->pws);
    auto t3 = clk::now();
    DOFData U;
    U.ux.assign(c->pb.mesh.numNodes, 0.0); U.uy.assign(c->pb.mesh.numNodes, 0.0); U.uz.assign(c->pb.mesh.numNodes, 0.0);
    scatter_from_free(c->pb, c->uWarm, U);
    double C = ComputeCompliance(c->pb, E, U, ce);
    std::vector<float> dc(ne), xdc(ne), dcf;
    for (int e = 0; e < ne; e++) {
        float rho = std::clamp(c->x[e], 0.0f, 1.0f);
        float dEdrho = P.simpPenalty * static_cast<float>(std::pow(rho, P.simpPenalty - 1.0f)) *
                       (P.youngsModulus - P.youngsModulusMin);
        dc[e] = -dEdrho * static_cast<float>(ce[e] / C);
        xdc[e] = c->x[e] * dc[e];
    }
    auto t4 = clk::now();
    ApplyPDEFilter(c->pb, c->pf, xdc, dcf, c->fws);
    auto t5 = clk::now();
    for (int e = 0; e < ne; e++) dc[e] = dcf[e] / std::max(1.0e-3f, c->x[e]);
    float l1 = 0.0f, l2 = 1e9f, move = 0.2f;
    std::vector<float> xnew(ne);
    while ((l2 - l1) / (l1 + l2) > 1e-6) {
        float lmid = 0.5f * (l1 + l2);
        for (int e = 0; e < ne; e++) {
            float val = std::sqrt(std::max(1e-30f, -dc[e] / lmid));
            float xe = std::clamp(c->x[e] * val, c->x[e] - move, c->x[e] + move);
            xe = std::clamp(xe, 0.0f, 1.0f);
            xnew[e] = std::max(1.0e-3f, xe);
        }
        float vol = std::accumulate(xnew.begin(), xnew.end(), 0.0f, [](float s, float v) { return s + v; }) /
                    static_cast<float>(ne);
        if (vol - V0 > 0) l1 = lmid; else l2 = lmid;
    }
    c->x.swap(xnew);
    auto t6 = clk::now();
    times[0] = secs(t0, t1); times[1] = secs(t1, t2); times[2] = secs(t2, t3);
    times[3] = secs(t3, t4); times[4] = secs(t4, t5); times[5] = secs(t5, t6);
    return it;
}

// The reference's own surface export (io.cpp:80-87) of densities in Morton order, written to `path`.
int ref_export_stl(void* h, const float* xphys, const char* path, float iso) {
    RefCtx* c = static_cast<RefCtx*>(h);
    std::vector<float> x(xphys, xphys + c->pb.mesh.numElements);
    real_stl(c->pb, x, std::string(path), iso);
    return 0;
}

}  // extern "C"
