// Host runtime of the B200 library: one context = one cantilever design on one GPU.  Owns every
// device buffer (allocated once at creation, none afterwards on the design-loop path), orchestrates
// the kernels of the design iteration on one stream, captures the PCG iteration in CUDA graphs and
// implements the C-ABI declared in include/t3d_b200.h.
#include "t3d_b200.h"
#include "hex8.hpp"
#include "kernels.hpp"
#include "topvoxel.hpp"
#include "context.hpp"

#include <algorithm>
#include <cmath>
#include <memory>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace t3d {

namespace {
thread_local std::string g_err;
}

int set_error(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

int set_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof buf, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    g_err = buf;
    return e == cudaErrorMemoryAllocation ? T3D_ERR_OOM : T3D_ERR_CUDA;
}

// ------------------------------------------------------------------ host-side model constants
// (the hex8 element stiffness is in hex8.hpp)

// PDE-filter 8x8 kernel r^2 KEF0 + KEF1 (filter.cpp:11-54) followed by its 8 row sums (:56-62)
static void filter_kernel(float rmin, double* kf) {
    static const double sg[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    static const double tg[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    static const double pg[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    double N[8][8], dS[24][8];
    for (int g = 0; g < 8; ++g) {
        const double s = sg[g] / std::sqrt(3.0), t = tg[g] / std::sqrt(3.0), q = pg[g] / std::sqrt(3.0);
        for (int a = 0; a < 8; ++a) {
            N[g][a] = 0.125 * (1 + sg[a] * s) * (1 + tg[a] * t) * (1 + pg[a] * q);
            dS[3 * g + 0][a] = 0.125 * sg[a] * (1 + tg[a] * t) * (1 + pg[a] * q);
            dS[3 * g + 1][a] = 0.125 * tg[a] * (1 + sg[a] * s) * (1 + pg[a] * q);
            dS[3 * g + 2][a] = 0.125 * pg[a] * (1 + sg[a] * s) * (1 + tg[a] * t);
        }
    }
    const double rr = ((double)rmin * 1.0) / (2.0 * std::sqrt(3.0));
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) {
            double k0 = 0.0, k1 = 0.0;
            for (int k = 0; k < 24; ++k) k0 += dS[k][i] * dS[k][j];
            for (int g = 0; g < 8; ++g) k1 += N[g][i] * (1.0 / 8.0) * N[g][j];
            kf[i * 8 + j] = rr * rr * k0 + k1;
        }
    for (int a = 0; a < 8; ++a) {
        double s = 0.0;
        for (int b = 0; b < 8; ++b) s += kf[a * 8 + b];
        kf[64 + a] = s;
    }
}

static int pad_levels(uint64_t nvox) {   // padding.hpp:23-33
    int L = 0;
    while (nvox >= 50000u) { ++L; nvox = (nvox + 4u) / 8u; }
    return L < 3 ? 3 : L;
}
static int pad_dim(int n, int L) {
    const int s = 1 << L;
    return ((n + s - 1) / s) * s;
}


static int update_ke_pattern(Context* c);

// W^T Ke W for the child positions of the first coarsening (the 'Standard' V-cycle's level-1 Galerkin)
static int upload_gpos(Context* c) {
    const int s1 = c->lv[1].span;
    std::vector<double> G((size_t)s1 * s1 * s1 * 576);
    galerkin_positions(s1, c->Ke_h, G.data());
    T3D_CUDA_OK(cudaMemcpy(c->Gpos, G.data(), G.size() * sizeof(double), cudaMemcpyHostToDevice));
    return T3D_OK;
}

int launch_check(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error(e, what, __FILE__, __LINE__);
    return T3D_OK;
}

int sync(Context* c) {
    T3D_CUDA_OK(cudaStreamSynchronize(c->st));
    return T3D_OK;
}

// ------------------------------------------------------------------ creation
static int build_levels(Context* c) {
    // hierarchy.cpp:84-138: span 4 first (non-dyadic), then 2, exact divisibility, stop at min dim <= 2
    int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
    c->nlev = 0;
    MgLevel& L0 = c->lv[c->nlev++];
    L0.nx = nx; L0.ny = ny; L0.nz = nz; L0.span = 1;
    for (int li = 1; li < c->prm.mg_max_levels && li < 8; ++li) {
        const int s = (li == 1 && c->prm.mg_nondyadic) ? 4 : 2;
        if (nx % s || ny % s || nz % s) break;
        if (nx / s < 1 || ny / s < 1 || nz / s < 1) break;
        nx /= s; ny /= s; nz /= s;
        MgLevel& L = c->lv[c->nlev++];
        L.nx = nx; L.ny = ny; L.nz = nz; L.span = s;
        if (std::min(nx, std::min(ny, nz)) <= 2) break;
    }
    if (c->nlev < 2) return set_error(T3D_ERR_UNSUPPORTED, "grid admits no coarse multigrid level");
    for (int l = 0; l < c->nlev; ++l) {
        MgLevel& L = c->lv[l];
        L.nn = (int64_t)(L.nx + 1) * (L.ny + 1) * (L.nz + 1);
        CHECK(c->alloc(&L.diag, 3 * L.nn));
        if (l == 0) L.mask = c->mask0;
        else {
            CHECK(c->alloc(&L.mask, L.nn));
            CHECK(c->alloc(&L.r, 3 * L.nn));
            CHECK(c->alloc(&L.x, 3 * L.nn));
        }
    }
    const int N = (int)(3 * c->lv[c->nlev - 1].nn);
    c->Nc = (N <= 1000) ? N : 0;   // NlimitDofs (preconditioner.cpp:52-54)
    if (c->Nc) {
        const MgLevel& Lc = c->lv[c->nlev - 1];
        CHECK(c->alloc(&c->Kce, (size_t)Lc.nx * Lc.ny * Lc.nz * 576));
        CHECK(c->alloc(&c->Kc, (size_t)N * N));
        CHECK(c->alloc(&c->LT, (size_t)N * N));
        CHECK(c->alloc(&c->Lrow, (size_t)N * N));
        CHECK(c->alloc(&c->Xc, (size_t)N * N));
    }
    for (int l = 0; l + 1 < c->nlev; ++l) {
        const MgLevel &Lf = c->lv[l], &Lc = c->lv[l + 1];
        CHECK(c->alloc(&c->ra1[l], (size_t)3 * (Lf.nz + 1) * (Lf.ny + 1) * (Lc.nx + 1)));
        CHECK(c->alloc(&c->ra2[l], (size_t)3 * (Lf.nz + 1) * (Lc.ny + 1) * (Lc.nx + 1)));
    }
    CHECK(c->alloc(&c->chol_status, 1));
    T3D_CUDA_OK(cudaMemsetAsync(c->chol_status, 0, sizeof(int), c->st));
    for (int l = 0; l + 1 < c->nlev; ++l) launch_mask_restrict(c->lv[l + 1], c->lv[l], c->st);
    c->standard = c->prm.mg_vcycle == T3D_VCYCLE_STANDARD;
    if (c->standard) {
        for (int l = 1; l < c->nlev; ++l) {
            const MgLevel& L = c->lv[l];
            CHECK(c->alloc(&c->Kel[l], (size_t)L.nx * L.ny * L.nz * 576));
            CHECK(c->alloc(&c->KelT[l], (size_t)L.nx * L.ny * L.nz * 576));
            CHECK(c->alloc(&c->vtmp[l], 3 * L.nn));
        }
        const int s1 = c->lv[1].span;
        CHECK(c->alloc(&c->E_mg, c->g.NE));
        CHECK(c->alloc(&c->Gpos, (size_t)s1 * s1 * s1 * 576));
        CHECK(upload_gpos(c));
    }
    return launch_check("mask restriction");
}

// A TMA-staged K(E)p records a bounded mbarrier wait that gave up in c->tma_err (the kernel went on and
// returned); its results are then void.  Reads the flag (synchronising the stream).
int check_tma(Context* c) {
    int e = 0;
    T3D_CUDA_OK(cudaMemcpyAsync(&e, c->tma_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    T3D_CUDA_OK(cudaStreamSynchronize(c->st));
    if (e) return set_error(T3D_ERR_CUDA, "TMA-staged K(E)p: an mbarrier wait timed out");
    return T3D_OK;
}

static int build_mixed(Context* c) {
    const Grid& g = c->g;
    // finest-level FP32 images are pitched (Grid::px, Grid::pex); their pads stay zero
    CHECK(c->alloc(&c->Ke32, 576));
    CHECK(c->alloc(&c->E32, g.NEp));
    T3D_CUDA_OK(cudaMemsetAsync(c->E32, 0, g.NEp * sizeof(float), c->st));
    for (float** v : {&c->r32, &c->d32, &c->z32, &c->p32, &c->Ap32}) {
        CHECK(c->alloc(v, 3 * g.NNp));
        T3D_CUDA_OK(cudaMemsetAsync(*v, 0, 3 * g.NNp * sizeof(float), c->st));
    }
    CHECK(c->alloc(&c->S32, 1));
    T3D_CUDA_OK(cudaMemsetAsync(c->S32, 0, sizeof(PcgScalars), c->st));
    CHECK(c->alloc(&c->tma_err, 1));
    T3D_CUDA_OK(cudaMemsetAsync(c->tma_err, 0, sizeof(int), c->st));
    for (int l = 0; l < c->nlev; ++l) {
        const MgLevel& L = c->lv[l];
        MgLevel32& M = c->lv32[l];
        M.nx = L.nx; M.ny = L.ny; M.nz = L.nz; M.span = L.span; M.nn = L.nn; M.mask = L.mask;
        M.pitch = l == 0 ? g.px : L.nx + 1;
        M.cs = l == 0 ? g.NNp : L.nn;
        CHECK(c->alloc(&M.diag, 3 * M.cs));
        T3D_CUDA_OK(cudaMemsetAsync(M.diag, 0, 3 * M.cs * sizeof(float), c->st));
        if (l > 0) {
            CHECK(c->alloc(&M.r, 3 * L.nn));
            CHECK(c->alloc(&M.x, 3 * L.nn));
        }
    }
    for (int l = 0; l + 1 < c->nlev; ++l) {
        const MgLevel &Lf = c->lv[l], &Lc = c->lv[l + 1];
        CHECK(c->alloc(&c->ra1_32[l], (size_t)3 * (Lf.nz + 1) * (Lf.ny + 1) * (Lc.nx + 1)));
    }
    if (c->standard) {
        CHECK(c->alloc(&c->E_mg32, g.NEp));
        T3D_CUDA_OK(cudaMemsetAsync(c->E_mg32, 0, g.NEp * sizeof(float), c->st));
        for (int l = 1; l < c->nlev; ++l) {
            const MgLevel& L = c->lv[l];
            CHECK(c->alloc(&c->Kel32[l], (size_t)L.nx * L.ny * L.nz * 300));   // symmetric-packed
            CHECK(c->alloc(&c->vtmp32[l], 3 * L.nn));
        }
    }
    float k32[576];
    for (int i = 0; i < 576; ++i) k32[i] = (float)c->Ke_h[i];
    T3D_CUDA_OK(cudaMemcpyAsync(c->Ke32, k32, sizeof k32, cudaMemcpyHostToDevice, c->st));
    c->modal = c->prm.matvec32_form == T3D_MATVEC32_AUTO && modal_ke_from(c->Ke_h, &c->kh, &c->modal_off);
    // the tile shape of the modal kernel is chosen by timing each one on this grid (zero vectors)
    if (c->prm.matvec32_tile > 0) CHECK(modal_tiling(g, c->dev, c->prm.matvec32_tile - 1, &c->mt));
    else CHECK(modal_autotune(g, c->dev, c->kh, c->E32, c->mask0, c->p32, c->Ap32, c->tma_err, c->st, &c->mt));
    CHECK(sync(c));
    return check_tma(c);
}

// FP32 K(E)p on the FP32 images (moduli E, default E32; x -> y); with dot.partial, x.y goes to S->denom.
// mark = 0 for the operator inside the Standard V-cycle (leaves the PCG's S->xit alone).
static void matvec32(Context* c, const float* x, float* y, RedSlot dot, PcgScalars* S, int mark = 1,
                     const float* E = nullptr) {
    c->launches += 1;
    if (!E) E = c->E32;
    if (c->modal) launch_matvec32_modal(c->g, c->kh, c->mt, E, c->mask0, x, y, dot, S, mark, c->tma_err, c->st);
    else launch_matvec32(c->g, c->Ke32, E, c->mask0, x, y, dot, S, mark, c->st);
}

// Load vector b of the context's load case on its free DOFs (fixed DOFs are skipped).
//   T3D_LOAD_TIP_LINE: the reference cantilever, F_z = -1/count on nodes ix = nelx, iz <= max(1, nz/6),
//     every iy of the padded grid (fea.cpp:388-403);
//   T3D_LOAD_TOP_TRACTION: total -1 in z spread evenly over the nodes of the top face iz = nelz;
//   T3D_LOAD_TORSION: +1 in y spread over the line ix = nelx, iz = nelz and -1 in y over ix = nelx,
//     iz = 0 (a couple about the x axis at the free end).
static int setup_load(Context* c) {
    const Grid& g = c->g;
    const Cuboid& q = c->cub;
    T3D_CUDA_OK(cudaMemsetAsync(c->b, 0, 3 * g.NN * sizeof(double), c->st));
    const int y0 = g.ny - q.nely, y1 = g.ny;    // node rows of the solid region (grid y)
    if (c->load_case == T3D_LOAD_TIP_LINE) {
        const int ix_load = std::min(q.nelx, g.nnx - 1);
        const int iz_max = std::max(1, g.nz / 6);
        const int count = (iz_max + 1) * g.nny;
        launch_setup_load(g, ix_load, iz_max, -1.0 / (double)count, c->mask0, c->b, c->st);
    } else if (c->load_case == T3D_LOAD_TOP_TRACTION) {
        const double f = -1.0 / ((double)(q.nelx + 1) * (q.nely + 1));
        launch_setup_box_load(g, 0, q.nelx, y0, y1, q.nelz, q.nelz, 2, f, c->mask0, c->b, c->st);
    } else {
        const double f = 1.0 / (double)(q.nely + 1);
        launch_setup_box_load(g, q.nelx, q.nelx, y0, y1, q.nelz, q.nelz, 1, f, c->mask0, c->b, c->st);
        launch_setup_box_load(g, q.nelx, q.nelx, y0, y1, 0, 0, 1, -f, c->mask0, c->b, c->st);
    }
    return launch_check("load set-up");
}

// External model (TopVoxel, TOP3D_XL.m:458-586): solid cells from the voxel list (passive elements as
// solid = 2), fixations and loads from the node lists.  The reference's x = 0 fixation does not apply;
// nodes touched by no solid element stay fixed, as for every model.  File coordinates (x, y, z) are the
// reference's element / node coordinates: cell (x, ny-1-y, z), grid node (x, ny-y, z).
static int setup_voxel_model(Context* c) {
    const Grid& g = c->g;
    const VoxelModel& v = *c->vox;
    std::vector<uint8_t> cells((size_t)g.NE, 0);
    for (int z = 0; z < v.nelz; ++z)
        for (int x = 0; x < v.nelx; ++x)
            for (int y = 0; y < v.nely; ++y) {
                const uint8_t s = v.voxel[(size_t)y + (size_t)v.nely * ((size_t)x + (size_t)v.nelx * z)];
                if (s) cells[(size_t)g.cell(x, g.ny - 1 - y, z)] = s;
            }
    auto grid_node = [&](int64_t m) {
        const int64_t py = v.nely + 1, px = v.nelx + 1;
        const int y = (int)(m % py), x = (int)((m / py) % px), z = (int)(m / (py * px));
        return (int32_t)g.node(x, g.ny - y, z);
    };
    // fixation nodes, then the loaded nodes of case 0, 1, ... ; forces of all cases in the same order
    const int nf = (int)v.fix_node.size();
    std::vector<int32_t> nodes;
    std::vector<double> forces;
    std::vector<int> case_off{nf}, case_n;
    for (int i = 0; i < nf; ++i) nodes.push_back(grid_node(v.fix_node[i]));
    for (int k = 0; k < c->ncases; ++k) {
        const std::vector<int64_t>& ln = k ? v.case_node[k - 1] : v.load_node;
        const std::vector<double>& lf = k ? v.case_f[k - 1] : v.load_f;
        for (int64_t m : ln) nodes.push_back(grid_node(m));
        forces.insert(forces.end(), lf.begin(), lf.end());
        case_n.push_back((int)ln.size());
        case_off.push_back(case_off.back() + (int)ln.size());
    }
    int32_t* d_nodes = nullptr;
    uint8_t* d_bits = nullptr;
    double* d_f = nullptr;
    cudaError_t e = cudaMalloc(&d_nodes, (nodes.size() + 1) * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&d_bits, (size_t)nf + 1);
    if (e == cudaSuccess) e = cudaMalloc(&d_f, (forces.size() + 1) * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->solid, cells.data(), cells.size(), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess && !nodes.empty())
        e = cudaMemcpyAsync(d_nodes, nodes.data(), nodes.size() * sizeof(int32_t), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess && nf) e = cudaMemcpyAsync(d_bits, v.fix_bits.data(), nf, cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess && !forces.empty())
        e = cudaMemcpyAsync(d_f, forces.data(), forces.size() * sizeof(double), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) {
        launch_setup_mask0(g, c->solid, 0, c->mask0, c->st);
        launch_setup_fix_list(nf, d_nodes, d_bits, c->mask0, c->st);
        const int64_t n3 = 3 * g.NN;
        for (int k = 0; k < c->ncases; ++k) {   // case 0 into b, and every case into its slot of b_cases
            double* bk = c->ncases > 1 ? c->b_cases + k * n3 : c->b;
            launch_setup_load_list(g, case_n[k], d_nodes + case_off[k], d_f + 3 * (size_t)(case_off[k] - nf),
                                   c->mask0, bk, c->st);
        }
        if (c->ncases > 1) e = cudaMemcpyAsync(c->b, c->b_cases, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c->st);
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);   // the host vectors and temporaries end here
    cudaFree(d_nodes);
    cudaFree(d_bits);
    cudaFree(d_f);
    if (e != cudaSuccess) return set_cuda_error(e, "external model set-up", __FILE__, __LINE__);
    return T3D_OK;
}

int create(int nely, int nelx, int nelz, const t3d_params* prm, const t3d_problem* pb, Context* c) {
    if (nely <= 0 || nelx <= 0 || nelz <= 0) return set_error(T3D_ERR_INVALID, "element counts must be positive");
    if (pb) {
        if (pb->load_case < T3D_LOAD_TIP_LINE || pb->load_case > T3D_LOAD_TORSION)
            return set_error(T3D_ERR_INVALID, "unknown load case");
        if (pb->num_voids < 0 || pb->num_voids > T3D_MAX_VOIDS)
            return set_error(T3D_ERR_INVALID, "num_voids must be in [0, T3D_MAX_VOIDS]");
        c->load_case = pb->load_case;
        c->voids.n = pb->num_voids;
        for (int k = 0; k < pb->num_voids; ++k)
            for (int d = 0; d < 3; ++d) {
                if (!(pb->voids[k][3 + d] > 0.0)) return set_error(T3D_ERR_INVALID, "void radii must be positive");
                c->voids.c[k][d] = pb->voids[k][d];
                c->voids.r[k][d] = pb->voids[k][3 + d];
            }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_error(T3D_ERR_NO_DEVICE, "no CUDA device available (the library has no CPU path)");
    }
    if (prm) c->prm = *prm;
    else t3d_params_default(&c->prm);
    if (c->prm.device < 0 || c->prm.device >= ndev) return set_error(T3D_ERR_NO_DEVICE, "device index out of range");
    if (c->prm.precision != T3D_FP64 && c->prm.precision != T3D_MIXED)
        return set_error(T3D_ERR_UNSUPPORTED, "precision must be T3D_FP64 or T3D_MIXED");
    if (c->prm.mg_coarse_assembly != T3D_COARSE_REFERENCE && c->prm.mg_coarse_assembly != T3D_COARSE_FULL)
        return set_error(T3D_ERR_UNSUPPORTED, "mg_coarse_assembly must be T3D_COARSE_REFERENCE or T3D_COARSE_FULL");
    if (c->prm.matvec32_form != T3D_MATVEC32_AUTO && c->prm.matvec32_form != T3D_MATVEC32_DENSE)
        return set_error(T3D_ERR_UNSUPPORTED, "matvec32_form must be T3D_MATVEC32_AUTO or T3D_MATVEC32_DENSE");
    if (c->prm.matvec64_form != T3D_MATVEC64_AUTO && c->prm.matvec64_form != T3D_MATVEC64_NODES)
        return set_error(T3D_ERR_UNSUPPORTED, "matvec64_form must be T3D_MATVEC64_AUTO or T3D_MATVEC64_NODES");
    if (c->prm.mg_vcycle != T3D_VCYCLE_ADAPTED && c->prm.mg_vcycle != T3D_VCYCLE_STANDARD)
        return set_error(T3D_ERR_UNSUPPORTED, "mg_vcycle must be T3D_VCYCLE_ADAPTED or T3D_VCYCLE_STANDARD");
    // fields that were reserved (zero) in earlier versions of t3d_params: 0 selects the default
    if (c->prm.mg_rebuild_period == 0) c->prm.mg_rebuild_period = 5;
    if (c->prm.mg_standard_weight == 0.0f) c->prm.mg_standard_weight = 0.35f;
    if (c->prm.mg_rebuild_period < 1) return set_error(T3D_ERR_INVALID, "mg_rebuild_period must be >= 1");
    if (c->prm.mg_vcycle == T3D_VCYCLE_STANDARD && !(c->prm.mg_standard_weight > 0.0f))
        return set_error(T3D_ERR_INVALID, "mg_standard_weight must be positive");
    c->mixed = c->prm.precision == T3D_MIXED;
    c->dev = c->prm.device;
    T3D_CUDA_OK(cudaSetDevice(c->dev));
    T3D_CUDA_OK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    for (auto& e : c->ev) T3D_CUDA_OK(cudaEventCreate(&e));
    c->use_graph = std::getenv("T3D_NO_GRAPH") == nullptr;

    // padding (padding.hpp:42-53, fea.cpp:189-197): the level count comes from the number of solid voxels,
    // the whole cuboid for the built-in problems, the file's solid voxels for an external model
    // (numel(find(voxelizedVolume_)), TOP3D_XL.m:1765-1774)
    const uint64_t nvox = c->vox ? (uint64_t)c->vox->num_solid : (uint64_t)nelx * nely * nelz;
    const int L = pad_levels(nvox);
    const int nx = pad_dim(nelx, L), ny = pad_dim(nely, L), nz = pad_dim(nelz, L);
    if ((int64_t)(nx + 1) * (ny + 1) * (nz + 1) * 3 >= (int64_t)INT32_MAX)
        return set_error(T3D_ERR_UNSUPPORTED, "grid too large for 32-bit DOF indices");
    c->g = make_grid(nx, ny, nz);
    c->cub = Cuboid{nelx, nely, nelz};
    c->ne = (int64_t)nelx * nely * nelz;
    if (c->voids.n > 0) {   // solid elements = cuboid minus the void ellipsoids (same test as k_setup_cells)
        int64_t ne = 0;
        for (int ez = 0; ez < nelz; ++ez)
            for (int ey = 0; ey < nely; ++ey)
                for (int ex = 0; ex < nelx; ++ex) ne += in_void(c->voids, ex, ey, ez) ? 0 : 1;
        if (ne == 0) return set_error(T3D_ERR_INVALID, "the voids remove every element");
        c->ne = ne;
    }
    if (c->vox) c->ne = c->vox->num_solid;
    const Grid& g = c->g;
    c->mv64_stream = c->prm.matvec64_form == T3D_MATVEC64_AUTO;
    if (c->mv64_stream) CHECK(stream64_tiling(g, c->dev, &c->st64));

    CHECK(c->alloc(&c->Ke, 576));
    CHECK(c->alloc(&c->Kd, KE_MAX_DISTINCT));
    CHECK(c->alloc(&c->kf, 72));
    CHECK(c->alloc(&c->solid, g.NE));
    CHECK(c->alloc(&c->mask0, g.NN));
    CHECK(c->alloc(&c->E, g.NE));
    CHECK(c->alloc(&c->ce, g.NE));
    CHECK(c->alloc(&c->x, g.NE));
    CHECK(c->alloc(&c->xnew, g.NE));
    CHECK(c->alloc(&c->dc, g.NE));
    CHECK(c->alloc(&c->xdc, g.NE));
    CHECK(c->alloc(&c->dcf, g.NE));
    for (double** v : {&c->b, &c->u, &c->r, &c->z, &c->p, &c->Ap}) CHECK(c->alloc(v, 3 * g.NN));
    for (double** v : {&c->frhs, &c->fx, &c->fr, &c->fz, &c->fp, &c->fAp, &c->flastx, &c->flastrhs, &c->fdiag})
        CHECK(c->alloc(v, g.NN));
    if (c->vox && c->vox->num_additional_loads > 0) {
        c->ncases = 1 + c->vox->num_additional_loads;
        CHECK(c->alloc(&c->b_cases, (size_t)c->ncases * 3 * g.NN));
        CHECK(c->alloc(&c->u_cases, (size_t)c->ncases * 3 * g.NN));
        CHECK(c->alloc(&c->ce_acc, g.NE));
        CHECK(c->alloc(&c->one, 1));
        const double one = 1.0;
        T3D_CUDA_OK(cudaMemcpy(c->one, &one, sizeof one, cudaMemcpyHostToDevice));
        T3D_CUDA_OK(cudaMemsetAsync(c->b_cases, 0, (size_t)c->ncases * 3 * g.NN * sizeof(double), c->st));
        T3D_CUDA_OK(cudaMemsetAsync(c->u_cases, 0, (size_t)c->ncases * 3 * g.NN * sizeof(double), c->st));
    }
    CHECK(c->alloc(&c->S, 1));
    CHECK(c->alloc(&c->FS, 1));
    CHECK(c->alloc(&c->OC, 1));
    CHECK(c->alloc(&c->scal, 8));
    double* part = nullptr;
    unsigned int* cnt = nullptr;
    CHECK(c->alloc(&part, 4 * RED_BLOCKS));
    CHECK(c->alloc(&cnt, 4));
    T3D_CUDA_OK(cudaMemsetAsync(cnt, 0, 4 * sizeof(unsigned int), c->st));
    for (int i = 0; i < 4; ++i) c->slot[i] = RedSlot{part + i * RED_BLOCKS, cnt + i};
    T3D_CUDA_OK(cudaMallocHost(&c->S_h, sizeof(PcgScalars)));
    T3D_CUDA_OK(cudaMallocHost(&c->OC_h, sizeof(OcState)));
    T3D_CUDA_OK(cudaMallocHost(&c->FS_h, sizeof(FilterScalars)));
    T3D_CUDA_OK(cudaMallocHost(&c->scal_h, 8 * sizeof(double)));
    T3D_CUDA_OK(cudaMallocHost(&c->flag_h, 2 * sizeof(int)));

    // element stiffness (fea.cpp:345 passes nu = 0.3 literally) and filter kernel
    hex8_stiffness(0.3, 1.0, c->Ke_h);
    T3D_CUDA_OK(cudaMemcpyAsync(c->Ke, c->Ke_h, sizeof c->Ke_h, cudaMemcpyHostToDevice, c->st));
    CHECK(update_ke_pattern(c));
    double kf[72];
    filter_kernel(c->prm.filter_rmin, kf);
    T3D_CUDA_OK(cudaMemcpyAsync(c->kf, kf, sizeof kf, cudaMemcpyHostToDevice, c->st));

    // zero every array once: ghost cells and non-solid cells stay exactly zero from here on
    T3D_CUDA_OK(cudaMemsetAsync(c->E, 0, g.NE * sizeof(double), c->st));
    T3D_CUDA_OK(cudaMemsetAsync(c->ce, 0, g.NE * sizeof(double), c->st));
    for (float* v : {c->x, c->xnew, c->dc, c->xdc, c->dcf})
        T3D_CUDA_OK(cudaMemsetAsync(v, 0, g.NE * sizeof(float), c->st));
    for (double* v : {c->b, c->u, c->r, c->z, c->p, c->Ap})
        T3D_CUDA_OK(cudaMemsetAsync(v, 0, 3 * g.NN * sizeof(double), c->st));
    for (double* v : {c->frhs, c->fx, c->fr, c->fz, c->fp, c->fAp, c->flastx, c->flastrhs})
        T3D_CUDA_OK(cudaMemsetAsync(v, 0, g.NN * sizeof(double), c->st));
    T3D_CUDA_OK(cudaMemsetAsync(c->S, 0, sizeof(PcgScalars), c->st));
    T3D_CUDA_OK(cudaMemsetAsync(c->scal, 0, 8 * sizeof(double), c->st));

    // model: solid cells, fixed DOFs, load (fea.cpp:181-447)
    if (c->vox) {
        CHECK(setup_voxel_model(c));
    } else {
        launch_setup_cells(g, c->cub, c->voids, c->solid, c->st);
        launch_setup_mask0(g, c->solid, 1, c->mask0, c->st);
        CHECK(launch_check("model set-up"));
        CHECK(setup_load(c));
    }
    CHECK(build_levels(c));
    if (c->mixed) CHECK(build_mixed(c));
    launch_filter_diag(g, c->solid, c->kf, c->fdiag, c->st);
    CHECK(launch_check("filter set-up"));
    return sync(c);
}

// ------------------------------------------------------------------ lazily built layout maps
// Morton order of the solid elements (fea.cpp:289-317): octree walk visiting children in key order
// (x bit most significant, then y, then z), emitting grid cell indices.
static void morton_walk(const Context* c, int x0, int y0, int z0, int h, std::vector<int32_t>& out) {
    const Cuboid& q = c->cub;
    if (x0 >= q.nelx || y0 >= q.nely || z0 >= q.nelz) return;
    if (h == 1) {
        const bool solid = c->vox ? c->vox->voxel[(size_t)y0 + (size_t)q.nely * ((size_t)x0 + (size_t)q.nelx * z0)] != 0
                                  : !in_void(c->voids, x0, y0, z0);
        if (solid) out.push_back((int32_t)c->g.cell(x0, c->g.ny - 1 - y0, z0));
        return;
    }
    const int m = h / 2;
    for (int k = 0; k < 8; ++k) morton_walk(c, x0 + ((k >> 2) & 1) * m, y0 + ((k >> 1) & 1) * m, z0 + (k & 1) * m, m, out);
}

int ensure_morton(Context* c) {
    if (c->morton) return T3D_OK;
    int h = 1;
    while (h < std::max(c->cub.nelx, std::max(c->cub.nely, c->cub.nelz))) h *= 2;
    c->morton_h.clear();
    c->morton_h.reserve(c->ne);
    morton_walk(c, 0, 0, 0, h, c->morton_h);
    CHECK(c->alloc(&c->morton, c->ne));
    T3D_CUDA_OK(cudaMemcpy(c->morton, c->morton_h.data(), c->ne * sizeof(int32_t), cudaMemcpyHostToDevice));
    return T3D_OK;
}

static int ensure_free(Context* c) {
    if (c->free_d) return T3D_OK;
    std::vector<uint8_t> m(c->g.NN);
    T3D_CUDA_OK(cudaMemcpy(m.data(), c->mask0, c->g.NN, cudaMemcpyDeviceToHost));
    c->free_h.clear();
    for (int64_t n = 0; n < c->g.NN; ++n)
        for (int k = 0; k < 3; ++k)
            if (!((m[n] >> k) & 1)) c->free_h.push_back((int32_t)(3 * n + k));
    CHECK(c->alloc(&c->free_d, c->free_h.size()));
    T3D_CUDA_OK(cudaMemcpy(c->free_d, c->free_h.data(), c->free_h.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    return T3D_OK;
}

static int ensure_stage(Context* c) {
    CHECK(ensure_free(c));
    CHECK(ensure_morton(c));
    const size_t need = std::max(c->free_h.size(), (size_t)c->ne);
    if (c->stage_n >= need) return T3D_OK;
    CHECK(c->alloc(&c->stage, need));
    c->stage_n = need;
    return T3D_OK;
}

// host free vector -> device grid vector (fixed DOFs zero)
static int upload_free(Context* c, const double* h, double* grid) {
    CHECK(ensure_stage(c));
    const int64_t nf = (int64_t)c->free_h.size();
    T3D_CUDA_OK(cudaMemsetAsync(grid, 0, 3 * c->g.NN * sizeof(double), c->st));
    T3D_CUDA_OK(cudaMemcpyAsync(c->stage, h, nf * sizeof(double), cudaMemcpyHostToDevice, c->st));
    launch_scatter_free(nf, c->free_d, c->stage, c->g.NN, grid, c->st);
    return launch_check("scatter_free");
}
static int download_free(Context* c, const double* grid, double* h) {
    CHECK(ensure_stage(c));
    const int64_t nf = (int64_t)c->free_h.size();
    launch_gather_free(nf, c->free_d, grid, c->g.NN, c->stage, c->st);
    CHECK(launch_check("gather_free"));
    T3D_CUDA_OK(cudaMemcpyAsync(h, c->stage, nf * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}
static int upload_cells_f64(Context* c, const double* h, double* cells) {
    CHECK(ensure_stage(c));
    T3D_CUDA_OK(cudaMemsetAsync(cells, 0, c->g.NE * sizeof(double), c->st));
    T3D_CUDA_OK(cudaMemcpyAsync(c->stage, h, c->ne * sizeof(double), cudaMemcpyHostToDevice, c->st));
    launch_cells_from_morton_f64(c->ne, c->morton, c->stage, cells, c->st);
    return launch_check("cells_from_morton");
}
static int download_cells_f64(Context* c, const double* cells, double* h) {
    CHECK(ensure_stage(c));
    launch_cells_to_morton_f64(c->ne, c->morton, cells, c->stage, c->st);
    CHECK(launch_check("cells_to_morton"));
    T3D_CUDA_OK(cudaMemcpyAsync(h, c->stage, c->ne * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}
static int upload_cells_f32(Context* c, const float* h, float* cells) {
    CHECK(ensure_stage(c));
    float* st = reinterpret_cast<float*>(c->stage);
    T3D_CUDA_OK(cudaMemsetAsync(cells, 0, c->g.NE * sizeof(float), c->st));
    T3D_CUDA_OK(cudaMemcpyAsync(st, h, c->ne * sizeof(float), cudaMemcpyHostToDevice, c->st));
    launch_cells_from_morton_f32(c->ne, c->morton, st, cells, c->st);
    return launch_check("cells_from_morton");
}
static int download_cells_f32(Context* c, const float* cells, float* h) {
    CHECK(ensure_stage(c));
    float* st = reinterpret_cast<float*>(c->stage);
    launch_cells_to_morton_f32(c->ne, c->morton, cells, st, c->st);
    CHECK(launch_check("cells_to_morton"));
    T3D_CUDA_OK(cudaMemcpyAsync(h, st, c->ne * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

// ------------------------------------------------------------------ multigrid
// make_diagonal_preconditioner_from_static for the moduli in c->E (preconditioner.cpp:38-79)
static int mg_setup(Context* c) {
    c->launches += 1 + (c->nlev - 1) + (c->Nc ? 3 : 0);
    launch_diag0(c->g, c->Ke, c->E, c->mask0, c->lv[0].diag, c->st);
    if (c->standard) {   // Galerkin element matrices and their diagonals on every coarse level
        // the cycle's level-0 operator is K(E) of these moduli, so that a hierarchy kept between rebuilds
        // (loop 1 and every 5th, driver.cpp:132) stays one symmetric positive definite preconditioner
        T3D_CUDA_OK(cudaMemcpyAsync(c->E_mg, c->E, c->g.NE * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
        launch_galerkin_fine(c->g, c->lv[1], c->E, c->mask0, c->Gpos, c->Ke, c->Kel[1], c->st);
        for (int l = 2; l < c->nlev; ++l) launch_galerkin_coarse(c->lv[l - 1], c->lv[l], c->Kel[l - 1], c->Kel[l], c->st);
        for (int l = 1; l < c->nlev; ++l) {
            launch_level_diag(c->lv[l], c->Kel[l], c->st);
            const MgLevel& L = c->lv[l];
            launch_kel_transpose((int64_t)L.nx * L.ny * L.nz, c->Kel[l], c->KelT[l], c->st);
        }
        c->launches += 3 * (c->nlev - 1);
        if (c->Nc) {
            const MgLevel& Lc = c->lv[c->nlev - 1];
            launch_to_coarse_layout(Lc, c->Kel[c->nlev - 1], c->Kce, c->st);
            launch_coarse_assemble(Lc, c->Kce, c->Kc, c->st);
            c->launches += launch_cholesky(c->Kc, c->LT, c->Lrow, c->Nc, c->chol_status, c->st);
            launch_coarse_inverse(c->LT, c->Lrow, c->Nc, c->chol_status, c->Xc, c->st);
        }
        if (c->mixed) {   // FP32 images: level-0 moduli, coarse element matrices, reciprocal diagonals
            launch_cells_to32(c->g, c->E_mg, c->E_mg32, c->st);
            for (int l = 1; l < c->nlev; ++l) {
                const MgLevel& L = c->lv[l];
                launch_kel_pack32((int64_t)L.nx * L.ny * L.nz, c->Kel[l], c->Kel32[l], c->st);
            }
            for (int l = 0; l < c->nlev; ++l) {
                const MgLevel32& M = c->lv32[l];
                launch_recip_diag32(3 * (int64_t)(M.ny + 1) * (M.nz + 1), M.nx + 1, M.pitch, c->lv[l].diag, M.diag,
                                    c->st);
            }
            c->launches += 2 * c->nlev;
        }
        c->mg_ready = true;
        return launch_check("mg set-up");
    }
    for (int l = 0; l + 1 < c->nlev; ++l) launch_diag_coarsen(c->lv[l + 1], c->lv[l], c->st);
    if (c->Nc) {
        const MgLevel& Lc = c->lv[c->nlev - 1];
        // the reference samples s^3 fine elements per coarse element with s the coarsest level's own span
        // (coarsest.cpp:138-323; a corner sub-block of the grid when there are more than 2 levels); the full
        // Galerkin form samples all of them (s = product of the spans)
        int span = Lc.span;
        if (c->prm.mg_coarse_assembly == T3D_COARSE_FULL) span = c->g.nx / Lc.nx;
        launch_coarse_element_matrices(c->g, Lc, span, c->mask0, c->E, c->Ke, (double)c->prm.Emin, c->Kce, c->st);
        launch_coarse_assemble(Lc, c->Kce, c->Kc, c->st);
        c->launches += launch_cholesky(c->Kc, c->LT, c->Lrow, c->Nc, c->chol_status, c->st);
        launch_coarse_inverse(c->LT, c->Lrow, c->Nc, c->chol_status, c->Xc, c->st);
    }
    if (c->mixed) {
        for (int l = 0; l < c->nlev; ++l) {
            const MgLevel32& M = c->lv32[l];
            launch_recip_diag32(3 * (int64_t)(M.ny + 1) * (M.nz + 1), M.nx + 1, M.pitch, c->lv[l].diag, M.diag, c->st);
        }
        c->launches += c->nlev;
    }
    c->mg_ready = true;
    return launch_check("mg set-up");
}

// Selects the FP64 streaming kernel's coefficient form for c->Ke_h (ordered on c->st)
static int update_ke_pattern(Context* c) {
    static_assert(sizeof(c->Ke_h) == 576 * sizeof(double), "Ke_h");
    double D[KE_MAX_DISTINCT] = {0};
    c->ke_pat = ke_pattern_magnitudes(c->Ke_h, D);
    if (c->ke_pat) T3D_CUDA_OK(cudaMemcpyAsync(c->Kd, D, sizeof D, cudaMemcpyHostToDevice, c->st));
    return T3D_OK;
}

// FP64 y = K(E) u on c->E (bit-identical in both forms); with dot.partial, u.y goes to S->denom unless
// S->done.  Returns the number of kernels launched.
int matvec64(Context* c, const double* u, double* y, RedSlot dot, PcgScalars* S) {
    if (!c->mv64_stream) {
        launch_matvec64(c->g, c->Ke, c->E, c->mask0, u, y, dot, S, c->st);
        return 1;
    }
    launch_matvec64_stream(c->g, c->st64, c->Ke_h, c->ke_pat ? c->Kd : nullptr, c->E, c->mask0, u, y, S, c->st);
    if (!dot.partial) return 1;
    launch_dot_pcg(c->g, u, y, dot, S, c->st);
    return 2;
}

// y = K_l x on level l (level 0: K(E) of the moduli the hierarchy was built from)
static void level_matvec(Context* c, int l, const double* x, double* y, const PcgScalars* S) {
    if (l == 0)
        launch_matvec64_stream(c->g, c->st64, c->Ke_h, c->ke_pat ? c->Kd : nullptr, c->E_mg, c->mask0, x, y, S,
                               c->st);
    else
        launch_level_matvec(c->lv[l], c->KelT[l], x, y, S, c->st);
}

// kernels of one V-cycle
static int vcycle_launches(const Context* c) {
    const int L = c->nlev;
    return c->standard ? 9 * (L - 1) + 2 : 4 * (L - 1) + 1;
}

// The 'Standard' cycle (see k_mg_standard.cu); level 0 uses Ap as scratch (free between the PCG update
// and the next K(E)p)
static void vcycle_standard(Context* c, const double* r, double* z, PcgScalars* S, RedSlot dot) {
    const int L = c->nlev;
    const double w = (double)c->prm.mg_standard_weight;
    c->launches += vcycle_launches(c);
    for (int l = 0; l + 1 < L; ++l) {
        const double* rl = l == 0 ? r : c->lv[l].r;
        double* xl = l == 0 ? z : c->lv[l].x;
        double* t = l == 0 ? c->Ap : c->vtmp[l];
        launch_jacobi_init(c->lv[l], rl, xl, w, S, c->st);
        level_matvec(c, l, xl, t, S);
        launch_residual(c->lv[l], rl, t, S, c->st);
        launch_restrict(c->lv[l + 1], c->lv[l], t, c->lv[l + 1].r, c->ra1[l], c->ra2[l], S, c->st, false);
    }
    launch_coarse_solve(c->lv[L - 1], c->Xc, c->Nc, c->chol_status, S, c->st);
    for (int l = L - 2; l >= 0; --l) {
        const double* rl = l == 0 ? r : c->lv[l].r;
        double* xl = l == 0 ? z : c->lv[l].x;
        double* t = l == 0 ? c->Ap : c->vtmp[l];
        launch_prolong_add(c->lv[l + 1], c->lv[l], c->lv[l + 1].x, xl, S, c->st);
        level_matvec(c, l, xl, t, S);
        launch_jacobi_correct(c->lv[l], rl, t, xl, w, S, c->st);
    }
    if (S) launch_dot_rz(c->g.NN, r, z, dot, S, c->st);
}

// z = M r for grid vectors; with S, r.z goes to S (rz / beta)
static void vcycle(Context* c, const double* r, double* z, PcgScalars* S, RedSlot dot) {
    if (c->standard) {
        vcycle_standard(c, r, z, S, dot);
        return;
    }
    const int L = c->nlev;
    c->launches += 4 * (L - 1) + 1;
    for (int l = 0; l + 1 < L; ++l)
        launch_restrict(c->lv[l + 1], c->lv[l], l == 0 ? r : c->lv[l].r, c->lv[l + 1].r, c->ra1[l], c->ra2[l], S,
                        c->st);
    launch_coarse_solve(c->lv[L - 1], c->Xc, c->Nc, c->chol_status, S, c->st);
    for (int l = L - 2; l >= 1; --l)
        launch_prolong_smooth(c->lv[l + 1], c->lv[l], c->lv[l + 1].x, c->lv[l].r, c->lv[l].x,
                              (double)c->prm.mg_weight, S, c->st);
    launch_prolong_smooth0(c->lv[1], c->lv[0], c->lv[1].x, r, z, (double)c->prm.mg_weight, dot, S, c->st);
}

// ------------------------------------------------------------------ PCG (solver.cpp:87-217)
static void pcg_iteration(Context* c) {
    c->launches += 2 + matvec64(c, c->p, c->Ap, c->slot[0], c->S);
    launch_pcg_update(c->g, c->u, c->r, c->p, c->Ap, c->slot[1], c->S, c->st);
    vcycle(c, c->r, c->z, c->S, c->slot[2]);
    launch_pcg_direction(c->g, c->z, c->p, c->S, c->st);
}

static constexpr int PCG_CHUNK = 16;

static int ensure_pcg_graph(Context* c) {
    if (!c->use_graph || c->pcg_graph) return T3D_OK;
    cudaGraph_t graph;
    T3D_CUDA_OK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < PCG_CHUNK; ++k) pcg_iteration(c);
    T3D_CUDA_OK(cudaStreamEndCapture(c->st, &graph));
    cudaError_t e = cudaGraphInstantiate(&c->pcg_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGraphInstantiate", __FILE__, __LINE__);
    c->pcg_graph_len = PCG_CHUNK;
    return T3D_OK;
}

// Solves K(E) u = b on device-resident c->E, c->b, warm start c->u.  Returns the PCG_free
// iteration count in *iters.
static int pcg_solve(Context* c, double tol, int maxit, int* iters) {
    if (!c->mg_ready) return set_error(T3D_ERR_INVALID, "multigrid preconditioner not set up");
    CHECK(ensure_pcg_graph(c));
    c->launches += 1 + matvec64(c, c->u, c->Ap, RedSlot{nullptr, nullptr}, nullptr);
    launch_pcg_init(c->g, c->b, c->Ap, c->r, c->slot[1], c->S, tol, c->st);
    vcycle(c, c->r, c->z, c->S, c->slot[2]);
    launch_pcg_start(c->g, c->z, c->p, c->st);
    CHECK(launch_check("pcg start"));
    int queued = 0, chunk = 0;
    bool done = false;
    while (queued < maxit && !done) {
        const int n = std::min(PCG_CHUNK, maxit - queued);
        if (c->use_graph && n == PCG_CHUNK) {
            T3D_CUDA_OK(cudaGraphLaunch(c->pcg_graph, c->st));
            c->launches += (int64_t)PCG_CHUNK * ((c->mv64_stream ? 4 : 3) + vcycle_launches(c));
        } else {
            for (int k = 0; k < n; ++k) pcg_iteration(c);
            CHECK(launch_check("pcg iteration"));
        }
        queued += n;
        const int slot = chunk & 1;
        T3D_CUDA_OK(cudaMemcpyAsync(&c->flag_h[slot], &c->S->done, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        T3D_CUDA_OK(cudaEventRecord(c->ev[slot], c->st));
        if (chunk >= 1) {   // poll the previous chunk while this one runs
            T3D_CUDA_OK(cudaEventSynchronize(c->ev[slot ^ 1]));
            done = c->flag_h[slot ^ 1] != 0;
        }
        ++chunk;
    }
    T3D_CUDA_OK(cudaMemcpyAsync(c->S_h, c->S, sizeof(PcgScalars), cudaMemcpyDeviceToHost, c->st));
    CHECK(sync(c));
    *iters = c->S_h->done ? c->S_h->result : maxit;
    return T3D_OK;
}

// ------------------------------------------------------------------ mixed-precision solve
// The Standard cycle in FP32 (k_mg_standard32.cu): the same steps as vcycle_standard; level 0 uses Ap32 as
// scratch and the modal FP32 K(E) of the hierarchy's moduli as its operator
static void vcycle32_standard(Context* c, const float* r, float* z, PcgScalars* S, RedSlot dot) {
    const int L = c->nlev;
    const float w = c->prm.mg_standard_weight;
    // level 0 with the modal TMA kernel: the residual and the correction (with r.z) run in its epilogue
    const bool fuse = c->modal && modal_fused_available(c->mt);
    auto level_op = [&](int l, const float* x, float* y) {
        if (l == 0) matvec32(c, x, y, RedSlot{nullptr, nullptr}, S, 0, c->E_mg32);
        else {
            launch_level_matvec32(c->lv32[l], c->Kel32[l], x, y, S, c->st);
            c->launches += 1;
        }
    };
    for (int l = 0; l + 1 < L; ++l) {
        const float* rl = l == 0 ? r : c->lv32[l].r;
        float* xl = l == 0 ? z : c->lv32[l].x;
        float* t = l == 0 ? c->Ap32 : c->vtmp32[l];
        launch_jacobi_init32(c->lv32[l], rl, xl, w, S, c->st);
        c->launches += 1;
        if (l == 0 && fuse) {
            launch_matvec32_fused(1, c->g, c->kh, c->mt, c->E_mg32, c->mask0, xl, t, rl, nullptr, w,
                                  RedSlot{nullptr, nullptr}, S, c->tma_err, c->st);
            c->launches += 1;
        } else {
            level_op(l, xl, t);
            launch_residual32(c->lv32[l], rl, t, S, c->st);
            c->launches += 1;
        }
        launch_restrict32(c->lv32[l + 1], c->lv32[l], t, c->lv32[l + 1].r, c->ra1_32[l], S, c->st, false);
        c->launches += c->lv32[l + 1].span == 4 ? 2 : 1;
    }
    launch_coarse_solve32(c->lv32[L - 1], c->Xc, c->Nc, c->chol_status, S, c->st);
    c->launches += 1;
    for (int l = L - 2; l >= 1; --l) {
        const float* rl = c->lv32[l].r;
        float* xl = c->lv32[l].x;
        launch_prolong_add32(c->lv32[l + 1], c->lv32[l], c->lv32[l + 1].x, xl, xl, S, c->st);
        level_op(l, xl, c->vtmp32[l]);
        launch_jacobi_correct32(c->lv32[l], rl, c->vtmp32[l], xl, w, S, c->st);
        c->launches += 2;
    }
    // level 0: T = z + P x_1 into Ap32, then z = T + w (r - K T) / D with r.z, fused; else the separate steps
    if (fuse) {
        launch_prolong_add32(c->lv32[1], c->lv32[0], c->lv32[1].x, z, c->Ap32, S, c->st);
        launch_matvec32_fused(2, c->g, c->kh, c->mt, c->E_mg32, c->mask0, c->Ap32, z, r, c->lv32[0].diag, w, dot, S,
                              c->tma_err, c->st);
        c->launches += 2;
        return;
    }
    launch_prolong_add32(c->lv32[1], c->lv32[0], c->lv32[1].x, z, z, S, c->st);
    level_op(0, z, c->Ap32);
    launch_jacobi_correct32(c->lv32[0], r, c->Ap32, z, w, S, c->st);
    launch_dot_rz32(3 * c->g.NNp, r, z, dot, S, c->st);
    c->launches += 3;
}

static void vcycle32(Context* c, const float* r, float* z, PcgScalars* S, RedSlot dot) {
    if (c->standard) {
        vcycle32_standard(c, r, z, S, dot);
        return;
    }
    const int L = c->nlev;
    // per transition: restriction (x + y-z passes for span 4, one x-y-z pass for span 2) and prolongation
    for (int l = 0; l + 1 < L; ++l) c->launches += c->lv32[l + 1].span == 2 ? 2 : 3;
    c->launches += 1;
    for (int l = 0; l + 1 < L; ++l)
        launch_restrict32(c->lv32[l + 1], c->lv32[l], l == 0 ? r : c->lv32[l].r, c->lv32[l + 1].r, c->ra1_32[l], S,
                          c->st);
    launch_coarse_solve32(c->lv32[L - 1], c->Xc, c->Nc, c->chol_status, S, c->st);
    for (int l = L - 2; l >= 1; --l)
        launch_prolong_smooth32(c->lv32[l + 1], c->lv32[l], c->lv32[l + 1].x, c->lv32[l].r, c->lv32[l].x,
                                c->prm.mg_weight, S, c->st);
    launch_prolong_smooth0_32(c->lv32[1], c->lv32[0], c->lv32[1].x, r, z, c->prm.mg_weight, dot, S, c->st);
}

int member_vcycle32(Context* c, const float* r, float* z, PcgScalars* S, RedSlot dot) {
    vcycle32(c, r, z, S, dot);
    return launch_check("V-cycle");
}

static void pcg32_iteration(Context* c) {
    c->launches += 2;
    matvec32(c, c->p32, c->Ap32, c->slot[0], c->S32);
    launch_pcg_update32(c->g, c->d32, c->r32, c->p32, c->Ap32, c->slot[1], c->S32, c->st);
    vcycle32(c, c->r32, c->z32, c->S32, c->slot[2]);
    launch_pcg_direction32(c->g, c->z32, c->p32, c->d32, c->S32, c->st);
}

static int ensure_pcg32_graph(Context* c) {
    if (!c->use_graph || c->pcg32_graph) return T3D_OK;
    cudaGraph_t graph;
    const int64_t l0 = c->launches;
    T3D_CUDA_OK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < PCG_CHUNK; ++k) pcg32_iteration(c);
    T3D_CUDA_OK(cudaStreamEndCapture(c->st, &graph));
    c->pcg32_graph_launches = (c->launches - l0) / PCG_CHUNK;   // kernels per iteration in the graph
    c->launches = l0;
    cudaError_t e = cudaGraphInstantiate(&c->pcg32_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGraphInstantiate", __FILE__, __LINE__);
    return T3D_OK;
}

// Defect correction: r64 = b - K64 u64 (FP64), stop when |r64| < max(1e-30,|b|)*tol (the reference's
// test, solver.cpp:149,184, applied to the true residual); else solve K32 d = r32 with the FP32
// MG-PCG (at most the remaining budget of max_it iterations, inner target max(stop, 1e-5|r64|))
// and add d to u64.  *iters = inner iterations used (max_it when the budget ran out unconverged).
static int mixed_solve(Context* c, double tol, int maxit, int* iters) {
    if (!c->mg_ready) return set_error(T3D_ERR_INVALID, "multigrid preconditioner not set up");
    CHECK(ensure_pcg32_graph(c));
    const Grid& g = c->g;
    launch_cells_to32(g, c->E, c->E32, c->st);
    launch_dot(g, 3, c->b, c->b, c->slot[3], c->scal + 5, c->st);
    c->launches += 2;
    T3D_CUDA_OK(cudaMemcpyAsync(c->scal_h + 5, c->scal + 5, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CHECK(sync(c));
    const double nb = std::sqrt(c->scal_h[5]);
    const double stop = (1.0e-30 < nb ? nb : 1.0e-30) * tol;
    int budget = maxit, used = 0, outer = 0;
    bool converged = false;
    for (; outer < 64; ++outer) {
        c->launches += 1 + matvec64(c, c->u, c->Ap, RedSlot{nullptr, nullptr}, nullptr);
        launch_mixed_residual(g, c->b, c->Ap, c->r32, c->d32, c->slot[3], c->scal + 6, c->st);
        CHECK(launch_check("mixed residual"));
        T3D_CUDA_OK(cudaMemcpyAsync(c->scal_h + 6, c->scal + 6, sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CHECK(sync(c));
        const double rn = std::sqrt(c->scal_h[6]);
        if (rn < stop) { converged = true; break; }
        if (budget <= 0) break;
        PcgScalars init{};
        init.stop = std::max(stop, 1e-5 * rn);
        init.tol = tol;
        init.first = 1;
        init.maxit = budget;
        T3D_CUDA_OK(cudaMemcpyAsync(c->S32, &init, sizeof init, cudaMemcpyHostToDevice, c->st));
        vcycle32(c, c->r32, c->z32, c->S32, c->slot[2]);
        T3D_CUDA_OK(cudaMemcpyAsync(c->p32, c->z32, 3 * g.NNp * sizeof(float), cudaMemcpyDeviceToDevice, c->st));
        int queued = 0, chunk = 0;
        bool done = false;
        while (queued < budget && !done) {
            const int n = std::min(PCG_CHUNK, budget - queued);
            if (c->use_graph && n == PCG_CHUNK) {
                T3D_CUDA_OK(cudaGraphLaunch(c->pcg32_graph, c->st));
                c->launches += (int64_t)PCG_CHUNK * c->pcg32_graph_launches;
            } else {
                for (int k = 0; k < n; ++k) pcg32_iteration(c);
                CHECK(launch_check("pcg32 iteration"));
            }
            queued += n;
            const int slot = chunk & 1;
            T3D_CUDA_OK(cudaMemcpyAsync(&c->flag_h[slot], &c->S32->done, sizeof(int), cudaMemcpyDeviceToHost, c->st));
            T3D_CUDA_OK(cudaEventRecord(c->ev[slot], c->st));
            if (chunk >= 1) {
                T3D_CUDA_OK(cudaEventSynchronize(c->ev[slot ^ 1]));
                done = c->flag_h[slot ^ 1] != 0;
            }
            ++chunk;
        }
        launch_mixed_accumulate(g, c->u, c->d32, c->st);
        c->launches += 1;
        T3D_CUDA_OK(cudaMemcpyAsync(c->S_h, c->S32, sizeof(PcgScalars), cudaMemcpyDeviceToHost, c->st));
        CHECK(sync(c));
        used += c->S_h->it;
        budget -= c->S_h->it;
    }
    c->last_outer = outer;
    *iters = converged ? used : maxit;
    return check_tma(c);
}

static int solve(Context* c, double tol, int maxit, int* iters) {
    return c->mixed ? mixed_solve(c, tol, maxit, iters) : pcg_solve(c, tol, maxit, iters);
}

// ------------------------------------------------------------------ PDE filter (filter.cpp:175-275)
static int filter_apply(Context* c, const float* src_cells, float* dst_cells) {
    const Grid& g = c->g;
    launch_filter_rhs(g, c->solid, src_cells, c->frhs, c->st);
    launch_filter_norms(g, c->frhs, c->flastrhs, c->slot[0], c->slot[1], c->FS, c->st);
    launch_filter_x0(g, c->flastx, c->fx, c->FS, c->st);
    launch_filter_matvec(g, c->solid, c->kf, c->fx, c->fAp, RedSlot{nullptr, nullptr}, c->FS, c->st);
    launch_filter_r0(g, c->frhs, c->fAp, c->fdiag, c->fr, c->fz, c->fp, c->slot[0], c->slot[1], c->FS, c->st);
    CHECK(launch_check("filter start"));
    for (int it = 0; it < 80; it += 8) {
        for (int k = 0; k < 8 && it + k < 80; ++k) {
            c->launches += 4;
            launch_filter_matvec(g, c->solid, c->kf, c->fp, c->fAp, c->slot[2], c->FS, c->st);
            launch_filter_update(g, c->fx, c->fr, c->fp, c->fAp, c->slot[3], c->FS, c->st);
            launch_filter_precond(g, c->fr, c->fdiag, c->fz, c->slot[0], c->FS, c->st);
            launch_filter_direction(g, c->fz, c->fp, c->FS, c->st);
        }
        CHECK(launch_check("filter iteration"));
        T3D_CUDA_OK(cudaMemcpyAsync(c->flag_h, &c->FS->done, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        CHECK(sync(c));
        if (c->flag_h[0]) break;
    }
    launch_filter_to_cells(g, c->solid, c->fx, dst_cells, c->st);
    c->launches += 6;
    T3D_CUDA_OK(cudaMemcpyAsync(c->flastx, c->fx, g.NN * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    T3D_CUDA_OK(cudaMemcpyAsync(c->flastrhs, c->frhs, g.NN * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    return launch_check("filter finish");
}

// ------------------------------------------------------------------ OC (driver.cpp:170-189)
static constexpr int OC_MAX_PASSES = 400;

static int oc_update(Context* c, float V0) {
    const int fp64 = c->prm.oc_sum_order == T3D_SUM_FP64;
    if (!fp64) CHECK(ensure_morton(c));
    launch_oc_init(c->OC, c->st);
    int passes = 0;
    for (;;) {
        for (int k = 0; k < 16; ++k) {
            c->launches += fp64 ? 1 : 2;
            launch_oc_pass(c->g, c->solid, c->x, c->dc, c->xnew, c->OC, fp64, V0, c->ne, c->slot[0], c->st);
            if (!fp64) launch_oc_vec8_vol(c->ne, c->morton, c->xnew, c->OC, V0, c->st);
        }
        CHECK(launch_check("oc pass"));
        passes += 16;
        T3D_CUDA_OK(cudaMemcpyAsync(c->flag_h, &c->OC->done, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        CHECK(sync(c));
        if (c->flag_h[0]) break;
        if (passes >= OC_MAX_PASSES) return set_error(T3D_ERR_NUMERIC, "OC bisection did not terminate");
    }
    launch_oc_finish(c->g, c->solid, c->x, c->xnew, c->OC, fp64, c->ne, c->slot[0], c->slot[1], c->st);
    c->launches += 3 + (fp64 ? 0 : 1);
    if (!fp64) launch_oc_vec8_stats(c->ne, c->morton, c->x, c->OC, c->st);
    CHECK(launch_check("oc finish"));
    T3D_CUDA_OK(cudaMemcpyAsync(c->OC_h, c->OC, sizeof(OcState), cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

// ------------------------------------------------------------------ design loop (driver.cpp:60-216)
static int fill_cells(Context* c, float v) {
    std::vector<float> h((size_t)c->ne, v);
    return upload_cells_f32(c, h.data(), c->x);
}

// Solves every load case on c->E and leaves the element compliance in c->ce and its E-weighted sum in
// *C.  Several cases (external models): each is solved from its own previous displacement, and
// ce = sum_k ce_k / K (TOP3D_XL.m:105,125,605-621); c->b and c->u are left holding case 0.
static int solve_all(Context* c, double tol, int maxit, int* iters, double* C) {
    const Grid& g = c->g;
    if (c->ncases == 1) {
        CHECK(solve(c, tol, maxit, iters));
        launch_compliance64(g, c->Ke, c->E, c->u, c->ce, c->slot[0], C, c->st);
        c->launches += 1;
        return T3D_OK;
    }
    const int64_t n3 = 3 * g.NN;
    const size_t bytes = n3 * sizeof(double);
    const double w = 1.0 / c->ncases;
    int total = 0;
    for (int k = 0; k < c->ncases; ++k) {
        T3D_CUDA_OK(cudaMemcpyAsync(c->b, c->b_cases + k * n3, bytes, cudaMemcpyDeviceToDevice, c->st));
        T3D_CUDA_OK(cudaMemcpyAsync(c->u, c->u_cases + k * n3, bytes, cudaMemcpyDeviceToDevice, c->st));
        int its = 0;
        CHECK(solve(c, tol, maxit, &its));
        total += its;
        T3D_CUDA_OK(cudaMemcpyAsync(c->u_cases + k * n3, c->u, bytes, cudaMemcpyDeviceToDevice, c->st));
        launch_compliance64(g, c->Ke, c->E, c->u, c->ce, c->slot[0], c->scal + 3, c->st);
        launch_cells_axpy(g.NE, k == 0, w, c->ce, c->ce_acc, c->st);
        c->launches += 2;
    }
    T3D_CUDA_OK(cudaMemcpyAsync(c->ce, c->ce_acc, g.NE * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    launch_objective(g, c->E, c->ce, c->one, c->slot[0], C, c->st);   // sum E ce
    T3D_CUDA_OK(cudaMemcpyAsync(c->b, c->b_cases, bytes, cudaMemcpyDeviceToDevice, c->st));
    T3D_CUDA_OK(cudaMemcpyAsync(c->u, c->u_cases, bytes, cudaMemcpyDeviceToDevice, c->st));
    c->launches += 1;
    *iters = total;
    return launch_check("load cases");
}

int design_init(Context* c, float V0, double* Csolid) {
    CHECK(ensure_morton(c));
    c->V0 = V0;
    c->loop = 0;
    CHECK(fill_cells(c, V0));
    {   // eleMod = E0 for every element for the solid reference solve (driver.cpp:67, 85-103)
        std::vector<double> e((size_t)c->ne, (double)c->prm.E0);
        CHECK(upload_cells_f64(c, e.data(), c->E));
    }
    T3D_CUDA_OK(cudaMemsetAsync(c->u, 0, 3 * c->g.NN * sizeof(double), c->st));
    if (c->ncases > 1)
        T3D_CUDA_OK(cudaMemsetAsync(c->u_cases, 0, (size_t)c->ncases * 3 * c->g.NN * sizeof(double), c->st));
    T3D_CUDA_OK(cudaMemsetAsync(c->flastx, 0, c->g.NN * sizeof(double), c->st));
    T3D_CUDA_OK(cudaMemsetAsync(c->flastrhs, 0, c->g.NN * sizeof(double), c->st));
    CHECK(mg_setup(c));
    int its = 0;
    CHECK(solve_all(c, (double)c->prm.cg_tol, c->prm.cg_max_it, &its, c->scal + 1));
    CHECK(launch_check("solid compliance"));
    T3D_CUDA_OK(cudaMemcpyAsync(c->scal_h, c->scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CHECK(sync(c));
    if (Csolid) *Csolid = c->scal_h[1];
    c->design_ready = true;
    return T3D_OK;
}

int design_pre(Context* c) {
    if (!c->design_ready) return set_error(T3D_ERR_INVALID, "t3d_design_init not called");
    const t3d_params& P = c->prm;
    ++c->loop;
    T3D_CUDA_OK(cudaEventRecord(c->ev[2], c->st));
    launch_simp(c->g, c->solid, c->x, P.E0, P.Emin, P.penal, c->E, c->st);
    c->launches += 4;   // simp, objective, sensitivities, dc scale
    if (!c->mg_ready || c->loop == 1 || c->loop % c->prm.mg_rebuild_period == 0) CHECK(mg_setup(c));
    return T3D_OK;
}

static int design_step(Context* c, t3d_iter_record* rec) {
    CHECK(design_pre(c));
    int its = 0;
    CHECK(solve_all(c, (double)c->prm.cg_tol, c->prm.cg_max_it, &its, c->scal + 0));
    return design_post(c, its, rec);
}

int design_post(Context* c, int its, t3d_iter_record* rec) {
    const Grid& g = c->g;
    const t3d_params& P = c->prm;
    cudaEvent_t e0 = c->ev[2], e1 = c->ev[3], e2 = c->ev[4], e3 = c->ev[5], e4 = c->ev[6];
    T3D_CUDA_OK(cudaEventRecord(e1, c->st));
    launch_objective(g, c->E, c->ce, c->scal + 1, c->slot[1], c->scal + 2, c->st);
    launch_sens(g, c->solid, c->x, c->ce, c->scal + 1, P.E0, P.Emin, P.penal, c->dc, c->xdc, c->st);
    CHECK(launch_check("sensitivities"));
    T3D_CUDA_OK(cudaEventRecord(e2, c->st));
    CHECK(filter_apply(c, c->xdc, c->dcf));
    T3D_CUDA_OK(cudaEventRecord(e3, c->st));
    launch_dc_scale(g, c->solid, c->dcf, c->x, c->dc, c->st);
    CHECK(oc_update(c, c->V0));
    T3D_CUDA_OK(cudaEventRecord(e4, c->st));
    T3D_CUDA_OK(cudaMemcpyAsync(c->scal_h, c->scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CHECK(sync(c));
    if (rec) {
        float tcg = 0, topt1 = 0, tf = 0, topt2 = 0;
        cudaEventElapsedTime(&tcg, e0, e1);
        cudaEventElapsedTime(&topt1, e1, e2);
        cudaEventElapsedTime(&tf, e2, e3);
        cudaEventElapsedTime(&topt2, e3, e4);
        rec->loop = c->loop;
        rec->pcg_iters = its;
        rec->obj = c->scal_h[2];
        rec->vol = c->OC_h->volfrac;
        rec->sharp = c->OC_h->sharp;
        rec->cons = c->OC_h->volfrac - c->V0;
        rec->change = c->OC_h->change;
        rec->lmid = c->OC_h->lmid;
        rec->bisections = c->OC_h->passes;
        rec->t_cg = tcg * 1e-3;
        rec->t_filter = tf * 1e-3;
        rec->t_opt = (topt1 + tf + topt2) * 1e-3;
        rec->t_total = (tcg + topt1 + tf + topt2) * 1e-3;
    }
    return T3D_OK;
}

}  // namespace t3d

// ====================================================================== C-ABI

#define API_GUARD(ctx)                                                                  \
    if (!(ctx)) return t3d::set_error(T3D_ERR_INVALID, "null context");                \
    if (cudaSetDevice((ctx)->dev) != cudaSuccess) return t3d::set_error(T3D_ERR_CUDA, "cudaSetDevice failed")

extern "C" {

int t3d_params_default(t3d_params* p) {
    if (!p) return t3d::set_error(T3D_ERR_INVALID, "null params");
    std::memset(p, 0, sizeof *p);
    p->E0 = 1.0f; p->Emin = 1.0e-6f; p->nu = 0.3f; p->penal = 3.0f;     // core.hpp:28-31
    p->cg_tol = 1.0e-3f; p->cg_max_it = 800;                             // core.hpp:35-36
    p->mg_nondyadic = 1; p->mg_max_levels = 5; p->mg_weight = 0.6f;      // driver.cpp:54
    p->mg_standard_weight = 0.35f;
    p->mg_rebuild_period = 5;                                            // driver.cpp:132
    p->filter_rmin = std::sqrt(3.0f);                                    // top3d_cli.cpp:33
    p->oc_sum_order = T3D_SUM_REFERENCE;
    p->precision = T3D_FP64;
    p->device = 0;
    return T3D_OK;
}

const char* t3d_last_error(void) { return t3d::g_err.c_str(); }

int t3d_create_problem(int nely, int nelx, int nelz, const t3d_params* p, const t3d_problem* problem,
                       t3d_context** out) {
    if (!out || !problem) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    *out = nullptr;
    t3d_context* c = new (std::nothrow) t3d_context();
    if (!c) return t3d::set_error(T3D_ERR_OOM, "host allocation failed");
    int rc = t3d::create(nely, nelx, nelz, p, problem, c);
    if (rc != T3D_OK) {
        delete c;
        return rc;
    }
    *out = c;
    return T3D_OK;
}

int t3d_topvoxel_info(const char* path, int64_t* info) {
    if (!path || !info) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    t3d::VoxelModel m;
    std::string err;
    if (!t3d::parse_topvoxel(path, &m, &err)) return t3d::set_error(T3D_ERR_INVALID, err);
    const int64_t v[8] = {m.nelx, m.nely, m.nelz, m.num_solid, m.num_passive, (int64_t)m.fix_node.size(),
                          (int64_t)m.load_node.size(), m.num_additional_loads};
    std::memcpy(info, v, sizeof v);
    return T3D_OK;
}

int t3d_create_from_topvoxel(const char* path, const t3d_params* p, t3d_context** out) {
    if (!out || !path) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    *out = nullptr;
    auto m = std::make_shared<t3d::VoxelModel>();
    std::string err;
    if (!t3d::parse_topvoxel(path, m.get(), &err)) return t3d::set_error(T3D_ERR_INVALID, err);
    if (m->fix_node.empty())
        return t3d::set_error(T3D_ERR_INVALID, "TopVoxel file fixes no DOF: the stiffness would be singular");
    if (m->load_node.empty()) return t3d::set_error(T3D_ERR_INVALID, "TopVoxel file has no loads");
    t3d_context* c = new (std::nothrow) t3d_context();
    if (!c) return t3d::set_error(T3D_ERR_OOM, "host allocation failed");
    c->vox = m;
    int rc = t3d::create(m->nely, m->nelx, m->nelz, p, nullptr, c);
    if (rc != T3D_OK) {
        delete c;
        return rc;
    }
    *out = c;
    return T3D_OK;
}

int t3d_create(int nely, int nelx, int nelz, const t3d_params* p, t3d_context** out) {
    if (!out) return t3d::set_error(T3D_ERR_INVALID, "null output pointer");
    *out = nullptr;
    t3d_context* c = new (std::nothrow) t3d_context();
    if (!c) return t3d::set_error(T3D_ERR_OOM, "host allocation failed");
    int rc = t3d::create(nely, nelx, nelz, p, nullptr, c);
    if (rc != T3D_OK) {
        delete c;
        return rc;
    }
    *out = c;
    return T3D_OK;
}

int t3d_destroy(t3d_context* ctx) {
    if (!ctx) return T3D_OK;
    cudaSetDevice(ctx->dev);
    cudaStreamSynchronize(ctx->st);
    delete ctx;
    return T3D_OK;
}

int t3d_get_info(const t3d_context* ctx, t3d_info* info) {
    if (!ctx || !info) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    std::memset(info, 0, sizeof *info);
    info->res[0] = ctx->g.nx; info->res[1] = ctx->g.ny; info->res[2] = ctx->g.nz;
    info->orig[0] = ctx->cub.nelx; info->orig[1] = ctx->cub.nely; info->orig[2] = ctx->cub.nelz;
    info->num_elements = ctx->ne;
    info->num_nodes = ctx->g.NN;
    // free DOFs: nodes used by a solid element and not on the x=0 face (the built-in cuboid), else counted
    if (ctx->voids.n == 0 && !ctx->vox) {
        const int64_t ux = ctx->cub.nelx + 1, uy = ctx->cub.nely + 1, uz = ctx->cub.nelz + 1;
        info->num_free = 3 * (ux - 1) * uy * uz;
    } else {
        t3d_context* mc = const_cast<t3d_context*>(ctx);   // the free-DOF list is a lazily built cache
        CHECK(t3d::ensure_free(mc));
        info->num_free = (int64_t)mc->free_h.size();
    }
    info->num_levels = ctx->nlev;
    for (int l = 0; l < ctx->nlev; ++l) {
        info->levels[l][0] = ctx->lv[l].nx; info->levels[l][1] = ctx->lv[l].ny;
        info->levels[l][2] = ctx->lv[l].nz; info->levels[l][3] = ctx->lv[l].span;
    }
    info->coarse_n = ctx->Nc;
    int st = 0;
    if (ctx->Nc && ctx->mg_ready) cudaMemcpy(&st, ctx->chol_status, sizeof(int), cudaMemcpyDeviceToHost);
    info->coarse_cholesky_ok = st;
    info->device_bytes = (int64_t)ctx->bytes;
    info->kernel_launches = ctx->launches;
    info->matvec32_modal = ctx->modal ? 1 : 0;
    info->matvec64_kernel = !ctx->mv64_stream ? 0 : ctx->ke_pat ? 2 : 1;
    if (ctx->mixed) {
        int d[4];
        t3d::modal_variant_desc(ctx->mt.variant, d);
        for (int k = 0; k < 4; ++k) info->matvec32_tile[k] = d[k];
        info->matvec32_variant = ctx->mt.variant;
        info->last_outer_passes = ctx->last_outer;
    }
    return T3D_OK;
}

int t3d_voxel_ke(double nu, double cell_size, double* ke) {
    if (!ke) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    if (!(cell_size > 0.0) || !std::isfinite(cell_size) || !(nu > -1.0 && nu < 0.5))
        return t3d::set_error(T3D_ERR_INVALID, "need cell_size > 0 and -1 < nu < 0.5");
    t3d::hex8_stiffness(nu, cell_size, ke);
    return T3D_OK;
}

int t3d_get_ke(const t3d_context* ctx, double* ke) {
    if (!ctx || !ke) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    std::memcpy(ke, ctx->Ke_h, sizeof ctx->Ke_h);
    return T3D_OK;
}

int t3d_set_ke(t3d_context* ctx, const double* ke) {
    API_GUARD(ctx);
    if (!ke) return t3d::set_error(T3D_ERR_INVALID, "null Ke");
    std::memcpy(ctx->Ke_h, ke, sizeof ctx->Ke_h);
    T3D_CUDA_OK(cudaMemcpy(ctx->Ke, ctx->Ke_h, sizeof ctx->Ke_h, cudaMemcpyHostToDevice));
    CHECK(t3d::update_ke_pattern(ctx));
    if (ctx->standard) CHECK(t3d::upload_gpos(ctx));   // the Standard V-cycle's level-1 Galerkin products
    ctx->mg_ready = false;   // the hierarchy was built with the old Ke: rebuilt by the next design step or t3d_mg_setup
    T3D_CUDA_OK(cudaStreamSynchronize(ctx->st));
    if (ctx->Ke32) {
        float k32[576];
        for (int i = 0; i < 576; ++i) k32[i] = (float)ctx->Ke_h[i];
        T3D_CUDA_OK(cudaMemcpy(ctx->Ke32, k32, sizeof k32, cudaMemcpyHostToDevice));
        ctx->modal = ctx->prm.matvec32_form == T3D_MATVEC32_AUTO &&
                     t3d::modal_ke_from(ctx->Ke_h, &ctx->kh, &ctx->modal_off);
    }
    // the captured PCG iterations hold Ke (FP64 streaming form) and the modal coefficients by value
    if (ctx->pcg_graph) cudaGraphExecDestroy(ctx->pcg_graph);
    if (ctx->pcg32_graph) cudaGraphExecDestroy(ctx->pcg32_graph);
    ctx->pcg_graph = nullptr;
    ctx->pcg32_graph = nullptr;
    return T3D_OK;
}

int t3d_get_element_map(t3d_context* ctx, int32_t* out) {
    API_GUARD(ctx);
    if (!out) return t3d::set_error(T3D_ERR_INVALID, "null output");
    CHECK(t3d::ensure_morton(ctx));
    const t3d::Grid& g = ctx->g;
    for (int64_t k = 0; k < ctx->ne; ++k) {   // grid cell -> reference full index ny*nx*ez + ny*ex + (ny-1-ey)
        const int64_t ci = ctx->morton_h[k];
        const int cx = (int)(ci % g.ex) - 1, cy = (int)((ci / g.ex) % g.ey) - 1, cz = (int)(ci / ((int64_t)g.ex * g.ey)) - 1;
        out[k] = (int32_t)((int64_t)g.ny * g.nx * cz + (int64_t)g.ny * cx + cy);
    }
    return T3D_OK;
}

int t3d_get_free_dofs(t3d_context* ctx, int32_t* out) {
    API_GUARD(ctx);
    if (!out) return t3d::set_error(T3D_ERR_INVALID, "null output");
    CHECK(t3d::ensure_free(ctx));
    std::memcpy(out, ctx->free_h.data(), ctx->free_h.size() * sizeof(int32_t));
    return T3D_OK;
}

int t3d_get_load(t3d_context* ctx, double* b) {
    API_GUARD(ctx);
    if (!b) return t3d::set_error(T3D_ERR_INVALID, "null output");
    return t3d::download_free(ctx, ctx->b, b);
}

int t3d_matvec(t3d_context* ctx, const double* E, const double* u, double* y) {
    API_GUARD(ctx);
    if (!E || !u || !y) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    CHECK(t3d::upload_cells_f64(ctx, E, ctx->E));
    CHECK(t3d::upload_free(ctx, u, ctx->p));
    ctx->launches += t3d::matvec64(ctx, ctx->p, ctx->Ap, t3d::RedSlot{nullptr, nullptr}, nullptr);
    CHECK(t3d::launch_check("matvec"));
    return t3d::download_free(ctx, ctx->Ap, y);
}

int t3d_matvec32(t3d_context* ctx, const double* E, const double* u, double* y) {
    API_GUARD(ctx);
    if (!E || !u || !y) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    if (!ctx->mixed) return t3d::set_error(T3D_ERR_INVALID, "FP32 kernels need precision T3D_MIXED");
    CHECK(t3d::upload_cells_f64(ctx, E, ctx->E));
    CHECK(t3d::upload_free(ctx, u, ctx->p));
    t3d::launch_cells_to32(ctx->g, ctx->E, ctx->E32, ctx->st);
    t3d::launch_nodes_to32(ctx->g, ctx->p, ctx->p32, ctx->st);
    ctx->launches += 2;
    t3d::matvec32(ctx, ctx->p32, ctx->Ap32, t3d::RedSlot{nullptr, nullptr}, nullptr);
    t3d::launch_nodes_from32(ctx->g, ctx->Ap32, ctx->Ap, ctx->st);
    ctx->launches += 1;
    CHECK(t3d::launch_check("matvec32"));
    CHECK(t3d::check_tma(ctx));
    return t3d::download_free(ctx, ctx->Ap, y);
}

int t3d_mg_setup(t3d_context* ctx, const double* E) {
    API_GUARD(ctx);
    if (!E) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    CHECK(t3d::upload_cells_f64(ctx, E, ctx->E));
    CHECK(t3d::mg_setup(ctx));
    return t3d::sync(ctx);
}

int t3d_vcycle(t3d_context* ctx, const double* r, double* z) {
    API_GUARD(ctx);
    if (!r || !z) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    if (!ctx->mg_ready) return t3d::set_error(T3D_ERR_INVALID, "t3d_mg_setup not called");
    CHECK(t3d::upload_free(ctx, r, ctx->r));
    T3D_CUDA_OK(cudaMemsetAsync(ctx->S, 0, sizeof(t3d::PcgScalars), ctx->st));
    t3d::vcycle(ctx, ctx->r, ctx->z, ctx->S, ctx->slot[2]);
    CHECK(t3d::launch_check("vcycle"));
    return t3d::download_free(ctx, ctx->z, z);
}

int t3d_vcycle32(t3d_context* ctx, const double* r, double* z) {
    API_GUARD(ctx);
    if (!r || !z) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    if (!ctx->mixed) return t3d::set_error(T3D_ERR_INVALID, "FP32 kernels need precision T3D_MIXED");
    if (!ctx->mg_ready) return t3d::set_error(T3D_ERR_INVALID, "t3d_mg_setup not called");
    CHECK(t3d::upload_free(ctx, r, ctx->r));
    t3d::launch_nodes_to32(ctx->g, ctx->r, ctx->r32, ctx->st);
    T3D_CUDA_OK(cudaMemsetAsync(ctx->S32, 0, sizeof(t3d::PcgScalars), ctx->st));
    ctx->launches += 1;
    t3d::vcycle32(ctx, ctx->r32, ctx->z32, ctx->S32, ctx->slot[2]);
    t3d::launch_nodes_from32(ctx->g, ctx->z32, ctx->z, ctx->st);
    ctx->launches += 1;
    CHECK(t3d::launch_check("vcycle32"));
    return t3d::download_free(ctx, ctx->z, z);
}

int t3d_pcg(t3d_context* ctx, const double* E, const double* b, double* x, double tol, int max_it, int* iters) {
    API_GUARD(ctx);
    if (!E || !b || !x || max_it < 0) return t3d::set_error(T3D_ERR_INVALID, "bad argument");
    if (!ctx->mg_ready) return t3d::set_error(T3D_ERR_INVALID, "t3d_mg_setup not called");
    // the preconditioner keeps the moduli it was built with; the operator uses E
    CHECK(t3d::upload_cells_f64(ctx, E, ctx->E));
    CHECK(t3d::upload_free(ctx, b, ctx->b));
    CHECK(t3d::upload_free(ctx, x, ctx->u));
    int its = 0;
    CHECK(t3d::pcg_solve(ctx, tol, max_it, &its));
    if (iters) *iters = its;
    CHECK(t3d::download_free(ctx, ctx->u, x));
    // restore the context's load for later design iterations
    CHECK(t3d::setup_load(ctx));
    return t3d::sync(ctx);
}

int t3d_compliance(t3d_context* ctx, const double* E, const double* u, double* ce, double* C) {
    API_GUARD(ctx);
    if (!E || !u) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    CHECK(t3d::upload_cells_f64(ctx, E, ctx->E));
    CHECK(t3d::upload_free(ctx, u, ctx->u));
    t3d::launch_compliance64(ctx->g, ctx->Ke, ctx->E, ctx->u, ctx->ce, ctx->slot[0], ctx->scal + 3, ctx->st);
    CHECK(t3d::launch_check("compliance"));
    if (ce) CHECK(t3d::download_cells_f64(ctx, ctx->ce, ce));
    T3D_CUDA_OK(cudaMemcpyAsync(ctx->scal_h, ctx->scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CHECK(t3d::sync(ctx));
    if (C) *C = ctx->scal_h[3];
    return T3D_OK;
}

int t3d_mg_get_diag(t3d_context* ctx, int level, double* out) {
    API_GUARD(ctx);
    if (!out || level < 0 || level >= ctx->nlev) return t3d::set_error(T3D_ERR_INVALID, "bad level");
    const t3d::MgLevel& L = ctx->lv[level];
    std::vector<double> soa(3 * L.nn);
    T3D_CUDA_OK(cudaMemcpy(soa.data(), L.diag, soa.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int64_t n = 0; n < L.nn; ++n)
        for (int c = 0; c < 3; ++c) out[3 * n + c] = soa[c * L.nn + n];
    return T3D_OK;
}

int t3d_mg_get_mask(t3d_context* ctx, int level, uint8_t* out) {
    API_GUARD(ctx);
    if (!out || level < 0 || level >= ctx->nlev) return t3d::set_error(T3D_ERR_INVALID, "bad level");
    const t3d::MgLevel& L = ctx->lv[level];
    std::vector<uint8_t> m(L.nn);
    T3D_CUDA_OK(cudaMemcpy(m.data(), L.mask, L.nn, cudaMemcpyDeviceToHost));
    for (int64_t n = 0; n < L.nn; ++n)
        for (int c = 0; c < 3; ++c) out[3 * n + c] = (m[n] >> c) & 1;
    return T3D_OK;
}

int t3d_mg_coarse_matrix(t3d_context* ctx, const double* E, double* Kc) {
    API_GUARD(ctx);
    if (!E || !Kc) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    if (!ctx->Nc) return t3d::set_error(T3D_ERR_UNSUPPORTED, "coarsest level uses the Jacobi fallback");
    CHECK(t3d::upload_cells_f64(ctx, E, ctx->E));
    CHECK(t3d::mg_setup(ctx));
    T3D_CUDA_OK(cudaMemcpyAsync(Kc, ctx->Kc, (size_t)ctx->Nc * ctx->Nc * sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->st));
    return t3d::sync(ctx);
}

int t3d_filter_apply(t3d_context* ctx, const float* src, float* dst) {
    API_GUARD(ctx);
    if (!src || !dst) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    CHECK(t3d::upload_cells_f32(ctx, src, ctx->xdc));
    CHECK(t3d::filter_apply(ctx, ctx->xdc, ctx->dcf));
    return t3d::download_cells_f32(ctx, ctx->dcf, dst);
}

int t3d_filter_setup(t3d_context* ctx, float rmin) {
    API_GUARD(ctx);
    if (!(rmin > 0.0f) || !std::isfinite(rmin)) return t3d::set_error(T3D_ERR_INVALID, "filter radius must be positive");
    ctx->prm.filter_rmin = rmin;
    double kf[72];
    t3d::filter_kernel(rmin, kf);
    T3D_CUDA_OK(cudaMemcpyAsync(ctx->kf, kf, sizeof kf, cudaMemcpyHostToDevice, ctx->st));
    t3d::launch_filter_diag(ctx->g, ctx->solid, ctx->kf, ctx->fdiag, ctx->st);
    CHECK(t3d::launch_check("filter set-up"));
    T3D_CUDA_OK(cudaMemsetAsync(ctx->flastx, 0, ctx->g.NN * sizeof(double), ctx->st));
    T3D_CUDA_OK(cudaMemsetAsync(ctx->flastrhs, 0, ctx->g.NN * sizeof(double), ctx->st));
    return t3d::sync(ctx);
}

int t3d_filter_get_state(t3d_context* ctx, double* last_x, double* last_rhs, double* diag) {
    API_GUARD(ctx);
    const size_t nb = ctx->g.NN * sizeof(double);
    if (last_x) T3D_CUDA_OK(cudaMemcpy(last_x, ctx->flastx, nb, cudaMemcpyDeviceToHost));
    if (last_rhs) T3D_CUDA_OK(cudaMemcpy(last_rhs, ctx->flastrhs, nb, cudaMemcpyDeviceToHost));
    if (diag) T3D_CUDA_OK(cudaMemcpy(diag, ctx->fdiag, nb, cudaMemcpyDeviceToHost));
    return T3D_OK;
}

int t3d_filter_set_state(t3d_context* ctx, const double* last_x, const double* last_rhs) {
    API_GUARD(ctx);
    if (!last_x || !last_rhs) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    const size_t nb = ctx->g.NN * sizeof(double);
    T3D_CUDA_OK(cudaMemcpy(ctx->flastx, last_x, nb, cudaMemcpyHostToDevice));
    T3D_CUDA_OK(cudaMemcpy(ctx->flastrhs, last_rhs, nb, cudaMemcpyHostToDevice));
    return T3D_OK;
}

int t3d_simp(t3d_context* ctx, const float* xphys, double* E) {
    API_GUARD(ctx);
    if (!xphys || !E) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    CHECK(t3d::upload_cells_f32(ctx, xphys, ctx->x));
    t3d::launch_simp(ctx->g, ctx->solid, ctx->x, ctx->prm.E0, ctx->prm.Emin, ctx->prm.penal, ctx->E, ctx->st);
    CHECK(t3d::launch_check("simp"));
    return t3d::download_cells_f64(ctx, ctx->E, E);
}

int t3d_sensitivity(t3d_context* ctx, const float* xphys, const double* ce, double c_solid, float* dc) {
    API_GUARD(ctx);
    if (!xphys || !ce || !dc) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    CHECK(t3d::upload_cells_f32(ctx, xphys, ctx->x));
    CHECK(t3d::upload_cells_f64(ctx, ce, ctx->ce));
    T3D_CUDA_OK(cudaMemcpy(ctx->scal + 4, &c_solid, sizeof(double), cudaMemcpyHostToDevice));
    t3d::launch_sens(ctx->g, ctx->solid, ctx->x, ctx->ce, ctx->scal + 4, ctx->prm.E0, ctx->prm.Emin, ctx->prm.penal,
                     ctx->dc, ctx->xdc, ctx->st);
    CHECK(t3d::launch_check("sensitivity"));
    return t3d::download_cells_f32(ctx, ctx->dc, dc);
}

int t3d_dc_scale(t3d_context* ctx, const float* dcf, const float* x, float* dc) {
    API_GUARD(ctx);
    if (!dcf || !x || !dc) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    CHECK(t3d::upload_cells_f32(ctx, dcf, ctx->dcf));
    CHECK(t3d::upload_cells_f32(ctx, x, ctx->x));
    t3d::launch_dc_scale(ctx->g, ctx->solid, ctx->dcf, ctx->x, ctx->dc, ctx->st);
    CHECK(t3d::launch_check("dc_scale"));
    return t3d::download_cells_f32(ctx, ctx->dc, dc);
}

int t3d_oc_update(t3d_context* ctx, const float* x, const float* dc, float V0, float* xnew, float* change,
                  float* lmid, int* bis) {
    API_GUARD(ctx);
    if (!x || !dc || !xnew) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    CHECK(t3d::upload_cells_f32(ctx, x, ctx->x));
    CHECK(t3d::upload_cells_f32(ctx, dc, ctx->dc));
    CHECK(t3d::oc_update(ctx, V0));
    if (change) *change = ctx->OC_h->change;
    if (lmid) *lmid = ctx->OC_h->lmid;
    if (bis) *bis = ctx->OC_h->passes;
    return t3d::download_cells_f32(ctx, ctx->x, xnew);
}

int t3d_design_init(t3d_context* ctx, float V0, double* c_solid) {
    API_GUARD(ctx);
    return t3d::design_init(ctx, V0, c_solid);
}

int t3d_design_step(t3d_context* ctx, t3d_iter_record* rec) {
    API_GUARD(ctx);
    return t3d::design_step(ctx, rec);
}

int t3d_design_step_host(t3d_context* ctx, const float* x_in, float* x_out, t3d_iter_record* rec) {
    API_GUARD(ctx);
    if (!x_in || !x_out) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    CHECK(t3d::upload_cells_f32(ctx, x_in, ctx->x));
    CHECK(t3d::design_step(ctx, rec));
    return t3d::download_cells_f32(ctx, ctx->x, x_out);
}

int t3d_get_density(t3d_context* ctx, float* x) {
    API_GUARD(ctx);
    if (!x) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    return t3d::download_cells_f32(ctx, ctx->x, x);
}

int t3d_get_displacement(t3d_context* ctx, double* u) {
    API_GUARD(ctx);
    if (!u) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    return t3d::download_free(ctx, ctx->u, u);
}

int t3d_set_density(t3d_context* ctx, const float* x) {
    API_GUARD(ctx);
    if (!x) return t3d::set_error(T3D_ERR_INVALID, "null argument");
    CHECK(t3d::upload_cells_f32(ctx, x, ctx->x));
    return t3d::sync(ctx);
}

int t3d_run_global(t3d_context* ctx, float V0, int n_loop, double* c_solid, t3d_iter_record* records, int* n_records,
                   float* x_final) {
    API_GUARD(ctx);
    CHECK(t3d::design_init(ctx, V0, c_solid));
    float change = 1.0f, sharp = 1.0f;
    int n = 0;
    while (n < n_loop && change > 1e-4 && sharp > 0.01) {   // driver.cpp:112
        t3d_iter_record rec;
        CHECK(t3d::design_step(ctx, &rec));
        change = rec.change;
        sharp = rec.sharp;
        if (records) records[n] = rec;
        ++n;
    }
    if (n_records) *n_records = n;
    if (x_final) CHECK(t3d::download_cells_f32(ctx, ctx->x, x_final));
    return T3D_OK;
}

int t3d_synchronize(t3d_context* ctx) {
    API_GUARD(ctx);
    return t3d::sync(ctx);
}

int t3d_profile(t3d_context* ctx, int what, int reps, double* ms) {
    API_GUARD(ctx);
    if (reps <= 0 || !ms || what < T3D_PROFILE_MATVEC || what > T3D_PROFILE_VCYCLE32)
        return t3d::set_error(T3D_ERR_INVALID, "bad profile request");
    if (what != T3D_PROFILE_MATVEC && !ctx->mg_ready) return t3d::set_error(T3D_ERR_INVALID, "MG not set up");
    if (what >= T3D_PROFILE_MATVEC32 && !ctx->mixed)
        return t3d::set_error(T3D_ERR_INVALID, "FP32 kernels need precision T3D_MIXED");
    T3D_CUDA_OK(cudaMemsetAsync(ctx->S, 0, sizeof(t3d::PcgScalars), ctx->st));
    if (ctx->mixed) {   // the FP32 kernels see the FP32 images of the current E, p and r
        T3D_CUDA_OK(cudaMemsetAsync(ctx->S32, 0, sizeof(t3d::PcgScalars), ctx->st));
        t3d::launch_cells_to32(ctx->g, ctx->E, ctx->E32, ctx->st);
        t3d::launch_nodes_to32(ctx->g, ctx->p, ctx->p32, ctx->st);
        t3d::launch_nodes_to32(ctx->g, ctx->r, ctx->r32, ctx->st);
    }
    auto once = [&]() {
        if (what == T3D_PROFILE_MATVEC) {
            ctx->launches += t3d::matvec64(ctx, ctx->p, ctx->Ap, ctx->slot[0], ctx->S);
        } else if (what == T3D_PROFILE_VCYCLE) {
            t3d::vcycle(ctx, ctx->r, ctx->z, ctx->S, ctx->slot[2]);
        } else if (what == T3D_PROFILE_MATVEC32) {
            t3d::matvec32(ctx, ctx->p32, ctx->Ap32, ctx->slot[0], ctx->S32);
        } else {
            t3d::vcycle32(ctx, ctx->r32, ctx->z32, ctx->S32, ctx->slot[2]);
        }
    };
    once();
    T3D_CUDA_OK(cudaEventRecord(ctx->ev[6], ctx->st));
    for (int k = 0; k < reps; ++k) once();
    T3D_CUDA_OK(cudaEventRecord(ctx->ev[7], ctx->st));
    CHECK(t3d::launch_check("profile"));
    T3D_CUDA_OK(cudaEventSynchronize(ctx->ev[7]));
    float t = 0;
    T3D_CUDA_OK(cudaEventElapsedTime(&t, ctx->ev[6], ctx->ev[7]));
    *ms = (double)t / reps;
    return ctx->mixed ? t3d::check_tma(ctx) : T3D_OK;
}

int t3d_export_stl(t3d_context* ctx, const float* xphys, float iso, const char* path, int64_t* ntri) {
    API_GUARD(ctx);
    if (!path) return t3d::set_error(T3D_ERR_INVALID, "null path");
    const t3d::Grid& g = ctx->g;
    const float* dens = ctx->x;
    if (xphys) {   // densities given in the reference's element order: staged into xnew (cells)
        CHECK(t3d::upload_cells_f32(ctx, xphys, ctx->xnew));
        dens = ctx->xnew;
    }
    const int nb = t3d::stl_chunks(g);
    unsigned* bsum = nullptr;
    uint16_t* body = nullptr;
    unsigned faces = 0;
    int rc = T3D_OK;
    cudaError_t e = cudaMalloc(&bsum, (size_t)(nb + 1) * sizeof(unsigned));
    if (e != cudaSuccess) return t3d::set_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
    t3d::launch_stl_count(g, dens, iso, bsum, ctx->st);
    e = cudaMemcpyAsync(&faces, bsum + nb, sizeof faces, cudaMemcpyDeviceToHost, ctx->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    const int64_t n_tri = 2 * (int64_t)faces;
    std::vector<char> host;
    if (e == cudaSuccess && n_tri > 0) {
        e = cudaMalloc(&body, (size_t)n_tri * 50);
        if (e == cudaSuccess) {
            t3d::launch_stl_write(g, dens, iso, bsum, body, ctx->st);
            host.resize((size_t)n_tri * 50);
            e = cudaMemcpyAsync(host.data(), body, host.size(), cudaMemcpyDeviceToHost, ctx->st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
        }
    }
    if (e != cudaSuccess) rc = t3d::set_cuda_error(e, "stl export", __FILE__, __LINE__);
    cudaFree(bsum);
    if (body) cudaFree(body);
    if (rc != T3D_OK) return rc;
    // export_stl.hpp:14-33: 80-byte header, triangle count, records
    FILE* f = std::fopen(path, "wb");
    if (!f) return t3d::set_error(T3D_ERR_INVALID, std::string("cannot open ") + path);
    char header[80] = {0};
    std::strncpy(header, "Generated by TOP3D_XL", 79);
    const uint32_t n32 = (uint32_t)n_tri;
    bool ok = std::fwrite(header, 1, 80, f) == 80 && std::fwrite(&n32, 4, 1, f) == 1 &&
              (host.empty() || std::fwrite(host.data(), 1, host.size(), f) == host.size());
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return t3d::set_error(T3D_ERR_INVALID, std::string("write failed: ") + path);
    if (ntri) *ntri = n_tri;
    return T3D_OK;
}

}  // extern "C"
