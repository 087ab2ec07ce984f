/* Test infrastructure only -- CPU oracle (single-threaded C11 restatement) of the
 * per-design-iteration hot path of natashahirt/AlgorithmEngineering_AltProject.
 * See t3d_oracle.h for layouts and its role.  Every function cites the reference
 * file:line it restates (paths relative to the reference project root).
 *
 * Evaluation-order notes.  The reference is built with -O3 -ffast-math; where the
 * compiled reference evaluates an expression differently from its source text and the
 * difference is visible in float results, this oracle follows the compiled form and
 * says so (these were read off the x86 assembly of the reference build made here):
 *   - SIMP modulus uses a fused multiply-add (driver.cpp:120);
 *   - the sensitivity is ceNorm*(pw*((Emin-E0)*p)) with ceNorm=(float)(ce*(1/Csolid))
 *     (driver.cpp:151-157);
 *   - OC computes -dc*(2/(l1+l2)) instead of -dc/lmid and sums the volume with an
 *     8-lane vector reduction (driver.cpp:173-183).
 */
#define _GNU_SOURCE
#include "t3d_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <immintrin.h>

/* ------------------------------------------------------------------ structures */
typedef struct orc_level {
    int nx, ny, nz, span;
    int64_t nn;
    uint8_t* mask;   /* [3*nn] 1 = fixed */
    double* diag;    /* [3*nn] */
    double* r;       /* [3*nn] */
    double* x;       /* [3*nn] */
} orc_level;

struct orc_problem {
    orc_params p;
    int nelx, nely, nelz;          /* original element counts */
    int nx, ny, nz;                /* padded (resX,resY,resZ) */
    int nnx, nny, nnz;
    int64_t nn, ndof, nf;
    int ne;
    int32_t* ele_full;             /* [ne] full element index ny*nx*ez + ny*ex + (ny-1-ey) */
    int32_t* enod;                 /* [ne*8] */
    int32_t* bucket;               /* [ne] elements grouped by colour, Morton order inside */
    int32_t bucket_start[9];
    uint8_t* isfree;               /* [ndof] */
    int32_t* free_dofs;            /* [nf] */
    int32_t* dof2free;             /* [ndof] */
    double* F;                     /* [ndof] interleaved 3n+c */
    /* external model (TopVoxel, TOP3D_XL.m:458-586); NULL voxel = the built-in cuboid */
    const uint8_t* voxel;          /* [nelx*nely*nelz], k = y + nely*(x + nelx*z): 0 void, 1 solid, 2 passive */
    int nfix;                      /* fixations: file nodes m = y + (nely+1)*(x + (nelx+1)*z), DOF bits */
    const int64_t* fix_node;
    const uint8_t* fix_bits;
    int ncases;                    /* load cases; loads concatenated: case k has case_n[k] nodes */
    const int* case_n;
    const int64_t* load_node;
    const double* load_f;          /* 3 per loaded node */
    double* Fcases;                /* [ncases*ndof] when ncases > 1 */
    uint8_t* passive;              /* [ne] 1 = passive element (kept at 1 by the OC update) */
    double Ke[576];
    int nlev;
    orc_level lv[8];
    double* Lc;                    /* coarsest Cholesky factor, row-major, lower */
    double* Xc;                    /* red_mode 1: coarsest inverse, column j = solve(L L', e_j) */
    int Nc;                        /* 0 -> Jacobi coarsest */
    double* tmpf;                  /* [3*nn0] prolongation scratch */
    double *r, *z, *pp, *Ap;       /* PCG workspace [nf] */
    /* PDE filter */
    double kf[64];
    double* fdiag;
    double* flastx;
    double* flastrhs;
    double *frhs, *fx, *fr, *fz, *fp, *fAp;
    int filter_ready;
};

typedef double (*canon_step)(double part, int64_t item, const void* ctx);
static double canon_fold(int64_t nitems, canon_step step, const void* ctx);
static int32_t* cell_to_element(const orc_problem* P);

static void* xcalloc(size_t n, size_t sz) {
    void* p = calloc(n ? n : 1, sz);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}

/* ------------------------------------------------------------------ parameters */
void orc_params_default(orc_params* p) {
    /* GlobalParams defaults core.hpp:26-42; MG config driver.cpp:54 */
    p->E0 = 1.0f; p->Emin = 1.0e-6f; p->nu = 0.3f; p->penal = 3.0f;
    p->cg_tol = 1.0e-3f; p->cg_max_it = 800;
    p->mg_nondyadic = 1; p->mg_max_levels = 5; p->mg_weight = 0.6f;
    p->pow_mode = 0; p->vol_mode = 0; p->approx_mode = 0; p->red_mode = 0;
    p->coarse_full = 0;
}

/* ------------------------------------------------------------------ padding
 * padding.hpp:23-53: L = number of (n+4)/8 reductions while n >= 50000, at least 3;
 * each dimension is padded up to a multiple of 2^L. */
static int pad_levels(uint64_t nvox) {
    int L = 0;
    while (nvox >= 50000u) { ++L; nvox = (nvox + 4u) / 8u; }
    return L < 3 ? 3 : L;
}
static int pad_dim(int n, int L) {
    const int s = 1 << L;
    return ((n + s - 1) / s) * s;
}

/* ------------------------------------------------------------------ element stiffness
 * fea.cpp:117-179: unit-modulus hex8, 2x2x2 Gauss, Voigt order [xx,yy,zz,yz,xz,xy],
 * local DOF 3a+c, natural-coordinate node order (-,-,-),(+,-,-),(+,+,-),(-,+,-), then +z. */
static void hex8_stiffness(double nu, double h, double* Ke) {
    const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = 1.0 / (2.0 * (1.0 + nu));
    double D[6][6] = {{0}};
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) D[i][j] = lam;
        D[i][i] = lam + 2.0 * mu;
        D[3 + i][3 + i] = mu;
    }
    static const double sg[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    static const double tg[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    static const double pg[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    const double g = 1.0 / sqrt(3.0);
    const double detJ = (h * h * h) / 8.0;
    const double sc = 2.0 / h;
    memset(Ke, 0, 576 * sizeof(double));
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c) {
                const double s = a ? g : -g, t = b ? g : -g, q = c ? g : -g;
                double dx[8], dy[8], dz[8];
                for (int n = 0; n < 8; ++n) {
                    dx[n] = 0.125 * sg[n] * (1 + tg[n] * t) * (1 + pg[n] * q) * sc;
                    dy[n] = 0.125 * tg[n] * (1 + sg[n] * s) * (1 + pg[n] * q) * sc;
                    dz[n] = 0.125 * pg[n] * (1 + sg[n] * s) * (1 + tg[n] * t) * sc;
                }
                double B[6][24];
                memset(B, 0, sizeof B);
                for (int n = 0; n < 8; ++n) {
                    B[0][3 * n + 0] = dx[n];
                    B[1][3 * n + 1] = dy[n];
                    B[2][3 * n + 2] = dz[n];
                    B[3][3 * n + 1] = dz[n]; B[3][3 * n + 2] = dy[n];
                    B[4][3 * n + 0] = dz[n]; B[4][3 * n + 2] = dx[n];
                    B[5][3 * n + 0] = dy[n]; B[5][3 * n + 1] = dx[n];
                }
                double DB[6][24];
                for (int i = 0; i < 6; ++i)
                    for (int j = 0; j < 24; ++j) {
                        double acc = 0.0;
                        for (int k = 0; k < 6; ++k) acc += D[i][k] * B[k][j];
                        DB[i][j] = acc;
                    }
                for (int i = 0; i < 24; ++i)
                    for (int j = 0; j < 24; ++j) {
                        double acc = 0.0;
                        for (int k = 0; k < 6; ++k) acc += B[k][i] * DB[k][j];
                        Ke[i * 24 + j] += acc * detJ;
                    }
            }
}

/* ------------------------------------------------------------------ mesh
 * fea.cpp:181-358.  Element (ex,ey,ez) with ey counted from the top of the padded grid;
 * its local nodes in reference order sit at (ex+dx, ny-ey-1+dy, ez+dz) with
 * (dx,dy,dz) given by CORNER below (fea.cpp:257-264). */
static const int CORNER[8][3] = {{0, 1, 0}, {1, 1, 0}, {1, 0, 0}, {0, 0, 0},
                                 {0, 1, 1}, {1, 1, 1}, {1, 0, 1}, {0, 0, 1}};

static uint64_t spread_bits3(uint32_t v) {
    uint64_t r = 0;
    for (int b = 0; b < 21; ++b) r |= (uint64_t)((v >> b) & 1u) << (3 * b);
    return r;
}

typedef struct { uint64_t key; int32_t full; } keyed;
static int cmp_keyed(const void* a, const void* b) {
    const uint64_t x = ((const keyed*)a)->key, y = ((const keyed*)b)->key;
    return (x > y) - (x < y);
}

static int64_t node_id(const orc_problem* P, int ix, int iy, int iz) {
    return (int64_t)P->nnx * P->nny * iz + (int64_t)P->nnx * iy + ix;
}

static int voxel_of(const orc_problem* P, int ex, int ey, int ez) {   /* 1 for the built-in cuboid */
    return P->voxel ? P->voxel[(int64_t)ey + (int64_t)P->nely * (ex + (int64_t)P->nelx * ez)] : 1;
}

static void build_mesh(orc_problem* P) {
    const int nx = P->nx, ny = P->ny;
    keyed* k = xcalloc((size_t)P->nelx * P->nely * P->nelz, sizeof(keyed));
    int n = 0;
    /* solid region: ex < nelx, ey < nely, ez < nelz (fea.cpp:204-215), or the external model's voxels */
    for (int ez = 0; ez < P->nelz; ++ez)
        for (int ex = 0; ex < P->nelx; ++ex)
            for (int ey = 0; ey < P->nely; ++ey) {
                if (!voxel_of(P, ex, ey, ez)) continue;
                k[n].key = (spread_bits3((uint32_t)ex) << 2) | (spread_bits3((uint32_t)ey) << 1) |
                           spread_bits3((uint32_t)ez);
                k[n].full = ny * nx * ez + ny * ex + (ny - 1 - ey);
                ++n;
            }
    qsort(k, (size_t)n, sizeof(keyed), cmp_keyed);   /* keys are unique */
    P->ne = n;
    P->ele_full = xcalloc((size_t)n, sizeof(int32_t));
    P->passive = xcalloc((size_t)n, 1);
    P->enod = xcalloc((size_t)n * 8, sizeof(int32_t));
    uint8_t* color = xcalloc((size_t)n, 1);
    for (int e = 0; e < n; ++e) {
        const int full = k[e].full;
        P->ele_full[e] = full;
        const int ez = full / (nx * ny), rem = full % (nx * ny);
        const int ex = rem / ny, ey = ny - 1 - rem % ny;
        for (int a = 0; a < 8; ++a)
            P->enod[8 * e + a] = (int32_t)node_id(P, ex + CORNER[a][0], ny - ey - 1 + CORNER[a][1], ez + CORNER[a][2]);
        color[e] = (uint8_t)((ex & 1) | ((ey & 1) << 1) | ((ez & 1) << 2));   /* fea.cpp:300 */
        P->passive[e] = voxel_of(P, ex, ey, ez) == 2;
    }
    /* colour buckets in Morton order (fea.cpp:318-326) */
    P->bucket = xcalloc((size_t)n, sizeof(int32_t));
    int pos = 0;
    for (int c = 0; c < 8; ++c) {
        P->bucket_start[c] = pos;
        for (int e = 0; e < n; ++e)
            if (color[e] == c) P->bucket[pos++] = e;
    }
    P->bucket_start[8] = pos;
    free(color);
    free(k);
}

/* fea.cpp:360-447: x=0 face fixed, -Z load slab on ix=origNx over iz<=max(1,nz/6) of the
 * padded grid, nodes touched by no solid element fixed, free list ascending. */
static void build_bcs(orc_problem* P) {
    const int64_t nn = P->nn;
    P->isfree = xcalloc((size_t)P->ndof, 1);
    P->F = xcalloc((size_t)P->ndof, sizeof(double));
    memset(P->isfree, 1, (size_t)P->ndof);
    if (P->voxel) {   /* external model: listed fixations and loads; file node (x, y, z) = grid node (x, ny-y, z) */
        const int64_t py = P->nely + 1, px = P->nelx + 1;
#define GRID_NODE(m) node_id(P, (int)(((m) / py) % px), P->ny - (int)((m) % py), (int)((m) / (py * px)))
        for (int i = 0; i < P->nfix; ++i) {
            const int64_t nd = GRID_NODE(P->fix_node[i]);
            for (int c = 0; c < 3; ++c)
                if ((P->fix_bits[i] >> c) & 1) P->isfree[3 * nd + c] = 0;
        }
        if (P->ncases > 1) P->Fcases = xcalloc((size_t)P->ncases * P->ndof, sizeof(double));
        int off = 0;
        for (int k = 0; k < P->ncases; ++k) {
            double* Fk = P->ncases > 1 ? P->Fcases + (int64_t)k * P->ndof : P->F;
            for (int i = off; i < off + P->case_n[k]; ++i) {
                const int64_t nd = GRID_NODE(P->load_node[i]);
                for (int c = 0; c < 3; ++c) Fk[3 * nd + c] = P->load_f[3 * i + c];
            }
            off += P->case_n[k];
        }
        if (P->ncases > 1) memcpy(P->F, P->Fcases, (size_t)P->ndof * sizeof(double));
#undef GRID_NODE
    } else {
        for (int iz = 0; iz < P->nnz; ++iz)
            for (int iy = 0; iy < P->nny; ++iy) {
                const int64_t nd = node_id(P, 0, iy, iz);
                P->isfree[3 * nd] = P->isfree[3 * nd + 1] = P->isfree[3 * nd + 2] = 0;
            }
        const int ixl = P->nelx < P->nnx - 1 ? P->nelx : P->nnx - 1;
        const int izmax = (P->nz / 6) > 1 ? (P->nz / 6) : 1;
        const int count = (izmax + 1) * P->nny;
        const double fz = -1.0 / (double)count;
        for (int iz = 0; iz <= izmax; ++iz)
            for (int iy = 0; iy < P->nny; ++iy) P->F[3 * node_id(P, ixl, iy, iz) + 2] += fz;
    }
    uint8_t* used = xcalloc((size_t)nn, 1);
    for (int64_t i = 0; i < (int64_t)P->ne * 8; ++i) used[P->enod[i]] = 1;
    for (int64_t v = 0; v < nn; ++v)
        if (!used[v]) P->isfree[3 * v] = P->isfree[3 * v + 1] = P->isfree[3 * v + 2] = 0;
    free(used);
    int64_t nf = 0;
    for (int64_t d = 0; d < P->ndof; ++d) nf += P->isfree[d];
    P->nf = nf;
    P->free_dofs = xcalloc((size_t)nf, sizeof(int32_t));
    P->dof2free = xcalloc((size_t)P->ndof, sizeof(int32_t));
    nf = 0;
    for (int64_t d = 0; d < P->ndof; ++d) {
        if (P->isfree[d]) { P->dof2free[d] = (int32_t)nf; P->free_dofs[nf++] = (int32_t)d; }
        else P->dof2free[d] = -1;
    }
}

/* ------------------------------------------------------------------ K(E) u on free DOFs
 * fea.cpp:692-837: colour by colour, Morton order inside a colour; fe = Ke ue as an FMA
 * chain over j; y += fe * E; elements with E <= 1e-16 are skipped. */
void orc_matvec(orc_problem* P, const double* E, const double* u, double* y) {
    memset(y, 0, (size_t)P->nf * sizeof(double));
    for (int c = 0; c < 8; ++c)
        for (int b = P->bucket_start[c]; b < P->bucket_start[c + 1]; ++b) {
            const int e = P->bucket[b];
            const double Ee = E[e];
            if (Ee <= 1.0e-16) continue;
            int idx[24];
            double ue[24];
            for (int a = 0; a < 8; ++a)
                for (int d = 0; d < 3; ++d) {
                    const int f = P->dof2free[3 * (int64_t)P->enod[8 * e + a] + d];
                    idx[3 * a + d] = f;
                    ue[3 * a + d] = f >= 0 ? u[f] : 0.0;
                }
            for (int i = 0; i < 24; ++i) {
                if (idx[i] < 0) continue;
                double fe = 0.0;
                for (int j = 0; j < 24; ++j) fe = fma(P->Ke[i * 24 + j], ue[j], fe);
                y[idx[i]] = fma(fe, Ee, y[idx[i]]);
            }
        }
}

/* fea.cpp:587-677, 851-864: ce_e = ue' Ke ue (0 when E <= 1e-16), C = sum E ce.
 * u is a free vector; fixed DOFs read as 0 (scatter_from_free into zeroed U). */
typedef struct { const int32_t* cell2e; const double* w; const double* v; double scale; } cell_sum_ctx;
static double step_cell_wv(double part, int64_t k, const void* vctx) {   /* part + w*v over live cells */
    const cell_sum_ctx* c = (const cell_sum_ctx*)vctx;
    const int e = c->cell2e[k];
    if (e < 0 || c->w[e] <= 1.0e-16) return part;
    return part + c->w[e] * c->v[e];
}
static double step_cell_obj(double part, int64_t k, const void* vctx) {  /* part + E*(ce*rc) */
    const cell_sum_ctx* c = (const cell_sum_ctx*)vctx;
    const int e = c->cell2e[k];
    if (e < 0 || c->w[e] == 0.0) return part;
    return part + c->w[e] * (c->v[e] * c->scale);
}

double orc_compliance(orc_problem* P, const double* E, const double* u, double* ce) {
    double C = 0.0;
    for (int e = 0; e < P->ne; ++e) {
        if (E[e] <= 1.0e-16) { ce[e] = 0.0; continue; }
        double ue[24];
        for (int a = 0; a < 8; ++a)
            for (int d = 0; d < 3; ++d) {
                const int f = P->dof2free[3 * (int64_t)P->enod[8 * e + a] + d];
                ue[3 * a + d] = f >= 0 ? u[f] : 0.0;
            }
        double s = 0.0;
        for (int i = 0; i < 24; ++i) {
            double row = 0.0;
            for (int j = 0; j < 24; ++j) row += P->Ke[i * 24 + j] * ue[j];
            s += ue[i] * row;
        }
        ce[e] = s;
        C += E[e] * s;
    }
    if (P->p.red_mode == 1) {
        int32_t* m = cell_to_element(P);
        cell_sum_ctx c = {m, E, ce, 1.0};
        C = canon_fold((int64_t)P->nx * P->ny * P->nz, step_cell_wv, &c);
        free(m);
    }
    return C;
}

/* printed objective Cdisp (driver.cpp:144-150) */
double orc_objective(const orc_problem* P, const double* E, const double* ce, double Csolid) {
    if (P->p.red_mode == 1) {
        int32_t* m = cell_to_element(P);
        cell_sum_ctx c = {m, E, ce, 1.0 / Csolid};
        const double s = canon_fold((int64_t)P->nx * P->ny * P->nz, step_cell_obj, &c);
        free(m);
        return Csolid > 0 ? s * Csolid : s;
    }
    double cobj = 0.0;
    for (int e = 0; e < P->ne; ++e) cobj += E[e] * (ce[e] / Csolid);
    return Csolid > 0 ? cobj * Csolid : cobj;
}

/* ------------------------------------------------------------------ multigrid hierarchy
 * hierarchy.cpp:84-138: first span 4 (non-dyadic) then 2; a level needs exact
 * divisibility; stop when min dim <= 2 or at the level cap. */
static void build_hierarchy(orc_problem* P) {
    int nx = P->nx, ny = P->ny, nz = P->nz;
    P->nlev = 0;
    orc_level* L0 = &P->lv[P->nlev++];
    L0->nx = nx; L0->ny = ny; L0->nz = nz; L0->span = 1;
    for (int li = 1; li < P->p.mg_max_levels && li < 8; ++li) {
        const int s = (li == 1 && P->p.mg_nondyadic) ? 4 : 2;
        if (nx % s || ny % s || nz % s) break;
        if (nx / s < 1 || ny / s < 1 || nz / s < 1) break;
        nx /= s; ny /= s; nz /= s;
        orc_level* L = &P->lv[P->nlev++];
        L->nx = nx; L->ny = ny; L->nz = nz; L->span = s;
        int m = nx < ny ? nx : ny;
        m = m < nz ? m : nz;
        if (m <= 2) break;
    }
    for (int l = 0; l < P->nlev; ++l) {
        orc_level* L = &P->lv[l];
        L->nn = (int64_t)(L->nx + 1) * (L->ny + 1) * (L->nz + 1);
        L->mask = xcalloc((size_t)(3 * L->nn), 1);
        L->diag = xcalloc((size_t)(3 * L->nn), sizeof(double));
        L->r = xcalloc((size_t)(3 * L->nn), sizeof(double));
        L->x = xcalloc((size_t)(3 * L->nn), sizeof(double));
    }
    P->tmpf = xcalloc((size_t)(3 * P->lv[0].nn), sizeof(double));
}

/* Normalised hat-weighted average over the fine window [c*s-(s-1), c*s+(s-1)]^3 clipped to
 * the fine grid (transfers.cpp:95-191 for one component, :449-533 for three).  `divide`
 * selects valSum/wSum (strided form, used for the masks) or valSum*(1/wSum) (Vec3 form,
 * used by the V-cycle). */
static void restrict_nodes(const orc_level* Lc, const orc_level* Lf, const double* rf, int ncomp,
                           int divide, double* rc) {
    const int s = Lc->span, ws = 2 * s - 1;
    const double inv = 1.0 / s;
    double W[8];
    for (int i = 0; i < ws; ++i) W[i] = 1.0 - fabs((double)(i - (s - 1))) * inv;
    const int fnx = Lf->nx + 1, fny = Lf->ny + 1, fnz = Lf->nz + 1;
    const int cnx = Lc->nx + 1, cny = Lc->ny + 1, cnz = Lc->nz + 1;
    for (int cz = 0; cz < cnz; ++cz)
        for (int cy = 0; cy < cny; ++cy)
            for (int cx = 0; cx < cnx; ++cx) {
                double v[3] = {0, 0, 0}, wsum = 0.0;
                for (int iz = 0; iz < ws; ++iz) {
                    const int fz = cz * s + iz - (s - 1);
                    if (fz < 0 || fz >= fnz) continue;
                    for (int iy = 0; iy < ws; ++iy) {
                        const int fy = cy * s + iy - (s - 1);
                        if (fy < 0 || fy >= fny) continue;
                        const double wzy = W[iz] * W[iy];
                        for (int ix = 0; ix < ws; ++ix) {
                            const int fx = cx * s + ix - (s - 1);
                            if (fx < 0 || fx >= fnx) continue;
                            const double w = wzy * W[ix];
                            const int64_t f = ((int64_t)fz * fny + fy) * fnx + fx;
                            for (int c = 0; c < ncomp; ++c) v[c] += rf[f * ncomp + c] * w;
                            wsum += w;
                        }
                    }
                }
                const int64_t ci = ((int64_t)cz * cny + cy) * cnx + cx;
                if (wsum > 1e-12) {
                    if (divide) {
                        for (int c = 0; c < ncomp; ++c) rc[ci * ncomp + c] = v[c] / wsum;
                    } else {
                        const double iw = 1.0 / wsum;
                        for (int c = 0; c < ncomp; ++c) rc[ci * ncomp + c] = v[c] * iw;
                    }
                } else {
                    for (int c = 0; c < ncomp; ++c) rc[ci * ncomp + c] = 0.0;
                }
            }
}

/* Canonical (red_mode 1) restriction: the same normalised hat average evaluated separably,
 * first along x for every fine (z,y) row of the window, then along y, then along z, each sum in
 * increasing index order from 0; the weight sum (exact in binary) is the product of the 1D sums. */
static void restrict_nodes_separable(const orc_level* Lc, const orc_level* Lf, const double* rf, double* rc) {
    const int s = Lc->span, ws = 2 * s - 1;
    const double inv = 1.0 / s;
    double W[8];
    for (int i = 0; i < ws; ++i) W[i] = 1.0 - fabs((double)(i - (s - 1))) * inv;
    const int fnx = Lf->nx + 1, fny = Lf->ny + 1, fnz = Lf->nz + 1;
    const int cnx = Lc->nx + 1, cny = Lc->ny + 1, cnz = Lc->nz + 1;
    for (int cz = 0; cz < cnz; ++cz)
        for (int cy = 0; cy < cny; ++cy)
            for (int cx = 0; cx < cnx; ++cx) {
                double vz[3] = {0, 0, 0}, swz = 0.0, swy = 0.0, swx = 0.0;
                for (int ix = 0; ix < ws; ++ix) {
                    const int fx = cx * s + ix - (s - 1);
                    if (fx >= 0 && fx < fnx) swx = swx + W[ix];
                }
                for (int iy = 0; iy < ws; ++iy) {
                    const int fy = cy * s + iy - (s - 1);
                    if (fy >= 0 && fy < fny) swy = swy + W[iy];
                }
                for (int iz = 0; iz < ws; ++iz) {
                    const int fz = cz * s + iz - (s - 1);
                    if (fz < 0 || fz >= fnz) continue;
                    swz = swz + W[iz];
                    double vy[3] = {0, 0, 0};
                    for (int iy = 0; iy < ws; ++iy) {
                        const int fy = cy * s + iy - (s - 1);
                        if (fy < 0 || fy >= fny) continue;
                        double vx[3] = {0, 0, 0};
                        for (int ix = 0; ix < ws; ++ix) {
                            const int fx = cx * s + ix - (s - 1);
                            if (fx < 0 || fx >= fnx) continue;
                            const int64_t f = ((int64_t)fz * fny + fy) * fnx + fx;
                            for (int c = 0; c < 3; ++c) vx[c] = vx[c] + W[ix] * rf[f * 3 + c];
                        }
                        for (int c = 0; c < 3; ++c) vy[c] = vy[c] + W[iy] * vx[c];
                    }
                    for (int c = 0; c < 3; ++c) vz[c] = vz[c] + W[iz] * vy[c];
                }
                const double wsum = swz * swy * swx;
                const int64_t ci = ((int64_t)cz * cny + cy) * cnx + cx;
                const double iw = 1.0 / wsum;
                for (int c = 0; c < 3; ++c) rc[ci * 3 + c] = wsum > 1e-12 ? vz[c] * iw : 0.0;
            }
}

/* Trilinear interpolation from the coarse cell floor(f/s), clamped to the last cell
 * (transfers.cpp:378-445). */
static void prolongate_nodes(const orc_level* Lc, const orc_level* Lf, const double* xc, double* xf) {
    const int s = Lc->span;
    const double inv = 1.0 / s;
    const int fnx = Lf->nx + 1, fny = Lf->ny + 1, fnz = Lf->nz + 1;
    const int cnx = Lc->nx + 1, cny = Lc->ny + 1;
    for (int fz = 0; fz < fnz; ++fz)
        for (int fy = 0; fy < fny; ++fy)
            for (int fx = 0; fx < fnx; ++fx) {
                int cx = fx / s, cy = fy / s, cz = fz / s;
                int rx = fx % s, ry = fy % s, rz = fz % s;
                if (cx >= Lc->nx) { cx = Lc->nx - 1; rx = s; }
                if (cy >= Lc->ny) { cy = Lc->ny - 1; ry = s; }
                if (cz >= Lc->nz) { cz = Lc->nz - 1; rz = s; }
                const double wx1 = rx * inv, wx0 = 1.0 - wx1;
                const double wy1 = ry * inv, wy0 = 1.0 - wy1;
                const double wz1 = rz * inv, wz0 = 1.0 - wz1;
                const int64_t b = ((int64_t)cz * cny + cy) * cnx + cx;
                const int64_t n000 = b, n100 = b + 1, n010 = b + cnx, n110 = b + cnx + 1;
                const int64_t pz = (int64_t)cnx * cny;
                const int64_t f = (((int64_t)fz * fny + fy) * fnx + fx) * 3;
                for (int c = 0; c < 3; ++c) {
                    xf[f + c] = xc[3 * n000 + c] * wx0 * wy0 * wz0 + xc[3 * n100 + c] * wx1 * wy0 * wz0 +
                                xc[3 * n010 + c] * wx0 * wy1 * wz0 + xc[3 * n110 + c] * wx1 * wy1 * wz0 +
                                xc[3 * (n000 + pz) + c] * wx0 * wy0 * wz1 + xc[3 * (n100 + pz) + c] * wx1 * wy0 * wz1 +
                                xc[3 * (n010 + pz) + c] * wx0 * wy1 * wz1 + xc[3 * (n110 + pz) + c] * wx1 * wy1 * wz1;
                }
            }
}

/* masks.cpp:11-37: fine mask = fixed DOFs; coarse mask = restricted 0/1 field > 0.5 */
static void build_masks(orc_problem* P) {
    for (int64_t d = 0; d < P->ndof; ++d) P->lv[0].mask[d] = P->isfree[d] ? 0 : 1;
    for (int l = 0; l + 1 < P->nlev; ++l) {
        orc_level* Lf = &P->lv[l];
        orc_level* Lc = &P->lv[l + 1];
        double* rf = xcalloc((size_t)Lf->nn, sizeof(double));
        double* rc = xcalloc((size_t)Lc->nn, sizeof(double));
        for (int c = 0; c < 3; ++c) {
            for (int64_t n = 0; n < Lf->nn; ++n) rf[n] = Lf->mask[3 * n + c] ? 1.0 : 0.0;
            restrict_nodes(Lc, Lf, rf, 1, 1, rc);
            for (int64_t n = 0; n < Lc->nn; ++n) Lc->mask[3 * n + c] = rc[n] > 0.5 ? 1 : 0;
        }
        free(rf);
        free(rc);
    }
}

/* Level-l trilinear weight of coarse corner a at fine sub-node (ix,iy,iz) of a coarse
 * element (hierarchy.cpp:13-42). */
static double corner_weight(int s, int ix, int iy, int iz, int a) {
    const double xi = -1.0 + 2.0 * ((double)ix / (double)s);
    const double eta = -1.0 + 2.0 * ((double)iy / (double)s);
    const double zeta = -1.0 + 2.0 * ((double)iz / (double)s);
    static const double sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    static const double sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    static const double sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    return 0.125 * (1.0 + sx[a] * xi) * (1.0 + sy[a] * eta) * (1.0 + sz[a] * zeta);
}

/* Jacobi diagonals (diagonal.cpp:11-160).  Fine: sum of E*Ke_ii over the colour-ordered
 * elements, non-positive -> 1, fixed -> 1.  Coarse: w^2-weighted average of the fine
 * diagonal over each coarse element's (s+1)^3 sub-nodes, coarse elements in colour order. */
static void build_diagonals(orc_problem* P, const double* E) {
    orc_level* L0 = &P->lv[0];
    double* d0 = L0->diag;
    memset(d0, 0, (size_t)(3 * L0->nn) * sizeof(double));
    for (int c = 0; c < 8; ++c)
        for (int b = P->bucket_start[c]; b < P->bucket_start[c + 1]; ++b) {
            const int e = P->bucket[b];
            for (int a = 0; a < 8; ++a)
                for (int d = 0; d < 3; ++d) {
                    const int l = 3 * a + d;
                    d0[3 * (int64_t)P->enod[8 * e + a] + d] += P->Ke[l * 24 + l] * E[e];
                }
        }
    for (int64_t i = 0; i < 3 * L0->nn; ++i)
        if (!(d0[i] > 0.0)) d0[i] = 1.0;
    for (int64_t i = 0; i < 3 * L0->nn; ++i)
        if (L0->mask[i]) d0[i] = 1.0;

    for (int l = 0; l + 1 < P->nlev; ++l) {
        const orc_level* Lf = &P->lv[l];
        orc_level* Lc = &P->lv[l + 1];
        const int s = Lc->span;
        double* dc = Lc->diag;
        double* wsum = xcalloc((size_t)(3 * Lc->nn), sizeof(double));
        memset(dc, 0, (size_t)(3 * Lc->nn) * sizeof(double));
        const int fnx = Lf->nx + 1, fny = Lf->ny + 1;
        const int cnx = Lc->nx + 1, cny = Lc->ny + 1;
        for (int color = 0; color < 8; ++color)
            for (int cez = 0; cez < Lc->nz; ++cez)
                for (int cex = 0; cex < Lc->nx; ++cex)
                    for (int cey = 0; cey < Lc->ny; ++cey) {
                        if (((cex & 1) | ((cey & 1) << 1) | ((cez & 1) << 2)) != color) continue;
                        int64_t cn[8];
                        for (int a = 0; a < 8; ++a)
                            cn[a] = ((int64_t)(cez + CORNER[a][2]) * cny + (Lc->ny - cey - 1 + CORNER[a][1])) * cnx +
                                    (cex + CORNER[a][0]);
                        const int fx0 = cex * s, fy0 = (Lc->ny - cey) * s, fz0 = cez * s;
                        for (int iz = 0; iz <= s; ++iz)
                            for (int iy = 0; iy <= s; ++iy)
                                for (int ix = 0; ix <= s; ++ix) {
                                    const int64_t fn = ((int64_t)(fz0 + iz) * fny + (fy0 - iy)) * fnx + (fx0 + ix);
                                    for (int a = 0; a < 8; ++a) {
                                        const double w = corner_weight(s, ix, iy, iz, a);
                                        const double w2 = w * w;
                                        for (int d = 0; d < 3; ++d) {
                                            const int64_t cd = 3 * cn[a] + d, fd = 3 * fn + d;
                                            if (Lc->mask[cd] || Lf->mask[fd]) continue;
                                            dc[cd] += w2 * Lf->diag[fd];
                                            wsum[cd] += w2;
                                        }
                                    }
                                }
                    }
        for (int64_t i = 0; i < 3 * Lc->nn; ++i) {
            if (Lc->mask[i]) dc[i] = 1.0;
            else if (wsum[i] > 0) {
                dc[i] /= wsum[i];
                if (!(dc[i] > 0.0)) dc[i] = 1.0;
            } else dc[i] = 1.0;
        }
        free(wsum);
    }
}

/* Coarsest dense Galerkin matrix (coarsest.cpp:126-323 + preconditioner.cpp:56-73).
 * For every coarse element, the s^3 fine elements at (cex*s+ix, (resYc-cey)*s-iy-1, cez*s+iz)
 * of the FINEST grid (s = the coarsest level's own span) contribute T'(max(Emin,E_f) Ke)T;
 * fine elements touching a fixed DOF have those rows/cols replaced by identity first.
 * Lower triangle only, then coarsest BC rows/cols -> identity.  Returns N or 0. */
static int assemble_coarse(orc_problem* P, const double* E, double* Kc) {
    const orc_level* Lf = &P->lv[0];
    const orc_level* Lc = &P->lv[P->nlev - 1];
    const int N = (int)(3 * Lc->nn);
    if (P->nlev == 1 || N > 1000) return 0;
    memset(Kc, 0, (size_t)N * N * sizeof(double));
    const int s = P->p.coarse_full ? P->nx / Lc->nx : Lc->span;
    /* full-grid moduli: padding elements read 0 (EleMod_CompactToFull_Finest) */
    double* Efull = xcalloc((size_t)P->nx * P->ny * P->nz, sizeof(double));
    for (int e = 0; e < P->ne; ++e) Efull[P->ele_full[e]] = E[e];
    const double emin = (double)P->p.Emin;
    const int cnx = Lc->nx + 1, cny = Lc->ny + 1;
    double T[576], M[576], Kf[576], Kce[576];
    for (int cez = 0; cez < Lc->nz; ++cez)
        for (int cex = 0; cex < Lc->nx; ++cex)
            for (int cey = 0; cey < Lc->ny; ++cey) {
                int cdof[24];
                for (int a = 0; a < 8; ++a) {
                    const int64_t cn = ((int64_t)(cez + CORNER[a][2]) * cny + (Lc->ny - cey - 1 + CORNER[a][1])) * cnx +
                                       (cex + CORNER[a][0]);
                    for (int d = 0; d < 3; ++d) cdof[3 * a + d] = (int)(3 * cn + d);
                }
                memset(Kce, 0, sizeof Kce);
                for (int iz = 0; iz < s; ++iz)
                    for (int iy = 0; iy < s; ++iy)
                        for (int ix = 0; ix < s; ++ix) {
                            const int fex = cex * s + ix, fey = (Lc->ny - cey) * s - iy - 1, fez = cez * s + iz;
                            const int full = Lf->ny * Lf->nx * fez + Lf->ny * fex + (Lf->ny - 1 - fey);
                            double Ee = Efull[full];
                            if (Ee < emin) Ee = emin;
                            /* The sub-element's nodes (and so its BC mask) are those of the cell whose
                               lower node row is fey, i.e. the cell geometrically inside the coarse
                               element; its modulus is read through the full element index above,
                               which names the y-mirrored cell (coarsest.cpp:156-158,246-253). */
                            int fnode[8];
                            int masked = 0;
                            for (int v = 0; v < 8; ++v) {
                                fnode[v] = (int)node_id(P, fex + CORNER[v][0], fey + CORNER[v][1], fez + CORNER[v][2]);
                                for (int d = 0; d < 3; ++d) masked |= Lf->mask[3 * (int64_t)fnode[v] + d];
                            }
                            /* T maps coarse element DOFs to this sub-element's DOFs */
                            memset(T, 0, sizeof T);
                            for (int v = 0; v < 8; ++v) {
                                const int vx = CORNER[v][0], vz = CORNER[v][2];
                                /* sub-element corner v sits at sub-node (ix+vx, iy+(1-vyc), iz+vz) in the
                                   coarse element's natural-coordinate grid */
                                const int vy = (v == 0 || v == 1 || v == 4 || v == 5) ? 0 : 1;
                                for (int a = 0; a < 8; ++a) {
                                    const double w = corner_weight(s, ix + vx, iy + vy, iz + vz, a);
                                    for (int d = 0; d < 3; ++d) T[(3 * v + d) * 24 + 3 * a + d] = w;
                                }
                            }
                            for (int i = 0; i < 576; ++i) Kf[i] = masked ? Ee * P->Ke[i] : P->Ke[i];
                            if (masked) {
                                for (int v = 0; v < 8; ++v)
                                    for (int d = 0; d < 3; ++d)
                                        if (Lf->mask[3 * (int64_t)fnode[v] + d]) {
                                            const int q = 3 * v + d;
                                            for (int j = 0; j < 24; ++j) { Kf[q * 24 + j] = 0.0; Kf[j * 24 + q] = 0.0; }
                                            Kf[q * 24 + q] = 1.0;
                                        }
                            }
                            for (int i = 0; i < 24; ++i)
                                for (int j = 0; j < 24; ++j) {
                                    double acc = 0.0;
                                    for (int k = 0; k < 24; ++k) acc += Kf[i * 24 + k] * T[k * 24 + j];
                                    M[i * 24 + j] = acc;
                                }
                            for (int i = 0; i < 24; ++i)
                                for (int j = 0; j < 24; ++j) {
                                    double acc = 0.0;
                                    for (int k = 0; k < 24; ++k) acc += T[k * 24 + i] * M[k * 24 + j];
                                    /* unmasked: template (T'KeT) scaled by Ee; masked: already scaled */
                                    Kce[i * 24 + j] += masked ? acc : Ee * acc;
                                }
                        }
                for (int i = 0; i < 24; ++i)
                    for (int j = 0; j < 24; ++j)
                        if (cdof[i] >= cdof[j]) Kc[(int64_t)cdof[i] * N + cdof[j]] += Kce[i * 24 + j];
            }
    free(Efull);
    for (int64_t n = 0; n < Lc->nn; ++n)
        for (int d = 0; d < 3; ++d)
            if (Lc->mask[3 * n + d]) {
                const int q = (int)(3 * n + d);
                for (int j = 0; j < N; ++j) { Kc[(int64_t)q * N + j] = 0.0; Kc[(int64_t)j * N + q] = 0.0; }
                Kc[(int64_t)q * N + q] = 1.0;
            }
    return N;
}

/* coarsest.cpp:13-90 (row-oriented Cholesky on the lower triangle) */
static int cholesky_lower(double* A, int N) {
    for (int i = 0; i < N; ++i) {
        for (int j = 0; j <= i; ++j) {
            double s = A[(int64_t)i * N + j];
            for (int k = 0; k < j; ++k) s -= A[(int64_t)i * N + k] * A[(int64_t)j * N + k];
            if (i == j) {
                if (s <= 0.0) return 0;
                A[(int64_t)i * N + i] = sqrt(s);
            } else {
                A[(int64_t)i * N + j] = s / A[(int64_t)j * N + j];
            }
        }
        for (int j = i + 1; j < N; ++j) A[(int64_t)i * N + j] = 0.0;
    }
    return 1;
}

/* coarsest.cpp:92-122 */
static void cholesky_solve(const double* L, const double* b, double* x, int N) {
    for (int i = 0; i < N; ++i) x[i] = b[i];
    for (int i = 0; i < N; ++i) {
        double s = x[i];
        for (int k = 0; k < i; ++k) s -= L[(int64_t)i * N + k] * x[k];
        x[i] = s / L[(int64_t)i * N + i];
    }
    for (int i = N - 1; i >= 0; --i) {
        x[i] /= L[(int64_t)i * N + i];
        const double xi = x[i];
        for (int k = 0; k < i; ++k) x[k] -= L[(int64_t)i * N + k] * xi;
    }
}

/* make_diagonal_preconditioner_from_static (preconditioner.cpp:38-79) */
void orc_mg_build(orc_problem* P, const double* E) {
    build_diagonals(P, E);
    free(P->Lc);
    P->Lc = NULL;
    P->Nc = 0;
    const orc_level* Lc = &P->lv[P->nlev - 1];
    const int N = (int)(3 * Lc->nn);
    if (P->nlev > 1 && N <= 1000) {
        double* K = xcalloc((size_t)N * N, sizeof(double));
        assemble_coarse(P, E, K);
        if (cholesky_lower(K, N)) { P->Lc = K; P->Nc = N; }
        else free(K);
    }
    free(P->Xc);
    P->Xc = NULL;
    if (P->Nc && P->p.red_mode == 1) {
        /* canonical coarsest solve: X[:,j] = L'^-1 L^-1 e_j by the reference's substitutions */
        const int n = P->Nc;
        P->Xc = xcalloc((size_t)n * n, sizeof(double));
        double* e = xcalloc((size_t)n, sizeof(double));
        for (int j = 0; j < n; ++j) {
            memset(e, 0, (size_t)n * sizeof(double));
            e[j] = 1.0;
            cholesky_solve(P->Lc, e, P->Xc + (int64_t)j * n, n);   /* column j stored contiguously */
        }
        free(e);
    }
}

int orc_mg_coarse_n(const orc_problem* P) { return P->Nc; }

int orc_coarse_matrix(orc_problem* P, const double* E, double* out) { return assemble_coarse(P, E, out); }

/* Additive V-cycle (preconditioner.cpp:88-265) */
void orc_vcycle(orc_problem* P, const double* r, double* z) {
    const double w = (double)P->p.mg_weight;
    orc_level* L0 = &P->lv[0];
    memset(L0->r, 0, (size_t)(3 * L0->nn) * sizeof(double));
    memset(L0->x, 0, (size_t)(3 * L0->nn) * sizeof(double));
    for (int64_t i = 0; i < P->nf; ++i) L0->r[P->free_dofs[i]] = r[i];
    for (int64_t d = 0; d < 3 * L0->nn; ++d)
        if (L0->mask[d]) L0->r[d] = 0.0;
    for (int l = 0; l + 1 < P->nlev; ++l) {
        orc_level* Lf = &P->lv[l];
        orc_level* Lc = &P->lv[l + 1];
        for (int64_t d = 0; d < 3 * Lf->nn; ++d) {
            double dd = Lf->diag[d] > 1.0e-30 ? Lf->diag[d] : 1.0e-30;
            Lf->x[d] = Lf->mask[d] ? 0.0 : w * Lf->r[d] / dd;
        }
        if (P->p.red_mode == 1) restrict_nodes_separable(Lc, Lf, Lf->r, Lc->r);
        else restrict_nodes(Lc, Lf, Lf->r, 3, 0, Lc->r);
        for (int64_t d = 0; d < 3 * Lc->nn; ++d)
            if (Lc->mask[d]) Lc->r[d] = 0.0;
    }
    orc_level* LL = &P->lv[P->nlev - 1];
    if (P->Nc > 0 && P->Nc == 3 * LL->nn && P->Xc) {
        const int n = P->Nc;
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int j = 0; j < n; ++j) acc = acc + P->Xc[(int64_t)j * n + i] * LL->r[j];
            LL->x[i] = acc;
        }
    } else if (P->Nc > 0 && P->Nc == 3 * LL->nn) {
        cholesky_solve(P->Lc, LL->r, LL->x, P->Nc);
    } else {
        for (int64_t d = 0; d < 3 * LL->nn; ++d) {
            double dd = LL->diag[d] > 1.0e-30 ? LL->diag[d] : 1.0e-30;
            LL->x[d] = LL->mask[d] ? 0.0 : LL->r[d] / dd;
        }
    }
    for (int64_t d = 0; d < 3 * LL->nn; ++d)
        if (LL->mask[d]) LL->x[d] = 0.0;
    for (int l = P->nlev - 2; l >= 0; --l) {
        orc_level* Lf = &P->lv[l];
        prolongate_nodes(&P->lv[l + 1], Lf, P->lv[l + 1].x, P->tmpf);
        for (int64_t d = 0; d < 3 * Lf->nn; ++d) {
            Lf->x[d] += P->tmpf[d];
            if (Lf->mask[d]) Lf->x[d] = 0.0;
            else {
                double dd = Lf->diag[d] > 1.0e-30 ? Lf->diag[d] : 1.0e-30;
                Lf->x[d] += w * Lf->r[d] / dd;
            }
        }
    }
    for (int64_t i = 0; i < P->nf; ++i) z[i] = L0->x[P->free_dofs[i]];
}

static double dot(const double* a, const double* b, int64_t n) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* ------------------------------------------------------------------ canonical reduction order
 * Emulates the CUDA path's deterministic reductions: item i (a node or a cell) belongs to thread
 * gid = i mod (RB*RT); each thread folds its items in increasing order into a partial starting at 0
 * through `step`; the 32 partials of a warp are combined by an xor butterfly (offsets 16..1), the 8
 * warp sums of a block by the same butterfly padded with zeros, and the RB block partials by a last
 * pass where thread t sums partials t, t+RT, ... in order, followed by the two butterflies. */
#define RB 1184
#define RT 256

static double butterfly32(double* v) {
    double t[32];
    for (int off = 16; off > 0; off >>= 1) {
        for (int l = 0; l < 32; ++l) t[l] = v[l] + v[l ^ off];
        memcpy(v, t, sizeof t);
    }
    return v[0];
}

static double fold_block(const double* lanes /* RT */) {
    double w[8];
    for (int k = 0; k < 8; ++k) {
        double v[32];
        memcpy(v, lanes + 32 * k, sizeof v);
        w[k] = butterfly32(v);
    }
    double v[32];
    for (int l = 0; l < 32; ++l) v[l] = l < 8 ? w[l] : 0.0;
    return butterfly32(v);
}

/* per-thread partial of thread t of block b; `active` says whether block b has any work */
typedef double (*canon_thread)(int b, int t, const void* ctx);
typedef int (*canon_active)(int b, const void* ctx);

static double canon_fold_threads(canon_thread part_of, canon_active active, const void* ctx) {
    static double partial[RB];
    double lanes[RT];
    for (int b = 0; b < RB; ++b) {
        if (!active(b, ctx)) {   /* threads without items: the butterflies of +0 give +0 */
            partial[b] = 0.0;
            continue;
        }
        for (int t = 0; t < RT; ++t) lanes[t] = part_of(b, t, ctx);
        partial[b] = fold_block(lanes);
    }
    for (int t = 0; t < RT; ++t) {
        double s = 0.0;
        for (int i = t; i < RB; i += RT) s = s + partial[i];
        lanes[t] = s;
    }
    return fold_block(lanes);
}

/* item i of a linear grid-stride loop belongs to thread (b,t) with i = b*RT + t (mod RB*RT) */
typedef struct { int64_t nitems; canon_step step; const void* ctx; } linear_ctx;
static double linear_part(int b, int t, const void* vctx) {
    const linear_ctx* c = (const linear_ctx*)vctx;
    double p = 0.0;
    for (int64_t i = (int64_t)b * RT + t; i < c->nitems; i += (int64_t)RB * RT) p = c->step(p, i, c->ctx);
    return p;
}
static int linear_active(int b, const void* vctx) { return (int64_t)b * RT < ((const linear_ctx*)vctx)->nitems; }

static double canon_fold(int64_t nitems, canon_step step, const void* ctx) {
    linear_ctx c = {nitems, step, ctx};
    return canon_fold_threads(linear_part, linear_active, &c);
}

/* node-item step: sum over the three DOFs of node i of a*b (free vectors; fixed DOFs read 0) */
typedef struct { const orc_problem* P; const double* a; const double* b; } node_dot_ctx;
static double step_node_dot(double part, int64_t n, const void* vctx) {
    const node_dot_ctx* c = (const node_dot_ctx*)vctx;
    for (int d = 0; d < 3; ++d) {
        const int f = c->P->dof2free[3 * n + d];
        const double av = f >= 0 ? c->a[f] : 0.0, bv = f >= 0 ? c->b[f] : 0.0;
        part = part + av * bv;
    }
    return part;
}

/* inner product of two free-DOF vectors in the selected order */
static double free_dot(const orc_problem* P, const double* a, const double* b) {
    if (P->p.red_mode == 0) return dot(a, b, P->nf);
    node_dot_ctx c = {P, a, b};
    return canon_fold(P->nn, step_node_dot, &c);
}

/* inner product of two node vectors (filter) in the selected order */
typedef struct { const double* a; const double* b; } vec_dot_ctx;
static double step_vec_dot(double part, int64_t n, const void* vctx) {
    const vec_dot_ctx* c = (const vec_dot_ctx*)vctx;
    return part + c->a[n] * c->b[n];
}
static double node_dot(const orc_problem* P, const double* a, const double* b) {
    if (P->p.red_mode == 0) return dot(a, b, P->nn);
    vec_dot_ctx c = {a, b};
    return canon_fold(P->nn, step_vec_dot, &c);
}

/* canonical cell order: k = (cz*ny + cy)*nx + cx over the padded grid; cell2e maps k to the
   compact (Morton) element or -1 for a void cell */
static int32_t* cell_to_element(const orc_problem* P) {
    const int64_t ncell = (int64_t)P->nx * P->ny * P->nz;
    int32_t* m = xcalloc((size_t)ncell, sizeof(int32_t));
    for (int64_t k = 0; k < ncell; ++k) m[k] = -1;
    for (int e = 0; e < P->ne; ++e) {
        const int full = P->ele_full[e];   /* ny*nx*cz + ny*cx + cy */
        const int cz = full / (P->nx * P->ny), rem = full % (P->nx * P->ny);
        const int cx = rem / P->ny, cy = rem % P->ny;
        m[((int64_t)cz * P->ny + cy) * P->nx + cx] = e;
    }
    return m;
}

/* PCG_free (solver.cpp:87-217) with the multigrid preconditioner built by orc_mg_build */
int orc_pcg(orc_problem* P, const double* E, const double* b, double* x, double tol, int maxit) {
    const int64_t n = P->nf;
    double *r = P->r, *z = P->z, *p = P->pp, *Ap = P->Ap;
    orc_matvec(P, E, x, Ap);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - Ap[i];
    orc_vcycle(P, r, z);
    double rz = free_dot(P, r, z);
    memcpy(p, z, (size_t)n * sizeof(double));
    const double nb = sqrt(free_dot(P, b, b));
    const double stop = (nb > 1.0e-30 ? nb : 1.0e-30) * tol;
    for (int it = 0; it < maxit; ++it) {
        orc_matvec(P, E, p, Ap);
        const double den = free_dot(P, p, Ap);
        const double alpha = rz / (den > 1.0e-30 ? den : 1.0e-30);
        double rn2 = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
            rn2 += r[i] * r[i];
        }
        if (P->p.red_mode == 1) rn2 = free_dot(P, r, r);
        if (sqrt(rn2) < stop) return it + 1;
        orc_vcycle(P, r, z);
        const double rzn = free_dot(P, r, z);
        const double beta = rzn / (rz > 1.0e-30 ? rz : 1.0e-30);
        rz = rzn;
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    return maxit;
}

/* ------------------------------------------------------------------ PDE filter
 * filter.cpp:9-75: 8x8 kernel r^2*KEF0 + KEF1 with r = rMin/(2 sqrt 3), inverse row-sum
 * Jacobi preconditioner accumulated over elements in compact order. */
void orc_filter_setup(orc_problem* P, float rmin) {
    static const double sg[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    static const double tg[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    static const double pg[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    double N[8][8], dS[24][8];
    for (int g = 0; g < 8; ++g) {
        const double s = sg[g] / sqrt(3.0), t = tg[g] / sqrt(3.0), q = pg[g] / sqrt(3.0);
        for (int a = 0; a < 8; ++a) {
            N[g][a] = 0.125 * (1 + sg[a] * s) * (1 + tg[a] * t) * (1 + pg[a] * q);
            dS[3 * g + 0][a] = 0.125 * sg[a] * (1 + tg[a] * t) * (1 + pg[a] * q);
            dS[3 * g + 1][a] = 0.125 * tg[a] * (1 + sg[a] * s) * (1 + pg[a] * q);
            dS[3 * g + 2][a] = 0.125 * pg[a] * (1 + sg[a] * s) * (1 + tg[a] * t);
        }
    }
    const double rr = ((double)rmin * 1.0) / (2.0 * sqrt(3.0));
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) {
            double k0 = 0.0, k1 = 0.0;
            for (int k = 0; k < 24; ++k) k0 += dS[k][i] * dS[k][j];
            for (int g = 0; g < 8; ++g) k1 += N[g][i] * (1.0 / 8.0) * N[g][j];
            P->kf[i * 8 + j] = rr * rr * k0 + k1;
        }
    double rs[8];
    for (int a = 0; a < 8; ++a) {
        double s = 0.0;
        for (int b = 0; b < 8; ++b) s += P->kf[a * 8 + b];
        rs[a] = s;
    }
    const int64_t nn = P->nn;
    if (!P->fdiag) {
        P->fdiag = xcalloc((size_t)nn, sizeof(double));
        P->flastx = xcalloc((size_t)nn, sizeof(double));
        P->flastrhs = xcalloc((size_t)nn, sizeof(double));
        P->frhs = xcalloc((size_t)nn, sizeof(double));
        P->fx = xcalloc((size_t)nn, sizeof(double));
        P->fr = xcalloc((size_t)nn, sizeof(double));
        P->fz = xcalloc((size_t)nn, sizeof(double));
        P->fp = xcalloc((size_t)nn, sizeof(double));
        P->fAp = xcalloc((size_t)nn, sizeof(double));
    }
    memset(P->fdiag, 0, (size_t)nn * sizeof(double));
    for (int e = 0; e < P->ne; ++e)
        for (int a = 0; a < 8; ++a) P->fdiag[P->enod[8 * e + a]] += rs[a];
    for (int64_t i = 0; i < nn; ++i) P->fdiag[i] = P->fdiag[i] > 0 ? 1.0 / P->fdiag[i] : 1.0;
    memset(P->flastx, 0, (size_t)nn * sizeof(double));
    memset(P->flastrhs, 0, (size_t)nn * sizeof(double));
    P->filter_ready = 1;
}

/* filter.cpp:77-173 (colour order, Morton order inside a colour) */
static void filter_matvec(const orc_problem* P, const double* x, double* y) {
    memset(y, 0, (size_t)P->nn * sizeof(double));
    for (int c = 0; c < 8; ++c)
        for (int b = P->bucket_start[c]; b < P->bucket_start[c + 1]; ++b) {
            const int32_t* en = P->enod + 8 * P->bucket[b];
            double u[8];
            for (int a = 0; a < 8; ++a) u[a] = x[en[a]];
            for (int a = 0; a < 8; ++a) {
                double s = 0.0;
                for (int j = 0; j < 8; ++j) s += P->kf[a * 8 + j] * u[j];
                y[en[a]] += s;
            }
        }
}

static void filter_to_elements(const orc_problem* P, const double* x, float* dst) {
    for (int e = 0; e < P->ne; ++e) {
        double s = 0.0;
        for (int a = 0; a < 8; ++a) s += x[P->enod[8 * e + a]];
        dst[e] = (float)(s * (1.0 / 8.0));
    }
}

/* ApplyPDEFilter (filter.cpp:175-275) */
void orc_filter_apply(orc_problem* P, const float* src, float* dst) {
    const int64_t nn = P->nn;
    double* rhs = P->frhs;
    memset(rhs, 0, (size_t)nn * sizeof(double));
    for (int e = 0; e < P->ne; ++e) {
        const double v = (double)src[e] * (1.0 / 8.0);
        for (int a = 0; a < 8; ++a) rhs[P->enod[8 * e + a]] += v;
    }
    double nr = 0.0, df = 0.0;
    for (int64_t i = 0; i < nn; ++i) {
        const double d = rhs[i] - P->flastrhs[i];
        nr += rhs[i] * rhs[i];
        df += d * d;
    }
    if (P->p.red_mode == 1) {
        double* dv = xcalloc((size_t)nn, sizeof(double));
        for (int64_t i = 0; i < nn; ++i) dv[i] = rhs[i] - P->flastrhs[i];
        nr = node_dot(P, rhs, rhs);
        df = node_dot(P, dv, dv);
        free(dv);
    }
    nr = sqrt(nr);
    df = sqrt(df);
    const int warm = (nr > 0.0) && (df / (nr > 1.0e-30 ? nr : 1.0e-30) < 1000.0);
    double *x = P->fx, *r = P->fr, *z = P->fz, *p = P->fp, *Ap = P->fAp;
    if (warm) memcpy(x, P->flastx, (size_t)nn * sizeof(double));
    else memset(x, 0, (size_t)nn * sizeof(double));
    if (warm) {
        filter_matvec(P, x, Ap);
        for (int64_t i = 0; i < nn; ++i) r[i] = rhs[i] - Ap[i];
    } else {
        memcpy(r, rhs, (size_t)nn * sizeof(double));
    }
    double rz = 0.0;
    for (int64_t i = 0; i < nn; ++i) {
        z[i] = P->fdiag[i] * r[i];
        rz += r[i] * z[i];
    }
    if (P->p.red_mode == 1) rz = node_dot(P, r, z);
    if (rz == 0) rz = 1.0;
    memcpy(p, z, (size_t)nn * sizeof(double));
    const double rn0 = sqrt(node_dot(P, r, r));
    if (!(rn0 < 1.0e-2)) {
        for (int it = 0; it < 80; ++it) {
            filter_matvec(P, p, Ap);
            const double den = node_dot(P, p, Ap);
            const double alpha = rz / (den > 1.0e-30 ? den : 1.0e-30);
            for (int64_t i = 0; i < nn; ++i) x[i] += alpha * p[i];
            for (int64_t i = 0; i < nn; ++i) r[i] -= alpha * Ap[i];
            const double rn = sqrt(node_dot(P, r, r));
            if (rn < 1e-3) break;
            double rzn = 0.0;
            for (int64_t i = 0; i < nn; ++i) {
                z[i] = P->fdiag[i] * r[i];
                rzn += r[i] * z[i];
            }
            if (P->p.red_mode == 1) rzn = node_dot(P, r, z);
            const double beta = rzn / (rz > 1.0e-30 ? rz : 1.0e-30);
            for (int64_t i = 0; i < nn; ++i) p[i] = z[i] + beta * p[i];
            rz = rzn;
        }
    }
    filter_to_elements(P, x, dst);
    memcpy(P->flastx, x, (size_t)nn * sizeof(double));
    memcpy(P->flastrhs, rhs, (size_t)nn * sizeof(double));
}

void orc_filter_state(const orc_problem* P, double* lastx, double* lastrhs, double* diag) {
    const size_t nb = (size_t)P->nn * sizeof(double);
    if (lastx) memcpy(lastx, P->flastx, nb);
    if (lastrhs) memcpy(lastrhs, P->flastrhs, nb);
    if (diag) memcpy(diag, P->fdiag, nb);
}

void orc_filter_set_state(orc_problem* P, const double* lastx, const double* lastrhs) {
    const size_t nb = (size_t)P->nn * sizeof(double);
    memcpy(P->flastx, lastx, nb);
    memcpy(P->flastrhs, lastrhs, nb);
}

/* ------------------------------------------------------------------ float pow
 * pow_mode 0: x^p rounded once to float from double arithmetic (integer p by repeated
 * multiplication, else pow());  pow_mode 1: glibc libmvec powf in the blocking of the
 * reference build's vectorised loops (8-wide AVX2 blocks from index 0, then one 4-wide
 * block when 4..7 remain, then scalar powf). */
static float powf_rounded(float x, float p) {
    const double xd = (double)x;
    if (p == 3.0f) return (float)(xd * xd * xd);
    if (p == 2.0f) return (float)(xd * xd);
    if (p == 1.0f) return x;
    return (float)pow(xd, (double)p);
}

__m256 _ZGVdN8vv_powf(__m256, __m256);
__m128 _ZGVbN4vv_powf(__m128, __m128);

__attribute__((target("avx2,fma"))) static void powf_reference_blocks(const float* x, float p, float* out, int n) {
    int i = 0;
    if (n >= 8) {
        const int nb = n / 8;
        for (int b = 0; b < nb; ++b, i += 8)
            _mm256_storeu_ps(out + i, _ZGVdN8vv_powf(_mm256_loadu_ps(x + i), _mm256_set1_ps(p)));
    }
    if (n - i >= 4) {
        _mm_storeu_ps(out + i, _ZGVbN4vv_powf(_mm_loadu_ps(x + i), _mm_set1_ps(p)));
        i += 4;
    }
    for (; i < n; ++i) out[i] = powf(x[i], p);
}

static void pow_array(const orc_problem* P, const float* x, float p, float* out, int n) {
    if (P->p.pow_mode == 1) powf_reference_blocks(x, p, out, n);
    else
        for (int i = 0; i < n; ++i) out[i] = powf_rounded(x[i], p);
}

static float clamp01(float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); }

/* SIMP modulus driver.cpp:117-121: E = fma(rho^p, E0-Emin, Emin) in float, stored as double */
void orc_simp(const orc_problem* P, const float* xphys, double* E) {
    const int n = P->ne;
    float* rho = xcalloc((size_t)n, sizeof(float));
    float* pw = xcalloc((size_t)n, sizeof(float));
    for (int e = 0; e < n; ++e) rho[e] = clamp01(xphys[e]);
    pow_array(P, rho, P->p.penal, pw, n);
    const float dE = P->p.E0 - P->p.Emin;
    for (int e = 0; e < n; ++e) E[e] = (double)fmaf(pw[e], dE, P->p.Emin);
    free(rho);
    free(pw);
}

/* sensitivities driver.cpp:151-157 (compiled form: dc = ceNorm*(pw*((Emin-E0)*p)),
 * ceNorm = (float)(ce*(1/Csolid))) */
void orc_sens(const orc_problem* P, const float* xphys, const double* ce, double Csolid, float* dc) {
    const int n = P->ne;
    float* rho = xcalloc((size_t)n, sizeof(float));
    float* pw = xcalloc((size_t)n, sizeof(float));
    for (int e = 0; e < n; ++e) rho[e] = clamp01(xphys[e]);
    pow_array(P, rho, P->p.penal - 1.0f, pw, n);
    const float K = (P->p.Emin - P->p.E0) * P->p.penal;
    const double rc = 1.0 / Csolid;
    for (int e = 0; e < n; ++e) {
        const float cn = Csolid > 0 ? (float)(ce[e] * rc) : (float)ce[e];
        dc[e] = cn * (pw[e] * K);
    }
    free(rho);
    free(pw);
}

/* ------------------------------------------------------------------ float sums
 * Order of the reference build's vectorised std::accumulate (driver.cpp:181,188,201):
 * 8 lane sums over the first 8*floor(n/8) values, folded as
 * ((l0+l4)+(l2+l6)) + ((l1+l5)+(l3+l7)); a remainder of 4..7 values is added lane-wise to
 * (l0+l4,l1+l5,l2+l6,l3+l7) and folded as (m0+m2)+(m1+m3), then the last 0..3 values are
 * added one by one.  n <= 7 starts from zero lanes. */
static float fold4(const float m[4]) { return (m[1] + m[3]) + (m[0] + m[2]); }

static float vec8_sum(const float* t, int n) {
    float l[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int i = 0;
    float s;
    float h[4];
    if (n >= 8) {
        const int nb = n / 8;
        for (int b = 0; b < nb; ++b, i += 8)
            for (int j = 0; j < 8; ++j) l[j] = l[j] + t[i + j];
        for (int j = 0; j < 4; ++j) h[j] = l[j + 4] + l[j];
        s = fold4(h);
    } else {
        for (int j = 0; j < 4; ++j) h[j] = 0.0f;
        s = 0.0f;
    }
    const int rem = n - i;
    if (rem >= 4) {
        float m[4];
        for (int j = 0; j < 4; ++j) m[j] = h[j] + t[i + j];
        s = fold4(m);
        i += 4;
    }
    for (; i < n; ++i) s = s + t[i];
    return s;
}

static float seq_sum(const float* t, int n) {
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s = s + t[i];
    return s;
}

typedef struct { const int32_t* cell2e; const float* x; int sharp; } cell_f_ctx;
static double step_cell_f(double part, int64_t k, const void* vctx) {
    const cell_f_ctx* c = (const cell_f_ctx*)vctx;
    const int e = c->cell2e[k];
    if (e < 0) return part;
    const float v = c->x[e];
    return part + (double)(c->sharp ? v * (1.0f - v) : v);
}
/* FP64 sum of x (or x(1-x)) over the elements: canonical cell order when red_mode = 1 */
static double fp64_sum(const orc_problem* P, const float* x, int sharp) {
    if (P->p.red_mode == 1) {
        int32_t* m = cell_to_element(P);
        cell_f_ctx c = {m, x, sharp};
        const double s = canon_fold((int64_t)P->nx * P->ny * P->nz, step_cell_f, &c);
        free(m);
        return s;
    }
    double s = 0.0;
    for (int i = 0; i < P->ne; ++i) s += (double)(sharp ? x[i] * (1.0f - x[i]) : x[i]);
    return s;
}

float orc_vol_sum(const orc_problem* P, const float* x, int n) {
    if (P->p.vol_mode == 0) return vec8_sum(x, n);
    if (P->p.vol_mode == 1) return seq_sum(x, n);
    return (float)fp64_sum(P, x, 0);
}

/* sharpness 4*sum(x(1-x))/ne (driver.cpp:188) */
float orc_sharpness(const orc_problem* P, const float* x, int n) {
    if (P->p.vol_mode == 2) return 4.0f * (float)fp64_sum(P, x, 1) / (float)n;
    float* t = xcalloc((size_t)n, sizeof(float));
    for (int i = 0; i < n; ++i) t[i] = x[i] * (1.0f - x[i]);
    const float s = P->p.vol_mode == 0 ? vec8_sum(t, n) : seq_sum(t, n);
    free(t);
    return 4.0f * s / (float)n;
}

/* sqrt(max(1e-30, -dc*rl)) as the reference build's vectorised OC loop computes it:
 * y = rsqrt_approx(q); t = y*q; s = fma(y, t, -3) * (t * -0.5) on 8-wide blocks from index 0
 * and one 4-wide block, IEEE sqrt on the remaining 0..3 elements (and for n <= 3). */
__attribute__((target("avx2,fma"))) static void rsqrt_newton_blocks(const float* dc, float rl, float* out, int n) {
    int i = 0;
    if (n > 3) {
        const __m256 vr = _mm256_set1_ps(rl), tiny = _mm256_set1_ps(1e-30f);
        const __m256 m3 = _mm256_set1_ps(-3.0f), mh = _mm256_set1_ps(-0.5f);
        const __m256 sgn = _mm256_set1_ps(-0.0f), zero = _mm256_setzero_ps();
        for (; i + 8 <= n; i += 8) {
            __m256 q = _mm256_xor_ps(_mm256_mul_ps(_mm256_loadu_ps(dc + i), vr), sgn);
            q = _mm256_max_ps(q, tiny);
            __m256 y = _mm256_and_ps(_mm256_rsqrt_ps(q), _mm256_cmp_ps(zero, q, _CMP_NEQ_UQ));
            __m256 t = _mm256_mul_ps(y, q);
            __m256 e = _mm256_fmadd_ps(y, t, m3);
            _mm256_storeu_ps(out + i, _mm256_mul_ps(e, _mm256_mul_ps(t, mh)));
        }
        if (n - i >= 4) {
            const __m128 vr4 = _mm_set1_ps(rl), tiny4 = _mm_set1_ps(1e-30f);
            __m128 q = _mm_xor_ps(_mm_mul_ps(_mm_loadu_ps(dc + i), vr4), _mm_set1_ps(-0.0f));
            q = _mm_max_ps(q, tiny4);
            __m128 y = _mm_and_ps(_mm_rsqrt_ps(q), _mm_cmpneq_ps(_mm_setzero_ps(), q));
            __m128 t = _mm_mul_ps(y, q);
            __m128 e = _mm_fmadd_ps(y, t, _mm_set1_ps(-3.0f));
            _mm_storeu_ps(out + i, _mm_mul_ps(e, _mm_mul_ps(t, _mm_set1_ps(-0.5f))));
            i += 4;
        }
    }
    for (; i < n; ++i) {
        float q = -(dc[i] * rl);
        if (q < 1e-30f) q = 1e-30f;
        out[i] = sqrtf(q);
    }
}

/* dc = dcf / max(1e-3, x) (driver.cpp:166); approx_mode 1: r = rcp_approx(m),
 * r' = (r + r) - r*(r*m), dc = r' * dcf on 8/4-wide blocks, IEEE division on the rest. */
__attribute__((target("avx2,fma"))) static void rcp_newton_blocks(const float* dcf, const float* x, float* out, int n) {
    int i = 0;
    if (n > 3) {
        const __m256 lo = _mm256_set1_ps(1.0e-3f);
        for (; i + 8 <= n; i += 8) {
            const __m256 m = _mm256_max_ps(lo, _mm256_loadu_ps(x + i));
            const __m256 r = _mm256_rcp_ps(m);
            const __m256 rr = _mm256_mul_ps(r, _mm256_mul_ps(r, m));
            const __m256 r1 = _mm256_sub_ps(_mm256_add_ps(r, r), rr);
            _mm256_storeu_ps(out + i, _mm256_mul_ps(r1, _mm256_loadu_ps(dcf + i)));
        }
        if (n - i >= 4) {
            const __m128 m = _mm_max_ps(_mm_set1_ps(1.0e-3f), _mm_loadu_ps(x + i));
            const __m128 r = _mm_rcp_ps(m);
            const __m128 rr = _mm_mul_ps(r, _mm_mul_ps(r, m));
            const __m128 r1 = _mm_sub_ps(_mm_add_ps(r, r), rr);
            _mm_storeu_ps(out + i, _mm_mul_ps(r1, _mm_loadu_ps(dcf + i)));
            i += 4;
        }
    }
    for (; i < n; ++i) out[i] = dcf[i] / (1.0e-3f < x[i] ? x[i] : 1.0e-3f);
}

void orc_dc_scale(const orc_problem* P, const float* dcf, const float* x, float* dc) {
    const int n = P->ne;
    if (P->p.approx_mode == 1) rcp_newton_blocks(dcf, x, dc, n);
    else
        for (int e = 0; e < n; ++e) dc[e] = dcf[e] / (1.0e-3f < x[e] ? x[e] : 1.0e-3f);
}

/* ------------------------------------------------------------------ OC update
 * driver.cpp:170-184 (compiled form: -dc*(2/(l1+l2)), volume = sum * (1/(float)ne)) */
int orc_oc(const orc_problem* P, const float* x, const float* dc, float V0, float* xnew, float* change, float* lmid_out) {
    const int n = P->ne;
    float l1 = 0.0f, l2 = 1e9f, lmid = 0.0f;
    const float move = 0.2f;
    const float rne = 1.0f / (float)n;
    int passes = 0;
    float* sq = P->p.approx_mode == 1 ? xcalloc((size_t)n, sizeof(float)) : NULL;
    while ((double)((l2 - l1) / (l1 + l2)) > 1e-6) {
        lmid = 0.5f * (l1 + l2);
        const float rl = 2.0f / (l1 + l2);
        if (sq) rsqrt_newton_blocks(dc, rl, sq, n);
        for (int e = 0; e < n; ++e) {
            float q = -(dc[e] * rl);
            if (q < 1e-30f) q = 1e-30f;
            const float val = sq ? sq[e] : sqrtf(q);
            const float lo = x[e] - move, hi = x[e] + move;
            float xe = x[e] * val;
            xe = xe < lo ? lo : (hi < xe ? hi : xe);
            xe = xe < 0.0f ? 0.0f : (1.0f < xe ? 1.0f : xe);
            xnew[e] = 1.0e-3f < xe ? xe : 1.0e-3f;
            if (P->passive[e]) xnew[e] = 1.0f;   /* passive elements stay solid (TOP3D_XL.m:152,166) */
        }
        float vol;
        if (P->p.vol_mode == 2) vol = orc_vol_sum(P, xnew, n) / (float)n;
        else vol = orc_vol_sum(P, xnew, n) * rne;
        if (vol - V0 > 0) l1 = lmid;
        else l2 = lmid;
        ++passes;
    }
    free(sq);
    float ch = 0.0f;
    for (int e = 0; e < n; ++e) {
        const float d = fabsf(xnew[e] - x[e]);
        if (d > ch) ch = d;
    }
    *change = ch;
    if (lmid_out) *lmid_out = lmid;
    return passes;
}

/* ------------------------------------------------------------------ driver loop
 * TOP3D_XL_GLOBAL (driver.cpp:23-218): solid reference solve, then SIMP -> (lazy MG
 * rebuild at loop 1 and every 5th) -> warm-started PCG -> compliance -> sensitivities ->
 * PDE filter of x*dc -> OC -> change/sharpness, while loop<nLoop && change>1e-4 &&
 * sharpness>0.01. */
int orc_design_loop(orc_problem* P, float V0, int nLoop, float rMin, double* Csolid_out, orc_iter_record* recs,
                    float* xfinal) {
    const int ne = P->ne;
    const int64_t nf = P->nf;
    orc_filter_setup(P, rMin);
    float* x = xcalloc((size_t)ne, sizeof(float));
    float* xnew = xcalloc((size_t)ne, sizeof(float));
    float* dc = xcalloc((size_t)ne, sizeof(float));
    float* xdc = xcalloc((size_t)ne, sizeof(float));
    float* dcf = xcalloc((size_t)ne, sizeof(float));
    double* E = xcalloc((size_t)ne, sizeof(double));
    double* ce = xcalloc((size_t)ne, sizeof(double));
    /* load cases (external models, TOP3D_XL.m:105,125,605-621): each solved from its own previous
     * displacement; ce = sum_k ce_k / K accumulated as acc = w ce_0, then acc + w ce_k; C = sum E ce */
    const int K = P->ncases > 1 ? P->ncases : 1;
    const double w = 1.0 / K;
    double* b = xcalloc((size_t)nf * K, sizeof(double));
    double* u = xcalloc((size_t)nf * K, sizeof(double));
    double* cek = K > 1 ? xcalloc((size_t)ne, sizeof(double)) : NULL;
    for (int e = 0; e < ne; ++e) { x[e] = V0; E[e] = (double)P->p.E0; }
    for (int k = 0; k < K; ++k) {
        const double* Fk = K > 1 ? P->Fcases + (int64_t)k * P->ndof : P->F;
        for (int64_t i = 0; i < nf; ++i) b[k * nf + i] = Fk[P->free_dofs[i]];
    }
    const double tol = (double)P->p.cg_tol;
#define SOLVE_CASES(ITS, CTOTAL)                                                                   \
    do {                                                                                           \
        if (K == 1) {                                                                              \
            ITS = orc_pcg(P, E, b, u, tol, P->p.cg_max_it);                                        \
            CTOTAL = orc_compliance(P, E, u, ce);                                                  \
        } else {                                                                                   \
            ITS = 0;                                                                               \
            for (int k = 0; k < K; ++k) {                                                          \
                ITS += orc_pcg(P, E, b + k * nf, u + k * nf, tol, P->p.cg_max_it);                 \
                orc_compliance(P, E, u + k * nf, cek);                                             \
                for (int e = 0; e < ne; ++e) ce[e] = k == 0 ? w * cek[e] : ce[e] + w * cek[e];     \
            }                                                                                      \
            CTOTAL = orc_objective(P, E, ce, 1.0);                                                 \
        }                                                                                          \
    } while (0)
    orc_mg_build(P, E);
    int its0 = 0;
    double Csolid = 0.0;
    SOLVE_CASES(its0, Csolid);
    (void)its0;
    if (Csolid_out) *Csolid_out = Csolid;
    int loop = 0;
    float change = 1.0f, sharp = 1.0f;
    while (loop < nLoop && change > 1e-4 && sharp > 0.01) {
        ++loop;
        orc_simp(P, x, E);
        if (loop == 1 || loop % 5 == 0) orc_mg_build(P, E);
        int its = 0;
        double Cdummy = 0.0;
        SOLVE_CASES(its, Cdummy);
        (void)Cdummy;
        const double Cdisp = orc_objective(P, E, ce, Csolid);
        orc_sens(P, x, ce, Csolid, dc);
        for (int e = 0; e < ne; ++e) xdc[e] = x[e] * dc[e];
        orc_filter_apply(P, xdc, dcf);
        orc_dc_scale(P, dcf, x, dc);
        float lm = 0.0f;
        const int passes = orc_oc(P, x, dc, V0, xnew, &change, &lm);
        memcpy(x, xnew, (size_t)ne * sizeof(float));
        sharp = orc_sharpness(P, x, ne);
        const float vf = orc_vol_sum(P, x, ne) / (float)ne;
        orc_iter_record* R = &recs[loop - 1];
        R->loop = loop; R->pcg_iters = its; R->obj = Cdisp; R->vol = vf; R->sharp = sharp;
        R->cons = vf - V0; R->change = change; R->lmid = lm; R->bisections = passes;
    }
    if (xfinal) memcpy(xfinal, x, (size_t)ne * sizeof(float));
#undef SOLVE_CASES
    free(x); free(xnew); free(dc); free(xdc); free(dcf); free(E); free(ce); free(b); free(u); free(cek);
    return loop;
}

/* ------------------------------------------------------------------ lifecycle, accessors */
static orc_problem* create_common(orc_problem* P, int nely, int nelx, int nelz);

orc_problem* orc_create(int nely, int nelx, int nelz, const orc_params* prm) {
    orc_problem* P = xcalloc(1, sizeof(orc_problem));
    if (prm) P->p = *prm;
    else orc_params_default(&P->p);
    return create_common(P, nely, nelx, nelz);
}

/* An external model (TopVoxel, TOP3D_XL.m:458-586) in the file's index spaces; the arrays must outlive
 * the problem.  Fixations and loads are on distinct nodes (the file reader keeps the first row). */
orc_problem* orc_create_voxel(int nely, int nelx, int nelz, const orc_params* prm, const uint8_t* voxel, int nfix,
                              const int64_t* fix_node, const uint8_t* fix_bits, int ncases, const int* case_n,
                              const int64_t* load_node, const double* load_f) {
    orc_problem* P = xcalloc(1, sizeof(orc_problem));
    if (prm) P->p = *prm;
    else orc_params_default(&P->p);
    P->voxel = voxel;
    P->nfix = nfix; P->fix_node = fix_node; P->fix_bits = fix_bits;
    P->ncases = ncases; P->case_n = case_n; P->load_node = load_node; P->load_f = load_f;
    return create_common(P, nely, nelx, nelz);
}

static orc_problem* create_common(orc_problem* P, int nely, int nelx, int nelz) {
    P->nelx = nelx; P->nely = nely; P->nelz = nelz;
    /* L from the solid voxel count (fea.cpp:190 for the cuboid; numel(find(voxelizedVolume_)) for an external
     * model, TOP3D_XL.m:1765-1774) */
    uint64_t nsolid = (uint64_t)nelx * nely * nelz;
    if (P->voxel) {
        nsolid = 0;
        for (int64_t k = 0; k < (int64_t)nelx * nely * nelz; ++k) nsolid += P->voxel[k] != 0;
    }
    const int L = pad_levels(nsolid);
    P->nx = pad_dim(nelx, L); P->ny = pad_dim(nely, L); P->nz = pad_dim(nelz, L);
    P->nnx = P->nx + 1; P->nny = P->ny + 1; P->nnz = P->nz + 1;
    P->nn = (int64_t)P->nnx * P->nny * P->nnz;
    P->ndof = 3 * P->nn;
    build_mesh(P);
    build_bcs(P);
    hex8_stiffness(0.3, 1.0, P->Ke);   /* fea.cpp:345 passes nu=0.3 literally */
    build_hierarchy(P);
    build_masks(P);
    P->r = xcalloc((size_t)P->nf, sizeof(double));
    P->z = xcalloc((size_t)P->nf, sizeof(double));
    P->pp = xcalloc((size_t)P->nf, sizeof(double));
    P->Ap = xcalloc((size_t)P->nf, sizeof(double));
    return P;
}

void orc_destroy(orc_problem* P) {
    if (!P) return;
    free(P->ele_full); free(P->enod); free(P->bucket); free(P->isfree); free(P->free_dofs);
    free(P->dof2free); free(P->F); free(P->Fcases); free(P->passive);
    for (int l = 0; l < P->nlev; ++l) { free(P->lv[l].mask); free(P->lv[l].diag); free(P->lv[l].r); free(P->lv[l].x); }
    free(P->Lc); free(P->Xc); free(P->tmpf); free(P->r); free(P->z); free(P->pp); free(P->Ap);
    free(P->fdiag); free(P->flastx); free(P->flastrhs); free(P->frhs); free(P->fx); free(P->fr); free(P->fz);
    free(P->fp); free(P->fAp);
    free(P);
}

void orc_info(const orc_problem* P, int64_t* info) {
    info[0] = P->nx; info[1] = P->ny; info[2] = P->nz;
    info[3] = P->ne; info[4] = P->nn; info[5] = P->nf; info[6] = P->nlev;
    for (int l = 0; l < P->nlev; ++l) {
        info[7 + 4 * l + 0] = P->lv[l].nx;
        info[7 + 4 * l + 1] = P->lv[l].ny;
        info[7 + 4 * l + 2] = P->lv[l].nz;
        info[7 + 4 * l + 3] = P->lv[l].span;
    }
}

void orc_ele_map_back(const orc_problem* P, int32_t* out) { memcpy(out, P->ele_full, (size_t)P->ne * 4); }
void orc_free_dofs(const orc_problem* P, int32_t* out) { memcpy(out, P->free_dofs, (size_t)P->nf * 4); }
void orc_bfree(const orc_problem* P, double* out) {
    for (int64_t i = 0; i < P->nf; ++i) out[i] = P->F[P->free_dofs[i]];
}
void orc_ke(const orc_problem* P, double* out) { memcpy(out, P->Ke, sizeof P->Ke); }
void orc_set_ke(orc_problem* P, const double* Ke) { memcpy(P->Ke, Ke, sizeof P->Ke); }
void orc_mg_diag(const orc_problem* P, int level, double* out) {
    memcpy(out, P->lv[level].diag, (size_t)(3 * P->lv[level].nn) * sizeof(double));
}
void orc_mg_mask(const orc_problem* P, int level, uint8_t* out) {
    memcpy(out, P->lv[level].mask, (size_t)(3 * P->lv[level].nn));
}

/* ------------------------------------------------------------------ surface export (test infrastructure)
 * io.cpp:80-87 scatters xPhys onto vol[ny*nx*ez + ny*ex + y] (y is the flipped row, fea.cpp:222);
 * voxel_surface.hpp:44-92 visits z, then x, then y, and per voxel the faces -X, +X, -Y, +Y, -Z, +Z of an
 * inside voxel (value >= iso) whose neighbour is outside or absent; each face is 4 vertices (x, y, z)
 * and 2 triangles (0,1,2), (0,2,3) (voxel_surface.hpp:17-43); export_stl.hpp:14-33 writes an 80-byte
 * header, the triangle count and 50-byte records (zero normal, 3 vertices, zero attribute). */
static void stl_face(FILE* f, int axis, float y0, float x0, float z0) {
    float v[4][3];
    for (int i = 0; i < 4; ++i) { v[i][0] = x0; v[i][1] = y0; v[i][2] = z0; }
    if (axis == 0) {        /* plane x = const: vary y, z */
        v[1][1] += 1.0f; v[2][1] += 1.0f; v[2][2] += 1.0f; v[3][2] += 1.0f;
    } else if (axis == 1) { /* plane y = const: vary x, z */
        v[1][0] += 1.0f; v[2][0] += 1.0f; v[2][2] += 1.0f; v[3][2] += 1.0f;
    } else {                /* plane z = const: vary x, y */
        v[1][0] += 1.0f; v[2][0] += 1.0f; v[2][1] += 1.0f; v[3][1] += 1.0f;
    }
    static const int tri[2][3] = {{0, 1, 2}, {0, 2, 3}};
    const float n[3] = {0.0f, 0.0f, 0.0f};
    const uint16_t attr = 0;
    for (int t = 0; t < 2; ++t) {
        fwrite(n, 4, 3, f);
        for (int k = 0; k < 3; ++k) fwrite(v[tri[t][k]], 4, 3, f);
        fwrite(&attr, 2, 1, f);
    }
}

int64_t orc_export_stl(const orc_problem* P, const float* xphys, const char* path, float iso) {
    const int ny = P->ny, nx = P->nx, nz = P->nz;
    const int64_t nv = (int64_t)ny * nx * nz;
    float* vol = xcalloc((size_t)nv, sizeof(float));
    for (int64_t e = 0; e < P->ne; ++e) vol[P->ele_full[e]] = xphys[e];
    FILE* f = fopen(path, "wb");
    if (!f) { free(vol); return -1; }
    char header[80];
    memset(header, 0, sizeof header);
    strncpy(header, "Generated by TOP3D_XL", 79);
    fwrite(header, 1, 80, f);
    uint32_t ntri = 0;
    fwrite(&ntri, 4, 1, f);   /* patched below */
#define AT(y, x, z) (vol[(int64_t)(y) + (int64_t)ny * (x) + (int64_t)ny * nx * (z)] >= iso)
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                if (!AT(y, x, z)) continue;
                if (x == 0 || !AT(y, x - 1, z)) { stl_face(f, 0, (float)y, (float)x, (float)z); ntri += 2; }
                if (x == nx - 1 || !AT(y, x + 1, z)) { stl_face(f, 0, (float)y, (float)(x + 1), (float)z); ntri += 2; }
                if (y == 0 || !AT(y - 1, x, z)) { stl_face(f, 1, (float)y, (float)x, (float)z); ntri += 2; }
                if (y == ny - 1 || !AT(y + 1, x, z)) { stl_face(f, 1, (float)(y + 1), (float)x, (float)z); ntri += 2; }
                if (z == 0 || !AT(y, x, z - 1)) { stl_face(f, 2, (float)y, (float)x, (float)z); ntri += 2; }
                if (z == nz - 1 || !AT(y, x, z + 1)) { stl_face(f, 2, (float)y, (float)x, (float)(z + 1)); ntri += 2; }
            }
#undef AT
    fseek(f, 80, SEEK_SET);
    fwrite(&ntri, 4, 1, f);
    fclose(f);
    free(vol);
    return (int64_t)ntri;
}
