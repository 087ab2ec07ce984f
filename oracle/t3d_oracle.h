/* Test infrastructure only -- the CPU oracle for the per-design-iteration hot path of
 * natashahirt/AlgorithmEngineering_AltProject (`top3d_xl_cli GLOBAL`).
 *
 * A single-threaded C11 restatement of the reference algorithm, used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the CHECKER of the CUDA
 * path.  It is never linked into, or called by, the product.
 *
 * All arrays use the reference's own layouts:
 *   element arrays  [ne]       compact element order = 64-bit Morton order of (ex,ey,ez)
 *                              (reference cpp/src/fea.cpp:289-317)
 *   free vectors    [nfree]    ascending global DOF 3*node+c over free DOFs
 *                              (fea.cpp:420-421), node = nnx*nny*iz + nnx*iy + ix
 *   node vectors    [numNodes] lexicographic nodes (fea.cpp:253-255)
 *
 * Pinning: tests/test_oracle_pin.py checks this file against the reference built from
 * its unmodified sources (oracle/_ref/libt3d_ref.so, see oracle/Makefile) and against the
 * golden vectors in tests/golden/ that were generated from that build.
 */
#ifndef T3D_ORACLE_H
#define T3D_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
    float E0, Emin, nu, penal;      /* GlobalParams core.hpp:26-42 (nu is not used: Ke uses 0.3, fea.cpp:345) */
    float cg_tol;                   /* core.hpp:35 */
    int   cg_max_it;                /* core.hpp:36 */
    int   mg_nondyadic;             /* MGPrecondConfig multigrid.hpp:9-13, driver.cpp:54 */
    int   mg_max_levels;
    float mg_weight;
    int   pow_mode;                 /* 0: correctly rounded float pow;
                                       1: glibc libmvec powf blocking of the reference build (driver.cpp:117-121,151-157) */
    int   vol_mode;                 /* OC volume sum: 0 = 8-lane vector-sum order of the reference build,
                                       1 = sequential float (source order), 2 = FP64 */
    int   approx_mode;              /* 0 = IEEE sqrtf and division (source semantics);
                                       1 = the reference build's x86 approximations: vrsqrtps + one Newton
                                           step for the OC square root (driver.cpp:176) and vrcpps + one
                                           Newton step for dc/max(1e-3,x) (driver.cpp:166), both on 8/4-wide
                                           blocks with exact IEEE ops on the last 0..3 elements.  Their bits
                                           depend on the x86 CPU's rsqrt/rcp approximation tables. */
    int   red_mode;                 /* inner products and sums: 0 = sequential in the reference's loop order;
                                       1 = the CUDA path's canonical deterministic order (grid-stride over
                                           nodes/cells with 1184 x 256 threads, warp and block butterflies),
                                           so that the two can be compared bit for bit */
    int   coarse_full;              /* 0 = the reference's coarsest assembly (s = coarsest level's own span);
                                       1 = full Galerkin operator of the grid (s = product of the spans) */
} orc_params;

typedef struct orc_iter_record {    /* one line of driver.cpp:205-211 */
    int    loop;
    int    pcg_iters;
    double obj;                     /* Cdisp */
    float  vol, sharp, cons, change;
    float  lmid;                    /* final OC multiplier */
    int    bisections;
} orc_iter_record;

typedef struct orc_problem orc_problem;

void orc_params_default(orc_params* p);
orc_problem* orc_create(int nely, int nelx, int nelz, const orc_params* p);
/* external model (TopVoxel): voxel[k], k = y + nely*(x + nelx*z), 0 void / 1 solid / 2 passive; fixations
 * and loads on file nodes m = y + (nely+1)*(x + (nelx+1)*z); load cases concatenated, case k has case_n[k]
 * nodes (3 forces each).  The arrays must outlive the problem. */
orc_problem* orc_create_voxel(int nely, int nelx, int nelz, const orc_params* prm, const uint8_t* voxel, int nfix,
                              const int64_t* fix_node, const uint8_t* fix_bits, int ncases, const int* case_n,
                              const int64_t* load_node, const double* load_f);
void orc_destroy(orc_problem* P);

/* info: resX,resY,resZ, numElements, numNodes, nFree, nLevels, then per level (resX,resY,resZ,span) */
void orc_info(const orc_problem* P, int64_t* info);
void orc_ele_map_back(const orc_problem* P, int32_t* out);
void orc_free_dofs(const orc_problem* P, int32_t* out);
void orc_bfree(const orc_problem* P, double* out);
void orc_ke(const orc_problem* P, double* out);
void orc_set_ke(orc_problem* P, const double* Ke);

void   orc_matvec(orc_problem* P, const double* E, const double* u, double* y);
void   orc_mg_build(orc_problem* P, const double* E);
int    orc_mg_coarse_n(const orc_problem* P);
void   orc_mg_diag(const orc_problem* P, int level, double* out);
void   orc_mg_mask(const orc_problem* P, int level, uint8_t* out);
int    orc_coarse_matrix(orc_problem* P, const double* E, double* out);
void   orc_vcycle(orc_problem* P, const double* r, double* z);
int    orc_pcg(orc_problem* P, const double* E, const double* b, double* x, double tol, int maxit);
double orc_compliance(orc_problem* P, const double* E, const double* u, double* ce);
double orc_objective(const orc_problem* P, const double* E, const double* ce, double Csolid);

void orc_filter_setup(orc_problem* P, float rmin);
void orc_filter_apply(orc_problem* P, const float* src, float* dst);
void orc_filter_state(const orc_problem* P, double* lastx, double* lastrhs, double* diag);
void orc_filter_set_state(orc_problem* P, const double* lastx, const double* lastrhs);

void  orc_simp(const orc_problem* P, const float* xphys, double* E);
void  orc_sens(const orc_problem* P, const float* xphys, const double* ce, double Csolid, float* dc);
void  orc_dc_scale(const orc_problem* P, const float* dcf, const float* x, float* dc);
int   orc_oc(const orc_problem* P, const float* x, const float* dc, float V0, float* xnew, float* change, float* lmid);
float orc_vol_sum(const orc_problem* P, const float* x, int n);
float orc_sharpness(const orc_problem* P, const float* x, int n);

/* full driver loop (driver.cpp:23-218) for one simulation; returns number of records */
int orc_design_loop(orc_problem* P, float V0, int nLoop, float rMin, double* Csolid,
                    orc_iter_record* recs, float* xfinal);

/* export_surface_stl (io.cpp:80-87): element densities (Morton order) scattered onto the padded
 * [ny][nx][nz] volume, boundary faces at threshold iso (voxel_surface.hpp:12-93), binary STL
 * (export_stl.hpp:14-33).  Returns the triangle count, or -1 when the file cannot be written. */
int64_t orc_export_stl(const orc_problem* P, const float* xphys, const char* path, float iso);

#ifdef __cplusplus
}
#endif
#endif
