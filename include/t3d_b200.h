/* t3d_b200 -- C-ABI of the B200 (sm_100a) implementation of the per-design-iteration hot path of
 * natashahirt/AlgorithmEngineering_AltProject (`top3d_xl_cli GLOBAL`): the matrix-free hex8
 * K(rho)u product inside PCG, the geometric-multigrid V-cycle preconditioner, the PDE filter and
 * the OC update.
 *
 * Conventions shared by every entry point:
 *   - plain pointers to HOST memory, sizes as int64; no CUDA or C++ types cross the boundary;
 *   - every call returns an int status (T3D_OK = 0); t3d_last_error() gives the message;
 *   - element arrays use the reference's compact element order (64-bit Morton order of the
 *     element indices, fea.cpp:289-317), length num_elements;
 *   - free-DOF vectors use the reference's order (ascending global DOF 3*node+c over free DOFs,
 *     fea.cpp:420-421), length num_free;
 *   - node arrays use the reference's lexicographic nodes (fea.cpp:253-255), length num_nodes;
 *   - all device state (moduli, displacement, MG hierarchy, filter warm start) lives in the
 *     context; a context is bound to one GPU and is not thread-safe (like the reference's
 *     Preconditioner closure and PDEFilter, preconditioner.cpp:82-88, filter.hpp:8-14).
 * The library needs a CUDA device; there is no CPU fallback: without one t3d_create fails with
 * T3D_ERR_NO_DEVICE.
 */
#ifndef T3D_B200_H
#define T3D_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    T3D_OK = 0,
    T3D_ERR_INVALID = 1,       /* bad argument or call order */
    T3D_ERR_CUDA = 2,          /* CUDA runtime error */
    T3D_ERR_OOM = 3,           /* device allocation failed */
    T3D_ERR_NO_DEVICE = 4,     /* no CUDA device / device index out of range */
    T3D_ERR_UNSUPPORTED = 5,   /* configuration the library does not handle */
    T3D_ERR_NUMERIC = 6        /* non-finite value or non-converging bisection */
};

enum { T3D_SUM_REFERENCE = 0, T3D_SUM_FP64 = 1 };   /* OC volume / sharpness summation order */
/* solver precision of the design loop: T3D_FP64 = PCG_free in FP64; T3D_MIXED = FP32 inner MG-PCG (FP64
 * inner products, alpha/beta, coarsest solve) inside FP64 defect correction on the true residual */
enum { T3D_FP64 = 0, T3D_MIXED = 1 };
/* FP32 K(E)p of the mixed form: AUTO = the modal (corner-Hadamard, 45-nonzero) form whenever Ke is the
 * stiffness of an axis-aligned cubic isotropic voxel (always for the built-in Ke), else the dense
 * 24x24 form; DENSE = always the dense form */
enum { T3D_MATVEC32_AUTO = 0, T3D_MATVEC32_DENSE = 1 };
/* dense coarsest operator: REFERENCE = the reference's assembly (coarsest.cpp:138-323), which samples the
 * s^3 fine elements of each coarse element with s the coarsest level's own span, i.e. only a corner
 * sub-block of the grid when there are more than two levels (on some grids PCG then stalls);
 * FULL = the Galerkin operator of the whole grid (s = product of all spans) */
enum { T3D_COARSE_REFERENCE = 0, T3D_COARSE_FULL = 1 };
/* FP64 K(E)u (t3d_matvec, FP64 PCG, the mixed form's outer residual): AUTO = element-streaming kernel,
 * NODES = node-centric gather kernel.  Both are bit-identical to the reference's product. */
enum { T3D_MATVEC64_AUTO = 0, T3D_MATVEC64_NODES = 1 };
/* V-cycle: ADAPTED = the reference's (preconditioner.cpp:88-265: no residual smoothing, restricted
 * diagonals); STANDARD = smoothing with the true residual on every level, Galerkin coarse operators and
 * the transposed prolongation as restriction (the MATLAB original's 'Standard', TOP3D_XL.m:772-807);
 * FP64 precision only */
enum { T3D_VCYCLE_ADAPTED = 0, T3D_VCYCLE_STANDARD = 1 };

typedef struct t3d_params {
    float E0, Emin, nu, penal;    /* GlobalParams core.hpp:26-33 (Ke always uses nu = 0.3, fea.cpp:345) */
    float cg_tol;                 /* core.hpp:35 */
    int   cg_max_it;              /* core.hpp:36 */
    int   mg_nondyadic;           /* MGPrecondConfig multigrid.hpp:9-13 as set in driver.cpp:54 */
    int   mg_max_levels;
    float mg_weight;
    float filter_rmin;            /* top3d_cli.cpp:33: sqrt(3) cells */
    int   oc_sum_order;           /* T3D_SUM_REFERENCE (bit-identical bisection) or T3D_SUM_FP64 */
    int   precision;              /* T3D_FP64 or T3D_MIXED (design loop only; t3d_pcg is always FP64) */
    int   device;                 /* CUDA device ordinal */
    int   matvec32_form;          /* mixed precision only: T3D_MATVEC32_AUTO or T3D_MATVEC32_DENSE */
    int   mg_coarse_assembly;     /* T3D_COARSE_REFERENCE (default) or T3D_COARSE_FULL */
    int   matvec64_form;          /* T3D_MATVEC64_AUTO (default) or T3D_MATVEC64_NODES */
    int   mg_vcycle;              /* T3D_VCYCLE_ADAPTED (default) or T3D_VCYCLE_STANDARD */
    float mg_standard_weight;     /* Jacobi weight of the Standard V-cycle (0 = the default 0.35): below 2 / 5.36, where
                                     5.36 bounds lambda_max(D^-1 K) for the hex8 Ke and any moduli (Gershgorin),
                                     so its residual smoother converges; the reference's 0.6 does not */
    int   mg_rebuild_period;      /* design iterations between MG rebuilds: 5 = the reference's loop 1 and every
                                     5th (driver.cpp:132); 1 = every iteration; 0 = the default (5) */
    int   matvec32_tile;          /* tile shape of the modal FP32 K(E)p: 0 = chosen by timing every shape on the
                                     grid (the default); k >= 1 = shape k-1 (all shapes give identical results) */
} t3d_params;

/* Problem spec beyond the reference's built-in cantilever (the reference hard-codes one load case and a
 * full cuboid, fea.cpp:181-447; the MATLAB original reads loads and passive regions from files,
 * TOP3D_XL.m:1319-1362,1536-1612).  Fixations stay the reference's: the x = 0 face and every node
 * touched by no solid element (fea.cpp:374-417). */
enum { T3D_LOAD_TIP_LINE = 0, T3D_LOAD_TOP_TRACTION = 1, T3D_LOAD_TORSION = 2 };
#define T3D_MAX_VOIDS 4
typedef struct t3d_problem {
    int    load_case;             /* T3D_LOAD_*: TIP_LINE = the reference's -Z line load at x = nelx;
                                     TOP_TRACTION = total -1 in z over the top-face nodes (z = nelz);
                                     TORSION = +1 / -1 in y over the lines x = nelx, z = nelz / z = 0 */
    int    num_voids;             /* passive-void ellipsoids, 0..T3D_MAX_VOIDS */
    double voids[T3D_MAX_VOIDS][6]; /* centre (ex, ey, ez) and radii (rx, ry, rz) in element units of the
                                     reference's element coordinates; an element whose centre
                                     (ex+0.5, ey+0.5, ez+0.5) lies inside is absent from the model */
} t3d_problem;

typedef struct t3d_info {
    int64_t res[3];               /* padded element counts resX,resY,resZ (padding.hpp:42-53) */
    int64_t orig[3];              /* original nelx, nely, nelz */
    int64_t num_elements;         /* solid elements */
    int64_t num_nodes;
    int64_t num_free;
    int64_t num_levels;           /* multigrid levels (hierarchy.cpp:84-138) */
    int64_t levels[8][4];         /* per level resX,resY,resZ,span */
    int64_t coarse_n;             /* dense coarsest system size, 0 = Jacobi coarsest */
    int64_t coarse_cholesky_ok;   /* 1 when the last MG set-up factorised the coarsest matrix */
    int64_t device_bytes;         /* device memory held by the context */
    int64_t kernel_launches;      /* kernels launched by this context so far (graph nodes included) */
    int64_t matvec32_modal;       /* 1 when the mixed form's FP32 K(E)p uses the modal kernel */
    int64_t matvec32_tile[4];     /* tile shape the modal kernel's autotuner chose: threads in x, threads in y,
                                     plane-ring slots, plane staging (0 per-thread cp.async, 1 the same with packed
                                     FP32x2 arithmetic, 2 packed arithmetic with TMA bulk tensor copies) */
    int64_t matvec64_kernel;      /* FP64 K(E)u kernel: 0 node-centric, 1 streaming with Ke from the constant bank,
                                     2 streaming with the built-in Ke's magnitudes in registers */
    int64_t matvec32_variant;     /* index of the modal tile shape (params.matvec32_tile - 1 selects it) */
    int64_t last_outer_passes;    /* mixed precision: FP64 defect-correction passes of the last solve */
} t3d_info;

typedef struct t3d_iter_record {  /* one design iteration (driver.cpp:205-216) */
    int    loop;
    int    pcg_iters;
    double obj;                   /* Cdisp */
    float  vol, sharp, cons, change;
    float  lmid;
    int    bisections;
    double t_total, t_cg, t_opt, t_filter;  /* seconds, CUDA-event timed */
} t3d_iter_record;

/* --------------------------------------------------------------- lifecycle */
int  t3d_params_default(t3d_params* p);
/* CreateVoxelFEAmodel_Cuboid + ApplyBoundaryConditions + mg::build_static_once + SetupPDEFilter
 * (fea.cpp:181-447, preconditioner.cpp:19-34, filter.cpp:9-75) for the built-in cantilever. */
int  t3d_create(int nely, int nelx, int nelz, const t3d_params* p, struct t3d_context** out);
/* t3d_create for a problem spec: load case and passive voids.  Element arrays cover only the solid
 * (non-void) elements, in the reference's Morton order of those elements */
int  t3d_create_problem(int nely, int nelx, int nelz, const t3d_params* p, const t3d_problem* problem,
                        struct t3d_context** out);
/* External design domains in the MATLAB original's TopVoxel format, version 1.0 (CreateVoxelFEAmodel,
 * TOP3D_XL.m:458-586): solid voxels, passive elements (kept at density 1 by the OC update,
 * TOP3D_XL.m:152,166), per-node DOF fixations and per-node loads; the reference's built-in x = 0
 * fixation and tip load are not applied.  Element arrays cover the solid voxels in the reference's Morton
 * order.  Further load cases are solved one after the other in each design iteration and the element
 * compliance is their mean (TOP3D_XL.m:605-621); the load and displacement the context exposes are
 * case 1's.  t3d_topvoxel_info parses only (no device needed): info[8] = nelx, nely, nelz, solid
 * voxels, passive elements, fixed nodes, loaded nodes (case 1), additional load cases. */
int  t3d_topvoxel_info(const char* path, int64_t* info8);
int  t3d_create_from_topvoxel(const char* path, const t3d_params* p, struct t3d_context** out);
int  t3d_destroy(struct t3d_context* ctx);
int  t3d_get_info(const struct t3d_context* ctx, t3d_info* info);
const char* t3d_last_error(void);

/* --------------------------------------------------------------- model data (reference layouts) */
/* ComputeVoxelKe (fea.hpp:37, fea.cpp:117-179): unit-modulus hex8 stiffness of a cubic voxel of edge
 * cell_size, row-major 24x24, local DOF 3a+c; host only, no device or context needed */
int  t3d_voxel_ke(double nu, double cell_size, double* ke576);
int  t3d_get_ke(const struct t3d_context* ctx, double* ke576);            /* ComputeVoxelKe fea.cpp:117 */
int  t3d_set_ke(struct t3d_context* ctx, const double* ke576);   /* invalidates the MG hierarchy: the next
                                                                     design step rebuilds it, t3d_pcg / t3d_vcycle
                                                                     need t3d_mg_setup first */
int  t3d_get_element_map(struct t3d_context* ctx, int32_t* ele_map_back); /* mesh.eleMapBack core.hpp:60 */
int  t3d_get_free_dofs(struct t3d_context* ctx, int32_t* free_dofs);      /* Problem::freeDofIndex core.hpp:88 */
int  t3d_get_load(struct t3d_context* ctx, double* b_free);               /* restrict_to_free(F) solver.cpp:12 */

/* --------------------------------------------------------------- operators (host buffers) */
/* K_times_u_finest (fea.hpp:42-45, fea.cpp:763-837) */
int  t3d_matvec(struct t3d_context* ctx, const double* ele_E, const double* u_free, double* y_free);
/* K_times_u_finest in the FP32 form used by the mixed-precision inner solve (mixed contexts only):
 * inputs rounded to FP32, y returned widened to FP64; same layouts as t3d_matvec */
int  t3d_matvec32(struct t3d_context* ctx, const double* ele_E, const double* u_free, double* y_free);
/* mg::make_diagonal_preconditioner_from_static (multigrid.hpp:66-68, preconditioner.cpp:38-79) */
int  t3d_mg_setup(struct t3d_context* ctx, const double* ele_E);
/* the preconditioner closure z = M^-1 r (preconditioner.cpp:88-265) */
int  t3d_vcycle(struct t3d_context* ctx, const double* r_free, double* z_free);
/* the preconditioner in the FP32 form of the mixed-precision inner solve (mixed contexts, after
 * t3d_mg_setup): r rounded to FP32, z returned widened to FP64 */
int  t3d_vcycle32(struct t3d_context* ctx, const double* r_free, double* z_free);
/* PCG_free (solver.hpp:24-27, solver.cpp:87-217) with the preconditioner of t3d_mg_setup;
 * x_free is the warm start on entry and the solution on return */
int  t3d_pcg(struct t3d_context* ctx, const double* ele_E, const double* b_free, double* x_free, double tol,
             int max_it, int* iters);
/* ComputeCompliance (fea.hpp:47, fea.cpp:851-864): ce per element, returns C */
int  t3d_compliance(struct t3d_context* ctx, const double* ele_E, const double* u_free, double* ce, double* C);
/* MG internals for inspection: per-level Jacobi diagonal / BC mask (interleaved 3n+c), coarsest matrix */
int  t3d_mg_get_diag(struct t3d_context* ctx, int level, double* diag);
int  t3d_mg_get_mask(struct t3d_context* ctx, int level, uint8_t* mask);
int  t3d_mg_coarse_matrix(struct t3d_context* ctx, const double* ele_E, double* Kc);
/* ApplyPDEFilter (filter.hpp:28, filter.cpp:175-275); warm-start state lives in the context */
int  t3d_filter_apply(struct t3d_context* ctx, const float* src, float* dst);
/* SetupPDEFilter (filter.hpp:17, filter.cpp:9-75) for radius rmin (cells): kernel r^2 KEF0 + KEF1,
 * inverse-row-sum preconditioner, zero warm start (t3d_create sets it up for params.filter_rmin) */
int  t3d_filter_setup(struct t3d_context* ctx, float rmin);
int  t3d_filter_get_state(struct t3d_context* ctx, double* last_x, double* last_rhs, double* diag_precond);
int  t3d_filter_set_state(struct t3d_context* ctx, const double* last_x, const double* last_rhs);
/* SIMP moduli (driver.cpp:117-121) and sensitivities (driver.cpp:151-157) */
int  t3d_simp(struct t3d_context* ctx, const float* x_phys, double* ele_E);
int  t3d_sensitivity(struct t3d_context* ctx, const float* x_phys, const double* ce, double c_solid, float* dc);
/* dc_filt / max(1e-3, x) (driver.cpp:166) and the OC bisection (driver.cpp:170-184) */
int  t3d_dc_scale(struct t3d_context* ctx, const float* dc_filt, const float* x, float* dc);
int  t3d_oc_update(struct t3d_context* ctx, const float* x, const float* dc, float V0, float* x_new, float* change,
                   float* lmid, int* bisections);

/* --------------------------------------------------------------- device-resident design loop */
/* x = V0, solid reference solve (driver.cpp:60-103); *c_solid = compliance of the solid domain */
int  t3d_design_init(struct t3d_context* ctx, float V0, double* c_solid);
/* one design iteration (driver.cpp:112-216) on device-resident state */
int  t3d_design_step(struct t3d_context* ctx, t3d_iter_record* rec);
/* the same iteration through host buffers: x_in -> device, step, device -> x_out (Morton order) */
int  t3d_design_step_host(struct t3d_context* ctx, const float* x_in, float* x_out, t3d_iter_record* rec);
int  t3d_get_density(struct t3d_context* ctx, float* x);
int  t3d_set_density(struct t3d_context* ctx, const float* x);
/* the design loop's displacement U restricted to the free DOFs (driver.cpp:128-136 uFreeWarm) */
int  t3d_get_displacement(struct t3d_context* ctx, double* u_free);
/* TOP3D_XL_GLOBAL (driver.hpp:4, driver.cpp:23-280) for one simulation: records[nLoop], x_final[num_elements] */
int  t3d_run_global(struct t3d_context* ctx, float V0, int n_loop, double* c_solid, t3d_iter_record* records,
                    int* n_records, float* x_final);
int  t3d_synchronize(struct t3d_context* ctx);

/* --------------------------------------------------------------- batched designs (no reference counterpart;
 * the reference runs one design per process, driver.cpp:23).  n designs of uneven grid size share one device
 * arena and step together: each design iteration runs the members' SIMP / MG rebuild, then ONE inner FP32
 * MG-PCG for all members in which every kernel of the PCG iteration (K(E)p with p.Ap, update, restrictions,
 * coarsest solve, prolongations, direction) is a single persistent launch walking an (instance, block) work
 * list, with per-instance convergence masks and the steady iterations captured in a CUDA graph, inside the
 * members' FP64 defect-correction loops; then the members' compliance, sensitivities, filter and OC.  Every
 * member's results equal the ones its own context gives with the same parameters.
 * Members: precision T3D_MIXED, the Adapted V-cycle, one load case (built-in cuboid problems); the FP32
 * K(E)p tile shape is set to the batched one (params.matvec32_tile is overridden to T3D_BATCH_TILE).
 *   dims: n x {nely, nelx, nelz};  params, problems: n each (problems may be NULL: the tip-line cantilever). */
enum { T3D_BATCH_TILE = 7 };
struct t3d_batch;
int  t3d_batch_create(int n, const int* dims, const t3d_params* params, const t3d_problem* problems,
                      struct t3d_batch** out);
/* member i's context (owned by the batch; use it for queries such as t3d_get_density, not t3d_destroy) */
int  t3d_batch_member(struct t3d_batch* b, int i, struct t3d_context** out);
/* Continuous batching (a request loop): an empty batch on `device`; t3d_batch_adopt moves a context created
 * and initialised alone (t3d_create_problem with the member rules above and matvec32_tile = T3D_BATCH_TILE,
 * then t3d_design_init) into the batch, appended as the last member, from the next t3d_batch_design_step on;
 * t3d_batch_release takes member i out again (later members move down by one) and hands its context back to
 * the caller, who destroys it.  Members created by t3d_batch_create live in the batch's arena and cannot be
 * released. */
int  t3d_batch_open(int device, struct t3d_batch** out);
int  t3d_batch_adopt(struct t3d_batch* b, struct t3d_context* ctx);
int  t3d_batch_release(struct t3d_batch* b, int i, struct t3d_context** out);
/* t3d_design_init of every member: V0[n] in, c_solid[n] out (may be NULL) */
int  t3d_batch_design_init(struct t3d_batch* b, const float* V0, double* c_solid);
/* one design iteration of every member: recs[n] */
int  t3d_batch_design_step(struct t3d_batch* b, t3d_iter_record* recs);
/* steps[i] design iterations of member i; recs receives member 0's records, then member 1's, ... (sum of
 * steps).  Members advance independently (each on its own host thread and stream); only their inner solves
 * share the batched launches, so a member with a short solve does not wait for one with a long solve. */
int  t3d_batch_run(struct t3d_batch* b, const int* steps, t3d_iter_record* recs);
/* Submitted work (a request loop), on a batch from t3d_batch_open: t3d_batch_submit hands over a context
 * created and initialised alone (t3d_design_init) to run `steps` design iterations in the batch, starting at
 * once; t3d_batch_collect waits up to timeout_ms for a finished one and returns its context (the caller's
 * again: destroy it), its records (up to cap) and its status in *status (*ctx NULL: none finished yet).
 * t3d_batch_destroy waits for submitted work still running.  While submitted work exists, t3d_batch_run,
 * t3d_batch_design_step, t3d_batch_adopt and t3d_batch_release are refused. */
int  t3d_batch_submit(struct t3d_batch* b, struct t3d_context* ctx, int steps);
int  t3d_batch_collect(struct t3d_batch* b, int timeout_ms, struct t3d_context** ctx, t3d_iter_record* recs, int cap,
                       int* nrec, int* status);
/* info[0] arena bytes, [1] members, [2] batched kernel launches so far, [3] kernels of one batched PCG
 * iteration, [4] logical blocks of one batched PCG iteration, [5] member kernels launched so far */
int  t3d_batch_info(struct t3d_batch* b, int64_t* info);
int  t3d_batch_destroy(struct t3d_batch* b);

/* --------------------------------------------------------------- profiling (no reference counterpart)
 * Times `reps` back-to-back launches of one device-resident kernel sequence with CUDA events on the
 * context's stream, after one untimed launch: T3D_PROFILE_MATVEC = K(E)p with the fused p.Ap,
 * T3D_PROFILE_VCYCLE = one V-cycle z = M r.  Operates on the current device state (E, p, r) and
 * overwrites Ap / z; *ms = mean milliseconds per launch. */
/* T3D_PROFILE_MATVEC32 / T3D_PROFILE_VCYCLE32: the FP32 forms of the mixed-precision inner solve
 * (contexts created with precision T3D_MIXED only). */
enum { T3D_PROFILE_MATVEC = 0, T3D_PROFILE_VCYCLE = 1, T3D_PROFILE_MATVEC32 = 2, T3D_PROFILE_VCYCLE32 = 3 };
int  t3d_profile(struct t3d_context* ctx, int what, int reps, double* ms);

/* --------------------------------------------------------------- allocation-free compliance
 * No counterpart in the reference.  For callers that cannot allocate device memory (a host that owns
 * the device heap, a serving loop that must not enter the allocator, a caller without a context):
 * ComputeCompliance on DEVICE pointers in the library's grid layout, with no cudaMalloc and no context.
 *   d_E, d_ce : (nx+2)*(ny+2)*(nz+2) doubles, padded grid with a zero ghost ring; cell (cx,cy,cz) at
 *               ((cz+1)*(ny+2)+cy+1)*(nx+2)+cx+1 is reference element (cx, ny-1-cy, cz); E = 0 off the
 *               cuboid; d_ce is written for the nx*ny*nz interior cells;
 *   d_u       : 3 planes of (nx+1)*(ny+1)*(nz+1) doubles, node (ix,iy,iz) of component c at
 *               c*NN + (iz*(ny+1)+iy)*(nx+1)+ix, zero on fixed DOFs;
 *   d_C       : one double, sum E*ce;  ke576: HOST pointer to Ke;  stream: a cudaStream_t (0 = default).
 * nx,ny,nz are the padded counts of t3d_create for (nely,nelx,nelz).  Scratch: a static device array of
 * 65536+1 doubles (512 KiB per GPU that loads the library, held until exit), one partial per 256
 * padded cells, so grids above 16,777,216 padded cells are rejected with T3D_ERR_UNSUPPORTED.  The
 * first call on a device looks up the array's address for that device (do it before any stream
 * capture); the address is the one in the device's primary context, so callers that make another
 * driver context current, or reset the device, are not supported.  Every call shares the array:
 * calls that overlap on the GPU race.  Asynchronous on `stream`. */
int  t3d_compliance_noalloc(int nely, int nelx, int nelz, const double* ke576, const double* d_E, const double* d_u,
                            double* d_ce, double* d_C, void* stream);

/* export_surface_stl (io.cpp:80-87): binary STL of the boundary faces of the voxels with density >= iso
 * (the reference exports at iso 0.3, driver.cpp:274), byte-identical to the reference's file.  xphys:
 * densities in the reference's element order, or NULL for the context's current design density.
 * *ntri receives the triangle count. */
int  t3d_export_stl(struct t3d_context* ctx, const float* xphys, float iso, const char* path, int64_t* ntri);

#ifdef __cplusplus
}
#endif
#endif
