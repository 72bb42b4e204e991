/*
 * cfd_b200.h — C ABI of the B200-native explicit finite-volume residual/update path.
 *
 * Plain C types only (pointers, sizes, doubles); no CUDA or torch types in any signature.
 * The library owns all device memory of a context; host pointers are borrowed for the call.
 * No function calls exit(): every failure is a status code (the reference exits on errors,
 * e.g. src/Basic_Functions.cpp:151-155, src/Numerical_Method.cpp:66-75).
 * One context per host thread; contexts are independent; a context is not re-entrant.
 *
 * Reference entry points (rameshkolluru43/CFD_Solver_withCUDA) each function replaces are
 * cited beside it.  Indices, face order and ghost numbering follow the reference's mesh
 * layout (include/Globals.h:313-328; ghosts numbered from No_Physical_Cells, cell-major,
 * face-minor, src/Read_Gmsh_File.cpp:360-402).
 */
#ifndef CFD_B200_H
#define CFD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CFD_OK = 0,
  CFD_ERR_BAD_ARG = 1,
  CFD_ERR_CUDA = 2,
  CFD_ERR_NONPHYSICAL = 3,    /* NaN sound speed (negative pressure/density); see cfd_step_info.bad_cell */
  CFD_ERR_DT_NONPOSITIVE = 4, /* global time step <= 0 (src/Numerical_Method.cpp:66-75) */
  CFD_ERR_TIMEOUT = 5,        /* a bounded device wait ran out */
  CFD_ERR_DIVERGED = 6,       /* residual growth beyond the configured limit */
  CFD_ERR_MESH = 7,
  CFD_ERR_IO = 8,
  CFD_ERR_NO_DEVICE = 9
} cfd_status;

/* Message for the last error on this thread. */
const char *cfd_last_error(void);
/* Library version string. */
const char *cfd_version(void);

/* ------------------------------------------------------------------------------------------
 * Mesh layer (host only; no device needed).  Replaces the reference's mesh ingest
 * Read_VTK_Grid (src/Read_Gmsh_File.cpp:11) + Construct_Ghost_Cells
 * (src/Grid_Computations.cpp:394) + Calculate_Cell_Center_Distances (:802), and adds seeded
 * generators for the benchmark geometries.
 * ------------------------------------------------------------------------------------------ */
typedef struct cfd_mesh cfd_mesh;

/* Boundary kinds of a (cell, face, ghost) entry: the reference's Inlet/Exit/Wall/Symmetry
 * cell lists (include/Globals.h:385). */
enum { CFD_BC_INLET = 0, CFD_BC_EXIT = 1, CFD_BC_WALL = 2, CFD_BC_SYMMETRY = 3 };

/* Borrowed view of a mesh in the reference's layout.  Arrays are indexed by reference cell id. */
typedef struct {
  int n_physical;                 /* No_Physical_Cells */
  int n_ghost;                    /* No_Ghost_Cells */
  const int *n_faces;             /* [NP] Cell::numFaces (3 or 4) */
  const int *neighbours;          /* [NP*4] Cell::Neighbours, -1 padded */
  const double *face_normals;     /* [NP*8] Cell::Face_Normals (nx, ny per face) */
  const double *face_lengths;     /* [NP*4] Cell::Face_Areas */
  const double *center_distances; /* [NP*4] Cell::Cell_Center_Distances */
  const double *center_vectors;   /* [NP*8] Cell::Cell_Center_Vector (x, y of N - c per face);
                                     needed by the gradient MUSCL form only, may be NULL */
  const double *area;             /* [NP] Cell::Area */
  const double *inv_area;         /* [NP] Cell::Inv_Area */
  int n_boundary;                 /* number of boundary entries (== n_ghost) */
  const int *boundary;            /* [n_boundary*4] kind, cell, face, ghost */
} cfd_mesh_desc;

cfd_status cfd_mesh_box(int nx, int ny, double x0, double x1, double y0, double y1, cfd_mesh **out);
cfd_status cfd_mesh_half_cylinder(int ntheta, int nr, double r_body, double r_outer, double ratio, cfd_mesh **out);
/* open_top = 0: boundary kinds by the reference reader's bounding-box rule (top = wall);
 * open_top = 1: top and right outflow, left inflow, lower boundary wall. */
cfd_status cfd_mesh_ramp(int nx, int ny, double length, double height, double x_corner, double angle_deg,
                         int open_top, cfd_mesh **out);
cfd_status cfd_mesh_bump(int nx, int ny, double length, double height, double thickness, int n_quad_layers,
                         double jitter, uint64_t seed, int triangles, cfd_mesh **out);
cfd_status cfd_mesh_read_vtk(const char *path, cfd_mesh **out);
cfd_status cfd_mesh_write_vtk(const cfd_mesh *m, const char *path);
cfd_status cfd_mesh_describe(const cfd_mesh *m, cfd_mesh_desc *out);
/* Cell centres of physical and ghost cells, [(NP+NG)*3] (Cell::Cell_Center). */
cfd_status cfd_mesh_centers(const cfd_mesh *m, double *out);
/* The structured-block numbering of reorder 4 (host only, no device needed): when the mesh is a
 * single block of ni x nj quads, *ni, *nj, *lh (1 when the face slots run clockwise in the block's
 * (i, j) axes) and, if cells is not NULL, cells[j * ni + i] = the mesh cell at (i, j) (n_physical
 * entries).  The i axis is the one whose length is a multiple of 32 if only one is, else the longer.
 * CFD_ERR_MESH (with the reason in cfd_last_error) for any other mesh. */
cfd_status cfd_mesh_block_order(const cfd_mesh_desc *d, int *ni, int *nj, int *lh, int *cells);
/* Points and cell node lists as given ([npts*3], [ncells*4] -1 padded). */
cfd_status cfd_mesh_points(const cfd_mesh *m, int *n_points, const double **points);
void cfd_mesh_destroy(cfd_mesh *m);

/* ------------------------------------------------------------------------------------------
 * Solver configuration: the reference's Solver_Config keys (json_Files/Solver_Config.json:1-38,
 * read at src/Configuration_Read.cpp:23-87) plus additive keys.
 * ------------------------------------------------------------------------------------------ */
/* Flux schemes.  The reference's Dissipation_Type switch (src/Net_Flux.cpp:74-91,109-126):
 * 1 LLF, 2 MOVERS / MOVERS_2O (src/MOVERS.cpp:45,169), 3 ROE / ROE_2O, 4 RICCA / RICCA_2O
 * (src/RICCA.cpp:61,129), 5 MOVERS_NWSC / MOVERS_NWSC_2O (src/MOVERS_NWSC.cpp:23,109); 2, 4 and 5
 * in the reference's per-cell form only (muscl = CFD_MUSCL_REFERENCE, FP64).  Additive: 6 AUSM,
 * 7 HLLC, and CFD_DISS_AUSM_GPU, the face flux of the reference's GPU kernel ausm_flux_kernel
 * (CUDA_KERNELS/Flux_Calculations_Cuda_Kernels.cu:37-113), gradient-MUSCL (face-based) form only. */
enum { CFD_DISS_LLF = 1, CFD_DISS_MOVERS = 2, CFD_DISS_ROE = 3, CFD_DISS_RICCA = 4, CFD_DISS_MOVERS_NWSC = 5,
       CFD_DISS_AUSM = 6, CFD_DISS_HLLC = 7, CFD_DISS_AUSM_GPU = 8 };
enum { CFD_LIM_REF_MINMOD = 0, CFD_LIM_MINMOD = 1, CFD_LIM_VANLEER = 2, CFD_LIM_SUPERBEE = 3, CFD_LIM_VANALBADA = 4 };
/* Integrators.  CFD_INT_RK3_GPU_REF / CFD_INT_RK4_GPU_REF: the stage updates of the reference's
 * GPU kernels tvd_rk3_kernel and rk4_complete_kernel (CUDA_KERNELS/Time_Integration_Cuda_Kernels.cu
 * :94-131 and :11-73; the RK4 one is not the classical scheme: its last stage uses only the last
 * residual), with dt taken at the first stage. */
enum { CFD_INT_REFERENCE = 0, CFD_INT_RK4 = 1, CFD_INT_SSPRK3 = 2, CFD_INT_RK3_GPU_REF = 3, CFD_INT_RK4_GPU_REF = 4 };
/* CFD_INLET_FARFIELD: Riemann-invariant far field of the reference's GPU kernel farfield_bc_kernel
 * (CUDA_KERNELS/Boundary_Conditions_Cuda_Kernels.cu:257-325), free stream (inlet_rho, inlet_u,
 * inlet_v, inlet_p).  CFD_EXIT_FIXED_P_REF: the reference's Subsonic_Exit_Boundary_Condition
 * (src/Exit_Boundary_Conditions.cpp:8-66, not called by its own driver) with P_f = exit_p (the
 * reference hard-codes 0.9/1.4). */
enum { CFD_INLET_SUPERSONIC = 0, CFD_INLET_SUBSONIC_REF = 1, CFD_INLET_TOTAL_PT = 2, CFD_INLET_FIXED = 3,
       CFD_INLET_FARFIELD = 4 };
enum { CFD_EXIT_SUPERSONIC = 0, CFD_EXIT_SUBSONIC_REF = 1, CFD_EXIT_STATIC_P = 2, CFD_EXIT_FIXED_P_REF = 3 };
enum { CFD_PREC_FP64 = 0, CFD_PREC_FP32_FLUX = 1 };
enum { CFD_MUSCL_REFERENCE = 0, CFD_MUSCL_GRADIENT = 1 };

typedef struct {
  int dissipation_type;      /* Dissipation_Type: CFD_DISS_* (1 LLF, 2 MOVERS, 3 ROE, 4 RICCA,
                                5 MOVERS_NWSC; additive 6 AUSM, 7 HLLC, 8 GPU AUSM) */
  int is_second_order;       /* Is_Second_Order */
  int time_accurate;         /* Time_Accurate: 1 -> Runge_Kutta_Method, 0 -> Explicit_Method */
  int local_time_stepping;   /* Local_Time_Stepping */
  int integrator;            /* CFD_INT_*: reference forms, classical RK4, standard SSP-RK3,
                                reference GPU RK3 / RK4 kernels */
  int limiter;               /* CFD_LIM_*: 0 = reference 2-argument MinMod (src/Limiters.cpp:58-63) */
  int reconstruct_primitive; /* MUSCL on (rho,u,v,p) instead of conserved variables */
  int muscl;                 /* CFD_MUSCL_REFERENCE: the reference's directional stencil
                                (src/Limiters.cpp:97-200) in ROE_2O; CFD_MUSCL_GRADIENT:
                                Green-Gauss-gradient MUSCL on (rho,u,v,p), Roe flux of the two
                                reconstructed face states */
  int inlet_bc;              /* CFD_INLET_* (reference: Is_Inlet_SubSonic) */
  int exit_bc;               /* CFD_EXIT_*  (reference: Is_Exit_SubSonic) */
  int precision;             /* CFD_PREC_* */
  int reorder;               /* device cell numbering: 0 as given, 1 reverse Cuthill-McKee,
                                2 patches of 128 cells grown breadth-first in RCM seed order,
                                3 patches of 128 cells by recursive coordinate bisection (needs
                                centre vectors; face-based per-cell-dt forms then run each
                                stage as one kernel per patch, option "patch_stage"),
                                4 a single structured block of ni x nj quads numbered j*ni+i
                                (CFD_ERR_MESH otherwise; see cfd_mesh_block_order); the
                                gradient-MUSCL forms with a per-cell dt and three stages then run
                                each stage as one kernel per 32 x 8 tile, option "tile_stage") */
  double cfl;                /* CFL */
  double limiter_zeta;       /* Limiter_Zeta */
  double limiter_zeta1;      /* Limiter_Zeta1 */
  double inlet_rho, inlet_p, inlet_u, inlet_v; /* inletCond (Rho, P, u, v) */
  double inlet_p0, inlet_t0;                   /* total pressure / temperature (CFD_INLET_TOTAL_PT) */
  double exit_p;                               /* static exit pressure (CFD_EXIT_STATIC_P) */
  double r_gas;                                /* gas constant for total-temperature inflow */
  int device;                /* CUDA device ordinal */
  void *stream;              /* cudaStream_t to launch on (NULL: the context creates its own) */
  int weno;                  /* Is_WENO: the reference's WENO path (Evaluate_Cell_Net_Flux_WENO,
                                src/WENO2D.cpp:395-456; quad cells; replaces the MUSCL forms) */
  int weno_characteristic;   /* Is_Char: WENO on characteristic variables (src/WENO2D.cpp:228-236) */
  double entropy_fix_linear; /* Harten's entropy fix on the linear (entropy and shear) waves of the
                                Roe flux in the gradient-MUSCL form: |Un| below delta = value *
                                a_Roe becomes (Un^2/delta + delta)/2.  0 (default): only the
                                acoustic waves are fixed, with delta = 0.1 * a_Roe, as in the
                                reference's ROE.  No reference counterpart; it suppresses the
                                carbuncle of grid-aligned strong shocks (0.2 - 0.4 typical). */
  double shock_fix;          /* Shock-stable hybrid of the gradient-MUSCL Roe flux: on a face where
                                either cell's pressure gradient marks a shock, |grad p| |d| >
                                value * p (d: centre-to-centre vector), the Roe dissipation is
                                replaced by the Rusanov dissipation 1/2 max(|Vn| + a) (U_R - U_L) dl.
                                0 (default): Roe everywhere.  No reference counterpart. */
  int movers_single_alpha;   /* Is_MOVERS_1: MOVERS uses the energy component's wave-speed
                                coefficient for all four components (src/MOVERS.cpp:142-152) */
  int movers_entropy_fix;    /* Enable_Entropy_Fix: MOVERS' entropy fix of the coefficients
                                (src/MOVERS.cpp:7-17,153-160) */
} cfd_config;

/* Defaults of json_Files/Solver_Config.json with Dissipation_Type = ROE. */
void cfd_config_default(cfd_config *cfg);
/* Parses a Solver_Config JSON file (the reference schema; // comments allowed) into cfg.
 * Is_MOVERS_1 and Enable_Entropy_Fix are read as the reference reads them
 * (src/Configuration_Read.cpp:72-73).
 * Unknown keys are ignored; additive keys: Limiter_Type, Flux_Scheme, Integrator, Precision,
 * Inlet_BC, Exit_BC, Reorder, MUSCL, Reconstruction, Entropy_Fix_Linear. */
cfd_status cfd_config_read_json(const char *path, cfd_config *cfg);

/* ------------------------------------------------------------------------------------------
 * Solver context
 * ------------------------------------------------------------------------------------------ */
typedef struct cfd_ctx cfd_ctx;

typedef struct {
  int iterations;      /* iterations (src/Solver.cpp:116) */
  double min_dt;       /* Min_dt after the last step */
  double total_time;   /* Total_Time */
  double error[4];     /* Error[0..3] of Estimate_Error (src/Error_Estimate_Update.cpp:10-28) */
  double res_l2[4];    /* plain ||R_k||_2 over physical cells of the last stage */
  int bad_cell;        /* first cell (reference id) with a NaN sound speed, or -1 */
  int status;          /* cfd_status of the step */
} cfd_step_info;

cfd_status cfd_create(const cfd_mesh_desc *mesh, const cfd_config *cfg, cfd_ctx **out);
void cfd_destroy(cfd_ctx *ctx);

/* Uploads conserved variables U [n*4] (rows in reference cell order; n = NP or NP+NG) and
 * recomputes primitives on the device, as Initialize_TestCase does (src/Initialize_TestCase.cpp:36-58).
 * With n = NP, ghost rows are initialised from their owner cell. */
cfd_status cfd_upload_state(cfd_ctx *ctx, const double *U, int n);

/* Whole pseudo-steps: n_steps repetitions of the loop body of Inviscid_Solver
 * (src/Solver.cpp:94-125): Apply_Boundary_Conditions -> Runge_Kutta_Method | Explicit_Method ->
 * Total_Time += Min_dt -> Estimate_Error -> Update.  Stops early when t_end > 0 and
 * Total_Time >= t_end.  info may be NULL. */
cfd_status cfd_step(cfd_ctx *ctx, int n_steps, double t_end, cfd_step_info *info);

/* Enqueue n pseudo-steps on the context's stream without waiting; cfd_sync waits and
 * collects the status (used to time the device path without host round trips). */
cfd_status cfd_step_async(cfd_ctx *ctx, int n_steps);
cfd_status cfd_sync(cfd_ctx *ctx, cfd_step_info *info);
/* Runtime options: "keep_delu" (write Cells_DelU in fused steps, default 1),
 * "use_graph" (replay pseudo-steps from a captured CUDA graph, default 1),
 * "profile" (time every launch with CUDA events; disables graph replay, default 0),
 * "fuse_gather" (face-based forms with per-cell dt: one kernel for the face-flux gather and
 * the stage update, default 1), "faces_shape" (face-flux kernel launch shape 0-4, default 3),
 * "flux_lanes" (threads per cell of the per-cell flux kernel, 1 or 4, default 1),
 * "flux_minb" (the one-lane second-order kernels with the directional limiter -- ROE_2O, RICCA_2O,
 * MOVERS_NWSC_2O -- register-capped for 1 (uncapped), 6 or 8 resident blocks per SM, default 1),
 * "pdl" (launch the kernels of a pseudo-step with programmatic dependent launch, default 0),
 * "patch_stage" (with reorder 3, the face-based forms with a per-cell dt frozen per step run each
 * stage as one kernel: a thread block per 128-cell patch computes the records, face fluxes, gather
 * and update of its cells in shared memory; default 0, tried by cfd_autotune),
 * "l2_persist" (face-based forms: the per-cell (rho, u, v, p) rows and the face-flux array are kept
 * in L2 as persisting lines between the kernels of a stage, when they fit in the device's largest
 * persisting set-aside; default 1.  Creating such a context
 * raises the device's persisting-L2 set-aside, cudaLimitPersistingL2CacheSize, to hold them, up to
 * the device maximum; it is never lowered and lasts as long as the process's CUDA context),
 * "persistent" (face-based forms with a per-cell dt: each RK stage as one persistent cooperative
 * kernel over the cells, faces and cells again, with bounded grid barriers between the phases and
 * one CUDA graph per RK stage; default 0; the batched solves' form, see cfd_batch_set_option),
 * "persist_minb" (the persistent kernel's register budget: built for 4, 6 or 8 resident blocks per
 * SM; default 0: 6 in FP64 and 8 in the FP32-flux form, the faster of each on B200),
 * "barrier_timeout_test" (a test of the bounded barriers: every barrier of the persistent form
 * waits for `value` more blocks than it has, so each wait runs out and the step reports
 * CFD_ERR_TIMEOUT; default 0),
 * "tile_stage" (with reorder 4 on a structured block, the gradient-MUSCL forms with a per-cell dt
 * frozen per step and three stages (CFD_INT_SSPRK3, CFD_INT_RK3_GPU_REF with local time stepping)
 * run each stage as one kernel: a thread block per tile of 32 x 8 cells stages the (rho, u, v, p)
 * rows of the tile and two rings around it in shared memory and forms the gradients, face fluxes,
 * gather and update of its cells there.  1: each phase loads what it reads; 2: the TMA form, in
 * which the tile's state rows and face records arrive by tensor bulk copies (cp.async.bulk.tensor)
 * and its cells' stage inputs by cp.async, all issued at block start; 3: the TMA form with the
 * stage inputs loaded where used (three blocks per SM); 4: form 2 with 288 threads per block.
 * Default 0 (on B200 the three kernels are faster), tried by cfd_autotune; where the form does not
 * apply (or, for 2-4, the device offers no tensor copies) setting it is CFD_ERR_BAD_ARG),
 * "tile_prefetch" (tile forms 2-4: each block also prefetches into L2 the inputs of the tile that
 * starts one wave later; default 0).
 * None of the options changes a state bit (the persistent form sums the error norms in another
 * order). */
cfd_status cfd_set_option(cfd_ctx *ctx, const char *name, double value);
/* Times every combination of the options above that applies to this configuration over `steps`
 * pseudo-steps of the context's own mesh and state, keeps the fastest and restores the state
 * (the solve is not advanced).  report (may be NULL) receives one line per candidate. */
cfd_status cfd_autotune(cfd_ctx *ctx, int steps, char *report, size_t report_len);

/* Entry points of the reference path, one call each, same semantics and post-conditions. */
cfd_status cfd_apply_boundary_conditions(cfd_ctx *ctx); /* Apply_Boundary_Conditions, src/Boundary_Conditions.cpp:12 */
cfd_status cfd_evaluate_net_flux(cfd_ctx *ctx);         /* Evaluate_Cell_Net_Flux_1O/2O, src/Net_Flux.cpp:46,97 */
cfd_status cfd_explicit_method(cfd_ctx *ctx);           /* Explicit_Method, src/Numerical_Method.cpp:26 */
cfd_status cfd_runge_kutta_method(cfd_ctx *ctx);        /* Runge_Kutta_Method, src/Numerical_Method.cpp:342 */
cfd_status cfd_estimate_error(cfd_ctx *ctx, double error[4]); /* Estimate_Error, src/Error_Estimate_Update.cpp:10 */
cfd_status cfd_update(cfd_ctx *ctx);                    /* Update(), src/Error_Estimate_Update.cpp:31 */
/* Set_DelU, src/Basic_Functions.cpp:9-18: dU [NP][4] (reference order) becomes the increment the
 * next cfd_update adds to U (the reference, SSP-RK3 and RK4 integrators). */
cfd_status cfd_set_delu(cfd_ctx *ctx, const double *dU);
cfd_status cfd_get_min_dt(cfd_ctx *ctx, double *min_dt); /* get_Min_dt, src/Numerical_Method.cpp:322 */
/* Lax_Fedrichs, src/Numerical_Method.cpp:459-481 (declared in the reference's Solver.h, called by
 * none of its drivers): U_c = 0.25 (sum of the four neighbours' U) - Min_dt / A_c * R_c, in place
 * with the reference's sweep semantics (neighbours earlier in reference cell order are read with
 * their new values), from the last net-flux evaluation; primitives are left as they are.  Quad
 * meshes only (CFD_ERR_MESH otherwise). */
cfd_status cfd_lax_friedrichs(cfd_ctx *ctx);

/* Downloads (reference cell order).  Any pointer may be NULL.
 *   U      [(NP+NG)*4] U_Cells
 *   prim   [(NP+NG)*11] Primitive_Cells (all 11 slots, src/Basic_Functions.cpp:162-219)
 *   dt     [NP] Cell::del_t of the last flux evaluation
 *   net    [NP*4] Cells_Net_Flux of the last flux evaluation
 *   delu   [NP*4] Cells_DelU */
cfd_status cfd_download(cfd_ctx *ctx, double *U, double *prim, double *dt, double *net, double *delu);
/* Conserved rows U_Cells [(NP+NG)*4] only (gathered into reference order on the device; a
 * pinned destination gives full PCIe/C2C bandwidth). */
cfd_status cfd_download_U(cfd_ctx *ctx, double *U);
/* Asynchronous forms of cfd_upload_state (all NP+NG rows) and cfd_download_U for pipelines of
 * independent solves: the copy and its gather kernels are enqueued on the context's stream and the
 * call returns at once; cfd_sync waits and reports the status (a non-physical uploaded state
 * included).  U must stay valid, and unchanged for an upload, until then, and must be page-locked
 * for the copy to overlap other work: with two contexts on two streams, one solve's copies run
 * while the other computes.  No reference counterpart (the reference keeps its state on the host). */
cfd_status cfd_upload_state_async(cfd_ctx *ctx, const double *U, int n);
cfd_status cfd_download_U_async(cfd_ctx *ctx, double *U);
/* Stage state [NP*4]: after Runge_Kutta_Method it holds U_Cells_RK_2 (the stage buffer is
 * shared by U_Cells_RK_1 and U_Cells_RK_2, src/Numerical_Method.cpp:372-416). */
cfd_status cfd_download_stage_state(cfd_ctx *ctx, double *S);

/* Green-Gauss gradient of primitive slot var (0 rho, 1 u, 2 v, 4 p) at cell centres, [NP*2]
 * (Calculate_Gradient_At_Cell_Center, src/Grid_Refine_Functions.cpp:221-246). */
cfd_status cfd_gradient(cfd_ctx *ctx, int var, double *grad);
/* AMR indicator [NP] and tags [NP] (Compute_Gradient_Refinement_Indicator / TagRefinableCells,
 * src/Grid_Refine_Functions.cpp:8-63).  Either output may be NULL. */
cfd_status cfd_amr_tags(cfd_ctx *ctx, double threshold, double max_fraction, double *indicator, uint8_t *tags);

/* ------------------------------------------------------------------------------------------
 * Solution files in the reference's formats.
 * cfd_write_solution: Write_Solution type 1 (src/output_files.cpp:492-556): the header integers
 *   (the reference writes nx_c ny_c nz_c for Grid_Type 0), No_Physical_Cells, iterations, then
 *   one row per cell: id, del_t, rho, p, T, u, v, M, p0 (default stream precision).
 * cfd_read_solution: the restart Initialize(const string &) (src/Initialize.cpp:125-176): physical
 *   cells' U from the rows' rho, p, u, v, and the iteration count; n_header integers are skipped.
 * cfd_vtk_copy_grid / cfd_vtk_append_solution: Read_Write_Grid and Append_Solution
 *   (src/Create_Vtk_File.cpp:5-157): the grid of a VTK file copied, then the cell data of a
 *   solution file appended (pressure, temperature, density, velocities, total pressure, entropy,
 *   Mach number, velocity vectors).  Host only.
 * ------------------------------------------------------------------------------------------ */
cfd_status cfd_write_solution(cfd_ctx *ctx, const char *path, const int *header, int n_header);
cfd_status cfd_read_solution(cfd_ctx *ctx, const char *path, int n_header);
cfd_status cfd_vtk_copy_grid(const char *grid_vtk, const char *out_vtk);
cfd_status cfd_vtk_append_solution(const char *solution_txt, const char *out_vtk, int n_header);

/* Pointwise evaluation of the face functions on host arrays (runs on `device`): the limiter
 * phi(a, b) of CFD_LIM_MINMOD..CFD_LIM_VANALBADA for n pairs (the phi(r) family of
 * CUDA_KERNELS/Limiter_Cuda_Kernels.cu:89-154: r = a/b, phi = 0 when |b| < 1e-12 or r <= 0), and
 * the face flux of scheme CFD_DISS_ROE / _AUSM / _HLLC / _AUSM_GPU for n conserved left/right
 * states [n*4], outward unit normals [n*2] and face lengths [n], into F [n*4], in precision
 * CFD_PREC_FP64 or CFD_PREC_FP32_FLUX.  The same device functions as the solver's face kernel. */
cfd_status cfd_eval_limiter(int limiter, const double *a, const double *b, int n, double *out, int device);
cfd_status cfd_eval_face_flux(int scheme, int precision, const double *UL, const double *UR, const double *normals,
                              const double *lengths, int n, double *F, int device);

/* Device arrays of one net-flux evaluation, in the device layout this library uses internally
 * (no renumbering): face-major [4][NP] per-face arrays, component-major state planes. */
typedef struct {
  int n_physical;                 /* NP */
  int n_total;                    /* NP + NG */
  const int *n_faces;             /* [NP] */
  const int *neighbours;          /* [4][NP] neighbour or ghost id of face f of cell c at f*NP+c */
  const double *nx, *ny, *dl;     /* [4][NP] face normal and length */
  const double *area, *inv_area;  /* [NP] */
  const int *second_neighbours;   /* [4][NP] second cell of the directional limiter stencil (2nd order) */
  const double *d1, *d2;          /* [4][NP] centre distances of that stencil (2nd order) */
  const uint8_t *degenerate;      /* [NP] bit f set when |n_f| < 1e-12 */
  const double *prim;             /* [5][NT] rho, u, v, p, a */
  const double *U;                /* [4][NT] conserved state, ghost rows included */
  double *net_flux;               /* out [4][NP] per-cell residual (sum of face fluxes) */
  double *dt;                     /* out [NP] per-cell time step */
  double *min_dt;                 /* out [1] minimum time step over the cells */
} cfd_flux_arrays;

/* The per-cell residual, per-cell time step and minimum time step (what cfd_evaluate_net_flux
 * computes) on caller-owned device arrays, WITHOUT allocating device memory.  It has no
 * counterpart in the reference.  It exists for callers that cannot let this library call
 * cudaMalloc: their own pool allocator owns the GPU's memory, or their loop cannot take
 * cudaMalloc's device synchronisation or its possible failure.
 * The kernel's scratch (control block, completion counter, one partial minimum per thread block)
 * is a fixed static device array of 262,168 doubles (2 MiB) per GPU, held until the process
 * exits; at most 8,388,608 physical cells per call (larger sizes are rejected with
 * CFD_ERR_BAD_ARG).  The array is placed on the device when the library's device code is loaded
 * into the CUDA context; with lazy module loading (the CUDA default) that is the first call in a
 * context, which then needs 2 MiB of free device memory and synchronises the device.  So make the
 * first call on each device before your pool reserves the GPU's memory (or run with
 * CUDA_MODULE_LOADING=EAGER), and before any stream capture.  The array's device address is
 * looked up in the current context on every call.  Calls share the array and every call clears
 * what must start at zero: calls that overlap on the GPU (different streams, other threads) race.
 * Reference MUSCL stencil, FP64; ROE, MOVERS, RICCA, MOVERS_NWSC (first and second order) or
 * first-order LLF.
 * stream: cudaStream_t (NULL = default stream). */
cfd_status cfd_evaluate_net_flux_noalloc(const cfd_flux_arrays *a, const cfd_config *cfg, void *stream);

/* ------------------------------------------------------------------------------------------
 * Batched solves: many independent meshes (uneven sizes) run together as one union mesh through
 * the same kernels; work lists restrict every launch to instances that have not converged; the
 * whole pseudo-step is replayed from a CUDA graph that is re-captured when the active set
 * changes.  No reference counterpart (the reference solves one mesh per process).
 * Gradient-MUSCL form only, no renumbering (cfg->muscl = 1, cfg->reorder = 0).
 * inflow: [n*4] (rho, u, v, p) per instance for CFD_INLET_FIXED inlet entries (may be NULL).
 * ------------------------------------------------------------------------------------------ */
typedef struct cfd_batch cfd_batch;
cfd_status cfd_batch_create(int n, const cfd_mesh_desc *meshes, const double *inflow, const cfd_config *cfg,
                            cfd_batch **out);
/* U: for each instance in order, its NP_i + NG_i rows in reference order.  Uploading restarts
 * every instance (all active again). */
cfd_status cfd_batch_upload_state(cfd_batch *b, const double *U);
/* Per-instance boundary values (either pointer may be NULL): inlet [n*4] read by the configured
 * inlet kind (CFD_INLET_FIXED / CFD_INLET_FARFIELD: rho, u, v, p; CFD_INLET_TOTAL_PT: p0, T0, -, -),
 * exit_p [n] the exit pressure of CFD_EXIT_STATIC_P / CFD_EXIT_FIXED_P_REF. */
cfd_status cfd_batch_set_boundary_values(cfd_batch *b, const double *inlet, const double *exit_p);
/* Per-instance residual normalisers r0 [n] for cfd_batch_run's tolerance test (NULL: each
 * instance's first-step residual), so that runs from different starts share one absolute target. */
cfd_status cfd_batch_set_reference_residual(cfd_batch *b, const double *r0);
/* ||R_rho||_2 of each instance's last residual evaluation, [n]. */
cfd_status cfd_batch_residuals(cfd_batch *b, double *res);
cfd_status cfd_batch_download_state(cfd_batch *b, double *U);
/* Runs until every instance's plain residual ||R_rho||_2 has dropped by the factor tol from its
 * first-step value (or from the normaliser set by cfd_batch_set_reference_residual), or
 * max_steps; the residuals are checked every check_every steps (each check
 * synchronises).  Per instance: steps_to_tol (-1 if not reached), time_to_tol (seconds since the
 * call, -1 if not reached), res_ratio (last ||R_rho|| / first).  cell_updates counts the cells
 * actually advanced.  Any output pointer may be NULL. */
cfd_status cfd_batch_run(cfd_batch *b, int max_steps, double tol, int check_every, int *steps_to_tol,
                         double *time_to_tol, double *res_ratio, long long *cell_updates, int *steps_done);
/* Run-time options of the batch's solver context (cfd_set_option), e.g. "persistent" = 1: each RK
 * stage of every instance runs as one persistent cooperative kernel over the (instance, block)
 * work lists, bounded grid barriers between its phases, one CUDA graph per RK stage (results
 * bit-identical to the three-kernel form; CFD_ERR_TIMEOUT when a barrier wait runs out).
 * "divergence_ratio" = x > 0: in cfd_batch_run an instance whose residual ratio exceeds x at a
 * check stops updating and gets steps_to_tol = -2 (residual growth; 0 = never). */
cfd_status cfd_batch_set_option(cfd_batch *b, const char *name, double value);
void cfd_batch_destroy(cfd_batch *b);

/* ------------------------------------------------------------------------------------------
 * Kernels of the warm-start surrogate (message passing on the cell graph of a mesh; no reference
 * counterpart).  Device pointers, float32, launched on `stream` (cudaStream_t, NULL = default).
 * Segment sum: out[r, :] = sum over j in [ptr[r], ptr[r+1]) of x[idx[j], :] in list order
 * (deterministic; width columns).  Adam: one bias-corrected step (`step` counts from 1).
 * ------------------------------------------------------------------------------------------ */
cfd_status cfd_mpnn_segment_sum(const float *x, const int *ptr, const int *idx, int n_rows, int width, float *out,
                                void *stream);
cfd_status cfd_mpnn_adam(float *param, const float *grad, float *m, float *v, int n, float lr, float beta1,
                         float beta2, float eps, int step, void *stream);

/* Dense blocks on the tensor cores: y = W2 silu(W1 x + b1) + b2 (+ r), hidden width 64, BF16
 * operands (rounded when staged), FP32 accumulation and epilogues.  The input row x is up to three
 * segments side by side (total width <= 192); segment s supplies columns of row
 * (idx ? idx[row] : row) of src (leading dimension ld), through silu() when silu = 1. */
typedef struct {
  const float *src;
  const int *idx; /* row map of the segment, or NULL */
  int width, ld;
  int silu;       /* 1: values pass through silu(z) = z / (1 + exp(-z)) when loaded */
} cfd_mlp_seg;

typedef struct {
  int rows;
  int nseg;
  cfd_mlp_seg seg[3];
  int out;                 /* output width, 1..64 */
  const float *w1, *b1;    /* [64][in_width], [64] */
  const float *w2, *b2;    /* [out][64], [out] */
  const float *resid;      /* optional residual added to y, [rows][ld_resid] */
  int ld_resid;
  float *z1;               /* out (optional): hidden pre-activation [rows][64] */
  float *y;                /* out [rows][ld_y] */
  int ld_y;
  int engine;              /* 0: mma.sync m16n8k16 (64-row tiles); 1: tcgen05.mma with the accumulators in
                              tensor memory (128-row tiles, operands in shared memory by matrix
                              descriptors); the two agree up to the FP32 summation order */
} cfd_mlp_fwd;
cfd_status cfd_mpnn_mlp_forward(const cfd_mlp_fwd *a, void *stream);
/* Status word of the tcgen05 kernels (0, or CFD_ERR_TIMEOUT when a bounded wait ran out); reset = 1
 * clears it.  Synchronises with the device. */
cfd_status cfd_mpnn_status(int *status, int reset);

/* Backward data path of one dense block: dz1 = (dy W2) * silu'(z1) and dx = dz1 W1. */
typedef struct {
  int rows, in_width, out;
  const float *dy;         /* [rows][ld_dy] */
  int ld_dy;
  const float *z1;         /* [rows][64] from the forward pass */
  const float *w1, *w2;
  float *dz1;              /* out [rows][64] */
  float *dx;               /* out (optional) [rows][ld_dx] */
  int ld_dx;
  int engine;              /* 0: mma.sync; 1: tcgen05.mma with tensor-memory accumulators */
} cfd_mlp_bwd;
cfd_status cfd_mpnn_mlp_backward(const cfd_mlp_bwd *a, void *stream);

/* Weight gradient of one linear layer: dw = dz^T x ([n][in_width]) and db = column sums of dz, with
 * x given as segments as above (n = 64, or n <= 16).  Each of at most CFD_MPNN_WGRAD_BLOCKS thread
 * blocks accumulates its rows into one partial in `workspace` (CFD_MPNN_WGRAD_BLOCKS * (n *
 * in_width + n) floats); the partials are summed in block order, so results repeat bit for bit.
 * accumulate = 1 adds to dw and db instead of overwriting them. */
#define CFD_MPNN_WGRAD_BLOCKS 296
typedef struct {
  int rows, n;
  const float *dz;
  int ld_dz;
  int nseg;
  cfd_mlp_seg seg[3];
  float *workspace;
  float *dw, *db;
  int accumulate;
} cfd_mlp_wgrad;
cfd_status cfd_mpnn_weight_grad(const cfd_mlp_wgrad *a, void *stream);
int cfd_mpnn_wgrad_blocks(void);

/* Helpers of the training step (float32, device pointers, leading dimensions in elements):
 * out = a + b on a [rows][width] window; out[r] += src[idx[r]]; out[r] (+)= sum over the CSR list
 * of row r of x[idx[j]] in list order; the mean-squared error of n values with its gradient
 * 2 (pred - target) / n (loss to a device scalar, fixed-order sum). */
cfd_status cfd_mpnn_add(float *out, int ldo, const float *a, int lda, const float *b, int ldb, int rows, int width,
                        void *stream);
cfd_status cfd_mpnn_gather_add(float *out, int ldo, const float *src, int lds, const int *idx, int rows, int width,
                               void *stream);
cfd_status cfd_mpnn_segment_sum_acc(const float *x, int ldx, const int *ptr, const int *idx, int n_rows, int width,
                                    float *out, int ldo, int accumulate, void *stream);
cfd_status cfd_mpnn_mse(const float *pred, const float *target, int n, float *grad, float *loss, void *stream);

/* Accumulated device time of one kernel family ("flux", "stage", "bc", and for the face-based
 * forms "gradients", "faces", "gather_stage", "patch") over the launches made while option "profile" was
 * set (CUDA events on the context's stream around each launch). */
cfd_status cfd_kernel_time(cfd_ctx *ctx, const char *kernel, double *total_ms, long long *launches);
/* Number of unique faces of the face-based forms (0 for the per-cell reference forms). */
int cfd_face_count(const cfd_ctx *ctx);
/* Number of CUDA kernel launches this context has issued so far. */
long long cfd_kernel_launches(const cfd_ctx *ctx);
/* Device bytes held by the context. */
size_t cfd_device_bytes(const cfd_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* CFD_B200_H */
