/*
 * adh_sw2_gpu.h -- C ABI of the B200 (sm_100a) implementation of AdH-Kraken's
 * implicit SW2 time step.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and reports
 * failures through its int return value (SW2G_OK = 0) and sw2g_last_error().
 * Host-buffer entry points copy their inputs to the device and their outputs
 * back, so they drop in where the reference's C routines are called today; the
 * *_state / sw2g_step entry points keep the solution resident in HBM.
 *
 * Conventions are the reference's: node-major dofs (dof = 3*node + {0:h, 1:u, 2:v},
 * src/structs/sivar_position/sivar_position.c:61-81), the serial CSR of
 * slin_sys_init_sparsity_mono (sorted unique columns per row), element order =
 * triangles then boundary segments, and bc_mask entries equal to 1 for Dirichlet
 * dofs (the reference's YES).
 *
 * Not reentrant on one model: calls on a model must come from one host thread,
 * as in the reference (module-level static work buffers, e.g.
 * src/la/bcgstab_solver.c:5-22).  Different models are independent.
 */
#ifndef ADH_SW2_GPU_H
#define ADH_SW2_GPU_H
#ifdef __cplusplus
extern "C" {
#endif

#define SW2G_OK 0
#define SW2G_ERR_ARG (-1)       /* bad argument or size */
#define SW2G_ERR_CUDA (-2)      /* CUDA runtime error (message in sw2g_last_error) */
#define SW2G_ERR_NOMEM (-3)     /* device or host allocation failed */
#define SW2G_ERR_MESH (-4)      /* mesh / CSR structure not usable */
#define SW2G_ERR_NONFINITE (-5) /* NaN or Inf in a residual norm (the reference exits, newton_tools.c:344-349) */

typedef struct sw2g_model sw2g_model;

typedef struct {
    int nnodes, ntri, nseg;
    const double *xyz;      /* [3*nnodes] x, y, bed elevation z */
    const int *tri;         /* [3*ntri] counter-clockwise node ids */
    const int *seg;         /* [2*nseg] boundary segments; node order gives the outward normal */
    const int *seg_kind;    /* [nseg] 0 = "NB VEL" (fe_sw2_bc_vel), 1 = "DEPTH" (fe_sw2_bc_h),
                               2 = discharge (fe_sw2_bc_discharge, src/models/sw2/sw2_bc_discharge.c.bk:57),
                               3 = tailwater (fe_sw2_bc_tailwater, src/models/sw2/sw2_bc_tailwater.c.bk:57),
                               4 = outflow (fe_sw2_bc_outflow, src/models/sw2/sw2_bc_outflow.c.bk:58),
                               5 = flux (fe_sw2_bc_flux, src/models/sw2/sw2_bc_flux.c.bk:58) */
    const int *indptr;      /* optional [3*nnodes+1]: the caller's CSR, checked against ours; NULL to build */
    const int *cols;        /* optional [nnz] */
    double gravity;         /* sm->gravity, 9.8 by default */
} sw2g_mesh;

typedef struct {
    double tol_nonlin;        /* sm->tol_nonlin, absolute max-norm, default 1e-8 */
    double inc_nonlin;        /* sm->inc_nonlin, default 1e-6 */
    int max_nonlin_it;        /* sm->max_nonlin_it, default 10 */
    int max_linesearch_cuts;  /* sm->max_nonlin_linesearch_cuts, default 5 */
    int krylov_max_it;        /* Krylov iteration cap per Newton correction */
    double krylov_tol;        /* BiCGStab: stopping tolerance (bcgstab_solver.c:20-21: 1e-11); GMRES: forcing
                                 term, max|r| <= max(krylov_tol * max|R|, tol_nonlin / 10 (relative Newton test)
                                 or / 100 (absolute)) on the unscaled linear residual */
    int krylov_precision;     /* 64: FP64 BiCGStab; 32: FP32 BiCGStab inside FP64 iterative refinement */
    double refine_tol;        /* FP32 inner solve relative reduction per refinement pass (32-bit mode) */
    int max_refine;           /* refinement passes per Newton correction (32-bit mode) */
    int use_guess;            /* 1: start Newton from the buffer given to sw2g_set_guess when its residual
                                 L2 norm is below that of sol_old (else sol_old, the reference's start) */
    int precond;              /* SW2G_PC_AMG (default), SW2G_PC_BILU0 or SW2G_PC_BLOCK_JACOBI */
    int krylov_method;        /* SW2G_KRYLOV_GMRES (default; needs SW2G_PC_AMG or SW2G_PC_BILU0) or SW2G_KRYLOV_BICGSTAB */
    double tol_nonlin_rel;    /* > 0: Newton residual test relative to the residual max-norm at the previous
                                 step's state (the reference's starting point, the same whatever the initial
                                 guess): max|R| <= tol_nonlin_rel * max|R(sol_old)| (replaces tol_nonlin);
                                 0 (default): the reference's absolute test */
    int krylov_basis_precision; /* GMRES with krylov_precision 32: 64 (default) keeps the Krylov basis, the SpMV
                                 and the Gram-Schmidt in FP64 around the FP32 preconditioner; 32 runs the whole
                                 cycle in FP32, each cycle refined from the FP64 residual */
    int krylov_restart;       /* GMRES restart length, 1..200 (default 30); the basis holds restart+1 vectors */
    int amg_chunks;           /* AMG chunk corrections (exact solves on chunks of the nodes whose block-Jacobi
                                 smoothing the l1 fix-up weakens): 0 off (default), 1 after each V-cycle,
                                 2 inside it.  They remove the stall of the linear solve at shallow wet/dry
                                 nodes on some steps and slow or break it on others (nearly singular chunk
                                 blocks), so they are off unless asked for. */
    double tol_nonlin_min;    /* with tol_nonlin_rel > 0: the tolerance is max(tol_nonlin_rel * max|R(sol_old)|,
                                 tol_nonlin_min) (default 0).  A time loop that covers an interval in smaller
                                 steps after a failed solve passes the interval's own tolerance here: the
                                 residual at the start of a short step shrinks with its dt, the attainable
                                 accuracy does not. */
} sw2g_newton_opts;

/* Krylov methods of the Newton correction.  BiCGStab is the reference's
 * (bcgstab_solver.c:65-330).  GMRES(m) (m = krylov_restart), right-preconditioned and restarted from
 * the true FP64 residual, is robust where an approximate preconditioner leaves a
 * far-from-normal operator (BiCGStab's residual then swings or diverges). */
#define SW2G_KRYLOV_BICGSTAB 0
#define SW2G_KRYLOV_GMRES 1

/* preconditioners standing in for the reference's full UMFPACK LU (bcgstab_solver.c:371-420) */
#define SW2G_PC_BLOCK_JACOBI 0   /* 3x3 nodal block-Jacobi */
#define SW2G_PC_BILU0 1          /* multicolour 3x3 block ILU(0) over the node graph */
#define SW2G_PC_AMG 2            /* aggregation AMG V-cycle over the node blocks (l1 block-Jacobi smoothing) */

typedef struct {
    int newton_its;           /* Newton iterations of the step */
    int krylov_its;           /* Krylov (BiCGStab or GMRES) iterations summed over the step */
    int linesearch_cuts;      /* line-search halvings summed over the step */
    int refine_passes;        /* FP64 refinement passes (32-bit mode) */
    int success;              /* fe_newton's TRUE/FALSE: max|R| <= tolerance, or the increment max-norm <=
                                 inc_nonlin after a linear solve that reached its target */
    int krylov_breakdowns;    /* Krylov solves that stopped on a zero/non-finite denominator */
    double resid_max;         /* final max |R| over non-Dirichlet dofs */
    double resid_l2;          /* final sqrt(sum R^2)/ndofs */
    double inc_max;           /* last max |increment| */
    double initial_resid_max; /* max |R| at the initial guess */
    double prev_resid_max;    /* max |R| at the previous-step state (the reference's initial guess) */
    int guess_used;           /* 1: the sw2g_set_guess guess had the smaller residual L2 norm and started Newton */
    double initial_resid_l2;  /* sqrt(sum R^2)/ndofs at the initial guess */
    int guess_fallback;       /* 1: Newton from the guess failed and was repeated from the previous step
                                 (the counts above include both attempts) */
    int linear_unconverged;   /* Newton iterations whose linear solve stopped before its target (iteration
                                 cap, stall, breakdown); their increment test does not count as convergence */
    double tol_used;          /* the Newton residual tolerance applied (tol_nonlin, or tol_nonlin_rel times
                                 max|R(sol_old)|) */
} sw2g_newton_stats;

/* --- lifetime ------------------------------------------------------------ */
/* Builds the device model: element geometry (selem2d/selem1d), the bit-exact CSR
 * (src/structs/slin_sys/slin_sys_init_sparsity_mono.c:28), the element-to-CSR
 * assembly maps and all work buffers.  `cuda_stream` may be NULL (own stream).
 * Replaces the linear-system part of smodel_design_init_no_read
 * (src/structs/smodel_design/smodel_design_init_no_read.c:110-135). */
int sw2g_create(const sw2g_mesh *mesh, void *cuda_stream, sw2g_model **out);
void sw2g_destroy(sw2g_model *m);
const char *sw2g_last_error(void);
void sw2g_default_opts(sw2g_newton_opts *opts);
int sw2g_sizes(const sw2g_model *m, int *ndofs, int *nnz);
/* The CSR structure the device uses: identical to the reference's serial CSR. */
int sw2g_get_sparsity(const sw2g_model *m, int *indptr, int *cols);
/* Per-step scalars: dt = ts->dt / nsubsteps, tau_temporal, and the step-averaged
 * values of series 0 (depth) and 1/2 (velocity x/y) (sseries_setall_ts_valuesAVG,
 * src/structs/sseries/sseries.c:673). */
int sw2g_set_step(sw2g_model *m, double dt, double tau_temporal, double bc_depth, double bc_vx, double bc_vy);
/* The values of the discharge and tailwater segments (kinds 2 and 3) for the coming
 * steps: the discharge string's series value (sseries_get_value of its ol_flow series,
 * sw2_bc_discharge.c.bk:161), its conveyance (STR_VALUE.conveyance, sstr_value.h:63),
 * the boundary strings' equivalent roughness height (FRICTION.eqrheight; the drag is
 * fr_bedshstr_drag_coef's, zero for a height <= DBL_EPSILON as in fe_sw2_get_roughness,
 * src/models/sw2/sw2_get_roughness.c:24) and the tailwater elevation (the series value of
 * sw2_bc_tailwater.c.bk:154).  As in the reference, a discharge segment with zero drag
 * divides by zero (the residual turns non-finite).  Defaults: 0, 1, 0, 0.  Non-finite
 * values or a zero conveyance give SW2G_ERR_ARG. */
int sw2g_set_bc_structures(sw2g_model *m, double q_series, double conveyance, double rough_height, double tail_elev);
/* The series value of the flux strings (kind 5) for the coming steps: the unit flux
 * whose negative the strings carry into the domain (sw2_bc_flux.c.bk:151-153).
 * Default 0; a non-finite value gives SW2G_ERR_ARG. */
int sw2g_set_bc_flux(sw2g_model *m, double flux_series);

/* --- drop-in host-buffer entry points ------------------------------------ */
/* fe_sw2_wdflag_legacy (src/models/sw2/sw2_wdflag_legacy.c:34): [ntri] flags 0/1/2 */
int sw2g_wd_flags(sw2g_model *m, const double *sol, const double *sol_old, int *wd_flag);
/* Element residuals as the reference's resid plugins return them
 * (fe_sw2_body_resid sw2_body_resid.c:44, fe_sw2_bc_vel sw2_bc_vel.c:58,
 * fe_sw2_bc_h sw2_bc_h.c:57): [ntri*9] and [nseg*6].  Uses the wet/dry flags of
 * (sol, sol_old). */
int sw2g_elem_resid(sw2g_model *m, const double *sol, const double *sol_old, const double *sol_older,
                    double *out_tri, double *out_seg);
/* Central-difference element Jacobians (perturb_var, src/jacobian/assemble_jacobian.c:304):
 * [ntri*81] and [nseg*36], row-major element matrices. */
int sw2g_elem_jac(sw2g_model *m, const double *sol, const double *sol_old, const double *sol_older,
                  double *out_tri, double *out_seg);
/* assemble_residual(SMODEL_SUPER*, SGRID*) (src/residual/residual.h:5): [ndofs] */
int sw2g_assemble_residual(sw2g_model *m, const double *sol, const double *sol_old, const double *sol_older,
                           double *residual);
/* assemble_jacobian(SMODEL_SUPER*) (src/jacobian/jacobian.h:5): CSR values [nnz] */
int sw2g_assemble_jacobian(sw2g_model *m, const double *sol, const double *sol_old, const double *sol_older,
                           double *vals);
/* The same assemblies with the caller's wet/dry flags [ntri] (0, 1 or 2): what
 * assemble_residual / assemble_jacobian compute inside fe_newton, whose element
 * routines read sm->dvars.elem_flags[_WDFLAG] as fe_sw2_init set it at the start of
 * the Newton solve (src/newton/newton_tools.c:21-53, src/models/sw2/sw2_body_resid.c:88). */
int sw2g_assemble_residual_wd(sw2g_model *m, const double *sol, const double *sol_old, const double *sol_older,
                              const int *wd_flag, double *residual);
int sw2g_assemble_jacobian_wd(sw2g_model *m, const double *sol, const double *sol_old, const double *sol_older,
                              const int *wd_flag, double *vals);
/* check_diag + apply_Dirichlet_BC (src/la/la.h:12-13) + scale_linear_system (la.h:46):
 * vals [nnz], residual [ndofs], x [ndofs] and bc_mask [ndofs] in/out; scale [ndofs] out. */
int sw2g_prepare_system(sw2g_model *m, double *vals, double *residual, double *x, int *bc_mask, double *scale);
/* solve_linear_sys_bcgstab (src/la/la.h:22-29), serial branch: x in/out (the x0 shift
 * and the unscaling are the reference's), b is overwritten with M^-1 b as in the
 * reference.  The exact UMFPACK LU preconditioner is replaced by `precond`
 * (SW2G_PC_*).  Returns the iteration count in *iters (negative on breakdown). */
int sw2g_solve_linear_sys_bcgstab(sw2g_model *m, double *x, const double *vals, double *b, const double *scale_vect,
                                  int max_it, double tol, int precond, int *iters);
/* fe_newton(SMODEL_SUPER*) (src/newton/newton.h:19) for one time step: sol out;
 * sol_old/sol_older in; bc_mask in/out (permanent Dirichlet marks); dirichlet in. */
int sw2g_fe_newton(sw2g_model *m, double *sol, const double *sol_old, const double *sol_older, int *bc_mask,
                   const double *dirichlet, const sw2g_newton_opts *opts, sw2g_newton_stats *stats);

/* Mass balance of a state.  out[0] = tl_find_grid_mass_elem2d(density, .., depth, grid, ..)
 * (src/tools/tl_grid_mass.c:198): density times the sum over triangles of the depth
 * integral, with the reference's dry-vertex rule (depth < 0 is dry).  out[1] = one
 * step's boundary mass inflow, the boundary loop of tl_find_grid_mass_error_elem2d
 * (tl_grid_mass.c:310-320): -density dt sum over boundary segments of the integral of
 * h (v . n), each segment with its own length (the reference takes the first
 * segment's length for all of them).  The reference's mass error after k steps is
 * |out[0] - (sum of the k inflows) - initial mass|.  sol: host [ndofs], or NULL for
 * the resident state (after sw2g_step / sw2g_load_state); elem_mass: optional host
 * [ntri], each triangle's term before the density factor.  The sums run in a fixed
 * order (run-to-run identical); they differ from the reference's serial sum only by
 * rounding. */
int sw2g_grid_mass(sw2g_model *m, const double *sol, double density, double dt, double *out, double *elem_mass);

/* The residual of sw2g_assemble_residual, on device buffers, for callers that cannot
 * allocate device memory when they call in (an application that gave all free device
 * memory to its own pool at start-up, a time loop that must not allocate inside its
 * steps).  No counterpart in the reference.  The call allocates nothing: its work
 * arrays are fixed-size device arrays inside the library (about 10.5 MB, held by every
 * GPU that loads it until the process exits), so the mesh may have at most 131072
 * elements (triangles + segments) and 131072 nodes; larger meshes get SW2G_ERR_ARG.
 * d_sol, d_sol_old, d_sol_older [ndofs] and d_residual [ndofs] are device pointers on
 * the model's device; the step parameters come from sw2g_set_step.  The model's device
 * (the one current at sw2g_create) must be the current device when this is called
 * (SW2G_ERR_ARG otherwise).  The first call on a device looks the arrays' device
 * addresses up (once per device); make it before any stream capture.  Every call shares the arrays, so calls that overlap on the GPU
 * (other models, streams or host threads) race; the call returns after its kernels
 * have finished on the model's stream. */
int sw2g_assemble_residual_noalloc(sw2g_model *m, const double *d_sol, const double *d_sol_old,
                                   const double *d_sol_older, double *d_residual);

/* --- device-resident time stepping --------------------------------------- */
int sw2g_load_state(sw2g_model *m, const double *sol, const double *sol_old, const double *sol_older,
                    const int *bc_mask, const double *dirichlet);
int sw2g_store_state(sw2g_model *m, double *sol, double *sol_old, double *sol_older, int *bc_mask);
/* Optional Newton initial guess for the next sw2g_step (host [ndofs] or device pointer). */
int sw2g_set_guess(sw2g_model *m, const double *guess, int guess_on_device);
/* One time step on the resident state: smodel_super_prep_sol (sol_older <- sol_old
 * <- sol) then fe_newton, as advance_time does (src/timeloop/time_loop.c:56-89). */
int sw2g_step(sw2g_model *m, const sw2g_newton_opts *opts, sw2g_newton_stats *stats);
/* Undo the last sw2g_step: the levels go back to what they were before it (sol =
 * the step's start state, sol_old = its previous level), so that the same interval
 * can be tried again, e.g. with a smaller dt after a failed Newton solve.  The
 * reference instead scales dt by DT_REDUCE_FACTOR (tc_scale, src/tools/tc_scale.c:10,
 * called at src/newton/fe_newton.c:887) and ends its time loop (time_loop.c:37).
 * The step overwrote the sol_older level, so this is refused (SW2G_ERR_ARG) under
 * the three-level scheme (tau_temporal != 0), after sw2g_load_state or any entry
 * point that loads states, and a second time in a row.  The permanent Dirichlet
 * marks the step added stay, as they do in the reference. */
int sw2g_undo_step(sw2g_model *m);
/* Device pointers of the resident state (for device-side consumers such as the
 * learned initial-guess network). */
int sw2g_device_state(sw2g_model *m, double **sol, double **sol_old, double **sol_older);
void *sw2g_stream(sw2g_model *m);

/* --- instrumentation ------------------------------------------------------ */
/* The AMG's chunk corrections at the last preconditioner set-up: info[0] nodes whose
 * smoother block the l1 fix-up weakened, info[1] chunks, info[2] chunk nodes (with
 * overlap), info[3] entries of the inverse rows kept, info[4] chunks left uncorrected
 * because their block was singular.  No counterpart in the reference (its UMFPACK LU
 * needs no such correction). */
int sw2g_precond_info(sw2g_model *m, long long *info);
/* Per kernel class, CUDA-event time (ms) and launch counts since the last reset:
 * classes 0 residual, 1 FD Jacobian, 2 Jacobian gather, 3 Dirichlet/scale/precond
 * setup, 4 BiCGStab, 5 other.  Timing adds events around each class. */
#define SW2G_NCLASSES 6
int sw2g_set_profiling(sw2g_model *m, int on);
int sw2g_get_profile(sw2g_model *m, double *ms, long long *launches);
int sw2g_reset_profile(sw2g_model *m);
/* Times `reps` launches of one kernel on the resident data (CUDA events on the
 * model's stream) and returns the mean launch time and the algorithmic bytes of
 * one launch: 0 FP64 SpMV, 1 FD Jacobian element kernels, 2 element residual,
 * 3 Jacobian gather, 4 AMG level-0 smoothing sweep (FP64), 5 the same sweep on FP32
 * values and vectors, 6 one FP32 AMG V-cycle (bytes: its four level-0 matrix passes),
 * 7 FP32 SpMV, 8 one whole FP32 GMRES cycle with its stopping test off (bytes: the
 * cycle's iteration count, so avg_ms / bytes is one iteration; needs a prior FP32 GMRES
 * solve), 9 the AMG's chunk corrections in FP32 (bytes: inverse rows and residuals read).
 * Instrumentation for roofline
 * reporting; no counterpart in the reference. */
int sw2g_time_kernel(sw2g_model *m, int which, int reps, double *avg_ms, double *bytes);

#ifdef __cplusplus
}
#endif
#endif
