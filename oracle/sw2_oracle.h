/*
 * CPU restatement of the reference's SW2 implicit time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.  It is
 * pinned against the reference's own compiled code (oracle/_ref/) by the tests in
 * tests/test_oracle_vs_reference.py and by the committed fixtures in tests/golden/.
 *
 * Every routine restates one reference routine with the same floating-point
 * operation order (built without FMA contraction), so its element residuals and
 * element Jacobians are bit-identical to the reference's.  File:line citations are
 * relative to the reference project root.
 */
#ifndef SW2_ORACLE_H
#define SW2_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nnodes, ntri, nseg;
    const double *xyz;       /* 3*nnodes: x, y, bed z */
    const int *tri;          /* 3*ntri, counter-clockwise */
    const int *seg;          /* 2*nseg, node order gives the outward normal */
    const int *seg_kind;     /* nseg: 0 = NB VEL (fe_sw2_bc_vel), 1 = DEPTH (fe_sw2_bc_h),
                                2 = discharge (sw2_bc_discharge.c.bk), 3 = tailwater (sw2_bc_tailwater.c.bk),
                                4 = outflow (sw2_bc_outflow.c.bk), 5 = flux (sw2_bc_flux.c.bk) */
    const double *tri_djac;  /* ntri: element area */
    const double *tri_grad;  /* 6*ntri: grad phi_a (x,y) for a = 0..2 */
    const double *seg_djac;  /* nseg: segment length */
    const double *seg_nrml;  /* 2*nseg: outward unit normal */
    int ndof, nnz;
    const int *indptr;       /* ndof+1 */
    const int *cols;         /* nnz, sorted within each row */
    double gravity;
    double dt;               /* ts->dt / nsubsteps (nsubsteps = 1) */
    double tau_temporal;     /* alpha of the 3-level scheme, 0 = backward Euler */
    double bc_depth, bc_vx, bc_vy; /* step-averaged series values (ids 0, 1, 2) */
    int *wd_flag;            /* ntri, written by sw2o_wd_flags */
    double bc_qs;            /* discharge string's series value */
    double bc_convey;        /* discharge string's conveyance */
    double bc_rough;         /* boundary strings' equivalent roughness height */
    double bc_tail;          /* tailwater elevation */
    double bc_flux;          /* flux string's series value */
} sw2o_model;

/* geometry: selem2d_get_triangle_linear_djac_nrml_gradPhi (src/structs/selem/selem_2d.c:270-350),
 * selem1d_load (src/structs/selem/selem_1d.c:27-58) */
void sw2o_geometry(int nnodes, int ntri, int nseg, const double *xyz, const int *tri, const int *seg,
                   double *tri_djac, double *tri_grad, double *seg_djac, double *seg_nrml);

/* sparsity: slin_sys_init_sparsity_mono (src/structs/slin_sys/slin_sys_init_sparsity_mono.c:28) */
int sw2o_sparsity_nnz(int nnodes, int ntri, int nseg, const int *tri, const int *seg);
void sw2o_sparsity(int nnodes, int ntri, int nseg, const int *tri, const int *seg, int *indptr, int *cols);

/* wet/dry flags: fe_sw2_wdflag_legacy (src/models/sw2/sw2_wdflag_legacy.c:34) */
void sw2o_wd_flags(sw2o_model *m, const double *sol, const double *sol_old);

/* element residuals (unperturbed) for every triangle (9 each) and segment (6 each) */
void sw2o_elem_resid_all(const sw2o_model *m, const double *sol, const double *sol_old,
                         const double *sol_older, double *out_tri, double *out_seg);
/* one triangle with an optional perturbation (pvar < 0: none) */
void sw2o_body_resid(const sw2o_model *m, const double *sol, const double *sol_old, const double *sol_older,
                     int e, double pert, int pnode, int pvar, int psign, double *elem_rhs);
/* element FD Jacobians: 81 per triangle, 36 per segment, row-major [row][col] */
void sw2o_elem_jac_all(const sw2o_model *m, const double *sol, const double *sol_old,
                       const double *sol_older, double *out_tri, double *out_seg);

/* assemble_residual (src/residual/assemble_residual.c:69) */
void sw2o_assemble_residual(const sw2o_model *m, const double *sol, const double *sol_old,
                            const double *sol_older, double *residual);
/* assemble_jacobian (src/jacobian/assemble_jacobian.c:20) */
void sw2o_assemble_jacobian(const sw2o_model *m, const double *sol, const double *sol_old,
                            const double *sol_older, double *vals);

/* check_diag, apply_Dirichlet_BC (src/la/matrix_utilities.c:120,42) */
void sw2o_check_diag(const sw2o_model *m, const double *vals, int *bc_mask);
void sw2o_apply_dirichlet(const sw2o_model *m, const int *bc_mask, double *vals, double *residual);
/* scale_linear_system (src/la/scale_linear_system.c:31) */
void sw2o_scale_system(const sw2o_model *m, double *vals, double *b, double *x, double *scale_vect);
/* split_CSR_mat_vec_mult, serial branch (src/la/matrix_utilities.c:203-215) */
void sw2o_spmv(int n, const int *indptr, const int *cols, const double *vals, const double *x, double *y);

/* Left-preconditioned BiCGStab of src/la/bcgstab_solver.c:65-330 with the exact LU
 * replaced by a 3x3 nodal block-Jacobi preconditioner.  Returns the iteration count
 * (negative on breakdown).  x is in/out as in the reference (x0 shift, unscaled). */
int sw2o_bicgstab_bj(int n, const int *indptr, const int *cols, const double *vals, double *x,
                     double *b, const double *scale_vect, int max_it, double tol);

/* fe_newton (src/newton/fe_newton.c:44) for one time step with block-Jacobi BiCGStab.
 * On entry sol_old/sol_older hold the previous levels; sol receives the result (on
 * failure, the start of the step again, as fe_newton resets it).
 * bc_mask (ndof) and dirichlet (ndof) persist across steps like sm->bc_mask.
 * stats[0] = Newton iterations, stats[1] = total Krylov iterations,
 * stats[2] = final residual max norm, stats[3] = success flag, stats[4] = line-search
 * halvings over all Newton iterations. */
int sw2o_newton(sw2o_model *m, double *sol, const double *sol_old, const double *sol_older,
                int *bc_mask, const double *dirichlet, double tol_nonlin, double inc_nonlin,
                int max_nonlin_it, int max_linesearch_cuts, int krylov_max_it, double krylov_tol,
                double *stats);

/* mass balance: tl_find_grid_mass_elem2d (src/tools/tl_grid_mass.c:198) of the depths in sol,
 * one triangle's term of it, and one step's boundary mass flux (inflow positive) of the
 * boundary loop of tl_find_grid_mass_error_elem2d (tl_grid_mass.c:310-320); that loop
 * weights every segment by the first segment's length, which first_seg_length = 1
 * reproduces (0: each segment's own length, what the CUDA path computes) */
double sw2o_grid_mass(const sw2o_model *m, const double *sol, double density);
double sw2o_elem_mass(const sw2o_model *m, const double *sol, int e);
double sw2o_boundary_mass_flux(const sw2o_model *m, const double *sol, double density, double dt,
                                int first_seg_length);

/* flop counter for one unperturbed triangle residual evaluation (fully wet path) */
long sw2o_body_resid_flops(void);

#ifdef __cplusplus
}
#endif
#endif
