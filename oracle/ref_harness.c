/*
 * Reference harness: drives the reference's own, unmodified SW2 C code (compiled
 * from the reference tree by oracle/Makefile into oracle/_ref/) on a mesh and
 * state read from a case file, and writes what the reference computes.  It is the
 * pin for the CPU restatement in oracle/sw2_oracle.c and for the CUDA path.
 * Test infrastructure only: the product never links or runs it.
 *
 * Model set-up follows the reference's no-read path, the one its own tests use
 * (src/test/test_sw2_nb.c:40-330, commented out upstream):
 *   smodel_design_init_no_read -> smodel_super_no_read -> slin_sys_init_ptrs
 *   -> slin_sys_init_sparsity_mono   (src/structs/smodel_design/smodel_design_init_no_read.c)
 * The grid is built with the reference's selem2d_load / selem1d_load (the same
 * calls create_rectangular_grid makes, src/tools/create_rectangular_grid.c:173-440).
 *
 * Fix-ups for latent reference bugs (each keeps the reference's arithmetic):
 *  (i)   sm->str_values is never allocated but is read at
 *        str_values[elem2d->string] with string = UNSET_INT (sw2_body_resid.c:87)
 *        and at str_values[mat].ol_flow.ivx/ivy (sw2_bc_vel.c:147-150): we give it
 *        a zeroed table with three entries before index 0 and set ivx/ivy.
 *  (ii)  dvars.elem_flags has one row but is indexed [adh_def._WDFLAG]
 *        (sdvar.c:105, sw2_body_resid.c:88): we re-point a full row table.
 *  (iii) the no-read path never sets pde->init; the file path sets fe_sw2_init
 *        for the SW2 model (read_bc_MODEL.c:124): we do the same.
 *  (iv)  smodel_super_no_read indexes a boundary material's pde by the running
 *        boundary counter instead of the per-material counter
 *        (smodel_super_no_read.c: "pde = &mat->pde[bc_ctr]"), which writes past
 *        the second boundary material's one-entry pde array.  We register every
 *        material as model "SW2" (imod = _SW2, the same imod select_bresid_func
 *        returns for both SW2 boundary kinds, sadh_def.c:279-297) and then set the
 *        boundary materials' resid pointers to what select_bresid_func returns:
 *        fe_sw2_bc_vel for "NB VEL", fe_sw2_bc_h for "DEPTH".
 *  (v)   series: id 0 = the depth series (hard-coded in sw2_bc_h.c:156), ids 1/2 =
 *        the velocity x/y series named by str_values[mat].ol_flow.ivx/ivy.
 *        Slopes and trapezoid areas are filled as sseries_read does
 *        (sseries.c:94-105) with the reference's tc_trap_area.
 *  (vi)  selem1d_init_alloc_array writes through node arrays it never allocated
 *        (selem_1d.c:86-125); see build_grid.
 *
 * Built a second time with -DSW2_REFGLUE into adh_refglue_harness: the reference's
 * objects without src/residual/assemble_residual.c and src/jacobian/assemble_jacobian.c,
 * linked with adh_kraken_b200/refglue/sw2_refglue.c, whose assemble_residual /
 * assemble_jacobian run on the GPU; mode "loop" then runs the reference's own Newton
 * on GPU assemblies and mode "loop_gpu" installs fe_newton_gpu as the stepper.
 *
 * Usage: adh_ref_harness <dump|run|loop|time|mass> <case.bin> <out.bin> [every|reps]
 *        adh_ref_harness init <case.bin> <out.bin> <init file base>
 *        adh_ref_harness geo <grid.geo> <out.bin>
 *        adh_ref_harness rect - <out.bin> xmin xmax ymin ymax npx npy a0 ax
 */
#include "adh.h"
#include <stdint.h>
#ifdef SW2_REFGLUE
#include "sw2_refglue.h"
#endif

SADH_DEF adh_def; /* defined by src/main/adh.c in the reference binary */

/* Stand-in for src/structs/sflags/sflags.c:21, which does not compile without
 * _HDF5: every flag off, and the per-model switch array that model_flag_switch
 * (read_bc_MODEL.c:9) writes, filled with UNSET_INT as the original does. */
void sflags_init(SFLAGS *f) {
    memset(f, 0, sizeof(SFLAGS));
    f->model = (int *)tl_alloc(sizeof(int), adh_def.nmodels);
    sarray_init_value_int(f->model, adh_def.nmodels, UNSET_INT);
}

/* ---------------------------------------------------------------- output file */
static FILE *g_out = NULL;
static void out_rec(const char *name, char type, const void *data, int64_t count) {
    char nm[32]; memset(nm, 0, sizeof nm); strncpy(nm, name, 31);
    fwrite(nm, 1, 32, g_out);
    fwrite(&type, 1, 1, g_out);
    fwrite(&count, sizeof(int64_t), 1, g_out);
    size_t es = (type == 'd') ? sizeof(double) : sizeof(int);
    if (count > 0) fwrite(data, es, (size_t)count, g_out);
}

/* ---------------------------------------------------------------- case file */
typedef struct {
    int nnodes, ntri, nseg, nsteps;
    double dt, t0, tol_nonlin, inc_nonlin, gravity;
    int max_nonlin_it;
    double *xyz; int *tri; int *seg; int *seg_kind;
    double *sol, *sol_old, *sol_older;
    int nseries; int *ser_id, *ser_n; double **ser_t, **ser_v;
} CASE;

static void rd(void *p, size_t sz, size_t n, FILE *f) {
    if (fread(p, sz, n, f) != n) { fprintf(stderr, "harness: short case file\n"); exit(2); }
}

static CASE read_case(const char *path) {
    CASE c; memset(&c, 0, sizeof c);
    FILE *f = fopen(path, "rb");
    if (!f) { fprintf(stderr, "harness: cannot open %s\n", path); exit(2); }
    int32_t magic, version; rd(&magic, 4, 1, f); rd(&version, 4, 1, f);
    if (magic != 0x43325753 || version != 1) { fprintf(stderr, "harness: bad case header\n"); exit(2); }
    int32_t iv[5]; rd(iv, 4, 5, f);
    c.nnodes = iv[0]; c.ntri = iv[1]; c.nseg = iv[2]; c.nsteps = iv[3]; c.max_nonlin_it = iv[4];
    double dv[5]; rd(dv, 8, 5, f);
    c.dt = dv[0]; c.t0 = dv[1]; c.tol_nonlin = dv[2]; c.inc_nonlin = dv[3]; c.gravity = dv[4];
    c.xyz = malloc(sizeof(double) * 3 * c.nnodes); rd(c.xyz, 8, 3 * (size_t)c.nnodes, f);
    c.tri = malloc(sizeof(int) * 3 * c.ntri); rd(c.tri, 4, 3 * (size_t)c.ntri, f);
    c.seg = malloc(sizeof(int) * 2 * (c.nseg + 1)); rd(c.seg, 4, 2 * (size_t)c.nseg, f);
    c.seg_kind = malloc(sizeof(int) * (c.nseg + 1)); rd(c.seg_kind, 4, (size_t)c.nseg, f);
    size_t nd = 3 * (size_t)c.nnodes;
    c.sol = malloc(8 * nd); c.sol_old = malloc(8 * nd); c.sol_older = malloc(8 * nd);
    rd(c.sol, 8, nd, f); rd(c.sol_old, 8, nd, f); rd(c.sol_older, 8, nd, f);
    int32_t ns; rd(&ns, 4, 1, f); c.nseries = ns;
    c.ser_id = malloc(sizeof(int) * ns); c.ser_n = malloc(sizeof(int) * ns);
    c.ser_t = malloc(sizeof(double *) * ns); c.ser_v = malloc(sizeof(double *) * ns);
    for (int s = 0; s < ns; s++) {
        int32_t h[2]; rd(h, 4, 2, f); c.ser_id[s] = h[0]; c.ser_n[s] = h[1];
        c.ser_t[s] = malloc(8 * h[1]); c.ser_v[s] = malloc(8 * h[1]);
        rd(c.ser_t[s], 8, h[1], f); rd(c.ser_v[s], 8, h[1], f);
    }
    fclose(f);
    return c;
}

/* ---------------------------------------------------------------- model build */
static SMODEL_DESIGN g_dm;
static SMODEL_SUPER *g_sm;

static void build_grid(const CASE *c) {
    SGRID *grid = (SGRID *)tl_alloc(sizeof(SGRID), 1);
    memset(grid, 0, sizeof(SGRID));
    grid->nnodes = c->nnodes; grid->max_nnodes = c->nnodes;
    grid->nelems3d = 0; grid->nelems2d = c->ntri; grid->nelems1d = c->nseg;
    grid->max_nelems1d = c->nseg; grid->max_nelems2d = c->ntri; grid->max_nelems3d = 0;
    grid->nTris = c->ntri;
    grid->nnodes_sur = c->nnodes;
    grid->inv_per_node = (int *)tl_alloc(sizeof(int), c->nnodes);
    grid->macro_nnodes = c->nnodes; grid->macro_nnodes_sur = c->nnodes;
    grid->macro_nelems2d = c->ntri; grid->macro_nelems1d = c->nseg; grid->macro_nTris = c->ntri;
    grid->orig_macro_nnodes = c->nnodes; grid->orig_macro_nnodes_sur = c->nnodes;
    grid->orig_macro_nelems1d = c->nseg; grid->orig_macro_nelems2d = c->ntri;
    grid->my_nnodes = c->nnodes; grid->my_nnodes_sur = c->nnodes;
    grid->my_nelems2d = c->ntri; grid->my_nelems1d = c->nseg; grid->my_nTris = c->ntri;
    if (c->nseg > 0) {
        /* fix-up (vi): selem1d_init_alloc_array (selem_1d.c:119) initialises
         * elements whose node arrays were never allocated; allocate zeroed
         * elements and let selem1d_load allocate the arrays. */
        selem1d_alloc_array(&(grid->elem1d), c->nseg);
        memset(grid->elem1d, 0, sizeof(SELEM_1D) * (size_t)c->nseg);
        for (int k = 0; k < c->nseg; k++) selem1d_init(&grid->elem1d[k]);
    }
    selem2d_init_alloc_array(&(grid->elem2d), c->ntri);
    snode_init_alloc_array(&(grid->node), c->nnodes);
    for (int i = 0; i < c->nnodes; i++) {
        grid->node[i].id = i; grid->node[i].original_id = i; grid->node[i].gid = i;
        grid->node[i].x = c->xyz[3 * i]; grid->node[i].y = c->xyz[3 * i + 1]; grid->node[i].z = c->xyz[3 * i + 2];
    }
    for (int k = 0; k < c->ntri; k++) {
        int ids[3]; SVECT nds[3];
        for (int a = 0; a < 3; a++) {
            ids[a] = c->tri[3 * k + a];
            nds[a].x = grid->node[ids[a]].x; nds[a].y = grid->node[ids[a]].y; nds[a].z = grid->node[ids[a]].z;
        }
        selem2d_init(&grid->elem2d[k]);
        selem2d_load(&(grid->elem2d[k]), k, k, 3, ids, 0, nds, 0);
        grid->elem2d[k].bflag = BODY;
    }
    for (int k = 0; k < c->nseg; k++) {
        int ids[2]; SVECT nds[2];
        for (int a = 0; a < 2; a++) {
            ids[a] = c->seg[2 * k + a];
            nds[a].x = grid->node[ids[a]].x; nds[a].y = grid->node[ids[a]].y; nds[a].z = grid->node[ids[a]].z;
        }
        selem1d_load(&(grid->elem1d[k]), k, k, 2, ids, 0, nds, 0);
    }
    g_dm.grid = grid;
}

static void add_series(const CASE *c) {
    g_sm->series_head = NULL; g_sm->series_curr = NULL;
    for (int s = 0; s < c->nseries; s++) {
        SSERIES *series;
        sseries_alloc(&series, c->ser_n[s], TIME_SERIES, 0);
        series->id = c->ser_id[s]; series->infact = 1; series->outfact = 1;
        for (int e = 0; e < c->ser_n[s]; e++) {
            series->entry[e].time = c->ser_t[s][e];
            series->entry[e].value[0] = c->ser_v[s][e];
        }
        for (int e = 1; e < series->size; e++)
            series->entry[e - 1].slope[0] = (series->entry[e].value[0] - series->entry[e - 1].value[0]) /
                                            (series->entry[e].time - series->entry[e - 1].time);
        for (int e = 0; e < series->size - 1; e++)
            series->entry[e].area[0] = tc_trap_area(series->entry[e].value[0], series->entry[e + 1].value[0],
                                                    series->entry[e].time, series->entry[e + 1].time);
        sseries_add(series, &(g_sm->series_head), &(g_sm->series_curr), TRUE);
        sseries_free(series);
    }
}

static void build_model(const CASE *c) {
    smodel_design_defaults(&g_dm);
    build_grid(c);
    double tf = c->t0 + c->dt * (c->nsteps > 0 ? c->nsteps : 1);
    int nSuper = 1;
    int nmat = 3;
    int nphys[1] = {3};
    int npdes_m[3] = {1, 1, 1};
    int *npdes[1] = {npdes_m};
    int mvb_m[3] = {1, 1, 1}; /* fix-up (iv): all registered as model SW2 */
    int *mvb[1] = {mvb_m};
    char *ms_m[3] = {"SW2", "SW2", "SW2"};
    char **ms[1] = {ms_m};
    char *bp_m[1] = {"SW2"}; char **bp[1] = {bp_m};
    char *bt_m[1] = {"NB"}; char **bt[1] = {bt_m};
    char *bv_m[1] = {"VEL"}; char **bv[1] = {bv_m};
    int bs_m[1] = {0}; int *bs[1] = {bs_m};
    int nel = c->ntri + c->nseg;
    int *mat_ids_m = (int *)malloc(sizeof(int) * (nel + 1));
    for (int j = 0; j < c->ntri; j++) mat_ids_m[j] = 0;
    for (int j = 0; j < c->nseg; j++) mat_ids_m[c->ntri + j] = (c->seg_kind[j] == 0) ? 1 : 2;
    int *mat_ids[1] = {mat_ids_m};
    (void)nmat;
    smodel_design_init_no_read(&g_dm, c->dt, c->t0, tf, nSuper, nphys, npdes, mvb, ms, bp, bt, bv, bs, mat_ids);
    g_sm = &(g_dm.superModel[0]);
    SMODEL_SUPER *sm = g_sm;
    /* fix-up (iv): boundary resid pointers as select_bresid_func returns them */
    sm->mat_physics_elem[1].pde[0].resid = fe_sw2_bc_vel;
    sm->mat_physics_elem[2].pde[0].resid = fe_sw2_bc_h;
    /* fix-up (iii) */
    sm->mat_physics_elem[0].pde[0].init = fe_sw2_init;
    /* fix-up (i) */
    STR_VALUE *sv = (STR_VALUE *)calloc(3 + 8, sizeof(STR_VALUE));
    sm->str_values = sv + 3;
    sm->str_values[1].ol_flow.ivx = 1;
    sm->str_values[1].ol_flow.ivy = 2;
    /* fix-up (ii) */
    int *row = sm->dvars.elem_flags[0];
    int **rows = (int **)calloc(MAX_NDVARS, sizeof(int *));
    for (int k = 0; k < MAX_NDVARS; k++) rows[k] = row;
    sm->dvars.elem_flags = rows;
    /* fix-up (v) */
    add_series(c);
    /* solver settings */
    sm->tol_nonlin = c->tol_nonlin;
    sm->inc_nonlin = c->inc_nonlin;
    sm->max_nonlin_it = c->max_nonlin_it;
    sm->gravity = c->gravity;
    g_dm.ts.dt = c->dt; g_dm.ts.t_prev = c->t0; g_dm.ts.t_init = c->t0; g_dm.ts.t_final = tf;
    /* alpha of the three-level temporal scheme; the reference's default is 0 (sdt.c:24) */
    g_dm.ts.tau_temporal = getenv("HARNESS_TAU") ? atof(getenv("HARNESS_TAU")) : 0.;
    for (int i = 0; i < sm->ndofs; i++) {
        sm->sol[i] = c->sol[i]; sm->sol_old[i] = c->sol_old[i]; sm->sol_older[i] = c->sol_older[i];
        sm->dirichlet_data[i] = 0.; sm->lin_sys->dsol[i] = 0.;
    }
}

/* ---------------------------------------------------------------- modes */
/* The reference's own time loop (src/timeloop/time_loop.c:14-89: tc_init, update_dt,
 * advance_time -> adh_time_stepper[sm->forward_step]) over the case's steps.  The
 * stepper installed in adh_time_stepper[FE_NEWTON] is wrapped so that every step's
 * state, success flag and Newton count are recorded as the loop runs. */
static int (*g_inner_stepper)(SMODEL_SUPER *) = NULL;
static int g_loop_steps = 0, g_loop_cap = 0;
static double *g_loop_sol = NULL;
static int *g_loop_ok = NULL, *g_loop_its = NULL;
static double *g_loop_secs = NULL;

static double now_s(void);
static int recording_stepper(SMODEL_SUPER *sm) {
    const int before = sm->it_count_nonlin;
    const double t0 = now_s();
    const int r = g_inner_stepper(sm);
    if (g_loop_steps < g_loop_cap) {
        memcpy(g_loop_sol + (size_t)sm->ndofs * g_loop_steps, sm->sol, sizeof(double) * sm->ndofs);
        g_loop_ok[g_loop_steps] = r;
        g_loop_its[g_loop_steps] = sm->it_count_nonlin - before;
        g_loop_secs[g_loop_steps] = now_s() - t0;
    }
    g_loop_steps++;
    return r;
}

static void mode_loop(const CASE *c, int (*stepper)(SMODEL_SUPER *)) {
    SMODEL_SUPER *sm = g_sm;
    g_loop_cap = c->nsteps + 2;
    g_loop_sol = calloc((size_t)sm->ndofs * g_loop_cap, sizeof(double));
    g_loop_ok = calloc(g_loop_cap, sizeof(int));
    g_loop_its = calloc(g_loop_cap, sizeof(int));
    g_loop_secs = calloc(g_loop_cap, sizeof(double));
    g_inner_stepper = stepper;
    adh_time_stepper[FE_NEWTON] = recording_stepper;
    time_loop(&g_dm);
    const int n = g_loop_steps < g_loop_cap ? g_loop_steps : g_loop_cap;
    out_rec("newton_its", 'i', g_loop_its, n);
    out_rec("step_ok", 'i', g_loop_ok, n);
    out_rec("step_seconds", 'd', g_loop_secs, n);
    out_rec("sol_steps", 'd', g_loop_sol, (int64_t)sm->ndofs * n);
    out_rec("bc_mask", 'i', sm->bc_mask, sm->ndofs);
}

static double now_s(void) { struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts); return ts.tv_sec + 1e-9 * ts.tv_nsec; }

#ifndef SW2_REFGLUE
static void mode_dump(const CASE *c) {
    SMODEL_SUPER *sm = g_sm; SGRID *grid = sm->grid; SLIN_SYS *ls = sm->lin_sys;
    int V = grid->nnodes, T = grid->nelems2d, S = grid->nelems1d, N = sm->ndofs;
    int nnz = ls->nnz_diag;
    sseries_setall_ts_valuesAVG(sm->series_head, c->t0, c->t0 + c->dt);
    fe_sw2_wdflag_legacy(sm);
    int *dof = malloc(sizeof(int) * 3 * V);
    for (int v = 0; v < 3; v++) for (int i = 0; i < V; i++) dof[v * V + i] = sm->ivars[v][i];
    out_rec("dofmap", 'i', dof, 3 * (int64_t)V);
    out_rec("indptr", 'i', ls->indptr_diag, N + 1);
    out_rec("cols", 'i', ls->cols_diag, nnz);
    out_rec("wd_flag", 'i', sm->dvars.elem_flags[adh_def._WDFLAG], T);
    double bcv[3] = {sseries_get_value(0, sm->series_head, 0), 0., 0.};
    if (c->nseries > 1) { bcv[1] = sseries_get_value(1, sm->series_head, 0); bcv[2] = sseries_get_value(2, sm->series_head, 0); }
    out_rec("bc_values", 'd', bcv, 3);
    double *er = calloc((size_t)T * 9 + 1, sizeof(double));
    double buf[64];
    for (int e = 0; e < T; e++) {
        memset(buf, 0, sizeof buf);
        fe_sw2_body_resid(sm, buf, e, 0.0, UNSET_INT, UNSET_INT, 0, 0);
        memcpy(er + 9 * (size_t)e, buf, 9 * sizeof(double));
    }
    out_rec("elem_rhs_tri", 'd', er, 9 * (int64_t)T);
    double *es = calloc((size_t)S * 6 + 1, sizeof(double));
    for (int e = 0; e < S; e++) {
        memset(buf, 0, sizeof buf);
        int m = sm->elem1d_physics_mat[e];
        sm->mat_physics_elem[m].pde[0].resid(sm, buf, e, 0.0, UNSET_INT, UNSET_INT, 0, 0);
        memcpy(es + 6 * (size_t)e, buf, 6 * sizeof(double));
    }
    out_rec("elem_rhs_seg", 'd', es, 6 * (int64_t)S);
    /* element FD Jacobians through the reference's own load_elem_mat */
    int md = sm->ivar_pos.n * MAX_NNODE;
    double **em = malloc(sizeof(double *) * md);
    for (int k = 0; k < md; k++) em[k] = calloc(md, sizeof(double));
    double *ej = calloc((size_t)T * 81 + 1, sizeof(double));
    for (int e = 0; e < T; e++) {
        sarray_init_double_2d(em, md, md);
        load_elem_mat(sm, 3, grid->elem2d[e].nodes, sm->elem2d_physics_mat[e], e, em);
        for (int i = 0; i < 9; i++) for (int j = 0; j < 9; j++) ej[81 * (size_t)e + 9 * i + j] = em[i][j];
    }
    out_rec("elem_jac_tri", 'd', ej, 81 * (int64_t)T);
    double *sj = calloc((size_t)S * 36 + 1, sizeof(double));
    for (int e = 0; e < S; e++) {
        sarray_init_double_2d(em, md, md);
        load_elem_mat(sm, 2, grid->elem1d[e].nodes, sm->elem1d_physics_mat[e], e, em);
        for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) sj[36 * (size_t)e + 6 * i + j] = em[i][j];
    }
    out_rec("elem_jac_seg", 'd', sj, 36 * (int64_t)S);
    assemble_residual(sm, grid);
    out_rec("residual", 'd', ls->residual, N);
    assemble_jacobian(sm);
    out_rec("jac_vals", 'd', ls->vals_diag, nnz);
    for (int i = 0; i < N; i++) if (sm->bc_mask[i] != YES) sm->bc_mask[i] = 0;
    check_diag(sm);
    apply_Dirichlet_BC(sm);
    out_rec("bc_mask", 'i', sm->bc_mask, N);
    out_rec("jac_vals_dirichlet", 'd', ls->vals_diag, nnz);
    out_rec("residual_dirichlet", 'd', ls->residual, N);
    sarray_init_dbl(ls->dsol, N);
    scale_linear_system(ls->indptr_diag, ls->cols_diag, ls->vals_diag, ls->indptr_off_diag, ls->cols_off_diag,
                        ls->vals_off_diag, ls->residual, ls->dsol, ls->scale_vect, *(ls->local_size), *(ls->size), 0,
                        ls->ghosts, ls->nghost);
    out_rec("scale_vect", 'd', ls->scale_vect, N);
    out_rec("jac_vals_scaled", 'd', ls->vals_diag, nnz);
    out_rec("residual_scaled", 'd', ls->residual, N);
    if (getenv("HARNESS_SKIP_SOLVE") == NULL) {
        prep_umfpack(ls->indptr_diag, ls->cols_diag, ls->vals_diag, *(ls->local_size));
        solve_linear_sys_bcgstab(ls->dsol, ls->indptr_diag, ls->cols_diag, ls->vals_diag, ls->indptr_off_diag,
                                 ls->cols_off_diag, ls->vals_off_diag, ls->residual, ls->scale_vect,
                                 *(ls->local_size), *(ls->size), 0, ls->ghosts, ls->nghost);
        out_rec("dsol", 'd', ls->dsol, N);
    }
}

#endif

static void mode_run(const CASE *c, int every) {
    SMODEL_SUPER *sm = g_sm; int N = sm->ndofs;
    int nsteps = c->nsteps;
    int *its = calloc(nsteps + 1, sizeof(int));
    int *ok = calloc(nsteps + 1, sizeof(int));
    double *secs = calloc(nsteps + 1, sizeof(double));
    double *bcv = calloc(3 * (size_t)nsteps + 3, sizeof(double));
    int nkeep = 0;
    double *keep = calloc((size_t)N * (nsteps / every + 2), sizeof(double));
    int done = 0;
    for (int ts = 0; ts < nsteps; ts++) {
        g_dm.ts.t_prev += g_dm.ts.dt;
        smodel_super_prep_sol(sm);
        sseries_setall_ts_valuesAVG(sm->series_head, sm->ts->t_prev - sm->ts->dt, sm->ts->t_prev);
        bcv[3 * ts] = sseries_get_value(0, sm->series_head, 0);
        if (c->nseries > 1) { bcv[3 * ts + 1] = sseries_get_value(1, sm->series_head, 0); bcv[3 * ts + 2] = sseries_get_value(2, sm->series_head, 0); }
        int before = sm->it_count_nonlin;
        double t0 = now_s();
        int r = fe_newton(sm);
        secs[ts] = now_s() - t0;
        its[ts] = sm->it_count_nonlin - before;
        ok[ts] = r;
        done = ts + 1;
        if ((ts + 1) % every == 0 || ts + 1 == nsteps || !r) {
            memcpy(keep + (size_t)N * nkeep, sm->sol, sizeof(double) * N);
            nkeep++;
        }
        if (!r) break;
    }
    out_rec("newton_its", 'i', its, done);
    out_rec("step_ok", 'i', ok, done);
    out_rec("step_seconds", 'd', secs, done);
    out_rec("bc_values", 'd', bcv, 3 * (int64_t)done);
    out_rec("sol_kept", 'd', keep, (int64_t)N * nkeep);
    out_rec("bc_mask", 'i', sm->bc_mask, N);
}

/* CPU-baseline timing of the reference's per-Newton-iteration assembly: one
 * assemble_residual + one assemble_jacobian at the case state, repeated. */
static void mode_time(const CASE *c, int reps) {
    SMODEL_SUPER *sm = g_sm;
    sseries_setall_ts_valuesAVG(sm->series_head, c->t0, c->t0 + c->dt);
    fe_sw2_wdflag_legacy(sm);
    double tr = 0, tj = 0;
    for (int r = 0; r < reps; r++) {
        double a = now_s(); assemble_residual(sm, sm->grid); double b = now_s();
        assemble_jacobian(sm); double d = now_s();
        tr += b - a; tj += d - b;
    }
    double v[3] = {tr / reps, tj / reps, (double)reps};
    out_rec("assembly_seconds", 'd', v, 3);
}

/* The reference's mass-balance tools on the case state (density 1, no flags):
 * tl_find_grid_mass_elem2d (src/tools/tl_grid_mass.c:198) of sol and of sol_old,
 * and tl_find_grid_mass_error_elem2d (tl_grid_mass.c:280) of sol with sol_old's
 * mass as the initial mass, which also returns one step's boundary mass flux. */
static void mode_mass(const CASE *c) {
    SMODEL_SUPER *sm = g_sm; SGRID *grid = sm->grid; int V = grid->nnodes;
    int *ih = sm->ivars[sm->ivar_pos.var[adh_def._H]];
    int *iu = sm->ivars[sm->ivar_pos.var[adh_def._UDA]], *iv = sm->ivars[sm->ivar_pos.var[adh_def._VDA]];
    double *head = malloc(sizeof(double) * V), *head_old = malloc(sizeof(double) * V);
    SVECT2D *vel = malloc(sizeof(SVECT2D) * V);
    for (int i = 0; i < V; i++) {
        head[i] = sm->sol[ih[i]]; head_old[i] = sm->sol_old[ih[i]];
        vel[i].x = sm->sol[iu[i]]; vel[i].y = sm->sol[iv[i]];
    }
    SFLAGS flags; memset(&flags, 0, sizeof flags);
    double m_new = tl_find_grid_mass_elem2d(1.0, NULL, NULL, head, grid, flags);
    double m_old = tl_find_grid_mass_elem2d(1.0, NULL, NULL, head_old, grid, flags);
    double flux_T = 0.;
    double err = tl_find_grid_mass_error_elem2d(1.0, head, vel, grid, flags, m_old, NULL, NULL, c->dt, &flux_T);
    double v[4] = {m_new, m_old, flux_T, err};
    out_rec("grid_mass", 'd', v, 4);
}

/* The reference's .geo reader, sgrid_read (src/structs/sgrid/sgrid_read.c:22), on a
 * grid file: node coordinates, triangle and segment node ids (0-based) and triangle
 * areas as the reader stores them.  argv = geo path, out path. */
static void mode_geo(char **argv) {
    SGRID *g = NULL;
    sgrid_read(&g, argv[2]);
    double *xyz = malloc(sizeof(double) * 3 * (g->nnodes + 1));
    for (int i = 0; i < g->nnodes; i++) { xyz[3*i] = g->node[i].x; xyz[3*i+1] = g->node[i].y; xyz[3*i+2] = g->node[i].z; }
    int *tri = malloc(sizeof(int) * 3 * (g->nelems2d + 1));
    double *djac = malloc(sizeof(double) * (g->nelems2d + 1));
    for (int e = 0; e < g->nelems2d; e++) {
        for (int a = 0; a < 3; a++) tri[3*e+a] = g->elem2d[e].nodes[a];
        djac[e] = g->elem2d[e].djac;
    }
    int *seg = malloc(sizeof(int) * 2 * (g->nelems1d + 1));
    for (int e = 0; e < g->nelems1d; e++) { seg[2*e] = g->elem1d[e].nodes[0]; seg[2*e+1] = g->elem1d[e].nodes[1]; }
    out_rec("xyz", 'd', xyz, 3 * (int64_t)g->nnodes);
    out_rec("tri", 'i', tri, 3 * (int64_t)g->nelems2d);
    out_rec("djac", 'd', djac, g->nelems2d);
    out_rec("seg", 'i', seg, 2 * (int64_t)g->nelems1d);
}

/* The reference's .init reader, smodel_super_read_init (src/structs/smodel_super/
 * smodel_super_read_init.c:26), on the case's model: the three solution levels start at
 * zero as smodel_super_read allocates them (smodel_super_read.c), then the file's
 * DATASETs fill them.  argv[4] = file base (the reader appends ".init"). */
static void mode_init(char *filebase) {
    SMODEL_SUPER *sm = g_sm;
    for (int i = 0; i < sm->ndofs; i++) { sm->sol[i] = 0.; sm->sol_old[i] = 0.; sm->sol_older[i] = 0.; }
    smodel_super_read_init(sm, filebase);
    out_rec("sol", 'd', sm->sol, sm->ndofs);
    out_rec("sol_old", 'd', sm->sol_old, sm->ndofs);
    out_rec("sol_older", 'd', sm->sol_older, sm->ndofs);
}

/* The reference's own structured-grid generator (src/tools/create_rectangular_grid.c:4),
 * used to pin the flume mesh builder: argv = xmin xmax ymin ymax npx npy a0 ax. */
static void mode_rect(int argc, char **argv) {
    if (argc < 12) { fprintf(stderr, "rect: xmin xmax ymin ymax npx npy a0 ax\n"); exit(2); }
    SGRID g = create_rectangular_grid(atof(argv[4]), atof(argv[5]), atof(argv[6]), atof(argv[7]),
                                      atoi(argv[8]), atoi(argv[9]), 0.0, 1, atof(argv[10]), atof(argv[11]),
                                      0., 0., 0., 0., 0., 0., 0., 0);
    double *xyz = malloc(sizeof(double) * 3 * g.nnodes);
    for (int i = 0; i < g.nnodes; i++) { xyz[3*i] = g.node[i].x; xyz[3*i+1] = g.node[i].y; xyz[3*i+2] = g.node[i].z; }
    int *tri = malloc(sizeof(int) * 3 * g.nelems2d);
    double *djac = malloc(sizeof(double) * g.nelems2d);
    double *grad = malloc(sizeof(double) * 6 * g.nelems2d);
    for (int e = 0; e < g.nelems2d; e++) {
        for (int a = 0; a < 3; a++) { tri[3*e+a] = g.elem2d[e].nodes[a]; grad[6*e+2*a] = g.elem2d[e].grad_shp[a].x; grad[6*e+2*a+1] = g.elem2d[e].grad_shp[a].y; }
        djac[e] = g.elem2d[e].djac;
    }
    out_rec("xyz", 'd', xyz, 3 * (int64_t)g.nnodes);
    out_rec("tri", 'i', tri, 3 * (int64_t)g.nelems2d);
    out_rec("djac", 'd', djac, g.nelems2d);
    out_rec("grad_shp", 'd', grad, 6 * (int64_t)g.nelems2d);
}

/* Mode "bcx": the discharge, tailwater, outflow and flux segment residuals of
 * sw2_bc_discharge.c.bk, sw2_bc_tailwater.c.bk, sw2_bc_outflow.c.bk and sw2_bc_flux.c.bk
 * (kinds 2-5; a flux record carries its series value in the q_series slot).  Those
 * files are not part of the reference's build and do not compile against its live
 * structures (the discharge file reads a NULL str_values, the others call an older
 * dof-map API), so their top-level steps are followed here line
 * by line while every integral, the roughness law and the drag coefficient are the
 * reference's own compiled functions (fe_sw2_1d_explicit_flow, fe_sw2_1d_wall_friction,
 * fe_sw2_1d_implicit_flow, fe_sw2_1d_pressure in src/fe/fe_sw2_boundary_integrals.c,
 * fe_sw2_get_roughness in src/models/sw2/sw2_get_roughness.c).  Input: int32 n, then n
 * records of 21 doubles {kind, nx, ny, djac, dt, g, h0, h1, u0, v0, u1, v1, z0, q_series,
 * conveyance, rough_height, tail_elev, perturbation, perturb_node, perturb_var (-1 none,
 * 0 h, 1 u, 2 v), perturb_sign}; output record "seg_resid", 6 doubles per segment. */
static void bcx_one(const double *in, double *out) {
    int kind = (int)in[0];
    SVECT2D nrml; nrml.x = in[1]; nrml.y = in[2];
    double djac = in[3], dt = in[4], g = in[5];
    double elem_head[2] = {in[6], in[7]};
    SVECT2D elem_vel[2];
    elem_vel[0].x = in[8]; elem_vel[0].y = in[9]; elem_vel[1].x = in[10]; elem_vel[1].y = in[11];
    double z0 = in[12], qs = in[13], convey = in[14], rough = in[15], tail = in[16];
    double perturbation = in[17];
    int perturb_node = (int)in[18], perturb_var = (int)in[19], perturb_sign = (int)in[20];
    int PRESSURE_FLAG = ON;
    if (perturb_var == 0) elem_head[perturb_node] += perturb_sign * perturbation;
    else if (perturb_var == 1) { elem_vel[perturb_node].x += perturb_sign * perturbation; PRESSURE_FLAG = OFF; }
    else if (perturb_var == 2) { elem_vel[perturb_node].y += perturb_sign * perturbation; PRESSURE_FLAG = OFF; }
    for (int i = 0; i < 6; i++) out[i] = 0.0;
    SELEM_1D elem1d; memset(&elem1d, 0, sizeof elem1d);
    STR_VALUE str; memset(&str, 0, sizeof str);
    str.fterms.sav_flag = NO; str.fterms.urv_flag = NO; str.fterms.icethick = UNSET_FLT; str.fterms.eqrheight = rough;
    SMODEL_SUPER mod; memset(&mod, 0, sizeof mod);
    mod.str_values = &str;
    if (kind == 2) {                       /* sw2_bc_discharge.c.bk:111-172 */
        double u_tan = one_2 * (elem_vel[0].x + elem_vel[1].x) * nrml.y - one_2 * (elem_vel[0].y + elem_vel[1].y) * nrml.x;
        double mag_utan = fabs(u_tan);
        double u[2] = {elem_vel[0].x, elem_vel[1].x}, v[2] = {elem_vel[0].y, elem_vel[1].y};
        double h_avg = one_2 * (elem_head[0] + elem_head[1]); if (h_avg < SMALL) h_avg = SMALL;
        double roughness[2], resistance[2];
        roughness[0] = fe_sw2_get_roughness(&mod, elem_head[0], 0.0, 0, UNUSED);
        roughness[1] = fe_sw2_get_roughness(&mod, elem_head[1], 0.0, 0, UNUSED);
        resistance[0] = one_2 * roughness[0] * mag_utan;
        resistance[1] = one_2 * roughness[1] * mag_utan;
        if (elem_head[0] < SMALL || elem_head[1] < SMALL) return;
        double troughness[2], discharge[2], three_2 = 3.0 / 2.0;
        troughness[0] = fe_sw2_get_roughness(&mod, elem_head[0], mag_utan, 0, UNUSED);
        troughness[1] = fe_sw2_get_roughness(&mod, elem_head[1], mag_utan, 0, UNUSED);
        double fact = -1.0 * qs * sqrt(2. * g / troughness[0]) / convey;
        discharge[0] = fact * pow(elem_head[0], three_2);
        fact = -1.0 * qs * sqrt(2. * g / troughness[1]) / convey;
        discharge[1] = fact * pow(elem_head[0], three_2);
        double elem_avg_discharge = one_2 * (discharge[0] + discharge[1]);
        fe_sw2_1d_explicit_flow(out, elem1d, 0, nrml, djac, dt, elem_avg_discharge, h_avg, u, v, OFF, OFF);
        fe_sw2_1d_wall_friction(out, elem1d, 0, nrml, djac, dt, u, v, resistance, OFF, OFF);
    } else if (kind == 4) {                /* sw2_bc_outflow.c.bk:144 */
        fe_sw2_1d_implicit_flow(out, elem1d, 0, nrml, djac, dt, elem_vel, elem_head, OFF, OFF);
    } else if (kind == 5) {                /* sw2_bc_flux.c.bk:114-116,151-153; the series value in the q_series slot */
        double u[2] = {elem_vel[0].x, elem_vel[1].x}, v[2] = {elem_vel[0].y, elem_vel[1].y};
        double h_avg = one_2 * (elem_head[0] + elem_head[1]); if (h_avg < SMALL) h_avg = SMALL;
        double flux = -1.0 * qs;
        fe_sw2_1d_explicit_flow(out, elem1d, 0, nrml, djac, dt, flux, h_avg, u, v, OFF, OFF);
    } else if (kind == 3) {                /* sw2_bc_tailwater.c.bk:152-170 */
        double elem_depth[2];
        elem_depth[0] = tail - z0;
        elem_depth[1] = tail - z0;
        if (elem_depth[0] < SMALL || elem_depth[1] < SMALL || elem_head[0] < SMALL || elem_head[1] < SMALL) return;
        fe_sw2_1d_implicit_flow(out, elem1d, 0, nrml, djac, dt, elem_vel, elem_head, OFF, OFF);
        if (PRESSURE_FLAG == ON) {
            fe_sw2_1d_pressure(out, elem1d, 0, nrml, djac, dt, elem_depth, g, OFF, OFF);
            fe_sw2_1d_pressure(out, elem1d, 0, nrml, djac, dt, elem_head, -g, OFF, OFF);
        }
    }
}

static int mode_bcx(const char *in_path, const char *out_path) {
    FILE *f = fopen(in_path, "rb");
    if (!f) { fprintf(stderr, "harness: cannot read %s\n", in_path); return 2; }
    int32_t n = 0;
    if (fread(&n, sizeof n, 1, f) != 1 || n < 0) { fclose(f); return 2; }
    double *in = malloc(sizeof(double) * 21 * ((size_t)n + 1));
    double *out = malloc(sizeof(double) * 6 * ((size_t)n + 1));
    if (!in || !out || fread(in, sizeof(double), 21 * (size_t)n, f) != 21 * (size_t)n) { fclose(f); return 2; }
    fclose(f);
    for (int32_t k = 0; k < n; k++) bcx_one(in + 21 * (size_t)k, out + 6 * (size_t)k);
    g_out = fopen(out_path, "wb");
    if (!g_out) { fprintf(stderr, "harness: cannot write %s\n", out_path); return 2; }
    out_rec("seg_resid", 'd', out, 6 * (int64_t)n);
    fclose(g_out);
    free(in); free(out);
    return 0;
}

/* Mode "params": the series pass of smodel_super_read
 * (src/structs/smodel_super/smodel_super_read.c:42-61) on a .params file, through the
 * reference's own tokenizer and sseries_read_allocate; output records "ids", "sizes",
 * "times" and "values" of the BC series in list order.  WIND and WAVE series are not
 * handled here (their station arrays need a node count). */
static int mode_params(const char *in_path, const char *out_path) {
    FILE *fp = fopen(in_path, "r");
    if (!fp) { fprintf(stderr, "harness: cannot read %s\n", in_path); return 2; }
    SSERIES *head = NULL, *curr = NULL;
    char *line = NULL, *token = NULL;
    size_t len = 0;
    while (getline(&line, &len, fp) != -1) {
        get_token(line, &token); if (token == NULL) continue;
        if (strcmp(token, "SERIES") == 0) {
            get_next_token(&token);
            if (token && strcmp(token, "BC") == 0)
                sseries_read_allocate(fp, &head, &curr, TIME_SERIES, &token, UNSET_INT);
            else { fprintf(stderr, "harness: series type not handled\n"); fclose(fp); return 2; }
        }
    }
    fclose(fp);
    int n = 0, tot = 0;
    for (SSERIES *p = head; p; p = p->next) { n++; tot += p->size; }
    int *ids = malloc(sizeof(int) * (n + 1)), *sizes = malloc(sizeof(int) * (n + 1));
    double *times = malloc(sizeof(double) * (tot + 1)), *vals = malloc(sizeof(double) * (tot + 1));
    int k = 0, e = 0;
    for (SSERIES *p = head; p; p = p->next, k++) {
        ids[k] = p->id; sizes[k] = p->size;
        for (int j = 0; j < p->size; j++, e++) { times[e] = p->entry[j].time; vals[e] = p->entry[j].value[0]; }
    }
    g_out = fopen(out_path, "wb");
    if (!g_out) { fprintf(stderr, "harness: cannot write %s\n", out_path); return 2; }
    out_rec("ids", 'i', ids, n);
    out_rec("sizes", 'i', sizes, n);
    out_rec("times", 'd', times, tot);
    out_rec("values", 'd', vals, tot);
    fclose(g_out);
    free(ids); free(sizes); free(times); free(vals);
    return 0;
}

int main(int argc, char **argv) {
    if (argc >= 4 && strcmp(argv[1], "geo") == 0) {
        if (getenv("HARNESS_VERBOSE") == NULL) { if (!freopen("/dev/null", "w", stdout)) return 2; }
        debug_initialize();
        sadh_def_init();
        g_out = fopen(argv[3], "wb");
        if (!g_out) { fprintf(stderr, "harness: cannot write %s\n", argv[3]); return 2; }
        mode_geo(argv);
        fclose(g_out);
        return 0;
    }
    if (argc >= 4 && strcmp(argv[1], "params") == 0) {
        if (getenv("HARNESS_VERBOSE") == NULL) { if (!freopen("/dev/null", "w", stdout)) return 2; }
        debug_initialize();
        sadh_def_init();
        return mode_params(argv[2], argv[3]);
    }
    if (argc >= 4 && strcmp(argv[1], "bcx") == 0) {
        if (getenv("HARNESS_VERBOSE") == NULL) { if (!freopen("/dev/null", "w", stdout)) return 2; }
        debug_initialize();
        sadh_def_init();
        return mode_bcx(argv[2], argv[3]);
    }
    if (argc >= 4 && strcmp(argv[1], "rect") == 0) {
        if (getenv("HARNESS_VERBOSE") == NULL) { if (!freopen("/dev/null", "w", stdout)) return 2; }
        debug_initialize();
        sadh_def_init();
        g_out = fopen(argv[3], "wb");
        mode_rect(argc, argv);
        fclose(g_out);
        return 0;
    }
    if (argc < 4) { fprintf(stderr, "usage: %s <dump|run|time> case.bin out.bin [every|reps]\n", argv[0]); return 2; }
    /* the reference prints progress from its init path; keep our stdout clean */
    if (getenv("HARNESS_VERBOSE") == NULL) { if (!freopen("/dev/null", "w", stdout)) return 2; }
#ifndef _MESSG
    debug_initialize();
#endif
    sadh_def_init();
    set_function_pointers(adh_time_stepper);
    CASE c = read_case(argv[2]);
    build_model(&c);
    g_out = fopen(argv[3], "wb");
    if (!g_out) { fprintf(stderr, "harness: cannot write %s\n", argv[3]); return 2; }
#ifndef SW2_REFGLUE
    if (strcmp(argv[1], "dump") == 0) mode_dump(&c);
    else
#endif
    if (strcmp(argv[1], "loop") == 0) mode_loop(&c, fe_newton);
#ifdef SW2_REFGLUE
    else if (strcmp(argv[1], "loop_gpu") == 0) { mode_loop(&c, fe_newton_gpu); sw2_gpu_detach_all(); }
#endif
    else if (strcmp(argv[1], "run") == 0) mode_run(&c, argc > 4 ? atoi(argv[4]) : 1);
    else if (strcmp(argv[1], "time") == 0) mode_time(&c, argc > 4 ? atoi(argv[4]) : 1);
    else if (strcmp(argv[1], "mass") == 0) mode_mass(&c);
    else if (strcmp(argv[1], "init") == 0 && argc > 4) mode_init(argv[4]);
    else { fprintf(stderr, "harness: unknown mode %s\n", argv[1]); return 2; }
    fclose(g_out);
    return 0;
}
