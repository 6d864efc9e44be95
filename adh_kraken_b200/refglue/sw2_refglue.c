/*
 * sw2_refglue.c -- assemble_residual, assemble_jacobian and an fe_newton-compatible
 * stepper of the reference, on the B200 C ABI (include/adh_sw2_gpu.h).  Declarations
 * and scope in sw2_refglue.h.
 */
#include "adh.h"
#include "sw2_refglue.h"

#ifdef _MESSG
#error "sw2_refglue.c is the serial (one GPU) path: build the reference without _MESSG"
#endif

#define SW2_GLUE_MAX_MODELS 16

static struct {
    SMODEL_SUPER *sm;
    sw2g_model *g;
    int ivx, ivy;        /* velocity series of the NB VEL strings (-1: none) */
    int has_depth;       /* a DEPTH string exists: series 0 is read (sw2_bc_h.c:156) */
} g_tab[SW2_GLUE_MAX_MODELS];
static int g_nmodels = 0;
static sw2g_newton_opts g_opts;
static int g_opts_set = 0;
static sw2g_newton_stats g_last;

static void glue_fail(const char *where, int rc) {
    char msg[512];
    snprintf(msg, sizeof msg, "%s: sw2g error %d: %s\n", where, rc, sw2g_last_error());
    tl_error(msg);
}

static int glue_index(SMODEL_SUPER *sm) {
    for (int i = 0; i < g_nmodels; i++)
        if (g_tab[i].sm == sm) return i;
    return -1;
}

int sw2_gpu_attach(SMODEL_SUPER *sm) {
    if (glue_index(sm) >= 0) return SW2G_OK;
    if (g_nmodels == SW2_GLUE_MAX_MODELS) return SW2G_ERR_ARG;
    SGRID *g = sm->grid;
    if (sm->nsubsteps != 1 || g->nelems3d != 0) return SW2G_ERR_ARG;
    const int V = g->nnodes, T = g->nelems2d, S = g->nelems1d;
    for (int e = 0; e < T; e++)
        if (g->elem2d[e].nnodes != 3 || sm->mat_physics_elem[sm->elem2d_physics_mat[e]].pde[0].resid != fe_sw2_body_resid)
            return SW2G_ERR_ARG;
    double *xyz = (double *)malloc(sizeof(double) * 3 * (size_t)V);
    int *tri = (int *)malloc(sizeof(int) * 3 * (size_t)T);
    int *seg = (int *)malloc(sizeof(int) * 2 * (size_t)(S + 1));
    int *kind = (int *)malloc(sizeof(int) * (size_t)(S + 1));
    int ivx = -1, ivy = -1, has_depth = 0, rc = SW2G_OK;
    for (int i = 0; i < V; i++) {
        xyz[3 * i] = g->node[i].x; xyz[3 * i + 1] = g->node[i].y; xyz[3 * i + 2] = g->node[i].z;
    }
    for (int e = 0; e < T; e++)
        for (int a = 0; a < 3; a++) tri[3 * e + a] = g->elem2d[e].nodes[a];
    for (int s = 0; s < S && rc == SW2G_OK; s++) {
        const int mat = sm->elem1d_physics_mat[s];
        seg[2 * s] = g->elem1d[s].nodes[0]; seg[2 * s + 1] = g->elem1d[s].nodes[1];
        if (sm->mat_physics_elem[mat].pde[0].resid == fe_sw2_bc_h) {
            kind[s] = 1; has_depth = 1;
        } else if (sm->mat_physics_elem[mat].pde[0].resid == fe_sw2_bc_vel) {
            /* fe_sw2_bc_vel reads its series from str_values[mat].ol_flow (sw2_bc_vel.c:147-150) */
            const int x = sm->str_values[mat].ol_flow.ivx, y = sm->str_values[mat].ol_flow.ivy;
            if ((ivx >= 0 && x != ivx) || (ivy >= 0 && y != ivy)) rc = SW2G_ERR_ARG;   /* one pair only */
            ivx = x; ivy = y; kind[s] = 0;
        } else {
            rc = SW2G_ERR_ARG;
        }
    }
    sw2g_model *m = NULL;
    if (rc == SW2G_OK) {
        sw2g_mesh mesh = {V, T, S, xyz, tri, seg, kind, sm->lin_sys->indptr_diag, sm->lin_sys->cols_diag, sm->gravity};
        rc = sw2g_create(&mesh, NULL, &m);
    }
    free(xyz); free(tri); free(seg); free(kind);
    if (rc != SW2G_OK) return rc;
    g_tab[g_nmodels].sm = sm; g_tab[g_nmodels].g = m;
    g_tab[g_nmodels].ivx = ivx; g_tab[g_nmodels].ivy = ivy; g_tab[g_nmodels].has_depth = has_depth;
    g_nmodels++;
    return SW2G_OK;
}

sw2g_model *sw2_gpu_model(SMODEL_SUPER *sm) {
    const int i = glue_index(sm);
    return i < 0 ? NULL : g_tab[i].g;
}

void sw2_gpu_detach_all(void) {
    for (int i = 0; i < g_nmodels; i++) sw2g_destroy(g_tab[i].g);
    g_nmodels = 0;
}

void sw2_gpu_set_newton_opts(const sw2g_newton_opts *opts) {
    if (opts) { g_opts = *opts; g_opts_set = 1; } else g_opts_set = 0;
}

const sw2g_newton_stats *sw2_gpu_last_stats(void) { return &g_last; }

/* the model of sm, with the scalars the element plugins read from sm for this step:
 * dt and tau_temporal (sw2_body_resid.c:81-82) and the step-averaged series values
 * (sw2_bc_h.c:156, sw2_bc_vel.c:147-150) */
static sw2g_model *glue_model_for_step(SMODEL_SUPER *sm, const char *who) {
    int rc = sw2_gpu_attach(sm);
    if (rc != SW2G_OK) glue_fail(who, rc);
    const int i = glue_index(sm);
    const double depth = g_tab[i].has_depth ? sseries_get_value(0, sm->series_head, 0) : 0.0;
    const double vx = g_tab[i].ivx >= 0 ? sseries_get_value(g_tab[i].ivx, sm->series_head, 0) : 0.0;
    const double vy = g_tab[i].ivy >= 0 ? sseries_get_value(g_tab[i].ivy, sm->series_head, 0) : 0.0;
    rc = sw2g_set_step(g_tab[i].g, sm->ts->dt / sm->nsubsteps, sm->ts->tau_temporal, depth, vx, vy);
    if (rc != SW2G_OK) glue_fail(who, rc);
    return g_tab[i].g;
}

void assemble_residual(SMODEL_SUPER *sm, SGRID *grid) {
    (void)grid;   /* the device model holds sm->grid */
    sw2g_model *m = glue_model_for_step(sm, "assemble_residual");
    const int rc = sw2g_assemble_residual_wd(m, sm->sol, sm->sol_old, sm->sol_older,
                                             sm->dvars.elem_flags[adh_def._WDFLAG], sm->lin_sys->residual);
    if (rc != SW2G_OK) glue_fail("assemble_residual", rc);
}

void assemble_jacobian(SMODEL_SUPER *sm) {
    sw2g_model *m = glue_model_for_step(sm, "assemble_jacobian");
    const int rc = sw2g_assemble_jacobian_wd(m, sm->sol, sm->sol_old, sm->sol_older,
                                             sm->dvars.elem_flags[adh_def._WDFLAG], sm->lin_sys->vals_diag);
    if (rc != SW2G_OK) glue_fail("assemble_jacobian", rc);
}

/* fe_newton (src/newton/fe_newton.c:44-915) on the device: TRUE when the step
 * converged; on failure the state is back at the start of the step and dt is scaled
 * by tc_scale, as fe_newton leaves them (fe_newton.c:887-899). */
int fe_newton_gpu(SMODEL_SUPER *sm) {
    sw2g_model *m = glue_model_for_step(sm, "fe_newton_gpu");
    sw2g_newton_opts o;
    if (g_opts_set) o = g_opts; else sw2g_default_opts(&o);
    o.tol_nonlin = sm->tol_nonlin;
    o.inc_nonlin = sm->inc_nonlin;
    o.max_nonlin_it = sm->max_nonlin_it;
    o.max_linesearch_cuts = sm->max_nonlin_linesearch_cuts;
    memset(&g_last, 0, sizeof g_last);
    const int rc = sw2g_fe_newton(m, sm->sol, sm->sol_old, sm->sol_older, sm->bc_mask, sm->dirichlet_data, &o, &g_last);
    if (rc == SW2G_ERR_NONFINITE) {   /* the reference exits on a NaN residual (newton_tools.c:344-349) */
        glue_fail("fe_newton_gpu", rc);
    } else if (rc != SW2G_OK) {
        glue_fail("fe_newton_gpu", rc);
    }
    sm->it_count_nonlin += g_last.newton_its;
    if (!g_last.success) {
        tc_scale(&sm->ts->dt);
        sm->it_count_nonlin_failed += g_last.newton_its;
        return FALSE;
    }
    return TRUE;
}
