/*
 * CPU restatement of the reference's SW2 implicit time-step hot path.
 * TEST INFRASTRUCTURE ONLY -- see sw2_oracle.h.  Built with -ffp-contract=off.
 *
 * Operation order follows the reference expression by expression (C evaluates
 * a*b*c as (a*b)*c and a+b+c as (a+b)+c); integer literals such as the 3 in
 * 3*h1*h1 are converted to double exactly as the reference's C does.
 */
#include "sw2_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#define SMALL DBL_EPSILON            /* src/include/define.h:31 */
#define NOT_QUITE_SMALL FLT_EPSILON  /* src/include/define.h:32 */
#define one_2 0.5e+0                 /* src/include/define.h:37-52 */
#define one_3 0.333333333333333333333333
#define one_6 0.166666666666666666666667
#define one_12 0.083333333333333333333333
#define one_30 0.033333333333333333333333
#define one_60 0.016666666666666666666667

static inline double dmax(double a, double b) { return a > b ? a : b; } /* MAX, macro.h:845 */

typedef struct { double x, y; } v2;

/* ------------------------------------------------------------------ geometry */
void sw2o_geometry(int nnodes, int ntri, int nseg, const double *xyz, const int *tri, const int *seg,
                   double *tri_djac, double *tri_grad, double *seg_djac, double *seg_nrml) {
    (void)nnodes;
    for (int e = 0; e < ntri; e++) {
        const double *p1 = xyz + 3 * tri[3 * e], *p2 = xyz + 3 * tri[3 * e + 1], *p3 = xyz + 3 * tri[3 * e + 2];
        double s1x = p2[0] - p1[0], s1y = p2[1] - p1[1];
        double s2x = p3[0] - p1[0], s2y = p3[1] - p1[1];
        double djac = (s1x * s2y) - (s2x * s1y);            /* selem_2d.c:326 */
        double inv = 1. / djac;                              /* svect2d_scale_replace_array(.., 1./djac) */
        double *g = tri_grad + 6 * e;
        g[0] = (s1y - s2y) * inv; g[1] = (s2x - s1x) * inv;
        g[2] = s2y * inv;         g[3] = -s2x * inv;
        g[4] = -s1y * inv;        g[5] = s1x * inv;
        tri_djac[e] = djac * (1.0 / 2.0);                    /* SCALE_FOR_MASTER_TRI_VOLUME */
    }
    for (int k = 0; k < nseg; k++) {
        const double *a = xyz + 3 * seg[2 * k], *b = xyz + 3 * seg[2 * k + 1];
        double d = sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1])); /* DIST_2D */
        seg_djac[k] = d;
        seg_nrml[2 * k] = (b[1] - a[1]) / d;
        seg_nrml[2 * k + 1] = -(b[0] - a[0]) / d;
    }
}

/* ------------------------------------------------------------------ sparsity */
static int cmp_int(const void *a, const void *b) { int x = *(const int *)a, y = *(const int *)b; return (x > y) - (x < y); }

/* node adjacency (each node with itself) from triangles and segments, sorted unique */
static int *node_adj(int nnodes, int ntri, int nseg, const int *tri, const int *seg, int **adj_ptr_out) {
    int *cnt = calloc((size_t)nnodes + 1, sizeof(int));
    for (int e = 0; e < ntri; e++) for (int a = 0; a < 3; a++) cnt[tri[3 * e + a]] += 3;
    for (int e = 0; e < nseg; e++) for (int a = 0; a < 2; a++) cnt[seg[2 * e + a]] += 2;
    int *ptr = malloc(sizeof(int) * ((size_t)nnodes + 1));
    ptr[0] = 0;
    for (int i = 0; i < nnodes; i++) ptr[i + 1] = ptr[i] + cnt[i];
    int *buf = malloc(sizeof(int) * ((size_t)ptr[nnodes] + 1));
    memset(cnt, 0, sizeof(int) * (size_t)nnodes);
    for (int e = 0; e < ntri; e++) for (int a = 0; a < 3; a++) { int i = tri[3 * e + a]; for (int b = 0; b < 3; b++) buf[ptr[i] + cnt[i]++] = tri[3 * e + b]; }
    for (int e = 0; e < nseg; e++) for (int a = 0; a < 2; a++) { int i = seg[2 * e + a]; for (int b = 0; b < 2; b++) buf[ptr[i] + cnt[i]++] = seg[2 * e + b]; }
    int *uptr = malloc(sizeof(int) * ((size_t)nnodes + 1));
    uptr[0] = 0;
    int w = 0;
    for (int i = 0; i < nnodes; i++) {
        int *row = buf + ptr[i]; int n = ptr[i + 1] - ptr[i];
        qsort(row, (size_t)n, sizeof(int), cmp_int);
        int start = w;
        for (int k = 0; k < n; k++) if (k == 0 || row[k] != row[k - 1]) buf[w++] = row[k];
        uptr[i + 1] = uptr[i] + (w - start);
    }
    free(cnt); free(ptr);
    *adj_ptr_out = uptr;
    return buf;
}

int sw2o_sparsity_nnz(int nnodes, int ntri, int nseg, const int *tri, const int *seg) {
    int *ap; int *adj = node_adj(nnodes, ntri, nseg, tri, seg, &ap);
    int nnz = 9 * ap[nnodes];
    free(ap); free(adj);
    return nnz;
}

/* Each row of dof (node, var) holds the columns 3*b + k of every neighbour b
 * (node itself included), k = 0..2, sorted: the sorted-unique column lists of
 * slin_sys_init_sparsity_mono.c:335-436 for an all-SW2 mesh with dof = 3*node+var
 * (sivar_position.c:74-79). */
void sw2o_sparsity(int nnodes, int ntri, int nseg, const int *tri, const int *seg, int *indptr, int *cols) {
    int *ap; int *adj = node_adj(nnodes, ntri, nseg, tri, seg, &ap);
    int w = 0;
    indptr[0] = 0;
    for (int i = 0; i < nnodes; i++) {
        for (int v = 0; v < 3; v++) {
            for (int k = ap[i]; k < ap[i + 1]; k++)
                for (int c = 0; c < 3; c++) cols[w++] = 3 * adj[k] + c;
            indptr[3 * i + v + 1] = w;
        }
    }
    free(ap); free(adj);
}

/* ------------------------------------------------------------------ wet/dry flags */
void sw2o_wd_flags(sw2o_model *m, const double *sol, const double *sol_old) {
    int *tmp = calloc((size_t)m->nnodes, sizeof(int));
    for (int e = 0; e < m->ntri; e++) {
        int wet = 0;
        for (int a = 0; a < 3; a++) if (sol[m->tri[3 * e + a] * 3] > 0.0) wet++;
        if (wet != 3) for (int a = 0; a < 3; a++) tmp[m->tri[3 * e + a]] = 1;
    }
    for (int e = 0; e < m->ntri; e++) {
        const int *n = m->tri + 3 * e;
        int f = 0;
        for (int a = 0; a < 3; a++) if (tmp[n[a]] != 0) f = 1;
        if (sol[n[0] * 3] < 0 && sol[n[1] * 3] < 0 && sol[n[2] * 3] < 0 &&
            sol_old[n[0] * 3] < 0 && sol_old[n[1] * 3] < 0 && sol_old[n[2] * 3] < 0) f = 2;
        m->wd_flag[e] = f;
    }
    free(tmp);
}

/* ------------------------------------------------------------------ triangle integrals
 * src/fe/fe_integrals_2d.c */
static inline void tri_phi_f(double djac, double c, const double *f, double *I) {          /* :25 */
    double f_sum = f[0] + f[1] + f[2];
    double t1 = djac * c * one_12;
    I[0] += t1 * (f_sum + f[0]); I[1] += t1 * (f_sum + f[1]); I[2] += t1 * (f_sum + f[2]);
}
static inline void tri_phi_f_lump(double djac, double c, const double *f, double *I) {     /* :33 */
    double t1 = djac * c * one_3;
    I[0] += t1 * f[0]; I[1] += t1 * f[1]; I[2] += t1 * f[2];
}
static inline void tri_gradPhi_dot_f_v(const v2 *g, double djac, double c, const double *f, const v2 *v, double *I) {
    double p1 = (2 * f[0] + f[1] + f[2]);
    double p2 = (f[0] + 2 * f[1] + f[2]);
    double p3 = (f[0] + f[1] + 2 * f[2]);
    double tx = (p1 * v[0].x + p2 * v[1].x + p3 * v[2].x);
    double ty = (p1 * v[0].y + p2 * v[1].y + p3 * v[2].y);
    double con = djac * one_12 * c;
    for (int i = 0; i < 3; i++) I[i] += con * (g[i].x * tx + g[i].y * ty);
}
static inline void tri_dphi_f_g_h(const v2 *g, double djac, double c, const double *f, const double *gg,
                                  const double *h, double *Ix, double *Iy) {
    double ff1 = (3 * f[0] + f[1] + f[2]), ff2 = (2 * f[0] + 2 * f[1] + f[2]), ff3 = (2 * f[0] + f[1] + 2 * f[2]);
    double ff4 = (f[0] + 3 * f[1] + f[2]), ff5 = (f[0] + 2 * f[1] + 2 * f[2]), ff6 = (f[0] + f[1] + 3 * f[2]);
    double gg1 = (2 * ff1 * gg[0] + ff2 * gg[1] + ff3 * gg[2]);
    double gg2 = (ff2 * gg[0] + 2 * ff4 * gg[1] + ff5 * gg[2]);
    double gg3 = (ff3 * gg[0] + ff5 * gg[1] + 2 * ff6 * gg[2]);
    double con = djac * one_60 * c * (gg1 * h[0] + gg2 * h[1] + gg3 * h[2]);
    for (int i = 0; i < 3; i++) Ix[i] += con * g[i].x;
    for (int i = 0; i < 3; i++) Iy[i] += con * g[i].y;
}
static inline void tri_dphi_f_f_h(const v2 *g, double djac, double c, const double *f, const double *h,
                                  double *Ix, double *Iy) {
    double f1_2 = f[0] * f[0], f2_2 = f[1] * f[1], f3_2 = f[2] * f[2];
    double p1 = (3 * f1_2 + 2 * f[0] * f[1] + f2_2 + (2 * f[0] + f[1]) * f[2] + f3_2);
    double p2 = (f1_2 + 2 * f[0] * f[1] + 3 * f2_2 + (f[0] + 2 * f[1]) * f[2] + f3_2);
    double p3 = (f1_2 + f[0] * f[1] + f2_2 + 2 * (f[0] + f[1]) * f[2] + 3 * f3_2);
    double con = djac * one_30 * c * (p1 * h[0] + p2 * h[1] + p3 * h[2]);
    if (Ix) for (int i = 0; i < 3; i++) Ix[i] += con * g[i].x;
    if (Iy) for (int i = 0; i < 3; i++) Iy[i] += con * g[i].y;
}
static inline void tri_dphi_f_f(const v2 *g, double djac, double c, const double *f, double *Ix, double *Iy) {
    double int_f_f = (c * one_6 * djac * (f[0] * f[0] + f[0] * f[1] + f[1] * f[1] + f[0] * f[2] + f[1] * f[2] + f[2] * f[2]));
    for (int i = 0; i < 3; i++) Ix[i] += g[i].x * int_f_f;
    for (int i = 0; i < 3; i++) Iy[i] += g[i].y * int_f_f;
}
static inline void tri_phi_h_df(double djac, double c, const double *h, v2 df, double *Ix, double *Iy) {
    double con, sum_h = h[0] + h[1] + h[2];
    con = djac * one_12 * c * df.x;
    for (int i = 0; i < 3; i++) Ix[i] += con * (sum_h + h[i]);
    con = djac * one_12 * c * df.y;
    for (int i = 0; i < 3; i++) Iy[i] += con * (sum_h + h[i]);
}
/* src/fe/fe_integrals_1d.c */
static inline void line_phi_h_h(double djac, double c, double h1, double h2, double *I) {    /* :16 */
    double t1 = djac * one_12 * c;
    I[0] += t1 * (3 * h1 * h1 + 2 * h1 * h2 + h2 * h2);
    I[1] += t1 * (h1 * h1 + 2 * h1 * h2 + 3 * h2 * h2);
}
static inline void line_phi_h_v_dot_n(double djac, double c, const double *h, const v2 *v, v2 n, double *I) {
    double t1 = djac * one_12 * c;
    I[0] += t1 * (n.x * ((3 * h[0] + h[1]) * v[0].x + (h[0] + h[1]) * v[1].x) + n.y * ((3 * h[0] + h[1]) * v[0].y + (h[0] + h[1]) * v[1].y));
    I[1] += t1 * (n.x * ((h[0] + h[1]) * v[0].x + (h[0] + 3 * h[1]) * v[1].x) + n.y * ((h[0] + h[1]) * v[0].y + (h[0] + 3 * h[1]) * v[1].y));
}
static inline void line_phi_f_g_h(double djac, double c, double f1, double f2, double g1, double g2,
                                  double h1, double h2, double *I) {
    double t1 = one_60 * djac * c;
    I[0] += t1 * ((3 * (4 * f1 + f2) * g1 + (3 * f1 + 2 * f2) * g2) * h1 + ((3 * f1 + 2 * f2) * g1 + (2 * f1 + 3 * f2) * g2) * h2);
    I[1] += t1 * (((3 * f1 + 2 * f2) * g1 + (2 * f1 + 3 * f2) * g2) * h1 + ((2 * f1 + 3 * f2) * g1 + 3 * (f1 + 4 * f2) * g2) * h2);
}

/* ------------------------------------------------------------------ wet/dry integrands
 * src/fe/fe_wet_dry_integrations.c.  One signature, as the reference's function pointer. */
typedef struct {
    const v2 *x;          /* 3 vertices (only x,y used) */
    const double *h;
    const v2 *grad;       /* may be NULL */
    const v2 *v;          /* may be NULL */
    const v2 *vwd;        /* may be NULL */
    const double *fwd;    /* may be NULL */
    double djac;
    double vars0, vars1;
} wd_args;
typedef void (*wd_func)(const wd_args *a, double *rhs);

static void wd_convection(const wd_args *a, double *rhs) {           /* :45 */
    double c = a->vars1; c *= a->vars0;
    double rc[3] = {0, 0, 0}, rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
    double uu[3], vv[3];
    for (int i = 0; i < 3; i++) { uu[i] = a->vwd[i].x; vv[i] = a->vwd[i].y; }
    tri_gradPhi_dot_f_v(a->grad, a->djac, c, a->h, a->vwd, rc);
    tri_dphi_f_g_h(a->grad, a->djac, c, uu, vv, a->h, ry, rx);
    tri_dphi_f_f_h(a->grad, a->djac, c, uu, a->h, rx, NULL);
    tri_dphi_f_f_h(a->grad, a->djac, c, vv, a->h, NULL, ry);
    for (int i = 0; i < 3; i++) { rhs[3 * i] += rc[i]; rhs[3 * i + 1] += rx[i]; rhs[3 * i + 2] += ry[i]; }
}
static void wd_continuity_temporal(const wd_args *a, double *rhs) {  /* :92 */
    double rc[3] = {0, 0, 0};
    tri_phi_f(a->djac, a->vars1, a->h, rc);
    for (int i = 0; i < 3; i++) rhs[3 * i] += rc[i];
}
static void wd_pressure(const wd_args *a, double *rhs) {             /* :112 */
    double rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
    tri_dphi_f_f(a->grad, a->djac, a->vars1, a->h, rx, ry);
    for (int i = 0; i < 3; i++) { rhs[3 * i + 1] += rx[i]; rhs[3 * i + 2] += ry[i]; }
}
static void wd_bodyForce(const wd_args *a, double *rhs) {            /* :131 */
    double rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
    tri_phi_h_df(a->djac, a->vars1, a->h, *a->v, rx, ry);
    for (int i = 0; i < 3; i++) { rhs[3 * i + 1] += rx[i]; rhs[3 * i + 2] += ry[i]; }
}
static void wd_boundaryPressure(const wd_args *a, double *rhs) {     /* :146 */
    static const int n1s[3] = {0, 1, 2}, n2s[3] = {1, 2, 0};
    for (int e = 0; e < 3; e++) {
        int n1 = n1s[e], n2 = n2s[e];
        double delx = a->x[n1].x - a->x[n2].x;
        double dely = a->x[n2].y - a->x[n1].y;
        double r[2] = {0., 0.};
        line_phi_h_h(1., a->vars1, a->h[n1], a->h[n2], r);
        rhs[n1 * 3 + 1] += dely * r[0];
        rhs[n2 * 3 + 1] += dely * r[1];
        rhs[n1 * 3 + 2] += delx * r[0];
        rhs[n2 * 3 + 2] += delx * r[1];
    }
}
static void wd_integrate_f(const wd_args *a, double *rhs) {          /* :250 */
    double t1 = (a->h[0] + a->h[1] + a->h[2]) / 3.0, t2 = 0.0, t3 = 0.0;
    if (a->vwd) {
        t2 = (a->vwd[0].x + a->vwd[1].x + a->vwd[2].x) / 3.0;
        t3 = (a->vwd[0].y + a->vwd[1].y + a->vwd[2].y) / 3.0;
    }
    rhs[0] += a->djac * t1; rhs[1] += a->djac * t2; rhs[2] += a->djac * t3;
}
static void wd_gls_convection(const wd_args *a, double *rhs) {       /* :270 */
    const double *f = a->fwd; const v2 *w = a->vwd; const v2 *g = a->grad;
    double dt = a->vars0, c = a->vars1;
    double h_avg = one_3 * (f[0] + f[1] + f[2]);
    double u_avg = one_3 * (w[0].x + w[1].x + w[2].x);
    double v_avg = one_3 * (w[0].y + w[1].y + w[2].y);
    double dhdx = g[0].x * f[0] + g[1].x * f[1] + g[2].x * f[2];
    double dhdy = g[0].y * f[0] + g[1].y * f[1] + g[2].y * f[2];
    double dudx = g[0].x * w[0].x + g[1].x * w[1].x + g[2].x * w[2].x;
    double dudy = g[0].y * w[0].x + g[1].y * w[1].x + g[2].y * w[2].x;
    double dvdx = g[0].x * w[0].y + g[1].x * w[1].y + g[2].x * w[2].y;
    double dvdy = g[0].y * w[0].y + g[1].y * w[1].y + g[2].y * w[2].y;
    rhs[0] += a->djac * dt * c * (u_avg * dhdx + h_avg * dudx + v_avg * dhdy + h_avg * dvdy);
    rhs[1] += a->djac * dt * c * (u_avg * dudx + v_avg * dudy);
    rhs[2] += a->djac * dt * c * (u_avg * dvdx + v_avg * dvdy);
}

/* ------------------------------------------------------------------ wet/dry wrapper
 * fe_sw2_wet_dry_wrapper, src/fe/fe_wet_dry_wrapper.c:104-304 */
static double wd_wrapper(double *elem_rhs, const v2 *x, const double *h, const v2 *grad, const v2 *v,
                         const v2 *vwd, const double *fwd, double djac, int redistribute,
                         double vars0, double vars1, wd_func fn) {
    int passcode = 0, total = 0;
    for (int i = 0; i < 3; i++) { int d = (h[i] <= 0.0) ? 1 : 0; total += d; passcode += (d << i); }
    wd_args a = {x, h, grad, v, vwd, fwd, djac, vars0, vars1};
    if (total == 3) return 0;
    if (total == 0) { fn(&a, elem_rhs); return 1.0; }
    if (total == 1) fn(&a, elem_rhs);
    else passcode = 7 - passcode;
    int only = passcode / 2;
    double new_h[3] = {0.0, 0.0, 0.0}, new_f[3] = {0, 0, 0};
    v2 new_x[3], new_v[3] = {{0, 0}, {0, 0}, {0, 0}};
    for (int i = 0; i < 3; i++) {
        if (i != only) {
            double xsi = h[i] / (h[i] - h[only]);
            new_x[i].x = x[i].x + xsi * (x[only].x - x[i].x);         /* FIXED_POS, macro.h:756 */
            new_x[i].y = x[i].y + xsi * (x[only].y - x[i].y);
            if (vwd) {
                new_v[i].x = vwd[i].x + xsi * (vwd[only].x - vwd[i].x);
                new_v[i].y = vwd[i].y + xsi * (vwd[only].y - vwd[i].y);
            }
            if (fwd) new_f[i] = fwd[i] + xsi * (fwd[only] - fwd[i]);
        } else {
            new_x[i] = x[i]; new_h[i] = h[i];
            if (fwd) new_f[i] = fwd[i];
            if (vwd) new_v[i] = vwd[i];
        }
    }
    double elem_djac = djac;
    {   /* TRI_AREA, macro.h:771 */
        double ax = new_x[1].x - new_x[0].x, ay = new_x[1].y - new_x[0].y;
        double bx = new_x[2].x - new_x[0].x, by = new_x[2].y - new_x[0].y;
        djac = (ax * by - ay * bx) / 2.0;
    }
    if (djac / elem_djac < SMALL) return (double)(total % 2);
    v2 ng[3];
    if (grad) {  /* GRAD_SHAPE, macro.h:778 */
        ng[0].x = 0.5 * (new_x[1].y - new_x[2].y) / djac;
        ng[1].x = 0.5 * (new_x[2].y - new_x[0].y) / djac;
        ng[2].x = 0.5 * (new_x[0].y - new_x[1].y) / djac;
        ng[0].y = 0.5 * (new_x[2].x - new_x[1].x) / djac;
        ng[1].y = 0.5 * (new_x[0].x - new_x[2].x) / djac;
        ng[2].y = 0.5 * (new_x[1].x - new_x[0].x) / djac;
    }
    double nr[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    wd_args b = {new_x, new_h, grad ? ng : NULL, v, vwd ? new_v : NULL, fwd ? new_f : NULL, djac, vars0, vars1};
    fn(&b, nr);
    double factor = (total >> 1) - (total % 2);
    if (redistribute) {  /* RE_DISTRIBUTE, macro.h:788 */
        for (int i = 0; i < 3; i++) {
            if (i == only) continue;
            double v0x = new_x[i].x - x[only].x, v0y = new_x[i].y - x[only].y;
            double v1x = x[i].x - x[only].x, v1y = x[i].y - x[only].y;
            double l0 = v0x * v0x + v0y * v0y, l1 = v1x * v1x + v1y * v1y;
            double xsi = sqrt(l0 / l1);
            for (int k = 0; k < 3; k++) nr[only * 3 + k] += (1.0 - xsi) * nr[i * 3 + k];
            for (int k = 0; k < 3; k++) nr[i * 3 + k] *= xsi;
        }
    }
    for (int i = 0; i < 9; i++) elem_rhs[i] += factor * nr[i];
    factor *= djac / elem_djac;
    return factor + ((factor < 0) ? 1.0 : 0.0);
}

/* fe_sw2_wet_dry_factor, fe_wet_dry_wrapper.c:29 */
static double wd_factor(const v2 *x, const double *h, double djac) {
    int passcode = 0, total = 0;
    for (int i = 0; i < 3; i++) { int d = (h[i] <= 0.0) ? 1 : 0; total += d; passcode += (d << i); }
    if (total == 3) return 0.0;
    if (total == 0) return 1.0;
    if (total != 1) passcode = 7 - passcode;
    int only = passcode / 2;
    v2 nx[3];
    for (int i = 0; i < 3; i++) {
        if (i != only) {
            double xsi = h[i] / (h[i] - h[only]);
            nx[i].x = x[i].x + xsi * (x[only].x - x[i].x);
            nx[i].y = x[i].y + xsi * (x[only].y - x[i].y);
        } else nx[i] = x[i];
    }
    double elem_djac = djac;
    double ax = nx[1].x - nx[0].x, ay = nx[1].y - nx[0].y, bx = nx[2].x - nx[0].x, by = nx[2].y - nx[0].y;
    djac = (ax * by - ay * bx) / 2.0;
    if (djac / elem_djac < SMALL) return (double)(total % 2);
    double factor = (total >> 1) - (total % 2);
    factor *= djac / elem_djac;
    return factor + ((factor < 0) ? 1.0 : 0.0);
}

/* fe_sw2_wd_average, src/fe/fe_wet_dry_integrations.c:40-59 */
static void wd_average(const v2 *x, const double *h, const v2 *v, double djac, double *havg, v2 *vavg) {
    double av[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double factor = wd_wrapper(av, x, h, NULL, NULL, v, h, djac, 0, 1., 1., wd_integrate_f);
    *havg = 0.;
    vavg->x = 0.; vavg->y = 0.;
    if (factor > 0.0) {
        double wet_area = djac * factor;
        *havg = av[0] / wet_area;
        vavg->x = av[1] / wet_area;
        vavg->y = av[2] / wet_area;
    }
}

/* fe_sw2_temporal, src/models/sw2/sw2_body_resid.c:1195 */
static void temporal(const v2 *x, double djac, const double *head, const v2 *vel, double wd_fac,
                     double dt_factor, double *elem_rhs, int wd_flag) {
    double con = dt_factor * wd_fac;
    double rhs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double uh[3], vh[3], rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
    for (int i = 0; i < 3; i++) {
        uh[i] = vel[i].x * dmax(head[i], 1e-6);
        vh[i] = vel[i].y * dmax(head[i], 1e-6);
    }
    wd_wrapper(rhs, x, head, NULL, NULL, NULL, NULL, djac, 1, 1.0, dt_factor, wd_continuity_temporal);
    tri_phi_f_lump(djac, con, uh, rx);
    tri_phi_f_lump(djac, con, vh, ry);
    for (int i = 0; i < 3; i++) {
        if (wd_flag != 2) elem_rhs[i * 3] += rhs[i * 3];
        elem_rhs[i * 3 + 1] += rx[i];
        elem_rhs[i * 3 + 2] += ry[i];
    }
}

/* ------------------------------------------------------------------ body residual
 * fe_sw2_body_resid, src/models/sw2/sw2_body_resid.c:44-1176 (triangles).  Terms
 * whose coefficients the reference hard-codes to zero (shock capturing :352-400,
 * eddy-viscosity diffusion :476-499, Coriolis :596-610, wind, rain) add a signed
 * zero to an entry that already holds the +0 it was initialised to or a non-zero
 * value, which leaves it unchanged for finite inputs; they are not evaluated. */
void sw2o_body_resid(const sw2o_model *m, const double *sol, const double *sol_old, const double *sol_older,
                     int e, double pert, int pnode, int pvar, int psign, double *elem_rhs) {
    const int *nd = m->tri + 3 * e;
    const double *gp = m->tri_grad + 6 * e;
    v2 g[3] = {{gp[0], gp[1]}, {gp[2], gp[3]}, {gp[4], gp[5]}};
    double djac = m->tri_djac[e];
    double dt = m->dt, alpha = m->tau_temporal, grav = m->gravity;
    int wd_flag = m->wd_flag[e];
    int pressure = 1;
    v2 x[3]; double z[3];
    double head[3], oh[3], ooh[3];
    v2 vel[3], ov[3], oov[3];
    for (int i = 0; i < 3; i++) {
        const double *p = m->xyz + 3 * nd[i];
        x[i].x = p[0]; x[i].y = p[1]; z[i] = p[2];
        head[i] = sol[3 * nd[i]]; vel[i].x = sol[3 * nd[i] + 1]; vel[i].y = sol[3 * nd[i] + 2];
        oh[i] = sol_old[3 * nd[i]]; ov[i].x = sol_old[3 * nd[i] + 1]; ov[i].y = sol_old[3 * nd[i] + 2];
        ooh[i] = sol_older[3 * nd[i]]; oov[i].x = sol_older[3 * nd[i] + 1]; oov[i].y = sol_older[3 * nd[i] + 2];
    }
    if (pvar == 0) head[pnode] += psign * pert;
    else if (pvar == 1) { vel[pnode].x += psign * pert; pressure = 0; }
    else if (pvar == 2) { vel[pnode].y += psign * pert; pressure = 0; }

    /* element averages and gradients (:185-201) */
    double h_avg = (head[0] + head[1] + head[2]) / 3.0;
    double u_avg = (vel[0].x + vel[1].x + vel[2].x) / 3.0;
    double v_avg = (vel[0].y + vel[1].y + vel[2].y) / 3.0;
    v2 grad_z = {0, 0}, grad_h = {0, 0};
    for (int i = 0; i < 3; i++) { grad_z.x += z[i] * g[i].x; grad_z.y += z[i] * g[i].y; }
    for (int i = 0; i < 3; i++) { grad_h.x += head[i] * g[i].x; grad_h.y += head[i] * g[i].y; }
    (void)u_avg; (void)v_avg;

    /* wet/dry averages and factors (:228-236) */
    double h_wd, oh_wd;
    v2 vel_wd, ovel_wd;
    wd_average(x, head, vel, djac, &h_wd, &vel_wd);
    wd_average(x, oh, ov, djac, &oh_wd, &ovel_wd);
    (void)h_avg; (void)oh_wd;
    double factor = wd_factor(x, head, djac);
    double factor_old = wd_factor(x, oh, djac);
    double factor_older = wd_factor(x, ooh, djac);
    double vel_wd_mag = sqrt(vel_wd.x * vel_wd.x + vel_wd.y * vel_wd.y);
    double roughness = 0.002;                                   /* :241 */

    /* advection (:413-434) */
    {
        double rhs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        wd_wrapper(rhs, x, head, g, vel, vel, NULL, djac, 1, dt, -1, wd_convection);
        for (int i = 0; i < 9; i++) elem_rhs[i] += rhs[i];
    }
    /* temporal (:456-463) */
    temporal(x, djac, head, vel, factor, (1. + alpha / 2.), elem_rhs, -3);
    temporal(x, djac, oh, ov, factor_old, (-1.) * (1. + alpha), elem_rhs, wd_flag);
    temporal(x, djac, ooh, oov, factor_older, (alpha / 2.), elem_rhs, wd_flag);
    /* friction (:520-539) */
    double resistance = roughness / (2.0 * grav);
    {
        double fx[3], fy[3], rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
        for (int i = 0; i < 3; i++) {
            double t = sqrt(vel[i].x * vel[i].x + vel[i].y * vel[i].y);
            fx[i] = vel[i].x * t; fy[i] = vel[i].y * t;
        }
        double t1 = dt * grav * resistance * factor;
        tri_phi_f(djac, t1, fx, rx);
        tri_phi_f(djac, t1, fy, ry);
        for (int i = 0; i < 3; i++) { elem_rhs[3 * i + 1] += rx[i]; elem_rhs[3 * i + 2] += ry[i]; }
    }
    v2 bed_stress = {resistance * vel_wd.x * vel_wd_mag, resistance * vel_wd.y * vel_wd_mag};
    /* pressure, bed slope, boundary pressure (:710-804) */
    if (pressure) {
        double rhs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double t1 = -one_2 * grav * dt;
        wd_wrapper(rhs, x, head, g, NULL, NULL, NULL, djac, 1, 1, t1, wd_pressure);
        for (int i = 0; i < 9; i++) elem_rhs[i] += rhs[i];
        double r2[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        t1 = grav * dt;
        wd_wrapper(r2, x, head, NULL, &grad_z, NULL, NULL, djac, 1, 1, t1, wd_bodyForce);
        for (int i = 0; i < 9; i++) elem_rhs[i] += r2[i];
        double r3[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        t1 = one_2 * dt * grav;
        wd_wrapper(r3, x, head, NULL, NULL, NULL, NULL, djac, 1, 1, t1, wd_boundaryPressure);
        for (int i = 0; i < 9; i++) elem_rhs[i] += r3[i];
    }
    /* SUPG (:921-1142) */
    if (fabs(h_wd) >= SMALL) {
        double g_factor = (1 + 0.0) * grav;
        double hden = dmax(h_wd, NOT_QUITE_SMALL);
        /* fe_get_supg_tau_sw (src/tools/get_supg_tau.c:43), le = sqrt(area) (:126).  The wet
         * fraction can round to a tiny negative value for an element whose wet part is almost
         * empty (depths ~1e-13); the reference then takes the square root of a negative number
         * and its residual turns NaN.  Clamping at zero changes nothing where the reference's
         * result is finite. */
        double le = sqrt(djac * (factor_old > 0.0 ? factor_old : 0.0));
        double cel2 = g_factor * hden;
        if (hden <= 0.0) cel2 = 0.;
        double sr = sqrt(vel_wd.x * vel_wd.x + vel_wd.y * vel_wd.y + cel2 + SMALL);
        double tau = 0.5 * le / sr;
        double dfdt[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, adv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        factor_old = wd_wrapper(dfdt, x, oh, NULL, NULL, ov, oh, djac, 0, 1, 1, wd_integrate_f);
        double dudt = -dfdt[1], dvdt = -dfdt[2], dhdt = -dfdt[0];
        for (int i = 0; i < 9; i++) dfdt[i] = 0;
        factor = wd_wrapper(dfdt, x, head, NULL, NULL, vel, head, djac, 0, 1, 1, wd_integrate_f);
        dudt += dfdt[1]; dvdt += dfdt[2]; dhdt += dfdt[0];
        factor = wd_wrapper(adv, x, head, g, NULL, vel, head, djac, 0, dt, 1, wd_gls_convection);
        double x_pressure = g_factor * (grad_h.x + grad_z.x) * dt * factor + 0.0 * dt * factor;
        double y_pressure = g_factor * (grad_h.y + grad_z.y) * dt * factor + 0.0 * dt * factor;
        double x_friction = grav * bed_stress.x * dt * factor;
        double y_friction = grav * bed_stress.y * dt * factor;
        double c_eq = dhdt + adv[0] + factor * 0.0 * djac * dt;
        double x_eq = dudt + adv[1] + (x_pressure + x_friction / hden) * djac + (0.0 - 0.0 / hden) * djac * factor * dt;
        double y_eq = dvdt + adv[2] + (y_pressure + y_friction / hden) * djac + (0.0 - 0.0 / hden) * djac * factor * dt;
        for (int i = 0; i < 3; i++) {
            double rc = (g[i].x * (tau * vel_wd.x * c_eq + tau * h_wd * x_eq) +
                         g[i].y * (tau * vel_wd.y * c_eq + tau * h_wd * y_eq));
            double rx = (g[i].x * (tau * g_factor * h_wd * c_eq + tau * vel_wd.x * h_wd * x_eq) +
                         g[i].y * (tau * vel_wd.y * h_wd * x_eq));
            double ry = (g[i].y * (tau * g_factor * h_wd * c_eq + tau * vel_wd.y * h_wd * y_eq) +
                         g[i].x * (tau * vel_wd.x * h_wd * y_eq));
            elem_rhs[3 * i] += rc; elem_rhs[3 * i + 1] += rx; elem_rhs[3 * i + 2] += ry;
        }
    }
}

/* ------------------------------------------------------------------ boundary residuals */
/* fe_sw2_1d_implicit_flow, src/fe/fe_sw2_boundary_integrals.c:125 */
static void implicit_flow(double *elem_rhs, v2 n, double djac, double dt, const v2 *v, const double *h) {
    double rc[2] = {0, 0}, rx[2] = {0, 0}, ry[2] = {0, 0};
    double u1 = v[0].x, u2 = v[1].x, v1 = v[0].y, v2_ = v[1].y, h1 = h[0], h2 = h[1];
    double ur1 = v[0].x, ur2 = v[1].x, vr1 = v[0].y, vr2 = v[1].y;
    double d0 = v[0].x * n.x + v[0].y * n.y, d1 = v[1].x * n.x + v[1].y * n.y;
    if (d0 < SMALL) { ur1 = 0.; vr1 = 0.; }
    if (d1 < SMALL) { ur2 = 0.; vr2 = 0.; }
    line_phi_h_v_dot_n(djac, 1., h, v, n, rc);
    line_phi_f_g_h(djac, n.x, ur1, ur2, u1, u2, h1, h2, rx);
    line_phi_f_g_h(djac, n.y, vr1, vr2, v1, v2_, h1, h2, ry);
    line_phi_f_g_h(djac, n.y, ur1, ur2, v1, v2_, h1, h2, rx);
    line_phi_f_g_h(djac, n.x, vr1, vr2, u1, u2, h1, h2, ry);
    for (int i = 0; i < 2; i++) {
        elem_rhs[i * 3] += dt * rc[i]; elem_rhs[i * 3 + 1] += dt * rx[i]; elem_rhs[i * 3 + 2] += dt * ry[i];
    }
}
/* fe_sw2_1d_pressure, fe_sw2_boundary_integrals.c:260 */
static void pressure_1d(double *elem_rhs, v2 n, double djac, double dt, const double *h, double g) {
    double r[2] = {0., 0.};
    line_phi_h_h(djac, 1., h[0], h[1], r);
    double t1 = dt * one_2 * g;
    for (int i = 0; i < 2; i++) { elem_rhs[i * 3 + 1] += t1 * n.x * r[i]; elem_rhs[i * 3 + 2] += t1 * n.y * r[i]; }
}
/* fr_bedshstr_drag_coef, src/friction/fr_bedshstr_drag_coef.c:18-42 */
static double bedshstr_drag_coef(double depth, double rh) {
    depth = depth > 1.E-8 ? depth : 1.E-8;
    rh = rh > 1.E-8 ? rh : 1.E-8;
    double depth_rh = (rh > 29.7 * depth) ? 1. / 29.7 : depth / rh;
    double bta = 29.7 * depth_rh;
    double phi = pow((.4 * bta) / ((bta + 1) * (log(bta + 1) - 1) + 1), 2.);
    return 2. * phi;
}
/* fe_sw2_get_roughness (src/models/sw2/sw2_get_roughness.c:24-49), string without vegetation or ice */
static double bc_roughness(double depth, double rh) { return rh > SMALL ? bedshstr_drag_coef(depth, rh) : 0.0; }
/* integrate_line_phi / integrate_line_phi_f, src/fe/fe_integrals_1d.c:54,67 */
static void line_phi(double djac, double c, double *q) { double t1 = one_2 * djac * c; q[0] += t1; q[1] += t1; }
static void line_phi_f(double djac, double c, const double *f, double *q) {
    double t1 = one_6 * djac * c;
    q[0] += t1 * (2 * f[0] + f[1]);
    q[1] += t1 * (f[0] + 2 * f[1]);
}
/* fe_sw2_1d_explicit_flow, src/fe/fe_sw2_boundary_integrals.c:56-82 */
static void explicit_flow(double *elem_rhs, v2 n, double djac, double dt, double flux, double h_avg,
                          const double *u, const double *v) {
    double rc[2] = {0., 0.}, rx[2] = {0., 0.}, ry[2] = {0., 0.};
    line_phi(djac, 1., rc);
    if (flux < 0) {
        double u_star = 0., v_star = 0.;
        if (h_avg > 0) { u_star = flux * n.x / h_avg; v_star = flux * n.y / h_avg; }
        line_phi(djac, u_star, rx);
        line_phi(djac, v_star, ry);
    } else {
        line_phi_f(djac, 1., u, rx);
        line_phi_f(djac, 1., v, ry);
    }
    double t1 = dt * flux;
    for (int i = 0; i < 2; i++) {
        elem_rhs[i * 3] += t1 * rc[i]; elem_rhs[i * 3 + 1] += t1 * rx[i]; elem_rhs[i * 3 + 2] += t1 * ry[i];
    }
}
/* fe_sw2_1d_wall_friction, src/fe/fe_sw2_boundary_integrals.c:205-219 */
static void wall_friction(double *elem_rhs, v2 n, double djac, double dt, const double *u, const double *v,
                          const double *res) {
    double rx[2] = {0., 0.}, ry[2] = {0., 0.};
    line_phi_f(djac, fabs(n.y), u, rx);
    line_phi_f(djac, fabs(n.x), v, ry);
    for (int i = 0; i < 2; i++) { elem_rhs[i * 3 + 1] += dt * res[i] * rx[i]; elem_rhs[i * 3 + 2] += dt * res[i] * ry[i]; }
}
/* fe_sw2_bc_discharge (src/models/sw2/sw2_bc_discharge.c.bk:111-172): the discharge law
 * -q sqrt(2 g / c_f) h^(3/2) / conveyance with the first node's head at both nodes, as an
 * explicit flux, plus wall friction along the segment */
static void discharge_resid(const sw2o_model *m, v2 n, double djac, double dt, const double *head, const v2 *vel,
                            double *elem_rhs) {
    double u_tan = one_2 * (vel[0].x + vel[1].x) * n.y - one_2 * (vel[0].y + vel[1].y) * n.x;
    double mag_utan = fabs(u_tan);
    double u[2] = {vel[0].x, vel[1].x}, v[2] = {vel[0].y, vel[1].y};
    double h_avg = one_2 * (head[0] + head[1]);
    if (h_avg < SMALL) h_avg = SMALL;
    double res[2] = {one_2 * bc_roughness(head[0], m->bc_rough) * mag_utan,
                     one_2 * bc_roughness(head[1], m->bc_rough) * mag_utan};
    if (head[0] < SMALL || head[1] < SMALL) return;
    double g = m->gravity;
    double fact = -1.0 * m->bc_qs * sqrt(2. * g / bc_roughness(head[0], m->bc_rough)) / m->bc_convey;
    double d0 = fact * pow(head[0], 1.5);
    fact = -1.0 * m->bc_qs * sqrt(2. * g / bc_roughness(head[1], m->bc_rough)) / m->bc_convey;
    double d1 = fact * pow(head[0], 1.5);
    explicit_flow(elem_rhs, n, djac, dt, one_2 * (d0 + d1), h_avg, u, v);
    wall_friction(elem_rhs, n, djac, dt, u, v, res);
}
/* fe_sw2_bc_vel (src/models/sw2/sw2_bc_vel.c:58), fe_sw2_bc_h (sw2_bc_h.c:57), and the
 * discharge, tailwater, outflow and flux conditions of sw2_bc_discharge.c.bk,
 * sw2_bc_tailwater.c.bk, sw2_bc_outflow.c.bk and sw2_bc_flux.c.bk */
static void seg_resid(const sw2o_model *m, const double *sol, int k, double pert, int pnode, int pvar, int psign,
                      double *elem_rhs) {
    const int *nd = m->seg + 2 * k;
    v2 n = {m->seg_nrml[2 * k], m->seg_nrml[2 * k + 1]};
    double djac = m->seg_djac[k], dt = m->dt;
    double head[2]; v2 vel[2];
    int pressure = 1;
    for (int i = 0; i < 2; i++) { head[i] = sol[3 * nd[i]]; vel[i].x = sol[3 * nd[i] + 1]; vel[i].y = sol[3 * nd[i] + 2]; }
    if (pvar == 0) head[pnode] += psign * pert;
    else if (pvar == 1) { vel[pnode].x += psign * pert; pressure = 0; }
    else if (pvar == 2) { vel[pnode].y += psign * pert; pressure = 0; }
    if (m->seg_kind[k] == 0) {
        vel[0].x = m->bc_vx; vel[0].y = m->bc_vy; vel[1].x = m->bc_vx; vel[1].y = m->bc_vy;
        implicit_flow(elem_rhs, n, djac, dt, vel, head);
    } else if (m->seg_kind[k] == 1) {
        double dep[2] = {m->bc_depth, m->bc_depth};
        if (dep[0] < SMALL || dep[1] < SMALL || head[0] < SMALL || head[1] < SMALL) return;
        implicit_flow(elem_rhs, n, djac, dt, vel, dep);
        if (pressure) {
            pressure_1d(elem_rhs, n, djac, dt, dep, m->gravity);
            pressure_1d(elem_rhs, n, djac, dt, head, -m->gravity);
        }
    } else if (m->seg_kind[k] == 2) {
        discharge_resid(m, n, djac, dt, head, vel, elem_rhs);
    } else if (m->seg_kind[k] == 4) {   /* sw2_bc_outflow.c.bk:144 */
        implicit_flow(elem_rhs, n, djac, dt, vel, head);
    } else if (m->seg_kind[k] == 5) {   /* sw2_bc_flux.c.bk:151-153 */
        double u[2] = {vel[0].x, vel[1].x}, v[2] = {vel[0].y, vel[1].y};
        double h_avg = one_2 * (head[0] + head[1]);
        if (h_avg < SMALL) h_avg = SMALL;
        explicit_flow(elem_rhs, n, djac, dt, -1.0 * m->bc_flux, h_avg, u, v);
    } else {   /* sw2_bc_tailwater.c.bk:152-170: depth below the elevation at the first node, at both */
        double z0 = m->xyz[3 * nd[0] + 2];
        double dep[2] = {m->bc_tail - z0, m->bc_tail - z0};
        if (dep[0] < SMALL || dep[1] < SMALL || head[0] < SMALL || head[1] < SMALL) return;
        implicit_flow(elem_rhs, n, djac, dt, vel, head);
        if (pressure) {
            pressure_1d(elem_rhs, n, djac, dt, dep, m->gravity);
            pressure_1d(elem_rhs, n, djac, dt, head, -m->gravity);
        }
    }
}

void sw2o_elem_resid_all(const sw2o_model *m, const double *sol, const double *sol_old,
                         const double *sol_older, double *out_tri, double *out_seg) {
    #pragma omp parallel for schedule(static)
    for (int e = 0; e < m->ntri; e++) {
        double r[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        sw2o_body_resid(m, sol, sol_old, sol_older, e, 0.0, -1, -1, 0, r);
        memcpy(out_tri + 9 * (size_t)e, r, sizeof r);
    }
    for (int k = 0; k < m->nseg; k++) {
        double r[6] = {0, 0, 0, 0, 0, 0};
        seg_resid(m, sol, k, 0.0, -1, -1, 0, r);
        memcpy(out_seg + 6 * (size_t)k, r, sizeof r);
    }
}

/* ------------------------------------------------------------------ FD element Jacobian
 * perturb_var + elem_matrix_deriv, src/jacobian/assemble_jacobian.c:304-397 */
static inline double fd_eps(double u) {     /* NUM_DIFF_EPSILON, macro.h:669 with 1e-4 (:313) */
    double e = fabs(u) * (1. + 1e-4);
    e -= fabs(u);
    if (e < 1e-4) e = 1e-4;
    return e;
}

static void tri_jac(const sw2o_model *m, const double *sol, const double *sol_old, const double *sol_older,
                    int e, double *J /* 81 */) {
    const int *nd = m->tri + 3 * e;
    for (int k = 0; k < 3; k++) {
        for (int i = 0; i < 3; i++) {
            double eps = fd_eps(sol[3 * nd[i] + k]);
            double eps2 = 2.0 * eps;
            double P[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, M[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            sw2o_body_resid(m, sol, sol_old, sol_older, e, eps, i, k, +1, P);
            sw2o_body_resid(m, sol, sol_old, sol_older, e, eps, i, k, -1, M);
            int col = i * 3 + k;
            for (int r = 0; r < 9; r++) J[r * 9 + col] = (P[r] - M[r]) / eps2;
        }
    }
}

static void seg_jac(const sw2o_model *m, const double *sol, int k_, double *J /* 36 */) {
    const int *nd = m->seg + 2 * k_;
    for (int k = 0; k < 3; k++) {
        for (int i = 0; i < 2; i++) {
            double eps = fd_eps(sol[3 * nd[i] + k]);
            double eps2 = 2.0 * eps;
            double P[6] = {0, 0, 0, 0, 0, 0}, M[6] = {0, 0, 0, 0, 0, 0};
            seg_resid(m, sol, k_, eps, i, k, +1, P);
            seg_resid(m, sol, k_, eps, i, k, -1, M);
            int col = i * 3 + k;
            for (int r = 0; r < 6; r++) J[r * 6 + col] = (P[r] - M[r]) / eps2;
        }
    }
}

void sw2o_elem_jac_all(const sw2o_model *m, const double *sol, const double *sol_old,
                       const double *sol_older, double *out_tri, double *out_seg) {
    #pragma omp parallel for schedule(static)
    for (int e = 0; e < m->ntri; e++) tri_jac(m, sol, sol_old, sol_older, e, out_tri + 81 * (size_t)e);
    for (int k = 0; k < m->nseg; k++) seg_jac(m, sol, k, out_seg + 36 * (size_t)k);
}

/* ------------------------------------------------------------------ assembly */
void sw2o_assemble_residual(const sw2o_model *m, const double *sol, const double *sol_old,
                            const double *sol_older, double *residual) {
    double *et = malloc(sizeof(double) * 9 * ((size_t)m->ntri + 1));
    double *es = malloc(sizeof(double) * 6 * ((size_t)m->nseg + 1));
    sw2o_elem_resid_all(m, sol, sol_old, sol_older, et, es);
    for (int i = 0; i < m->ndof; i++) residual[i] = 0.0;
    /* load_pdes: elem_rhs = 0 + (-1.0)*eq_rhs, then residual[dof] += elem_rhs (:4-60,160) */
    for (int e = 0; e < m->ntri; e++)
        for (int a = 0; a < 3; a++)
            for (int v = 0; v < 3; v++) residual[3 * m->tri[3 * e + a] + v] += 0.0 + -1.0 * et[9 * (size_t)e + 3 * a + v];
    for (int k = 0; k < m->nseg; k++)
        for (int a = 0; a < 2; a++)
            for (int v = 0; v < 3; v++) residual[3 * m->seg[2 * k + a] + v] += 0.0 + -1.0 * es[6 * (size_t)k + 3 * a + v];
    free(et); free(es);
}

static inline int find_slot(const int *indptr, const int *cols, int row, int col) {
    int lo = indptr[row], hi = indptr[row + 1] - 1;
    while (lo <= hi) { int mid = (lo + hi) >> 1; if (cols[mid] < col) lo = mid + 1; else if (cols[mid] > col) hi = mid - 1; else return mid; }
    return -1;
}

void sw2o_assemble_jacobian(const sw2o_model *m, const double *sol, const double *sol_old,
                            const double *sol_older, double *vals) {
    double *jt = malloc(sizeof(double) * 81 * ((size_t)m->ntri + 1));
    double *js = malloc(sizeof(double) * 36 * ((size_t)m->nseg + 1));
    sw2o_elem_jac_all(m, sol, sol_old, sol_older, jt, js);
    for (int i = 0; i < m->nnz; i++) vals[i] = 0.0;
    for (int e = 0; e < m->ntri; e++) {
        int dofs[9];
        for (int a = 0; a < 3; a++) for (int v = 0; v < 3; v++) dofs[3 * a + v] = 3 * m->tri[3 * e + a] + v;
        for (int i = 0; i < 9; i++) for (int j = 0; j < 9; j++)
            vals[find_slot(m->indptr, m->cols, dofs[i], dofs[j])] += jt[81 * (size_t)e + 9 * i + j];
    }
    for (int k = 0; k < m->nseg; k++) {
        int dofs[6];
        for (int a = 0; a < 2; a++) for (int v = 0; v < 3; v++) dofs[3 * a + v] = 3 * m->seg[2 * k + a] + v;
        for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++)
            vals[find_slot(m->indptr, m->cols, dofs[i], dofs[j])] += js[36 * (size_t)k + 6 * i + j];
    }
    free(jt); free(js);
}

/* ------------------------------------------------------------------ linear system */
void sw2o_check_diag(const sw2o_model *m, const double *vals, int *bc_mask) {
    for (int r = 0; r < m->ndof; r++) {
        int s = find_slot(m->indptr, m->cols, r, r);
        if (fabs(vals[s]) < SMALL) bc_mask[r] = 1;
    }
}

void sw2o_apply_dirichlet(const sw2o_model *m, const int *bc_mask, double *vals, double *residual) {
    for (int r = 0; r < m->ndof; r++)
        for (int k = m->indptr[r]; k < m->indptr[r + 1]; k++)
            if (bc_mask[m->cols[k]] == 1) vals[k] = 0.0;
    for (int r = 0; r < m->ndof; r++) {
        if (bc_mask[r] == 1) {
            residual[r] = 0.0;
            for (int k = m->indptr[r]; k < m->indptr[r + 1]; k++) vals[k] = (m->cols[k] == r) ? 1.0 : 0.0;
        }
    }
}

void sw2o_scale_system(const sw2o_model *m, double *vals, double *b, double *x, double *s) {
    int n = m->ndof;
    for (int i = 0; i < n; i++) {
        double mx = 0;
        for (int k = m->indptr[i]; k < m->indptr[i + 1]; k++) { double t = fabs(vals[k]); if (t > mx) mx = t; }
        s[i] = mx;
    }
    double small = DBL_EPSILON, small_factor = 1.0 / sqrt(small);
    for (int i = 0; i < n; i++) s[i] = (s[i] < small) ? small_factor : 1.0 / sqrt(fabs(s[i]));
    for (int i = 0; i < n; i++) { double f = s[i]; b[i] *= f; x[i] /= f; }
    for (int i = 0; i < n; i++)
        for (int k = m->indptr[i]; k < m->indptr[i + 1]; k++) vals[k] *= s[i] * s[m->cols[k]];
}

void sw2o_spmv(int n, const int *indptr, const int *cols, const double *vals, const double *x, double *y) {
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        double a = 0.0;
        for (int k = indptr[i]; k < indptr[i + 1]; k++) a += vals[k] * x[cols[k]];
        y[i] = a;
    }
}

/* 3x3 nodal block-Jacobi: invert the diagonal block of every node (Gauss-Jordan
 * with partial pivoting); a singular block falls back to the identity. */
static void bj_setup(int n, const int *indptr, const int *cols, const double *vals, double *inv) {
    int nn = n / 3;
    #pragma omp parallel for schedule(static)
    for (int b = 0; b < nn; b++) {
        double a[3][6];
        for (int r = 0; r < 3; r++) {
            int row = 3 * b + r;
            for (int c = 0; c < 3; c++) { a[r][c] = 0.0; a[r][3 + c] = (r == c) ? 1.0 : 0.0; }
            for (int k = indptr[row]; k < indptr[row + 1]; k++) {
                int c = cols[k] - 3 * b;
                if (c >= 0 && c < 3) a[r][c] = vals[k];
            }
        }
        int ok = 1;
        for (int c = 0; c < 3 && ok; c++) {
            int p = c; double pv = fabs(a[c][c]);
            for (int r = c + 1; r < 3; r++) if (fabs(a[r][c]) > pv) { pv = fabs(a[r][c]); p = r; }
            if (pv == 0.0) { ok = 0; break; }
            if (p != c) for (int k = 0; k < 6; k++) { double t = a[c][k]; a[c][k] = a[p][k]; a[p][k] = t; }
            double d = a[c][c];
            for (int k = 0; k < 6; k++) a[c][k] /= d;
            for (int r = 0; r < 3; r++) if (r != c) { double f = a[r][c]; for (int k = 0; k < 6; k++) a[r][k] -= f * a[c][k]; }
        }
        for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) inv[9 * b + 3 * r + c] = ok ? a[r][3 + c] : (r == c ? 1.0 : 0.0);
    }
}
static void bj_apply(int n, const double *inv, const double *x, double *y) {
    int nn = n / 3;
    #pragma omp parallel for schedule(static)
    for (int b = 0; b < nn; b++) {
        const double *M = inv + 9 * b; const double *xi = x + 3 * b;
        for (int r = 0; r < 3; r++) y[3 * b + r] = M[3 * r] * xi[0] + M[3 * r + 1] * xi[1] + M[3 * r + 2] * xi[2];
    }
}
static double dot(int n, const double *a, const double *b) { double s = 0; for (int i = 0; i < n; i++) s += a[i] * b[i]; return s; }
static double linf(int n, const double *a) { double s = 0; for (int i = 0; i < n; i++) { double t = fabs(a[i]); if (t > s) s = t; } return s; }

int sw2o_bicgstab_bj(int n, const int *indptr, const int *cols, const double *vals, double *x,
                     double *b, const double *scale_vect, int max_it, double tol) {
    double *inv = malloc(sizeof(double) * 3 * (size_t)n);
    bj_setup(n, indptr, cols, vals, inv);
    double *r = calloc((size_t)n, 8), *p = calloc((size_t)n, 8), *Ap = calloc((size_t)n, 8), *Mp = calloc((size_t)n, 8);
    double *q = calloc((size_t)n, 8), *s = calloc((size_t)n, 8), *As = calloc((size_t)n, 8), *Ms = calloc((size_t)n, 8);
    double *x0 = malloc(8 * (size_t)n);
    memcpy(x0, x, 8 * (size_t)n);
    for (int i = 0; i < n; i++) x[i] = 0;
    /* b <- M^-1 b;  x = M^-1 b;  r = b - M^-1 A x   (bcgstab_solver.c:137-176) */
    memcpy(p, b, 8 * (size_t)n);
    bj_apply(n, inv, p, b);
    for (int i = 0; i < n; i++) p[i] = 0;
    memcpy(x, b, 8 * (size_t)n);
    sw2o_spmv(n, indptr, cols, vals, x, Mp);
    bj_apply(n, inv, Mp, Ap);
    for (int i = 0; i < n; i++) r[i] = b[i] + -1 * Ap[i];
    for (int i = 0; i < n; i++) { Mp[i] = 0; Ap[i] = 0; }
    memcpy(q, r, 8 * (size_t)n);
    double rnorm = linf(n, r), bnorm = linf(n, b);
    double rhop = 1.0, alpha = 1.0, omega = 1.0, rho = dot(n, r, q), gamma, beta;
    int it = 0, status = 0;
    while (rnorm > (tol + bnorm * tol) && it < max_it) {
        it++;
        beta = (rho * alpha) / (rhop * omega);
        for (int i = 0; i < n; i++) p[i] += -omega * Ap[i];
        for (int i = 0; i < n; i++) p[i] *= beta;
        for (int i = 0; i < n; i++) p[i] += 1 * r[i];
        sw2o_spmv(n, indptr, cols, vals, p, Mp);
        bj_apply(n, inv, Mp, Ap);
        gamma = dot(n, q, Ap);
        if (gamma == 0.0 || !isfinite(gamma)) { status = -1; break; }
        alpha = rho / gamma;
        for (int i = 0; i < n; i++) s[i] = r[i] + -alpha * Ap[i];
        sw2o_spmv(n, indptr, cols, vals, s, Ms);
        bj_apply(n, inv, Ms, As);
        omega = dot(n, As, s);
        gamma = dot(n, As, As);
        if (gamma == 0.0) { /* s is exactly zero: x += alpha p solves the system */
            for (int i = 0; i < n; i++) x[i] += alpha * p[i];
            for (int i = 0; i < n; i++) r[i] = s[i];
            rnorm = linf(n, r);
            break;
        }
        omega = omega / gamma;
        rhop = rho;
        rho = -1.0 * omega * dot(n, As, q);
        for (int i = 0; i < n; i++) x[i] += alpha * p[i];
        for (int i = 0; i < n; i++) x[i] += omega * s[i];
        for (int i = 0; i < n; i++) r[i] = s[i] + -omega * As[i];
        rnorm = linf(n, r);
        if (!isfinite(rnorm)) { status = -1; break; }
    }
    /* unscale_linear_system (scale_linear_system.c:137) */
    for (int i = 0; i < n; i++) x[i] += x0[i];
    for (int i = 0; i < n; i++) x[i] *= scale_vect[i];
    free(inv); free(r); free(p); free(Ap); free(Mp); free(q); free(s); free(As); free(Ms); free(x0);
    return status < 0 ? -it - 1 : it;
}

/* ------------------------------------------------------------------ Newton step
 * fe_newton (src/newton/fe_newton.c:44-915) with the serial, non-PETSc branch. */
static void resid_norms(int n, const double *res, const double *dsol, const int *bc_mask,
                        double *rmax, double *rl2, double *imax) {
    double l2 = 0, mx = 0, im = 0;
    for (int i = 0; i < n; i++) {
        int inc = (bc_mask[i] == 1) ? 0 : 1;
        if (fabs(dsol[i]) > im && inc) im = fabs(dsol[i]);
        if (fabs(res[i]) > mx && inc) mx = fabs(res[i]);
        if (inc) l2 += res[i] * res[i];
    }
    *rmax = mx; *rl2 = sqrt(l2) / n; *imax = im;
}

int sw2o_newton(sw2o_model *m, double *sol, const double *sol_old, const double *sol_older,
                int *bc_mask, const double *dirichlet, double tol_nonlin, double inc_nonlin,
                int max_nonlin_it, int max_linesearch_cuts, int krylov_max_it, double krylov_tol,
                double *stats) {
    int n = m->ndof;
    double *res = malloc(8 * (size_t)n), *dsol = calloc((size_t)n, 8), *vals = malloc(8 * (size_t)m->nnz);
    double *sv = malloc(8 * (size_t)n);
    /* initialize_system: sol <- sol_old; fe_sw2_init (wd flags, dry-node masks) */
    memcpy(sol, sol_old, 8 * (size_t)n);
    sw2o_wd_flags(m, sol, sol_old);
    for (int i = 0; i < m->nnodes; i++)
        if (sol_old[3 * i] <= 0.) { bc_mask[3 * i + 1] = 1; bc_mask[3 * i + 2] = 1; }
    for (int i = 0; i < n; i++) if (bc_mask[i] == 1) sol[i] = dirichlet[i];
    sw2o_assemble_residual(m, sol, sol_old, sol_older, res);
    double rmax, rl2, imax, old_l2;
    resid_norms(n, res, dsol, bc_mask, &rmax, &rl2, &imax);
    int it = 0, kry_total = 0, cuts_total = 0, ok = 1, keep;
    do {
        sw2o_assemble_jacobian(m, sol, sol_old, sol_older, vals);
        sw2o_check_diag(m, vals, bc_mask);
        sw2o_apply_dirichlet(m, bc_mask, vals, res);
        for (int i = 0; i < n; i++) dsol[i] = 0;
        sw2o_scale_system(m, vals, res, dsol, sv);
        int kit = sw2o_bicgstab_bj(n, m->indptr, m->cols, vals, dsol, res, sv, krylov_max_it, krylov_tol);
        kry_total += kit < 0 ? -kit - 1 : kit;
        for (int i = 0; i < n; i++) sol[i] += dsol[i];
        for (int i = 0; i < n; i++) dsol[i] = -dsol[i];
        old_l2 = rl2;
        sw2o_assemble_residual(m, sol, sol_old, sol_older, res);
        resid_norms(n, res, dsol, bc_mask, &rmax, &rl2, &imax);
        if (isnan(rl2) || isinf(rl2)) ok = 0;
        int cuts = 0;
        while (rmax > tol_nonlin && rl2 > old_l2 && cuts < max_linesearch_cuts) {
            for (int i = 0; i < n; i++) dsol[i] *= 0.5;
            for (int i = 0; i < n; i++) sol[i] += dsol[i];
            sw2o_assemble_residual(m, sol, sol_old, sol_older, res);
            resid_norms(n, res, dsol, bc_mask, &rmax, &rl2, &imax);
            cuts++;
        }
        cuts_total += cuts;
        it++;
        keep = ok && it < max_nonlin_it && rmax < 1.0E+20 && rmax > tol_nonlin && imax > inc_nonlin;
    } while (keep);
    int success = !(((rmax > tol_nonlin) && (imax > inc_nonlin)) || (rmax >= 1.0E+20) || !ok);
    if (!success) {   /* fe_newton.c:893-899: initialize_system, then initialize_dirichlet_bc */
        memcpy(sol, sol_old, 8 * (size_t)n);
        sw2o_wd_flags(m, sol, sol_old);
        for (int i = 0; i < m->nnodes; i++)
            if (sol_old[3 * i] <= 0.) { bc_mask[3 * i + 1] = 1; bc_mask[3 * i + 2] = 1; }
        for (int i = 0; i < n; i++) if (bc_mask[i] == 1) sol[i] = dirichlet[i];
    }
    stats[0] = it; stats[1] = kry_total; stats[2] = rmax; stats[3] = success; stats[4] = cuts_total;
    free(res); free(dsol); free(vals); free(sv);
    return success;
}

/* ------------------------------------------------------------------ mass balance */

/* fe_3m2d_dry_wet_factornew, src/tools/tl_grid_mass.c:442-515: the wet fraction
 * of a triangle for the mass integral.  Unlike the residual's wet/dry factor, a
 * vertex is dry only when its depth is strictly negative (:462). */
static double mass_wet_factor(const v2 *x, const double *h, double djac, int *num_dry) {
    int passcode = 0, total = 0;
    for (int i = 0; i < 3; i++) { int d = (h[i] < 0.0) ? 1 : 0; total += d; passcode += (d << i); }
    if (total == 3) { *num_dry = 3; return 0.0; }
    if (total == 0) { *num_dry = 0; return 1.0; }
    if (total != 1) passcode = 7 - passcode;
    int only = passcode / 2;
    v2 nx[3];
    for (int i = 0; i < 3; i++) {
        if (i != only) {
            double xsi = h[i] / (h[i] - h[only]);
            nx[i].x = x[i].x + xsi * (x[only].x - x[i].x);           /* FIXED_POS, macro.h:756 */
            nx[i].y = x[i].y + xsi * (x[only].y - x[i].y);
        } else nx[i] = x[i];
    }
    double elem_djac = djac;
    double ax = nx[1].x - nx[0].x, ay = nx[1].y - nx[0].y;           /* TRI_AREA, macro.h:771 */
    double bx = nx[2].x - nx[0].x, by = nx[2].y - nx[0].y;
    djac = (ax * by - ay * bx) / 2.0;
    if (djac / elem_djac < SMALL) {                                   /* :506-509 */
        int odd = total % 2;
        *num_dry = (odd == 1) ? 0 : 3;
        return (double)odd;
    }
    double factor = (total >> 1) - (total % 2);
    *num_dry = total;
    factor *= djac / elem_djac;
    return factor + ((factor < 0) ? 1.0 : 0.0);
}

/* integrate_triangle_f, src/fe/fe_integrals_2d.c:25 */
static inline double tri_int_f(double djac, double c, const double *f) {
    return (c * djac * (f[0] + f[1] + f[2]) / 3.0);
}

double sw2o_elem_mass(const sw2o_model *m, const double *sol, int e) {
    /* one triangle's term of tl_find_grid_mass_elem2d, src/tools/tl_grid_mass.c:209-258 */
    double head[3], hneg[3] = {0.0, 0.0, 0.0};
    v2 x[3];
    for (int a = 0; a < 3; a++) {
        int nd = m->tri[3 * e + a];
        head[a] = sol[3 * nd];
        x[a].x = m->xyz[3 * nd]; x[a].y = m->xyz[3 * nd + 1];
    }
    double djac = m->tri_djac[e];
    int num_dry;
    double factor = mass_wet_factor(x, head, djac, &num_dry);
    double f1, f2;
    switch (num_dry) {
        case 1:     /* the wet part plus the (negative) dry vertex depth counted as positive mass */
            for (int a = 0; a < 3; a++) if (head[a] < 0.0) hneg[a] = head[a];
            f1 = 1.0; f2 = -1.0 * (1.0 - factor);
            break;
        case 2:
            for (int a = 0; a < 3; a++) if (head[a] < 0.0) { hneg[a] = head[a]; head[a] = 0.0; }
            f1 = factor; f2 = 0.0;
            break;
        default:
            f1 = factor; f2 = 0.0;
            break;
    }
    return tri_int_f(djac, f1, head) + tri_int_f(djac, f2, hneg);
}

double sw2o_grid_mass(const sw2o_model *m, const double *sol, double density) {
    double mass = 0.0;
    for (int e = 0; e < m->ntri; e++) mass += sw2o_elem_mass(m, sol, e);
    return mass * density;
}

double sw2o_boundary_mass_flux(const sw2o_model *m, const double *sol, double density, double dt,
                                int first_seg_length) {
    /* the boundary loop of tl_find_grid_mass_error_elem2d, src/tools/tl_grid_mass.c:310-320:
     * minus the integral of h (v . n) over every boundary segment, times density dt
     * (inflow positive).  Each segment uses its own length; the reference passes the
     * first segment's length (grid->elem1d->djac, :318) for all of them, which
     * first_seg_length = 1 reproduces. */
    double total = 0.0;
    for (int k = 0; k < m->nseg; k++) {
        double vn[2], h[2];
        for (int a = 0; a < 2; a++) {
            int nd = m->seg[2 * k + a];
            vn[a] = sol[3 * nd + 1] * m->seg_nrml[2 * k] + sol[3 * nd + 2] * m->seg_nrml[2 * k + 1];
            h[a] = sol[3 * nd];
        }
        /* integrate_line_h_f, src/fe/fe_integrals_1d.c:42, with h = v . n and f = depth */
        double len = first_seg_length ? m->seg_djac[0] : m->seg_djac[k];
        double t1 = len * one_6 * (density * dt);
        total -= (t1 * ((2 * vn[0] + vn[1]) * h[0] + (vn[0] + 2 * vn[1]) * h[1]));
    }
    return total;
}
