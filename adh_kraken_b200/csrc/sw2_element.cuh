// SW2 element residuals on the device: the triangle body residual
// (fe_sw2_body_resid, src/models/sw2/sw2_body_resid.c:44-1176) and the two
// weak boundary residuals (fe_sw2_bc_vel, src/models/sw2/sw2_bc_vel.c:58;
// fe_sw2_bc_h, src/models/sw2/sw2_bc_h.c:57).
//
// Parity contract: every expression keeps the reference's floating-point
// operation order and this file is compiled with --fmad=false, so a residual is
// bit-identical to the reference CPU build (IEEE division and square root are
// correctly rounded on both sides).  Terms whose coefficients the reference
// hard-codes to zero (shock capturing :352-400, eddy-viscosity diffusion
// :476-499, Coriolis :596-610, wind and rain) add a signed zero to an entry that
// holds a non-zero value or the +0 it started from, so they are not evaluated.
//
// Layout: everything lives in registers.  Arrays are indexed only with
// compile-time constants; the one data-dependent vertex of the wet/dry
// sub-triangle is handled with selects so nothing spills to local memory.
#pragma once
#include <cuda_runtime.h>

namespace sw2 {

// src/include/define.h:31-52
#define SW2_SMALL 2.220446049250313080847e-16          // DBL_EPSILON
#define SW2_NOT_QUITE_SMALL 1.1920928955078125e-07     // FLT_EPSILON, widened exactly
#define SW2_ONE_2 0.5e+0
#define SW2_ONE_3 0.333333333333333333333333
#define SW2_ONE_6 0.166666666666666666666667
#define SW2_ONE_12 0.083333333333333333333333
#define SW2_ONE_30 0.033333333333333333333333
#define SW2_ONE_60 0.016666666666666666666667

struct V2 { double x, y; };

__device__ __forceinline__ double dmax_(double a, double b) { return a > b ? a : b; }  // MAX, macro.h:845

template <class T>
__device__ __forceinline__ T sel3(const T a[3], int i) { return i == 0 ? a[0] : (i == 1 ? a[1] : a[2]); }

// ----------------------------------------------------------------------------
// closed-form P1 integrals, src/fe/fe_integrals_2d.c and fe_integrals_1d.c
__device__ __forceinline__ void tri_phi_f(double djac, double c, const double f[3], double I[3]) {
    double f_sum = f[0] + f[1] + f[2];
    double t1 = djac * c * SW2_ONE_12;
    I[0] += t1 * (f_sum + f[0]); I[1] += t1 * (f_sum + f[1]); I[2] += t1 * (f_sum + f[2]);
}
__device__ __forceinline__ void tri_phi_f_lump(double djac, double c, const double f[3], double I[3]) {
    double t1 = djac * c * SW2_ONE_3;
    I[0] += t1 * f[0]; I[1] += t1 * f[1]; I[2] += t1 * f[2];
}
__device__ __forceinline__ void line_phi_h_h(double djac, double c, double h1, double h2, double I[2]) {
    double t1 = djac * SW2_ONE_12 * c;
    I[0] += t1 * (3 * h1 * h1 + 2 * h1 * h2 + h2 * h2);
    I[1] += t1 * (h1 * h1 + 2 * h1 * h2 + 3 * h2 * h2);
}
__device__ __forceinline__ void line_phi_f_g_h(double djac, double c, double f1, double f2, double g1, double g2,
                                               double h1, double h2, double I[2]) {
    double t1 = SW2_ONE_60 * djac * c;
    I[0] += t1 * ((3 * (4 * f1 + f2) * g1 + (3 * f1 + 2 * f2) * g2) * h1 + ((3 * f1 + 2 * f2) * g1 + (2 * f1 + 3 * f2) * g2) * h2);
    I[1] += t1 * (((3 * f1 + 2 * f2) * g1 + (2 * f1 + 3 * f2) * g2) * h1 + ((2 * f1 + 3 * f2) * g1 + 3 * (f1 + 4 * f2) * g2) * h2);
}

// ----------------------------------------------------------------------------
// The partially wet sub-triangle of fe_sw2_wet_dry_wrapper (src/fe/fe_wet_dry_wrapper.c:104-304):
// classify the vertices, cut the triangle along h = 0, and describe the piece that
// is integrated and added with weight +1 (two dry vertices: the wet corner) or
// -1 (one dry vertex: the dry corner, subtracted from the full-element integral).
struct Cut {
    int total;        // number of vertices with h <= 0
    int only;         // the corner vertex of the sub-triangle
    double xsi[3];    // interpolation weights of the non-corner vertices
    V2 nx[3];         // sub-triangle vertices
    double nh[3];     // depths on the sub-triangle (0 on the cut)
    double area;      // sub-triangle area (TRI_AREA, macro.h:771)
};

__device__ __forceinline__ int classify(const double h[3], int* only) {
    int passcode = 0, total = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) { int d = (h[i] <= 0.0) ? 1 : 0; total += d; passcode += (d << i); }
    if (total != 1) passcode = 7 - passcode;
    *only = passcode / 2;
    return total;
}

__device__ __forceinline__ void make_cut(const V2 x[3], const double h[3], Cut& c) {
    c.total = classify(h, &c.only);
    const int o = c.only;
    const double ho = sel3(h, o);
    const V2 xo = sel3(x, o);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (i != o) {
            double xsi = h[i] / (h[i] - ho);
            c.xsi[i] = xsi;
            c.nx[i].x = x[i].x + xsi * (xo.x - x[i].x);   // FIXED_POS, macro.h:756
            c.nx[i].y = x[i].y + xsi * (xo.y - x[i].y);
            c.nh[i] = 0.0;
        } else {
            c.xsi[i] = 0.0;
            c.nx[i] = x[i];
            c.nh[i] = h[i];
        }
    }
    double ax = c.nx[1].x - c.nx[0].x, ay = c.nx[1].y - c.nx[0].y;
    double bx = c.nx[2].x - c.nx[0].x, by = c.nx[2].y - c.nx[0].y;
    c.area = (ax * by - ay * bx) / 2.0;
}

// interpolate a nodal quantity onto the sub-triangle (FIXED_POS with the cut's weights)
__device__ __forceinline__ void cut_interp(const Cut& c, const double f[3], double nf[3]) {
    const double fo = sel3(f, c.only);
#pragma unroll
    for (int i = 0; i < 3; i++) nf[i] = (i != c.only) ? f[i] + c.xsi[i] * (fo - f[i]) : f[i];
}
__device__ __forceinline__ void cut_interp(const Cut& c, const V2 f[3], V2 nf[3]) {
    const V2 fo = sel3(f, c.only);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (i != c.only) { nf[i].x = f[i].x + c.xsi[i] * (fo.x - f[i].x); nf[i].y = f[i].y + c.xsi[i] * (fo.y - f[i].y); }
        else nf[i] = f[i];
    }
}
// GRAD_SHAPE, macro.h:778
__device__ __forceinline__ void cut_grad(const Cut& c, V2 g[3]) {
    const V2* v = c.nx;
    g[0].x = 0.5 * (v[1].y - v[2].y) / c.area;
    g[1].x = 0.5 * (v[2].y - v[0].y) / c.area;
    g[2].x = 0.5 * (v[0].y - v[1].y) / c.area;
    g[0].y = 0.5 * (v[2].x - v[1].x) / c.area;
    g[1].y = 0.5 * (v[0].x - v[2].x) / c.area;
    g[2].y = 0.5 * (v[1].x - v[0].x) / c.area;
}
// RE_DISTRIBUTE, macro.h:788: move the cut vertices' share back to the corner
__device__ __forceinline__ void cut_redistribute(const Cut& c, const V2 x[3], double nr[9]) {
    const V2 xo = sel3(x, c.only);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (i == c.only) continue;
        double v0x = c.nx[i].x - xo.x, v0y = c.nx[i].y - xo.y;
        double v1x = x[i].x - xo.x, v1y = x[i].y - xo.y;
        double l0 = v0x * v0x + v0y * v0y, l1 = v1x * v1x + v1y * v1y;
        double xsi = sqrt(l0 / l1);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double add = (1.0 - xsi) * nr[i * 3 + k];
            // nr[only*3+k] += add, with the corner selected by predicate
            if (c.only == 0) nr[k] += add; else if (c.only == 1) nr[3 + k] += add; else nr[6 + k] += add;
        }
#pragma unroll
        for (int k = 0; k < 3; k++) nr[i * 3 + k] *= xsi;
    }
}

// Apply the wrapper's rule around an integrand `f(rhs, x, h, ...)`.  `sub(nr)` must
// evaluate the integrand on the sub-triangle described by the Cut.  Returns the
// wrapper's wet fraction.
template <class Full, class Sub>
__device__ __forceinline__ double wd_wrap(double r[9], const V2 x[3], const double h[3], double djac, bool redist,
                                          Full full, Sub sub) {
    int only;
    int total = classify(h, &only);
    if (total == 3) return 0.0;
    if (total == 0) { full(r); return 1.0; }
    if (total == 1) full(r);
    Cut c;
    make_cut(x, h, c);
    if (c.area / djac < SW2_SMALL) return (double)(total % 2);
    double nr[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    sub(c, nr);
    double factor = (total >> 1) - (total % 2);
    if (redist) cut_redistribute(c, x, nr);
#pragma unroll
    for (int i = 0; i < 9; i++) r[i] += factor * nr[i];
    factor *= c.area / djac;
    return factor + ((factor < 0) ? 1.0 : 0.0);
}

// fe_sw2_wet_dry_factor, fe_wet_dry_wrapper.c:29
__device__ __forceinline__ double wd_factor(const V2 x[3], const double h[3], double djac) {
    int only;
    int total = classify(h, &only);
    if (total == 3) return 0.0;
    if (total == 0) return 1.0;
    Cut c;
    make_cut(x, h, c);
    if (c.area / djac < SW2_SMALL) return (double)(total % 2);
    double factor = (total >> 1) - (total % 2);
    factor *= c.area / djac;
    return factor + ((factor < 0) ? 1.0 : 0.0);
}

// ----------------------------------------------------------------------------
// integrands of src/fe/fe_wet_dry_integrations.c, each on explicit vertex data
__device__ __forceinline__ void ig_convection(double r[9], const V2 g[3], double djac, double c,
                                              const double h[3], const V2 w[3]) {   // :94
    double rc[3] = {0, 0, 0}, rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
    double uu[3] = {w[0].x, w[1].x, w[2].x}, vv[3] = {w[0].y, w[1].y, w[2].y};
    {   // integrate_triangle_gradPhi_dot_f_v
        double p1 = (2 * h[0] + h[1] + h[2]);
        double p2 = (h[0] + 2 * h[1] + h[2]);
        double p3 = (h[0] + h[1] + 2 * h[2]);
        double tx = (p1 * w[0].x + p2 * w[1].x + p3 * w[2].x);
        double ty = (p1 * w[0].y + p2 * w[1].y + p3 * w[2].y);
        double con = djac * SW2_ONE_12 * c;
#pragma unroll
        for (int i = 0; i < 3; i++) rc[i] += con * (g[i].x * tx + g[i].y * ty);
    }
    {   // integrate_triangle_dphi_f_g_h(.., uu, vv, h, rhs_y, rhs_x)
        const double* f = uu; const double* gg = vv;
        double ff1 = (3 * f[0] + f[1] + f[2]), ff2 = (2 * f[0] + 2 * f[1] + f[2]), ff3 = (2 * f[0] + f[1] + 2 * f[2]);
        double ff4 = (f[0] + 3 * f[1] + f[2]), ff5 = (f[0] + 2 * f[1] + 2 * f[2]), ff6 = (f[0] + f[1] + 3 * f[2]);
        double gg1 = (2 * ff1 * gg[0] + ff2 * gg[1] + ff3 * gg[2]);
        double gg2 = (ff2 * gg[0] + 2 * ff4 * gg[1] + ff5 * gg[2]);
        double gg3 = (ff3 * gg[0] + ff5 * gg[1] + 2 * ff6 * gg[2]);
        double con = djac * SW2_ONE_60 * c * (gg1 * h[0] + gg2 * h[1] + gg3 * h[2]);
#pragma unroll
        for (int i = 0; i < 3; i++) ry[i] += con * g[i].x;
#pragma unroll
        for (int i = 0; i < 3; i++) rx[i] += con * g[i].y;
    }
    // integrate_triangle_dphi_f_f_h for uu (x only) and vv (y only)
#pragma unroll
    for (int d = 0; d < 2; d++) {
        const double* f = d == 0 ? uu : vv;
        double f1_2 = f[0] * f[0], f2_2 = f[1] * f[1], f3_2 = f[2] * f[2];
        double p1 = (3 * f1_2 + 2 * f[0] * f[1] + f2_2 + (2 * f[0] + f[1]) * f[2] + f3_2);
        double p2 = (f1_2 + 2 * f[0] * f[1] + 3 * f2_2 + (f[0] + 2 * f[1]) * f[2] + f3_2);
        double p3 = (f1_2 + f[0] * f[1] + f2_2 + 2 * (f[0] + f[1]) * f[2] + 3 * f3_2);
        double con = djac * SW2_ONE_30 * c * (p1 * h[0] + p2 * h[1] + p3 * h[2]);
        if (d == 0) {
#pragma unroll
            for (int i = 0; i < 3; i++) rx[i] += con * g[i].x;
        } else {
#pragma unroll
            for (int i = 0; i < 3; i++) ry[i] += con * g[i].y;
        }
    }
#pragma unroll
    for (int i = 0; i < 3; i++) { r[3 * i] += rc[i]; r[3 * i + 1] += rx[i]; r[3 * i + 2] += ry[i]; }
}

__device__ __forceinline__ void ig_continuity_temporal(double r[9], double djac, double c, const double h[3]) {  // :244
    double rc[3] = {0, 0, 0};
    tri_phi_f(djac, c, h, rc);
#pragma unroll
    for (int i = 0; i < 3; i++) r[3 * i] += rc[i];
}

__device__ __forceinline__ void ig_pressure(double r[9], const V2 g[3], double djac, double c, const double f[3]) {  // :292
    double int_f_f = (c * SW2_ONE_6 * djac * (f[0] * f[0] + f[0] * f[1] + f[1] * f[1] + f[0] * f[2] + f[1] * f[2] + f[2] * f[2]));
    double rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < 3; i++) rx[i] += g[i].x * int_f_f;
#pragma unroll
    for (int i = 0; i < 3; i++) ry[i] += g[i].y * int_f_f;
#pragma unroll
    for (int i = 0; i < 3; i++) { r[3 * i + 1] += rx[i]; r[3 * i + 2] += ry[i]; }
}

__device__ __forceinline__ void ig_body_force(double r[9], double djac, double c, const double h[3], V2 df) {  // :349
    double rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
    double con, sum_h = h[0] + h[1] + h[2];
    con = djac * SW2_ONE_12 * c * df.x;
#pragma unroll
    for (int i = 0; i < 3; i++) rx[i] += con * (sum_h + h[i]);
    con = djac * SW2_ONE_12 * c * df.y;
#pragma unroll
    for (int i = 0; i < 3; i++) ry[i] += con * (sum_h + h[i]);
#pragma unroll
    for (int i = 0; i < 3; i++) { r[3 * i + 1] += rx[i]; r[3 * i + 2] += ry[i]; }
}

__device__ __forceinline__ void ig_boundary_pressure(double r[9], const V2 x[3], double c, const double h[3]) {  // :389
#pragma unroll
    for (int e = 0; e < 3; e++) {
        const int n1 = e, n2 = (e + 1) % 3;
        double delx = x[n1].x - x[n2].x;
        double dely = x[n2].y - x[n1].y;
        double q[2] = {0., 0.};
        line_phi_h_h(1., c, h[n1], h[n2], q);
        r[n1 * 3 + 1] += dely * q[0];
        r[n2 * 3 + 1] += dely * q[1];
        r[n1 * 3 + 2] += delx * q[0];
        r[n2 * 3 + 2] += delx * q[1];
    }
}

__device__ __forceinline__ void ig_average(double r[9], double djac, const double h[3], const V2 w[3]) {  // :643
    double t1 = (h[0] + h[1] + h[2]) / 3.0;
    double t2 = (w[0].x + w[1].x + w[2].x) / 3.0;
    double t3 = (w[0].y + w[1].y + w[2].y) / 3.0;
    r[0] += djac * t1; r[1] += djac * t2; r[2] += djac * t3;
}

__device__ __forceinline__ void ig_gls_convection(double r[9], const V2 g[3], double djac, double dt, double c,
                                                  const double f[3], const V2 w[3]) {  // :700
    double h_avg = SW2_ONE_3 * (f[0] + f[1] + f[2]);
    double u_avg = SW2_ONE_3 * (w[0].x + w[1].x + w[2].x);
    double v_avg = SW2_ONE_3 * (w[0].y + w[1].y + w[2].y);
    double dhdx = g[0].x * f[0] + g[1].x * f[1] + g[2].x * f[2];
    double dhdy = g[0].y * f[0] + g[1].y * f[1] + g[2].y * f[2];
    double dudx = g[0].x * w[0].x + g[1].x * w[1].x + g[2].x * w[2].x;
    double dudy = g[0].y * w[0].x + g[1].y * w[1].x + g[2].y * w[2].x;
    double dvdx = g[0].x * w[0].y + g[1].x * w[1].y + g[2].x * w[2].y;
    double dvdy = g[0].y * w[0].y + g[1].y * w[1].y + g[2].y * w[2].y;
    r[0] += djac * dt * c * (u_avg * dhdx + h_avg * dudx + v_avg * dhdy + h_avg * dvdy);
    r[1] += djac * dt * c * (u_avg * dudx + v_avg * dudy);
    r[2] += djac * dt * c * (u_avg * dvdx + v_avg * dvdy);
}

// ----------------------------------------------------------------------------
// wrapped terms
__device__ __forceinline__ void wd_average(const V2 x[3], const double h[3], const V2 v[3], double djac,
                                           double* havg, V2* vavg) {  // fe_sw2_wd_average, :40
    double av[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double factor = wd_wrap(av, x, h, djac, false,
        [&](double* r) { ig_average(r, djac, h, v); },
        [&](const Cut& c, double* nr) { V2 nv[3]; cut_interp(c, v, nv); ig_average(nr, c.area, c.nh, nv); });
    *havg = 0.; vavg->x = 0.; vavg->y = 0.;
    if (factor > 0.0) {
        double wet_area = djac * factor;
        *havg = av[0] / wet_area;
        vavg->x = av[1] / wet_area;
        vavg->y = av[2] / wet_area;
    }
}

// fe_sw2_temporal, sw2_body_resid.c:1195
__device__ __forceinline__ void temporal(double r[9], const V2 x[3], double djac, const double h[3], const V2 v[3],
                                         double wd_fac, double dt_factor, bool add_continuity) {
    double con = dt_factor * wd_fac;
    double rhs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double uh[3], vh[3], rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < 3; i++) { uh[i] = v[i].x * dmax_(h[i], 1e-6); vh[i] = v[i].y * dmax_(h[i], 1e-6); }
    wd_wrap(rhs, x, h, djac, true,
        [&](double* q) { ig_continuity_temporal(q, djac, dt_factor, h); },
        [&](const Cut& c, double* nr) { ig_continuity_temporal(nr, c.area, dt_factor, c.nh); });
    tri_phi_f_lump(djac, con, uh, rx);
    tri_phi_f_lump(djac, con, vh, ry);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (add_continuity) r[i * 3] += rhs[i * 3];
        r[i * 3 + 1] += rx[i];
        r[i * 3 + 2] += ry[i];
    }
}

// ----------------------------------------------------------------------------
// Triangle data as the residual reads it.  `h,u,v` may carry a perturbation.
struct TriData {
    V2 x[3]; double z[3];
    V2 g[3]; double djac;
    double h[3]; V2 vel[3];      // t^{n+1}
    double ho[3]; V2 velo[3];    // t^n
    double hoo[3]; V2 veloo[3];  // t^{n-1}
    int wd_flag;
};

// fe_sw2_body_resid for a triangle.  PRESSURE is false exactly when the
// reference perturbs a velocity (sw2_body_resid.c:124-129).
template <bool PRESSURE>
__device__ __forceinline__ void body_resid(const TriData& T, double dt, double alpha, double grav, double r[9]) {
    const V2* x = T.x;
    const V2* g = T.g;
    const double djac = T.djac;
#pragma unroll
    for (int i = 0; i < 9; i++) r[i] = 0.0;

    V2 grad_z = {0, 0}, grad_h = {0, 0};
#pragma unroll
    for (int i = 0; i < 3; i++) { grad_z.x += T.z[i] * g[i].x; grad_z.y += T.z[i] * g[i].y; }
#pragma unroll
    for (int i = 0; i < 3; i++) { grad_h.x += T.h[i] * g[i].x; grad_h.y += T.h[i] * g[i].y; }

    double h_wd, oh_wd;
    V2 vel_wd, ovel_wd;
    wd_average(x, T.h, T.vel, djac, &h_wd, &vel_wd);
    wd_average(x, T.ho, T.velo, djac, &oh_wd, &ovel_wd);
    double factor = wd_factor(x, T.h, djac);
    double factor_old = wd_factor(x, T.ho, djac);
    double factor_older = wd_factor(x, T.hoo, djac);
    double vel_wd_mag = sqrt(vel_wd.x * vel_wd.x + vel_wd.y * vel_wd.y);
    const double roughness = 0.002;   // sw2_body_resid.c:241

    {   // advection, :413-434
        double rhs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double c = -1; c *= dt;
        wd_wrap(rhs, x, T.h, djac, true,
            [&](double* q) { ig_convection(q, g, djac, c, T.h, T.vel); },
            [&](const Cut& cu, double* nr) { V2 ng[3], nv[3]; cut_grad(cu, ng); cut_interp(cu, T.vel, nv);
                                             ig_convection(nr, ng, cu.area, c, cu.nh, nv); });
#pragma unroll
        for (int i = 0; i < 9; i++) r[i] += rhs[i];
    }
    // temporal, :456-463
    temporal(r, x, djac, T.h, T.vel, factor, (1. + alpha / 2.), true);
    temporal(r, x, djac, T.ho, T.velo, factor_old, (-1.) * (1. + alpha), T.wd_flag != 2);
    temporal(r, x, djac, T.hoo, T.veloo, factor_older, (alpha / 2.), T.wd_flag != 2);
    // friction, :520-539
    double resistance = roughness / (2.0 * grav);
    {
        double fx[3], fy[3], rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
#pragma unroll
        for (int i = 0; i < 3; i++) {
            double t = sqrt(T.vel[i].x * T.vel[i].x + T.vel[i].y * T.vel[i].y);
            fx[i] = T.vel[i].x * t; fy[i] = T.vel[i].y * t;
        }
        double t1 = dt * grav * resistance * factor;
        tri_phi_f(djac, t1, fx, rx);
        tri_phi_f(djac, t1, fy, ry);
#pragma unroll
        for (int i = 0; i < 3; i++) { r[3 * i + 1] += rx[i]; r[3 * i + 2] += ry[i]; }
    }
    V2 bed_stress = {resistance * vel_wd.x * vel_wd_mag, resistance * vel_wd.y * vel_wd_mag};
    if (PRESSURE) {   // :710-804
        double rhs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double t1 = -SW2_ONE_2 * grav * dt;
        wd_wrap(rhs, x, T.h, djac, true,
            [&](double* q) { ig_pressure(q, g, djac, t1, T.h); },
            [&](const Cut& cu, double* nr) { V2 ng[3]; cut_grad(cu, ng); ig_pressure(nr, ng, cu.area, t1, cu.nh); });
#pragma unroll
        for (int i = 0; i < 9; i++) r[i] += rhs[i];
        double r2[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double t2 = grav * dt;
        wd_wrap(r2, x, T.h, djac, true,
            [&](double* q) { ig_body_force(q, djac, t2, T.h, grad_z); },
            [&](const Cut& cu, double* nr) { ig_body_force(nr, cu.area, t2, cu.nh, grad_z); });
#pragma unroll
        for (int i = 0; i < 9; i++) r[i] += r2[i];
        double r3[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double t3 = SW2_ONE_2 * dt * grav;
        wd_wrap(r3, x, T.h, djac, true,
            [&](double* q) { ig_boundary_pressure(q, x, t3, T.h); },
            [&](const Cut& cu, double* nr) { ig_boundary_pressure(nr, cu.nx, t3, cu.nh); });
#pragma unroll
        for (int i = 0; i < 9; i++) r[i] += r3[i];
    }
    // SUPG, :921-1142 (tau from fe_get_supg_tau_sw, src/tools/get_supg_tau.c:43, le = sqrt(area))
    if (fabs(h_wd) >= SW2_SMALL) {
        const double g_factor = (1 + 0.0) * grav;
        double hden = dmax_(h_wd, SW2_NOT_QUITE_SMALL);
        // a wet fraction that rounds below zero (an almost empty wet part) would make this NaN, as in
        // the reference; clamped at zero, which changes nothing where the reference is finite
        double le = sqrt(djac * (factor_old > 0.0 ? factor_old : 0.0));
        double cel2 = g_factor * hden;
        if (hden <= 0.0) cel2 = 0.;
        double sr = sqrt(vel_wd.x * vel_wd.x + vel_wd.y * vel_wd.y + cel2 + SW2_SMALL);
        double tau = 0.5 * le / sr;
        double dfdt[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        wd_wrap(dfdt, x, T.ho, djac, false,
            [&](double* q) { ig_average(q, djac, T.ho, T.velo); },
            [&](const Cut& cu, double* nr) { V2 nv[3]; cut_interp(cu, T.velo, nv); ig_average(nr, cu.area, cu.nh, nv); });
        double dudt = -dfdt[1], dvdt = -dfdt[2], dhdt = -dfdt[0];
        double dfn[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        wd_wrap(dfn, x, T.h, djac, false,
            [&](double* q) { ig_average(q, djac, T.h, T.vel); },
            [&](const Cut& cu, double* nr) { V2 nv[3]; cut_interp(cu, T.vel, nv); ig_average(nr, cu.area, cu.nh, nv); });
        dudt += dfn[1]; dvdt += dfn[2]; dhdt += dfn[0];
        double adv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double fac = wd_wrap(adv, x, T.h, djac, false,
            [&](double* q) { ig_gls_convection(q, g, djac, dt, 1, T.h, T.vel); },
            [&](const Cut& cu, double* nr) { V2 ng[3], nv[3]; double nf[3]; cut_grad(cu, ng); cut_interp(cu, T.vel, nv);
                                             cut_interp(cu, T.h, nf); ig_gls_convection(nr, ng, cu.area, dt, 1, nf, nv); });
        double x_pressure = g_factor * (grad_h.x + grad_z.x) * dt * fac + 0.0 * dt * fac;
        double y_pressure = g_factor * (grad_h.y + grad_z.y) * dt * fac + 0.0 * dt * fac;
        double x_friction = grav * bed_stress.x * dt * fac;
        double y_friction = grav * bed_stress.y * dt * fac;
        double c_eq = dhdt + adv[0] + fac * 0.0 * djac * dt;
        double x_eq = dudt + adv[1] + (x_pressure + x_friction / hden) * djac + (0.0 - 0.0 / hden) * djac * fac * dt;
        double y_eq = dvdt + adv[2] + (y_pressure + y_friction / hden) * djac + (0.0 - 0.0 / hden) * djac * fac * dt;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            double rc = (g[i].x * (tau * vel_wd.x * c_eq + tau * h_wd * x_eq) +
                         g[i].y * (tau * vel_wd.y * c_eq + tau * h_wd * y_eq));
            double rx = (g[i].x * (tau * g_factor * h_wd * c_eq + tau * vel_wd.x * h_wd * x_eq) +
                         g[i].y * (tau * vel_wd.y * h_wd * x_eq));
            double ry = (g[i].y * (tau * g_factor * h_wd * c_eq + tau * vel_wd.y * h_wd * y_eq) +
                         g[i].x * (tau * vel_wd.x * h_wd * y_eq));
            r[3 * i] += rc; r[3 * i + 1] += rx; r[3 * i + 2] += ry;
        }
    }
}

// ----------------------------------------------------------------------------
// boundary segments
struct SegData {
    V2 n; double djac;
    double h[2]; V2 vel[2];
    double z0;  // bed elevation of the segment's first node
    int kind;   // 0 velocity (fe_sw2_bc_vel), 1 depth (fe_sw2_bc_h), 2 discharge, 3 tailwater, 4 outflow, 5 flux
};

// The boundary values of one step, shared by every segment of a kind.
struct SegBC {
    double depth, vx, vy;   // series 0, 1, 2: fe_sw2_bc_h's depth, fe_sw2_bc_vel's velocity
    double q_series;        // discharge string's series value (sw2_bc_discharge.c.bk:161)
    double conveyance;      // discharge string's conveyance (sstr_value.h:63)
    double rough_height;    // equivalent roughness height of the boundary strings (FRICTION.eqrheight)
    double tail_elev;       // tailwater elevation series value (sw2_bc_tailwater.c.bk:154)
    double flux_series;     // flux string's series value (sw2_bc_flux.c.bk:152)
};

// fr_bedshstr_drag_coef, src/friction/fr_bedshstr_drag_coef.c:18-42
__device__ __forceinline__ double bedshstr_drag_coef(double depth, double rh) {
    depth = depth > 1.E-8 ? depth : 1.E-8;
    rh = rh > 1.E-8 ? rh : 1.E-8;
    double depth_rh = (rh > 29.7 * depth) ? 1. / 29.7 : depth / rh;
    double bta = 29.7 * depth_rh;
    double phi = pow((.4 * bta) / ((bta + 1) * (log(bta + 1) - 1) + 1), 2.);
    return 2. * phi;
}

// fe_sw2_get_roughness (src/models/sw2/sw2_get_roughness.c:24-49) for a string with
// neither vegetation nor ice: the bed-shear drag of its roughness height, else zero drag
__device__ __forceinline__ double bc_roughness(double depth, double rh) {
    return rh > SW2_SMALL ? bedshstr_drag_coef(depth, rh) : 0.0;
}

// integrate_line_phi (src/fe/fe_integrals_1d.c:54)
__device__ __forceinline__ void line_phi(double djac, double c, double q[2]) {
    double t1 = SW2_ONE_2 * djac * c;
    q[0] += t1; q[1] += t1;
}

// integrate_line_phi_f (src/fe/fe_integrals_1d.c:67)
__device__ __forceinline__ void line_phi_f(double djac, double c, const double f[2], double q[2]) {
    double t1 = SW2_ONE_6 * djac * c;
    q[0] += t1 * (2 * f[0] + f[1]);
    q[1] += t1 * (f[0] + 2 * f[1]);
}

// fe_sw2_1d_explicit_flow, src/fe/fe_sw2_boundary_integrals.c:56-82 (flux < 0 is inflow)
__device__ __forceinline__ void explicit_flow(double r[6], V2 n, double djac, double dt, double flux, double h_avg,
                                              const double u[2], const double v[2]) {
    double rc[2] = {0., 0.}, rx[2] = {0., 0.}, ry[2] = {0., 0.};
    line_phi(djac, 1., rc);
    if (flux < 0) {
        double u_star = 0., v_star = 0.;
        if (h_avg > 0) {
            u_star = flux * n.x / h_avg;
            v_star = flux * n.y / h_avg;
        }
        line_phi(djac, u_star, rx);
        line_phi(djac, v_star, ry);
    } else {
        line_phi_f(djac, 1., u, rx);
        line_phi_f(djac, 1., v, ry);
    }
    double t1 = dt * flux;
#pragma unroll
    for (int i = 0; i < 2; i++) { r[i * 3] += t1 * rc[i]; r[i * 3 + 1] += t1 * rx[i]; r[i * 3 + 2] += t1 * ry[i]; }
}

// fe_sw2_1d_wall_friction, src/fe/fe_sw2_boundary_integrals.c:205-219
__device__ __forceinline__ void wall_friction(double r[6], V2 n, double djac, double dt, const double u[2],
                                              const double v[2], const double res[2]) {
    double rx[2] = {0., 0.}, ry[2] = {0., 0.};
    line_phi_f(djac, fabs(n.y), u, rx);
    line_phi_f(djac, fabs(n.x), v, ry);
#pragma unroll
    for (int i = 0; i < 2; i++) { r[i * 3 + 1] += dt * res[i] * rx[i]; r[i * 3 + 2] += dt * res[i] * ry[i]; }
}

// fe_sw2_1d_implicit_flow, src/fe/fe_sw2_boundary_integrals.c:125
__device__ __forceinline__ void implicit_flow(double r[6], V2 n, double djac, double dt, const V2 v[2], const double h[2]) {
    double rc[2] = {0, 0}, rx[2] = {0, 0}, ry[2] = {0, 0};
    double u1 = v[0].x, u2 = v[1].x, v1 = v[0].y, v2 = v[1].y, h1 = h[0], h2 = h[1];
    double ur1 = v[0].x, ur2 = v[1].x, vr1 = v[0].y, vr2 = v[1].y;
    double d0 = v[0].x * n.x + v[0].y * n.y, d1 = v[1].x * n.x + v[1].y * n.y;
    if (d0 < SW2_SMALL) { ur1 = 0.; vr1 = 0.; }
    if (d1 < SW2_SMALL) { ur2 = 0.; vr2 = 0.; }
    {   // integrate_line_phi_h_v_dot_n(djac, 1., h, v, nrml)
        double t1 = djac * SW2_ONE_12 * 1.;
        rc[0] += t1 * (n.x * ((3 * h[0] + h[1]) * v[0].x + (h[0] + h[1]) * v[1].x) + n.y * ((3 * h[0] + h[1]) * v[0].y + (h[0] + h[1]) * v[1].y));
        rc[1] += t1 * (n.x * ((h[0] + h[1]) * v[0].x + (h[0] + 3 * h[1]) * v[1].x) + n.y * ((h[0] + h[1]) * v[0].y + (h[0] + 3 * h[1]) * v[1].y));
    }
    line_phi_f_g_h(djac, n.x, ur1, ur2, u1, u2, h1, h2, rx);
    line_phi_f_g_h(djac, n.y, vr1, vr2, v1, v2, h1, h2, ry);
    line_phi_f_g_h(djac, n.y, ur1, ur2, v1, v2, h1, h2, rx);
    line_phi_f_g_h(djac, n.x, vr1, vr2, u1, u2, h1, h2, ry);
#pragma unroll
    for (int i = 0; i < 2; i++) { r[i * 3] += dt * rc[i]; r[i * 3 + 1] += dt * rx[i]; r[i * 3 + 2] += dt * ry[i]; }
}

// fe_sw2_1d_pressure, fe_sw2_boundary_integrals.c:260
__device__ __forceinline__ void pressure_1d(double r[6], V2 n, double djac, double dt, const double h[2], double g) {
    double q[2] = {0., 0.};
    line_phi_h_h(djac, 1., h[0], h[1], q);
    double t1 = dt * SW2_ONE_2 * g;
#pragma unroll
    for (int i = 0; i < 2; i++) { r[i * 3 + 1] += t1 * n.x * q[i]; r[i * 3 + 2] += t1 * n.y * q[i]; }
}

template <bool PRESSURE>
__device__ __forceinline__ void seg_resid(const SegData& S, double dt, double grav, const SegBC& B, double r[6]) {
#pragma unroll
    for (int i = 0; i < 6; i++) r[i] = 0.0;
    if (S.kind == 0) {   // sw2_bc_vel.c:147-159: the boundary velocity replaces u, v
        V2 v[2] = {{B.vx, B.vy}, {B.vx, B.vy}};
        implicit_flow(r, S.n, S.djac, dt, v, S.h);
    } else if (S.kind == 1) {   // sw2_bc_h.c:150-172
        double dep[2] = {B.depth, B.depth};
        if (dep[0] < SW2_SMALL || dep[1] < SW2_SMALL || S.h[0] < SW2_SMALL || S.h[1] < SW2_SMALL) return;
        implicit_flow(r, S.n, S.djac, dt, S.vel, dep);
        if (PRESSURE) {
            pressure_1d(r, S.n, S.djac, dt, dep, grav);
            pressure_1d(r, S.n, S.djac, dt, S.h, -grav);
        }
    } else if (S.kind == 2) {   // sw2_bc_discharge.c.bk:111-172
        double u_tan = SW2_ONE_2 * (S.vel[0].x + S.vel[1].x) * S.n.y - SW2_ONE_2 * (S.vel[0].y + S.vel[1].y) * S.n.x;
        double mag_utan = fabs(u_tan);
        double u[2] = {S.vel[0].x, S.vel[1].x}, v[2] = {S.vel[0].y, S.vel[1].y};
        double h_avg = SW2_ONE_2 * (S.h[0] + S.h[1]);
        if (h_avg < SW2_SMALL) h_avg = SW2_SMALL;
        double res[2] = {SW2_ONE_2 * bc_roughness(S.h[0], B.rough_height) * mag_utan,
                         SW2_ONE_2 * bc_roughness(S.h[1], B.rough_height) * mag_utan};
        if (S.h[0] < SW2_SMALL || S.h[1] < SW2_SMALL) return;
        // the discharge law takes the first node's head at both nodes (.bk:164-167)
        double fact = -1.0 * B.q_series * sqrt(2. * grav / bc_roughness(S.h[0], B.rough_height)) / B.conveyance;
        double d0 = fact * pow(S.h[0], 1.5);
        fact = -1.0 * B.q_series * sqrt(2. * grav / bc_roughness(S.h[1], B.rough_height)) / B.conveyance;
        double d1 = fact * pow(S.h[0], 1.5);
        explicit_flow(r, S.n, S.djac, dt, SW2_ONE_2 * (d0 + d1), h_avg, u, v);
        wall_friction(r, S.n, S.djac, dt, u, v, res);
    } else if (S.kind == 4) {   // sw2_bc_outflow.c.bk:144: implicit flow with the computed depth and velocity
        implicit_flow(r, S.n, S.djac, dt, S.vel, S.h);
    } else if (S.kind == 5) {   // sw2_bc_flux.c.bk:151-153: the series value as a unit inflow
        double u[2] = {S.vel[0].x, S.vel[1].x}, v[2] = {S.vel[0].y, S.vel[1].y};
        double h_avg = SW2_ONE_2 * (S.h[0] + S.h[1]);
        if (h_avg < SW2_SMALL) h_avg = SW2_SMALL;
        explicit_flow(r, S.n, S.djac, dt, -1.0 * B.flux_series, h_avg, u, v);
    } else {                    // kind 3: sw2_bc_tailwater.c.bk:152-170
        // depth below the tailwater elevation at the first node, used at both nodes (.bk:155-156)
        double dep[2] = {B.tail_elev - S.z0, B.tail_elev - S.z0};
        if (dep[0] < SW2_SMALL || dep[1] < SW2_SMALL || S.h[0] < SW2_SMALL || S.h[1] < SW2_SMALL) return;
        implicit_flow(r, S.n, S.djac, dt, S.vel, S.h);
        if (PRESSURE) {
            pressure_1d(r, S.n, S.djac, dt, dep, grav);
            pressure_1d(r, S.n, S.djac, dt, S.h, -grav);
        }
    }
}

// NUM_DIFF_EPSILON (macro.h:669) with the 1e-4 floor of perturb_var (assemble_jacobian.c:313)
__device__ __forceinline__ double fd_eps(double u) {
    double e = fabs(u) * (1. + 1e-4);
    e -= fabs(u);
    if (e < 1e-4) e = 1e-4;
    return e;
}

}  // namespace sw2
