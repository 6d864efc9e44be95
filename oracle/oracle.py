"""Test infrastructure: ctypes front-end of the CPU restatement (liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import this.
``OracleModel`` wraps one SW2 case: geometry, the bit-exact CSR sparsity, and the
residual / Jacobian / linear-system / Newton routines of sw2_oracle.c.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Model(C.Structure):
    _fields_ = [
        ("nnodes", C.c_int), ("ntri", C.c_int), ("nseg", C.c_int),
        ("xyz", _dp), ("tri", _ip), ("seg", _ip), ("seg_kind", _ip),
        ("tri_djac", _dp), ("tri_grad", _dp), ("seg_djac", _dp), ("seg_nrml", _dp),
        ("ndof", C.c_int), ("nnz", C.c_int), ("indptr", _ip), ("cols", _ip),
        ("gravity", C.c_double), ("dt", C.c_double), ("tau_temporal", C.c_double),
        ("bc_depth", C.c_double), ("bc_vx", C.c_double), ("bc_vy", C.c_double),
        ("wd_flag", _ip),
        ("bc_qs", C.c_double), ("bc_convey", C.c_double), ("bc_rough", C.c_double), ("bc_tail", C.c_double),
        ("bc_flux", C.c_double),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True, capture_output=True)
        _LIB = C.CDLL(path)
    return _LIB


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def series_average(times, values, t1, t2):
    """Step average of a piecewise-linear series over [t1, t2]: the trapezoid
    integral divided by t2 - t1 (sseries_set_values_average, src/structs/sseries/sseries.c:622-667,
    with sseries_get_interval :746 and tc_eval_series, src/tools/tc_eval_series.c)."""
    eps = np.finfo(np.float64).eps

    def interval(t):
        n = len(times)
        i = 0
        while i < n - 1 and t >= times[i] * (1.0 - eps):
            i += 1
        return i - 1

    def evalv(iv, t):
        if iv == len(times) - 1:
            return values[-1]
        lt, rt, lv, rv = times[iv], times[iv + 1], values[iv], values[iv + 1]
        delta = rt - lt
        theta = (rt - t) / delta
        return theta * lv + (1.0 - theta) * rv

    def trap(lv, rv, lt, rt):  # tc_trap_area, src/tools/tc_trap_area.c
        delta = rt - lt
        return 0.0 if delta < eps else (lv + rv) * 0.5 * delta

    i1, i2 = interval(t1), interval(t2)
    v1, v2 = evalv(i1, t1), evalv(i2, t2)
    if i1 == i2:
        area = trap(v1, v2, t1, t2)
    else:
        area = 0.0
        for k in range(i1 + 1, i2):
            area += trap(values[k], values[k + 1], times[k], times[k + 1])
        area += trap(v1, values[i1 + 1], t1, times[i1 + 1])
        area += trap(values[i2], v2, times[i2], t2)
    return area / (t2 - t1)


class OracleModel:
    def __init__(self, case, tau_temporal=0.0):
        L = lib()
        self.case = case
        V, T, S = case.nnodes, case.ntri, case.nseg
        self.xyz = np.ascontiguousarray(case.xyz, dtype=np.float64).ravel()
        self.tri = np.ascontiguousarray(case.tri, dtype=np.int32).ravel()
        self.seg = np.ascontiguousarray(case.seg, dtype=np.int32).ravel() if S else np.zeros(2, np.int32)
        self.seg_kind = np.ascontiguousarray(case.seg_kind, dtype=np.int32) if S else np.zeros(1, np.int32)
        self.tri_djac = np.zeros(T); self.tri_grad = np.zeros(6 * T)
        self.seg_djac = np.zeros(max(S, 1)); self.seg_nrml = np.zeros(2 * max(S, 1))
        L.sw2o_geometry(V, T, S, _d(self.xyz), _i(self.tri), _i(self.seg), _d(self.tri_djac), _d(self.tri_grad),
                        _d(self.seg_djac), _d(self.seg_nrml))
        nnz = L.sw2o_sparsity_nnz(V, T, S, _i(self.tri), _i(self.seg))
        self.indptr = np.zeros(3 * V + 1, np.int32); self.cols = np.zeros(nnz, np.int32)
        L.sw2o_sparsity(V, T, S, _i(self.tri), _i(self.seg), _i(self.indptr), _i(self.cols))
        self.wd_flag = np.zeros(T, np.int32)
        m = _Model()
        m.nnodes, m.ntri, m.nseg = V, T, S
        m.xyz, m.tri, m.seg, m.seg_kind = _d(self.xyz), _i(self.tri), _i(self.seg), _i(self.seg_kind)
        m.tri_djac, m.tri_grad, m.seg_djac, m.seg_nrml = _d(self.tri_djac), _d(self.tri_grad), _d(self.seg_djac), _d(self.seg_nrml)
        m.ndof, m.nnz, m.indptr, m.cols = 3 * V, nnz, _i(self.indptr), _i(self.cols)
        m.gravity, m.dt, m.tau_temporal = case.gravity, case.dt, float(tau_temporal)
        m.wd_flag = _i(self.wd_flag)
        m.bc_convey = float(getattr(case, "bc_conveyance", 1.0))
        m.bc_rough = float(getattr(case, "bc_rough_height", 0.0))
        self.m = m
        self.ndof, self.nnz = 3 * V, nnz
        self.set_bc_window(case.t0, case.t0 + case.dt)

    # -- forcing
    def bc_values(self, t1, t2):
        s = self.case.series
        out = [series_average(*s[0], t1, t2)]
        for k in (1, 2):
            out.append(series_average(*s[k], t1, t2) if k in s else 0.0)
        return out

    def set_bc_window(self, t1, t2):
        self.m.bc_depth, self.m.bc_vx, self.m.bc_vy = self.bc_values(t1, t2)
        s = self.case.series
        self.m.bc_qs = series_average(*s[3], t1, t2) if 3 in s else 0.0
        self.m.bc_tail = series_average(*s[4], t1, t2) if 4 in s else 0.0
        self.m.bc_flux = series_average(*s[5], t1, t2) if 5 in s else 0.0

    # -- kernels
    def wd_flags(self, sol, sol_old):
        lib().sw2o_wd_flags(C.byref(self.m), _d(sol), _d(sol_old))
        return self.wd_flag.copy()

    def elem_resid(self, sol, sol_old, sol_older):
        et = np.zeros(9 * self.case.ntri); es = np.zeros(6 * max(self.case.nseg, 1))
        lib().sw2o_elem_resid_all(C.byref(self.m), _d(sol), _d(sol_old), _d(sol_older), _d(et), _d(es))
        return et, es[: 6 * self.case.nseg]

    def elem_jac(self, sol, sol_old, sol_older):
        jt = np.zeros(81 * self.case.ntri); js = np.zeros(36 * max(self.case.nseg, 1))
        lib().sw2o_elem_jac_all(C.byref(self.m), _d(sol), _d(sol_old), _d(sol_older), _d(jt), _d(js))
        return jt, js[: 36 * self.case.nseg]

    def residual(self, sol, sol_old, sol_older):
        r = np.zeros(self.ndof)
        lib().sw2o_assemble_residual(C.byref(self.m), _d(sol), _d(sol_old), _d(sol_older), _d(r))
        return r

    def jacobian(self, sol, sol_old, sol_older):
        v = np.zeros(self.nnz)
        lib().sw2o_assemble_jacobian(C.byref(self.m), _d(sol), _d(sol_old), _d(sol_older), _d(v))
        return v

    def check_diag(self, vals, bc_mask):
        lib().sw2o_check_diag(C.byref(self.m), _d(vals), _i(bc_mask))

    def apply_dirichlet(self, bc_mask, vals, res):
        lib().sw2o_apply_dirichlet(C.byref(self.m), _i(bc_mask), _d(vals), _d(res))

    def scale_system(self, vals, b, x):
        s = np.zeros(self.ndof)
        lib().sw2o_scale_system(C.byref(self.m), _d(vals), _d(b), _d(x), _d(s))
        return s

    def spmv(self, vals, x):
        y = np.zeros(self.ndof)
        lib().sw2o_spmv(self.ndof, _i(self.indptr), _i(self.cols), _d(vals), _d(x), _d(y))
        return y

    def bicgstab(self, vals, x, b, scale_vect, max_it=100, tol=1e-11):
        return lib().sw2o_bicgstab_bj(self.ndof, _i(self.indptr), _i(self.cols), _d(vals), _d(x), _d(b),
                                      _d(scale_vect), max_it, C.c_double(tol))

    def grid_mass(self, sol, density=1.0):
        f = lib().sw2o_grid_mass
        f.restype = C.c_double
        return f(C.byref(self.m), _d(sol), C.c_double(density))

    def elem_mass(self, sol):
        f = lib().sw2o_elem_mass
        f.restype = C.c_double
        return np.array([f(C.byref(self.m), _d(sol), e) for e in range(self.case.ntri)])

    def boundary_mass_flux(self, sol, density=1.0, dt=None, first_seg_length=False):
        f = lib().sw2o_boundary_mass_flux
        f.restype = C.c_double
        dt = self.case.dt if dt is None else dt
        return f(C.byref(self.m), _d(sol), C.c_double(density), C.c_double(dt), int(first_seg_length))

    def newton(self, sol, sol_old, sol_older, bc_mask, dirichlet, krylov_max_it=100, krylov_tol=1e-11):
        c = self.case
        stats = np.zeros(5)
        lib().sw2o_newton(C.byref(self.m), _d(sol), _d(sol_old), _d(sol_older), _i(bc_mask), _d(dirichlet),
                          C.c_double(c.tol_nonlin), C.c_double(c.inc_nonlin), c.max_nonlin_it, 5, krylov_max_it,
                          C.c_double(krylov_tol), _d(stats))
        return {"newton_its": int(stats[0]), "krylov_its": int(stats[1]), "resid_max": stats[2], "ok": bool(stats[3]),
                "linesearch_cuts": int(stats[4])}

    def run(self, nsteps=None, krylov_max_it=100, krylov_tol=1e-11):
        """Time loop of src/timeloop/time_loop.c:14-89: rotate levels, average the
        forcing over the step, one Newton solve per step; stops at a failed step."""
        c = self.case
        nsteps = c.nsteps if nsteps is None else nsteps
        sol = c.sol0.astype(np.float64).copy(); sol_old = sol.copy(); sol_older = sol.copy()
        bc_mask = np.zeros(self.ndof, np.int32); dirichlet = np.zeros(self.ndof)
        t = c.t0
        hist = []
        for _ in range(nsteps):
            t += c.dt
            sol_older[:] = sol_old; sol_old[:] = sol
            self.set_bc_window(t - c.dt, t)
            st = self.newton(sol, sol_old, sol_older, bc_mask, dirichlet, krylov_max_it, krylov_tol)
            hist.append(st)
            if not st["ok"]:
                break
        return sol, hist
