"""ctypes binding of the C ABI in include/adh_sw2_gpu.h.

This is the Python face of the drop-in boundary: every call goes through the
extern "C" entry points of the in-tree libadh_sw2_gpu.so.  There is no CPU
fallback -- if the library or a GPU is missing, construction fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libadh_sw2_gpu.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

# every symbol declared in include/adh_sw2_gpu.h
EXPORTED = [
    "sw2g_create", "sw2g_destroy", "sw2g_last_error", "sw2g_default_opts", "sw2g_sizes", "sw2g_get_sparsity",
    "sw2g_set_step", "sw2g_set_bc_structures", "sw2g_set_bc_flux", "sw2g_wd_flags", "sw2g_elem_resid", "sw2g_elem_jac", "sw2g_assemble_residual",
    "sw2g_assemble_jacobian", "sw2g_prepare_system", "sw2g_solve_linear_sys_bcgstab", "sw2g_fe_newton",
    "sw2g_load_state", "sw2g_store_state", "sw2g_set_guess", "sw2g_step", "sw2g_device_state", "sw2g_stream",
    "sw2g_set_profiling", "sw2g_get_profile", "sw2g_reset_profile", "sw2g_time_kernel",
    "sw2g_assemble_residual_noalloc", "sw2g_grid_mass", "sw2g_undo_step",
    "sw2g_assemble_residual_wd", "sw2g_assemble_jacobian_wd", "sw2g_precond_info",
    # include/adh_sw2_gnn.h (learned initial guess)
    "sw2n_agg_fwd", "sw2n_agg_bwd", "sw2n_dense_fwd", "sw2n_dense_bwd", "sw2n_adam", "sw2n_to_bf16",
    "sw2n_features", "sw2n_targets", "sw2n_mse", "sw2n_apply_guess", "sw2n_smooth3", "sw2n_smooth3_adj",
]


class Mesh(C.Structure):
    _fields_ = [("nnodes", C.c_int), ("ntri", C.c_int), ("nseg", C.c_int), ("xyz", _dp), ("tri", _ip),
                ("seg", _ip), ("seg_kind", _ip), ("indptr", _ip), ("cols", _ip), ("gravity", C.c_double)]


class NewtonOpts(C.Structure):
    _fields_ = [("tol_nonlin", C.c_double), ("inc_nonlin", C.c_double), ("max_nonlin_it", C.c_int),
                ("max_linesearch_cuts", C.c_int), ("krylov_max_it", C.c_int), ("krylov_tol", C.c_double),
                ("krylov_precision", C.c_int), ("refine_tol", C.c_double), ("max_refine", C.c_int),
                ("use_guess", C.c_int), ("precond", C.c_int), ("krylov_method", C.c_int),
                ("tol_nonlin_rel", C.c_double), ("krylov_basis_precision", C.c_int), ("krylov_restart", C.c_int),
                ("amg_chunks", C.c_int), ("tol_nonlin_min", C.c_double)]

PC_BLOCK_JACOBI = 0
PC_BILU0 = 1
PC_AMG = 2
KRYLOV_BICGSTAB = 0
KRYLOV_GMRES = 1


class NewtonStats(C.Structure):
    _fields_ = [("newton_its", C.c_int), ("krylov_its", C.c_int), ("linesearch_cuts", C.c_int),
                ("refine_passes", C.c_int), ("success", C.c_int), ("krylov_breakdowns", C.c_int),
                ("resid_max", C.c_double), ("resid_l2", C.c_double), ("inc_max", C.c_double),
                ("initial_resid_max", C.c_double), ("prev_resid_max", C.c_double), ("guess_used", C.c_int),
                ("initial_resid_l2", C.c_double), ("guess_fallback", C.c_int), ("linear_unconverged", C.c_int),
                ("tol_used", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_LIB = None


def lib():
    """Load the in-tree CUDA library (building it first if it is absent)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _b
            _b.build()
        L = C.CDLL(LIB_PATH)
        L.sw2g_last_error.restype = C.c_char_p
        L.sw2g_stream.restype = C.c_void_p
        L.sw2g_create.argtypes = [C.POINTER(Mesh), C.c_void_p, C.POINTER(C.c_void_p)]
        for name in ("sw2g_destroy",):
            getattr(L, name).argtypes = [C.c_void_p]
        _LIB = L
    return _LIB


ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_MESH, ERR_NONFINITE = -1, -2, -3, -4, -5   # SW2G_ERR_* of adh_sw2_gpu.h


class SW2Error(RuntimeError):
    """A non-zero status from the C ABI; ``rc`` holds the SW2G_ERR_* code (None when raised
    by host code)."""

    def __init__(self, msg, rc=None):
        super().__init__(msg)
        self.rc = rc


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def default_opts(**kw) -> NewtonOpts:
    o = NewtonOpts()
    lib().sw2g_default_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class SW2Model:
    """One SW2 mesh on the GPU (a ``sw2g_model``)."""

    def __init__(self, case, stream=None, check_csr=None):
        L = lib()
        self.case = case
        self._keep = []
        xyz = np.ascontiguousarray(case.xyz, dtype=np.float64).ravel()
        tri = np.ascontiguousarray(case.tri, dtype=np.int32).ravel()
        seg = np.ascontiguousarray(case.seg, dtype=np.int32).ravel() if case.nseg else np.zeros(2, np.int32)
        kind = np.ascontiguousarray(case.seg_kind, dtype=np.int32) if case.nseg else np.zeros(1, np.int32)
        self._keep += [xyz, tri, seg, kind]
        mesh = Mesh(case.nnodes, case.ntri, case.nseg, _d(xyz), _i(tri), _i(seg), _i(kind), None, None, case.gravity)
        if check_csr is not None:
            ip, cl = (np.ascontiguousarray(a, dtype=np.int32) for a in check_csr)
            self._keep += [ip, cl]
            mesh.indptr, mesh.cols = _i(ip), _i(cl)
        h = C.c_void_p()
        self._check(L.sw2g_create(C.byref(mesh), C.c_void_p(stream) if stream else None, C.byref(h)))
        self.h = h
        nd, nz = C.c_int(), C.c_int()
        self._check(L.sw2g_sizes(self.h, C.byref(nd), C.byref(nz)))
        self.ndofs, self.nnz = nd.value, nz.value

    # ------------------------------------------------------------- plumbing
    def _check(self, rc):
        if rc != 0:
            raise SW2Error(f"sw2g error {rc}: {lib().sw2g_last_error().decode()}", rc)

    def close(self):
        if getattr(self, "h", None):
            lib().sw2g_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return lib().sw2g_stream(self.h)

    # ------------------------------------------------------------- API
    def sparsity(self):
        ip = np.zeros(self.ndofs + 1, np.int32)
        cl = np.zeros(self.nnz, np.int32)
        self._check(lib().sw2g_get_sparsity(self.h, _i(ip), _i(cl)))
        return ip, cl

    def set_bc_structures(self, q_series, conveyance, rough_height, tail_elev):
        """Values of the discharge (kind 2) and tailwater (kind 3) segments."""
        self._check(lib().sw2g_set_bc_structures(self.h, C.c_double(q_series), C.c_double(conveyance),
                                                 C.c_double(rough_height), C.c_double(tail_elev)))

    def set_bc_flux(self, flux_series):
        """Series value of the flux segments (kind 5)."""
        self._check(lib().sw2g_set_bc_flux(self.h, C.c_double(flux_series)))

    def set_step(self, dt, bc_depth, bc_vx, bc_vy, tau_temporal=0.0):
        self._check(lib().sw2g_set_step(self.h, C.c_double(dt), C.c_double(tau_temporal), C.c_double(bc_depth),
                                        C.c_double(bc_vx), C.c_double(bc_vy)))

    def wd_flags(self, sol, sol_old):
        out = np.zeros(self.case.ntri, np.int32)
        self._check(lib().sw2g_wd_flags(self.h, _d(_f64(sol)), _d(_f64(sol_old)), _i(out)))
        return out

    def elem_resid(self, sol, sol_old, sol_older):
        t = np.zeros(9 * self.case.ntri); s = np.zeros(6 * max(self.case.nseg, 1))
        self._check(lib().sw2g_elem_resid(self.h, _d(_f64(sol)), _d(_f64(sol_old)), _d(_f64(sol_older)), _d(t), _d(s)))
        return t, s[: 6 * self.case.nseg]

    def elem_jac(self, sol, sol_old, sol_older):
        t = np.zeros(81 * self.case.ntri); s = np.zeros(36 * max(self.case.nseg, 1))
        self._check(lib().sw2g_elem_jac(self.h, _d(_f64(sol)), _d(_f64(sol_old)), _d(_f64(sol_older)), _d(t), _d(s)))
        return t, s[: 36 * self.case.nseg]

    def residual(self, sol, sol_old, sol_older):
        r = np.zeros(self.ndofs)
        self._check(lib().sw2g_assemble_residual(self.h, _d(_f64(sol)), _d(_f64(sol_old)), _d(_f64(sol_older)), _d(r)))
        return r

    def jacobian(self, sol, sol_old, sol_older):
        v = np.zeros(self.nnz)
        self._check(lib().sw2g_assemble_jacobian(self.h, _d(_f64(sol)), _d(_f64(sol_old)), _d(_f64(sol_older)), _d(v)))
        return v

    def residual_wd(self, sol, sol_old, sol_older, wd_flag):
        """The residual with the caller's wet/dry flags (sw2g_assemble_residual_wd)."""
        r = np.zeros(self.ndofs)
        wd = np.ascontiguousarray(wd_flag, dtype=np.int32)
        self._check(lib().sw2g_assemble_residual_wd(self.h, _d(_f64(sol)), _d(_f64(sol_old)), _d(_f64(sol_older)),
                                                    _i(wd), _d(r)))
        return r

    def jacobian_wd(self, sol, sol_old, sol_older, wd_flag):
        """The CSR values with the caller's wet/dry flags (sw2g_assemble_jacobian_wd)."""
        v = np.zeros(self.nnz)
        wd = np.ascontiguousarray(wd_flag, dtype=np.int32)
        self._check(lib().sw2g_assemble_jacobian_wd(self.h, _d(_f64(sol)), _d(_f64(sol_old)), _d(_f64(sol_older)),
                                                    _i(wd), _d(v)))
        return v

    def prepare_system(self, vals, residual, x, bc_mask):
        vals = _f64(vals).copy(); residual = _f64(residual).copy(); x = _f64(x).copy()
        bc_mask = np.ascontiguousarray(bc_mask, dtype=np.int32).copy()
        scale = np.zeros(self.ndofs)
        self._check(lib().sw2g_prepare_system(self.h, _d(vals), _d(residual), _d(x), _i(bc_mask), _d(scale)))
        return vals, residual, x, bc_mask, scale

    def bicgstab(self, vals, b, x, scale, max_it=4000, tol=1e-11, precond=PC_AMG):
        x = _f64(x).copy(); b = _f64(b).copy()
        it = C.c_int()
        self._check(lib().sw2g_solve_linear_sys_bcgstab(self.h, _d(x), _d(_f64(vals)), _d(b), _d(_f64(scale)),
                                                        int(max_it), C.c_double(tol), int(precond), C.byref(it)))
        return x, b, it.value

    def fe_newton(self, sol_old, sol_older, bc_mask, dirichlet=None, opts=None):
        sol = np.zeros(self.ndofs)
        bc_mask = np.ascontiguousarray(bc_mask, dtype=np.int32)
        dirichlet = np.zeros(self.ndofs) if dirichlet is None else _f64(dirichlet)
        st = NewtonStats()
        o = opts or default_opts()
        self._check(lib().sw2g_fe_newton(self.h, _d(sol), _d(_f64(sol_old)), _d(_f64(sol_older)), _i(bc_mask),
                                         _d(dirichlet), C.byref(o), C.byref(st)))
        return sol, st.as_dict()

    def load_state(self, sol, sol_old, sol_older, bc_mask=None, dirichlet=None):
        bm = None if bc_mask is None else np.ascontiguousarray(bc_mask, dtype=np.int32)
        di = None if dirichlet is None else _f64(dirichlet)
        self._check(lib().sw2g_load_state(self.h, _d(_f64(sol)), _d(_f64(sol_old)), _d(_f64(sol_older)),
                                          _i(bm) if bm is not None else None, _d(di) if di is not None else None))

    def store_state(self):
        a, b, c = np.zeros(self.ndofs), np.zeros(self.ndofs), np.zeros(self.ndofs)
        m = np.zeros(self.ndofs, np.int32)
        self._check(lib().sw2g_store_state(self.h, _d(a), _d(b), _d(c), _i(m)))
        return a, b, c, m

    def set_guess(self, guess=None, device_ptr=None):
        if device_ptr is not None:
            self._check(lib().sw2g_set_guess(self.h, C.c_void_p(device_ptr), 1))
        elif guess is not None:
            g = _f64(guess)
            self._check(lib().sw2g_set_guess(self.h, _d(g), 0))
        else:
            self._check(lib().sw2g_set_guess(self.h, None, 0))

    def step(self, opts=None):
        st = NewtonStats()
        self._check(lib().sw2g_step(self.h, C.byref(opts or default_opts()), C.byref(st)))
        return st.as_dict()

    def undo_step(self):
        self._check(lib().sw2g_undo_step(self.h))

    def device_state(self):
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        self._check(lib().sw2g_device_state(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def grid_mass(self, sol=None, density=1.0, dt=None, elem=False):
        """(density * grid mass, one step's boundary mass inflow[, per-triangle terms]) of
        `sol` (host [ndofs]) or, with sol None, of the resident state."""
        out = np.zeros(2)
        em = np.zeros(max(self.case.ntri, 1)) if elem else None
        dt = self.case.dt if dt is None else dt
        src = None if sol is None else _f64(sol)
        self._check(lib().sw2g_grid_mass(self.h, _d(src) if src is not None else None, C.c_double(density),
                                         C.c_double(dt), _d(out), _d(em) if em is not None else None))
        if elem:
            return out[0], out[1], em[: self.case.ntri]
        return out[0], out[1]

    def set_profiling(self, on=True):
        self._check(lib().sw2g_set_profiling(self.h, int(on)))
        self.profiling = bool(on)

    def profile(self):
        ms = np.zeros(6); n = np.zeros(6, np.int64)
        self._check(lib().sw2g_get_profile(self.h, _d(ms), n.ctypes.data_as(C.POINTER(C.c_longlong))))
        return ms, n

    def precond_info(self):
        """The AMG's chunk corrections at the last preconditioner set-up (sw2g_precond_info)."""
        info = np.zeros(5, np.int64)
        self._check(lib().sw2g_precond_info(self.h, info.ctypes.data_as(C.POINTER(C.c_longlong))))
        return dict(zip(("flagged_nodes", "chunks", "chunk_nodes", "inverse_entries", "singular_chunks"),
                        (int(v) for v in info)))

    def reset_profile(self):
        self._check(lib().sw2g_reset_profile(self.h))

    def time_kernel(self, which, reps=20):
        """(mean ms per launch, algorithmic bytes per launch) of kernel family `which`:
        0 FP64 SpMV, 1 FD Jacobian, 2 element residual, 3 Jacobian gather, 4 AMG smoothing sweep (FP64),
        5 AMG smoothing sweep (FP32), 6 FP32 V-cycle, 7 FP32 SpMV, 8 one FP32 GMRES cycle (second value: its
        iterations), 9 the AMG chunk corrections (FP32)."""
        ms, by = C.c_double(), C.c_double()
        self._check(lib().sw2g_time_kernel(self.h, int(which), int(reps), C.byref(ms), C.byref(by)))
        return ms.value, by.value


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)
