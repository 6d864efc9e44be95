"""Host-side time loop around the GPU Newton step.

Mirrors the reference's driver layer: time_loop / update_dt / advance_time
(src/timeloop/time_loop.c:14-125) and the step averaging of the boundary series
(sseries_setall_ts_valuesAVG, src/structs/sseries/sseries.c:622-682).  The
per-step work -- residuals, FD Jacobian, assembly, Dirichlet/scaling, BiCGStab,
Newton -- runs on the device through the C ABI (capi.SW2Model).
"""
from __future__ import annotations

import numpy as np

from .capi import ERR_NONFINITE, SW2Error, SW2Model, default_opts

_EPS = np.finfo(np.float64).eps
DT_REDUCE_FACTOR = 0.25        # tc_scale's factor after a failed Newton solve (src/include/define.h:127)
NOT_QUITE_SMALL = float(np.finfo(np.float32).eps)   # update_dt's end-of-run slack (src/include/define.h:32)


def _interval(times, t):
    # sseries_get_interval (sseries.c:746-773)
    i = 0
    n = len(times)
    while i < n - 1 and t >= times[i] * (1.0 - _EPS):
        i += 1
    return i - 1


def _eval(times, values, iv, t):
    # tc_eval_series (src/tools/tc_eval_series.c)
    if iv == len(times) - 1:
        return values[-1]
    lt, rt = times[iv], times[iv + 1]
    theta = (rt - t) / (rt - lt)
    return theta * values[iv] + (1.0 - theta) * values[iv + 1]


def _trap(lv, rv, lt, rt):
    # tc_trap_area (src/tools/tc_trap_area.c)
    d = rt - lt
    return 0.0 if d < _EPS else (lv + rv) * 0.5 * d


def series_step_average(times, values, t1, t2):
    """Average of a piecewise-linear series over [t1, t2] (sseries_set_values_average)."""
    times = np.asarray(times, dtype=np.float64)
    values = np.asarray(values, dtype=np.float64)
    if t1 < times[0] * (1.0 - _EPS) or t2 > times[-1] * (1.0 + _EPS):
        raise ValueError(f"time window [{t1}, {t2}] is outside the series range")
    i1, i2 = _interval(times, t1), _interval(times, t2)
    v1, v2 = _eval(times, values, i1, t1), _eval(times, values, i2, t2)
    if i1 == i2:
        area = _trap(v1, v2, t1, t2)
    else:
        area = 0.0
        for k in range(i1 + 1, i2):
            area += _trap(values[k], values[k + 1], times[k], times[k + 1])
        area += _trap(v1, values[i1 + 1], t1, times[i1 + 1])
        area += _trap(values[i2], v2, times[i2], t2)
    return area / (t2 - t1)


class SW2Simulation:
    """A time-stepping SW2 run whose state stays resident on the GPU."""

    def __init__(self, case, opts=None, stream=None, model=None):
        self.case = case
        self.model = model if model is not None else SW2Model(case, stream=stream)
        self.opts = opts or default_opts(tol_nonlin=case.tol_nonlin, inc_nonlin=case.inc_nonlin,
                                         max_nonlin_it=case.max_nonlin_it)
        self.t = case.t0
        sol0 = case.sol0.astype(np.float64)
        self.model.load_state(sol0, sol0, sol0)
        self.history = []        # every Newton solve tried, failed ones included
        self.nsteps_done = 0     # successful steps (what a checkpoint counts)
        # advance(): after an interval needed a cut, the next intervals start at the reduced
        # step (the reference keeps a cut dt too: tc_scale writes sm->ts->dt and nothing
        # restores it); after keep_reduced_dt such intervals the step grows by 1/DT_REDUCE_FACTOR
        # toward the case's dt.  0 turns the carry-over off.
        self._has_discharge = bool(np.any(np.asarray(case.seg_kind) == 2))
        self.keep_reduced_dt = 4
        self.dt_hold = None      # the reduced step carried over, None = the case's dt
        self.hold_count = 0      # intervals completed at dt_hold
        self.mass_log = None
        self.log = None     # a writable text stream: one JSON line per step (set_log)

    def bc_values(self, t1, t2):
        s = self.case.series
        out = [series_step_average(*s[0], t1, t2)]
        for k in (1, 2):
            out.append(series_step_average(*s[k], t1, t2) if k in s else 0.0)
        return out

    def prepare_step(self, dt=None):
        """update_dt + the series averaging of advance_time for the next step."""
        dt = self.case.dt if dt is None else dt
        t_new = self.t + dt
        d, vx, vy = self.bc_values(t_new - dt, t_new)
        self.model.set_step(dt, d, vx, vy)
        s = self.case.series
        if self._has_discharge and not self.case.bc_rough_height > np.finfo(np.float64).eps:
            # the discharge law divides by the strings' drag, zero without a roughness height
            raise ValueError("discharge segments need SW2Case.bc_rough_height > 0")
        if 3 in s or 4 in s:    # discharge / tailwater segments
            qs = series_step_average(*s[3], t_new - dt, t_new) if 3 in s else 0.0
            tw = series_step_average(*s[4], t_new - dt, t_new) if 4 in s else 0.0
            self.model.set_bc_structures(qs, self.case.bc_conveyance, self.case.bc_rough_height, tw)
        if 5 in s:              # flux segments
            self.model.set_bc_flux(series_step_average(*s[5], t_new - dt, t_new))
        return t_new

    def _attempt(self, opts, dt):
        """One Newton solve over [t, t + dt]; the clock stays.  A non-finite residual
        (SW2G_ERR_NONFINITE) is a failed solve like any other; every other error --
        bad arguments, CUDA errors, errors of set_step -- propagates."""
        t_new = self.prepare_step(dt)
        try:
            st = self.model.step(opts or self.opts)
        except SW2Error as e:
            if e.rc != ERR_NONFINITE:
                raise
            st = {"success": 0, "newton_its": 0, "krylov_its": 0, "error": str(e)}
        return st, t_new

    def _record(self, st, t_new, dt, moved):
        self.history.append(st)
        rec = None
        if moved:
            self.t = t_new
        if st["success"]:
            self.nsteps_done += 1
            if self.mass_log is not None:
                m, inflow = self.model.grid_mass(None, self.density, dt)
                self.inflow_total += inflow
                self.mass_log.append((t_new, m, inflow))
                rec = (m, inflow)
        if self.log is not None:
            self._write_log(t_new, dt, st, rec)

    def step(self, opts=None, dt=None):
        """One Newton solve over [t, t + dt] (dt: the case's step by default) with the
        reference's semantics: a failed solve leaves the state at the step's start, as
        fe_newton does, and time moves on (the reference's time loop then stops,
        src/timeloop/time_loop.c:37).  advance() is the form that retries instead."""
        dt = self.case.dt if dt is None else dt
        st, t_new = self._attempt(opts, dt)
        self._record(st, t_new, dt, moved=True)
        return st

    def set_log(self, stream) -> None:
        """Write one JSON line per Newton solve to ``stream`` (None stops): time, dt, the
        Newton statistics, the grid mass and boundary inflow when the mass balance is on,
        and the device time per kernel class accumulated since the last profile reset
        when the model profiles (set_profiling)."""
        self.log = stream

    def _write_log(self, t, dt, st, mass):
        import json
        keys = ("success", "newton_its", "krylov_its", "linesearch_cuts", "resid_max", "initial_resid_max",
                "guess_used", "guess_fallback")
        out = {"t": t, "dt": dt}
        out.update({k: (float(st[k]) if isinstance(st[k], (float, np.floating)) else int(st[k]))
                    for k in keys if k in st})
        if mass is not None:
            out["mass"], out["inflow"] = float(mass[0]), float(mass[1])
        prof = getattr(self.model, "profile", None)
        if getattr(self.model, "profiling", False) and prof is not None:
            ms, n = prof()
            out["class_ms_total"] = [round(float(x), 3) for x in ms]
        self.log.write(json.dumps(out) + "\n")

    def advance(self, opts=None, max_cuts=3, before_attempt=None):
        """One interval of the case's dt that survives failed Newton solves.  A failed
        solve is undone and the interval is tried again with dt scaled by
        DT_REDUCE_FACTOR, as tc_scale scales it (src/tools/tc_scale.c:10, called at
        src/newton/fe_newton.c:887); the rest of the interval is then covered in
        steps of the reduced size.  The reference instead ends its time loop at the
        first failure (src/timeloop/time_loop.c:37).  Gives up after max_cuts
        reductions (success 0, the state and the clock at the last good substep).  With
        the relative Newton test, the shorter steps keep the tolerance of the interval's
        first attempt (sw2g_newton_opts.tol_nonlin_min).
        After an interval that needed a cut, the next ``keep_reduced_dt`` intervals start
        at the reduced step (with the interval's tolerance), then the step grows back by
        1/DT_REDUCE_FACTOR per such run of intervals.
        ``before_attempt(sim, dt)``, when given, runs before every Newton solve (e.g.
        to set an initial guess for a step of that dt).  Failed attempts are undone before anything else runs:
        the clock never moves for them and the mass log never sees them."""
        target = self.t + self.case.dt
        dt, cuts, subs, failed = self.case.dt, 0, [], []
        o_cur = opts or self.opts
        rel = getattr(o_cur, "tol_nonlin_rel", 0)
        held = self.keep_reduced_dt > 0 and self.dt_hold is not None and self.dt_hold < self.case.dt
        if held:
            dt = self.dt_hold
        h_start = dt
        if held:
            if rel > 0:
                # R(sol_old) scales with the step's length (sol = sol_old makes the temporal
                # terms vanish), so rel x dt/h keeps the tolerance of the whole interval
                o_cur = type(o_cur).from_buffer_copy(o_cur)
                o_cur.tol_nonlin_rel = rel * self.case.dt / dt
        first = True
        while self.t + NOT_QUITE_SMALL * self.case.dt < target:
            h = min(dt, target - self.t)
            if before_attempt is not None:
                before_attempt(self, h)
            st, t_new = self._attempt(o_cur, h)
            if first and rel > 0 and st.get("tol_used") and (held or not st["success"]):
                # the shorter steps keep the interval's tolerance: the residual at the start of a
                # short step shrinks with its dt, the attainable accuracy does not
                o_cur = type(o_cur).from_buffer_copy(o_cur)
                o_cur.tol_nonlin_min = float(st["tol_used"])
                o_cur.tol_nonlin_rel = rel
            first = False
            if st["success"]:
                self._record(st, t_new, h, moved=True)
                subs.append(st)
                continue
            self.model.undo_step()
            self._record(st, t_new, h, moved=False)
            failed.append(st)
            cuts += 1
            if cuts > max_cuts:
                break
            dt = h * DT_REDUCE_FACTOR
        ok = cuts <= max_cuts
        if ok and self.keep_reduced_dt > 0:
            if cuts > 0:
                self.dt_hold, self.hold_count = dt, 0
            elif held:
                self.hold_count += 1
                if self.hold_count >= self.keep_reduced_dt:
                    grown = dt / DT_REDUCE_FACTOR
                    self.dt_hold = None if grown >= self.case.dt * (1 - NOT_QUITE_SMALL) else grown
                    self.hold_count = 0
        out = {"success": int(ok), "substeps": len(subs), "dt_cuts": cuts, "step_start": h_start,
               "newton_its": sum(s["newton_its"] for s in subs + failed),
               "krylov_its": sum(s["krylov_its"] for s in subs + failed),
               "linear_unconverged": sum(s.get("linear_unconverged", 0) for s in subs + failed)}
        if subs:
            last = subs[-1]
            for k in ("resid_max", "inc_max", "tol_used"):
                if k in last:
                    out[k] = last[k]
            for k in ("prev_resid_max", "initial_resid_max", "guess_used"):
                if k in subs[0]:
                    out[k] = subs[0][k]
        return out

    def start_mass_balance(self, density=1.0):
        """Start the mass bookkeeping of tl_find_grid_mass_error_elem2d
        (src/tools/tl_grid_mass.c:280) from the resident state: every later successful
        step records the grid mass of its result and its boundary mass inflow."""
        self.density = float(density)
        self.mass0, _ = self.model.grid_mass(None, self.density, self.case.dt)
        self.inflow_total = 0.0
        self.mass_log = []

    def mass_balance(self):
        """Grid mass now, at the start, the boundary inflow since, and the reference's
        mass error |mass - inflow - initial mass|."""
        if self.mass_log is None:
            raise RuntimeError("start_mass_balance() was not called")
        m = self.mass_log[-1][1] if self.mass_log else self.mass0
        err = abs(m - self.inflow_total - self.mass0)
        return {"initial_mass": self.mass0, "mass": m, "inflow": self.inflow_total, "error": err,
                "rel_error": err / self.mass0 if self.mass0 else None, "steps": len(self.mass_log)}

    def run(self, nsteps, opts=None, stop_on_failure=True):
        for _ in range(nsteps):
            st = self.step(opts)
            if stop_on_failure and not st["success"]:
                break
        return self.history

    def state(self):
        return self.model.store_state()

    def checkpoint(self, path: str) -> None:
        """Write the resident state -- the three solution levels, the Dirichlet marks,
        the time, the count of successful steps and, when the mass balance is on, its
        totals and log -- to ``path`` (.npz).  Resuming from it with :meth:`restore`
        takes the same next step, and reports the same mass error, as the
        uninterrupted run."""
        sol, sol_old, sol_older, bc_mask = self.model.store_state()
        extra = {}
        if self.mass_log is not None:
            extra = {"mass_density": self.density, "mass0": self.mass0, "mass_inflow_total": self.inflow_total,
                     "mass_log": np.asarray(self.mass_log, dtype=np.float64).reshape(-1, 3)}
        np.savez(path, sol=sol, sol_old=sol_old, sol_older=sol_older, bc_mask=bc_mask, t=self.t,
                 dt=self.case.dt, steps=self.nsteps_done,
                 dt_hold=-1.0 if self.dt_hold is None else self.dt_hold, hold_count=self.hold_count, **extra)

    def restore(self, path: str) -> None:
        z = np.load(path)
        if float(z["dt"]) != self.case.dt or z["sol"].size != 3 * self.case.nnodes:
            raise ValueError("checkpoint does not belong to this case")
        self.model.load_state(z["sol"], z["sol_old"], z["sol_older"], bc_mask=z["bc_mask"])
        self.t = float(z["t"])
        self.nsteps_done = int(z["steps"])
        if "dt_hold" in z:
            self.dt_hold = None if float(z["dt_hold"]) < 0 else float(z["dt_hold"])
            self.hold_count = int(z["hold_count"])
        if "mass0" in z:
            self.density = float(z["mass_density"])
            self.mass0 = float(z["mass0"])
            self.inflow_total = float(z["mass_inflow_total"])
            self.mass_log = [tuple(float(v) for v in row) for row in z["mass_log"]]
        else:
            self.mass_log = None
