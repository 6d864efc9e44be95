#!/usr/bin/env python
"""SW2 implicit time steps per second on the 4M-triangle wet/dry beach.

Workload: 40 km x 10 km sloping beach (bed -20 m .. +3 m plus N(0, 0.2 m) noise,
seed 3), jittered Delaunay of a 2828 x 707 grid = 3 991 724 triangles, 1 999 396
nodes, 5 998 188 dofs; inflow hydrograph Q(t) = 500 + 1500 sin^2(pi t / 6 h) as a
velocity BC, dt = 120 s.  A "step" is one implicit time step: fe_newton to
tol_nonlin = 1e-8 on the reference's unscaled max-norm residual (FD Jacobian,
CSR assembly, Dirichlet/scaling, preconditioned Krylov solve per Newton
iteration).  Synthetic input generated here; every array is far larger than L2.

Two paths are timed from the same state after warm-up:
  * fast:  Krylov with the preconditioner in FP32 (FP64 basis and residuals) and,
           with --guess learned, the message-passing network's initial guess;
  * plain: everything FP64, previous-step initial guess.
`value` is the fast path (the product); the plain path is reported beside it.

`python bench.py --impl reference` times the reference's own C code (compiled
from its sources, UMFPACK replaced by a banded LU) on the host cores for a
bounded sample of the same workload and reports the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "SW2 timesteps/s @4M tris: learned+FP32-Krylov vs plain FP64 GPU at equal Newton tol"
UNIT = "timesteps/s"
NTRI_FULL = 3991724
SAMPLE_NX, SAMPLE_NY = 240, 60            # reference CPU sample: same beach, coarser grid


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--nx", type=int, default=2828)
    p.add_argument("--ny", type=int, default=707)
    p.add_argument("--krylov-tol", type=float, default=1e-6,
                   help="inexact-Newton forcing: linear residual <= tol * Newton residual (floor: a tenth of "
                        "tol_nonlin with the relative Newton test, a hundredth with the absolute one)")
    p.add_argument("--guess", choices=["none", "learned"], default="learned")
    p.add_argument("--weights", default=None, help="trained initial-guess weights (default: the committed ones)")
    p.add_argument("--tol-rel", type=float, default=1e-8,
                   help="Newton test max|R| <= tol_rel * max|R(previous step)|; 0: the reference's absolute 1e-8")
    p.add_argument("--basis", type=int, choices=[32, 64], default=32,
                   help="fast path: FP32 (default) or FP64 GMRES basis around the FP32 preconditioner")
    p.add_argument("--restart", type=int, default=50, help="GMRES restart length of both paths (1..50)")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-steps", type=int, default=4)
    return p.parse_args()


# ----------------------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local, dist


def max_over_ranks(x, dist, device="cuda"):
    """The slowest rank's value (every rank calls this at the same point)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_reference_sample(nsteps_total, skip):
    """Reference fe_newton (compiled from its C sources) on the SAMPLE_NX x SAMPLE_NY beach:
    seconds per step of steps skip..nsteps_total-1, and the sample's triangle count."""
    from adh_kraken_b200.mesh import beach_case
    from oracle import refio
    case = beach_case(nx=SAMPLE_NX, ny=SAMPLE_NY, nsteps=nsteps_total)
    rec = refio.run_harness("run", case, extra=(nsteps_total,), timeout=1800)
    secs = np.asarray(rec["step_seconds"], dtype=np.float64)
    ok = np.asarray(rec["step_ok"])
    use = secs[skip:] if len(secs) > skip else secs
    return use, int(case.ntri), int(ok.sum()), len(ok)


# ----------------------------------------------------------------------------- reference arm
def run_reference(args, world, rank, dist):
    if rank != 0:
        return
    if not os.path.exists(os.path.join(HERE, "oracle", "_ref", "adh_ref_harness")):
        print(json.dumps({"impl": "reference", "unavailable": "reference harness not built (oracle/_ref)"}))
        return
    secs, ntri, nok, nrun = cpu_reference_sample(args.warmup + args.steps, args.warmup)
    per_step_full = float(np.mean(secs)) * NTRI_FULL / ntri
    value = 1.0 / per_step_full
    sample = (f"reference fe_newton on the {SAMPLE_NX}x{SAMPLE_NY} beach ({ntri} tris, same dt/forcing), "
              f"{len(secs)} timed steps after {args.warmup} warm-up, {float(np.mean(secs)):.3f} s/step, scaled "
              f"linearly by triangle count to {NTRI_FULL} (a lower bound on CPU time: its LU scales worse); "
              f"UMFPACK replaced by a banded LU; {nok}/{nrun} steps converged")
    out = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step_full * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "beach4M", "ntri": NTRI_FULL, "dt_s": 120.0, "tol_nonlin": 1e-8,
                      "sample_ntri": ntri},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ----------------------------------------------------------------------------- our arm
def run_ours(args, world, rank, local, dist):
    import torch
    from adh_kraken_b200.capi import default_opts, NewtonStats, SW2Error, lib
    from adh_kraken_b200.mesh import beach_case
    from adh_kraken_b200.timeloop import SW2Simulation
    import ctypes as C

    torch.cuda.set_device(local)
    K, W = args.steps, args.warmup
    case = beach_case(nx=args.nx, ny=args.ny, nsteps=W + 2 * K + 4)
    base = dict(tol_nonlin=1e-8, tol_nonlin_rel=args.tol_rel, inc_nonlin=1e-6, max_nonlin_it=10,
                krylov_max_it=20000, krylov_tol=args.krylov_tol, precond=2, krylov_method=1,
                krylov_restart=args.restart)
    opts_fast = default_opts(krylov_precision=32, krylov_basis_precision=args.basis, **base)
    opts_plain = default_opts(krylov_precision=64, **base)
    guesser = None
    if args.guess == "learned":
        from adh_kraken_b200 import learned
        guesser = learned.load_guesser(case, args.weights) if args.weights else learned.load_guesser(case)
    if guesser is not None:
        opts_fast.use_guess = 1

    fast = SW2Simulation(case, opts=opts_fast)

    def safe_step(sim):
        try:
            return sim.step()
        except SW2Error as e:                 # a non-finite residual: the step fails, the state is kept
            return {"success": 0, "newton_its": -1, "krylov_its": -1, "initial_resid_max": float("nan"),
                    "resid_max": float("nan"), "error": str(e)}

    def fast_step(sim):
        if guesser is not None:
            guesser.predict_into(sim)        # device-side guess from the resident state
        return safe_step(sim)

    # warm-up (spin-up of the hydrograph and of every graph / hierarchy)
    for _ in range(W):
        fast_step(fast)
    state0 = fast.state()
    t0 = fast.t
    plain = None
    if not args.no_plain:
        plain = SW2Simulation(case, opts=opts_plain)
        plain.model.load_state(*state0[:3], bc_mask=state0[3])
        plain.t = t0
        safe_step(plain)                        # builds its hierarchy / graphs
        plain.model.load_state(*state0[:3], bc_mask=state0[3])
        plain.t = t0

    def timed(sim, stepper, clocks=None):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        hist = []
        sim.start_mass_balance(1000.0)          # water density, kg/m^3
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        sim.model.set_profiling(True)
        sim.model.reset_profile()
        s = torch.cuda.ExternalStream(sim.model.stream)
        ev0.record(s)
        for _ in range(K):
            hist.append(stepper(sim))
        ev1.record(s)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        prof_ms, prof_n = sim.model.profile()
        sim.model.set_profiling(False)
        if dist is not None:
            ms = max_over_ranks(ms, dist)
            dist.barrier()
        return ms, hist, prof_ms, prof_n

    with ClockSampler(local) as clk:
        ms_fast, hist_fast, prof_ms, prof_n = timed(fast, fast_step)
    clocks = clk.summary()
    ms_plain, hist_plain = None, None
    if plain is not None:
        ms_plain, hist_plain, _, _ = timed(plain, safe_step)

    # roofline of the dominant kernel of the fast path: the FP32 AMG smoothing sweep
    rf_ms, rf_bytes = fast.model.time_kernel(5, 20)
    spmv_ms, spmv_bytes = fast.model.time_kernel(0, 20)
    fd_ms, fd_bytes = fast.model.time_kernel(1, 5)
    peaks = {}
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    hbm = float(peaks.get("hbm_gbs", 0) or 0)
    peak_src = "measured"
    if hbm <= 0:
        hbm, peak_src = 6650.0, "fallback"
    achieved = rf_bytes / (rf_ms * 1e-3) / 1e9
    traffic = None
    tfile = os.path.join(HERE, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            with open(tfile) as fh:
                traffic = json.load(fh).get("amg_smooth_fp32_bytes_per_launch")
        except (OSError, ValueError):
            traffic = None

    # end to end through the C ABI with host buffers (sw2g_fe_newton per step)
    e2e = None
    if not args.no_e2e:
        m = fast.model
        n = m.ndofs
        sol_h = torch.empty(n, dtype=torch.float64, pin_memory=True)
        old_h = torch.empty(n, dtype=torch.float64, pin_memory=True)
        older_h = torch.empty(n, dtype=torch.float64, pin_memory=True)
        mask_h = torch.empty(n, dtype=torch.int32, pin_memory=True)
        dir_h = torch.zeros(n, dtype=torch.float64, pin_memory=True)
        s, so, soo, mk = state0
        old_h.numpy()[:] = s; older_h.numpy()[:] = so; mask_h.numpy()[:] = mk
        st = NewtonStats()
        L = lib()
        t_e = t0
        e2e_fail = 0
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for _ in range(K):
            t_e += case.dt
            d, vx, vy = fast.bc_values(t_e - case.dt, t_e)
            m.set_step(case.dt, d, vx, vy)
            if guesser is not None:
                guesser.predict_host(m, old_h.numpy(), older_h.numpy())
            rc = L.sw2g_fe_newton(m.h, C.c_void_p(sol_h.data_ptr()), C.c_void_p(old_h.data_ptr()),
                                  C.c_void_p(older_h.data_ptr()), C.c_void_p(mask_h.data_ptr()),
                                  C.c_void_p(dir_h.data_ptr()), C.byref(opts_fast), C.byref(st))
            if rc not in (0, -5):                 # -5: non-finite residual, a failed step (state kept)
                raise RuntimeError(L.sw2g_last_error().decode())
            e2e_fail += int(rc != 0 or not st.success)
            older_h.numpy()[:] = old_h.numpy(); old_h.numpy()[:] = sol_h.numpy()
        wall = time.perf_counter() - w0
        wall = max_over_ranks(wall, dist)
        e2e = {"value": world * K / wall, "unit": UNIT,
               "h2d_bytes_per_step": 3 * 8 * n + 4 * n + 8 * n + (8 * n if guesser is not None else 0),
               "d2h_bytes_per_step": 8 * n + 4 * n, "failed_steps": e2e_fail,
               "api": "sw2g_fe_newton (host buffers, pinned)"}

    # CPU baseline (rank 0, bounded sample)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        try:
            secs, ntri, nok, nrun = cpu_reference_sample(args.cpu_steps + 1, 1)
            per_full = float(np.mean(secs)) * NTRI_FULL / ntri
            cpu = {"value": 1.0 / per_full, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": (f"reference fe_newton, {SAMPLE_NX}x{SAMPLE_NY} beach ({ntri} tris), {len(secs)} steps "
                              f"at {float(np.mean(secs)):.3f} s/step scaled linearly to {NTRI_FULL} tris; "
                              f"banded LU in place of UMFPACK; single-threaded code")}
        except Exception as e:  # noqa: BLE001 - reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    if rank != 0:
        _cleanup(fast, plain, guesser)
        if dist is not None:
            dist.destroy_process_group()
        return
    kfail = sum(1 for h in hist_fast if not h["success"])
    names = ["residual", "fd_jacobian", "jacobian_gather", "prepare_precond_setup", "krylov", "other"]
    out = {
        "metric": METRIC, "value": world * K / (ms_fast * 1e-3), "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": ms_fast / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
        "config": {"workload": "beach4M", "ntri": case.ntri, "nnodes": case.nnodes, "ndofs": 3 * case.nnodes,
                   "nnz": fast.model.nnz, "dt_s": case.dt, "tol_nonlin": 1e-8, "tol_nonlin_rel": args.tol_rel,
                   "krylov": f"GMRES({args.restart})+AMG",
                   "krylov_forcing": args.krylov_tol, "guess": args.guess if guesser is not None else "none",
                   "fast_precision": ("AMG preconditioner FP32, Krylov/residual/FD FP64" if args.basis == 64 else
                                      "GMRES cycle (basis, SpMV, AMG) FP32 inside FP64 refinement; residual/FD FP64"),
                   "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (1.5 GB matrix)"},
        "plain_fp64": None if ms_plain is None else {
            "value": world * K / (ms_plain * 1e-3), "ms_per_step": ms_plain / K,
            "newton_its": [h["newton_its"] for h in hist_plain], "krylov_its": [h["krylov_its"] for h in hist_plain],
            "failed_steps": sum(1 for h in hist_plain if not h["success"]),
            "mass_balance": plain.mass_balance()},
        "fast_detail": {"newton_its": [h["newton_its"] for h in hist_fast],
                        "krylov_its": [h["krylov_its"] for h in hist_fast], "failed_steps": kfail,
                        "initial_resid": [h["initial_resid_max"] for h in hist_fast],
                        "initial_resid_l2": [h.get("initial_resid_l2") for h in hist_fast],
                        "prev_resid": [h.get("prev_resid_max") for h in hist_fast],
                        "final_resid": [h["resid_max"] for h in hist_fast],
                        "guess_used": [h.get("guess_used", 0) for h in hist_fast],
                        "guess_fallback": [h.get("guess_fallback", 0) for h in hist_fast],
                        "class_ms": dict(zip(names, [round(float(x), 2) for x in prof_ms])),
                        "mass_balance": fast.mass_balance()},
        "gpu_launches": int(np.sum(prof_n)),
        "clocks": clocks,
        "roofline": {"kernel": "k_amg_l0<float,1> (AMG level-0 smoothing sweep, FP32)", "bound": "hbm",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": peak_src, "traffic": traffic, "algorithmic_bytes": rf_bytes,
                     "avg_launch_ms": rf_ms,
                     "spmv_fp64": {"achieved": spmv_bytes / (spmv_ms * 1e-3) / 1e9, "avg_launch_ms": spmv_ms,
                                   "frac": spmv_bytes / (spmv_ms * 1e-3) / 1e9 / hbm},
                     "fd_jacobian": {"achieved_gbs": fd_bytes / (fd_ms * 1e-3) / 1e9, "avg_launch_ms": fd_ms}},
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    if out["plain_fp64"] is not None:
        out["speedup_vs_plain_fp64"] = ms_plain / ms_fast
    print(json.dumps(out), flush=True)
    _cleanup(fast, plain, guesser)
    if dist is not None:
        dist.destroy_process_group()


def _cleanup(*objs):
    """Release device objects in a fixed order before interpreter shutdown."""
    import torch
    torch.cuda.synchronize()
    for o in objs:
        if o is None:
            continue
        model = getattr(o, "model", None)
        if model is not None:
            model.close()
    torch.cuda.synchronize()


def main():
    args = parse()
    world, rank, local, dist = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank, dist)
        if dist is not None:
            dist.destroy_process_group()
        return
    run_ours(args, world, rank, local, dist)


if __name__ == "__main__":
    main()
