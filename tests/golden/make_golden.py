"""Generate the golden fixtures in tests/golden/ by running the reference's own
compiled SW2 code (oracle/_ref/adh_ref_harness, built by oracle/Makefile from the
reference sources).  Run it on a machine that has the reference tree:

    make -C oracle all && python tests/golden/make_golden.py

Each fixture is a compressed .npz holding the case inputs (mesh, states, series)
and what the reference computed for them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from adh_kraken_b200.mesh import basin_case, flume_case, small_delaunay_case, still_beach_case  # noqa: E402
from oracle.refio import run_harness  # noqa: E402


def perturbed_states(case, seed):
    rng = np.random.default_rng(seed)
    V = case.nnodes
    sol = case.sol0.copy(); sol_old = case.sol0.copy(); sol_older = case.sol0.copy()
    sol[0::3] += 0.01 * rng.standard_normal(V)
    sol[1::3] += 0.05 * rng.standard_normal(V)
    sol[2::3] += 0.05 * rng.standard_normal(V)
    sol_older[0::3] -= 0.01 * rng.standard_normal(V)
    return sol, sol_old, sol_older


def case_arrays(case):
    out = {"xyz": case.xyz, "tri": case.tri, "seg": case.seg, "seg_kind": case.seg_kind, "sol0": case.sol0,
           "dt": case.dt, "nsteps": case.nsteps, "t0": case.t0}
    for k, (t, v) in case.series.items():
        out[f"series{k}_t"] = t
        out[f"series{k}_v"] = v
    return out


def edge_depths(case, sol, seed):
    """Put a sixth of the nodes at depths on the wet/dry boundary: exactly 0, -0,
    +-1e-20 and 1e-300 (the current level only; the old level keeps the wet/dry flags
    of the perturbed state)."""
    rng = np.random.default_rng(seed)
    nodes = rng.choice(case.nnodes, size=case.nnodes // 6, replace=False)
    vals = np.array([0.0, -1e-20, 1e-20, 1e-300, -0.0])
    sol = sol.copy()
    sol[3 * nodes] = vals[np.arange(len(nodes)) % len(vals)]
    return sol


def dump_fixture(name, case, seed, tau=0.0, edge=False):
    sol, sol_old, sol_older = perturbed_states(case, seed)
    if edge:
        sol = edge_depths(case, sol, seed + 1)
    env = {"HARNESS_TAU": repr(tau), "HARNESS_SKIP_SOLVE": "1"} if (tau or edge) else None
    d = run_harness("dump", case, sol=sol, sol_old=sol_old, sol_older=sol_older, env=env)
    arrs = case_arrays(case)
    arrs.update({"sol": sol, "sol_old": sol_old, "sol_older": sol_older, "tau": tau})
    arrs.update({f"ref_{k}": v for k, v in d.items()})
    np.savez_compressed(os.path.join(HERE, name), **arrs)


def run_fixture(name, case, every=1):
    r = run_harness("run", case, extra=(every,))
    arrs = case_arrays(case)
    arrs.update({f"ref_{k}": v for k, v in r.items() if k != "step_seconds"})
    np.savez_compressed(os.path.join(HERE, name), **arrs)


def mass_states(case, seed, run_name=None):
    """State triples for the mass-balance fixture: perturbed states, one with nodes
    at exactly zero depth and at -1e-20 (the near-empty dry-corner branch of
    fe_3m2d_dry_wet_factornew), and the reference run's last kept state."""
    out = [perturbed_states(case, seed)]
    sol, sol_old, sol_older = perturbed_states(case, seed + 1)
    rng = np.random.default_rng(seed + 2)
    nodes = rng.choice(case.nnodes, size=max(2, case.nnodes // 8), replace=False)
    half = len(nodes) // 2
    sol[3 * nodes[:half]] = 0.0
    sol[3 * nodes[half:]] = -1e-20
    out.append((sol, sol_old, sol_older))
    if run_name is not None:
        z = np.load(os.path.join(HERE, run_name))
        kept = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)
        last = kept[-1].copy()
        prev = kept[-2].copy() if len(kept) > 1 else case.sol0.copy()
        out.append((last, prev, prev))
    return out


def mass_fixture(name, case, seed, run_name=None):
    states = mass_states(case, seed, run_name)
    res = []
    for sol, sol_old, sol_older in states:
        d = run_harness("mass", case, sol=sol, sol_old=sol_old, sol_older=sol_older)
        res.append(d["grid_mass"])
    arrs = case_arrays(case)
    arrs["sol"] = np.stack([s[0] for s in states])
    arrs["sol_old"] = np.stack([s[1] for s in states])
    arrs["ref_grid_mass"] = np.stack(res)   # per state: mass(sol), mass(sol_old), boundary flux, mass error
    np.savez_compressed(os.path.join(HERE, name), **arrs)


def main():
    dump_fixture("dump_flume_21x6.npz", flume_case(nsteps=1, npx=21, npy=6), seed=11)
    dump_fixture("dump_wetdry_12.npz", small_delaunay_case(n=12, seed=5, nsteps=1), seed=12)
    dump_fixture("dump_wetdry_12_tau05.npz", small_delaunay_case(n=12, seed=5, nsteps=1), seed=13, tau=0.5)
    dump_fixture("dump_wetdry_12_edge_depths.npz", small_delaunay_case(n=12, seed=5, nsteps=1), seed=17, edge=True)
    run_fixture("run_flume_21x6_8steps.npz", flume_case(nsteps=8, npx=21, npy=6))
    run_fixture("run_wetdry_12_4steps.npz", small_delaunay_case(n=12, seed=5, nsteps=4))
    run_fixture("run_still_beach_16x6_1440steps.npz", still_beach_case(nsteps=1440), every=240)
    # the CPU-runnable benchmark configuration: 101 x 11 flume, 100 steps of 60 s (every 10th state kept)
    run_fixture("run_flume_101x11_100steps.npz", flume_case(nsteps=100), every=10)
    run_fixture("run_basin_12_6steps.npz", basin_case(n=12, seed=2, nsteps=6))
    # dt 600 s: four line-search halvings in the first Newton solve; dt 150 s: a failed solve
    run_fixture("run_wetdry_12_dt600_6steps.npz", small_delaunay_case(n=12, seed=5, nsteps=6, dt=600.0))
    run_fixture("run_wetdry_12_dt150_fail.npz", small_delaunay_case(n=12, seed=5, nsteps=3, dt=150.0))
    mass_fixture("mass_flume_21x6.npz", flume_case(nsteps=8, npx=21, npy=6), 31, "run_flume_21x6_8steps.npz")
    mass_fixture("mass_wetdry_12.npz", small_delaunay_case(n=12, seed=5, nsteps=4), 41, "run_wetdry_12_4steps.npz")
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
