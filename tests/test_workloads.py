"""The synthetic workloads' construction (no GPU): the learned-guess basin with inflow
hydrographs keeps config 2's mesh, bathymetry and tide, adds a velocity string on the
east edge, draws its peak discharge from the seed, and runs on the CPU oracle."""
import numpy as np

from adh_kraken_b200.mesh import basin_case, basin_hydro_case
from oracle.oracle import OracleModel


def test_basin_hydro_case_keeps_the_basin_and_adds_the_inflow():
    base = basin_case(n=20, seed=2, nsteps=3)
    c = basin_hydro_case(44, n=20, nsteps=3)
    assert np.array_equal(c.xyz, base.xyz) and np.array_equal(c.tri, base.tri)
    assert np.array_equal(c.seg[: base.nseg], base.seg) and (c.seg_kind[: base.nseg] == 1).all()
    east = c.seg[base.nseg:]
    assert len(east) == 19 and (c.seg_kind[base.nseg:] == 0).all()
    assert np.allclose(c.xyz[east.ravel(), 0], 20000.0)
    # outward normal (dy, -dx) of the east string points to +x
    a, b = c.xyz[east[:, 0], :2], c.xyz[east[:, 1], :2]
    assert ((b[:, 1] - a[:, 1]) > 0).all()
    assert 1000.0 <= c.q_peak <= 3000.0
    assert c.q_peak != basin_hydro_case(45, n=20, nsteps=3).q_peak
    t, v = c.series[1]
    assert np.isclose(v[0], -200.0 / 2e5) and v.min() >= -c.q_peak / 2e5 - 1e-15


def test_basin_hydro_case_steps_on_the_oracle():
    c = basin_hydro_case(41, n=16, nsteps=2)
    sol, hist = OracleModel(c).run(2, krylov_max_it=20000)
    assert all(h["ok"] for h in hist)
    assert np.isfinite(sol).all() and sol[0::3].min() > 0


def test_estuary_case_has_tide_river_and_dry_land():
    from adh_kraken_b200.mesh import estuary_case
    c = estuary_case(nx=240, ny=120, nsteps=2)
    depth_edge = c.seg[c.seg_kind == 1]
    river = c.seg[c.seg_kind == 0]
    assert len(depth_edge) == 119 and len(river) >= 1
    assert np.allclose(c.xyz[np.unique(depth_edge.ravel()), 2], -30.0)     # flat tidal edge
    assert np.allclose(c.xyz[river.ravel(), 0], 80000.0)
    dry = (c.sol0[0::3] <= 0).mean()
    assert 0.0 < dry < 0.2                                                 # partial wet/dry
    t, v = c.series[0]
    assert np.allclose(v, 30.0 + 1.5 * np.sin(2 * np.pi * t / (12.42 * 3600.0)))
    assert np.isclose(c.series[1][1][0], -0.4)                             # 800 m^3/s through 500 m x 4 m
