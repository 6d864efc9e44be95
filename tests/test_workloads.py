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
