"""Mass balance on the GPU (sw2g_grid_mass) against the CPU oracle, which
test_oracle_golden.py pins to the reference's tl_find_grid_mass_elem2d and
tl_find_grid_mass_error_elem2d (src/tools/tl_grid_mass.c:198, :280).

Per-triangle terms are bit-identical; the totals are sums in a different order
(block partials instead of the reference's serial loop), so they agree to a
relative 1e-13."""
import numpy as np
import pytest

from fixtures import load
from oracle.oracle import OracleModel

pytestmark = pytest.mark.gpu

MASS = ["mass_flume_21x6.npz", "mass_wetdry_12.npz"]
SUM_RTOL = 1e-13


def gpu_model(case):
    from adh_kraken_b200.capi import SW2Model
    o = OracleModel(case)
    return SW2Model(case, check_csr=(o.indptr, o.cols)), o


@pytest.mark.parametrize("name", MASS)
def test_grid_mass_matches_reference(name):
    case, z = load(name)
    g, o = gpu_model(case)
    for k in range(z["sol"].shape[0]):
        sol = z["sol"][k]
        m_new, _, flux_ref, _ = z["ref_grid_mass"][k]
        mass, flux, em = g.grid_mass(sol, elem=True)
        assert np.array_equal(em, o.elem_mass(sol))
        assert abs(mass - m_new) <= SUM_RTOL * abs(m_new)
        assert abs(flux - o.boundary_mass_flux(sol)) <= SUM_RTOL * max(abs(flux_ref), 1.0)
        assert abs(flux - flux_ref) <= SUM_RTOL * max(abs(flux_ref), 1.0)
        rho_mass, rho_flux = g.grid_mass(sol, density=1000.0, dt=2.0 * case.dt)
        assert abs(rho_mass - 1000.0 * mass) <= SUM_RTOL * abs(rho_mass)
        assert abs(rho_flux - 2000.0 * flux) <= SUM_RTOL * max(abs(rho_flux), 1.0)


def test_resident_state_mass_and_run_to_run_identical():
    case, z = load("mass_wetdry_12.npz")
    g, _ = gpu_model(case)
    sol = z["sol"][0]
    g.load_state(sol, z["sol_old"][0], z["sol_old"][0])
    a = g.grid_mass(None)
    b = g.grid_mass(sol)
    assert a == b and g.grid_mass(None) == a


def test_grid_mass_beach_strip_elementwise():
    """A 120k-triangle wet/dry beach strip: every per-triangle term bit-identical to
    the oracle, and the total equal to the exactly rounded sum of the terms to 1e-13."""
    import math
    from adh_kraken_b200.mesh import beach_case
    case = beach_case(nx=1000, ny=60, seed=3, nsteps=1, ly=850.0)
    g, o = gpu_model(case)
    rng = np.random.default_rng(7)
    sol = case.sol0.copy()
    sol[0::3] += 0.05 * rng.standard_normal(case.nnodes)
    mass, flux, em = g.grid_mass(sol, elem=True)
    ref = o.elem_mass(sol)
    assert np.array_equal(em, ref)
    exact = math.fsum(ref.tolist())
    assert abs(mass - exact) <= SUM_RTOL * abs(exact)
    assert abs(flux - o.boundary_mass_flux(sol)) <= SUM_RTOL * max(abs(flux), 1.0)
