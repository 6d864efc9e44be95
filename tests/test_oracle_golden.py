"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the compiled reference)."""
import numpy as np
import pytest

from fixtures import load, rel_err
from oracle.oracle import OracleModel

DUMPS = ["dump_flume_21x6.npz", "dump_wetdry_12.npz"]
# the three-level temporal scheme (tau_temporal = 0.5; the reference's default is 0), and
# depths on the wet/dry boundary (exactly 0, -0, +-1e-20, 1e-300) at a sixth of the nodes
DUMPS_TAU = DUMPS + ["dump_wetdry_12_tau05.npz", "dump_wetdry_12_edge_depths.npz"]


def oracle_for(case, z):
    return OracleModel(case, tau_temporal=float(z["tau"]) if "tau" in z.files else 0.0)
RUNS = ["run_flume_21x6_8steps.npz", "run_wetdry_12_4steps.npz",
        "run_basin_12_6steps.npz",          # tidal depth boundary, a 1 m / 12.42 h sine series
        "run_wetdry_12_dt600_6steps.npz"]   # line-search halvings in the first solve


@pytest.mark.parametrize("name", DUMPS)
def test_structure_and_maps(name):
    case, z = load(name)
    o = OracleModel(case)
    assert np.array_equal(o.indptr, z["ref_indptr"])
    assert np.array_equal(o.cols, z["ref_cols"])
    V = case.nnodes
    assert np.array_equal(z["ref_dofmap"].reshape(3, V).T.ravel(), np.arange(3 * V)), "dof = 3*node + var"


@pytest.mark.parametrize("name", DUMPS)
def test_bc_series_average(name):
    case, z = load(name)
    o = OracleModel(case)
    assert np.array_equal(np.array(o.bc_values(case.t0, case.t0 + case.dt)), z["ref_bc_values"])


@pytest.mark.parametrize("name", DUMPS_TAU)
def test_element_level_bit_exact(name):
    case, z = load(name)
    o = oracle_for(case, z)
    sol, old, older = z["sol"], z["sol_old"], z["sol_older"]
    assert np.array_equal(o.wd_flags(sol, old), z["ref_wd_flag"])
    et, es = o.elem_resid(sol, old, older)
    assert np.array_equal(et, z["ref_elem_rhs_tri"])
    assert np.array_equal(es, z["ref_elem_rhs_seg"])
    jt, js = o.elem_jac(sol, old, older)
    assert np.array_equal(jt, z["ref_elem_jac_tri"])
    assert np.array_equal(js, z["ref_elem_jac_seg"])


@pytest.mark.parametrize("name", DUMPS_TAU)
def test_assembly_and_linear_system_bit_exact(name):
    case, z = load(name)
    o = oracle_for(case, z)
    sol, old, older = z["sol"], z["sol_old"], z["sol_older"]
    o.wd_flags(sol, old)
    r = o.residual(sol, old, older)
    v = o.jacobian(sol, old, older)
    assert np.array_equal(r, z["ref_residual"])
    assert np.array_equal(v, z["ref_jac_vals"])
    bc = np.zeros(o.ndof, np.int32)
    o.check_diag(v, bc)
    o.apply_dirichlet(bc, v, r)
    assert np.array_equal(bc, (z["ref_bc_mask"] == 1).astype(np.int32))
    assert np.array_equal(v, z["ref_jac_vals_dirichlet"])
    assert np.array_equal(r, z["ref_residual_dirichlet"])
    x = np.zeros(o.ndof)
    s = o.scale_system(v, r, x)
    assert np.array_equal(s, z["ref_scale_vect"])
    assert np.array_equal(v, z["ref_jac_vals_scaled"])
    assert np.array_equal(r, z["ref_residual_scaled"])


@pytest.mark.parametrize("name", DUMPS)
def test_bicgstab_block_jacobi_solves_reference_system(name):
    """Block-Jacobi BiCGStab reaches the reference's exact-LU solution of the same
    scaled system to solver tolerance."""
    case, z = load(name)
    o = OracleModel(case)
    v = z["ref_jac_vals_scaled"].copy(); b = z["ref_residual_scaled"].copy(); x = np.zeros(o.ndof)
    it = o.bicgstab(v, x, b, z["ref_scale_vect"], max_it=20000, tol=1e-13)
    ref = z["ref_dsol"]
    assert it > 0
    # the two preconditioners reach the same solution to the conditioning of the system
    assert np.abs(x - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("name", RUNS)
def test_time_steps_match_reference(name):
    """Several implicit steps with block-Jacobi BiCGStab land on the reference's
    converged states (exact LU preconditioner) within 1e-8 relative."""
    case, z = load(name)
    o = OracleModel(case)
    sol, hist = o.run(case.nsteps, krylov_max_it=20000)
    assert all(h["ok"] for h in hist)
    ref = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)[-1]
    assert max(rel_err(sol, ref)) < 1e-8


@pytest.mark.parametrize("name", RUNS)
def test_step_averaged_series_every_step(name):
    """sseries_setall_ts_valuesAVG over each step's [t - dt, t], bit for bit, on every
    step of the runs (the basin's tide has four samples per step)."""
    case, z = load(name)
    o = OracleModel(case)
    n = len(z["ref_step_ok"])
    mine = [o.bc_values(case.t0 + k * case.dt, case.t0 + (k + 1) * case.dt) for k in range(n)]
    assert np.array_equal(np.array(mine).ravel(), z["ref_bc_values"])


def test_line_search_is_exercised():
    """The dt = 600 s run halves its first Newton increments (fe_newton.c:681-741)
    and still lands on the reference's states (test_time_steps_match_reference)."""
    case, z = load("run_wetdry_12_dt600_6steps.npz")
    o = OracleModel(case)
    _, hist = o.run(2, krylov_max_it=20000)
    assert hist[0]["linesearch_cuts"] >= 3 and hist[0]["newton_its"] == int(z["ref_newton_its"][0])


def test_failed_newton_solve_resets_like_the_reference():
    """dt = 150 s: the first solve fails after max_nonlin_it iterations in the
    reference as in the oracle; both reset the state to the start of the step with the
    Dirichlet values and the dry-node marks (fe_newton.c:893-899), bit for bit."""
    case, z = load("run_wetdry_12_dt150_fail.npz")
    assert z["ref_step_ok"].tolist() == [0]
    o = OracleModel(case)
    sol = case.sol0.copy(); old = sol.copy(); older = sol.copy()
    bc = np.zeros(o.ndof, np.int32)
    o.set_bc_window(case.t0, case.t0 + case.dt)
    st = o.newton(sol, old, older, bc, np.zeros(o.ndof), krylov_max_it=20000)
    assert not st["ok"] and st["newton_its"] == int(z["ref_newton_its"][0])
    assert np.array_equal(sol, z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)[-1])
    assert np.array_equal(bc, (z["ref_bc_mask"] == 1).astype(np.int32))


MASS = ["mass_flume_21x6.npz", "mass_wetdry_12.npz"]


@pytest.mark.parametrize("name", MASS)
def test_grid_mass_and_boundary_flux_bit_exact(name):
    """tl_find_grid_mass_elem2d and the boundary loop of tl_find_grid_mass_error_elem2d
    (src/tools/tl_grid_mass.c:198, :280): the oracle sums the same per-element terms
    in the same element order, so totals agree to the bit."""
    case, z = load(name)
    o = OracleModel(case)
    for k in range(z["sol"].shape[0]):
        sol, old = z["sol"][k], z["sol_old"][k]
        m_new, m_old, flux, err = z["ref_grid_mass"][k]
        assert o.grid_mass(sol) == m_new
        assert o.grid_mass(old) == m_old
        # the reference weights every boundary segment by the first one's length
        f = o.boundary_mass_flux(sol, first_seg_length=True)
        assert f == flux
        assert abs(o.grid_mass(sol) - f - o.grid_mass(old)) == err
        # segment lengths agree to rounding in these meshes: own lengths change the last bits only
        assert abs(o.boundary_mass_flux(sol) - flux) <= 1e-13 * max(abs(flux), 1.0)


def test_grid_mass_covers_every_dry_branch():
    """The wet/dry fixture's states reach every case of fe_3m2d_dry_wet_factornew:
    0-3 dry vertices and the near-empty dry corner that counts as wet."""
    case, z = load("mass_wetdry_12.npz")
    tri = case.tri
    seen = set()
    for k in range(z["sol"].shape[0]):
        h = z["sol"][k][0::3][tri]
        seen |= set(np.unique((h < 0).sum(axis=1)).tolist())
        if np.any(h == -1e-20):
            seen.add("tiny")
    assert seen >= {0, 1, 2, 3, "tiny"}


def still_beach_checks(case, states, mass_of):
    """The still-water beach (src/test/test_sw2_wd.c:232-263): the water stays at
    rest (sum |u| + sum |v| below the test's 1e-7), wet depths stay put, and the mass
    is kept.  Dry nodes (h0 < 0) go to h = 0 in the first step, in the reference as
    here, which the reference test's sum |h - h0| would count as an error."""
    h0 = case.sol0[0::3]
    wet = h0 > 0.0
    m0 = mass_of(case.sol0)
    for s in states:
        assert np.abs(s[1::3]).sum() + np.abs(s[2::3]).sum() < 1e-7
        assert np.abs(s[0::3][wet] - h0[wet]).sum() < 1e-7
        assert np.abs(s[0::3][~wet]).max() < 1e-9
        assert abs(mass_of(s) - m0) <= 1e-12 * m0


def test_still_beach_kat_matches_reference():
    case, z = load("run_still_beach_16x6_1440steps.npz")
    o = OracleModel(case)
    ref = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)
    assert z["ref_step_ok"].all() and len(ref) == 6
    sol = case.sol0.copy(); old = sol.copy(); older = sol.copy()
    bc_mask = np.zeros(o.ndof, np.int32); dirichlet = np.zeros(o.ndof)
    t, kept = case.t0, []
    for k in range(case.nsteps):
        t += case.dt
        older[:] = old; old[:] = sol
        o.set_bc_window(t - case.dt, t)
        st = o.newton(sol, old, older, bc_mask, dirichlet)
        assert st["ok"]
        if (k + 1) % 240 == 0:
            kept.append(sol.copy())
    assert np.abs(np.array(kept) - ref).max() < 1e-10
    still_beach_checks(case, ref, o.grid_mass)
    still_beach_checks(case, kept, o.grid_mass)
