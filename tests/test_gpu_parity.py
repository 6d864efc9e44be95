"""GPU parity: the CUDA path through the C ABI against the CPU oracle (which is
pinned to the reference by test_oracle_golden.py) and against the reference's
golden outputs directly."""
import numpy as np
import pytest

from fixtures import load, rel_err
from oracle.oracle import OracleModel

pytestmark = pytest.mark.gpu

DUMPS = ["dump_flume_21x6.npz", "dump_wetdry_12.npz"]
# the three-level scheme (tau_temporal 0.5) and a sixth of the nodes at depths 0, -0,
# +-1e-20 and 1e-300: element and assembly parity only (no solve in these dumps)
DUMPS_ALL = DUMPS + ["dump_wetdry_12_tau05.npz", "dump_wetdry_12_edge_depths.npz"]
RUNS = ["run_flume_21x6_8steps.npz", "run_wetdry_12_4steps.npz"]


def gpu_model(case, tau=0.0):
    from adh_kraken_b200.capi import SW2Model
    o = OracleModel(case)
    g = SW2Model(case, check_csr=(o.indptr, o.cols))
    d, vx, vy = o.bc_values(case.t0, case.t0 + case.dt)
    g.set_step(case.dt, d, vx, vy, tau_temporal=tau)
    return g, o


def _tau(z):
    return float(z["tau"]) if "tau" in z.files else 0.0


@pytest.mark.parametrize("name", DUMPS_ALL)
def test_csr_structure_bit_exact(name):
    case, z = load(name)
    g, _ = gpu_model(case, _tau(z))
    ip, cl = g.sparsity()
    assert np.array_equal(ip, z["ref_indptr"]) and np.array_equal(cl, z["ref_cols"])


@pytest.mark.parametrize("name", DUMPS_ALL)
def test_element_residuals_and_jacobians_bit_exact(name):
    case, z = load(name)
    g, _ = gpu_model(case, _tau(z))
    sol, old, older = z["sol"], z["sol_old"], z["sol_older"]
    assert np.array_equal(g.wd_flags(sol, old), z["ref_wd_flag"])
    et, es = g.elem_resid(sol, old, older)
    assert np.array_equal(et, z["ref_elem_rhs_tri"]), np.abs(et - z["ref_elem_rhs_tri"]).max()
    assert np.array_equal(es, z["ref_elem_rhs_seg"])
    jt, js = g.elem_jac(sol, old, older)
    assert np.array_equal(jt, z["ref_elem_jac_tri"]), np.abs(jt - z["ref_elem_jac_tri"]).max()
    assert np.array_equal(js, z["ref_elem_jac_seg"])


@pytest.mark.parametrize("name", DUMPS_ALL)
def test_assembly_bit_exact(name):
    case, z = load(name)
    g, _ = gpu_model(case, _tau(z))
    sol, old, older = z["sol"], z["sol_old"], z["sol_older"]
    assert np.array_equal(g.residual(sol, old, older), z["ref_residual"])
    assert np.array_equal(g.jacobian(sol, old, older), z["ref_jac_vals"])


@pytest.mark.parametrize("name", DUMPS_ALL)
def test_dirichlet_and_scaling_bit_exact(name):
    case, z = load(name)
    g, _ = gpu_model(case, _tau(z))
    vals, res, x, bc, scale = g.prepare_system(z["ref_jac_vals"], z["ref_residual"], np.zeros(3 * case.nnodes),
                                               np.zeros(3 * case.nnodes, np.int32))
    assert np.array_equal(bc, (z["ref_bc_mask"] == 1).astype(np.int32))
    assert np.array_equal(scale, z["ref_scale_vect"])
    assert np.array_equal(vals, z["ref_jac_vals_scaled"])
    assert np.array_equal(res, z["ref_residual_scaled"])


PRECONDS = [0, 1, 2]   # block-Jacobi, block ILU(0), aggregation AMG


@pytest.mark.parametrize("precond", PRECONDS)
@pytest.mark.parametrize("name", DUMPS)
def test_bicgstab_reaches_reference_solution(name, precond):
    case, z = load(name)
    g, _ = gpu_model(case)
    x, b, it = g.bicgstab(z["ref_jac_vals_scaled"], z["ref_residual_scaled"], np.zeros(3 * case.nnodes),
                          z["ref_scale_vect"], max_it=20000, tol=1e-13, precond=precond)
    assert it > 0
    ref = z["ref_dsol"]
    # the two preconditioners reach the same solution to the conditioning of the system
    assert np.abs(x - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("name", RUNS)
def test_time_steps_match_reference(name):
    from adh_kraken_b200.timeloop import SW2Simulation
    case, z = load(name)
    sim = SW2Simulation(case)
    hist = sim.run(case.nsteps)
    assert len(hist) == case.nsteps and all(h["success"] for h in hist)
    sol = sim.state()[0]
    ref = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)[-1]
    assert max(rel_err(sol, ref)) < 1e-8, rel_err(sol, ref)


@pytest.mark.parametrize("krylov", [0, 1])   # BiCGStab, restarted GMRES
@pytest.mark.parametrize("precond", [1, 2])
@pytest.mark.parametrize("name", RUNS)
def test_time_steps_match_reference_each_solver(name, precond, krylov):
    from adh_kraken_b200.capi import default_opts
    from adh_kraken_b200.timeloop import SW2Simulation
    case, z = load(name)
    sim = SW2Simulation(case, opts=default_opts(precond=precond, krylov_method=krylov))
    hist = sim.run(case.nsteps)
    assert all(h["success"] for h in hist)
    sol = sim.state()[0]
    ref = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)[-1]
    assert max(rel_err(sol, ref)) < 1e-8, rel_err(sol, ref)


@pytest.mark.parametrize("krylov", [0, 1])
@pytest.mark.parametrize("precond", [1, 2])
@pytest.mark.parametrize("name", RUNS)
def test_fp32_krylov_with_refinement_matches_reference(name, precond, krylov):
    from adh_kraken_b200.capi import default_opts
    from adh_kraken_b200.timeloop import SW2Simulation
    case, z = load(name)
    sim = SW2Simulation(case, opts=default_opts(krylov_precision=32, precond=precond, krylov_method=krylov))
    hist = sim.run(case.nsteps)
    assert all(h["success"] for h in hist)
    sol = sim.state()[0]
    ref = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)[-1]
    assert max(rel_err(sol, ref)) < 1e-8, rel_err(sol, ref)


@pytest.mark.parametrize("name", RUNS)
def test_fp32_gmres_cycles_in_fp64_refinement_match_reference(name):
    """Whole GMRES cycles in FP32 (basis, SpMV, AMG), refined from the FP64 residual."""
    from adh_kraken_b200.capi import default_opts
    from adh_kraken_b200.timeloop import SW2Simulation
    case, z = load(name)
    sim = SW2Simulation(case, opts=default_opts(krylov_precision=32, krylov_basis_precision=32, precond=2,
                                                krylov_method=1))
    hist = sim.run(case.nsteps)
    assert all(h["success"] for h in hist)
    sol = sim.state()[0]
    ref = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)[-1]
    assert max(rel_err(sol, ref)) < 1e-8, rel_err(sol, ref)


def test_still_beach_kat_matches_reference():
    """Still water on a sloping beach with a dry upper part and no boundary
    segments (src/test/test_sw2_wd.c): 1440 steps, the kept states within 1e-8 of
    the reference's run, the water at rest, wet depths unchanged, mass kept."""
    from adh_kraken_b200.timeloop import SW2Simulation
    case, z = load("run_still_beach_16x6_1440steps.npz")
    ref = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)
    sim = SW2Simulation(case)
    kept = []
    for k in range(case.nsteps):
        assert sim.step()["success"]
        if (k + 1) % 240 == 0:
            kept.append(sim.state()[0])
    kept = np.array(kept)
    assert np.abs(kept - ref).max() < 1e-8
    h0 = case.sol0[0::3]
    wet = h0 > 0.0
    m0 = sim.model.grid_mass(case.sol0)[0]
    for s in kept:
        assert np.abs(s[1::3]).sum() + np.abs(s[2::3]).sum() < 1e-7
        assert np.abs(s[0::3][wet] - h0[wet]).sum() < 1e-7
        assert np.abs(s[0::3][~wet]).max() < 1e-9
        assert abs(sim.model.grid_mass(s)[0] - m0) <= 1e-12 * m0


def test_undo_step_retries_the_interval():
    """A failed Newton solve undone with sw2g_undo_step, then the same interval
    again: the result is the state an unbroken first step reaches."""
    from adh_kraken_b200.capi import SW2Error, default_opts
    from adh_kraken_b200.timeloop import SW2Simulation
    case, z = load("run_flume_21x6_8steps.npz")
    a = SW2Simulation(case)
    assert a.step()["success"]
    sa = a.state()[0]
    b = SW2Simulation(case)
    st = b.step(opts=default_opts(max_nonlin_it=1, krylov_max_it=1))
    assert not st["success"]
    b.model.undo_step()
    b.t -= case.dt
    with pytest.raises(SW2Error):
        b.model.undo_step()                  # only once per step
    assert b.step()["success"]
    assert max(rel_err(b.state()[0], sa)) < 1e-10
    c = SW2Simulation(case)
    adv = c.advance()
    assert adv["success"] == 1 and adv["substeps"] == 1 and adv["dt_cuts"] == 0
    assert max(rel_err(c.state()[0], sa)) < 1e-10


BENCH_OPTS = dict(tol_nonlin=1e-8, tol_nonlin_rel=1e-8, inc_nonlin=1e-6, max_nonlin_it=10, krylov_max_it=20000,
                  krylov_tol=1e-6, precond=2, krylov_method=1, krylov_restart=100)


@pytest.mark.parametrize("mode", ["reference_test", "bench_fast", "bench_plain"])
def test_config1_flume_100_steps_match_reference(mode):
    """The CPU-runnable benchmark configuration (101 x 11 flume, 2000 triangles, 100
    steps of 60 s): every 10th state within 1e-8 relative (h, u, v) of the reference's
    run, with the reference's absolute Newton test and with the benchmark's options
    (relative Newton test 1e-8, forcing 1e-6, GMRES(50) + AMG; the fast path in FP32
    GMRES cycles inside FP64 refinement, the plain path in FP64)."""
    from adh_kraken_b200.capi import default_opts
    from adh_kraken_b200.timeloop import SW2Simulation
    case, z = load("run_flume_101x11_100steps.npz")
    ref = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)
    if mode == "reference_test":
        opts = default_opts()
    elif mode == "bench_fast":
        opts = default_opts(krylov_precision=32, krylov_basis_precision=32, **BENCH_OPTS)
    else:
        opts = default_opts(krylov_precision=64, **BENCH_OPTS)
    sim = SW2Simulation(case, opts=opts)
    worst = 0.0
    for k in range(case.nsteps):
        assert sim.step()["success"], k
        if (k + 1) % 10 == 0:
            worst = max(worst, max(rel_err(sim.state()[0], ref[(k + 1) // 10 - 1])))
    assert worst < 1e-8, worst


@pytest.mark.parametrize("name", ["run_wetdry_12_4steps.npz", "run_still_beach_16x6_1440steps.npz"])
def test_amg_chunk_corrections_are_exercised_and_match_reference(name):
    """The AMG's chunk corrections (amg_chunks = 2: exact solves on the chunks of nodes whose
    block-Jacobi smoothing the l1 fix-up weakens, inside the V-cycle) run on wet/dry meshes,
    invert every chunk, and the steps still land on the reference's states to 1e-8."""
    from adh_kraken_b200.capi import default_opts
    from adh_kraken_b200.timeloop import SW2Simulation
    case, z = load(name)
    sim = SW2Simulation(case, opts=default_opts(precond=2, krylov_method=1, amg_chunks=2))
    nsteps = min(case.nsteps, 6)
    seen = 0
    for _ in range(nsteps):
        assert sim.step()["success"]
        info = sim.model.precond_info()
        assert info["singular_chunks"] == 0
        seen = max(seen, info["chunks"])
    assert seen > 0
    if nsteps == case.nsteps:
        ref = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)[-1]
        assert max(rel_err(sim.state()[0], ref)) < 1e-8
