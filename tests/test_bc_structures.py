"""The discharge, tailwater, outflow and flux boundary conditions (segment kinds 2-5)
of src/models/sw2/sw2_bc_discharge.c.bk, sw2_bc_tailwater.c.bk, sw2_bc_outflow.c.bk
and sw2_bc_flux.c.bk.

CPU: the oracle's segment residuals and FD Jacobians against the reference's own
boundary integrals, roughness law and drag coefficient composed as the two files do
(harness mode bcx), bit for bit, including dry and edge depths; the oracle's Newton
loop over the structures flume.  GPU: the CUDA element residuals and Jacobians against
the oracle, and the device time loop against the oracle's over 20 steps."""
import numpy as np
import pytest

from adh_kraken_b200.mesh import flume_flux_outflow_case, flume_structures_case
from oracle import refio
from oracle.oracle import OracleModel


def _states(case, seed):
    """Three random states about the initial one; a fifth of the nodes get depths
    0, -0, 1e-300, 1e-20 or small negatives (the dry branches)."""
    rng = np.random.default_rng(seed)
    V = case.nnodes
    sol = case.sol0.copy()
    sol[0::3] += rng.normal(0, 0.2, V)
    sol[1::3] = rng.normal(0.2, 0.3, V)
    sol[2::3] = rng.normal(0, 0.1, V)
    edge = rng.choice(V, V // 5, replace=False)
    sol[3 * edge] = rng.choice([0.0, -0.0, 1e-300, 1e-20, -1e-3], len(edge))
    for kind in np.unique(case.seg_kind):   # one dry node on the first segment of each kind
        sol[3 * case.seg[case.seg_kind == kind][0, 0]] = 0.0
    old = sol + rng.normal(0, 0.01, 3 * V)
    older = old + rng.normal(0, 0.01, 3 * V)
    return sol, old, older


def _fd_eps(u):
    """NUM_DIFF_EPSILON with the 1e-4 floor (src/jacobian/assemble_jacobian.c:313)."""
    e = abs(u) * (1.0 + 1e-4)
    e -= abs(u)
    return e if e >= 1e-4 else 1e-4


def _records(o, case, sol, pert=None):
    """bcx records of every segment; pert = (perturbation, node, var, sign) or None."""
    recs = []
    for k in range(case.nseg):
        a, b = case.seg[k]
        p = (0.0, -1, -1, 0) if pert is None else pert(k)
        recs.append([case.seg_kind[k], o.seg_nrml[2 * k], o.seg_nrml[2 * k + 1], o.seg_djac[k], o.m.dt, case.gravity,
                     sol[3 * a], sol[3 * b], sol[3 * a + 1], sol[3 * a + 2], sol[3 * b + 1], sol[3 * b + 2],
                     case.xyz[a, 2], o.m.bc_flux if case.seg_kind[k] == 5 else o.m.bc_qs, o.m.bc_convey,
                     o.m.bc_rough, o.m.bc_tail, *p])
    return np.array(recs, dtype=np.float64)


needs_harness = pytest.mark.skipif(not refio.harness_available(), reason="reference harness not built")


CASES = {"discharge_tailwater": flume_structures_case, "flux_outflow": flume_flux_outflow_case}


@needs_harness
@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("name", list(CASES))
def test_oracle_structure_residuals_match_reference_integrals(name, seed):
    case = CASES[name](npx=21, npy=6)
    o = OracleModel(case)
    sol, old, older = _states(case, seed)
    o.wd_flags(sol, old)
    _, es = o.elem_resid(sol, old, older)
    ref = refio.run_bcx(_records(o, case, sol))
    assert np.array_equal(es.reshape(-1, 6), ref), np.abs(es.reshape(-1, 6) - ref).max()
    # both kinds took their wet branches somewhere and their dry returns somewhere
    nz = np.abs(ref).sum(1) > 0
    for kind in np.unique(case.seg_kind):
        assert nz[case.seg_kind == kind].any()
        if kind in (2, 3):                 # the two with a dry return
            assert not nz[case.seg_kind == kind].all()


@needs_harness
def test_oracle_structure_residuals_tailwater_below_bed_and_zero_drag():
    """A tailwater elevation below the outlet bed leaves the tailwater segments out;
    zero roughness height gives zero drag, and the discharge law divides by it (both
    sides turn non-finite alike)."""
    case = flume_structures_case(npx=21, npy=6)
    o = OracleModel(case)
    sol, old, older = _states(case, 4)
    o.m.bc_tail = float(case.xyz[:, 2].min()) - 1.0
    o.m.bc_rough = 0.0
    o.wd_flags(sol, old)
    _, es = o.elem_resid(sol, old, older)
    ref = refio.run_bcx(_records(o, case, sol))
    es = es.reshape(-1, 6)
    assert np.array_equal(np.isfinite(es), np.isfinite(ref))
    assert np.array_equal(es[np.isfinite(ref)], ref[np.isfinite(ref)])
    assert not np.isfinite(ref[case.seg_kind == 2]).all()
    assert (ref[case.seg_kind == 3] == 0).all()


@needs_harness
@pytest.mark.parametrize("name", list(CASES))
def test_oracle_structure_jacobians_match_reference_integrals(name):
    case = CASES[name](npx=21, npy=6)
    o = OracleModel(case)
    sol, old, older = _states(case, 3)
    o.wd_flags(sol, old)
    _, js = o.elem_jac(sol, old, older)
    js = js.reshape(-1, 6, 6)
    for node in range(2):
        for var in range(3):
            col = node * 3 + var

            def pert(k, sign):
                u = sol[3 * case.seg[k][node] + var]
                return (_fd_eps(u), node, var, sign)
            P = refio.run_bcx(_records(o, case, sol, lambda k: pert(k, +1)))
            M = refio.run_bcx(_records(o, case, sol, lambda k: pert(k, -1)))
            eps2 = np.array([2.0 * _fd_eps(sol[3 * case.seg[k][node] + var]) for k in range(case.nseg)])
            ref = (P - M) / eps2[:, None]
            assert np.array_equal(js[:, :, col], ref), (col, np.abs(js[:, :, col] - ref).max())


def test_oracle_newton_runs_the_structures_flume():
    """The discharge string feeds ~0.5 m^2/s into the flume and the tailwater string
    holds the outlet: 20 Newton steps converge and the inflow velocity approaches
    q / h = 0.25 m/s."""
    case = flume_structures_case(nsteps=20)
    sol, hist = OracleModel(case).run(20)
    assert len(hist) == 20 and all(h["ok"] for h in hist)
    up = case.seg[case.seg_kind == 2].ravel()
    assert 0.15 < sol[3 * up + 1].mean() < 0.35


def test_oracle_newton_runs_the_flux_outflow_flume():
    """The flux string carries 0.5 m^2/s in and the outflow string lets the water out:
    20 Newton steps converge."""
    case = flume_flux_outflow_case(nsteps=20)
    sol, hist = OracleModel(case).run(20)
    assert len(hist) == 20 and all(h["ok"] for h in hist)
    assert (sol[0::3] > 1.0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_structure_residuals_and_jacobians_match_oracle(name, seed):
    """pow and log are CUDA's on the device and glibc's on the host (each within a few
    ulp of the exact value), so the discharge entries agree to 1e-13 relative to the
    largest entry; the other kinds, which take neither, agree bit for bit."""
    from adh_kraken_b200.capi import SW2Model
    case = CASES[name](npx=21, npy=6)
    o = OracleModel(case)
    g = SW2Model(case, check_csr=(o.indptr, o.cols))
    d, vx, vy = o.bc_values(case.t0, case.t0 + case.dt)
    g.set_step(case.dt, d, vx, vy)
    g.set_bc_structures(o.m.bc_qs, o.m.bc_convey, o.m.bc_rough, o.m.bc_tail)
    g.set_bc_flux(o.m.bc_flux)
    sol, old, older = _states(case, seed)
    o.wd_flags(sol, old)
    _, es = g.elem_resid(sol, old, older)
    _, es_o = o.elem_resid(sol, old, older)
    _, js = g.elem_jac(sol, old, older)
    _, js_o = o.elem_jac(sol, old, older)
    es, es_o = es.reshape(-1, 6), es_o.reshape(-1, 6)
    js, js_o = js.reshape(-1, 36), js_o.reshape(-1, 36)
    tw = case.seg_kind != 2                 # every kind but the discharge takes neither pow nor log
    assert np.array_equal(es[tw], es_o[tw]) and np.array_equal(js[tw], js_o[tw])
    assert np.abs(es - es_o).max() <= 1e-13 * np.abs(es_o).max()
    assert np.abs(js - js_o).max() <= 1e-12 * np.abs(js_o).max()
    r = g.residual(sol, old, older)
    r_o = o.residual(sol, old, older)
    assert np.abs(r - r_o).max() <= 1e-13 * np.abs(r_o).max()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_time_loop_with_structures_matches_oracle(name):
    from adh_kraken_b200.timeloop import SW2Simulation
    from fixtures import rel_err
    case = CASES[name](nsteps=20)
    sim = SW2Simulation(case)
    hist = sim.run(20)
    assert len(hist) == 20 and all(h["success"] for h in hist)
    ref, oh = OracleModel(case).run(20)
    assert all(h["ok"] for h in oh)
    assert max(rel_err(sim.state()[0], ref)) < 1e-8, rel_err(sim.state()[0], ref)
