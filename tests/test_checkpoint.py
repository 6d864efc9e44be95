"""Checkpoint / resume of the time loop, on CPU: SW2Simulation drives a stand-in
model that steps with the CPU oracle (test infrastructure), so the host logic --
level rotation, forcing windows, state files -- is checked with real numerics.
A resumed run takes the same steps as the uninterrupted one, bit for bit."""
import numpy as np

from adh_kraken_b200.deck import read_init, write_init
from adh_kraken_b200.mesh import small_delaunay_case
from adh_kraken_b200.timeloop import SW2Simulation
from oracle.oracle import OracleModel


class OracleStepper:
    """The calls SW2Simulation makes on its model, answered by the oracle."""

    def __init__(self, case):
        self.o = OracleModel(case)
        n = 3 * case.nnodes
        self.sol, self.old, self.older = np.zeros(n), np.zeros(n), np.zeros(n)
        self.mask, self.dirichlet = np.zeros(n, np.int32), np.zeros(n)

    def set_step(self, dt, d, vx, vy, tau_temporal=0.0):
        self.o.m.dt = dt
        self.o.m.bc_depth, self.o.m.bc_vx, self.o.m.bc_vy = d, vx, vy

    def load_state(self, sol, sol_old, sol_older, bc_mask=None, dirichlet=None):
        self.sol, self.old, self.older = (np.array(a, dtype=np.float64) for a in (sol, sol_old, sol_older))
        self.mask = np.zeros(self.sol.size, np.int32) if bc_mask is None else np.array(bc_mask, np.int32)

    def store_state(self):
        return self.sol.copy(), self.old.copy(), self.older.copy(), self.mask.copy()

    def step(self, opts=None):
        self.before = (self.sol.copy(), self.old.copy(), self.older.copy())
        self.older, self.old = self.old, self.sol.copy()      # smodel_super_prep_sol
        st = self.o.newton(self.sol, self.old, self.older, self.mask, self.dirichlet, krylov_max_it=20000)
        return {"success": int(st["ok"]), "newton_its": st["newton_its"], "krylov_its": st["krylov_its"]}

    def undo_step(self):
        # as sw2g_undo_step turns the level rotation back: the start state and its
        # previous level return, the sol_older level keeps the failed step's buffer
        failed = self.sol
        self.sol, self.old = self.before[0], self.before[1]
        self.older = failed

    def grid_mass(self, sol=None, density=1.0, dt=None):
        s = self.sol if sol is None else sol
        return self.o.grid_mass(s, density), self.o.boundary_mass_flux(s, density, dt)


def test_resume_from_checkpoint_is_bit_exact(tmp_path):
    case = small_delaunay_case(n=12, seed=5, nsteps=4)
    full = SW2Simulation(case, model=OracleStepper(case))
    full.run(4)
    first = SW2Simulation(case, model=OracleStepper(case))
    first.run(2)
    ck = str(tmp_path / "ck.npz")
    first.checkpoint(ck)
    resumed = SW2Simulation(case, model=OracleStepper(case))
    resumed.restore(ck)
    resumed.run(2)
    assert resumed.t == full.t
    for a, b in zip(resumed.state(), full.state()):
        assert np.array_equal(a, b)
    assert [h["newton_its"] for h in first.history + resumed.history] == [h["newton_its"] for h in full.history]


def test_resume_through_the_reference_restart_format(tmp_path):
    """The same through an .init file (the reference's DATASET restart format): the
    three levels round-trip exactly, so the resumed step is the same."""
    case = small_delaunay_case(n=12, seed=5, nsteps=3)
    full = SW2Simulation(case, model=OracleStepper(case))
    full.run(3)
    first = SW2Simulation(case, model=OracleStepper(case))
    first.run(2)
    sol, old, older, mask = first.state()
    init = str(tmp_path / "restart.init")
    write_init(init, sol, old, older, nelems=case.ntri, t=first.t)
    resumed = SW2Simulation(case, model=OracleStepper(case))
    resumed.model.load_state(*read_init(init, case.nnodes), bc_mask=mask)
    resumed.t = first.t
    resumed.run(1)
    assert np.array_equal(resumed.state()[0], full.state()[0])


def test_mass_balance_and_retry_on_the_oracle_stepper():
    """Mass bookkeeping over real steps: the error |mass - inflow - initial| is what
    the reference's tl_find_grid_mass_error_elem2d reports for the same states."""
    case = small_delaunay_case(n=12, seed=5, nsteps=3)
    sim = SW2Simulation(case, model=OracleStepper(case))
    sim.start_mass_balance(1.0)
    m0 = sim.mass0
    inflow = 0.0
    for _ in range(3):
        sim.step()
        sol = sim.state()[0]
        inflow += sim.model.o.boundary_mass_flux(sol, 1.0, case.dt)
    mb = sim.mass_balance()
    assert mb["steps"] == 3 and mb["inflow"] == inflow
    assert mb["error"] == abs(sim.model.o.grid_mass(sim.state()[0]) - inflow - m0)


def test_failed_step_is_retried_with_a_quarter_dt():
    """dt = 150 s fails on the wet/dry case (in the reference too); advance() undoes
    it and covers the interval in four steps of 37.5 s, which converge and equal four
    plain 37.5 s steps from the same start."""
    import dataclasses
    from adh_kraken_b200.timeloop import DT_REDUCE_FACTOR
    case = small_delaunay_case(n=12, seed=5, nsteps=3, dt=150.0)
    sim = SW2Simulation(case, model=OracleStepper(case))
    st = sim.advance()
    assert st["success"] == 1 and st["dt_cuts"] == 1 and st["substeps"] == 4
    assert sim.t == case.t0 + case.dt and not sim.history[0]["success"]
    small = dataclasses.replace(case, dt=case.dt * DT_REDUCE_FACTOR)
    ref = SW2Simulation(small, model=OracleStepper(small))
    ref.run(4)
    assert np.array_equal(sim.state()[0], ref.state()[0])


def test_nan_state_fails_every_retry():
    """A NaN planted in the state (host side): every attempt fails, advance() gives up
    after its reductions and leaves the state and the clock at the step's start."""
    case = small_delaunay_case(n=12, seed=5, nsteps=3)
    sim = SW2Simulation(case, model=OracleStepper(case))
    sol = case.sol0.copy()
    sol[3 * 7] = np.nan
    sim.model.load_state(sol, sol, sol)
    st = sim.advance(max_cuts=2)
    assert st["success"] == 0 and st["dt_cuts"] == 3 and st["substeps"] == 0
    assert sim.t == case.t0
    assert np.isnan(sim.state()[0][3 * 7])


def test_per_step_json_log():
    import io
    import json
    case = small_delaunay_case(n=12, seed=5, nsteps=3)
    sim = SW2Simulation(case, model=OracleStepper(case))
    buf = io.StringIO()
    sim.set_log(buf)
    sim.start_mass_balance(1000.0)
    sim.run(3)
    lines = [json.loads(x) for x in buf.getvalue().splitlines()]
    assert len(lines) == 3
    assert [ln["newton_its"] for ln in lines] == [h["newton_its"] for h in sim.history]
    assert lines[-1]["t"] == sim.t and lines[0]["dt"] == case.dt and all(ln["success"] == 1 for ln in lines)
    assert [ln["mass"] for ln in lines] == [m for _, m, _ in sim.mass_log]


def test_resume_keeps_step_count_and_mass_balance(tmp_path):
    """The checkpoint carries the count of successful steps and the mass bookkeeping
    (initial mass, boundary inflow so far, the per-step log): a resumed run reports the
    same mass error as the uninterrupted one."""
    case = small_delaunay_case(n=12, seed=5, nsteps=4)
    full = SW2Simulation(case, model=OracleStepper(case))
    full.start_mass_balance(1000.0)
    full.run(4)
    first = SW2Simulation(case, model=OracleStepper(case))
    first.start_mass_balance(1000.0)
    first.run(2)
    ck = str(tmp_path / "ck.npz")
    first.checkpoint(ck)
    resumed = SW2Simulation(case, model=OracleStepper(case))
    resumed.restore(ck)
    assert resumed.nsteps_done == 2
    resumed.run(2)
    assert resumed.nsteps_done == full.nsteps_done == 4
    assert resumed.mass_balance() == full.mass_balance()
    assert resumed.mass_log == full.mass_log
