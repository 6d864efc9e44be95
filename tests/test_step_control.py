"""Host logic of the time loop's step control (SW2Simulation.advance) and mass
bookkeeping, on a stand-in for the device model: no GPU needed."""
import numpy as np
import pytest

from adh_kraken_b200.mesh import flume_case
from adh_kraken_b200.timeloop import DT_REDUCE_FACTOR, SW2Simulation


class FakeModel:
    """Succeeds on steps no longer than `dt_ok`; a failed step leaves the state, and
    undo_step must follow it before the next step."""

    def __init__(self, dt_ok, fail_nonfinite=False):
        self.dt_ok, self.fail_nonfinite = dt_ok, fail_nonfinite
        self.calls, self.undos, self.dt = [], 0, None
        self.pending_undo = False
        self.mass = 100.0

    def load_state(self, *a, **k):
        pass

    def set_step(self, dt, d, vx, vy, tau_temporal=0.0):
        self.dt = dt

    def step(self, opts=None):
        from adh_kraken_b200.capi import ERR_NONFINITE, SW2Error
        assert not self.pending_undo, "a failed step was not undone"
        self.calls.append(self.dt)
        if self.dt > self.dt_ok * (1 + 1e-12):
            self.pending_undo = True
            if self.fail_nonfinite:
                raise SW2Error("non-finite residual norm during Newton", ERR_NONFINITE)
            return {"success": 0, "newton_its": 10, "krylov_its": 5}
        self.mass += 2.0 * self.dt
        return {"success": 1, "newton_its": 2, "krylov_its": 7}

    def undo_step(self):
        assert self.pending_undo
        self.pending_undo = False
        self.undos += 1

    def grid_mass(self, sol=None, density=1.0, dt=None):
        return density * self.mass, density * 2.0 * dt


@pytest.mark.parametrize("nonfinite", [False, True])
def test_advance_reduces_dt_and_covers_the_interval(nonfinite):
    case = flume_case(nsteps=4, npx=5, npy=3)
    fake = FakeModel(dt_ok=case.dt * DT_REDUCE_FACTOR, fail_nonfinite=nonfinite)
    sim = SW2Simulation(case, model=fake)
    st = sim.advance()
    assert st["success"] == 1 and st["dt_cuts"] == 1 and st["substeps"] == 4
    assert fake.calls == [case.dt] + [case.dt * DT_REDUCE_FACTOR] * 4
    assert fake.undos == 1
    assert sim.t == pytest.approx(case.t0 + case.dt, abs=0)


def test_advance_two_reductions_and_giving_up():
    case = flume_case(nsteps=4, npx=5, npy=3)
    fake = FakeModel(dt_ok=case.dt / 16)
    sim = SW2Simulation(case, model=fake)
    st = sim.advance()
    assert st["success"] == 1 and st["dt_cuts"] == 2 and st["substeps"] == 16
    assert sim.t == case.t0 + case.dt
    fake2 = FakeModel(dt_ok=case.dt / 1000)
    sim2 = SW2Simulation(case, model=fake2)
    st2 = sim2.advance(max_cuts=2)
    assert st2["success"] == 0 and st2["substeps"] == 0 and sim2.t == case.t0
    assert fake2.calls == [case.dt, case.dt / 4, case.dt / 16]


def test_mass_bookkeeping_counts_successful_steps_only():
    case = flume_case(nsteps=4, npx=5, npy=3)
    fake = FakeModel(dt_ok=case.dt * DT_REDUCE_FACTOR)
    sim = SW2Simulation(case, model=fake)
    sim.start_mass_balance(density=2.0)
    sim.advance()
    mb = sim.mass_balance()
    assert mb["steps"] == 4
    assert mb["inflow"] == pytest.approx(2.0 * 2.0 * case.dt)
    assert mb["error"] == pytest.approx(0.0, abs=1e-9)


def test_advance_keeps_a_reduced_dt_then_grows_it_back():
    """After a cut, the next keep_reduced_dt intervals start at the reduced step (no
    failed full-dt attempt), then the full dt is tried again; keep_reduced_dt = 0 tries
    it every interval."""
    case = flume_case(nsteps=8, npx=5, npy=3)
    q = case.dt * DT_REDUCE_FACTOR
    fake = FakeModel(dt_ok=q)
    sim = SW2Simulation(case, model=fake)
    cuts = [sim.advance()["dt_cuts"] for _ in range(7)]
    assert cuts == [1, 0, 0, 0, 0, 1, 0]
    assert fake.calls == ([case.dt] + [q] * 4) + [q] * 16 + ([case.dt] + [q] * 4) + [q] * 4
    assert sim.t == pytest.approx(case.t0 + 7 * case.dt)
    fake0 = FakeModel(dt_ok=q)
    sim0 = SW2Simulation(case, model=fake0)
    sim0.keep_reduced_dt = 0
    assert [sim0.advance()["dt_cuts"] for _ in range(3)] == [1, 1, 1]


def test_held_step_keeps_the_interval_tolerance():
    """A held step h starts with tol_nonlin_rel x dt / h (R(sol_old) scales with the step's
    length), and its later substeps keep the first one's tolerance as the floor."""
    from adh_kraken_b200.capi import default_opts
    case = flume_case(nsteps=4, npx=5, npy=3)
    seen = []

    class Recording(FakeModel):
        def step(self, opts=None):
            seen.append((self.dt, opts.tol_nonlin_rel, opts.tol_nonlin_min))
            st = super().step(opts)
            st["tol_used"] = 1e-8 * (self.dt / case.dt) * opts.tol_nonlin_rel / 1e-8 * 3.0
            return st

    fake = Recording(dt_ok=case.dt * DT_REDUCE_FACTOR)
    sim = SW2Simulation(case, model=fake, opts=default_opts(tol_nonlin_rel=1e-8))
    sim.advance()
    seen.clear()
    sim.advance()
    q = case.dt * DT_REDUCE_FACTOR
    assert seen[0] == (q, pytest.approx(1e-8 / DT_REDUCE_FACTOR), 0.0)
    first_tol = 1e-8 * DT_REDUCE_FACTOR * (1e-8 / DT_REDUCE_FACTOR) / 1e-8 * 3.0
    assert all(s[1] == pytest.approx(1e-8) and s[2] == pytest.approx(first_tol) for s in seen[1:])


def test_advance_reports_the_step_it_started_with():
    case = flume_case(nsteps=8, npx=5, npy=3)
    q = case.dt * DT_REDUCE_FACTOR
    sim = SW2Simulation(case, model=FakeModel(dt_ok=q))
    starts = [sim.advance()["step_start"] for _ in range(3)]
    assert starts == [case.dt, q, q]
    sim2 = SW2Simulation(case, model=FakeModel(dt_ok=q * DT_REDUCE_FACTOR))
    sim2.advance()                       # two cuts: holds q / 4
    sim2.model.dt_ok = q * DT_REDUCE_FACTOR ** 3
    st = sim2.advance()                  # starts at q / 4, cuts twice more
    assert st["step_start"] == q * DT_REDUCE_FACTOR and st["dt_cuts"] == 2


def test_discharge_segments_without_roughness_are_refused():
    """The discharge law divides by the boundary strings' drag: a case with discharge
    segments and no roughness height is refused before any step."""
    import dataclasses
    from adh_kraken_b200.mesh import flume_structures_case
    case = dataclasses.replace(flume_structures_case(nsteps=2), bc_rough_height=0.0)
    sim = SW2Simulation(case, model=FakeModel(dt_ok=case.dt))
    with pytest.raises(ValueError):
        sim.step()
