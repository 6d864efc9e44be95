"""Checkpoint / resume of the time loop on the device model: the three resident
levels, the permanent Dirichlet marks, the clock, the step count and the mass
bookkeeping go through a checkpoint file, and the resumed run takes the same steps
as the uninterrupted one, bit for bit."""
import numpy as np
import pytest

from fixtures import load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["run_wetdry_12_4steps.npz", "run_flume_21x6_8steps.npz"])
def test_resume_on_the_device_model_is_bit_exact(tmp_path, name):
    from adh_kraken_b200.timeloop import SW2Simulation
    case, _ = load(name)
    full = SW2Simulation(case)
    full.start_mass_balance(1000.0)
    for _ in range(4):
        assert full.step()["success"]
    first = SW2Simulation(case)
    first.start_mass_balance(1000.0)
    for _ in range(2):
        assert first.step()["success"]
    ck = str(tmp_path / "ck.npz")
    first.checkpoint(ck)
    first.model.close()
    resumed = SW2Simulation(case)
    resumed.restore(ck)
    for _ in range(2):
        assert resumed.step()["success"]
    assert resumed.t == full.t and resumed.nsteps_done == full.nsteps_done == 4
    for a, b in zip(resumed.state(), full.state()):
        assert np.array_equal(a, b)
    assert resumed.mass_balance() == full.mass_balance()
