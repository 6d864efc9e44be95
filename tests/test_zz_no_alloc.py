"""sw2g_assemble_residual_noalloc: the residual assembly for callers that cannot
allocate device memory when they call in (an application that gave all free
device memory to its own pool at start-up, or a time loop that must not allocate
inside its steps).  Its work arrays are fixed-size device arrays inside the
library, so it serves meshes of at most 131072 elements and nodes.  This file is
collected last so that a run stopping at the first failure has run every other
test before it."""
import ctypes as C

import numpy as np
import pytest

from fixtures import load

pytestmark = pytest.mark.gpu


def _model(case):
    from adh_kraken_b200.capi import SW2Model
    from oracle.oracle import OracleModel
    o = OracleModel(case)
    g = SW2Model(case)
    d, vx, vy = o.bc_values(case.t0, case.t0 + case.dt)
    g.set_step(case.dt, d, vx, vy)
    return g


def _noalloc(g, sol, old, older):
    import torch
    from adh_kraken_b200.capi import lib
    dev = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in (sol, old, older)]
    out = torch.full((g.ndofs,), float("nan"), dtype=torch.float64, device="cuda")
    rc = lib().sw2g_assemble_residual_noalloc(g.h, *(C.c_void_p(t.data_ptr()) for t in dev), C.c_void_p(out.data_ptr()))
    return rc, out.cpu().numpy()


@pytest.mark.parametrize("name", ["dump_flume_21x6.npz", "dump_wetdry_12.npz"])
def test_noalloc_residual_matches_assemble_residual_twice(name):
    case, z = load(name)
    g = _model(case)
    states = [(z["sol"], z["sol_old"], z["sol_older"]),
              (z["sol_old"], z["sol_old"], z["sol_older"])]   # a second, different call reuses the arrays
    for sol, old, older in states:
        ref = g.residual(sol, old, older)                      # the existing entry point (host buffers)
        rc, got = _noalloc(g, sol, old, older)
        assert rc == 0
        assert np.array_equal(got, ref), np.abs(got - ref).max()   # bit-exact, as the other residual tests


def test_noalloc_rejects_meshes_above_its_limit():
    from adh_kraken_b200.capi import lib
    from adh_kraken_b200.mesh import beach_case
    case = beach_case(nx=300, ny=300, nsteps=1)                # 178 802 triangles > 131072
    g = _model(case)
    rc, _ = _noalloc(g, case.sol0, case.sol0, case.sol0)
    assert rc != 0
    assert b"131072" in lib().sw2g_last_error()
