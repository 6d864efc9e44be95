"""The partitioned Newton loop with the device model as each rank's element
evaluator: two gloo ranks (two processes on the one GPU, exchanging only through the
host) assemble their rows with the CUDA kernels on their halo sub-meshes and run the
reference's Newton loop over the split CSR.  They must take the same Newton iterations
and line-search cuts as the single-process oracle and as the same ranks with the oracle
as evaluator, and end at the same state."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from adh_kraken_b200.mesh import small_delaunay_case
from oracle.oracle import OracleModel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nsteps, evaluator, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    from adh_kraken_b200.partition import DeviceRankModel, RankNewton
    case = small_delaunay_case(n=12, seed=5, nsteps=nsteps)
    o = OracleModel(case)
    make = DeviceRankModel if evaluator == "device" else OracleModel
    rn = RankNewton(case, o.indptr, o.cols, world, rank, make)
    r0, r1 = rn.r0, rn.r1
    sol = case.sol0[r0:r1].copy(); old = sol.copy()
    mask = np.zeros(r1 - r0, np.int32); dirichlet = np.zeros(r1 - r0)
    hist, t = [], case.t0
    for _ in range(nsteps):
        t += case.dt
        older, old = old, sol
        rn.model.set_bc_window(t - case.dt, t)
        sol, st = rn.solve(old, older, mask, dirichlet, dist, krylov_max_it=20000)
        hist.append((st["newton_its"], st["linesearch_cuts"], st["ok"]))
    if evaluator == "device":
        rn.model.close()
    out[(evaluator, rank)] = (sol, hist)
    dist.barrier()
    dist.destroy_process_group()


def _run(evaluator, world, nsteps, out):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, nsteps, evaluator, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]


def test_partitioned_newton_with_device_assembly_matches_oracle_ranks():
    world, nsteps = 2, 4
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    _run("oracle", world, nsteps, out)
    _run("device", world, nsteps, out)
    case = small_delaunay_case(n=12, seed=5, nsteps=nsteps)
    sol1, hist1 = OracleModel(case).run(nsteps, krylov_max_it=20000)
    for ev in ("oracle", "device"):
        assert out[(ev, 0)][1] == out[(ev, 1)][1]
        assert [h[:2] for h in out[(ev, 0)][1]] == [(h["newton_its"], h["linesearch_cuts"]) for h in hist1]
        assert all(h[2] for h in out[(ev, 0)][1])
    s_or = np.concatenate([out[("oracle", r)][0] for r in range(world)])
    s_dev = np.concatenate([out[("device", r)][0] for r in range(world)])
    # the device rows equal the oracle's bit for bit, so the two runs are expected to agree exactly
    print("device ranks equal oracle ranks bit for bit:", np.array_equal(s_dev, s_or))
    for k in range(3):
        assert np.abs(s_dev[k::3] - s_or[k::3]).max() <= 1e-12 * max(np.abs(s_or[k::3]).max(), 1e-300), k
    for k in range(3):
        assert np.abs(s_dev[k::3] - sol1[k::3]).max() <= 1e-10 * max(np.abs(sol1[k::3]).max(), 1e-300), k
