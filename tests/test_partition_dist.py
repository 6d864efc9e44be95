"""The multi-rank plumbing of the linear algebra on CPU: node partition, split CSR,
halo plan, and the distributed matrix-vector and dot products over gloo ranks
(world size 2 and 3) against the single-process product."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from adh_kraken_b200.mesh import small_delaunay_case
from adh_kraken_b200.partition import matvec_local, node_ranges, split
from oracle.oracle import OracleModel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def system(seed=0):
    case = small_delaunay_case(n=12, seed=5, nsteps=1)
    o = OracleModel(case)
    rng = np.random.default_rng(seed)
    vals = rng.standard_normal(o.nnz)
    x = rng.standard_normal(o.ndof)
    return case, o, vals, x


def emulate(parts, x):
    """Every rank's product with its ghost values taken straight from x."""
    out = []
    for p in parts:
        x_ext = np.concatenate([x[p.row0:p.row0 + p.nrows], x[p.ghosts]])
        out.append(matvec_local(p, x_ext))
    return np.concatenate(out)


def test_node_ranges_follow_the_reference_split():
    assert node_ranges(10, 3).tolist() == [0, 3, 6, 10]      # nnodes / npes each, the rest on the last
    assert node_ranges(7, 1).tolist() == [0, 7]


@pytest.mark.parametrize("npes", [1, 2, 3])
def test_split_csr_and_halo_plan(npes):
    case, o, vals, x = system()
    parts = split(o.indptr, o.cols, vals, case.nnodes, npes)
    assert sum(p.nrows for p in parts) == o.ndof
    assert sum(p.cols_diag.size + p.cols_off.size for p in parts) == o.nnz
    for p in parts:
        own = (p.ghosts >= p.row0) & (p.ghosts < p.row0 + p.nrows)
        assert not own.any()
        for q, pos in p.recv.items():
            assert np.array_equal(parts[q].send[p.rank], p.ghosts[pos])
        assert sorted(np.concatenate(list(p.recv.values())).tolist() if p.recv else []) == list(range(p.ghosts.size))
    y = emulate(parts, x)
    ref = o.spmv(vals, x)
    assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()
    if npes == 1:
        assert np.array_equal(y, ref)      # one rank: the diagonal block is the whole row, same order


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from adh_kraken_b200.partition import dot, matvec, split as split_
    case, o, vals, x = system()
    p = split_(o.indptr, o.cols, vals, case.nnodes, world)[rank]
    own = x[p.row0:p.row0 + p.nrows]
    y = matvec(p, own, dist)
    d = dot(own, own, dist)
    out[rank] = (p.row0, y, d)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_distributed_matvec_and_dot_over_gloo(world):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    case, o, vals, x = system()
    parts = split(o.indptr, o.cols, vals, case.nnodes, world)
    y = np.concatenate([out[r][1] for r in range(world)])
    assert np.array_equal(y, emulate(parts, x))          # the exchanged ghosts are the owners' values
    assert all(abs(out[r][2] - float(np.dot(x, x))) <= 1e-12 * float(np.dot(x, x)) for r in range(world))


def _bicg_worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from fixtures import load
    from adh_kraken_b200.partition import bicgstab_bj, split as split_
    case, z = load("dump_wetdry_12.npz")
    o = OracleModel(case)
    p = split_(o.indptr, o.cols, z["ref_jac_vals_scaled"], case.nnodes, world)[rank]
    sl = slice(p.row0, p.row0 + p.nrows)
    x, it = bicgstab_bj(p, np.zeros(p.nrows), z["ref_residual_scaled"][sl].copy(), z["ref_scale_vect"][sl], dist,
                        max_it=20000, tol=1e-13)
    out[rank] = (x, it)
    dist.barrier()
    dist.destroy_process_group()


def test_distributed_block_jacobi_bicgstab_matches_the_single_process_solve():
    """The reference's BiCGStab recurrence on two ranks (halo exchange per product,
    all-reduce per dot and max-norm) against the oracle's single-process solve of the
    same scaled system from the reference's dump."""
    from fixtures import load
    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_bicg_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    assert all(p.exitcode == 0 for p in procs)
    case, z = load("dump_wetdry_12.npz")
    o = OracleModel(case)
    v = z["ref_jac_vals_scaled"].copy(); b = z["ref_residual_scaled"].copy(); x1 = np.zeros(o.ndof)
    it1 = o.bicgstab(v, x1, b, z["ref_scale_vect"], max_it=20000, tol=1e-13)
    xd = np.concatenate([out[r][0] for r in range(world)])
    its = {out[r][1] for r in range(world)}
    assert len(its) == 1 and it1 > 0 and abs(its.pop() - it1) <= 2
    assert np.abs(xd - x1).max() <= 1e-9 * np.abs(x1).max()
    assert np.abs(xd - z["ref_dsol"]).max() <= 1e-6 * np.abs(z["ref_dsol"]).max()


@pytest.mark.parametrize("npes", [2, 3, 4])
def test_per_rank_assembly_is_bit_exact(npes):
    """Each rank assembles its own residual rows and Jacobian rows from the elements
    within two rings of its nodes, in global element order: identical to the
    single-process assembly, with no element contributions exchanged."""
    from fixtures import load
    from adh_kraken_b200.partition import assembly_parts, part_case
    case, z = load("dump_wetdry_12.npz")
    sol, old, older = z["sol"], z["sol_old"], z["sol_older"]
    o = OracleModel(case)
    o.wd_flags(sol, old)
    R, J = o.residual(sol, old, older), o.jacobian(sol, old, older)
    assert np.array_equal(R, z["ref_residual"]) and np.array_equal(J, z["ref_jac_vals"])
    for p in assembly_parts(case.tri, case.seg, case.nnodes, npes):
        sc, dofs = part_case(case, p)
        so = OracleModel(sc)
        so.wd_flags(sol[dofs], old[dofs])
        r = so.residual(sol[dofs], old[dofs], older[dofs])
        v = so.jacobian(sol[dofs], old[dofs], older[dofs])
        own = (3 * p.owned_local[:, None] + np.arange(3)).ravel()
        assert np.array_equal(r[own], R[3 * p.lo:3 * p.hi])
        for rl, rg in zip(own, range(3 * p.lo, 3 * p.hi)):
            cl = so.cols[so.indptr[rl]:so.indptr[rl + 1]]
            assert np.array_equal(3 * p.nodes[cl // 3] + cl % 3, o.cols[o.indptr[rg]:o.indptr[rg + 1]])
            assert np.array_equal(v[so.indptr[rl]:so.indptr[rl + 1]], J[o.indptr[rg]:o.indptr[rg + 1]])


def _assembly_worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from fixtures import load
    from adh_kraken_b200.partition import assembly_parts, exchange_state, part_case, state_halo
    case, z = load("dump_wetdry_12.npz")
    parts = assembly_parts(case.tri, case.seg, case.nnodes, world)
    send, recv = state_halo(parts, case.nnodes)
    p = parts[rank]
    loc = [exchange_state(p, send[rank], recv[rank], z[k][3 * p.lo:3 * p.hi], dist)
           for k in ("sol", "sol_old", "sol_older")]
    sc, _ = part_case(case, p)
    so = OracleModel(sc)
    so.wd_flags(loc[0], loc[1])
    r = so.residual(*loc)
    own = (3 * p.owned_local[:, None] + np.arange(3)).ravel()
    out[rank] = r[own]
    dist.barrier()
    dist.destroy_process_group()


def test_distributed_residual_over_gloo():
    """Owned states plus a two-ring state halo exchanged between gloo ranks give every
    rank its rows of the reference's assembled residual, bit for bit."""
    from fixtures import load
    world = 3
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_assembly_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    assert all(p.exitcode == 0 for p in procs)
    case, z = load("dump_wetdry_12.npz")
    assert np.array_equal(np.concatenate([out[r] for r in range(world)]), z["ref_residual"])


def _newton_worker(rank, world, port, nsteps, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    from adh_kraken_b200.partition import RankNewton
    case = small_delaunay_case(n=12, seed=5, nsteps=nsteps)
    o = OracleModel(case)
    rn = RankNewton(case, o.indptr, o.cols, world, rank, OracleModel)
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
    out[rank] = (sol, hist)
    dist.barrier()
    dist.destroy_process_group()


def test_distributed_newton_steps_follow_the_single_process_run():
    """Two ranks run the reference's Newton loop on their halo sub-meshes (norms, dots
    and ghost columns through gloo): the same Newton iterations and line-search cuts as
    the single-process oracle, the same states to 1e-10, and the reference's run to 1e-8."""
    from fixtures import load
    world, nsteps = 2, 4
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_newton_worker, args=(r, world, port, nsteps, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs)
    case = small_delaunay_case(n=12, seed=5, nsteps=nsteps)
    sol1, hist1 = OracleModel(case).run(nsteps, krylov_max_it=20000)
    sold = np.concatenate([out[r][0] for r in range(world)])
    assert out[0][1] == out[1][1]
    assert [h[:2] for h in out[0][1]] == [(h["newton_its"], h["linesearch_cuts"]) for h in hist1]
    assert all(h[2] for h in out[0][1])
    for k in range(3):
        a, b = sold[k::3], sol1[k::3]
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(b).max(), 1e-300), k
    _, z = load("run_wetdry_12_4steps.npz")
    ref = z["ref_sol_kept"].reshape(-1, 3 * case.nnodes)[-1]
    for k in range(3):
        assert np.abs(sold[k::3] - ref[k::3]).max() <= 1e-8 * np.abs(ref[k::3]).max(), k
