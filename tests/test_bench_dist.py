"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): the timing is
the maximum over ranks, and the reference arm runs on rank 0 only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    v = bench.max_over_ranks(1.5 + rank, dist, device="cpu")
    args = type("A", (), {"warmup": 0, "steps": 1, "gpus": world})()
    buf = io.StringIO()
    if rank != 0:
        with redirect_stdout(buf):
            bench.run_reference(args, world, rank, dist)     # non-zero ranks return at once, printing nothing
    dist.barrier()
    out[rank] = (v, buf.getvalue())
    dist.destroy_process_group()


def test_max_over_ranks_and_rank0_only_reference():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    assert out[0][0] == 2.5 and out[1][0] == 2.5
    assert out[1][1] == ""
