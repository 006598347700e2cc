"""The multi-rank logic of bench.py on CPU (gloo, world size 2): the max over
ranks of the per-rank times, the barrier, per-rank seeds (replicas), and the
reference arm running on rank 0 only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    r, w, lr = bench.dist_env()
    m = bench.max_over_ranks(torch, 1.5 + rank, None)
    bench.barrier(torch)
    f = bench.make_initial_fields(64, bench.CFG["field_seed"] + rank)
    buf = io.StringIO()

    class A:
        steps, warmup = 1, 0
    with redirect_stdout(buf):
        rc = bench.reference_arm(A(), rank, world) if rank == 1 else 0
    dist.destroy_process_group()
    out.put((rank, r, w, lr, m, float(np.sum(f)), rc, buf.getvalue()))


@pytest.mark.timeout(300)
def test_two_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, r, w, lr, m, fsum, rc, printed in res:
        assert (r, w, lr) == (rank, world, rank)
        assert m == 2.5  # max over ranks
        assert rc == 0
        assert printed == ""  # the reference arm prints on rank 0 only
    assert res[0][5] != res[1][5]  # replicas draw different initial fields

