"""bench.py's multi-GPU arithmetic on CPU: two gloo ranks (replicas) report
the max of their timed milliseconds and the sum of their droplet-substeps,
and every rank takes the same collective steps."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t, n = bench.reduce_over_ranks(dist, 10.0 + rank, 1000 * (rank + 1), device="cpu")
    t2, n2 = bench.reduce_over_ranks(None, 10.0 + rank, 7)
    out.put((rank, t, n, t2, n2))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_reduction():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, n, t2, n2 in res:
        assert t == 11.0 and n == 3000  # max time, summed work
        assert t2 == 10.0 + rank and n2 == 7  # no group: unchanged
