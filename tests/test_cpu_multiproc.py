"""The multi-GPU host logic of bench.py on CPU: two gloo ranks (127.0.0.1).

bench.py runs independent replicas (no data-path collective); the only
cross-rank steps are the barrier and the max-over-ranks of each timed region.
Here rank r reports a time of (r + 1) seconds: both ranks must see the maximum,
and the whole-job rate must be (world * units) / slowest time.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        m = bench.max_over_ranks(rank + 1.0)
        dist.barrier()
        q.put((rank, m, bench.rate(12, world, m)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rate_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, r in res:
        assert m == 2.0
        assert r == pytest.approx(2 * 12 / 2.0)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.rate(12, 1, 2.0) == 6.0
