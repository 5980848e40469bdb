"""The N>1 path of bench.py on CPU: two gloo ranks (no GPU).

Each rank solves its own realisations (replicas, no data-path collective);
the only collectives are the whole-job aggregation: total converged pairs
over the slowest rank's time.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r converged 100*(r+1) pairs in (1 + r) seconds
        value, total, smax = bench.aggregate(100.0 * (rank + 1), 1.0 + rank, world, device="cpu")
        q.put((rank, value, total, smax, bench.rank_seed0(rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, value, total, smax, seed in res:
        assert total == 300.0 and smax == 2.0
        assert value == pytest.approx(150.0)
    assert res[0][4] != res[1][4]   # disjoint realisations per rank


def test_single_rank_aggregation():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate(200.0, 0.5, 1) == (400.0, 200.0, 0.5)
