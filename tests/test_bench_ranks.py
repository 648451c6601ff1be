"""bench.py's N > 1 plumbing on CPU: two gloo ranks (127.0.0.1) reduce their
times to the slowest rank's, and the whole-job throughput counts every
replica's cells over that time."""
import datetime
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank 1 is the slow one for the first quantity, rank 0 for the second
        a = bench.max_over_ranks(10.0 + 5.0 * rank, 2, device="cpu")
        b = bench.max_over_ranks(7.0 - 3.0 * rank, 2, device="cpu")
        q.put((rank, a, b, bench.job_mlups(2, 1000, 10, a)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get() for _ in range(2))
    for rank, a, b, v in got:
        assert a == 15.0 and b == 7.0
        assert abs(v - 2 * 1000 * 10 / 15e-3 / 1e6) < 1e-12


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_mlups(1, 16777216, 200, 142.2) == 16777216 * 200 / 0.1422 / 1e6
