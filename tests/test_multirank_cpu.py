"""The multi-GPU bench path on CPU: two gloo ranks (replicas, weak scaling).

bench.py times each rank's replica, takes the maximum over ranks of the
timed milliseconds and reports every rank's units over that time.  The same
helpers run here with the gloo backend on 127.0.0.1."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        slowest = bench.max_over_ranks(torch, dist, world, values[rank])
        dist.barrier()
        out[rank] = slowest
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    world = 2
    values = [12.5, 17.25]
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, values, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        got = dict(out)
    assert got == {0: 17.25, 1: 17.25}
    sys.path.insert(0, ROOT)
    import bench
    # 65,536 entries per rank per step, 10 steps, slowest rank 17.25 ms in total
    assert bench.job_rate(world, 65536, 10, 17.25) == pytest.approx(2 * 65536 * 10 / 0.01725)
    assert bench.max_over_ranks(torch, None, 1, 3.0) == 3.0
