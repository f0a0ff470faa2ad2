"""Gram sharding across ranks (sigpde_b200.distributed) on CPU: gloo ranks on
127.0.0.1, with the float64 oracle standing in for each rank's GPU solve.

What is checked is the host logic: the row partition (equal blocks for a
Gram, lower-triangle-area blocks for a symmetric Gram), the diagonal block
solved as a symmetric Gram, the all-gather of row blocks of unequal heights,
the mirror of the lower triangle, and the robust lambdas computed in shards
and all-gathered.  Each entry of the oracle depends only on its own pair, so
the assembled matrices equal the oracle's single-process results exactly, on
every rank.  The reference's tile loop being distributed is
sigpde/torch/kernel.py:100-122 (and :143-169 for the symmetric Gram).
"""
import os
import socket
import sys

import numpy as np
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


def _oracle_hooks(order):
    from oracle import oracle

    def solve(xr, yc, sx, sy):
        xs = None if sx is None else sx.double().numpy()
        if yc is None:
            return torch.from_numpy(oracle.gram(xr.double().numpy(), None, order, xs))
        ys = None if sy is None else sy.double().numpy()
        scaled = xs is not None or ys is not None
        return torch.from_numpy(oracle.gram(xr.double().numpy(), yc.double().numpy(), order,
                                            xs if scaled else None, ys if scaled else None))

    def lam(x):
        return torch.from_numpy(oracle.normalization(x.double().numpy(), order))

    return solve, lam


def _inputs():
    from oracle import oracle
    x = torch.from_numpy(oracle.brownian(11, 12, 3, 71))
    y = torch.from_numpy(oracle.brownian(7, 10, 3, 72))
    rng = np.random.default_rng(5)
    sx = torch.from_numpy(np.exp(rng.uniform(-0.3, 0.3, 11)))
    sy = torch.from_numpy(np.exp(rng.uniform(-0.3, 0.3, 7)))
    xr = torch.from_numpy(oracle.brownian(9, 12, 3, 73, scale=np.exp(rng.uniform(np.log(0.5), np.log(4.0), 9))))
    return x, y, sx, sy, xr


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from sigpde_b200 import distributed as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        solve, lam = _oracle_hooks(1)
        x, y, sx, sy, xr = _inputs()
        res = {
            "gram": D.sharded_gram(x, y, solve=solve).numpy(),
            "gram_scaled": D.sharded_gram(x, y, sx, sy, solve=solve).numpy(),
            "sym": D.sharded_gram(x, solve=solve).numpy(),
            "sym_scaled": D.sharded_gram(x, None, sx, solve=solve).numpy(),
            "robust_sym": D.sharded_robust_gram(xr, dyadic_order=1, solve=solve, lam=lam).numpy(),
            "robust": D.sharded_robust_gram(xr, x, dyadic_order=1, solve=solve, lam=lam).numpy(),
        }
        dist.barrier()
        out[rank] = res
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_gram_with_gloo_ranks(world, oracle):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
            assert p.exitcode == 0
        got = dict(out)
    x, y, sx, sy, xr = (t.numpy() for t in _inputs())
    lx = oracle.normalization(xr, 1)
    ly = oracle.normalization(x, 1)
    want = {
        "gram": oracle.gram(x, y, 1),
        "gram_scaled": oracle.gram(x, y, 1, sx, sy),
        "sym": oracle.gram(x, None, 1),
        "sym_scaled": oracle.gram(x, None, 1, sx),
        "robust_sym": oracle.gram(xr, None, 1, lx),
        "robust": oracle.gram(xr, x, 1, lx, ly),
    }
    for rank in range(world):
        for k, w in want.items():
            np.testing.assert_array_equal(got[rank][k], w, err_msg=f"rank {rank}: {k}")


def test_partitions():
    sys.path.insert(0, ROOT)
    from sigpde_b200.distributed import row_blocks, triangle_blocks
    for n in (1, 2, 7, 100, 512, 1000):
        for w in (1, 2, 3, 4, 8):
            for blocks in (row_blocks(n, w), triangle_blocks(n, w)):
                assert len(blocks) == w and blocks[0][0] == 0 and blocks[-1][1] == n
                assert all(blocks[i][1] == blocks[i + 1][0] for i in range(w - 1))
                assert all(e >= s for s, e in blocks)
    areas = [(e * (e + 1) - s * (s + 1)) // 2 for s, e in triangle_blocks(512, 4)]
    assert max(areas) - min(areas) <= 512  # within one row of equal
    assert [e - s for s, e in row_blocks(10, 4)] == [3, 3, 2, 2]
