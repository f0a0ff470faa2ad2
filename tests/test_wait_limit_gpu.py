"""A bounded device wait that runs out ends in a status, not a hang or a fault.

The uneven-batch kernel solves each band of a multi-band pair on its own warp;
a band waits (bounded polling of a progress counter in global memory, no
asynchronous copies in flight) for the band above to publish its bottom row.
With the wait limit set to 0 polls (sigk_set_wait_limit), the first band-1
wait finds nothing published yet and gives up: the pair's result is NaN, the
launch's error word gets its timeout bit, and sigk_ragged_status returns
SIGK_ETIMEDOUT.  The kernel still returns, the context stays usable, and with
the default limit restored the same plan solves every pair again (bitwise the
results of a normal launch, which match the float64 oracle).

The reference has no waits; its failure convention is NaN -> inf in the
results (sigpde/torch/kernel.py:183, sigpde/cuda_pairwise_kernels.py:132).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _batch(oracle):
    # 48 pairs of 2 bands each (511 coarse cells at order 1 = 1022 refined rows, 16 rows a lane)
    rng = np.random.default_rng(11)
    xs = [oracle.brownian(1, 512, 4, int(rng.integers(1 << 30)))[0] for _ in range(48)]
    ys = [oracle.brownian(1, 300, 4, int(rng.integers(1 << 30)))[0] for _ in range(48)]
    X = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in xs]
    Y = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in ys]
    return X, Y


def test_band_wait_timeout_returns_status(oracle):
    from sigpde_b200 import _lib
    from sigpde_b200.torch.ragged import RaggedPairwise

    X, Y = _batch(oracle)
    orders = [1] * len(X)
    solver = RaggedPairwise([x.shape[0] for x in X], [y.shape[0] for y in Y], orders, 4, torch.float64, "cuda")
    assert int(solver.pair_bands.max()) >= 2
    solver.load(X, Y)
    normal = solver.solve().clone()
    solver.check()
    assert solver.error_flag() == 0
    want = np.array([oracle.pairwise(X[b].cpu().numpy()[None], Y[b].cpu().numpy()[None], 1)[0] for b in range(4)])
    got = normal[:4].cpu().numpy()
    assert float(np.max(np.abs(got - want) / np.abs(want))) <= 1e-9

    prev = _lib.set_wait_limit(0)
    try:
        out = solver.solve().clone()
        with pytest.raises(_lib.SigkError) as ei:
            solver.check()
        assert ei.value.status == _lib.SIGK_ETIMEDOUT
        assert solver.error_flag() & 2
    finally:
        _lib.set_wait_limit(prev)
    o = out.cpu().numpy()
    n = normal.cpu().numpy()
    bad = np.isnan(o)
    assert bad.any(), "every multi-band pair should have timed out at 0 polls"
    np.testing.assert_array_equal(o[~bad], n[~bad])

    # the context is usable and the default limit solves every pair again
    again = solver.solve().clone()
    solver.check()
    np.testing.assert_array_equal(again.cpu().numpy(), n)
    assert _lib.set_wait_limit(-1) == prev
