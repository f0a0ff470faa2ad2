"""The uneven-batch autotuner (sigpde_b200.torch.autotune).

CPU: bucket keys, candidate sets and the JSON round trip.  GPU: tuning picks a
valid rows-per-lane for every bucket a batch uses, and the tuned plan gives
bitwise the same results as the default plan (rows per lane only change which
lane computes a cell, not its arithmetic)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_buckets_and_candidates():
    from sigpde_b200.torch import autotune as at
    assert at.bucket_of(508, 2) == (9, 2)
    assert at.bucket_of(4088, 3) == (12, 3)
    assert at.bucket_of(15, 7) == (4, 4)
    assert at.candidates(40) == [2]              # one band of 64 rows already
    assert at.candidates(200) == [2, 4, 8]       # 8 covers 200 in one band; 16 adds nothing
    assert at.candidates(4088) == [2, 4, 8, 16]  # 64, 32, 16, 8 bands
    assert at.candidates(5000) == [4, 8, 16]     # 2 rows a lane would need 79 bands
    for n in (2, 17, 63, 64, 65, 511, 512, 513, 2047, 9000):
        for R in at.candidates(n):
            assert R in at.ROWS and -(-n // (32 * R)) <= at.MAX_BANDS


def test_table_round_trip(tmp_path):
    from sigpde_b200.torch import autotune as at
    t = at.RaggedTuner.__new__(at.RaggedTuner)
    t.dim, t.precision, t.table, t.timings = 32, "tc64", {(9, 2): 8, (12, 3): 16}, {(9, 2): {8: 1.0, 16: 2.0}}
    t.device = torch.device("cpu")
    import unittest.mock as um
    with um.patch("torch.cuda.get_device_name", return_value="test"):
        t.save(tmp_path / "t.json")
    u = at.RaggedTuner.__new__(at.RaggedTuner)
    u.dim, u.precision, u.table = 32, "tc64", {}
    u.load(tmp_path / "t.json")
    assert u.table == t.table
    assert u.rows_for(400, 2) == 8 and u.rows_for(4000, 3) == 16
    v = at.RaggedTuner.__new__(at.RaggedTuner)
    v.dim, v.precision, v.table = 16, "tc64", {}
    v.load(tmp_path / "t.json")  # another dim: not applied
    assert v.table == {}


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "tc64"])
def test_tuned_plan_gives_identical_results(oracle, prec):
    import sigpde_b200.torch as sig
    rng = np.random.default_rng(9)
    n = 96
    lx = rng.integers(16, 300, n)
    ly = rng.integers(16, 300, n)
    orders = rng.integers(0, 4, n)
    X = [torch.tensor(oracle.brownian(1, int(a), 8, int(s))[0], dtype=torch.float32, device="cuda")
         for a, s in zip(lx, rng.integers(1 << 30, size=n))]
    Y = [torch.tensor(oracle.brownian(1, int(a), 8, int(s))[0], dtype=torch.float32, device="cuda")
         for a, s in zip(ly, rng.integers(1 << 30, size=n))]
    base = sig.ragged.RaggedPairwise(lx, ly, orders, 8, precision=prec)
    base.load(X, Y)
    want = base.solve().clone()
    tuner = sig.autotune.RaggedTuner(8, precision=prec, pairs_per_bucket=64)
    tuned = sig.ragged.RaggedPairwise(lx, ly, orders, 8, precision=prec, tuner=tuner)
    assert tuner.table, "every bucket of the batch is tuned"
    for (lg, o), R in tuner.table.items():
        assert R in sig.autotune.ROWS
    tuned.load(X, Y)
    got = tuned.solve()
    assert torch.equal(got, want)
