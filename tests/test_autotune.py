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
    assert at.bucket_of(508, 2, 8) == (9, 3, 2)
    assert at.bucket_of(4088, 3, 32) == (12, 5, 3)
    assert at.bucket_of(15, 7, 16) == (4, 4, 4)
    assert at.dim_bucket(1) == 1 and at.dim_bucket(5) == 3 and at.dim_bucket(32) == 5 and at.dim_bucket(33) == 6
    assert at.candidates(40) == [2]              # one band of 64 rows already
    assert at.candidates(200) == [2, 4, 8]       # 8 covers 200 in one band; 16 adds nothing
    assert at.candidates(4088) == [2, 4, 8, 16]  # 64, 32, 16, 8 bands
    assert at.candidates(5000) == [4, 8, 16]     # 2 rows a lane would need 79 bands
    for n in (2, 17, 63, 64, 65, 511, 512, 513, 2047, 9000):
        for R in at.candidates(n):
            assert R in at.ROWS and -(-n // (32 * R)) <= at.MAX_BANDS
    assert at.source_candidates("tc64", 32) == [("matrix", 256), ("matrix", 128), ("fused", 256)]
    assert at.source_candidates("tc32", 40) == [("fused", 256)]
    assert at.source_candidates("fp64", 8) == [("matrix", 256), ("fused", 256)]
    assert at.source_candidates("fp32", 8) == [("fused", 256)]


def test_table_round_trip(tmp_path):
    from sigpde_b200.torch import autotune as at
    t = at.RaggedTuner.__new__(at.RaggedTuner)
    t.dim, t.precision = 32, "tc64"
    t.table, t.timings = {(9, 5, 2): 8, (12, 5, 3): 16}, {(9, 5, 2): {8: 1.0, 16: 2.0}}
    t.batch, t.batch_timings = {5: {"source": "matrix", "tile_n": 128}}, {5: {"matrix/128": 1.0}}
    t.device = torch.device("cpu")
    import unittest.mock as um
    with um.patch("torch.cuda.get_device_name", return_value="test"):
        t.save(tmp_path / "t.json")
    u = at.RaggedTuner.__new__(at.RaggedTuner)
    u.dim, u.precision, u.table, u.batch = 32, "tc64", {}, {}
    u.load(tmp_path / "t.json")
    assert u.table == t.table and u.batch == t.batch
    assert u.rows_for(400, 2) == 8 and u.rows_for(4000, 3) == 16
    assert u.choice() == {"source": "matrix", "tile_n": 128}
    rep = u.report()
    assert rep["rows_per_lane"]["n<=2^9,d<=2^5,order=2"] == 8 and rep["tile_n"] == 128
    v = at.RaggedTuner.__new__(at.RaggedTuner)
    v.dim, v.precision, v.table, v.batch = 16, "tc64", {}, {}
    v.load(tmp_path / "t.json")  # another dim: not applied
    assert v.table == {} and v.batch == {}


def _batch(oracle, n, d, seed):
    rng = np.random.default_rng(seed)
    lx = rng.integers(16, 300, n)
    ly = rng.integers(16, 300, n)
    orders = rng.integers(0, 4, n)
    X = [torch.tensor(oracle.brownian(1, int(a), d, int(s))[0], dtype=torch.float32, device="cuda")
         for a, s in zip(lx, rng.integers(1 << 30, size=n))]
    Y = [torch.tensor(oracle.brownian(1, int(a), d, int(s))[0], dtype=torch.float32, device="cuda")
         for a, s in zip(ly, rng.integers(1 << 30, size=n))]
    return lx, ly, orders, X, Y


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "tc64"])
def test_tuned_plan_matches_the_default_plan(oracle, prec):
    """Every knob is tuned; the tuned plan equals the default bitwise when it keeps
    the default increment source, and within the precision's tolerance when it
    switches source (float64 cells: 1e-12 relative between sources)."""
    import sigpde_b200.torch as sig
    lx, ly, orders, X, Y = _batch(oracle, 96, 16, 9)
    base = sig.ragged.RaggedPairwise(lx, ly, orders, 16, precision=prec)
    base.load(X, Y)
    want = base.solve().clone()
    tuner = sig.autotune.RaggedTuner(16, precision=prec, pairs_per_bucket=64)
    tuned = sig.ragged.RaggedPairwise(lx, ly, orders, 16, precision=prec, tuner=tuner)
    assert tuner.table, "every bucket of the batch is tuned"
    for (lg, db, o), R in tuner.table.items():
        assert R in sig.autotune.ROWS and db == sig.autotune.dim_bucket(16)
    assert tuned.source == tuner.choice()["source"] and sig.autotune.dim_bucket(16) in tuner.batch_timings
    tuned.load(X, Y)
    got = tuned.solve()
    if tuned.source == base.source and tuned.tile_n == base.tile_n:
        assert torch.equal(got, want)
    elif prec == "fp64":
        assert float(((got.double() - want.double()).abs() / want.double().abs()).max()) <= 1e-6  # float32 outputs
    else:
        assert torch.isfinite(got).all()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "tc64"])
def test_every_rows_and_tile_candidate_gives_identical_results(oracle, prec):
    """Rows per lane (bands per pair) and the GEMM tile width change which warp or
    tile computes a value, not its arithmetic: bitwise equal results."""
    import sigpde_b200.torch as sig
    lx, ly, orders, X, Y = _batch(oracle, 40, 8, 10)
    tiles = (256, 128) if prec == "tc64" else (256,)
    ref = None
    for tile_n in tiles:
        for R in (2, 4, 8, 16):
            solver = sig.ragged.RaggedPairwise(lx, ly, orders, 8, precision=prec, source="matrix", tile_n=tile_n,
                                               rows_fn=lambda n, o, R=R: R)
            assert solver.tile_n == tile_n
            solver.load(X, Y)
            got = solver.solve().clone()
            solver.check()
            if ref is None:
                ref = got
            else:
                assert torch.equal(got, ref), f"tile_n={tile_n} R={R}"
