"""Uneven batched pairwise solves (sigk_pairwise_ragged) against the float64
oracle, pair by pair.  Tolerances as in test_parity_gpu: float64 cells, so
the bound is 1e-9 relative for float64 outputs and 2.5e-7 (float32 output
rounding) for float32 outputs."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _batch(oracle, specs, seed, dtype):
    rng = np.random.default_rng(seed)
    xs, ys = [], []
    for i, (lx, ly, d, o) in enumerate(specs):
        xs.append(oracle.brownian(1, lx, d, int(rng.integers(1 << 30)))[0])
        ys.append(oracle.brownian(1, ly, d, int(rng.integers(1 << 30)))[0])
    X = [torch.tensor(a, dtype=dtype, device="cuda") for a in xs]
    Y = [torch.tensor(a, dtype=dtype, device="cuda") for a in ys]
    return X, Y


def _want(oracle, X, Y, orders, sx=None, sy=None):
    out = []
    for b, (x, y, o) in enumerate(zip(X, Y, orders)):
        xin = x.double().cpu().numpy()[None]
        yin = y.double().cpu().numpy()[None]
        s1 = None if sx is None else np.array([float(sx[b])])
        s2 = None if sy is None else np.array([float(sy[b])])
        out.append(oracle.pairwise(xin, yin, o, s1, s2)[0])
    return np.array(out)


def _rel(got, want):
    return float(np.max(np.abs(got - want) / np.abs(want)))


SPECS = [
    # (len x, len y, dim, order)
    (16, 40, 4, 0), (40, 16, 4, 0), (33, 33, 4, 1), (70, 20, 4, 2), (9, 120, 4, 3),
    (130, 150, 4, 2),   # two bands on the shorter side (516 rows)
    (300, 90, 4, 1),    # swapped: 89 * 2 = 178 rows, 598 columns
    (2, 2, 4, 0), (3, 7, 4, 5), (520, 517, 4, 0),
]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_ragged_matches_oracle(sig, oracle, dtype):
    X, Y = _batch(oracle, SPECS, 1, dtype)
    orders = [s[3] for s in SPECS]
    got = sig.ragged.pairwise(X, Y, orders).double().cpu().numpy()
    want = _want(oracle, X, Y, orders)
    tol = 1e-9 if dtype is torch.float64 else 2.5e-7
    assert _rel(got, want) <= tol


def _cs_err(oracle, X, Y, orders, got, sx=None, sy=None):
    want = _want(oracle, X, Y, orders, sx, sy)
    kxx = _want(oracle, X, X, orders, sx, sx)
    kyy = _want(oracle, Y, Y, orders, sy, sy)
    return float(np.max(np.abs(got - want) / np.sqrt(np.abs(kxx * kyy))))


@pytest.mark.parametrize("prec", ["tc64", "tc32"])
def test_ragged_tensor_core_increments(sig, oracle, prec):
    """Increments from the grouped split-TF32 GEMM (tensor-core plan): CS-normalised
    error <= 1e-5 with float64 cells, <= 4x the fp32-cell mode's own error with
    float32 cells; the float64-cell run is also checked against fp64 mode."""
    specs = SPECS + [(200, 300, 32, 1), (64, 64, 17, 3)]
    for d in (4, 32, 17):
        sp = [(a, b, d, o) for (a, b, _, o) in specs]
        X, Y = _batch(oracle, sp, 11 + d, torch.float64)
        orders = [s[3] for s in sp]
        got = sig.ragged.pairwise(X, Y, orders, precision=prec).cpu().numpy()
        err = _cs_err(oracle, X, Y, orders, got)
        if prec == "tc64":
            assert err <= 1e-5, err
        else:
            ref = sig.ragged.pairwise(X, Y, orders, precision="fp32").cpu().numpy()
            assert err <= 4 * _cs_err(oracle, X, Y, orders, ref) + 1e-7, err


def test_ragged_tensor_core_graph_replay_and_scales(sig, oracle):
    specs = [(30 + 11 * i, 25 + 5 * i, 8, (i % 3) + 1) for i in range(20)] + [(600, 90, 8, 1)]
    orders = [s[3] for s in specs]
    solver = sig.ragged.RaggedPairwise([s[0] for s in specs], [s[1] for s in specs], orders, 8,
                                       dtype=torch.float32, device="cuda", precision="tc64")
    assert solver.tc is not None
    sx = np.linspace(0.5, 1.5, len(specs))
    sy = np.linspace(1.4, 0.6, len(specs))
    for seed in (4, 5):
        X, Y = _batch(oracle, specs, seed, torch.float32)
        solver.load(X, Y, sx, sy)
        if seed == 4:
            solver.capture()
        got = solver.solve().double().cpu().numpy()
        assert _cs_err(oracle, X, Y, orders, got, sx, sy) <= 1e-5
        assert solver.error_flag() == 0


def test_ragged_scales_and_dimension(sig, oracle):
    specs = [(20 + 7 * i, 60 - 3 * i, 32, i % 4) for i in range(12)]
    X, Y = _batch(oracle, specs, 2, torch.float64)
    orders = [s[3] for s in specs]
    sx = np.linspace(0.5, 1.5, 12)
    sy = np.linspace(1.4, 0.6, 12)
    got = sig.ragged.pairwise(X, Y, orders, x_scale=sx, y_scale=sy).cpu().numpy()
    assert _rel(got, _want(oracle, X, Y, orders, sx, sy)) <= 1e-9


@pytest.mark.parametrize("dim", [16, 40])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_ragged_float64_increment_matrix(sig, oracle, monkeypatch, dim, dtype):
    """fp64 batches with d >= 16 take float64 increments from one FP64 GEMM over the
    plan's tiles: the oracle's values, and the fused path's up to the order of the
    scalings (rows on the shorter path, scales on either side)."""
    from sigpde_b200.torch import ragged as rg
    specs = [(lx, ly, dim, o) for lx, ly, _, o in SPECS]
    X, Y = _batch(oracle, specs, 7, dtype)
    orders = [s[3] for s in specs]
    sx = np.linspace(0.6, 1.3, len(specs))
    sy = np.linspace(1.2, 0.7, len(specs))
    got = sig.ragged.pairwise(X, Y, orders, x_scale=sx, y_scale=sy).double().cpu().numpy()
    tol = 1e-9 if dtype is torch.float64 else 2.5e-7
    # the scales are held in the paths' dtype, as the reference holds them
    sxe = torch.tensor(sx, dtype=dtype).double().numpy()
    sye = torch.tensor(sy, dtype=dtype).double().numpy()
    assert _rel(got, _want(oracle, X, Y, orders, sxe, sye)) <= tol
    monkeypatch.setattr(rg, "MAT64_MIN_DIM", 1 << 30)  # the fused form
    fused = sig.ragged.pairwise(X, Y, orders, x_scale=sx, y_scale=sy).double().cpu().numpy()
    assert _rel(got, fused) <= (1e-12 if dtype is torch.float64 else 2.5e-7)


@pytest.mark.parametrize("dim", [16, 24, 32])
def test_ragged_pipelined_dgemm_bit_identical(sig, oracle, monkeypatch, dim):
    """The pipelined float64 GEMM (half-tiles sharing their A rows, next B rows
    prefetched) gives exactly the one-piece-per-CTA GEMM's increments."""
    specs = [(lx, ly, dim, o) for lx, ly, _, o in SPECS]
    X, Y = _batch(oracle, specs, 11, torch.float64)
    orders = [s[3] for s in specs]
    sx = np.linspace(0.6, 1.3, len(specs))
    pipe = sig.ragged.pairwise(X, Y, orders, x_scale=sx).cpu().numpy()
    monkeypatch.setenv("SIGK_NO_DGEMM_PIPE", "1")
    single = sig.ragged.pairwise(X, Y, orders, x_scale=sx).cpu().numpy()
    monkeypatch.delenv("SIGK_NO_DGEMM_PIPE")
    assert np.all(np.isfinite(pipe))
    np.testing.assert_array_equal(pipe, single)
    sxe = torch.tensor(sx, dtype=torch.float64).numpy()
    assert _rel(pipe, _want(oracle, X, Y, orders, sxe, np.ones(len(specs)))) <= 1e-9


def test_ragged_graph_replay_with_new_values(sig, oracle):
    specs = [(30 + 11 * i, 25 + 5 * i, 8, (i % 3) + 1) for i in range(20)]
    orders = [s[3] for s in specs]
    solver = sig.ragged.RaggedPairwise([s[0] for s in specs], [s[1] for s in specs], orders, 8,
                                       dtype=torch.float64, device="cuda")
    X1, Y1 = _batch(oracle, specs, 3, torch.float64)
    solver.load(X1, Y1)
    solver.capture()
    for seed in (4, 5):
        X, Y = _batch(oracle, specs, seed, torch.float64)
        solver.load(X, Y)
        got = solver.solve().cpu().numpy()
        assert _rel(got, _want(oracle, X, Y, orders)) <= 1e-9


def test_ragged_long_pairs_split_into_band_pipelines(sig, oracle):
    """Pairs of 4 to 8 bands run as pipelines of warps; mixed with short pairs."""
    specs = [(512, 500, 8, 3), (300, 512, 8, 3), (130, 140, 8, 2)] + [(12 + i, 30 - i, 8, i % 3) for i in range(10)]
    X, Y = _batch(oracle, specs, 7, torch.float32)
    orders = [s[3] for s in specs]
    solver = sig.ragged.RaggedPairwise([s[0] for s in specs], [s[1] for s in specs], orders, 8,
                                       dtype=torch.float32, device="cuda")
    assert int(solver.pair_bands.max()) >= 8
    solver.load(X, Y)
    got = solver.solve().double().cpu().numpy()
    assert _rel(got, _want(oracle, X, Y, orders)) <= 2.5e-7
    assert solver.error_flag() == 0


def test_ragged_plan_is_consistent():
    import sigpde_b200.torch.ragged as rg
    pl = rg.plan([20, 600, 40], [500, 30, 41], [3, 1, 0], 32, 8)
    # every pair's bands are consecutive and ordered; longest pair first
    assert pl["item_pair"][0] == 0
    for b in range(3):
        idx = np.nonzero(pl["item_pair"] == b)[0]
        assert np.all(np.diff(idx) == 1) and list(pl["item_band"][idx]) == list(range(pl["bands"][b]))


def test_ragged_invalid_pairs_give_nan_without_faulting(sig, oracle):
    from sigpde_b200 import _lib
    specs = [(10, 12, 2, 1), (10, 12, 2, 1)]
    solver = sig.ragged.RaggedPairwise([s[0] for s in specs], [s[1] for s in specs], [1, 1], 2,
                                       dtype=torch.float64, device="cuda")
    X, Y = _batch(oracle, specs, 6, torch.float64)
    solver.load(X, Y)
    solver.order[1] = 13  # outside [0, 12]: refused by the kernel, not solved
    got = solver.solve().cpu().numpy()
    assert np.isfinite(got[0]) and np.isnan(got[1])
    assert solver.error_flag() == 1
    assert _lib.lib().sigk_ragged_workspace_size(0, 0, 0, 2, 0, 0, 0) == 0


@pytest.fixture(scope="module")
def sig():
    import sigpde_b200.torch as sig
    return sig
