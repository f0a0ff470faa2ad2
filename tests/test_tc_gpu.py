"""Tensor-core increments (precision "tc32" / "tc64") against the float64 oracle.

The increments <dx_i, dy_j> of all pairs come from one split-TF32 tcgen05
GEMM (hi*hi + hi*lo + lo*hi, float32 accumulation) and are read back by the
streaming wavefront.  Tolerances, with errors normalised by the
Cauchy-Schwarz bound sqrt(k(x,x) k(y,y)) (the cells grow to that size, so a
pointwise bound on near-zero entries is not available in float32 storage):
  * "tc64" (float64 cells): at most 1e-5, the accuracy target for the fast
    modes on Brownian paths;
  * "tc32" (float32 cells): at most 6x the reference's own float32 GPU
    numerics on the same inputs, plus 1e-7 (the "fp32" bound of 4x, widened
    for the split-TF32 increments' own ~2^-21 relative error, which adds to
    the float32 cell rounding on long paths).
Pairs of several bands of rows, or with fewer than 32 column blocks, read
the same matrix from the per-pair kernel.  dim > 32 is outside the TC plan:
those increments are formed on the CUDA cores and, with float64 cells, meet
the fp64 bound of 1e-9 relative.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

CS_TC64 = 1e-5


@pytest.fixture(scope="module")
def sig():
    import sigpde_b200.torch as sig
    return sig


def cuda(a, dtype=torch.float32):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device="cuda")


def host(t):
    return t.detach().double().cpu().numpy()


def cs(got, want, kxx, kyy):
    return float(np.max(np.abs(got - want) / np.sqrt(np.abs(kxx * kyy))))


def _check(oracle, got, x, y, order, prec, sx=None, sy=None, sym=False, pairwise=False):
    if pairwise:
        want = oracle.pairwise(x, y, order, sx, sy)
        ref = oracle.pairwise(x, y, order, sx, sy, store_f32=True)
        kxx = oracle.pairwise(x, None, order, sx, sx)
        kyy = oracle.pairwise(y, None, order, sy, sy)
    else:
        want = oracle.gram(x, None if sym else y, order, sx, sy)
        ref = oracle.gram(x, None if sym else y, order, sx, sy, store_f32=True)
        yy, syy = (x, sx) if sym else (y, sy)
        kxx = oracle.pairwise(x, None, order, sx, sx)[:, None]
        kyy = oracle.pairwise(yy, None, order, syy, syy)[None, :]
    err = cs(got, want, kxx, kyy)
    if prec == "tc64":
        assert err <= CS_TC64, f"tc64 CS-normalised error {err:.3e}"
    else:
        tol = 6.0 * cs(ref, want, kxx, kyy) + 1e-7
        assert err <= tol, f"tc32 CS-normalised error {err:.3e} > {tol:.3e}"
    return err


SHAPES = [
    # (n_x, n_y, L, d, order)
    (12, 10, 40, 8, 2),
    (9, 14, 33, 5, 1),
    (6, 7, 20, 16, 4),
    (8, 8, 40, 32, 0),
    (5, 6, 128, 8, 2),
]


@pytest.mark.parametrize("prec", ["tc64", "tc32"])
@pytest.mark.parametrize("shape", SHAPES)
def test_tc_gram(sig, oracle, prec, shape):
    nx, ny, L, d, o = shape
    X = cuda(oracle.brownian(nx, L, d, 11 + L))
    Y = cuda(oracle.brownian(ny, L + 3, d, 12 + L))
    k = sig.SigPDE(sig.kernels.LinearKernel(), o, precision=prec)
    got = host(k.gram(X, Y))
    _check(oracle, got, host(X), host(Y), o, prec)


@pytest.mark.parametrize("prec", ["tc64", "tc32"])
def test_tc_symmetric_gram_and_pairwise(sig, oracle, prec):
    X = cuda(oracle.brownian(15, 64, 16, 21))
    Y = cuda(oracle.brownian(15, 64, 16, 22))
    k = sig.SigPDE(sig.kernels.LinearKernel(), 1, precision=prec)
    G = host(k.gram(X))
    assert np.array_equal(G, G.T)
    _check(oracle, G, host(X), None, 1, prec, sym=True)
    _check(oracle, host(k.pairwise(X, Y)), host(X), host(Y), 1, prec, pairwise=True)


def test_tc_scales_and_float64_inputs(sig, oracle):
    x = oracle.brownian(10, 50, 8, 31)
    y = oracle.brownian(7, 45, 8, 32)
    sx = np.linspace(0.5, 1.7, 10)
    sy = np.linspace(1.3, 0.4, 7)
    k = sig.SigPDE(sig.kernels.LinearKernel(1.7), 2, precision="tc64")
    got = host(k.gram(cuda(x, torch.float64), cuda(y, torch.float64), cuda(sx, torch.float64),
                      cuda(sy, torch.float64)))
    _check(oracle, got, x * np.sqrt(1.7), y * np.sqrt(1.7), 2, "tc64", sx, sy)
    got = host(k.gram(cuda(x, torch.float64), None, cuda(sx, torch.float64)))
    _check(oracle, got, x * np.sqrt(1.7), None, 2, "tc64", sx, sx, sym=True)


def test_tc_chunked_matches_unchunked(sig, oracle, monkeypatch):
    """Chunks of x paths (forced with a 1 MB matrix cap) give the same numbers."""
    x = oracle.brownian(24, 64, 8, 41)
    y = oracle.brownian(20, 64, 8, 42)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 1, precision="tc64")
    X, Y = cuda(x), cuda(y)
    full = [host(k.gram(X, Y)), host(k.gram(X)), host(k.pairwise(X, Y[:20].repeat(2, 1, 1)[:24]))]
    monkeypatch.setenv("SIGK_TC_CHUNK_MB", "1")
    part = [host(k.gram(X, Y)), host(k.gram(X)), host(k.pairwise(X, Y[:20].repeat(2, 1, 1)[:24]))]
    for a, b in zip(full, part):
        np.testing.assert_array_equal(a, b)


def test_tc_is_deterministic(sig, oracle):
    x = oracle.brownian(16, 128, 8, 51)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 2, precision="tc32")
    X = cuda(x)
    a = host(k.gram(X, X))
    b = host(k.gram(X, X))
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("prec", ["tc64", "tc32"])
@pytest.mark.parametrize("shape", [(3, 4, 600, 4, 0), (5, 4, 170, 32, 2), (6, 5, 20, 8, 0)])
def test_tc_multi_band_and_short_pairs(sig, oracle, shape, prec):
    """Pairs of several bands of rows (n > 512) or fewer than 32 column blocks read the
    increment matrix from the per-pair kernel: Gram, symmetric Gram and pairwise."""
    nx, ny, L, d, o = shape
    X = cuda(oracle.brownian(nx, L, d, 61))
    Y = cuda(oracle.brownian(ny, L + 5, d, 62))
    k = sig.SigPDE(sig.kernels.LinearKernel(), o, precision=prec)
    _check(oracle, host(k.gram(X, Y)), host(X), host(Y), o, prec)
    _check(oracle, host(k.gram(X)), host(X), None, o, prec, sym=True)
    Yp = cuda(oracle.brownian(nx, L + 5, d, 63))
    _check(oracle, host(k.pairwise(X, Yp)), host(X), host(Yp), o, prec, pairwise=True)


def test_tc_modes_outside_the_plan_use_cuda_core_increments(sig, oracle):
    """dim > 32 runs CUDA-core increments with float64 cells (fp64 bound)."""
    x = oracle.brownian(4, 30, 40, 61)
    y = oracle.brownian(3, 30, 40, 62)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 1, precision="tc64")
    got = host(k.gram(cuda(x, torch.float64), cuda(y, torch.float64)))
    want = oracle.gram(x, y, 1)
    assert np.max(np.abs(got - want) / np.abs(want)) <= 1e-9
