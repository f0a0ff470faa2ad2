"""RBF / L1-RBF Grams with the static kernel evaluated from the path points on
the device (sigk_gram_static), against the float64 oracle.

The oracle builds the static Gram of all point pairs in float64
(oracle.static_gram, the formulas of sigpde/torch/static_kernels.py:13-53),
the 4-term second difference / 4^order (sigpde/torch/kernel.py:18-21) and the
solve.  Tolerance: relative error <= 1e-8 per entry for float64 outputs (the
RBF distance |x|^2 + |y|^2 - 2<x,y> and the second difference cancel; in
float64 that leaves ~1e-11 relative on the increments), and the float32
rounding of the output (2.5e-7) for float32 paths, whose results are float32
as in the reference.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

RTOL = 1e-8
RTOL_OUT32 = 2.5e-7


def cuda(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device="cuda")


def host(t):
    return t.detach().double().cpu().numpy()


def assert_rel(got, want, rtol, msg=""):
    err = np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300))
    assert err <= rtol, f"{msg}: max relative error {err:.3e} > {rtol:.1e}"


@pytest.fixture(scope="module")
def sig():
    import sigpde_b200.torch as sig
    return sig


def static_kernel(sig, kind, sigma):
    return sig.kernels.RBFKernel(sigma) if kind == "rbf" else sig.kernels.L1RBFKernel(sigma)


SHAPES = [
    # (n_x, n_y, L_x, L_y, d, order)
    (5, 4, 9, 11, 3, 1),      # rows padded (ncx = 8 -> 8), short y: per-pair kernel
    (6, 7, 2, 3, 1, 0),       # one coarse row; y paths of 2 cells
    (4, 5, 5, 4, 2, 2),       # ncx = 4 = rows_x: no padding row
    (9, 8, 40, 37, 8, 2),     # streaming wavefront
    (7, 6, 33, 40, 17, 1),    # dimension padded to 32
    (3, 4, 30, 34, 32, 4),    # order 4: several steps per coarse column
    (3, 3, 70, 66, 5, 3),     # 552 refined rows: several bands
    (40, 3, 6, 6, 4, 0),      # many x paths per warp (6 points each)
]


@pytest.mark.parametrize("kind", ["rbf", "l1rbf"])
@pytest.mark.parametrize("shape", SHAPES)
def test_static_gram(sig, oracle, kind, shape):
    nx, ny, lx, ly, d, o = shape
    x = oracle.brownian(nx, lx, d, 100 + lx)
    y = oracle.brownian(ny, ly, d, 200 + ly)
    sigma = 0.9
    k = sig.SigPDE(static_kernel(sig, kind, sigma), o)
    got = host(k.gram(cuda(x), cuda(y)))
    want = oracle.gram(x, y, o, static=kind, static_param=sigma)
    assert_rel(got, want, RTOL, f"{kind} gram {shape}")


@pytest.mark.parametrize("kind", ["rbf", "l1rbf"])
@pytest.mark.parametrize("shape", [(9, 21, 5, 1), (5, 40, 8, 2), (4, 70, 3, 3), (33, 7, 16, 0)])
def test_static_symmetric_gram(sig, oracle, kind, shape):
    n, L, d, o = shape
    x = oracle.brownian(n, L, d, 300 + L)
    k = sig.SigPDE(static_kernel(sig, kind, 1.3), o)
    G = host(k.gram(cuda(x)))
    assert np.array_equal(G, G.T)
    assert_rel(G, oracle.gram(x, None, o, static=kind, static_param=1.3), RTOL, f"{kind} sym {shape}")


@pytest.mark.parametrize("kind", ["rbf", "l1rbf"])
def test_static_scales_and_float32_inputs(sig, oracle, kind):
    x = oracle.brownian(6, 25, 4, 41)
    y = oracle.brownian(5, 30, 4, 42)
    sx = np.linspace(0.5, 1.7, 6)
    sy = np.linspace(1.3, 0.4, 5)
    k = sig.SigPDE(static_kernel(sig, kind, 0.7), 2)
    got = host(k.gram(cuda(x), cuda(y), cuda(sx), cuda(sy)))
    assert_rel(got, oracle.gram(x, y, 2, sx, sy, static=kind, static_param=0.7), RTOL, "scaled")
    got = host(k.gram(cuda(x), None, cuda(sx)))
    assert_rel(got, oracle.gram(x, None, 2, sx, static=kind, static_param=0.7), RTOL, "sym scaled")
    # a [1] scale is broadcast (sigpde/torch/kernel.py:40-41)
    got = host(k.gram(cuda(x), cuda(y), cuda([1.4])))
    assert_rel(got, oracle.gram(x, y, 2, np.full(6, 1.4), np.ones(5), static=kind, static_param=0.7), RTOL,
               "broadcast")
    # float32 paths: the same float32 values, float32 results
    x32, y32 = cuda(x, torch.float32), cuda(y, torch.float32)
    G32 = k.gram(x32, y32)
    assert G32.dtype == torch.float32
    want = oracle.gram(host(x32), host(y32), 2, static=kind, static_param=0.7)
    assert_rel(host(G32), want, RTOL_OUT32, "float32 in/out")


def test_static_chunks_and_tc64_are_bitwise_the_same(sig, oracle, monkeypatch):
    """Chunks of x paths (a 1 MB matrix cap) and precision "tc64" (float64
    cells, the same increments) give the same bits."""
    x = oracle.brownian(40, 48, 6, 51)
    y = oracle.brownian(30, 52, 6, 52)
    X, Y = cuda(x), cuda(y)
    k = sig.SigPDE(sig.kernels.RBFKernel(2.0), 1)
    full = [host(k.gram(X, Y)), host(k.gram(X))]
    kt = sig.SigPDE(sig.kernels.RBFKernel(2.0), 1, precision="tc64")
    for a, b in zip(full, [host(kt.gram(X, Y)), host(kt.gram(X))]):
        np.testing.assert_array_equal(a, b)
    monkeypatch.setenv("SIGK_TC_CHUNK_MB", "1")
    for a, b in zip(full, [host(k.gram(X, Y)), host(k.gram(X))]):
        np.testing.assert_array_equal(a, b)
    assert_rel(full[0], oracle.gram(x, y, 1, static="rbf", static_param=2.0), RTOL, "gram")


def test_static_matches_the_generic_route(sig, oracle):
    """The device-evaluated static Gram and the reference's route (torch static
    Gram and 4-term difference, then the increment solver) agree on float64
    inputs; wide paths (d > 32) keep the reference's route."""
    from sigpde_b200.torch import kernel as kmod
    x = oracle.brownian(7, 30, 5, 61)
    y = oracle.brownian(6, 26, 5, 62)
    X, Y = cuda(x), cuda(y)
    sk = sig.kernels.L1RBFKernel(1.1)
    k = sig.SigPDE(sk, 2)
    fused = host(k.gram(X, Y))
    inc = kmod.gram_inner_product(X, Y, sk, 2)
    generic = torch.empty((7, 6), dtype=torch.float64, device="cuda")
    k._solve_gram_inc(inc, None, None, generic, 0, 0, False)
    assert_rel(fused, host(generic), 1e-10, "fused vs generic")
    xw = oracle.brownian(3, 12, 33, 63)
    kw = sig.SigPDE(sig.kernels.RBFKernel(8.0), 1)
    assert not kw._static_on_device(cuda(xw))
    assert_rel(host(kw.gram(cuda(xw))), oracle.gram(xw, None, 1, static="rbf", static_param=8.0), RTOL, "d=33")


@pytest.mark.parametrize("kind", ["rbf", "l1rbf"])
def test_robust_gram_with_static_kernels(sig, oracle, kind):
    """RobustSigPDE.gram: lambda from the normalisation, then the scaled Gram on
    the device-evaluated static kernel."""
    x = oracle.brownian(6, 20, 3, 71) * 3.0
    y = oracle.brownian(5, 22, 3, 72) * 3.0
    rk = sig.RobustSigPDE(static_kernel(sig, kind, 0.8), 1)
    lx = host(rk.normalization(cuda(x)))
    ly = host(rk.normalization(cuda(y)))
    got = host(rk.gram(cuda(x), cuda(y)))
    want = oracle.gram(x, y, 1, lx, ly, static=kind, static_param=0.8)
    assert_rel(got, want, 1e-7, "robust gram")


def _cs_err(got, want, kxx, kyy):
    return np.abs(got - want) / np.sqrt(np.abs(kxx * kyy))


@pytest.mark.parametrize("prec", ["fp32", "tc32"])
@pytest.mark.parametrize("kind", ["rbf", "l1rbf"])
@pytest.mark.parametrize("shape", [(9, 8, 40, 37, 8, 2), (5, 4, 9, 11, 3, 1), (3, 3, 70, 66, 5, 3), (7, 6, 33, 40, 17, 1)])
@pytest.mark.parametrize("in64", [False, True])
def test_static_gram_float32_cells(sig, oracle, prec, kind, shape, in64):
    """Float32 cells (precision fp32 / tc32) read the device-evaluated increments
    rounded once to float32, from float32 or float64 input paths.  Tolerance as
    for the linear kernel's float32 cells: error normalised by
    sqrt(k(x,x) k(y,y)) at most 4x that of the reference's own numerics on the
    same inputs (float64 arithmetic, float32 storage of every cell: the oracle
    with store_f32=True), plus 1e-7."""
    nx, ny, lx, ly, d, o = shape
    x = oracle.brownian(nx, lx, d, 500 + lx)
    y = oracle.brownian(ny, ly, d, 600 + ly)
    sigma = 0.9
    k = sig.SigPDE(static_kernel(sig, kind, sigma), o, precision=prec)
    dt = torch.float64 if in64 else torch.float32
    X, Y = cuda(x, dt), cuda(y, dt)
    assert k._static_on_device(X)
    xin, yin = host(X), host(Y)
    got = host(k.gram(X, Y))
    want = oracle.gram(xin, yin, o, static=kind, static_param=sigma)
    ref = oracle.gram(xin, yin, o, static=kind, static_param=sigma, store_f32=True)
    kxx = oracle.pairwise(xin, None, o, static=kind, static_param=sigma)[:, None]
    kyy = oracle.pairwise(yin, None, o, static=kind, static_param=sigma)[None, :]
    tol = 4.0 * float(_cs_err(ref, want, kxx, kyy).max()) + 1e-7
    err = float(_cs_err(got, want, kxx, kyy).max())
    assert err <= tol, f"{prec} {kind} {shape}: CS-normalised error {err:.3e} > {tol:.3e}"
    G = host(k.gram(X))
    assert np.array_equal(G, G.T)
    wsym = oracle.gram(xin, None, o, static=kind, static_param=sigma)
    rsym = oracle.gram(xin, None, o, static=kind, static_param=sigma, store_f32=True)
    tol = 4.0 * float(_cs_err(rsym, wsym, kxx, kxx.T).max()) + 1e-7
    assert float(_cs_err(G, wsym, kxx, kxx.T).max()) <= tol
