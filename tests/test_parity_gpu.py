"""Parity of the CUDA engine (through the sigpde_b200.torch API and the C ABI)
against the float64 oracle and the reference's golden vectors.

Tolerances (stated per test):
  * precision="fp64" (float64 cells, the default): relative error <= 1e-9 per
    entry against the float64 oracle on the same inputs when the output is
    float64; float32 inputs return float32 results (as the reference does), so
    their bound is the float32 rounding of the output, 2.5e-7 (2 ulp);
  * precision="fp32" (float32 cells): error normalised by the Cauchy-Schwarz
    bound sqrt(k(x,x) k(y,y)) at most 4x that of the reference's own GPU
    numerics on the same inputs (float64 arithmetic, every cell stored as
    float32; the oracle emulates it with store_f32=True), plus 1e-7: both
    round each cell once at the magnitude of K.  Float32
    cells cannot give a pointwise bound on near-zero entries: the cells grow to
    ~sqrt(k(x,x) k(y,y));
  * robust lambda: relative error <= 1e-6 (absolute 1e-9 near 0).
"""
import re

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

RTOL64 = 1e-9
RTOL_OUT32 = 2.5e-7
CS32 = 2e-5
LAM_RTOL = 1e-6


def cuda(a, dtype=torch.float32):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device="cuda")


def host(t):
    return t.detach().double().cpu().numpy()


def _keys(golden, pattern):
    rx = re.compile(pattern)
    return sorted({m.group(1) for k in golden for m in [rx.match(k)] if m})


def _order(key):
    return int(re.search(r"_o(\d+)", key).group(1))


@pytest.fixture(scope="module")
def sig():
    import sigpde_b200.torch as sig
    return sig


def rtol_for(dt):
    return RTOL64 if dt is torch.float64 else RTOL_OUT32


def assert_rel(got, want, rtol=RTOL64, msg=""):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    err = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    assert np.all(np.isfinite(got)), msg
    assert err.max() <= rtol, f"{msg}: max rel err {err.max():.3e} > {rtol:.1e}"


def cs_err(got, want, kxx, kyy):
    return np.abs(np.asarray(got) - np.asarray(want)) / np.sqrt(np.abs(np.asarray(kxx) * np.asarray(kyy)))


def assert_cs(got, want, kxx, kyy, tol=CS32, msg=""):
    err = cs_err(got, want, kxx, kyy)
    assert err.max() <= tol, f"{msg}: max CS-normalised err {err.max():.3e} > {tol:.1e}"


def fp32_tol(ref_sem, want, kxx, kyy):
    """4x the CS-normalised error of the reference's float32 GPU numerics, + 1e-7."""
    return 4.0 * float(cs_err(ref_sem, want, kxx, kyy).max()) + 1e-7


# ----------------------------------------------------------------------------- golden vectors
def test_golden_pairwise(sig, golden):
    lin = sig.kernels.LinearKernel()
    for dt_name, dt in (("f64", torch.float64), ("f32", torch.float32)):
        for key in _keys(golden, rf"(pw_{dt_name}_L\d+_d\d+_o\d+)_out$"):
            x, y, o = golden[key + "_x"], golden[key + "_y"], _order(key)
            k = sig.SigPDE(lin, o)
            got = host(k.pairwise(cuda(x, dt), cuda(y, dt)))
            if dt is torch.float64:
                assert_rel(got, golden[key + "_out"], RTOL64, key)
            sx, sy = golden[key + "_sx"], golden[key + "_sy"]
            got_s = host(k.pairwise(cuda(x, dt), cuda(y, dt), cuda(sx, dt), cuda(sy, dt)))
            got_ss = host(k.pairwise(cuda(x, dt), None, cuda(sx, dt)))
            if dt is torch.float64:
                assert_rel(got_s, golden[key + "_scaled_out"], RTOL64, key + " scaled")
                assert_rel(got_ss, golden[key + "_self_scaled_out"], RTOL64, key + " self scaled")


def test_golden_gram(sig, golden):
    lin = sig.kernels.LinearKernel()
    for key in _keys(golden, r"(gr_f64_\d+x\d+_L\d+_d\d+_o\d+)_out$"):
        x, y, o = golden[key + "_x"], golden[key + "_y"], _order(key)
        k = sig.SigPDE(lin, o)
        X, Y = cuda(x, torch.float64), cuda(y, torch.float64)
        assert_rel(host(k.gram(X, Y)), golden[key + "_out"], RTOL64, key)
        assert_rel(host(k.gram(X, Y, max_batch=4)), golden[key + "_tiled_out"], RTOL64, key + " tiled")
        sx, sy = cuda(golden[key + "_sx"], torch.float64), cuda(golden[key + "_sy"], torch.float64)
        assert_rel(host(k.gram(X, Y, sx, sy)), golden[key + "_scaled_out"], RTOL64, key + " scaled")
        assert_rel(host(k.gram(X)), golden[key + "_sym_out"], RTOL64, key + " sym")
        assert_rel(host(k.gram(Y)), golden[key + "_sym_tiled_out"], RTOL64, key + " sym (y)")
        assert_rel(host(k.gram(X, None, sx)), golden[key + "_sym_scaled_out"], RTOL64, key + " sym scaled")


def test_golden_config1(sig, golden, oracle):
    """Config 1: SigPDE.pairwise, LinearKernel, B=8, L=20, d=5, order 1."""
    if "cfg1_f64_out" not in golden:
        pytest.skip("config-1 vectors not generated")
    k = sig.SigPDE(sig.kernels.LinearKernel(), 1)
    got = host(k.pairwise(cuda(golden["cfg1_f64_x"], torch.float64), cuda(golden["cfg1_f64_y"], torch.float64)))
    assert_rel(got, golden["cfg1_f64_out"], RTOL64, "cfg1 f64")
    x32, y32 = golden["cfg1_f32_x"], golden["cfg1_f32_y"]
    got = host(k.pairwise(cuda(x32), cuda(y32)))
    assert_rel(got, oracle.pairwise(x32, y32, 1), RTOL_OUT32, "cfg1 f32 inputs, fp64 cells")


def test_golden_robust(sig, golden):
    lin = sig.kernels.LinearKernel()
    for key in _keys(golden, r"(rn_f64_N\d+_L\d+_d\d+_o\d+(?:_pow)?)_out$"):
        x, o = golden[key + "_x"], _order(key)
        nrm = (lambda s: 2 - 1 / s.pow(0.1)) if key.endswith("_pow") else None
        lam = host(sig.RobustSigPDE(lin, o).normalization(cuda(x, torch.float64), normalizer=nrm))
        np.testing.assert_allclose(lam, golden[key + "_out"], rtol=LAM_RTOL, atol=1e-9, err_msg=key)
    for key in _keys(golden, r"(rb_f64_N\d+_L\d+_d\d+_o\d+)_pw_out$"):
        x, y, y2 = (cuda(golden[key + s], torch.float64) for s in ("_x", "_y", "_y2"))
        o = _order(key)
        rk = sig.RobustSigPDE(lin, o)
        np.testing.assert_allclose(host(rk.pairwise(x, y)), golden[key + "_pw_out"], rtol=1e-7, err_msg=key)
        np.testing.assert_allclose(host(rk.pairwise(x)), golden[key + "_pwself_out"], rtol=1e-7, err_msg=key)
        np.testing.assert_allclose(host(rk.gram(x, y2)), golden[key + "_gram_out"], rtol=1e-7, err_msg=key)
        np.testing.assert_allclose(host(rk.gram(x)), golden[key + "_gramsym_out"], rtol=1e-7, err_msg=key)


# ----------------------------------------------------------------------------- shapes vs oracle
SHAPES = [
    # (B, Lx, Ly, d, order)
    (5, 2, 2, 1, 0),
    (4, 3, 17, 2, 0),
    (3, 33, 33, 3, 0),
    (6, 20, 20, 5, 1),
    (3, 40, 23, 4, 2),
    (2, 9, 30, 6, 3),
    (2, 5, 7, 3, 4),
    (2, 4, 6, 2, 5),
    (3, 130, 90, 8, 2),      # n = 516 rows: two bands
    (2, 300, 64, 3, 1),      # n = 598 rows: two bands, short columns
    (2, 70, 70, 33, 0),      # d not a multiple of anything
    (2, 64, 64, 160, 1),     # dx staging does not fit: read from global
]


@pytest.mark.parametrize("B,Lx,Ly,d,o", SHAPES)
@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_pairwise_shapes(sig, oracle, B, Lx, Ly, d, o, dt):
    rng = np.random.default_rng(B * 1000 + Lx * 10 + d + o)
    x = oracle.brownian(B, Lx, d, int(rng.integers(1 << 30)))
    y = oracle.brownian(B, Ly, d, int(rng.integers(1 << 30)))
    X, Y = cuda(x, dt), cuda(y, dt)
    xin, yin = host(X), host(Y)
    k = sig.SigPDE(sig.kernels.LinearKernel(), o)
    got = host(k.pairwise(X, Y))
    assert_rel(got, oracle.pairwise(xin, yin, o), rtol_for(dt), f"pairwise {B, Lx, Ly, d, o}")
    sx = rng.uniform(0.5, 2.0, B)
    sy = rng.uniform(0.5, 2.0, B)
    got = host(k.pairwise(X, Y, cuda(sx, dt), cuda(sy, dt)))
    assert_rel(got, oracle.pairwise(xin, yin, o, host(cuda(sx, dt)), host(cuda(sy, dt))), rtol_for(dt), "scaled")


@pytest.mark.parametrize("Nx,Ny,L,d,o", [(3, 4, 10, 3, 1), (5, 2, 64, 8, 2), (4, 4, 140, 2, 2), (7, 7, 9, 2, 3)])
def test_gram_shapes(sig, oracle, Nx, Ny, L, d, o):
    x = oracle.brownian(Nx, L, d, 3)
    y = oracle.brownian(Ny, L + 3, d, 4)
    X, Y = cuda(x), cuda(y)
    k = sig.SigPDE(sig.kernels.LinearKernel(), o)
    assert_rel(host(k.gram(X, Y)), oracle.gram(host(X), host(Y), o), RTOL_OUT32, "gram")
    assert_rel(host(k.gram(X)), oracle.gram(host(X), None, o), RTOL_OUT32, "gram sym")
    sx = cuda(np.linspace(0.5, 2.0, Nx))
    assert_rel(host(k.gram(X, None, sx)), oracle.gram(host(X), None, o, host(sx)), RTOL_OUT32, "gram sym scaled")
    assert_rel(host(k.gram(X, Y, sx)), oracle.gram(host(X), host(Y), o, host(sx), None), RTOL_OUT32,
               "gram x scaled")


# shapes that take the streaming kernel (one band of <= 512 refined rows, >= 32 column blocks)
STREAM_SHAPES = [
    # (Nx, Ny, Lx, Ly, d, order)
    (5, 7, 40, 50, 3, 0),
    (3, 9, 33, 33, 1, 1),
    (6, 6, 100, 70, 8, 2),
    (3, 4, 40, 36, 4, 3),
    (2, 3, 20, 40, 2, 4),
    (2, 2, 10, 35, 2, 5),
]


@pytest.mark.parametrize("Nx,Ny,Lx,Ly,d,o", STREAM_SHAPES)
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_stream_kernel(sig, oracle, Nx, Ny, Lx, Ly, d, o, prec):
    x = oracle.brownian(Nx, Lx, d, 100 + o)
    y = oracle.brownian(Ny, Ly, d, 200 + o)
    X, Y = cuda(x), cuda(y)
    xin, yin = host(X), host(Y)
    k = sig.SigPDE(sig.kernels.LinearKernel(), o, precision=prec)
    sx = cuda(np.linspace(0.6, 1.4, Nx))
    sy = cuda(np.linspace(1.3, 0.7, Ny))
    got = {"gram": host(k.gram(X, Y)), "gram_scaled": host(k.gram(X, Y, sx, sy)), "sym": host(k.gram(Y)),
           "pairwise": host(k.pairwise(X[:2], Y[:2]))}
    want = {"gram": oracle.gram(xin, yin, o), "gram_scaled": oracle.gram(xin, yin, o, host(sx), host(sy)),
            "sym": oracle.gram(yin, None, o), "pairwise": oracle.pairwise(xin[:2], yin[:2], o)}
    for name in got:
        if prec == "fp64":
            assert_rel(got[name], want[name], RTOL_OUT32, name)
        else:
            kx = oracle.pairwise(xin, None, o)
            ky = oracle.pairwise(yin, None, o)
            if name == "gram":
                ref = oracle.gram(xin, yin, o, store_f32=True)
                kk = (kx[:, None], ky[None, :])
            elif name == "sym":
                ref = oracle.gram(yin, None, o, store_f32=True)
                kk = (ky[:, None], ky[None, :])
            elif name == "pairwise":
                ref = oracle.pairwise(xin[:2], yin[:2], o, store_f32=True)
                kk = (kx[:2], ky[:2])
            else:
                continue
            assert_cs(got[name], want[name], *kk, fp32_tol(ref, want[name], *kk), name)


def test_stream_and_per_pair_kernels_agree(sig, oracle, monkeypatch):
    x = oracle.brownian(37, 60, 5, 301)
    y = oracle.brownian(29, 60, 5, 302)
    X, Y = cuda(x, torch.float64), cuda(y, torch.float64)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 2)
    a = host(k.gram(X, Y))
    monkeypatch.setenv("SIGK_NO_STREAM", "1")
    b = host(k.gram(X, Y))
    monkeypatch.delenv("SIGK_NO_STREAM")
    assert_rel(a, b, 1e-13, "stream vs per-pair")
    assert_rel(a, oracle.gram(x, y, 2), RTOL64, "stream vs oracle")


@pytest.mark.parametrize("Nx,Ny,Lx,Ly,d,o", STREAM_SHAPES + [(7, 5, 128, 130, 8, 2), (1, 1, 60, 64, 5, 1)])
def test_paired_fp32_stream_bit_identical(sig, oracle, monkeypatch, Nx, Ny, Lx, Ly, d, o):
    """float32 cells: the two-pairs-per-lane kernel (paired f32x2 instructions)
    returns exactly the one-pair kernel's values, for odd and even runs of
    items (Gram, scaled Gram, symmetric Gram, pairwise)."""
    X = cuda(oracle.brownian(Nx, Lx, d, 400 + o))
    Y = cuda(oracle.brownian(Ny, Ly, d, 500 + o))
    sx = cuda(np.linspace(0.6, 1.4, Nx))
    k = sig.SigPDE(sig.kernels.LinearKernel(), o, precision="fp32")
    n = min(Nx, Ny)

    def run():
        return [host(k.gram(X, Y)), host(k.gram(X, Y, sx)), host(k.gram(Y)), host(k.pairwise(X[:n], Y[:n]))]

    paired = run()
    monkeypatch.setenv("SIGK_NO_PAIRED_F32", "1")
    single = run()
    monkeypatch.delenv("SIGK_NO_PAIRED_F32")
    for a, b in zip(paired, single):
        assert np.all(np.isfinite(a))
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("Nx,Ny,Lx,Ly,d,o", STREAM_SHAPES + [(7, 5, 128, 130, 8, 2), (3, 2, 60, 64, 5, 1),
                                                     (2, 1, 60, 64, 5, 1), (4, 3, 40, 40, 32, 0)])
def test_dual_fp64_stream_bit_identical(sig, oracle, monkeypatch, Nx, Ny, Lx, Ly, d, o):
    """float64 cells: the two-entries-per-lane Gram kernel returns exactly the
    one-entry kernel's values (odd and even numbers of y paths, scaled and
    unscaled, float32 and float64 inputs)."""
    X = cuda(oracle.brownian(Nx, Lx, d, 600 + o), torch.float64)
    Y = cuda(oracle.brownian(Ny, Ly, d, 700 + o), torch.float64)
    sx = cuda(np.linspace(0.6, 1.4, Nx), torch.float64)
    sy = cuda(np.linspace(1.2, 0.8, Ny), torch.float64)
    k = sig.SigPDE(sig.kernels.LinearKernel(), o)

    def run():
        return [host(k.gram(X, Y)), host(k.gram(X, Y, sx, sy)), host(k.gram(X.float(), Y.float()))]

    dual = run()
    monkeypatch.setenv("SIGK_NO_DUAL_F64", "1")
    single = run()
    monkeypatch.delenv("SIGK_NO_DUAL_F64")
    for a, b in zip(dual, single):
        assert np.all(np.isfinite(a))
        np.testing.assert_array_equal(a, b)
    assert_rel(dual[0], oracle.gram(host(X), host(Y), o), RTOL64, "dual fp64 gram vs oracle")


@pytest.mark.parametrize("Nx,Ny,L,d,o", [(9, 7, 40, 16, 1), (6, 11, 33, 24, 0), (5, 4, 70, 32, 2), (13, 1, 20, 17, 3)])
def test_pipelined_dgemm_increments_bit_identical(sig, oracle, monkeypatch, Nx, Ny, L, d, o):
    """fp64 Grams of wide paths take their increments from a float64 GEMM; the
    pipelined GEMM (A tile kept, B tiles prefetched) gives exactly the
    one-tile-per-CTA GEMM's results (Gram, scaled, symmetric)."""
    X = cuda(oracle.brownian(Nx, L, d, 800 + d), torch.float64)
    Y = cuda(oracle.brownian(Ny, L + 5, d, 900 + d), torch.float64)
    sx = cuda(np.linspace(0.7, 1.3, Nx), torch.float64)
    k = sig.SigPDE(sig.kernels.LinearKernel(), o)

    def run():
        return [host(k.gram(X, Y)), host(k.gram(X, Y, sx)), host(k.gram(X)), host(k.gram(X, None, sx))]

    pipe = run()
    monkeypatch.setenv("SIGK_NO_DGEMM_PIPE", "1")
    single = run()
    monkeypatch.delenv("SIGK_NO_DGEMM_PIPE")
    for a, b in zip(pipe, single):
        assert np.all(np.isfinite(a))
        np.testing.assert_array_equal(a, b)
    assert_rel(pipe[0], oracle.gram(host(X), host(Y), o), RTOL64, "pipelined dgemm gram vs oracle")
    assert_rel(pipe[2], oracle.gram(host(X), None, o), RTOL64, "pipelined dgemm sym gram vs oracle")


def test_static_scale_and_broadcast(sig, oracle):
    x = oracle.brownian(4, 12, 3, 11)
    y = oracle.brownian(4, 12, 3, 12)
    X, Y = cuda(x, torch.float64), cuda(y, torch.float64)
    k = sig.SigPDE(sig.kernels.LinearKernel(0.3), 1)
    assert_rel(host(k.pairwise(X, Y)), oracle.pairwise(x, y, 1, static_param=0.3), RTOL64)
    k1 = sig.SigPDE(sig.kernels.LinearKernel(), 1)
    s = cuda([1.7], torch.float64)
    assert_rel(host(k1.pairwise(X, Y, s)), oracle.pairwise(x, y, 1, np.full(4, 1.7), np.ones(4)), RTOL64)
    assert_rel(host(k1.gram(X, Y, None, s)), oracle.gram(x, y, 1, None, np.full(4, 1.7)), RTOL64)


def test_fp32_cells_error_bound(sig, oracle):
    x = oracle.brownian(16, 64, 8, 31)
    y = oracle.brownian(16, 64, 8, 32)
    X, Y = cuda(x), cuda(y)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 2, precision="fp32")
    got = host(k.gram(X, Y))
    want = oracle.gram(host(X), host(Y), 2)
    kxx = oracle.pairwise(host(X), None, 2)
    kyy = oracle.pairwise(host(Y), None, 2)
    ref = oracle.gram(host(X), host(Y), 2, store_f32=True)
    tol = fp32_tol(ref, want, kxx[:, None], kyy[None, :])
    assert_cs(got, want, kxx[:, None], kyy[None, :], tol, "fp32 gram")
    got = host(k.pairwise(X, Y))
    assert_cs(got, np.diag(want), kxx, kyy, tol, "fp32 pairwise")


# ----------------------------------------------------------------------------- robust
def test_robust_normalization_config3_shape(sig, oracle):
    """Config-3 shape (L=64, d=16, order 1, scales log-uniform in [0.5, 4]), 48 paths."""
    rng = np.random.default_rng(3)
    scales = np.exp(rng.uniform(np.log(0.5), np.log(4.0), 48))
    x = oracle.brownian(48, 64, 16, 33, scale=scales)
    X = cuda(x)
    rk = sig.RobustSigPDE(sig.kernels.LinearKernel(), 1)
    lam = host(rk.normalization(X))
    want = oracle.normalization(host(X), 1)
    np.testing.assert_allclose(lam, want, rtol=LAM_RTOL, atol=1e-9)
    assert (want > 0).sum() >= 24
    # custom normalizer (two-phase path: k on device, f on the host side, lambda on device)
    nrm = lambda s: 2 - 1 / s.pow(0.1)  # noqa: E731
    lam = host(rk.normalization(X, normalizer=nrm))
    np.testing.assert_allclose(lam, oracle.normalization(host(X), 1, nrm), rtol=LAM_RTOL, atol=1e-9)


@pytest.mark.parametrize("L,d,order", [(70, 3, 3), (130, 2, 1), (12, 40, 2), (128, 32, 1)])
def test_robust_normalization_increment_sources(sig, oracle, L, d, order, monkeypatch):
    """The shared-memory increment tile and the precomputed-difference source
    (longer paths, or SIGK_NO_NORM_TILE=1), one CTA per path with the bands as
    a warp pipeline or one warp per path (SIGK_NO_NORM_PIPE=1), with one and
    several bands of rows, against the oracle and against each other."""
    rng = np.random.default_rng(L + d)
    scales = np.exp(rng.uniform(np.log(0.5), np.log(4.0), 10))
    x = oracle.brownian(10, L, d, 61 + L, scale=scales)
    X = cuda(x, torch.float64)
    rk = sig.RobustSigPDE(sig.kernels.LinearKernel(), order)
    lam = host(rk.normalization(X))
    want = oracle.normalization(x, order)
    np.testing.assert_allclose(lam, want, rtol=LAM_RTOL, atol=1e-9)
    assert (want > 0).sum() >= 3
    monkeypatch.setenv("SIGK_NORM_PIPE", "1")  # the pipelined kernel wherever a path has >= 2 bands
    np.testing.assert_array_equal(host(rk.normalization(X)), lam)
    monkeypatch.delenv("SIGK_NORM_PIPE")
    monkeypatch.setenv("SIGK_NO_NORM_TILE", "1")
    lam_delta = host(rk.normalization(X))
    np.testing.assert_allclose(lam_delta, lam, rtol=1e-12, atol=1e-14)
    # one warp per path (all bands in sequence) instead of one CTA per path (bands as a warp pipeline):
    # the same cells from the same increments, so the same lambdas
    monkeypatch.setenv("SIGK_NO_NORM_PIPE", "1")
    lam_warp = host(rk.normalization(X))
    np.testing.assert_array_equal(lam_warp, lam_delta)
    monkeypatch.delenv("SIGK_NO_NORM_TILE")
    np.testing.assert_array_equal(host(rk.normalization(X)), lam)


@pytest.mark.parametrize("shape", [(7, 6, 40, 24, 2), (9, 9, 64, 32, 0), (5, 4, 300, 24, 1), (6, 6, 12, 16, 4),
                                   (7, 6, 40, 16, 2)])
def test_fp64_wide_paths_use_a_float64_increment_matrix(sig, oracle, shape, monkeypatch):
    """fp64 Grams with d >= 16 first write the float64 increments of all pairs with one GEMM on the
    CUDA cores and the wavefront reads them; each increment is summed in the fused kernels' order, so
    the results are bitwise those of the fused path (SIGK_NO_DGEMM_INC=1), and meet the fp64 bound.
    (A Gram of order 2-3 whose lanes hold dx in registers, like the Gram of (7, 6, 40, 16, 2), takes
    the register kernel instead; its symmetric Gram keeps the matrix.)"""
    nx, ny, L, d, o = shape
    X = cuda(oracle.brownian(nx, L, d, 71 + L), torch.float64)
    Y = cuda(oracle.brownian(ny, L + 7, d, 72 + L), torch.float64)
    s = cuda(np.linspace(0.6, 1.4, nx), torch.float64)
    k = sig.SigPDE(sig.kernels.LinearKernel(1.3), o)
    got = [host(k.gram(X, Y)), host(k.gram(X)), host(k.gram(X, None, s))]
    monkeypatch.setenv("SIGK_NO_DGEMM_INC", "1")
    fused = [host(k.gram(X, Y)), host(k.gram(X)), host(k.gram(X, None, s))]
    for a, b in zip(got, fused):
        np.testing.assert_array_equal(a, b)
    x, y = host(X) * np.sqrt(1.3), host(Y) * np.sqrt(1.3)
    assert_rel(got[0], oracle.gram(x, y, o), RTOL64, "gram")
    assert_rel(got[1], oracle.gram(x, None, o), RTOL64, "sym")


def test_robust_normalization_alternating_shared_memory_sizes(sig, oracle):
    """One kernel instance launched with large, then smaller, then large
    shared-memory tiles (the per-function opt-in must cover all of them)."""
    rk = sig.RobustSigPDE(sig.kernels.LinearKernel(), 2)
    for L in (52, 30, 52, 40, 60):
        x = oracle.brownian(4, L, 32, 70 + L, scale=np.array([0.6, 1.5, 2.5, 3.5]))
        lam = host(rk.normalization(cuda(x, torch.float64)))
        np.testing.assert_allclose(lam, oracle.normalization(x, 2), rtol=LAM_RTOL, atol=1e-9)


def test_robust_gram_and_pairwise(sig, oracle):
    rng = np.random.default_rng(4)
    scales = np.exp(rng.uniform(np.log(0.5), np.log(4.0), 6))
    x = oracle.brownian(6, 20, 4, 41, scale=scales)
    y = oracle.brownian(6, 20, 4, 42, scale=scales[::-1])
    X, Y = cuda(x, torch.float64), cuda(y, torch.float64)
    rk = sig.RobustSigPDE(sig.kernels.LinearKernel(), 1)
    np.testing.assert_allclose(host(rk.gram(X)), oracle.robust_gram(x, None, 1), rtol=1e-7)
    np.testing.assert_allclose(host(rk.gram(X, Y)), oracle.robust_gram(x, y, 1), rtol=1e-7)
    np.testing.assert_allclose(host(rk.pairwise(X, Y)), oracle.robust_pairwise(x, y, 1), rtol=1e-7)
    # explicit scales skip the normalisation (kernel.py:294-298)
    s = cuda(np.linspace(0.2, 0.9, 6), torch.float64)
    np.testing.assert_allclose(host(rk.gram(X, None, s)), oracle.gram(x, None, 1, host(s)), rtol=1e-9)


# ----------------------------------------------------------------------------- generic static kernels
@pytest.mark.parametrize("kind", ["rbf", "l1rbf"])
def test_generic_static_kernels(sig, oracle, kind):
    x = oracle.brownian(5, 9, 3, 51)
    y = oracle.brownian(5, 11, 3, 52)
    X, Y = cuda(x, torch.float64), cuda(y, torch.float64)
    sk = sig.kernels.RBFKernel(0.8) if kind == "rbf" else sig.kernels.L1RBFKernel(0.8)
    k = sig.SigPDE(sk, 1)
    assert_rel(host(k.pairwise(X, Y)), oracle.pairwise(x, y, 1, static=kind, static_param=0.8), 1e-8, "pw")
    assert_rel(host(k.gram(X, Y, max_batch=4)), oracle.gram(x, y, 1, static=kind, static_param=0.8), 1e-8, "gram")
    assert_rel(host(k.gram(X, max_batch=4)), oracle.gram(x, None, 1, static=kind, static_param=0.8), 1e-8, "sym")
    s = cuda(np.linspace(0.5, 1.5, 5), torch.float64)
    assert_rel(host(k.gram(X, None, s, max_batch=9)), oracle.gram(x, None, 1, host(s), static=kind,
                                                                    static_param=0.8), 1e-8, "sym scaled")
    rk = sig.RobustSigPDE(sk, 1)
    lam = host(rk.normalization(X * 3))
    np.testing.assert_allclose(lam, oracle.normalization(x * 3, 1, static=kind, static_param=0.8), rtol=1e-6,
                               atol=1e-9)


def test_duck_typed_linear_kernel_is_fused(sig, oracle):
    class LinearKernel:  # same name and attribute as the reference's class
        def __init__(self, scale=1.0):
            self.scale = scale

        def pairwise(self, X, Y):
            raise AssertionError("the fused path must not materialise the static Gram")

        gram = pairwise

    x = oracle.brownian(3, 10, 2, 61)
    X = cuda(x, torch.float64)
    assert_rel(host(sig.SigPDE(LinearKernel(2.0), 1).pairwise(X)), oracle.pairwise(x, None, 1, static_param=2.0))


# ----------------------------------------------------------------------------- full-size properties
def test_config2_gram_sampled_and_properties(sig, oracle):
    """Config 2: Gram 256x256, L=128, d=8, order 2, fp32 Brownian paths.

    128 sampled entries against the oracle, and size-independent properties on
    the full matrix: gram(x) equals gram(x, x), pairwise equals diag(gram)."""
    x = oracle.brownian(256, 128, 8, 2001)
    y = oracle.brownian(256, 128, 8, 2002)
    X, Y = cuda(x), cuda(y)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 2)
    G = host(k.gram(X, Y))
    rng = np.random.default_rng(0)
    flat = rng.choice(256 * 256, 128, replace=False)
    want = oracle.gram(host(X), host(Y), 2, pairs=flat)
    assert_rel(G.reshape(-1)[flat], want, RTOL_OUT32, "config2 sampled")
    P = host(k.pairwise(X, Y))
    assert_rel(P, np.diag(G), 1e-12, "pairwise vs diag(gram)")
    S = host(k.gram(X))
    Gxx = host(k.gram(X, X))
    assert_rel(S, Gxx, 1e-12, "gram(x) vs gram(x, x)")
    # float64 inputs give the float64 result itself
    G64 = host(k.gram(X.double()[:16], Y.double()[:16]))
    want = oracle.gram(host(X)[:16], host(Y)[:16], 2)
    assert_rel(G64, want, RTOL64, "config2 rows, float64 output")
    np.testing.assert_array_equal(S, S.T)


def test_long_paths_many_bands(sig, oracle):
    """Config-4 extremes: L=512 at order 3 (4088 refined rows = 8 bands)."""
    x = oracle.brownian(2, 512, 32, 71)
    y = oracle.brownian(2, 300, 32, 72)
    X, Y = cuda(x), cuda(y)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 3)
    assert_rel(host(k.pairwise(X, Y)), oracle.pairwise(host(X), host(Y), 3), RTOL_OUT32, "long")
    assert_rel(host(k.pairwise(X.double(), Y.double())), oracle.pairwise(host(X), host(Y), 3), 1e-8, "long f64")


# ----------------------------------------------------------------------------- edge cases and errors
def test_edge_cases(sig):
    k = sig.SigPDE(sig.kernels.LinearKernel(), 1)
    empty = torch.zeros((0, 5, 2), device="cuda")
    assert k.pairwise(empty).shape == (0,)
    assert k.gram(empty).shape == (0, 0)
    with pytest.raises(ValueError):
        k.pairwise(torch.zeros((2, 5, 2)))  # CPU tensor
    with pytest.raises(TypeError):
        k.pairwise(torch.zeros((2, 5, 2), device="cuda", dtype=torch.float16))
    with pytest.raises(ValueError):
        k.pairwise(torch.zeros((2, 1, 2), device="cuda"))  # one point per path
    const = torch.ones((3, 6, 2), device="cuda", dtype=torch.float64)
    y = torch.randn((3, 6, 2), device="cuda", dtype=torch.float64)
    np.testing.assert_array_equal(host(k.pairwise(const, y)), np.ones(3))


def test_non_default_stream(sig, oracle):
    x = oracle.brownian(8, 30, 4, 81)
    X = cuda(x, torch.float64)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        r = sig.SigPDE(sig.kernels.LinearKernel(), 2).gram(X)
    s.synchronize()
    assert_rel(host(r), oracle.gram(x, None, 2), RTOL64)


def test_c_abi_errors_are_reported(sig):
    from sigpde_b200 import _lib
    X = torch.zeros((2, 5, 3), device="cuda")
    out = torch.empty(2, device="cuda")
    st = _lib.lib().sigk_pairwise(X.data_ptr(), X.data_ptr(), 2, 5, 1, 3, 0, 0, 1.0, None, None, out.data_ptr(), 0,
                                  None, 0, None)
    assert st == _lib.SIGK_EINVAL and "length" in _lib.last_error()
    st = _lib.lib().sigk_pairwise(X.data_ptr(), X.data_ptr(), 2, 5, 5, 3, 7, 0, 1.0, None, None, out.data_ptr(), 0,
                                  None, 0, None)
    assert st == _lib.SIGK_EINVAL and "dtype" in _lib.last_error()
    host_buf = np.zeros(30, np.float32)
    st = _lib.lib().sigk_pairwise(host_buf.ctypes.data, X.data_ptr(), 2, 5, 5, 3, 0, 0, 1.0, None, None,
                                  out.data_ptr(), 0, None, 0, None)
    assert st == _lib.SIGK_EINVAL and "device pointer" in _lib.last_error()
