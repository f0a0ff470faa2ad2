"""The fused tensor-core Gram (fused_tc.cuh): tcgen05 increments handed from
TMEM through shared memory to the wavefront, no increment matrix in HBM.

The route is the default for tc64 Grams of order >= 2 where it applies;
SIGK_FUSED_TC=1 takes it at every order and SIGK_FUSED_TC=0 never, which is
how these tests choose the two routes.  Its arithmetic is the two-phase
path's (tc_gemm_kernel writing the float32 increment matrix, stream_inc_kernel
reading it): the same split-TF32 MMAs per increment and the same float64
cells, so the results must be bitwise equal to that path.  Against the float64
oracle the tc64 bound applies: error normalised by sqrt(k(x,x) k(y,y)) at most
1e-5.  Shapes cover every instantiated (rows per lane, order), time lines
padded to 16 columns, odd numbers of x and y paths (a last x block of fewer
than 8 paths, a last y pair of one path), fewer groups than CTAs, runs that
cross x blocks (the A operand restaged mid-run), both ring sizes (a boundary
every 16 steps, or every 8 where the operands of dimensions up to 32 need the
shared memory), scales, float64 inputs and dimensions 1..32.  Each case first checks that the fused route is the one
taken (its workspace has no increment matrix).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

CS_TC64 = 1e-5

SHAPES = [
    # (nx, ny, len_x, len_y, dim, order)
    (48, 37, 128, 128, 8, 2),   # config 2's path shape: 16 rows a lane, 4 coarse rows
    (9, 11, 40, 57, 3, 1),      # 78 rows: 4 rows a lane
    (5, 6, 20, 33, 16, 0),      # 19 rows: 2 rows a lane at order 0
    (7, 13, 100, 71, 8, 1),     # 198 rows: 8 a lane
    (6, 5, 64, 40, 5, 3),       # 504 rows at order 3: 16 a lane, 2 coarse rows
    (3, 2, 30, 18, 1, 2),       # 116 rows: 4 a lane at order 2 (1 coarse row); 1 group
    (33, 3, 17, 129, 16, 0),    # one y block of 3 paths, ncy = 128
    (4, 9, 66, 64, 8, 2),       # 260 rows: 16 a lane, 4 coarse rows (one row of padding)
    (64, 81, 40, 35, 4, 1),     # 328 groups on 148 CTAs: runs cross x blocks; last y pair of one path
    (5, 1, 40, 41, 8, 2),       # a single y path: every y pair has one path
    (1, 6, 33, 30, 2, 2),       # a single x path: 7 of the block's 8 rows are absent
    (24, 37, 128, 128, 16, 2),  # d = 16 at 4 coarse rows a lane: 8-slot ring (taken when forced)
    (9, 11, 60, 57, 32, 2),     # d = 32 at 2 coarse rows a lane: 8-slot ring
    (7, 5, 60, 50, 12, 3),      # d = 12 at order 3 (16-slot ring)
]


def _fused_taken(monkeypatch, nx, ny, lx, ly, d, o, in64):
    from sigpde_b200 import _lib
    lib = _lib.lib()
    dt = _lib.SIGK_F64 if in64 else _lib.SIGK_F32
    monkeypatch.setenv("SIGK_FUSED_TC", "1")
    fused = lib.sigk_workspace_size(_lib.SIGK_OP_GRAM, nx, ny, lx, ly, d, o, dt, _lib.SIGK_PREC_TC64)
    monkeypatch.setenv("SIGK_FUSED_TC", "0")
    two = lib.sigk_workspace_size(_lib.SIGK_OP_GRAM, nx, ny, lx, ly, d, o, dt, _lib.SIGK_PREC_TC64)
    return fused != two


def host(t):
    return t.detach().double().cpu().numpy()


@pytest.fixture(scope="module")
def sig():
    import sigpde_b200.torch as s
    return s


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("in64", [False, True])
def test_fused_equals_two_phase_and_oracle(sig, oracle, monkeypatch, shape, in64):
    nx, ny, lx, ly, d, o = shape
    assert _fused_taken(monkeypatch, nx, ny, lx, ly, d, o, in64)
    dt = torch.float64 if in64 else torch.float32
    X = torch.tensor(oracle.brownian(nx, lx, d, 1000 + lx), dtype=dt, device="cuda")
    Y = torch.tensor(oracle.brownian(ny, ly, d, 2000 + ly), dtype=dt, device="cuda")
    sx = torch.linspace(0.6, 1.4, nx, dtype=dt, device="cuda")
    k = sig.SigPDE(sig.kernels.LinearKernel(0.8), o, precision="tc64")
    for scales in ((None, None), (sx, None)):
        monkeypatch.setenv("SIGK_FUSED_TC", "1")
        fused = k.gram(X, Y, *scales)
        monkeypatch.setenv("SIGK_FUSED_TC", "0")
        two = k.gram(X, Y, *scales)
        torch.cuda.synchronize()
        assert torch.equal(fused, two), f"{shape} in64={in64} scaled={scales[0] is not None}"
    monkeypatch.setenv("SIGK_FUSED_TC", "1")
    G = host(k.gram(X, Y))
    monkeypatch.delenv("SIGK_FUSED_TC", raising=False)
    x, y = host(X), host(Y)
    want = oracle.gram(x, y, o, static_param=0.8)
    kxx = oracle.pairwise(x, None, o, static_param=0.8)[:, None]
    kyy = oracle.pairwise(y, None, o, static_param=0.8)[None, :]
    assert float(np.max(np.abs(G - want) / np.sqrt(kxx * kyy))) <= CS_TC64


def test_fused_route_is_taken_and_small(sig):
    """By default a tc64 Gram at order 2 takes the fused route, whose workspace
    holds only the operand images (no increment matrix): 256 x 256 paths of
    length 128 in 8 dims need ~4 MB, against 4.26 GB for the two-phase matrix."""
    import os
    from sigpde_b200 import _lib
    lib = _lib.lib()
    os.environ.pop("SIGK_FUSED_TC", None)
    default = lib.sigk_workspace_size(_lib.SIGK_OP_GRAM, 256, 256, 128, 128, 8, 2, _lib.SIGK_F32,
                                      _lib.SIGK_PREC_TC64)
    os.environ["SIGK_FUSED_TC"] = "0"
    try:
        two = lib.sigk_workspace_size(_lib.SIGK_OP_GRAM, 256, 256, 128, 128, 8, 2, _lib.SIGK_F32,
                                      _lib.SIGK_PREC_TC64)
    finally:
        os.environ.pop("SIGK_FUSED_TC", None)
    assert default < 8 << 20 < (1 << 30) < two


def test_fused_config2_size(sig, oracle, monkeypatch):
    """The full 256 x 256 Gram at L = 128, d = 8, order 2 (28 groups per CTA,
    each run crossing an x block): bitwise the two-phase result, and 16 sampled
    entries within the tc64 bound of the float64 oracle."""
    X = torch.tensor(oracle.brownian(256, 128, 8, 1), dtype=torch.float32, device="cuda")
    Y = torch.tensor(oracle.brownian(256, 128, 8, 2), dtype=torch.float32, device="cuda")
    assert _fused_taken(monkeypatch, 256, 256, 128, 128, 8, 2, False)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 2, precision="tc64")
    monkeypatch.setenv("SIGK_FUSED_TC", "1")
    fused = k.gram(X, Y)
    monkeypatch.setenv("SIGK_FUSED_TC", "0")
    two = k.gram(X, Y)
    torch.cuda.synchronize()
    assert torch.equal(fused, two)
    G = host(fused)
    x, y = host(X), host(Y)
    rng = np.random.default_rng(3)
    flat = rng.choice(256 * 256, 16, replace=False)
    want = oracle.gram(x, y, 2, pairs=flat)
    i, j = flat // 256, flat % 256
    kxx = oracle.pairwise(x[i], None, 2)
    kyy = oracle.pairwise(y[j], None, 2)
    assert float(np.max(np.abs(G.reshape(-1)[flat] - want) / np.sqrt(kxx * kyy))) <= CS_TC64


def test_fused_random_shapes_bitwise(sig, oracle, monkeypatch):
    """40 seeded random Gram shapes (paths 1..40, lengths 5..130, dimensions
    1..32, orders 0..3): wherever the fused route is eligible (forced with
    SIGK_FUSED_TC=1) its results equal the two-phase route's bitwise."""
    from sigpde_b200 import _lib
    rng = np.random.default_rng(2024)
    taken = 0
    for _ in range(40):
        nx, ny = int(rng.integers(1, 41)), int(rng.integers(1, 41))
        lx, ly = int(rng.integers(5, 131)), int(rng.integers(5, 131))
        d, o = int(rng.integers(1, 33)), int(rng.integers(0, 4))
        if not _fused_taken(monkeypatch, nx, ny, lx, ly, d, o, False):
            continue
        taken += 1
        X = torch.tensor(oracle.brownian(nx, lx, d, int(rng.integers(1 << 30))), dtype=torch.float32, device="cuda")
        Y = torch.tensor(oracle.brownian(ny, ly, d, int(rng.integers(1 << 30))), dtype=torch.float32, device="cuda")
        k = sig.SigPDE(sig.kernels.LinearKernel(), o, precision="tc64")
        monkeypatch.setenv("SIGK_FUSED_TC", "1")
        fused = k.gram(X, Y)
        monkeypatch.setenv("SIGK_FUSED_TC", "0")
        two = k.gram(X, Y)
        monkeypatch.delenv("SIGK_FUSED_TC", raising=False)
        torch.cuda.synchronize()
        assert torch.equal(fused, two), (nx, ny, lx, ly, d, o)
        assert bool(torch.all(torch.isfinite(fused)))
    assert taken >= 10, f"only {taken} of 40 random shapes were eligible"
