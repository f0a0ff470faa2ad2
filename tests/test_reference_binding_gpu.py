"""The reference-side binding of INTEGRATION.md, run for real.

The unmodified stojl/SigPDE package (installed under baseline/_ref) keeps its
own sigpde/torch/kernel.py -- increments built with torch, tile loops,
cuda.synchronize() -- while its three solver classes
(sigpde/PDESolvers.py:37-245) are swapped for the ctypes stubs below, which
call libsigk's generic-increment entry points.  The reference's SigPDE.pairwise
/ gram / symmetric gram (plain and scaled) and RobustSigPDE.normalization /
gram then run through libsigk and are compared with the float64 oracle:
float64 inputs, so the bound is 1e-9 relative for kernel values and 1e-6 for
the robust lambdas.  Skipped when the reference or numba is not installed.
"""
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "baseline", "_ref")

# ---------------------------------------------------------------- the stubs
from sigpde_b200 import _lib  # noqa: E402  (argtypes of every entry point are set there)

F32, F64, PREC_FP64 = 0, 1, 0
OP_PAIRWISE, OP_GRAM, OP_NORMALIZE = 0, 1, 3


def _dt(t):
    return F64 if t.dtype == torch.float64 else F32


def _ws(op, nx, ny, ncx, ncy, order, dt):
    n = _lib.lib().sigk_workspace_size(op, nx, ny, ncx + 1, ncy + 1, 0, order, dt, PREC_FP64)
    return (torch.empty(n, dtype=torch.uint8, device="cuda"), n) if n else (None, 0)


def _p(t):
    return None if t is None else t.data_ptr()


def _st():
    return torch.cuda.current_stream().cuda_stream


def _ok(status):
    assert status == 0, _lib.last_error()


class PairwisePDESolver:  # sigpde/PDESolvers.py:37-135
    def __init__(self, batch_size, x_length, y_length, dtype=None, dyadic_order=0, max_batch=1000,
                 max_threads=1024):
        self.order = dyadic_order
        self.batch_size = batch_size
        self.max_batch = min(max_batch, batch_size)

    def solve(self, inc, result, sx=None, sy=None):
        B, ncx, ncy = inc.shape
        ws, n = _ws(OP_PAIRWISE, B, B, ncx, ncy, self.order, _dt(inc))
        _ok(_lib.lib().sigk_pairwise_inc(_p(inc), B, ncx, ncy, *inc.stride(), _dt(inc), self.order, _p(sx), _p(sy),
                                         _p(result), PREC_FP64, _p(ws), n, _st()))

    def solve_scaled(self, inc, sx, sy, result):
        self.solve(inc, result, sx, sy)

    def solve_norms(self, inc, fk, k, result, tol=1e-8, maxit=100):
        # the reference passes f(k) as `norms` and k as `f_norms` (sigpde/torch/kernel.py:186-193)
        B, nc, _ = inc.shape
        ws, n = _ws(OP_NORMALIZE, B, B, nc, nc, self.order, _dt(inc))
        k64, fk64 = k.double().contiguous(), fk.double().contiguous()
        _ok(_lib.lib().sigk_normalize_inc(_p(inc), B, nc, *inc.stride(), _dt(inc), self.order, _p(k64), _p(fk64),
                                          float(tol), int(maxit), _p(result), None, _p(ws), n, _st()))


class GramPDESolver:  # sigpde/PDESolvers.py:137-190
    def __init__(self, x_batch_size, y_batch_size, x_length, y_length, dtype=None, dyadic_order=0, max_batch=1000,
                 max_threads=1024):
        self.order = dyadic_order
        self.batch_size_x, self.batch_size_y = x_batch_size, y_batch_size
        self.max_batch_x, self.max_batch_y = min(max_batch, x_batch_size), min(max_batch, y_batch_size)

    def solve(self, inc, result, sx=None, sy=None):
        # the tile's values go to result[0:nx, 0:ny]; the caller copies them out (kernel.py:100-122)
        nx, ny, ncx, ncy = inc.shape
        ws, n = _ws(OP_GRAM, nx, ny, ncx, ncy, self.order, _dt(inc))
        _ok(_lib.lib().sigk_gram_inc(_p(inc), nx, ny, ncx, ncy, *inc.stride(), _dt(inc), self.order, _p(sx), _p(sy),
                                     0, _p(result), result.stride(0), PREC_FP64, _p(ws), n, _st()))

    def solve_scaled(self, inc, sx, sy, result):
        self.solve(inc, result, sx, sy)


class SymmetricGramPDESolver:  # sigpde/PDESolvers.py:192-245
    def __init__(self, batch_size, length, dtype=None, dyadic_order=0, max_batch=1000, max_threads=1024):
        self.order = dyadic_order
        self.batch_size = batch_size
        self.max_batch = min(max_batch, batch_size)

    def solve(self, inc, x_offset, y_offset, result, sx=None, sy=None):
        # as the reference's kernel (cuda_gram_kernels.py:79-120): tiles above the diagonal are skipped,
        # the diagonal tile is solved on its lower triangle and mirrored, a tile below the diagonal is
        # solved whole and written at both (i, j) and (j, i)
        if x_offset < y_offset:
            return
        nx, ny, ncx, ncy = inc.shape
        out = result[x_offset:x_offset + nx, y_offset:y_offset + ny]
        sym = int(x_offset == y_offset)
        ws, n = _ws(OP_GRAM, nx, ny, ncx, ncy, self.order, _dt(inc))
        _ok(_lib.lib().sigk_gram_inc(_p(inc), nx, ny, ncx, ncy, *inc.stride(), _dt(inc), self.order, _p(sx), _p(sy),
                                     sym, _p(out), result.stride(0), PREC_FP64, _p(ws), n, _st()))
        if not sym:
            result[y_offset:y_offset + ny, x_offset:x_offset + nx] = out.t()

    def solve_scaled(self, inc, sx, sy, x_offset, y_offset, result):
        self.solve(inc, x_offset, y_offset, result, sx, sy)


# ---------------------------------------------------------------- the reference with the stubs swapped in
@pytest.fixture(scope="module")
def refsig():
    if not os.path.isdir(os.path.join(REF, "sigpde")):
        pytest.skip("the reference is not installed under baseline/_ref")
    sys.path.insert(0, REF)
    try:
        import warnings
        warnings.filterwarnings("ignore")
        import sigpde.torch as rs
        import sigpde.torch.kernel as rk
    except Exception as e:  # numba missing or without a CUDA target
        pytest.skip(f"the reference does not import: {type(e).__name__}: {e}")
    saved = (rk.PairwisePDESolver, rk.GramPDESolver, rk.SymmetricGramPDESolver)
    rk.PairwisePDESolver, rk.GramPDESolver, rk.SymmetricGramPDESolver = (PairwisePDESolver, GramPDESolver,
                                                                         SymmetricGramPDESolver)
    yield rs
    rk.PairwisePDESolver, rk.GramPDESolver, rk.SymmetricGramPDESolver = saved


def cuda64(a):
    return torch.tensor(a, dtype=torch.float64, device="cuda")


def rel(got, want):
    return float(np.max(np.abs(got - want) / np.abs(want)))


def test_reference_pairwise_and_gram_through_the_stubs(refsig, oracle):
    x = oracle.brownian(40, 20, 5, 901)
    y = oracle.brownian(37, 23, 5, 902)
    k = refsig.SigPDE(refsig.kernels.LinearKernel(), 1)
    X, Y = cuda64(x), cuda64(y)
    P = k.pairwise(X[:37], Y).cpu().numpy()
    assert rel(P, oracle.pairwise(x[:37], y, 1)) <= 1e-9
    G = k.gram(X, Y).cpu().numpy()  # 32-path tiles: 2 x 2
    assert rel(G, oracle.gram(x, y, 1)) <= 1e-9
    S = k.gram(X).cpu().numpy()  # symmetric: tiles below, on and above the diagonal
    np.testing.assert_array_equal(S, S.T)
    assert rel(S, oracle.gram(x, None, 1)) <= 1e-9
    sx = np.exp(np.random.default_rng(1).uniform(-0.5, 0.5, 40))
    sy = np.exp(np.random.default_rng(2).uniform(-0.5, 0.5, 37))
    Gs = k.gram(X, Y, cuda64(sx), cuda64(sy)).cpu().numpy()
    assert rel(Gs, oracle.gram(x, y, 1, sx, sy)) <= 1e-9
    Ss = k.gram(X, None, cuda64(sx)).cpu().numpy()
    assert rel(Ss, oracle.gram(x, None, 1, sx)) <= 1e-9


def test_reference_robust_through_the_stubs(refsig, oracle):
    rng = np.random.default_rng(3)
    x = oracle.brownian(36, 30, 6, 903, scale=np.exp(rng.uniform(np.log(0.5), np.log(4.0), 36)))
    rk = refsig.RobustSigPDE(refsig.kernels.LinearKernel(), 1)
    X = cuda64(x)
    lam = rk.normalization(X).cpu().numpy()
    want = oracle.normalization(x, 1)
    assert (want > 0).sum() >= 8
    np.testing.assert_allclose(lam, want, rtol=1e-6, atol=1e-9)
    G = rk.gram(X).cpu().numpy()
    assert rel(G, oracle.gram(x, None, 1, lam)) <= 1e-9
