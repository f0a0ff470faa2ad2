"""Backward pass (sigk_backward, autograd through sigpde_b200.torch) against
the oracle's gradients, which are pinned by central differences of the
oracle's solve (tests/test_oracle_grad.py).

Tolerance: float64 paths, max |got - want| <= 1e-9 * max |want| (the adjoint
runs in float64 with the same increments as the forward; only summation
order differs); float32 paths return float32 gradients: 2e-6 relative to
max |want|.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL64 = 1e-9
TOL32 = 2e-6


def cuda(a, dtype=torch.float64, grad=False):
    t = torch.as_tensor(np.asarray(a), dtype=dtype, device="cuda")
    return t.requires_grad_(grad)


def host(t):
    return t.detach().double().cpu().numpy()


def close(got, want, tol, msg=""):
    err = np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300)
    assert err <= tol, f"{msg}: error {err:.3e} relative to max |grad| > {tol:.1e}"


@pytest.fixture(scope="module")
def sig():
    import sigpde_b200.torch as sig
    return sig


@pytest.mark.parametrize("shape", [
    # (batch, L_x, L_y, d, order)
    (5, 9, 11, 3, 0),
    (4, 20, 17, 4, 1),
    (3, 33, 40, 2, 2),
    (3, 12, 9, 5, 3),
    (2, 8, 10, 3, 4),
    (2, 70, 30, 2, 3),   # 552 refined rows: two bands of 512
    (6, 2, 3, 1, 0),     # one coarse row
])
def test_pairwise_gradients(sig, oracle, shape):
    B, lx, ly, d, o = shape
    x = oracle.brownian(B, lx, d, 1 + lx)
    y = oracle.brownian(B, ly, d, 2 + ly)
    w = np.linspace(-1.0, 1.5, B)
    X, Y = cuda(x, grad=True), cuda(y, grad=True)
    k = sig.SigPDE(sig.kernels.LinearKernel(0.8), o)
    out = k.pairwise(X, Y)
    np.testing.assert_allclose(host(out), oracle.pairwise(x, y, o, static_param=0.8), rtol=1e-9)
    out.backward(cuda(w))
    gx, gy = oracle.grad_pairwise(x, y, o, w, static_scale=0.8)
    close(host(X.grad), gx, TOL64, "grad x")
    close(host(Y.grad), gy, TOL64, "grad y")


@pytest.mark.parametrize("shape", [(4, 3, 15, 13, 3, 1), (3, 5, 40, 33, 8, 2), (6, 2, 7, 70, 2, 0)])
def test_gram_gradients_with_scales(sig, oracle, shape):
    nx, ny, lx, ly, d, o = shape
    x = oracle.brownian(nx, lx, d, 10 + lx)
    y = oracle.brownian(ny, ly, d, 20 + ly)
    sx = np.linspace(0.6, 1.4, nx)
    sy = np.linspace(1.2, 0.7, ny)
    w = np.random.default_rng(5).standard_normal((nx, ny))
    X, Y = cuda(x, grad=True), cuda(y, grad=True)
    k = sig.SigPDE(sig.kernels.LinearKernel(), o)
    G = k.gram(X, Y, cuda(sx), cuda(sy))
    (G * cuda(w)).sum().backward()
    gx, gy = oracle.grad_gram(x, y, o, w, sx, sy)
    close(host(X.grad), gx, TOL64, "grad x")
    close(host(Y.grad), gy, TOL64, "grad y")


def test_symmetric_gram_and_self_pairwise_gradients(sig, oracle):
    x = oracle.brownian(5, 24, 3, 31)
    w = np.random.default_rng(6).standard_normal((5, 5))
    X = cuda(x, grad=True)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 2)
    (k.gram(X) * cuda(w)).sum().backward()
    close(host(X.grad), oracle.grad_gram(x, None, 2, w), TOL64, "symmetric gram")
    X2 = cuda(x, grad=True)
    wp = np.linspace(0.5, 2.0, 5)
    (k.pairwise(X2) * cuda(wp)).sum().backward()
    gx, gy = oracle.grad_pairwise(x, x, 2, wp)
    close(host(X2.grad), gx + gy, TOL64, "pairwise(x)")


def test_float32_paths_and_one_sided_gradients(sig, oracle):
    x = oracle.brownian(4, 18, 3, 41)
    y = oracle.brownian(3, 21, 3, 42)
    X = cuda(x, torch.float32, grad=True)
    Y = cuda(y, torch.float32)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 1)
    G = k.gram(X, Y)
    assert G.requires_grad and G.dtype == torch.float32
    G.sum().backward()
    assert X.grad.dtype == torch.float32 and Y.grad is None
    gx, _ = oracle.grad_gram(host(X), host(Y), 1, np.ones((4, 3)))
    close(host(X.grad), gx, TOL32, "float32 grad x")


def test_chunked_backward_matches(sig, oracle, monkeypatch):
    """Chunks of x paths (a 1 MB cap) give the same gradients up to summation order."""
    x = oracle.brownian(9, 30, 3, 51)
    y = oracle.brownian(7, 26, 3, 52)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 2)
    w = cuda(np.random.default_rng(7).standard_normal((9, 7)))

    def grads():
        X, Y = cuda(x, grad=True), cuda(y, grad=True)
        (k.gram(X, Y) * w).sum().backward()
        return host(X.grad), host(Y.grad)

    a = grads()
    monkeypatch.setenv("SIGK_GRAD_CHUNK_MB", "1")
    b = grads()
    for u, v in zip(a, b):
        close(v, u, 1e-13, "chunked")


def test_gradcheck_small(sig):
    """torch.autograd.gradcheck: the backward against finite differences of the forward."""
    rng = np.random.default_rng(8)
    x = cuda(rng.standard_normal((2, 5, 2)) * 0.4, grad=True)
    y = cuda(rng.standard_normal((3, 4, 2)) * 0.4, grad=True)
    k = sig.SigPDE(sig.kernels.LinearKernel(), 1)
    assert torch.autograd.gradcheck(lambda a, b: k.gram(a, b), (x, y), eps=1e-6, atol=1e-7, rtol=1e-6)
    assert torch.autograd.gradcheck(lambda a, b: k.pairwise(a, b[:2]), (x, y), eps=1e-6, atol=1e-7, rtol=1e-6)


@pytest.mark.parametrize("kind", ["rbf", "l1rbf"])
def test_static_kernel_gradients(sig, oracle, kind):
    """RBF / L1-RBF: autograd through the torch static Gram of the increment route and
    sigk_backward_inc, against the oracle's adjoint and chain rule."""
    x = oracle.brownian(5, 14, 3, 61)
    y = oracle.brownian(4, 17, 3, 62) + 0.05
    sk = sig.kernels.RBFKernel(0.9) if kind == "rbf" else sig.kernels.L1RBFKernel(0.9)
    k = sig.SigPDE(sk, 2)
    w = np.random.default_rng(9).standard_normal((5, 4))
    X, Y = cuda(x, grad=True), cuda(y, grad=True)
    G = k.gram(X, Y, max_batch=9)  # 3 x 3 path tiles, as the reference tiles
    np.testing.assert_allclose(host(G), oracle.gram(x, y, 2, static=kind, static_param=0.9), rtol=1e-9)
    (G * cuda(w)).sum().backward()
    gx, gy = oracle.grad_static_gram(kind, x, y, 2, w, 0.9)
    close(host(X.grad), gx, TOL64, "grad x")
    close(host(Y.grad), gy, TOL64, "grad y")
    # pairwise with scales, and the symmetric Gram
    X2, Y2 = cuda(x[:4], grad=True), cuda(y, grad=True)
    sx, sy = np.linspace(0.7, 1.2, 4), np.linspace(1.1, 0.8, 4)
    wp = np.array([1.0, -2.0, 0.5, 0.25])
    (k.pairwise(X2, Y2, cuda(sx), cuda(sy)) * cuda(wp)).sum().backward()
    gx, gy = oracle.grad_static_pairs(kind, x[:4], y, 2, wp, 0.9, sx, sy)
    close(host(X2.grad), gx, TOL64, "pairwise grad x")
    close(host(Y2.grad), gy, TOL64, "pairwise grad y")
    xs = x + np.linspace(0, 0.2, 5)[:, None, None]
    X3 = cuda(xs, grad=True)
    ws = np.random.default_rng(10).standard_normal((5, 5))
    (k.gram(X3, max_batch=4) * cuda(ws)).sum().backward()
    close(host(X3.grad), oracle.grad_static_gram(kind, xs, None, 2, ws, 0.9), TOL64, "symmetric")


def test_duck_typed_kernel_gradcheck(sig):
    """Any object with the static-kernel protocol is differentiable through the
    increment route: gradcheck on a polynomial kernel (1 + <x, y>)^2."""
    class PolyKernel:
        def pairwise(self, X, Y):
            return (1 + torch.bmm(X, Y.transpose(1, 2))) ** 2

        def gram(self, X, Y):
            return (1 + torch.einsum("ipk,jqk->ijpq", X, Y)) ** 2

    rng = np.random.default_rng(11)
    x = cuda(rng.standard_normal((2, 4, 2)) * 0.3, grad=True)
    y = cuda(rng.standard_normal((3, 5, 2)) * 0.3, grad=True)
    k = sig.SigPDE(PolyKernel(), 1)
    assert torch.autograd.gradcheck(lambda a, b: k.gram(a, b), (x, y), eps=1e-6, atol=1e-7, rtol=1e-6)
    assert torch.autograd.gradcheck(lambda a, b: k.pairwise(a, b[:2, :4]), (x, y), eps=1e-6, atol=1e-7, rtol=1e-6)


def _fd(f, arr, h=1e-6):
    g = np.zeros_like(arr)
    for idx in np.ndindex(arr.shape):
        a = arr.copy()
        a[idx] += h
        fp = f(a)
        a[idx] -= 2 * h
        g[idx] = (fp - f(a)) / (2 * h)
    return g


def test_scale_gradients(sig, oracle):
    """Gradients with respect to the per-path scales (linear: through the scaled
    paths; RBF: through the scaled increments), against central differences."""
    x = oracle.brownian(3, 9, 2, 71)
    y = oracle.brownian(2, 8, 2, 72) + 0.05
    sx, sy = np.array([0.7, 1.1, 0.9]), np.array([1.3, 0.6])
    w = np.array([[1.0, -0.5], [0.3, 2.0], [-1.2, 0.4]])
    for kind, sk in (("linear", sig.kernels.LinearKernel()), ("rbf", sig.kernels.RBFKernel(1.3))):
        k = sig.SigPDE(sk, 1)
        X, Y = cuda(x, grad=True), cuda(y, grad=True)
        SX, SY = cuda(sx, grad=True), cuda(sy, grad=True)
        (k.gram(X, Y, SX, SY) * cuda(w)).sum().backward()
        param = 1.0 if kind == "linear" else 1.3

        def f(ax=sx, ay=sy, xx=x):
            return float(np.sum(w * oracle.gram(xx, y, 1, ax, ay, static=kind, static_param=param)))

        close(host(SX.grad), _fd(lambda a: f(ax=a), sx), 1e-6, f"{kind} d/d scale_x")
        close(host(SY.grad), _fd(lambda a: f(ay=a), sy), 1e-6, f"{kind} d/d scale_y")
        close(host(X.grad), _fd(lambda a: f(xx=a), x), 1e-6, f"{kind} d/dx with scales")


@pytest.mark.parametrize("kind", ["linear", "rbf"])
def test_robust_gradients(sig, oracle, kind):
    """RobustSigPDE is differentiable through lambda(x) (implicit function theorem),
    against central differences of the oracle's robust kernel (tight root tolerance)."""
    x = oracle.brownian(3, 8, 2, 81) * 3.0
    y = oracle.brownian(2, 9, 2, 82) * 2.5 + 0.05
    sk = sig.kernels.LinearKernel() if kind == "linear" else sig.kernels.RBFKernel(0.5)
    param = 1.0 if kind == "linear" else 0.5
    rk = sig.RobustSigPDE(sk, 1)
    tol, maxit = 1e-13, 200
    lam = oracle.normalization(x, 1, None, tol, maxit, static=kind, static_param=param)
    assert np.all(lam > 0) and np.all(lam < 1), lam  # the normalisation is active on every path
    w = np.array([[1.0, -0.5], [0.3, 2.0], [-1.2, 0.4]])
    X, Y = cuda(x, grad=True), cuda(y, grad=True)
    (rk.gram(X, Y, tol=tol, maxit=maxit) * cuda(w)).sum().backward()

    def f(xx, yy):
        lx = oracle.normalization(xx, 1, None, tol, maxit, static=kind, static_param=param)
        ly = oracle.normalization(yy, 1, None, tol, maxit, static=kind, static_param=param)
        return float(np.sum(w * oracle.gram(xx, yy, 1, lx, ly, static=kind, static_param=param)))

    close(host(X.grad), _fd(lambda a: f(a, y), x), 1e-5, "robust gram d/dx")
    close(host(Y.grad), _fd(lambda a: f(x, a), y), 1e-5, "robust gram d/dy")
    X2 = cuda(x, grad=True)
    wp = np.array([0.5, -1.0, 2.0])
    (rk.pairwise(X2, tol=tol, maxit=maxit) * cuda(wp)).sum().backward()

    def fp(xx):
        lx = oracle.normalization(xx, 1, None, tol, maxit, static=kind, static_param=param)
        return float(np.dot(wp, oracle.pairwise(xx, None, 1, lx, lx, static=kind, static_param=param)))

    close(host(X2.grad), _fd(fp, x), 1e-5, "robust pairwise(x) d/dx")


def test_backward_refusals(sig):
    x = cuda(np.zeros((2, 5, 2)), grad=True)
    from sigpde_b200._lib import SigkError
    with pytest.raises(SigkError, match="order <= 4"):
        sig.SigPDE(sig.kernels.LinearKernel(), 5).gram(x, x).sum().backward()
    # robust Gram with fixed scales is differentiable in the paths
    g = sig.RobustSigPDE(sig.kernels.LinearKernel(), 1).gram(x, None, cuda([0.5, 0.9]))
    g.sum().backward()
    assert x.grad is not None
