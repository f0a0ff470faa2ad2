"""The oracle's gradients (adjoint of the float64 scheme, oracle/sigk_oracle.c
sko_grad_solve, with the chain rule through the LinearKernel increments in
oracle/oracle.py) against central differences of the oracle's own solve.  The
reference has no backward pass, so the gradient oracle is pinned by the
pinned forward oracle: bound 1e-7 absolute on gradients of size ~1-20 (the
central differences with h = 1e-5 carry ~1e-9)."""
import numpy as np
import pytest


def _fd(f, arr, h=1e-5):
    g = np.zeros_like(arr)
    for idx in np.ndindex(arr.shape):
        a = arr.copy()
        a[idx] += h
        fp = f(a)
        a[idx] -= 2 * h
        g[idx] = (fp - f(a)) / (2 * h)
    return g


@pytest.mark.parametrize("order", [0, 1, 2, 3])
def test_pairwise_gradient_matches_central_differences(oracle, order):
    x = oracle.brownian(2, 6, 3, 11)
    y = oracle.brownian(2, 7, 3, 12)
    w = np.array([0.7, -1.3])
    sx, sy = np.array([0.8, 1.2]), np.array([1.1, 0.6])
    gx, gy = oracle.grad_pairwise(x, y, order, w, sx, sy, 1.3)

    def f(xx, yy):
        return float(np.dot(w, oracle.pairwise(xx, yy, order, sx, sy, static_param=1.3)))

    np.testing.assert_allclose(gx, _fd(lambda a: f(a, y), x), atol=1e-7)
    np.testing.assert_allclose(gy, _fd(lambda a: f(x, a), y), atol=1e-7)


def test_gram_and_symmetric_gram_gradients(oracle):
    x = oracle.brownian(3, 5, 2, 21)
    y = oracle.brownian(2, 6, 2, 22)
    w = np.array([[0.5, -1.0], [2.0, 0.3], [-0.7, 1.1]])
    gx, gy = oracle.grad_gram(x, y, 1, w)

    def f(xx, yy):
        return float(np.sum(w * oracle.gram(xx, yy, 1)))

    np.testing.assert_allclose(gx, _fd(lambda a: f(a, y), x), atol=1e-7)
    np.testing.assert_allclose(gy, _fd(lambda a: f(x, a), y), atol=1e-7)
    ws = np.arange(9.0).reshape(3, 3) / 9 - 0.3
    g = oracle.grad_gram(x, None, 2, ws, np.array([0.9, 1.1, 1.4]))
    np.testing.assert_allclose(g, _fd(lambda a: float(np.sum(ws * oracle.gram(a, None, 2, np.array([0.9, 1.1, 1.4])))),
                                      x), atol=1e-7)


def test_grad_of_increments_is_linear_in_the_weight(oracle):
    inc = np.random.default_rng(3).standard_normal((4, 5)) * 0.2
    g1, k1 = oracle.grad_increments(inc, 2, None, np.array([1.0]))
    g2, k2 = oracle.grad_increments(inc, 2, None, np.array([-2.5]))
    np.testing.assert_allclose(g2, -2.5 * g1, rtol=1e-14)
    assert k1[0] == k2[0] == oracle.solve_increments(inc, 2)[0]


@pytest.mark.parametrize("kind", ["rbf", "l1rbf"])
def test_static_kernel_gradients(oracle, kind):
    """RBF / L1-RBF: the adjoint plus the chain rule through the static Gram and its
    second difference, against central differences."""
    x = oracle.brownian(2, 5, 2, 31)
    y = oracle.brownian(2, 6, 2, 32) + 0.05  # no coincident coordinates: |.| has a kink at 0
    w = np.array([1.2, -0.4])
    gx, gy = oracle.grad_static_pairs(kind, x, y, 1, w, 0.9, np.array([0.8, 1.1]), np.array([1.3, 0.7]))

    def f(xx, yy):
        return float(np.dot(w, oracle.pairwise(xx, yy, 1, np.array([0.8, 1.1]), np.array([1.3, 0.7]),
                                               static=kind, static_param=0.9)))

    np.testing.assert_allclose(gx, _fd(lambda a: f(a, y), x), atol=1e-7)
    np.testing.assert_allclose(gy, _fd(lambda a: f(x, a), y), atol=1e-7)
    x = x + np.array([0.0, 0.03])[:, None, None]  # the two paths start apart
    g = oracle.grad_static_gram(kind, x, None, 2, np.array([[1.0, 0.5], [-0.3, 2.0]]), 1.1)
    fd = _fd(lambda a: float(np.sum(np.array([[1.0, 0.5], [-0.3, 2.0]]) *
                                    oracle.gram(a, None, 2, static=kind, static_param=1.1))), x)
    np.testing.assert_allclose(g, fd, atol=1e-7)
