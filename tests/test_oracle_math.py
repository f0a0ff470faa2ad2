"""Known answers from the mathematics of the signature-kernel PDE, and the C
oracle against the pure-Python anti-diagonal restatement (CPU only)."""
import math

import numpy as np


def test_c_solver_equals_python_antidiagonal_loop(oracle):
    rng = np.random.default_rng(5)
    for (ncx, ncy, o) in ((1, 1, 0), (3, 5, 0), (4, 3, 1), (2, 3, 2), (3, 2, 3)):
        inc = rng.normal(scale=0.3, size=(ncx, ncy))
        a = oracle.solve_increments(inc[None], o)[0]
        b = oracle.py_solve(inc, o)
        assert a == b, (ncx, ncy, o, a, b)
        a = oracle.solve_increments(inc[None], o, sx=[1.7], sy=[0.6])[0]
        b = oracle.py_solve(inc, o, 1.7 * 0.6)
        assert abs(a - b) <= 1e-15 * abs(b), (a, b)


def test_constant_path_has_kernel_one(oracle):
    x = np.ones((2, 7, 3))
    y = np.random.default_rng(1).normal(size=(2, 9, 3))
    np.testing.assert_array_equal(oracle.pairwise(x, y, 2), np.ones(2))


def test_symmetry_and_translation_invariance(oracle):
    x = oracle.brownian(3, 11, 4, 7)
    y = oracle.brownian(3, 13, 4, 8)
    a = oracle.pairwise(x, y, 1)
    b = oracle.pairwise(y, x, 1)
    np.testing.assert_allclose(a, b, rtol=1e-12)
    np.testing.assert_allclose(oracle.pairwise(x + 3.0, y - 1.5, 1), a, rtol=1e-11)


def test_scale_equals_prescaled_path(oracle):
    x = oracle.brownian(3, 9, 3, 3)
    y = oracle.brownian(3, 9, 3, 4)
    s = np.array([0.5, 1.3, 2.2])
    np.testing.assert_allclose(oracle.pairwise(x, y, 1, s, None), oracle.pairwise(x * s[:, None, None], y, 1),
                               rtol=1e-11)


def test_gram_consistency(oracle):
    x = oracle.brownian(4, 8, 3, 9)
    g = oracle.gram(x, x, 1)
    gs = oracle.gram(x, None, 1)
    np.testing.assert_allclose(gs, g, rtol=1e-11)
    np.testing.assert_allclose(np.diag(g), oracle.pairwise(x, None, 1), rtol=1e-12)


def test_single_segment_converges_to_bessel(oracle):
    """L=2: k -> sum_n c^n/(n!)^2 = I0(2 sqrt(c)) as the dyadic order grows."""
    c = 0.8
    x = np.array([[[0.0, 0.0], [1.0, 0.0]]])
    y = np.array([[[0.0, 0.0], [c, 0.0]]])
    exact = sum(c ** n / math.factorial(n) ** 2 for n in range(30))
    errs = [abs(oracle.pairwise(x, y, o)[0] - exact) for o in range(3, 9)]
    assert errs[-1] < 2e-7 * exact
    # second-order scheme: once in the asymptotic range each refinement divides the error by about 4
    assert all(3.3 < e1 / e2 < 4.5 for e1, e2 in zip(errs, errs[1:]))


def test_robust_lambda_solves_its_equation(oracle):
    x = oracle.brownian(4, 12, 3, 21, scale=[0.7, 1.5, 2.5, 3.5])
    lam, k, fk, it = oracle.normalization(x, 1, return_iters=True)
    for b in range(4):
        if k[b] < 1:
            assert lam[b] == 0
            continue
        kl = oracle.pairwise(x[b:b + 1] * lam[b], None, 1)[0]
        assert abs(kl - fk[b]) < 1e-7, (b, kl, fk[b])
        assert it[b] < 100


def test_generic_static_kernels_match_linear_definition(oracle):
    x = oracle.brownian(2, 6, 3, 2)
    y = oracle.brownian(3, 7, 3, 3)
    g = oracle.static_gram("linear", x, y)
    np.testing.assert_allclose(g, np.einsum("ipk,jqk->ijpq", x, y), rtol=1e-15)
    rbf = oracle.static_gram("rbf", x, y, 0.7)
    d2 = ((x[:, None, :, None, :] - y[None, :, None, :, :]) ** 2).sum(-1)
    np.testing.assert_allclose(rbf, np.exp(-d2 / 0.7), rtol=1e-12)
    l1 = oracle.static_gram("l1rbf", x, y, 0.7)
    d1 = np.abs(x[:, None, :, None, :] - y[None, :, None, :, :]).sum(-1)
    np.testing.assert_allclose(l1, np.exp(-d1 / 0.7), rtol=1e-12)
