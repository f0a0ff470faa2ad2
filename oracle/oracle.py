"""FP64 CPU oracle for the SigPDE signature-kernel hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker the CUDA product is
compared against.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg may import it; the product package never does.

It wraps ``sigk_oracle.c`` (a plain-C float64 restatement, OpenMP over pairs)
and adds the small pieces of host logic the reference keeps in Python:

* scale broadcasting of ``SigPDE.pairwise`` / ``_gram``      sigpde/torch/kernel.py:31-41, 75-84
* symmetric Gram ``gram(x)``                                 sigpde/torch/kernel.py:67-73, 128-171
* the robust normalisation (NaN -> inf, f(k), Chandrupatla, lambda = 0 for k < 1)
                                                             sigpde/torch/kernel.py:180-230
* RobustSigPDE.pairwise / gram                               sigpde/torch/kernel.py:232-301
* static-kernel Grams (linear / RBF / L1-RBF) in float64     sigpde/torch/static_kernels.py:3-53
* gradients of pairwise / Gram (LinearKernel) by the adjoint of the solve (no
  reference counterpart; pinned by central differences of the solve in tests/)

Inputs are upcast to float64 before anything is computed, so the rounding of
float32 inputs is not charged to the kernel under test.  Parity of this
restatement is pinned against the reference itself (run under
NUMBA_ENABLE_CUDASIM=1) by the fixtures in ``tests/golden``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsigk_oracle.so")
_lib = None
_lock = threading.Lock()

_d = ctypes.c_double
_i64 = ctypes.c_int64
_int = ctypes.c_int
_pd = ctypes.POINTER(ctypes.c_double)
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pint = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile ``libsigk_oracle.so`` with the committed Makefile (gcc, -ffp-contract=off)."""
    src = os.path.join(_HERE, "sigk_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(_LIB_PATH)
            L.sko_solve.argtypes = [_pd, _i64, _i64, _int, _d, _int, _pd]
            L.sko_solve.restype = _d
            L.sko_increments_linear.argtypes = [_pd, _pd, _i64, _i64, _i64, _int, _d, _pd]
            L.sko_solve_batch.argtypes = [_pd, _i64, _i64, _i64, _int, _pd, _pd, _int, _pd]
            L.sko_pairwise_linear.argtypes = [_pd, _pd, _i64, _i64, _i64, _i64, _int, _d, _pd, _pd, _int, _pd]
            L.sko_gram_linear.argtypes = [_pd, _pd, _i64, _i64, _i64, _i64, _i64, _int, _d, _pd, _pd, _int,
                                          _pi64, _i64, _pd]
            L.sko_chandrupatla.argtypes = [_pd, _i64, _int, _d, _d, _d, _int, _int, _pint]
            L.sko_chandrupatla.restype = _d
            L.sko_chandrupatla_batch.argtypes = [_pd, _i64, _i64, _int, _pd, _pd, _d, _int, _int, _pd, _pint]
            L.sko_grad_solve.argtypes = [_pd, _i64, _i64, _int, _d, _d, _pd]
            L.sko_grad_solve.restype = _d
            L.sko_grad_solve_batch.argtypes = [_pd, _i64, _i64, _i64, _int, _pd, _pd, _pd, _pd]
            L.sko_num_threads.restype = _int
            L.sko_set_num_threads.argtypes = [_int]
            _lib = L
    return _lib


def num_threads() -> int:
    return lib().sko_num_threads()


def set_num_threads(n: int) -> None:
    lib().sko_set_num_threads(int(n))


def _f64(a) -> np.ndarray:
    if hasattr(a, "detach"):
        a = a.detach().cpu().double().numpy()
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_pd)


def _scale_vec(s, n):
    """Scale broadcast of sigpde/torch/kernel.py:40-41 (shape [1] -> [n])."""
    if s is None:
        return None
    s = _f64(s).reshape(-1)
    if s.shape[0] == 1:
        s = np.repeat(s, n)
    return np.ascontiguousarray(s)


# --------------------------------------------------------------------------- increments
def static_gram(kind: str, X, Y, param: float = 1.0) -> np.ndarray:
    """Static kernel on all point pairs, float64: (A,M,d) x (B,N,d) -> (A,B,M,N).

    linear: param * <x,y>                 static_kernels.py:3-11
    rbf:    exp(-|x-y|^2 / param)          static_kernels.py:13-36
    l1rbf:  exp(-|x-y|_1 / param)          static_kernels.py:38-53
    """
    X = _f64(X)
    Y = _f64(Y)
    if kind == "linear":
        return param * np.einsum("ipk,jqk->ijpq", X, Y)
    if kind == "rbf":
        Xs = np.sum(X ** 2, axis=2)
        Ys = np.sum(Y ** 2, axis=2)
        dist = -2.0 * np.einsum("ipk,jqk->ijpq", X, Y)
        dist += Xs[:, None, :, None] + Ys[None, :, None, :]
        return np.exp(-dist / param)
    if kind == "l1rbf":
        dist = np.abs(X[:, None, :, None, :] - Y[None, :, None, :, :]).sum(-1)
        return np.exp(-dist / param)
    raise ValueError(f"unknown static kernel {kind!r}")


def second_difference(ip: np.ndarray, order: int) -> np.ndarray:
    """4-term difference / 4^order over the last two axes (kernel.py:13-21)."""
    d = ip[..., 1:, 1:] + ip[..., :-1, :-1] - ip[..., 1:, :-1] - ip[..., :-1, 1:]
    return d / float(2 ** (2 * order))


def increments_linear(x, y, order: int, static_scale: float = 1.0) -> np.ndarray:
    """LinearKernel increments of one pair, via the C restatement."""
    x = _f64(x)
    y = _f64(y)
    Lx, d = x.shape
    Ly = y.shape[0]
    out = np.empty((Lx - 1, Ly - 1), np.float64)
    lib().sko_increments_linear(_ptr(x), _ptr(y), Lx, Ly, d, int(order), float(static_scale), _ptr(out))
    return out


# --------------------------------------------------------------------------- solves
def solve_increments(incs, order: int, sx=None, sy=None, store_f32: bool = False) -> np.ndarray:
    """Solve a batch of precomputed coarse increments (npairs, ncx, ncy)."""
    incs = _f64(incs)
    if incs.ndim == 2:
        incs = incs[None]
    B, ncx, ncy = incs.shape
    sx = None if sx is None else _f64(sx).reshape(B)
    sy = None if sy is None else _f64(sy).reshape(B)
    out = np.empty(B, np.float64)
    lib().sko_solve_batch(_ptr(incs), B, ncx, ncy, int(order), _ptr(sx), _ptr(sy), int(store_f32), _ptr(out))
    return out


def py_solve(inc, order: int, scale: float = 1.0) -> float:
    """Pure-Python restatement of the anti-diagonal loop, for tiny cases only.

    Walks anti-diagonals p = 2..N-1 exactly as sigpde/cuda_pairwise_kernels.py:17-39,
    with a full (lx, ly) grid instead of the 3-slot rotation.
    """
    inc = _f64(inc)
    ncx, ncy = inc.shape
    lx = (ncx << order) + 1
    ly = (ncy << order) + 1
    N = lx + ly - 1
    K = [[1.0] * ly for _ in range(lx)]
    for p in range(2, N):
        for i in range(1, min(lx, p)):
            j = p - i
            if 1 <= j < ly:
                c = float(inc[(i - 1) >> order, (j - 1) >> order]) * scale
                k00, k01, k10 = K[i - 1][j - 1], K[i - 1][j], K[i][j - 1]
                c2 = c * c
                K[i][j] = (k01 + k10) * (1. + 0.5 * c + (1. / 12) * c2) - k00 * (1. - (1. / 12) * c2)
    return K[lx - 1][ly - 1]


def pairwise(x, y=None, order: int = 0, x_scale=None, y_scale=None, static: str = "linear",
             static_param: float = 1.0, store_f32: bool = False) -> np.ndarray:
    """SigPDE.pairwise (sigpde/torch/kernel.py:31-65) in float64."""
    if y is None:
        y_scale = x_scale
        y = x
    x = _f64(x)
    y = _f64(y)
    B = x.shape[0]
    scaled = x_scale is not None or y_scale is not None
    sx = _scale_vec(x_scale, B) if scaled else None
    sy = _scale_vec(y_scale, B) if scaled else None
    if scaled:
        sx = np.ones(B) if sx is None else sx
        sy = np.ones(B) if sy is None else sy
    if static == "linear":
        Lx, d = x.shape[1], x.shape[2]
        Ly = y.shape[1]
        out = np.empty(B, np.float64)
        lib().sko_pairwise_linear(_ptr(x), _ptr(y), B, Lx, Ly, d, int(order), float(static_param),
                                  _ptr(sx), _ptr(sy), int(store_f32), _ptr(out))
        return out
    incs = np.stack([second_difference(static_gram(static, x[b:b + 1], y[b:b + 1], static_param)[0, 0], order)
                     for b in range(B)])
    return solve_increments(incs, order, sx, sy, store_f32)


def gram(x, y=None, order: int = 0, x_scale=None, y_scale=None, static: str = "linear",
         static_param: float = 1.0, store_f32: bool = False, pairs=None) -> np.ndarray:
    """SigPDE.gram (sigpde/torch/kernel.py:67-171) in float64.

    ``y=None`` is the symmetric Gram with ``y_scale = x_scale`` (the reference
    computes the lower triangle and mirrors it, cuda_gram_kernels.py:85-113; the
    mirrored values equal a direct solve of k(x_j, x_i) only up to the symmetry of
    the PDE, so the oracle computes the lower triangle and mirrors too).
    ``pairs`` (flat indices i*Ny+j) restricts the computation for sampled checks;
    the return value is then the 1-D vector of those entries.
    """
    sym = y is None
    if sym:
        y = x
        y_scale = x_scale
    x = _f64(x)
    y = _f64(y)
    Nx, Ny = x.shape[0], y.shape[0]
    scaled = x_scale is not None or y_scale is not None
    sx = _scale_vec(x_scale, Nx) if scaled else None
    sy = _scale_vec(y_scale, Ny) if scaled else None
    if scaled:
        sx = np.ones(Nx) if sx is None else sx
        sy = np.ones(Ny) if sy is None else sy
    if sym and pairs is None:
        tri = np.array([i * Ny + j for i in range(Nx) for j in range(i + 1)], dtype=np.int64)
        vals = gram(x, x, order, sx, sy, static, static_param, store_f32, pairs=tri)
        out = np.empty((Nx, Ny), np.float64)
        ii, jj = tri // Ny, tri % Ny
        out[ii, jj] = vals
        out[jj, ii] = vals
        return out
    if static == "linear":
        Lx, d = x.shape[1], x.shape[2]
        Ly = y.shape[1]
        if pairs is not None:
            pairs = np.ascontiguousarray(np.asarray(pairs, dtype=np.int64))
            out = np.empty(pairs.shape[0], np.float64)
            pp, npairs = pairs.ctypes.data_as(_pi64), pairs.shape[0]
        else:
            out = np.empty((Nx, Ny), np.float64)
            pp, npairs = None, 0
        lib().sko_gram_linear(_ptr(x), _ptr(y), Nx, Ny, Lx, Ly, d, int(order), float(static_param),
                              _ptr(sx), _ptr(sy), int(store_f32), pp, npairs, _ptr(out))
        return out
    flat = np.arange(Nx * Ny) if pairs is None else np.asarray(pairs)
    incs = np.stack([second_difference(static_gram(static, x[f // Ny:f // Ny + 1], y[f % Ny:f % Ny + 1],
                                                   static_param)[0, 0], order) for f in flat])
    vx = None if sx is None else sx[flat // Ny]
    vy = None if sy is None else sy[flat % Ny]
    vals = solve_increments(incs, order, vx, vy, store_f32)
    return vals if pairs is not None else vals.reshape(Nx, Ny)


# --------------------------------------------------------------------------- gradients
def grad_increments(incs, order: int, scale=None, w=None):
    """w * dk/dc for a batch of increment blocks (npairs, ncx, ncy), c = inc * scale:
    the adjoint of the solve (sko_grad_solve).  Returns (G, k)."""
    incs = _f64(incs)
    if incs.ndim == 2:
        incs = incs[None]
    B, ncx, ncy = incs.shape
    scale = None if scale is None else _f64(scale).reshape(B)
    w = None if w is None else _f64(w).reshape(B)
    G = np.empty((B, ncx, ncy), np.float64)
    k = np.empty(B, np.float64)
    lib().sko_grad_solve_batch(_ptr(incs), B, ncx, ncy, int(order), _ptr(scale), _ptr(w), _ptr(G), _ptr(k))
    return G, k


def _chain_linear(H, x, y):
    """Gradients of sum_ij H_ij <dx_i, dy_j> with respect to the points of x and y."""
    dx = np.diff(x, axis=0)
    dy = np.diff(y, axis=0)
    hx = H @ dy          # (ncx, d): d/d dx_i
    hy = H.T @ dx        # (ncy, d): d/d dy_j
    gx = np.zeros_like(x)
    gy = np.zeros_like(y)
    gx[1:] += hx
    gx[:-1] -= hx
    gy[1:] += hy
    gy[:-1] -= hy
    return gx, gy


def grad_pairwise(x, y, order: int, grad_out, x_scale=None, y_scale=None, static_scale: float = 1.0):
    """Gradients of sum_b grad_out[b] * k(x_b, y_b) (LinearKernel) with respect to x and y,
    float64, by the adjoint of each solve and the chain rule through the increments
    inc_ij = static_scale * <dx_i, dy_j> / 4^order, c = inc * x_scale * y_scale."""
    x = _f64(x)
    y = _f64(y)
    B = x.shape[0]
    w = _f64(grad_out).reshape(B)
    sx = _scale_vec(x_scale, B)
    sy = _scale_vec(y_scale, B)
    s = np.ones(B) * (1.0 if sx is None else sx) * (1.0 if sy is None else sy)
    incs = np.stack([increments_linear(x[b], y[b], order, static_scale) for b in range(B)])
    G, _ = grad_increments(incs, order, s, w)
    gx = np.zeros_like(x)
    gy = np.zeros_like(y)
    f = static_scale / float(4 ** order)
    for b in range(B):
        gx[b], gy[b] = _chain_linear(G[b] * (s[b] * f), x[b], y[b])
    return gx, gy


def grad_gram(x, y, order: int, grad_out, x_scale=None, y_scale=None, static_scale: float = 1.0):
    """Gradients of sum_ij grad_out[i, j] * k(x_i, y_j) (LinearKernel Gram) with respect to x
    and y (y=None: the symmetric Gram of x, both sides' contributions to x)."""
    sym = y is None
    x = _f64(x)
    y = x if sym else _f64(y)
    Nx, Ny = x.shape[0], y.shape[0]
    w = _f64(grad_out).reshape(Nx, Ny)
    sx = _scale_vec(x_scale, Nx)
    sy = sx if sym else _scale_vec(y_scale, Ny)
    sxv = np.ones(Nx) if sx is None else sx
    syv = np.ones(Ny) if sy is None else sy
    ii, jj = np.meshgrid(np.arange(Nx), np.arange(Ny), indexing="ij")
    ii, jj = ii.reshape(-1), jj.reshape(-1)
    incs = np.stack([increments_linear(x[i], y[j], order, static_scale) for i, j in zip(ii, jj)])
    s = sxv[ii] * syv[jj]
    G, _ = grad_increments(incs, order, s, w.reshape(-1))
    gx = np.zeros_like(x)
    gy = np.zeros_like(y)
    f = static_scale / float(4 ** order)
    for t, (i, j) in enumerate(zip(ii, jj)):
        a, b = _chain_linear(G[t] * (s[t] * f), x[i], y[j])
        gx[i] += a
        gy[j] += b
    if sym:
        return gx + gy
    return gx, gy


def _chain_static(kind, H, x, y, param):
    """Gradients of sum_pq H[p, q] k(x_p, y_q) for the RBF / L1-RBF static kernels
    (sigpde/torch/static_kernels.py:13-53) with respect to the points."""
    S = static_gram(kind, x[None], y[None], param)[0, 0]
    diff = x[:, None, :] - y[None, :, :]                 # (Lx, Ly, d)
    if kind == "rbf":
        W = H * S * (-2.0 / param)
        gx = np.einsum("pq,pqk->pk", W, diff)
        gy = -np.einsum("pq,pqk->qk", W, diff)
    elif kind == "l1rbf":
        W = H * S * (-1.0 / param)
        sg = np.sign(diff)
        gx = np.einsum("pq,pqk->pk", W, sg)
        gy = -np.einsum("pq,pqk->qk", W, sg)
    else:
        raise ValueError(kind)
    return gx, gy


def _second_difference_adjoint(Ginc, f):
    """dL/dS for inc = f * (S[1:,1:] + S[:-1,:-1] - S[1:,:-1] - S[:-1,1:])."""
    ncx, ncy = Ginc.shape
    H = np.zeros((ncx + 1, ncy + 1))
    H[1:, 1:] += Ginc
    H[:-1, :-1] += Ginc
    H[1:, :-1] -= Ginc
    H[:-1, 1:] -= Ginc
    return H * f


def grad_static_pairs(kind, x, y, order, w, param, sx=None, sy=None):
    """Per-pair gradients of sum_b w[b] k(x_b, y_b) for a static kernel of the
    generic route (increments from the static Gram), float64.  Returns (gx, gy)."""
    x = _f64(x)
    y = _f64(y)
    B = x.shape[0]
    s = np.ones(B) * (1.0 if sx is None else _f64(sx).reshape(B)) * (1.0 if sy is None else _f64(sy).reshape(B))
    incs = np.stack([second_difference(static_gram(kind, x[b:b + 1], y[b:b + 1], param)[0, 0], order)
                     for b in range(B)])
    G, _ = grad_increments(incs, order, s, _f64(w).reshape(B))
    f = 1.0 / float(4 ** order)
    gx = np.zeros_like(x)
    gy = np.zeros_like(y)
    for b in range(B):
        H = _second_difference_adjoint(G[b] * s[b], f)
        gx[b], gy[b] = _chain_static(kind, H, x[b], y[b], param)
    return gx, gy


def grad_static_gram(kind, x, y, order, w, param, sx=None, sy=None):
    """Gradients of sum_ij w[i, j] k(x_i, y_j) for RBF / L1-RBF (y=None: the
    symmetric Gram, both sides' contributions to x)."""
    sym = y is None
    x = _f64(x)
    y = x if sym else _f64(y)
    Nx, Ny = x.shape[0], y.shape[0]
    w = _f64(w).reshape(Nx, Ny)
    sxv = np.ones(Nx) if sx is None else _scale_vec(sx, Nx)
    syv = sxv if sym else (np.ones(Ny) if sy is None else _scale_vec(sy, Ny))
    ii, jj = np.meshgrid(np.arange(Nx), np.arange(Ny), indexing="ij")
    ii, jj = ii.reshape(-1), jj.reshape(-1)
    gxp, gyp = grad_static_pairs(kind, x[ii], y[jj], order, w.reshape(-1), param, sxv[ii], syv[jj])
    gx = np.zeros_like(x)
    gy = np.zeros_like(y)
    np.add.at(gx, ii, gxp)
    np.add.at(gy, jj, gyp)
    if sym:
        return gx + gy
    return gx, gy


# --------------------------------------------------------------------------- robust
def log_normalizer(k):
    """Default normalizer f(s) = 2 - 1/(1 + log s) (sigpde/torch/kernel.py:23-24)."""
    return 2 - 1 / (1 + np.log(k))


def _apply_normalizer(normalizer, k: np.ndarray) -> np.ndarray:
    if normalizer is None:
        with np.errstate(all="ignore"):
            return log_normalizer(k)
    try:
        import torch
        r = normalizer(torch.from_numpy(k.copy()))
        if hasattr(r, "detach"):
            return r.detach().cpu().double().numpy()
        return np.asarray(r, np.float64)
    except ImportError:  # pragma: no cover
        return np.asarray(normalizer(k), np.float64)


def normalization(x, order: int = 0, normalizer=None, tol: float = 1e-8, maxit: int = 100,
                  static: str = "linear", static_param: float = 1.0, return_iters: bool = False):
    """RobustSigPDE.normalization (sigpde/torch/kernel.py:180-230) in float64.

    k = k(x,x); NaN -> +inf; fk = f(k); lambda from the Chandrupatla loop;
    lambda = 0 where k < 1.
    """
    x = _f64(x)
    B, L = x.shape[0], x.shape[1]
    if static == "linear":
        incs = np.stack([increments_linear(x[b], x[b], order, static_param) for b in range(B)])
    else:
        incs = np.stack([second_difference(static_gram(static, x[b:b + 1], x[b:b + 1], static_param)[0, 0], order)
                         for b in range(B)])
    incs = np.ascontiguousarray(incs)
    k = solve_increments(incs, order)
    k[np.isnan(k)] = np.inf
    fk = np.ascontiguousarray(_apply_normalizer(normalizer, k), dtype=np.float64)
    lam = np.empty(B, np.float64)
    iters = np.zeros(B, np.int32)
    with np.errstate(all="ignore"):
        lib().sko_chandrupatla_batch(_ptr(incs), B, L - 1, int(order), _ptr(k), _ptr(fk), float(tol), int(maxit), 0,
                                     _ptr(lam), iters.ctypes.data_as(_pint))
    if return_iters:
        return lam, k, fk, iters
    return lam


def robust_pairwise(x, y=None, order: int = 0, normalizer=None, tol: float = 1e-8, maxit: int = 100):
    """RobustSigPDE.pairwise (sigpde/torch/kernel.py:232-291) in float64."""
    lx = normalization(x, order, normalizer, tol, maxit)
    if y is None:
        return pairwise(x, None, order, lx, lx)
    ly = normalization(y, order, normalizer, tol, maxit)
    return pairwise(x, y, order, lx, ly)


def robust_gram(x, y=None, order: int = 0, x_scale=None, y_scale=None, normalizer=None, tol: float = 1e-8,
                maxit: int = 100):
    """RobustSigPDE.gram (sigpde/torch/kernel.py:293-301) in float64."""
    xs = normalization(x, order, normalizer, tol, maxit) if x_scale is None else x_scale
    if y is None:
        return gram(x, None, order, xs, None)
    ys = normalization(y, order, normalizer, tol, maxit) if y_scale is None else y_scale
    return gram(x, y, order, xs, ys)


# --------------------------------------------------------------------------- inputs
def brownian(n: int, length: int, dim: int, seed: int, scale=None) -> np.ndarray:
    """Seeded Brownian paths, float64: x[:,0] = 0, x[:,t] = cumsum of N(0, 1/(L-1)).

    Uses numpy's PCG64 so the same paths can be rebuilt on any host.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    inc = rng.standard_normal((n, length - 1, dim)) / np.sqrt(max(length - 1, 1))
    x = np.zeros((n, length, dim))
    x[:, 1:, :] = np.cumsum(inc, axis=1)
    if scale is not None:
        x = x * np.asarray(scale, np.float64).reshape(n, 1, 1)
    return x
