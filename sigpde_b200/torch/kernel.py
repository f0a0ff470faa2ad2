"""`SigPDE` and `RobustSigPDE` with the API of sigpde/torch/kernel.py, backed
by libsigk.so (hand-written sm_100a CUDA).

Differences from the reference that a caller can observe:
  * the work is enqueued on torch's current CUDA stream and the call returns
    without a device-wide synchronise (the reference calls
    numba.cuda.synchronize(), kernel.py:56-63,124,169,228,289); results are
    ordinary torch tensors, so stream order keeps every later torch op correct;
  * PDE cells are float64 by default (`precision="fp64"`), also for float32
    inputs, and the robust normalisation always runs in float64, including
    k(x,x) and f(k(x,x)); the reference rounds every cell to the input dtype
    and overflows k(x,x) to inf in float32 (17.6% of the paths of the robust
    benchmark, N=512 L=64 d=16, scales log-uniform in [0.5, 4]).
    `precision="fp32"` gives float32 cells; "tc32" / "tc64" form the
    linear-kernel increments with one split-TF32 tensor-core GEMM and solve
    float32 / float64 cells (sigk.h describes where they apply);
  * `max_batch` / `max_threads` are accepted and only bound the memory of the
    generic-increment path (non-linear static kernels); the linear kernel runs
    any batch in one launch.
"""
from __future__ import annotations

import math

import torch

from .. import _lib
from . import static_kernels

_PREC = {"fp64": _lib.SIGK_PREC_FP64, "fp32": _lib.SIGK_PREC_FP32, "tc32": _lib.SIGK_PREC_TC32,
         "tc64": _lib.SIGK_PREC_TC64}


def _dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return _lib.SIGK_F32
    if t.dtype == torch.float64:
        return _lib.SIGK_F64
    raise TypeError(f"signature kernels take float32 or float64 paths, got {t.dtype}")


def _check_paths(x: torch.Tensor, name: str) -> None:
    if not isinstance(x, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if not x.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (this package has no CPU path)")
    if x.dim() != 3:
        raise ValueError(f"{name} must have shape (batch, length, dim), got {tuple(x.shape)}")
    if x.shape[1] < 2:
        raise ValueError(f"{name} needs at least 2 points per path, got length {x.shape[1]}")
    _dtype_code(x)


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _ptr(t):
    return None if t is None else t.data_ptr()


def _workspace(op, nx, ny, lx, ly, d, order, dtype_code, prec, device):
    n = _lib.lib().sigk_workspace_size(op, nx, ny, lx, ly, d, order, dtype_code, prec)
    if n == 0:
        return None, 0
    return torch.empty(n, dtype=torch.uint8, device=device), n


def _broadcast_scale(s, n, like: torch.Tensor):
    """Scale broadcast of sigpde/torch/kernel.py:38-41 ([1] -> [n])."""
    if s is None:
        return None
    if not isinstance(s, torch.Tensor):
        s = torch.as_tensor(s, dtype=like.dtype, device=like.device)
    s = s.reshape(-1).to(device=like.device, dtype=like.dtype)
    if s.shape[0] == 1:
        s = s.repeat(n)
    if s.shape[0] != n:
        raise ValueError(f"scale has {s.shape[0]} entries, expected 1 or {n}")
    return s.contiguous()


def _is_fused_linear(static_kernel) -> bool:
    """The linear kernel (ours, or any object named LinearKernel with a float
    `scale`, such as the reference's) is contracted on the device."""
    if isinstance(static_kernel, static_kernels.LinearKernel):
        return True
    return type(static_kernel).__name__ == "LinearKernel" and isinstance(getattr(static_kernel, "scale", None),
                                                                          (int, float))


def _static_kind(static_kernel):
    """(kind, sigma) for an RBF or L1-RBF kernel whose static Gram the device
    evaluates from the points (ours, or the reference's classes of the same
    name with a float sigma), else None."""
    name = type(static_kernel).__name__
    kind = {"RBFKernel": _lib.SIGK_STATIC_RBF, "L1RBFKernel": _lib.SIGK_STATIC_L1RBF}.get(name)
    sigma = getattr(static_kernel, "sigma", None)
    if kind is None or isinstance(sigma, bool) or not isinstance(sigma, (int, float)):
        return None
    if not (isinstance(static_kernel, (static_kernels.RBFKernel, static_kernels.L1RBFKernel)) or
            type(static_kernel).__module__.startswith("sigpde")):
        return None
    return kind, float(sigma)


def pairwise_inner_product(x, y, static_kernel, dyadic_order):
    """Coarse increments of each pair: 4-term second difference of the static
    Gram divided by 4^order (sigpde/torch/kernel.py:13-16)."""
    ip = static_kernel.pairwise(x, y)
    ip = ip[:, 1:, 1:] + ip[:, :-1, :-1] - ip[:, 1:, :-1] - ip[:, :-1, 1:]
    return ip / float(4 ** dyadic_order)


def gram_inner_product(x, y, static_kernel, dyadic_order):
    """Gram version of pairwise_inner_product (sigpde/torch/kernel.py:18-21)."""
    ip = static_kernel.gram(x, y)
    ip = ip[:, :, 1:, 1:] + ip[:, :, :-1, :-1] - ip[:, :, 1:, :-1] - ip[:, :, :-1, 1:]
    return ip / float(4 ** dyadic_order)


def log_normalizer(x):
    """Default robust normaliser f(s) = 2 - 1/(1 + log s) (sigpde/torch/kernel.py:23-24)."""
    return 2 - 1 / (1 + x.log())


def _wants_grad(*ts) -> bool:
    return torch.is_grad_enabled() and any(isinstance(t, torch.Tensor) and t.requires_grad for t in ts)


class _LinearSigKernel(torch.autograd.Function):
    """Differentiable LinearKernel values: pairwise, Gram and symmetric Gram.

    The forward is the solver's own path (any precision); the backward runs
    sigk_backward, the adjoint of the float64 scheme, for the gradients with
    respect to the points of x and y.  Per-path scales are constants.  The
    reference has no backward pass (its Numba kernels end autograd)."""

    @staticmethod
    def forward(ctx, x, y, sx, sy, solver, op):
        if op == "pairwise":
            out = solver.pairwise(x, y, sx, sy)
        elif op == "gram":
            out = solver._gram(x, y, sx, sy, 1000)
        else:
            out = solver._gram_sym(x, sx, 1000)
        ctx.solver = solver
        ctx.op = op
        ctx.save_for_backward(x, y, sx, sy)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        x, y, sx, sy = ctx.saved_tensors
        solver, op = ctx.solver, ctx.op
        self_pairs = y is None  # k(x_i, x_j) / k(x_b, x_b): both sides are x
        yy = x if self_pairs else y
        if self_pairs:
            sy = sx
        kop = _lib.SIGK_OP_PAIRWISE if op == "pairwise" else _lib.SIGK_OP_GRAM
        need_x = ctx.needs_input_grad[0]
        need_y = (not self_pairs) and ctx.needs_input_grad[1]
        if not (need_x or need_y):
            return None, None, None, None, None, None
        x = x.contiguous()
        yy = yy.contiguous()
        g = grad_out.detach().to(dtype=x.dtype).contiguous()
        gx = torch.empty_like(x) if (need_x or self_pairs) else None
        gy = torch.empty_like(yy) if (need_y or self_pairs) else None
        Nx, Ny = x.shape[0], yy.shape[0]
        dt = _dtype_code(x)
        with torch.cuda.device(x.device):
            n = _lib.lib().sigk_backward_workspace_size(kop, Nx, Ny, x.shape[1], yy.shape[1], x.shape[2],
                                                        solver.dyadic_order, dt)
            ws = torch.empty(n, dtype=torch.uint8, device=x.device)
            _lib.call("sigk_backward", kop, _ptr(x), _ptr(yy), Nx, Ny, x.shape[1], yy.shape[1], x.shape[2], dt,
                      solver.dyadic_order, float(solver.static_kernel.scale), _ptr(sx), _ptr(sy), _ptr(g), _ptr(gx),
                      _ptr(gy), _ptr(ws), n, _stream())
        if self_pairs:
            return gx + gy, None, None, None, None, None
        return gx, gy, None, None, None, None


class _IncSolve(torch.autograd.Function):
    """k of each pair from caller's increments (sigk_pairwise_inc), differentiable
    with respect to the increments (sigk_backward_inc, the float64 adjoint), so
    that autograd continues through whatever torch code built them: any static
    kernel of the duck-typed protocol.  Scales are constants."""

    @staticmethod
    def forward(ctx, inc, sx, sy, solver):
        B, ncx, ncy = inc.shape
        out = torch.empty(B, device=inc.device, dtype=inc.dtype)
        solver._solve_pairwise_inc(inc, sx, sy, out)
        ctx.solver = solver
        ctx.save_for_backward(inc, sx, sy)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        inc, sx, sy = ctx.saved_tensors
        if not ctx.needs_input_grad[0]:
            return None, None, None, None
        B, ncx, ncy = inc.shape
        g = grad_out.detach().to(dtype=inc.dtype).contiguous()
        ginc = torch.empty(inc.shape, dtype=inc.dtype, device=inc.device)
        dt = _dtype_code(inc)
        order = ctx.solver.dyadic_order
        with torch.cuda.device(inc.device):
            n = _lib.lib().sigk_backward_inc_workspace_size(B, ncx, ncy, order)
            ws = torch.empty(n, dtype=torch.uint8, device=inc.device)
            _lib.call("sigk_backward_inc", _ptr(inc), B, ncx, ncy, inc.stride(0), inc.stride(1), inc.stride(2), dt,
                      order, _ptr(sx), _ptr(sy), _ptr(g), _ptr(ginc), ginc.stride(0), ginc.stride(1),
                      ginc.stride(2), _ptr(ws), n, _stream())
        return ginc, None, None, None


def _generic_differentiable(solver, op, x, y, x_scale, y_scale, max_batch):
    """Differentiable values for a static kernel other than the linear one: the
    reference's route (torch builds the increments of each tile, so autograd
    sees the static kernel) with _IncSolve for the solves."""
    _check_paths(x, "x")
    if op == "pairwise":
        yv = x if y is None else y
        _check_paths(yv, "y")
        B = x.shape[0]
        ys = x_scale if y is None else y_scale
        scaled = x_scale is not None or ys is not None
        sx = _broadcast_scale(x_scale, B, x) if scaled else None
        sy = _broadcast_scale(ys, B, yv) if scaled else None
        parts = []
        for s0, s1 in _batches(B, max_batch):
            inc = pairwise_inner_product(x[s0:s1], yv[s0:s1], solver.static_kernel, solver.dyadic_order).to(x.dtype)
            if scaled:  # in torch, so that autograd reaches the scales (sigpde/cuda_pairwise_kernels.py:61,69)
                inc = inc * (sx[s0:s1] * sy[s0:s1])[:, None, None]
            parts.append(_IncSolve.apply(inc, None, None, solver))
        return torch.cat(parts)
    sym = y is None
    yv = x if sym else y
    _check_paths(yv, "y")
    Nx, Ny = x.shape[0], yv.shape[0]
    ys = x_scale if sym else y_scale
    scaled = x_scale is not None or ys is not None
    sx = _broadcast_scale(x_scale, Nx, x) if scaled else None
    sy = _broadcast_scale(ys, Ny, yv) if scaled else None
    tile = math.ceil(math.sqrt(max_batch))  # sigpde/torch/kernel.py:68
    blocks = {}
    rows = []
    for x0, x1 in _batches(Nx, tile):
        row = []
        for y0, y1 in _batches(Ny, tile):
            if sym and y0 > x0:  # upper tiles are the transposed lower ones
                row.append(None)
                continue
            inc = gram_inner_product(x[x0:x1], yv[y0:y1], solver.static_kernel, solver.dyadic_order).to(x.dtype)
            if scaled:  # in torch, so that autograd reaches the scales (sigpde/cuda_gram_kernels.py:52,60)
                inc = inc * (sx[x0:x1][:, None] * sy[y0:y1][None, :])[:, :, None, None]
            tx, ty, ncx, ncy = inc.shape
            blk = _IncSolve.apply(inc.reshape(tx * ty, ncx, ncy), None, None, solver).reshape(tx, ty)
            blocks[(x0, y0)] = blk
            row.append(blk)
        rows.append(row)
    xs = list(_batches(Nx, tile))
    ysb = list(_batches(Ny, tile))
    out_rows = []
    for a, (x0, _) in enumerate(xs):
        out_rows.append(torch.cat([rows[a][b] if rows[a][b] is not None else blocks[(y0, x0)].t()
                                   for b, (y0, _) in enumerate(ysb)], dim=1))
    return torch.cat(out_rows, dim=0)


def _differentiable(solver, op, x, y, x_scale, y_scale, n_y, max_batch=1000):
    """Route a call whose paths or scales require grad through _LinearSigKernel
    (linear kernel) or the increment route with _IncSolve (any other static
    kernel)."""
    if not _is_fused_linear(solver.static_kernel):
        return _generic_differentiable(solver, "pairwise" if op == "pairwise" else "gram", x, y, x_scale,
                                       y_scale, max_batch)
    if _wants_grad(x_scale, y_scale):
        # the linear kernel's increments scaled by s_x s_y are those of the paths scaled by s_x and s_y,
        # so autograd reaches the scales through the paths
        _check_paths(x, "x")
        n_x = x.shape[0]
        sx = _broadcast_scale(x_scale, n_x, x) if x_scale is not None else None
        xs = x if sx is None else x * sx[:, None, None]
        if op == "gram_sym" or (op == "pairwise" and y is None):
            return _differentiable(solver, op, xs, None, None, None, n_y, max_batch)
        _check_paths(y, "y")
        sy = _broadcast_scale(y_scale, y.shape[0], y) if y_scale is not None else None
        ys = y if sy is None else y * sy[:, None, None]
        return _differentiable(solver, op, xs, ys, None, None, n_y, max_batch)
    _check_paths(x, "x")
    if y is not None:
        _check_paths(y, "y")
    n_x = x.shape[0]
    if op == "pairwise":
        yv = x if y is None else y
        ys = x_scale if y is None else y_scale
        scaled = x_scale is not None or ys is not None
        sx = _broadcast_scale(x_scale, n_x, x) if scaled else None
        sy = _broadcast_scale(ys, n_x, yv) if scaled else None
        return _LinearSigKernel.apply(x, y, sx, sy, solver, op)
    if op == "gram":
        scaled = x_scale is not None or y_scale is not None
        sx = _broadcast_scale(x_scale, n_x, x) if scaled else None
        sy = _broadcast_scale(y_scale, n_y, y) if scaled else None
        return _LinearSigKernel.apply(x, y, sx, sy, solver, op)
    sx = _broadcast_scale(x_scale, n_x, x)
    return _LinearSigKernel.apply(x, None, sx, None, solver, op)


def _batches(n, size):
    size = max(1, int(size))
    for start in range(0, n, size):
        yield start, min(n, start + size)


class SigPDE:
    """Untruncated signature kernel by the Goursat PDE (sigpde/torch/kernel.py:26-171)."""

    def __init__(self, static_kernel, dyadic_order=0, precision="fp64"):
        if precision not in _PREC:
            raise ValueError(f"precision must be one of {sorted(_PREC)}")
        if int(dyadic_order) < 0:
            raise ValueError("dyadic_order must be >= 0")
        self.static_kernel = static_kernel
        self.dyadic_order = int(dyadic_order)
        self.precision = precision

    # ------------------------------------------------------------------ pairwise
    def pairwise(self, x, y=None, x_scale=None, y_scale=None, max_batch=1000, max_threads=1024):
        if _wants_grad(x, y, x_scale, y_scale):
            return _differentiable(self, "pairwise", x, y, x_scale, y_scale, None, max_batch)
        y_scale = x_scale if y is None else y_scale
        y = x if y is None else y
        _check_paths(x, "x")
        _check_paths(y, "y")
        if y.dtype != x.dtype or y.device != x.device:
            raise ValueError("x and y must share dtype and device")
        B = x.shape[0]
        if y.shape[0] != B:
            raise ValueError(f"pairwise needs equal batch sizes, got {B} and {y.shape[0]}")
        if y.shape[2] != x.shape[2]:
            raise ValueError("x and y must have the same dimension")
        scaled = x_scale is not None or y_scale is not None
        sx = _broadcast_scale(x_scale, B, x) if scaled else None
        sy = _broadcast_scale(y_scale, B, y) if scaled else None
        result = torch.empty(B, device=x.device, dtype=x.dtype)
        if B == 0:
            return result
        dt = _dtype_code(x)
        prec = _PREC[self.precision]
        with torch.cuda.device(x.device):
            if _is_fused_linear(self.static_kernel):
                x = x.contiguous()
                y = y.contiguous()
                ws, nws = _workspace(_lib.SIGK_OP_PAIRWISE, B, B, x.shape[1], y.shape[1], x.shape[2],
                                     self.dyadic_order, dt, prec, x.device)
                _lib.call("sigk_pairwise", _ptr(x), _ptr(y), B, x.shape[1], y.shape[1], x.shape[2], dt,
                          self.dyadic_order, float(self.static_kernel.scale), _ptr(sx), _ptr(sy), _ptr(result),
                          prec, _ptr(ws), nws, _stream())
                return result
            for s0, s1 in _batches(B, max_batch):
                inc = pairwise_inner_product(x[s0:s1], y[s0:s1], self.static_kernel, self.dyadic_order)
                self._solve_pairwise_inc(inc, None if sx is None else sx[s0:s1],
                                         None if sy is None else sy[s0:s1], result[s0:s1])
        return result

    def _solve_pairwise_inc(self, inc, sx, sy, out):
        inc = inc.to(out.dtype)
        nb, ncx, ncy = inc.shape
        dt = _dtype_code(inc)
        prec = _PREC[self.precision]
        ws, nws = _workspace(_lib.SIGK_OP_PAIRWISE, nb, nb, ncx + 1, ncy + 1, 0, self.dyadic_order, dt, prec,
                             inc.device)
        _lib.call("sigk_pairwise_inc", _ptr(inc), nb, ncx, ncy, inc.stride(0), inc.stride(1), inc.stride(2), dt,
                  self.dyadic_order, _ptr(sx), _ptr(sy), _ptr(out), prec, _ptr(ws), nws, _stream())

    # ------------------------------------------------------------------ gram
    def gram(self, x, y=None, x_scale=None, y_scale=None, max_batch=1000, max_threads=1024):
        if _wants_grad(x, y, x_scale, y_scale):
            if y is None:
                return _differentiable(self, "gram_sym", x, None, x_scale, None, None, max_batch)
            return _differentiable(self, "gram", x, y, x_scale, y_scale, y.shape[0], max_batch)
        if y is None:
            return self._gram_sym(x, x_scale, max_batch)
        return self._gram(x, y, x_scale, y_scale, max_batch)

    def _gram(self, x, y, x_scale, y_scale, max_batch):
        _check_paths(x, "x")
        _check_paths(y, "y")
        if y.dtype != x.dtype or y.device != x.device:
            raise ValueError("x and y must share dtype and device")
        if y.shape[2] != x.shape[2]:
            raise ValueError("x and y must have the same dimension")
        Nx, Ny = x.shape[0], y.shape[0]
        scaled = x_scale is not None or y_scale is not None
        sx = _broadcast_scale(x_scale, Nx, x) if scaled else None
        sy = _broadcast_scale(y_scale, Ny, y) if scaled else None
        result = torch.empty((Nx, Ny), device=x.device, dtype=x.dtype)
        if Nx == 0 or Ny == 0:
            return result
        dt = _dtype_code(x)
        prec = _PREC[self.precision]
        with torch.cuda.device(x.device):
            if _is_fused_linear(self.static_kernel):
                x = x.contiguous()
                y = y.contiguous()
                ws, nws = _workspace(_lib.SIGK_OP_GRAM, Nx, Ny, x.shape[1], y.shape[1], x.shape[2],
                                     self.dyadic_order, dt, prec, x.device)
                _lib.call("sigk_gram", _ptr(x), _ptr(y), Nx, Ny, x.shape[1], y.shape[1], x.shape[2], dt,
                          self.dyadic_order, float(self.static_kernel.scale), _ptr(sx), _ptr(sy), _ptr(result),
                          prec, _ptr(ws), nws, _stream())
                return result
            if self._static_on_device(x):
                self._gram_static(_lib.SIGK_OP_GRAM, x, y, sx, sy, result)
                return result
            tile = math.ceil(math.sqrt(max_batch))  # sigpde/torch/kernel.py:68
            for y0, y1 in _batches(Ny, tile):
                for x0, x1 in _batches(Nx, tile):
                    inc = gram_inner_product(x[x0:x1], y[y0:y1], self.static_kernel, self.dyadic_order)
                    self._solve_gram_inc(inc, None if sx is None else sx[x0:x1], None if sy is None else sy[y0:y1],
                                         result, x0, y0, False)
        return result

    def _gram_sym(self, x, x_scale, max_batch):
        _check_paths(x, "x")
        N = x.shape[0]
        sx = _broadcast_scale(x_scale, N, x)
        result = torch.empty((N, N), device=x.device, dtype=x.dtype)
        if N == 0:
            return result
        dt = _dtype_code(x)
        prec = _PREC[self.precision]
        with torch.cuda.device(x.device):
            if _is_fused_linear(self.static_kernel):
                x = x.contiguous()
                ws, nws = _workspace(_lib.SIGK_OP_GRAM_SYM, N, N, x.shape[1], x.shape[1], x.shape[2],
                                     self.dyadic_order, dt, prec, x.device)
                _lib.call("sigk_gram_sym", _ptr(x), N, x.shape[1], x.shape[2], dt, self.dyadic_order,
                          float(self.static_kernel.scale), _ptr(sx), _ptr(result), prec, _ptr(ws), nws, _stream())
                return result
            if self._static_on_device(x):
                self._gram_static(_lib.SIGK_OP_GRAM_SYM, x, None, sx, None, result)
                return result
            tile = math.ceil(math.sqrt(max_batch))
            for y0, y1 in _batches(N, tile):
                for x0, x1 in _batches(N, tile):
                    if x0 < y0:
                        continue  # upper tiles are mirrored from the lower ones
                    inc = gram_inner_product(x[x0:x1], x[y0:y1], self.static_kernel, self.dyadic_order)
                    self._solve_gram_inc(inc, None if sx is None else sx[x0:x1], None if sx is None else sx[y0:y1],
                                         result, x0, y0, x0 == y0)
                    if x0 != y0:
                        result[y0:y1, x0:x1] = result[x0:x1, y0:y1].t()
        return result

    def _static_on_device(self, x):
        """RBF / L1-RBF Grams with dim <= 32 evaluate the static kernel from
        the points on the device (sigk_gram_static; float64 increments for
        float64 cells, rounded once to float32 for float32 cells); wider
        paths build the increments with torch (the reference's route)."""
        return (getattr(self, "_device_static", True) and _static_kind(self.static_kernel) is not None
                and x.shape[2] <= 32)

    def _gram_static(self, op, x, y, sx, sy, result):
        kind, sigma = _static_kind(self.static_kernel)
        x = x.contiguous()
        y = x if y is None else y.contiguous()
        dt = _dtype_code(x)
        prec = _PREC[self.precision]
        n = _lib.lib().sigk_static_workspace_size(op, kind, x.shape[0], y.shape[0], x.shape[1], y.shape[1],
                                                  x.shape[2], self.dyadic_order, dt, prec)
        ws = torch.empty(n, dtype=torch.uint8, device=x.device) if n else None
        _lib.call("sigk_gram_static", op, kind, sigma, _ptr(x), None if op == _lib.SIGK_OP_GRAM_SYM else _ptr(y),
                  x.shape[0], y.shape[0], x.shape[1], y.shape[1], x.shape[2], dt, self.dyadic_order, _ptr(sx),
                  _ptr(sy), _ptr(result), prec, _ptr(ws), n, _stream())

    def _solve_gram_inc(self, inc, sx, sy, result, x0, y0, symmetric):
        inc = inc.to(result.dtype)
        nx, ny, ncx, ncy = inc.shape
        dt = _dtype_code(inc)
        prec = _PREC[self.precision]
        out = result[x0:, y0:]
        op = _lib.SIGK_OP_GRAM_SYM if symmetric else _lib.SIGK_OP_GRAM
        ws, nws = _workspace(op, nx, ny, ncx + 1, ncy + 1, 0, self.dyadic_order, dt, prec, inc.device)
        _lib.call("sigk_gram_inc", _ptr(inc), nx, ny, ncx, ncy, inc.stride(0), inc.stride(1), inc.stride(2),
                  inc.stride(3), dt, self.dyadic_order, _ptr(sx), _ptr(sy), int(symmetric), _ptr(out),
                  result.stride(0), prec, _ptr(ws), nws, _stream())


class _RobustLambda(torch.autograd.Function):
    """The robust normalisation lambda(x) of each path, differentiable by the
    implicit function theorem.  lambda solves phi = k(lambda^2 inc) - f(k(inc)) = 0
    (inc: the path's self-increments, k: the PDE solution; lambda = 0 where
    k(inc) < 1, sigpde/torch/kernel.py:180-195), so
        dlambda/dx = -(d phi / dx) / (d phi / d lambda),
    both from autograd through the increments and _IncSolve's adjoint, the
    normaliser's derivative from autograd on the normaliser."""

    @staticmethod
    def forward(ctx, x, robust, normalizer, tol, maxit, max_batch):
        lam = robust._normalization(x, normalizer, tol, maxit, max_batch)[0]
        ctx.robust = robust
        ctx.normalizer = robust.normalizer if normalizer is None else normalizer
        ctx.max_batch = max_batch
        ctx.save_for_backward(x, lam)
        return lam

    @staticmethod
    def backward(ctx, g_lam):
        x, lam = ctx.saved_tensors
        if not ctx.needs_input_grad[0]:
            return None, None, None, None, None, None
        rk = ctx.robust
        solver = SigPDE(rk.static_kernel, rk.dyadic_order, "fp64")
        with torch.enable_grad():
            xg = x.detach().requires_grad_()
            inc = pairwise_inner_product(xg, xg, rk.static_kernel, rk.dyadic_order).to(torch.float64)
            lv = lam.detach().to(torch.float64).requires_grad_()
            k_lam = _IncSolve.apply(inc * (lv * lv)[:, None, None], None, None, solver)
            k_0 = _IncSolve.apply(inc, None, None, solver)
            kk = k_0.detach().clone().requires_grad_()
            fk = torch.as_tensor(ctx.normalizer(kk))
            (fprime,) = torch.autograd.grad(fk.sum(), kk)
            (phi_lam,) = torch.autograd.grad(k_lam.sum(), lv, retain_graph=True)
            valid = (lv.detach() > 0) & torch.isfinite(k_0.detach()) & torch.isfinite(fprime) & (phi_lam != 0)
            v = torch.where(valid, -g_lam.to(torch.float64) / torch.where(valid, phi_lam, torch.ones_like(phi_lam)),
                            torch.zeros_like(phi_lam))
            total = (v * k_lam).sum() - (v * fprime.detach() * k_0).sum()
            (gx,) = torch.autograd.grad(total, xg)
        return gx.to(x.dtype), None, None, None, None, None


class RobustSigPDE:
    """Robust (tensor-normalised) signature kernel (sigpde/torch/kernel.py:174-301)."""

    def __init__(self, static_kernel, dyadic_order=0, normalizer=None, precision="fp64"):
        if precision not in _PREC:
            raise ValueError(f"precision must be one of {sorted(_PREC)}")
        self.static_kernel = static_kernel
        self.dyadic_order = int(dyadic_order)
        self.normalizer = log_normalizer if normalizer is None else normalizer
        self.precision = precision

    def normalization(self, x, normalizer=None, tol=1e-8, maxit=100, max_batch=1000, max_threads=1024):
        """Per-path scale lambda with k(lambda x, lambda x) = f(k(x, x)), and
        lambda = 0 where k(x, x) < 1 (sigpde/torch/kernel.py:180-230)."""
        return self._normalization(x, normalizer, tol, maxit, max_batch)[0]

    def _normalization(self, x, normalizer, tol, maxit, max_batch, want_iters=False):
        normalizer = self.normalizer if normalizer is None else normalizer
        _check_paths(x, "x")
        N, L, d = x.shape
        lam = torch.empty(N, device=x.device, dtype=x.dtype)
        iters = torch.empty(N, device=x.device, dtype=torch.int32) if want_iters else None
        if N == 0:
            return lam, iters
        dt = _dtype_code(x)
        order = self.dyadic_order
        with torch.cuda.device(x.device):
            if _is_fused_linear(self.static_kernel):
                x = x.contiguous()
                scale = float(self.static_kernel.scale)
                ws, nws = _workspace(_lib.SIGK_OP_NORMALIZE, N, N, L, L, d, order, dt, _lib.SIGK_PREC_FP64,
                                     x.device)
                if normalizer is log_normalizer:
                    _lib.call("sigk_normalize", _ptr(x), N, L, d, dt, order, scale, None, None, float(tol),
                              int(maxit), _ptr(lam), _ptr(iters), _ptr(ws), nws, _stream())
                    return lam, iters
                knorm = torch.empty(N, device=x.device, dtype=torch.float64)
                _lib.call("sigk_self_norms", _ptr(x), N, L, d, dt, order, scale, _ptr(knorm), _ptr(ws), nws,
                          _stream())
                fnorm = torch.as_tensor(normalizer(knorm), dtype=torch.float64, device=x.device).contiguous()
                _lib.call("sigk_normalize", _ptr(x), N, L, d, dt, order, scale, _ptr(knorm), _ptr(fnorm),
                          float(tol), int(maxit), _ptr(lam), _ptr(iters), _ptr(ws), nws, _stream())
                return lam, iters
            # generic static kernel: torch builds the self-increments, in float64
            for s0, s1 in _batches(N, max_batch):
                inc = pairwise_inner_product(x[s0:s1], x[s0:s1], self.static_kernel, order).to(torch.float64)
                nb, nc, _ = inc.shape
                knorm = torch.empty(nb, device=x.device, dtype=torch.float64)
                ws, nws = _workspace(_lib.SIGK_OP_NORMALIZE, nb, nb, nc + 1, nc + 1, 0, order, _lib.SIGK_F64,
                                     _lib.SIGK_PREC_FP64, x.device)
                _lib.call("sigk_pairwise_inc", _ptr(inc), nb, nc, nc, inc.stride(0), inc.stride(1), inc.stride(2),
                          _lib.SIGK_F64, order, None, None, _ptr(knorm), _lib.SIGK_PREC_FP64, _ptr(ws), nws,
                          _stream())
                knorm = torch.where(torch.isnan(knorm), torch.full_like(knorm, math.inf), knorm)
                fnorm = torch.as_tensor(normalizer(knorm), dtype=torch.float64, device=x.device).contiguous()
                lam64 = torch.empty(nb, device=x.device, dtype=torch.float64)
                _lib.call("sigk_normalize_inc", _ptr(inc), nb, nc, inc.stride(0), inc.stride(1), inc.stride(2),
                          _lib.SIGK_F64, order, _ptr(knorm), _ptr(fnorm), float(tol), int(maxit), _ptr(lam64),
                          None if iters is None else _ptr(iters[s0:s1]), _ptr(ws), nws, _stream())
                lam[s0:s1] = lam64.to(x.dtype)
        return lam, iters

    def pairwise(self, x, y=None, normalizer=None, tol=1e-8, maxit=100, max_batch=1000, max_threads=1024):
        """Robust pairwise kernel (sigpde/torch/kernel.py:232-291)."""
        solver = SigPDE(self.static_kernel, self.dyadic_order, self.precision)
        if _wants_grad(x, y):
            lx = _RobustLambda.apply(x, self, normalizer, tol, maxit, max_batch)
            if y is None:
                return solver.pairwise(x, None, lx, None, max_batch, max_threads)
            ly = _RobustLambda.apply(y, self, normalizer, tol, maxit, max_batch)
            return solver.pairwise(x, y, lx, ly, max_batch, max_threads)
        lx = self.normalization(x, normalizer, tol, maxit, max_batch, max_threads)
        if y is None:
            return solver.pairwise(x, None, lx, None, max_batch, max_threads)
        ly = self.normalization(y, normalizer, tol, maxit, max_batch, max_threads)
        return solver.pairwise(x, y, lx, ly, max_batch, max_threads)

    def gram(self, x, y=None, x_scale=None, y_scale=None, normalizer=None, tol=1e-8, maxit=100, max_batch=1000,
             max_threads=1024):
        """Robust Gram (sigpde/torch/kernel.py:293-301): given scales skip the normalisation."""
        if _wants_grad(x, y):
            xs = _RobustLambda.apply(x, self, normalizer, tol, maxit, max_batch) if x_scale is None else x_scale
            ys = None
            if y is not None:
                ys = _RobustLambda.apply(y, self, normalizer, tol, maxit, max_batch) if y_scale is None else y_scale
            solver = SigPDE(self.static_kernel, self.dyadic_order, self.precision)
            return solver.gram(x, y, xs, ys, max_batch, max_threads)
        xs = self.normalization(x, normalizer, tol, maxit, max_batch, max_threads) if x_scale is None else x_scale
        if y is None:
            ys = None
        else:
            ys = self.normalization(y, normalizer, tol, maxit, max_batch, max_threads) if y_scale is None else y_scale
        solver = SigPDE(self.static_kernel, self.dyadic_order, self.precision)
        return solver.gram(x, y, xs, ys, max_batch, max_threads)
