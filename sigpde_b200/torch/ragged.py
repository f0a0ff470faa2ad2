"""Uneven batched pairwise signature kernels (one persistent launch).

The reference solves a batch with one `SigPDE.pairwise` call per shape: every
path in a call has the same length and the whole call one dyadic order
(sigpde/torch/kernel.py:31-65).  A batch of pairs with their own lengths and
orders therefore costs it one call per (len x, len y, order) bucket.  Here the
pairs go in one launch of `sigk_pairwise_ragged`: paths are packed back to
back and each pair is cut into bands of rows; warps take bands longest pair
first from a work counter, so a long pair runs on several warps at once as a
pipeline while short pairs fill the rest of the GPU.  The plan (rows per lane,
bands, boundary-buffer offsets, item order) is built here once per batch shape.

    from sigpde_b200.torch import ragged
    k = ragged.pairwise(x_paths, y_paths, orders)          # lists of (L_b, d) tensors

`RaggedPairwise` keeps the packed layout, the work order and the workspace of
one batch shape, and can capture the launch in a CUDA graph for repeated
solves of new values with the same shapes (for example a serving loop).
"""
from __future__ import annotations

import torch

from .. import _lib
from .kernel import _PREC, _dtype_code, _is_fused_linear, _ptr, _stream

__all__ = ["pack", "pairwise", "RaggedPairwise"]


def pack(paths, dtype=None, device=None):
    """Pack a list of (L_i, d) paths into (sum L_i, d) plus int64 offsets and lengths."""
    if len(paths) == 0:
        raise ValueError("no paths")
    d = paths[0].shape[-1]
    dtype = paths[0].dtype if dtype is None else dtype
    device = paths[0].device if device is None else device
    lens = [int(p.shape[0]) for p in paths]
    for p in paths:
        if p.dim() != 2 or p.shape[1] != d:
            raise ValueError("every path must be a (length, dim) tensor with the same dim")
    packed = torch.cat([p.to(device=device, dtype=dtype) for p in paths], 0).contiguous()
    lengths = torch.tensor(lens, dtype=torch.int64)
    offsets = torch.zeros_like(lengths)
    offsets[1:] = torch.cumsum(lengths, 0)[:-1]
    return packed, offsets.to(device), lengths.to(device), lens


STAGE_BYTES_PER_WARP = 16 * 1024  # the kernel's dx staging budget per warp
MAT64_MIN_DIM = 16                # fp64 batches of this dimension or more take the float64 increment matrix


def rows_per_lane(n, d, order, tsize, staged=True):
    """Rows per lane R for a pair with n refined rows: the smallest of 2, 4, 8,
    16 covering the rows in one band of 32 R; with `staged` (increments formed
    from staged differences) shrunk while the lane's dx tile (coarse rows per
    lane x d) does not fit the kernel's staging budget."""
    R = 2 if n <= 64 else 4 if n <= 128 else 8 if n <= 256 else 16
    if not staged:
        return R
    cap = STAGE_BYTES_PER_WARP // tsize
    while R > 2:
        rc = 1 if order >= 4 else max(R >> order, 1)
        if rc * d * 32 <= cap:
            break
        R >>= 1
    return R


def staging_fits(R, d, order, tsize):
    """Whether the lane's dx tile of rows-per-lane R fits the staging budget."""
    rc = 1 if order >= 4 else max(R >> order, 1)
    return rc * d * 32 <= STAGE_BYTES_PER_WARP // tsize


def tc_plan(x_lengths, y_lengths, tile_m=128, tile_n=256):
    """Tensor-core plan of a ragged batch (sigk_ragged_tc_plan in include/sigk.h):
    operand-image rows and increment-block offsets per pair, and the GEMM tiles."""
    import numpy as np
    lx = np.asarray(x_lengths, np.int64)
    ly = np.asarray(y_lengths, np.int64)
    rows = np.minimum(lx, ly) - 1       # the row path is the shorter one
    cols = np.maximum(lx, ly) - 1
    r8 = (rows + 7) // 8 * 8
    c8 = (cols + 7) // 8 * 8
    ld = (rows + 3) // 4 * 4
    a_row0 = np.zeros_like(rows)
    a_row0[1:] = np.cumsum(r8)[:-1]
    b_row0 = np.zeros_like(cols)
    b_row0[1:] = np.cumsum(c8)[:-1]
    blk = cols * ld
    inc_off = np.zeros_like(blk)
    inc_off[1:] = np.cumsum(blk)[:-1]
    # tiles (i, j) of every pair, i over 128-row blocks, j over 256-column blocks; largest pairs first
    ti = (rows + tile_m - 1) // tile_m
    tj = (cols + tile_n - 1) // tile_n
    order = np.argsort(-(rows * cols).astype(np.float64), kind="stable")
    cnt = (ti * tj)[order]
    pb = np.repeat(order, cnt)
    local = np.arange(int(cnt.sum()), dtype=np.int64) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    i = local // tj[pb]
    j = local - i * tj[pb]
    tiles = np.stack([a_row0[pb] + tile_m * i, b_row0[pb] + tile_n * j, np.minimum(tile_m, rows[pb] - tile_m * i),
                      np.minimum(tile_n, cols[pb] - tile_n * j), inc_off[pb] + tile_n * j * ld[pb] + tile_m * i,
                      ld[pb]], axis=1).astype(np.int64)
    return {"a_row0": a_row0, "b_row0": b_row0, "a_rows": int(r8.sum()) + tile_m, "b_rows": int(c8.sum()) + tile_n,
            "inc_off": inc_off, "inc_elems": int(blk.sum()), "tiles": tiles.reshape(-1, 6), "tile_n": int(tile_n)}


def default_source(precision, dim):
    """Where a batch's increments come from when nothing was tuned: a GEMM into
    per-pair blocks for the tensor-core precisions (dim <= 32) and for fp64 with
    dim >= MAT64_MIN_DIM (the d FMAs per coarse cell dominate the fused form
    there), else formed inside the wavefront."""
    if precision in ("tc32", "tc64"):
        return "matrix" if dim <= 32 else "fused"
    return "matrix" if precision == "fp64" and dim >= MAT64_MIN_DIM else "fused"


def plan(x_lengths, y_lengths, orders, dim, tsize, staged=True, rows_fn=None):
    """Band plan of a ragged batch (see sigk_pairwise_ragged in include/sigk.h).
    `staged`: increments are formed from staged differences (CUDA-core modes);
    `rows_fn(n, order)`: rows per lane chosen elsewhere (the autotuner), or None."""
    import numpy as np
    lx = np.asarray(x_lengths, np.int64)
    ly = np.asarray(y_lengths, np.int64)
    od = np.asarray(orders, np.int64)
    n = (np.minimum(lx, ly) - 1) << od
    m = (np.maximum(lx, ly) - 1) << od
    if rows_fn is not None:
        rows = np.array([rows_fn(int(a), int(o)) for a, o in zip(n, od)], np.int64)
    else:  # rows_per_lane, vectorised
        rows = np.where(n <= 64, 2, np.where(n <= 128, 4, np.where(n <= 256, 8, 16))).astype(np.int64)
        if staged:
            cap = STAGE_BYTES_PER_WARP // tsize
            for _ in range(3):
                rc = np.where(od >= 4, 1, np.maximum(rows >> np.minimum(od, 4), 1))
                shrink = (rows > 2) & (rc * dim * 32 > cap)
                rows = np.where(shrink, rows >> 1, rows)
    bands = (n + 32 * rows - 1) // (32 * rows)
    sizes = (bands - 1) * (m + 1)
    bnd_off = np.zeros_like(sizes)
    bnd_off[1:] = np.cumsum(sizes)[:-1]
    order_of_start = np.argsort(-(n * m).astype(np.float64), kind="stable")  # longest first
    item_pair = np.repeat(order_of_start, bands[order_of_start])
    item_band = np.concatenate([np.arange(bands[b]) for b in order_of_start]).astype(np.int64)
    return {"rows": rows, "bands": bands, "bnd_off": bnd_off, "bnd_elems": int(sizes.sum()),
            "item_pair": item_pair, "item_band": item_band}


class RaggedPairwise:
    """Solver for one ragged batch shape: packed inputs, work order and workspace
    are built once; `solve()` runs the launch (optionally replaying a captured
    CUDA graph).  `tuner` (autotune.RaggedTuner) or `rows_fn(n, order)` choose
    the rows per lane (hence bands) per pair instead of the default rule."""

    def __init__(self, x_lengths, y_lengths, orders, dim, dtype=torch.float32, device="cuda", precision="fp64",
                 static_scale=1.0, tuner=None, rows_fn=None, source=None, tile_n=None):
        if precision not in _PREC:
            raise ValueError(f"precision must be one of {sorted(_PREC)}")
        x_lengths = [int(v) for v in x_lengths]
        y_lengths = [int(v) for v in y_lengths]
        orders = [int(v) for v in orders]
        if not (len(x_lengths) == len(y_lengths) == len(orders)) or not x_lengths:
            raise ValueError("x_lengths, y_lengths and orders must be non-empty and of equal length")
        if min(x_lengths + y_lengths) < 2:
            raise ValueError("every path needs at least 2 points")
        if min(orders) < 0 or max(orders) > 12:
            raise ValueError("dyadic orders must lie in [0, 12]")
        self.device = torch.device(device)
        self.dtype = dtype
        self.dim = int(dim)
        self.n = len(orders)
        self.prec = _PREC[precision]
        self.static_scale = float(static_scale)
        xl = torch.tensor(x_lengths, dtype=torch.int64)
        yl = torch.tensor(y_lengths, dtype=torch.int64)
        xo = torch.zeros_like(xl)
        xo[1:] = torch.cumsum(xl, 0)[:-1]
        yo = torch.zeros_like(yl)
        yo[1:] = torch.cumsum(yl, 0)[:-1]
        od = torch.tensor(orders, dtype=torch.int32)
        self.x_len, self.y_len = xl.to(self.device), yl.to(self.device)
        self.x_off, self.y_off = xo.to(self.device), yo.to(self.device)
        self.order = od.to(self.device)
        tsize = 8 if precision in ("fp64", "tc64") else 4
        if tuner is not None:  # increment source, tile width and rows per lane from measurements (autotune.py)
            choice = tuner.tune_for(x_lengths, y_lengths, orders)
            source = choice["source"] if source is None else source
            tile_n = choice["tile_n"] if tile_n is None else tile_n
            if rows_fn is None:
                rows_fn = tuner.rows_for
        if source is None:
            source = default_source(precision, self.dim)
        if source not in ("matrix", "fused"):
            raise ValueError("source must be 'matrix' or 'fused'")
        # "matrix": the increments of all pairs from one GEMM into per-pair blocks (tensor cores for tc32 /
        # tc64 with dim <= 32, the FP64 GEMM for fp64), read by the wavefront; "fused": each lane forms its
        # increments from staged differences on the CUDA cores (the tensor-core precisions then keep their
        # cells, with float64 dot products)
        use_tc = source == "matrix" and (precision == "fp64" or (precision in ("tc32", "tc64") and self.dim <= 32))
        self.source = "matrix" if use_tc else "fused"
        if tile_n is None or not use_tc or precision == "fp64":
            tile_n = 256
        if tile_n not in (128, 256):
            raise ValueError("tile_n must be 128 or 256")
        self.tile_n = int(tile_n)
        pl = plan(x_lengths, y_lengths, orders, self.dim, tsize, staged=not use_tc, rows_fn=rows_fn)
        self.item_pair = torch.as_tensor(pl["item_pair"], device=self.device)
        self.item_band = torch.as_tensor(pl["item_band"], dtype=torch.int32, device=self.device)
        self.pair_rows = torch.as_tensor(pl["rows"], dtype=torch.int32, device=self.device)
        self.pair_bands = torch.as_tensor(pl["bands"], dtype=torch.int32, device=self.device)
        self.pair_bnd_off = torch.as_tensor(pl["bnd_off"], device=self.device)
        self.bnd_elems = pl["bnd_elems"]
        self.nitems = int(pl["item_pair"].shape[0])
        self.x_pack = torch.zeros((int(xl.sum()), self.dim), dtype=dtype, device=self.device)
        self.y_pack = torch.zeros((int(yl.sum()), self.dim), dtype=dtype, device=self.device)
        self.out = torch.empty(self.n, dtype=dtype, device=self.device)
        self.x_points = int(xl.sum())
        self.y_points = int(yl.sum())
        self.tc = None
        if use_tc:
            tp = tc_plan(x_lengths, y_lengths, tile_n=self.tile_n)
            self._tc_arrays = {k: torch.as_tensor(tp[k], device=self.device)
                               for k in ("a_row0", "b_row0", "inc_off", "tiles")}
            self.tc = _lib.RaggedTcPlan(_ptr(self._tc_arrays["a_row0"]), _ptr(self._tc_arrays["b_row0"]), tp["a_rows"],
                                        tp["b_rows"], _ptr(self._tc_arrays["inc_off"]), tp["inc_elems"],
                                        _ptr(self._tc_arrays["tiles"]), int(tp["tiles"].shape[0]), self.tile_n)
            nws = _lib.lib().sigk_ragged_tc_workspace_size(self.n, self.dim, self.nitems, self.bnd_elems, self.prec,
                                                           self.tc)
        else:
            nws = _lib.lib().sigk_ragged_workspace_size(self.n, self.x_points, self.y_points, self.dim, self.nitems,
                                                        self.bnd_elems, self.prec)
        self.ws = torch.empty(nws, dtype=torch.uint8, device=self.device)
        self.x_scale = None
        self.y_scale = None
        self.graph = None

    def load_packed(self, x_pack, y_pack, x_scale=None, y_scale=None):
        """Copy already packed paths ((x_points, dim) and (y_points, dim), same layout as `pack`)."""
        self.x_pack.copy_(x_pack)
        self.y_pack.copy_(y_pack)
        self.x_scale = self._scale_buffer(self.x_scale, x_scale)
        self.y_scale = self._scale_buffer(self.y_scale, y_scale)

    def load(self, x_paths, y_paths, x_scale=None, y_scale=None):
        """Copy new path values (same shapes) into the packed buffers."""
        torch.cat([p.to(self.device, self.dtype) for p in x_paths], 0, out=self.x_pack)
        torch.cat([p.to(self.device, self.dtype) for p in y_paths], 0, out=self.y_pack)
        self.x_scale = self._scale_buffer(self.x_scale, x_scale)
        self.y_scale = self._scale_buffer(self.y_scale, y_scale)

    def _scale_buffer(self, buf, values):
        # new values go into the existing buffer, so a captured graph keeps reading the right memory
        if values is None:
            return None
        v = torch.as_tensor(values, dtype=self.dtype, device=self.device).reshape(-1)
        if buf is not None and buf.shape == v.shape:
            buf.copy_(v)
            return buf
        return v.clone()

    def _launch(self):
        args = (_ptr(self.x_pack), _ptr(self.x_off), _ptr(self.x_len), self.x_points, _ptr(self.y_pack),
                _ptr(self.y_off), _ptr(self.y_len), self.y_points, _ptr(self.order), _ptr(self.item_pair),
                _ptr(self.item_band), self.nitems, _ptr(self.pair_rows), _ptr(self.pair_bands),
                _ptr(self.pair_bnd_off), self.bnd_elems, self.n, self.dim, _dtype_code(self.x_pack),
                self.static_scale, _ptr(self.x_scale), _ptr(self.y_scale), _ptr(self.out), self.prec)
        if self.tc is not None:
            _lib.call("sigk_pairwise_ragged_tc", *args, self.tc, _ptr(self.ws), self.ws.numel(), _stream())
        else:
            _lib.call("sigk_pairwise_ragged", *args, _ptr(self.ws), self.ws.numel(), _stream())

    def capture(self):
        """Capture the launch (counter reset + kernel) in a CUDA graph; later
        `solve()` calls replay it.  Scales present at capture time stay bound."""
        self._launch()  # warm-up outside the capture (loads the module, sizes the grid)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        c0 = _lib.launch_count()
        with torch.cuda.graph(g):
            self._launch()
        self.graph_kernels = _lib.launch_count() - c0  # kernels each replay runs
        self.graph = g
        return self

    def error_flag(self):
        """Error word of the last launch (synchronises): bit 1 an item was refused,
        bit 2 a band wait ran out; 0 when every pair was solved."""
        return int(self.ws[8:12].view(torch.int32).item())

    def check(self):
        """Raise SigkError (SIGK_ETIMEDOUT / SIGK_EINVAL) if the last launch left a
        pair unsolved (its result is NaN); synchronises the current stream."""
        _lib.call("sigk_ragged_status", _ptr(self.ws), _stream())

    def solve(self):
        with torch.cuda.device(self.device):
            if self.graph is not None:
                self.graph.replay()
            else:
                self._launch()
        return self.out


def pairwise(x_paths, y_paths, orders, static_kernel=None, x_scale=None, y_scale=None, precision="fp64"):
    """k(x_b, y_b) for pairs with their own lengths and dyadic orders.

    x_paths, y_paths: lists of (L_b, d) CUDA tensors (float32 or float64);
    orders: list of ints.  Returns a (B,) tensor in the paths' dtype.
    """
    if static_kernel is not None and not _is_fused_linear(static_kernel):
        raise NotImplementedError("ragged batches support the linear static kernel")
    scale = 1.0 if static_kernel is None else float(static_kernel.scale)
    if not (len(x_paths) == len(y_paths) == len(orders)):
        raise ValueError("x_paths, y_paths and orders must have the same length")
    dev = x_paths[0].device
    if dev.type != "cuda":
        raise ValueError("paths must be CUDA tensors (this package has no CPU path)")
    dtype = x_paths[0].dtype
    _dtype_code(x_paths[0])
    solver = RaggedPairwise([p.shape[0] for p in x_paths], [p.shape[0] for p in y_paths], orders,
                            x_paths[0].shape[1], dtype, dev, precision, scale)
    solver.load(x_paths, y_paths, x_scale, y_scale)
    return solver.solve().clone()
