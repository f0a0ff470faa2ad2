"""Gram matrices sharded across GPUs (one process per GPU, torch.distributed).

Every Gram entry and every robust lambda is independent, so the work splits
with no exchange during the solve: each rank solves a block of Gram rows and
the blocks are all-gathered afterwards (NCCL over NVLink on GPUs; the payload
is the result itself, N_x * N_y values).  This distributes the host tile loop
of the reference (sigpde/torch/kernel.py:100-122 for the Gram, :143-169 for
the symmetric Gram) over ranks instead of over 32x32 tiles.

* Gram(x, y): rows of x are cut into `world` contiguous blocks of equal size.
* Symmetric Gram(x): rank r solves rows [r0, r1) of the lower triangle: the
  block left of its diagonal block as a Gram (columns [0, r0)) and the diagonal
  block as a symmetric Gram; the cut points balance the lower-triangle area,
  sum over rows of (i + 1), across ranks.  After the gather the lower triangle
  is mirrored, so the result is exactly symmetric.
* RobustSigPDE.gram(x[, y]): the paths' lambdas are computed in equal shards
  and all-gathered (N values) before the Gram rows are solved with them.

Inputs are replicated: every rank holds the full x (and y), which for this
path is small next to the Gram (paths of N x L x d against N^2 entries).

The hooks `solve(x_rows, y_cols, x_scale, y_scale) -> (rows, cols)` (y_cols
None: the symmetric Gram of x_rows, x_scale on both sides) and
`lam(x) -> (n,)` default to this package's CUDA engine; the host logic --
partition, collectives, assembly -- does not depend on them.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple

import torch
import torch.distributed as dist


def _world(group) -> Tuple[int, int]:
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def row_blocks(n: int, world: int) -> List[Tuple[int, int]]:
    """Equal contiguous row blocks [r0, r1) of n rows over `world` ranks."""
    q, r = divmod(n, world)
    out, s = [], 0
    for k in range(world):
        e = s + q + (1 if k < r else 0)
        out.append((s, e))
        s = e
    return out


def triangle_blocks(n: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous row blocks [r0, r1) of an n x n lower triangle whose areas
    (rows i contribute i + 1 entries) are as equal as the row boundaries allow."""
    total = n * (n + 1) // 2
    out, s = [], 0
    for k in range(world):
        if k == world - 1:
            e = n
        else:
            target = total * (k + 1) / world
            e = s
            while e < n and (e + 1) * (e + 2) // 2 <= target:
                e += 1
            # take the boundary that lands nearer the target
            if e < n and abs((e + 1) * (e + 2) / 2 - target) < abs(e * (e + 1) / 2 - target):
                e += 1
            e = max(e, s)
        out.append((s, e))
        s = e
    return out


def _gather_rows(block: torch.Tensor, blocks: List[Tuple[int, int]], ncols: int, group) -> torch.Tensor:
    """All-gather row blocks of different heights into the full (n, ncols) matrix."""
    rank, world = _world(group)
    if world == 1:
        return block
    hmax = max(e - s for s, e in blocks)
    buf = torch.zeros((hmax, ncols), dtype=block.dtype, device=block.device)
    buf[: block.shape[0], : block.shape[1]] = block
    parts = torch.empty((world * hmax, ncols), dtype=block.dtype, device=block.device)
    dist.all_gather_into_tensor(parts, buf, group=group)  # the ranks' buffers concatenated along rows
    parts = parts.view(world, hmax, ncols)
    return torch.cat([parts[k, : e - s] for k, (s, e) in enumerate(blocks)], 0)


def _gather_vec(part: torch.Tensor, blocks: List[Tuple[int, int]], group) -> torch.Tensor:
    rank, world = _world(group)
    if world == 1:
        return part
    hmax = max(e - s for s, e in blocks)
    buf = torch.zeros(hmax, dtype=part.dtype, device=part.device)
    buf[: part.shape[0]] = part
    parts = torch.empty(world * hmax, dtype=part.dtype, device=part.device)
    dist.all_gather_into_tensor(parts, buf, group=group)
    parts = parts.view(world, hmax)
    return torch.cat([parts[k, : e - s] for k, (s, e) in enumerate(blocks)], 0)


def _engine_gram(static_kernel, order: int, precision: str) -> Callable:
    from .torch import SigPDE

    solver = SigPDE(static_kernel, order, precision=precision)

    def gram(xr, yc, sx, sy):
        return solver.gram(xr, yc, sx, sy)

    return gram


def _engine_lam(static_kernel, order: int, normalizer, tol: float, maxit: int) -> Callable:
    from .torch import RobustSigPDE

    rk = RobustSigPDE(static_kernel, order, normalizer)

    def lam(x):
        return rk.normalization(x, tol=tol, maxit=maxit)

    return lam


def rank_rows(x: torch.Tensor, y: Optional[torch.Tensor], x_scale, y_scale, rank: int, world: int,
              solve: Callable):
    """The row blocks of all ranks and this rank's block of the Gram (the rows it
    solves, all columns; for a symmetric Gram the entries right of its diagonal
    block are zero)."""
    n = x.shape[0]
    if y is None:
        blocks = triangle_blocks(n, world)
        r0, r1 = blocks[rank]
        sx = None if x_scale is None else x_scale[r0:r1]
        block = torch.zeros((r1 - r0, n), dtype=x.dtype, device=x.device)
        if r1 > r0:
            if r0 > 0:  # the rows' part left of the diagonal block
                block[:, :r0] = solve(x[r0:r1], x[:r0], sx, None if x_scale is None else x_scale[:r0])
            block[:, r0:r1] = solve(x[r0:r1], None, sx, None)  # the diagonal block: a symmetric Gram
        return blocks, block
    blocks = row_blocks(n, world)
    r0, r1 = blocks[rank]
    sx = None if x_scale is None else x_scale[r0:r1]
    if r1 > r0:
        return blocks, solve(x[r0:r1], y, sx, y_scale)
    return blocks, torch.empty((0, y.shape[0]), dtype=x.dtype, device=x.device)


def assemble(full: torch.Tensor, symmetric: bool) -> torch.Tensor:
    """The gathered rows as the Gram: a symmetric Gram's lower triangle mirrored."""
    if not symmetric:
        return full
    return torch.tril(full) + torch.tril(full, -1).t()


def sharded_gram(x: torch.Tensor, y: Optional[torch.Tensor] = None, x_scale=None, y_scale=None, *,
                 static_kernel=None, dyadic_order: int = 0, precision: str = "fp64", group=None,
                 solve: Optional[Callable] = None) -> torch.Tensor:
    """SigPDE.gram(x, y, x_scale, y_scale) solved by all ranks of `group`
    together; every rank returns the full matrix.  Outside a process group it
    is the single-process Gram."""
    if solve is None:
        from .torch import kernels
        solve = _engine_gram(static_kernel or kernels.LinearKernel(), dyadic_order, precision)
    rank, world = _world(group)
    n = x.shape[0]
    if x_scale is not None and x_scale.numel() == 1:
        x_scale = x_scale.reshape(1).expand(n).contiguous()
    if y is not None and y_scale is not None and y_scale.numel() == 1:
        y_scale = y_scale.reshape(1).expand(y.shape[0]).contiguous()
    blocks, block = rank_rows(x, y, x_scale, y_scale, rank, world, solve)
    full = _gather_rows(block, blocks, n if y is None else y.shape[0], group)
    return assemble(full, y is None)


def sharded_robust_gram(x: torch.Tensor, y: Optional[torch.Tensor] = None, *, static_kernel=None,
                        dyadic_order: int = 0, normalizer=None, tol: float = 1e-8, maxit: int = 100,
                        precision: str = "fp64", group=None, solve: Optional[Callable] = None,
                        lam: Optional[Callable] = None) -> torch.Tensor:
    """RobustSigPDE.gram(x, y) solved by all ranks: lambdas in shards, all-gathered,
    then the Gram rows (sigpde/torch/kernel.py:293-301)."""
    from .torch import kernels

    sk = static_kernel or kernels.LinearKernel()
    if lam is None:
        lam = _engine_lam(sk, dyadic_order, normalizer, tol, maxit)
    rank, world = _world(group)

    def lambdas(p):
        blocks = row_blocks(p.shape[0], world)
        s, e = blocks[rank]
        part = lam(p[s:e]) if e > s else torch.empty(0, dtype=p.dtype, device=p.device)
        return _gather_vec(part, blocks, group)

    lx = lambdas(x)
    ly = None if y is None else lambdas(y)
    return sharded_gram(x, y, lx, ly, static_kernel=sk, dyadic_order=dyadic_order, precision=precision,
                        group=group, solve=solve)
