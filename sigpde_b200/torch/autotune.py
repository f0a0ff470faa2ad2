"""Autotuner for uneven batches (the ragged launch of ragged.py).

Three knobs, all chosen by measurement on the current device:

* increment source and tile shape, per (dimension bucket, precision): the
  increments of all pairs from one GEMM into per-pair blocks ("matrix": the
  split-TF32 tensor-core GEMM for tc32 / tc64, in 128 x 256 or 128 x 128
  tiles, or the FP64 GEMM for fp64) or formed inside the wavefront from
  staged differences on the CUDA cores ("fused").  Timed on the batch's own
  shape with synthetic values; the faster wins.
* warps per pair, per (ceil(log2 n), ceil(log2 d), order) bucket, n the
  pair's refined rows: the ragged launch cuts pair b into ceil(n / (32 R))
  bands of 32 R rows, one warp each, pipelined; R (rows per lane) in
  {2, 4, 8, 16} sets the band count.  Few bands mean little pipeline overhead
  but long pairs that finish late; many bands mean more overlap but more
  boundary traffic and waiting.  Each bucket is timed on a synthetic batch
  of that bucket with every valid R.
* the dyadic unroll is not a knob here: every wavefront step advances one
  coarse column (2^order refined columns, 8 above order 3), because the
  stencil coefficients are hoisted per coarse cell and a step's R x 2^order
  block shares them; a partial coarse column per step would recompute them.

Rows per lane and tile width change which warp or tile computes a value, not
its arithmetic, so results are bitwise the same for every choice; the source
changes the increment arithmetic (float64 dot products instead of tensor-core
ones, or summed in another place) within the precision's stated tolerance.

    from sigpde_b200.torch import autotune, ragged
    tuner = autotune.RaggedTuner(dim=32, precision="tc64")
    solver = ragged.RaggedPairwise(lx, ly, orders, 32, precision="tc64", tuner=tuner)
    tuner.save("ragged_tuning.json")      # reload with RaggedTuner(..., cache=path)

The fixed heuristics this replaces are the reference's threads-per-block and
rows-per-thread rule (sigpde/PDESolvers.py:30-35, sigpde/utils.py:3-19).
"""
from __future__ import annotations

import json
import math
import os
import statistics

import torch

__all__ = ["RaggedTuner", "bucket_of", "candidates", "dim_bucket"]

ROWS = (2, 4, 8, 16)
MAX_BANDS = 64
TILE_NS = (256, 128)


def dim_bucket(d: int) -> int:
    """ceil(log2 d): 1 for d <= 2, 3 for d in (4, 8], 5 for d in (16, 32], ..."""
    return max(int(math.ceil(math.log2(max(int(d), 2)))), 1)


def bucket_of(n: int, order: int, dim: int = 8):
    """Bucket key of a pair with n refined rows: (ceil(log2 n), ceil(log2 d), min(order, 4))."""
    return (max(int(math.ceil(math.log2(max(n, 2)))), 1), dim_bucket(dim), min(int(order), 4))


def candidates(n: int):
    """Rows per lane worth trying for n refined rows: every R of 2, 4, 8, 16
    whose band count stays within MAX_BANDS (a lone warp per pair at most 16
    rows a lane; more rows than needed to cover n in one band add nothing)."""
    out = []
    for R in ROWS:
        bands = -(-n // (32 * R))
        if bands > MAX_BANDS:
            continue
        if R > 2 and -(-n // (32 * (R // 2))) == 1:
            continue  # R/2 already covers n in one band
        out.append(R)
    return out or [16]


def source_candidates(precision: str, dim: int):
    """(source, tile_n) pairs a batch of this precision and dimension can take."""
    out = []
    if precision in ("tc32", "tc64") and dim <= 32:
        out += [("matrix", t) for t in TILE_NS]
    elif precision == "fp64":
        out.append(("matrix", 256))
    out.append(("fused", 256))
    return out


class RaggedTuner:
    """Measured choices for one dimension and precision: the batch-level
    increment source and tile width, and rows per lane per bucket."""

    def __init__(self, dim, precision="fp64", dtype=torch.float32, device="cuda", pairs_per_bucket=None,
                 cache=None):
        self.dim = int(dim)
        self.precision = precision
        self.dtype = dtype
        self.device = torch.device(device)
        self.pairs_per_bucket = pairs_per_bucket
        self.table = {}        # bucket -> rows per lane
        self.batch = {}        # dim bucket -> {"source": ..., "tile_n": ...}
        self.timings = {}      # bucket -> {R: ms}
        self.batch_timings = {}  # dim bucket -> {"source/tile_n": ms}
        if cache and os.path.exists(cache):
            self.load(cache)

    # ------------------------------------------------------------------ tables
    def choice(self):
        """The batch-level choice for this dimension (the default rule if not tuned)."""
        from .ragged import default_source
        return self.batch.get(dim_bucket(self.dim), {"source": default_source(self.precision, self.dim),
                                                     "tile_n": 256})

    def rows_for(self, n, order):
        """Tuned R for a pair with n refined rows at this order (the planner's
        default rule for buckets that were not tuned)."""
        from .ragged import rows_per_lane
        key = bucket_of(n, order, self.dim)
        if key in self.table:
            R = self.table[key]
            if R in ROWS:
                return R
        tsize = 8 if self.precision in ("fp64", "tc64") else 4
        staged = self.choice()["source"] == "fused"
        return rows_per_lane(n, self.dim, order, tsize, staged)

    def save(self, path):
        data = {"dim": self.dim, "precision": self.precision, "device": torch.cuda.get_device_name(self.device),
                "batch": [[k, v["source"], v["tile_n"]] for k, v in sorted(self.batch.items())],
                "table": [[k[0], k[1], k[2], v] for k, v in sorted(self.table.items())],
                "timings_ms": [[k[0], k[1], k[2], {str(r): t for r, t in v.items()}] for k, v in
                               sorted(self.timings.items())],
                "batch_timings_ms": [[k, v] for k, v in sorted(self.batch_timings.items())]}
        with open(path, "w") as f:
            json.dump(data, f, indent=1)

    def load(self, path):
        with open(path) as f:
            data = json.load(f)
        if data.get("dim") != self.dim or data.get("precision") != self.precision:
            return
        self.table = {(int(a), int(b), int(c)): int(r) for a, b, c, r in data.get("table", [])}
        self.batch = {int(k): {"source": s, "tile_n": int(t)} for k, s, t in data.get("batch", [])}

    def report(self):
        """Human-readable table of the choices (for logs and bench output)."""
        return {"dim_bucket": dim_bucket(self.dim), "precision": self.precision, **self.choice(),
                "rows_per_lane": {f"n<=2^{k[0]},d<=2^{k[1]},order={k[2]}": v for k, v in sorted(self.table.items())}}

    # ------------------------------------------------------------------ measurement
    def tune_for(self, x_lengths, y_lengths, orders):
        """Tune the batch-level choice (once per dimension bucket) and every
        bucket the batch uses that has not been tuned yet; returns the choice."""
        db = dim_bucket(self.dim)
        if db not in self.batch:
            self.batch[db] = self._tune_source(x_lengths, y_lengths, orders)
        need = {}
        for lx, ly, o in zip(x_lengths, y_lengths, orders):
            n = (min(int(lx), int(ly)) - 1) << int(o)
            key = bucket_of(n, o, self.dim)
            if key not in self.table:
                # representative pair of the bucket: its largest n, the batch's longer side at most
                m = (max(int(lx), int(ly)) - 1) << int(o)
                prev = need.get(key)
                if prev is None or n > prev[0]:
                    need[key] = (n, m, int(o))
        for key, (n, m, o) in sorted(need.items()):
            self.table[key] = self._tune_one(key, n, m, o)
        return self.choice()

    def _time(self, solver, reps=3):
        solver.solve()
        torch.cuda.synchronize(self.device)
        ts = []
        for _ in range(reps):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            solver.solve()
            e.record()
            e.synchronize()
            ts.append(s.elapsed_time(e))
        return statistics.median(ts)

    def _paths(self, lengths, seed):
        gen = torch.Generator(device="cpu").manual_seed(seed)
        out = []
        for L in lengths:
            p = torch.randn(int(L), self.dim, generator=gen, dtype=torch.float64).cumsum(0).mul(1 / math.sqrt(L))
            out.append(p.to(self.device, self.dtype))
        return out

    def _tune_source(self, x_lengths, y_lengths, orders):
        from .ragged import RaggedPairwise
        cands = source_candidates(self.precision, self.dim)
        if len(cands) == 1:
            return {"source": cands[0][0], "tile_n": cands[0][1]}
        xs = self._paths(x_lengths, 4321)
        ys = self._paths(y_lengths, 8765)
        best, best_t, times = None, math.inf, {}
        for source, tile_n in cands:
            solver = RaggedPairwise(x_lengths, y_lengths, orders, self.dim, self.dtype, self.device, self.precision,
                                    source=source, tile_n=tile_n)
            solver.load(xs, ys)
            t = self._time(solver)
            times[f"{source}/{tile_n}"] = t
            if t < best_t:
                best, best_t = {"source": source, "tile_n": tile_n}, t
            del solver
        self.batch_timings[dim_bucket(self.dim)] = times
        return best

    def _tune_one(self, key, n, m, order):
        from .ragged import RaggedPairwise
        cands = candidates(n)
        if len(cands) == 1:
            return cands[0]
        lx = (n >> order) + 1
        ly = max((m >> order) + 1, lx)
        # enough pairs to fill the device once with single-band work
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        P = self.pairs_per_bucket or max(sms * 8, 256)
        X = self._paths([lx, lx], 1234 + 31 * key[0] + 7 * key[1] + key[2])
        Y = self._paths([ly, ly], 5678 + 31 * key[0] + 7 * key[1] + key[2])
        xs = [X[i % 2] for i in range(P)]
        ys = [Y[i % 2] for i in range(P)]
        ch = self.choice()
        best, best_t = cands[0], math.inf
        times = {}
        for R in cands:
            solver = RaggedPairwise([lx] * P, [ly] * P, [order] * P, self.dim, self.dtype, self.device,
                                    self.precision, rows_fn=lambda a, o, R=R: R, source=ch["source"],
                                    tile_n=ch["tile_n"])
            solver.load(xs, ys)
            t = self._time(solver)
            times[R] = t
            if t < best_t:
                best, best_t = R, t
        self.timings[key] = times
        return best
