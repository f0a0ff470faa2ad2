"""Autotuner for uneven batches: rows per lane, hence bands (warps working on
one pair as a pipeline), per (refined-rows bucket, dyadic order).

The ragged launch cuts pair b into ceil(n_b / (32 R_b)) bands of 32 R_b rows.
Few bands mean little pipeline overhead but long pairs that finish late and
idle warps at the end; many bands mean more overlap but more boundary traffic
and waiting.  The best R depends on n, the order (columns per step), the cell
precision, where the increments come from and the device.  `RaggedTuner`
measures it: for each bucket it times a synthetic batch of pairs of that
bucket with every valid R (CUDA events, median of three runs after a warm-up)
and keeps the fastest.  Results are bitwise the same for every R (each cell is
computed by the same arithmetic from the same inputs; boundary rows are
passed in the cell precision), so tuning changes speed only.

    from sigpde_b200.torch import autotune, ragged
    tuner = autotune.RaggedTuner(dim=32, precision="tc64")
    solver = ragged.RaggedPairwise(lx, ly, orders, 32, precision="tc64", tuner=tuner)
    tuner.save("ragged_tuning.json")      # reload with RaggedTuner(..., cache=path)
"""
from __future__ import annotations

import json
import math
import os
import statistics

import torch

__all__ = ["RaggedTuner", "bucket_of", "candidates"]

ROWS = (2, 4, 8, 16)
MAX_BANDS = 64


def bucket_of(n: int, order: int):
    """Bucket key of a pair with n refined rows: (ceil(log2 n), min(order, 4))."""
    return (max(int(math.ceil(math.log2(max(n, 2)))), 1), min(int(order), 4))


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


class RaggedTuner:
    """Per-bucket rows-per-lane table, measured on the current device."""

    def __init__(self, dim, precision="fp64", dtype=torch.float32, device="cuda", pairs_per_bucket=None,
                 cache=None):
        self.dim = int(dim)
        self.precision = precision
        self.dtype = dtype
        self.device = torch.device(device)
        self.pairs_per_bucket = pairs_per_bucket
        self.table = {}
        self.timings = {}
        if cache and os.path.exists(cache):
            self.load(cache)

    # ------------------------------------------------------------------ table
    def rows_for(self, n, order):
        """Tuned R for a pair with n refined rows at this order (the planner's
        default rule for buckets that were not tuned)."""
        from .ragged import rows_per_lane
        key = bucket_of(n, order)
        if key in self.table:
            R = self.table[key]
            if R in ROWS:
                return R
        tsize = 8 if self.precision in ("fp64", "tc64") else 4
        from .ragged import MAT64_MIN_DIM
        staged = not ((self.precision in ("tc32", "tc64") and self.dim <= 32) or
                      (self.precision == "fp64" and self.dim >= MAT64_MIN_DIM))
        return rows_per_lane(n, self.dim, order, tsize, staged)

    def save(self, path):
        data = {"dim": self.dim, "precision": self.precision, "device": torch.cuda.get_device_name(self.device),
                "table": [[k[0], k[1], v] for k, v in sorted(self.table.items())],
                "timings_ms": [[k[0], k[1], {str(r): t for r, t in v.items()}] for k, v in
                               sorted(self.timings.items())]}
        with open(path, "w") as f:
            json.dump(data, f, indent=1)

    def load(self, path):
        with open(path) as f:
            data = json.load(f)
        if data.get("dim") != self.dim or data.get("precision") != self.precision:
            return
        self.table = {(int(a), int(b)): int(r) for a, b, r in data.get("table", [])}

    # ------------------------------------------------------------------ measurement
    def tune_for(self, x_lengths, y_lengths, orders):
        """Tune every bucket the batch uses and has not been tuned yet."""
        need = {}
        for lx, ly, o in zip(x_lengths, y_lengths, orders):
            n = (min(int(lx), int(ly)) - 1) << int(o)
            key = bucket_of(n, o)
            if key not in self.table:
                # representative pair of the bucket: its largest n, the batch's longer side at most
                m = (max(int(lx), int(ly)) - 1) << int(o)
                prev = need.get(key)
                if prev is None or n > prev[0]:
                    need[key] = (n, m, int(o))
        for key, (n, m, o) in sorted(need.items()):
            self.table[key] = self._tune_one(key, n, m, o)
        return self.table

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
        gen = torch.Generator(device="cpu").manual_seed(1234 + 31 * key[0] + key[1])
        X = [torch.randn(lx, self.dim, generator=gen, dtype=torch.float64).cumsum(0).mul(1 / math.sqrt(lx))
             for _ in range(2)]
        Y = [torch.randn(ly, self.dim, generator=gen, dtype=torch.float64).cumsum(0).mul(1 / math.sqrt(ly))
             for _ in range(2)]
        xs = [X[i % 2].to(self.device, self.dtype) for i in range(P)]
        ys = [Y[i % 2].to(self.device, self.dtype) for i in range(P)]
        best, best_t = cands[0], math.inf
        times = {}
        for R in cands:
            solver = RaggedPairwise([lx] * P, [ly] * P, [order] * P, self.dim, self.dtype, self.device,
                                    self.precision, rows_fn=lambda a, o, R=R: R)
            solver.load(xs, ys)
            t = self._time(solver)
            times[R] = t
            if t < best_t:
                best, best_t = R, t
        self.timings[key] = times
        return best
