"""Request server for signature-kernel Gram solves with continuous batching.

Requests (a Gram k(x_i, y_j), a symmetric Gram k(x_i, x_j), or a robust Gram
with per-path normalisation) arrive at any time.  A scheduler thread admits
them in arrival order as soon as two resources allow it:

* a slot: one of `max_inflight` CUDA streams is free;
* device memory: the request's footprint (paths, result, kernel workspace,
  robust scratch), estimated before admission, fits in the HBM budget next to
  the footprints of the requests already on the device.

With `batch_small=True`, small symmetric requests that wait together are
batched at the kernel level: the lower triangles of their Grams become the
pairs of ONE uneven-batch launch (sigpde_b200.torch.ragged: every pair with
its own path length and dyadic order; a robust request's lambdas become
per-pair scales), and the pair results are scattered back into each
request's matrix.  Results are bitwise those of the requests alone.  It is
off by default: the uneven-batch launch copies each path once per pair and
(tensor-core modes) gives every pair its own GEMM tiles, so on the measured
traces it is slower than running the small requests' own Gram launches
concurrently.

Among the requests waiting, the cheapest (fewest PDE cells) is admitted
first; a request that has waited longer than `max_wait_s` goes first
regardless, so nothing starves.  An admitted request is enqueued on its own
stream: host-to-device copy of its paths (pinned staging), the solve with the
kernel variant that fits its shape, and the device-to-host copy of the
result.  A large Gram is solved in row blocks of about `chunk_cells` cells,
one launch each: a persistent kernel holds every SM until it ends, so
chunking lets requests admitted meanwhile get SMs between chunks instead of
waiting for the whole large request.  Requests admitted while others are
running execute concurrently on the device, and copies overlap compute.  Completion
is detected with CUDA events; the result, the timestamps (arrival, admission,
completion) and any error are delivered on the request's handle.

Paths can be kept resident: `put(name, paths)` copies a path set to the
device once and returns a PathSet that requests name as x or y.  Such
requests skip the copy-in, are not charged for the paths (the store's bytes
come out of the budget once), and robust requests on the set compute its
normalisation scales once per (dyadic order, precision): later requests wait
for the event of the stream that wrote them and reuse them.

Every solve is deterministic and a request's kernels only read its own
buffers (and stored paths and scales, which nothing overwrites), so a
request's result does not depend on what else is in flight.

`serve_sequential` runs the same requests one at a time (copy in, solve, copy
out, synchronise) -- the per-request plain-launch baseline.
"""
from __future__ import annotations

import collections
import dataclasses
import queue
import threading
import time
from typing import Optional

import torch

from . import _lib
from .torch import kernel as _k
from .torch import static_kernels as _sk

__all__ = ["GramRequest", "RequestHandle", "GramServer", "PathSet", "serve_sequential", "footprint_bytes",
           "request_cells", "request_pairs", "batch_footprint_bytes"]


class PathSet:
    """Paths resident on the server's device (GramServer.put).  A request names
    a PathSet as its x or y instead of a tensor: the paths are not copied per
    request and not charged to the request's footprint (the store holds them
    once), and robust requests reuse the set's normalisation scales per
    (dyadic order, precision) -- computed by the first robust request that
    needs them, on its stream, and read by later ones after waiting for that
    stream's event.  `host` keeps a pinned copy for per-request baselines."""

    def __init__(self, name, tensor: torch.Tensor, host: torch.Tensor):
        self.name = name
        self.tensor = tensor
        self.host = host
        self.nbytes = tensor.numel() * tensor.element_size()
        self.lam_hits = 0
        self.lam_misses = 0
        self._lam = {}  # (order, precision) -> (scales, event recorded after they were written)
        self._lock = threading.Lock()

    @property
    def shape(self):
        return self.tensor.shape

    @property
    def dtype(self):
        return self.tensor.dtype

    def dim(self):
        return self.tensor.dim()

    def element_size(self):
        return self.tensor.element_size()

    def numel(self):
        return self.tensor.numel()

    def scales(self, rk, order: int, precision: str, stream, use_cache: bool = True):
        """Normalisation scales of the set (RobustSigPDE.normalization), enqueued on `stream`."""
        if not use_cache:
            return rk.normalization(self.tensor)
        key = (int(order), precision)
        with self._lock:
            hit = self._lam.get(key)
            if hit is not None:
                self.lam_hits += 1
        if hit is not None:
            lam, ev = hit
            stream.wait_event(ev)
            return lam
        lam = rk.normalization(self.tensor)
        ev = torch.cuda.Event()
        ev.record(stream)
        with self._lock:
            self._lam.setdefault(key, (lam, ev))
            self.lam_misses += 1
        return lam


def _resident(t) -> bool:
    return isinstance(t, PathSet)


def _on_device(t, device, use_host: bool = False):
    """The request operand on the device: a PathSet's resident tensor (or, for a baseline that copies
    per request, its pinned host copy sent over), else the tensor copied in (no copy if already there)."""
    if _resident(t):
        return t.host.to(device, non_blocking=True) if use_host else t.tensor
    return t.to(device, non_blocking=True)


@dataclasses.dataclass
class GramRequest:
    """One request.  x (and y) are (N, L, d) float32/float64 tensors, on the
    host (pinned or pageable) or on the device, or PathSets resident in the
    server's store.  kind: "gram" (k(x_i, y_j), or the symmetric Gram when y
    is None) or "robust" (RobustSigPDE.gram with the default normaliser)."""

    x: torch.Tensor
    y: Optional[torch.Tensor] = None
    order: int = 0
    kind: str = "gram"
    rid: int = -1
    arrival: float = 0.0  # seconds on the server's clock (time.perf_counter)


class RequestHandle:
    """Result of one request: `wait()` returns the (Nx, Ny) host tensor or raises."""

    def __init__(self, req: GramRequest):
        self.req = req
        self._done = threading.Event()
        self.cost = 0
        self.result: Optional[torch.Tensor] = None
        self.error: Optional[BaseException] = None
        self.t_admit = None
        self.t_done = None

    def _finish(self, result=None, error=None):
        self.result = result
        self.error = error
        self.t_done = time.perf_counter()
        self._done.set()

    def done(self) -> bool:
        return self._done.is_set()

    def wait(self, timeout=None):
        if not self._done.wait(timeout):
            raise TimeoutError(f"request {self.req.rid} not finished")
        if self.error is not None:
            raise self.error
        return self.result

    @property
    def latency(self) -> Optional[float]:
        return None if self.t_done is None else self.t_done - self.req.arrival


def footprint_bytes(req: GramRequest, precision: str = "fp64") -> int:
    """Device bytes a request holds while in flight (paths, result, workspace, robust scratch)."""
    x = req.x
    y = x if req.y is None else req.y
    nx, lx, d = x.shape
    ny, ly = y.shape[0], y.shape[1]
    es = x.element_size()
    prec = _k._PREC[precision]
    dt = _k._dtype_code(x)
    sym = req.y is None
    op = _lib.SIGK_OP_GRAM_SYM if sym else _lib.SIGK_OP_GRAM
    ws = _lib.lib().sigk_workspace_size(op, nx, ny, lx, ly, d, req.order, dt, prec)
    # resident paths are held by the server's store, not by the request
    paths = (0 if _resident(x) else x.numel() * es) + (0 if sym or _resident(y) else y.numel() * es)
    total = paths + nx * ny * es + ws
    if req.kind == "robust":
        nws = _lib.lib().sigk_workspace_size(_lib.SIGK_OP_NORMALIZE, nx, nx, lx, lx, d, req.order, dt, prec)
        total += nws + (nx + ny) * (8 + es)
    return int(total)


class _Inflight:
    """One admitted unit: a single request, or a batch of small requests solved by one launch."""
    __slots__ = ("handles", "stream", "event", "bytes", "out_hosts", "keep")

    def __init__(self, handles, stream, event, nbytes, out_hosts, keep):
        self.handles = handles
        self.stream = stream
        self.event = event
        self.bytes = nbytes
        self.out_hosts = out_hosts
        self.keep = keep


def request_pairs(req: GramRequest) -> int:
    """PDE solves of a request (the lower triangle, diagonal included, for a symmetric Gram)."""
    nx = int(req.x.shape[0])
    return nx * (nx + 1) // 2 if req.y is None else nx * int(req.y.shape[0])


def batch_footprint_bytes(reqs, precision: str = "fp64") -> int:
    """Device bytes of a batch of small symmetric requests solved by one ragged launch (an upper
    estimate): the paths, the per-pair path packs and their differences or tensor-core operands and
    increment blocks, the band boundary rows, the pair results and the Gram results."""
    total = 0
    tc = precision in ("tc32", "tc64")
    for r in reqs:
        N, L, d = r.x.shape
        es = r.x.element_size()
        P = N * (N + 1) // 2
        n = (L - 1) << r.order
        bands = -(-n // 512)
        total += r.x.numel() * es + N * N * es + 2 * P * (es + 8) + 8 * P * 4
        total += 2 * P * L * d * es                      # x and y packs
        if tc:
            kp = (d + 7) // 8 * 8
            total += P * (L - 1) * ((L - 1 + 3) // 4 * 4) * 4 + 4 * P * (L + 8) * kp * 4
        else:
            total += 2 * P * (L - 1) * d * 8
        total += P * max(bands - 1, 0) * (n + 1) * 8 + 4 * P * bands
    return int(total + (64 << 20))  # plus the tile table, images' tile padding and counters


def _solve_batch_on_stream(reqs, precision: str, device, stream):
    """Enqueue several small symmetric requests as ONE uneven-batch launch on `stream`: the lower
    triangle of every request's Gram becomes pairs of one ragged batch (paths of their own length
    and dyadic order; robust requests bring their lambdas as per-pair scales), and the pair results
    are scattered back into each request's matrix.  Returns (pinned host results, keep-alive)."""
    import numpy as np
    from .torch import ragged as _rg
    with torch.cuda.stream(stream):
        xs, parts_x, parts_y, sx_parts, sy_parts, lens, ords, tris = [], [], [], [], [], [], [], []
        for r in reqs:
            if r.kind not in ("gram", "robust") or r.y is not None:
                raise ValueError("only symmetric gram / robust requests are batched")
            x = _on_device(r.x, device)
            N, L, d = x.shape
            ii, jj = torch.tril_indices(N, N, device=device)  # i >= j: x_i on the rows, as the symmetric Gram
            if r.kind == "robust":
                rk = _k.RobustSigPDE(_sk.LinearKernel(), r.order, precision=precision)
                lam = r.x.scales(rk, r.order, precision, stream) if _resident(r.x) else rk.normalization(x)
                sx_parts.append(lam.index_select(0, ii))
                sy_parts.append(lam.index_select(0, jj))
            else:
                one = torch.ones(ii.numel(), dtype=x.dtype, device=device)
                sx_parts.append(one)
                sy_parts.append(one)
            parts_x.append(x.index_select(0, ii).reshape(-1, d))
            parts_y.append(x.index_select(0, jj).reshape(-1, d))
            P = int(ii.numel())
            lens.append(np.full(P, L, np.int64))
            ords.append(np.full(P, r.order, np.int64))
            xs.append(x)
            tris.append((N, ii, jj, P))
        lens = np.concatenate(lens)
        ords = np.concatenate(ords)
        solver = _rg.RaggedPairwise(lens, lens, ords, xs[0].shape[2], xs[0].dtype, device, precision)
        solver.load_packed(torch.cat(parts_x), torch.cat(parts_y), torch.cat(sx_parts), torch.cat(sy_parts))
        out = solver.solve()
        hosts, results = [], []
        off = 0
        for N, ii, jj, P in tris:
            v = out[off:off + P]
            off += P
            res = torch.empty((N, N), dtype=out.dtype, device=device)
            res[ii, jj] = v
            res[jj, ii] = v
            host = torch.empty((N, N), dtype=out.dtype, pin_memory=True)
            host.copy_(res, non_blocking=True)
            hosts.append(host)
            results.append(res)
    return hosts, (xs, parts_x, parts_y, sx_parts, sy_parts, solver, out, results, tris)


def request_cells(req: GramRequest) -> int:
    """Refined PDE cells of a request (its cost, for ordering and chunking)."""
    x = req.x
    y = x if req.y is None else req.y
    n = (x.shape[1] - 1) << req.order
    m = (y.shape[1] - 1) << req.order
    return int(x.shape[0]) * int(y.shape[0]) * n * m


def _solve_on_stream(req: GramRequest, precision: str, device, stream, chunk_cells: int = 0, staging=None,
                     use_store: bool = True):
    """Enqueue copy-in, solve and copy-out of one request on `stream`.
    Returns (pinned host result, tensors to keep alive until the event).
    chunk_cells > 0 splits a large (non-symmetric or robust) Gram into row
    blocks of about that many cells, one launch each.  use_store=False treats
    a PathSet operand like a host tensor (copied in, scales recomputed): the
    per-request baseline."""
    with torch.cuda.stream(stream):
        x = _on_device(req.x, device, use_host=not use_store)
        y = None if req.y is None else _on_device(req.y, device, use_host=not use_store)
        lin = _sk.LinearKernel()
        if req.kind not in ("gram", "robust"):
            raise ValueError(f"unknown request kind {req.kind!r}")
        k = _k.SigPDE(lin, req.order, precision=precision)
        sx = sy = None
        if req.kind == "robust":
            rk = _k.RobustSigPDE(lin, req.order, precision=precision)

            def scales(operand, dev_paths):
                if _resident(operand) and use_store:
                    return operand.scales(rk, req.order, precision, stream)
                return rk.normalization(dev_paths)

            sx = scales(req.x, x)
            sy = sx if y is None else scales(req.y, y)
        cells = request_cells(req)
        rows = x.shape[0]
        if chunk_cells > 0 and cells > chunk_cells and rows > 1:
            step = max(1, int(rows * chunk_cells // cells))
            if y is None:
                # symmetric: per row block, the diagonal block with the symmetric kernel and the
                # block to its left with x_i on the rows -- the orientation the symmetric kernel
                # uses for i >= j -- mirrored, so every entry is the unchunked entry bit for bit
                out = torch.empty((rows, rows), dtype=x.dtype, device=device)
                for i0 in range(0, rows, step):
                    i1 = min(rows, i0 + step)
                    s_blk = None if sx is None else sx[i0:i1]
                    out[i0:i1, i0:i1] = k.gram(x[i0:i1], None, s_blk)
                    if i0 > 0:
                        left = k.gram(x[i0:i1], x[:i0], s_blk, None if sx is None else sx[:i0])
                        out[i0:i1, :i0] = left
                        out[:i0, i0:i1] = left.t()
            else:
                out = torch.empty((rows, y.shape[0]), dtype=x.dtype, device=device)
                for i0 in range(0, rows, step):
                    i1 = min(rows, i0 + step)
                    out[i0:i1] = k.gram(x[i0:i1], y, None if sx is None else sx[i0:i1], sy)
        else:
            out = k.gram(x, y, sx, sy if y is not None else None)
        if staging is not None:  # the server's pinned buffer of this stream (no page-locked allocation per request)
            host = staging(out.numel() * out.element_size()).view(out.dtype)[:out.numel()].view(out.shape)
        else:
            host = torch.empty(out.shape, dtype=out.dtype, pin_memory=True)
        host.copy_(out, non_blocking=True)
    return host, (x, y, out, sx, sy)


class GramServer:
    """Continuous-batching server (see the module docstring).

    hbm_budget_bytes: device memory the in-flight requests may hold together
    (default: 80% of the memory free at start, counting blocks that the
    caching allocator holds but does not use).  A request larger than the
    whole budget fails at admission with MemoryError instead of waiting
    forever.
    """

    def __init__(self, device="cuda", max_inflight: int = 8, hbm_budget_bytes: Optional[int] = None,
                 precision: str = "fp64", poll_interval_s: float = 50e-6, chunk_cells: int = 2 * 10 ** 12,
                 max_wait_s: float = 2.0, batch_small: bool = False, small_pairs: int = 8192,
                 small_cells: int = 2 * 10 ** 9, batch_pairs: int = 1 << 17):
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.precision = precision
        self.max_inflight = int(max_inflight)
        # Start from a clean allocator pool: blocks cached by earlier work in the process (an earlier
        # server's requests, say) are released, so that this server's requests are not carved out of a
        # pool shaped by other sizes.  Measured: a second and third server in one process (light trace,
        # burst) served 764-790 requests/s from the pool the first left, 1151-1610 from a clean one.
        with torch.cuda.device(self.device):
            torch.cuda.empty_cache()
        if hbm_budget_bytes is None:
            # memory this process can use: what the driver has free plus what the caching allocator holds
            # without using (blocks cached by earlier work, which the driver counts as taken); from the
            # driver's figure alone, a second server in a process that already served would get only the
            # scraps the first one left
            free, _ = torch.cuda.mem_get_info(self.device)
            cached = torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
            hbm_budget_bytes = int(0.8 * (free + max(cached, 0)))
        self.budget = int(hbm_budget_bytes)
        self.poll = poll_interval_s
        self.chunk_cells = int(chunk_cells)
        self.max_wait_s = float(max_wait_s)
        # kernel-level batching: small symmetric requests waiting together go into one ragged launch
        self.batch_small = bool(batch_small)
        self.small_pairs = int(small_pairs)
        self.small_cells = int(small_cells)
        self.batch_pairs = int(batch_pairs)
        self.batches = 0
        self.batched_requests = 0
        self._q: "queue.Queue[RequestHandle]" = queue.Queue()
        self._pending: collections.deque = collections.deque()
        self._inflight: list = []
        self._streams = [torch.cuda.Stream(self.device) for _ in range(self.max_inflight)]
        self._free_streams = list(self._streams)
        # one pinned staging buffer per stream for device-to-host result copies, grown by doubling:
        # allocating page-locked memory per request (cudaHostAlloc) can stall behind work in flight
        self._staging = {id(st): None for st in self._streams}
        self._used = 0
        self._store = {}       # name -> PathSet resident on the device
        self._store_bytes = 0  # held by the store, outside the requests' share of the budget
        self._stop = threading.Event()
        self._ids = 0
        self._lock = threading.Lock()
        self.peak_inflight = 0
        self.peak_bytes = 0
        self._thread = threading.Thread(target=self._run, name="sigk-server", daemon=True)
        self._thread.start()

    # ------------------------------------------------------------------ client side
    def submit(self, req: GramRequest) -> RequestHandle:
        with self._lock:
            if req.rid < 0:
                req.rid = self._ids
            self._ids += 1
        if not req.arrival:
            req.arrival = time.perf_counter()
        h = RequestHandle(req)
        try:
            h.cost = request_cells(req)
        except Exception:
            h.cost = 0
        self._q.put(h)
        return h

    def put(self, name, paths) -> PathSet:
        """Keep `paths` ((N, L, d) float32/float64) resident on the server's device
        under `name` and return the PathSet that requests can name as x or y.
        The store's bytes come out of the HBM budget the requests share."""
        t = torch.as_tensor(paths)
        if t.dim() != 3:
            raise ValueError("paths must be (N, L, d)")
        nbytes = t.numel() * t.element_size()
        with self._lock:
            if name in self._store:
                raise KeyError(f"a path set named {name!r} is already stored")
            if self._store_bytes + nbytes > self.budget:
                raise MemoryError(f"storing {nbytes} bytes would exceed the budget of {self.budget}")
            self._store_bytes += nbytes
        host = t.detach().to("cpu").pin_memory()
        with torch.cuda.device(self.device):
            dev = host.to(self.device)
            torch.cuda.synchronize(self.device)  # resident before any request stream reads it
        ps = PathSet(name, dev, host)
        with self._lock:
            self._store[name] = ps
        return ps

    def drop(self, name):
        """Release a stored path set (requests in flight keep their references until they finish)."""
        with self._lock:
            ps = self._store.pop(name)
            self._store_bytes -= ps.nbytes

    def store_stats(self):
        """Per stored set: bytes and hits / misses of its cached normalisation scales."""
        with self._lock:
            return {n: {"bytes": p.nbytes, "scale_hits": p.lam_hits, "scale_misses": p.lam_misses}
                    for n, p in self._store.items()}

    def close(self, wait: bool = True):
        self._stop.set()
        if wait:
            self._thread.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ scheduler
    def _next(self):
        """The waiting request to admit next: one that waited too long, else the cheapest."""
        now = time.perf_counter()
        old = [h for h in self._pending if now - h.req.arrival > self.max_wait_s]
        pool = old if old else self._pending
        return min(pool, key=lambda h: (h.req.arrival if old else h.cost))

    def _small(self, req) -> bool:
        try:
            return (self.batch_small and req.y is None and req.kind in ("gram", "robust") and req.x.dim() == 3
                    and req.x.shape[1] >= 2 and req.x.shape[0] >= 1 and request_pairs(req) <= self.small_pairs
                    and request_cells(req) <= self.small_cells)
        except Exception:
            return False

    def _admit_batch(self, first) -> bool:
        """Admit `first` with the other small waiting requests of the same dim and dtype as one
        launch; False (nothing admitted) when memory is short."""
        key = (int(first.req.x.shape[2]), first.req.x.dtype)
        group = [first]
        pairs = request_pairs(first.req)
        for h in sorted(self._pending, key=lambda g: g.cost):
            if h is first or not self._small(h.req) or (int(h.req.x.shape[2]), h.req.x.dtype) != key:
                continue
            p = request_pairs(h.req)
            if pairs + p > self.batch_pairs:
                continue
            group.append(h)
            pairs += p
        budget = self.budget - self._store_bytes
        need = batch_footprint_bytes([h.req for h in group], self.precision)
        while len(group) > 1 and need > budget:
            group.pop()
            need = batch_footprint_bytes([h.req for h in group], self.precision)
        if len(group) == 1 or self._used + need > budget:
            return False
        for h in group:
            self._pending.remove(h)
        stream = self._free_streams.pop()
        now = time.perf_counter()
        for h in group:
            h.t_admit = now
        try:
            with torch.cuda.device(self.device):
                hosts, keep = _solve_batch_on_stream([h.req for h in group], self.precision, self.device, stream)
                ev = torch.cuda.Event()
                ev.record(stream)
        except Exception as e:
            self._free_streams.append(stream)
            for h in group:
                h._finish(error=e)
            return True
        self._used += need
        self._inflight.append(_Inflight(group, stream, ev, need, hosts, keep))
        self.batches += 1
        self.batched_requests += len(group)
        self.peak_inflight = max(self.peak_inflight, len(self._inflight))
        self.peak_bytes = max(self.peak_bytes, self._used)
        return True

    def _admit(self):
        while self._pending and self._free_streams:
            h = self._next()
            if self._small(h.req) and self._admit_batch(h):
                continue
            try:
                need = footprint_bytes(h.req, self.precision)
            except Exception as e:  # malformed request: fail it, keep serving
                self._pending.remove(h)
                h._finish(error=e)
                continue
            budget = self.budget - self._store_bytes
            if need > budget:
                self._pending.remove(h)
                h._finish(error=MemoryError(f"request {h.req.rid} needs {need} bytes, budget is {budget}"))
                continue
            if self._used + need > budget:
                return  # wait for memory to free up
            self._pending.remove(h)
            stream = self._free_streams.pop()
            h.t_admit = time.perf_counter()
            try:
                with torch.cuda.device(self.device):
                    out_host, keep = _solve_on_stream(h.req, self.precision, self.device, stream,
                                                      self.chunk_cells, self._staging_for(stream))
                    ev = torch.cuda.Event()
                    ev.record(stream)
            except Exception as e:
                self._free_streams.append(stream)
                h._finish(error=e)
                continue
            self._used += need
            self._inflight.append(_Inflight([h], stream, ev, need, [out_host], keep))
            self.peak_inflight = max(self.peak_inflight, len(self._inflight))
            self.peak_bytes = max(self.peak_bytes, self._used)

    def _staging_for(self, stream):
        def get(nbytes):
            buf = self._staging[id(stream)]
            if buf is None or buf.numel() < nbytes:
                size = 1 << max(20, (int(nbytes) - 1).bit_length())
                buf = torch.empty(size, dtype=torch.uint8, pin_memory=True)
                self._staging[id(stream)] = buf
            return buf[:nbytes]
        return get

    def _reap(self):
        still = []
        for f in self._inflight:
            if f.event.query():
                self._used -= f.bytes
                self._free_streams.append(f.stream)
                f.keep = None
                for h, host in zip(f.handles, f.out_hosts):
                    # results staged in the stream's pinned buffer are copied out before it is reused
                    h._finish(result=host.clone())
            else:
                still.append(f)
        self._inflight = still

    def _run(self):
        torch.cuda.set_device(self.device)
        while True:
            while True:
                try:
                    self._pending.append(self._q.get_nowait())
                except queue.Empty:
                    break
            self._reap()
            self._admit()
            if self._stop.is_set() and not self._pending and not self._inflight and self._q.empty():
                return
            if not self._inflight and not self._pending:
                try:
                    self._pending.append(self._q.get(timeout=0.01))
                except queue.Empty:
                    pass
            else:
                time.sleep(self.poll)


def serve_sequential(requests, precision: str = "fp64", device="cuda", arrivals=None):
    """The per-request plain-launch baseline: each request alone (copy in,
    solve, copy out, synchronise), in arrival order, starting no earlier than
    its arrival; PathSet operands are copied in from their host copies and
    their scales recomputed, as a plain call would.  Returns a list of
    RequestHandle."""
    device = torch.device(device)
    stream = torch.cuda.Stream(device)
    handles = []
    t0 = time.perf_counter()
    for i, req in enumerate(requests):
        if arrivals is not None:
            target = t0 + arrivals[i]
            while time.perf_counter() < target:
                time.sleep(max(0.0, min(1e-3, target - time.perf_counter())))
            req.arrival = target
        elif not req.arrival:
            req.arrival = time.perf_counter()
        h = RequestHandle(req)
        h.t_admit = time.perf_counter()
        try:
            host, _ = _solve_on_stream(req, precision, device, stream, use_store=False)
            stream.synchronize()
            h._finish(result=host)
        except Exception as e:
            h._finish(error=e)
        handles.append(h)
    return handles
