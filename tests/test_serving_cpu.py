"""Host-side logic of the request server (sigpde_b200.serving), without a GPU:
request cost and footprint accounting, including path sets kept resident by
the server (their bytes are the store's, not the request's), the cached
normalisation scales of a path set (computed once per (order, precision)),
and the admission order (cheapest first, oldest first past the wait limit)."""
import numpy as np
import pytest
import torch


def _paths(n, length, d, seed=0):
    rng = np.random.default_rng(seed)
    return torch.tensor(np.cumsum(rng.normal(size=(n, length, d)) / np.sqrt(length), axis=1), dtype=torch.float32)


def test_resident_paths_leave_the_footprint():
    from sigpde_b200.serving import GramRequest, PathSet, footprint_bytes, request_cells
    x, y = _paths(12, 40, 8, 1), _paths(7, 33, 8, 2)
    px, py = PathSet("x", x, x), PathSet("y", y, y)
    for kind in ("gram", "robust"):
        for order in (0, 2):
            host = GramRequest(x=x, y=y, order=order, kind=kind)
            res = GramRequest(x=px, y=py, order=order, kind=kind)
            assert footprint_bytes(host) - footprint_bytes(res) == x.numel() * 4 + y.numel() * 4
            assert request_cells(host) == request_cells(res) == 12 * 7 * (39 << order) * (32 << order)
            sym_host = GramRequest(x=x, order=order, kind=kind)
            sym_res = GramRequest(x=px, order=order, kind=kind)
            assert footprint_bytes(sym_host) - footprint_bytes(sym_res) == x.numel() * 4
    assert px.shape == x.shape and px.dtype == x.dtype and px.dim() == 3 and px.nbytes == x.numel() * 4


class _FakeRobust:
    def __init__(self):
        self.calls = 0

    def normalization(self, t):
        self.calls += 1
        return t[:, 0, 0] * 0 + self.calls


class _FakeStream:
    def __init__(self):
        self.waited = []

    def wait_event(self, ev):
        self.waited.append(ev)


def test_path_set_scales_are_cached_per_order_and_precision(monkeypatch):
    """The first robust request of a (order, precision) computes the scales and
    records an event on its stream; later ones wait for that event and reuse
    them; use_cache=False always recomputes (the per-request baseline)."""
    from sigpde_b200 import serving

    class _Ev:
        def record(self, stream):
            self.stream = stream

    monkeypatch.setattr(serving.torch.cuda, "Event", _Ev)
    x = _paths(5, 20, 3, 4)
    ps = serving.PathSet("p", x, x)
    rk = _FakeRobust()
    s1, s2 = _FakeStream(), _FakeStream()
    a = ps.scales(rk, 1, "fp64", s1)
    b = ps.scales(rk, 1, "fp64", s2)
    assert rk.calls == 1 and b is a and len(s2.waited) == 1 and s2.waited[0].stream is s1
    c = ps.scales(rk, 2, "fp64", s2)
    d = ps.scales(rk, 1, "tc64", s2)
    assert rk.calls == 3 and c is not a and d is not a
    e = ps.scales(rk, 1, "fp64", s1, use_cache=False)
    assert rk.calls == 4 and e is not a
    assert (ps.lam_hits, ps.lam_misses) == (1, 3)


class _Req:
    def __init__(self, arrival):
        self.arrival = arrival


class _Handle:
    def __init__(self, name, cost, arrival):
        self.name = name
        self.cost = cost
        self.req = _Req(arrival)


class _Queue:
    def __init__(self, handles, max_wait_s):
        self._pending = handles
        self.max_wait_s = max_wait_s


def test_admission_order_cheapest_first_with_aging():
    """The next request admitted is the cheapest waiting one, unless some waited longer than
    max_wait_s: then the oldest of those (so that large requests are not starved)."""
    import time
    from sigpde_b200.serving import GramServer
    now = time.perf_counter()
    a, b, c = _Handle("a", 50.0, now - 0.01), _Handle("b", 5.0, now - 0.02), _Handle("c", 20.0, now)
    assert GramServer._next(_Queue([a, b, c], max_wait_s=10.0)).name == "b"
    old1, old2 = _Handle("old1", 900.0, now - 30.0), _Handle("old2", 100.0, now - 20.0)
    assert GramServer._next(_Queue([a, b, old2, old1, c], max_wait_s=10.0)).name == "old1"
    assert GramServer._next(_Queue([a, b, old2, c], max_wait_s=10.0)).name == "old2"


def test_request_pairs_count_the_lower_triangle_of_a_symmetric_gram():
    from sigpde_b200.serving import GramRequest, request_pairs
    x, y = _paths(9, 12, 3, 3), _paths(4, 15, 3, 4)
    assert request_pairs(GramRequest(x=x, y=y, order=1)) == 36
    assert request_pairs(GramRequest(x=x, order=1)) == 45
