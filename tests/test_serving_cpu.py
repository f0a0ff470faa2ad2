"""Host-side logic of the request server (sigpde_b200.serving), without a GPU:
request cost and footprint accounting, including path sets kept resident by
the server (their bytes are the store's, not the request's), and the cached
normalisation scales of a path set (computed once per (order, precision))."""
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
