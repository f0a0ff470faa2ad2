"""The request server (sigpde_b200.serving): continuous batching with
HBM-footprint admission.

* each request's result in a concurrent mix equals the same request solved
  alone through the API (the solves are deterministic and only read their own
  buffers, so the tolerance is 0: bitwise equal), also when small requests are
  batched into one uneven-batch launch (the same arithmetic per cell);
* requests overlap on the device (more than one in flight at once);
* the in-flight footprint never exceeds the HBM budget; a request larger than
  the whole budget fails alone with MemoryError;
* a malformed request fails alone, the others complete;
* float64 spot checks against the oracle (float32 outputs: 2.5e-7 relative).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _requests(oracle, n, seed, dtype=torch.float32):
    from sigpde_b200.serving import GramRequest
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        N = int(rng.integers(3, 40))
        L = int(rng.integers(8, 80))
        d = int(rng.choice([2, 8, 32]))
        o = int(rng.integers(0, 3))
        kind = "robust" if rng.random() < 0.3 else "gram"
        sc = np.exp(rng.uniform(np.log(0.5), np.log(4.0), N)) if kind == "robust" else None
        x = torch.tensor(oracle.brownian(N, L, d, int(rng.integers(1 << 30)), scale=sc), dtype=dtype).pin_memory()
        y = None
        if kind == "gram" and rng.random() < 0.5:
            y = torch.tensor(oracle.brownian(int(rng.integers(2, 30)), L + int(rng.integers(0, 20)), d,
                                             int(rng.integers(1 << 30))), dtype=dtype).pin_memory()
        reqs.append(GramRequest(x=x, y=y, order=o, kind=kind))
    return reqs


def _alone(req):
    import sigpde_b200.torch as sig
    x = req.x.cuda()
    y = None if req.y is None else req.y.cuda()
    if req.kind == "robust":
        return sig.RobustSigPDE(sig.kernels.LinearKernel(), req.order).gram(x, y).cpu()
    return sig.SigPDE(sig.kernels.LinearKernel(), req.order).gram(x, y).cpu()


def test_results_in_the_mix_equal_results_alone(oracle):
    from sigpde_b200.serving import GramServer
    reqs = _requests(oracle, 24, 1)
    with GramServer(max_inflight=6) as srv:
        handles = [srv.submit(r) for r in reqs]
        results = [h.wait(timeout=120) for h in handles]
        peak = srv.peak_inflight
    assert peak > 1, "requests should overlap on the device"
    for r, got in zip(reqs, results):
        np.testing.assert_array_equal(got.numpy(), _alone(r).numpy())
    # float64 spot checks on a few entries
    rng = np.random.default_rng(0)
    for r, got in list(zip(reqs, results))[:6]:
        x = r.x.double().numpy()
        y = None if r.y is None else r.y.double().numpy()
        i = int(rng.integers(got.shape[0]))
        j = int(rng.integers(got.shape[1]))
        if r.kind == "robust":
            want = oracle.robust_gram(x, y, r.order)[i, j]
        else:
            yy = x if y is None else y
            want = oracle.gram(x, yy, r.order, pairs=[i * yy.shape[0] + j])[0]
        assert abs(float(got[i, j]) - want) <= 2.5e-7 * abs(want) + 1e-300


@pytest.mark.parametrize("precision", ["fp64", "tc64"])
def test_small_requests_are_batched_into_one_launch(oracle, precision):
    """Small symmetric requests waiting together run as one uneven-batch launch; each
    result equals the request solved alone through the API with the same precision."""
    import sigpde_b200.torch as sig
    from sigpde_b200.serving import GramServer
    reqs = [r for r in _requests(oracle, 30, 7) if r.y is None]
    with GramServer(max_inflight=2, precision=precision, batch_small=True) as srv:
        handles = [srv.submit(r) for r in reqs]
        results = [h.wait(timeout=120) for h in handles]
        assert srv.batches >= 1 and srv.batched_requests >= 2
    for r, got in zip(reqs, results):
        x = r.x.cuda()
        if r.kind == "robust":
            want = sig.RobustSigPDE(sig.kernels.LinearKernel(), r.order, precision=precision).gram(x).cpu()
        else:
            want = sig.SigPDE(sig.kernels.LinearKernel(), r.order, precision=precision).gram(x).cpu()
        np.testing.assert_array_equal(got.numpy(), want.numpy())


def test_admission_respects_the_hbm_budget(oracle):
    from sigpde_b200.serving import GramServer, footprint_bytes
    reqs = _requests(oracle, 12, 2)
    sizes = [footprint_bytes(r) for r in reqs]
    budget = 2 * max(sizes)
    big = _requests(oracle, 1, 3)[0]
    big_size = footprint_bytes(big)
    small_budget = max(budget, 1)
    with GramServer(max_inflight=8, hbm_budget_bytes=small_budget) as srv:
        handles = [srv.submit(r) for r in reqs]
        for h in handles:
            h.wait(timeout=120)
        assert srv.peak_bytes <= small_budget
    if big_size > small_budget:
        with GramServer(max_inflight=2, hbm_budget_bytes=small_budget) as srv:
            h = srv.submit(big)
            with pytest.raises(MemoryError):
                h.wait(timeout=60)


def test_a_bad_request_fails_alone(oracle):
    from sigpde_b200.serving import GramRequest, GramServer
    reqs = _requests(oracle, 6, 4)
    bad = GramRequest(x=torch.zeros((4, 1, 3)), order=1)  # one point per path: rejected by the API
    with GramServer(max_inflight=4) as srv:
        handles = [srv.submit(r) for r in reqs[:3]] + [srv.submit(bad)] + [srv.submit(r) for r in reqs[3:]]
        with pytest.raises(ValueError):
            handles[3].wait(timeout=60)
        for h, r in zip(handles[:3] + handles[4:], reqs):
            np.testing.assert_array_equal(h.wait(timeout=120).numpy(), _alone(r).numpy())


def test_chunked_large_requests_match(oracle):
    """Row-block chunking of large Grams (forced with a tiny chunk size) gives the same result."""
    from sigpde_b200.serving import GramServer
    reqs = _requests(oracle, 8, 6)
    with GramServer(max_inflight=3, chunk_cells=10 ** 5) as srv:
        handles = [srv.submit(r) for r in reqs]
        for h, r in zip(handles, reqs):
            np.testing.assert_array_equal(h.wait(timeout=120).numpy(), _alone(r).numpy())


def test_sequential_baseline_gives_the_same_results(oracle):
    from sigpde_b200.serving import serve_sequential
    reqs = _requests(oracle, 5, 5)
    handles = serve_sequential(reqs)
    for h, r in zip(handles, reqs):
        np.testing.assert_array_equal(h.wait().numpy(), _alone(r).numpy())


def test_resident_path_sets(oracle):
    """Path sets kept on the device (GramServer.put): requests naming them as x or
    y give bitwise the results of the same paths sent from the host, robust
    requests on a set compute its scales once per (order, precision) and reuse
    them (hits counted), the store's bytes come out of the budget and the
    requests' footprints leave the stored paths out, and the per-request
    baseline (serve_sequential) recomputes from the host copies."""
    import sigpde_b200.torch as sig
    from sigpde_b200.serving import GramRequest, GramServer, footprint_bytes, serve_sequential
    rng = np.random.default_rng(7)
    sets = {}
    for i in range(4):
        N, L = int(rng.integers(4, 30)), int(rng.integers(10, 60))
        sc = np.exp(rng.uniform(np.log(0.5), np.log(4.0), N))
        sets[f"s{i}"] = torch.tensor(oracle.brownian(N, L, 8, 100 + i, scale=sc), dtype=torch.float32)
    with GramServer(max_inflight=4) as srv:
        budget0 = srv.budget - srv._store_bytes
        stored = {k: srv.put(k, v) for k, v in sets.items()}
        assert srv.budget - srv._store_bytes == budget0 - sum(v.numel() * 4 for v in sets.values())
        with pytest.raises(KeyError):
            srv.put("s0", sets["s0"])
        reqs = []
        for i in range(24):
            a = f"s{int(rng.integers(0, 4))}"
            kind = "robust" if i % 2 == 0 else "gram"
            o = int(rng.integers(0, 3))
            y = None
            if kind == "gram" and i % 4 == 1:
                b = f"s{int(rng.integers(0, 4))}"
                y = stored[b]
            reqs.append(GramRequest(x=stored[a], y=y, order=o, kind=kind))
        # footprints leave the resident paths out
        for r in reqs[:4]:
            host_req = GramRequest(x=r.x.host, y=None if r.y is None else r.y.host, order=r.order, kind=r.kind)
            paths = r.x.nbytes + (0 if r.y is None else r.y.nbytes)
            assert footprint_bytes(host_req) - footprint_bytes(r) == paths
        handles = [srv.submit(r) for r in reqs]
        results = [h.wait(timeout=120) for h in handles]
        stats = srv.store_stats()
    for r, got in zip(reqs, results):
        x = r.x.host.cuda()
        y = None if r.y is None else r.y.host.cuda()
        if r.kind == "robust":
            want = sig.RobustSigPDE(sig.kernels.LinearKernel(), r.order).gram(x, y).cpu()
        else:
            want = sig.SigPDE(sig.kernels.LinearKernel(), r.order).gram(x, y).cpu()
        np.testing.assert_array_equal(got.numpy(), want.numpy())
    robust_keys = {(r.x.name, r.order) for r in reqs if r.kind == "robust"}
    robust_reqs = sum(r.kind == "robust" for r in reqs)
    hits = sum(v["scale_hits"] for v in stats.values())
    misses = sum(v["scale_misses"] for v in stats.values())
    assert hits + misses == robust_reqs
    assert misses >= len(robust_keys) and hits >= robust_reqs - 2 * len(robust_keys) and hits > 0
    # the per-request baseline copies the host paths and recomputes: the same results
    seq = serve_sequential(reqs[:6])
    for h, got in zip(seq, results[:6]):
        np.testing.assert_array_equal(h.result.numpy(), got.numpy())


def test_default_budget_counts_the_allocator_cache():
    """Memory the caching allocator holds without using (left by earlier work in
    the process) is usable by a new server: its default budget must not shrink
    by it (a second server in a process that already served once used to get
    only the scraps, and refused ordinary requests)."""
    import gc
    from sigpde_b200.serving import GramServer
    gc.collect()
    torch.cuda.empty_cache()
    with GramServer(max_inflight=2) as srv:
        b0 = srv.budget
    block = torch.empty(4 << 30, dtype=torch.uint8, device="cuda")
    del block  # cached by the allocator, free for this process
    with GramServer(max_inflight=2) as srv:
        b1 = srv.budget
    assert b1 > b0 - (256 << 20), (b0, b1)
