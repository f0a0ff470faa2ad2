"""Full-size parity of the benchmark configurations that are not the default
Gram (which test_parity_gpu.test_config2_gram_sampled_and_properties covers):

* robust512 -- RobustSigPDE.gram(x) + normalization(x), N=512 Brownian paths
  scaled log-uniform in [0.5, 4], L=64, d=16, order 1: all 512 lambdas against
  the float64 oracle's Chandrupatla restatement (relative 1e-6, absolute 1e-9
  near 0), the full 512x512 Gram exactly symmetric, and 256 sampled lower-
  triangle entries against the oracle solved with this engine's lambdas
  (float32 output rounding: 2.5e-7 relative);
* uneven4096 -- 4096 (x, y) pairs, lengths uniform in [16, 512] per path,
  d=32, order uniform in {0, 1, 2, 3}, in one uneven-batch launch: 64 sampled
  pairs against the oracle with float64 cells (2.5e-7, the float32 output
  rounding) and with tensor-core increments (tc64: error normalised by
  sqrt(k(x,x) k(y,y)) at most 1e-5);
* serve200 -- a seeded trace of 200 Gram requests drawn like the serving
  configuration (N log-uniform in [8, 1024], L log-uniform in [32, 1024],
  d in {2, 8, 32}, order in {0, 1, 2}, 30% RobustSigPDE): every result of the
  concurrent mix bitwise equal to the request solved alone, and float64 spot
  checks of two entries in every tenth request.

The reference paths: sigpde/torch/kernel.py:197-230 and :293-301 (robust),
:31-65 (pairwise per length bucket), :67-126 (Gram).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

LAM_RTOL = 1e-6
RTOL_OUT32 = 2.5e-7
CS_TC64 = 1e-5


def host(t):
    return t.detach().double().cpu().numpy()


def rel(got, want):
    return float(np.max(np.abs(got - want) / np.abs(want)))


def test_robust512_full(oracle):
    import sigpde_b200.torch as sig
    from sigpde_b200 import synthetic

    scales = synthetic.log_uniform(512, 0.5, 4.0, 513)
    X = torch.tensor(synthetic.brownian_np(512, 64, 16, 512, scale=scales), dtype=torch.float32, device="cuda")
    rk = sig.RobustSigPDE(sig.kernels.LinearKernel(), 1)
    lam = host(rk.normalization(X))
    x64 = host(X)
    want = oracle.normalization(x64, 1)
    np.testing.assert_allclose(lam, want, rtol=LAM_RTOL, atol=1e-9)
    assert (want > 0).sum() > 256, "most config-3 paths have k(x,x) > 1"
    G = host(rk.gram(X))
    np.testing.assert_array_equal(G, G.T)
    rng = np.random.default_rng(3)
    ii = rng.integers(0, 512, 256)
    jj = (rng.random(256) * (ii + 1)).astype(np.int64)
    flat = ii * 512 + jj
    ref = oracle.gram(x64, x64, 1, lam, lam, pairs=flat)
    live = np.abs(ref) > 0
    assert rel(G.reshape(-1)[flat][live], ref[live]) <= RTOL_OUT32
    np.testing.assert_array_equal(G.reshape(-1)[flat][~live], ref[~live])


def _uneven4096():
    from sigpde_b200 import synthetic
    rng = np.random.Generator(np.random.PCG64(4096))
    lx = rng.integers(16, 513, 4096)
    ly = rng.integers(16, 513, 4096)
    orders = rng.choice(np.array([0, 1, 2, 3]), 4096)
    xs = [synthetic.brownian_np(1, int(L), 32, 4096 * 100003 + 2 * b)[0] for b, L in enumerate(lx)]
    ys = [synthetic.brownian_np(1, int(L), 32, 4096 * 100003 + 2 * b + 1)[0] for b, L in enumerate(ly)]
    return xs, ys, orders.tolist()


@pytest.mark.parametrize("precision", ["fp64", "tc64"])
def test_uneven4096_full(oracle, precision):
    import sigpde_b200.torch as sig
    xs, ys, orders = _uneven4096()
    X = [torch.tensor(a, dtype=torch.float32, device="cuda") for a in xs]
    Y = [torch.tensor(a, dtype=torch.float32, device="cuda") for a in ys]
    got = host(sig.ragged.pairwise(X, Y, orders, precision=precision))
    assert got.shape == (4096,) and np.all(np.isfinite(got))
    pick = np.random.default_rng(4).choice(4096, 64, replace=False)
    want, kxx, kyy = [], [], []
    for b in pick:
        x = host(X[b])[None]
        y = host(Y[b])[None]
        want.append(oracle.pairwise(x, y, orders[b])[0])
        if precision == "tc64":
            kxx.append(oracle.pairwise(x, None, orders[b])[0])
            kyy.append(oracle.pairwise(y, None, orders[b])[0])
    want = np.array(want)
    if precision == "fp64":
        assert rel(got[pick], want) <= RTOL_OUT32
    else:
        err = np.abs(got[pick] - want) / np.sqrt(np.array(kxx) * np.array(kyy))
        assert float(err.max()) <= CS_TC64


def _serve_trace(n, seed):
    from sigpde_b200 import synthetic
    from sigpde_b200.serving import GramRequest
    rng = np.random.Generator(np.random.PCG64(seed))
    reqs = []
    for i in range(n):
        N = int(round(np.exp(rng.uniform(np.log(8), np.log(1024)))))
        L = int(round(np.exp(rng.uniform(np.log(32), np.log(1024)))))
        d = int(rng.choice([2, 8, 32]))
        o = int(rng.choice([0, 1, 2]))
        kind = "robust" if rng.random() < 0.3 else "gram"
        x = synthetic.brownian_np(N, L, d, int(rng.integers(1 << 31)))
        reqs.append(GramRequest(x=torch.tensor(x, dtype=torch.float32).pin_memory(), order=o, kind=kind, rid=i))
    return reqs


def test_serve200_trace(oracle):
    import sigpde_b200.torch as sig
    from sigpde_b200.serving import GramServer
    reqs = _serve_trace(200, 55)
    with GramServer() as srv:
        handles = [srv.submit(r) for r in reqs]
        mixed = [h.wait(timeout=600) for h in handles]
        peak = srv.peak_inflight
    assert peak > 1, "requests should overlap on the device"
    rng = np.random.default_rng(5)
    for i, (r, got) in enumerate(zip(reqs, mixed)):
        x = r.x.cuda()
        if r.kind == "robust":
            rk = sig.RobustSigPDE(sig.kernels.LinearKernel(), r.order)
            alone = rk.gram(x).cpu()
        else:
            alone = sig.SigPDE(sig.kernels.LinearKernel(), r.order).gram(x).cpu()
        np.testing.assert_array_equal(got.numpy(), alone.numpy(), err_msg=f"request {i} differs alone and mixed")
        if i % 10:
            continue
        # float64 spot check of two lower-triangle entries
        N = r.x.shape[0]
        a = rng.integers(0, N, 2)
        b = (rng.random(2) * (a + 1)).astype(np.int64)
        idx = np.unique(np.concatenate([a, b]))
        x64 = r.x.double().numpy()
        sub = {int(p): k for k, p in enumerate(idx)}
        if r.kind == "robust":
            lam = host(rk.normalization(x))
            np.testing.assert_allclose(lam[idx], oracle.normalization(x64[idx], r.order), rtol=LAM_RTOL, atol=1e-9)
            s = lam[idx]
        else:
            s = None
        want = oracle.gram(x64[idx], x64[idx], r.order, s, s,
                           pairs=np.array([sub[int(p)] * len(idx) + sub[int(q)] for p, q in zip(a, b)]))
        vals = got.double().numpy()[a, b]
        live = np.abs(want) > 0
        assert rel(vals[live], want[live]) <= RTOL_OUT32, f"request {i}"
