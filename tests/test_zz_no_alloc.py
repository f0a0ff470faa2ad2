"""sigk_gram_noalloc: the Gram entry point for callers that cannot allocate.

Some callers cannot call cudaMalloc, for example a host program that links only
libsigk.so and runs inside a device-memory budget fixed up front.  sigk_gram
takes its scratch (the scaled path differences its streaming kernel reads)
from the caller; sigk_gram_noalloc takes it from an 8 MiB array built into
the library instead.  These tests call both entry points through the C ABI on
the same inputs and require the same results, on two calls in a row (the second
with other paths, so leftover scratch from the first call cannot leak into it),
and check that a Gram needing more than 8 MiB of scratch is refused with a
clear error.  This file is collected last on purpose.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

RTOL_OUT32 = 2.5e-7  # float32 outputs: 2 ulp, the bound the parity tests use
NOALLOC_BYTES = 8 << 20


def _paths(n, length, dim, seed):
    from sigpde_b200 import synthetic
    return synthetic.brownian(n, length, dim, seed, device="cuda")


def _gram_with_workspace(lib, X, Y, order, sx, sy, prec=0):
    from sigpde_b200 import _lib
    nx, lx, d = X.shape
    ny, ly, _ = Y.shape
    out = torch.empty((nx, ny), device="cuda", dtype=X.dtype)
    nws = lib.sigk_workspace_size(_lib.SIGK_OP_GRAM, nx, ny, lx, ly, d, order, _lib.SIGK_F32, prec)
    ws = torch.empty(max(nws, 1), dtype=torch.uint8, device="cuda")
    st = lib.sigk_gram(X.data_ptr(), Y.data_ptr(), nx, ny, lx, ly, d, _lib.SIGK_F32, order, 1.0,
                       None if sx is None else sx.data_ptr(), None if sy is None else sy.data_ptr(), out.data_ptr(),
                       prec, ws.data_ptr(), nws, torch.cuda.current_stream().cuda_stream)
    assert st == 0, _lib.last_error()
    return out, nws


def _gram_noalloc(lib, X, Y, order, sx, sy, prec=0):
    from sigpde_b200 import _lib
    nx, lx, d = X.shape
    ny, ly, _ = Y.shape
    out = torch.full((nx, ny), float("nan"), device="cuda", dtype=X.dtype)
    st = lib.sigk_gram_noalloc(X.data_ptr(), Y.data_ptr(), nx, ny, lx, ly, d, _lib.SIGK_F32, order, 1.0,
                               None if sx is None else sx.data_ptr(), None if sy is None else sy.data_ptr(),
                               out.data_ptr(), prec, torch.cuda.current_stream().cuda_stream)
    assert st == 0, _lib.last_error()
    return out


def test_noalloc_gram_matches_gram_on_two_calls():
    from sigpde_b200 import _lib
    lib = _lib.lib()
    calls = [
        # (nx, ny, length, dim, order, scaled) -- both take the streaming kernel
        (48, 40, 64, 8, 2, False),
        (33, 57, 40, 5, 1, True),
    ]
    for i, (nx, ny, L, d, o, scaled) in enumerate(calls):
        X = _paths(nx, L, d, 500 + i)
        Y = _paths(ny, L + 3, d, 600 + i)
        sx = torch.linspace(0.5, 1.5, nx, device="cuda") if scaled else None
        sy = torch.linspace(1.2, 0.8, ny, device="cuda") if scaled else None
        want, nws = _gram_with_workspace(lib, X, Y, o, sx, sy)
        assert 0 < nws <= NOALLOC_BYTES
        got = _gram_noalloc(lib, X, Y, o, sx, sy)
        torch.cuda.synchronize()
        g = got.double().cpu().numpy()
        w = want.double().cpu().numpy()
        assert np.all(np.isfinite(g)), f"call {i}: unwritten entries"
        err = np.max(np.abs(g - w) / np.abs(w))
        assert err <= RTOL_OUT32, f"call {i}: max rel diff {err:.3e}"


def test_noalloc_gram_matches_gram_on_the_matrix_routes():
    """The two routes whose scratch holds an increment matrix: tensor-core
    increments (tc64: split-TF32 GEMM into a float32 matrix, float64 cells) and
    float64 increments from the FP64 GEMM (fp64 with dim >= 16).  Both fit the
    8 MiB array at these sizes; each is called twice in a row with other paths."""
    from sigpde_b200 import _lib
    lib = _lib.lib()
    for prec, d in ((_lib.SIGK_PREC_TC64, 8), (_lib.SIGK_PREC_FP64, 16)):
        for i in range(2):
            X = _paths(24, 40, d, 700 + 10 * prec + i)
            Y = _paths(20, 37, d, 800 + 10 * prec + i)
            want, nws = _gram_with_workspace(lib, X, Y, 1, None, None, prec)
            assert 0 < nws <= NOALLOC_BYTES
            got = _gram_noalloc(lib, X, Y, 1, None, None, prec)
            torch.cuda.synchronize()
            g = got.double().cpu().numpy()
            w = want.double().cpu().numpy()
            assert np.all(np.isfinite(g)), f"precision {prec} call {i}: unwritten entries"
            err = np.max(np.abs(g - w) / np.abs(w))
            assert err <= RTOL_OUT32, f"precision {prec} call {i}: max rel diff {err:.3e}"


def test_noalloc_gram_refuses_more_than_its_scratch():
    from sigpde_b200 import _lib
    lib = _lib.lib()
    # 2048 x 2048 paths of length 128 in 8 dimensions: ~33 MB of scratch
    n, L, d = 2048, 128, 8
    need = lib.sigk_workspace_size(_lib.SIGK_OP_GRAM, n, n, L, L, d, 2, _lib.SIGK_F32, _lib.SIGK_PREC_FP64)
    assert need > NOALLOC_BYTES
    X = torch.zeros((n, L, d), device="cuda")
    out = torch.empty((n, n), device="cuda")
    st = lib.sigk_gram_noalloc(X.data_ptr(), X.data_ptr(), n, n, L, L, d, _lib.SIGK_F32, 2, 1.0, None, None,
                               out.data_ptr(), _lib.SIGK_PREC_FP64, torch.cuda.current_stream().cuda_stream)
    assert st == _lib.SIGK_EINVAL
    msg = _lib.last_error()
    assert "8 MiB" in msg and "sigk_gram_noalloc" in msg
