"""CPU-only checks: the C ABI library loads and exports every symbol that
include/sigk.h declares, and the host-side logic of sigpde_b200.torch
(argument checks, scale broadcasting, generic increment builders, static
kernels) matches the reference's conventions."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    src = open(os.path.join(ROOT, "include", "sigk.h")).read()
    return re.findall(r"^SIGK_API\s+[\w\s\*]+?\b(sigk_\w+)\s*\(", src, flags=re.M)


@pytest.fixture(scope="module")
def built_lib():
    from sigpde_b200 import build
    return build.build()


def test_header_declares_the_entry_points():
    fns = _header_functions()
    for name in ("sigk_pairwise", "sigk_gram", "sigk_gram_sym", "sigk_normalize", "sigk_self_norms",
                 "sigk_pairwise_inc", "sigk_gram_inc", "sigk_normalize_inc", "sigk_workspace_size",
                 "sigk_last_error_string", "sigk_version"):
        assert name in fns, name


def test_library_exports_every_declared_symbol(built_lib):
    lib = ctypes.CDLL(built_lib)
    for name in _header_functions():
        assert hasattr(lib, name), f"{name} declared in include/sigk.h but not exported"


def test_binding_table_matches_header(built_lib):
    from sigpde_b200 import _lib
    assert set(_lib.SIGNATURES) == set(_header_functions())
    assert _lib.version().startswith("sigk ")
    assert _lib.last_error() == ""


def test_library_needs_no_cuda_runtime_on_the_loader_path(built_lib):
    # cudart is linked statically: loading never depends on LD_LIBRARY_PATH
    deps = os.popen(f"ldd {built_lib}").read()
    assert "libcudart" not in deps


def test_cpu_tensors_are_rejected_before_any_device_call():
    import sigpde_b200.torch as sig
    k = sig.SigPDE(sig.kernels.LinearKernel(), 1)
    x = torch.zeros((2, 5, 3))
    with pytest.raises(ValueError, match="CUDA"):
        k.pairwise(x)
    with pytest.raises(ValueError, match="CUDA"):
        k.gram(x, x)
    with pytest.raises(ValueError, match="CUDA"):
        sig.RobustSigPDE(sig.kernels.LinearKernel()).normalization(x)
    with pytest.raises(ValueError):
        sig.SigPDE(sig.kernels.LinearKernel(), 1, precision="fp16")


def test_scale_broadcast_rules():
    from sigpde_b200.torch.kernel import _broadcast_scale
    like = torch.zeros(1, dtype=torch.float64)
    assert _broadcast_scale(None, 4, like) is None
    s = _broadcast_scale(torch.tensor([2.0]), 4, like)
    assert s.dtype == torch.float64 and s.tolist() == [2.0] * 4
    with pytest.raises(ValueError):
        _broadcast_scale(torch.ones(3), 4, like)


def test_increment_builders_match_oracle(oracle):
    from sigpde_b200.torch import gram_inner_product, pairwise_inner_product, kernels
    x = oracle.brownian(3, 7, 4, 1)
    y = oracle.brownian(3, 9, 4, 2)
    X, Y = torch.tensor(x), torch.tensor(y)
    for order in (0, 2):
        inc = pairwise_inner_product(X, Y, kernels.LinearKernel(), order).numpy()
        for b in range(3):
            np.testing.assert_allclose(inc[b], oracle.increments_linear(x[b], y[b], order), rtol=1e-12, atol=1e-15)
        g = gram_inner_product(X, Y, kernels.RBFKernel(0.5), order).numpy()
        want = oracle.second_difference(oracle.static_gram("rbf", x, y, 0.5), order)
        np.testing.assert_allclose(g, want, rtol=1e-9, atol=1e-13)


@pytest.mark.parametrize("name,param", [("LinearKernel", 0.7), ("RBFKernel", 0.9), ("L1RBFKernel", 1.3)])
def test_static_kernels_match_oracle(oracle, name, param):
    from sigpde_b200.torch import kernels
    kind = {"LinearKernel": "linear", "RBFKernel": "rbf", "L1RBFKernel": "l1rbf"}[name]
    k = getattr(kernels, name)(param)
    x = oracle.brownian(2, 5, 3, 3)
    y = oracle.brownian(3, 6, 3, 4)
    g = k.gram(torch.tensor(x), torch.tensor(y)).numpy()
    np.testing.assert_allclose(g, oracle.static_gram(kind, x, y, param), rtol=1e-10, atol=1e-13)
    p = k.pairwise(torch.tensor(x[:2]), torch.tensor(y[:2])).numpy()
    want = oracle.static_gram(kind, x[:2], y[:2], param)
    np.testing.assert_allclose(p, np.stack([want[0, 0], want[1, 1]]), rtol=1e-10, atol=1e-13)


def test_static_kernel_detection():
    """RBF / L1-RBF kernels (ours or classes of the reference's names from a
    sigpde module) go to sigk_gram_static; other objects keep the generic route."""
    from sigpde_b200 import _lib
    from sigpde_b200.torch import kernels
    from sigpde_b200.torch.kernel import _static_kind
    assert _static_kind(kernels.RBFKernel(0.5)) == (_lib.SIGK_STATIC_RBF, 0.5)
    assert _static_kind(kernels.L1RBFKernel(2)) == (_lib.SIGK_STATIC_L1RBF, 2.0)
    assert _static_kind(kernels.LinearKernel(2.0)) is None

    class RBFKernel:  # same name, foreign module: may compute anything else
        sigma = 1.0
    assert _static_kind(RBFKernel()) is None
    ref_like = type("RBFKernel", (), {"__module__": "sigpde.torch.static_kernels", "sigma": 0.25})
    assert _static_kind(ref_like()) == (_lib.SIGK_STATIC_RBF, 0.25)
    assert _static_kind(type("L1RBFKernel", (), {"__module__": "sigpde.torch.static_kernels",
                                                  "sigma": torch.tensor(1.0)})()) is None


def test_static_gram_argument_checks(built_lib):
    """sigk_gram_static rejects bad arguments before any device call."""
    from sigpde_b200 import _lib
    L = _lib.lib()

    def call(op=_lib.SIGK_OP_GRAM, kind=_lib.SIGK_STATIC_RBF, param=1.0, dim=4, prec=_lib.SIGK_PREC_FP64, y=None):
        return L.sigk_gram_static(op, kind, param, None, y, 3, 3, 10, 10, dim, _lib.SIGK_F32, 1, None, None, None,
                                  prec, None, 0, None)

    assert call(op=_lib.SIGK_OP_PAIRWISE) == _lib.SIGK_EINVAL
    assert call(kind=7) == _lib.SIGK_EINVAL
    assert call(param=0.0) == _lib.SIGK_EINVAL
    assert call(param=float("nan")) == _lib.SIGK_EINVAL
    assert call(prec=9) == _lib.SIGK_EINVAL
    # float32 cells are accepted (increments rounded once to float32): these calls get as far as
    # the null path pointer
    for prec in (_lib.SIGK_PREC_FP32, _lib.SIGK_PREC_TC32):
        assert call(prec=prec) == _lib.SIGK_EINVAL
        assert "x" in _lib.last_error()
    assert call(dim=33) == _lib.SIGK_EUNSUPPORTED
    assert "dim <= 32" in _lib.last_error()
    assert call(op=_lib.SIGK_OP_GRAM_SYM, y=1024) == _lib.SIGK_EINVAL
    assert L.sigk_static_workspace_size(_lib.SIGK_OP_PAIRWISE, _lib.SIGK_STATIC_RBF, 3, 3, 10, 10, 4, 1,
                                        _lib.SIGK_F32, _lib.SIGK_PREC_FP64) == 0
    assert L.sigk_static_workspace_size(_lib.SIGK_OP_GRAM, 9, 3, 3, 10, 10, 4, 1, _lib.SIGK_F32,
                                        _lib.SIGK_PREC_FP64) == 0


def test_backward_argument_checks(built_lib):
    """sigk_backward rejects bad arguments before any device call."""
    from sigpde_b200 import _lib
    L = _lib.lib()

    def call(op=_lib.SIGK_OP_GRAM, order=1, dim=3, length=8):
        return L.sigk_backward(op, None, None, 2, 3, length, length, dim, _lib.SIGK_F32, order, 1.0, None, None,
                               None, None, None, None, 0, None)

    assert call(op=_lib.SIGK_OP_GRAM_SYM) == _lib.SIGK_EINVAL
    assert call(order=5) == _lib.SIGK_EUNSUPPORTED
    assert "order <= 4" in _lib.last_error()
    assert call(dim=0) == _lib.SIGK_EINVAL
    assert call(length=1) == _lib.SIGK_EINVAL
    assert call() == _lib.SIGK_OK  # no gradient requested: nothing to do
    assert L.sigk_backward_workspace_size(_lib.SIGK_OP_GRAM_SYM, 2, 3, 8, 8, 3, 1, _lib.SIGK_F32) == 0
    assert L.sigk_backward_workspace_size(_lib.SIGK_OP_GRAM, 2, 3, 8, 8, 3, 5, _lib.SIGK_F32) == 0


def test_gradient_routing():
    """Calls are routed to the differentiable path only when a path or a scale
    requires grad and grad mode is on; CPU tensors are still rejected there."""
    import sigpde_b200.torch as sig
    from sigpde_b200.torch.kernel import _wants_grad
    x = torch.zeros((2, 5, 3), requires_grad=True)
    s = torch.ones(2, requires_grad=True)
    assert _wants_grad(x) and _wants_grad(None, s) and not _wants_grad(x.detach(), None, 1.0)
    with torch.no_grad():
        assert not _wants_grad(x, s)
    for k in (sig.SigPDE(sig.kernels.LinearKernel(), 1), sig.SigPDE(sig.kernels.RBFKernel(), 1)):
        with pytest.raises(ValueError, match="CUDA"):
            k.gram(x, x)
        with pytest.raises(ValueError, match="CUDA"):
            k.pairwise(x)


def test_route_choices_by_workspace(built_lib, monkeypatch):
    """Route choices visible through sigk_workspace_size (host-only planning).

    A tc64 Gram of order >= 2 takes the fused tensor-core kernel (operand
    images only: no increment matrix) unless SIGK_FUSED_TC=0, except where its
    operands leave room for only an 8-slot ring at 4 coarse rows a lane; order
    1 keeps the two-phase matrix unless SIGK_FUSED_TC=1.  An fp64 Gram of d >= 16 writes the
    float64 increment matrix, except at order 2-3 when the lanes' dx tile fits
    registers (then it needs only the path differences, as with
    SIGK_NO_DGEMM_INC=1); its symmetric Gram keeps the matrix.  Float32 matrices
    read at order 1 by half-warp pipelines are chunked at 1 GiB."""
    from sigpde_b200 import _lib
    lib = _lib.lib()
    G, S, F32 = _lib.SIGK_OP_GRAM, _lib.SIGK_OP_GRAM_SYM, _lib.SIGK_F32
    TC64, FP64 = _lib.SIGK_PREC_TC64, _lib.SIGK_PREC_FP64

    def ws(op, nx, ny, lx, ly, d, o, prec, **env):
        for k in ("SIGK_FUSED_TC", "SIGK_NO_DGEMM_INC", "SIGK_TC_CHUNK_MB"):
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        n = lib.sigk_workspace_size(op, nx, ny, lx, ly, d, o, F32, prec)
        for k in env:
            monkeypatch.delenv(k)
        return n

    # tc64, order 2: fused by default (~4 MB), two-phase when disabled (the 4.26 GB matrix, chunked)
    fused = ws(G, 256, 256, 128, 128, 8, 2, TC64)
    two = ws(G, 256, 256, 128, 128, 8, 2, TC64, SIGK_FUSED_TC="0")
    assert fused < 8 << 20 < 1 << 30 < two
    # tc64, order 1: two-phase by default, fused on request
    assert ws(G, 256, 256, 128, 128, 8, 1, TC64) > 1 << 30 > ws(G, 256, 256, 128, 128, 8, 1, TC64, SIGK_FUSED_TC="1")
    # tc64, d = 16 at 4 coarse rows a lane (the 8-slot ring): two-phase by default, fused on request
    assert ws(G, 256, 256, 128, 128, 16, 2, TC64) > 1 << 30 > ws(G, 256, 256, 128, 128, 16, 2, TC64, SIGK_FUSED_TC="1")
    # tc64, d = 32 at 2 coarse rows a lane (8-slot ring): fused by default
    assert ws(G, 256, 256, 64, 64, 32, 3, TC64) < 16 << 20 < ws(G, 256, 256, 64, 64, 32, 3, TC64, SIGK_FUSED_TC="0")
    # tc64, d = 32 at 4 coarse rows a lane: the operands do not fit shared memory, two-phase even on request
    assert ws(G, 256, 256, 128, 128, 32, 2, TC64, SIGK_FUSED_TC="1") == ws(G, 256, 256, 128, 128, 32, 2, TC64)
    # fp64, d = 16, order 2, 156 rows (8 a lane, 2 coarse rows x 16 dims in registers): no matrix
    g = ws(G, 7, 6, 40, 47, 16, 2, FP64)
    assert g == ws(G, 7, 6, 40, 47, 16, 2, FP64, SIGK_NO_DGEMM_INC="1")
    assert ws(S, 7, 7, 40, 40, 16, 2, FP64) > ws(S, 7, 7, 40, 40, 16, 2, FP64, SIGK_NO_DGEMM_INC="1")
    # fp64, d = 24 (a 32-wide padded tile: too wide for registers) keeps the matrix at order 2
    assert ws(G, 7, 6, 40, 47, 24, 2, FP64) > ws(G, 7, 6, 40, 47, 24, 2, FP64, SIGK_NO_DGEMM_INC="1")
    # tc64 float32 matrices at order 1 with at most 128 refined rows (half-warp readers): chunks of at
    # most 1 GiB (the robust workload's 2.08 GB matrix in 3 chunks); a larger SIGK_TC_CHUNK_MB overrides;
    # order 0 and longer paths keep the 6 GiB cap (one chunk here)
    c3 = ws(S, 512, 512, 64, 64, 16, 1, TC64)
    assert c3 < (1 << 30) + (64 << 20) < (2 << 30) < ws(S, 512, 512, 64, 64, 16, 1, TC64, SIGK_TC_CHUNK_MB="6144")
    assert ws(S, 512, 512, 128, 128, 8, 0, TC64) > 4 << 30
    assert ws(S, 512, 512, 128, 128, 8, 1, TC64) > 4 << 30
