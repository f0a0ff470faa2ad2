"""The float64 oracle against golden vectors produced by the reference itself.

tests/golden/golden.npz holds outputs of the unmodified stojl/SigPDE code run
under NUMBA_ENABLE_CUDASIM=1 (tests/golden/gen_golden.py).  float64 cases pin
the oracle to ~1e-12 relative (the remaining difference is the summation order
of the static Gram: torch.bmm/einsum in the reference, a plain loop here).
float32 cases ran with the simulator's float32 arithmetic, so they only pin the
oracle to the float32 rounding of the reference.
"""
import re

import numpy as np
import pytest

F64_RTOL = 1e-11


def _keys(golden, pattern):
    rx = re.compile(pattern)
    return sorted({m.group(1) for k in golden for m in [rx.match(k)] if m})


def _order(key):
    return int(re.search(r"_o(\d+)", key).group(1))


def _cs_err(a, b, kxx, kyy):
    """|a - b| / sqrt(k(x,x) k(y,y)): error normalised by the Cauchy-Schwarz bound."""
    return np.abs(a - b) / np.sqrt(np.abs(kxx * kyy))


def test_golden_file_present(golden):
    assert "meta_generator" in golden
    assert len(_keys(golden, r"(pw_f64_.*)_out$")) >= 4
    assert len(_keys(golden, r"(gr_f64_.*)_out$")) >= 2
    assert len(_keys(golden, r"(rn_f64_.*)_out$")) >= 4


def test_pairwise_f64(golden, oracle):
    keys = _keys(golden, r"(pw_f64_L\d+_d\d+_o\d+)_out$")
    assert keys
    for key in keys:
        x, y, o = golden[key + "_x"], golden[key + "_y"], _order(key)
        np.testing.assert_allclose(oracle.pairwise(x, y, o), golden[key + "_out"], rtol=F64_RTOL, err_msg=key)
        sx, sy = golden[key + "_sx"], golden[key + "_sy"]
        np.testing.assert_allclose(oracle.pairwise(x, y, o, sx, sy), golden[key + "_scaled_out"], rtol=F64_RTOL,
                                   err_msg=key + " scaled")
        np.testing.assert_allclose(oracle.pairwise(x, None, o, sx), golden[key + "_self_scaled_out"],
                                   rtol=F64_RTOL, err_msg=key + " self scaled")


def test_gram_f64(golden, oracle):
    keys = _keys(golden, r"(gr_f64_\d+x\d+_L\d+_d\d+_o\d+)_out$")
    assert keys
    for key in keys:
        x, y, o = golden[key + "_x"], golden[key + "_y"], _order(key)
        g = oracle.gram(x, y, o)
        np.testing.assert_allclose(g, golden[key + "_out"], rtol=F64_RTOL, err_msg=key)
        np.testing.assert_allclose(g, golden[key + "_tiled_out"], rtol=F64_RTOL, err_msg=key + " tiled")
        sx, sy = golden[key + "_sx"], golden[key + "_sy"]
        np.testing.assert_allclose(oracle.gram(x, y, o, sx, sy), golden[key + "_scaled_out"], rtol=F64_RTOL,
                                   err_msg=key + " scaled")
        np.testing.assert_allclose(oracle.gram(x, None, o), golden[key + "_sym_out"], rtol=F64_RTOL,
                                   err_msg=key + " sym")
        np.testing.assert_allclose(oracle.gram(y, None, o), golden[key + "_sym_tiled_out"], rtol=F64_RTOL,
                                   err_msg=key + " sym tiled")
        np.testing.assert_allclose(oracle.gram(x, None, o, sx), golden[key + "_sym_scaled_out"], rtol=F64_RTOL,
                                   err_msg=key + " sym scaled")


def test_config1_f64(golden, oracle):
    if "cfg1_f64_out" not in golden:
        pytest.skip("config-1 vectors not generated")
    np.testing.assert_allclose(oracle.pairwise(golden["cfg1_f64_x"], golden["cfg1_f64_y"], 1), golden["cfg1_f64_out"],
                               rtol=F64_RTOL)


def test_float32_vectors_within_float32_rounding(golden, oracle):
    """Simulator float32 outputs vs the float64 oracle on the same float32 inputs."""
    worst = 0.0
    for key in _keys(golden, r"(pw_f32_L\d+_d\d+_o\d+)_out$") + (["cfg1_f32"] if "cfg1_f32_out" in golden else []):
        x, y = golden[key + "_x"], golden[key + "_y"]
        o = 1 if key == "cfg1_f32" else _order(key)
        ref = golden[key + "_out"]
        ora = oracle.pairwise(x, y, o)
        kxx = oracle.pairwise(x, None, o)
        kyy = oracle.pairwise(y, None, o)
        worst = max(worst, float(_cs_err(ref, ora, kxx, kyy).max()))
    assert worst < 1e-5, worst


def test_robust_normalization_f64(golden, oracle):
    keys = _keys(golden, r"(rn_f64_N\d+_L\d+_d\d+_o\d+(?:_pow)?)_out$")
    assert keys
    for key in keys:
        x, o = golden[key + "_x"], _order(key)
        nrm = (lambda s: 2 - 1 / s.pow(0.1)) if key.endswith("_pow") else None
        lam = oracle.normalization(x, o, nrm)
        np.testing.assert_allclose(lam, golden[key + "_out"], rtol=1e-9, atol=1e-12, err_msg=key)


def test_robust_normalization_f32(golden, oracle):
    """Reference float32 lambdas (float32 norms and f(k)) against the float64 oracle."""
    keys = _keys(golden, r"(rn_f32_N\d+_L\d+_d\d+_o\d+(?:_pow)?)_out$")
    for key in keys:
        x, o = golden[key + "_x"], _order(key)
        nrm = (lambda s: 2 - 1 / s.pow(0.1)) if key.endswith("_pow") else None
        lam = oracle.normalization(x, o, nrm)
        np.testing.assert_allclose(lam, golden[key + "_out"], rtol=1e-4, atol=1e-6, err_msg=key)


def test_robust_pairwise_and_gram_f64(golden, oracle):
    keys = _keys(golden, r"(rb_f64_N\d+_L\d+_d\d+_o\d+)_pw_out$")
    assert keys
    for key in keys:
        x, y, y2, o = golden[key + "_x"], golden[key + "_y"], golden[key + "_y2"], _order(key)
        np.testing.assert_allclose(oracle.robust_pairwise(x, y, o), golden[key + "_pw_out"], rtol=1e-9,
                                   err_msg=key + " pairwise")
        np.testing.assert_allclose(oracle.robust_pairwise(x, None, o), golden[key + "_pwself_out"], rtol=1e-9,
                                   err_msg=key + " pairwise self")
        np.testing.assert_allclose(oracle.robust_gram(x, y2, o), golden[key + "_gram_out"], rtol=1e-9,
                                   err_msg=key + " gram")
        np.testing.assert_allclose(oracle.robust_gram(x, None, o), golden[key + "_gramsym_out"], rtol=1e-9,
                                   err_msg=key + " gram sym")
