"""The RBF increment kernel's exponential (exp_nonpos in
sigpde_b200/csrc/static_inc.cuh: Cody-Waite reduction and a degree-13 Taylor
polynomial) against CUDA's exp on 4M arguments in [-707.5, 0] and a few just
above 0.  Bound: 2 units in the last place (the relative difference is then
below 4.5e-16)."""
import os
import re
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_exp_nonpos_matches_cuda_exp(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "exp_check"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "sigpde_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), "-o", str(exe), os.path.join(ROOT, "tests", "exp_nonpos_check.cu")],
                   check=True, capture_output=True, timeout=600)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=120).stdout
    m = re.search(r"max_rel ([0-9.e+-]+) max_ulp ([0-9.e+-]+)", out)
    assert m, out
    assert float(m.group(2)) <= 2.0, out
    assert float(m.group(1)) <= 4.5e-16, out
