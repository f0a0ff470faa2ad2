"""Build libsigk.so (the sm_100a CUDA engine) in-tree with nvcc.

Usage:  python -m sigpde_b200.build [--force] [-j N]

The kernel instantiations are split across several translation units that
are compiled in parallel and linked into one shared library next to this
file.  Only sm_100a code is generated (no PTX for other targets).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsigk.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["sigk_api.cu", "kernels_pair_f64.cu", "kernels_pair_f32.cu", "kernels_norm.cu", "kernels_stream.cu",
           "kernels_stream_reg_f64.cu", "kernels_stream_reg_f32.cu", "kernels_stream_reg_f32x2.cu", "kernels_stream_reg_f64x2.cu", "kernels_ragged.cu", "kernels_tc.cu", "kernels_norm_pipe.cu",
           "kernels_grad.cu", "kernels_fused_tc.cu"]
HEADERS = ["wave.cuh", "sigk_kernels.cuh", "stream.cuh", "dispatch.h", "kernels_stream_reg.inc", "ragged.cuh", "tc.cuh", "norm_pipe.cuh", "dgemm_inc.cuh", "static_inc.cuh", "grad.cuh", "fused_tc.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "-DSIGK_BUILD"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, extra) -> str:
    obj = os.path.join(BUILD, os.path.splitext(os.path.basename(src))[0] + ".o")
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "sigk.h"), __file__]
    if _stale(obj, deps):
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + list(extra) + ["-I", INCLUDE, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if r.stderr.strip() and "-Xptxas" in " ".join(extra):
            sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, jobs: int = 0, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    jobs = jobs or min(len(srcs), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), srcs))
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("--ptxas-v", action="store_true", help="print register / spill / smem usage")
    a = ap.parse_args()
    print(build(a.force, a.j, a.ptxas_v))


if __name__ == "__main__":
    main()
