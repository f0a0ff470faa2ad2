"""The CPU reference arm of bench.py: one JSON line with the keys the GPU arm's
line carries and the same `config`, measured on the host cores by the float64
oracle (so no GPU is needed), and silence on ranks other than 0."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


def _bench(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=e,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, ROOT)
    import bench as b
    return b


@pytest.mark.parametrize("workload", ["gram256", "uneven4096"])
def test_reference_arm_line(bench, workload):
    lines = _bench(["--impl", "reference", "--workload", workload, "--steps", "1", "--warmup", "1",
                    "--cpu-seconds", "1"])
    assert len(lines) == 1
    d = lines[0]
    for k in KEYS:
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["ms_per_step"] > 0
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1 and d["higher_is_better"] is True
    w = bench.WORKLOADS[workload]
    want = bench.gram_config(w, 1, "fp64") if workload == "gram256" else bench.ragged_config(w, "fp64")
    assert d["config"] == want  # the GPU arm's config at its default precision
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    lines = _bench(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--cpu-seconds", "1"],
                   env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert lines == []
