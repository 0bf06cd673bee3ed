"""The reference arm of bench.py (--impl reference) runs on the host cores
alone: the reference's own CPU PDLP (oracle/_ref, built from the reference's
sources) on a bounded sample of the workload. Checked here on CPU, with small
samples, for the JSON line the benchmark contract asks for."""
import json
import os
import subprocess
import sys

import pytest

import oracle as O
from conftest import ROOT

pytestmark = pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref is not built")

KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"}


def run_arm(*args):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                         capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


def check_line(d):
    assert KEYS <= set(d), KEYS - set(d)
    assert d["impl"] == "reference" and d["unit"] == "solves/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_small_lp():
    d = run_arm("--workload", "small", "--steps", "1", "--warmup", "1", "--cpu-sample-iters", "8")
    check_line(d)
    assert d["cpu_baseline"]["cores"] == (os.cpu_count() or 1)  # one single-threaded solve per core


@pytest.mark.parametrize("workload", ["batch", "serve"])
def test_reference_arm_all_cores(workload):
    d = run_arm("--workload", workload, "--steps", "1", "--warmup", "0", "--cpu-budget-s", "1")
    check_line(d)
    assert d["cpu_baseline"]["cores"] == (os.cpu_count() or 1)
    assert all(st["converged"] == st["lps"] for st in d["steps_detail"])
