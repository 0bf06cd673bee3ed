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


def test_reference_arm_never_loads_the_product_library():
    """The reference arm builds its LPs with the oracle's generators and hands
    them to the reference's own build_pdlp_form -> scale: the product library
    must not be mapped into its process."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'small', '--steps', '1', "
            "'--warmup', '0']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('PRODUCT_MAPPED' if 'libb200pdlp' in maps else 'PRODUCT_NOT_MAPPED'); "
            "print('ORACLE_MAPPED' if 'liboracle' in maps else 'ORACLE_NOT_MAPPED')")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    # the LP came from the oracle's generator; the solves ran in spawned workers that import only the oracle
    assert "PRODUCT_NOT_MAPPED" in out.stdout and "ORACLE_MAPPED" in out.stdout, out.stdout[-2000:]


def test_reference_arm_sampled_line_is_labelled_as_extrapolated():
    d = run_arm("--workload", "transport", "--steps", "1", "--warmup", "0", "--cpu-sample-iters", "4")
    check_line(d)
    assert d["extrapolated"] is True and d["sampled_attempts"] == 4
    assert d["attempts_per_solve_source"].startswith("reference")
    assert d["ms_per_step"] > 0


def test_bench_batch_family_equals_the_library_draw():
    sys.path.insert(0, ROOT)
    import bench
    import b200pdlp as B
    assert bench.family_shapes(300, 0) == B.batch_family_shapes(300, seed=0)
    assert bench.family_shapes(50, 5, m_hi=900) == B.batch_family_shapes(50, seed=5, m_hi=900)
