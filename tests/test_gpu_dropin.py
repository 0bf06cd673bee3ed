"""The drop-in boundary seen from the reference's side: the reference's own
end-to-end checks (tests/run_checks.cpp) and its CPU-vs-GPU audit tool
(tools/audit_lp.cpp), compiled from the reference's sources and linked against
this engine's solve_pdhg_gpu symbol (team-suprema_b200/csrc/shim_solve_pdhg_gpu.cpp)
in place of gpu/pdlp_gpu_solve.cu (oracle/Makefile, target dropin).

* run_checks drives solve_mps, whose LP portfolio races the CPU engine against
  solve_pdhg_gpu (src/solve.cpp:108-122) and, in check [6c], hands the PDLP
  point to crossover and simplex (src/solve.cpp:317-338, tests/run_checks.cpp:144-166).
* audit_lp runs solve_pdhg (CPU) and solve_pdhg_gpu (this engine) unraced on the
  same presolved and scaled form, certifies both with verify() on the original
  problem after postsolve, and fails on a CPU/GPU objective gap above 1e-4 or
  either engine above 1e-4 of the published Netlib optimum
  (tools/audit_lp.cpp:241-280).

Both binaries run with cwd oracle/_ref, where the build copied the fixtures
they read by relative path. Their full output is printed (pytest -s shows it).
"""
import os
import re
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

REF_DIR = os.path.join(ROOT, "oracle", "_ref")
RUN_CHECKS = os.path.join(REF_DIR, "run_checks_b200")
AUDIT = os.path.join(REF_DIR, "audit_lp_b200")

if not (os.path.exists(RUN_CHECKS) and os.path.exists(AUDIT)):
    pytest.skip("the reference's run_checks/audit_lp linked against the engine are not built (make -C oracle dropin)",
                allow_module_level=True)


def run(cmd, timeout):
    p = subprocess.run(cmd, cwd=REF_DIR, capture_output=True, text=True, timeout=timeout)
    print(p.stdout[-20000:])
    print(p.stderr[-4000:])
    return p


def test_reference_run_checks_pass_with_the_b200_engine():
    p = run([RUN_CHECKS], 900)
    assert p.returncode == 0, p.stdout[-3000:]
    assert "ALL CHECKS PASSED" in p.stdout


# Fixtures audited at 1e-6. share1b is left out: the reference's own CPU engine
# fails the audit's original-space check on it too (its PDLP-form point at 1e-6
# maps to eps_P ~ 3.8e-5 after postsolve), so the file fails whichever GPU
# engine is linked; test_audit_share1b_fails_alike_for_both_engines covers it.
AUDITED = ["afiro", "adlittle", "blend", "sc50a", "sc50b", "sc105", "kb2", "scagr7", "israel", "beaconfd"]


def verdicts(out: str):
    """{file stem: verdict} from audit_lp's report."""
    res, cur = {}, None
    for ln in out.splitlines():
        m = re.match(r"^=== (\S+\.mps) ===", ln.strip())
        if m:
            cur = os.path.splitext(os.path.basename(m.group(1)))[0]
        v = re.search(r"VERDICT:\s*(PASS|WARN|FAIL)", ln)
        if v and cur:
            res[cur] = v.group(1)
    return res


def test_reference_audit_agrees_cpu_and_b200_engine():
    files = [os.path.join("sample_problems", f"{n}.mps") for n in AUDITED]
    p = run([AUDIT, "--tol", "1e-6", "--max-iter", "500000", *files], 900)
    assert p.returncode == 0, p.stdout[-4000:]
    m = re.search(r"(\d+) problem\(s\) audited, (\d+) FAIL, (\d+) WARN, (\d+) PASS", p.stdout)
    assert m, p.stdout[-2000:]
    total, fail, warn, ok = (int(g) for g in m.groups())
    assert total == len(AUDITED) and fail == 0
    got = verdicts(p.stdout)
    # a WARN is a CPU/GPU objective gap between 1e-6 and 1e-4 with both engines at 1e-6 KKT, which
    # two points certified at 1e-6 can show (each may lie ~2e-6 from the optimum); FAIL is any
    # engine off its KKT claim, off the published optimum by 1e-4, or a gap above 1e-4
    assert sorted(got) == sorted(AUDITED) and all(v in ("PASS", "WARN") for v in got.values()), got


def test_audit_share1b_fails_alike_for_both_engines():
    """share1b fails the audit for the reference CPU engine itself: both engines
    converge in PDLP form, and both points exceed 1e-6 after postsolve. The
    engine must not add a failure of its own (no GPU-only note)."""
    p = run([AUDIT, "--tol", "1e-6", "--max-iter", "500000", os.path.join("sample_problems", "share1b.mps")], 600)
    out = p.stdout
    assert verdicts(out).get("share1b") in ("PASS", "WARN", "FAIL"), out[-2000:]
    cpu_note = "CPU claims converged but its own KKT residual exceeds tol" in out
    gpu_note = "GPU claims converged but its own KKT residual exceeds tol" in out
    assert cpu_note == gpu_note, out[-3000:]
    assert "GPU did not converge" not in out
    assert "disagreement exceeds 1e-4" not in out
    assert "GPU objective does not match" not in out
