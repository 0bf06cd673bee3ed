"""Shared test setup: the gpu marker, import paths, and golden-fixture loaders."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "team-suprema_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import b200pdlp  # noqa: E402
import oracle  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product kernels")


def golden_index() -> dict:
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


def fixture_names():
    return sorted(golden_index()["fixtures"].keys())


def load_fixture(name: str):
    """(unscaled PDLP form, scaled form, Dr, Dc) exactly as the reference hands
    them to solve_pdhg_gpu, as oracle.LPForm objects."""
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    m, n = (int(v) for v in z["u_dims"])
    off = float(z["u_off"][0])
    U = oracle.LPForm(m, n, z["u_row"], z["u_col"], z["u_val"], z["u_c"], z["u_rL"], z["u_rU"], z["u_l"],
                      z["u_u"], off)
    S = oracle.LPForm(m, n, z["u_row"], z["u_col"], z["s_val"], z["s_c"], z["s_rL"], z["s_rU"], z["s_l"],
                      z["s_u"], off)
    return U.normalized(), S.normalized(), np.array(z["Dr"]), np.array(z["Dc"])


def random_case(key: str):
    """A random-family LP of the golden index, regenerated from its seed and
    prepared without presolve: (raw LP, unscaled form, scaled form, Dr, Dc, golden entry)."""
    g = golden_index()["random"][key]
    lp = b200pdlp.gen_random_lp(g["m"], g["n"], g["k"], g["seed"], g["fp32"])
    U, S, Dr, Dc, _ = b200pdlp.prepare(lp)
    return lp, U, S, Dr, Dc, g


def as_form(lp) -> "oracle.LPForm":
    return oracle.LPForm(lp.m, lp.n, lp.row, lp.col, lp.val, lp.c, lp.rL, lp.rU, lp.l, lp.u,
                         lp.obj_offset).normalized()


def digest(lp) -> str:
    """Content hash of a generated LP (same recipe as tests/golden/make_golden.py)."""
    import hashlib
    h = hashlib.sha256()
    for a in (lp.row, lp.col, lp.val, lp.c, lp.rL, lp.rU, lp.l, lp.u):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def rel(a: float, b: float) -> float:
    return abs(a - b) / max(1.0, abs(b))


# Objective bounds. The north star's 1e-6 applies to the objective of a point
# certified at 1e-8 (tests at tol 1e-8) and to the random benchmark family. A
# point certified at tol = 1e-6 has eps_G <= 1e-6, i.e. |c'x - D| <= 1e-6 (1 +
# |c'x| + |D|), about 2e-6 of the objective, plus the slack its primal and dual
# residuals leave; such a point is held to GAP_BOUND_1E6 of the dual simplex's
# optimum, and to GAP_BOUND_1E6 plus the reference PDLP's own distance from the
# optimum when compared with the reference PDLP's 1e-6 point (the reference's
# own 1e-6 point lands up to 1.54e-6 from the optimum, on adlittle).
OBJ_TOL = 1e-6
GAP_BOUND_1E6 = 2.5e-6


def fixture_obj_tol(name: str) -> float:
    """Bound on a fixture's objective, solved to 1e-6, against the dual simplex."""
    return GAP_BOUND_1E6


def fixture_ref_tol(name: str) -> float:
    """Bound on a fixture's objective, solved to 1e-6, against the reference
    CPU PDLP's own 1e-6 point: GAP_BOUND_1E6 plus that point's distance from the
    dual simplex optimum."""
    g = golden_index()["fixtures"][name]
    return GAP_BOUND_1E6 + rel(g["pdlp"]["1e-06"]["form_objective"], g["simplex"]["objective"])


@pytest.fixture(scope="session")
def golden():
    return golden_index()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
