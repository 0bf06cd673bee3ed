"""Host preparation of an LP as the caller has it (no GPU): this library's
presolve / postsolve (b2_presolve, b2_postsolve) and PDLP form
(b2_pdlp_form_build / _extract).

* The PDLP form equals the reference's build_pdlp_form (src/pdlp.cpp:8-82)
  entry for entry, on the fixtures' LPs as the reference reads them
  (tests/golden/orig_<name>.npz) and on an LP with every kind of row.
* presolve -> PDLP form -> the oracle's PDLP (the restated reference
  algorithm) -> extract -> postsolve gives a point that verify() certifies on
  the ORIGINAL LP (primal and dual values), with the published optimum.
* Presolve reports infeasible / unbounded LPs its reductions expose.
"""
import os

import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import GOLDEN, golden_index, rel

G = golden_index()
ORIG = sorted(f[5:-4] for f in os.listdir(GOLDEN) if f.startswith("orig_") and f.endswith(".npz"))
SOLVABLE = [n for n in ORIG if n in G["fixtures"]]


def load_original(name) -> B.RangedLP:
    z = np.load(os.path.join(GOLDEN, f"orig_{name}.npz"))
    m, n = (int(v) for v in z["o_dims"])
    return B.RangedLP(m, n, z["o_row"], z["o_col"], z["o_val"], z["o_c"], z["o_rL"], z["o_rU"], z["o_l"], z["o_u"],
                      float(z["o_off"][0]))


def as_oracle(lp) -> O.LPForm:
    return O.LPForm(lp.m, lp.n, lp.row, lp.col, lp.val, lp.c, lp.rL, lp.rU, lp.l, lp.u, lp.obj_offset).normalized()


def every_row_kind():
    """Equality, >=, <=, ranged and free rows; fixed, free and bounded columns."""
    rng = np.random.default_rng(5)
    m, n = 9, 7
    A = rng.uniform(-1, 1, (m, n)) * (rng.random((m, n)) < 0.6)
    r, c = np.nonzero(A)
    inf = np.inf
    rL = np.array([1.0, -inf, 0.5, -2.0, -inf, 3.0, 0.0, -inf, -1.0])
    rU = np.array([1.0, 4.0, inf, 2.0, inf, 3.0, inf, 0.25, 5.0])
    l = np.array([0.0, -inf, 1.0, 0.0, -3.0, 2.0, 0.0])
    u = np.array([10.0, inf, 1.0, inf, 3.0, 2.0, 1.0])
    return B.RangedLP(m, n, r, c, A[r, c], rng.normal(size=n), rL, rU, l, u, 1.5)


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref is not built")
@pytest.mark.parametrize("name", ORIG + ["every_row_kind"])
def test_pdlp_form_equals_the_references(name):
    lp = every_row_kind() if name == "every_row_kind" else load_original(name)
    P = O.RefProblem.from_form(as_oracle(lp), use_presolve=False)
    # the reference builds its form from its (not presolved) working copy of the LP,
    # whose entries it keeps in column order: both builders get that same input
    src = P.form(P.PRESOLVED)
    lp = B.RangedLP(src.m, src.n, src.row, src.col, src.val, src.c, src.rL, src.rU, src.l, src.u, src.obj_offset)
    F = B.PdlpForm(lp)
    R = P.form(P.PDLP_FORM)
    f = F.form
    assert (f.m, f.n) == (R.m, R.n)
    for a, b in ((f.row, R.row), (f.col, R.col), (f.val, R.val), (f.c, R.c), (f.rL, R.rL), (f.rU, R.rU),
                 (f.l, R.l), (f.u, R.u)):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b))
    assert f.obj_offset == R.obj_offset
    # extract: x is the first n columns, y goes back to the input rows with the row signs
    rng = np.random.default_rng(0)
    x2, y2 = rng.normal(size=f.n), rng.normal(size=f.m)
    x, y = F.extract(x2, y2)
    np.testing.assert_array_equal(x, x2[:lp.n])
    assert y.shape == (lp.m,)


def solve_original_on_cpu(lp, tol=1e-8):
    """presolve -> PDLP form -> scale -> the oracle's PDLP -> extract -> postsolve."""
    pre = B.Presolved(lp)
    assert pre.status == 0
    F = B.PdlpForm(pre.reduced)
    U = as_oracle(F.form)
    S, Dr, Dc = O.scale(U)
    r = O.pdlp_run(U, S, Dr, Dc, max_iterations=500000, tol=tol)
    assert r["converged"]
    xr, yr = F.extract(r["x"], r["y"])
    return pre, pre.postsolve(xr, yr)


@pytest.mark.parametrize("name", SOLVABLE)
def test_presolve_postsolve_certified_on_the_original(name):
    lp = load_original(name)
    pre, (x, y) = solve_original_on_cpu(lp)
    v = O.verify(as_oracle(lp), x, y)
    # 1e-8 on the reduced PDLP form; the postsolved point is judged on the original LP
    assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6, v
    ref = G["fixtures"][name]["simplex"]["objective"]
    assert rel(v["objective"], ref) <= 1e-6, (v["objective"], ref)


def test_presolve_reduces_the_fixtures():
    """The reductions fire on the Netlib fixtures (fixed columns, singleton rows)."""
    shrunk = 0
    for name in SOLVABLE:
        lp = load_original(name)
        pre = B.Presolved(lp)
        assert pre.status == 0
        assert pre.reduced.m <= lp.m and pre.reduced.n <= lp.n
        shrunk += (pre.reduced.m < lp.m) or (pre.reduced.n < lp.n)
    assert shrunk >= 3


def test_singleton_rows_and_fixed_columns_postsolve_duals():
    """min 2 x0 + x1 with x0 + x1 + x2 = 4, a singleton row 2 x0 >= 6 (active
    at the optimum x0 = 3, x1 = 0.5) and a fixed column x2 = 0.5: the singleton
    row's multiplier comes back from x0's reduced cost; verify() certifies the
    postsolved point."""
    inf = np.inf
    row = np.array([0, 0, 0, 1]); col = np.array([0, 1, 2, 0]); val = np.array([1.0, 1.0, 1.0, 2.0])
    lp = B.RangedLP(2, 3, row, col, val, np.array([2.0, 1.0, 0.0]), np.array([4.0, 6.0]), np.array([4.0, inf]),
                    np.array([0.0, 0.0, 0.5]), np.array([10.0, 10.0, 0.5]))
    pre = B.Presolved(lp)
    assert pre.status == 0 and pre.reduced.m == 1 and pre.reduced.n == 2
    pre2, (x, y) = solve_original_on_cpu(lp)
    v = O.verify(as_oracle(lp), x, y)
    assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6, (x, y, v)
    assert v["objective"] == pytest.approx(2 * 3.0 + 0.5, abs=1e-6)
    assert y[1] > 0  # the singleton row x0 >= 3 carries the multiplier


def test_presolve_reports_infeasible_and_unbounded():
    inf = np.inf
    # an empty row 1 <= 0 <= 2
    lp = B.RangedLP(2, 2, np.array([0, 0]), np.array([0, 1]), np.array([1.0, 1.0]), np.array([1.0, 1.0]),
                    np.array([0.0, 1.0]), np.array([5.0, 2.0]), np.zeros(2), np.full(2, 10.0))
    assert B.Presolved(lp).status == 1
    # an empty column with negative cost and no upper bound
    lp = B.RangedLP(1, 2, np.array([0]), np.array([0]), np.array([1.0]), np.array([1.0, -1.0]),
                    np.array([0.0]), np.array([5.0]), np.zeros(2), np.array([10.0, inf]))
    assert B.Presolved(lp).status == 2
    # contradictory singleton rows: x >= 3 and x <= 1
    lp = B.RangedLP(2, 1, np.array([0, 1]), np.array([0, 0]), np.array([1.0, 1.0]), np.array([1.0]),
                    np.array([3.0, -inf]), np.array([inf, 1.0]), np.zeros(1), np.full(1, 10.0))
    assert B.Presolved(lp).status == 1
