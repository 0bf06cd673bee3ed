"""End-to-end parity of the device PDLP engine with the reference.

Every returned point is certified by the oracle's restated verify()
(src/verify.cpp:24-103) on the unscaled PDLP form -- not by the engine's own
numbers -- and its objective is compared with the reference CPU PDLP and the
reference FP64 dual simplex on the same inputs (golden fixtures made by
running the reference, tests/golden/make_golden.py). Tolerances:
  * tol 1e-6: eps_P, eps_D, eps_G <= 1e-6 (certified); the engine's own
    eps_P/eps_D/eps_G agree with the independent check; objective within
    2.5e-6 relative of the dual simplex (what eps_G <= 1e-6 allows, see
    conftest.GAP_BOUND_1E6) and within 2.5e-6 plus the reference PDLP's own
    distance from the optimum of the reference CPU PDLP's 1e-6 point; the
    random family within 1e-6 of both;
  * tol 1e-8: objective within 1e-6 relative of the dual simplex and of the
    reference PDLP at 1e-8.
"""
import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import (OBJ_TOL, as_form, fixture_names, fixture_obj_tol, fixture_ref_tol, golden_index, load_fixture,
                      random_case, rel)

pytestmark = pytest.mark.gpu

G = golden_index()


def certified(U, res, tol):
    v = O.verify(as_form(U), res.x, res.y)
    worst = max(v["eps_P"], v["eps_D"], v["eps_G"])
    return v, worst


@pytest.mark.parametrize("precision", [B.PREC_FP64, B.PREC_MIXED])
@pytest.mark.parametrize("name", fixture_names())
def test_fixture_tol_1e6(name, precision):
    U, S, Dr, Dc = load_fixture(name)
    g = G["fixtures"][name]
    r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 500000, 64, 1e-6, precision=precision)
    assert r.converged, (r.iterations, r.eps_P, r.eps_D, r.eps_G)
    v, worst = certified(U, r, 1e-6)
    assert worst <= 1e-6 * (1 + 1e-9), v
    # the engine's own report (its device-side KKT check) agrees with the independent check
    assert r.eps_P == pytest.approx(v["eps_P"], rel=1e-6, abs=1e-12)
    assert r.eps_D == pytest.approx(v["eps_D"], rel=1e-6, abs=1e-12)
    assert r.eps_G == pytest.approx(v["eps_G"], rel=1e-6, abs=1e-12)
    b_spx, b_ref = fixture_obj_tol(name), fixture_ref_tol(name)
    e_spx = rel(v["objective"], g["simplex"]["objective"])
    e_ref = rel(v["objective"], g["pdlp"]["1e-06"]["form_objective"])
    print(f"OBJ {name} prec={precision} vs_simplex={e_spx:.2e} (bound {b_spx:.2e}) vs_ref_pdlp={e_ref:.2e} "
          f"(bound {b_ref:.2e})")
    assert e_spx <= b_spx and e_ref <= b_ref, (e_spx, e_ref, b_spx, b_ref)


@pytest.mark.parametrize("name", ["afiro", "sc50a", "blend", "beaconfd", "israel", "share1b"])
def test_fixture_tol_1e8(name):
    U, S, Dr, Dc = load_fixture(name)
    g = G["fixtures"][name]
    r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 500000, 64, 1e-8)
    assert r.converged
    v, worst = certified(U, r, 1e-8)
    assert worst <= 1e-8 * (1 + 1e-6)
    assert rel(v["objective"], g["simplex"]["objective"]) <= 1e-6
    assert rel(v["objective"], g["pdlp"]["1e-08"]["form_objective"]) <= 1e-6


@pytest.mark.parametrize("key", sorted(G["random"].keys()))
def test_random_family(key):
    lp, U, S, Dr, Dc, g = random_case(key)
    for tol in (1e-6, 1e-8):
        r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 500000, 64, tol)
        assert r.converged
        v, worst = certified(U, r, tol)
        assert worst <= tol * (1 + 1e-6)
        assert r.eps_P == pytest.approx(v["eps_P"], rel=1e-6, abs=1e-12)
        assert r.eps_D == pytest.approx(v["eps_D"], rel=1e-6, abs=1e-12)
        assert r.eps_G == pytest.approx(v["eps_G"], rel=1e-6, abs=1e-12)
        e_spx = rel(v["objective"], g["simplex"]["objective"])
        e_ref = rel(v["objective"], g["pdlp"][f"{tol:g}"]["form_objective"])
        print(f"OBJ {key} tol={tol:g} vs_simplex={e_spx:.2e} vs_ref_pdlp={e_ref:.2e}")
        assert e_spx <= OBJ_TOL and e_ref <= OBJ_TOL, (e_spx, e_ref)


@pytest.mark.parametrize("name", ["afiro", "blend", "israel", "share1b"])
def test_fp64_trajectory_matches_restatement(name):
    """FP64 mode takes the reference's decisions. PDHG amplifies rounding
    (a 1e-15 perturbation of A moves the reference's own iterate by up to 3e-4
    after 200 attempts on israel), so the point is compared after 64 attempts
    (one KKT check, one restart decision) and the decision counts after 200."""
    U, S, Dr, Dc = load_fixture(name)
    ref = O.pdlp_run(U, S, Dr, Dc, max_iterations=64, check_every=64, tol=1e-12)
    r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 64, 64, 1e-12, precision=B.PREC_FP64)
    assert r.iterations == ref["iterations"] == 64
    assert r.restarts == ref["restarts"]
    assert r.stats["accepted"] == ref["accepted"]
    scale_x = 1.0 + np.abs(ref["x"]).max()
    scale_y = 1.0 + np.abs(ref["y"]).max()
    assert np.abs(r.x - ref["x"]).max() <= 1e-7 * scale_x
    assert np.abs(r.y - ref["y"]).max() <= 1e-7 * scale_y
    ref = O.pdlp_run(U, S, Dr, Dc, max_iterations=200, check_every=64, tol=1e-12)
    r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 200, 64, 1e-12, precision=B.PREC_FP64)
    assert r.iterations == ref["iterations"]
    assert r.restarts == ref["restarts"]
    assert r.stats["accepted"] == ref["accepted"]


def test_engine_resident_repeat_is_deterministic():
    U, S, Dr, Dc = load_fixture("share1b")
    with B.Engine(U, S, Dr, Dc) as e:
        a = e.solve(tol=1e-6, max_iterations=500000)
        b = e.solve(tol=1e-6, max_iterations=500000)
    assert a.iterations == b.iterations
    np.testing.assert_array_equal(a.x, b.x)
    np.testing.assert_array_equal(a.y, b.y)


def test_stop_flag_before_start_returns_best_unconverged():
    """stop_flag semantics of include/pdlp.hpp:30-34: return early, converged=false."""
    U, S, Dr, Dc = load_fixture("share1b")
    f = B.StopFlag()
    f.set()
    r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 500000, 64, 1e-6, stop_flag=f)
    assert not r.converged
    assert r.stats["exit_reason"] == B.EXIT_STOPPED
    assert r.iterations <= 32
    assert np.all(np.isfinite(r.x)) and np.all(np.isfinite(r.y))
    v, _ = certified(U, r, 1e-6)
    assert r.eps_P == pytest.approx(v["eps_P"], rel=1e-6, abs=1e-12)


def test_stop_callback_stops_a_running_solve():
    """b2_solve_opts::stop_poll (what the shim passes for the reference's
    std::atomic<bool> stop flag): polled by the waiting thread while the
    persistent kernel runs; a nonzero answer stops it like stop_flag."""
    import ctypes as C
    lp = B.gen_random_lp(20_000, 60_000, 6, 7, True)
    U, S, Dr, Dc, _ = B.prepare(lp)
    calls = [0]

    @C.CFUNCTYPE(C.c_int32, C.c_void_p)
    def poll(_ctx):
        calls[0] += 1
        return 1 if calls[0] > 50 else 0

    r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 10_000_000, 64, 1e-12, precision=B.PREC_FP64,
                         stop_poll=C.cast(poll, C.c_void_p).value)
    assert not r.converged
    assert r.stats["exit_reason"] == B.EXIT_STOPPED
    assert calls[0] > 50
    assert np.all(np.isfinite(r.x)) and np.all(np.isfinite(r.y))


def test_iteration_limit_reports_best_point():
    U, S, Dr, Dc = load_fixture("share1b")
    r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 1000, 64, 1e-9, precision=B.PREC_FP64)
    assert not r.converged
    assert r.iterations == 1000
    assert r.stats["exit_reason"] == B.EXIT_MAX_ITER
    v, _ = certified(U, r, 1e-9)
    assert r.eps_P == pytest.approx(v["eps_P"], rel=1e-6, abs=1e-12)


def test_time_limit_exits_cleanly():
    lp = B.gen_random_lp(3000, 9000, 6, 3, True)
    U, S, Dr, Dc, _ = B.prepare(lp)
    r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 10_000_000, 64, 1e-12, time_limit_s=0.02, precision=B.PREC_FP64)
    assert not r.converged
    assert r.stats["exit_reason"] == B.EXIT_TIME_LIMIT


def test_barrier_timeout_reports_error_and_engine_stays_usable():
    """A device-side wait that runs out (CTA 0 held back 50 ms, 1 ms limit) ends the kernel with
    B2_ERR_TIMEOUT; the context stays usable and the next solve succeeds."""
    lp = B.gen_random_lp(3000, 9000, 6, 4, True)
    U, S, Dr, Dc, _ = B.prepare(lp)
    with B.Engine(U, S, Dr, Dc) as e:
        assert e.info()["ctas"] >= 2
        with pytest.raises(B.B2Error) as err:
            e.solve(tol=1e-6, barrier_timeout_s=1e-3, max_ctas=4, debug_delay_us=50000)
        assert err.value.code == B.B2_ERR_TIMEOUT
        r = e.solve(tol=1e-6, max_iterations=500000)
        assert r.converged


def test_inequality_rows_and_free_columns():
    """>= rows (sign projection of y) and free / one-sided columns (dual sign
    rules of verify.cpp:42-57)."""
    rng = np.random.default_rng(8)
    m, n = 40, 90
    A = (rng.random((m, n)) < 0.15) * rng.uniform(-1, 1, (m, n))
    A[np.arange(m), rng.integers(0, n, m)] += 1.0
    x0 = rng.uniform(0, 2, n)
    b = A @ x0
    r_, c_ = np.nonzero(A)
    l = np.zeros(n); u = np.full(n, 5.0)
    l[:10] = -np.inf; u[:5] = np.inf          # five free columns, five with only an upper bound
    rL = b - np.where(np.arange(m) % 2 == 0, 0.0, 1.0)
    rU = np.where(np.arange(m) % 2 == 0, b, np.inf)
    cost = A.T @ rng.normal(size=m) + rng.uniform(0, 1, n)
    cost[:5] = A[:, :5].T @ rng.normal(size=m) * 0  # free columns must have a dual-feasible cost
    lp = B.RangedLP(m, n, r_, c_, A[r_, c_], cost, rL, rU, l, u)
    U, S, Dr, Dc, _ = B.prepare(lp)
    ref = O.pdlp_run(as_form(U), as_form(S), Dr, Dc, max_iterations=400000, tol=1e-7)
    r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 400000, 64, 1e-7)
    assert r.converged == ref["converged"]
    if ref["converged"]:
        v, worst = certified(U, r, 1e-7)
        assert worst <= 1e-7 * (1 + 1e-6)
        vr = O.verify(as_form(U), ref["x"], ref["y"])
        # both points within 1e-7 KKT of the same optimum
        assert rel(v["objective"], vr["objective"]) <= OBJ_TOL


def test_transport_split_layout_solve_certified():
    """A transportation LP on the whole-GPU layout (tuned, split slices) and on
    the batched layout (neither): both certified, objectives agree."""
    lp = B.gen_transport(300, 500, 7)
    U, S, Dr, Dc, _ = B.prepare(lp)
    r = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 500000, 64, 1e-6)
    assert r.converged
    v = O.verify(as_form(U), r.x, r.y)
    assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6 * (1 + 1e-9)
    with B.Batch([(U, S, Dr, Dc)]) as bt:
        res, _ = bt.solve(max_iterations=500000, tol=1e-6)
        x, y = bt.solution(0)
    assert res[0]["converged"]
    v2 = O.verify(as_form(U), x, y)
    assert max(v2["eps_P"], v2["eps_D"], v2["eps_G"]) <= 1e-6 * (1 + 1e-9)
    assert rel(v["objective"], v2["objective"]) <= OBJ_TOL
    # repeated solves on the split layout are bit-identical (fixed segment order)
    with B.Engine(U, S, Dr, Dc) as eng:
        a = eng.solve(max_iterations=3000, tol=1e-9)
        b = eng.solve(max_iterations=3000, tol=1e-9)
    np.testing.assert_array_equal(a.x, b.x)
    np.testing.assert_array_equal(a.y, b.y)
