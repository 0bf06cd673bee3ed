"""The batched engine (many LPs, one persistent launch, one CTA per LP).

* every LP's answer is certified by the oracle's restated verify() and agrees
  with the reference's dual simplex / reference PDLP (golden fixtures);
* an LP's answer is bit-identical alone and inside any batch (its arithmetic
  never depends on the other LPs);
* the batch answer agrees with the single-LP engine within the solve tolerance.
"""
import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import OBJ_TOL, fixture_obj_tol, as_form, fixture_names, golden_index, load_fixture, random_case, rel

pytestmark = pytest.mark.gpu

G = golden_index()


def fixture_problems():
    names = fixture_names()
    return names, [load_fixture(n) for n in names]


@pytest.mark.parametrize("precision", [B.PREC_FP64, B.PREC_MIXED])
def test_batch_of_fixtures_certified(precision):
    names, probs = fixture_problems()
    keys = sorted(G["random"].keys())
    for k in keys:
        _, U, S, Dr, Dc, _ = random_case(k)
        probs.append((U, S, Dr, Dc))
    with B.Batch(probs) as bt:
        res, ms = bt.solve(max_iterations=500000, tol=1e-6, precision=precision)
        assert ms > 0
        for i, (U, S, Dr, Dc) in enumerate(probs):
            r = res[i]
            assert r["converged"], (i, r)
            x, y = bt.solution(i)
            v = O.verify(as_form(U), x, y)
            assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6 * (1 + 1e-9)
            assert r["eps_P"] == pytest.approx(v["eps_P"], rel=1e-6, abs=1e-12)
            ref = (G["fixtures"][names[i]]["simplex"]["objective"] if i < len(names)
                   else G["random"][keys[i - len(names)]]["simplex"]["objective"])
            bound = fixture_obj_tol(names[i]) if i < len(names) else OBJ_TOL
            assert rel(v["objective"], ref) <= bound


def test_answer_is_identical_alone_and_in_the_mix():
    names, probs = fixture_problems()
    with B.Batch(probs) as bt:
        res, _ = bt.solve(max_iterations=500000, tol=1e-6)
        mixed = [bt.solution(i) for i in range(len(probs))]
    for i in (0, 3, len(probs) - 1):
        with B.Batch([probs[i]]) as one:
            r1, _ = one.solve(max_iterations=500000, tol=1e-6)
            x, y = one.solution(0)
        assert r1[0]["iterations"] == res[i]["iterations"]
        np.testing.assert_array_equal(x, mixed[i][0])
        np.testing.assert_array_equal(y, mixed[i][1])
    # a different batch composition and order
    sub = [probs[j] for j in (5, 0, 9, 2)]
    with B.Batch(sub) as bt2:
        bt2.solve(max_iterations=500000, tol=1e-6)
        x, y = bt2.solution(1)
    np.testing.assert_array_equal(x, mixed[0][0])


def test_batch_matches_single_engine():
    U, S, Dr, Dc = load_fixture("israel")
    single = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 500000, 64, 1e-8)
    with B.Batch([(U, S, Dr, Dc)]) as bt:
        res, _ = bt.solve(max_iterations=500000, tol=1e-8)
        x, y = bt.solution(0)
    assert res[0]["converged"] and single.converged
    v1 = O.verify(as_form(U), single.x, single.y)
    v2 = O.verify(as_form(U), x, y)
    assert rel(v1["objective"], v2["objective"]) <= 1e-6


def test_uneven_random_batch():
    shapes = [s for s in B.batch_family_shapes(48, seed=5, m_lo=50, m_hi=600)]
    probs = []
    for (m, n, k, seed) in shapes:
        lp = B.gen_random_lp(m, n, k, seed, True)
        U, S, Dr, Dc, _ = B.prepare(lp)
        probs.append((U, S, Dr, Dc))
    with B.Batch(probs) as bt:
        res, ms = bt.solve(max_iterations=400000, tol=1e-6)
        assert all(r["converged"] for r in res)
        for i in (0, 17, 47):
            x, y = bt.solution(i)
            v = O.verify(as_form(probs[i][0]), x, y)
            assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6 * (1 + 1e-9)


def test_batch_stop_flag():
    _, probs = fixture_problems()
    f = B.StopFlag()
    f.set()
    with B.Batch(probs) as bt:
        res, _ = bt.solve(max_iterations=500000, tol=1e-9, stop_flag=f)
    assert all(not r["converged"] for r in res if r["iterations"] > 64)
    assert all(r["exit_reason"] in (B.EXIT_STOPPED, B.EXIT_CONVERGED) for r in res)


def test_cluster_path_certified():
    """LPs above the cluster threshold are solved by a cluster of 16 CTAs
    (hardware cluster barrier); answers are certified like the one-CTA path."""
    names, probs = fixture_problems()
    with B.Batch(probs) as bt:
        res, _ = bt.solve(max_iterations=500000, tol=1e-6, batch_cluster_nnz=1500)
        for i, (U, S, Dr, Dc) in enumerate(probs):
            assert res[i]["converged"], (names[i], res[i])
            x, y = bt.solution(i)
            v = O.verify(as_form(U), x, y)
            assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6 * (1 + 1e-9)
            assert rel(v["objective"], G["fixtures"][names[i]]["simplex"]["objective"]) <= fixture_obj_tol(names[i])
        # the cluster answer is deterministic and independent of the batch
        x0, _ = bt.solution(len(probs) - 2)
    with B.Batch([probs[len(probs) - 2]]) as one:
        one.solve(max_iterations=500000, tol=1e-6, batch_cluster_nnz=1500)
        x1, _ = one.solution(0)
    np.testing.assert_array_equal(x0, x1)


def test_tail_lane_certified_deterministic_and_untouched_below_the_switch():
    """The tail lane (batch_tail_attempts): LPs still running at 300 attempts
    yield there and finish on 16-CTA clusters in a second launch. Every answer
    is certified; two runs give the same bits; LPs that finish before the
    switch are bit-identical to the batch without a tail lane."""
    names, probs = fixture_problems()
    keys = sorted(G["random"].keys())
    for k in keys:
        _, U, S, Dr, Dc, _ = random_case(k)
        probs.append((U, S, Dr, Dc))
    runs = []
    for tail in (300, 300, 0):
        with B.Batch(probs) as bt:
            res, _ = bt.solve(max_iterations=500000, tol=1e-6, batch_tail_attempts=tail)
            runs.append((res, [bt.solution(i) for i in range(len(probs))]))
    (r1, s1), (r2, s2), (r0, s0) = runs
    moved = [i for i, r in enumerate(r1) if r["group_ctas"] > 1]
    assert moved and len(moved) < len(probs)
    for i, (U, S, Dr, Dc) in enumerate(probs):
        assert r1[i]["converged"], (i, r1[i])
        assert r1[i]["iterations"] == r2[i]["iterations"]
        np.testing.assert_array_equal(s1[i][0], s2[i][0])
        v = O.verify(as_form(U), *s1[i])
        assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6 * (1 + 1e-9)
        if i not in moved:
            assert r1[i]["iterations"] == r0[i]["iterations"] <= 300 + 64
            np.testing.assert_array_equal(s1[i][0], s0[i][0])
