"""The served stream (b2_server_*): LPs arriving over time, continuous batching.

* every answer is certified by the oracle's restated verify() and agrees with
  the reference's dual simplex (golden fixtures);
* rounds pause LPs at their deadline and resume them in the next round; the
  answer is bit-identical to the uninterrupted batched solve of the same LP;
* an LP's answer is bit-identical alone and in a mix that arrives around it;
* the whole-GPU lane (time-sliced one-LP engine) returns the one-LP engine's
  answer bit for bit;
* admission keeps the resident footprint under the HBM budget; a malformed
  request fails alone and the server keeps serving.
"""
import time

import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import OBJ_TOL, as_form, fixture_names, fixture_obj_tol, golden_index, load_fixture, random_case, rel

pytestmark = pytest.mark.gpu

G = golden_index()
TOL = 1e-6


def fixture_problems():
    names = fixture_names()
    return names, [load_fixture(n) for n in names]


def certified(U, res, ref_obj, name=None):
    """Certified by the oracle's verify; objective within 1e-6 of the dual
    simplex (the fixture's own bound for a named fixture, see fixture_obj_tol)."""
    v = O.verify(as_form(U), res.x, res.y)
    assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= TOL * (1 + 1e-9), v
    bound = fixture_obj_tol(name) if name else OBJ_TOL
    assert rel(v["objective"], ref_obj) <= bound, (name, rel(v["objective"], ref_obj), bound)
    return v


@pytest.mark.parametrize("precision", [B.PREC_MIXED, B.PREC_FP64])
def test_served_answers_certified_and_equal_to_uninterrupted_batch(precision):
    names, probs = fixture_problems()
    keys = sorted(G["random"].keys())
    refs = [G["fixtures"][n]["simplex"]["objective"] for n in names]
    for k in keys:
        _, U, S, Dr, Dc, g = random_case(k)
        probs.append((U, S, Dr, Dc))
        refs.append(g["simplex"]["objective"])
    # tiny rounds: every LP is paused and resumed many times
    with B.Server(round_ms=0.2, precision=precision, max_iterations=500000, tol=TOL) as srv:
        tickets = [srv.submit(U) for (U, _, _, _) in probs]
        out = [srv.wait(t, timeout_s=300.0) for t in tickets]
    assert all(o is not None for o in out)
    assert max(info["rounds"] for _, info in out) > 3
    with B.Batch(probs) as bt:
        res, _ = bt.solve(max_iterations=500000, tol=TOL, precision=precision)
        for i, (U, S, Dr, Dc) in enumerate(probs):
            r, info = out[i]
            assert r.converged, (i, r.stats)
            assert info["lane"] == 0
            certified(U, r, refs[i], names[i] if i < len(names) else None)
            x, y = bt.solution(i)
            assert r.iterations == res[i]["iterations"]
            np.testing.assert_array_equal(r.x, x)
            np.testing.assert_array_equal(r.y, y)


def test_answer_is_identical_alone_and_in_an_arriving_mix():
    names, probs = fixture_problems()
    target = names.index("israel")
    U = probs[target][0]
    with B.Server(round_ms=0.5) as srv:
        alone, _ = srv.wait(srv.submit(U), timeout_s=300.0)
    shapes = B.batch_family_shapes(40, seed=11, m_lo=50, m_hi=800)
    others = []
    for (m, n, k, seed) in shapes:
        lp = B.gen_random_lp(m, n, k, seed, True)
        others.append(B.prepare(lp)[0])
    with B.Server(round_ms=0.5) as srv:
        early = [srv.submit(o) for o in others[:20]]
        time.sleep(0.01)
        t = srv.submit(U)
        time.sleep(0.005)
        late = [srv.submit(o) for o in others[20:]]
        mixed, info = srv.wait(t, timeout_s=300.0)
        rest = [srv.wait(k, timeout_s=300.0) for k in early + late]
        st = srv.stats()
    assert all(r is not None and r[0].converged for r in rest)
    assert st["completed"] == 41 and st["failed"] == 0 and st["rounds"] >= 1
    assert alone.iterations == mixed.iterations
    np.testing.assert_array_equal(alone.x, mixed.x)
    np.testing.assert_array_equal(alone.y, mixed.y)
    certified(U, mixed, G["fixtures"]["israel"]["simplex"]["objective"], "israel")


@pytest.mark.parametrize("precision", [B.PREC_MIXED, B.PREC_FP64])
def test_whole_gpu_lane_matches_one_lp_engine(precision):
    _, U, S, Dr, Dc, g = random_case(sorted(G["random"].keys())[0])
    with B.Engine(U, S, Dr, Dc) as eng:
        ref = eng.solve(max_iterations=500000, tol=TOL, precision=precision)
    with B.Server(grid_nnz=1, grid_slice_ms=0.3, precision=precision, max_iterations=500000, tol=TOL) as srv:
        r, info = srv.wait(srv.submit(U), timeout_s=300.0)
        st = srv.stats()
    assert info["lane"] == 1 and info["rounds"] > 1 and st["grid_slices"] == info["rounds"]
    assert r.converged and r.iterations == ref.iterations
    np.testing.assert_array_equal(r.x, ref.x)
    np.testing.assert_array_equal(r.y, ref.y)
    certified(U, r, g["simplex"]["objective"])


def test_admission_keeps_footprint_under_budget():
    shapes = B.batch_family_shapes(24, seed=3, m_lo=200, m_hi=600)
    lps = [B.prepare(B.gen_random_lp(m, n, k, seed, True))[0] for (m, n, k, seed) in shapes]
    budget = 3_000_000  # a few LPs at a time
    with B.Server(hbm_budget_bytes=budget, round_ms=1.0) as srv:
        ts = [srv.submit(U) for U in lps]
        out = [srv.wait(t, timeout_s=300.0) for t in ts]
        st = srv.stats()
    assert all(r is not None and r[0].converged for r in out)
    sizes = [info["device_bytes"] for _, info in out]
    assert max(sizes) <= budget
    assert st["peak_bytes"] <= budget
    assert st["bytes_in_use"] == 0 and st["resident"] == 0


def test_malformed_request_fails_alone():
    U, S, Dr, Dc = load_fixture("afiro")
    bad = B.RangedLP.like(U)
    bad.col = bad.col.copy()
    bad.col[0] = U.n + 7
    with B.Server(round_ms=1.0) as srv:
        t_bad = srv.submit(bad)
        t_ok = srv.submit(U)
        with pytest.raises(B.B2Error) as e:
            srv.wait(t_bad, timeout_s=60.0)
        assert e.value.code == B.B2_ERR_INVALID
        r, _ = srv.wait(t_ok, timeout_s=60.0)
        st = srv.stats()
    assert r.converged and st["failed"] == 1 and st["completed"] == 1
    certified(U, r, G["fixtures"]["afiro"]["simplex"]["objective"], "afiro")


@pytest.mark.parametrize("cluster_nnz", [1, 3000])
def test_cluster_lane_equals_batched_cluster_path(cluster_nnz):
    """Served LPs above cluster_nnz stored entries run on 16-CTA clusters (beside
    a one-CTA launch for the rest); each answer is the batched engine's on the
    same path, bit for bit, however the rounds cut it."""
    names, probs = fixture_problems()
    with B.Server(round_ms=0.3, cluster_nnz=cluster_nnz, max_iterations=500000, tol=TOL) as srv:
        out = [srv.wait(t, timeout_s=300.0) for t in [srv.submit(U) for (U, _, _, _) in probs]]
    with B.Batch(probs) as bt:
        res, _ = bt.solve(max_iterations=500000, tol=TOL, batch_cluster_nnz=cluster_nnz)
        for i, (U, _, _, _) in enumerate(probs):
            r, _ = out[i]
            assert r.converged, names[i]
            x, y = bt.solution(i)
            assert r.iterations == res[i]["iterations"], names[i]
            np.testing.assert_array_equal(r.x, x)
            np.testing.assert_array_equal(r.y, y)
            certified(U, r, G["fixtures"][names[i]]["simplex"]["objective"], names[i])


def test_pending_result_and_shutdown_with_requests_in_flight():
    """wait() with a short timeout reports a running request as pending; closing
    the server with requests in flight stops them at their next poll and
    returns promptly."""
    lps = [B.prepare(B.gen_random_lp(20_000, 60_000, 6, s, True))[0] for s in (1, 2, 3)]
    srv = B.Server(round_ms=2.0, max_iterations=2_000_000, tol=1e-9)
    ts = [srv.submit(U) for U in lps]
    assert srv.wait(ts[0], timeout_s=0.05) is None
    st = srv.stats()
    assert st["submitted"] == 3 and st["completed"] == 0
    t0 = time.perf_counter()
    srv.close()
    assert time.perf_counter() - t0 < 30.0
    # a fresh server on the same device works afterwards
    U, S, Dr, Dc = load_fixture("afiro")
    with B.Server(round_ms=1.0) as s2:
        r, _ = s2.wait(s2.submit(U), timeout_s=60.0)
    certified(U, r, G["fixtures"]["afiro"]["simplex"]["objective"], "afiro")


def test_request_file_gives_the_same_answer(tmp_path):
    """An LP submitted as a request file (read on the server's threads) is
    solved exactly as the same LP submitted from memory; a bad path fails
    its ticket alone."""
    names, probs = fixture_problems()
    U = B.RangedLP.like(probs[names.index("israel")][0])
    path = str(tmp_path / "israel.b2lp")
    B.write_lp(path, U)
    with B.Server(round_ms=0.5) as srv:
        a, _ = srv.wait(srv.submit(U), timeout_s=300.0)
        b, _ = srv.wait(srv.submit_file(path), timeout_s=300.0)
    # the file holds A row by row; the same LP, but its entries in another order
    # may change the last bits, so the answers agree through the verifier
    assert a.converged and b.converged
    va = certified(U, a, G["fixtures"]["israel"]["simplex"]["objective"])
    vb = certified(U, b, G["fixtures"]["israel"]["simplex"]["objective"])
    assert rel(va["objective"], vb["objective"]) <= 1e-6
    # the round-tripped LP in memory and the file: bit for bit
    back = B.read_lp(path)
    with B.Server(round_ms=0.5) as srv:
        c, _ = srv.wait(srv.submit(back), timeout_s=300.0)
    np.testing.assert_array_equal(c.x, b.x)
    np.testing.assert_array_equal(c.y, b.y)
    # a file whose header is sound but whose column index is out of range
    import struct
    blob = bytearray(open(path, "rb").read())
    col0 = 32 + 8 * (U.m + 1)
    blob[col0:col0 + 4] = struct.pack("<i", U.n + 9)
    bad = str(tmp_path / "bad.b2lp")
    open(bad, "wb").write(bytes(blob))
    with B.Server(round_ms=0.5) as srv:
        t_bad = srv.submit_file(bad)
        t_ok = srv.submit(U)
        with pytest.raises(B.B2Error) as e:
            srv.wait(t_bad, timeout_s=60.0)
        assert e.value.code == B.B2_ERR_INVALID
        r, _ = srv.wait(t_ok, timeout_s=300.0)
    np.testing.assert_array_equal(r.x, a.x)


def test_server_presolves_lps_as_the_caller_has_them():
    """b2_server_submit_lp: LPs as the reference reads them (before presolve,
    tests/golden/orig_<name>.npz) are presolved, put in PDLP form and scaled on
    the server's threads; the answer comes back in the original LP's space,
    with verify()'s figures taken there, and the oracle's verify agrees."""
    import os
    from conftest import GOLDEN
    names = sorted(f[5:-4] for f in os.listdir(GOLDEN) if f.startswith("orig_") and f.endswith(".npz")
                   and f[5:-4] in G["fixtures"])

    def original(name):
        z = np.load(os.path.join(GOLDEN, f"orig_{name}.npz"))
        m, n = (int(v) for v in z["o_dims"])
        return B.RangedLP(m, n, z["o_row"], z["o_col"], z["o_val"], z["o_c"], z["o_rL"], z["o_rU"], z["o_l"],
                          z["o_u"], float(z["o_off"][0]))

    # 1e-7 on the PDLP form keeps the postsolved point within 1e-6 on the original LP
    with B.Server(max_iterations=500000, tol=1e-7) as srv:
        tickets = [(nm, srv.submit_lp(original(nm))) for nm in names]
        # an LP presolve proves infeasible fails its own ticket only
        bad = B.RangedLP(2, 2, np.array([0, 0]), np.array([0, 1]), np.array([1.0, 1.0]), np.array([1.0, 1.0]),
                         np.array([0.0, 1.0]), np.array([5.0, 2.0]), np.zeros(2), np.full(2, 10.0))
        tb = srv.submit_lp(bad)
        out = [(nm, srv.wait(t, timeout_s=300.0)) for nm, t in tickets]
        with pytest.raises(B.B2Error) as e:
            srv.wait(tb, timeout_s=60.0)
        assert e.value.code == B.B2_ERR_INFEASIBLE
    for nm, (r, info) in out:
        lp = original(nm)
        assert r.converged, (nm, r.stats)
        assert r.x.shape == (lp.n,) and r.y.shape == (lp.m,)
        assert info["presolved_m"] <= lp.m + 1 and max(info["form_eps"]) <= 1e-7 * (1 + 1e-9)
        v = O.verify(as_form(lp), r.x, r.y)
        assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6, (nm, v)
        # the server's own original-space figures are verify()'s
        assert r.eps_P == pytest.approx(v["eps_P"], rel=1e-6, abs=1e-12)
        assert r.eps_D == pytest.approx(v["eps_D"], rel=1e-6, abs=1e-12)
        assert r.eps_G == pytest.approx(v["eps_G"], rel=1e-6, abs=1e-12)
        assert rel(v["objective"], G["fixtures"][nm]["simplex"]["objective"]) <= fixture_obj_tol(nm)
