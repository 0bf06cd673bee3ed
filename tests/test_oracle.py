"""Pins the oracle: the C restatement (oracle/pdlp_oracle.c) against the golden
fixtures made by the reference itself, and -- where the reference library is
built (oracle/_ref) -- against the reference directly, bit for bit."""
import numpy as np
import pytest

import b200pdlp
import oracle as O
from conftest import fixture_names, golden_index, load_fixture, random_case

FIX = fixture_names()


@pytest.mark.parametrize("name", FIX)
def test_restatement_reproduces_reference_pdlp(name):
    """Same iterations, restarts, residuals and objective as the reference's
    solve_pdhg on the reference's own fixture (tests/run_checks.cpp cases)."""
    g = golden_index()["fixtures"][name]["pdlp"]["1e-06"]
    U, S, Dr, Dc = load_fixture(name)
    r = O.pdlp_run(U, S, Dr, Dc, max_iterations=500000, check_every=64, tol=1e-6)
    assert r["iterations"] == g["iterations"]
    assert r["restarts"] == g["restarts"]
    assert r["converged"] == g["converged"]
    assert r["eps_P"] == pytest.approx(g["eps_P"], rel=1e-9, abs=1e-300)
    v = O.verify(U, r["x"], r["y"])
    assert v["objective"] == pytest.approx(g["form_objective"], rel=1e-12)


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built here")
@pytest.mark.parametrize("name", ["afiro", "sc50a", "blend", "beaconfd", "israel"])
def test_restatement_bitexact_with_reference(name):
    U, S, Dr, Dc = load_fixture(name)
    r = O.pdlp_run(U, S, Dr, Dc, max_iterations=500000, tol=1e-6)
    lib = O.reference()
    h = lib.ref_from_arrays(U.m, U.n, U.nnz, U.row, U.col, U.val, U.c, U.rL, U.rU, U.l, U.u, U.obj_offset, 0)
    P = O.RefProblem(h, lib)
    # same form in, no presolve: the reference pipeline rebuilds the PDLP form and scaling
    ref = P.solve_pdhg(max_iterations=500000, tol=1e-6)
    assert ref["iterations"] == r["iterations"]
    np.testing.assert_array_equal(ref["x"], r["x"])
    np.testing.assert_array_equal(ref["y"], r["y"])


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built here")
@pytest.mark.parametrize("name", FIX)
def test_verify_and_scale_bitexact_with_reference(name):
    U, S, Dr, Dc = load_fixture(name)
    rng = np.random.default_rng(3)
    x = rng.normal(size=U.n)
    y = rng.normal(size=U.m)
    lib = O.reference()
    h = lib.ref_from_arrays(U.m, U.n, U.nnz, U.row, U.col, U.val, U.c, U.rL, U.rU, U.l, U.u, U.obj_offset, 0)
    P = O.RefProblem(h, lib)
    a = P.verify_form(P.ORIGINAL, x, y)
    b = O.verify(U, x, y)
    for k in ("eps_P", "eps_D", "eps_G", "objective"):
        assert a[k] == b[k] or (np.isinf(a[k]) and np.isinf(b[k]))
    s1, Dr1, Dc1 = O.scale(U)
    s2, Dr2, Dc2 = O.ref_scale(U)
    np.testing.assert_array_equal(s1.val, s2.val)
    np.testing.assert_array_equal(Dr1, Dr2)
    np.testing.assert_array_equal(Dc1, Dc2)
    # and the fixture's stored scaling is what scale() gives
    np.testing.assert_array_equal(s1.val, S.val)
    np.testing.assert_array_equal(Dr1, Dr)


@pytest.mark.parametrize("key", sorted(golden_index()["random"].keys()))
def test_random_family_regenerates_bitexact(key):
    """The seeded generator still produces the LP the golden results were made on."""
    from conftest import digest
    lp, *_ , g = random_case(key)
    assert digest(lp) == g["digest"]


@pytest.mark.parametrize("key", sorted(golden_index()["random"].keys()))
def test_oracle_generator_equals_product_generator(key):
    """The oracle's restated generator (used where the product library must not
    be loaded: the benchmark's reference arm, the golden records) builds the
    same LP, bit for bit, as the product's."""
    from conftest import digest
    g = golden_index()["random"][key]
    lp = O.gen_random_lp(g["m"], g["n"], g["k"], g["seed"], g["fp32"])
    assert digest(lp) == g["digest"]
    assert digest(lp) == digest(b200pdlp.gen_random_lp(g["m"], g["n"], g["k"], g["seed"], g["fp32"]))


@pytest.mark.parametrize("S,D,seed", [(7, 5, 0), (60, 40, 3), (2000, 500, 1)])
def test_oracle_transport_generator_equals_product_generator(S, D, seed):
    from conftest import digest
    assert digest(O.gen_transport(S, D, seed)) == digest(b200pdlp.gen_transport(S, D, seed))


def test_large_records_pin_the_generated_lps():
    """tests/golden/large.json stores the content digests of the benchmark-size
    LPs the reference solved; the oracle's generator still builds them."""
    import json
    import os
    from conftest import GOLDEN, digest
    path = os.path.join(GOLDEN, "large.json")
    if not os.path.exists(path):
        pytest.skip("no large-LP records")
    rec = json.load(open(path))
    p = rec["transport"]["lp"]
    assert digest(O.gen_transport(p["S"], p["D"], p["seed"])) == rec["transport"]["digest"]
    p = rec["large"]["lp"]
    assert digest(O.gen_random_lp(p["m"], p["n"], p["k"], p["seed"], p["fp32"])) == rec["large"]["digest"]


def test_restatement_small_random_lp_matches_reference_objective():
    key = "rand_m300_n900_k4_s7_f32"
    lp, U, S, Dr, Dc, g = random_case(key)
    r = O.pdlp_run(O.LPForm(U.m, U.n, U.row, U.col, U.val, U.c, U.rL, U.rU, U.l, U.u),
                   O.LPForm(S.m, S.n, S.row, S.col, S.val, S.c, S.rL, S.rU, S.l, S.u), Dr, Dc, tol=1e-8,
                   max_iterations=500000)
    assert r["converged"]
    obj = float(np.dot(U.c, r["x"]))
    ref = g["simplex"]["objective"]
    assert abs(obj - ref) / max(1.0, abs(ref)) < 1e-6


@pytest.mark.parametrize("kind", ["random", "transport"])
def test_generated_lp_round_trips_through_the_reference_mps_reader(kind, tmp_path):
    """Generated benchmark LPs are handed to the reference's own tools as MPS
    (%.17g, written by oracle/ref_capi.cpp): the reference's read_mps must give
    back the same LP, value for value."""
    import b200pdlp as B
    if not O.reference_available():
        pytest.skip("oracle/_ref is not built")
    lp = B.gen_random_lp(300, 900, 6, 5, False) if kind == "random" else B.gen_transport(40, 30, 2)
    P = O.RefProblem.from_form(O.LPForm(lp.m, lp.n, lp.row, lp.col, lp.val, lp.c, lp.rL, lp.rU, lp.l, lp.u),
                               use_presolve=False)
    path = str(tmp_path / "gen.mps")
    P.write_mps(path)
    a = P.form(P.ORIGINAL)
    b = O.RefProblem.from_mps(path, use_presolve=False).form(O.RefProblem.ORIGINAL)
    assert (a.m, a.n, a.nnz) == (b.m, b.n, b.nnz)
    ka = np.lexsort((a.col, a.row))
    kb = np.lexsort((b.col, b.row))
    np.testing.assert_array_equal(a.row[ka], b.row[kb])
    np.testing.assert_array_equal(a.col[ka], b.col[kb])
    np.testing.assert_array_equal(a.val[ka], b.val[kb])
    for f in ("c", "rL", "rU", "l", "u"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
    assert a.obj_offset == b.obj_offset


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built here")
@pytest.mark.parametrize("seed", range(2, 10))
def test_restatement_bitexact_with_reference_c0_seed_sweep(seed):
    """The 600 x 1,800 random LP (6 nonzeros per column, FP64 values, the CPU
    configuration) over a sweep of seeds: the restatement takes the reference's
    solve_pdhg steps to 1e-6, bit for bit, and converges with it."""
    import b200pdlp as B
    lp = B.gen_random_lp(600, 1800, 6, seed, False)
    U, S, Dr, Dc, _ = B.prepare(lp)
    fU = O.LPForm(U.m, U.n, U.row, U.col, U.val, U.c, U.rL, U.rU, U.l, U.u, U.obj_offset)
    fS = O.LPForm(S.m, S.n, S.row, S.col, S.val, S.c, S.rL, S.rU, S.l, S.u, S.obj_offset)
    r = O.pdlp_run(fU, fS, Dr, Dc, max_iterations=500000, tol=1e-6)
    ref = O.RefProblem.from_form(fU, use_presolve=False).solve_pdhg(max_iterations=500000, tol=1e-6)
    assert r["converged"] and ref["converged"]
    assert ref["iterations"] == r["iterations"] and ref["restarts"] == r["restarts"]
    np.testing.assert_array_equal(ref["x"], r["x"])
    np.testing.assert_array_equal(ref["y"], r["y"])
