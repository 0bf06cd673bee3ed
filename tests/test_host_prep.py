"""Host-side preparation of the product (no GPU): scaling, PDLP form and the
benchmark generators, checked against the oracle and the reference."""
import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import as_form, fixture_names, load_fixture


@pytest.mark.parametrize("name", fixture_names())
def test_product_scaling_bitexact_with_oracle(name):
    """b2_scale restates src/scaling.cpp:25-84; it must give the same bits."""
    U, S, Dr, Dc = load_fixture(name)
    s, dr, dc = B.scale(B.RangedLP.like(U))
    np.testing.assert_array_equal(s.val, S.val)
    np.testing.assert_array_equal(s.c, S.c)
    np.testing.assert_array_equal(s.l, S.l)
    np.testing.assert_array_equal(s.u, S.u)
    np.testing.assert_array_equal(s.rL, S.rL)
    np.testing.assert_array_equal(dr, Dr)
    np.testing.assert_array_equal(dc, Dc)


def test_product_scaling_random_family():
    lp = B.gen_random_lp(200, 600, 5, 11, False)
    s, dr, dc = B.scale(lp)
    s2, dr2, dc2 = O.scale(as_form(lp))
    np.testing.assert_array_equal(s.val, s2.val)
    np.testing.assert_array_equal(dr, dr2)
    np.testing.assert_array_equal(dc, dc2)


@pytest.mark.parametrize("shape", [(150_000, 300_000, 4, 21, True), (2_500, 1_000_000, None, 3, None)])
def test_product_scaling_on_threads_is_bitexact(shape):
    """From 262,144 entries b2_scale runs on several threads (per-thread
    maxima, row and column sums in COO order through stable orders); the bits
    must still be the serial restatement's. One random LP and a transport LP
    (1M columns of 2 entries, rows of 500 and 2,000)."""
    m, n, k, seed, fp32 = shape
    lp = B.gen_random_lp(m, n, k, seed, fp32) if k else B.gen_transport(2000, 500, seed)
    assert lp.nnz >= 1 << 18
    s, dr, dc = B.scale(lp)
    s2, dr2, dc2 = O.scale(as_form(lp))
    np.testing.assert_array_equal(s.val, s2.val)
    np.testing.assert_array_equal(s.c, s2.c)
    np.testing.assert_array_equal(s.l, s2.l)
    np.testing.assert_array_equal(s.u, s2.u)
    np.testing.assert_array_equal(s.rL, s2.rL)
    np.testing.assert_array_equal(s.rU, s2.rU)
    np.testing.assert_array_equal(dr, dr2)
    np.testing.assert_array_equal(dc, dc2)


def _mixed_rows_lp():
    # rows: E, L, G, ranged, free, E ; columns with finite / infinite bounds
    rng = np.random.default_rng(5)
    m, n = 6, 5
    row, col, val = [], [], []
    for i in range(m):
        for j in rng.choice(n, 3, replace=False):
            row.append(i); col.append(int(j)); val.append(float(rng.uniform(-2, 2)))
    inf = np.inf
    rL = np.array([1.0, -inf, 0.5, -1.0, -inf, 2.0])
    rU = np.array([1.0, 3.0, inf, 4.0, inf, 2.0])
    l = np.array([0.0, -inf, -1.0, 0.0, -inf])
    u = np.array([5.0, inf, 2.0, inf, 3.0])
    c = rng.normal(size=n)
    return B.RangedLP(m, n, np.array(row), np.array(col), np.array(val), c, rL, rU, l, u, 1.5)


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built here")
def test_build_pdlp_form_matches_reference():
    """Row order, signs, slack columns and dropped free rows as src/pdlp.cpp:8-82."""
    lp = _mixed_rows_lp()
    form, meta = B.build_pdlp_form(lp)
    P = O.RefProblem.from_form(as_form(lp), use_presolve=False)
    ref = P.form(P.PDLP_FORM)
    assert (form.m, form.n, form.nnz) == (ref.m, ref.n, ref.nnz)
    key = lambda f: sorted(zip(f.row.tolist(), f.col.tolist(), f.val.tolist()))  # noqa: E731
    assert key(form) == key(ref)
    for a in ("c", "rL", "rU", "l", "u"):
        np.testing.assert_array_equal(getattr(form, a), getattr(ref, a))
    assert form.obj_offset == ref.obj_offset


def test_transport_generator_shape_and_balance():
    S, D = 20, 7
    lp = B.gen_transport(S, D, 3)
    assert (lp.m, lp.n, lp.nnz) == (S + D, S * D, 2 * S * D)
    assert np.all(lp.val == 1.0)
    supply, demand = lp.rL[:S], lp.rL[S:]
    assert np.all((supply >= 100) & (supply <= 1000)) and np.all(supply == np.round(supply))
    assert supply.sum() == demand.sum()
    assert np.all(demand >= 1) and np.all(demand == np.round(demand))
    assert np.all((lp.c >= 1) & (lp.c <= 100)) and np.all(lp.c == np.round(lp.c))
    assert np.all(lp.l == 0) and np.all(np.isinf(lp.u))
    counts = np.bincount(lp.col, minlength=lp.n)
    assert np.all(counts == 2)


def test_random_generator_shape_and_determinism():
    m, n, k = 50, 150, 6
    a = B.gen_random_lp(m, n, k, 9, True)
    b = B.gen_random_lp(m, n, k, 9, True)
    for f in ("row", "col", "val", "c", "rL"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
    assert np.all(np.bincount(a.col, minlength=n) == k)
    for j in range(n):  # distinct rows per column
        rows = a.row[a.col == j]
        assert len(set(rows.tolist())) == k
    assert np.all(np.abs(a.val) <= 1.0) and np.all(a.val != 0)
    assert np.all(a.val == a.val.astype(np.float32).astype(np.float64))
    np.testing.assert_array_equal(a.rL, a.rU)
    assert np.all(a.l == 0) and np.all(a.u == 10)


def test_random_lp_is_feasible_by_construction():
    """b = A x0 for some x0 in [0,5]^n: the LP is feasible (the CPU oracle solves it)."""
    lp = B.gen_random_lp(40, 120, 4, 21, False)
    U, S, Dr, Dc, _ = B.prepare(lp)
    r = O.pdlp_run(as_form(U), as_form(S), Dr, Dc, tol=1e-7, max_iterations=200000)
    assert r["converged"]
    v = O.verify(as_form(U), r["x"], r["y"])
    assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-7


def _layout_cases():
    cases = [load_fixture(n) for n in ("afiro", "israel", "share1b")]
    # sizes that cut every parallel stage into several chunks (entries, sigma
    # windows, columns) as well as small ones that stay on one thread
    for lp in (B.gen_random_lp(30_000, 90_000, 8, 3, True), B.gen_random_lp(150_000, 300_000, 4, 5, True),
               B.gen_transport(300, 200, 2),
               B.gen_random_lp(2_000, 5_000, 6, 4, False)):
        U, S, Dr, Dc, _ = B.prepare(lp)
        cases.append((U, S, Dr, Dc))
    return cases


@pytest.mark.parametrize("whole_gpu", [True, False])
def test_layout_does_not_depend_on_host_threads(whole_gpu):
    """The device layout (CSR builds, sigma sort, tuned and split slices,
    permuted vectors, step seeds) is built on several host threads for the
    one-LP engine; every thread count must hand the device the same bytes."""
    for U, S, Dr, Dc in _layout_cases():
        d1 = B.layout_digest(U, S, Dr, Dc, threads=1, whole_gpu=whole_gpu)
        for t in (2, 3, 8):
            assert B.layout_digest(U, S, Dr, Dc, threads=t, whole_gpu=whole_gpu) == d1, (U.m, U.n, t)


def test_layout_errors_name_the_first_bad_entry_at_any_thread_count():
    U, S, Dr, Dc, _ = B.prepare(B.gen_random_lp(30_000, 90_000, 8, 3, True))
    for bad in (5, 400_000):
        V = B.RangedLP.like(U)
        V.col = V.col.copy()
        V.col[bad] = U.n + 1
        V.col[bad + 1000] = -1
        for t in (1, 8):
            with pytest.raises(B.B2Error) as e:
                B.layout_digest(V, S, Dr, Dc, threads=t)
            assert e.value.code == B.B2_ERR_INVALID
            assert f"entry {bad}" in str(e.value)
    V = B.RangedLP.like(U)
    V.val = V.val.copy()
    V.val[7] = np.nan
    with pytest.raises(B.B2Error) as e:
        B.layout_digest(V, S, Dr, Dc, threads=8)
    assert e.value.code == B.B2_ERR_NONFINITE and "entry 7" in str(e.value)


def test_dense_run_records_of_the_whole_gpu_layout():
    """b2_layout_get_stats: on the 2,000 x 500 transportation LP nearly every
    slice record of A is a dense run (source rows: 500 consecutive arcs; sink
    rows: 32 consecutive sinks a warp, one source a step), none of A^T is, and
    a random LP has none; the batch layout never marks any."""
    U, S, Dr, Dc, _ = B.prepare(B.gen_transport(2000, 500, 1))
    st = B.layout_stats(U, S, Dr, Dc)
    assert st["a_slices"] == 4109 and st["a_groups"] == 17
    assert st["a_dense"] >= 4000, st
    assert st["at_dense"] == 0
    assert B.layout_stats(U, S, Dr, Dc, whole_gpu=False)["a_dense"] == 0
    U, S, Dr, Dc, _ = B.prepare(B.gen_random_lp(2000, 4000, 8, 3, True))
    st = B.layout_stats(U, S, Dr, Dc)
    assert st["a_dense"] == 0 and st["at_dense"] == 0


def test_dense_run_needs_every_stored_column_on_the_run():
    """One dense row of 4,096 columns is one long dense run (split into
    segments, each a dense record). The layout keeps a row's entries in their
    input order, so two swapped entries take their segment off the run, and a
    shuffled row has no dense record at all."""
    n = 4096

    def one_row(cols):
        row = np.zeros(n, dtype=np.int64)
        lp = B.RangedLP(1, n, row, np.asarray(cols), np.ones(n), np.ones(n), np.array([1.0]), np.array([1.0]),
                        np.zeros(n), np.full(n, 10.0))
        U, S, Dr, Dc, _ = B.prepare(lp)
        return B.layout_stats(U, S, Dr, Dc)

    st = one_row(np.arange(n))
    assert st["a_dense"] == st["a_slices"] > 1, st
    perm = np.arange(n)
    perm[[100, 101]] = perm[[101, 100]]
    st2 = one_row(perm)
    assert st2["a_slices"] == st["a_slices"] and st2["a_dense"] == st["a_dense"] - 1, st2
    rng = np.random.default_rng(0)
    st3 = one_row(rng.permutation(n))
    assert st3["a_dense"] == 0, st3


def test_slices_stay_inside_sigma_windows():
    """Rows are sorted longest first inside each sigma window; a slice that
    ran on into the next window would take that window's longest row as its
    length. The layout widens such a slice's lanes per row instead, so a
    random LP of short rows has no split (overlong) slices at all."""
    U, S, Dr, Dc, _ = B.prepare(B.gen_random_lp(20000, 40000, 8, 1, True))
    st = B.layout_stats(U, S, Dr, Dc)
    assert st["a_groups"] == 0 and st["at_groups"] == 0, st
    assert st["a_padded"] < 1.04 * U.nnz, st
