"""The two-phase product layout of the whole-GPU engine (csrc/pb_layout.cpp),
checked on the host without a GPU: y = A x evaluated phase by phase through
the layout (b2_two_phase_spmv_host: products placed by their destination,
bins summed from their slots) must equal the oracle's CSR product
(include/sparse.hpp:52-59 restated) bit for bit -- the layout adds each row's
products in the row's CSR order, products of FP32-exact values rounded once."""
import numpy as np
import pytest

import b200pdlp as B
import oracle as O


def as_lp(lp):
    return B.RangedLP(lp.m, lp.n, lp.row, lp.col, lp.val, lp.c, lp.rL, lp.rU, lp.l, lp.u)


@pytest.mark.parametrize("m,n,k,seed,chunks,bins", [
    (20_000, 40_000, 8, 1, 296, 8192), (3_000, 9_000, 6, 2, 296, 8192), (500, 1_500, 4, 3, 7, 64),
    (5_000, 15_000, 10, 4, 148, 1024), (50, 120, 4, 5, 296, 16)])
def test_two_phase_layout_equals_csr_product(m, n, k, seed, chunks, bins):
    lp = O.gen_random_lp(m, n, k, seed, True)
    x = np.random.default_rng(seed).uniform(-1, 1, n)
    y = B.two_phase_spmv_host(as_lp(lp), x, chunks=chunks, bin_entries=bins)
    ptr, idx, dat = O.csr(lp)
    np.testing.assert_array_equal(y, O.matvec(ptr, idx, dat, x))
    # and the transposed direction, as the engine's A^T y' runs
    t = O.LPForm(n, m, lp.col, lp.row, lp.val, np.zeros(m), np.zeros(n), np.zeros(n), np.zeros(m), np.zeros(m))
    yy = np.random.default_rng(seed + 1).normal(size=m)
    z = B.two_phase_spmv_host(as_lp(t), yy, chunks=chunks, bin_entries=bins)
    tp, ti, td = O.csr(lp, transpose=True)
    np.testing.assert_array_equal(z, O.matvec(tp, ti, td, yy))


def test_empty_rows_and_columns_and_transport_rows():
    lp = O.gen_transport(40, 30, 2)  # rows of 30 and 40 entries
    x = np.random.default_rng(0).uniform(0, 1, lp.n)
    y = B.two_phase_spmv_host(as_lp(lp), x, chunks=16, bin_entries=64)
    ptr, idx, dat = O.csr(lp)
    np.testing.assert_array_equal(y, O.matvec(ptr, idx, dat, x))
    # an empty row and an empty column
    row = np.array([0, 0, 2, 2]); col = np.array([0, 2, 0, 2]); val = np.array([1.0, -2.0, 0.5, 4.0])
    e = B.RangedLP(3, 4, row, col, val, np.zeros(4), np.zeros(3), np.zeros(3), np.zeros(4), np.zeros(4))
    y = B.two_phase_spmv_host(e, np.array([1.0, 5.0, 2.0, 7.0]), chunks=3, bin_entries=2)
    np.testing.assert_array_equal(y, [1.0 - 4.0, 0.0, 0.5 + 8.0])


def test_row_longer_than_a_bin_is_refused():
    lp = O.gen_transport(40, 30, 2)
    with pytest.raises(B.B2Error) as e:
        B.two_phase_spmv_host(as_lp(lp), np.zeros(lp.n), chunks=16, bin_entries=16)
    assert e.value.code == B.B2_ERR_UNSUPPORTED
