"""Device SpMV (sliced-ELL, the kernel inside every PDLP pass) against the
oracle's serial CSR matvec (include/sparse.hpp:52-59) on the same inputs."""
import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import as_form, fixture_names, load_fixture

pytestmark = pytest.mark.gpu


def _check_engine(U, S, Dr, Dc, seed=0, **opts):
    Uf = as_form(U)
    a = O.csr(Uf, False)
    at = O.csr(Uf, True)
    rng = np.random.default_rng(seed)
    with B.Engine(B.RangedLP.like(U), B.RangedLP.like(S), Dr, Dc, **opts) as e:
        for _ in range(2):
            x = rng.normal(size=U.n)
            y = rng.normal(size=U.m)
            ax = e.spmv(0, x)
            aty = e.spmv(1, y)
            ref_ax = O.matvec(*a, x)
            ref_aty = O.matvec(*at, y)
            # FP64 accumulation in a different order: |err| <= n_row * eps * sum|a_ij x_j|
            bound_ax = 1e-13 * (O.matvec(a[0], a[1], np.abs(a[2]), np.abs(x)) + 1e-300)
            bound_aty = 1e-13 * (O.matvec(at[0], at[1], np.abs(at[2]), np.abs(y)) + 1e-300)
            assert np.all(np.abs(ax - ref_ax) <= bound_ax)
            assert np.all(np.abs(aty - ref_aty) <= bound_aty)


@pytest.mark.parametrize("name", fixture_names())
def test_spmv_fixtures(name):
    _check_engine(*load_fixture(name))


@pytest.mark.parametrize("shape", [(600, 1800, 6, True), (1000, 3000, 6, False), (97, 301, 3, True)])
def test_spmv_random_family(shape):
    m, n, k, f32 = shape
    lp = B.gen_random_lp(m, n, k, 5, f32)
    U, S, Dr, Dc, _ = B.prepare(lp)
    _check_engine(U, S, Dr, Dc)


@pytest.mark.parametrize("lane_target", [2, 4, 16, 64])
def test_spmv_transport_long_rows(lane_target):
    """Skewed rows (transport: rows of D and S entries, columns of 2): every
    lanes-per-row choice of the sliced format gives the same product."""
    lp = B.gen_transport(40, 300, 1)
    U, S, Dr, Dc, _ = B.prepare(lp)
    _check_engine(U, S, Dr, Dc, lane_target=lane_target)


def test_spmv_empty_rows_and_columns():
    # an LP whose A has an empty row and an empty column
    m, n = 5, 6
    row = np.array([0, 0, 1, 3, 3, 4], np.int32)
    col = np.array([0, 2, 2, 3, 0, 4], np.int32)
    val = np.array([1.0, -2.0, 0.5, 3.0, 1.25, -1.0])
    c = np.ones(n); rL = np.array([1.0, 0.5, 0.0, 2.0, -1.0]); rU = rL.copy()
    lp = B.RangedLP(m, n, row, col, val, c, rL, rU, np.zeros(n), np.full(n, 10.0))
    s, Dr, Dc = B.scale(lp)
    _check_engine(lp, s, Dr, Dc)


@pytest.mark.parametrize("shape", [(300, 700), (700, 300)])
def test_spmv_transport_tuned_and_split_slices(shape):
    """Long rows on the whole-GPU layout: lanes-per-row chosen by the sector
    cost model, slices longer than 32 steps split over several warps whose
    partial sums one warp adds in segment order."""
    lp = B.gen_transport(shape[0], shape[1], 3)
    U, S, Dr, Dc, _ = B.prepare(lp)
    _check_engine(U, S, Dr, Dc, seed=2)
