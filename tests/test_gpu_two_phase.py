"""The whole-GPU engine's two-phase products (A x' and A^T y' as coalesced
product streams plus per-bin sums in shared memory, csrc/pb_layout.cpp and
device.cuh pb_produce / pb_consume) against its sliced-ELL gathers, on the
same engine: both answers are certified by the oracle's verify, agree in the
objective within 1e-6 relative, and the two-phase solve repeats bit for bit.
The two add a row's entries in different orders, so their iterates differ in
the last bits; after 64 FP64 attempts they agree to 1e-9 of their scale."""
import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import OBJ_TOL, as_form, rel

pytestmark = pytest.mark.gpu


def certified(U, r, tol=1e-6):
    v = O.verify(as_form(U), r.x, r.y)
    assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= tol * (1 + 1e-9), v
    assert r.eps_P == pytest.approx(v["eps_P"], rel=1e-6, abs=1e-12)
    return v


@pytest.mark.parametrize("precision", [B.PREC_MIXED, B.PREC_FP64])
def test_two_phase_solve_certified_deterministic_and_equal_to_gathers(precision):
    U, S, Dr, Dc, _ = B.prepare(B.gen_random_lp(50_000, 150_000, 6, 3, True))
    with B.Engine(U, S, Dr, Dc, product=B.PRODUCT_TWO_PHASE) as eng:
        assert eng.info()["two_phase"] == 1
        kw = dict(max_iterations=500_000, tol=1e-6, precision=precision)
        a = eng.solve(product=B.PRODUCT_TWO_PHASE, **kw)
        b = eng.solve(product=B.PRODUCT_TWO_PHASE, **kw)
        s = eng.solve(product=B.PRODUCT_SLICED, **kw)
    assert a.converged and s.converged
    assert a.iterations == b.iterations
    np.testing.assert_array_equal(a.x, b.x)
    np.testing.assert_array_equal(a.y, b.y)
    va, vs = certified(U, a), certified(U, s)
    assert rel(va["objective"], vs["objective"]) <= OBJ_TOL
    print(f"TWO_PHASE prec={precision} attempts {a.iterations} ({a.stats['device_ms']:.1f} ms) vs gathers "
          f"{s.iterations} ({s.stats['device_ms']:.1f} ms)")


def test_two_phase_short_trajectory_matches_gathers():
    U, S, Dr, Dc, _ = B.prepare(B.gen_random_lp(20_000, 60_000, 6, 7, True))
    with B.Engine(U, S, Dr, Dc, product=B.PRODUCT_TWO_PHASE) as eng:
        assert eng.info()["two_phase"] == 1
        a = eng.solve(max_iterations=64, tol=1e-12, precision=B.PREC_FP64, product=B.PRODUCT_TWO_PHASE,
                      return_current=1)
        s = eng.solve(max_iterations=64, tol=1e-12, precision=B.PREC_FP64, product=B.PRODUCT_SLICED,
                      return_current=1)
    assert a.iterations == s.iterations == 64
    assert a.stats["accepted"] == s.stats["accepted"] and a.restarts == s.restarts
    assert np.abs(a.x - s.x).max() <= 1e-9 * (1 + np.abs(s.x).max())
    assert np.abs(a.y - s.y).max() <= 1e-9 * (1 + np.abs(s.y).max())


def test_large_lp_takes_two_phase_by_default():
    """The automatic choice: the 500,000 x 1,000,000 random LP (8 nonzeros a
    column, 16 a row) runs the two-phase products; the transportation LP, whose
    rows hold 500 and 2,000 entries, keeps the gathers."""
    U, S, Dr, Dc, _ = B.prepare(B.gen_random_lp(500_000, 1_000_000, 8, 1, True))
    with B.Engine(U, S, Dr, Dc) as eng:
        assert eng.info()["two_phase"] == 1
    U, S, Dr, Dc, _ = B.prepare(B.gen_transport(2000, 500, 1))
    with B.Engine(U, S, Dr, Dc) as eng:
        assert eng.info()["two_phase"] == 0
