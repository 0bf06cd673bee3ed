"""Scaling on the GPU (b2_scale_gpu) against the host restatement (b2_scale)
and the reference's own scale() (src/scaling.cpp:25-84): bit for bit."""
import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import as_form, fixture_names, load_fixture

pytestmark = pytest.mark.gpu


def _same(lp):
    s_h, dr_h, dc_h = B.scale(lp)
    s_g, dr_g, dc_g = B.scale(lp, on_gpu=True)
    np.testing.assert_array_equal(dr_g, dr_h)
    np.testing.assert_array_equal(dc_g, dc_h)
    for f in ("val", "c", "rL", "rU", "l", "u"):
        np.testing.assert_array_equal(getattr(s_g, f), getattr(s_h, f))
    return s_g, dr_g, dc_g


@pytest.mark.parametrize("name", fixture_names())
def test_gpu_scaling_equals_host_and_reference_on_fixtures(name):
    U, _, _, _ = load_fixture(name)
    s, dr, dc = _same(B.RangedLP.like(U))
    if O.reference_available():
        ref, rdr, rdc = O.ref_scale(as_form(U))
        np.testing.assert_array_equal(dr, rdr)
        np.testing.assert_array_equal(dc, rdc)
        np.testing.assert_array_equal(s.val, ref.val)


@pytest.mark.parametrize("kind", ["random", "transport", "wide"])
def test_gpu_scaling_equals_host_on_generated(kind):
    if kind == "random":
        lp = B.gen_random_lp(20_000, 60_000, 6, 4, True)
    elif kind == "transport":
        lp = B.gen_transport(300, 200, 2)
    else:  # a few very long rows and many short ones: order-dependent sums matter
        rng = np.random.default_rng(9)
        m, n = 40, 50_000
        row = rng.integers(0, m, 400_000).astype(np.int32)
        col = rng.integers(0, n, 400_000).astype(np.int32)
        val = rng.normal(size=400_000) * 10.0 ** rng.integers(-3, 4, 400_000)
        lp = B.RangedLP(m, n, row, col, val, rng.normal(size=n), np.zeros(m), np.zeros(m), np.zeros(n),
                        np.full(n, 5.0))
    _same(lp)
