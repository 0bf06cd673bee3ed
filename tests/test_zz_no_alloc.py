"""The allocation-free entry point, b2_solve_pdhg_gpu_noalloc.

Some callers cannot allocate GPU memory: a process whose device memory is
reserved up front by another runtime's allocator or a pool it does not own,
and latency-critical paths that must stay out of the driver's allocator. For
them the library keeps one static 32 MiB device array and runs the one-CTA
solve entirely inside it. This test calls that entry point through the C ABI
and checks that it returns what the ordinary entry point
(b2_solve_pdhg_gpu_ex, which allocates its working memory) returns for the
same LPs, on two calls in a row -- the second call runs on an array that still
holds the first call's data -- in both precision modes (mixed: an FP32 launch
handing over to an FP64 one; FP64: the FP64 launch from the start). Each
answer is also certified by the oracle's restated verify().
"""
import ctypes as C

import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import load_fixture

pytestmark = pytest.mark.gpu


def _solve(fn_name, U, S, Dr, Dc, precision):
    lib = B.lib()
    U = B.RangedLP.like(U)
    S = B.RangedLP.like(S)
    Dr = np.ascontiguousarray(Dr, np.float64)
    Dc = np.ascontiguousarray(Dc, np.float64)
    o = B.default_opts(max_iterations=500000, check_every=64, tol=1e-6, precision=precision)
    x = np.zeros(max(U.n, 1))
    y = np.zeros(max(U.m, 1))
    r = B._Result()
    uv, sv = U.view(), S.view()
    if fn_name == "noalloc":
        rc = lib.b2_solve_pdhg_gpu_noalloc(C.byref(uv), C.byref(sv), Dr.ctypes.data, Dc.ctypes.data, C.byref(o),
                                           x.ctypes.data, y.ctypes.data, C.byref(r))
    else:
        rc = lib.b2_solve_pdhg_gpu_ex(C.byref(uv), C.byref(sv), Dr.ctypes.data, Dc.ctypes.data, C.byref(o), None,
                                      x.ctypes.data, y.ctypes.data, C.byref(r))
    assert rc == B.B2_OK, lib.b2_last_error().decode()
    return x[:U.n], y[:U.m], r


@pytest.mark.parametrize("precision", [B.PREC_MIXED, B.PREC_FP64])
def test_noalloc_matches_allocating_entry_point_on_two_calls(precision):
    for name in ("share1b", "israel"):          # two calls in a row, different LPs
        U, S, Dr, Dc = load_fixture(name)
        x1, y1, r1 = _solve("noalloc", U, S, Dr, Dc, precision)
        x0, y0, r0 = _solve("ex", U, S, Dr, Dc, precision)
        assert r1.converged == r0.converged == 1
        assert r1.iterations == r0.iterations
        assert r1.eps_P == pytest.approx(r0.eps_P, rel=1e-9, abs=1e-15)
        # same tolerance as the other GPU parity tests use for points
        np.testing.assert_allclose(x1, x0, rtol=1e-9, atol=1e-9 * (1 + np.abs(x0).max()))
        np.testing.assert_allclose(y1, y0, rtol=1e-9, atol=1e-9 * (1 + np.abs(y0).max()))
        assert r1.objective == pytest.approx(r0.objective, rel=1e-12)
        v = O.verify(U, x1, y1)
        assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6 * (1 + 1e-9), (name, v)
