"""The whole-grid kernel's staged y' (one bulk copy into every CTA's shared
memory after the rows barrier, for LPs with few rows), with several engines
alive in one process: their staging sizes differ, and the kernel's dynamic
shared-memory limit is process-wide, so creating an engine with a smaller y'
must not stop an older one with a larger y' from launching. Each answer is
certified by the oracle's verify and a repeat solve gives the same bits."""
import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import as_form

pytestmark = pytest.mark.gpu


def test_engines_with_different_staged_rows_solve_in_any_order():
    lps = [B.gen_random_lp(8000, 16000, 8, 3, True), B.gen_transport(200, 50, 2)]
    forms = [B.prepare(lp) for lp in lps]
    engines = [B.Engine(U, S, Dr, Dc) for (U, S, Dr, Dc, _) in forms]
    try:
        for e in engines:
            assert e.info()["ctas"] > 1  # the whole-grid kernel, where y' is staged
        for order in ((0, 1), (1, 0)):
            for i in order:
                U = forms[i][0]
                r1 = engines[i].solve(max_iterations=200_000, tol=1e-6)
                r2 = engines[i].solve(max_iterations=200_000, tol=1e-6)
                assert r1.converged and r2.converged, (i, r1.stats)
                np.testing.assert_array_equal(r1.x, r2.x)
                v = O.verify(as_form(U), r1.x, r1.y)
                assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6 * (1 + 1e-9), (i, v)
    finally:
        for e in engines:
            e.close()
