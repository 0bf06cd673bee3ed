"""The shape-class autotuner (b2_batch_autotune) on the B200: it returns a
lane target from {4, 8, 16, 32} for each class present in the LPs it is given
(0 for the others) with the chosen target's measured time per attempt, and a
batch built with the tuned table solves every LP to a certified 1e-6 answer.
Tables are data: the same table gives bit-identical answers twice."""
import numpy as np
import pytest

import b200pdlp as B
import oracle as O
from conftest import as_form

pytestmark = pytest.mark.gpu


def family(count, seed=11, m_hi=2000):
    probs = []
    for (m, n, k, sd) in B.batch_family_shapes(count, seed=seed, m_hi=m_hi):
        U, S, Dr, Dc, _ = B.prepare(B.gen_random_lp(m, n, k, sd, True))
        probs.append((U, S, Dr, Dc))
    return probs


def test_autotune_table_and_tuned_batch_certified():
    probs = family(48)
    t = B.autotune(probs)
    present = {B.shape_class(U.m, U.n, U.nnz) for (U, _, _, _) in probs}
    for k in range(B.TUNE_CLASSES):
        if k in present:
            assert t.lane_target[k] in (4, 8, 16, 32) and t.us_per_attempt[k] > 0
        else:
            assert t.lane_target[k] == 0
    print("TUNE " + str({k: (t.lane_target[k], round(t.us_per_attempt[k], 2)) for k in sorted(present)}))
    sols = []
    for _ in range(2):
        with B.Batch(probs, tune=t) as bt:
            res, _ = bt.solve(max_iterations=500_000, tol=1e-6)
            assert all(r["converged"] for r in res)
            sols.append([bt.solution(i) for i in range(len(probs))])
    for i, (U, S, Dr, Dc) in enumerate(probs):
        x, y = sols[0][i]
        np.testing.assert_array_equal(x, sols[1][i][0])
        v = O.verify(as_form(U), x, y)
        assert max(v["eps_P"], v["eps_D"], v["eps_G"]) <= 1e-6 * (1 + 1e-9)
