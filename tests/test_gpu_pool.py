"""A pool of servers in one process (b2_pool_*): each submit goes to the
member with the least unfinished work, and every answer is bit-identical to
a single server's (each LP is solved as alone, whichever member takes it).
The box has one GPU, so the pool's two members share device 0; their
kernels never wait on each other (one-CTA groups and hardware clusters)."""
import numpy as np
import pytest

import b200pdlp as B
from conftest import fixture_names, golden_index, load_fixture, random_case

pytestmark = pytest.mark.gpu

G = golden_index()


def _lps():
    lps = [load_fixture(n)[0] for n in fixture_names()]
    for k in sorted(G["random"].keys()):
        lps.append(random_case(k)[1])
    return lps


def test_pool_routes_to_the_least_backlog_and_answers_match_one_server():
    lps = _lps()
    with B.Server(round_ms=0.5, max_iterations=500000, tol=1e-6) as srv:
        ref = [srv.wait(t, timeout_s=300.0) for t in [srv.submit(U) for U in lps]]
    with B.Pool([0, 0], round_ms=0.5, max_iterations=500000, tol=1e-6) as pool:
        ts = [pool.submit(U) for U in lps]
        out = [pool.wait(t, timeout_s=300.0) for t in ts]
        st = [pool.stats(k) for k in range(2)]
    # empty pool: the first LP goes to member 0, the next to the idle member 1
    assert out[0][1]["member"] == 0 and out[1][1]["member"] == 1
    assert {info["member"] for _, info in out} == {0, 1}
    assert sum(s["completed"] for s in st) == len(lps) and all(s["failed"] == 0 for s in st)
    assert all(s["backlog_work"] == 0 and s["bytes_in_use"] == 0 for s in st)
    for (a, _), (b, _) in zip(ref, out):
        assert a.converged and b.converged
        assert a.iterations == b.iterations
        np.testing.assert_array_equal(a.x, b.x)
        np.testing.assert_array_equal(a.y, b.y)


def test_backlog_counts_unfinished_work_and_pool_closes_in_flight():
    lps = [B.prepare(B.gen_random_lp(20_000, 60_000, 6, s, True))[0] for s in (4, 5, 6)]
    work = [B.request_work(U.m, U.n, U.nnz) for U in lps]
    pool = B.Pool([0, 0], round_ms=2.0, max_iterations=2_000_000, tol=1e-9)
    ts = [pool.submit(U) for U in lps]
    # two members: LPs 0 and 2 on member 0 (equal backlogs go to the lower member), LP 1 on member 1
    st = [pool.stats(k) for k in range(2)]
    assert st[0]["backlog_work"] == work[0] + work[2]
    assert st[1]["backlog_work"] == work[1]
    assert pool.wait(ts[0], timeout_s=0.05) is None
    pool.close()
    with pytest.raises(B.B2Error) as e:
        B.Pool([0, 99])
    assert e.value.code == B.B2_ERR_INVALID
