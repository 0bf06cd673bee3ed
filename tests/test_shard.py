"""Shares of a batch or a stream over several GPUs (b2_shard_plan,
b2_request_work, b2_pool_create), host side only.

The plan is checked against a plain restatement of its two rules (longest
load first to the least-loaded share; arrival order to the least-loaded share
so far), for the longest-first bound of 4/3 of the best split, and through
two gloo ranks that each compute their own share of the same batch and stream
without a collective: the shares must be disjoint, cover everything, and be
the same on both ranks."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import b200pdlp as B
from conftest import GOLDEN, ROOT

sys.path.insert(0, ROOT)


def plan_restated(work, parts, online):
    order = list(range(len(work)))
    if not online:
        order.sort(key=lambda i: (-work[i], i))
    load = [0] * parts
    out = [0] * len(work)
    for i in order:
        best = min(range(parts), key=lambda r: (load[r], r))
        load[best] += work[i]
        out[i] = best
    return out


@pytest.mark.parametrize("online", [False, True])
def test_plan_matches_its_rules(online):
    rng = np.random.default_rng(5)
    for count in (0, 1, 7, 64, 500):
        for parts in (1, 2, 3, 8):
            # many equal loads, so the tie rules are exercised
            work = rng.integers(0, 20, count).astype(np.int64) * 1000
            got = B.shard_plan(work, parts, online=online)
            assert got.tolist() == plan_restated(work.tolist(), parts, online)
            assert got.size == count and (count == 0 or (got.min() >= 0 and got.max() < parts))


def test_longest_first_is_within_four_thirds_of_the_best_split():
    rng = np.random.default_rng(1)
    for parts in (2, 4, 8):
        shapes = B.batch_family_shapes(512, seed=int(rng.integers(1 << 30)))
        work = np.array([B.request_work(m, n, n * k) for (m, n, k, _) in shapes], np.int64)
        plan = B.shard_plan(work, parts)
        loads = np.bincount(plan, weights=work, minlength=parts)
        lower = max(work.sum() / parts, work.max())
        assert loads.max() <= (4 / 3) * lower
        assert loads.sum() == work.sum()


def test_request_work_and_errors():
    assert B.request_work(3, 4, 10) == 27
    assert B.request_work(0, 0, 0) == 0
    with pytest.raises(B.B2Error) as e:
        B.shard_plan([1, 2], 0)
    assert e.value.code == B.B2_ERR_INVALID
    with pytest.raises(B.B2Error) as e:
        B.shard_plan([1, -2], 2)
    assert e.value.code == B.B2_ERR_INVALID


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_pool_without_a_device_fails_cleanly():
    with pytest.raises(B.B2Error) as e:
        B.Pool([0, 1])
    assert e.value.code == B.B2_ERR_NO_DEVICE


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import b200pdlp as B_
    w, r, _ = bench.dist_setup(world)
    shapes = bench.batch_shapes("batch", 96, 0, w)
    batch = bench.my_share(B_, [B_.request_cost(m, n, n * k) for (m, n, k, _) in shapes], w, r)
    full = bench.serve_stream(2000.0 * w, 0.05, 0)
    stream = bench.my_share(B_, [B_.request_cost(m, n, n * k) for (_, m, n, k, _) in full], w, r, online=True)
    total = bench.dist_sum(float(len(batch)), w)
    out[rank] = (batch, stream, len(shapes), len(full), total)
    import torch.distributed as dist
    dist.destroy_process_group()


def test_two_gloo_ranks_take_disjoint_covering_shares():
    world, port = 2, _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
    (b0, s0, nb, ns, t0), (b1, s1, _, _, t1) = out[0], out[1]
    assert nb == 192 and t0 == t1 == nb
    assert sorted(b0 + b1) == list(range(nb)) and b0 and b1
    assert sorted(s0 + s1) == list(range(ns)) and s0 and s1
    # the loads of the two batch shares are close (longest first)
    import bench
    shapes = bench.batch_shapes("batch", 96, 0, 2)
    work = np.array([B.request_work(m, n, n * k) for (m, n, k, _) in shapes])
    l0, l1 = work[b0].sum(), work[b1].sum()
    assert abs(l0 - l1) <= work.max()


def test_request_cost_model_and_measured_batch_shares():
    """b2_request_cost = work x round(167 m^0.657). The attempts each LP of the
    4,096-LP batch took on a B200 (tests/golden/batch_attempts.csv, made by
    make_batch_attempts.py) give each LP's measured cost, work x attempts.
    The model's attempts follow the measured ones; shares of the whole batch
    planned on either load end within 5 % of each other; shares of smaller
    batches (256 LPs over 8 GPUs, averaged over 20 draws) end closer together
    when planned on the cost."""
    for (m, n, z) in ((1, 1, 1), (100, 300, 2000), (5000, 15000, 100000)):
        assert B.request_cost(m, n, z) == B.request_work(m, n, z) * round(167.0 * m ** 0.657)
    assert B.request_cost(0, 0, 0) == 0
    rows = np.loadtxt(os.path.join(GOLDEN, "batch_attempts.csv"), delimiter=",", skiprows=1, dtype=np.int64)
    assert rows.shape == (4096, 4)
    m, n, z, att = rows.T
    assert att.min() > 0
    measured = ((2 * z + m + n) * att).astype(np.float64)
    model = 167.0 * m.astype(np.float64) ** 0.657
    assert np.corrcoef(np.log(model), np.log(att))[0, 1] > 0.85
    work = np.array([B.request_work(int(a), int(b), int(c)) for a, b, c in zip(m, n, z)], np.int64)
    cost = np.array([B.request_cost(int(a), int(b), int(c)) for a, b, c in zip(m, n, z)], np.int64)

    def spread(load, idx, parts):
        got = np.bincount(B.shard_plan(load[idx], parts), weights=measured[idx], minlength=parts)
        return got.max() / got.mean()

    everything = np.arange(4096)
    for parts in (2, 4, 8):
        assert spread(work, everything, parts) < 1.05 and spread(cost, everything, parts) < 1.05
    rng = np.random.default_rng(0)
    draws = [rng.choice(4096, 256, replace=False) for _ in range(20)]
    by_work = np.mean([spread(work, d, 8) for d in draws])
    by_cost = np.mean([spread(cost, d, 8) for d in draws])
    assert by_cost < by_work, (by_cost, by_work)
