"""The multi-process path of bench.py on CPU: two gloo ranks, each with its own
replica timing; the job's time is the max over ranks and its throughput
counts every rank's units (no data-path collective: replicas only)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    w, r, _ = bench.dist_setup(world)
    assert (w, r) == (world, rank)
    bench.dist_barrier(w)
    # rank r "took" 100 * (r + 1) ms for 3 steps
    mx = bench.dist_max(100.0 * (r + 1), w)
    out[rank] = (mx, bench.job_rate(w, 3, mx))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_and_count_all_replicas():
    world, port = 2, _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1]
    mx, rate = out[0]
    assert mx == pytest.approx(200.0)
    assert rate == pytest.approx(2 * 3 / 0.2)


def test_job_rate_single_rank():
    import bench
    assert bench.job_rate(1, 4, 2000.0) == pytest.approx(2.0)
