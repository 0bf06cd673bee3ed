"""Benchmark of the B200 PDLP engine on the single large LP of the benchmark
family: equality-form random LP, m = 500,000 rows, n = 1,000,000 columns,
8 nonzeros per column (8M nnz), values stored in FP32, solved to 1e-6 relative
KKT (every answer checked by the engine's device-side restatement of the
reference verifier). One step = one full solve from a cold start.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0). Under torchrun with N > 1 every rank solves its
own replica of the LP (one LP is not partitioned: that would need an exchange
of x' and y' every attempt) and `value` is the total solves/s of the job, timed
as the max over ranks. The batch and the served stream (--workload batch|serve)
are sharded instead: every rank takes its share from the same deterministic
plan (b2_shard_plan), with no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "team-suprema_b200"))

METRIC = "LP solves/s & p50/p99 latency at 1e-6 rel KKT vs plain PDLP; SpMV HBM GB/s"
UNIT = "solves/s"

WORKLOADS = {
    # name: (kind, params)
    "large": ("random", dict(m=500_000, n=1_000_000, k=8, seed=1, fp32=True)),
    "transport": ("transport", dict(S=2000, D=500, seed=1)),
    "small": ("random", dict(m=600, n=1800, k=6, seed=0, fp32=False)),
    "medium": ("random", dict(m=50_000, n=150_000, k=6, seed=3, fp32=True)),
    "batch": ("batch", dict(count=4096, seed=0)),
    # Poisson arrivals at 2,000 LPs/s: 80% m~U[100,2000], 19% m~U[2000,50000],
    # 1% m=500,000; n=3m, 6 nnz/col, per-request seeds (a window of `seconds`)
    "serve": ("serve", dict(rate=2000.0, seconds=0.1, seed=0)),
}


# DRAM bytes (read + write) per attempt of the persistent solve kernel, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of 256-attempt solves of the workload with FP32
# and with FP64 iterates (`bench.py --mode solve --max-attempts 256`). A profiler cannot run
# inside the timed region, so the roofline's `traffic` is this capture scaled by the attempts
# of each timed launch, and the line labels it so.
TRAFFIC_PER_ATTEMPT = {"large": (137.0e6, 184.3e6)}


def describe(name, count=0, seconds=0.0, world=1):
    kind, p = WORKLOADS[name]
    if kind == "serve":
        return (f"served stream: Poisson arrivals at {p['rate'] * world:.0f} LPs/s for {seconds or p['seconds']} s; "
                f"sizes 80% m~U[100,2000], 19% m~U[2000,50000], 1% m=500000; n=3m, 6 nnz/col, FP32 values, "
                f"seed {p['seed']}")
    if kind == "batch":
        return (f"batch of {(count or p['count']) * world} random equality LPs, m log-uniform [50,5000], "
                f"n=round(U[2,4] m), U{{4..10}} nnz/col, FP32 values, seed {p['seed']}")
    if kind == "random":
        return (f"random equality LP m={p['m']} n={p['n']} {p['k']} nnz/col values "
                f"{'FP32' if p['fp32'] else 'FP64'} U[-1,1], 0<=x<=10, seed {p['seed']}")
    return f"transportation LP {p['S']}x{p['D']} (n={p['S'] * p['D']}, m={p['S'] + p['D']}), seed {p['seed']}"


def make_lp(B, name):
    kind, p = WORKLOADS[name]
    if kind == "random":
        return B.gen_random_lp(p["m"], p["n"], p["k"], p["seed"], p["fp32"])
    return B.gen_transport(p["S"], p["D"], p["seed"])


def algorithmic_bytes(m, n, z, p):
    """Per accepted PDHG iteration with p-byte iterates: B_spmv(A) + B_spmv(A^T)
    + primal pass (read x, A^T y, c, l, u, xsum; write x', xsum) + dual pass
    (read y, Ax', Ax, b, ysum; write y', ysum); B_spmv = 8Z + 4(R+1) + p C + p R."""
    spmv_a = 8 * z + 4 * (m + 1) + p * n + p * m
    spmv_at = 8 * z + 4 * (n + 1) + p * m + p * n
    return spmv_a + spmv_at + 8 * p * n + 7 * p * m


def spmv_bytes(rows, cols, z, p=4):
    return 8 * z + 4 * (rows + 1) + p * cols + p * rows


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return world, rank, local


def dist_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_sum(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def my_share(B, work, world, rank, online=False):
    """Indices of this rank's share of a batch (online=False) or a stream in
    arrival order (online=True): every rank computes the same plan from the
    same loads (b2_shard_plan), so no collective is needed to decide it."""
    if world == 1:
        return list(range(len(work)))
    plan = B.shard_plan(work, world, online=online)
    return [i for i in range(len(work)) if plan[i] == rank]


def job_rate(world: int, units_per_rank: float, max_ms: float) -> float:
    """Whole-job throughput of `world` replicas that each processed
    units_per_rank units, timed as the max over ranks (ms)."""
    return world * units_per_rank / (max_ms / 1e3)


def dist_barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


_ref_worker_problem = None


def ref_lp(name):
    """The workload's LP built by the oracle's restated generators (the same
    bits as the product's; pinned by tests/test_oracle.py), so the reference
    arm never loads the product library."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    kind, p = WORKLOADS[name]
    if kind == "random":
        return O.gen_random_lp(p["m"], p["n"], p["k"], p["seed"], p["fp32"])
    return O.gen_transport(p["S"], p["D"], p["seed"])


def ref_attempts_per_solve(name):
    """(attempts, source) one solve of the workload's LP takes at 1e-6 by the
    reference algorithm, from runs of the reference itself recorded in
    tests/golden/ (make_golden*.py): its FP64 GPU engine's full solve of the
    large LP, its CPU engine's full solves of the transportation and small
    LPs. (None, None) when no reference record exists."""
    try:
        big = json.load(open(os.path.join(ROOT, "tests", "golden", "large.json")))
        small = json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))["random"]
    except (OSError, ValueError, KeyError):
        return None, None
    if name == "large" and "gpu_fp64_1e-06" in big.get("large", {}):
        return int(big["large"]["gpu_fp64_1e-06"]["attempts"]), "reference FP64 GPU engine, full solve"
    if name == "transport" and "cpu_pdlp_1e-06" in big.get("transport", {}):
        return int(big["transport"]["cpu_pdlp_1e-06"]["attempts"]), "reference CPU PDLP, full solve"
    if name == "small" and "rand_m600_n1800_k6_s0_f64" in small:
        return int(small["rand_m600_n1800_k6_s0_f64"]["pdlp"]["1e-06"]["iterations"]), "reference CPU PDLP, full solve"
    return None, None


def _ref_worker_init(workload):
    """Pool-worker set-up: the workload's raw LP (regenerated from its seed:
    the same bits in every process) through the reference's own
    build_pdlp_form -> scale (src/pdlp.cpp:8-82, src/scaling.cpp:25-84), without
    presolve, i.e. the PDLP form the B200 engine receives."""
    global _ref_worker_problem
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    _ref_worker_problem = O.RefProblem.from_form(ref_lp(workload), use_presolve=False)


def _ref_worker_attempts(iters):
    r = _ref_worker_problem.solve_pdhg(max_iterations=iters, check_every=64, tol=1e-6)
    return r["seconds"], r["iterations"], r["converged"]


def reference_arm(args, world, rank):
    """The reference's own CPU PDLP (solve_pdhg, src/pdlp.cpp:146, built from
    its sources into oracle/_ref) on every host core: the engine is
    single-threaded, so each core runs its own solve of the LP, all at once
    (they share the memory bandwidth).

    Where one solve fits a step (the small LP), every step is full solves on
    every core and solves/s is measured. Otherwise each step is a bounded
    sample of cpu_sample_iters attempts per core; solves/s is then
    extrapolated from the cores' summed attempts/s with the attempts per solve
    the reference itself took (ref_attempts_per_solve), and the line says so
    (extrapolated, sampled_attempts, attempts_per_solve_source). ms_per_step is
    always the measured wall time of a step."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.reference_available():
        return {"impl": "reference", "unavailable": "reference CPU engine not built (oracle/_ref/libsovref.so)"}
    import concurrent.futures as cf
    import multiprocessing as mp
    lp = ref_lp(args.workload)
    attempts, source = ref_attempts_per_solve(args.workload)
    full = args.workload == "small"
    if attempts is None and not full:
        return {"impl": "reference", "unavailable": f"no reference attempt count recorded for {args.workload}"}
    # one process per core, as many as half the host memory holds: a worker
    # keeps the reference's forms of the LP (1.8 GB peak for the 8M-nonzero
    # LP; 250 bytes per nonzero leaves headroom)
    mem = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES")
    per_worker = max(1 << 28, 250 * lp.nnz)
    cores = max(1, min(os.cpu_count() or 1, int(0.5 * mem // per_worker)))
    iters = 2_000_000 if full else args.cpu_sample_iters
    per_step, step_ms, solved = [], [], 0
    with cf.ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn"),
                                initializer=_ref_worker_init, initargs=(args.workload,)) as ex:
        # every worker holds its problem before the first step (each answers with its pid)
        seen = set()
        for _ in range(20):
            seen |= set(ex.map(_ref_warm, range(cores)))
            if len(seen) >= cores:
                break
        for s in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            res = [f.result() for f in [ex.submit(_ref_worker_attempts, iters) for _ in range(cores)]]
            wall = time.perf_counter() - t0
            if full:
                per_step.append(sum(1 for _, _, ok in res if ok) / wall)
                if s >= args.warmup:
                    solved += sum(1 for _, _, ok in res if ok)
            else:
                per_step.append(sum(it / sec for sec, it, _ in res if sec > 0))
            step_ms.append(wall * 1e3)
    timed = per_step[args.warmup:] or per_step[-1:]
    timed_ms = step_ms[args.warmup:] or step_ms[-1:]
    if full:
        value = float(np.mean(timed))
        sample = (f"full solves of solve_pdhg to 1e-6, one per core on {cores} cores per step, "
                  f"{solved} solved in the timed steps; solves/s measured")
    else:
        value = float(np.mean(timed)) / attempts
        sample = (f"{iters} attempts of solve_pdhg per core per step, {cores} single-threaded solves of this LP at "
                  f"once; solves/s = summed attempts/s / {attempts} attempts per solve ({source})")
    cb = {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample}
    cfg = workload_config(args, lp, None)
    cfg["parallelism"] = f"{cores} host cores, one solve per core"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean(timed_ms)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference", "config": cfg,
            "cpu_baseline": cb, "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0},
            "extrapolated": not full}
    if not full:
        line.update(sampled_attempts=iters, attempts_per_solve=attempts, attempts_per_solve_source=source,
                    attempts_per_s_per_core=float(np.mean(timed)) / cores)
    return line


_ref_problem_cache = {}


def _form_arrays(U):
    return (U.m, U.n, U.row, U.col, U.val, U.c, U.rL, U.rU, U.l, U.u, U.obj_offset)


def _ref_warm(_i=0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.reference()
    time.sleep(0.3)  # held long enough that every worker process takes one
    return os.getpid()


def _ref_solve(arrs):
    """One full solve by the reference CPU PDLP (solve_pdhg, src/pdlp.cpp:146)
    in a pool worker: (seconds of the solve by the reference's clock, attempts,
    converged)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    m, n, row, col, val, c, rL, rU, l, u, off = arrs
    P = O.RefProblem.from_form(O.LPForm(m, n, row, col, val, c, rL, rU, l, u, off), use_presolve=False)
    r = P.solve_pdhg(max_iterations=2_000_000, check_every=64, tol=1e-6)
    return r["seconds"], r["iterations"], r["converged"]


def cpu_all_cores(lps, budget_s):
    """The reference CPU PDLP on every host core: independent single-threaded
    solves, one spawned process per core, of the LPs in `lps` (unscaled PDLP
    forms, in order) until budget_s of wall time has passed (solves already
    started finish). Returns (solves/s, dict): the rate is cores x solved
    LPs / the sum of their solve seconds, i.e. the cores kept busy all the
    time, an upper bound on what the CPU sustains on this mix."""
    import concurrent.futures as cf
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    with cf.ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_ref_warm, range(cores)))  # every worker up and the library loaded before the clock
        t0 = time.perf_counter()
        pending, it = set(), iter(lps)
        out = []
        while True:
            while len(pending) < cores and time.perf_counter() - t0 < budget_s:
                U = next(it, None)
                if U is None:
                    break
                pending.add(ex.submit(_ref_solve, _form_arrays(U)))
            if not pending:
                break
            fin, pending = cf.wait(pending, return_when=cf.FIRST_COMPLETED)
            out.extend(f.result() for f in fin)
        wall = time.perf_counter() - t0
    solved = [o for o in out if o[2]]
    busy = sum(o[0] for o in out)
    rate = cores * len(solved) / busy if busy > 0 else 0.0
    return rate, {"cores": cores, "lps": len(out), "converged": len(solved), "busy_s": busy, "wall_s": wall}


def cpu_sample(O, U, iters):
    key = id(U)
    if key not in _ref_problem_cache:
        _ref_problem_cache[key] = O.RefProblem.from_form(O.LPForm(U.m, U.n, U.row, U.col, U.val, U.c, U.rL, U.rU,
                                                                  U.l, U.u, U.obj_offset), use_presolve=False)
    P = _ref_problem_cache[key]
    r = P.solve_pdhg(max_iterations=iters, check_every=64, tol=1e-6)
    return {"seconds": r["seconds"], "iterations": r["iterations"]}


def workload_config(args, U, lp):
    return {"workload": describe(args.workload), "m": U.m, "n": U.n, "nnz": U.nnz, "tol": args.tol,
            "check_every": 64, "precision": args.precision,
            "l2": "inputs larger than L2 (working set > 126 MB)" if U.nnz * 16 > 126e6 else
                  "inputs smaller than L2; no flush (every solve re-reads them)",
            "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single GPU"}


def family_shapes(count: int, seed: int, m_lo: int = 50, m_hi: int = 5000):
    """The uneven batch family: m log-uniform on [m_lo, m_hi], n = round(U[2,4] m),
    nonzeros per column uniform on {4..10}, one derived seed per LP; a list of
    (m, n, k, seed). The same draw as the library's batch_family_shapes (a test
    pins the two), restated here so the reference arm does not load the library."""
    rng = np.random.default_rng(seed)
    m = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), count)).round().astype(int)
    n = np.round(rng.uniform(2.0, 4.0, count) * m).astype(int)
    k = rng.integers(4, 11, count)
    seeds = rng.integers(0, 2**62, count)
    return [(int(a), int(b), int(c), int(d)) for a, b, c, d in zip(m, n, k, seeds)]


def batch_shapes(name, count=0, m_hi=0, world=1):
    """The batch of `count` LPs per GPU: world x count shapes drawn from one
    master seed (the single-GPU batch is the first draw of the same family)."""
    _, p = WORKLOADS[name]
    return family_shapes((count or p["count"]) * world, p["seed"], m_hi=m_hi or 5000)


def make_batch(B, name, count=0, m_hi=0, world=1, rank=0):
    """This rank's share of the batch (all of it on one GPU), balanced by load."""
    shapes = batch_shapes(name, count, m_hi, world)
    mine = my_share(B, [B.request_cost(m, n, n * k) for (m, n, k, _) in shapes], world, rank)
    probs = []
    for i in mine:
        m, n, k, seed = shapes[i]
        lp = B.gen_random_lp(m, n, k, seed, True)
        U, S, Dr, Dc, _ = B.prepare(lp)
        probs.append((U, S, Dr, Dc))
    return probs, len(shapes)


def batch_bench(args, world, rank, local):
    """One step = one persistent launch solving the whole batch to 1e-6."""
    import torch
    import b200pdlp as B
    torch.cuda.set_device(local)
    prec = B.PREC_MIXED if args.precision == "mixed" else B.PREC_FP64
    t0 = time.time()
    probs, n_total = make_batch(B, args.workload, args.batch_count, args.batch_mhi, world, rank)
    t_prep = time.time() - t0
    t0 = time.time()
    bt = B.Batch(probs)
    t_create = time.time() - t0
    info = bt.info()
    bopts = dict(precision=prec, batch_block=args.batch_block, batch_cluster_nnz=args.batch_cluster_nnz,
                 batch_tail_attempts=args.batch_tail_attempts)
    for _ in range(args.warmup):
        bt.solve(max_iterations=2_000_000, tol=args.tol, **bopts)
    dist_barrier(world)
    steps = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            res, ms = bt.solve(max_iterations=2_000_000, tol=args.tol, **bopts)
            steps.append((res, ms))
    dist_barrier(world)
    ms_total = dist_max(sum(ms for _, ms in steps), world)
    n_lp = len(probs)
    # every rank solves its own share: the job's throughput is all LPs over the slowest rank
    value = n_total * args.steps / (ms_total / 1e3)
    res = steps[-1][0]
    lat = sorted(r["device_ms"] for r in res)
    lp_cta_ms = float(sum(r["device_ms"] * max(1, r["group_ctas"]) for r in res))
    launch_ctas = bt.info()["last_launch_ctas"]
    conv = int(dist_sum(sum(r["converged"] for r in res), world))
    attempts = np.array([r["iterations"] for r in res])
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the batch's LPs are drawn independently, so its first ones are a sample of the mix
        rate, st = cpu_all_cores([pr[0] for pr in probs], args.cpu_budget_s)
        cpu = {"value": rate, "unit": UNIT, "cores": st["cores"], "kind": "reference",
               "sample": f"the reference solve_pdhg to 1e-6 on the batch's first {st['lps']} LPs, one process per "
                         f"core ({st['converged']} converged; {st['busy_s']:.1f} s of solves in {st['wall_s']:.1f} s); "
                         "solves/s = cores x LPs / solve seconds"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if prec == B.PREC_MIXED else "f64",
            "data": "synthetic",
            "config": {"workload": describe(args.workload, count=args.batch_count, world=world), "lps": n_total,
                       "lps_rank0": n_lp,
                       "m_hi": args.batch_mhi or 5000, "sum_m_rank0": info["sum_m"],
                       "sum_n_rank0": info["sum_n"], "sum_nnz_rank0": info["sum_nnz"], "tol": args.tol,
                       "batch_block": bt.info()["threads_per_cta"], "batch_cluster_nnz": args.batch_cluster_nnz,
                       "parallelism": f"sharded x{world} (load-balanced shares, no collective)" if world > 1
                       else "single GPU"},
            "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[int(0.99 * (len(lat) - 1))], "max": lat[-1],
                           "note": "per-LP time on its CTA inside the launch (rank 0's share)"},
            "occupancy": {"lp_cta_ms": lp_cta_ms, "ctas": launch_ctas,
                          "busy_fraction": lp_cta_ms / (steps[-1][1] * max(1, launch_ctas)),
                          "note": "sum over LPs of (time on its CTAs x CTAs in its group) over (launch time x "
                                  "CTAs the launch used), last step"},
            "converged": conv, "attempts": {"median": float(np.median(attempts)), "max": int(attempts.max()),
                                            "total": int(attempts.sum())},
            "clocks": clk.summary(), "gpu_launches": args.steps, "prep_s": t_prep, "create_s": t_create,
            "device_bytes": info["device_bytes"], "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    bt.close()


def serve_stream(rate, seconds, seed):
    """Arrival times and (m, n, k, seed) of the request stream."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            return out
        u = rng.random()
        if u < 0.80:
            m = int(rng.integers(100, 2001))
        elif u < 0.99:
            m = int(rng.integers(2000, 50001))
        else:
            m = 500_000
        out.append((t, m, 3 * m, 6, int(rng.integers(1, 2**62))))


def serve_bench(args, world, rank, local):
    """One step = the whole request stream: submitted at its arrival times to
    the server (b2_server_*), every result waited for; value = completed / makespan."""
    import torch
    import b200pdlp as B
    torch.cuda.set_device(local)
    prec = B.PREC_MIXED if args.precision == "mixed" else B.PREC_FP64
    _, p = WORKLOADS[args.workload]
    # the offered rate grows with the GPUs (weak scaling); each rank serves its
    # share of the one stream, routed in arrival order to the least-loaded rank
    full = serve_stream(p["rate"] * world, args.serve_seconds or p["seconds"], p["seed"])
    mine = my_share(B, [B.request_cost(m, n, n * k) for (_, m, n, k, _) in full], world, rank, online=True)
    stream = [full[i] for i in mine]
    t0 = time.time()
    lps = [B.gen_random_lp(m, n, k, sd, True) for (_, m, n, k, sd) in stream]
    t_gen = time.time() - t0
    warm = [B.gen_random_lp(m, 3 * m, 6, 1000 + i, True) for i, m in enumerate((300, 900, 1500))]
    with B.Server(round_ms=args.round_ms, precision=prec, max_iterations=2_000_000, tol=args.tol) as srv:
        for _ in range(args.warmup):
            for t in [srv.submit(w) for w in warm]:
                srv.wait(t)
        st0 = srv.stats()
        dist_barrier(world)
        tickets = []
        with ClockSampler(local) as clk:
            start = time.perf_counter()
            for (ta, *_), lp in zip(stream, lps):
                d = start + ta - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets.append(srv.submit(lp))
            out = [srv.wait(t) for t in tickets]
            wall = time.perf_counter() - start
        st1 = srv.stats()
    dist_barrier(world)
    lat = np.array([(info["done_s"] - info["submit_s"]) * 1e3 for _, info in out])
    # from the stream's first arrival to the last answer on any rank (the ranks
    # start their arrival clocks together, after the barrier)
    end = 0.0
    if out:
        first = min(info["submit_s"] for _, info in out)
        last = max(info["done_s"] for _, info in out)
        end = last - first + stream[0][0]
    makespan = dist_max(end, world) - full[0][0]
    value = len(full) / makespan
    conv = int(dist_sum(sum(r.converged for r, _ in out), world))
    worst = dist_max(max((max(r.eps_P, r.eps_D, r.eps_G) for r, _ in out), default=0.0), world)
    lanes = [info["lane"] for _, info in out]
    sizes = np.array([m for (_, m, *_rest) in stream])
    sizes_all = np.array([m for (_, m, *_rest) in full])
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = serve_cpu_baseline(B, stream, lps, out)
    if rank == 0:
        q = lambda a, f: float(np.quantile(a, f)) if len(a) else None  # noqa: E731
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": 1, "warmup": args.warmup,
            "ms_per_step": makespan * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if prec == B.PREC_MIXED else "f64", "data": "synthetic",
            "config": {"workload": describe(args.workload, seconds=args.serve_seconds, world=world),
                       "requests": len(full), "requests_rank0": len(out),
                       "offered_per_s": len(full) / (args.serve_seconds or p["seconds"]),
                       "classes": {"m<=2000": int((sizes_all <= 2000).sum()),
                                   "2000<m<=50000": int(((sizes_all > 2000) & (sizes_all <= 50000)).sum()),
                                   "m=500000": int((sizes_all == 500_000).sum())},
                       "tol": args.tol, "round_ms": args.round_ms, "hbm_budget_gb": 150,
                       "parallelism": f"sharded x{world} (requests routed in arrival order to the least-loaded "
                                      "rank, no collective)" if world > 1 else "single GPU"},
            "latency_ms": {"p50": q(lat, 0.5), "p99": q(lat, 0.99), "p999": q(lat, 0.999),
                           "max": float(lat.max()) if len(lat) else None,
                           "of": "rank 0's requests" if world > 1 else "all requests",
                           "p50_small": q(lat[sizes <= 2000], 0.5), "p99_small": q(lat[sizes <= 2000], 0.99)},
            "converged": int(conv), "worst_kkt": worst, "whole_gpu_lane": int(sum(lanes)),
            "server": {"rounds": st1["rounds"] - st0["rounds"], "grid_slices": st1["grid_slices"] - st0["grid_slices"],
                       "busy_ms": st1["busy_ms"] - st0["busy_ms"], "peak_bytes": st1["peak_bytes"]},
            "wall_s": wall, "gen_s": t_gen, "clocks": clk.summary(), "cpu_baseline": cpu,
            "gpu_launches": int(st1["rounds"] - st0["rounds"] + st1["grid_slices"] - st0["grid_slices"]),
        }
        print(json.dumps(line), flush=True)


def serve_cpu_baseline(B, stream, lps, out):
    """The reference CPU PDLP serving the whole stream on every host core,
    estimated per size class: the larger requests take a CPU minutes
    (m <= 50,000) to hours (m = 500,000) each, too long to run. Up to three
    requests per class get two bounded runs (8 and 40 attempts, one core),
    which give the class's set-up and time per attempt; a request's CPU time
    is set-up + its attempts (the attempts this engine's served answer took)
    x time per attempt. With C cores the stream needs at least
    max(sum / C, longest request) seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.reference_available():
        return None
    cores = os.cpu_count() or 1
    sizes = np.array([m for (_, m, *_r) in stream])
    classes = {"m<=2000": sizes <= 2000, "2000<m<500000": (sizes > 2000) & (sizes < 500_000),
               "m=500000": sizes >= 500_000}
    times = np.zeros(len(stream))
    model = {}
    for name, mask in classes.items():
        idx = np.flatnonzero(mask)
        if idx.size == 0:
            continue
        setups, pers = [], []
        for i in idx[np.linspace(0, idx.size - 1, min(3, idx.size)).astype(int)]:
            U = B.prepare(lps[i])[0]
            P = O.RefProblem.from_form(O.LPForm(*_form_arrays(U)), use_presolve=False)
            r1 = P.solve_pdhg(max_iterations=8, check_every=64, tol=1e-6)
            r2 = P.solve_pdhg(max_iterations=40, check_every=64, tol=1e-6)
            per = (r2["seconds"] - r1["seconds"]) / max(1, r2["iterations"] - r1["iterations"])
            setups.append(max(0.0, r1["seconds"] - r1["iterations"] * per))
            pers.append(per)
        setup, per = float(np.mean(setups)), float(np.mean(pers))
        for i in idx:
            times[i] = setup + out[i][0].iterations * per
        model[name] = {"requests": int(idx.size), "ms_per_attempt": per * 1e3, "cpu_s": float(times[idx].sum())}
    span = max(times.sum() / cores, times.max())
    return {"value": float(len(stream) / span), "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"per size class, bounded runs (8 and 40 attempts) of the reference solve_pdhg on up to 3 "
                      f"requests; each request = set-up + its attempts x time per attempt; the stream on {cores} "
                      f"cores takes max(sum / cores, longest) = {span:.1f} s",
            "classes": model}


def reference_many(args, world, rank):
    """--impl reference for the batch and the served stream: the reference CPU
    PDLP as independent single-threaded solves on every host core (the
    reference solves one LP per call and has no batching or serving); each
    step is a bounded sample of the workload's LPs."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.reference_available():
        return {"impl": "reference", "unavailable": "reference CPU engine not built (oracle/_ref/libsovref.so)"}
    kind, p = WORKLOADS[args.workload]
    if kind == "batch":
        shapes = batch_shapes(args.workload, args.batch_count, args.batch_mhi, 1)
        gen = ((m, n, k, sd) for (m, n, k, sd) in shapes)
        what = "the batch's LPs in order"
    else:
        stream = serve_stream(p["rate"], args.serve_seconds or p["seconds"], p["seed"])
        gen = ((m, n, k, sd) for (_, m, n, k, sd) in stream if m <= 2000)
        what = "the stream's m <= 2000 requests in arrival order (an upper bound for the whole mix)"
    rates, stats = [], []
    for _ in range(args.warmup + args.steps):
        lps = []
        for (m, n, k, sd) in gen:
            lps.append(O.gen_random_lp(m, n, k, sd, True))
            if len(lps) >= 4 * (os.cpu_count() or 1):
                break
        if not lps:
            break
        r, st = cpu_all_cores(lps, args.cpu_budget_s)
        rates.append(r)
        stats.append(st)
    timed = rates[args.warmup:] or rates[-1:]
    timed_wall = [st["wall_s"] for st in (stats[args.warmup:] or stats[-1:])]
    value = float(np.mean(timed))
    cb = {"value": value, "unit": UNIT, "cores": stats[-1]["cores"], "kind": "reference",
          "sample": f"per step up to {4 * stats[-1]['cores']} of {what}, solve_pdhg to 1e-6, one process per core "
                    f"for about {args.cpu_budget_s:.0f} s; solves/s = cores x LPs / solve seconds"}
    cfg = {"workload": describe(args.workload, count=args.batch_count, seconds=args.serve_seconds),
           "parallelism": f"{stats[-1]['cores']} host cores, one solve per core"}
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": len(timed),
            "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(timed_wall)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": cfg, "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "steps_detail": stats}


def other_configs(args, peak_gbs):
    """The other benchmark configurations, measured after the headline LP on
    one GPU so that every config has a number in the same run: the 2,000 x 500
    transportation LP (K solves from HBM-resident data, CUDA events) and the
    4,096-LP batch (one persistent launch per step). Each entry carries its
    own clocks record."""
    import torch
    import b200pdlp as B
    out = {}
    prec = B.PREC_MIXED if args.precision == "mixed" else B.PREC_FP64
    # transportation LP
    lp = make_lp(B, "transport")
    U, S, Dr, Dc, _ = B.prepare(lp)
    stream = torch.cuda.Stream()
    with B.Engine(U, S, Dr, Dc, precision=prec, stream=stream.cuda_stream) as eng:
        def one():
            return eng.solve(max_iterations=2_000_000, tol=args.tol, copy_out=False, precision=prec,
                             stream=stream.cuda_stream)
        for _ in range(3):
            one()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        res = []
        with ClockSampler(torch.cuda.current_device()) as clk:
            ev[0].record(stream)
            for _ in range(args.extra_steps):
                res.append(one())
            ev[1].record(stream)
            torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1])
        m, n, z = U.m, U.n, U.nnz
        tot_b = sum(r.stats["fp32_accepted"] * algorithmic_bytes(m, n, z, 4)
                    + (r.stats["accepted"] - r.stats["fp32_accepted"]) * algorithmic_bytes(m, n, z, 8) for r in res)
        dev_ms = sum(r.stats["device_ms"] for r in res)
        a_ms = eng.spmv_bench(0, B.PREC_MIXED, 50, stream.cuda_stream)
        r0 = res[-1]
        out["transport"] = {
            "workload": describe("transport"), "value": args.extra_steps / (ms / 1e3), "unit": UNIT,
            "ms_per_step": ms / args.extra_steps, "steps": args.extra_steps, "warmup": 3,
            "attempts": r0.iterations, "fp32_attempts": r0.stats["fp32_attempts"], "converged": r0.converged,
            "eps": [r0.eps_P, r0.eps_D, r0.eps_G],
            "roofline": {"bound": "hbm", "achieved": tot_b / (dev_ms / 1e3) / 1e9, "peak": peak_gbs, "unit": "GB/s",
                         "frac": tot_b / (dev_ms / 1e3) / 1e9 / peak_gbs, "kernel": "k_pdlp (persistent solve)"},
            "spmv_A_frac": spmv_bytes(m, n, z) / (a_ms / 1e3) / 1e9 / peak_gbs, "clocks": clk.summary()}
    # the uneven batch
    probs, n_total = make_batch(B, "batch")
    with B.Batch(probs) as bt:
        info = bt.info()
        bt.solve(max_iterations=2_000_000, tol=args.tol, precision=prec)
        with ClockSampler(torch.cuda.current_device()) as clk:
            res, ms = bt.solve(max_iterations=2_000_000, tol=args.tol, precision=prec)
        lat = sorted(r["device_ms"] for r in res)
        out["batch"] = {
            "workload": describe("batch"), "value": n_total / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
            "steps": 1, "warmup": 1, "converged": int(sum(r["converged"] for r in res)), "lps": n_total,
            "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[int(0.99 * (len(lat) - 1))], "max": lat[-1],
                           "note": "per-LP time on its CTA inside the launch"},
            "sum_nnz": info["sum_nnz"], "clocks": clk.summary()}
    return out


def profile_mode(args):
    """Short runs for profiler captures: builds the engine for the workload and
    launches only the kernel under study."""
    import b200pdlp as B
    lp = make_lp(B, args.workload)
    U, S, Dr, Dc, _ = B.prepare(lp)
    prec = B.PREC_MIXED if args.precision == "mixed" else B.PREC_FP64
    with B.Engine(U, S, Dr, Dc, long_rows=args.long_rows) as eng:
        if args.mode == "spmv":
            a = eng.spmv_bench(0, prec, args.reps)
            t = eng.spmv_bench(1, prec, args.reps)
            print(f"spmv A {a * 1e3:.1f} us, A^T {t * 1e3:.1f} us ({args.precision} vectors)")
        else:
            extra = {"switch_tol": args.switch_tol} if args.switch_tol > 0 else {}
            r = eng.solve(max_iterations=args.max_attempts, tol=args.tol, precision=prec, copy_out=False, **extra)
            print(f"solve: {r.iterations} attempts ({r.stats['fp32_attempts']} FP32), "
                  f"{r.stats['device_ms']:.2f} ms, {1e3 * r.stats['device_ms'] / max(1, r.iterations):.1f} us/attempt, "
                  f"tol {args.tol:g}, converged {r.converged}, eps {r.eps_P:.3e} {r.eps_D:.3e} {r.eps_G:.3e}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large", choices=sorted(WORKLOADS))
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-sample-iters", type=int, default=40)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="large LP: skip the transport LP and batch measurements added to the line")
    ap.add_argument("--extra-steps", type=int, default=5, help="timed solves of the transport LP in other_configs")
    ap.add_argument("--cpu-budget-s", type=float, default=15.0,
                    help="batch / serve: wall seconds of the all-cores reference CPU sample (per step)")
    ap.add_argument("--mode", default="bench", choices=["bench", "spmv", "solve"],
                    help="spmv / solve: one short run of that kernel for profiling (ncu), no JSON line")
    ap.add_argument("--max-attempts", type=int, default=256, help="--mode solve: attempt limit")
    ap.add_argument("--long-rows", type=int, default=0, choices=[0, 1],
                    help="--mode solve/spmv: long rows by the sector cost model (0) or the length rule (1)")
    ap.add_argument("--switch-tol", type=float, default=0.0,
                    help="--mode solve, mixed precision: KKT level of the FP32 -> FP64 hand-over (0: default)")
    ap.add_argument("--reps", type=int, default=1, help="--mode spmv: timed launches per product")
    ap.add_argument("--batch-block", type=int, default=0, help="batch: threads per CTA (128/256/512, 0 auto)")
    ap.add_argument("--batch-count", type=int, default=0, help="batch: LPs (0: 4096)")
    ap.add_argument("--batch-mhi", type=int, default=0, help="batch: largest m of the family (0: 5000; profiling)")
    ap.add_argument("--serve-seconds", type=float, default=0.0, help="serve: arrival window (0: workload default)")
    ap.add_argument("--round-ms", type=float, default=5.0, help="serve: device time of one batched round")
    ap.add_argument("--batch-tail-attempts", type=int, default=0,
                    help="batch: LPs still running at this many attempts finish on 16-CTA clusters (0: off)")
    ap.add_argument("--batch-cluster-nnz", type=int, default=0,
                    help="batch: stored entries from which an LP is solved by a cluster (0 auto, <0 never)")
    args = ap.parse_args()
    world, rank, local = dist_setup(args.gpus)
    if args.mode != "bench":
        return profile_mode(args)
    if args.impl == "reference" and WORKLOADS[args.workload][0] in ("batch", "serve"):
        line = reference_many(args, world, rank)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
        return
    if WORKLOADS[args.workload][0] == "batch":
        return batch_bench(args, world, rank, local)
    if WORKLOADS[args.workload][0] == "serve":
        return serve_bench(args, world, rank, local)

    if args.impl == "reference":
        line = reference_arm(args, world, rank)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
        return

    import torch
    import b200pdlp as B
    torch.cuda.set_device(local)
    prec = B.PREC_MIXED if args.precision == "mixed" else B.PREC_FP64

    t0 = time.time()
    lp = make_lp(B, args.workload)
    U, S, Dr, Dc, _ = B.prepare(lp)
    t_prep = time.time() - t0
    stream = torch.cuda.Stream()
    opts = dict(precision=prec, stream=stream.cuda_stream)
    eng = B.Engine(U, S, Dr, Dc, **opts)
    info = eng.info()

    def one_solve():
        return eng.solve(max_iterations=2_000_000, check_every=64, tol=args.tol, copy_out=False, **opts)

    for _ in range(args.warmup):
        r = one_solve()
    dist_barrier(world)
    torch.cuda.synchronize()
    results = []
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    with ClockSampler(local) as clk:
        ev[0].record(stream)
        for _ in range(args.steps):
            results.append(one_solve())
        ev[1].record(stream)
        torch.cuda.synchronize()
    dist_barrier(world)
    ms_total = ev[0].elapsed_time(ev[1])
    ms_total = dist_max(ms_total, world)
    value = job_rate(world, args.steps, ms_total)
    lat = sorted(r.stats["device_ms"] for r in results)

    # roofline of the persistent kernel: algorithmic bytes of the accepted
    # iterations (FP32 and FP64 phases) over the kernel's own CUDA-event time
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    peak_gbs = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    m, n, z = U.m, U.n, U.nnz
    tot_bytes, tot_ms = 0.0, 0.0
    for r in results:
        acc32 = r.stats["fp32_accepted"]
        acc64 = r.stats["accepted"] - acc32
        tot_bytes += acc32 * algorithmic_bytes(m, n, z, 4) + acc64 * algorithmic_bytes(m, n, z, 8)
        tot_ms += r.stats["device_ms"]
    achieved = tot_bytes / (tot_ms / 1e3) / 1e9
    launches = sum(1 + (1 if 0 < r.stats["fp32_attempts"] < r.iterations else 0) for r in results)
    traffic = None
    if args.workload in TRAFFIC_PER_ATTEMPT and args.precision == "mixed":
        t32, t64 = TRAFFIC_PER_ATTEMPT[args.workload]
        traffic = sum(r.stats["fp32_attempts"] * t32 + (r.iterations - r.stats["fp32_attempts"]) * t64
                      for r in results) / launches

    # standalone SpMV (A x, FP32), the kernel every pass is built on
    spmv_ms = eng.spmv_bench(0, B.PREC_MIXED, 50, stream.cuda_stream)
    spmv_t_ms = eng.spmv_bench(1, B.PREC_MIXED, 50, stream.cuda_stream)
    spmv_gbs = spmv_bytes(m, n, z) / (spmv_ms / 1e3) / 1e9
    spmv_t_gbs = spmv_bytes(n, m, z) / (spmv_t_ms / 1e3) / 1e9

    # e2e: the drop-in C-ABI call with host buffers (layout build, H2D, solve, D2H)
    e2e_ms = []
    for i in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        re = B.solve_pdhg_gpu(U, S, Dr, Dc, 0.99, 2_000_000, 64, args.tol, precision=prec)
        e2e_ms.append((time.perf_counter() - t1) * 1e3)
    e2e_ms = e2e_ms[1:]
    e2e_max = dist_max(sum(e2e_ms), world)
    e2e_value = job_rate(world, len(e2e_ms), e2e_max)
    h2d = info["device_bytes"]
    d2h = 8 * (m + n)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O
            if O.reference_available():
                s = cpu_sample(O, U, args.cpu_sample_iters)
                attempts, source = ref_attempts_per_solve(args.workload)
                if attempts is None:
                    attempts, source = int(statistics.median(r.iterations for r in results)), "this engine's count"
                cpu = {"value": 1.0 / (s["seconds"] / s["iterations"] * attempts), "unit": UNIT, "cores": 1,
                       "kind": "reference", "extrapolated": True,
                       "sample": f"{s['iterations']} attempts of the reference solve_pdhg ({s['seconds']:.2f} s) "
                                 f"on this LP, extrapolated to {attempts} attempts per solve ({source})"}
        except Exception as e:  # the baseline is reported, not required
            cpu = {"error": str(e)}

    others = None
    if rank == 0 and world == 1 and args.workload == "large" and not args.no_other_configs:
        others = other_configs(args, peak_gbs)

    if rank == 0:
        clocks = clk.summary()
        r0 = results[-1]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if prec == B.PREC_MIXED else "f64",
            "data": "synthetic", "config": workload_config(args, U, lp),
            "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                           "max": lat[-1]},
            "solve": {"attempts": r0.iterations, "accepted": r0.stats["accepted"],
                      "fp32_attempts": r0.stats["fp32_attempts"], "restarts": r0.restarts,
                      "checks": r0.stats["checks"], "eps": [r0.eps_P, r0.eps_D, r0.eps_G],
                      "converged": r0.converged, "attempts_per_s": r0.iterations / (r0.stats["device_ms"] / 1e3)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak_gbs, "unit": "GB/s",
                         "frac": achieved / peak_gbs, "traffic": traffic,
                         "algorithmic_bytes_per_launch": tot_bytes / launches,
                         "traffic_note": "bytes per launch: DRAM bytes per attempt from an ncu capture of 256-attempt "
                                         "solves, x the launch's attempts"
                                         if traffic else None,
                         "kernel": "k_pdlp (persistent solve)", "peak_source": peak_src},
            "spmv": {"A_gbs": spmv_gbs, "AT_gbs": spmv_t_gbs, "A_ms": spmv_ms, "AT_ms": spmv_t_ms,
                     "frac_A": spmv_gbs / peak_gbs, "frac_AT": spmv_t_gbs / peak_gbs},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": statistics.mean(e2e_ms)},
            "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
            "prep_s": t_prep, "layout": {k: info[k] for k in ("ctas", "a_padded", "at_padded", "values_exact_fp32")},
            "other_configs": others,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
