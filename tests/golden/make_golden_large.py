"""Golden records of the benchmark-size LPs, produced by the reference itself.

    python tests/golden/make_golden_large.py --part cpu            # here: the reference CPU engines
    python tests/golden/make_golden_large.py --part gpu --out F    # on a B200: the reference FP64 GPU engine

The LPs are the benchmark's synthetic ones, built by the oracle's restated
generators (oracle/pdlp_oracle.c; the same bits as the product's generators,
pinned by the content digest stored here), and handed to the reference's own
pipeline without presolve -- build_pdlp_form (src/pdlp.cpp:8-82) -> scale
(src/scaling.cpp:25-84) -- so the reference engines solve exactly the PDLP
form the B200 engine receives:

* large: random equality LP, m = 500,000, n = 1,000,000, 8 nonzeros per
  column, FP32 values, seed 1. The reference's FP64 GPU engine
  (gpu/pdlp_gpu_solve.cu:261-267, built for sm_100a into oracle/_ref) solves it
  to 1e-6; its CPU engine and dual simplex cannot finish it in hours.
* transport: transportation LP, 2,000 sources x 500 sinks (n = 1,000,000,
  m = 2,500), seed 1. The reference CPU PDLP (solve_pdhg, src/pdlp.cpp:146) at
  1e-6 and 1e-8, its dual simplex (solve_mps_simplex, src/solve.cpp:234) on the
  same LP written as MPS, and (gpu part) its FP64 GPU engine at 1e-6.

Each record stores attempts, restarts, eps of the engine's own report, the
PDLP-form objective by the oracle's verify and the wall seconds of the solve
call. The file is tests/golden/large.json; the gpu part runs on a B200 and its
output is merged into that file.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import platform
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

LARGE = dict(m=500_000, n=1_000_000, k=8, seed=1, fp32=True)
TRANSPORT = dict(S=2000, D=500, seed=1)


def digest(lp) -> str:
    h = hashlib.sha256()
    for a in (lp.row, lp.col, lp.val, lp.c, lp.rL, lp.rU, lp.l, lp.u):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def build(name):
    if name == "large":
        p = LARGE
        return O.gen_random_lp(p["m"], p["n"], p["k"], p["seed"], p["fp32"])
    p = TRANSPORT
    return O.gen_transport(p["S"], p["D"], p["seed"])


def record(P, U, r):
    v = O.verify(U, r["x"], r["y"])
    return dict(attempts=r["iterations"], restarts=r["restarts"], converged=r["converged"],
                eps=[r["eps_P"], r["eps_D"], r["eps_G"]],
                verify=dict(eps_P=v["eps_P"], eps_D=v["eps_D"], eps_G=v["eps_G"]),
                form_objective=v["objective"], seconds=r["seconds"])


def host():
    cpu = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                cpu = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return dict(cpu=cpu, cores=os.cpu_count(), python=platform.python_version())


def part_cpu(out):
    lp = build("transport")
    P = O.RefProblem.from_form(lp, use_presolve=False)
    U = P.form(P.PDLP_FORM)
    rec = dict(lp=TRANSPORT, digest=digest(lp), form_dims=[U.m, U.n, U.nnz], host=host())
    for tol in (1e-6, 1e-8):
        r = P.solve_pdhg(max_iterations=2_000_000, check_every=64, tol=tol)
        rec[f"cpu_pdlp_{tol:g}"] = record(P, U, r)
        print("transport cpu pdlp", tol, rec[f"cpu_pdlp_{tol:g}"]["attempts"], rec[f"cpu_pdlp_{tol:g}"]["seconds"],
              flush=True)
    tmp = os.path.join("/tmp", f"b200_golden_transport_{os.getpid()}.mps")
    P.write_mps(tmp)
    try:
        s = O.ref_solve_simplex_mps(tmp, time_limit=1200.0)
    finally:
        os.unlink(tmp)
    rec["dual_simplex"] = dict(objective=s["objective"], status=s["status"], pivots=s["iterations"],
                               seconds=s["seconds"], eps=[s["eps_P"], s["eps_D"], s["eps_G"]])
    print("transport dual simplex", s["status"], s["objective"], s["seconds"], flush=True)
    out.setdefault("transport", {}).update(rec)
    big = build("large")
    out.setdefault("large", {}).update(dict(lp=LARGE, digest=digest(big)))


def part_gpu(out):
    for name in ("transport", "large"):
        lp = build(name)
        P = O.RefProblem.from_form(lp, use_presolve=False, gpu=True)
        U = P.form(P.PDLP_FORM)
        t0 = time.time()
        r = P.solve_pdhg(max_iterations=2_000_000, check_every=64, tol=1e-6, gpu=True)
        rec = record(P, U, r)
        rec["wall_s"] = time.time() - t0
        rec["host"] = host()
        try:
            import subprocess
            rec["gpu"] = subprocess.run(["nvidia-smi", "--query-gpu=name,clocks.max.sm", "--format=csv,noheader"],
                                        capture_output=True, text=True, timeout=30).stdout.strip()
        except Exception:  # noqa: BLE001 - the GPU name is informational
            rec["gpu"] = None
        out.setdefault(name, {}).update({"lp": LARGE if name == "large" else TRANSPORT, "digest": digest(lp),
                                         "gpu_fp64_1e-06": rec})
        print(name, "reference FP64 GPU engine:", rec["attempts"], "attempts", f"{rec['seconds']:.1f} s",
              "objective", rec["form_objective"], flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--part", choices=["cpu", "gpu"], required=True)
    ap.add_argument("--out", default=os.path.join(HERE, "large.json"))
    args = ap.parse_args()
    out = {}
    if os.path.exists(args.out):
        with open(args.out) as f:
            out = json.load(f)
    (part_cpu if args.part == "cpu" else part_gpu)(out)
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True, default=float)


if __name__ == "__main__":
    main()
