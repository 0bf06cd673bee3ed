"""Generates the golden fixtures of the PDLP path from the reference itself.

Run in a container that has the reference tree and the oracle built
(``make -C oracle``):  python tests/golden/make_golden.py [--ref /root/reference]

For every LP fixture the reference's own tests solve with PDLP
(tests/run_checks.cpp:23-107, :144-166) it stores, in ``<name>.npz``:
  * the PDLP-form problem exactly as solve_pdhg_gpu receives it -- presolve
    (src/presolve.cpp:524) -> build_pdlp_form (src/pdlp.cpp:8-82) -> scale
    (src/scaling.cpp:25-84): unscaled form, scaled values/vectors, Dr, Dc;
in ``orig_<name>.npz`` the LP as read (to_ranged_lp, before presolve); and in ``golden.json``:
  * the reference CPU PDLP result on that form (solve_pdhg, src/pdlp.cpp:146) at
    tol 1e-6 and 1e-8: iterations, restarts, eps, the PDLP-form objective, and the
    original-space objective/eps after extract_solution + postsolve + verify;
  * the reference dual simplex (solve_mps_simplex, src/solve.cpp:234) objective;
  * the published optimum the reference's tests pin (tests/run_checks.cpp:116-121).
For the synthetic random-LP family (generated by this repo's seeded generator,
regenerated from its seed at test time) only the reference results are stored.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

# objective optima pinned by the reference's tests (tests/run_checks.cpp:116-121)
PUBLISHED = {
    "afiro": -464.75314286, "adlittle": 225494.96316, "blend": -30.812149846, "sc50a": -64.575077059,
    "sc50b": -70.0, "sc105": -52.202061212, "kb2": -1749.9001299, "scagr7": -2331389.8243,
    "israel": -896644.82186, "share1b": -76589.318579, "beaconfd": 33592.485807, "tiny_range": 10.0,
}
# PDLP fixtures of tests/run_checks.cpp ([1]-[4], [6c]); adlittle is added as one more Netlib case.
CASES = ["afiro", "blend", "sc50a", "sc50b", "kb2", "sc105", "scagr7", "share1b", "beaconfd", "israel",
         "adlittle", "tiny_range"]
# random LP family of the benchmark (m, n, nnz per column, seed, fp32 values)
RANDOM = [(600, 1800, 6, 0, False), (600, 1800, 6, 1, False), (300, 900, 4, 7, True), (1000, 3000, 6, 2, True)]


def form_arrays(prefix, f):
    return {f"{prefix}_row": f.row, f"{prefix}_col": f.col, f"{prefix}_val": f.val, f"{prefix}_c": f.c,
            f"{prefix}_rL": f.rL, f"{prefix}_rU": f.rU, f"{prefix}_l": f.l, f"{prefix}_u": f.u,
            f"{prefix}_dims": np.array([f.m, f.n], np.int64), f"{prefix}_off": np.array([f.obj_offset])}


def ref_results(P, U):
    out = {}
    for tol in (1e-6, 1e-8):
        r = P.solve_pdhg(max_iterations=500000, check_every=64, tol=tol)
        vf = O.verify(U, r["x"], r["y"])
        fin = P.finish(r["x"], r["y"])
        out[f"{tol:g}"] = dict(iterations=r["iterations"], restarts=r["restarts"], converged=r["converged"],
                               eps_P=r["eps_P"], eps_D=r["eps_D"], eps_G=r["eps_G"],
                               form_objective=vf["objective"], final=fin, seconds=r["seconds"])
    return out


def digest(lp) -> str:
    h = hashlib.sha256()
    for a in (lp.row, lp.col, lp.val, lp.c, lp.rL, lp.rU, lp.l, lp.u):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def originals(ref: str):
    """orig_<name>.npz: each fixture's LP as the reference reads it, before
    presolve (read_mps -> to_ranged_lp, include/ranged_lp.hpp:39-62), for the
    presolve and PDLP-form tests."""
    for name in CASES + ["tiny_infeasible", "tiny_unbounded"]:
        path = os.path.join(ref, "sample_problems", f"{name}.mps")
        if not os.path.exists(path):
            continue
        P = O.RefProblem.from_mps(path, use_presolve=False)
        f = P.form(P.ORIGINAL)
        np.savez_compressed(os.path.join(HERE, f"orig_{name}.npz"), **form_arrays("o", f))
        print("original", name, f.m, f.n, f.nnz)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--originals", action="store_true", help="only write the orig_<name>.npz files")
    args = ap.parse_args()
    if args.originals:
        originals(args.ref)
        return
    gold = {"fixtures": {}, "random": {}}
    for name in CASES:
        path = os.path.join(args.ref, "sample_problems", f"{name}.mps")
        P = O.RefProblem.from_mps(path)
        if P.status != 0:
            print("skip", name, "status", P.status)
            continue
        U = P.form(P.PDLP_FORM)
        S = P.form(P.SCALED)
        Dr, Dc = P.scaling()
        arrays = form_arrays("u", U)
        arrays.update({"s_val": S.val, "s_c": S.c, "s_rL": S.rL, "s_rU": S.rU, "s_l": S.l, "s_u": S.u,
                       "Dr": Dr, "Dc": Dc})
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        spx = O.ref_solve_simplex_mps(path)
        gold["fixtures"][name] = dict(m=U.m, n=U.n, nnz=U.nnz, pdlp=ref_results(P, U),
                                      simplex=dict(objective=spx["objective"], status=spx["status"]),
                                      published=PUBLISHED.get(name))
        print(name, U.m, U.n, U.nnz, gold["fixtures"][name]["pdlp"]["1e-06"]["iterations"])

    sys.path.insert(0, os.path.join(ROOT, "team-suprema_b200"))
    import b200pdlp as pkg
    tmp = os.path.join("/tmp", "b200_golden_tmp.mps")
    for (m, n, k, seed, f32) in RANDOM:
        lp = pkg.gen_random_lp(m, n, k, seed, f32)
        P = O.RefProblem.from_form(O.LPForm(lp.m, lp.n, lp.row, lp.col, lp.val, lp.c, lp.rL, lp.rU, lp.l, lp.u))
        U = P.form(P.PDLP_FORM)
        key = f"rand_m{m}_n{n}_k{k}_s{seed}_{'f32' if f32 else 'f64'}"
        P.write_mps(tmp)
        spx = O.ref_solve_simplex_mps(tmp, time_limit=600.0)
        gold["random"][key] = dict(m=m, n=n, k=k, seed=seed, fp32=f32, digest=digest(lp),
                                   presolved_dims=[U.m, U.n, U.nnz], pdlp=ref_results(P, U),
                                   simplex=dict(objective=spx["objective"], status=spx["status"]))
        print(key, gold["random"][key]["pdlp"]["1e-06"]["iterations"], spx["status"])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(gold, f, indent=1, sort_keys=True, default=float)
    originals(args.ref)


if __name__ == "__main__":
    main()
