"""Random LPs of the benchmark family to a relative KKT tolerance: the
mixed-precision solve against the FP64-only solve of the same engine (whose
decisions are the reference algorithm's, pinned on the fixtures), each answer
certified by the oracle's restated verify() (src/verify.cpp:24-103) on the
unscaled PDLP form.

* the 500,000 x 1,000,000 LP (8M nonzeros) at 1e-6;
* a 20,000 x 40,000 LP of the same family at 1e-8 (the large LP needs about
  1.1M attempts, ~110 s per solve, for 1e-8: measured by
  `bench.py --mode solve --tol 1e-8`, not repeated here).

Measured figures (device seconds, attempts, the objective error of the mixed
solve against the FP64 one) are printed as LARGE_ACCURACY lines."""
import json

import pytest

import b200pdlp as B
import oracle as O
from conftest import as_form, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,tol", [(500_000, 1_000_000, 1e-6), (20_000, 40_000, 1e-8)])
def test_mixed_against_fp64_at_tolerance(m, n, tol):
    U, S, Dr, Dc, _ = B.prepare(B.gen_random_lp(m, n, 8, 1, True))
    form = as_form(U)
    out = {}
    with B.Engine(U, S, Dr, Dc) as eng:
        eng.solve(max_iterations=1000, tol=1e-6)  # warm-up
        for name, prec in (("mixed", B.PREC_MIXED), ("fp64", B.PREC_FP64)):
            r = eng.solve(max_iterations=1_000_000, tol=tol, precision=prec)
            assert r.converged, (name, tol, r.stats)
            v = O.verify(form, r.x, r.y)
            worst = max(v["eps_P"], v["eps_D"], v["eps_G"])
            assert worst <= tol * (1 + 1e-6), (name, tol, v)
            out[name] = {"seconds": r.stats["device_ms"] / 1e3, "attempts": r.iterations,
                         "fp32_attempts": r.stats["fp32_attempts"], "objective": v["objective"], "kkt": worst}
    err = rel(out["mixed"]["objective"], out["fp64"]["objective"])
    print("LARGE_ACCURACY " + json.dumps({"m": m, "n": n, "tol": tol, "objective_rel_err_mixed_vs_fp64": err, **out}))
    # both points satisfy the same KKT bound; their objectives agree to the gap it allows
    assert err <= 10 * tol
