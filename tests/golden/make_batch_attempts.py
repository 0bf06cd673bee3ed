"""Writes tests/golden/batch_attempts.csv: for each of the 4,096 LPs of the
uneven batch family (seed 0, m log-uniform on [50, 5000], the benchmark's
batch), its PDLP-form dimensions and the attempts this engine's batched
solve took to 1e-6 on a B200. The shard-plan test uses the attempts as the
measured cost of each LP. Needs a GPU; run from the repository root:

    python tests/golden/make_batch_attempts.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "team-suprema_b200"))
import b200pdlp as B  # noqa: E402


def main():
    shapes = B.batch_family_shapes(4096, seed=0, m_hi=5000)
    probs = []
    for (m, n, k, sd) in shapes:
        U, S, Dr, Dc, _ = B.prepare(B.gen_random_lp(m, n, k, sd, True))
        probs.append((U, S, Dr, Dc))
    with B.Batch(probs) as bt:
        res, _ = bt.solve(max_iterations=500000, tol=1e-6)
    assert all(r["converged"] for r in res)
    with open(os.path.join(HERE, "batch_attempts.csv"), "w") as f:
        f.write("m,n,nnz,attempts\n")
        for (U, _, _, _), r in zip(probs, res):
            f.write(f"{U.m},{U.n},{int(U.nnz)},{r['iterations']}\n")


if __name__ == "__main__":
    main()
