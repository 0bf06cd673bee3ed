"""The whole-grid kernel's work-balanced schedule of slice records
(schedule_records in the library's host code), checked on the CPU through a
small C++ program linked against the library: for the layouts of the
2,000 x 500 transportation LP (dense runs and split groups), a random LP and
one long dense row (255-segment split groups), at several warp counts, the
schedule is a permutation of the records in contiguous per-warp ranges;
inside a warp no record that waits (a subgroup leader, a group owner) comes
before one that waits for nothing, and no owner before a leader, so every
wait of a split group ends; and no warp holds more than the average load
plus the costliest record (the longest-first bound)."""
import os
import subprocess

import numpy as np

import b200pdlp as B
from conftest import ROOT

PROGRAM = r"""
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "internal.h"

static std::vector<char> slurp(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) std::exit(2);
    std::vector<char> b;
    char buf[1 << 16];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) b.insert(b.end(), buf, buf + k);
    std::fclose(f);
    return b;
}

struct Reader {
    const char* p;
    template <class T> const T* take(size_t n) { const T* q = reinterpret_cast<const T*>(p); p += n * sizeof(T); return q; }
};

static int check(const b2::SellHost& S, int warps, const char* tag) {
    std::vector<int32_t> seq, start;
    b2::schedule_records(S, warps, 8, 16, seq, start);
    const int64_t n = S.n_slices();
    if ((int64_t)seq.size() != n || (int64_t)start.size() != warps + 1 || start[0] != 0 || start[warps] != n) return 10;
    std::vector<char> seen((size_t)n, 0);
    for (int32_t r : seq) { if (r < 0 || r >= n || seen[(size_t)r]) return 11; seen[(size_t)r] = 1; }
    auto cost = [&](int32_t r) -> int64_t {
        const int64_t len = (int64_t)((uint32_t)S.slice[(size_t)(4 * r + 1)] & b2::kLenMask);
        const bool dense = !S.aff.empty() && S.aff[(size_t)(2 * r)] >= 0;
        return dense ? (len + 7) / 8 + 2 : len + 4;
    };
    auto cls = [&](int32_t r) {
        const uint32_t w = (uint32_t)S.slice[(size_t)(4 * r + 3)];
        if (w == 0) return 0;
        const int q = (int)(w >> 24);
        return q == 0 ? 2 : (q % 16 == 0 ? 1 : 0);
    };
    int64_t total = 0, most = 0, top = 0;
    for (int64_t r = 0; r < n; ++r) { total += cost((int32_t)r); top = std::max(top, cost((int32_t)r)); }
    int waiting = 0;
    for (int w = 0; w < warps; ++w) {
        if (start[w + 1] < start[w]) return 12;
        int64_t load = 0;
        int last = 0;
        for (int32_t k = start[w]; k < start[w + 1]; ++k) {
            const int c = cls(seq[(size_t)k]);
            if (c < last) return 13;
            last = c;
            waiting += c > 0;
            load += cost(seq[(size_t)k]);
        }
        most = std::max(most, load);
    }
    const double mean = (double)total / warps;
    if ((double)most > mean + (double)top + 1e-9) return 14;
    std::printf("%s warps %d records %lld waiting %d max %lld mean %.1f top %lld\n", tag, warps, (long long)n, waiting,
                (long long)most, mean, (long long)top);
    return 0;
}

int main(int argc, char** argv) {
    for (int a = 1; a < argc; ++a) {
        std::vector<char> buf = slurp(argv[a]);
        Reader rd{buf.data()};
        const int64_t* dims = rd.take<int64_t>(3);
        b2_lp_view U{}, Sv{};
        U.m = Sv.m = (int32_t)dims[0];
        U.n = Sv.n = (int32_t)dims[1];
        U.nnz = Sv.nnz = dims[2];
        U.row_idx = Sv.row_idx = rd.take<int32_t>((size_t)U.nnz);
        U.col_idx = Sv.col_idx = rd.take<int32_t>((size_t)U.nnz);
        U.val = rd.take<double>((size_t)U.nnz);
        Sv.val = rd.take<double>((size_t)U.nnz);
        for (b2_lp_view* v : {&U, &Sv}) {
            v->c = rd.take<double>((size_t)U.n);
            v->rL = rd.take<double>((size_t)U.m);
            v->rU = rd.take<double>((size_t)U.m);
            v->l = rd.take<double>((size_t)U.n);
            v->u = rd.take<double>((size_t)U.n);
        }
        const double* Dr = rd.take<double>((size_t)U.m);
        const double* Dc = rd.take<double>((size_t)U.n);
        b2::BuildParams bp;
        bp.split = true;
        b2::Layout L;
        b2::build_layout(U, Sv, Dr, Dc, bp, L);
        for (int warps : {1, 2, 64, 4736}) {
            int e = check(L.A, warps, "A");
            if (e) return e;
            e = check(L.AT, warps, "AT");
            if (e) return e;
        }
    }
    std::printf("schedule ok\n");
    return 0;
}
"""


def write_lp(path, lp):
    U, S, Dr, Dc, _ = B.prepare(lp)
    U, S = B.RangedLP.like(U), B.RangedLP.like(S)
    with open(path, "wb") as f:
        f.write(np.array([U.m, U.n, U.nnz], np.int64).tobytes())
        f.write(np.asarray(U.row, np.int32).tobytes())
        f.write(np.asarray(U.col, np.int32).tobytes())
        f.write(np.asarray(U.val, np.float64).tobytes())
        f.write(np.asarray(S.val, np.float64).tobytes())
        for v in (U, S):
            for a in (v.c, v.rL, v.rU, v.l, v.u):
                f.write(np.asarray(a, np.float64).tobytes())
        f.write(np.asarray(Dr, np.float64).tobytes())
        f.write(np.asarray(Dc, np.float64).tobytes())


def test_schedule_is_a_balanced_wait_safe_permutation(tmp_path):
    n = 80_000
    dense_row = B.RangedLP(1, n, np.zeros(n, np.int64), np.arange(n), np.ones(n), np.ones(n), np.array([1.0]),
                           np.array([1.0]), np.zeros(n), np.full(n, 10.0))
    files = []
    for name, lp in (("transport", B.gen_transport(2000, 500, 1)), ("random", B.gen_random_lp(20000, 40000, 8, 1, True)),
                     ("dense_row", dense_row)):
        p = tmp_path / f"{name}.bin"
        write_lp(p, lp)
        files.append(str(p))
    src = tmp_path / "sched.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "sched"
    libdir = os.path.dirname(B.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(libdir, "csrc"),
           str(src), "-o", str(exe), "-L", libdir, "-lb200pdlp", f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)] + files, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    assert "schedule ok" in r.stdout
    # the split groups' leaders and owners were there to be ordered
    assert any("waiting" in l and " waiting 0 " not in l for l in r.stdout.splitlines())
