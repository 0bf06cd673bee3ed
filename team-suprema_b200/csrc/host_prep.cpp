// host_prep.cpp -- host side of the engine that needs no GPU:
//   * validation of the PDLP form handed over by solve_pdhg_gpu's callers,
//   * the device layout (row/column permutations and the sliced-ELL format of
//     A and A^T, with per-row/per-column vectors in the same permuted order),
//   * Ruiz + Pock-Chambolle scaling (same algorithm as src/scaling.cpp:25-84),
//   * seeded generators for the benchmark LP shapes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <queue>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace b2 {

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

// Runs f(begin, end, chunk) over [0, n) cut into contiguous chunks, one per
// thread (at most `threads`, none shorter than `grain`); the calling thread
// takes chunk 0. Returns the number of chunks.
template <class F>
int parallel_chunks(int threads, int64_t n, int64_t grain, F&& f) {
    const int nch = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(1, threads), n / std::max<int64_t>(1, grain)));
    if (nch <= 1) {
        f(int64_t(0), n, 0);
        return 1;
    }
    const int64_t per = (n + nch - 1) / nch;
    std::vector<std::thread> pool;
    for (int t = 1; t < nch; ++t) {
        const int64_t b = std::min(n, t * per), e = std::min(n, b + per);
        pool.emplace_back([&f, b, e, t] { f(b, e, t); });
    }
    f(int64_t(0), std::min(n, per), 0);
    for (auto& th : pool) th.join();
    return nch;
}

// Smallest k in [0, n) with bad(k), or -1; chunks searched in parallel.
template <class P>
int64_t first_bad(int threads, int64_t n, P&& bad) {
    std::vector<int64_t> hit((size_t)std::max(1, threads), -1);
    parallel_chunks(threads, n, 1 << 16, [&](int64_t b, int64_t e, int t) {
        for (int64_t k = b; k < e; ++k)
            if (bad(k)) {
                hit[t] = k;
                return;
            }
    });
    for (int64_t h : hit)
        if (h >= 0) return h;  // chunks are in index order
    return -1;
}

// CSR with the stable fill order of include/sparse.hpp:24-40 (entries of a row
// keep their COO order). With several threads, each takes a contiguous run of
// the COO entries: it counts its entries per row, the counts are turned into
// per-run start offsets (earlier runs first inside every row), and each run
// scatters its own entries, so the result is the serial one.
void coo_to_csr(int64_t rows, int64_t nnz, const int32_t* r, const int32_t* c, const double* v,
                std::vector<int64_t>& ptr, std::vector<int32_t>& idx, std::vector<double>& val, int threads = 1) {
    ptr.assign(rows + 1, 0);
    idx.resize(nnz);
    val.resize(nnz);
    const int nch = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(1, threads), nnz / (1 << 18)));
    if (nch <= 1) {
        for (int64_t k = 0; k < nnz; ++k) ptr[r[k] + 1]++;
        for (int64_t i = 0; i < rows; ++i) ptr[i + 1] += ptr[i];
        std::vector<int64_t> cur(ptr.begin(), ptr.end() - 1);
        for (int64_t k = 0; k < nnz; ++k) {
            int64_t p = cur[r[k]]++;
            idx[p] = c[k];
            val[p] = v[k];
        }
        return;
    }
    const int64_t per = (nnz + nch - 1) / nch;
    std::vector<std::vector<int64_t>> cur((size_t)nch);
    auto runs = [&](auto&& body) {
        std::vector<std::thread> pool;
        for (int t = 1; t < nch; ++t) pool.emplace_back([&body, t] { body(t); });
        body(0);
        for (auto& th : pool) th.join();
    };
    runs([&](int t) {
        cur[t].assign((size_t)rows, 0);
        const int64_t b = std::min(nnz, t * per), e = std::min(nnz, b + per);
        for (int64_t k = b; k < e; ++k) cur[t][r[k]]++;
    });
    parallel_chunks(nch, rows, 1 << 14, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; ++i) {
            int64_t tot = 0;
            for (int t = 0; t < nch; ++t) tot += cur[t][i];
            ptr[i + 1] = tot;
        }
    });
    for (int64_t i = 0; i < rows; ++i) ptr[i + 1] += ptr[i];
    parallel_chunks(nch, rows, 1 << 14, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; ++i) {
            int64_t off = ptr[i];
            for (int t = 0; t < nch; ++t) {
                const int64_t cnt = cur[t][i];
                cur[t][i] = off;
                off += cnt;
            }
        }
    });
    runs([&](int t) {
        const int64_t b = std::min(nnz, t * per), e = std::min(nnz, b + per);
        int64_t* cu = cur[t].data();
        for (int64_t k = b; k < e; ++k) {
            const int64_t p = cu[r[k]]++;
            idx[p] = c[k];
            val[p] = v[k];
        }
    });
}

// Rows sorted by length, longest first, inside windows of `window` rows; the
// window keeps neighbouring rows together so gathers keep their locality.
std::vector<int32_t> sigma_sort(const std::vector<int64_t>& ptr, int window, int threads = 1) {
    const int32_t rows = (int32_t)ptr.size() - 1;
    std::vector<int32_t> perm(rows);
    std::iota(perm.begin(), perm.end(), 0);
    if (window <= 1) return perm;
    const int64_t windows = ((int64_t)rows + window - 1) / window;
    parallel_chunks(threads, windows, 64, [&](int64_t wb, int64_t we, int) {
        for (int64_t wi = wb; wi < we; ++wi) {
            const int64_t w0 = wi * window, w1 = std::min<int64_t>(w0 + window, rows);
            std::stable_sort(perm.begin() + w0, perm.begin() + w1, [&](int32_t a, int32_t b) {
                return ptr[a + 1] - ptr[a] > ptr[b + 1] - ptr[b];
            });
        }
    });
    return perm;
}

int pick_lanes(int64_t len, int lane_target) {
    int g = 1;
    while (g < 32 && (len + g - 1) / g > lane_target) g <<= 1;
    return g;
}

// Memory cost of one slice: the 32-byte sectors of x (4-byte values) its
// gathers touch, step by step, plus the col/val stream (32 lanes x 8 bytes =
// 8 sectors per step, padding included). Rows perm[i .. i+nr), g lanes per row.
double slice_cost(const std::vector<int64_t>& ptr, const std::vector<int32_t>& idx, const std::vector<int32_t>& perm,
                  const std::vector<int32_t>& inv_col, int32_t i, int32_t nr, int g, int64_t len) {
    // at most 64 evenly spaced steps are counted and scaled to the slice
    const int64_t stride = std::max<int64_t>(1, len / 64);
    double sectors = 0.0;
    int64_t samples = 0;
    uint32_t ids[32];
    for (int64_t k = 0; k < len; k += stride) {
        ++samples;
        int cnt = 0;
        for (int lane = 0; lane < 32; ++lane) {
            const int32_t rl = lane / g, sub = lane % g;
            if (rl >= nr) break;
            const int32_t r = perm[i + rl];
            const int64_t b = ptr[r], e = ptr[r + 1];
            if (e == b) continue;
            // a padding entry gathers the lane's last real column again
            int64_t p = b + sub + k * g;
            if (p >= e) p = b + sub + ((e - 1 - b - sub) / g) * g;
            if (p < b || p >= e) p = b;
            ids[cnt++] = (uint32_t)inv_col[idx[p]] >> 3;
        }
        std::sort(ids, ids + cnt);
        sectors += (double)(std::unique(ids, ids + cnt) - ids);
    }
    return 8.0 * (double)len + (samples ? sectors * (double)len / (double)samples : 0.0);
}

// Builds the sliced format of the rows `perm` (device order) of a CSR whose
// column indices are mapped through `inv_col`.
void build_sell(const std::vector<int64_t>& ptr, const std::vector<int32_t>& idx, const std::vector<double>& val,
                const std::vector<int32_t>& perm, const std::vector<int32_t>& inv_col, int n_cols, int lane_target,
                bool keep64, const BuildParams& bp, SellHost& S) {
    const int32_t rows = (int32_t)perm.size();
    S.n_rows = rows;
    S.n_cols = n_cols;
    S.slice.clear();
    S.seg.clear();
    S.seg_slots = 0;
    S.seg_max = 0;
    // pass 1: slice shapes
    struct Shape { int32_t row0, nrows, lg; int64_t len, blk; };
    std::vector<Shape> shapes;
    int64_t blk = 0;
    // A slice does not run on into the next sigma window: rows are sorted
    // longest first inside a window, so such a slice would take the next
    // window's longest row as its length (padding every shorter row up to it,
    // and splitting the slice once it is longer than split_steps). A slice
    // always covers 32 / g rows (the device derives a lane's row from that;
    // only the matrix's last slice may hold fewer), so a slice that would
    // cross the window's end takes more lanes per row instead: the largest
    // power of two of rows that still fits.
    const int window = bp.sigma_window > 0 ? bp.sigma_window : 1024;
    auto shape_of = [&](int32_t i, int& g, int32_t& nr, int64_t& len) {
        const int64_t wend = ((int64_t)i / window + 1) * window;
        if (wend < rows && wend - i < 32 / g) {
            int64_t p = 1;
            while (p * 2 <= wend - i) p *= 2;
            g = (int)(32 / p);
        }
        nr = (int32_t)std::min<int64_t>(32 / g, rows - i);
        if (nr != 32 / g && i + nr != rows) fail(B2_ERR_INVALID, "sliced layout: a slice short of rows inside the matrix");
        int64_t lmax = 0;
        for (int32_t t = 0; t < nr; ++t) lmax = std::max<int64_t>(lmax, ptr[perm[i + t] + 1] - ptr[perm[i + t]]);
        len = (lmax + g - 1) / g;
    };
    // the tuned choice is kept for a shape class: rows of the same length in
    // the same sigma window
    int64_t class_len = -1, class_win = -1;
    int class_g = 0;
    for (int32_t i = 0; i < rows;) {
        const int32_t r0 = perm[i];
        const int64_t rlen = ptr[r0 + 1] - ptr[r0];
        int g = pick_lanes(rlen, lane_target);
        int32_t nr = 0;
        int64_t len = 0;
        shape_of(i, g, nr, len);
        if (bp.split && rlen >= bp.tune_len && rlen == class_len && i / window == class_win) {
            if (class_g != g) {
                g = class_g;
                shape_of(i, g, nr, len);
            }
        } else if (bp.split && rlen >= bp.tune_len) {
            // long rows: the lanes-per-row whose slice touches the fewest
            // sectors per entry wins if it beats the length rule by 20%
            auto entries = [&](int32_t a, int32_t cnt) {
                int64_t e = 0;
                for (int32_t t = 0; t < cnt; ++t) e += ptr[perm[a + t] + 1] - ptr[perm[a + t]];
                return (double)std::max<int64_t>(e, 1);
            };
            const double base = slice_cost(ptr, idx, perm, inv_col, i, nr, g, len) / entries(i, nr);
            double best = base * 0.8;
            int best_g = g;
            for (int cg = 1; cg <= 32; cg <<= 1) {
                int eg = cg;  // the lanes per row the slice gets (more at a window's end)
                int32_t cnr = 0;
                int64_t clen = 0;
                shape_of(i, eg, cnr, clen);
                if (eg == g) continue;
                const double c = slice_cost(ptr, idx, perm, inv_col, i, cnr, eg, clen) / entries(i, cnr);
                if (c < best) { best = c; best_g = eg; }
            }
            if (best_g != g) {
                g = best_g;
                shape_of(i, g, nr, len);
            }
            class_len = rlen;
            class_win = i / window;
            class_g = g;
        }
        if (len > (int64_t)kLenMask) fail(B2_ERR_UNSUPPORTED, "row too long for the sliced format");
        int lg = 0;
        while ((1 << lg) < g) ++lg;
        shapes.push_back({i, nr, lg, len, blk});
        blk += len;
        i += nr;
    }
    if (blk >= (int64_t)std::numeric_limits<uint32_t>::max()) fail(B2_ERR_UNSUPPORTED, "matrix too large");
    S.padded = blk * 32;
    S.col.assign((size_t)S.padded, 0u);
    S.val32.assign((size_t)S.padded, 0.0f);
    if (keep64) S.val64.assign((size_t)S.padded, 0.0);
    else S.val64.clear();
    // slice records: a slice longer than split_steps becomes segments of at
    // most that many steps (at most 255 of them), consecutive slice records
    // over the same rows and storage
    const int64_t split_at = bp.split ? std::max(1, bp.split_steps) : INT64_MAX;
    S.slice.reserve(shapes.size() * 4);
    std::vector<std::pair<int32_t, int64_t>> rec;  // slice record -> (shape, first step)
    rec.reserve(shapes.size());
    for (size_t s = 0; s < shapes.size(); ++s) {
        const Shape& sh = shapes[s];
        if (sh.len > split_at) {
            const int64_t seg_steps = std::max<int64_t>(split_at, (sh.len + 254) / 255);
            const int64_t q_count = (sh.len + seg_steps - 1) / seg_steps;
            const int64_t group = S.n_groups();
            if (group + 1 >= (1 << 24)) fail(B2_ERR_UNSUPPORTED, "too many split slices");
            S.seg.push_back((int32_t)q_count);
            S.seg.push_back((int32_t)S.seg_slots);
            S.seg_slots += q_count;
            S.seg_max = std::max<int32_t>(S.seg_max, (int32_t)q_count);
            for (int64_t q = 0; q < q_count; ++q) {
                const int64_t l0 = q * seg_steps, l1 = std::min(sh.len, l0 + seg_steps);
                rec.emplace_back((int32_t)s, l0);
                S.slice.push_back(sh.row0);
                S.slice.push_back((int32_t)((uint32_t)(l1 - l0) | ((uint32_t)sh.lg << kLenBits)));
                S.slice.push_back((int32_t)(uint32_t)(sh.blk + l0));
                S.slice.push_back((int32_t)((uint32_t)(group + 1) | ((uint32_t)q << 24)));
            }
        } else {
            rec.emplace_back((int32_t)s, 0);
            S.slice.push_back(sh.row0);
            S.slice.push_back((int32_t)((uint32_t)sh.len | ((uint32_t)sh.lg << kLenBits)));
            S.slice.push_back((int32_t)(uint32_t)sh.blk);
            S.slice.push_back(0);
        }
    }
    // fill: every slice owns its storage range, so ranges of slices fill in
    // parallel (the result does not depend on the thread count)
    auto fill = [&](size_t s0, size_t s1) {
        for (size_t s = s0; s < s1; ++s) {
            const Shape& sh = shapes[s];
            const int g = 1 << sh.lg;
            for (int lane = 0; lane < 32; ++lane) {
                const int32_t rl = lane / g, sub = lane % g;
                uint32_t last_col = 0;
                int64_t k = 0;
                if (rl < sh.nrows) {
                    const int32_t r = perm[sh.row0 + rl];
                    const int64_t b = ptr[r], e = ptr[r + 1];
                    if (e > b) last_col = (uint32_t)inv_col[idx[b]];
                    for (int64_t p = b + sub; p < e; p += g, ++k) {
                        const size_t pos = (size_t)((sh.blk + k) * 32 + lane);
                        last_col = (uint32_t)inv_col[idx[p]];
                        S.col[pos] = last_col;
                        S.val32[pos] = (float)val[p];
                        if (keep64) S.val64[pos] = val[p];
                    }
                }
                for (; k < sh.len; ++k) S.col[(size_t)((sh.blk + k) * 32 + lane)] = last_col;  // value stays 0
            }
        }
    };
    const size_t nth = std::max<size_t>(1, std::min<size_t>((size_t)std::max(1, bp.threads), shapes.size() / 256 + 1));
    if (nth <= 1) {
        fill(0, shapes.size());
    } else {
        std::vector<std::thread> pool;
        const size_t per = (shapes.size() + nth - 1) / nth;
        for (size_t t = 0; t < nth; ++t) {
            const size_t s0 = std::min(shapes.size(), t * per), s1 = std::min(shapes.size(), s0 + per);
            pool.emplace_back(fill, s0, s1);
        }
        for (auto& th : pool) th.join();
    }
    if (!bp.split) return;
    // dense runs: each record is checked on its own; most fail on the first
    // lanes, and a record that passes is read once more in full
    S.aff.assign(rec.size() * 2, 0);
    S.n_dense = 0;
    for (size_t r = 0; r < rec.size(); ++r) {
        S.aff[2 * r] = -1;
        const Shape& sh = shapes[(size_t)rec[r].first];
        const int64_t l0 = rec[r].second;
        const int64_t len = (int64_t)((uint32_t)S.slice[4 * r + 1] & kLenMask);
        const int64_t blk0 = sh.blk + l0;
        const int g = 1 << sh.lg;
        // stored entries of each lane: a row of e entries gives lane sub of it
        // ceil((e - sub) / g) of them
        int64_t cnt[32];
        for (int lane = 0; lane < 32; ++lane) {
            const int32_t rl = lane / g, sub = lane % g;
            cnt[lane] = 0;
            if (rl < sh.nrows) {
                const int32_t row = perm[sh.row0 + rl];
                const int64_t e = ptr[row + 1] - ptr[row];
                cnt[lane] = e > sub ? (e - sub + g - 1) / g : 0;
            }
        }
        if (len < 1 || cnt[0] <= l0 || (len > 1 && cnt[0] <= l0 + 1)) continue;
        const int64_t c0 = S.col[(size_t)(blk0 * 32)];
        const int64_t ks = len > 1 ? (int64_t)S.col[(size_t)((blk0 + 1) * 32)] - c0 : 0;
        bool ok = ks >= INT32_MIN && ks <= INT32_MAX;
        for (int64_t k = 0; k < len && ok; ++k)
            for (int lane = 0; lane < 32 && ok; ++lane) {
                const int64_t want = c0 + k * ks + lane;
                if (want < 0 || want >= (int64_t)S.n_cols) ok = false;
                else if (l0 + k < cnt[lane] && (int64_t)S.col[(size_t)((blk0 + k) * 32 + lane)] != want) ok = false;
            }
        if (!ok) continue;
        S.aff[2 * r] = (int32_t)c0;
        S.aff[2 * r + 1] = (int32_t)ks;
        ++S.n_dense;
    }
    if (S.n_dense == 0) S.aff.clear();
}

double finite_inf_norm(const double* v, int64_t len) {
    double m = 0.0;
    for (int64_t i = 0; i < len; ++i)
        if (std::isfinite(v[i])) m = std::max(m, std::fabs(v[i]));
    return m;
}

}  // namespace

void build_layout(const b2_lp_view& U, const b2_lp_view& S, const double* Dr, const double* Dc,
                  const BuildParams& bp, Layout& L) {
    const int32_t m = U.m, n = U.n;
    const int64_t nnz = U.nnz;
    if (m < 0 || n < 0 || nnz < 0) fail(B2_ERR_INVALID, "negative dimension");
    if (S.m != m || S.n != n || S.nnz != nnz) fail(B2_ERR_INVALID, "scaled form does not match the unscaled form");
    if (nnz > 0 && (!U.row_idx || !U.col_idx || !U.val || !S.val)) fail(B2_ERR_INVALID, "null matrix pointer");
    if ((n > 0 && (!U.c || !U.l || !U.u || !S.c || !S.l || !S.u || !Dc)) ||
        (m > 0 && (!U.rL || !U.rU || !S.rL || !Dr)))
        fail(B2_ERR_INVALID, "null vector pointer");
    const int th = std::max(1, bp.threads);
    // the entries are checked in parallel; the first bad one is reported
    const int64_t bad = first_bad(th, nnz, [&](int64_t k) {
        return U.row_idx[k] < 0 || U.row_idx[k] >= m || U.col_idx[k] < 0 || U.col_idx[k] >= n ||
               !std::isfinite(U.val[k]) || !std::isfinite(S.val[k]);
    });
    if (bad >= 0) {
        const int64_t k = bad;
        if (U.row_idx[k] < 0 || U.row_idx[k] >= m || U.col_idx[k] < 0 || U.col_idx[k] >= n)
            fail(B2_ERR_INVALID, "matrix index out of range at entry " + std::to_string(k));
        fail(B2_ERR_NONFINITE, "non-finite matrix value at entry " + std::to_string(k));
    }
    // PDLP-form invariant (src/pdlp.cpp:59-62): rL finite, rU == rL or +inf.
    for (int32_t i = 0; i < m; ++i) {
        if (!std::isfinite(U.rL[i])) fail(B2_ERR_NONFINITE, "rL must be finite in the PDLP form (row " + std::to_string(i) + ")");
        if (!(U.rU[i] == U.rL[i] || (std::isinf(U.rU[i]) && U.rU[i] > 0)))
            fail(B2_ERR_INVALID, "row " + std::to_string(i) + " is neither an equality nor a >= row");
        if (!(Dr[i] > 0) || !std::isfinite(Dr[i])) fail(B2_ERR_INVALID, "Dr must be positive and finite");
    }
    auto col_bad = [&](int64_t j) {
        const double want = Dc[j] * U.c[j];
        return !std::isfinite(U.c[j]) || !std::isfinite(S.c[j]) || std::isnan(U.l[j]) || std::isnan(U.u[j]) ||
               U.l[j] > U.u[j] || !(Dc[j] > 0) || !std::isfinite(Dc[j]) ||
               std::fabs(S.c[j] - want) > 1e-9 * (1.0 + std::fabs(want));
    };
    const int64_t jb = first_bad(th, n, col_bad);
    if (jb >= 0) {
        const int64_t j = jb;
        if (!std::isfinite(U.c[j]) || !std::isfinite(S.c[j])) fail(B2_ERR_NONFINITE, "non-finite cost at column " + std::to_string(j));
        if (std::isnan(U.l[j]) || std::isnan(U.u[j]) || U.l[j] > U.u[j])
            fail(B2_ERR_INVALID, "bad bounds at column " + std::to_string(j));
        if (!(Dc[j] > 0) || !std::isfinite(Dc[j])) fail(B2_ERR_INVALID, "Dc must be positive and finite");
        fail(B2_ERR_INVALID, "scaled cost is not Dc * cost at column " + std::to_string(j));
    }

    L.m = m; L.n = n; L.nnz = nnz;
    std::vector<int64_t> aptr, tptr;
    std::vector<int32_t> aidx, tidx;
    std::vector<double> aval, tval;
    coo_to_csr(m, nnz, U.row_idx, U.col_idx, U.val, aptr, aidx, aval, th);
    coo_to_csr(n, nnz, U.col_idx, U.row_idx, U.val, tptr, tidx, tval, th);

    L.exact32 = first_bad(th, nnz, [&](int64_t k) { return (double)(float)U.val[k] != U.val[k]; }) < 0;

    const int window = bp.sigma_window > 0 ? bp.sigma_window : 1024;
    const int target = bp.lane_target > 0 ? bp.lane_target : 16;
    L.perm_r = sigma_sort(aptr, window, th);
    L.perm_c = sigma_sort(tptr, window, th);
    L.inv_r.assign(m, 0);
    L.inv_c.assign(n, 0);
    for (int32_t i = 0; i < m; ++i) L.inv_r[L.perm_r[i]] = i;
    parallel_chunks(th, n, 1 << 16, [&](int64_t b, int64_t e, int) {
        for (int64_t j = b; j < e; ++j) L.inv_c[L.perm_c[j]] = (int32_t)j;
    });

    if (bp.threads > 1) {
        BuildParams half = bp;
        half.threads = std::max(1, bp.threads / 2);
        std::thread ta([&] { build_sell(aptr, aidx, aval, L.perm_r, L.inv_c, n, target, !L.exact32, half, L.A); });
        build_sell(tptr, tidx, tval, L.perm_c, L.inv_r, m, target, !L.exact32, half, L.AT);
        ta.join();
    } else {
        build_sell(aptr, aidx, aval, L.perm_r, L.inv_c, n, target, !L.exact32, bp, L.A);
        build_sell(tptr, tidx, tval, L.perm_c, L.inv_r, m, target, !L.exact32, bp, L.AT);
    }

    L.b.resize(m); L.rU.resize(m); L.dr2.resize(m);
    for (int32_t i = 0; i < m; ++i) {
        const int32_t o = L.perm_r[i];
        L.b[i] = U.rL[o];
        L.rU[i] = U.rU[o];
        const double w = Dr[o] * Dr[o];
        L.dr2[i] = (U.rL[o] != U.rU[o]) ? -w : w;
    }
    L.c.resize(n); L.l.resize(n); L.u.resize(n); L.dc2.resize(n); L.x0.resize(n);
    parallel_chunks(th, n, 1 << 16, [&](int64_t b, int64_t e, int) {
        for (int64_t j = b; j < e; ++j) {
            const int32_t o = L.perm_c[j];
            L.c[j] = U.c[o];
            L.l[j] = U.l[o];
            L.u[j] = U.u[o];
            L.dc2[j] = Dc[o] * Dc[o];
            // initial point of include/pdlp_algo.hpp:69, mapped to unscaled space
            L.x0[j] = Dc[o] * std::min(std::max(0.0, S.l[o]), S.u[o]);
        }
    });
    // one pair of bounds for every column (bitwise): the kernels then read no l, u
    L.lu_const = n > 0 && first_bad(th, n, [&](int64_t j) {
                              return std::memcmp(&L.l[j], &L.l[0], sizeof(double)) != 0 ||
                                     std::memcmp(&L.u[j], &L.u[0], sizeof(double)) != 0;
                          }) < 0;
    L.l_all = n > 0 ? L.l[0] : 0.0;
    L.u_all = n > 0 ? L.u[0] : 0.0;
    // step size and primal weight seeds (include/pdlp_algo.hpp:70-77), on the
    // scaled form; a maximum does not depend on the order it is taken in
    std::vector<double> amax_t((size_t)th, 0.0);
    parallel_chunks(th, nnz, 1 << 16, [&](int64_t b, int64_t e, int t) {
        double a = 0.0;
        for (int64_t k = b; k < e; ++k) a = std::max(a, std::fabs(S.val[k]));
        amax_t[t] = a;
    });
    double amax = 0.0;
    for (double a : amax_t) amax = std::max(amax, a);
    L.eta0 = amax > 0 ? 1.0 / amax : 1.0;
    double cn = 0.0, bn = 0.0;
    for (int32_t j = 0; j < n; ++j) cn += S.c[j] * S.c[j];
    for (int32_t i = 0; i < m; ++i)
        if (std::isfinite(S.rL[i])) bn += S.rL[i] * S.rL[i];
    cn = std::sqrt(cn);
    bn = std::sqrt(bn);
    L.omega0 = (cn > 1e-10 && bn > 1e-10) ? cn / bn : 1.0;
    // KKT denominators of src/verify.cpp:39,56 (unscaled form)
    L.denom_p = 1.0 + std::max(finite_inf_norm(U.rL, m), finite_inf_norm(U.rU, m));
    L.denom_d = 1.0 + finite_inf_norm(U.c, n);
    L.obj_offset = U.obj_offset;
}

void schedule_records(const SellHost& S, int warps, int dense_unroll, int sub_seg, std::vector<int32_t>& seq,
                      std::vector<int32_t>& start) {
    const int64_t n = S.n_slices();
    if (warps < 1 || dense_unroll < 1 || sub_seg < 1) fail(B2_ERR_INVALID, "schedule: bad arguments");
    std::vector<int64_t> cost((size_t)n);
    for (int64_t r = 0; r < n; ++r) {
        const int64_t len = (int64_t)((uint32_t)S.slice[(size_t)(4 * r + 1)] & kLenMask);
        const bool dense = !S.aff.empty() && S.aff[(size_t)(2 * r)] >= 0;
        cost[(size_t)r] = dense ? (len + dense_unroll - 1) / dense_unroll + 2 : len + 4;
    }
    std::vector<int32_t> ord((size_t)n);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int32_t a, int32_t b) { return cost[(size_t)a] > cost[(size_t)b]; });
    using Load = std::pair<int64_t, int32_t>;
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
    for (int32_t w = 0; w < warps; ++w) heap.push({0, w});
    std::vector<int32_t> warp_of((size_t)n);
    for (int32_t r : ord) {
        const Load top = heap.top();
        heap.pop();
        warp_of[(size_t)r] = top.second;
        heap.push({top.first + cost[(size_t)r], top.second});
    }
    auto cls = [&](int32_t r) {
        const uint32_t w = (uint32_t)S.slice[(size_t)(4 * r + 3)];
        if (w == 0) return 0;
        const int q = (int)(w >> 24);
        if (q == 0) return 2;
        return q % sub_seg == 0 ? 1 : 0;
    };
    seq.resize((size_t)n);
    std::iota(seq.begin(), seq.end(), 0);
    std::stable_sort(seq.begin(), seq.end(), [&](int32_t a, int32_t b) {
        if (warp_of[(size_t)a] != warp_of[(size_t)b]) return warp_of[(size_t)a] < warp_of[(size_t)b];
        return cls(a) < cls(b);
    });
    start.assign((size_t)warps + 1, 0);
    for (int32_t r : seq) ++start[(size_t)warp_of[(size_t)r] + 1];
    for (int32_t w = 0; w < warps; ++w) start[(size_t)w + 1] += start[(size_t)w];
}

// FNV-1a over every array and scalar of a layout: two layouts with the same
// digest hand the device the same bytes.
uint64_t layout_digest(const Layout& L) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](const void* p, size_t bytes) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < bytes; ++i) h = (h ^ b[i]) * 1099511628211ull;
    };
    auto vec = [&](const auto& v) {
        const uint64_t len = v.size();
        mix(&len, sizeof(len));
        if (!v.empty()) mix(v.data(), v.size() * sizeof(v[0]));
    };
    auto sell = [&](const SellHost& S) {
        mix(&S.n_rows, sizeof(S.n_rows));
        mix(&S.n_cols, sizeof(S.n_cols));
        vec(S.slice); vec(S.col); vec(S.val32); vec(S.val64); vec(S.seg); vec(S.aff);
        mix(&S.padded, sizeof(S.padded));
        mix(&S.seg_slots, sizeof(S.seg_slots));
        mix(&S.seg_max, sizeof(S.seg_max));
    };
    mix(&L.m, sizeof(L.m));
    mix(&L.n, sizeof(L.n));
    mix(&L.nnz, sizeof(L.nnz));
    vec(L.perm_r); vec(L.perm_c); vec(L.inv_r); vec(L.inv_c);
    sell(L.A);
    sell(L.AT);
    const char e32 = L.exact32 ? 1 : 0, luc = L.lu_const ? 1 : 0;
    mix(&e32, 1);
    mix(&luc, 1);
    mix(&L.l_all, sizeof(double));
    mix(&L.u_all, sizeof(double));
    vec(L.b); vec(L.rU); vec(L.dr2); vec(L.c); vec(L.l); vec(L.u); vec(L.x0); vec(L.dc2);
    const double sc[5] = {L.eta0, L.omega0, L.denom_p, L.denom_d, L.obj_offset};
    mix(sc, sizeof(sc));
    return h;
}

// ----------------------------------------------------------------- scaling
namespace {

// Entry positions k grouped by key (rows or columns), each group in
// increasing k: the order in which the serial loop adds a group's entries.
void stable_groups(int64_t groups, int64_t nnz, const int32_t* key, int threads, std::vector<int64_t>& ptr,
                   std::vector<int64_t>& pos) {
    // a stable counting sort, as in coo_to_csr: contiguous entry runs counted
    // per group, turned into per-run offsets (earlier runs first), scattered
    ptr.assign(groups + 1, 0);
    pos.resize(nnz);
    const int nch = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(1, threads), nnz / (1 << 18)));
    const int64_t per = (nnz + nch - 1) / nch;
    std::vector<std::vector<int64_t>> cur((size_t)nch);
    auto runs = [&](auto&& body) {
        std::vector<std::thread> pool;
        for (int t = 1; t < nch; ++t) pool.emplace_back([&body, t] { body(t); });
        body(0);
        for (auto& th : pool) th.join();
    };
    runs([&](int t) {
        cur[t].assign((size_t)groups, 0);
        const int64_t b = std::min(nnz, t * per), e = std::min(nnz, b + per);
        for (int64_t k = b; k < e; ++k) cur[t][key[k]]++;
    });
    for (int64_t i = 0; i < groups; ++i) {
        int64_t off = ptr[i];
        for (int t = 0; t < nch; ++t) {
            const int64_t c = cur[t][i];
            cur[t][i] = off;
            off += c;
        }
        ptr[i + 1] = off;
    }
    runs([&](int t) {
        const int64_t b = std::min(nnz, t * per), e = std::min(nnz, b + per);
        int64_t* cu = cur[t].data();
        for (int64_t k = b; k < e; ++k) pos[cu[key[k]]++] = k;
    });
}

// The scaling of scale_lp on several threads, with the serial loops' bits:
// maxima and products do not depend on the order they are taken in, and the
// Pock-Chambolle sums add every row's (column's) entries in increasing k, as
// the serial loop does.
void scale_lp_parallel(const b2_lp_view& lp, int ruiz_passes, int th, double* val_s, double* Dr, double* Dc,
                       std::vector<double>& rs, std::vector<double>& cs) {
    const int32_t m = lp.m, n = lp.n;
    const int64_t nnz = lp.nnz;
    const int32_t* R = lp.row_idx;
    const int32_t* Cc = lp.col_idx;
    const int64_t grain = 1 << 16;
    std::vector<std::vector<double>> part((size_t)th);
    // per-thread maxima over contiguous entry runs, then the maximum of those
    auto group_max = [&](const int32_t* key, int64_t groups, std::vector<double>& out) {
        const int nch = parallel_chunks(th, nnz, grain, [&](int64_t b, int64_t e, int t) {
            std::vector<double>& p = part[t];
            p.assign((size_t)groups, 0.0);
            for (int64_t k = b; k < e; ++k) p[key[k]] = std::max(p[key[k]], std::fabs(val_s[k]));
        });
        parallel_chunks(th, groups, grain, [&](int64_t b, int64_t e, int) {
            for (int64_t i = b; i < e; ++i) {
                double v = 0.0;
                for (int t = 0; t < nch; ++t) v = std::max(v, part[t][i]);
                out[i] = v > 0 ? 1.0 / std::sqrt(v) : 1.0;
            }
        });
    };
    for (int pass = 0; pass < ruiz_passes; ++pass) {
        group_max(R, m, rs);
        parallel_chunks(th, nnz, grain, [&](int64_t b, int64_t e, int) {
            for (int64_t k = b; k < e; ++k) val_s[k] = val_s[k] * rs[R[k]];
        });
        for (int32_t i = 0; i < m; ++i) Dr[i] *= rs[i];
        group_max(Cc, n, cs);
        parallel_chunks(th, nnz, grain, [&](int64_t b, int64_t e, int) {
            for (int64_t k = b; k < e; ++k) val_s[k] = val_s[k] * cs[Cc[k]];
        });
        for (int32_t j = 0; j < n; ++j) Dc[j] *= cs[j];
    }
    std::vector<int64_t> ptr, pos;
    auto group_sum = [&](const int32_t* key, int64_t groups, std::vector<double>& out) {
        stable_groups(groups, nnz, key, th, ptr, pos);
        parallel_chunks(th, groups, grain / 16, [&](int64_t b, int64_t e, int) {
            for (int64_t i = b; i < e; ++i) {
                double v = 0.0;
                for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) v += std::fabs(val_s[pos[p]]);
                out[i] = std::sqrt(v > 0 ? 1.0 / v : 1.0);
            }
        });
    };
    group_sum(R, m, rs);
    group_sum(Cc, n, cs);
    parallel_chunks(th, nnz, grain, [&](int64_t b, int64_t e, int) {
        for (int64_t k = b; k < e; ++k) val_s[k] = val_s[k] * rs[R[k]] * cs[Cc[k]];
    });
}

}  // namespace

void scale_lp(const b2_lp_view& lp, int ruiz_passes, double* val_s, double* c_s, double* rL_s, double* rU_s,
              double* l_s, double* u_s, double* Dr, double* Dc, int threads) {
    const int32_t m = lp.m, n = lp.n;
    const int64_t nnz = lp.nnz;
    const int th = std::max(1, threads);
    if (first_bad(th, nnz, [&](int64_t k) {
            return lp.row_idx[k] < 0 || lp.row_idx[k] >= m || lp.col_idx[k] < 0 || lp.col_idx[k] >= n;
        }) >= 0)
        fail(B2_ERR_INVALID, "matrix index out of range");
    const int32_t* R = lp.row_idx;
    const int32_t* Cc = lp.col_idx;
    std::copy(lp.val, lp.val + nnz, val_s);
    if (th > 1 && nnz >= (1 << 18)) {
        std::fill(Dr, Dr + m, 1.0);
        std::fill(Dc, Dc + n, 1.0);
        std::vector<double> rs(m), cs(n);
        scale_lp_parallel(lp, ruiz_passes, th, val_s, Dr, Dc, rs, cs);
        for (int32_t i = 0; i < m; ++i) Dr[i] *= rs[i];
        for (int32_t j = 0; j < n; ++j) Dc[j] *= cs[j];
        for (int32_t j = 0; j < n; ++j) {
            c_s[j] = Dc[j] * lp.c[j];
            l_s[j] = lp.l[j] / Dc[j];
            u_s[j] = lp.u[j] / Dc[j];
        }
        for (int32_t i = 0; i < m; ++i) {
            rL_s[i] = Dr[i] * lp.rL[i];
            rU_s[i] = Dr[i] * lp.rU[i];
        }
        return;
    }
    std::fill(Dr, Dr + m, 1.0);
    std::fill(Dc, Dc + n, 1.0);
    std::vector<double> rs(m), cs(n);
    for (int pass = 0; pass < ruiz_passes; ++pass) {
        std::fill(rs.begin(), rs.end(), 0.0);
        for (int64_t k = 0; k < nnz; ++k) rs[R[k]] = std::max(rs[R[k]], std::fabs(val_s[k]));
        for (int32_t i = 0; i < m; ++i) rs[i] = rs[i] > 0 ? 1.0 / std::sqrt(rs[i]) : 1.0;
        for (int64_t k = 0; k < nnz; ++k) val_s[k] = val_s[k] * rs[R[k]];
        for (int32_t i = 0; i < m; ++i) Dr[i] *= rs[i];
        std::fill(cs.begin(), cs.end(), 0.0);
        for (int64_t k = 0; k < nnz; ++k) cs[Cc[k]] = std::max(cs[Cc[k]], std::fabs(val_s[k]));
        for (int32_t j = 0; j < n; ++j) cs[j] = cs[j] > 0 ? 1.0 / std::sqrt(cs[j]) : 1.0;
        for (int64_t k = 0; k < nnz; ++k) val_s[k] = val_s[k] * cs[Cc[k]];
        for (int32_t j = 0; j < n; ++j) Dc[j] *= cs[j];
    }
    std::fill(rs.begin(), rs.end(), 0.0);
    std::fill(cs.begin(), cs.end(), 0.0);
    for (int64_t k = 0; k < nnz; ++k) rs[R[k]] += std::fabs(val_s[k]);
    for (int64_t k = 0; k < nnz; ++k) cs[Cc[k]] += std::fabs(val_s[k]);
    for (int32_t i = 0; i < m; ++i) rs[i] = std::sqrt(rs[i] > 0 ? 1.0 / rs[i] : 1.0);
    for (int32_t j = 0; j < n; ++j) cs[j] = std::sqrt(cs[j] > 0 ? 1.0 / cs[j] : 1.0);
    for (int64_t k = 0; k < nnz; ++k) val_s[k] = val_s[k] * rs[R[k]] * cs[Cc[k]];
    for (int32_t i = 0; i < m; ++i) Dr[i] *= rs[i];
    for (int32_t j = 0; j < n; ++j) Dc[j] *= cs[j];
    for (int32_t j = 0; j < n; ++j) {
        c_s[j] = Dc[j] * lp.c[j];
        l_s[j] = lp.l[j] / Dc[j];
        u_s[j] = lp.u[j] / Dc[j];
    }
    for (int32_t i = 0; i < m; ++i) {
        rL_s[i] = Dr[i] * lp.rL[i];
        rU_s[i] = Dr[i] * lp.rU[i];
    }
}

// -------------------------------------------------------------- generators
namespace {

// xoshiro256** seeded through splitmix64 (Blackman & Vigna's published
// generators), so every benchmark input is reproducible from its seed.
struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t z = seed;
        for (auto& w : s) {
            z += 0x9E3779B97F4A7C15ull;
            uint64_t t = z;
            t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ull;
            t = (t ^ (t >> 27)) * 0x94D049BB133111EBull;
            w = t ^ (t >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }           // [0, 1)
    int64_t below(int64_t n) { return (int64_t)(uniform() * (double)n); }      // [0, n)
    double normal() {                                                         // Marsaglia polar
        for (;;) {
            double a = 2.0 * uniform() - 1.0, b = 2.0 * uniform() - 1.0, q = a * a + b * b;
            if (q > 0.0 && q < 1.0) return a * std::sqrt(-2.0 * std::log(q) / q);
        }
    }
};

}  // namespace

void gen_random_lp(int m, int n, int k, uint64_t seed, bool fp32_values, int32_t* row, int32_t* col, double* val,
                   double* c, double* rL, double* rU, double* l, double* u) {
    if (m <= 0 || n <= 0 || k <= 0 || k > m) fail(B2_ERR_INVALID, "bad generator sizes");
    Rng rng(seed);
    std::vector<int32_t> pick(k);
    for (int32_t j = 0; j < n; ++j) {
        for (int t = 0; t < k; ++t) {
            int32_t r;
            bool dup;
            do {
                r = (int32_t)rng.below(m);
                dup = false;
                for (int q = 0; q < t; ++q) dup |= pick[q] == r;
            } while (dup);
            pick[t] = r;
            double v;
            do {
                v = 2.0 * rng.uniform() - 1.0;
                if (fp32_values) v = (double)(float)v;
            } while (v == 0.0);
            const int64_t p = (int64_t)j * k + t;
            row[p] = r;
            col[p] = j;
            val[p] = v;
        }
    }
    std::vector<double> x0(n), y0(m);
    for (int32_t j = 0; j < n; ++j) x0[j] = 5.0 * rng.uniform();
    for (int32_t i = 0; i < m; ++i) y0[i] = rng.normal();
    std::fill(rL, rL + m, 0.0);
    for (int64_t p = 0; p < (int64_t)n * k; ++p) rL[row[p]] += val[p] * x0[col[p]];
    for (int32_t j = 0; j < n; ++j) {
        double s = 0.0;
        for (int t = 0; t < k; ++t) {
            const int64_t p = (int64_t)j * k + t;
            s += val[p] * y0[row[p]];
        }
        c[j] = s + rng.uniform();
        l[j] = 0.0;
        u[j] = 10.0;
    }
    std::copy(rL, rL + m, rU);
}

void gen_transport(int S, int D, uint64_t seed, int32_t* row, int32_t* col, double* val, double* c, double* rL,
                   double* rU, double* l, double* u) {
    if (S < 1 || D < 1) fail(B2_ERR_INVALID, "bad transport sizes");
    Rng rng(seed);
    std::vector<int64_t> supply(S), demand(D);
    int64_t total = 0;
    for (int i = 0; i < S; ++i) { supply[i] = 100 + rng.below(901); total += supply[i]; }
    std::vector<double> w(D);
    double wsum = 0.0;
    for (int j = 0; j < D; ++j) { w[j] = 0.5 + rng.uniform(); wsum += w[j]; }
    int64_t assigned = 0;
    for (int j = 0; j < D; ++j) {
        demand[j] = std::max<int64_t>(1, (int64_t)std::floor((double)total * w[j] / wsum));
        assigned += demand[j];
    }
    // integer partition: hand the remainder out one unit at a time, round robin
    for (int64_t r = total - assigned, j = 0; r != 0; j = (j + 1) % D) {
        if (r > 0) { demand[j]++; r--; }
        else if (demand[j] > 1) { demand[j]--; r++; }
    }
    const int64_t n = (int64_t)S * D;
    for (int i = 0; i < S; ++i)
        for (int j = 0; j < D; ++j) {
            const int64_t a = (int64_t)i * D + j;
            row[2 * a] = i;         col[2 * a] = (int32_t)a;     val[2 * a] = 1.0;
            row[2 * a + 1] = S + j; col[2 * a + 1] = (int32_t)a; val[2 * a + 1] = 1.0;
            c[a] = (double)(1 + rng.below(100));
            l[a] = 0.0;
            u[a] = kInf;
        }
    (void)n;
    for (int i = 0; i < S; ++i) rL[i] = rU[i] = (double)supply[i];
    for (int j = 0; j < D; ++j) rL[S + j] = rU[S + j] = (double)demand[j];
}

}  // namespace b2
