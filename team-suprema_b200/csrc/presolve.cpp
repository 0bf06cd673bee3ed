// presolve.cpp -- host-side preparation of an LP before the PDLP stage, run on
// the server's preparation threads for requests submitted as ranged LPs, and
// exposed through the C ABI (b2_presolve / b2_postsolve, b2_pdlp_form_*):
//
//   original ranged LP --presolve--> reduced LP --PDLP form--> equality rows
//   first, then A x >= b rows (what the engine solves)
//
// and back: PDLP-form point --extract--> reduced point --postsolve--> a point
// of the original LP, with the dual values (y) that verify() needs.
//
// The PDLP form is the reference's (build_pdlp_form / extract_solution,
// src/pdlp.cpp:8-90): equality rows first in input order, then the one-sided
// rows in input order with "<=" rows negated into ">=", a ranged row becomes
// an equality with a bounded slack column (value -1) appended after the
// original columns, free rows are dropped. Matching it entry for entry keeps
// a form built here interchangeable with one the reference built.
//
// The presolve is this engine's own, a small set of reductions whose
// postsolve is exact for both primal and dual values:
//   * free rows (both row bounds infinite) and empty rows are dropped (an
//     empty row whose bounds exclude 0 makes the LP infeasible);
//   * fixed columns (l == u) and empty columns are fixed at a value, their
//     entries moved into the row bounds and their cost into the offset (an
//     empty column whose cost pulls it to an infinite bound makes the LP
//     unbounded);
//   * singleton rows (one entry a x_j) become bounds on x_j.
// Reductions repeat until nothing changes. Postsolve undoes them in reverse
// order; for a singleton row the multiplier of x_j's active bound moves to
// the row when that bound came from the row, decided by the sign of x_j's
// reduced cost (as the reference's postsolve does, src/presolve.cpp:571-585).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "internal.h"

namespace b2 {

namespace {

constexpr double kInfP = std::numeric_limits<double>::infinity();

struct Step {
    enum Kind { DROP_ROW, FIX_COL, ROW_TO_BOUND } kind;
    int32_t i = -1, j = -1;
    double value = 0.0;            // FIX_COL: x_j
    double a = 0.0;                // ROW_TO_BOUND: the row's one coefficient
    bool lo_from_row = false;      // ROW_TO_BOUND: x_j's lower / upper bound came from the row
    bool hi_from_row = false;
};

}  // namespace

struct Presolved {
    // the original LP (kept for postsolve's reduced costs)
    int32_t m0 = 0, n0 = 0;
    std::vector<int32_t> row0, col0;
    std::vector<double> val0, c0;
    // the reduced LP, renumbered; row_ids / col_ids map reduced -> original
    std::vector<int32_t> row, col;
    std::vector<double> val, c, rL, rU, l, u;
    double obj_offset = 0.0;
    std::vector<int32_t> row_ids, col_ids;
    std::vector<Step> steps;
    int32_t status = 0;  // 0 reduced, 1 infeasible, 2 unbounded
};

struct PdlpForm {
    int32_t m_orig = 0, n_orig = 0, m = 0, n = 0;
    std::vector<int32_t> row, col;
    std::vector<double> val, c, rL, rU, l, u;
    double obj_offset = 0.0;
    std::vector<int32_t> row_perm;   // form row -> input row
    std::vector<double> row_sign;    // +1, or -1 for a negated "<=" row
};

namespace {

void check_view(const b2_lp_view& v) {
    if (v.m < 0 || v.n < 0 || v.nnz < 0) fail(B2_ERR_INVALID, "negative LP dimensions");
    for (int64_t k = 0; k < v.nnz; ++k) {
        if (v.row_idx[k] < 0 || v.row_idx[k] >= v.m || v.col_idx[k] < 0 || v.col_idx[k] >= v.n)
            fail(B2_ERR_INVALID, "matrix index out of range at entry " + std::to_string(k));
        if (!std::isfinite(v.val[k])) fail(B2_ERR_NONFINITE, "non-finite matrix value at entry " + std::to_string(k));
    }
    for (int32_t j = 0; j < v.n; ++j)
        if (!std::isfinite(v.c[j])) fail(B2_ERR_NONFINITE, "non-finite cost in column " + std::to_string(j));
}

}  // namespace

Presolved* presolve_lp(const b2_lp_view& v) {
    check_view(v);
    auto* P = new Presolved();
    Presolved& R = *P;
    const int32_t m = v.m, n = v.n;
    R.m0 = m;
    R.n0 = n;
    R.row0.assign(v.row_idx, v.row_idx + v.nnz);
    R.col0.assign(v.col_idx, v.col_idx + v.nnz);
    R.val0.assign(v.val, v.val + v.nnz);
    R.c0.assign(v.c, v.c + n);
    std::vector<double> rL(v.rL, v.rL + m), rU(v.rU, v.rU + m), l(v.l, v.l + n), u(v.u, v.u + n);
    double offset = v.obj_offset;
    // entry lists of every row and column (entry ids), with alive counts
    std::vector<int64_t> rp(m + 1, 0), cp(n + 1, 0);
    for (int64_t k = 0; k < v.nnz; ++k) { rp[v.row_idx[k] + 1]++; cp[v.col_idx[k] + 1]++; }
    for (int32_t i = 0; i < m; ++i) rp[i + 1] += rp[i];
    for (int32_t j = 0; j < n; ++j) cp[j + 1] += cp[j];
    std::vector<int64_t> re(v.nnz), ce(v.nnz);
    {
        std::vector<int64_t> a(rp.begin(), rp.end() - 1), b(cp.begin(), cp.end() - 1);
        for (int64_t k = 0; k < v.nnz; ++k) { re[a[v.row_idx[k]]++] = k; ce[b[v.col_idx[k]]++] = k; }
    }
    std::vector<char> row_alive(m, 1), col_alive(n, 1), ent_alive(v.nnz, 1);
    std::vector<int32_t> row_cnt(m), col_cnt(n);
    for (int32_t i = 0; i < m; ++i) row_cnt[i] = (int32_t)(rp[i + 1] - rp[i]);
    for (int32_t j = 0; j < n; ++j) col_cnt[j] = (int32_t)(cp[j + 1] - cp[j]);
    const double feas_tol = 1e-9;

    auto drop_row = [&](int32_t i) {
        row_alive[i] = 0;
        for (int64_t q = rp[i]; q < rp[i + 1]; ++q) {
            const int64_t k = re[q];
            if (!ent_alive[k]) continue;
            ent_alive[k] = 0;
            col_cnt[v.col_idx[k]]--;
        }
        row_cnt[i] = 0;
        Step s;
        s.kind = Step::DROP_ROW;
        s.i = i;
        R.steps.push_back(s);
    };
    auto fix_col = [&](int32_t j, double x) {
        col_alive[j] = 0;
        for (int64_t q = cp[j]; q < cp[j + 1]; ++q) {
            const int64_t k = ce[q];
            if (!ent_alive[k]) continue;
            ent_alive[k] = 0;
            const int32_t i = v.row_idx[k];
            row_cnt[i]--;
            rL[i] -= v.val[k] * x;
            rU[i] -= v.val[k] * x;
        }
        col_cnt[j] = 0;
        offset += v.c[j] * x;
        Step s;
        s.kind = Step::FIX_COL;
        s.j = j;
        s.value = x;
        R.steps.push_back(s);
    };

    bool changed = true;
    for (int pass = 0; changed && pass < 100 && R.status == 0; ++pass) {
        changed = false;
        for (int32_t i = 0; i < m && R.status == 0; ++i) {
            if (!row_alive[i]) continue;
            if (!std::isfinite(rL[i]) && !std::isfinite(rU[i])) { drop_row(i); changed = true; continue; }
            if (row_cnt[i] == 0) {
                if (rL[i] > feas_tol * (1 + std::fabs(rL[i])) || rU[i] < -feas_tol * (1 + std::fabs(rU[i]))) {
                    R.status = 1;
                    break;
                }
                drop_row(i);
                changed = true;
                continue;
            }
            if (row_cnt[i] == 1) {
                int64_t k = -1;
                for (int64_t q = rp[i]; q < rp[i + 1]; ++q)
                    if (ent_alive[re[q]]) { k = re[q]; break; }
                const int32_t j = v.col_idx[k];
                const double a = v.val[k];
                if (a == 0.0) {  // an explicit zero: the row is empty (checked next pass)
                    ent_alive[k] = 0;
                    row_cnt[i] = 0;
                    col_cnt[j]--;
                    changed = true;
                    continue;
                }
                double lo = a > 0 ? rL[i] / a : rU[i] / a;
                double hi = a > 0 ? rU[i] / a : rL[i] / a;
                if (!std::isfinite(a > 0 ? rL[i] : rU[i])) lo = -kInfP;
                if (!std::isfinite(a > 0 ? rU[i] : rL[i])) hi = kInfP;
                Step s;
                s.kind = Step::ROW_TO_BOUND;
                s.i = i;
                s.j = j;
                s.a = a;
                s.lo_from_row = std::isfinite(lo) && lo >= l[j];
                s.hi_from_row = std::isfinite(hi) && hi <= u[j];
                if (s.lo_from_row) l[j] = lo;
                if (s.hi_from_row) u[j] = hi;
                if (l[j] > u[j]) {
                    if (l[j] - u[j] > feas_tol * (1 + std::fabs(l[j]))) { R.status = 1; break; }
                    u[j] = l[j];
                }
                row_alive[i] = 0;
                ent_alive[k] = 0;
                row_cnt[i] = 0;
                col_cnt[j]--;
                R.steps.push_back(s);
                changed = true;
            }
        }
        for (int32_t j = 0; j < n && R.status == 0; ++j) {
            if (!col_alive[j]) continue;
            if (l[j] == u[j]) { fix_col(j, l[j]); changed = true; continue; }
            if (col_cnt[j] == 0) {
                const double cj = v.c[j];
                double x;
                if (cj > 0) x = l[j];
                else if (cj < 0) x = u[j];
                else x = std::min(std::max(0.0, l[j]), u[j]);
                if (!std::isfinite(x)) { R.status = 2; break; }
                fix_col(j, x);
                changed = true;
            }
        }
    }
    R.obj_offset = offset;
    if (R.status != 0) return P;
    // the reduced LP, renumbered in input order
    std::vector<int32_t> new_row(m, -1), new_col(n, -1);
    for (int32_t i = 0; i < m; ++i)
        if (row_alive[i]) { new_row[i] = (int32_t)R.row_ids.size(); R.row_ids.push_back(i); }
    for (int32_t j = 0; j < n; ++j)
        if (col_alive[j]) { new_col[j] = (int32_t)R.col_ids.size(); R.col_ids.push_back(j); }
    for (int64_t k = 0; k < v.nnz; ++k) {
        if (!ent_alive[k]) continue;
        R.row.push_back(new_row[v.row_idx[k]]);
        R.col.push_back(new_col[v.col_idx[k]]);
        R.val.push_back(v.val[k]);
    }
    for (int32_t i : R.row_ids) { R.rL.push_back(rL[i]); R.rU.push_back(rU[i]); }
    for (int32_t j : R.col_ids) { R.c.push_back(v.c[j]); R.l.push_back(l[j]); R.u.push_back(u[j]); }
    return P;
}

int32_t presolved_status(const Presolved& R) { return R.status; }
void presolved_free(Presolved* p) { delete p; }
void pdlp_form_free(PdlpForm* f) { delete f; }

void presolved_view(const Presolved& R, b2_lp_view& out) {
    out.m = (int32_t)R.row_ids.size();
    out.n = (int32_t)R.col_ids.size();
    out.nnz = (int64_t)R.val.size();
    out.row_idx = R.row.data();
    out.col_idx = R.col.data();
    out.val = R.val.data();
    out.c = R.c.data();
    out.rL = R.rL.data();
    out.rU = R.rU.data();
    out.l = R.l.data();
    out.u = R.u.data();
    out.obj_offset = R.obj_offset;
}

void postsolve_lp(const Presolved& R, const double* x_red, const double* y_red, double* x, double* y) {
    std::fill(x, x + R.n0, 0.0);
    std::fill(y, y + R.m0, 0.0);
    for (size_t t = 0; t < R.col_ids.size(); ++t) x[R.col_ids[t]] = x_red[t];
    for (size_t t = 0; t < R.row_ids.size(); ++t) y[R.row_ids[t]] = y_red[t];
    if (R.steps.empty()) return;
    // column entry lists of the original matrix, for reduced costs
    std::vector<int64_t> cp(R.n0 + 1, 0);
    for (int32_t j : R.col0) cp[j + 1]++;
    for (int32_t j = 0; j < R.n0; ++j) cp[j + 1] += cp[j];
    std::vector<int64_t> ce(R.col0.size());
    {
        std::vector<int64_t> a(cp.begin(), cp.end() - 1);
        for (size_t k = 0; k < R.col0.size(); ++k) ce[a[R.col0[k]]++] = (int64_t)k;
    }
    // rows removed before a step are not yet restored when that step is undone:
    // their y is still 0, so z_j below sums exactly the rows alive at the step
    for (size_t s = R.steps.size(); s-- > 0;) {
        const Step& st = R.steps[s];
        if (st.kind == Step::FIX_COL) {
            x[st.j] = st.value;
        } else if (st.kind == Step::ROW_TO_BOUND) {
            double z = R.c0[st.j];
            for (int64_t q = cp[st.j]; q < cp[st.j + 1]; ++q) {
                const int64_t k = ce[q];
                if (R.row0[k] != st.i) z -= R.val0[k] * y[R.row0[k]];
            }
            // z > 0: x_j rests on its lower bound; z < 0: on its upper bound
            if ((z > 0 && st.lo_from_row) || (z < 0 && st.hi_from_row)) y[st.i] = z / st.a;
        }
        // DROP_ROW: y_i stays 0
    }
}

// ---------------------------------------------------------------- PDLP form
PdlpForm* pdlp_form_build(const b2_lp_view& v) {
    check_view(v);
    auto* F = new PdlpForm();
    const int32_t m = v.m, n = v.n;
    F->m_orig = m;
    F->n_orig = n;
    // row order: equalities and ranged rows first, then one-sided rows, each in input order
    std::vector<int32_t> slack_of(m, -1);
    std::vector<int32_t> one_sided;
    std::vector<double> slack_lo, slack_hi;
    std::vector<double> rhs_eq, rhs_in;
    for (int32_t i = 0; i < m; ++i) {
        const double lo = v.rL[i], hi = v.rU[i];
        const bool flo = std::isfinite(lo), fhi = std::isfinite(hi);
        if (lo == hi || (flo && fhi)) {
            if (lo != hi) {
                slack_of[i] = (int32_t)slack_lo.size();
                slack_lo.push_back(lo);
                slack_hi.push_back(hi);
            }
            F->row_perm.push_back(i);
            F->row_sign.push_back(1.0);
            rhs_eq.push_back(lo == hi ? lo : 0.0);
        } else if (fhi || flo) {
            one_sided.push_back(i);
        }
    }
    const int32_t n_eq = (int32_t)F->row_perm.size();
    for (int32_t i : one_sided) {
        const bool upper = std::isfinite(v.rU[i]);
        F->row_perm.push_back(i);
        F->row_sign.push_back(upper ? -1.0 : 1.0);
        rhs_in.push_back(upper ? -v.rU[i] : v.rL[i]);
    }
    F->m = (int32_t)F->row_perm.size();
    F->n = n + (int32_t)slack_lo.size();
    std::vector<int32_t> pos(m, -1);
    for (int32_t p = 0; p < F->m; ++p) pos[F->row_perm[p]] = p;
    F->row.reserve(v.nnz + slack_lo.size());
    for (int64_t k = 0; k < v.nnz; ++k) {
        const int32_t p = pos[v.row_idx[k]];
        if (p < 0) continue;  // free row
        F->row.push_back(p);
        F->col.push_back(v.col_idx[k]);
        F->val.push_back(F->row_sign[p] * v.val[k]);
    }
    for (int32_t p = 0; p < n_eq; ++p) {
        const int32_t s = slack_of[F->row_perm[p]];
        if (s < 0) continue;
        F->row.push_back(p);
        F->col.push_back(n + s);
        F->val.push_back(-1.0);
    }
    F->rL = rhs_eq;
    F->rL.insert(F->rL.end(), rhs_in.begin(), rhs_in.end());
    F->rU = rhs_eq;
    F->rU.resize(F->m, kInfP);
    F->c.assign(v.c, v.c + n);
    F->c.resize(F->n, 0.0);
    F->l.assign(v.l, v.l + n);
    F->u.assign(v.u, v.u + n);
    F->l.insert(F->l.end(), slack_lo.begin(), slack_lo.end());
    F->u.insert(F->u.end(), slack_hi.begin(), slack_hi.end());
    F->obj_offset = v.obj_offset;
    return F;
}

void pdlp_form_view(const PdlpForm& F, b2_lp_view& out) {
    out.m = F.m;
    out.n = F.n;
    out.nnz = (int64_t)F.val.size();
    out.row_idx = F.row.data();
    out.col_idx = F.col.data();
    out.val = F.val.data();
    out.c = F.c.data();
    out.rL = F.rL.data();
    out.rU = F.rU.data();
    out.l = F.l.data();
    out.u = F.u.data();
    out.obj_offset = F.obj_offset;
}

void pdlp_form_extract(const PdlpForm& F, const double* x2, const double* y2, double* x, double* y) {
    std::copy(x2, x2 + F.n_orig, x);
    std::fill(y, y + F.m_orig, 0.0);
    for (int32_t p = 0; p < F.m; ++p) y[F.row_perm[p]] = F.row_sign[p] * y2[p];
}

// verify()'s KKT figures (src/verify.cpp:24-103) of a point of a ranged LP,
// on the host: out = {eps_P, eps_D, eps_G, objective}. Used to certify
// answers mapped back to the caller's LP after postsolve.
void kkt_host(const b2_lp_view& v, const double* x, const double* y, double* out) {
    std::vector<double> ax(v.m, 0.0), z(v.c, v.c + v.n);
    for (int64_t k = 0; k < v.nnz; ++k) {
        ax[v.row_idx[k]] += v.val[k] * x[v.col_idx[k]];
        z[v.col_idx[k]] -= v.val[k] * y[v.row_idx[k]];
    }
    auto finite_max = [](const double* a, int32_t len) {
        double mx = 0.0;
        for (int32_t i = 0; i < len; ++i)
            if (std::isfinite(a[i])) mx = std::max(mx, std::fabs(a[i]));
        return mx;
    };
    double p2 = 0.0, d2 = 0.0, D = 0.0, cx = 0.0;
    for (int32_t i = 0; i < v.m; ++i) {
        const double rl = v.rL[i], ru = v.rU[i], a = ax[i];
        const double rv = std::max(rl - a, 0.0) + std::max(a - ru, 0.0);
        p2 += rv * rv;
        double yv = y[i], sv = 0.0;
        if (!std::isfinite(rl) && yv > 0) { sv += yv; yv = 0.0; }
        if (!std::isfinite(ru) && yv < 0) { sv += -yv; yv = 0.0; }
        d2 += sv * sv;
        if (yv > 0) D += rl * yv;
        if (yv < 0) D += ru * yv;
    }
    for (int32_t j = 0; j < v.n; ++j) {
        const double lj = v.l[j], uj = v.u[j], xj = x[j];
        const double bv = std::max(lj - xj, 0.0) + std::max(xj - uj, 0.0);
        p2 += bv * bv;
        double zv = z[j], sv = 0.0;
        if (!std::isfinite(lj) && zv > 0) { sv += zv; zv = 0.0; }
        if (!std::isfinite(uj) && zv < 0) { sv += -zv; zv = 0.0; }
        d2 += sv * sv;
        if (zv > 0) D += lj * zv;
        if (zv < 0) D += uj * zv;
        cx += v.c[j] * xj;
    }
    const double denom_p = 1.0 + std::max(finite_max(v.rL, v.m), finite_max(v.rU, v.m));
    const double denom_d = 1.0 + finite_max(v.c, v.n);
    out[0] = std::sqrt(p2) / denom_p;
    out[1] = std::sqrt(d2) / denom_d;
    out[2] = std::fabs(cx - D) / (1.0 + std::fabs(cx) + std::fabs(D));
    out[3] = cx + v.obj_offset;
}

}  // namespace b2
