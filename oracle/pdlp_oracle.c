/* pdlp_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Serial FP64 restatement of the reference solver's PDLP path in plain C, so
 * the GPU engine can be checked against the reference algorithm on any host
 * (including one without the reference tree). It is itself pinned against the
 * reference library built from source (oracle/_ref/libsovref.so) by
 * tests/test_oracle.py on the reference's own fixtures.
 *
 * Restated, with the reference locations:
 *   or_coo_to_csr  include/sparse.hpp:24-50      (to_csr, to_csc_as_transposed_csr)
 *   or_matvec      include/sparse.hpp:52-59      (matvec)
 *   or_verify      src/verify.cpp:6-103          (verify, finite_inf_norm, vec_norm2)
 *   or_scale       src/scaling.cpp:4-84          (scale, LP case)
 *   or_pdlp_run    include/pdlp_algo.hpp:49-185 with the CPU backend of src/pdlp.cpp:97-142
 * plus the benchmark LP generators (or_gen_random_lp, or_gen_transport), which
 * restate this project's own generators, not the reference's.
 */
#include "pdlp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_INF (1.0 / 0.0)

void or_coo_to_csr(int rows, int cols, int64_t nnz, const int32_t* row, const int32_t* col, const double* val,
                   int transpose, int32_t* indptr, int32_t* indices, double* data) {
    /* sparse.hpp:24-40: count, prefix sum, then a stable scatter in COO order. */
    int nr = transpose ? cols : rows;
    const int32_t* r = transpose ? col : row;
    const int32_t* c = transpose ? row : col;
    memset(indptr, 0, sizeof(int32_t) * (size_t)(nr + 1));
    for (int64_t k = 0; k < nnz; ++k) indptr[r[k] + 1]++;
    for (int i = 0; i < nr; ++i) indptr[i + 1] += indptr[i];
    int32_t* cursor = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nr > 0 ? nr : 1));
    memcpy(cursor, indptr, sizeof(int32_t) * (size_t)nr);
    for (int64_t k = 0; k < nnz; ++k) {
        int32_t pos = cursor[r[k]]++;
        indices[pos] = c[k];
        data[pos] = val[k];
    }
    free(cursor);
}

void or_matvec(int rows, const int32_t* indptr, const int32_t* indices, const double* data, const double* x,
               double* y) {
    for (int i = 0; i < rows; ++i) {
        double s = 0.0;
        for (int32_t p = indptr[i]; p < indptr[i + 1]; ++p) s += data[p] * x[indices[p]];
        y[i] = s;
    }
}

static double finite_inf_norm(const double* v, int len) {
    /* verify.cpp:6-10 */
    double m = 0.0;
    int any = 0;
    for (int i = 0; i < len; ++i)
        if (isfinite(v[i])) { m = fmax(m, fabs(v[i])); any = 1; }
    return any ? m : 0.0;
}

void or_verify(int m, int n, const int32_t* a_ptr, const int32_t* a_idx, const double* a_val,
               const int32_t* at_ptr, const int32_t* at_idx, const double* at_val, const double* c,
               const double* rL, const double* rU, const double* l, const double* u, double obj_offset,
               const double* x, const double* y, double* out) {
    double* a = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    double* aty = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    or_matvec(m, a_ptr, a_idx, a_val, x, a);
    or_matvec(n, at_ptr, at_idx, at_val, y, aty);

    /* eps_P, verify.cpp:35-40 */
    double s = 0.0, max_row = 0.0, max_bnd = 0.0;
    for (int i = 0; i < m; ++i) {
        double v = fmax(rL[i] - a[i], 0.0) + fmax(a[i] - rU[i], 0.0);
        s += v * v;
        if (i == 0 || v > max_row) max_row = v;
    }
    for (int j = 0; j < n; ++j) {
        double v = fmax(l[j] - x[j], 0.0) + fmax(x[j] - u[j], 0.0);
        s += v * v;
        if (j == 0 || v > max_bnd) max_bnd = v;
    }
    double denom_p = 1.0 + fmax(finite_inf_norm(rL, m), finite_inf_norm(rU, m));
    double eps_P = sqrt(s) / denom_p;

    /* eps_D, verify.cpp:42-57 */
    s = 0.0;
    for (int i = 0; i < m; ++i) {
        double v = 0.0;
        if (!isfinite(rL[i]) && y[i] > 0) v += y[i];
        if (!isfinite(rU[i]) && y[i] < 0) v += -y[i];
        s += v * v;
    }
    for (int j = 0; j < n; ++j) {
        double z = c[j] - aty[j], v = 0.0;
        if (!isfinite(l[j]) && z > 0) v += z;
        if (!isfinite(u[j]) && z < 0) v += -z;
        s += v * v;
    }
    double eps_D = sqrt(s) / (1.0 + finite_inf_norm(c, n));

    /* dual objective, verify.cpp:59-87 */
    double D = 0.0;
    for (int i = 0; i < m; ++i) {
        double yv = y[i];
        if (!isfinite(rL[i]) && yv > 0) yv = 0.0;
        if (!isfinite(rU[i]) && yv < 0) yv = 0.0;
        double yp = fmax(yv, 0.0), yn = fmax(-yv, 0.0);
        if (yp > 0 && isfinite(rL[i])) D += rL[i] * yp;
        if (yn > 0 && isfinite(rU[i])) D += -rU[i] * yn;
        if (yp > 0 && !isfinite(rL[i])) D = -OR_INF;
        if (yn > 0 && !isfinite(rU[i])) D = -OR_INF;
    }
    for (int j = 0; j < n; ++j) {
        double zv = c[j] - aty[j];
        if (!isfinite(l[j]) && zv > 0) zv = 0.0;
        if (!isfinite(u[j]) && zv < 0) zv = 0.0;
        double zp = fmax(zv, 0.0), zn = fmax(-zv, 0.0);
        if (zp > 0 && isfinite(l[j])) D += l[j] * zp;
        if (zn > 0 && isfinite(u[j])) D += -u[j] * zn;
        if (zp > 0 && !isfinite(l[j])) D = -OR_INF;
        if (zn > 0 && !isfinite(u[j])) D = -OR_INF;
    }
    double cx = 0.0;
    for (int j = 0; j < n; ++j) cx += c[j] * x[j];
    double eps_G = isfinite(D) ? fabs(cx - D) / (1.0 + fabs(cx) + fabs(D)) : OR_INF;

    out[0] = eps_P; out[1] = eps_D; out[2] = eps_G;
    out[3] = cx + obj_offset;
    out[4] = isfinite(D) ? D + obj_offset : D;
    out[5] = m > 0 ? max_row : 0.0;
    out[6] = n > 0 ? max_bnd : 0.0;
    free(a);
    free(aty);
}

void or_scale(int m, int n, int64_t nnz, const int32_t* row, const int32_t* col, const double* val,
              const double* c, const double* rL, const double* rU, const double* l, const double* u,
              int ruiz_passes, double* val_s, double* c_s, double* rL_s, double* rU_s, double* l_s,
              double* u_s, double* Dr, double* Dc) {
    double* rs = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    double* cs = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    memcpy(val_s, val, sizeof(double) * (size_t)nnz);
    for (int i = 0; i < m; ++i) Dr[i] = 1.0;
    for (int j = 0; j < n; ++j) Dc[j] = 1.0;
    /* Ruiz: rows then columns (scaling.cpp:35-54) */
    for (int pass = 0; pass < ruiz_passes; ++pass) {
        for (int i = 0; i < m; ++i) rs[i] = 0.0;
        for (int64_t k = 0; k < nnz; ++k) rs[row[k]] = fmax(rs[row[k]], fabs(val_s[k]));
        for (int i = 0; i < m; ++i) rs[i] = rs[i] > 0 ? 1.0 / sqrt(rs[i]) : 1.0;
        for (int64_t k = 0; k < nnz; ++k) val_s[k] = val_s[k] * rs[row[k]] * 1.0;
        for (int i = 0; i < m; ++i) Dr[i] *= rs[i];
        for (int j = 0; j < n; ++j) cs[j] = 0.0;
        for (int64_t k = 0; k < nnz; ++k) cs[col[k]] = fmax(cs[col[k]], fabs(val_s[k]));
        for (int j = 0; j < n; ++j) cs[j] = cs[j] > 0 ? 1.0 / sqrt(cs[j]) : 1.0;
        for (int64_t k = 0; k < nnz; ++k) val_s[k] = val_s[k] * 1.0 * cs[col[k]];
        for (int j = 0; j < n; ++j) Dc[j] *= cs[j];
    }
    /* Pock-Chambolle alpha = 1 (scaling.cpp:56-66) */
    for (int i = 0; i < m; ++i) rs[i] = 0.0;
    for (int j = 0; j < n; ++j) cs[j] = 0.0;
    for (int64_t k = 0; k < nnz; ++k) rs[row[k]] += fabs(val_s[k]);
    for (int64_t k = 0; k < nnz; ++k) cs[col[k]] += fabs(val_s[k]);
    for (int i = 0; i < m; ++i) rs[i] = sqrt(rs[i] > 0 ? 1.0 / rs[i] : 1.0);
    for (int j = 0; j < n; ++j) cs[j] = sqrt(cs[j] > 0 ? 1.0 / cs[j] : 1.0);
    for (int64_t k = 0; k < nnz; ++k) val_s[k] = val_s[k] * rs[row[k]] * cs[col[k]];
    for (int i = 0; i < m; ++i) Dr[i] *= rs[i];
    for (int j = 0; j < n; ++j) Dc[j] *= cs[j];
    /* bounds and cost (scaling.cpp:68-82) */
    for (int j = 0; j < n; ++j) { c_s[j] = Dc[j] * c[j]; l_s[j] = l[j] / Dc[j]; u_s[j] = u[j] / Dc[j]; }
    for (int i = 0; i < m; ++i) { rL_s[i] = Dr[i] * rL[i]; rU_s[i] = Dr[i] * rU[i]; }
    free(rs);
    free(cs);
}

/* ------------------------------------------------------------------ PDLP -- */

typedef struct {
    int rows;
    int32_t *ptr, *idx;
    double* val;
} csr_t;

static csr_t make_csr(const or_lp* p, int transpose) {
    csr_t M;
    M.rows = transpose ? p->n : p->m;
    M.ptr = (int32_t*)malloc(sizeof(int32_t) * (size_t)(M.rows + 1));
    M.idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)(p->nnz > 0 ? p->nnz : 1));
    M.val = (double*)malloc(sizeof(double) * (size_t)(p->nnz > 0 ? p->nnz : 1));
    or_coo_to_csr(p->m, p->n, p->nnz, p->row, p->col, p->val, transpose, M.ptr, M.idx, M.val);
    return M;
}

static void free_csr(csr_t* M) { free(M->ptr); free(M->idx); free(M->val); }

static double* vzalloc(int len) { return (double*)calloc((size_t)(len > 0 ? len : 1), sizeof(double)); }

typedef struct { double eps_P, eps_D, eps_G; } kkt_t;

static double merit(kkt_t r) { return sqrt(r.eps_P * r.eps_P + r.eps_D * r.eps_D + r.eps_G * r.eps_G); }

/* pdlp_algo.hpp:58-64: map to unscaled space and verify there. */
static kkt_t unscaled_kkt(const or_lp* U, const csr_t* Au, const csr_t* AuT, const double* Dr, const double* Dc,
                          const double* xs, const double* ys, double* xu, double* yu) {
    for (int j = 0; j < U->n; ++j) xu[j] = Dc[j] * xs[j];
    for (int i = 0; i < U->m; ++i) yu[i] = Dr[i] * ys[i];
    double out[7];
    or_verify(U->m, U->n, Au->ptr, Au->idx, Au->val, AuT->ptr, AuT->idx, AuT->val, U->c, U->rL, U->rU, U->l,
              U->u, U->obj_offset, xu, yu, out);
    kkt_t k = {out[0], out[1], out[2]};
    return k;
}

int or_pdlp_run(const or_lp* U, const or_lp* S, const double* Dr, const double* Dc, int max_iterations,
                int check_every, double tol, double* x_out, double* y_out, int* info, double* eps_out,
                double* trace, int trace_len) {
    const int n = S->n, m = S->m;
    csr_t Au = make_csr(U, 0), AuT = make_csr(U, 1);
    csr_t A = make_csr(S, 0), AT = make_csr(S, 1); /* CpuBackend ctor, src/pdlp.cpp:104-108 */
    char* is_ineq = (char*)malloc((size_t)(m > 0 ? m : 1));
    for (int i = 0; i < m; ++i) is_ineq[i] = S->rL[i] != S->rU[i];
    const double* b = S->rL;

    /* initial point, step size, primal weight (pdlp_algo.hpp:67-77) */
    double *x = vzalloc(n), *y = vzalloc(m), *xn = vzalloc(n), *yn = vzalloc(m);
    double *ax = vzalloc(m), *axn = vzalloc(m), *aty = vzalloc(n);
    double *xsum = vzalloc(n), *ysum = vzalloc(m);
    double *hxs = vzalloc(n), *hys = vzalloc(m), *xu = vzalloc(n), *yu = vzalloc(m), *xu2 = vzalloc(n),
           *yu2 = vzalloc(m);
    double *x_last = vzalloc(n), *y_last = vzalloc(m), *best_x = vzalloc(n), *best_y = vzalloc(m);
    for (int j = 0; j < n; ++j) x[j] = fmin(fmax(0.0, S->l[j]), S->u[j]);
    double amax = 0.0;
    for (int64_t k = 0; k < S->nnz; ++k) amax = fmax(amax, fabs(S->val[k]));
    double eta = amax > 0 ? 1.0 / amax : 1.0;
    double cn = 0.0, bn = 0.0;
    for (int j = 0; j < n; ++j) cn += S->c[j] * S->c[j];
    for (int i = 0; i < m; ++i)
        if (isfinite(S->rL[i])) bn += S->rL[i] * S->rL[i];
    cn = sqrt(cn);
    bn = sqrt(bn);
    double omega = (cn > 1e-10 && bn > 1e-10) ? cn / bn : 1.0;

    or_matvec(m, A.ptr, A.idx, A.val, x, ax);
    or_matvec(n, AT.ptr, AT.idx, AT.val, y, aty);
    double wsum = 0.0;
    memcpy(x_last, x, sizeof(double) * (size_t)n);
    double merit_last_restart = OR_INF, merit_prev_cand = OR_INF;
    int since_restart = 0, restarts = 0, accepted = 0, attempts = 0;
    double best_merit = OR_INF;
    kkt_t best_k = {0, 0, 0};
    int converged = 0;

    while (attempts < max_iterations) {
        /* one PDHG step with adaptive step size (pdlp_algo.hpp:106-131) */
        while (attempts < max_iterations) {
            ++attempts;
            const double tau = eta / omega, sigma = eta * omega;
            for (int j = 0; j < n; ++j) xn[j] = fmin(fmax(x[j] - tau * (S->c[j] - aty[j]), S->l[j]), S->u[j]);
            or_matvec(m, A.ptr, A.idx, A.val, xn, axn);
            for (int i = 0; i < m; ++i) {
                double v = y[i] + sigma * (b[i] - (2.0 * axn[i] - ax[i]));
                yn[i] = (is_ineq[i] && v < 0.0) ? 0.0 : v;
            }
            double dx2 = 0.0, dy2 = 0.0, inter = 0.0;
            for (int j = 0; j < n; ++j) { double d = xn[j] - x[j]; dx2 += d * d; }
            for (int i = 0; i < m; ++i) { double d = yn[i] - y[i]; dy2 += d * d; inter += d * (axn[i] - ax[i]); }
            const double num = omega * dx2 + dy2 / omega;
            const double eta_bar = fabs(inter) > 0 ? num / (2.0 * fabs(inter)) : OR_INF;
            const double k1 = accepted + 2.0;
            const double grow = (1.0 + pow(k1, -0.6)) * eta;
            const double eta_next = isfinite(eta_bar) ? fmin((1.0 - pow(k1, -0.3)) * eta_bar, grow) : grow;
            const int acc = eta <= eta_bar;
            if (trace && attempts - 1 < trace_len) trace[attempts - 1] = acc ? eta : -eta;
            if (acc) {
                double* t;
                t = x; x = xn; xn = t;
                t = y; y = yn; yn = t;
                t = ax; ax = axn; axn = t;
                or_matvec(n, AT.ptr, AT.idx, AT.val, y, aty);
                for (int j = 0; j < n; ++j) xsum[j] += eta * x[j];
                for (int i = 0; i < m; ++i) ysum[i] += eta * y[i];
                wsum += eta;
                eta = eta_next;
                ++accepted;
                ++since_restart;
                break;
            }
            eta = eta_next;
        }

        if (accepted % check_every != 0 && attempts < max_iterations) continue;

        /* KKT check, current vs average (pdlp_algo.hpp:135-153) */
        if (wsum > 0) {
            for (int j = 0; j < n; ++j) hxs[j] = xsum[j] / wsum;
            for (int i = 0; i < m; ++i) hys[i] = ysum[i] / wsum;
        } else {
            memcpy(hxs, x, sizeof(double) * (size_t)n);
            memcpy(hys, y, sizeof(double) * (size_t)m);
        }
        kkt_t rc = unscaled_kkt(U, &Au, &AuT, Dr, Dc, x, y, xu, yu);
        kkt_t ra = unscaled_kkt(U, &Au, &AuT, Dr, Dc, hxs, hys, xu2, yu2);
        if (merit(rc) < best_merit) {
            best_merit = merit(rc); best_k = rc;
            memcpy(best_x, xu, sizeof(double) * (size_t)n); memcpy(best_y, yu, sizeof(double) * (size_t)m);
        }
        if (merit(ra) < best_merit) {
            best_merit = merit(ra); best_k = ra;
            memcpy(best_x, xu2, sizeof(double) * (size_t)n); memcpy(best_y, yu2, sizeof(double) * (size_t)m);
        }
        const int use_avg = merit(ra) < merit(rc);
        const kkt_t rep = use_avg ? ra : rc;
        const double mc = merit(rep);
        if (fmax(rep.eps_P, fmax(rep.eps_D, rep.eps_G)) <= tol) {
            memcpy(x_out, use_avg ? xu2 : xu, sizeof(double) * (size_t)n);
            memcpy(y_out, use_avg ? yu2 : yu, sizeof(double) * (size_t)m);
            eps_out[0] = rep.eps_P; eps_out[1] = rep.eps_D; eps_out[2] = rep.eps_G;
            converged = 1;
            break;
        }
        /* restart decision (pdlp_algo.hpp:155-174) */
        const int sufficient = mc <= 0.2 * merit_last_restart;
        const int necessary = mc <= 0.8 * merit_last_restart && mc > merit_prev_cand;
        const int artificial = since_restart >= 0.36 * accepted;
        merit_prev_cand = mc;
        if (sufficient || necessary || artificial) {
            const double* cx = use_avg ? hxs : x;
            const double* cy = use_avg ? hys : y;
            double ddx = 0.0, ddy = 0.0;
            for (int j = 0; j < n; ++j) ddx += (cx[j] - x_last[j]) * (cx[j] - x_last[j]);
            for (int i = 0; i < m; ++i) ddy += (cy[i] - y_last[i]) * (cy[i] - y_last[i]);
            ddx = sqrt(ddx);
            ddy = sqrt(ddy);
            if (ddx > 1e-10 && ddy > 1e-10) omega = exp(0.5 * log(ddy / ddx) + 0.5 * log(omega));
            memcpy(x_last, cx, sizeof(double) * (size_t)n);
            memcpy(y_last, cy, sizeof(double) * (size_t)m);
            if (use_avg) {
                memcpy(x, hxs, sizeof(double) * (size_t)n);
                memcpy(y, hys, sizeof(double) * (size_t)m);
                or_matvec(m, A.ptr, A.idx, A.val, x, ax);
                or_matvec(n, AT.ptr, AT.idx, AT.val, y, aty);
            }
            memset(xsum, 0, sizeof(double) * (size_t)n);
            memset(ysum, 0, sizeof(double) * (size_t)m);
            wsum = 0.0;
            since_restart = 0;
            ++restarts;
            merit_last_restart = mc;
            merit_prev_cand = OR_INF;
        }
    }

    if (!converged) {
        /* best-point fallback (pdlp_algo.hpp:177-184) */
        if (!isfinite(best_merit)) {
            kkt_t r = unscaled_kkt(U, &Au, &AuT, Dr, Dc, x, y, xu, yu);
            if (merit(r) < best_merit) {
                best_merit = merit(r); best_k = r;
                memcpy(best_x, xu, sizeof(double) * (size_t)n); memcpy(best_y, yu, sizeof(double) * (size_t)m);
            }
        }
        memcpy(x_out, best_x, sizeof(double) * (size_t)n);
        memcpy(y_out, best_y, sizeof(double) * (size_t)m);
        eps_out[0] = best_k.eps_P; eps_out[1] = best_k.eps_D; eps_out[2] = best_k.eps_G;
    }
    info[0] = attempts; info[1] = restarts; info[2] = converged; info[3] = accepted;

    free(x); free(y); free(xn); free(yn); free(ax); free(axn); free(aty); free(xsum); free(ysum);
    free(hxs); free(hys); free(xu); free(yu); free(xu2); free(yu2); free(x_last); free(y_last);
    free(best_x); free(best_y); free(is_ineq);
    free_csr(&Au); free_csr(&AuT); free_csr(&A); free_csr(&AT);
    return 0;
}

/* ------------------------------------------------------------ generators
 * The benchmark LPs are defined by this project's own seeded generators (the
 * reference's tools/gen_lp.cpp draws different supplies, so they are not the
 * reference's). These are independent C restatements of the product's
 * generators (team-suprema_b200/csrc/host_prep.cpp, gen_random_lp and
 * gen_transport), so that the reference arm of the benchmark and the golden
 * records can build the same LPs without loading the product library. A test
 * pins the two to the same content digest. The random source is xoshiro256**
 * seeded through splitmix64 (Blackman and Vigna's published generators). */
typedef struct { uint64_t s[4]; } or_rng;

static uint64_t or_rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static void or_rng_seed(or_rng* g, uint64_t seed) {
    uint64_t z = seed;
    for (int i = 0; i < 4; ++i) {
        z += 0x9E3779B97F4A7C15ull;
        uint64_t t = z;
        t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ull;
        t = (t ^ (t >> 27)) * 0x94D049BB133111EBull;
        g->s[i] = t ^ (t >> 31);
    }
}

static uint64_t or_rng_next(or_rng* g) {
    uint64_t* s = g->s;
    const uint64_t r = or_rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = or_rotl(s[3], 45);
    return r;
}

static double or_uniform(or_rng* g) { return (double)(or_rng_next(g) >> 11) * 0x1.0p-53; }
static int64_t or_below(or_rng* g, int64_t n) { return (int64_t)(or_uniform(g) * (double)n); }

static double or_normal(or_rng* g) {
    /* Marsaglia's polar method */
    for (;;) {
        double a = 2.0 * or_uniform(g) - 1.0, b = 2.0 * or_uniform(g) - 1.0, q = a * a + b * b;
        if (q > 0.0 && q < 1.0) return a * sqrt(-2.0 * log(q) / q);
    }
}

int or_gen_random_lp(int m, int n, int k, uint64_t seed, int fp32_values, int32_t* row, int32_t* col, double* val,
                     double* c, double* rL, double* rU, double* l, double* u) {
    if (m <= 0 || n <= 0 || k <= 0 || k > m) return 1;
    or_rng g;
    or_rng_seed(&g, seed);
    int32_t* pick = (int32_t*)malloc(sizeof(int32_t) * (size_t)k);
    double* x0 = (double*)malloc(sizeof(double) * (size_t)n);
    double* y0 = (double*)malloc(sizeof(double) * (size_t)m);
    for (int32_t j = 0; j < n; ++j) {
        for (int t = 0; t < k; ++t) {
            int32_t r;
            int dup;
            do { /* k distinct rows per column, uniform */
                r = (int32_t)or_below(&g, m);
                dup = 0;
                for (int q = 0; q < t; ++q) dup |= pick[q] == r;
            } while (dup);
            pick[t] = r;
            double v;
            do { /* U[-1,1] without zero, optionally rounded to FP32 */
                v = 2.0 * or_uniform(&g) - 1.0;
                if (fp32_values) v = (double)(float)v;
            } while (v == 0.0);
            const int64_t p = (int64_t)j * k + t;
            row[p] = r;
            col[p] = j;
            val[p] = v;
        }
    }
    for (int32_t j = 0; j < n; ++j) x0[j] = 5.0 * or_uniform(&g);
    for (int32_t i = 0; i < m; ++i) y0[i] = or_normal(&g);
    for (int32_t i = 0; i < m; ++i) rL[i] = 0.0;
    for (int64_t p = 0; p < (int64_t)n * k; ++p) rL[row[p]] += val[p] * x0[col[p]]; /* b = A x0 */
    for (int32_t j = 0; j < n; ++j) {
        double s = 0.0;
        for (int t = 0; t < k; ++t) {
            const int64_t p = (int64_t)j * k + t;
            s += val[p] * y0[row[p]];
        }
        c[j] = s + or_uniform(&g); /* c = A^T y0 + z0 */
        l[j] = 0.0;
        u[j] = 10.0;
    }
    for (int32_t i = 0; i < m; ++i) rU[i] = rL[i];
    free(pick);
    free(x0);
    free(y0);
    return 0;
}

int or_gen_transport(int S, int D, uint64_t seed, int32_t* row, int32_t* col, double* val, double* c, double* rL,
                     double* rU, double* l, double* u) {
    if (S < 1 || D < 1) return 1;
    or_rng g;
    or_rng_seed(&g, seed);
    int64_t* supply = (int64_t*)malloc(sizeof(int64_t) * (size_t)S);
    int64_t* demand = (int64_t*)malloc(sizeof(int64_t) * (size_t)D);
    double* w = (double*)malloc(sizeof(double) * (size_t)D);
    int64_t total = 0, assigned = 0;
    double wsum = 0.0;
    for (int i = 0; i < S; ++i) {
        supply[i] = 100 + or_below(&g, 901);
        total += supply[i];
    }
    for (int j = 0; j < D; ++j) {
        w[j] = 0.5 + or_uniform(&g);
        wsum += w[j];
    }
    for (int j = 0; j < D; ++j) {
        int64_t d = (int64_t)floor((double)total * w[j] / wsum);
        demand[j] = d > 1 ? d : 1;
        assigned += demand[j];
    }
    /* the remainder goes out one unit at a time, round robin, so demands are
     * an integer partition of the total supply */
    for (int64_t r = total - assigned, j = 0; r != 0; j = (j + 1) % D) {
        if (r > 0) { demand[j]++; r--; }
        else if (demand[j] > 1) { demand[j]--; r++; }
    }
    for (int i = 0; i < S; ++i)
        for (int j = 0; j < D; ++j) {
            const int64_t a = (int64_t)i * D + j;
            row[2 * a] = i;
            col[2 * a] = (int32_t)a;
            val[2 * a] = 1.0;
            row[2 * a + 1] = S + j;
            col[2 * a + 1] = (int32_t)a;
            val[2 * a + 1] = 1.0;
            c[a] = (double)(1 + or_below(&g, 100));
            l[a] = 0.0;
            u[a] = OR_INF;
        }
    for (int i = 0; i < S; ++i) rL[i] = rU[i] = (double)supply[i];
    for (int j = 0; j < D; ++j) rL[S + j] = rU[S + j] = (double)demand[j];
    free(supply);
    free(demand);
    free(w);
    return 0;
}
