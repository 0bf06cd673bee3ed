// ref_capi.cpp -- TEST INFRASTRUCTURE ONLY (the oracle). A flat extern "C"
// wrapper over the reference solver's own C++ pipeline so the Python tests
// and the CPU-baseline leg of bench.py can call it through ctypes. It is
// compiled together with the reference sources (see oracle/Makefile) into
// oracle/_ref/libsovref*.so; nothing in the product links it.
//
// Every entry point forwards to the reference's own functions:
//   read_mps                 src/mps_reader.cpp:54
//   to_ranged_lp             include/ranged_lp.hpp:39-62
//   presolve / postsolve     src/presolve.cpp:524 / :549
//   build_pdlp_form          src/pdlp.cpp:8-82, extract_solution :84-90
//   scale                    src/scaling.cpp:25-84
//   solve_pdhg               src/pdlp.cpp:146-152 (pdlp_run, include/pdlp_algo.hpp:49-185)
//   solve_pdhg_gpu           gpu/pdlp_gpu_solve.cu:261-267 (only in the CUDA variant)
//   verify                   src/verify.cpp:18-103
//   solve_mps / solve_mps_simplex   src/solve.cpp:150 / :234
#include "mps_reader.hpp"
#include "presolve.hpp"
#include "scaling.hpp"
#include "pdlp.hpp"
#include "pdlp_gpu.hpp"
#include "verify.hpp"
#include "solve.hpp"
#include "simplex.hpp"

#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>
#include <string>
#include <vector>

namespace {

struct RefProblem {
    RangedLP original;            // to_ranged_lp(read_mps(...)) or built from arrays
    PresolveResult pres;
    RangedLP pdlp_form;           // build_pdlp_form(pres.reduced).first
    PdlpFormMeta meta;
    ScalingResult sr;             // scale(pdlp_form)
    int status = 0;               // 0 ok, 1 infeasible, 2 unbounded, 3 reduced to nothing
    std::string error;
};

thread_local std::string g_err;

void prepare(RefProblem& P, bool use_presolve) {
    P.pres = presolve(P.original, use_presolve ? 500 : 0);
    if (P.pres.status == "infeasible") { P.status = 1; return; }
    if (P.pres.status == "unbounded") { P.status = 2; return; }
    if (P.pres.reduced.n() == 0 || P.pres.reduced.m() == 0) { P.status = 3; return; }
    auto built = build_pdlp_form(P.pres.reduced);
    P.pdlp_form = built.first;
    P.meta = built.second;
    P.sr = scale(P.pdlp_form);
    P.status = 0;
}

const RangedLP* pick(const RefProblem* P, int which) {
    if (which == 0) return &P->original;
    if (which == 1) return &P->pdlp_form;
    if (which == 2) return &P->sr.scaled;
    if (which == 3) return &P->pres.reduced;
    return nullptr;
}

void fill_names(RangedLP& r, int m, int n) {
    r.row_names.resize(m);
    r.col_names.resize(n);
    for (int i = 0; i < m; ++i) r.row_names[i] = "R" + std::to_string(i);
    for (int j = 0; j < n; ++j) r.col_names[j] = "C" + std::to_string(j);
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void* ref_load_mps(const char* path, int use_presolve) {
    try {
        auto* P = new RefProblem();
        P->original = to_ranged_lp(read_mps(path));
        prepare(*P, use_presolve != 0);
        return P;
    } catch (const std::exception& e) { g_err = e.what(); return nullptr; }
}

void* ref_from_arrays(int m, int n, int nnz, const int* row, const int* col, const double* val,
                      const double* c, const double* rL, const double* rU, const double* l, const double* u,
                      double obj_offset, int use_presolve) {
    try {
        auto* P = new RefProblem();
        RangedLP& r = P->original;
        r.name = "arrays";
        fill_names(r, m, n);
        r.A.rows = m; r.A.cols = n;
        r.A.row_idx.assign(row, row + nnz);
        r.A.col_idx.assign(col, col + nnz);
        r.A.val.assign(val, val + nnz);
        r.c.assign(c, c + n);
        r.rL.assign(rL, rL + m); r.rU.assign(rU, rU + m);
        r.l.assign(l, l + n); r.u.assign(u, u + n);
        r.obj_offset = obj_offset;
        r.original_sense = "min";
        prepare(*P, use_presolve != 0);
        return P;
    } catch (const std::exception& e) { g_err = e.what(); return nullptr; }
}

void ref_free(void* h) { delete static_cast<RefProblem*>(h); }

int ref_status(void* h) { return static_cast<RefProblem*>(h)->status; }

// which: 0 original, 1 PDLP form (unscaled), 2 scaled PDLP form, 3 presolved
int ref_form_dims(void* h, int which, int* m, int* n, int* nnz) {
    const RangedLP* r = pick(static_cast<RefProblem*>(h), which);
    if (!r) return 1;
    *m = r->m(); *n = r->n(); *nnz = r->A.nnz();
    return 0;
}

int ref_form_export(void* h, int which, int* row, int* col, double* val, double* c, double* rL, double* rU,
                    double* l, double* u, double* obj_offset) {
    const RangedLP* r = pick(static_cast<RefProblem*>(h), which);
    if (!r) return 1;
    std::copy(r->A.row_idx.begin(), r->A.row_idx.end(), row);
    std::copy(r->A.col_idx.begin(), r->A.col_idx.end(), col);
    std::copy(r->A.val.begin(), r->A.val.end(), val);
    std::copy(r->c.begin(), r->c.end(), c);
    std::copy(r->rL.begin(), r->rL.end(), rL);
    std::copy(r->rU.begin(), r->rU.end(), rU);
    std::copy(r->l.begin(), r->l.end(), l);
    std::copy(r->u.begin(), r->u.end(), u);
    *obj_offset = r->obj_offset;
    return 0;
}

int ref_scaling_export(void* h, double* Dr, double* Dc) {
    auto* P = static_cast<RefProblem*>(h);
    std::copy(P->sr.Dr.begin(), P->sr.Dr.end(), Dr);
    std::copy(P->sr.Dc.begin(), P->sr.Dc.end(), Dc);
    return 0;
}

// Reference scale() on a form given as arrays (used to pin the product's own
// Ruiz + Pock-Chambolle restatement).
int ref_scale_arrays(int m, int n, int nnz, const int* row, const int* col, const double* val,
                     const double* c, const double* rL, const double* rU, const double* l, const double* u,
                     double* val_out, double* c_out, double* rL_out, double* rU_out, double* l_out, double* u_out,
                     double* Dr, double* Dc) {
    try {
        RangedLP r;
        fill_names(r, m, n);
        r.A.rows = m; r.A.cols = n;
        r.A.row_idx.assign(row, row + nnz); r.A.col_idx.assign(col, col + nnz); r.A.val.assign(val, val + nnz);
        r.c.assign(c, c + n); r.rL.assign(rL, rL + m); r.rU.assign(rU, rU + m);
        r.l.assign(l, l + n); r.u.assign(u, u + n);
        ScalingResult s = scale(r);
        std::copy(s.scaled.A.val.begin(), s.scaled.A.val.end(), val_out);
        std::copy(s.scaled.c.begin(), s.scaled.c.end(), c_out);
        std::copy(s.scaled.rL.begin(), s.scaled.rL.end(), rL_out);
        std::copy(s.scaled.rU.begin(), s.scaled.rU.end(), rU_out);
        std::copy(s.scaled.l.begin(), s.scaled.l.end(), l_out);
        std::copy(s.scaled.u.begin(), s.scaled.u.end(), u_out);
        std::copy(s.Dr.begin(), s.Dr.end(), Dr);
        std::copy(s.Dc.begin(), s.Dc.end(), Dc);
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return 1; }
}

// info[0]=iterations (attempts) info[1]=restarts info[2]=converged
static int run_pdhg(RefProblem* P, bool gpu, int max_iter, int check_every, double tol, double* x, double* y,
                    int* info, double* eps, double* seconds) {
    try {
        auto t0 = std::chrono::steady_clock::now();
        PdlpResult r;
        if (gpu) {
#ifdef SOVEREIGN_WITH_CUDA
            r = solve_pdhg_gpu(P->pdlp_form, P->sr.scaled, P->sr.Dr, P->sr.Dc, 0.99, max_iter, check_every, tol, nullptr);
#else
            g_err = "this oracle build has no CUDA engine";
            return 2;
#endif
        } else {
            r = solve_pdhg(P->pdlp_form, P->sr.scaled, P->sr.Dr, P->sr.Dc, 0.99, max_iter, check_every, tol, nullptr);
        }
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::copy(r.x.begin(), r.x.end(), x);
        std::copy(r.y.begin(), r.y.end(), y);
        info[0] = r.iterations; info[1] = r.restarts; info[2] = r.converged ? 1 : 0;
        eps[0] = r.eps_P; eps[1] = r.eps_D; eps[2] = r.eps_G;
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return 1; }
}

int ref_solve_pdhg(void* h, int max_iter, int check_every, double tol, double* x, double* y, int* info,
                   double* eps, double* seconds) {
    return run_pdhg(static_cast<RefProblem*>(h), false, max_iter, check_every, tol, x, y, info, eps, seconds);
}

int ref_solve_pdhg_gpu(void* h, int max_iter, int check_every, double tol, double* x, double* y, int* info,
                       double* eps, double* seconds) {
    return run_pdhg(static_cast<RefProblem*>(h), true, max_iter, check_every, tol, x, y, info, eps, seconds);
}

// verify() on one of the handle's forms. out: eps_P, eps_D, eps_G, objective, dual_objective
int ref_verify_form(void* h, int which, const double* x, const double* y, double* out) {
    const RangedLP* r = pick(static_cast<RefProblem*>(h), which);
    if (!r) return 1;
    std::vector<double> xv(x, x + r->n()), yv(y, y + r->m());
    KKTReport k = verify(*r, xv, yv);
    out[0] = k.eps_P; out[1] = k.eps_D; out[2] = k.eps_G; out[3] = k.objective; out[4] = k.dual_objective;
    return 0;
}

// PDLP-form (x2, y2) -> extract_solution -> postsolve -> verify on the
// original problem, exactly as solve_mps does (src/solve.cpp:208-216).
// out: objective (reported sense), eps_P, eps_D, eps_G
int ref_finish(void* h, const double* x2, const double* y2, double* out) {
    auto* P = static_cast<RefProblem*>(h);
    try {
        std::vector<double> xv(x2, x2 + P->pdlp_form.n()), yv(y2, y2 + P->pdlp_form.m());
        std::vector<double> x_red, y_red, x_o, y_o, z_o;
        extract_solution(P->meta, xv, yv, x_red, y_red);
        const RangedLP& reduced = P->pres.reduced;
        CSR ATcsr = to_csc_as_transposed_csr(reduced.A);
        auto ATy = matvec_T(ATcsr, y_red);
        std::vector<double> z_red(reduced.n());
        for (int j = 0; j < reduced.n(); ++j) z_red[j] = reduced.c[j] - ATy[j];
        postsolve(P->original.n(), P->original.m(), P->pres.row_ids, P->pres.col_ids, x_red, y_red, z_red,
                  P->pres.steps, x_o, y_o, z_o);
        KKTReport k = verify(P->original, x_o, y_o);
        out[0] = report_objective(P->original, k.objective);
        out[1] = k.eps_P; out[2] = k.eps_D; out[3] = k.eps_G;
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return 1; }
}

// Full reference pipeline on an MPS file (src/solve.cpp:150). out: objective,
// eps_P, eps_D, eps_G, iterations, seconds. status_buf receives Solution::status.
int ref_solve_mps(const char* path, double tol, int max_iter, double* out, char* status_buf, int buflen) {
    try {
        auto t0 = std::chrono::steady_clock::now();
        Solution s = solve_mps(path, tol, max_iter);
        out[0] = s.objective; out[1] = s.eps_P; out[2] = s.eps_D; out[3] = s.eps_G; out[4] = s.iterations;
        out[5] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::snprintf(status_buf, buflen, "%s|%s", s.status.c_str(), s.engine_used.c_str());
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return 1; }
}

// Dual simplex pipeline (src/solve.cpp:234). out: objective, eps_P, eps_D, eps_G, pivots, seconds
int ref_solve_simplex_mps(const char* path, double time_limit, double* out, char* status_buf, int buflen) {
    try {
        SimplexOptions opt;
        opt.time_limit = time_limit;
        auto t0 = std::chrono::steady_clock::now();
        Solution s = solve_mps_simplex(path, opt);
        out[0] = s.objective; out[1] = s.eps_P; out[2] = s.eps_D; out[3] = s.eps_G; out[4] = s.iterations;
        out[5] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::snprintf(status_buf, buflen, "%s", s.status.c_str());
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return 1; }
}

// Writes the handle's original problem as a free-format MPS file that
// read_mps parses back (values printed with %.17g), so MPS-only reference
// entry points (dual simplex, solve_mps) can run on generated LPs.
int ref_write_mps(void* h, const char* path) {
    auto* P = static_cast<RefProblem*>(h);
    const RangedLP& r = P->original;
    std::FILE* f = std::fopen(path, "w");
    if (!f) { g_err = "cannot open output"; return 1; }
    std::fprintf(f, "NAME GEN\nROWS\n N  COST\n");
    std::vector<char> type(r.m());
    std::vector<double> rhs(r.m()), rng(r.m(), 0.0);
    std::vector<char> has_rng(r.m(), 0);
    for (int i = 0; i < r.m(); ++i) {
        double lo = r.rL[i], hi = r.rU[i];
        if (lo == hi) { type[i] = 'E'; rhs[i] = lo; }
        else if (std::isfinite(lo) && std::isfinite(hi)) { type[i] = 'G'; rhs[i] = lo; rng[i] = hi - lo; has_rng[i] = 1; }
        else if (std::isfinite(lo)) { type[i] = 'G'; rhs[i] = lo; }
        else if (std::isfinite(hi)) { type[i] = 'L'; rhs[i] = hi; }
        else { type[i] = 'N'; rhs[i] = 0.0; }
        std::fprintf(f, " %c  R%d\n", type[i] == 'N' ? 'N' : type[i], i);
    }
    std::fprintf(f, "COLUMNS\n");
    CSR AT = to_csc_as_transposed_csr(r.A);
    for (int j = 0; j < r.n(); ++j) {
        std::fprintf(f, "    C%d  COST  %.17g\n", j, r.c[j]);
        for (int p = AT.indptr[j]; p < AT.indptr[j + 1]; ++p)
            std::fprintf(f, "    C%d  R%d  %.17g\n", j, AT.indices[p], AT.data[p]);
    }
    std::fprintf(f, "RHS\n");
    if (r.obj_offset != 0.0) std::fprintf(f, "    RHS  COST  %.17g\n", -r.obj_offset);
    for (int i = 0; i < r.m(); ++i)
        if (rhs[i] != 0.0) std::fprintf(f, "    RHS  R%d  %.17g\n", i, rhs[i]);
    bool any_rng = false;
    for (int i = 0; i < r.m(); ++i) any_rng |= has_rng[i] != 0;
    if (any_rng) {
        std::fprintf(f, "RANGES\n");
        for (int i = 0; i < r.m(); ++i)
            if (has_rng[i]) std::fprintf(f, "    RNG  R%d  %.17g\n", i, rng[i]);
    }
    std::fprintf(f, "BOUNDS\n");
    for (int j = 0; j < r.n(); ++j) {
        double lo = r.l[j], hi = r.u[j];
        if (lo == hi) { std::fprintf(f, " FX BND  C%d  %.17g\n", j, lo); continue; }
        if (!std::isfinite(lo) && !std::isfinite(hi)) { std::fprintf(f, " FR BND  C%d\n", j); continue; }
        if (!std::isfinite(lo)) std::fprintf(f, " MI BND  C%d\n", j);
        else if (lo != 0.0) std::fprintf(f, " LO BND  C%d  %.17g\n", j, lo);
        if (std::isfinite(hi)) std::fprintf(f, " UP BND  C%d  %.17g\n", j, hi);
    }
    std::fprintf(f, "ENDATA\n");
    std::fclose(f);
    return 0;
}

}  // extern "C"
