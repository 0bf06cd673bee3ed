// capi.cpp -- the extern "C" boundary of libb200pdlp.so (include/b200_pdlp.h).
// Every entry point converts internal errors into a B2_ERR_* status plus a
// thread-local message; no exception crosses the ABI.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <thread>

#include "b200_pdlp.h"
#include "internal.h"

namespace b2 {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

[[noreturn]] void fail(int code, const std::string& msg) { throw Error{code, msg}; }

template <class F>
int guarded(F&& f) {
    try {
        f();
        g_last_error.clear();
        return B2_OK;
    } catch (const Error& e) {
        g_last_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return B2_ERR_OOM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return B2_ERR_INVALID;
    } catch (...) {
        g_last_error = "unknown error";
        return B2_ERR_INVALID;
    }
}

}  // namespace b2

struct b2_engine {
    b2::EngineImpl* impl;
};

struct b2_batch {
    b2::BatchImpl* impl;
};

struct b2_server {
    b2::ServerImpl* impl;
};

struct b2_pool {
    b2::PoolImpl* impl;
};

extern "C" {

void b2_default_opts(b2_solve_opts* o) {
    std::memset(o, 0, sizeof(*o));
    o->max_iterations = 200000;   // solve_pdhg default (include/pdlp.hpp:35-38)
    o->check_every = 64;
    o->tol = 1e-6;
    o->precision = B2_PREC_MIXED;
    o->switch_tol = 1e-5;
    o->stall_checks = 32;
    o->time_limit_s = 0.0;
    o->barrier_timeout_s = 10.0;
}

const char* b2_last_error(void) { return b2::g_last_error.c_str(); }

const char* b2_version(void) { return "b200-pdlp 0.1 (sm_100a)"; }

int b2_solve_pdhg_gpu_ex(const b2_lp_view* U, const b2_lp_view* S, const double* Dr, const double* Dc,
                         const b2_solve_opts* opts, const volatile int32_t* stop_flag, double* x_out, double* y_out,
                         b2_result* res) {
    return b2::guarded([&] {
        if (!U || !S || !opts) b2::fail(B2_ERR_INVALID, "null argument");
        const auto t0 = std::chrono::steady_clock::now();
        b2::EngineImpl* e = b2::engine_create(*U, *S, Dr, Dc, *opts);
        try {
            b2::engine_solve(e, *opts, stop_flag, x_out, y_out, res);
        } catch (...) {
            b2::engine_destroy(e);
            throw;
        }
        b2::engine_destroy(e);
        if (res) res->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    });
}

int b2_solve_pdhg_gpu(const b2_lp_view* U, const b2_lp_view* S, const double* Dr, const double* Dc, double /*eta*/,
                      int32_t max_iterations, int32_t check_every, double tol, const volatile int32_t* stop_flag,
                      double* x_out, double* y_out, b2_result* res) {
    b2_solve_opts o;
    b2_default_opts(&o);
    o.max_iterations = max_iterations;
    o.check_every = check_every;
    o.tol = tol;
    return b2_solve_pdhg_gpu_ex(U, S, Dr, Dc, &o, stop_flag, x_out, y_out, res);
}

int b2_solve_pdhg_gpu_noalloc(const b2_lp_view* U, const b2_lp_view* S, const double* Dr, const double* Dc,
                              const b2_solve_opts* opts, double* x_out, double* y_out, b2_result* res) {
    return b2::guarded([&] {
        if (!U || !S || !opts) b2::fail(B2_ERR_INVALID, "null argument");
        b2::solve_noalloc(*U, *S, Dr, Dc, *opts, x_out, y_out, res);
    });
}

int b2_engine_create(const b2_lp_view* U, const b2_lp_view* S, const double* Dr, const double* Dc,
                     const b2_solve_opts* opts, b2_engine** out) {
    return b2::guarded([&] {
        if (!U || !S || !out) b2::fail(B2_ERR_INVALID, "null argument");
        b2_solve_opts o;
        if (opts) o = *opts;
        else b2_default_opts(&o);
        *out = nullptr;
        b2::EngineImpl* e = b2::engine_create(*U, *S, Dr, Dc, o);
        *out = new b2_engine{e};
    });
}

int b2_engine_solve(b2_engine* e, const b2_solve_opts* opts, const volatile int32_t* stop_flag, double* x_out,
                    double* y_out, b2_result* res) {
    return b2::guarded([&] {
        if (!e || !opts) b2::fail(B2_ERR_INVALID, "null argument");
        b2::engine_solve(e->impl, *opts, stop_flag, x_out, y_out, res);
    });
}

void b2_engine_destroy(b2_engine* e) {
    if (!e) return;
    b2::engine_destroy(e->impl);
    delete e;
}

int b2_engine_get_info(b2_engine* e, b2_engine_info* info) {
    return b2::guarded([&] {
        if (!e || !info) b2::fail(B2_ERR_INVALID, "null argument");
        b2::engine_info(e->impl, info);
    });
}

int b2_engine_spmv(b2_engine* e, int32_t which, const double* x, double* y) {
    return b2::guarded([&] {
        if (!e || !x || !y || (which != 0 && which != 1)) b2::fail(B2_ERR_INVALID, "bad argument");
        b2::engine_spmv(e->impl, which, x, y);
    });
}

int b2_engine_spmv_bench(b2_engine* e, int32_t which, int32_t precision, int32_t reps, void* stream,
                         double* avg_ms) {
    return b2::guarded([&] {
        if (!e || !avg_ms || (which != 0 && which != 1) || reps < 0) b2::fail(B2_ERR_INVALID, "bad argument");
        b2::engine_spmv_bench(e->impl, which, precision, reps, stream, avg_ms);
    });
}

int b2_engine_trace(b2_engine* e, double* out, int32_t max_records, int32_t* count) {
    return b2::guarded([&] {
        if (!e || !count) b2::fail(B2_ERR_INVALID, "null argument");
        *count = b2::engine_trace(e->impl, out, max_records);
    });
}

int b2_server_create(const b2_server_opts* sopts, const b2_solve_opts* opts, b2_server** out) {
    return b2::guarded([&] {
        if (!out) b2::fail(B2_ERR_INVALID, "null argument");
        *out = nullptr;
        b2_server_opts so;
        std::memset(&so, 0, sizeof(so));
        if (sopts) so = *sopts;
        b2_solve_opts o;
        if (opts) o = *opts;
        else b2_default_opts(&o);
        b2::ServerImpl* s = b2::server_create(so, o);
        *out = new b2_server{s};
    });
}

int b2_server_submit(b2_server* s, const b2_lp_view* U, int64_t* ticket) {
    return b2::guarded([&] {
        if (!s || !U || !ticket) b2::fail(B2_ERR_INVALID, "null argument");
        *ticket = b2::server_submit(s->impl, *U);
    });
}

int b2_server_submit_file(b2_server* s, const char* path, int64_t* ticket) {
    return b2::guarded([&] {
        if (!s || !path || !ticket) b2::fail(B2_ERR_INVALID, "null argument");
        *ticket = b2::server_submit_file(s->impl, path);
    });
}

int b2_server_submit_lp(b2_server* s, const b2_lp_view* original, int32_t presolve, int64_t* ticket) {
    return b2::guarded([&] {
        if (!s || !original || !ticket) b2::fail(B2_ERR_INVALID, "null argument");
        *ticket = b2::server_submit_lp(s->impl, *original, presolve != 0);
    });
}

int b2_pdlp_form_build(const b2_lp_view* ranged, b2_pdlp_form** out) {
    return b2::guarded([&] {
        if (!ranged || !out) b2::fail(B2_ERR_INVALID, "null argument");
        *out = reinterpret_cast<b2_pdlp_form*>(b2::pdlp_form_build(*ranged));
    });
}

void b2_pdlp_form_view(const b2_pdlp_form* f, b2_lp_view* form) {
    if (f && form) b2::pdlp_form_view(*reinterpret_cast<const b2::PdlpForm*>(f), *form);
}

int b2_pdlp_form_extract(const b2_pdlp_form* f, const double* x2, const double* y2, double* x, double* y) {
    return b2::guarded([&] {
        if (!f || !x2 || !y2 || !x || !y) b2::fail(B2_ERR_INVALID, "null argument");
        b2::pdlp_form_extract(*reinterpret_cast<const b2::PdlpForm*>(f), x2, y2, x, y);
    });
}

void b2_pdlp_form_destroy(b2_pdlp_form* f) { b2::pdlp_form_free(reinterpret_cast<b2::PdlpForm*>(f)); }

int b2_presolve(const b2_lp_view* original, b2_presolved** out, int32_t* status) {
    return b2::guarded([&] {
        if (!original || !out) b2::fail(B2_ERR_INVALID, "null argument");
        b2::Presolved* p = b2::presolve_lp(*original);
        if (status) *status = b2::presolved_status(*p);
        *out = reinterpret_cast<b2_presolved*>(p);
    });
}

void b2_presolved_view(const b2_presolved* p, b2_lp_view* reduced) {
    if (p && reduced) b2::presolved_view(*reinterpret_cast<const b2::Presolved*>(p), *reduced);
}

int b2_postsolve(const b2_presolved* p, const double* x_red, const double* y_red, double* x, double* y) {
    return b2::guarded([&] {
        if (!p || !x || !y) b2::fail(B2_ERR_INVALID, "null argument");
        b2::postsolve_lp(*reinterpret_cast<const b2::Presolved*>(p), x_red, y_red, x, y);
    });
}

void b2_presolved_destroy(b2_presolved* p) { b2::presolved_free(reinterpret_cast<b2::Presolved*>(p)); }

int b2_lp_write(const char* path, const b2_lp_view* lp) {
    return b2::guarded([&] {
        if (!path || !lp) b2::fail(B2_ERR_INVALID, "null argument");
        b2::lp_write(path, *lp);
    });
}

int b2_lp_read_dims(const char* path, int32_t* m, int32_t* n, int64_t* nnz) {
    return b2::guarded([&] {
        if (!path || !m || !n || !nnz) b2::fail(B2_ERR_INVALID, "null argument");
        b2::lp_read_dims(path, m, n, nnz);
    });
}

int b2_lp_read(const char* path, int32_t* row, int32_t* col, double* val, double* c, double* rL, double* rU,
               double* l, double* u, double* obj_offset) {
    return b2::guarded([&] {
        if (!path) b2::fail(B2_ERR_INVALID, "null argument");
        b2::LpArrays a;
        b2::lp_read(path, a);
        auto cp = [](auto* dst, const auto& v) {
            if (!v.empty()) {
                if (!dst) b2::fail(B2_ERR_INVALID, "null output buffer");
                std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
            }
        };
        cp(row, a.row); cp(col, a.col); cp(val, a.val);
        cp(c, a.c); cp(l, a.l); cp(u, a.u); cp(rL, a.rL); cp(rU, a.rU);
        if (obj_offset) *obj_offset = a.obj_offset;
    });
}

int b2_server_wait(b2_server* s, int64_t ticket, double timeout_s, double* x, double* y, b2_result* res,
                   b2_request_info* info) {
    int rc = B2_OK;
    const int g = b2::guarded([&] {
        if (!s) b2::fail(B2_ERR_INVALID, "null argument");
        rc = b2::server_wait(s->impl, ticket, timeout_s, x, y, res, info);
    });
    if (g != B2_OK) return g;
    if (rc == B2_ERR_PENDING) b2::set_last_error("request not finished yet");
    return rc;
}

int b2_server_stats_get(b2_server* s, b2_server_stats* out) {
    return b2::guarded([&] {
        if (!s || !out) b2::fail(B2_ERR_INVALID, "null argument");
        b2::server_stats(s->impl, out);
    });
}

void b2_server_destroy(b2_server* s) {
    if (!s) return;
    b2::server_destroy(s->impl);
    delete s;
}

int b2_layout_digest(const b2_lp_view* U, const b2_lp_view* S, const double* Dr, const double* Dc, int32_t threads,
                     int32_t whole_gpu, uint64_t* digest) {
    return b2::guarded([&] {
        if (!U || !S || !digest) b2::fail(B2_ERR_INVALID, "null argument");
        b2::BuildParams bp;
        bp.split = whole_gpu != 0;
        bp.threads = threads > 0 ? threads : 1;
        b2::Layout L;
        b2::build_layout(*U, *S, Dr, Dc, bp, L);
        *digest = b2::layout_digest(L);
    });
}

int b2_layout_get_stats(const b2_lp_view* U, const b2_lp_view* S, const double* Dr, const double* Dc,
                        int32_t whole_gpu, b2_layout_stats* out) {
    return b2::guarded([&] {
        if (!U || !S || !out) b2::fail(B2_ERR_INVALID, "null argument");
        b2::BuildParams bp;
        bp.split = whole_gpu != 0;
        bp.threads = (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
        b2::Layout L;
        b2::build_layout(*U, *S, Dr, Dc, bp, L);
        out->a_slices = L.A.n_slices();
        out->at_slices = L.AT.n_slices();
        out->a_padded = L.A.padded;
        out->at_padded = L.AT.padded;
        out->a_groups = L.A.n_groups();
        out->at_groups = L.AT.n_groups();
        out->a_dense = L.A.n_dense;
        out->at_dense = L.AT.n_dense;
    });
}

int64_t b2_request_work(int32_t m, int32_t n, int64_t nnz) { return b2::request_work(m, n, nnz); }

int64_t b2_request_cost(int32_t m, int32_t n, int64_t nnz) { return b2::request_cost(m, n, nnz); }

int b2_shard_plan(const int64_t* work, int64_t count, int32_t parts, int32_t online, int32_t* rank_of) {
    return b2::guarded([&] { b2::shard_plan(work, count, parts, online != 0, rank_of); });
}

int b2_pool_create(const int32_t* devices, int32_t count, const b2_server_opts* sopts, const b2_solve_opts* opts,
                   b2_pool** out) {
    return b2::guarded([&] {
        if (!out) b2::fail(B2_ERR_INVALID, "null argument");
        *out = nullptr;
        b2_server_opts so;
        std::memset(&so, 0, sizeof(so));
        if (sopts) so = *sopts;
        b2_solve_opts o;
        if (opts) o = *opts;
        else b2_default_opts(&o);
        b2::PoolImpl* p = b2::pool_create(devices, count, so, o);
        *out = new b2_pool{p};
    });
}

int b2_pool_submit(b2_pool* p, const b2_lp_view* U, int64_t* ticket) {
    return b2::guarded([&] {
        if (!p || !U || !ticket) b2::fail(B2_ERR_INVALID, "null argument");
        *ticket = b2::pool_submit(p->impl, *U);
    });
}

int b2_pool_submit_file(b2_pool* p, const char* path, int64_t* ticket) {
    return b2::guarded([&] {
        if (!p || !path || !ticket) b2::fail(B2_ERR_INVALID, "null argument");
        *ticket = b2::pool_submit_file(p->impl, path);
    });
}

int b2_pool_wait(b2_pool* p, int64_t ticket, double timeout_s, double* x, double* y, b2_result* res,
                 b2_request_info* info, int32_t* member) {
    int rc = B2_OK;
    const int g = b2::guarded([&] {
        if (!p) b2::fail(B2_ERR_INVALID, "null argument");
        rc = b2::pool_wait(p->impl, ticket, timeout_s, x, y, res, info, member);
    });
    if (g != B2_OK) return g;
    if (rc == B2_ERR_PENDING) b2::set_last_error("request not finished yet");
    return rc;
}

int b2_pool_stats_get(b2_pool* p, int32_t member, b2_server_stats* out) {
    return b2::guarded([&] {
        if (!p || !out) b2::fail(B2_ERR_INVALID, "null argument");
        b2::pool_stats(p->impl, member, out);
    });
}

void b2_pool_destroy(b2_pool* p) {
    if (!p) return;
    b2::pool_destroy(p->impl);
    delete p;
}

int b2_batch_create(int32_t n_lp, const b2_lp_view* U, const b2_lp_view* S, const double* const* Dr,
                    const double* const* Dc, const b2_solve_opts* opts, b2_batch** out) {
    return b2::guarded([&] {
        if (!U || !S || !Dr || !Dc || !out) b2::fail(B2_ERR_INVALID, "null argument");
        b2_solve_opts o;
        if (opts) o = *opts;
        else b2_default_opts(&o);
        *out = nullptr;
        b2::BatchImpl* b = b2::batch_create(n_lp, U, S, Dr, Dc, o);
        *out = new b2_batch{b};
    });
}

int32_t b2_shape_class(int32_t m, int32_t n, int64_t nnz) { return b2::shape_class(m, n, nnz); }

void b2_default_tune_table(b2_tune_table* out) {
    if (out) b2::default_tune_table(*out);
}

int b2_batch_autotune(int32_t n_lp, const b2_lp_view* U, const b2_lp_view* S, const double* const* Dr,
                      const double* const* Dc, const b2_solve_opts* opts, b2_tune_table* out) {
    return b2::guarded([&] {
        if (!U || !S || !Dr || !Dc || !out || n_lp <= 0) b2::fail(B2_ERR_INVALID, "bad argument");
        b2_solve_opts o;
        if (opts) o = *opts;
        else b2_default_opts(&o);
        b2::batch_autotune(n_lp, U, S, Dr, Dc, o, *out);
    });
}

int b2_batch_solve(b2_batch* b, const b2_solve_opts* opts, const volatile int32_t* stop_flag, b2_result* results,
                   double* total_ms) {
    return b2::guarded([&] {
        if (!b || !opts) b2::fail(B2_ERR_INVALID, "null argument");
        b2::batch_solve(b->impl, *opts, stop_flag, results, total_ms);
    });
}

int b2_batch_get_solution(b2_batch* b, int32_t i, double* x, double* y) {
    return b2::guarded([&] {
        if (!b) b2::fail(B2_ERR_INVALID, "null argument");
        b2::batch_solution(b->impl, i, x, y);
    });
}

int b2_batch_get_info(b2_batch* b, b2_batch_info* info) {
    return b2::guarded([&] {
        if (!b || !info) b2::fail(B2_ERR_INVALID, "null argument");
        b2::batch_info(b->impl, info);
    });
}

int b2_batch_spmv(b2_batch* b, int32_t i, int32_t which, const double* x, double* y) {
    return b2::guarded([&] {
        if (!b || !x || !y || (which != 0 && which != 1)) b2::fail(B2_ERR_INVALID, "bad argument");
        b2::batch_spmv(b->impl, i, which, x, y);
    });
}

void b2_batch_destroy(b2_batch* b) {
    if (!b) return;
    b2::batch_destroy(b->impl);
    delete b;
}

int b2_scale(const b2_lp_view* lp, int32_t ruiz_passes, double* val_s, double* c_s, double* rL_s, double* rU_s,
             double* l_s, double* u_s, double* Dr, double* Dc) {
    return b2::guarded([&] {
        if (!lp) b2::fail(B2_ERR_INVALID, "null argument");
        b2::scale_lp(*lp, ruiz_passes, val_s, c_s, rL_s, rU_s, l_s, u_s, Dr, Dc,
                     (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency())));
    });
}

int b2_scale_gpu(const b2_lp_view* lp, int32_t ruiz_passes, double* val_s, double* c_s, double* rL_s, double* rU_s,
             double* l_s, double* u_s, double* Dr, double* Dc) {
    return b2::guarded([&] {
        if (!lp) b2::fail(B2_ERR_INVALID, "null argument");
        b2::scale_lp_gpu(*lp, ruiz_passes, val_s, c_s, rL_s, rU_s, l_s, u_s, Dr, Dc);
    });
}

int b2_gen_random_lp(int32_t m, int32_t n, int32_t k, uint64_t seed, int32_t fp32_values, int32_t* row,
                     int32_t* col, double* val, double* c, double* rL, double* rU, double* l, double* u) {
    return b2::guarded([&] { b2::gen_random_lp(m, n, k, seed, fp32_values != 0, row, col, val, c, rL, rU, l, u); });
}

int b2_gen_transport(int32_t S, int32_t D, uint64_t seed, int32_t* row, int32_t* col, double* val, double* c,
                     double* rL, double* rU, double* l, double* u) {
    return b2::guarded([&] { b2::gen_transport(S, D, seed, row, col, val, c, rL, rU, l, u); });
}

}  // extern "C"
