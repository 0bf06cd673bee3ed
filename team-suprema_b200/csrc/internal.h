// internal.h -- shared declarations of the host preparation (host_prep.cpp)
// and the CUDA engine (engine.cu). Not part of the C ABI.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "b200_pdlp.h"

namespace b2 {

// Error carried to the C ABI as (code, message).
struct Error {
    int code;
    std::string msg;
};
[[noreturn]] void fail(int code, const std::string& msg);
void set_last_error(const std::string& msg);

// Whether the caller asked a running solve to stop: its stop word or its
// stop callback (b2_solve_opts::stop_poll).
inline bool stop_requested(const b2_solve_opts& o, const volatile int32_t* stop_flag) {
    if (stop_flag && *stop_flag) return true;
    return o.stop_poll && o.stop_poll(o.stop_ctx) != 0;
}

// Sliced ELL with a per-slice lane count ("lanes per row", g = 1..32).
//
// A slice is one warp's unit of work: 32/g consecutive rows (in the permuted
// order), each row spread round-robin over g lanes. Entry e of a row lives in
// lane (row_in_slice * g + e % g) at step e / g; step k of lane l is stored at
// element 32 * (blk + k) + l, i.e. column-major inside the slice, so a warp's
// 32 lanes read 32 consecutive words per step. len = steps of the slice.
// slice[s] = {row0, len | (log2 g) << 27, blk, 0}.
struct SellHost {
    int32_t n_rows = 0, n_cols = 0;
    std::vector<int32_t> slice;       // 4 ints per slice
    std::vector<uint32_t> col;        // padded, 32 * total blocks
    std::vector<float> val32;
    std::vector<double> val64;        // only when values are not exact in FP32
    int64_t padded = 0;               // stored entries including padding
    // split slices: per group {segments, first segment slot}; slice.w of a
    // segment = group + 1 | segment << 24 (0: unsplit)
    std::vector<int32_t> seg;
    int64_t seg_slots = 0;            // segments in all groups (32 partial sums each)
    int32_t seg_max = 0;              // most segments in one group
    // dense runs (whole-GPU layout): per slice record {c0, ks} when lane l
    // of step k holds column c0 + k * ks + l for every stored entry (and
    // that index is a column for every padding entry), else {-1, 0}; empty
    // when no record is one
    std::vector<int32_t> aff;
    int64_t n_dense = 0;
    int64_t n_slices() const { return (int64_t)slice.size() / 4; }
    int64_t n_groups() const { return (int64_t)seg.size() / 2; }
};

constexpr int kLenBits = 27;
constexpr uint32_t kLenMask = (1u << kLenBits) - 1;

// Everything the device needs, in device (permuted) order.
struct Layout {
    int32_t m = 0, n = 0;
    int64_t nnz = 0;
    std::vector<int32_t> perm_r;      // device row i  -> caller row perm_r[i]
    std::vector<int32_t> perm_c;      // device col j  -> caller col perm_c[j]
    std::vector<int32_t> inv_r, inv_c;
    SellHost A, AT;
    bool exact32 = true;
    // rows
    std::vector<double> b, rU;        // b = rL of the PDLP form
    std::vector<double> dr2;          // Dr^2, negated on inequality rows
    // cols
    std::vector<double> c, l, u, x0;  // x0 = Dc * clamp(0, l_s, u_s)
    std::vector<double> dc2;          // Dc^2
    bool lu_const = false;            // every column has the bounds (l_all, u_all), bit for bit
    double l_all = 0.0, u_all = 0.0;
    // scalars
    double eta0 = 1.0, omega0 = 1.0, denom_p = 1.0, denom_d = 1.0, obj_offset = 0.0;
};

struct BuildParams {
    int lane_target = 16;   // entries per lane that decides lanes-per-row
    int sigma_window = 1024;
    // whole-GPU engine: rows of at least `tune_len` entries get the
    // lanes-per-row that touches the fewest memory sectors (cost model over
    // their actual column indices), and slices longer than `split_steps`
    // steps are split into segments that run on different warps
    bool split = false;
    int tune_len = 256;
    int split_steps = 16;
    int threads = 1;        // host threads for the layout (the one-LP engine uses several)
};

// Validates the PDLP form and builds the device layout. Throws Error.
void build_layout(const b2_lp_view& U, const b2_lp_view& S, const double* Dr, const double* Dc,
                  const BuildParams& bp, Layout& L);
uint64_t layout_digest(const Layout& L);

// The whole-grid kernel's work-balanced order of a matrix's slice records
// over `warps` warps: seq holds the record indices, warp w's records at
// seq[start[w] .. start[w + 1]). Records go costliest first to the
// least-loaded warp (ties: the lowest); a plain record costs its steps + 4, a
// dense-run record ceil(steps / dense_unroll) + 2. Inside a warp: records
// that wait for nothing (unsplit, subgroup members) first, then subgroup
// leaders (segment % sub_seg == 0), then group owners (segment 0), each in
// record order.
void schedule_records(const SellHost& S, int warps, int dense_unroll, int sub_seg, std::vector<int32_t>& seq,
                      std::vector<int32_t>& start);

// Ruiz + Pock-Chambolle on the host; the same bits with any number of threads.
void scale_lp(const b2_lp_view& lp, int ruiz_passes, double* val_s, double* c_s, double* rL_s, double* rU_s,
              double* l_s, double* u_s, double* Dr, double* Dc, int threads = 1);

// The same scaling on the GPU, bit for bit (scale.cu).
void scale_lp_gpu(const b2_lp_view& lp, int ruiz_passes, double* val_s, double* c_s, double* rL_s, double* rU_s,
                  double* l_s, double* u_s, double* Dr, double* Dc);

void gen_random_lp(int m, int n, int k, uint64_t seed, bool fp32_values, int32_t* row, int32_t* col, double* val,
                   double* c, double* rL, double* rU, double* l, double* u);
void gen_transport(int S, int D, uint64_t seed, int32_t* row, int32_t* col, double* val, double* c, double* rL,
                   double* rU, double* l, double* u);

// An LP held in owned arrays (COO), e.g. as read from a request file.
struct LpArrays {
    int32_t m = 0, n = 0;
    std::vector<int32_t> row, col;
    std::vector<double> val, c, rL, rU, l, u;
    double obj_offset = 0.0;
};

// Presolve, PDLP form and postsolve (presolve.cpp). Throw Error.
struct Presolved;
struct PdlpForm;
Presolved* presolve_lp(const b2_lp_view& original);
int32_t presolved_status(const Presolved& p);  // 0 reduced, 1 infeasible, 2 unbounded
void presolved_view(const Presolved& p, b2_lp_view& reduced);
void postsolve_lp(const Presolved& p, const double* x_red, const double* y_red, double* x, double* y);
void presolved_free(Presolved* p);
PdlpForm* pdlp_form_build(const b2_lp_view& ranged);
void pdlp_form_view(const PdlpForm& f, b2_lp_view& form);
void pdlp_form_extract(const PdlpForm& f, const double* x2, const double* y2, double* x, double* y);
void pdlp_form_free(PdlpForm* f);
// verify()'s figures on the host: out = {eps_P, eps_D, eps_G, objective}
void kkt_host(const b2_lp_view& lp, const double* x, const double* y, double* out);

// Shape classes and lane targets of batched / served LPs (batch.cu).
int32_t shape_class(int32_t m, int32_t n, int64_t nnz);
void default_tune_table(b2_tune_table& t);
// The lane target an LP of this shape gets under these options.
int lane_target_for(const b2_solve_opts& o, int32_t m, int32_t n, int64_t nnz);

// The binary request format (lp_io.cpp). All functions throw Error.
void lp_write(const std::string& path, const b2_lp_view& lp);
void lp_read_dims(const std::string& path, int32_t* m, int32_t* n, int64_t* nnz);
void lp_read(const std::string& path, LpArrays& out);

// The CUDA engine (engine.cu). All functions throw Error.
struct EngineImpl;
EngineImpl* engine_create(const b2_lp_view& U, const b2_lp_view& S, const double* Dr, const double* Dc,
                          const b2_solve_opts& o);
void engine_destroy(EngineImpl* e);
void engine_solve(EngineImpl* e, const b2_solve_opts& o, const volatile int32_t* stop, double* x, double* y,
                  b2_result* r);
void engine_info(EngineImpl* e, b2_engine_info* info);
void engine_spmv(EngineImpl* e, int which, const double* x, double* y);
int engine_trace(EngineImpl* e, double* out, int max_records);
void engine_spmv_bench(EngineImpl* e, int which, int precision, int reps, void* stream, double* avg_ms);
// An engine over a layout built beforehand (build_layout), and the
// time-sliced form of engine_solve used by the served stream: begin, slices of
// about slice_ms of device time (true when the solve has ended), finish.
EngineImpl* engine_create_from_layout(Layout&& L);
size_t engine_bytes(EngineImpl* e);
void engine_begin_slices(EngineImpl* e, const b2_solve_opts& o);
bool engine_slice(EngineImpl* e, const b2_solve_opts& o, double slice_ms, void* stream);
void engine_finish_slices(EngineImpl* e, double* x, double* y, b2_result* r);

// The allocation-free one-CTA solve (noalloc.cu). Throws Error.
void solve_noalloc(const b2_lp_view& U, const b2_lp_view& S, const double* Dr, const double* Dc,
                   const b2_solve_opts& o, double* x_out, double* y_out, b2_result* res);

// The batched engine (batch.cu). All functions throw Error.
struct BatchImpl;
BatchImpl* batch_create(int n, const b2_lp_view* U, const b2_lp_view* S, const double* const* Dr,
                        const double* const* Dc, const b2_solve_opts& o);
void batch_destroy(BatchImpl* b);
void batch_solve(BatchImpl* b, const b2_solve_opts& o, const volatile int32_t* stop, b2_result* res, double* ms);
void batch_solution(BatchImpl* b, int i, double* x, double* y);
void batch_info(BatchImpl* b, b2_batch_info* inf);
void batch_spmv(BatchImpl* b, int i, int which, const double* x, double* y);
void batch_autotune(int n, const b2_lp_view* U, const b2_lp_view* S, const double* const* Dr, const double* const* Dc,
                    const b2_solve_opts& o, b2_tune_table& out);

// The served stream (serve.cu). All functions throw Error.
struct ServerImpl;
ServerImpl* server_create(const b2_server_opts& so, const b2_solve_opts& o);
void server_destroy(ServerImpl* s);
int64_t server_submit(ServerImpl* s, const b2_lp_view& U);
int64_t server_submit_file(ServerImpl* s, const std::string& path);
int64_t server_submit_lp(ServerImpl* s, const b2_lp_view& original, bool presolve);
int server_wait(ServerImpl* s, int64_t ticket, double timeout_s, double* x, double* y, b2_result* res,
                b2_request_info* info);
void server_stats(ServerImpl* s, b2_server_stats* out);
int64_t server_backlog(ServerImpl* s);  // b2_server_stats.backlog_work

// Shares over several GPUs (pool.cpp). All functions throw Error.
int64_t request_work(int32_t m, int32_t n, int64_t nnz);
int64_t request_cost(int32_t m, int32_t n, int64_t nnz);
void shard_plan(const int64_t* work, int64_t count, int32_t parts, bool online, int32_t* rank_of);
struct PoolImpl;
PoolImpl* pool_create(const int32_t* devices, int32_t count, const b2_server_opts& so, const b2_solve_opts& o);
void pool_destroy(PoolImpl* p);
int64_t pool_submit(PoolImpl* p, const b2_lp_view& U);
int64_t pool_submit_file(PoolImpl* p, const std::string& path);
int pool_wait(PoolImpl* p, int64_t ticket, double timeout_s, double* x, double* y, b2_result* res,
              b2_request_info* info, int32_t* member);
void pool_stats(PoolImpl* p, int32_t member, b2_server_stats* out);

}  // namespace b2
