/* b200_pdlp.h -- C ABI of the B200 PDLP engine (libb200pdlp.so).
 *
 * The engine replaces the reference solver's CUDA backend behind its GPU
 * entry point
 *
 *     PdlpResult solve_pdhg_gpu(const RangedLP& unscaled_form, const RangedLP& scaled_form,
 *                               const std::vector<double>& Dr, const std::vector<double>& Dc,
 *                               double eta, int max_iterations, int check_every, double tol,
 *                               std::atomic<bool>* stop_flag);
 *     (include/pdlp_gpu.hpp:22-25, implemented by gpu/pdlp_gpu_solve.cu:261-267)
 *
 * Everything here is plain C: pointers, sizes and int status codes; no C++
 * types and no exceptions cross it. The C++ shim that gives the reference
 * its exact solve_pdhg_gpu symbol is team-suprema_b200/csrc/shim_solve_pdhg_gpu.cpp.
 *
 * Threading: every entry point is thread-safe for distinct engines; one
 * engine must not be used by two threads at once. Errors: a non-zero return
 * is one of the B2_ERR_* codes and b2_last_error() (thread-local) says why.
 */
#ifndef B200_PDLP_H
#define B200_PDLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define B2_OK 0
#define B2_ERR_INVALID 1     /* malformed input (indices, sizes, non-PDLP form)        */
#define B2_ERR_CUDA 2        /* CUDA runtime error                                       */
#define B2_ERR_OOM 3         /* device allocation failed                                 */
#define B2_ERR_TIMEOUT 4     /* a device-side barrier wait ran out of time (kernel exits) */
#define B2_ERR_NO_DEVICE 5   /* no CUDA device                                           */
#define B2_ERR_NONFINITE 6   /* NaN / inf where a finite number is required              */
#define B2_ERR_UNSUPPORTED 7 /* request outside what this build supports                 */
#define B2_ERR_PENDING 8     /* b2_server_wait: the request has not finished yet          */
#define B2_ERR_INFEASIBLE 9  /* presolve proved the LP infeasible                          */
#define B2_ERR_UNBOUNDED 10  /* presolve proved the LP unbounded                           */

/* ---- one LP, as the reference's RangedLP holds it ---------------------
 * rL <= A x <= rU, l <= x <= u, minimise c'x + obj_offset; A in COO
 * (SparseMatrix, include/sparse.hpp:14-22; RangedLP, include/ranged_lp.hpp:10-27). */
typedef struct b2_lp_view {
    int32_t m, n;
    int64_t nnz;
    const int32_t* row_idx;
    const int32_t* col_idx;
    const double* val;
    const double* c;
    const double* rL;
    const double* rU;
    const double* l;
    const double* u;
    double obj_offset;
} b2_lp_view;

/* ---- solve options ---------------------------------------------------- */
#define B2_PREC_FP64 0   /* FP64 iterates and accumulation throughout                       */
#define B2_PREC_MIXED 1  /* FP32 iterates / SpMV first, then FP64 iterates to `tol` (default) */

typedef struct b2_solve_opts {
    int32_t max_iterations;   /* attempts, counted as include/pdlp_algo.hpp:103-108      */
    int32_t check_every;      /* accepted steps between KKT checks (callers pass 64)      */
    double tol;               /* max(eps_P, eps_D, eps_G) on the unscaled PDLP form       */
    int32_t precision;        /* B2_PREC_*                                                 */
    double switch_tol;        /* MIXED: KKT level at which FP32 iterates hand over to FP64 */
    int32_t stall_checks;     /* MIXED: checks without a new best point before handing over */
    double time_limit_s;      /* <= 0: none. Device-side wall clock; exits like stop_flag  */
    double barrier_timeout_s; /* <= 0: 10 s. Bound on every device-side wait               */
    int32_t max_ctas;         /* <= 0: auto (co-resident CTAs of the persistent kernel)     */
    int32_t lane_target;      /* <= 0: auto. Entries per lane that picks lanes-per-row      */
    int32_t sigma_window;     /* <= 0: auto. Rows per sigma-sort window of the sliced format */
    int32_t return_current;   /* debug: return the current iterate, not the chosen/best    */
    void* stream;             /* cudaStream_t to launch on; NULL: the engine's own stream  */
    int32_t debug_delay_us;   /* test hook: CTA 0 reaches its first barrier this late (bounded),
                                 so a short barrier_timeout_s exercises the timeout path   */
    int32_t batch_cluster_nnz;/* batches: LPs with at least this many stored entries (A and A^T)
                                 are solved by a cluster of 16 CTAs; <= 0: never (default)     */
    int32_t batch_block;      /* batches: threads per CTA, 128, 256 or 512; 0: auto (512)     */
    /* Cancellation by callback, for callers whose stop flag is not a plain
       int32 word (the shim passes a reader of the reference's std::atomic<bool>):
       while a one-LP solve or a batch runs, the calling thread's wait loop calls
       stop_poll(stop_ctx) about every 20 us; a nonzero return stops the solve as
       a set stop_flag does. NULL: not used. */
    int32_t (*stop_poll)(void* stop_ctx);
    void* stop_ctx;
    /* Batches and served LPs: lanes-per-row target per shape class
       (b2_shape_class); NULL: the built-in table (b2_default_tune_table).
       An explicit lane_target > 0 overrides both. Read while b2_batch_create
       runs; a server copies it at b2_server_create. */
    const struct b2_tune_table* tune;
    /* Batches, the tail lane: > 0 -- an LP still running at this many attempts
       yields there, and once the one-CTA launch is done the yielded LPs finish
       on 16-CTA clusters on the whole GPU (a second launch). The switch point
       depends on the LP alone, so answers stay deterministic, but such an LP's
       bits differ from its solve on one CTA (the group size sets the order of
       its reductions). <= 0: off (default). Not with batch_cluster_nnz. */
    int32_t batch_tail_attempts;
    /* Whole-GPU engine, rows of 256+ entries: 0 -- the lanes per row that touch
       the fewest memory sectors (a cost model over the rows' own columns);
       1 -- the length rule of all other rows (lane_target). Read at create. */
    int32_t long_rows;
} b2_solve_opts;

/* ---- shape classes and the autotuner --------------------------------------
 * No counterpart in the reference. The sliced layout of a batched or served LP
 * spreads each row over g lanes, g the smallest power of two with
 * ceil(len / g) <= lane target; the lane target thus sets the rows per warp
 * (32 / g) and the steps per slice. b2_shape_class buckets an LP by size
 * (nonzeros: < 4K, < 16K, < 64K, < 256K, more) and entries per row (< 8, < 16,
 * < 32, more); b2_batch_autotune times, per class present in the given LPs, a
 * few of its LPs on one CTA each (512 FP64 attempts) under lane targets 4, 8,
 * 16 and 32 and keeps the fastest (16 unless another is 3 % faster). The table
 * is data: solves with a given table are deterministic, and the built-in one
 * came from this tuner run on a B200 over the batch family. */
#define B2_TUNE_CLASSES 20
typedef struct b2_tune_table {
    int32_t lane_target[B2_TUNE_CLASSES];    /* 0: class not tuned, 16 applies */
    double us_per_attempt[B2_TUNE_CLASSES];  /* the chosen target's measured time (0: not measured) */
} b2_tune_table;
int32_t b2_shape_class(int32_t m, int32_t n, int64_t nnz);
void b2_default_tune_table(struct b2_tune_table* out);

void b2_default_opts(b2_solve_opts* opts);

/* ---- result ------------------------------------------------------------
 * Mirrors PdlpResult (include/pdlp.hpp:18-24) plus engine counters. x/y are
 * written to caller buffers in unscaled PDLP-form space (x = Dc*x_s, y = Dr*y_s). */
#define B2_EXIT_CONVERGED 1
#define B2_EXIT_MAX_ITER 2
#define B2_EXIT_STOPPED 3
#define B2_EXIT_TIME_LIMIT 4

typedef struct b2_result {
    int32_t iterations;    /* attempts, as PdlpResult::iterations */
    int32_t restarts;
    int32_t converged;
    int32_t accepted;      /* accepted PDHG steps                  */
    double eps_P, eps_D, eps_G;
    double objective;      /* c'x + obj_offset of the returned point (PDLP form) */
    int32_t exit_reason;   /* B2_EXIT_*                            */
    int32_t checks;        /* KKT checks performed on the device   */
    int32_t fp32_attempts; /* attempts run with FP32 iterates      */
    int32_t fp32_accepted;
    double device_ms;      /* persistent-kernel time (CUDA events)  */
    double host_ms;        /* whole call, host clock                */
    double final_eta, final_omega;
    int32_t group_ctas;    /* CTAs that solved this LP together: 1, a cluster, or the whole launch */
} b2_result;

/* Drop-in for solve_pdhg_gpu (include/pdlp_gpu.hpp:22-25): same inputs in the
 * same order, `eta` ignored (adaptive, as gpu/pdlp_gpu_solve.cu:263), stop_flag
 * polled by the device about every 16 attempts (may be NULL). x_out (n) and
 * y_out (m) receive the returned point. Uses the default options above. */
int b2_solve_pdhg_gpu(const b2_lp_view* unscaled_form, const b2_lp_view* scaled_form, const double* Dr,
                      const double* Dc, double eta, int32_t max_iterations, int32_t check_every, double tol,
                      const volatile int32_t* stop_flag, double* x_out, double* y_out, b2_result* res);

/* Same, with explicit options (max_iterations / check_every / tol taken from opts). */
int b2_solve_pdhg_gpu_ex(const b2_lp_view* unscaled_form, const b2_lp_view* scaled_form, const double* Dr,
                         const double* Dc, const b2_solve_opts* opts, const volatile int32_t* stop_flag,
                         double* x_out, double* y_out, b2_result* res);

/* Allocation-free form of b2_solve_pdhg_gpu_ex (no counterpart in the
 * reference). For callers that must not allocate device memory: a process
 * whose GPU memory is reserved up front by another runtime's allocator or a
 * pool it does not own (so a cudaMalloc from this library would fail or
 * fragment that pool), and latency-critical paths that must stay out of the
 * driver's allocator. It runs the one-CTA solve with its whole device working
 * set (layout, iterates, averages, control state, outputs) in one static
 * device array of 32 MiB; LPs that need more (roughly above 200,000
 * nonzeros) get B2_ERR_UNSUPPORTED before any GPU work. It calls no
 * cudaMalloc / cudaFree or other allocating CUDA routine (host memory is
 * still used to build the layout). The array's memory: with CUDA's lazy
 * module loading (the default since CUDA 12.2) a device gets it at the first
 * call on that device, when the call looks up the array's address
 * (cudaGetSymbolAddress) with that device current, and keeps it until the
 * process exits; with eager loading (CUDA_MODULE_LOADING=EAGER) every device
 * gets it when the library is loaded, whether or not this entry point is
 * used. Make the first call on a device before any stream capture begins.
 * The work is issued on the legacy default stream with synchronous copies
 * and the call returns after its GPU work ends. All calls in the process
 * share the array, which keeps the previous call's contents (each call
 * clears what must start at zero); calls are serialized by a process-wide
 * lock, since GPU work of two calls that overlapped would race on the array.
 * Inputs, outputs and options mean what they mean for b2_solve_pdhg_gpu_ex,
 * except that stop_flag, time limit and stream are not supported. */
int b2_solve_pdhg_gpu_noalloc(const b2_lp_view* unscaled_form, const b2_lp_view* scaled_form, const double* Dr,
                              const double* Dc, const b2_solve_opts* opts, double* x_out, double* y_out,
                              b2_result* res);

/* ---- resident engine: upload once, solve many times ---------------------
 * b2_engine_create does what the reference's GpuBackend constructor does
 * (gpu/pdlp_gpu_solve.cu:198-205): builds the device layout of A and A^T and
 * uploads the problem. b2_engine_solve then runs from HBM-resident data.
 * Engine memory (and so that of b2_solve_pdhg_gpu, which makes an engine per
 * call) comes from the device's default stream-ordered memory pool, whose
 * release threshold is raised so that freed blocks stay cached for the next
 * engine; cudaMemPoolTrimTo on that pool hands them back to the driver. */
typedef struct b2_engine b2_engine;

int b2_engine_create(const b2_lp_view* unscaled_form, const b2_lp_view* scaled_form, const double* Dr,
                     const double* Dc, const b2_solve_opts* opts, b2_engine** out);
int b2_engine_solve(b2_engine* e, const b2_solve_opts* opts, const volatile int32_t* stop_flag, double* x_out,
                    double* y_out, b2_result* res);
void b2_engine_destroy(b2_engine* e);

typedef struct b2_engine_info {
    int32_t m, n;
    int64_t nnz;
    int64_t a_slices, at_slices;
    int64_t a_padded, at_padded;   /* stored entries incl. padding */
    int32_t values_exact_fp32;     /* 1: A's values are exact in FP32 (no FP64 copy kept) */
    int32_t ctas, threads_per_cta; /* persistent-kernel launch shape */
    int32_t sm_count;
    int64_t device_bytes;          /* HBM held by the engine */
} b2_engine_info;
int b2_engine_get_info(b2_engine* e, b2_engine_info* info);

/* y = A x (which = 0) or y = A^T x (which = 1) through the engine's device
 * SpMV (stored values, FP64 accumulation); x and y in the caller's order. */
int b2_engine_spmv(b2_engine* e, int32_t which, const double* x, double* y);

/* Times `reps` launches of the standalone SpMV kernel on resident data with
 * CUDA events on `stream` (NULL: the engine's stream). precision: B2_PREC_MIXED
 * times FP32 x/y, B2_PREC_FP64 times FP64 x/y (FP32 values either way when
 * they are exact). avg_ms receives the mean time per launch. */
int b2_engine_spmv_bench(b2_engine* e, int32_t which, int32_t precision, int32_t reps, void* stream,
                         double* avg_ms);

/* Per-check records of the engine's last solve, B2_TRACE_FIELDS doubles each:
 * attempts, accepted, eps_P/eps_D/eps_G of the current point, the same of the
 * average point, primal weight, step size, flags (1 restart, 2 restart to the
 * average, 4 FP32 iterates, 8/16 new best = current/average), weight of the
 * average. At most max_records are copied; *count receives how many. */
#define B2_TRACE_FIELDS 12
int b2_engine_trace(b2_engine* e, double* out, int32_t max_records, int32_t* count);

/* ---- batches: many LPs of uneven size in one persistent launch -----------
 * No counterpart in the reference, which solves one LP per call; each LP of a
 * batch is the same solve as b2_solve_pdhg_gpu on that LP (same inputs, same
 * options, bit-identical answer), run by one CTA that takes the next LP from
 * a device work queue when it finishes. unscaled[i], scaled[i], Dr[i], Dc[i]
 * describe LP i exactly as for b2_solve_pdhg_gpu. */
typedef struct b2_batch b2_batch;

typedef struct b2_batch_info {
    int32_t n_lp;
    int64_t sum_m, sum_n, sum_nnz, sum_padded;
    int32_t max_ctas, threads_per_cta;
    int64_t device_bytes;
    int32_t last_launch_ctas;      /* CTAs the last b2_batch_solve launched (both lanes) */
} b2_batch_info;

int b2_batch_create(int32_t n_lp, const b2_lp_view* unscaled, const b2_lp_view* scaled, const double* const* Dr,
                    const double* const* Dc, const b2_solve_opts* opts, b2_batch** out);
/* The autotuner (see b2_shape_class): fills `out` for the classes present in
 * the given LPs (others 0). Runs batches on the current GPU. */
int b2_batch_autotune(int32_t n_lp, const b2_lp_view* unscaled, const b2_lp_view* scaled, const double* const* Dr,
                      const double* const* Dc, const b2_solve_opts* opts, b2_tune_table* out);
/* Solves every LP of the batch; results[i] receives LP i's result (device_ms =
 * that LP's time on its CTA); *total_ms the whole launch (CUDA events). */
int b2_batch_solve(b2_batch* b, const b2_solve_opts* opts, const volatile int32_t* stop_flag, b2_result* results,
                   double* total_ms);
/* Copies LP i's returned point (unscaled PDLP-form space) of the last solve. */
int b2_batch_get_solution(b2_batch* b, int32_t i, double* x, double* y);
int b2_batch_get_info(b2_batch* b, b2_batch_info* info);
/* y = A x (which = 0) or A^T x (which = 1) of LP i through the batch's packed
 * device layout (FP64 accumulation); x, y in that LP's caller order. */
int b2_batch_spmv(b2_batch* b, int32_t i, int32_t which, const double* x, double* y);
void b2_batch_destroy(b2_batch* b);

/* ---- served stream: LPs arriving over time, continuous batching ----------
 * No counterpart in the reference, which solves one LP per call. A server
 * owns one GPU (the current device at creation) and three kinds of threads:
 * callers submit LPs and wait for tickets; preparation threads scale each LP
 * (Ruiz + Pock-Chambolle as src/scaling.cpp:25-84) and lay it out; one loop
 * thread admits prepared LPs, oldest first, while their device footprint fits
 * the HBM budget, uploads them while the GPU works, and runs rounds of the
 * batched kernel over every resident LP. A round lasts about round_ms of
 * device time; LPs still running then pause at an attempt boundary with
 * their state left on the device and go on in the next round, which also
 * takes in whatever arrived meanwhile. Each LP is solved by one CTA exactly
 * as one b2_batch LP is: its answer is bit-identical whatever else is in
 * flight. LPs with at least grid_nnz nonzeros are solved one at a time by the
 * whole GPU (the b2_engine solve), in slices of grid_slice_ms between rounds.
 * Every answer carries the engine's device-side KKT figures (the restatement
 * of the reference's verify(), src/verify.cpp:24-103). */
typedef struct b2_server b2_server;

typedef struct b2_server_opts {
    double hbm_budget_bytes;  /* device bytes resident LPs may hold; <= 0: 150e9       */
    double round_ms;          /* device time of one batched round; <= 0: 5 ms           */
    int32_t max_resident;     /* LPs resident at once (batched lane); <= 0: 65536       */
    int32_t prep_threads;     /* host preparation threads; <= 0: hardware threads (<=16) */
    int64_t grid_nnz;         /* nonzeros from which an LP takes the whole-GPU lane; <= 0: 4,000,000 */
    double grid_slice_ms;     /* device time of one whole-GPU slice; <= 0: 20 ms        */
    int64_t cluster_nnz;      /* stored entries (A and A^T) from which a batched LP is solved by
                                 a cluster of 16 CTAs; 0: 300,000; < 0: never             */
    int64_t gpu_scale_nnz;    /* nonzeros from which an LP is scaled on the GPU (b2_scale_gpu,
                                 the same bits); 0: 1,000,000; < 0: never                */
} b2_server_opts;

typedef struct b2_request_info {
    double submit_s, admit_s, done_s; /* server clock (seconds since creation)             */
    double prep_ms;                   /* host scaling + layout                               */
    int32_t rounds;                   /* rounds (or whole-GPU slices) the LP ran in          */
    int32_t lane;                     /* 0: batched, 1: whole GPU                            */
    int64_t device_bytes;             /* its footprint as admitted                           */
    double form_eps[3];               /* b2_server_submit_lp: eps_P/D/G of the PDLP form (device) */
    int32_t presolved_m, presolved_n; /* b2_server_submit_lp: the PDLP form's size           */
} b2_request_info;

typedef struct b2_server_stats {
    int64_t submitted, completed, failed;
    int64_t rounds, grid_slices;
    int32_t resident, queued;
    int64_t bytes_in_use, peak_bytes;
    double busy_ms;                   /* device time of rounds and slices                    */
    int64_t backlog_work;             /* sum of b2_request_work() over requests not finished  */
} b2_server_stats;

/* opts: solve options for every request (tol, precision, max_iterations, ...);
 * NULL: b2_default_opts. sopts NULL: all defaults. */
int b2_server_create(const b2_server_opts* sopts, const b2_solve_opts* opts, b2_server** out);
/* Submits one LP in unscaled PDLP form (as solve_pdhg_gpu's unscaled_form: rows
 * `=` or `>=`); the server copies it and returns at once with a ticket. */
int b2_server_submit(b2_server* s, const b2_lp_view* unscaled_form, int64_t* ticket);
/* Submits an LP stored in the binary request format (b2_lp_write); the file
 * is read and checked on the server's preparation threads, not the caller's.
 * A file that cannot be read or is malformed fails its ticket. */
int b2_server_submit_file(b2_server* s, const char* path, int64_t* ticket);
/* Submits an LP as the caller has it (a ranged LP, any row and column
 * bounds), as src/solve.cpp:150-195 prepares one for PDLP: on the server's
 * preparation threads it is presolved (when presolve != 0; b2_presolve),
 * put in PDLP form (b2_pdlp_form_build) and scaled. The answer b2_server_wait
 * hands over is the original LP's point (x: n, y: m of this LP), mapped back
 * by extract and postsolve; res->objective is c'x + obj_offset of the
 * original LP and res->eps_P/D/G are verify()'s figures on the original LP,
 * computed on the host after postsolve (the PDLP form's device figures are in
 * b2_request_info.form_eps). An LP that presolve proves infeasible or
 * unbounded fails its ticket with B2_ERR_INFEASIBLE / B2_ERR_UNBOUNDED; one
 * that presolve solves outright needs no GPU work. */
int b2_server_submit_lp(b2_server* s, const b2_lp_view* original, int32_t presolve, int64_t* ticket);
/* Waits up to timeout_s seconds (< 0: no limit) for a ticket. On B2_OK the
 * result is handed over (x: n, y: m in unscaled PDLP-form space, any may be
 * NULL) and the ticket is forgotten; B2_ERR_PENDING: not finished yet. A
 * request that failed returns its error code, once. */
int b2_server_wait(b2_server* s, int64_t ticket, double timeout_s, double* x, double* y, b2_result* res,
                   b2_request_info* info);
int b2_server_stats_get(b2_server* s, b2_server_stats* out);
/* Stops the server: running LPs stop at their next poll, unclaimed results are
 * dropped. No other call on this server may be in progress or follow. */
void b2_server_destroy(b2_server* s);

/* ---- several GPUs: shares of a batch or a stream -------------------------
 * No counterpart in the reference (one LP, one device). LPs are independent,
 * so a batch or a stream spreads over GPUs with no exchange between them:
 * each GPU solves its own share, one process per GPU (b2_shard_plan) or one
 * process driving a server per GPU (b2_pool). The unit of load is
 * b2_request_work(m, n, nnz) = 2 nnz + m + n, the matrix entries and vector
 * elements one PDHG attempt passes over (both products, both vector passes). */
int64_t b2_request_work(int32_t m, int32_t n, int64_t nnz);

/* The expected cost of a whole solve, for shares of a batch or a stream:
 * b2_request_work times the attempts an LP of m rows takes to 1e-6, modelled
 * as round(167 m^0.657) (a fit over the 4,096 LPs of the uneven batch family,
 * m 50..5,000). Larger LPs need more attempts as well as more work per
 * attempt, so shares planned on this cost end together more closely than
 * shares planned on the work of one attempt. */
int64_t b2_request_cost(int32_t m, int32_t n, int64_t nnz);

/* Assigns `count` items of load work[i] >= 0 to `parts` shares; rank_of[i]
 * receives item i's share. online = 0 (a batch known up front): items by
 * decreasing load (equal loads by index), each to the least-loaded share
 * (longest-processing-time first). online = 1 (a stream): items in the given
 * order, each to the share with the least load so far. Equal shares go to the
 * lower index. Deterministic: every rank computes the same plan from the same
 * list, so ranks agree on their shares without a collective. */
int b2_shard_plan(const int64_t* work, int64_t count, int32_t parts, int32_t online, int32_t* rank_of);

/* A pool of servers, one per listed device, in one process. Each submit goes
 * to the member with the least unfinished work (b2_server_stats.backlog_work;
 * equal backlogs to the lower member), so work finished on a fast GPU frees it
 * for the next request. Each LP is solved exactly as by a single server, so
 * its answer does not depend on which member took it. Tickets are the pool's
 * own. devices may repeat (several servers on one GPU). */
typedef struct b2_pool b2_pool;

int b2_pool_create(const int32_t* devices, int32_t count, const b2_server_opts* sopts, const b2_solve_opts* opts,
                   b2_pool** out);
int b2_pool_submit(b2_pool* p, const b2_lp_view* unscaled_form, int64_t* ticket);
int b2_pool_submit_file(b2_pool* p, const char* path, int64_t* ticket);
/* As b2_server_wait; member (may be NULL) receives the index (into the create
 * call's device list) of the server that solved the request. */
int b2_pool_wait(b2_pool* p, int64_t ticket, double timeout_s, double* x, double* y, b2_result* res,
                 b2_request_info* info, int32_t* member);
int b2_pool_stats_get(b2_pool* p, int32_t member, b2_server_stats* out);
void b2_pool_destroy(b2_pool* p);

/* Builds the device layout of an LP on the host (no GPU) exactly as
 * b2_engine_create (whole_gpu = 1: long rows tuned and split) or a batch /
 * server LP (whole_gpu = 0) does, with `threads` host threads, and returns a
 * 64-bit digest of every byte the device would receive. The layout does not
 * depend on the thread count; this is how that is checked. */
int b2_layout_digest(const b2_lp_view* unscaled_form, const b2_lp_view* scaled_form, const double* Dr,
                     const double* Dc, int32_t threads, int32_t whole_gpu, uint64_t* digest);

/* No counterpart in the reference. The shape of that layout, for callers
 * sizing or tuning it (no GPU): slice records of A and A^T (a split slice
 * counts once per segment), stored entries with padding, split groups, and
 * dense-run records (whole_gpu = 1 only), whose columns are an arithmetic run
 * c0 + k * ks + lane: the engine computes their addresses instead of reading a
 * column stream. */
typedef struct b2_layout_stats {
    int64_t a_slices, at_slices;
    int64_t a_padded, at_padded;
    int64_t a_groups, at_groups;
    int64_t a_dense, at_dense;
} b2_layout_stats;
int b2_layout_get_stats(const b2_lp_view* unscaled_form, const b2_lp_view* scaled_form, const double* Dr,
                        const double* Dc, int32_t whole_gpu, b2_layout_stats* out);

/* ---- host-side preparation (product side, no GPU needed) ---------------- */

/* Ruiz (ruiz_passes) + Pock-Chambolle alpha=1 scaling, as scale() in
 * src/scaling.cpp:25-84 (LP case). Outputs in caller buffers: scaled values in
 * COO order (nnz), c/l/u (n), rL/rU (m), Dr (m), Dc (n). */
int b2_scale(const b2_lp_view* lp, int32_t ruiz_passes, double* val_s, double* c_s, double* rL_s, double* rU_s,
             double* l_s, double* u_s, double* Dr, double* Dc);

/* The same scaling computed on the current GPU, bit for bit equal to b2_scale
 * (and so to the reference's scale()): maxima and products are exact, and the
 * Pock-Chambolle row / column sums add entries in COO order as the host loop
 * does. For ingest of large LPs, whose host scaling takes seconds. */
int b2_scale_gpu(const b2_lp_view* lp, int32_t ruiz_passes, double* val_s, double* c_s, double* rL_s,
                 double* rU_s, double* l_s, double* u_s, double* Dr, double* Dc);

/* PDLP form of a ranged LP, as build_pdlp_form (src/pdlp.cpp:8-82) builds it:
 * equality rows first in input order, then the one-sided rows in input order
 * as A x >= b ("<=" rows negated), a ranged row as an equality with a bounded
 * slack column (entry -1) after the original columns, free rows dropped. The
 * form's arrays belong to the b2_pdlp_form; b2_pdlp_form_view points into
 * them. b2_pdlp_form_extract maps a point of the form (x2: form n, y2: form m)
 * back to the input LP (x: n, y: m), as extract_solution (src/pdlp.cpp:84-90). */
typedef struct b2_pdlp_form b2_pdlp_form;
int b2_pdlp_form_build(const b2_lp_view* ranged, b2_pdlp_form** out);
void b2_pdlp_form_view(const b2_pdlp_form* f, b2_lp_view* form);
int b2_pdlp_form_extract(const b2_pdlp_form* f, const double* x2, const double* y2, double* x, double* y);
void b2_pdlp_form_destroy(b2_pdlp_form* f);

/* Presolve of a ranged LP before the PDLP stage (the role of the reference's
 * presolve / postsolve, src/presolve.cpp:524-628; this engine's own, smaller
 * set of reductions: free and empty rows dropped, fixed and empty columns
 * fixed, singleton rows turned into bounds, repeated to a fixed point).
 * status: 0 reduced, 1 infeasible, 2 unbounded (then the reduced LP is empty).
 * b2_presolved_view points into the handle. b2_postsolve maps a point of the
 * reduced LP (x_red: reduced n, y_red: reduced m) to the original LP (x: n,
 * y: m), dual values included, so that verify() on the original LP judges it. */
typedef struct b2_presolved b2_presolved;
int b2_presolve(const b2_lp_view* original, b2_presolved** out, int32_t* status);
void b2_presolved_view(const b2_presolved* p, b2_lp_view* reduced);
int b2_postsolve(const b2_presolved* p, const double* x_red, const double* y_red, double* x, double* y);
void b2_presolved_destroy(b2_presolved* p);

/* Binary LP request format (no counterpart in the reference, which reads MPS
 * text, src/mps_reader.cpp:66-308): the LP of a b2_lp_view with A in CSR
 * (format in team-suprema_b200/csrc/lp_io.cpp). b2_lp_read_dims gives the sizes
 * to allocate; b2_lp_read fills caller buffers (row/col/val: nnz, c/l/u: n,
 * rL/rU: m) with A in COO, rows in order. A malformed file is B2_ERR_INVALID. */
int b2_lp_write(const char* path, const b2_lp_view* lp);
int b2_lp_read_dims(const char* path, int32_t* m, int32_t* n, int64_t* nnz);
int b2_lp_read(const char* path, int32_t* row, int32_t* col, double* val, double* c, double* rL, double* rU,
               double* l, double* u, double* obj_offset);

/* Synthetic LPs of the benchmark shapes (seeded, deterministic):
 * equality-form LP min c'x, Ax = b, 0 <= x <= 10, `k` distinct uniform rows per
 * column with values U[-1,1] (rounded to FP32 when fp32_values), x0 ~ U[0,5],
 * b = A x0, y0 ~ N(0,1), z0 ~ U[0,1], c = A'y0 + z0. Buffers: row/col/val
 * (n*k), c/l/u (n), rL/rU (m). */
int b2_gen_random_lp(int32_t m, int32_t n, int32_t k, uint64_t seed, int32_t fp32_values, int32_t* row,
                     int32_t* col, double* val, double* c, double* rL, double* rU, double* l, double* u);

/* Balanced transportation LP: S sources x D sinks, n = S*D arcs, m = S + D
 * equality rows, 2 unit entries per column; supplies integer U[100,1000],
 * demands an integer partition of the total, costs integer U[1,100],
 * 0 <= x < inf. Buffers: row/col/val (2n), c/l/u (n), rL/rU (m). */
int b2_gen_transport(int32_t S, int32_t D, uint64_t seed, int32_t* row, int32_t* col, double* val, double* c,
                     double* rL, double* rU, double* l, double* u);

const char* b2_last_error(void);
const char* b2_version(void);

#ifdef __cplusplus
}
#endif
#endif /* B200_PDLP_H */
