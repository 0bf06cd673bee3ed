// serve.cu -- the served stream: LPs that arrive over time, solved by
// continuous batching on one GPU (b2_server_*).
//
// No counterpart in the reference, which solves one LP per call
// (solve_pdhg_gpu, include/pdlp_gpu.hpp:22-25). Each request is the same
// restarted PDLP as one b2_batch LP (device.cuh, solve_body over one CTA), so
// its answer does not depend on what else is in flight.
//
//   submit ──> prep threads: [an LP submitted as the caller has it: presolve
//              and PDLP form (presolve.cpp)], Ruiz + Pock-Chambolle scaling
//              (src/scaling.cpp:25-84 restated in host_prep.cpp), sliced
//              layout, the LP's device image
//          ──> admission, oldest first, while the LP's device footprint fits
//              the HBM budget and a descriptor slot is free: one device region
//              per LP (stream-ordered allocation) holding its matrix, vectors,
//              iterates, averages and control state, uploaded on the copy
//              stream while the GPU works
//          ──> rounds: one launch of the batched kernel (batch.cu) over every
//              resident LP, oldest first; CTAs pull LPs from the queue and yield
//              at the first attempt boundary past the round's deadline, state
//              left in the LP's region; the next round picks every LP up
//              exactly where it stopped (MODE_CONTINUE), new arrivals join it
//          ──> an LP whose exit reason is set is finished: its point and
//              control state are copied out, its region freed, the caller woken;
//              an LP submitted as the caller has it is mapped back (extract,
//              postsolve) and its KKT figures taken on the original LP, on the
//              waiting caller's thread.
//
// LPs with at least grid_nnz nonzeros take the whole-GPU lane instead: the
// cooperative one-LP engine (engine.cu) runs them one at a time in slices of
// grid_slice_ms that alternate with the batched rounds.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"

namespace b2 {
namespace {

using Clock = std::chrono::steady_clock;

// Byte offsets of one LP's pieces inside its device region. The constant part
// (matrix, vectors, permutations, initial control state) is a prefix that is
// uploaded from one host image; iterates and sums follow and are written by
// the solve itself.
struct RegionPlan {
    static constexpr size_t kNone = ~size_t(0);
    size_t bytes = 0, image_bytes = 0;
    size_t a_slice = 0, a_col = 0, a_v32 = 0, a_v64 = kNone;
    size_t at_slice = 0, at_col = 0, at_v32 = 0, at_v64 = kNone;
    size_t b = 0, rU = 0, dr2 = 0, c = 0, l = 0, u = 0, dc2 = 0, x0 = 0, perm_r = 0, perm_c = 0, ctl = 0;
    size_t itf[11] = {}, itd[11] = {};  // x0 x1 y0 y1 ax0 ax1 ax2 aty0 aty1 x_last y_last
    size_t xsum = 0, ysum = 0, best_x = 0, best_y = 0, out_x = 0, out_y = 0;
};

struct Planner {
    size_t used = 0;
    size_t take(size_t bytes) {
        used = (used + 255) & ~size_t(255);
        const size_t o = used;
        used += std::max<size_t>(bytes, 1);
        return o;
    }
};

RegionPlan plan_region(const Layout& L) {
    Planner p;
    RegionPlan r;
    const size_t m = (size_t)L.m, n = (size_t)L.n;
    r.a_slice = p.take(L.A.slice.size() * 4);
    r.a_col = p.take(L.A.col.size() * 4);
    r.a_v32 = p.take(L.A.val32.size() * 4);
    if (!L.A.val64.empty()) r.a_v64 = p.take(L.A.val64.size() * 8);
    r.at_slice = p.take(L.AT.slice.size() * 4);
    r.at_col = p.take(L.AT.col.size() * 4);
    r.at_v32 = p.take(L.AT.val32.size() * 4);
    if (!L.AT.val64.empty()) r.at_v64 = p.take(L.AT.val64.size() * 8);
    r.b = p.take(m * 8); r.rU = p.take(m * 8); r.dr2 = p.take(m * 8);
    r.c = p.take(n * 8); r.l = p.take(n * 8); r.u = p.take(n * 8); r.dc2 = p.take(n * 8); r.x0 = p.take(n * 8);
    r.perm_r = p.take(m * 4); r.perm_c = p.take(n * 4);
    r.ctl = p.take(sizeof(dev::Ctl));
    r.image_bytes = p.used;
    const size_t len[11] = {n, n, m, m, m, m, m, n, n, n, m};
    for (int k = 0; k < 11; ++k) r.itf[k] = p.take(len[k] * 4);
    for (int k = 0; k < 11; ++k) r.itd[k] = p.take(len[k] * 8);
    r.xsum = p.take(n * 8); r.best_x = p.take(n * 8); r.out_x = p.take(n * 8);
    r.ysum = p.take(m * 8); r.best_y = p.take(m * 8); r.out_y = p.take(m * 8);
    r.bytes = (p.used + 255) & ~size_t(255);
    return r;
}

template <class T>
void put(std::vector<unsigned char>& img, size_t off, const std::vector<T>& v) {
    if (!v.empty()) std::memcpy(img.data() + off, v.data(), v.size() * sizeof(T));
}

std::vector<unsigned char> build_image(const Layout& L, const RegionPlan& r, bool fp64_only) {
    std::vector<unsigned char> img(r.image_bytes, 0);
    put(img, r.a_slice, L.A.slice); put(img, r.a_col, L.A.col); put(img, r.a_v32, L.A.val32);
    if (r.a_v64 != RegionPlan::kNone) put(img, r.a_v64, L.A.val64);
    put(img, r.at_slice, L.AT.slice); put(img, r.at_col, L.AT.col); put(img, r.at_v32, L.AT.val32);
    if (r.at_v64 != RegionPlan::kNone) put(img, r.at_v64, L.AT.val64);
    put(img, r.b, L.b); put(img, r.rU, L.rU); put(img, r.dr2, L.dr2);
    put(img, r.c, L.c); put(img, r.l, L.l); put(img, r.u, L.u); put(img, r.dc2, L.dc2); put(img, r.x0, L.x0);
    put(img, r.perm_r, L.perm_r); put(img, r.perm_c, L.perm_c);
    dev::Ctl c;
    init_ctl(c, L, fp64_only);
    std::memcpy(img.data() + r.ctl, &c, sizeof(c));
    return img;
}

template <class T>
dev::Bufs<T> region_bufs(unsigned char* base, const size_t (&o)[11]) {
    dev::Bufs<T> B;
    auto at = [&](int k) { return reinterpret_cast<T*>(base + o[k]); };
    B.x[0] = at(0); B.x[1] = at(1); B.y[0] = at(2); B.y[1] = at(3);
    B.ax[0] = at(4); B.ax[1] = at(5); B.ax[2] = at(6);
    B.aty[0] = at(7); B.aty[1] = at(8);
    B.x_last = at(9); B.y_last = at(10);
    return B;
}

// Everything the server keeps of a prepared LP besides its image.
struct LpMeta {
    int32_t m = 0, n = 0;
    int64_t nnz = 0, a_slices = 0, at_slices = 0;
    bool exact32 = true;
    double denom_p = 1.0, denom_d = 1.0;
    bool lu_const = false;
    double l_all = 0.0, u_all = 0.0;
};

dev::LpDev region_desc(unsigned char* base, const RegionPlan& r, const LpMeta& M) {
    dev::LpDev d;
    std::memset(&d, 0, sizeof(d));
    auto D = [&](size_t off) { return reinterpret_cast<double*>(base + off); };
    d.m = M.m; d.n = M.n;
    d.A.n_rows = M.m; d.A.n_slices = (int)M.a_slices;
    d.A.slice = reinterpret_cast<const int4*>(base + r.a_slice);
    d.A.col = reinterpret_cast<const uint32_t*>(base + r.a_col);
    d.A.v32 = reinterpret_cast<const float*>(base + r.a_v32);
    d.A.v64 = r.a_v64 == RegionPlan::kNone ? nullptr : D(r.a_v64);
    d.AT.n_rows = M.n; d.AT.n_slices = (int)M.at_slices;
    d.AT.slice = reinterpret_cast<const int4*>(base + r.at_slice);
    d.AT.col = reinterpret_cast<const uint32_t*>(base + r.at_col);
    d.AT.v32 = reinterpret_cast<const float*>(base + r.at_v32);
    d.AT.v64 = r.at_v64 == RegionPlan::kNone ? nullptr : D(r.at_v64);
    d.b = D(r.b); d.rU = D(r.rU); d.dr2 = D(r.dr2);
    d.c = D(r.c); d.l = D(r.l); d.u = D(r.u); d.dc2 = D(r.dc2); d.x0 = D(r.x0);
    d.perm_r = reinterpret_cast<const int32_t*>(base + r.perm_r);
    d.perm_c = reinterpret_cast<const int32_t*>(base + r.perm_c);
    d.itf = region_bufs<float>(base, r.itf);
    d.itd = region_bufs<double>(base, r.itd);
    d.xsum = D(r.xsum); d.ysum = D(r.ysum); d.best_x = D(r.best_x); d.best_y = D(r.best_y);
    d.out_x = D(r.out_x); d.out_y = D(r.out_y);
    d.ctl = reinterpret_cast<dev::Ctl*>(base + r.ctl);
    d.denom_p = M.denom_p; d.denom_d = M.denom_d;
    d.exact32 = M.exact32 ? 1 : 0;
    d.lu_const = M.lu_const ? 1 : 0; d.l_all = M.l_all; d.u_all = M.u_all;
    return d;
}

enum ReqState { RQ_SUBMITTED = 0, RQ_PREPARED = 1, RQ_RESIDENT = 2, RQ_DONE = 3 };

struct Request {
    int64_t ticket = 0;
    std::string path;  // a request file, read on a preparation thread
    // b2_server_submit_lp: the LP as the caller has it, its presolve and its
    // PDLP form; the fields below then hold the PDLP form
    bool ranged = false, do_presolve = false, trivial = false;
    LpArrays orig;
    std::unique_ptr<Presolved, void (*)(Presolved*)> pre{nullptr, presolved_free};
    std::unique_ptr<PdlpForm, void (*)(PdlpForm*)> form{nullptr, pdlp_form_free};
    // the LP as submitted (unscaled PDLP form)
    int32_t m = 0, n = 0;
    std::vector<int32_t> row, col;
    std::vector<double> val, c, rL, rU, l, u;
    double obj_offset = 0.0;
    // prepared
    bool grid = false;
    bool cluster = false;  // batched lane, solved by a cluster of CTAs
    LpMeta meta;
    RegionPlan plan;
    std::vector<unsigned char> image;
    Layout layout;  // whole-GPU lane only (moved into its engine)
    // device
    unsigned char* region = nullptr;
    int slot = -1;
    EngineImpl* eng = nullptr;
    size_t dev_bytes = 0;
    uint64_t admit_seq = 0;
    // outcome
    int state = RQ_SUBMITTED;
    int err = 0;
    std::string err_msg;
    b2_result res{};
    std::vector<double> x, y;
    double t_submit = 0, t_prepared = 0, t_admit = 0, t_done = 0, prep_ms = 0;
    int rounds = 0;
    int qpos = -1;
    int64_t work = 0;  // request_work() of the LP, counted in the server's backlog until done
};

// Pinned staging for the copies out of finished LPs, so that one round's
// copies are issued back to back and waited for once.
struct Staging {
    unsigned char* p = nullptr;
    size_t cap = 0, used = 0;
    void reserve(size_t bytes) {
        if (bytes <= cap) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        cuda_ok(cudaHostAlloc((void**)&p, bytes, cudaHostAllocDefault), "cudaHostAlloc");
        cap = bytes;
    }
    ~Staging() {
        if (p) cudaFreeHost(p);
    }
};

}  // namespace

struct ServerImpl {
    b2_tune_table tune_copy{};
    b2_server_opts so{};
    b2_solve_opts o{};
    int device = 0, sm_count = 0, nt = 512, max_ctas = 0, max_clusters = 0, capacity = 0;
    BatchShape shape{};
    cudaStream_t cs = nullptr, cs2 = nullptr, ds = nullptr;  // compute (clusters, single CTAs), copies
    cudaEvent_t ev_small = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_copy = nullptr;
    cudaMemPool_t pool = nullptr;
    // device tables of the batched lane
    dev::BatchArgs args{};
    dev::LpDev* d_lps = nullptr;
    std::vector<void*> allocs;
    int* h_stop = nullptr;
    int* d_stop = nullptr;
    std::vector<int> free_slots;
    Staging stage;
    // requests
    std::mutex mu;
    std::condition_variable cv_prep, cv_loop, cv_done;
    std::deque<Request*> prep_q, admit_q;
    std::unordered_map<int64_t, Request*> reqs;
    std::vector<Request*> resident;       // batched lane, in admission order
    std::deque<Request*> grid_resident;   // whole-GPU lane, in admission order
    int64_t next_ticket = 1;
    uint64_t admit_counter = 0;
    size_t bytes_in_use = 0, peak_bytes = 0;
    bool stopping = false;
    int fatal = 0;
    std::string fatal_msg;
    b2_server_stats st{};
    Clock::time_point t_origin = Clock::now();
    std::vector<std::thread> preppers;
    std::thread loop;

    double now_s() const { return std::chrono::duration<double>(Clock::now() - t_origin).count(); }

    template <class T>
    T* dalloc_keep(size_t n) {
        size_t dummy = 0;
        T* p = dalloc<T>(n, dummy);
        allocs.push_back(p);
        return p;
    }

    void create(const b2_server_opts& sopt, const b2_solve_opts& opt) {
        so = sopt;
        o = opt;
        if (opt.tune) {  // the server keeps its own copy of the caller's table
            tune_copy = *opt.tune;
            o.tune = &tune_copy;
        }
        if (so.hbm_budget_bytes <= 0) so.hbm_budget_bytes = 150e9;
        if (so.round_ms <= 0) so.round_ms = 5.0;
        if (so.max_resident <= 0) so.max_resident = 65536;
        if (so.prep_threads <= 0) so.prep_threads = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        if (so.grid_nnz <= 0) so.grid_nnz = 4000000;
        if (so.grid_slice_ms <= 0) so.grid_slice_ms = 20.0;
        if (so.cluster_nnz == 0) so.cluster_nnz = 300000;
        if (so.gpu_scale_nnz == 0) so.gpu_scale_nnz = 1000000;
        if (o.max_iterations < 0) fail(B2_ERR_INVALID, "max_iterations < 0");
        nt = o.batch_block == 128 || o.batch_block == 256 ? o.batch_block : 512;
        capacity = so.max_resident;
        int ndev = 0;
        cuda_ok(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
        if (ndev == 0) fail(B2_ERR_NO_DEVICE, "no CUDA device");
        cuda_ok(cudaGetDevice(&device), "cudaGetDevice");
        cuda_ok(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device), "attr");
        cuda_ok(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_ok(cudaStreamCreateWithFlags(&ds, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_ok(cudaStreamCreateWithFlags(&cs2, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_ok(cudaEventCreateWithFlags(&ev_small, cudaEventDisableTiming), "event");
        cuda_ok(cudaEventCreate(&ev0), "event");
        cuda_ok(cudaEventCreate(&ev1), "event");
        cuda_ok(cudaEventCreateWithFlags(&ev_copy, cudaEventDisableTiming), "event");
        cuda_ok(cudaDeviceGetDefaultMemPool(&pool, device), "cudaDeviceGetDefaultMemPool");
        uint64_t keep = ~uint64_t(0);  // keep freed regions in the pool for the next LPs
        cuda_ok(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
        batch_kernel_shape(sm_count, shape);
        max_ctas = shape.max_ctas_nt[batch_nt_index(nt)];
        dev::BatchArgs& B = args;
        d_lps = dalloc_keep<dev::LpDev>(capacity);
        B.lps = d_lps;
        B.order = dalloc_keep<int>(capacity);
        B.next = dalloc_keep<unsigned>(1);
        B.order_large = dalloc_keep<int>(capacity);
        B.next_large = dalloc_keep<unsigned>(1);
        B.n_large = 0;
        max_clusters = shape.max_clusters_nt[batch_nt_index(nt)];
        B.cl_slot = dalloc_keep<int>(std::max(1, max_clusters));
        B.cl_scratch = dalloc_keep<double>((size_t)std::max(1, max_clusters) * dev::kClusterScratch);
        B.scratch = dalloc_keep<double>((size_t)max_ctas * 8);
        B.qstatus = dalloc_keep<int>(2 * (size_t)capacity);
        B.abort = dalloc_keep<int>(1);
        B.t_start = dalloc_keep<unsigned long long>(capacity);
        B.t_end = dalloc_keep<unsigned long long>(capacity);
        B.t0 = dalloc_keep<unsigned long long>(1);
        cuda_ok(cudaHostAlloc((void**)&h_stop, sizeof(int), cudaHostAllocMapped), "cudaHostAlloc");
        *h_stop = 0;
        cuda_ok(cudaHostGetDevicePointer((void**)&d_stop, h_stop, 0), "cudaHostGetDevicePointer");
        B.host_stop = d_stop;
        B.tol = o.tol;
        B.switch_tol = o.switch_tol;
        B.time_limit_ns = 0.0;
        B.max_iterations = o.max_iterations;
        B.check_every = std::max(1, o.check_every);
        B.stall_checks = o.stall_checks > 0 ? o.stall_checks : 32;
        B.mixed = o.precision == B2_PREC_MIXED;
        B.round_ns = (unsigned long long)(so.round_ms * 1e6);
        cuda_ok(cudaMemset(B.abort, 0, sizeof(int)), "memset");
        cuda_ok(cudaDeviceSynchronize(), "server create");
        free_slots.reserve(capacity);
        for (int i = capacity - 1; i >= 0; --i) free_slots.push_back(i);
        for (int t = 0; t < so.prep_threads; ++t) preppers.emplace_back([this] { prep_main(); });
        loop = std::thread([this] { loop_main(); });
    }

    ~ServerImpl() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stopping = true;
            if (h_stop) *(volatile int*)h_stop = 1;  // running LPs end at their next poll
        }
        cv_prep.notify_all();
        cv_loop.notify_all();
        for (auto& t : preppers) t.join();
        if (loop.joinable()) loop.join();
        // the caller may have another device current (a pool of servers)
        int caller = -1;
        if (cudaGetDevice(&caller) != cudaSuccess) caller = -1;
        if (cs) cudaSetDevice(device);
        if (cs) cudaStreamSynchronize(cs);
        if (ds) cudaStreamSynchronize(ds);
        for (auto& kv : reqs) release(kv.second), delete kv.second;
        if (ds) cudaStreamSynchronize(ds);
        for (void* p : allocs) cudaFree(p);
        if (h_stop) cudaFreeHost(h_stop);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_copy) cudaEventDestroy(ev_copy);
        if (ev_small) cudaEventDestroy(ev_small);
        if (cs2) cudaStreamDestroy(cs2);
        if (cs) cudaStreamDestroy(cs);
        if (ds) cudaStreamDestroy(ds);
        if (caller >= 0) cudaSetDevice(caller);
    }

    // ---- submission and preparation ----
    int64_t submit(const b2_lp_view& U) {
        if (U.m < 0 || U.n < 0 || U.nnz < 0) fail(B2_ERR_INVALID, "negative size");
        if (U.nnz > 0 && (!U.row_idx || !U.col_idx || !U.val)) fail(B2_ERR_INVALID, "null matrix arrays");
        if ((U.n > 0 && (!U.c || !U.l || !U.u)) || (U.m > 0 && (!U.rL || !U.rU))) fail(B2_ERR_INVALID, "null vectors");
        std::unique_ptr<Request> r(new Request());
        r->m = U.m;
        r->n = U.n;
        r->row.assign(U.row_idx, U.row_idx + U.nnz);
        r->col.assign(U.col_idx, U.col_idx + U.nnz);
        r->val.assign(U.val, U.val + U.nnz);
        r->c.assign(U.c, U.c + U.n);
        r->l.assign(U.l, U.l + U.n);
        r->u.assign(U.u, U.u + U.n);
        r->rL.assign(U.rL, U.rL + U.m);
        r->rU.assign(U.rU, U.rU + U.m);
        r->obj_offset = U.obj_offset;
        r->work = request_work(U.m, U.n, U.nnz);
        return enqueue(std::move(r));
    }

    int64_t submit_lp(const b2_lp_view& O, bool presolve) {
        if (O.m < 0 || O.n < 0 || O.nnz < 0) fail(B2_ERR_INVALID, "negative size");
        if (O.nnz > 0 && (!O.row_idx || !O.col_idx || !O.val)) fail(B2_ERR_INVALID, "null matrix arrays");
        if ((O.n > 0 && (!O.c || !O.l || !O.u)) || (O.m > 0 && (!O.rL || !O.rU))) fail(B2_ERR_INVALID, "null vectors");
        std::unique_ptr<Request> r(new Request());
        r->ranged = true;
        r->do_presolve = presolve;
        LpArrays& a = r->orig;
        a.m = O.m;
        a.n = O.n;
        a.row.assign(O.row_idx, O.row_idx + O.nnz);
        a.col.assign(O.col_idx, O.col_idx + O.nnz);
        a.val.assign(O.val, O.val + O.nnz);
        a.c.assign(O.c, O.c + O.n);
        a.l.assign(O.l, O.l + O.n);
        a.u.assign(O.u, O.u + O.n);
        a.rL.assign(O.rL, O.rL + O.m);
        a.rU.assign(O.rU, O.rU + O.m);
        a.obj_offset = O.obj_offset;
        r->work = request_work(O.m, O.n, O.nnz);
        return enqueue(std::move(r));
    }

    static b2_lp_view view_of(const LpArrays& a) {
        return b2_lp_view{a.m, a.n, (int64_t)a.val.size(), a.row.data(), a.col.data(), a.val.data(), a.c.data(),
                          a.rL.data(), a.rU.data(), a.l.data(), a.u.data(), a.obj_offset};
    }

    // The caller's LP -> [presolve] -> PDLP form, into the request's form
    // fields (src/solve.cpp:150-195 does the same before its PDLP stage).
    void to_pdlp_form(Request& r) {
        const b2_lp_view O = view_of(r.orig);
        b2_lp_view src = O;
        if (r.do_presolve) {
            r.pre.reset(presolve_lp(O));
            const int32_t st = presolved_status(*r.pre);
            if (st == 1) fail(B2_ERR_INFEASIBLE, "presolve: the LP is infeasible");
            if (st == 2) fail(B2_ERR_UNBOUNDED, "presolve: the LP is unbounded");
            presolved_view(*r.pre, src);
        }
        if (src.m == 0 || src.n == 0) {
            if (!r.do_presolve) fail(B2_ERR_INVALID, "an LP with no rows or no columns needs presolve");
            r.trivial = true;  // presolve solved it: no GPU work
            return;
        }
        r.form.reset(pdlp_form_build(src));
        b2_lp_view F;
        pdlp_form_view(*r.form, F);
        r.m = F.m;
        r.n = F.n;
        r.row.assign(F.row_idx, F.row_idx + F.nnz);
        r.col.assign(F.col_idx, F.col_idx + F.nnz);
        r.val.assign(F.val, F.val + F.nnz);
        r.c.assign(F.c, F.c + F.n);
        r.l.assign(F.l, F.l + F.n);
        r.u.assign(F.u, F.u + F.n);
        r.rL.assign(F.rL, F.rL + F.m);
        r.rU.assign(F.rU, F.rU + F.m);
        r.obj_offset = F.obj_offset;
    }

    // The PDLP-form answer of a ranged request -> the caller's LP, and
    // verify()'s figures there. Runs on the waiting caller's thread.
    void map_back(Request& r, std::vector<double>& x0, std::vector<double>& y0, b2_request_info* info) {
        const b2_lp_view O = view_of(r.orig);
        x0.assign(std::max(O.n, 1), 0.0);
        y0.assign(std::max(O.m, 1), 0.0);
        std::vector<double> xr, yr;
        b2_lp_view red = O;
        if (r.pre) presolved_view(*r.pre, red);
        xr.assign(std::max(red.n, 1), 0.0);
        yr.assign(std::max(red.m, 1), 0.0);
        if (r.form) pdlp_form_extract(*r.form, r.x.data(), r.y.data(), xr.data(), yr.data());
        if (r.pre) postsolve_lp(*r.pre, xr.data(), yr.data(), x0.data(), y0.data());
        else { x0 = xr; y0 = yr; }
        if (info) {
            info->form_eps[0] = r.res.eps_P;
            info->form_eps[1] = r.res.eps_D;
            info->form_eps[2] = r.res.eps_G;
            info->presolved_m = r.form ? r.m : 0;
            info->presolved_n = r.form ? r.n : 0;
        }
        double k[4];
        kkt_host(O, x0.data(), y0.data(), k);
        r.res.eps_P = k[0];
        r.res.eps_D = k[1];
        r.res.eps_G = k[2];
        r.res.objective = k[3];
    }

    int64_t submit_file(const std::string& path) {
        std::unique_ptr<Request> r(new Request());
        r->path = path;
        // the header alone sizes the backlog; a file that cannot be read
        // counts nothing and fails its ticket on a preparation thread
        try {
            int32_t m = 0, n = 0;
            int64_t nnz = 0;
            lp_read_dims(path, &m, &n, &nnz);
            r->work = request_work(m, n, nnz);
        } catch (const Error&) {
            r->work = 0;
        }
        return enqueue(std::move(r));
    }

    int64_t enqueue(std::unique_ptr<Request> r) {
        std::lock_guard<std::mutex> lk(mu);
        if (fatal) fail(fatal, "server stopped after an error: " + fatal_msg);
        if (stopping) fail(B2_ERR_INVALID, "server is shutting down");
        r->ticket = next_ticket++;
        r->t_submit = now_s();
        Request* p = r.release();
        reqs[p->ticket] = p;
        prep_q.push_back(p);
        st.submitted++;
        st.backlog_work += p->work;
        cv_prep.notify_one();
        return p->ticket;
    }

    void prep_main() {
        cudaSetDevice(device);  // large LPs are scaled on the GPU
        for (;;) {
            Request* r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_prep.wait(lk, [&] { return stopping || !prep_q.empty(); });
                if (stopping) return;
                r = prep_q.front();
                prep_q.pop_front();
            }
            const auto t0 = Clock::now();
            try {
                prepare(*r);
            } catch (const Error& e) {
                finish_failed(r, e.code, e.msg);
                continue;
            } catch (const std::bad_alloc&) {
                finish_failed(r, B2_ERR_OOM, "host allocation failed");
                continue;
            }
            r->prep_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
            if (r->trivial) {  // presolve left nothing to solve
                std::memset(&r->res, 0, sizeof(r->res));
                r->res.converged = 1;
                r->res.exit_reason = B2_EXIT_CONVERGED;
                {
                    std::lock_guard<std::mutex> lk(mu);
                    r->state = RQ_DONE;
                    st.backlog_work -= r->work;
                    r->t_prepared = r->t_admit = r->t_done = now_s();
                    st.completed++;
                }
                cv_done.notify_all();
                continue;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                r->state = RQ_PREPARED;
                r->t_prepared = now_s();
                admit_q.push_back(r);
            }
            cv_loop.notify_one();
        }
    }

    // Scaling (src/scaling.cpp:25-84, 10 Ruiz passes + Pock-Chambolle) and the
    // device layout; the batched lane also gets its region plan and image.
    void prepare(Request& r) {
        if (r.ranged) {
            to_pdlp_form(r);
            if (r.trivial) return;
        }
        if (!r.path.empty()) {
            LpArrays a;
            lp_read(r.path, a);
            r.m = a.m;
            r.n = a.n;
            r.row.swap(a.row); r.col.swap(a.col); r.val.swap(a.val);
            r.c.swap(a.c); r.l.swap(a.l); r.u.swap(a.u); r.rL.swap(a.rL); r.rU.swap(a.rU);
            r.obj_offset = a.obj_offset;
        }
        b2_lp_view U{r.m, r.n, (int64_t)r.val.size(), r.row.data(), r.col.data(), r.val.data(), r.c.data(),
                     r.rL.data(), r.rU.data(), r.l.data(), r.u.data(), r.obj_offset};
        std::vector<double> val_s(r.val.size()), c_s(r.n), l_s(r.n), u_s(r.n), rL_s(r.m), rU_s(r.m), Dr(r.m),
            Dc(r.n);
        // the GPU computes the same scaling bit for bit; it pays off for large LPs
        if (so.gpu_scale_nnz > 0 && (int64_t)r.val.size() >= so.gpu_scale_nnz)
            scale_lp_gpu(U, 10, val_s.data(), c_s.data(), rL_s.data(), rU_s.data(), l_s.data(), u_s.data(),
                         Dr.data(), Dc.data());
        else
            scale_lp(U, 10, val_s.data(), c_s.data(), rL_s.data(), rU_s.data(), l_s.data(), u_s.data(), Dr.data(),
                     Dc.data());
        b2_lp_view S{r.m, r.n, (int64_t)r.val.size(), r.row.data(), r.col.data(), val_s.data(), c_s.data(),
                     rL_s.data(), rU_s.data(), l_s.data(), u_s.data(), r.obj_offset};
        BuildParams bp;
        if (o.sigma_window > 0) bp.sigma_window = o.sigma_window;
        bp.split = (int64_t)r.val.size() >= so.grid_nnz;  // the whole-GPU lane lays out as b2_engine does
        // a batched-lane LP takes its shape class's lane target; the whole-GPU lane, the engine's
        bp.lane_target = bp.split ? o.lane_target : lane_target_for(o, r.m, r.n, (int64_t)r.val.size());
        if (bp.split) bp.threads = (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
        Layout L;
        build_layout(U, S, Dr.data(), Dc.data(), bp, L);
        r.meta.m = L.m; r.meta.n = L.n; r.meta.nnz = L.nnz;
        r.meta.a_slices = L.A.n_slices(); r.meta.at_slices = L.AT.n_slices();
        r.meta.exact32 = L.exact32;
        r.meta.denom_p = L.denom_p; r.meta.denom_d = L.denom_d;
        r.meta.lu_const = L.lu_const; r.meta.l_all = L.l_all; r.meta.u_all = L.u_all;
        r.grid = bp.split;
        r.cluster = !r.grid && so.cluster_nnz > 0 && L.A.padded + L.AT.padded >= so.cluster_nnz;
        r.plan = plan_region(L);
        if (r.grid) {
            r.layout = std::move(L);
        } else {
            r.image = build_image(L, r.plan, o.precision != B2_PREC_MIXED);
        }
        // the matrix copies are no longer needed; c stays for the objective
        std::vector<int32_t>().swap(r.row);
        std::vector<int32_t>().swap(r.col);
        std::vector<double>().swap(r.val);
        std::vector<double>().swap(r.rL);
        std::vector<double>().swap(r.rU);
        std::vector<double>().swap(r.l);
        std::vector<double>().swap(r.u);
    }

    // ---- completion ----
    void finish_failed(Request* r, int code, const std::string& msg) {
        {
            std::lock_guard<std::mutex> lk(mu);
            r->err = code ? code : B2_ERR_INVALID;
            r->err_msg = msg;
            r->state = RQ_DONE;
            st.backlog_work -= r->work;
            r->t_done = now_s();
            st.failed++;
        }
        cv_done.notify_all();
    }

    // Frees what a request holds on the device (the copy stream orders the
    // free after every use by earlier rounds, which the host has waited for).
    void release(Request* r) {
        if (r->region) {
            cudaFreeAsync(r->region, ds);
            r->region = nullptr;
        }
        if (r->eng) {
            engine_destroy(r->eng);
            r->eng = nullptr;
        }
        if (r->slot >= 0) {
            free_slots.push_back(r->slot);
            r->slot = -1;
        }
        if (r->dev_bytes) {
            bytes_in_use -= r->dev_bytes;
            r->dev_bytes = 0;
        }
    }

    // ---- the loop ----
    void loop_main() {
        try {
            cuda_ok(cudaSetDevice(device), "cudaSetDevice");
            for (;;) {
                {
                    std::unique_lock<std::mutex> lk(mu);
                    cv_loop.wait_for(lk, std::chrono::milliseconds(2), [&] {
                        return stopping || !admit_q.empty() || !resident.empty() || !grid_resident.empty();
                    });
                    if (stopping) return;
                }
                admit();
                if (!resident.empty()) run_round();
                admit();
                if (!grid_resident.empty()) run_grid_slice();
            }
        } catch (const Error& e) {
            fail_all(e.code, e.msg);
        } catch (const std::exception& e) {
            fail_all(B2_ERR_CUDA, e.what());
        }
    }

    void fail_all(int code, const std::string& msg) {
        std::vector<Request*> hit;
        {
            std::lock_guard<std::mutex> lk(mu);
            fatal = code ? code : B2_ERR_CUDA;
            fatal_msg = msg;
            for (auto& kv : reqs)
                if (kv.second->state != RQ_DONE) hit.push_back(kv.second);
        }
        for (Request* r : hit) finish_failed(r, fatal, "server stopped after an error: " + msg);
    }

    // Admits prepared LPs, oldest first, while their footprint fits the
    // budget and a slot is free; uploads on the copy stream.
    void admit(bool allow_grid = true) {
        for (;;) {
            Request* r = nullptr;
            {
                std::lock_guard<std::mutex> lk(mu);
                if (admit_q.empty()) return;
                Request* h = admit_q.front();
                const size_t need = h->plan.bytes;
                if ((double)(bytes_in_use + need) > so.hbm_budget_bytes && bytes_in_use > 0) return;
                if (!h->grid && free_slots.empty()) return;
                if (h->grid && !allow_grid) return;  // its engine is built between rounds
                admit_q.pop_front();
                r = h;
                bytes_in_use += need;
                r->dev_bytes = need;
                peak_bytes = std::max(peak_bytes, bytes_in_use);
                if (!r->grid) {
                    r->slot = free_slots.back();
                    free_slots.pop_back();
                }
            }
            try {
                if (r->grid) {
                    r->eng = engine_create_from_layout(std::move(r->layout));
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        bytes_in_use -= r->dev_bytes;
                        r->dev_bytes = engine_bytes(r->eng);
                        bytes_in_use += r->dev_bytes;
                        peak_bytes = std::max(peak_bytes, bytes_in_use);
                    }
                    engine_begin_slices(r->eng, o);
                } else {
                    void* p = nullptr;
                    cuda_ok(cudaMallocFromPoolAsync(&p, r->plan.bytes, pool, ds), "cudaMallocFromPoolAsync");
                    r->region = static_cast<unsigned char*>(p);
                    cuda_ok(cudaMemcpyAsync(r->region, r->image.data(), r->image.size(), cudaMemcpyHostToDevice, ds),
                            "LP upload");
                    const dev::LpDev d = region_desc(r->region, r->plan, r->meta);
                    cuda_ok(cudaMemcpyAsync(d_lps + r->slot, &d, sizeof(d), cudaMemcpyHostToDevice, ds), "desc upload");
                    cuda_ok(cudaEventRecord(ev_copy, ds), "event");
                    // pageable sources: the copies above have taken the bytes
                    std::vector<unsigned char>().swap(r->image);
                }
            } catch (const Error& e) {
                std::lock_guard<std::mutex> lk(mu);
                release(r);
                r->err = e.code;
                r->err_msg = e.msg;
                r->state = RQ_DONE;
                st.backlog_work -= r->work;
                r->t_done = now_s();
                st.failed++;
                cv_done.notify_all();
                if (e.code != B2_ERR_OOM) throw;
                continue;
            }
            std::lock_guard<std::mutex> lk(mu);
            r->state = RQ_RESIDENT;
            r->admit_seq = admit_counter++;
            r->t_admit = now_s();
            if (r->grid) grid_resident.push_back(r);
            else resident.push_back(r);
        }
    }

    // One round of the batched kernel over every resident LP (oldest first).
    void run_round() {
        const int nq = (int)resident.size();
        // two queues, each oldest first: LPs for clusters of CTAs, LPs for one CTA
        std::vector<int> order, order_large;
        std::vector<int> pos(nq);
        for (int k = 0; k < nq; ++k)
            if (!(resident[k]->cluster && max_clusters > 0)) pos[k] = (int)order.size(), order.push_back(resident[k]->slot);
        const int n_small = (int)order.size();
        for (int k = 0; k < nq; ++k)
            if (resident[k]->cluster && max_clusters > 0)
                pos[k] = n_small + (int)order_large.size(), order_large.push_back(resident[k]->slot);
        dev::BatchArgs B = args;
        B.n_inst = n_small;
        B.n_large = (int)order_large.size();
        cuda_ok(cudaStreamWaitEvent(cs, ev_copy, 0), "wait uploads");
        if (n_small)
            cuda_ok(cudaMemcpyAsync((void*)B.order, order.data(), sizeof(int) * n_small, cudaMemcpyHostToDevice, cs),
                    "queue");
        if (B.n_large)
            cuda_ok(cudaMemcpyAsync((void*)B.order_large, order_large.data(), sizeof(int) * B.n_large,
                                    cudaMemcpyHostToDevice, cs), "queue");
        cuda_ok(cudaMemsetAsync(B.qstatus, 0xff, sizeof(int) * nq, cs), "memset");
        cuda_ok(cudaMemsetAsync(B.next, 0, sizeof(unsigned), cs), "memset");
        cuda_ok(cudaMemsetAsync(B.next_large, 0, sizeof(unsigned), cs), "memset");
        cuda_ok(cudaMemsetAsync(B.t0, 0, sizeof(unsigned long long), cs), "memset");
        cuda_ok(cudaEventRecord(ev0, cs), "event");
        if (B.n_large) {
            // clusters for the large LPs on up to 3/4 of the GPU, and beside
            // them a one-CTA launch on the rest, so the small LPs never wait
            // for the large ones; both take from the same queues
            const int ncl = std::max(1, std::min(B.n_large, std::max(1, max_clusters * 3 / 4)));
            batch_kernel_launch(B, true, nt, ncl, cs);
            const int rest = max_ctas - ncl * dev::kMaxCluster;
            if (n_small && rest > 0) {
                cuda_ok(cudaStreamWaitEvent(cs2, ev0, 0), "wait");
                dev::BatchArgs Bs = B;
                Bs.n_large = 0;
                batch_kernel_launch(Bs, false, nt, std::min(rest, n_small), cs2);
                cuda_ok(cudaEventRecord(ev_small, cs2), "event");
                cuda_ok(cudaStreamWaitEvent(cs, ev_small, 0), "wait");
            }
        } else {
            batch_kernel_launch(B, false, nt, std::max(1, std::min(max_ctas, nq)), cs);
        }
        cuda_ok(cudaEventRecord(ev1, cs), "event");
        // overlap: admit (and upload) new arrivals while the round runs
        for (;;) {
            const cudaError_t q = cudaEventQuery(ev1);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) cuda_ok(q, "batched round");
            admit(false);
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
        float ms = 0.0f;
        cuda_ok(cudaEventElapsedTime(&ms, ev0, ev1), "elapsed");
        std::vector<int> qraw(nq), qs(nq);
        cuda_ok(cudaMemcpy(qraw.data(), B.qstatus, sizeof(int) * nq, cudaMemcpyDeviceToHost), "status");
        for (int k = 0; k < nq; ++k) qs[k] = qraw[pos[k]];
        // copy the finished LPs out through the pinned staging buffer
        std::vector<Request*> done;
        size_t need = 0;
        for (int k = 0; k < nq; ++k) {
            Request* r = resident[k];
            if (qs[k] != -1) r->rounds++;
            if (qs[k] > 0) {
                done.push_back(r);
                need += 256 + sizeof(dev::Ctl) + 16 + 8 * ((size_t)r->meta.m + r->meta.n);
            }
        }
        if (!done.empty()) {
            stage.reserve(std::max<size_t>(need, 1 << 20));
            std::vector<size_t> at(done.size());
            size_t off = 0;
            for (size_t i = 0; i < done.size(); ++i) {
                Request* r = done[i];
                const dev::LpDev d = region_desc(r->region, r->plan, r->meta);
                at[i] = off;
                cuda_ok(cudaMemcpyAsync(stage.p + off, d.ctl, sizeof(dev::Ctl), cudaMemcpyDeviceToHost, cs), "ctl");
                off += (sizeof(dev::Ctl) + 15) & ~size_t(15);
                cuda_ok(cudaMemcpyAsync(stage.p + off, args.t_start + r->slot, 8, cudaMemcpyDeviceToHost, cs), "t");
                cuda_ok(cudaMemcpyAsync(stage.p + off + 8, args.t_end + r->slot, 8, cudaMemcpyDeviceToHost, cs), "t");
                off += 16;
                if (r->meta.n)
                    cuda_ok(cudaMemcpyAsync(stage.p + off, d.out_x, 8 * (size_t)r->meta.n, cudaMemcpyDeviceToHost, cs), "x");
                off += 8 * (size_t)r->meta.n;
                if (r->meta.m)
                    cuda_ok(cudaMemcpyAsync(stage.p + off, d.out_y, 8 * (size_t)r->meta.m, cudaMemcpyDeviceToHost, cs), "y");
                off += 8 * (size_t)r->meta.m;
                off = (off + 255) & ~size_t(255);
            }
            cuda_ok(cudaStreamSynchronize(cs), "copy-out");
            for (size_t i = 0; i < done.size(); ++i) {
                Request* r = done[i];
                const unsigned char* p = stage.p + at[i];
                dev::Ctl f;
                std::memcpy(&f, p, sizeof(f));
                p += (sizeof(dev::Ctl) + 15) & ~size_t(15);
                unsigned long long t0 = 0, t1 = 0;
                std::memcpy(&t0, p, 8);
                std::memcpy(&t1, p + 8, 8);
                p += 16;
                r->x.assign(reinterpret_cast<const double*>(p), reinterpret_cast<const double*>(p) + r->meta.n);
                p += 8 * (size_t)r->meta.n;
                r->y.assign(reinterpret_cast<const double*>(p), reinterpret_cast<const double*>(p) + r->meta.m);
                fill_result(f, r->res);
                r->res.group_ctas = r->cluster && max_clusters > 0 ? dev::kMaxCluster : 1;
                r->res.device_ms = (double)(t1 - t0) * 1e-6;
                set_objective(r);
            }
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            st.rounds++;
            st.busy_ms += ms;
            const double t = now_s();
            std::vector<Request*> keep;
            keep.reserve(resident.size());
            for (int k = 0; k < nq; ++k) {
                Request* r = resident[k];
                if (qs[k] > 0) {
                    // the caller may take (and delete) it once it is marked done
                    release(r);
                    r->state = RQ_DONE;
                    st.backlog_work -= r->work;
                    r->t_done = t;
                    st.completed++;
                } else {
                    keep.push_back(r);
                }
            }
            for (size_t k = nq; k < resident.size(); ++k) keep.push_back(resident[k]);
            resident.swap(keep);
        }
        if (!done.empty()) cv_done.notify_all();
    }

    // c'x + offset in the caller's order (the reference reports the PDLP
    // form's objective the same way)
    static void set_objective(Request* r) {
        double obj = r->obj_offset;
        for (int32_t j = 0; j < r->n; ++j) obj += r->c[j] * r->x[j];
        r->res.objective = obj;
    }

    // One slice of the oldest whole-GPU LP.
    void run_grid_slice() {
        Request* r = grid_resident.front();
        const auto t0 = Clock::now();
        // short slices while the batched LPs could fill most of the GPU, long
        // ones when the LP is alone or the rounds would leave most SMs idle
        // (a round's CTAs: one per small LP, a cluster per large one)
        int64_t need = 0;
        for (const Request* q : resident) need += q->cluster && max_clusters > 0 ? dev::kMaxCluster : 1;
        const double slice_ms = need * 2 < max_ctas ? so.grid_slice_ms : std::min(so.grid_slice_ms, so.round_ms);
        const bool ended = engine_slice(r->eng, o, slice_ms, cs);
        r->rounds++;
        {
            std::lock_guard<std::mutex> lk(mu);
            st.grid_slices++;
            st.busy_ms += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        }
        if (!ended) return;
        r->x.resize(r->meta.n);
        r->y.resize(r->meta.m);
        engine_finish_slices(r->eng, r->x.data(), r->y.data(), &r->res);
        set_objective(r);
        {
            std::lock_guard<std::mutex> lk(mu);
            grid_resident.pop_front();
            release(r);
            r->state = RQ_DONE;
            st.backlog_work -= r->work;
            r->t_done = now_s();
            st.completed++;
        }
        cv_done.notify_all();
    }

    // ---- results ----
    int wait(int64_t ticket, double timeout_s, double* x, double* y, b2_result* res, b2_request_info* info) {
        std::unique_lock<std::mutex> lk(mu);
        auto it = reqs.find(ticket);
        if (it == reqs.end()) fail(B2_ERR_INVALID, "unknown ticket (or its result was already taken)");
        Request* r = it->second;
        auto ready = [&] { return r->state == RQ_DONE; };
        if (timeout_s < 0) cv_done.wait(lk, ready);
        else cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
        if (!ready()) return B2_ERR_PENDING;
        if (info) {
            std::memset(info, 0, sizeof(*info));
            info->submit_s = r->t_submit;
            info->admit_s = r->t_admit;
            info->done_s = r->t_done;
            info->prep_ms = r->prep_ms;
            info->rounds = r->rounds;
            info->lane = r->grid ? 1 : 0;
            info->device_bytes = (int64_t)r->plan.bytes;
        }
        const int err = r->err;
        const std::string msg = r->err_msg;
        reqs.erase(it);
        lk.unlock();
        // the request is the caller's alone now
        std::unique_ptr<Request> own(r);
        if (err) fail(err, msg);
        if (r->ranged) {
            std::vector<double> x0, y0;
            map_back(*r, x0, y0, info);
            if (x && r->orig.n) std::memcpy(x, x0.data(), sizeof(double) * r->orig.n);
            if (y && r->orig.m) std::memcpy(y, y0.data(), sizeof(double) * r->orig.m);
        } else {
            if (x && r->n) std::memcpy(x, r->x.data(), sizeof(double) * r->n);
            if (y && r->m) std::memcpy(y, r->y.data(), sizeof(double) * r->m);
        }
        if (res) *res = r->res;
        return B2_OK;
    }

    void stats(b2_server_stats* out) {
        std::lock_guard<std::mutex> lk(mu);
        *out = st;
        out->resident = (int32_t)(resident.size() + grid_resident.size());
        out->queued = (int32_t)(prep_q.size() + admit_q.size());
        out->bytes_in_use = (int64_t)bytes_in_use;
        out->peak_bytes = (int64_t)peak_bytes;
    }
};

ServerImpl* server_create(const b2_server_opts& so, const b2_solve_opts& o) {
    std::unique_ptr<ServerImpl> s(new ServerImpl());
    s->create(so, o);
    return s.release();
}
void server_destroy(ServerImpl* s) { delete s; }
int64_t server_submit(ServerImpl* s, const b2_lp_view& U) { return s->submit(U); }
int64_t server_submit_file(ServerImpl* s, const std::string& path) { return s->submit_file(path); }
int64_t server_submit_lp(ServerImpl* s, const b2_lp_view& O, bool presolve) { return s->submit_lp(O, presolve); }
int server_wait(ServerImpl* s, int64_t ticket, double timeout_s, double* x, double* y, b2_result* res,
                b2_request_info* info) {
    return s->wait(ticket, timeout_s, x, y, res, info);
}
void server_stats(ServerImpl* s, b2_server_stats* out) { s->stats(out); }
int64_t server_backlog(ServerImpl* s) {
    std::lock_guard<std::mutex> lk(s->mu);
    return s->st.backlog_work;
}

}  // namespace b2
