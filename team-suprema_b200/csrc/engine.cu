// engine.cu -- one large LP on the whole GPU: a cooperative launch of the
// persistent solve (device.cuh, solve_body over a grid group), plus the host
// side of the resident engine (b2_engine_*): layout upload, launch, mixed
// precision hand-over, cancellation, results.
#include <time.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <queue>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"

namespace b2 {
namespace dev {

// Grid-wide synchronisation state of a cooperative launch.
struct GridArgs {
    double* part;
    double* bcast;
    unsigned* bar;
    int* abort;
    unsigned long long timeout_ns;
    unsigned long long yield_ns;  // the solve yields this long after the launch starts; 0: never
    int svec_bytes;               // dynamic shared memory: the one-CTA launch's staged x' / y', the grid's y'
};

// y' staged per CTA for the grid kernel's columns pass: LPs whose y' fits in
// this much shared memory (12,288 rows in FP32, 6,144 in FP64)
constexpr size_t kYStageMax = 48 * 1024;

template <class T, class V>
__global__ void __launch_bounds__(kBlock, 2) k_pdlp(const KParams<T> P, const GridArgs ga) {
    Group g;
    g.rank = blockIdx.x;
    g.size = gridDim.x;
    g.gw = blockIdx.x * kWarps + (threadIdx.x >> 5);
    g.nw = gridDim.x * kWarps;
    g.gt = blockIdx.x * kBlock + threadIdx.x;
    g.nt = gridDim.x * kBlock;
    g.part = ga.part;
    g.bcast = ga.bcast;
    g.bar = ga.bar;
    g.abort = ga.abort;
    g.timeout_ns = ga.timeout_ns;
    g.spart = nullptr;
    if (ga.yield_ns) g.yield_at = gtimer() + ga.yield_ns;  // read on CTA 0 only
    extern __shared__ __align__(16) unsigned char s_vec[];
    g.svec = ga.svec_bytes > 0 ? s_vec : nullptr;
    g.svec_bytes = ga.svec_bytes;
    solve_body<GK_GRID, T, V>(P, g);
}

// A small LP on one CTA: the same solve as a CTA group (no grid barrier, no
// fences, partial sums in shared memory).
template <class T, class V>
__global__ void __launch_bounds__(kBlock, 2) k_pdlp_cta(const KParams<T> P, const GridArgs ga) {
    __shared__ double s_part[kCtaPartDoubles];
    extern __shared__ __align__(16) unsigned char s_vec[];
    Group g;
    g.rank = 0;
    g.size = 1;
    g.gw = threadIdx.x >> 5;
    g.nw = kWarps;
    g.gt = threadIdx.x;
    g.nt = kBlock;
    g.part = nullptr;
    g.bcast = ga.bcast;
    g.bar = nullptr;
    g.abort = ga.abort;
    g.timeout_ns = 0;
    g.spart = s_part;
    if (ga.yield_ns) g.yield_at = gtimer() + ga.yield_ns;
    g.svec = ga.svec_bytes > 0 ? s_vec : nullptr;
    g.svec_bytes = ga.svec_bytes;
    solve_body<GK_CTA, T, V, true>(P, g);
}

}  // namespace dev

void cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) fail(B2_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        fail(B2_ERR_NO_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
    fail(B2_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

// Device memory of one-LP engines comes from the device's stream-ordered pool,
// which keeps freed blocks (release threshold: all): the drop-in call creates
// and destroys an engine per solve, and the next one then reuses the blocks
// with no driver allocation or unmapping. A request the pool cannot meet
// first hands the cached blocks back to the driver and tries once more.
void* pool_alloc(size_t bytes, cudaMemPool_t pool, cudaStream_t st) {
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, st);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        cuda_ok(cudaStreamSynchronize(st), "sync");
        cuda_ok(cudaMemPoolTrimTo(pool, 0), "cudaMemPoolTrimTo");
        e = cudaMallocFromPoolAsync(&p, bytes, pool, st);
    }
    cuda_ok(e, "cudaMallocFromPoolAsync");
    return p;
}

}  // namespace

struct EngineImpl {
    int device = 0, sm_count = 0;
    cudaStream_t stream = nullptr;
    Layout L;
    size_t bytes = 0;
    std::vector<void*> allocs;
    dev::SellDev A{}, AT{};
    double *b = nullptr, *rU = nullptr, *c = nullptr, *l = nullptr, *u = nullptr, *x0 = nullptr;
    double *dr2 = nullptr, *dc2 = nullptr;
    dev::Bufs<float> itf{};
    dev::Bufs<double> itd{};
    double *xsum = nullptr, *ysum = nullptr, *best_x = nullptr, *best_y = nullptr, *out_x = nullptr,
           *out_y = nullptr, *part = nullptr, *bcast = nullptr;
    int32_t *perm_r = nullptr, *perm_c = nullptr;
    unsigned* bar = nullptr;
    int* abort_flag = nullptr;
    dev::Ctl* ctl = nullptr;
    static constexpr int kTraceCap = 65536;
    double* trace = nullptr;  // per-check records of the last solve
    int last_checks = 0;
    int* h_stop = nullptr;   // pinned, mapped
    int* d_stop = nullptr;
    int max_ctas = 0;
    int ystage_f = 0, ystage_d = 0;  // grid kernel's dynamic shared memory for y' (FP32 / FP64 iterates); 0: off
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    cudaMemPool_t mpool = nullptr;

    template <class T>
    T* alloc(size_t n) {
        const size_t b = (n > 0 ? n : 1) * sizeof(T);
        T* p = static_cast<T*>(pool_alloc(b, mpool, stream));
        allocs.push_back(p);
        bytes += b;
        return p;
    }
    template <class T>
    T* up(const std::vector<T>& h) {
        T* p = alloc<T>(h.size());
        if (!h.empty())
            cuda_ok(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream), "upload");
        return p;
    }

    ~EngineImpl() {
        // back to the pool in stream order (every solve has finished: solves block)
        if (stream) {
            for (void* p : allocs) cudaFreeAsync(p, stream);
            cudaStreamSynchronize(stream);
        }
        if (h_stop) cudaFreeHost(h_stop);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }

    // The whole-grid kernel's rows and columns passes run the slice records
    // on a work-balanced schedule over the grid's warps (schedule_records:
    // costliest first to the least-loaded warp; inside a warp, records that
    // wait for nothing first, then subgroup leaders, then group owners, so
    // every wait ends). The records are copied into that order, once per grid
    // size; the schedule is a function of the layout and the grid, so solves
    // stay deterministic.
    struct SchedDev {
        const int4* slice = nullptr;
        const int2* aff = nullptr;
        const int* start = nullptr;
    };
    struct Sched {
        SchedDev a, at;
    };
    std::map<int, Sched> scheds;  // by CTA count of the launch

    SchedDev build_sched(const SellHost& S, int nw) {
        SchedDev d;
        const int64_t n = S.n_slices();
        if (n == 0 || nw <= 1) return d;
        std::vector<int32_t> seq, start;
        schedule_records(S, nw, dev::kDenseUnroll, dev::kSubSeg, seq, start);
        std::vector<int32_t> recs((size_t)n * 4), affs(S.aff.empty() ? 0 : (size_t)n * 2);
        for (int64_t k = 0; k < n; ++k) {
            const size_t r = (size_t)seq[(size_t)k];
            for (int q = 0; q < 4; ++q) recs[(size_t)k * 4 + q] = S.slice[r * 4 + q];
            if (!affs.empty()) {
                affs[(size_t)k * 2] = S.aff[r * 2];
                affs[(size_t)k * 2 + 1] = S.aff[r * 2 + 1];
            }
        }
        d.slice = reinterpret_cast<const int4*>(up(recs));
        d.aff = affs.empty() ? nullptr : reinterpret_cast<const int2*>(up(affs));
        d.start = up(start);
        return d;
    }

    template <class T>
    void attach_sched(dev::KParams<T>& Q, int ctas) {
        auto it = scheds.find(ctas);
        if (it == scheds.end()) {
            Sched sc;
            sc.a = build_sched(L.A, ctas * dev::kWarps);
            sc.at = build_sched(L.AT, ctas * dev::kWarps);
            cuda_ok(cudaStreamSynchronize(stream), "schedule upload");
            it = scheds.emplace(ctas, sc).first;
        }
        Q.a_wslice = it->second.a.slice;
        Q.a_waff = it->second.a.aff;
        Q.a_wstart = it->second.a.start;
        Q.t_wslice = it->second.at.slice;
        Q.t_waff = it->second.at.aff;
        Q.t_wstart = it->second.at.start;
    }

    // split-slice arrival counters start every product at zero (an abandoned
    // solve may leave them counted up)
    void clear_seg_counters(cudaStream_t st) {
        for (const dev::SellDev* d : {&A, &AT})
            if (d->seg_cnt)
                cuda_ok(cudaMemsetAsync(d->seg_cnt, 0,
                                        sizeof(unsigned) * dev::kSegCounters * (size_t)(d == &A ? L.A : L.AT).n_groups(), st),
                        "memset");
    }

    dev::SellDev upload_sell(const SellHost& S) {
        dev::SellDev d{};
        d.n_rows = S.n_rows;
        d.n_slices = (int)S.n_slices();
        d.slice = reinterpret_cast<const int4*>(up(S.slice));
        d.col = up(S.col);
        d.v32 = up(S.val32);
        d.v64 = S.val64.empty() ? nullptr : up(S.val64);
        d.aff = S.aff.empty() ? nullptr : reinterpret_cast<const int2*>(up(S.aff));
        if (S.n_groups() > 0) {
            d.seg = reinterpret_cast<const int2*>(up(S.seg));
            d.seg_part = alloc<double>((size_t)S.seg_slots * 32);
            const size_t ncnt = (size_t)dev::kSegCounters * (size_t)S.n_groups();
            unsigned* cnt = alloc<unsigned>(ncnt);
            cuda_ok(cudaMemsetAsync(cnt, 0, sizeof(unsigned) * ncnt, stream), "memset");
            d.seg_cnt = cnt;
        }
        return d;
    }

    template <class T>
    void alloc_bufs(dev::Bufs<T>& B) {
        for (auto& p : B.x) p = alloc<T>(L.n);
        // rounded up to 4 entries: the grid kernel's bulk copy of y' moves whole 16-byte units
        for (auto& p : B.y) p = alloc<T>(((size_t)L.m + 3) / 4 * 4);
        for (auto& p : B.ax) p = alloc<T>(L.m);
        for (auto& p : B.aty) p = alloc<T>(L.n);
        B.x_last = alloc<T>(L.n);
        B.y_last = alloc<T>(L.m);
    }

    void create(const b2_lp_view& U, const b2_lp_view& S, const double* Dr, const double* Dc,
                const b2_solve_opts& o) {
        // host-side validation and layout first: malformed input is reported
        // as such even on a machine without a GPU
        BuildParams bp;
        bp.lane_target = o.lane_target;
        bp.sigma_window = o.sigma_window;
        bp.split = true;  // the whole GPU works on this LP: tune and split long rows
        if (o.long_rows == 1) bp.tune_len = INT32_MAX;  // the length rule for every row
        bp.threads = (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
        build_layout(U, S, Dr, Dc, bp, L);
        create_device();
    }

    void create_device() {
        int ndev = 0;
        cuda_ok(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
        if (ndev == 0) fail(B2_ERR_NO_DEVICE, "no CUDA device");
        cuda_ok(cudaGetDevice(&device), "cudaGetDevice");
        cuda_ok(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device), "attr");
        cuda_ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_ok(cudaEventCreate(&ev0), "event");
        cuda_ok(cudaEventCreate(&ev1), "event");
        cuda_ok(cudaDeviceGetDefaultMemPool(&mpool, device), "cudaDeviceGetDefaultMemPool");
        uint64_t keep = ~uint64_t(0);
        cuda_ok(cudaMemPoolSetAttribute(mpool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
        A = upload_sell(L.A);
        AT = upload_sell(L.AT);
        b = up(L.b); rU = up(L.rU); dr2 = up(L.dr2);
        c = up(L.c); l = up(L.l); u = up(L.u); dc2 = up(L.dc2); x0 = up(L.x0);
        perm_r = up(L.perm_r); perm_c = up(L.perm_c);
        alloc_bufs(itf);
        alloc_bufs(itd);
        xsum = alloc<double>(L.n); ysum = alloc<double>(L.m);
        best_x = alloc<double>(L.n); best_y = alloc<double>(L.m);
        out_x = alloc<double>(L.n); out_y = alloc<double>(L.m);
        bcast = alloc<double>(8);
        bar = alloc<unsigned>(1);
        abort_flag = alloc<int>(1);
        ctl = alloc<dev::Ctl>(1);
        trace = alloc<double>((size_t)kTraceCap * dev::kTraceFields);
        // host stop word: pinned and mapped so the device can poll it
        cuda_ok(cudaHostAlloc((void**)&h_stop, sizeof(int), cudaHostAllocMapped), "cudaHostAlloc");
        *h_stop = 0;
        cuda_ok(cudaHostGetDevicePointer((void**)&d_stop, h_stop, 0), "cudaHostGetDevicePointer");
        // co-resident CTAs of the widest instantiation bound the grid
        int occ[3] = {0, 0, 0};
        cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], dev::k_pdlp<float, float>, dev::kBlock, 0), "occ");
        cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], dev::k_pdlp<double, float>, dev::kBlock, 0), "occ");
        cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], dev::k_pdlp<double, double>, dev::kBlock, 0), "occ");
        int per_sm = std::min(occ[0], std::min(occ[1], occ[2]));
        if (per_sm < 1) fail(B2_ERR_CUDA, "persistent kernel does not fit on an SM");
        max_ctas = per_sm * sm_count;
        // y' staging (few rows): kept for a precision only if the grid keeps per_sm CTAs per SM
        auto stage = [&](const void* fn, size_t elem) -> int {
            const size_t bytes = ((size_t)L.m * elem + 15) / 16 * 16;
            if (L.m == 0 || bytes > dev::kYStageMax) return 0;
            // the kernel's limit is process-wide: every engine sets the same
            // largest size, so one engine's set-up never lowers another's
            if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dev::kYStageMax) !=
                cudaSuccess) {
                cudaGetLastError();
                return 0;
            }
            int o = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fn, dev::kBlock, bytes) != cudaSuccess) {
                cudaGetLastError();
                return 0;
            }
            return o >= per_sm ? (int)bytes : 0;
        };
        ystage_f = stage((const void*)dev::k_pdlp<float, float>, sizeof(float));
        const int d1 = stage((const void*)dev::k_pdlp<double, float>, sizeof(double));
        const int d2 = stage((const void*)dev::k_pdlp<double, double>, sizeof(double));
        ystage_d = d1 > 0 && d2 > 0 ? d1 : 0;
        part = alloc<double>((size_t)dev::NSLOTS * max_ctas * dev::kPartStride);
        cuda_ok(cudaDeviceSynchronize(), "create");
    }

    int pick_ctas(const b2_solve_opts& o) const {
        const int64_t work = L.A.padded + L.AT.padded + 4 * ((int64_t)L.m + L.n);
        int ctas = (int)std::min<int64_t>(max_ctas, std::max<int64_t>(1, work / 16384));
        if (o.max_ctas > 0) ctas = std::min(ctas, o.max_ctas);
        // split slices need the grid kernel with at least one warp per segment
        // of the longest group (their completion waits on the other segments)
        const int seg = std::max(L.A.seg_max, L.AT.seg_max);
        if (seg > 0) ctas = std::min(max_ctas, std::max(ctas, std::max(2, (seg + dev::kWarps - 1) / dev::kWarps)));
        return std::max(1, ctas);
    }

    template <class T>
    dev::KParams<T> params(const b2_solve_opts& o, dev::Bufs<T>& B) {
        dev::KParams<T> P{};
        P.m = L.m; P.n = L.n;
        P.A = A; P.AT = AT;
        P.b = b; P.rU = rU; P.c = c; P.l = l; P.u = u; P.x0 = x0; P.dr2 = dr2; P.dc2 = dc2;
        P.lu_const = L.lu_const ? 1 : 0; P.l_all = L.l_all; P.u_all = L.u_all;
        P.it = B;
        P.itf = itf;
        P.xsum = xsum; P.ysum = ysum; P.best_x = best_x; P.best_y = best_y; P.out_x = out_x; P.out_y = out_y;
        P.perm_r = perm_r; P.perm_c = perm_c;
        P.ctl = ctl;
        P.host_stop = d_stop;
        P.tol = o.tol;
        P.switch_tol = o.switch_tol;
        P.denom_p = L.denom_p; P.denom_d = L.denom_d;
        P.time_limit_ns = o.time_limit_s > 0 ? o.time_limit_s * 1e9 : 0.0;
        P.max_iterations = o.max_iterations;
        P.check_every = std::max(1, o.check_every);
        P.stall_checks = o.stall_checks > 0 ? o.stall_checks : 32;
        P.return_current = o.return_current;
        P.mixed = o.precision == B2_PREC_MIXED;
        P.debug_delay_ns = o.debug_delay_us > 0 ? (unsigned long long)o.debug_delay_us * 1000ull : 0ull;
        P.trace = trace;
        P.trace_cap = kTraceCap;
        return P;
    }

    dev::GridArgs grid_args(const b2_solve_opts& o) {
        dev::GridArgs ga{};
        ga.part = part;
        ga.bcast = bcast;
        ga.bar = bar;
        ga.abort = abort_flag;
        ga.timeout_ns = (unsigned long long)((o.barrier_timeout_s > 0 ? o.barrier_timeout_s : 10.0) * 1e9);
        return ga;
    }

    template <class T, class V>
    void launch(const dev::KParams<T>& P, const dev::GridArgs& ga, int ctas, cudaStream_t st) {
        cuda_ok(cudaMemsetAsync(bar, 0, sizeof(unsigned), st), "memset");
        cuda_ok(cudaMemsetAsync(abort_flag, 0, sizeof(int), st), "memset");
        clear_seg_counters(st);
        if (ctas == 1 && !P.debug_delay_ns) {
            // x' and y' in shared memory when they fit next to the static part
            dev::GridArgs g1 = ga;
            const size_t want = ((size_t)L.m + (size_t)L.n) * sizeof(T);
            cudaFuncAttributes fa{};
            cuda_ok(cudaFuncGetAttributes(&fa, dev::k_pdlp_cta<T, V>), "attr");
            int optin = 0;
            cuda_ok(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device), "attr");
            g1.svec_bytes = 0;
            if (want > 0 && want + fa.sharedSizeBytes <= (size_t)optin) {
                g1.svec_bytes = (int)((want + 255) / 256 * 256);
                if ((size_t)g1.svec_bytes + fa.sharedSizeBytes > (size_t)optin) g1.svec_bytes = (int)want;
                cuda_ok(cudaFuncSetAttribute(dev::k_pdlp_cta<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             g1.svec_bytes), "cudaFuncSetAttribute");
            }
            dev::k_pdlp_cta<T, V><<<1, dev::kBlock, (size_t)g1.svec_bytes, st>>>(P, g1);
            cuda_ok(cudaGetLastError(), "k_pdlp_cta");
            return;
        }
        dev::GridArgs gg = ga;
        gg.svec_bytes = sizeof(T) == 4 ? ystage_f : ystage_d;
        dev::KParams<T> Q = P;
        attach_sched(Q, ctas);
        void* args[] = {(void*)&Q, (void*)&gg};
        cuda_ok(cudaLaunchCooperativeKernel((const void*)dev::k_pdlp<T, V>, dim3(ctas), dim3(dev::kBlock), args,
                                            (size_t)gg.svec_bytes, st),
                "cudaLaunchCooperativeKernel");
    }

    void solve(const b2_solve_opts& o, const volatile int32_t* stop_flag, double* x_out, double* y_out,
               b2_result* res) {
        auto t_host0 = std::chrono::steady_clock::now();
        cudaStream_t st = o.stream ? (cudaStream_t)o.stream : stream;
        if (o.max_iterations < 0) fail(B2_ERR_INVALID, "max_iterations < 0");
        dev::Ctl h{};
        h.eta = L.eta0;
        h.omega = L.omega0;
        h.merit_last_restart = std::numeric_limits<double>::infinity();
        h.merit_prev_cand = std::numeric_limits<double>::infinity();
        h.best_merit = std::numeric_limits<double>::infinity();
        h.xi = 0; h.yi = 0; h.ax_cur = 0; h.ax_nxt = 1; h.ax_avg = 2; h.aty_cur = 0; h.aty_avg = 1;
        h.mode = dev::MODE_START;
        *h_stop = stop_requested(o, stop_flag) ? 1 : 0;
        cuda_ok(cudaMemcpyAsync(ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st), "ctl upload");
        const int ctas = pick_ctas(o);
        const bool mixed = o.precision == B2_PREC_MIXED;
        const bool exact = L.exact32;
        const dev::GridArgs ga = grid_args(o);
        cuda_ok(cudaEventRecord(ev0, st), "event");
        if (mixed) {
            auto P = params<float>(o, itf);
            launch<float, float>(P, ga, ctas, st);
            cuda_ok(cudaEventRecord(ev1, st), "event");
            wait(o, stop_flag);
            dev::Ctl back{};
            cuda_ok(cudaMemcpy(&back, ctl, sizeof(back), cudaMemcpyDeviceToHost), "ctl download");
            check_abort();
            if (back.switch_req && back.exit_reason == 0) {
                back.mode = dev::MODE_RESUME;
                back.switch_req = 0;
                back.best_merit = std::numeric_limits<double>::infinity();
                back.best_valid = 0;
                back.stall = 0;
                cuda_ok(cudaMemcpyAsync(ctl, &back, sizeof(back), cudaMemcpyHostToDevice, st), "ctl upload");
                auto Q = params<double>(o, itd);
                if (exact) launch<double, float>(Q, ga, ctas, st);
                else launch<double, double>(Q, ga, ctas, st);
                cuda_ok(cudaEventRecord(ev1, st), "event");
                wait(o, stop_flag);
                check_abort();
            }
        } else {
            auto Q = params<double>(o, itd);
            if (exact) launch<double, float>(Q, ga, ctas, st);
            else launch<double, double>(Q, ga, ctas, st);
            cuda_ok(cudaEventRecord(ev1, st), "event");
            wait(o, stop_flag);
            check_abort();
        }
        float ms = 0.0f;
        cuda_ok(cudaEventElapsedTime(&ms, ev0, ev1), "elapsed");
        dev::Ctl fin{};
        cuda_ok(cudaMemcpy(&fin, ctl, sizeof(fin), cudaMemcpyDeviceToHost), "ctl download");
        last_checks = fin.checks;
        if (x_out && L.n) cuda_ok(cudaMemcpy(x_out, out_x, sizeof(double) * L.n, cudaMemcpyDeviceToHost), "x download");
        if (y_out && L.m) cuda_ok(cudaMemcpy(y_out, out_y, sizeof(double) * L.m, cudaMemcpyDeviceToHost), "y download");
        if (res) {
            std::memset(res, 0, sizeof(*res));
            res->iterations = fin.attempts;
            res->restarts = fin.restarts;
            res->converged = fin.exit_reason == B2_EXIT_CONVERGED;
            res->accepted = fin.accepted;
            res->eps_P = fin.out_eps[0];
            res->eps_D = fin.out_eps[1];
            res->eps_G = fin.out_eps[2];
            res->exit_reason = fin.exit_reason;
            res->checks = fin.checks;
            res->fp32_attempts = fin.fp32_attempts;
            res->fp32_accepted = fin.fp32_accepted;
            res->device_ms = ms;
            res->final_eta = fin.eta;
            res->final_omega = fin.omega;
            res->group_ctas = ctas;
            res->objective = L.obj_offset;
            if (x_out) {
                // c'x in the caller's column order
                for (int32_t j = 0; j < L.n; ++j) res->objective += L.c[L.inv_c[j]] * x_out[j];
            }
            res->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
        }
    }

    // ---- time-sliced solve (the served stream's whole-GPU lane) ----
    // begin_slices uploads the initial control state; each slice runs the
    // current phase for about slice_ms of device time and returns true when
    // the solve has ended; finish_slices copies the answer out. The FP32 ->
    // FP64 hand-over happens between slices, as solve() does it in one call.
    dev::Ctl sl_ctl{};
    int sl_ctas = 0;
    double sl_ms = 0.0;

    void begin_slices(const b2_solve_opts& o) {
        if (o.max_iterations < 0) fail(B2_ERR_INVALID, "max_iterations < 0");
        dev::Ctl& h = sl_ctl;
        std::memset(&h, 0, sizeof(h));
        h.eta = L.eta0;
        h.omega = L.omega0;
        h.merit_last_restart = h.merit_prev_cand = h.best_merit = std::numeric_limits<double>::infinity();
        h.xi = 0; h.yi = 0; h.ax_cur = 0; h.ax_nxt = 1; h.ax_avg = 2; h.aty_cur = 0; h.aty_avg = 1;
        h.mode = dev::MODE_START;
        h.phase64 = o.precision == B2_PREC_MIXED ? 0 : 1;
        *h_stop = 0;
        cuda_ok(cudaMemcpy(ctl, &h, sizeof(h), cudaMemcpyHostToDevice), "ctl upload");
        sl_ctas = pick_ctas(o);
        sl_ms = 0.0;
    }

    bool slice(const b2_solve_opts& o, double slice_ms, cudaStream_t st) {
        dev::GridArgs ga = grid_args(o);
        ga.yield_ns = (unsigned long long)(std::max(0.01, slice_ms) * 1e6);
        cuda_ok(cudaEventRecord(ev0, st), "event");
        if (!sl_ctl.phase64) {
            auto P = params<float>(o, itf);
            launch<float, float>(P, ga, sl_ctas, st);
        } else {
            auto Q = params<double>(o, itd);
            if (L.exact32) launch<double, float>(Q, ga, sl_ctas, st);
            else launch<double, double>(Q, ga, sl_ctas, st);
        }
        cuda_ok(cudaEventRecord(ev1, st), "event");
        cuda_ok(cudaEventSynchronize(ev1), "slice");
        float ms = 0.0f;
        cuda_ok(cudaEventElapsedTime(&ms, ev0, ev1), "elapsed");
        sl_ms += ms;
        check_abort();
        cuda_ok(cudaMemcpy(&sl_ctl, ctl, sizeof(sl_ctl), cudaMemcpyDeviceToHost), "ctl download");
        if (sl_ctl.exit_reason != 0) return true;
        // a hand-over keeps the mode the phase started in (MODE_CONTINUE after
        // an earlier yield), so it is tested first
        if (sl_ctl.switch_req) {
            sl_ctl.mode = dev::MODE_RESUME;
            sl_ctl.switch_req = 0;
            sl_ctl.best_merit = std::numeric_limits<double>::infinity();
            sl_ctl.best_valid = 0;
            sl_ctl.stall = 0;
            sl_ctl.phase64 = 1;
            cuda_ok(cudaMemcpy(ctl, &sl_ctl, sizeof(sl_ctl), cudaMemcpyHostToDevice), "ctl upload");
            return false;
        }
        if (sl_ctl.mode == dev::MODE_CONTINUE) return false;  // yielded
        return true;
    }

    void finish_slices(double* x_out, double* y_out, b2_result* res) {
        last_checks = sl_ctl.checks;
        if (x_out && L.n) cuda_ok(cudaMemcpy(x_out, out_x, sizeof(double) * L.n, cudaMemcpyDeviceToHost), "x download");
        if (y_out && L.m) cuda_ok(cudaMemcpy(y_out, out_y, sizeof(double) * L.m, cudaMemcpyDeviceToHost), "y download");
        if (res) {
            fill_result(sl_ctl, *res);
            res->group_ctas = sl_ctas;
            res->device_ms = sl_ms;
            res->objective = L.obj_offset;
            if (x_out)
                for (int32_t j = 0; j < L.n; ++j) res->objective += L.c[L.inv_c[j]] * x_out[j];
        }
    }

    // Waits for the persistent kernel while mirroring the caller's stop flag
    // (or stop callback) into the mapped word the device polls.
    void wait(const b2_solve_opts& o, const volatile int32_t* stop_flag) {
        for (;;) {
            cudaError_t q = cudaEventQuery(ev1);
            if (q == cudaSuccess) return;
            if (q != cudaErrorNotReady) cuda_ok(q, "persistent kernel");
            if (stop_requested(o, stop_flag)) *(volatile int*)h_stop = 1;
            struct timespec ts{0, 20000};
            nanosleep(&ts, nullptr);
        }
    }

    void check_abort() {
        int ab = 0;
        cuda_ok(cudaMemcpy(&ab, abort_flag, sizeof(int), cudaMemcpyDeviceToHost), "abort flag");
        if (ab) fail(B2_ERR_TIMEOUT, "a device-side barrier wait timed out; the solve was abandoned");
    }

    void spmv(int which, const double* x, double* y) {
        const dev::SellDev& S = which == 0 ? A : AT;
        const int rows = which == 0 ? L.m : L.n, cols = which == 0 ? L.n : L.m;
        const std::vector<int32_t>& in_perm = which == 0 ? L.perm_c : L.perm_r;   // device col -> caller col
        const std::vector<int32_t>& out_perm = which == 0 ? L.perm_r : L.perm_c;  // device row -> caller row
        std::vector<double> xd(std::max(cols, 1)), yd(std::max(rows, 1));
        for (int j = 0; j < cols; ++j) xd[j] = x[in_perm[j]];
        double *dx = nullptr, *dy = nullptr;
        cuda_ok(cudaMalloc(&dx, xd.size() * sizeof(double)), "cudaMalloc");
        cuda_ok(cudaMalloc(&dy, yd.size() * sizeof(double)), "cudaMalloc");
        cuda_ok(cudaMemcpy(dx, xd.data(), xd.size() * sizeof(double), cudaMemcpyHostToDevice), "H2D");
        const int blocks = std::max(1, std::min(sm_count * 8, (S.n_slices + 7) / 8));
        clear_seg_counters(stream);
        if (S.n_slices > 0) {
            if (L.exact32) dev::k_spmv<double, float, double><<<blocks, 256, 0, stream>>>(S, dx, dy);
            else dev::k_spmv<double, double, double><<<blocks, 256, 0, stream>>>(S, dx, dy);
        }
        cuda_ok(cudaGetLastError(), "k_spmv");
        cuda_ok(cudaStreamSynchronize(stream), "k_spmv");
        cuda_ok(cudaMemcpy(yd.data(), dy, yd.size() * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
        cudaFree(dx);
        cudaFree(dy);
        for (int i = 0; i < rows; ++i) y[out_perm[i]] = yd[i];
    }

    void spmv_bench(int which, int precision, int reps, void* stream_in, double* avg_ms) {
        const dev::SellDev& S = which == 0 ? A : AT;
        cudaStream_t st = stream_in ? (cudaStream_t)stream_in : stream;
        const int blocks = std::max(1, std::min(sm_count * 8, (S.n_slices + 7) / 8));
        const bool f32 = precision == B2_PREC_MIXED;
        // reuse solver buffers of the right size as x / y
        const void* x = which == 0 ? (f32 ? (void*)itf.x[0] : (void*)itd.x[0]) : (f32 ? (void*)itf.y[0] : (void*)itd.y[0]);
        void* y = which == 0 ? (f32 ? (void*)itf.ax[2] : (void*)itd.ax[2]) : (f32 ? (void*)itf.aty[1] : (void*)itd.aty[1]);
        auto go = [&]() {
            if (S.n_slices == 0) return;
            if (f32) dev::k_spmv<float, float, float><<<blocks, 256, 0, st>>>(S, (const float*)x, (float*)y);
            else if (L.exact32) dev::k_spmv<double, float, double><<<blocks, 256, 0, st>>>(S, (const double*)x, (double*)y);
            else dev::k_spmv<double, double, double><<<blocks, 256, 0, st>>>(S, (const double*)x, (double*)y);
        };
        clear_seg_counters(st);
        go();
        cuda_ok(cudaGetLastError(), "k_spmv");
        cuda_ok(cudaEventRecord(ev0, st), "event");
        for (int r = 0; r < reps; ++r) go();
        cuda_ok(cudaEventRecord(ev1, st), "event");
        cuda_ok(cudaEventSynchronize(ev1), "sync");
        float ms = 0.0f;
        cuda_ok(cudaEventElapsedTime(&ms, ev0, ev1), "elapsed");
        *avg_ms = reps > 0 ? ms / reps : 0.0;
    }
};

// ---- thin interface used by the C ABI (capi.cpp) ----
EngineImpl* engine_create(const b2_lp_view& U, const b2_lp_view& S, const double* Dr, const double* Dc,
                          const b2_solve_opts& o) {
    std::unique_ptr<EngineImpl> e(new EngineImpl());
    e->create(U, S, Dr, Dc, o);
    return e.release();
}

EngineImpl* engine_create_from_layout(Layout&& L) {
    std::unique_ptr<EngineImpl> e(new EngineImpl());
    e->L = std::move(L);
    e->create_device();
    return e.release();
}

void engine_destroy(EngineImpl* e) { delete e; }

size_t engine_bytes(EngineImpl* e) { return e->bytes; }
void engine_begin_slices(EngineImpl* e, const b2_solve_opts& o) { e->begin_slices(o); }
bool engine_slice(EngineImpl* e, const b2_solve_opts& o, double slice_ms, void* stream) {
    return e->slice(o, slice_ms, stream ? (cudaStream_t)stream : e->stream);
}
void engine_finish_slices(EngineImpl* e, double* x, double* y, b2_result* r) { e->finish_slices(x, y, r); }

void engine_solve(EngineImpl* e, const b2_solve_opts& o, const volatile int32_t* stop, double* x, double* y,
                  b2_result* r) {
    e->solve(o, stop, x, y, r);
}

void engine_info(EngineImpl* e, b2_engine_info* info) {
    std::memset(info, 0, sizeof(*info));
    info->m = e->L.m;
    info->n = e->L.n;
    info->nnz = e->L.nnz;
    info->a_slices = e->L.A.n_slices();
    info->at_slices = e->L.AT.n_slices();
    info->a_padded = e->L.A.padded;
    info->at_padded = e->L.AT.padded;
    info->values_exact_fp32 = e->L.exact32 ? 1 : 0;
    b2_solve_opts o;
    b2_default_opts(&o);
    info->ctas = e->pick_ctas(o);
    info->threads_per_cta = dev::kBlock;
    info->sm_count = e->sm_count;
    info->device_bytes = (int64_t)e->bytes;
}

void engine_spmv(EngineImpl* e, int which, const double* x, double* y) { e->spmv(which, x, y); }

int engine_trace(EngineImpl* e, double* out, int max_records) {
    const int n = std::min(std::min(e->last_checks, EngineImpl::kTraceCap), std::max(0, max_records));
    if (n > 0 && out)
        cuda_ok(cudaMemcpy(out, e->trace, sizeof(double) * dev::kTraceFields * n, cudaMemcpyDeviceToHost), "trace");
    return n;
}

void engine_spmv_bench(EngineImpl* e, int which, int precision, int reps, void* stream, double* avg_ms) {
    e->spmv_bench(which, precision, reps, stream, avg_ms);
}

}  // namespace b2
