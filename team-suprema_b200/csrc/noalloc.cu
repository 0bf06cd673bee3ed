// noalloc.cu -- b2_solve_pdhg_gpu_noalloc: the one-CTA PDLP solve with every
// byte of its device working set (the LP's sliced layout, iterates, averages,
// best point, control state, outputs) carved out of one file-scope static
// __device__ array, so the call allocates no device memory.
//
// For callers that cannot call cudaMalloc: processes whose GPU memory is
// reserved up front by another runtime's allocator or a pool they do not own
// (a cudaMalloc from here would fail or fragment it), and latency-critical
// paths that must stay out of the driver's allocator.
//
// Limits and sharing:
//   * the array holds kNoAllocBytes (32 MiB): the layout, vectors and
//     iterates of LPs up to roughly 200,000 nonzeros; larger LPs are rejected
//     with B2_ERR_UNSUPPORTED before any GPU work;
//   * when a device holds the array: with lazy module loading (CUDA's default
//     since 12.2) from the first call on that device (its
//     cudaGetSymbolAddress loads this file's module) until the process exits;
//     with eager loading, on every device from library load;
//   * every call in the process shares the one array and leaves its contents
//     behind; whatever must start at zero is cleared by each call. Calls are
//     serialized by a process-wide lock and each returns only after its GPU
//     work is done; GPU work of two calls that overlapped would race on the
//     array;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins;
//   * the work runs on the legacy default stream, with synchronous copies.
// Host memory is still used to build the sliced layout before it is copied
// into the array.
#include <algorithm>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "device.cuh"

namespace b2 {

constexpr size_t kNoAllocBytes = 32u << 20;

namespace dev {

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// The same one-CTA solve as k_pdlp_cta in engine.cu.
template <class T, class V>
__global__ void __launch_bounds__(kBlock, 2) k_pdlp_cta_static(const KParams<T> P, double* bcast, int* abort_word) {
    __shared__ double s_part[kCtaPartDoubles];
    Group g;
    g.rank = 0;
    g.size = 1;
    g.gw = threadIdx.x >> 5;
    g.nw = kWarps;
    g.gt = threadIdx.x;
    g.nt = kBlock;
    g.part = nullptr;
    g.bcast = bcast;
    g.bar = nullptr;
    g.abort = abort_word;
    g.timeout_ns = 0;
    g.spart = s_part;
    solve_body<GK_CTA, T, V>(P, g);
}

}  // namespace dev

namespace {

std::mutex g_noalloc_lock;
std::vector<unsigned char*> g_noalloc_base;  // per device, from cudaGetSymbolAddress

// Bump allocation inside the static array (256-byte aligned pieces).
struct Carve {
    unsigned char* base;
    size_t used = 0;
    template <class T>
    T* take(size_t count) {
        const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
        used = (used + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + used);
        used += bytes;
        return p;
    }
};

template <class T>
void put(T* dst, const std::vector<T>& src) {
    if (!src.empty()) cuda_ok(cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice), "noalloc upload");
}

dev::SellDev carve_sell(Carve& c, const SellHost& S) {
    dev::SellDev d{};
    d.n_rows = S.n_rows;
    d.n_slices = (int)S.n_slices();
    int32_t* slice = c.take<int32_t>(S.slice.size());
    uint32_t* col = c.take<uint32_t>(S.col.size());
    float* v32 = c.take<float>(S.val32.size());
    double* v64 = S.val64.empty() ? nullptr : c.take<double>(S.val64.size());
    if (c.used <= kNoAllocBytes) {
        put(slice, S.slice);
        put(col, S.col);
        put(v32, S.val32);
        if (v64) put(v64, S.val64);
    }
    d.slice = reinterpret_cast<const int4*>(slice);
    d.col = col;
    d.v32 = v32;
    d.v64 = v64;
    return d;
}

template <class T>
dev::Bufs<T> carve_bufs(Carve& c, int m, int n) {
    dev::Bufs<T> B{};
    for (auto& p : B.x) p = c.take<T>(n);
    for (auto& p : B.y) p = c.take<T>(m);
    for (auto& p : B.ax) p = c.take<T>(m);
    for (auto& p : B.aty) p = c.take<T>(n);
    B.x_last = c.take<T>(n);
    B.y_last = c.take<T>(m);
    return B;
}

// Device bytes the carve below takes for this layout (with alignment slack).
size_t needed_bytes(const Layout& L) {
    Carve c{nullptr};
    auto sell = [&](const SellHost& S) {
        c.take<int32_t>(S.slice.size());
        c.take<uint32_t>(S.col.size());
        c.take<float>(S.val32.size());
        if (!S.val64.empty()) c.take<double>(S.val64.size());
    };
    sell(L.A);
    sell(L.AT);
    for (int k = 0; k < 3; ++k) c.take<double>(L.m);        // b, rU, dr2
    for (int k = 0; k < 5; ++k) c.take<double>(L.n);        // c, l, u, dc2, x0
    c.take<int32_t>(L.m);
    c.take<int32_t>(L.n);
    carve_bufs<float>(c, L.m, L.n);
    carve_bufs<double>(c, L.m, L.n);
    for (int k = 0; k < 3; ++k) c.take<double>(L.n);        // xsum, best_x, out_x
    for (int k = 0; k < 3; ++k) c.take<double>(L.m);        // ysum, best_y, out_y
    c.take<dev::Ctl>(1);
    c.take<double>(8);
    c.take<int>(1);
    return c.used;
}

}  // namespace

void solve_noalloc(const b2_lp_view& U, const b2_lp_view& S, const double* Dr, const double* Dc,
                   const b2_solve_opts& o, double* x_out, double* y_out, b2_result* res) {
    Layout L;
    BuildParams bp;
    bp.lane_target = o.lane_target;
    bp.sigma_window = o.sigma_window;
    build_layout(U, S, Dr, Dc, bp, L);
    const size_t need = needed_bytes(L);
    if (need > kNoAllocBytes)
        fail(B2_ERR_UNSUPPORTED, "this LP needs " + std::to_string(need) + " bytes of device working memory; the "
             "allocation-free entry point holds at most " + std::to_string(kNoAllocBytes) + " bytes (32 MiB)");
    if (o.max_iterations < 0) fail(B2_ERR_INVALID, "max_iterations < 0");

    std::lock_guard<std::mutex> lock(g_noalloc_lock);
    int device = 0;
    cuda_ok(cudaGetDevice(&device), "cudaGetDevice");
    if ((int)g_noalloc_base.size() <= device) g_noalloc_base.resize(device + 1, nullptr);
    if (!g_noalloc_base[device]) {
        // first call on this device: the array's device address
        void* p = nullptr;
        cuda_ok(cudaGetSymbolAddress(&p, dev::g_noalloc_scratch), "cudaGetSymbolAddress");
        g_noalloc_base[device] = static_cast<unsigned char*>(p);
    }
    Carve c{g_noalloc_base[device]};
    dev::SellDev A = carve_sell(c, L.A), AT = carve_sell(c, L.AT);
    double* b = c.take<double>(L.m); double* rU = c.take<double>(L.m); double* dr2 = c.take<double>(L.m);
    double* cc = c.take<double>(L.n); double* l = c.take<double>(L.n); double* u = c.take<double>(L.n);
    double* dc2 = c.take<double>(L.n); double* x0 = c.take<double>(L.n);
    int32_t* perm_r = c.take<int32_t>(L.m);
    int32_t* perm_c = c.take<int32_t>(L.n);
    put(b, L.b); put(rU, L.rU); put(dr2, L.dr2);
    put(cc, L.c); put(l, L.l); put(u, L.u); put(dc2, L.dc2); put(x0, L.x0);
    put(perm_r, L.perm_r); put(perm_c, L.perm_c);
    dev::Bufs<float> itf = carve_bufs<float>(c, L.m, L.n);
    dev::Bufs<double> itd = carve_bufs<double>(c, L.m, L.n);
    double* xsum = c.take<double>(L.n); double* best_x = c.take<double>(L.n); double* out_x = c.take<double>(L.n);
    double* ysum = c.take<double>(L.m); double* best_y = c.take<double>(L.m); double* out_y = c.take<double>(L.m);
    dev::Ctl* ctl = c.take<dev::Ctl>(1);
    double* bcast = c.take<double>(8);
    int* abort_word = c.take<int>(1);
    // left over from the previous call: clear what is read before it is written
    cuda_ok(cudaMemset(bcast, 0, 8 * sizeof(double)), "noalloc clear");
    cuda_ok(cudaMemset(abort_word, 0, sizeof(int)), "noalloc clear");

    auto params = [&](auto& P, auto& B) {
        P.m = L.m; P.n = L.n;
        P.A = A; P.AT = AT;
        P.b = b; P.rU = rU; P.c = cc; P.l = l; P.u = u; P.x0 = x0; P.dr2 = dr2; P.dc2 = dc2;
        P.lu_const = L.lu_const ? 1 : 0; P.l_all = L.l_all; P.u_all = L.u_all;
        P.it = B;
        P.itf = itf;
        P.xsum = xsum; P.ysum = ysum; P.best_x = best_x; P.best_y = best_y; P.out_x = out_x; P.out_y = out_y;
        P.perm_r = perm_r; P.perm_c = perm_c;
        P.ctl = ctl;
        P.host_stop = nullptr;
        P.tol = o.tol;
        P.switch_tol = o.switch_tol;
        P.denom_p = L.denom_p; P.denom_d = L.denom_d;
        P.time_limit_ns = 0.0;
        P.max_iterations = o.max_iterations;
        P.check_every = std::max(1, o.check_every);
        P.stall_checks = o.stall_checks > 0 ? o.stall_checks : 32;
        P.return_current = o.return_current;
        P.mixed = o.precision == B2_PREC_MIXED;
        P.debug_delay_ns = 0;
        P.trace = nullptr;
        P.trace_cap = 0;
    };
    dev::Ctl h{};
    h.eta = L.eta0;
    h.omega = L.omega0;
    h.merit_last_restart = h.merit_prev_cand = h.best_merit = std::numeric_limits<double>::infinity();
    h.ax_cur = 0; h.ax_nxt = 1; h.ax_avg = 2; h.aty_cur = 0; h.aty_avg = 1;
    h.mode = dev::MODE_START;
    cuda_ok(cudaMemcpy(ctl, &h, sizeof(h), cudaMemcpyHostToDevice), "ctl upload");
    // kernels run on the legacy default stream; the synchronous copies after
    // each launch wait for it
    bool run_fp64 = o.precision != B2_PREC_MIXED;
    if (!run_fp64) {
        dev::KParams<float> P{};
        params(P, itf);
        dev::k_pdlp_cta_static<float, float><<<1, dev::kBlock>>>(P, bcast, abort_word);
        cuda_ok(cudaGetLastError(), "k_pdlp_cta_static");
        dev::Ctl back{};
        cuda_ok(cudaMemcpy(&back, ctl, sizeof(back), cudaMemcpyDeviceToHost), "ctl download");
        if (back.switch_req && back.exit_reason == 0) {
            // hand the FP32 state over to the FP64 phase, as the resident engine does
            back.mode = dev::MODE_RESUME;
            back.switch_req = 0;
            back.best_merit = std::numeric_limits<double>::infinity();
            back.best_valid = 0;
            back.stall = 0;
            cuda_ok(cudaMemcpy(ctl, &back, sizeof(back), cudaMemcpyHostToDevice), "ctl upload");
            run_fp64 = true;
        }
    }
    if (run_fp64) {
        dev::KParams<double> Q{};
        params(Q, itd);
        if (L.exact32) dev::k_pdlp_cta_static<double, float><<<1, dev::kBlock>>>(Q, bcast, abort_word);
        else dev::k_pdlp_cta_static<double, double><<<1, dev::kBlock>>>(Q, bcast, abort_word);
        cuda_ok(cudaGetLastError(), "k_pdlp_cta_static");
    }
    dev::Ctl fin{};
    cuda_ok(cudaMemcpy(&fin, ctl, sizeof(fin), cudaMemcpyDeviceToHost), "ctl download");
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
        res->final_eta = fin.eta;
        res->final_omega = fin.omega;
        res->group_ctas = 1;
        res->objective = L.obj_offset;
        if (x_out)
            for (int32_t j = 0; j < L.n; ++j) res->objective += L.c[L.inv_c[j]] * x_out[j];
    }
}

}  // namespace b2
