// batch.cu -- many LPs of uneven size in one persistent launch.
//
// Each CTA is a group of one: it takes the next LP from a device work queue
// (an atomic counter over an order sorted longest-first), runs the whole
// restarted PDLP of that LP (device.cuh, solve_body over a CTA group, with
// __syncthreads as its barrier), writes the answer, and takes the next: a
// finished LP hands its CTA back at once. LPs are packed back to back in one
// set of pools (sliced ELL of A and A^T, per-row / per-column vectors,
// iterates, control state) with per-LP offsets.
//
// An LP's arithmetic depends only on its own data and the CTA shape, never on
// which other LPs share the launch, so every answer is bit-identical whether
// the LP is solved alone or in any batch (tests/test_gpu_batch.py).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"

namespace b2 {
namespace dev {

__device__ void fill_params(KParamsBase& P, const BatchArgs& B, const LpDev& d) {
    P.m = d.m;
    P.n = d.n;
    P.A = d.A;
    P.AT = d.AT;
    P.b = d.b; P.rU = d.rU; P.dr2 = d.dr2;
    P.c = d.c; P.l = d.l; P.u = d.u; P.dc2 = d.dc2; P.x0 = d.x0;
    P.lu_const = d.lu_const; P.l_all = d.l_all; P.u_all = d.u_all;
    P.itf = d.itf;
    P.xsum = d.xsum; P.ysum = d.ysum;
    P.best_x = d.best_x; P.best_y = d.best_y;
    P.out_x = d.out_x; P.out_y = d.out_y;
    P.perm_r = d.perm_r; P.perm_c = d.perm_c;
    P.ctl = d.ctl;
    P.host_stop = B.host_stop;
    P.tol = B.tol;
    P.switch_tol = B.switch_tol;
    P.denom_p = d.denom_p;
    P.denom_d = d.denom_d;
    P.time_limit_ns = B.time_limit_ns;
    P.max_iterations = B.max_iterations;
    P.check_every = B.check_every;
    P.stall_checks = B.stall_checks;
    P.return_current = 0;
    P.mixed = B.mixed;
    P.debug_delay_ns = 0;
    P.trace = nullptr;
    P.trace_cap = 0;
    P.yield_attempts = B.tail_attempts;
}

// One LP solved by a group (one CTA or one cluster): parameters into this
// CTA's shared copy, then the phase the LP is in -- FP32 iterates and, when
// they hand over, FP64 iterates. Returns the LP's exit reason, 0 when it
// yielded at the group's deadline (its state stays in its buffers).
template <int GK>
__device__ int solve_instance(const BatchArgs& B, int i, const Group& g, KParams<float>& Pf,
                              KParams<double>& Pd, int* s_exact) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        const LpDev& d = B.lps[i];
        fill_params(Pf, B, d);
        Pf.it = d.itf;
        fill_params(Pd, B, d);
        Pd.it = d.itd;
        *s_exact = d.exact32;
        if (g.rank == 0 && d.ctl->mode == MODE_START) B.t_start[i] = gtimer();
    }
    __syncthreads();
    Ctl* c = Pf.ctl;
    if (!ld_it<GK>(&c->phase64)) {
        solve_body<GK, float, float>(Pf, g);
        group_sync<GK>(g);
        if (g.rank == 0 && tid == 0 && c->switch_req && c->exit_reason == 0) {
            c->mode = MODE_RESUME;
            c->switch_req = 0;
            c->best_merit = kInfD;
            c->best_valid = 0;
            c->stall = 0;
            c->phase64 = 1;
        }
        group_sync<GK>(g);
    }
    // a yield or an exit in the FP32 phase leaves phase64 = 0
    if (ld_it<GK>(&c->phase64) && ld_it<GK>(&c->exit_reason) == 0) {
        if (*s_exact) solve_body<GK, double, float>(Pd, g);
        else solve_body<GK, double, double>(Pd, g);
    }
    group_sync<GK>(g);
    const int ex = ld_it<GK>(&c->exit_reason);
    if (g.rank == 0 && tid == 0 && ex != 0) B.t_end[i] = gtimer();
    __syncthreads();
    return ex;
}
__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_index() {
    unsigned r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}

// Round deadline shared by the whole launch: the first CTA to start fixes the
// base time; every group yields at its first attempt boundary past base +
// round_ns, and no CTA takes a new LP after it. 0: no deadline.
__device__ __forceinline__ unsigned long long launch_deadline(const BatchArgs& B) {
    if (B.round_ns == 0) return 0ull;
    const unsigned long long now = gtimer();
    const unsigned long long old = atomicCAS(B.t0, 0ull, now);
    return (old == 0ull ? now : old) + B.round_ns;
}

// CL = CTAs per cluster. With CL > 1 the kernel is launched in clusters of CL
// CTAs: each cluster first solves large LPs together (one at a time, from the
// large-LP queue); once that queue is empty its CTAs go on alone and take
// small LPs from the other queue, like every CTA of a CL = 1 launch.
// qstatus[k] receives the exit reason of the LP at queue position k (small
// queue first, then the large queue), 0 when it yielded; positions no group
// reached keep what the host put there.
template <int CL, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_pdlp_batch(const BatchArgs B) {
    __shared__ KParams<float> Pf;
    __shared__ KParams<double> Pd;
    __shared__ int s_inst, s_pos, s_exact;
    __shared__ unsigned long long s_deadline;
    __shared__ double s_part[kCtaPartDoubles];
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) s_deadline = launch_deadline(B);
    __syncthreads();
    const unsigned long long deadline = s_deadline;
    if (CL > 1) {
        const int rank = (int)cluster_rank();
        const int cid = (int)cluster_index();
        Group g;
        g.rank = rank;
        g.size = CL;
        g.gw = rank * (NT / 32) + warp;
        g.nw = CL * (NT / 32);
        g.gt = rank * NT + tid;
        g.nt = CL * NT;
        g.part = B.cl_scratch + (size_t)cid * kClusterScratch;
        g.bcast = g.part + NSLOTS * kMaxCluster * kPartStride;
        g.bar = nullptr;
        g.abort = B.abort;
        g.timeout_ns = 0;
        g.spart = nullptr;
        g.yield_at = deadline;
        for (;;) {
            if (rank == 0 && tid == 0) {
                int i = -1;
                if (deadline == 0 || gtimer() < deadline) {
                    const unsigned k = atomicAdd(B.next_large, 1u);
                    if (k < (unsigned)B.n_large) { i = B.order_large[k]; s_pos = B.n_inst + (int)k; }
                }
                B.cl_slot[cid] = i;
            }
            group_sync<GK_CLUSTER>(g);
            const int i = __ldcg(&B.cl_slot[cid]);
            if (i < 0) break;
            const int ex = solve_instance<GK_CLUSTER>(B, i, g, Pf, Pd, &s_exact);
            if (rank == 0 && tid == 0) B.qstatus[s_pos] = ex;
        }
    }
    Group g;
    g.rank = 0;
    g.size = 1;
    g.gw = warp;
    g.nw = NT / 32;
    g.gt = tid;
    g.nt = NT;
    g.part = nullptr;
    g.bcast = B.scratch + (size_t)blockIdx.x * 8;
    g.bar = nullptr;
    g.abort = B.abort;
    g.timeout_ns = 0;
    g.spart = s_part;
    g.yield_at = deadline;
    for (;;) {
        if (tid == 0) {
            int i = -1;
            if (deadline == 0 || gtimer() < deadline) {
                const unsigned k = atomicAdd(B.next, 1u);
                if (k < (unsigned)B.n_inst) { i = B.order[k]; s_pos = (int)k; }
            }
            s_inst = i;
        }
        __syncthreads();
        const int i = s_inst;
        if (i < 0) break;
        const int ex = solve_instance<GK_CTA>(B, i, g, Pf, Pd, &s_exact);
        if (tid == 0) B.qstatus[s_pos] = ex;
    }
}

template __global__ void k_pdlp_batch<1, 128>(const BatchArgs B);
template __global__ void k_pdlp_batch<kMaxCluster, 128>(const BatchArgs B);
template __global__ void k_pdlp_batch<1, 256>(const BatchArgs B);
template __global__ void k_pdlp_batch<kMaxCluster, 256>(const BatchArgs B);
template __global__ void k_pdlp_batch<1, 512>(const BatchArgs B);
template __global__ void k_pdlp_batch<kMaxCluster, 512>(const BatchArgs B);

}  // namespace dev

// ---- host-side launch helpers (also used by serve.cu) ----
namespace {

using BatchKernel = void (*)(dev::BatchArgs);

BatchKernel batch_kernel(int cl, int nt) {
    if (cl == 1) return nt == 128 ? dev::k_pdlp_batch<1, 128> : nt == 256 ? dev::k_pdlp_batch<1, 256>
                                                                         : dev::k_pdlp_batch<1, 512>;
    return nt == 128 ? dev::k_pdlp_batch<dev::kMaxCluster, 128>
                     : nt == 256 ? dev::k_pdlp_batch<dev::kMaxCluster, 256> : dev::k_pdlp_batch<dev::kMaxCluster, 512>;
}

void cluster_cfg(cudaLaunchConfig_t& cfg, cudaLaunchAttribute* at, int n_clusters, int nt, cudaStream_t st) {
    cfg.gridDim = dim3(n_clusters * dev::kMaxCluster);
    cfg.blockDim = dim3(nt);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = dev::kMaxCluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
}

template <class T>
T* upload_vec(const std::vector<T>& h, size_t& total) {
    T* d = dalloc<T>(h.size(), total);
    if (!h.empty()) cuda_ok(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return d;
}

}  // namespace

void batch_kernel_shape(int sm_count, BatchShape& out) {
    for (int v = 0; v < 3; ++v) {
        const int nt = 128 << v;
        int occ = 0;
        cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel(1, nt), nt, 0), "occ");
        if (occ < 1) fail(B2_ERR_CUDA, "batched kernel does not fit on an SM");
        out.max_ctas_nt[v] = occ * sm_count;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        cluster_cfg(cfg, at, 1, nt, nullptr);
        int ncl = 0;
        // clusters of 16 exceed the portable size of 8: allowed per kernel
        if (cudaFuncSetAttribute(batch_kernel(dev::kMaxCluster, nt), cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess)
            cudaGetLastError();
        if (cudaOccupancyMaxActiveClusters(&ncl, batch_kernel(dev::kMaxCluster, nt), &cfg) != cudaSuccess) {
            cudaGetLastError();
            ncl = 0;
        }
        out.max_clusters_nt[v] = ncl;
    }
}

void batch_kernel_launch(const dev::BatchArgs& B, bool clusters, int nt, int units, cudaStream_t st) {
    if (clusters) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        cluster_cfg(cfg, at, units, nt, st);
        cuda_ok(cudaLaunchKernelEx(&cfg, batch_kernel(dev::kMaxCluster, nt), B), "k_pdlp_batch launch");
    } else {
        batch_kernel(1, nt)<<<units, nt, 0, st>>>(B);
        cuda_ok(cudaGetLastError(), "k_pdlp_batch launch");
    }
}

// Offsets of one LP inside the batch pools.
struct PoolOffsets {
    int64_t a_slice, at_slice, a_cv, at_cv, row_off, col_off;
};

struct BatchImpl {
    int n = 0, sm_count = 0, max_ctas = 0, last_nt = 256;
    int last_ctas = 0;               // CTAs of the last launch (both lanes)
    std::vector<char> last_cluster;  // per LP: solved by a cluster in the last launch
    BatchShape shape{};
    cudaStream_t stream = nullptr, stream2 = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_small = nullptr;
    std::vector<Layout> L;
    std::vector<PoolOffsets> off;
    std::vector<dev::LpDev> lps;  // host copy of the descriptors
    std::vector<int> order;
    int64_t sum_m = 0, sum_n = 0, sum_nnz = 0, sum_padded = 0;
    size_t bytes = 0;
    std::vector<void*> allocs;
    dev::BatchArgs args{};
    int* h_stop = nullptr;
    int* d_stop = nullptr;
    std::vector<dev::Ctl> last_ctl;

    template <class T>
    T* alloc(size_t count) {
        T* p = dalloc<T>(count, bytes);
        allocs.push_back(p);
        return p;
    }
    template <class T>
    T* up(const std::vector<T>& h) {
        T* p = upload_vec(h, bytes);
        allocs.push_back(p);
        return p;
    }

    ~BatchImpl() {
        for (void* p : allocs) cudaFree(p);
        if (h_stop) cudaFreeHost(h_stop);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_small) cudaEventDestroy(ev_small);
        if (stream2) cudaStreamDestroy(stream2);
        if (stream) cudaStreamDestroy(stream);
    }

    template <class T>
    void alloc_bufs(dev::Bufs<T>& B) {
        for (auto& p : B.x) p = alloc<T>(sum_n);
        for (auto& p : B.y) p = alloc<T>(sum_m);
        for (auto& p : B.ax) p = alloc<T>(sum_m);
        for (auto& p : B.aty) p = alloc<T>(sum_n);
        B.x_last = alloc<T>(sum_n);
        B.y_last = alloc<T>(sum_m);
    }

    template <class T>
    static dev::Bufs<T> offset_bufs(const dev::Bufs<T>& B, int64_t row_off, int64_t col_off) {
        dev::Bufs<T> o;
        o.x[0] = B.x[0] + col_off; o.x[1] = B.x[1] + col_off;
        o.y[0] = B.y[0] + row_off; o.y[1] = B.y[1] + row_off;
        o.ax[0] = B.ax[0] + row_off; o.ax[1] = B.ax[1] + row_off; o.ax[2] = B.ax[2] + row_off;
        o.aty[0] = B.aty[0] + col_off; o.aty[1] = B.aty[1] + col_off;
        o.x_last = B.x_last + col_off;
        o.y_last = B.y_last + row_off;
        return o;
    }

    void create(int n_lp, const b2_lp_view* U, const b2_lp_view* S, const double* const* Dr, const double* const* Dc,
                const b2_solve_opts& o) {
        if (n_lp <= 0) fail(B2_ERR_INVALID, "empty batch");
        n = n_lp;
        L.resize(n);
        BuildParams bp;
        bp.sigma_window = o.sigma_window;
        // host layouts, in parallel over LPs (validation errors name the LP);
        // each LP's lane target from its shape class
        
        const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        std::vector<std::string> errs(hw);
        std::vector<int> codes(hw, 0);
        for (unsigned t = 0; t < hw; ++t)
            pool.emplace_back([&, t]() {
                for (int i = (int)t; i < n; i += (int)hw) {
                    try {
                        BuildParams bpi = bp;
                        bpi.lane_target = lane_target_for(o, U[i].m, U[i].n, U[i].nnz);
                        build_layout(U[i], S[i], Dr[i], Dc[i], bpi, L[i]);
                    } catch (const Error& e) {
                        codes[t] = e.code;
                        errs[t] = "LP " + std::to_string(i) + ": " + e.msg;
                        return;
                    }
                }
            });
        for (auto& th : pool) th.join();
        for (unsigned t = 0; t < hw; ++t)
            if (codes[t]) fail(codes[t], errs[t]);

        int ndev = 0;
        cuda_ok(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
        if (ndev == 0) fail(B2_ERR_NO_DEVICE, "no CUDA device");
        int device = 0;
        cuda_ok(cudaGetDevice(&device), "cudaGetDevice");
        cuda_ok(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device), "attr");
        cuda_ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_ok(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_ok(cudaEventCreateWithFlags(&ev_small, cudaEventDisableTiming), "event");
        cuda_ok(cudaEventCreate(&ev0), "event");
        cuda_ok(cudaEventCreate(&ev1), "event");

        // pack
        off.resize(n);
        int64_t slices = 0, cv = 0;
        bool any64 = false;
        for (int i = 0; i < n; ++i) {
            const Layout& l = L[i];
            PoolOffsets& d = off[i];
            d.a_slice = slices; slices += l.A.n_slices();
            d.at_slice = slices; slices += l.AT.n_slices();
            d.a_cv = cv; cv += l.A.padded;
            d.at_cv = cv; cv += l.AT.padded;
            d.row_off = sum_m; sum_m += l.m;
            d.col_off = sum_n; sum_n += l.n;
            any64 |= !l.exact32;
            sum_nnz += l.nnz;
            sum_padded += l.A.padded + l.AT.padded;
        }
        std::vector<int32_t> h_slice((size_t)slices * 4);
        std::vector<uint32_t> h_col((size_t)cv);
        std::vector<float> h_v32((size_t)cv);
        std::vector<double> h_v64(any64 ? (size_t)cv : 0);
        std::vector<double> hb(sum_m), hrU(sum_m), hdr2(sum_m), hc(sum_n), hl(sum_n), hu(sum_n), hdc2(sum_n), hx0(sum_n);
        std::vector<int32_t> hpr(sum_m), hpc(sum_n);
        for (int i = 0; i < n; ++i) {
            const Layout& l = L[i];
            const PoolOffsets& d = off[i];
            std::copy(l.A.slice.begin(), l.A.slice.end(), h_slice.begin() + d.a_slice * 4);
            std::copy(l.AT.slice.begin(), l.AT.slice.end(), h_slice.begin() + d.at_slice * 4);
            std::copy(l.A.col.begin(), l.A.col.end(), h_col.begin() + d.a_cv);
            std::copy(l.AT.col.begin(), l.AT.col.end(), h_col.begin() + d.at_cv);
            std::copy(l.A.val32.begin(), l.A.val32.end(), h_v32.begin() + d.a_cv);
            std::copy(l.AT.val32.begin(), l.AT.val32.end(), h_v32.begin() + d.at_cv);
            if (!l.exact32) {
                std::copy(l.A.val64.begin(), l.A.val64.end(), h_v64.begin() + d.a_cv);
                std::copy(l.AT.val64.begin(), l.AT.val64.end(), h_v64.begin() + d.at_cv);
            }
            std::copy(l.b.begin(), l.b.end(), hb.begin() + d.row_off);
            std::copy(l.rU.begin(), l.rU.end(), hrU.begin() + d.row_off);
            std::copy(l.dr2.begin(), l.dr2.end(), hdr2.begin() + d.row_off);
            std::copy(l.perm_r.begin(), l.perm_r.end(), hpr.begin() + d.row_off);
            std::copy(l.c.begin(), l.c.end(), hc.begin() + d.col_off);
            std::copy(l.l.begin(), l.l.end(), hl.begin() + d.col_off);
            std::copy(l.u.begin(), l.u.end(), hu.begin() + d.col_off);
            std::copy(l.dc2.begin(), l.dc2.end(), hdc2.begin() + d.col_off);
            std::copy(l.x0.begin(), l.x0.end(), hx0.begin() + d.col_off);
            std::copy(l.perm_c.begin(), l.perm_c.end(), hpc.begin() + d.col_off);
        }
        // longest LPs first, so the tail of the launch holds the short ones
        order.resize(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b2_) {
            return L[a].A.padded + L[a].AT.padded > L[b2_].A.padded + L[b2_].AT.padded;
        });

        dev::BatchArgs& B = args;
        B.order = alloc<int>(n);
        B.next = alloc<unsigned>(1);
        B.order_large = alloc<int>(n);
        B.next_large = alloc<unsigned>(1);
        const int4* slice = reinterpret_cast<const int4*>(up(h_slice));
        const uint32_t* col = up(h_col);
        const float* v32 = up(h_v32);
        const double* v64 = any64 ? up(h_v64) : nullptr;
        const double *b = up(hb), *rU = up(hrU), *dr2 = up(hdr2);
        const double *c = up(hc), *l = up(hl), *u = up(hu), *dc2 = up(hdc2), *x0 = up(hx0);
        const int32_t *perm_r = up(hpr), *perm_c = up(hpc);
        dev::Bufs<float> itf{};
        dev::Bufs<double> itd{};
        alloc_bufs(itf);
        alloc_bufs(itd);
        double* xsum = alloc<double>(sum_n); double* ysum = alloc<double>(sum_m);
        double* best_x = alloc<double>(sum_n); double* best_y = alloc<double>(sum_m);
        double* out_x = alloc<double>(sum_n); double* out_y = alloc<double>(sum_m);
        dev::Ctl* ctl = alloc<dev::Ctl>(n);
        lps.resize(n);
        for (int i = 0; i < n; ++i) {
            const Layout& li = L[i];
            const PoolOffsets& d = off[i];
            dev::LpDev& q = lps[i];
            std::memset(&q, 0, sizeof(q));
            q.m = li.m; q.n = li.n;
            q.A.n_rows = li.m; q.A.n_slices = (int)li.A.n_slices();
            q.A.slice = slice + d.a_slice; q.A.col = col + d.a_cv; q.A.v32 = v32 + d.a_cv;
            q.A.v64 = v64 ? v64 + d.a_cv : nullptr;
            q.AT.n_rows = li.n; q.AT.n_slices = (int)li.AT.n_slices();
            q.AT.slice = slice + d.at_slice; q.AT.col = col + d.at_cv; q.AT.v32 = v32 + d.at_cv;
            q.AT.v64 = v64 ? v64 + d.at_cv : nullptr;
            q.b = b + d.row_off; q.rU = rU + d.row_off; q.dr2 = dr2 + d.row_off;
            q.c = c + d.col_off; q.l = l + d.col_off; q.u = u + d.col_off; q.dc2 = dc2 + d.col_off;
            q.x0 = x0 + d.col_off;
            q.perm_r = perm_r + d.row_off; q.perm_c = perm_c + d.col_off;
            q.itf = offset_bufs(itf, d.row_off, d.col_off);
            q.itd = offset_bufs(itd, d.row_off, d.col_off);
            q.xsum = xsum + d.col_off; q.ysum = ysum + d.row_off;
            q.best_x = best_x + d.col_off; q.best_y = best_y + d.row_off;
            q.out_x = out_x + d.col_off; q.out_y = out_y + d.row_off;
            q.ctl = ctl + i;
            q.denom_p = li.denom_p; q.denom_d = li.denom_d;
            q.exact32 = li.exact32 ? 1 : 0;
            q.lu_const = li.lu_const ? 1 : 0; q.l_all = li.l_all; q.u_all = li.u_all;
        }
        B.lps = up(lps);
        B.abort = alloc<int>(1);
        B.t_start = alloc<unsigned long long>(n);
        B.t_end = alloc<unsigned long long>(n);
        B.t0 = alloc<unsigned long long>(1);
        B.qstatus = alloc<int>(n);
        B.round_ns = 0;
        batch_kernel_shape(sm_count, shape);
        max_ctas = *std::max_element(shape.max_ctas_nt, shape.max_ctas_nt + 3);
        const int ncl_max = *std::max_element(shape.max_clusters_nt, shape.max_clusters_nt + 3);
        B.scratch = alloc<double>((size_t)max_ctas * 8);
        B.cl_slot = alloc<int>(std::max(1, ncl_max));
        B.cl_scratch = alloc<double>((size_t)std::max(1, ncl_max) * dev::kClusterScratch);
        cuda_ok(cudaHostAlloc((void**)&h_stop, sizeof(int), cudaHostAllocMapped), "cudaHostAlloc");
        *h_stop = 0;
        cuda_ok(cudaHostGetDevicePointer((void**)&d_stop, h_stop, 0), "cudaHostGetDevicePointer");
        B.host_stop = d_stop;
        cuda_ok(cudaDeviceSynchronize(), "batch create");
        // host copies of the big layout arrays are no longer needed
        for (auto& li : L) {
            std::vector<uint32_t>().swap(li.A.col);
            std::vector<uint32_t>().swap(li.AT.col);
            std::vector<float>().swap(li.A.val32);
            std::vector<float>().swap(li.AT.val32);
            std::vector<double>().swap(li.A.val64);
            std::vector<double>().swap(li.AT.val64);
        }
    }

    void solve(const b2_solve_opts& o, const volatile int32_t* stop_flag, b2_result* res, double* total_ms) {
        cudaStream_t st = o.stream ? (cudaStream_t)o.stream : stream;
        // queues: LPs with at least `big` stored entries go to whole clusters,
        // the rest to single CTAs; both longest first
        // defaults from a sweep on the 4,096-LP family (B200): 512-thread CTAs,
        // no clusters (clusters of 8 cut the longest LP's time but cost more
        // CTA-time than they save)
        const int64_t big = o.batch_cluster_nnz > 0 ? o.batch_cluster_nnz : INT64_MAX;
        const int nt = o.batch_block == 128 || o.batch_block == 256 ? o.batch_block : 512;
        const int ntx = batch_nt_index(nt);
        last_nt = nt;
        std::vector<int> small_q, large_q;
        last_cluster.assign(n, 0);
        for (int i : order) {
            if (shape.max_clusters_nt[ntx] > 0 && L[i].A.padded + L[i].AT.padded >= big) {
                large_q.push_back(i);
                last_cluster[i] = 1;
            } else {
                small_q.push_back(i);
            }
        }
        if (o.max_iterations < 0) fail(B2_ERR_INVALID, "max_iterations < 0");
        std::vector<dev::Ctl> h(n);
        for (int i = 0; i < n; ++i) init_ctl(h[i], L[i], o.precision != B2_PREC_MIXED);
        dev::BatchArgs B = args;
        B.n_inst = (int)small_q.size();
        B.n_large = (int)large_q.size();
        if (!small_q.empty())
            cuda_ok(cudaMemcpyAsync((void*)B.order, small_q.data(), sizeof(int) * small_q.size(), cudaMemcpyHostToDevice, st), "queue");
        if (!large_q.empty())
            cuda_ok(cudaMemcpyAsync((void*)B.order_large, large_q.data(), sizeof(int) * large_q.size(), cudaMemcpyHostToDevice, st), "queue");
        B.tol = o.tol;
        B.switch_tol = o.switch_tol;
        B.time_limit_ns = o.time_limit_s > 0 ? o.time_limit_s * 1e9 : 0.0;
        B.max_iterations = o.max_iterations;
        B.check_every = std::max(1, o.check_every);
        B.stall_checks = o.stall_checks > 0 ? o.stall_checks : 32;
        B.mixed = o.precision == B2_PREC_MIXED;
        B.round_ns = 0;
        const bool tail = o.batch_tail_attempts > 0 && large_q.empty() && shape.max_clusters_nt[ntx] > 0;
        B.tail_attempts = tail ? o.batch_tail_attempts : 0;
        if (tail) cuda_ok(cudaMemsetAsync(B.qstatus, 0xff, sizeof(int) * small_q.size(), st), "memset");
        *h_stop = stop_requested(o, stop_flag) ? 1 : 0;
        cuda_ok(cudaMemcpyAsync(lps_ctl(0), h.data(), sizeof(dev::Ctl) * n, cudaMemcpyHostToDevice, st), "ctl upload");
        cuda_ok(cudaMemsetAsync(B.next, 0, sizeof(unsigned), st), "memset");
        cuda_ok(cudaMemsetAsync(B.next_large, 0, sizeof(unsigned), st), "memset");
        cuda_ok(cudaMemsetAsync(B.abort, 0, sizeof(int), st), "memset");
        cuda_ok(cudaMemsetAsync(B.t0, 0, sizeof(unsigned long long), st), "memset");
        cuda_ok(cudaEventRecord(ev0, st), "event");
        if (!large_q.empty()) {
            // clusters for the large LPs on at most half of the GPU, a one-CTA
            // launch on the rest beside them (second stream); both take from
            // the same queues, so the small LPs start at once
            int ncl = std::min((int)large_q.size(), std::max(1, shape.max_clusters_nt[ntx] / 2));
            if (o.max_ctas > 0) ncl = std::max(1, std::min(ncl, o.max_ctas / dev::kMaxCluster));
            batch_kernel_launch(B, true, nt, ncl, st);
            last_ctas = ncl * dev::kMaxCluster;
            const int rest = (o.max_ctas > 0 ? std::min(o.max_ctas, shape.max_ctas_nt[ntx]) : shape.max_ctas_nt[ntx]) -
                             ncl * dev::kMaxCluster;
            if (!small_q.empty() && rest > 0) {
                cuda_ok(cudaStreamWaitEvent(stream2, ev0, 0), "wait");
                dev::BatchArgs Bs = B;
                Bs.n_large = 0;
                batch_kernel_launch(Bs, false, nt, std::min(rest, (int)small_q.size()), stream2);
                last_ctas += std::min(rest, (int)small_q.size());
                cuda_ok(cudaEventRecord(ev_small, stream2), "event");
                cuda_ok(cudaStreamWaitEvent(st, ev_small, 0), "wait");
            }
        } else {
            const int ctas = std::max(1, std::min(shape.max_ctas_nt[ntx], o.max_ctas > 0 ? std::min(o.max_ctas, n) : n));
            batch_kernel_launch(B, false, nt, ctas, st);
            last_ctas = ctas;
        }
        auto wait_for = [&](cudaEvent_t ev) {
            for (;;) {
                cudaError_t q = cudaEventQuery(ev);
                if (q == cudaSuccess) break;
                if (q != cudaErrorNotReady) cuda_ok(q, "batched kernel");
                if (stop_requested(o, stop_flag)) *(volatile int*)h_stop = 1;
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
        };
        if (tail) {
            // the tail lane: LPs that yielded at batch_tail_attempts finish on
            // clusters of 16 CTAs, on the whole GPU, once the one-CTA launch is done
            cuda_ok(cudaEventRecord(ev1, st), "event");
            wait_for(ev1);
            std::vector<int> qs(small_q.size());
            if (!qs.empty())
                cuda_ok(cudaMemcpy(qs.data(), B.qstatus, sizeof(int) * qs.size(), cudaMemcpyDeviceToHost), "status");
            std::vector<int> yielded;
            for (size_t k = 0; k < qs.size(); ++k)
                if (qs[k] == 0) yielded.push_back(small_q[k]);
            if (!yielded.empty() && !*h_stop) {
                cuda_ok(cudaMemcpyAsync((void*)B.order_large, yielded.data(), sizeof(int) * yielded.size(),
                                        cudaMemcpyHostToDevice, st), "queue");
                cuda_ok(cudaMemsetAsync(B.next_large, 0, sizeof(unsigned), st), "memset");
                dev::BatchArgs Bt = B;
                Bt.n_inst = 0;
                Bt.n_large = (int)yielded.size();
                Bt.tail_attempts = 0;
                const int ncl = std::min((int)yielded.size(), shape.max_clusters_nt[ntx]);
                batch_kernel_launch(Bt, true, nt, ncl, st);
                last_ctas = std::max(last_ctas, ncl * dev::kMaxCluster);
                for (int i : yielded) last_cluster[i] = 1;
            }
        }
        cuda_ok(cudaEventRecord(ev1, st), "event");
        wait_for(ev1);
        float ms = 0.0f;
        cuda_ok(cudaEventElapsedTime(&ms, ev0, ev1), "elapsed");
        if (total_ms) *total_ms = ms;
        last_ctl.resize(n);
        cuda_ok(cudaMemcpy(last_ctl.data(), lps_ctl(0), sizeof(dev::Ctl) * n, cudaMemcpyDeviceToHost), "ctl download");
        std::vector<unsigned long long> t0(n), t1(n);
        cuda_ok(cudaMemcpy(t0.data(), B.t_start, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost), "t0");
        cuda_ok(cudaMemcpy(t1.data(), B.t_end, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost), "t1");
        if (res) {
            for (int i = 0; i < n; ++i) {
                fill_result(last_ctl[i], res[i]);
                res[i].device_ms = (double)(t1[i] - t0[i]) * 1e-6;
                res[i].objective = std::numeric_limits<double>::quiet_NaN();
                res[i].group_ctas = last_cluster[i] ? dev::kMaxCluster : 1;
            }
        }
    }

    // control states of the batch are contiguous (one pool)
    dev::Ctl* lps_ctl(int i) const { return lps[0].ctl + i; }

    void solution(int i, double* x, double* y) {
        if (i < 0 || i >= n) fail(B2_ERR_INVALID, "LP index out of range");
        if (x && L[i].n)
            cuda_ok(cudaMemcpy(x, lps[i].out_x, sizeof(double) * L[i].n, cudaMemcpyDeviceToHost), "x");
        if (y && L[i].m)
            cuda_ok(cudaMemcpy(y, lps[i].out_y, sizeof(double) * L[i].m, cudaMemcpyDeviceToHost), "y");
    }

    // y = A x (which 0) or A^T x (which 1) of LP i through the packed pools
    // and the solver's SpMV (FP64 accumulation); x, y in the caller's order.
    void spmv(int i, int which, const double* x, double* y) {
        if (i < 0 || i >= n) fail(B2_ERR_INVALID, "LP index out of range");
        const Layout& l = L[i];
        spmv_sell(which == 0 ? lps[i].A : lps[i].AT, l, which, l.exact32, stream, x, y);
    }

    void info(b2_batch_info* inf) {
        std::memset(inf, 0, sizeof(*inf));
        inf->n_lp = n;
        inf->sum_m = sum_m;
        inf->sum_n = sum_n;
        inf->sum_nnz = sum_nnz;
        inf->sum_padded = sum_padded;
        inf->max_ctas = max_ctas;
        inf->threads_per_cta = last_nt;
        inf->device_bytes = (int64_t)bytes;
        inf->last_launch_ctas = last_ctas;
    }
};

// Initial control state of an LP (pdlp_algo.hpp:67-102).
void init_ctl(dev::Ctl& c, const Layout& l, bool fp64_only) {
    std::memset(&c, 0, sizeof(c));
    c.eta = l.eta0;
    c.omega = l.omega0;
    c.merit_last_restart = c.merit_prev_cand = c.best_merit = std::numeric_limits<double>::infinity();
    c.ax_cur = 0; c.ax_nxt = 1; c.ax_avg = 2; c.aty_cur = 0; c.aty_avg = 1;
    c.mode = dev::MODE_START;
    c.phase64 = fp64_only ? 1 : 0;
}

void fill_result(const dev::Ctl& f, b2_result& r) {
    std::memset(&r, 0, sizeof(r));
    r.iterations = f.attempts;
    r.restarts = f.restarts;
    r.converged = f.exit_reason == B2_EXIT_CONVERGED;
    r.accepted = f.accepted;
    r.eps_P = f.out_eps[0];
    r.eps_D = f.out_eps[1];
    r.eps_G = f.out_eps[2];
    r.exit_reason = f.exit_reason;
    r.checks = f.checks;
    r.fp32_attempts = f.fp32_attempts;
    r.fp32_accepted = f.fp32_accepted;
    r.final_eta = f.eta;
    r.final_omega = f.omega;
}

// y = M x through a device sliced matrix (FP64 accumulation); x, y in the
// caller's order of that LP.
void spmv_sell(const dev::SellDev& S, const Layout& l, int which, bool exact32, cudaStream_t stream, const double* x,
               double* y) {
    const int rows = which == 0 ? l.m : l.n, cols = which == 0 ? l.n : l.m;
    const std::vector<int32_t>& in_perm = which == 0 ? l.perm_c : l.perm_r;
    const std::vector<int32_t>& out_perm = which == 0 ? l.perm_r : l.perm_c;
    std::vector<double> xd(std::max(cols, 1)), yd(std::max(rows, 1));
    for (int j = 0; j < cols; ++j) xd[j] = x[in_perm[j]];
    double *dx = nullptr, *dy = nullptr;
    cuda_ok(cudaMalloc(&dx, xd.size() * sizeof(double)), "cudaMalloc");
    cuda_ok(cudaMalloc(&dy, yd.size() * sizeof(double)), "cudaMalloc");
    cuda_ok(cudaMemcpy(dx, xd.data(), xd.size() * sizeof(double), cudaMemcpyHostToDevice), "H2D");
    if (S.n_slices > 0) {
        if (exact32) dev::k_spmv<double, float, double><<<std::max(1, S.n_slices / 8 + 1), 256, 0, stream>>>(S, dx, dy);
        else dev::k_spmv<double, double, double><<<std::max(1, S.n_slices / 8 + 1), 256, 0, stream>>>(S, dx, dy);
    }
    cuda_ok(cudaGetLastError(), "k_spmv");
    cuda_ok(cudaStreamSynchronize(stream), "k_spmv");
    cuda_ok(cudaMemcpy(yd.data(), dy, yd.size() * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
    cudaFree(dx);
    cudaFree(dy);
    for (int r = 0; r < rows; ++r) y[out_perm[r]] = yd[r];
}

BatchImpl* batch_create(int n, const b2_lp_view* U, const b2_lp_view* S, const double* const* Dr,
                        const double* const* Dc, const b2_solve_opts& o) {
    std::unique_ptr<BatchImpl> b(new BatchImpl());
    b->create(n, U, S, Dr, Dc, o);
    return b.release();
}
void batch_destroy(BatchImpl* b) { delete b; }
void batch_solve(BatchImpl* b, const b2_solve_opts& o, const volatile int32_t* stop, b2_result* res, double* ms) {
    b->solve(o, stop, res, ms);
}
void batch_solution(BatchImpl* b, int i, double* x, double* y) { b->solution(i, x, y); }
void batch_info(BatchImpl* b, b2_batch_info* inf) { b->info(inf); }
void batch_spmv(BatchImpl* b, int i, int which, const double* x, double* y) { b->spmv(i, which, x, y); }

// ------------------------------------------------------- shape classes
int32_t shape_class(int32_t m, int32_t n, int64_t nnz) {
    (void)n;
    const int64_t size_edges[4] = {4096, 16384, 65536, 262144};
    int sz = 0;
    while (sz < 4 && nnz >= size_edges[sz]) ++sz;
    const double per_row = m > 0 ? (double)nnz / (double)m : 0.0;
    const double row_edges[3] = {8.0, 16.0, 32.0};
    int rw = 0;
    while (rw < 3 && per_row >= row_edges[rw]) ++rw;
    return sz * 4 + rw;
}

// The built-in table: b2_batch_autotune on a B200 over 1,024 LPs of the batch
// family (m log-uniform on [50, 5,000], n = U[2,4] m, 4-10 entries a column),
// FP64 attempts, 512-thread CTAs. Measured time per attempt of the winner (us):
// class 1: 5.15, 2: 4.71, 3: 4.93, 5: 9.75, 6: 7.78, 7: 8.14, 9: 38.7,
// 10: 36.9, 11: 25.4, 13: 81.6, 14: 79.5, 15: 94.5. From 4K nonzeros, rows of
// 16 or more entries run faster at 32 entries per lane (half as many lanes per
// row); classes the family does not reach keep 16.
void default_tune_table(b2_tune_table& t) {
    static const int32_t kB200[B2_TUNE_CLASSES] = {16, 16, 16, 16, 16, 16, 32, 32, 16, 16,
                                                    32, 32, 16, 16, 32, 32, 16, 16, 16, 16};
    std::memset(&t, 0, sizeof(t));
    for (int k = 0; k < B2_TUNE_CLASSES; ++k) t.lane_target[k] = kB200[k];
}

int lane_target_for(const b2_solve_opts& o, int32_t m, int32_t n, int64_t nnz) {
    if (o.lane_target > 0) return o.lane_target;
    b2_tune_table def;
    const b2_tune_table* t = o.tune;
    if (!t) {
        default_tune_table(def);
        t = &def;
    }
    const int v = t->lane_target[shape_class(m, n, nnz)];
    return v > 0 ? v : 16;
}

// For every shape class present: up to four of its LPs, one CTA each, 512
// FP64 attempts under each candidate lane target; the fastest by summed
// device time per attempt wins, 16 unless another is at least 3 % faster.
void batch_autotune(int n, const b2_lp_view* U, const b2_lp_view* S, const double* const* Dr, const double* const* Dc,
                    const b2_solve_opts& o, b2_tune_table& out) {
    std::memset(&out, 0, sizeof(out));
    std::vector<std::vector<int>> members(B2_TUNE_CLASSES);
    for (int i = 0; i < n; ++i) {
        std::vector<int>& v = members[shape_class(U[i].m, U[i].n, U[i].nnz)];
        if (v.size() < 4) v.push_back(i);
    }
    const int cands[4] = {4, 8, 16, 32};
    for (int k = 0; k < B2_TUNE_CLASSES; ++k) {
        const std::vector<int>& v = members[k];
        if (v.empty()) continue;
        std::vector<b2_lp_view> u, s;
        std::vector<const double*> dr, dc;
        for (int i : v) {
            u.push_back(U[i]);
            s.push_back(S[i]);
            dr.push_back(Dr[i]);
            dc.push_back(Dc[i]);
        }
        double best = 0.0, t16 = 0.0;
        int pick = 16;
        double us[4] = {0, 0, 0, 0};
        for (int c = 0; c < 4; ++c) {
            b2_solve_opts oo = o;
            oo.lane_target = cands[c];
            oo.precision = B2_PREC_FP64;
            oo.max_iterations = 512;
            oo.tol = 1e-30;  // never converges: every candidate runs the same 512 attempts
            oo.time_limit_s = 0.0;
            std::unique_ptr<BatchImpl> b(new BatchImpl());
            b->create((int)v.size(), u.data(), s.data(), dr.data(), dc.data(), oo);
            std::vector<b2_result> res(v.size());
            double ms = 0.0;
            b->solve(oo, nullptr, res.data(), &ms);
            double dev = 0.0, att = 0.0;
            for (const b2_result& r : res) {
                dev += r.device_ms;
                att += r.iterations;
            }
            us[c] = att > 0 ? 1e3 * dev / att : 0.0;
            if (cands[c] == 16) t16 = us[c];
        }
        best = t16;
        for (int c = 0; c < 4; ++c)
            if (us[c] > 0 && us[c] < best * 0.97 && us[c] < best) { best = us[c]; pick = cands[c]; }
        out.lane_target[k] = pick;
        out.us_per_attempt[k] = best;
    }
}

}  // namespace b2
