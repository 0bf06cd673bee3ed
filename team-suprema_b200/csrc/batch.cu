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

#include "device.cuh"

namespace b2 {
namespace dev {

// Offsets of one LP inside the batch pools.
struct InstDesc {
    int m, n, a_nslices, at_nslices;
    long long a_slice, at_slice, a_cv, at_cv, row_off, col_off;
    double denom_p, denom_d;
    int exact32, pad;
};

struct BatchArgs {
    int n_inst;
    const int* order;
    unsigned* next;
    const InstDesc* inst;
    const int4* slice;
    const uint32_t* col;
    const float* v32;
    const double* v64;
    const double *b, *rU, *dr2, *c, *l, *u, *dc2, *x0;
    const int32_t *perm_r, *perm_c;
    Bufs<float> itf;
    Bufs<double> itd;
    double *xsum, *ysum, *best_x, *best_y, *out_x, *out_y;
    Ctl* ctl;
    double* scratch;  // per CTA: NSLOTS * kPartStride partials + 8 broadcast words
    const volatile int* host_stop;
    int* abort;
    unsigned long long *t_start, *t_end;
    double tol, switch_tol, time_limit_ns;
    int max_iterations, check_every, stall_checks, mixed;
    // large LPs, solved by a whole cluster
    int n_large;
    const int* order_large;
    unsigned* next_large;
    int* cl_slot;        // per cluster: the LP it is on
    double* cl_scratch;  // per cluster: partial sums + broadcast words
};

constexpr int kMaxCluster = 8;
constexpr int kClusterScratch = NSLOTS * kMaxCluster * kPartStride + 8;

template <class T>
__device__ Bufs<T> offset_bufs(const Bufs<T>& B, long long row_off, long long col_off) {
    Bufs<T> o;
    o.x[0] = B.x[0] + col_off; o.x[1] = B.x[1] + col_off;
    o.y[0] = B.y[0] + row_off; o.y[1] = B.y[1] + row_off;
    o.ax[0] = B.ax[0] + row_off; o.ax[1] = B.ax[1] + row_off; o.ax[2] = B.ax[2] + row_off;
    o.aty[0] = B.aty[0] + col_off; o.aty[1] = B.aty[1] + col_off;
    o.x_last = B.x_last + col_off;
    o.y_last = B.y_last + row_off;
    return o;
}

__device__ void fill_params(KParamsBase& P, const BatchArgs& B, const InstDesc& d, int i) {
    P.m = d.m;
    P.n = d.n;
    P.A.n_rows = d.m;
    P.A.n_slices = d.a_nslices;
    P.A.slice = B.slice + d.a_slice;
    P.A.col = B.col + d.a_cv;
    P.A.v32 = B.v32 + d.a_cv;
    P.A.v64 = B.v64 ? B.v64 + d.a_cv : nullptr;
    P.AT.n_rows = d.n;
    P.AT.n_slices = d.at_nslices;
    P.AT.slice = B.slice + d.at_slice;
    P.AT.col = B.col + d.at_cv;
    P.AT.v32 = B.v32 + d.at_cv;
    P.AT.v64 = B.v64 ? B.v64 + d.at_cv : nullptr;
    P.b = B.b + d.row_off; P.rU = B.rU + d.row_off; P.dr2 = B.dr2 + d.row_off;
    P.c = B.c + d.col_off; P.l = B.l + d.col_off; P.u = B.u + d.col_off; P.dc2 = B.dc2 + d.col_off;
    P.x0 = B.x0 + d.col_off;
    P.itf = offset_bufs(B.itf, d.row_off, d.col_off);
    P.xsum = B.xsum + d.col_off; P.ysum = B.ysum + d.row_off;
    P.best_x = B.best_x + d.col_off; P.best_y = B.best_y + d.row_off;
    P.out_x = B.out_x + d.col_off; P.out_y = B.out_y + d.row_off;
    P.perm_r = B.perm_r + d.row_off; P.perm_c = B.perm_c + d.col_off;
    P.ctl = B.ctl + i;
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
}

// One LP solved by a group (one CTA or one cluster): parameters into this
// CTA's shared copy, the FP32 phase and, when it hands over, the FP64 phase.
template <int GK>
__device__ void solve_instance(const BatchArgs& B, int i, const Group& g, KParams<float>& Pf,
                               KParams<double>& Pd) {
    const int tid = threadIdx.x;
    const InstDesc d = B.inst[i];
    if (tid == 0) {
        fill_params(Pf, B, d, i);
        Pf.it = offset_bufs(B.itf, d.row_off, d.col_off);
        fill_params(Pd, B, d, i);
        Pd.it = offset_bufs(B.itd, d.row_off, d.col_off);
        if (g.rank == 0) B.t_start[i] = gtimer();
    }
    __syncthreads();
    bool fp64 = !B.mixed;
    if (B.mixed) {
        solve_body<GK, float, float>(Pf, g);
        if (g.rank == 0 && tid == 0) {
            Ctl* c = B.ctl + i;
            if (c->switch_req && c->exit_reason == 0) {
                c->mode = MODE_RESUME;
                c->switch_req = 0;
                c->best_merit = kInfD;
                c->best_valid = 0;
                c->stall = 0;
            }
        }
        group_sync<GK>(g);
        fp64 = ld_it<GK>(&B.ctl[i].mode) == MODE_RESUME;
    }
    if (fp64) {
        if (d.exact32) solve_body<GK, double, float>(Pd, g);
        else solve_body<GK, double, double>(Pd, g);
    }
    if (g.rank == 0 && tid == 0) B.t_end[i] = gtimer();
    __syncthreads();
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

// CL = CTAs per cluster. With CL > 1 the kernel is launched in clusters of CL
// CTAs: each cluster first solves large LPs together (one at a time, from the
// large-LP queue); once that queue is empty its CTAs go on alone and take
// small LPs from the other queue, like every CTA of a CL = 1 launch.
template <int CL, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_pdlp_batch(const BatchArgs B) {
    __shared__ KParams<float> Pf;
    __shared__ KParams<double> Pd;
    __shared__ int s_inst;
    __shared__ double s_part[NSLOTS * kPartStride];
    const int tid = threadIdx.x, warp = tid >> 5;
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
        for (;;) {
            if (rank == 0 && tid == 0) {
                const unsigned k = atomicAdd(B.next_large, 1u);
                B.cl_slot[cid] = k < (unsigned)B.n_large ? B.order_large[k] : -1;
            }
            group_sync<GK_CLUSTER>(g);
            const int i = __ldcg(&B.cl_slot[cid]);
            if (i < 0) break;
            solve_instance<GK_CLUSTER>(B, i, g, Pf, Pd);
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
    for (;;) {
        if (tid == 0) {
            const unsigned k = atomicAdd(B.next, 1u);
            s_inst = k < (unsigned)B.n_inst ? B.order[k] : -1;
        }
        __syncthreads();
        const int i = s_inst;
        if (i < 0) break;
        solve_instance<GK_CTA>(B, i, g, Pf, Pd);
    }
}

template __global__ void k_pdlp_batch<1, 128>(const BatchArgs B);
template __global__ void k_pdlp_batch<kMaxCluster, 128>(const BatchArgs B);
template __global__ void k_pdlp_batch<1, 256>(const BatchArgs B);
template __global__ void k_pdlp_batch<kMaxCluster, 256>(const BatchArgs B);
template __global__ void k_pdlp_batch<1, 512>(const BatchArgs B);
template __global__ void k_pdlp_batch<kMaxCluster, 512>(const BatchArgs B);

}  // namespace dev

namespace {

template <class T>
T* upload_vec(const std::vector<T>& h, size_t& total) {
    T* d = dalloc<T>(h.size(), total);
    if (!h.empty()) cuda_ok(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return d;
}

}  // namespace

struct BatchImpl {
    int n = 0, sm_count = 0, max_ctas = 0, last_nt = 256;
    int max_ctas_nt[3] = {0, 0, 0}, max_clusters_nt[3] = {0, 0, 0};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<Layout> L;
    std::vector<dev::InstDesc> desc;
    std::vector<int64_t> row_off, col_off;
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

    void create(int n_lp, const b2_lp_view* U, const b2_lp_view* S, const double* const* Dr, const double* const* Dc,
                const b2_solve_opts& o) {
        if (n_lp <= 0) fail(B2_ERR_INVALID, "empty batch");
        n = n_lp;
        L.resize(n);
        BuildParams bp;
        bp.lane_target = o.lane_target;
        bp.sigma_window = o.sigma_window;
        // host layouts, in parallel over LPs (validation errors name the LP)
        const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        std::vector<std::string> errs(hw);
        std::vector<int> codes(hw, 0);
        for (unsigned t = 0; t < hw; ++t)
            pool.emplace_back([&, t]() {
                for (int i = (int)t; i < n; i += (int)hw) {
                    try {
                        build_layout(U[i], S[i], Dr[i], Dc[i], bp, L[i]);
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
        cuda_ok(cudaEventCreate(&ev0), "event");
        cuda_ok(cudaEventCreate(&ev1), "event");

        // pack
        desc.resize(n);
        row_off.resize(n);
        col_off.resize(n);
        int64_t slices = 0, cv = 0;
        bool any64 = false;
        for (int i = 0; i < n; ++i) {
            const Layout& l = L[i];
            dev::InstDesc& d = desc[i];
            d.m = l.m; d.n = l.n;
            d.a_nslices = (int)l.A.n_slices(); d.at_nslices = (int)l.AT.n_slices();
            d.a_slice = slices; slices += l.A.n_slices();
            d.at_slice = slices; slices += l.AT.n_slices();
            d.a_cv = cv; cv += l.A.padded;
            d.at_cv = cv; cv += l.AT.padded;
            d.row_off = row_off[i] = sum_m; sum_m += l.m;
            d.col_off = col_off[i] = sum_n; sum_n += l.n;
            d.denom_p = l.denom_p; d.denom_d = l.denom_d;
            d.exact32 = l.exact32 ? 1 : 0;
            d.pad = 0;
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
            const dev::InstDesc& d = desc[i];
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
        B.n_inst = n;
        B.order = alloc<int>(n);
        B.next = alloc<unsigned>(1);
        B.order_large = alloc<int>(n);
        B.next_large = alloc<unsigned>(1);
        B.inst = up(desc);
        B.slice = reinterpret_cast<const int4*>(up(h_slice));
        B.col = up(h_col);
        B.v32 = up(h_v32);
        B.v64 = any64 ? up(h_v64) : nullptr;
        B.b = up(hb); B.rU = up(hrU); B.dr2 = up(hdr2);
        B.c = up(hc); B.l = up(hl); B.u = up(hu); B.dc2 = up(hdc2); B.x0 = up(hx0);
        B.perm_r = up(hpr); B.perm_c = up(hpc);
        alloc_bufs(B.itf);
        alloc_bufs(B.itd);
        B.xsum = alloc<double>(sum_n); B.ysum = alloc<double>(sum_m);
        B.best_x = alloc<double>(sum_n); B.best_y = alloc<double>(sum_m);
        B.out_x = alloc<double>(sum_n); B.out_y = alloc<double>(sum_m);
        B.ctl = alloc<dev::Ctl>(n);
        B.abort = alloc<int>(1);
        B.t_start = alloc<unsigned long long>(n);
        B.t_end = alloc<unsigned long long>(n);
        for (int v = 0; v < 3; ++v) {
            const int nt = 128 << v;
            int occ = 0;
            cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel(1, nt), nt, 0), "occ");
            if (occ < 1) fail(B2_ERR_CUDA, "batched kernel does not fit on an SM");
            max_ctas_nt[v] = occ * sm_count;
            // clusters of kMaxCluster CTAs for the large LPs
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute at[1];
            cluster_cfg(cfg, at, 1, nt);
            int ncl = 0;
            if (cudaOccupancyMaxActiveClusters(&ncl, kernel(dev::kMaxCluster, nt), &cfg) != cudaSuccess) {
                cudaGetLastError();
                ncl = 0;
            }
            max_clusters_nt[v] = ncl;
        }
        max_ctas = *std::max_element(max_ctas_nt, max_ctas_nt + 3);
        const int ncl_max = *std::max_element(max_clusters_nt, max_clusters_nt + 3);
        B.scratch = alloc<double>((size_t)max_ctas * 8);
        B.cl_slot = alloc<int>(std::max(1, ncl_max));
        B.cl_scratch = alloc<double>((size_t)std::max(1, ncl_max) * dev::kClusterScratch);
        cuda_ok(cudaHostAlloc((void**)&h_stop, sizeof(int), cudaHostAllocMapped), "cudaHostAlloc");
        *h_stop = 0;
        cuda_ok(cudaHostGetDevicePointer((void**)&d_stop, h_stop, 0), "cudaHostGetDevicePointer");
        B.host_stop = d_stop;
        cuda_ok(cudaDeviceSynchronize(), "batch create");
        // host copies of the big layout arrays are no longer needed
        for (auto& l : L) {
            std::vector<uint32_t>().swap(l.A.col);
            std::vector<uint32_t>().swap(l.AT.col);
            std::vector<float>().swap(l.A.val32);
            std::vector<float>().swap(l.AT.val32);
            std::vector<double>().swap(l.A.val64);
            std::vector<double>().swap(l.AT.val64);
        }
    }

    static void (*kernel(int cl, int nt))(dev::BatchArgs) {
        if (cl == 1) return nt == 128 ? dev::k_pdlp_batch<1, 128> : nt == 256 ? dev::k_pdlp_batch<1, 256>
                                                                             : dev::k_pdlp_batch<1, 512>;
        return nt == 128 ? dev::k_pdlp_batch<dev::kMaxCluster, 128>
                         : nt == 256 ? dev::k_pdlp_batch<dev::kMaxCluster, 256> : dev::k_pdlp_batch<dev::kMaxCluster, 512>;
    }

    static int nt_index(int nt) { return nt == 128 ? 0 : nt == 256 ? 1 : 2; }

    void cluster_cfg(cudaLaunchConfig_t& cfg, cudaLaunchAttribute* at, int n_clusters, int nt) {
        cfg.gridDim = dim3(n_clusters * dev::kMaxCluster);
        cfg.blockDim = dim3(nt);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = dev::kMaxCluster;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
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
        const int ntx = nt_index(nt);
        last_nt = nt;
        std::vector<int> small_q, large_q;
        for (int i : order) {
            if (max_clusters_nt[ntx] > 0 && L[i].A.padded + L[i].AT.padded >= big) large_q.push_back(i);
            else small_q.push_back(i);
        }
        if (o.max_iterations < 0) fail(B2_ERR_INVALID, "max_iterations < 0");
        std::vector<dev::Ctl> h(n);
        for (int i = 0; i < n; ++i) {
            dev::Ctl& c = h[i];
            std::memset(&c, 0, sizeof(c));
            c.eta = L[i].eta0;
            c.omega = L[i].omega0;
            c.merit_last_restart = c.merit_prev_cand = c.best_merit = std::numeric_limits<double>::infinity();
            c.ax_cur = 0; c.ax_nxt = 1; c.ax_avg = 2; c.aty_cur = 0; c.aty_avg = 1;
            c.mode = dev::MODE_START;
        }
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
        *h_stop = stop_flag ? *stop_flag : 0;
        cuda_ok(cudaMemcpyAsync(B.ctl, h.data(), sizeof(dev::Ctl) * n, cudaMemcpyHostToDevice, st), "ctl upload");
        cuda_ok(cudaMemsetAsync(B.next, 0, sizeof(unsigned), st), "memset");
        cuda_ok(cudaMemsetAsync(B.next_large, 0, sizeof(unsigned), st), "memset");
        cuda_ok(cudaMemsetAsync(B.abort, 0, sizeof(int), st), "memset");
        cuda_ok(cudaEventRecord(ev0, st), "event");
        if (!large_q.empty()) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute at[1];
            int ncl = max_clusters_nt[ntx];
            if (o.max_ctas > 0) ncl = std::max(1, std::min(ncl, o.max_ctas / dev::kMaxCluster));
            cluster_cfg(cfg, at, ncl, nt);
            cfg.stream = st;
            cuda_ok(cudaLaunchKernelEx(&cfg, kernel(dev::kMaxCluster, nt), (const dev::BatchArgs)B), "k_pdlp_batch launch");
        } else {
            const int ctas = std::max(1, std::min(max_ctas_nt[ntx], o.max_ctas > 0 ? std::min(o.max_ctas, n) : n));
            kernel(1, nt)<<<ctas, nt, 0, st>>>(B);
        }
        cuda_ok(cudaGetLastError(), "k_pdlp_batch launch");
        cuda_ok(cudaEventRecord(ev1, st), "event");
        for (;;) {
            cudaError_t q = cudaEventQuery(ev1);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) cuda_ok(q, "batched kernel");
            if (stop_flag && *stop_flag) *(volatile int*)h_stop = 1;
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
        float ms = 0.0f;
        cuda_ok(cudaEventElapsedTime(&ms, ev0, ev1), "elapsed");
        if (total_ms) *total_ms = ms;
        last_ctl.resize(n);
        cuda_ok(cudaMemcpy(last_ctl.data(), B.ctl, sizeof(dev::Ctl) * n, cudaMemcpyDeviceToHost), "ctl download");
        std::vector<unsigned long long> t0(n), t1(n);
        cuda_ok(cudaMemcpy(t0.data(), B.t_start, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost), "t0");
        cuda_ok(cudaMemcpy(t1.data(), B.t_end, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost), "t1");
        if (res) {
            for (int i = 0; i < n; ++i) {
                const dev::Ctl& f = last_ctl[i];
                b2_result& r = res[i];
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
                r.device_ms = (double)(t1[i] - t0[i]) * 1e-6;
                r.final_eta = f.eta;
                r.final_omega = f.omega;
                r.objective = std::numeric_limits<double>::quiet_NaN();
            }
        }
    }

    void solution(int i, double* x, double* y) {
        if (i < 0 || i >= n) fail(B2_ERR_INVALID, "LP index out of range");
        if (x && L[i].n)
            cuda_ok(cudaMemcpy(x, args.out_x + col_off[i], sizeof(double) * L[i].n, cudaMemcpyDeviceToHost), "x");
        if (y && L[i].m)
            cuda_ok(cudaMemcpy(y, args.out_y + row_off[i], sizeof(double) * L[i].m, cudaMemcpyDeviceToHost), "y");
    }

    // y = A x (which 0) or A^T x (which 1) of LP i through the packed pools
    // and the solver's SpMV (FP64 accumulation); x, y in the caller's order.
    void spmv(int i, int which, const double* x, double* y) {
        if (i < 0 || i >= n) fail(B2_ERR_INVALID, "LP index out of range");
        const Layout& l = L[i];
        const dev::InstDesc& d = desc[i];
        dev::SellDev S{};
        S.n_rows = which == 0 ? d.m : d.n;
        S.n_slices = which == 0 ? d.a_nslices : d.at_nslices;
        S.slice = args.slice + (which == 0 ? d.a_slice : d.at_slice);
        S.col = args.col + (which == 0 ? d.a_cv : d.at_cv);
        S.v32 = args.v32 + (which == 0 ? d.a_cv : d.at_cv);
        S.v64 = args.v64 ? args.v64 + (which == 0 ? d.a_cv : d.at_cv) : nullptr;
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
            if (l.exact32) dev::k_spmv<double, float, double><<<std::max(1, S.n_slices / 8 + 1), 256, 0, stream>>>(S, dx, dy);
            else dev::k_spmv<double, double, double><<<std::max(1, S.n_slices / 8 + 1), 256, 0, stream>>>(S, dx, dy);
        }
        cuda_ok(cudaGetLastError(), "k_spmv");
        cuda_ok(cudaStreamSynchronize(stream), "k_spmv");
        cuda_ok(cudaMemcpy(yd.data(), dy, yd.size() * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
        cudaFree(dx);
        cudaFree(dy);
        for (int r = 0; r < rows; ++r) y[out_perm[r]] = yd[r];
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
    }
};

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

}  // namespace b2
