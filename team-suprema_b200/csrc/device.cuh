// device.cuh -- device side of the B200 PDLP engine: the restarted PDHG loop
// of include/pdlp_algo.hpp:49-185 as one device function, solve_body<GK, T, V>,
// run by a "group" of CTAs that cooperate on one LP:
//   * the whole grid of a cooperative launch for one large LP (engine.cu), its
//     barriers a bounded software grid barrier;
//   * a thread-block cluster per large LP in the batched kernel (batch.cu), its
//     barriers the hardware cluster barrier;
//   * a single CTA per small LP in the batched kernel, its barriers
//     __syncthreads.
//
// Design (what replaces the reference's gpu/pdlp_gpu_solve.cu):
//   * The reference launches 6+ kernels per attempt and makes one blocking
//     D2H copy per attempt for the step-size test (pdlp_gpu_solve.cu:232-243),
//     plus 4 full-vector D2H copies and 2 host verify() calls every 64
//     accepted steps (pdlp_algo.hpp:135-141). Here nothing leaves the device
//     until the solve ends: every CTA keeps a replica of the scalar control
//     state and takes identical decisions from identical, fixed-order sums.
//   * Two fused passes per attempt, separated by a group barrier:
//       rows: A x' (sliced ELL) + dual step + projection + |dy|^2, dy'(Ax'-Ax)
//             + the deferred ergodic-average update of y;
//       cols: [if accepted] A^T y' + the average update of x, then the primal
//             step + bound projection for the NEXT attempt + |dx|^2.
//   * The KKT check (verify.cpp:24-103 on the unscaled form) runs on the
//     device: A x and A^T y of the current point are carried with the
//     iterates, the average point takes one extra SpMV each way.
//   * Iterates live in unscaled coordinates (x_u = Dc x_s, y_u = Dr y_s), so
//     the matrix is stored with its ORIGINAL values (exact in FP32 for the
//     benchmark LPs) and Ruiz / Pock-Chambolle scaling becomes the diagonal
//     step weights tau Dc^2 and sigma Dr^2; the iteration is the reference's,
//     in a change of variables.
//   * Mixed precision: FP32 iterates and FP32-accumulated SpMV until the KKT
//     error reaches switch_tol, then FP64 iterates (same control state) until
//     `tol`. Reductions, step sizes, primal weight and KKT norms are FP64.
//   * Every device-side wait (the grid barrier) is bounded by a wall-clock
//     timeout; on expiry the kernel sets an abort flag, all CTAs leave, and the
//     host reports B2_ERR_TIMEOUT with the context intact.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"

namespace b2 {
namespace dev {

constexpr int kBlock = 512;          // CTA size of the one-LP kernels (and the largest CTA size)
constexpr int kWarps = kBlock / 32;
constexpr int kPartStride = 32;  // doubles per CTA (or per warp, one-CTA groups) per reduction slot
constexpr int kMaxNV = 22;
enum { SLOT_A = 0, SLOT_X = 1, SLOT_CK = 2, NSLOTS = 3 };
constexpr int kCtaPartDoubles = NSLOTS * kWarps * kPartStride;  // a one-CTA group's shared partials
enum { SEL_BEST = 0, SEL_CUR = 1, SEL_AVG = 2 };
// MODE_START: cold start. MODE_RESUME: the FP64 phase takes over from the
// FP32 phase (iterates widened, A x / A^T y recomputed). MODE_CONTINUE: the
// same phase goes on after a yield, from exactly the state it left.
enum { MODE_START = 0, MODE_RESUME = 1, MODE_CONTINUE = 2 };
// Group kinds: one CTA (barrier __syncthreads, partial sums in shared memory,
// iterates read through L1), a thread-block cluster (hardware cluster
// barrier), the whole grid of a cooperative launch (software grid barrier).
// Across SMs, iterates and partial sums go through L2 (ld.global.cg); the
// grid barrier fences once per CTA (thread 0, around its release/acquire), the
// cluster barrier in every thread, the one-CTA barrier not at all.
enum { GK_CTA = 0, GK_CLUSTER = 1, GK_GRID = 2 };
// one record per KKT check: attempts, accepted, eps_P/D/G of the current point,
// eps_P/D/G of the average, omega, eta, flags (restart | avg<<1 | fp32<<2 |
// best<<3), weight of the average
constexpr int kTraceFields = 12;
constexpr double kInfD = __builtin_huge_val();

struct SellDev {
    int n_rows;
    int n_slices;
    const int4* slice;
    const uint32_t* col;
    const float* v32;
    const double* v64;
    // split slices (long rows, whole-GPU engine only): per split group
    // {segments, first partial slot}, the partial sums (32 per segment) and
    // one arrival counter per group, zero between products
    const int2* seg;
    double* seg_part;
    unsigned* seg_cnt;
    // dense runs (whole-GPU engine only): per slice record {c0, ks} when lane
    // l of step k holds column c0 + k * ks + l, else {-1, 0}; null: none
    const int2* aff;
};

template <class T>
struct Bufs {
    T* x[2];
    T* y[2];
    T* ax[3];
    T* aty[2];
    T* x_last;
    T* y_last;
};

// Scalar state of pdlp_run (include/pdlp_algo.hpp:67-102), replicated per CTA.
struct Ctl {
    double eta, omega, wsum, pend_x, pend_y;
    double merit_last_restart, merit_prev_cand, best_merit;
    double best_eps[3], out_eps[3];
    double t_start;
    int attempts, accepted, since_restart, restarts, checks;
    int xi, yi, ax_cur, ax_nxt, ax_avg, aty_cur, aty_avg;
    int last_accepted, best_valid, stall, exit_reason, out_sel;
    int mode, check_now, switch_req, stop_req;
    int fp32_attempts, fp32_accepted;
    // yield / continue (rounds of a served batch): the phase the LP is in
    // (1: FP64 iterates), a pending yield, and the group total of |dx|^2 of
    // the primal step already taken for the next attempt
    int phase64, yield_req;
    double dx2_carry;
};

// Pointers and constants of one LP (independent of the iterate precision).
struct KParamsBase {
    int m, n;
    SellDev A, AT;
    const double *b, *rU, *c, *l, *u, *x0;
    const double *dr2, *dc2;  // Dr^2 (negated on >= rows), Dc^2
    // every column has the same bounds (l_all, u_all): l and u are not read
    int lu_const;
    double l_all, u_all;
    Bufs<float> itf;          // FP32 iterates (read when resuming in FP64)
    double *xsum, *ysum, *best_x, *best_y, *out_x, *out_y;
    const int32_t *perm_r, *perm_c;
    Ctl* ctl;
    const volatile int* host_stop;
    double tol, switch_tol, denom_p, denom_d, time_limit_ns;
    int max_iterations, check_every, stall_checks, return_current, mixed;
    unsigned long long debug_delay_ns;  // test hook: the group's first CTA arrives late at its first barrier
    double* trace;                      // per-check records (kTraceFields doubles), may be null
    int trace_cap;
    // > 0: the solve yields at its first attempt boundary from this attempt on
    // (a batch's tail lane; the point depends on the LP alone, not on timing)
    int yield_attempts;
    // whole-grid kernel: the slice records of A (a_) and A^T (t_), with their
    // dense-run pairs, again in the order of a work-balanced schedule over the
    // grid's warps; warp w runs records [start[w], start[w + 1]). Null:
    // round-robin over the matrices' own record order.
    const int4 *a_wslice, *t_wslice;
    const int2 *a_waff, *t_waff;
    const int *a_wstart, *t_wstart;
};

template <class T>
struct KParams : KParamsBase {
    Bufs<T> it;  // iterates at this precision
};

// Every device pointer and constant of one LP, for kernels that take LPs from
// a work queue (batches, served rounds): the LP may live in its own device
// region or at offsets inside shared pools.
struct LpDev {
    int m, n;
    SellDev A, AT;
    const double *b, *rU, *dr2, *c, *l, *u, *dc2, *x0;
    const int32_t *perm_r, *perm_c;
    Bufs<float> itf;
    Bufs<double> itd;
    double *xsum, *ysum, *best_x, *best_y, *out_x, *out_y;
    Ctl* ctl;
    double denom_p, denom_d;
    int exact32, lu_const;
    double l_all, u_all;  // the bounds of every column when lu_const
};

// The CTAs that cooperate on one LP, and this CTA's place in them.
struct Group {
    int rank, size;          // this CTA's index, number of CTAs
    int gw, nw, gt, nt;      // warp / thread index and count over the group
    double* part;            // partial sums: [NSLOTS][size][kPartStride]
    double* bcast;           // [0] stop, [1] time limit hit, [2] start time
    unsigned* bar;           // grid-barrier word (GK_GRID)
    int* abort;
    unsigned long long timeout_ns;
    double* spart;           // GK_CTA: warp partial sums in shared memory, [NSLOTS][kWarps][kPartStride]
    // global-timer deadline after which the solve yields at the next attempt
    // boundary (read on the group's first CTA only); 0: never
    unsigned long long yield_at = 0;
    // GK_CTA: shared memory for the two gathered iterates (x' for A x', y'
    // for A^T y'), used when both fit; null: gathers read global memory
    unsigned char* svec = nullptr;
    int svec_bytes = 0;
};

// ------------------------------------------------------------- primitives
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Matrix streams: read-only for the kernel's lifetime. A whole-GPU pass
// reads each entry once (no L1 allocation); a CTA that solves a small LP
// alone reads its matrix every attempt, so there it may stay in L1.
template <bool KEEP>
__device__ __forceinline__ uint32_t ld_mat(const uint32_t* p) {
    uint32_t v;
    if (KEEP) asm("ld.global.nc.u32 %0, [%1];" : "=r"(v) : "l"(p));
    else asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
template <bool KEEP>
__device__ __forceinline__ float ld_mat(const float* p) {
    float v;
    if (KEEP) asm("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
    else asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
template <bool KEEP>
__device__ __forceinline__ double ld_mat(const double* p) {
    double v;
    if (KEEP) asm("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    else asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
// Iterates are rewritten between passes, never read through the non-coherent
// path: inside one CTA a plain load (L1 holds the CTA's own stores), across
// SMs a load at L2.
template <int GK, class T>
__device__ __forceinline__ T ld_it(const T* p) {
    if (GK == GK_CTA) return *p;
    return __ldcg(p);
}

// One-dimensional bulk copy (TMA engine) from this GPU's global memory into
// this CTA's shared memory, completed on an mbarrier: the issuing thread
// announces the bytes (arrive.expect_tx) and the copy counts them off. Both
// addresses 16-byte aligned, bytes a multiple of 16; the copy lands in this
// CTA's shared memory only.
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bulk_to_smem(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
    // the source was written through the generic proxy (other SMs, ordered by
    // the grid barrier) and the destination last read through it: order both
    // before the async-proxy copy
    asm volatile("fence.proxy.async;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"((unsigned long long)__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_done(unsigned long long* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits (bounded) for the copy of phase `parity`; past the limit it raises
// `abort` and gives the copy, which still targets this CTA's shared memory, a
// second bounded wait before the caller goes on to the barrier that ends it.
__device__ __forceinline__ void mbar_wait(unsigned long long* bar, uint32_t parity, int* abort,
                                          unsigned long long timeout_ns) {
    if (mbar_done(bar, parity)) return;
    const unsigned long long t0 = gtimer();
    unsigned spins = 0;
    while (!mbar_done(bar, parity)) {
        if ((++spins & 63u) == 0 && gtimer() - t0 > timeout_ns) {
            atomicExch(abort, 1);
            const unsigned long long t1 = gtimer();
            while (!mbar_done(bar, parity) && gtimer() - t1 < timeout_ns) {
            }
            return;
        }
    }
}

template <class V>
__device__ __forceinline__ const V* vals(const SellDev& S);
template <>
__device__ __forceinline__ const float* vals<float>(const SellDev& S) { return S.v32; }
template <>
__device__ __forceinline__ const double* vals<double>(const SellDev& S) { return S.v64; }

// Sum over a warp, fixed tree; the result is taken from lane 0 and
// broadcast, so every lane (and every CTA) sees the same bits.
__device__ __forceinline__ double warp_total(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return __shfl_sync(0xffffffffu, v, 0);
}

// Group barrier. One CTA: __syncthreads. A cluster: fence + hardware cluster
// barrier. The grid of a cooperative launch: fence + one counter word; CTA 0
// adds 2^31 - (N-1), the others add 1, so the top bit flips exactly when the
// last CTA arrives. Arrival is a release, polling an acquire (gpu scope). The
// grid wait is bounded: past timeout_ns the CTA raises `abort` and every CTA
// leaves.
template <int GK>
__device__ __forceinline__ bool group_sync(const Group& g) {
    if (GK == GK_CTA) {
        // one CTA: bar.sync orders every thread's global and shared stores
        // before the other threads' loads after it (CTA scope), and the
        // iterates are read with plain (L1-coherent within the SM) loads
        __syncthreads();
        return true;
    }
    if (GK == GK_CLUSTER) {
        // the hardware cluster barrier has no timeout, so every thread also
        // fences its own stores at gpu scope first: a CTA of the cluster must
        // never decide from a value it cannot yet see
        __threadfence();
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
        return true;
    }
    __shared__ int s_ok;
    // bar.sync makes the CTA's stores observed by thread 0; its gpu-scope
    // fence and release then publish them cumulatively to the other CTAs,
    // which read them at L2 (ld.global.cg) after their acquire and bar.sync
    __syncthreads();
    if (g.size == 1) return true;
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned add = g.rank == 0 ? (0x80000000u - (unsigned)(g.size - 1)) : 1u;
        unsigned old;
        __threadfence();
        asm volatile("atom.add.release.gpu.u32 %0,[%1],%2;" : "=r"(old) : "l"(g.bar), "r"(add) : "memory");
        const unsigned long long t0 = gtimer();
        unsigned spins = 0;
        for (;;) {
            unsigned cur;
            asm volatile("ld.acquire.gpu.u32 %0,[%1];" : "=r"(cur) : "l"(g.bar) : "memory");
            if ((old ^ cur) & 0x80000000u) break;
            if ((++spins & 15u) == 0) {
                if (*(volatile int*)g.abort) { ok = 0; break; }
                if (gtimer() - t0 > g.timeout_ns) { atomicExch(g.abort, 1); ok = 0; break; }
            }
        }
        if (ok && *(volatile int*)g.abort) ok = 0;
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Per-CTA partial sums of NV values: k = 0..NV-1 go to index at + k of this
// CTA's row of the slot. Fixed order: warp tree, then warps in order.
//
// One CTA alone (GK_CTA) keeps the warp partials themselves, [slot][warp][k]
// in shared memory, and whoever reads the totals after the next barrier adds
// the warps in order (cta_sum): the same sums, two fewer barriers an attempt.
__device__ __forceinline__ double cta_sum(const Group& g, int slot, int k) {
    double s = 0.0;
    const int nwarps = blockDim.x >> 5;
    for (int w = 0; w < nwarps; ++w) s += g.spart[(slot * kWarps + w) * kPartStride + k];
    return s;
}

template <int NV, int GK>
__device__ __forceinline__ void cta_partial_at(double (&v)[NV], const Group& g, int slot, int at, double* s_red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (GK == GK_CTA) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = v[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) g.spart[(slot * kWarps + warp) * kPartStride + at + k] = t;
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) s_red[warp * NV + k] = t;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        const int nwarps = blockDim.x >> 5;
        for (int w = 0; w < nwarps; ++w) s += s_red[w * NV + threadIdx.x];
        g.part[((size_t)slot * g.size + g.rank) * kPartStride + at + threadIdx.x] = s;
    }
}

template <int NV, int GK>
__device__ __forceinline__ void cta_partial(double (&v)[NV], const Group& g, int slot, double* s_red) {
    cta_partial_at<NV, GK>(v, g, slot, 0, s_red);
}

// After a barrier: every CTA sums the CTA partials of one slot in CTA order.
// One lane's share of a sum over the group's CTAs: p[b * stride] for b = lane,
// lane + 32, ... < size, added in that order. The loads of up to 320 CTAs are
// issued before the first add, so the sum costs one L2 round trip, not one
// per CTA.
__device__ __forceinline__ double lane_parts(const double* p, int size, size_t stride, int lane) {
    constexpr int kIn = 10;
    double s = 0.0;
    for (int b0 = lane; b0 < size; b0 += 32 * kIn) {
        double v[kIn];
#pragma unroll
        for (int q = 0; q < kIn; ++q) v[q] = b0 + 32 * q < size ? __ldcg(p + (size_t)(b0 + 32 * q) * stride) : 0.0;
#pragma unroll
        for (int q = 0; q < kIn; ++q)
            if (b0 + 32 * q < size) s += v[q];
    }
    return s;
}

template <int NV, int GK>
__device__ __forceinline__ void group_totals(const Group& g, int slot, double* s_tot) {
    if (GK == GK_CTA) {
        if (threadIdx.x < NV) s_tot[threadIdx.x] = cta_sum(g, slot, threadIdx.x);
        __syncthreads();
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = warp; k < NV; k += (int)(blockDim.x >> 5)) {
        double s = lane_parts(g.part + (size_t)slot * g.size * kPartStride + k, g.size, kPartStride, lane);
        s = warp_total(s);
        if (lane == 0) s_tot[k] = s;
    }
    __syncthreads();
}

// Totals of the step-size statistics after a barrier: dy2 and dy'(Ax'-Ax)
// from the rows pass, |dx|^2 from the columns pass before it.
template <int GK>
__device__ __forceinline__ void step_totals(const Group& g, double* s_tot) {
    if (GK == GK_CTA) {
        // only thread 0 (the step decision) reads them: no barrier
        if (threadIdx.x == 0) {
            s_tot[0] = cta_sum(g, SLOT_A, 0);
            s_tot[1] = cta_sum(g, SLOT_A, 1);
            s_tot[2] = cta_sum(g, SLOT_X, 0);
        }
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp < 3) {
        const int slot = warp < 2 ? SLOT_A : SLOT_X, k = warp < 2 ? warp : 0;
        double s = lane_parts(g.part + (size_t)slot * g.size * kPartStride + k, g.size, kPartStride, lane);
        s = warp_total(s);
        if (lane == 0) s_tot[warp] = s;
    }
    __syncthreads();
}

// One slice of a sliced-ELL matrix times a gathered vector: every lane sums
// its share of its row in a fixed order, then the g lanes of a row are
// folded onto the row's first lane (fixed tree).
#ifndef B2_SLICE_UNROLL
#define B2_SLICE_UNROLL 4
#endif
constexpr int kUnroll = B2_SLICE_UNROLL;

// LOCAL: x is a copy in this CTA's shared memory (plain loads).
template <int GK, class AccT, class V, class XT, bool LOCAL = false>
__device__ __forceinline__ AccT slice_dot(const SellDev& S, const V* vbase, int4 sl, int lane, const XT* x) {
    constexpr bool KEEP = GK == GK_CTA;
    constexpr int GX = LOCAL ? GK_CTA : GK;
    const uint32_t len = (uint32_t)sl.y & kLenMask;
    const int lg = (int)((uint32_t)sl.y >> kLenBits);
    const size_t base = (size_t)(uint32_t)sl.z * 32u + (size_t)lane;
    const uint32_t* cp = S.col + base;
    const V* vp = vbase + base;
    AccT acc = AccT(0);
    uint32_t k = 0;
    // kUnroll gathers in flight per lane; the sum stays one sequential fma
    // chain, so the unroll depth never changes the result
    for (; k + kUnroll <= len; k += kUnroll) {
        uint32_t cc[kUnroll];
        V vv[kUnroll];
        AccT xx[kUnroll];
#pragma unroll
        for (int q = 0; q < kUnroll; ++q) {
            cc[q] = ld_mat<KEEP>(cp + 32 * q);
            vv[q] = ld_mat<KEEP>(vp + 32 * q);
        }
#pragma unroll
        for (int q = 0; q < kUnroll; ++q) xx[q] = (AccT)ld_it<GX>(x + cc[q]);
#pragma unroll
        for (int q = 0; q < kUnroll; ++q) acc = fma((AccT)vv[q], xx[q], acc);
        cp += 32 * kUnroll;
        vp += 32 * kUnroll;
    }
    for (; k < len; ++k) {
        acc = fma((AccT)ld_mat<KEEP>(vp), (AccT)ld_it<GX>(x + ld_mat<KEEP>(cp)), acc);
        cp += 32;
        vp += 32;
    }
    for (int o = (1 << lg) >> 1; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    return acc;
}

// The same product for a dense-run record (columns c0 + k * ks + lane): the
// gather addresses are computed, not read, so every step's value and x loads
// are independent and kDenseUnroll steps are in flight at once. The stored
// column stream holds the same indices; padding positions gather a column in
// range with a zero value, as the stream's padding does, so the sums are
// those of slice_dot.
constexpr int kDenseUnroll = 8;
template <int GK, class AccT, class V, class XT, bool LOCAL = false>
__device__ __forceinline__ AccT slice_dot_dense(const V* vbase, int4 sl, int2 af, int lane, const XT* x) {
    constexpr bool KEEP = GK == GK_CTA;
    constexpr int GX = LOCAL ? GK_CTA : GK;
    const uint32_t len = (uint32_t)sl.y & kLenMask;
    const int lg = (int)((uint32_t)sl.y >> kLenBits);
    const V* vp = vbase + (size_t)(uint32_t)sl.z * 32u + (size_t)lane;
    const XT* xp = x + (int64_t)af.x + lane;
    const int64_t ks = af.y;
    AccT acc = AccT(0);
    uint32_t k = 0;
    for (; k + kDenseUnroll <= len; k += kDenseUnroll) {
        V vv[kDenseUnroll];
        AccT xx[kDenseUnroll];
#pragma unroll
        for (int q = 0; q < kDenseUnroll; ++q) {
            vv[q] = ld_mat<KEEP>(vp + 32 * q);
            xx[q] = (AccT)ld_it<GX>(xp + (int64_t)q * ks);
        }
#pragma unroll
        for (int q = 0; q < kDenseUnroll; ++q) acc = fma((AccT)vv[q], xx[q], acc);
        vp += 32 * kDenseUnroll;
        xp += (int64_t)kDenseUnroll * ks;
    }
    for (; k < len; ++k) {
        acc = fma((AccT)ld_mat<KEEP>(vp), (AccT)ld_it<GX>(xp), acc);
        vp += 32;
        xp += ks;
    }
    for (int o = (1 << lg) >> 1; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    return acc;
}

// Split groups add their segments' partial sums in two levels: subgroups of
// kSubSeg consecutive segments are added in segment order, then the subgroup
// totals in subgroup order. The order is fixed by the layout, so every run
// gives the same bits, and the owner of the rows waits for a few subgroup
// totals instead of adding up to 255 partials in one chain.
constexpr int kSubSeg = 16;
// arrival counters per split group: [0] subgroup leaders, [1 + k] members of subgroup k
constexpr int kSegCounters = 1 + (255 + kSubSeg - 1) / kSubSeg;

template <class AccT>
__device__ __forceinline__ AccT sum_sub(const double* part, int first, int count, int lane) {
    // loads issued 8 at a time; the adds stay one chain in segment order
    AccT s = AccT(0);
    for (int h = 0; h < count; h += 8) {
        double v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = h + k < count ? __ldcg(part + (first + h + k) * 32 + lane) : 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (h + k < count) s += (AccT)v[k];
    }
    return s;
}

// The two-level sum of all `segments` partials of a lane (the order seg_finish
// uses), for the standalone product: a whole subgroup's loads in flight at once.
template <class AccT>
__device__ __forceinline__ AccT sum_partials(const double* part, int segments, int lane) {
    AccT tot = AccT(0);
    for (int f = 0; f < segments; f += kSubSeg) {
        const int count = min(kSubSeg, segments - f);
        double v[kSubSeg];
#pragma unroll
        for (int k = 0; k < kSubSeg; ++k) v[k] = k < count ? __ldcg(part + (f + k) * 32 + lane) : 0.0;
        AccT sub = AccT(0);
#pragma unroll
        for (int k = 0; k < kSubSeg; ++k)
            if (k < count) sub += (AccT)v[k];
        tot = f == 0 ? sub : tot + (AccT)(double)sub;
    }
    return tot;
}

// Lane 0 waits (bounded) until *cnt reaches want, then zeroes it for the next
// product; the warp learns whether the wait succeeded.
__device__ __forceinline__ bool seg_wait(unsigned* cnt, unsigned want, const Group& g, int lane) {
    int ok = 1;
    if (lane == 0 && want > 0) {
        const unsigned long long t0 = gtimer();
        unsigned spins = 0;
        for (;;) {
            unsigned cur;
            asm volatile("ld.acquire.gpu.u32 %0,[%1];" : "=r"(cur) : "l"(cnt) : "memory");
            if (cur == want) break;
            if ((++spins & 63u) == 0) {
                if (*(volatile int*)g.abort || gtimer() - t0 > g.timeout_ns) { atomicExch(g.abort, 1); ok = 0; break; }
            }
        }
        if (ok) *cnt = 0u;  // all have arrived: ready for the next product
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok != 0;
}

// A split slice is one of `segments` consecutive slice records over the same
// rows, each covering a range of steps (slice.w = group + 1 | segment << 24;
// 0 for an unsplit slice); only the whole-GPU layout has them. Every segment
// publishes its lanes' partial sums; a member counts itself in with its
// subgroup's leader (the subgroup's first segment), which waits (bounded) for
// the subgroup, adds its partials in order and leaves the subtotal in its own
// slot; the warp of segment 0 (leader of subgroup 0) owns the rows: it waits
// for the other leaders, adds the subtotals in order and alone runs the rows'
// epilogue, so the sums, and which CTA's reductions the rows land in, never
// depend on timing. Waits cannot form a cycle: a warp waits only on later
// slice records of its own group, and the launch keeps segments <= the
// group's warp count, so none of them is a later slice of the waiting warp.
// Returns whether this warp holds complete row sums in `acc`.
template <int GK, class AccT>
__device__ __forceinline__ bool seg_finish(const SellDev& S, int4 sl, int lane, AccT& acc, const Group& g) {
    if (GK != GK_GRID || sl.w == 0) return true;
    const int grp = (sl.w & 0xFFFFFF) - 1, q = (int)((unsigned)sl.w >> 24);
    const int2 info = __ldg(S.seg + grp);
    double* part = S.seg_part + (size_t)info.y * 32;
    unsigned* cnt = S.seg_cnt + (size_t)grp * kSegCounters;
    const int sub = q / kSubSeg, lead = sub * kSubSeg;
    const int members = min(kSubSeg, info.x - lead);
    __stcg(part + q * 32 + lane, (double)acc);
    __threadfence();
    __syncwarp();
    if (q != lead) {
        if (lane == 0) atomicAdd(cnt + 1 + sub, 1u);
        return false;
    }
    if (!seg_wait(cnt + 1 + sub, (unsigned)(members - 1), g, lane)) return false;  // abort: the next barrier reports it
    __threadfence();
    const AccT subtotal = sum_sub<AccT>(part, lead, members, lane);
    if (q != 0) {
        __stcg(part + q * 32 + lane, (double)subtotal);
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicAdd(cnt, 1u);
        return false;
    }
    const int nsub = (info.x + kSubSeg - 1) / kSubSeg;
    if (!seg_wait(cnt, (unsigned)(nsub - 1), g, lane)) return false;
    __threadfence();
    AccT tot = subtotal;
    for (int k = 1; k < nsub; ++k) tot += (AccT)__ldcg(part + k * kSubSeg * 32 + lane);
    acc = tot;
    return true;
}

// The same for a product with no reductions behind it (the standalone SpMV):
// whichever warp completes the group adds the partials in the same two-level
// order, so nobody waits and the sums are the same bits.
template <class AccT>
__device__ __forceinline__ bool seg_finish_last(const SellDev& S, int4 sl, int lane, AccT& acc) {
    if (sl.w == 0) return true;
    const int grp = (sl.w & 0xFFFFFF) - 1, q = (int)((unsigned)sl.w >> 24);
    const int2 info = __ldg(S.seg + grp);
    double* part = S.seg_part + (size_t)info.y * 32;
    unsigned* cnt = S.seg_cnt + (size_t)grp * kSegCounters;
    __stcg(part + q * 32 + lane, (double)acc);
    __threadfence();
    __syncwarp();
    unsigned last = 0;
    if (lane == 0) last = atomicAdd(cnt, 1u) == (unsigned)(info.x - 1) ? 1u : 0u;
    last = __shfl_sync(0xffffffffu, last, 0);
    __syncwarp();
    if (!last) return false;
    __threadfence();
    acc = sum_partials<AccT>(part, info.x, lane);
    if (lane == 0) *cnt = 0u;  // the next product comes after this kernel
    return true;
}

// A pass that needs no product over a split slice still runs the rows'
// epilogue once: in the warp of segment 0.
template <int GK>
__device__ __forceinline__ bool seg_first(int4 sl) {
    return GK != GK_GRID || sl.w == 0 || ((unsigned)sl.w >> 24) == 0u;
}

// verify.cpp:35-87 terms of one row: row violation^2, sign violation^2,
// dual-objective share, -inf flag.
__device__ __forceinline__ void kkt_row(double rl, double ru, double a, double y, double* v) {
    const double rv = fmax(rl - a, 0.0) + fmax(a - ru, 0.0);
    double sv = 0.0;
    if (!isfinite(rl) && y > 0) sv += y;
    if (!isfinite(ru) && y < 0) sv += -y;
    double yd = y;
    if (!isfinite(rl) && yd > 0) yd = 0.0;
    if (!isfinite(ru) && yd < 0) yd = 0.0;
    const double yp = fmax(yd, 0.0), yn = fmax(-yd, 0.0);
    double d = 0.0, ninf = 0.0;
    if (yp > 0 && isfinite(rl)) d += rl * yp;
    if (yn > 0 && isfinite(ru)) d += -ru * yn;
    if ((yp > 0 && !isfinite(rl)) || (yn > 0 && !isfinite(ru))) ninf = 1.0;
    v[0] += rv * rv;
    v[1] += sv * sv;
    v[2] += d;
    v[3] += ninf;
}

// The same for one column with reduced cost z = c - A^T y, plus c x.
__device__ __forceinline__ void kkt_col(double l, double u, double cc, double x, double z, double* v) {
    const double bv = fmax(l - x, 0.0) + fmax(x - u, 0.0);
    double sv = 0.0;
    if (!isfinite(l) && z > 0) sv += z;
    if (!isfinite(u) && z < 0) sv += -z;
    double zd = z;
    if (!isfinite(l) && zd > 0) zd = 0.0;
    if (!isfinite(u) && zd < 0) zd = 0.0;
    const double zp = fmax(zd, 0.0), zn = fmax(-zd, 0.0);
    double d = 0.0, ninf = 0.0;
    if (zp > 0 && isfinite(l)) d += l * zp;
    if (zn > 0 && isfinite(u)) d += -u * zn;
    if ((zp > 0 && !isfinite(l)) || (zn > 0 && !isfinite(u))) ninf = 1.0;
    v[0] += bv * bv;
    v[1] += sv * sv;
    v[2] += d;
    v[3] += ninf;
    v[4] += cc * x;
}

// Primal step of one column (pdlp_algo.hpp:110 / src/pdlp.cpp:122-124) in
// unscaled coordinates: x' = clamp(x - tau Dc^2 (c - A^T y), l, u).
template <class T>
__device__ __forceinline__ void primal_col_w(int j, T xv, double g, double tau, T* xn, double& dx2, T* xs,
                                             double w, double cj, double lj, double uj) {
    double v = (double)xv - tau * w * (cj - g);
    v = fmin(fmax(v, lj), uj);
    const T vt = (T)v;
    xn[j] = vt;
    if (xs) xs[j] = vt;  // the copy the next A x' gathers from
    const double d = (double)vt - (double)xv;
    dx2 += d * d / w;
}

// Bounds of column j: two loads, or none when every column has the same.
__device__ __forceinline__ void col_bounds(const KParamsBase& P, int j, double& lj, double& uj) {
    if (P.lu_const) {
        lj = P.l_all;
        uj = P.u_all;
    } else {
        lj = __ldg(P.l + j);
        uj = __ldg(P.u + j);
    }
}

template <class T>
__device__ __forceinline__ void primal_col(const KParams<T>& P, int j, T xv, double g, double tau, T* xn,
                                           double& dx2, T* xs) {
    double lj, uj;
    col_bounds(P, j, lj, uj);
    primal_col_w<T>(j, xv, g, tau, xn, dx2, xs, __ldg(P.dc2 + j), __ldg(P.c + j), lj, uj);
}

// --------------------------------------------------------------- passes

// Rows: A x' fused with the dual step (pdlp_algo.hpp:111-112, src/pdlp.cpp:125-130)
// and the step-size statistics (pdlp_gpu_solve.cu:119-131).
template <int GK, class T, class V>
__device__ void pass_rows_step(const KParams<T>& P, const Ctl& c, const Group& g, int lane, double* v, T* sx,
                               T* sy) {
    const T* xn = sx ? sx : P.it.x[1 - c.xi];
    const T* y = P.it.y[c.yi];
    T* yn = P.it.y[1 - c.yi];
    const T* ax = P.it.ax[c.ax_cur];
    T* axn = P.it.ax[c.ax_nxt];
    const double sigma = c.eta * c.omega, pend = c.pend_y;
    const V* vb = vals<V>(P.A);
    auto one = [&](const int4 sl, const int2 af) {
        const int lg = (int)((uint32_t)sl.y >> kLenBits);
        const int row = sl.x + (lane >> lg);
        const bool lead = (lane & ((1 << lg) - 1)) == 0 && row < P.m;
        // the epilogue's operands are loaded before the product, so their
        // latency hides behind its gathers
        T yv = T(0), axv = T(0);
        double w = 0.0, brow = 0.0, ys = 0.0;
        if (lead) {
            yv = ld_it<GK>(y + row);
            axv = ld_it<GK>(ax + row);
            w = __ldg(P.dr2 + row);
            brow = __ldg(P.b + row);
            if (pend != 0.0) ys = P.ysum[row];
        }
        T acc = af.x >= 0 ? slice_dot_dense<GK, T, V, T>(vb, sl, af, lane, xn) : slice_dot<GK, T, V, T>(P.A, vb, sl, lane, xn);
        if (!seg_finish<GK, T>(P.A, sl, lane, acc, g)) return;
        if (lead) {
            const double aw = fabs(w);
            double nv = (double)yv + sigma * aw * (brow - (2.0 * (double)acc - (double)axv));
            if (w < 0.0 && nv < 0.0) nv = 0.0;
            const T nt = (T)nv;
            yn[row] = nt;
            if (sy) sy[row] = nt;
            axn[row] = acc;
            const double d = (double)nt - (double)yv;
            v[0] += d * d / aw;
            v[1] += d * ((double)acc - (double)axv);
            if (pend != 0.0) P.ysum[row] = ys + pend * (double)yv;
        }
    };
    if (GK == GK_GRID && P.a_wstart) {
        // the whole grid: this warp's range of the work-balanced schedule
        const int s1 = __ldg(P.a_wstart + g.gw + 1);
        for (int s = __ldg(P.a_wstart + g.gw); s < s1; ++s)
            one(__ldg(P.a_wslice + s), P.a_waff ? __ldg(P.a_waff + s) : make_int2(-1, 0));
    } else {
        for (int s = g.gw; s < P.A.n_slices; s += g.nw)
            one(__ldg(P.A.slice + s), P.A.aff ? __ldg(P.A.aff + s) : make_int2(-1, 0));
    }
}

// Columns: [accepted] A^T y' + x-average update, then the next primal step.
template <int GK, class T, class V>
__device__ void pass_cols_step(const KParams<T>& P, const Ctl& c, const Group& g, int lane, double& dx2, T* sx,
                               const T* sy) {
    const T* x = P.it.x[c.xi];
    T* xn = P.it.x[1 - c.xi];
    T* aty = P.it.aty[c.aty_cur];
    const double tau = c.eta / c.omega, pend = c.pend_x;
    if (c.last_accepted) {
        const T* y = sy ? sy : P.it.y[c.yi];
        const V* vb = vals<V>(P.AT);
        auto one = [&](const int4 sl, const int2 af) {
            const int lg = (int)((uint32_t)sl.y >> kLenBits);
            const int j = sl.x + (lane >> lg);
            const bool lead = (lane & ((1 << lg) - 1)) == 0 && j < P.n;
            // the primal step's operands are loaded before the product
            T xv = T(0);
            double w = 1.0, cj = 0.0, lj = 0.0, uj = 0.0, xs = 0.0;
            if (lead) {
                xv = ld_it<GK>(x + j);
                w = __ldg(P.dc2 + j);
                cj = __ldg(P.c + j);
                col_bounds(P, j, lj, uj);
                if (pend != 0.0) xs = P.xsum[j];
            }
            T acc = af.x >= 0 ? (sy ? slice_dot_dense<GK, T, V, T, true>(vb, sl, af, lane, y)
                                    : slice_dot_dense<GK, T, V, T>(vb, sl, af, lane, y))
                              : (sy ? slice_dot<GK, T, V, T, true>(P.AT, vb, sl, lane, y)
                                    : slice_dot<GK, T, V, T>(P.AT, vb, sl, lane, y));
            if (!seg_finish<GK, T>(P.AT, sl, lane, acc, g)) return;
            if (lead) {
                aty[j] = acc;
                if (pend != 0.0) P.xsum[j] = xs + pend * (double)xv;
                primal_col_w<T>(j, xv, (double)acc, tau, xn, dx2, sx, w, cj, lj, uj);
            }
        };
        if (GK == GK_GRID && P.t_wstart) {
            // the whole grid: this warp's range of the work-balanced schedule
            const int s1 = __ldg(P.t_wstart + g.gw + 1);
            for (int s = __ldg(P.t_wstart + g.gw); s < s1; ++s)
                one(__ldg(P.t_wslice + s), P.t_waff ? __ldg(P.t_waff + s) : make_int2(-1, 0));
        } else {
            for (int s = g.gw; s < P.AT.n_slices; s += g.nw)
                one(__ldg(P.AT.slice + s), P.AT.aff ? __ldg(P.AT.aff + s) : make_int2(-1, 0));
        }
    } else {
        for (int j = g.gt; j < P.n; j += g.nt)
            primal_col<T>(P, j, ld_it<GK>(x + j), (double)ld_it<GK>(aty + j), tau, xn, dx2, sx);
    }
}

// KKT check, rows (verify.cpp:35-87 row terms) for the current and average
// points, the average's A x, the restart distance of y, and the pending
// y-average update.
template <int GK, class T, class V>
__device__ void pass_rows_check(const KParams<T>& P, const Ctl& c, const Group& g, int lane, double* v) {
    const T* y = P.it.y[c.yi];
    const T* ax = P.it.ax[c.ax_cur];
    T* axa = P.it.ax[c.ax_avg];
    const bool has_avg = c.wsum > 0;
    const double wsum = c.wsum, pend = c.pend_y;
    const V* vb = vals<V>(P.A);
    for (int s = g.gw; s < P.A.n_slices; s += g.nw) {
        const int4 sl = __ldg(P.A.slice + s);
        double acc = 0.0;
        if (has_avg) {
            acc = slice_dot<GK, double, V, double>(P.A, vb, sl, lane, P.xsum);
            if (!seg_finish<GK, double>(P.A, sl, lane, acc, g)) continue;
        } else if (!seg_first<GK>(sl)) {
            continue;
        }
        const int lg = (int)((uint32_t)sl.y >> kLenBits);
        const int i = sl.x + (lane >> lg);
        if ((lane & ((1 << lg) - 1)) == 0 && i < P.m) {
            const double yc = (double)ld_it<GK>(y + i);
            double ys = ld_it<GK>(P.ysum + i);
            if (pend != 0.0) { ys += pend * yc; P.ysum[i] = ys; }
            const double ac = (double)ld_it<GK>(ax + i);
            const double aa = has_avg ? acc / wsum : ac;
            const double ya = has_avg ? ys / wsum : yc;
            axa[i] = (T)aa;
            const double rl = __ldg(P.b + i), ru = __ldg(P.rU + i);
            kkt_row(rl, ru, ac, yc, v + 0);
            kkt_row(rl, ru, aa, ya, v + 4);
            const double w = fabs(__ldg(P.dr2 + i)), yl = (double)ld_it<GK>(P.it.y_last + i);
            v[8] += (yc - yl) * (yc - yl) / w;
            v[9] += (ya - yl) * (ya - yl) / w;
        }
    }
}

template <int GK, class T, class V>
__device__ void pass_cols_check(const KParams<T>& P, const Ctl& c, const Group& g, int lane, double* v) {
    const T* x = P.it.x[c.xi];
    const T* aty = P.it.aty[c.aty_cur];
    T* atya = P.it.aty[c.aty_avg];
    const bool has_avg = c.wsum > 0;
    const double wsum = c.wsum;
    const V* vb = vals<V>(P.AT);
    for (int s = g.gw; s < P.AT.n_slices; s += g.nw) {
        const int4 sl = __ldg(P.AT.slice + s);
        double acc = 0.0;
        if (has_avg) {
            acc = slice_dot<GK, double, V, double>(P.AT, vb, sl, lane, P.ysum);
            if (!seg_finish<GK, double>(P.AT, sl, lane, acc, g)) continue;
        } else if (!seg_first<GK>(sl)) {
            continue;
        }
        const int lg = (int)((uint32_t)sl.y >> kLenBits);
        const int j = sl.x + (lane >> lg);
        if ((lane & ((1 << lg) - 1)) == 0 && j < P.n) {
            const double xc = (double)ld_it<GK>(x + j), gc = (double)ld_it<GK>(aty + j);
            const double xa = has_avg ? ld_it<GK>(P.xsum + j) / wsum : xc;
            const double ga = has_avg ? acc / wsum : gc;
            atya[j] = (T)ga;
            const double cc = __ldg(P.c + j);
            double l, u;
            col_bounds(P, j, l, u);
            kkt_col(l, u, cc, xc, cc - gc, v + 0);
            kkt_col(l, u, cc, xa, cc - ga, v + 5);
            const double w = __ldg(P.dc2 + j), xl = (double)ld_it<GK>(P.it.x_last + j);
            v[10] += (xc - xl) * (xc - xl) / w;
            v[11] += (xa - xl) * (xa - xl) / w;
        }
    }
}

// After a check: copy the new best point, apply a restart (pdlp_algo.hpp:160-174)
// and, on restart, redo the next primal step with the new primal weight.
template <int GK, class T>
__device__ void pass_after_check(const KParams<T>& P, const Ctl& c, const Group& g, int best_sel, int restart,
                                 int use_avg, double wsum_old, double& dx2, T* sx) {
    const bool has_avg = wsum_old > 0;
    T* x = P.it.x[c.xi];
    T* xn = P.it.x[1 - c.xi];
    const double tau = c.eta / c.omega;
    for (int j = g.gt; j < P.n; j += g.nt) {
        const T xct = ld_it<GK>(x + j);
        const double xc = (double)xct;
        const double xa = has_avg ? ld_it<GK>(P.xsum + j) / wsum_old : xc;
        if (best_sel == SEL_CUR) P.best_x[j] = xc;
        else if (best_sel == SEL_AVG) P.best_x[j] = xa;
        if (restart) {
            const double cand = use_avg ? xa : xc;
            P.it.x_last[j] = (T)cand;
            T xnew = xct;
            if (use_avg) { xnew = (T)xa; x[j] = xnew; }
            P.xsum[j] = 0.0;
            const double gg = (double)ld_it<GK>((use_avg ? P.it.aty[c.aty_avg] : P.it.aty[c.aty_cur]) + j);
            primal_col<T>(P, j, xnew, gg, tau, xn, dx2, sx);
        }
    }
    T* y = P.it.y[c.yi];
    for (int i = g.gt; i < P.m; i += g.nt) {
        const T yct = ld_it<GK>(y + i);
        const double yc = (double)yct;
        const double ya = has_avg ? ld_it<GK>(P.ysum + i) / wsum_old : yc;
        if (best_sel == SEL_CUR) P.best_y[i] = yc;
        else if (best_sel == SEL_AVG) P.best_y[i] = ya;
        if (restart) {
            const double cand = use_avg ? ya : yc;
            P.it.y_last[i] = (T)cand;
            if (use_avg) y[i] = (T)ya;
            P.ysum[i] = 0.0;
        }
    }
}

__device__ __forceinline__ double merit3(double a, double b, double c) { return sqrt(a * a + b * b + c * c); }

// Check decision (pdlp_algo.hpp:135-174) from the 22 check totals; run by one
// thread per CTA on identical inputs. Returns, through `flags`, which point
// becomes the best point, whether to restart and whether to the average.
template <bool FP32>
__device__ void check_decision(const KParamsBase& B, Ctl& s, const double* t, bool evaluate_only, bool write_trace,
                               int* flags, double* wsum_old) {
    double eP[2], eD[2], eG[2], mer[2];
    for (int o = 0; o < 2; ++o) {
        const double* r = t + 4 * o;        // rows: rv2, sv2, D, ninf
        const double* q = t + 10 + 5 * o;   // cols: bv2, sv2, D, ninf, cx
        eP[o] = sqrt(r[0] + q[0]) / B.denom_p;
        eD[o] = sqrt(r[1] + q[1]) / B.denom_d;
        double D = r[2] + q[2];
        if (r[3] + q[3] > 0) D = -kInfD;
        const double cx = q[4];
        eG[o] = isfinite(D) ? fabs(cx - D) / (1.0 + fabs(cx) + fabs(D)) : kInfD;
        mer[o] = merit3(eP[o], eD[o], eG[o]);
    }
    s.checks++;
    int best_sel = 0, restart = 0, use_avg = 0;
    *wsum_old = s.wsum;
    if (evaluate_only) {
        // stopped before any check: report the current point (pdlp_algo.hpp:178-182)
        s.out_sel = SEL_CUR;
        s.out_eps[0] = eP[0]; s.out_eps[1] = eD[0]; s.out_eps[2] = eG[0];
        flags[0] = flags[1] = flags[2] = 0;
        return;
    }
    if (mer[0] < s.best_merit) {
        s.best_merit = mer[0]; best_sel = SEL_CUR;
        s.best_eps[0] = eP[0]; s.best_eps[1] = eD[0]; s.best_eps[2] = eG[0];
    }
    if (mer[1] < s.best_merit) {
        s.best_merit = mer[1]; best_sel = SEL_AVG;
        s.best_eps[0] = eP[1]; s.best_eps[1] = eD[1]; s.best_eps[2] = eG[1];
    }
    if (best_sel) { s.best_valid = 1; s.stall = 0; } else { s.stall++; }
    use_avg = mer[1] < mer[0];
    const int o = use_avg ? 1 : 0;
    const double mc = mer[o];
    const double worst = fmax(eP[o], fmax(eD[o], eG[o]));
    if (worst <= B.tol) {
        if (FP32) {
            s.switch_req = 1;  // confirm with FP64 iterates before terminating
            s.check_now = 1;
        } else {
            s.exit_reason = B2_EXIT_CONVERGED;
            s.out_sel = use_avg ? SEL_AVG : SEL_CUR;
            s.out_eps[0] = eP[o]; s.out_eps[1] = eD[o]; s.out_eps[2] = eG[o];
        }
    } else {
        const bool sufficient = mc <= 0.2 * s.merit_last_restart;
        const bool necessary = mc <= 0.8 * s.merit_last_restart && mc > s.merit_prev_cand;
        const bool artificial = s.since_restart >= 0.36 * s.accepted;
        s.merit_prev_cand = mc;
        if (sufficient || necessary || artificial) {
            restart = 1;
            const double ddx = sqrt(t[20 + o]), ddy = sqrt(t[8 + o]);
            if (ddx > 1e-10 && ddy > 1e-10) s.omega = exp(0.5 * log(ddy / ddx) + 0.5 * log(s.omega));
            s.since_restart = 0;
            s.restarts++;
            s.merit_last_restart = mc;
            s.merit_prev_cand = kInfD;
            s.wsum = 0.0;
        }
        if (FP32 && B.mixed && (worst <= B.switch_tol || s.stall >= B.stall_checks)) s.switch_req = 1;
        if (s.attempts >= B.max_iterations) s.exit_reason = B2_EXIT_MAX_ITER;
        else if (s.stop_req) s.exit_reason = s.stop_req;
    }
    flags[0] = best_sel;
    flags[1] = restart;
    flags[2] = use_avg;
    if (write_trace && B.trace && s.checks - 1 < B.trace_cap) {
        double* t_out = B.trace + (size_t)(s.checks - 1) * kTraceFields;
        t_out[0] = s.attempts; t_out[1] = s.accepted;
        t_out[2] = eP[0]; t_out[3] = eD[0]; t_out[4] = eG[0];
        t_out[5] = eP[1]; t_out[6] = eD[1]; t_out[7] = eG[1];
        t_out[8] = s.omega; t_out[9] = s.eta;
        t_out[10] = restart | (use_avg << 1) | ((FP32 ? 1 : 0) << 2) | (best_sel << 3);
        t_out[11] = *wsum_old;
    }
}

// The KKT check of the current and average points: two passes and two group
// barriers, then the decision in every CTA. Returns false if a barrier failed.
template <int GK, class T, class V>
__device__ bool run_check(const KParams<T>& P, Ctl& s, const Group& g, int lane, bool evaluate_only, double* s_red,
                          double* s_tot, int* s_flag, double* s_wsum_old) {
    constexpr bool kFP32 = sizeof(T) == 4;
    {
        double v[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) v[k] = 0.0;
        pass_rows_check<GK, T, V>(P, s, g, lane, v);
        cta_partial<10, GK>(v, g, SLOT_CK, s_red);
    }
    if (threadIdx.x == 0) s.pend_y = 0.0;
    if (!group_sync<GK>(g)) return false;
    {
        double v[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) v[k] = 0.0;
        pass_cols_check<GK, T, V>(P, s, g, lane, v);
        cta_partial_at<12, GK>(v, g, SLOT_CK, 10, s_red);
    }
    if (!group_sync<GK>(g)) return false;
    group_totals<22, GK>(g, SLOT_CK, s_tot);
    if (threadIdx.x == 0) check_decision<kFP32>(P, s, s_tot, evaluate_only, g.rank == 0, s_flag, s_wsum_old);
    __syncthreads();
    return true;
}

// Yield at an attempt boundary (after the columns pass and its barrier, or
// after a KKT check): the next attempt's primal step is taken, its |dx|^2
// partials wait in the group's scratch, everything else is in P's buffers
// and the control state. The group total of those partials is formed exactly
// as step_totals forms it and kept in the control state, which the group's
// first CTA writes back with mode MODE_CONTINUE.
template <int GK>
__device__ bool yield_state(const KParamsBase& P, Ctl& s, const Group& g) {
    __shared__ double s_carry;
    if (GK == GK_CTA) {
        if (threadIdx.x == 0) s_carry = cta_sum(g, SLOT_X, 0);
    } else if (threadIdx.x < 32) {
        double v = lane_parts(g.part + (size_t)SLOT_X * g.size * kPartStride, g.size, kPartStride, threadIdx.x);
        v = warp_total(v);
        if (threadIdx.x == 0) s_carry = v;
    }
    __syncthreads();
    if (g.rank == 0 && threadIdx.x == 0) {
        s.dx2_carry = s_carry;
        s.mode = MODE_CONTINUE;
        s.yield_req = 0;
        s.check_now = 0;
        *P.ctl = s;
    }
    __syncthreads();
    return true;
}

// ------------------------------------------------------------ the solve
//
// Per attempt:   rows pass -> barrier -> step decision -> cols pass -> barrier
// Per check:     rows check -> barrier -> cols check -> barrier -> decision
//                [-> best copy / restart pass -> barrier]
// The group's CTAs enter with the same P and leave together. The control
// state is read from P.ctl at entry and written back by the group's first CTA
// at exit. Returns false when a barrier wait timed out (abort).
template <int GK, class T, class V, bool STAGE = false>
__device__ bool solve_body(const KParams<T>& P, const Group& g) {
    __shared__ Ctl s;
    __shared__ double s_red[kWarps * kMaxNV];
    __shared__ double s_tot[kMaxNV];
    __shared__ int s_flag[4];
    __shared__ double s_wsum_old;
    __shared__ double s_pw[2];
    const int tid = threadIdx.x, lane = tid & 31;
    constexpr bool kFP32 = sizeof(T) == 4;

    if (tid == 0) s = *P.ctl;
    __syncthreads();
    const bool first_check = s.check_now != 0 && s.mode != MODE_CONTINUE;
    const bool ypoll = g.yield_at != 0;
    if (g.rank == 0 && tid == 0 && s.mode == MODE_START) s.t_start = (double)gtimer();
    // one CTA alone on the GPU (STAGE): x' and y' also live in shared memory
    // when they fit, and the SpMV gathers read them there (same values, same
    // order). Kernels that keep several CTAs per SM leave it off: the shared
    // memory would come out of the L1 that already caches their iterates.
    T* sx = nullptr;
    T* sy = nullptr;
    if (STAGE && GK == GK_CTA && g.svec && ((size_t)P.n + (size_t)P.m) * sizeof(T) <= (size_t)g.svec_bytes) {
        sx = reinterpret_cast<T*>(g.svec);
        sy = sx + P.n;
    }
    // The whole grid, an LP with few rows: every CTA takes a copy of y' into
    // its shared memory right after the rows barrier (one bulk copy, while the
    // step totals are formed), and the columns pass gathers y' from there.
    __shared__ __align__(8) unsigned long long s_ybar;
    T* ys = nullptr;
    uint32_t ybar_parity = 0;
    const uint32_t ybytes = (uint32_t)(((size_t)P.m * sizeof(T) + 15) & ~(size_t)15);
    if (GK == GK_GRID && g.svec && P.m > 0 && ybytes <= (uint32_t)g.svec_bytes &&
        ((reinterpret_cast<uintptr_t>(P.it.y[0]) | reinterpret_cast<uintptr_t>(P.it.y[1]) |
          reinterpret_cast<uintptr_t>(g.svec)) & 15u) == 0) {
        ys = reinterpret_cast<T*>(g.svec);
        if (tid == 0) mbar_init(&s_ybar, 1);
        __syncthreads();
    }

    // ---------------------------------------------------------- start-up
    if (s.mode == MODE_CONTINUE) {
        // after a yield: every iterate, A x, A^T y and the primal step of the
        // next attempt are where the yield left them; only the |dx|^2 partial
        // sums lived in the group's scratch. Put back the group total as rank
        // 0's partial and zeros for the others: the totals below then come
        // out bit-identical to the ones the uninterrupted solve would form.
        if (tid == 0) {
            if (GK == GK_CTA)
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
                    g.spart[(SLOT_X * kWarps + w) * kPartStride] = w == 0 ? s.dx2_carry : 0.0;
            else g.part[((size_t)SLOT_X * g.size + g.rank) * kPartStride] = g.rank == 0 ? s.dx2_carry : 0.0;
        }
        if (sx)
            for (int j = g.gt; j < P.n; j += g.nt) sx[j] = ld_it<GK>(P.it.x[1 - s.xi] + j);
        __syncthreads();
    } else {
        if (s.mode == MODE_START) {
            // x = x0, y = 0, A^T y = 0, sums = 0 (pdlp_algo.hpp:68-84)
            for (int j = g.gt; j < P.n; j += g.nt) {
                const T x0 = (T)__ldg(P.x0 + j);
                P.it.x[s.xi][j] = x0;
                P.it.x_last[j] = x0;
                P.it.aty[s.aty_cur][j] = T(0);
                P.xsum[j] = 0.0;
            }
            for (int i = g.gt; i < P.m; i += g.nt) {
                P.it.y[s.yi][i] = T(0);
                P.it.y_last[i] = T(0);
                P.ysum[i] = 0.0;
            }
        } else {
            // resume with FP64 iterates after the FP32 phase
            for (int j = g.gt; j < P.n; j += g.nt) {
                P.it.x[s.xi][j] = (T)P.itf.x[s.xi][j];
                P.it.x_last[j] = (T)P.itf.x_last[j];
            }
            for (int i = g.gt; i < P.m; i += g.nt) {
                P.it.y[s.yi][i] = (T)P.itf.y[s.yi][i];
                P.it.y_last[i] = (T)P.itf.y_last[i];
            }
        }
        if (P.debug_delay_ns && g.rank == 0 && tid == 0) {
            // test hook (bounded): hold the first CTA back so the others' barrier wait runs out
            const unsigned long long t0 = gtimer();
            while (gtimer() - t0 < P.debug_delay_ns) __nanosleep(1000);
        }
        if (!group_sync<GK>(g)) return false;
        {   // A x (and A^T y when resuming) at this precision
            const V* vb = vals<V>(P.A);
            T* ax = P.it.ax[s.ax_cur];
            for (int k = g.gw; k < P.A.n_slices; k += g.nw) {
                const int4 sl = __ldg(P.A.slice + k);
                T acc = slice_dot<GK, T, V, T>(P.A, vb, sl, lane, P.it.x[s.xi]);
                if (!seg_finish<GK, T>(P.A, sl, lane, acc, g)) continue;
                const int lg = (int)((uint32_t)sl.y >> kLenBits);
                const int i = sl.x + (lane >> lg);
                if ((lane & ((1 << lg) - 1)) == 0 && i < P.m) ax[i] = acc;
            }
            if (s.mode == MODE_RESUME) {
                const V* vt = vals<V>(P.AT);
                T* aty = P.it.aty[s.aty_cur];
                for (int k = g.gw; k < P.AT.n_slices; k += g.nw) {
                    const int4 sl = __ldg(P.AT.slice + k);
                    T acc = slice_dot<GK, T, V, T>(P.AT, vt, sl, lane, P.it.y[s.yi]);
                    if (!seg_finish<GK, T>(P.AT, sl, lane, acc, g)) continue;
                    const int lg = (int)((uint32_t)sl.y >> kLenBits);
                    const int j = sl.x + (lane >> lg);
                    if ((lane & ((1 << lg) - 1)) == 0 && j < P.n) aty[j] = acc;
                }
            }
        }
        if (!group_sync<GK>(g)) return false;
        {   // primal step of the first attempt
            double dx2[1] = {0.0};
            const double tau = s.eta / s.omega;
            for (int j = g.gt; j < P.n; j += g.nt)
                primal_col<T>(P, j, ld_it<GK>(P.it.x[s.xi] + j), (double)ld_it<GK>(P.it.aty[s.aty_cur] + j), tau,
                              P.it.x[1 - s.xi], dx2[0], sx);
            cta_partial<1, GK>(dx2, g, SLOT_X, s_red);
        }
        if (!group_sync<GK>(g)) return false;
    }

    // --------------------------------------------------------- main loop
    bool check_pending = first_check;
    for (;;) {
        if (!check_pending) {
            // ---- rows pass of one attempt ----
            // the step-size exponents (k+2)^-0.6 and (k+2)^-0.3 of this attempt
            // (pdlp_algo.hpp:120-121) are computed off the critical path by a
            // thread of the second warp while the pass runs
            if (tid == (blockDim.x > 32 ? 32 : 0)) {
                const double k1 = s.accepted + 2.0;
                s_pw[0] = pow(k1, -0.6);
                s_pw[1] = pow(k1, -0.3);
            }
            const bool poll = (s.attempts & 15) == 0;
            int hstop = 0;
            if (poll && g.rank == 0 && tid == 0 && P.host_stop) hstop = *P.host_stop;
            {
                double v[2] = {0.0, 0.0};
                pass_rows_step<GK, T, V>(P, s, g, lane, v, sx, sy);
                cta_partial<2, GK>(v, g, SLOT_A, s_red);
            }
            if (g.rank == 0 && tid == 0) {
                if (poll) {
                    g.bcast[0] = (double)hstop;
                    g.bcast[1] = (P.time_limit_ns > 0 && (double)gtimer() - s.t_start > P.time_limit_ns) ? 1.0 : 0.0;
                }
                if (ypoll) g.bcast[3] = gtimer() >= g.yield_at ? 1.0 : 0.0;
            }
            if (!group_sync<GK>(g)) return false;
            if (ys && tid == 0) bulk_to_smem(ys, P.it.y[1 - s.yi], ybytes, &s_ybar);
            step_totals<GK>(g, s_tot);
            if (tid == 0) {
                // adaptive step size (pdlp_algo.hpp:107-131)
                s.attempts++;
                if (kFP32) s.fp32_attempts++;
                const double dy2 = s_tot[0], inter = s_tot[1], dx2 = s_tot[2];
                const double num = s.omega * dx2 + dy2 / s.omega;
                const double eta_bar = fabs(inter) > 0 ? num / (2.0 * fabs(inter)) : kInfD;
                const double grow = (1.0 + s_pw[0]) * s.eta;
                const double eta_next = isfinite(eta_bar) ? fmin((1.0 - s_pw[1]) * eta_bar, grow) : grow;
                s.pend_y = 0.0;  // applied by the rows pass just finished
                s.pend_x = 0.0;
                if (s.eta <= eta_bar) {
                    s.xi ^= 1;
                    s.yi ^= 1;
                    const int t = s.ax_cur; s.ax_cur = s.ax_nxt; s.ax_nxt = t;
                    s.pend_x = s.eta;  // x-average update, in the cols pass below
                    s.pend_y = s.eta;  // y-average update, in the next rows pass
                    s.wsum += s.eta;
                    s.accepted++;
                    s.since_restart++;
                    s.last_accepted = 1;
                    if (kFP32) s.fp32_accepted++;
                } else {
                    s.last_accepted = 0;
                }
                s.eta = eta_next;
                if (poll) {
                    if (__ldcg(&g.bcast[0]) != 0.0) s.stop_req = B2_EXIT_STOPPED;
                    else if (__ldcg(&g.bcast[1]) != 0.0) s.stop_req = B2_EXIT_TIME_LIMIT;
                }
                if (ypoll && __ldcg(&g.bcast[3]) != 0.0) s.yield_req = 1;
                if (P.yield_attempts > 0 && s.attempts >= P.yield_attempts) s.yield_req = 1;
                s_flag[0] = (s.last_accepted && (s.accepted % P.check_every) == 0) || s.attempts >= P.max_iterations;
                if (ys) {
                    mbar_wait(&s_ybar, ybar_parity, g.abort, g.timeout_ns);
                    ybar_parity ^= 1u;
                }
            }
            __syncthreads();
            const bool check_due = s_flag[0] != 0;
            // ---- cols pass: A^T y' (if accepted) + next primal step ----
            {
                double dx2[1] = {0.0};
                pass_cols_step<GK, T, V>(P, s, g, lane, dx2[0], sx, GK == GK_GRID ? ys : sy);
                cta_partial<1, GK>(dx2, g, SLOT_X, s_red);
            }
            if (tid == 0) {
                s.pend_x = 0.0;
                if (!check_due && s.stop_req) s.exit_reason = s.stop_req;
            }
            if (!group_sync<GK>(g)) return false;
            if (!check_due) {
                if (s.exit_reason != 0) break;
                if (s.yield_req) return yield_state<GK>(P, s, g);
                continue;
            }
        }
        check_pending = false;

        // ---- KKT check on the unscaled problem: current vs average ----
        if (!run_check<GK, T, V>(P, s, g, lane, false, s_red, s_tot, s_flag, &s_wsum_old)) return false;
        if (s.exit_reason == B2_EXIT_CONVERGED) break;
        {
            const int best_sel = s_flag[0], restart = s_flag[1], use_avg = s_flag[2];
            if (best_sel != 0 || restart) {
                double dx2[1] = {0.0};
                pass_after_check<GK, T>(P, s, g, best_sel, restart, use_avg, s_wsum_old, dx2[0], sx);
                if (restart) cta_partial<1, GK>(dx2, g, SLOT_X, s_red);
                __syncthreads();
                if (tid == 0 && restart && use_avg) {
                    int t = s.ax_cur; s.ax_cur = s.ax_avg; s.ax_avg = t;
                    t = s.aty_cur; s.aty_cur = s.aty_avg; s.aty_avg = t;
                }
                if (!group_sync<GK>(g)) return false;
            }
        }
        if (s.switch_req || s.exit_reason != 0) break;
        if (s.yield_req) return yield_state<GK>(P, s, g);
    }

    // ------------------------------------------------------------- exit
    if (s.switch_req && s.exit_reason == 0) {
        // hand the state over to the FP64 phase
        if (g.rank == 0 && tid == 0) *P.ctl = s;
        __syncthreads();
        return true;
    }
    if (s.exit_reason != B2_EXIT_CONVERGED && !s.best_valid) {
        // no check has run yet: evaluate the current point to report it
        if (!run_check<GK, T, V>(P, s, g, lane, true, s_red, s_tot, s_flag, &s_wsum_old)) return false;
    } else if (s.exit_reason != B2_EXIT_CONVERGED) {
        if (tid == 0) {
            s.out_sel = SEL_BEST;
            s.out_eps[0] = s.best_eps[0]; s.out_eps[1] = s.best_eps[1]; s.out_eps[2] = s.best_eps[2];
        }
        __syncthreads();
    }
    {
        const int sel = P.return_current ? (int)SEL_CUR : s.out_sel;
        const T* x = P.it.x[s.xi];
        const T* y = P.it.y[s.yi];
        const double wsum = s.wsum;
        for (int j = g.gt; j < P.n; j += g.nt) {
            const double v = sel == SEL_CUR ? (double)ld_it<GK>(x + j)
                             : sel == SEL_AVG ? ld_it<GK>(P.xsum + j) / wsum : ld_it<GK>(P.best_x + j);
            P.out_x[P.perm_c[j]] = v;
        }
        for (int i = g.gt; i < P.m; i += g.nt) {
            const double v = sel == SEL_CUR ? (double)ld_it<GK>(y + i)
                             : sel == SEL_AVG ? ld_it<GK>(P.ysum + i) / wsum : ld_it<GK>(P.best_y + i);
            P.out_y[P.perm_r[i]] = v;
        }
        __syncthreads();
        if (g.rank == 0 && tid == 0) { s.out_sel = sel; *P.ctl = s; }
        __syncthreads();
    }
    return true;
}

// Standalone SpMV of a sliced matrix (y = M x), for b2_engine_spmv and the
// bandwidth benchmark; the same slice products the solver uses. The FP32
// product stays within 32 registers so that eight 256-thread CTAs fit on an
// SM (the launch is 8 CTAs per SM: one wave).
template <class AccT, class V, class XT>
__global__ void __launch_bounds__(256, sizeof(AccT) == 4 ? 8 : 6) k_spmv(SellDev S, const XT* x, AccT* y) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const V* vb = vals<V>(S);
    for (int s = gw; s < S.n_slices; s += nw) {
        const int4 sl = __ldg(S.slice + s);
        const int2 af = S.aff ? __ldg(S.aff + s) : make_int2(-1, 0);
        AccT acc = af.x >= 0 ? slice_dot_dense<GK_GRID, AccT, V, XT>(vb, sl, af, lane, x)
                             : slice_dot<GK_GRID, AccT, V, XT>(S, vb, sl, lane, x);
        if (!seg_finish_last<AccT>(S, sl, lane, acc)) continue;
        const int lg = (int)((uint32_t)sl.y >> kLenBits);
        const int r = sl.x + (lane >> lg);
        if ((lane & ((1 << lg) - 1)) == 0 && r < S.n_rows) y[r] = acc;
    }
}

}  // namespace dev

// ---------------------------------------------------- host-side helpers
void cuda_ok(cudaError_t e, const char* what);

template <class T>
T* dalloc(size_t count, size_t& total) {
    void* p = nullptr;
    const size_t bytes = (count > 0 ? count : 1) * sizeof(T);
    cuda_ok(cudaMalloc(&p, bytes), "cudaMalloc");
    total += bytes;
    return static_cast<T*>(p);
}

}  // namespace b2
