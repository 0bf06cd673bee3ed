// engine.cu -- the B200 PDLP engine: one persistent, cooperative kernel runs
// the whole restarted-PDHG loop of include/pdlp_algo.hpp:49-185 on the device.
//
// Design (what replaces the reference's gpu/pdlp_gpu_solve.cu):
//   * The reference launches 6+ kernels per attempt and makes one blocking
//     D2H copy per attempt for the step-size test (pdlp_gpu_solve.cu:232-243),
//     plus 4 full-vector D2H copies and 2 host verify() calls every 64
//     accepted steps (pdlp_algo.hpp:135-141). Here nothing leaves the device
//     until the solve ends: every CTA keeps a replica of the scalar control
//     state and takes identical decisions from identical, fixed-order sums.
//   * Two fused passes per attempt, separated by a grid barrier:
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
#include <cuda_runtime.h>

#include <time.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "internal.h"

namespace b2 {
namespace dev {

constexpr int kBlock = 512;
constexpr int kWarps = kBlock / 32;
constexpr int kPartStride = 32;  // doubles per CTA per reduction slot
constexpr int kMaxNV = 22;
enum { SLOT_A = 0, SLOT_X = 1, SLOT_CK = 2, NSLOTS = 3 };
enum { SEL_BEST = 0, SEL_CUR = 1, SEL_AVG = 2 };
// one record per KKT check: attempts, accepted, eps_P/D/G of the current point,
// eps_P/D/G of the average, omega, eta, flags (restart | avg<<1 | fp32<<2 |
// best<<3), weight of the average
constexpr int kTraceFields = 12;
enum { MODE_START = 0, MODE_RESUME = 1 };
constexpr double kInfD = __builtin_huge_val();

struct SellDev {
    int n_rows;
    int n_slices;
    const int4* slice;
    const uint32_t* col;
    const float* v32;
    const double* v64;
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
};

// Launch parameters that do not depend on the iterate precision.
struct KParamsBase {
    int m, n;
    SellDev A, AT;
    const double *b, *rU, *c, *l, *u, *x0;
    const double *dr2, *dc2;  // Dr^2 (negated on >= rows), Dc^2
    Bufs<float> itf;  // FP32 iterates (read when resuming in FP64)
    double *xsum, *ysum, *best_x, *best_y, *out_x, *out_y;
    const int32_t *perm_r, *perm_c;
    double* part;
    double* bcast;  // [0] stop, [1] time-limit hit, [2] start time
    unsigned* bar;
    int* abort;
    Ctl* ctl;
    const volatile int* host_stop;
    double tol, switch_tol, denom_p, denom_d, time_limit_ns;
    unsigned long long timeout_ns;
    int max_iterations, check_every, stall_checks, return_current, mixed;
    unsigned long long debug_delay_ns;  // test hook: CTA 0 arrives late at its first barrier
    double* trace;                      // per-check records (kTraceFields doubles), may be null
    int trace_cap;
};

template <class T>
struct KParams : KParamsBase {
    Bufs<T> it;  // iterates at this precision
};

// ------------------------------------------------------------- primitives
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Matrix streams: read-only for the kernel's lifetime, used once per pass.
__device__ __forceinline__ uint32_t ld_mat(const uint32_t* p) {
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float ld_mat(const float* p) {
    float v;
    asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double ld_mat(const double* p) {
    double v;
    asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
// Iterates are rewritten between passes by other CTAs: read them at L2, never
// through the non-coherent path.
template <class T>
__device__ __forceinline__ T ld_it(const T* p) { return __ldcg(p); }

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

struct Sync {
    unsigned* bar;
    int* abort;
    unsigned long long timeout_ns;
};

// Grid barrier for a cooperative launch. One counter word: CTA 0 adds
// 2^31 - (N-1), the others add 1, so the top bit flips exactly when the last
// CTA arrives. Arrival is a release, polling an acquire (gpu scope). The wait
// is bounded: past timeout_ns the CTA raises `abort` and every CTA leaves.
__device__ __forceinline__ bool grid_sync(const Sync& g) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        if (gridDim.x > 1) {
            const unsigned add = blockIdx.x == 0 ? (0x80000000u - (gridDim.x - 1)) : 1u;
            unsigned old;
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
        }
        if (ok && *(volatile int*)g.abort) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Per-CTA partial sums of NV values -> part[slot][cta][k].
// Values k = 0..NV-1 go to index at + k of the CTA's row of the slot.
template <int NV>
__device__ __forceinline__ void cta_partial_at(double (&v)[NV], double* part, int slot, int at, double* s_red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
        for (int w = 0; w < kWarps; ++w) s += s_red[w * NV + threadIdx.x];
        part[((size_t)slot * gridDim.x + blockIdx.x) * kPartStride + at + threadIdx.x] = s;
    }
}

template <int NV>
__device__ __forceinline__ void cta_partial(double (&v)[NV], double* part, int slot, double* s_red) {
    cta_partial_at<NV>(v, part, slot, 0, s_red);
}

// After a barrier: every CTA sums the CTA partials of one slot in CTA order.
template <int NV>
__device__ __forceinline__ void grid_totals(const double* part, int slot, double* s_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = warp; k < NV; k += kWarps) {
        double s = 0.0;
        for (int b = lane; b < (int)gridDim.x; b += 32)
            s += __ldcg(&part[((size_t)slot * gridDim.x + b) * kPartStride + k]);
        s = warp_total(s);
        if (lane == 0) s_tot[k] = s;
    }
    __syncthreads();
}

// One slice of a sliced-ELL matrix times a gathered vector: every lane sums
// its share of its row in a fixed order, then the g lanes of a row are
// folded onto the row's first lane (fixed tree).
template <class AccT, class V, class XT>
__device__ __forceinline__ AccT slice_dot(const SellDev& S, const V* vbase, int4 sl, int lane, const XT* x) {
    const uint32_t len = (uint32_t)sl.y & kLenMask;
    const int lg = (int)((uint32_t)sl.y >> kLenBits);
    const size_t base = (size_t)(uint32_t)sl.z * 32u + (size_t)lane;
    const uint32_t* cp = S.col + base;
    const V* vp = vbase + base;
    AccT acc = AccT(0);
    uint32_t k = 0;
    for (; k + 4 <= len; k += 4) {
        const uint32_t c0 = ld_mat(cp), c1 = ld_mat(cp + 32), c2 = ld_mat(cp + 64), c3 = ld_mat(cp + 96);
        const V v0 = ld_mat(vp), v1 = ld_mat(vp + 32), v2 = ld_mat(vp + 64), v3 = ld_mat(vp + 96);
        const AccT x0 = (AccT)ld_it(x + c0), x1 = (AccT)ld_it(x + c1), x2 = (AccT)ld_it(x + c2),
                   x3 = (AccT)ld_it(x + c3);
        acc = fma((AccT)v0, x0, acc);
        acc = fma((AccT)v1, x1, acc);
        acc = fma((AccT)v2, x2, acc);
        acc = fma((AccT)v3, x3, acc);
        cp += 128;
        vp += 128;
    }
    for (; k < len; ++k) {
        acc = fma((AccT)ld_mat(vp), (AccT)ld_it(x + ld_mat(cp)), acc);
        cp += 32;
        vp += 32;
    }
    for (int o = (1 << lg) >> 1; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    return acc;
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
__device__ __forceinline__ void primal_col(const KParams<T>& P, int j, T xv, double g, double tau, T* xn,
                                           double& dx2) {
    const double w = __ldg(P.dc2 + j);
    double v = (double)xv - tau * w * (__ldg(P.c + j) - g);
    v = fmin(fmax(v, __ldg(P.l + j)), __ldg(P.u + j));
    const T vt = (T)v;
    xn[j] = vt;
    const double d = (double)vt - (double)xv;
    dx2 += d * d / w;
}

// --------------------------------------------------------------- passes

// Rows: A x' fused with the dual step (pdlp_algo.hpp:111-112, src/pdlp.cpp:125-130)
// and the step-size statistics (pdlp_gpu_solve.cu:119-131).
template <class T, class V>
__device__ void pass_rows_step(const KParams<T>& P, const Ctl& c, int gw, int nw, int lane, double* v) {
    const T* xn = P.it.x[1 - c.xi];
    const T* y = P.it.y[c.yi];
    T* yn = P.it.y[1 - c.yi];
    const T* ax = P.it.ax[c.ax_cur];
    T* axn = P.it.ax[c.ax_nxt];
    const double sigma = c.eta * c.omega, pend = c.pend_y;
    const V* vb = vals<V>(P.A);
    for (int s = gw; s < P.A.n_slices; s += nw) {
        const int4 sl = __ldg(P.A.slice + s);
        const T acc = slice_dot<T, V, T>(P.A, vb, sl, lane, xn);
        const int lg = (int)((uint32_t)sl.y >> kLenBits);
        const int row = sl.x + (lane >> lg);
        if ((lane & ((1 << lg) - 1)) == 0 && row < P.m) {
            const T yv = ld_it(y + row), axv = ld_it(ax + row);
            const double w = __ldg(P.dr2 + row);
            const double aw = fabs(w);
            double nv = (double)yv + sigma * aw * (__ldg(P.b + row) - (2.0 * (double)acc - (double)axv));
            if (w < 0.0 && nv < 0.0) nv = 0.0;
            const T nt = (T)nv;
            yn[row] = nt;
            axn[row] = acc;
            const double d = (double)nt - (double)yv;
            v[0] += d * d / aw;
            v[1] += d * ((double)acc - (double)axv);
            if (pend != 0.0) P.ysum[row] += pend * (double)yv;
        }
    }
}

// Columns: [accepted] A^T y' + x-average update, then the next primal step.
template <class T, class V>
__device__ void pass_cols_step(const KParams<T>& P, const Ctl& c, int gw, int nw, int gt, int nt, int lane,
                               double& dx2) {
    const T* x = P.it.x[c.xi];
    T* xn = P.it.x[1 - c.xi];
    T* aty = P.it.aty[c.aty_cur];
    const double tau = c.eta / c.omega, pend = c.pend_x;
    if (c.last_accepted) {
        const T* y = P.it.y[c.yi];
        const V* vb = vals<V>(P.AT);
        for (int s = gw; s < P.AT.n_slices; s += nw) {
            const int4 sl = __ldg(P.AT.slice + s);
            const T acc = slice_dot<T, V, T>(P.AT, vb, sl, lane, y);
            const int lg = (int)((uint32_t)sl.y >> kLenBits);
            const int j = sl.x + (lane >> lg);
            if ((lane & ((1 << lg) - 1)) == 0 && j < P.n) {
                aty[j] = acc;
                const T xv = ld_it(x + j);
                if (pend != 0.0) P.xsum[j] += pend * (double)xv;
                primal_col<T>(P, j, xv, (double)acc, tau, xn, dx2);
            }
        }
    } else {
        for (int j = gt; j < P.n; j += nt) primal_col<T>(P, j, ld_it(x + j), (double)ld_it(aty + j), tau, xn, dx2);
    }
}

// KKT check, rows (verify.cpp:35-87 row terms) for the current and average
// points, the average's A x, the restart distance of y, and the pending
// y-average update.
template <class T, class V>
__device__ void pass_rows_check(const KParams<T>& P, const Ctl& c, int gw, int nw, int lane, double* v) {
    const T* y = P.it.y[c.yi];
    const T* ax = P.it.ax[c.ax_cur];
    T* axa = P.it.ax[c.ax_avg];
    const bool has_avg = c.wsum > 0;
    const double wsum = c.wsum, pend = c.pend_y;
    const V* vb = vals<V>(P.A);
    for (int s = gw; s < P.A.n_slices; s += nw) {
        const int4 sl = __ldg(P.A.slice + s);
        double acc = 0.0;
        if (has_avg) acc = slice_dot<double, V, double>(P.A, vb, sl, lane, P.xsum);
        const int lg = (int)((uint32_t)sl.y >> kLenBits);
        const int i = sl.x + (lane >> lg);
        if ((lane & ((1 << lg) - 1)) == 0 && i < P.m) {
            const double yc = (double)ld_it(y + i);
            double ys = __ldcg(P.ysum + i);
            if (pend != 0.0) { ys += pend * yc; P.ysum[i] = ys; }
            const double ac = (double)ld_it(ax + i);
            const double aa = has_avg ? acc / wsum : ac;
            const double ya = has_avg ? ys / wsum : yc;
            axa[i] = (T)aa;
            const double rl = __ldg(P.b + i), ru = __ldg(P.rU + i);
            kkt_row(rl, ru, ac, yc, v + 0);
            kkt_row(rl, ru, aa, ya, v + 4);
            const double w = fabs(__ldg(P.dr2 + i)), yl = (double)ld_it(P.it.y_last + i);
            v[8] += (yc - yl) * (yc - yl) / w;
            v[9] += (ya - yl) * (ya - yl) / w;
        }
    }
}

template <class T, class V>
__device__ void pass_cols_check(const KParams<T>& P, const Ctl& c, int gw, int nw, int lane, double* v) {
    const T* x = P.it.x[c.xi];
    const T* aty = P.it.aty[c.aty_cur];
    T* atya = P.it.aty[c.aty_avg];
    const bool has_avg = c.wsum > 0;
    const double wsum = c.wsum;
    const V* vb = vals<V>(P.AT);
    for (int s = gw; s < P.AT.n_slices; s += nw) {
        const int4 sl = __ldg(P.AT.slice + s);
        double acc = 0.0;
        if (has_avg) acc = slice_dot<double, V, double>(P.AT, vb, sl, lane, P.ysum);
        const int lg = (int)((uint32_t)sl.y >> kLenBits);
        const int j = sl.x + (lane >> lg);
        if ((lane & ((1 << lg) - 1)) == 0 && j < P.n) {
            const double xc = (double)ld_it(x + j), gc = (double)ld_it(aty + j);
            const double xa = has_avg ? __ldcg(P.xsum + j) / wsum : xc;
            const double ga = has_avg ? acc / wsum : gc;
            atya[j] = (T)ga;
            const double cc = __ldg(P.c + j), l = __ldg(P.l + j), u = __ldg(P.u + j);
            kkt_col(l, u, cc, xc, cc - gc, v + 0);
            kkt_col(l, u, cc, xa, cc - ga, v + 5);
            const double w = __ldg(P.dc2 + j), xl = (double)ld_it(P.it.x_last + j);
            v[10] += (xc - xl) * (xc - xl) / w;
            v[11] += (xa - xl) * (xa - xl) / w;
        }
    }
}

// After a check: copy the new best point, apply a restart (pdlp_algo.hpp:160-174)
// and, on restart, redo the next primal step with the new primal weight.
template <class T>
__device__ void pass_after_check(const KParams<T>& P, const Ctl& c, int best_sel, int restart, int use_avg,
                                 double wsum_old, int gt, int nt, double& dx2) {
    const bool has_avg = wsum_old > 0;
    T* x = P.it.x[c.xi];
    T* xn = P.it.x[1 - c.xi];
    const double tau = c.eta / c.omega;
    for (int j = gt; j < P.n; j += nt) {
        const T xct = ld_it(x + j);
        const double xc = (double)xct;
        const double xa = has_avg ? __ldcg(P.xsum + j) / wsum_old : xc;
        if (best_sel == SEL_CUR) P.best_x[j] = xc;
        else if (best_sel == SEL_AVG) P.best_x[j] = xa;
        if (restart) {
            const double cand = use_avg ? xa : xc;
            P.it.x_last[j] = (T)cand;
            T xnew = xct;
            if (use_avg) { xnew = (T)xa; x[j] = xnew; }
            P.xsum[j] = 0.0;
            const double g = (double)ld_it((use_avg ? P.it.aty[c.aty_avg] : P.it.aty[c.aty_cur]) + j);
            primal_col<T>(P, j, xnew, g, tau, xn, dx2);
        }
    }
    T* y = P.it.y[c.yi];
    for (int i = gt; i < P.m; i += nt) {
        const T yct = ld_it(y + i);
        const double yc = (double)yct;
        const double ya = has_avg ? __ldcg(P.ysum + i) / wsum_old : yc;
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

// Totals of the step-size statistics after a barrier: dy2 and dy'(Ax'-Ax)
// from the rows pass, |dx|^2 from the columns pass before it.
__device__ __forceinline__ void step_totals(const double* part, double* s_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp < 3) {
        const int slot = warp < 2 ? SLOT_A : SLOT_X, k = warp < 2 ? warp : 0;
        double s = 0.0;
        for (int b = lane; b < (int)gridDim.x; b += 32)
            s += __ldcg(&part[((size_t)slot * gridDim.x + b) * kPartStride + k]);
        s = warp_total(s);
        if (lane == 0) s_tot[warp] = s;
    }
    __syncthreads();
}

// Check decision (pdlp_algo.hpp:135-174) from the 22 check totals; run by one
// thread per CTA on identical inputs. Returns, through `flags`, which point
// becomes the best point, whether to restart and whether to the average.
template <bool FP32>
__device__ void check_decision(const KParamsBase& B, Ctl& s, const double* t, bool evaluate_only, int* flags,
                               double* wsum_old) {
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
    if (blockIdx.x == 0 && B.trace && s.checks - 1 < B.trace_cap) {
        double* t_out = B.trace + (size_t)(s.checks - 1) * kTraceFields;
        t_out[0] = s.attempts; t_out[1] = s.accepted;
        t_out[2] = eP[0]; t_out[3] = eD[0]; t_out[4] = eG[0];
        t_out[5] = eP[1]; t_out[6] = eD[1]; t_out[7] = eG[1];
        t_out[8] = s.omega; t_out[9] = s.eta;
        t_out[10] = restart | (use_avg << 1) | ((FP32 ? 1 : 0) << 2) | (best_sel << 3);
        t_out[11] = *wsum_old;
    }
}

// -------------------------------------------------------------- the kernel
//
// Per attempt:   rows pass -> barrier -> step decision -> cols pass -> barrier
// Per check:     rows check -> barrier -> cols check -> barrier -> decision
//                [-> best copy / restart pass -> barrier]
template <class T, class V>
__global__ void __launch_bounds__(kBlock, 2) k_pdlp(const KParams<T> P) {
    __shared__ Ctl s;
    __shared__ double s_red[kWarps * kMaxNV];
    __shared__ double s_tot[kMaxNV];
    __shared__ int s_flag[4];
    __shared__ double s_wsum_old;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gw = blockIdx.x * kWarps + warp, nw = gridDim.x * kWarps;
    const int gt = blockIdx.x * kBlock + tid, nt = gridDim.x * kBlock;
    constexpr bool kFP32 = sizeof(T) == 4;
    const Sync sy{P.bar, P.abort, P.timeout_ns};

    if (tid == 0) s = *P.ctl;
    __syncthreads();
    const bool first_check = s.check_now != 0;
    if (blockIdx.x == 0 && tid == 0 && s.mode == MODE_START) P.bcast[2] = (double)gtimer();

    // ---------------------------------------------------------- start-up
    if (s.mode == MODE_START) {
        // x = x0, y = 0, A^T y = 0, sums = 0 (pdlp_algo.hpp:68-84)
        for (int j = gt; j < P.n; j += nt) {
            const T x0 = (T)__ldg(P.x0 + j);
            P.it.x[s.xi][j] = x0;
            P.it.x_last[j] = x0;
            P.it.aty[s.aty_cur][j] = T(0);
            P.xsum[j] = 0.0;
        }
        for (int i = gt; i < P.m; i += nt) {
            P.it.y[s.yi][i] = T(0);
            P.it.y_last[i] = T(0);
            P.ysum[i] = 0.0;
        }
    } else {
        // resume with FP64 iterates after the FP32 phase
        for (int j = gt; j < P.n; j += nt) {
            P.it.x[s.xi][j] = (T)P.itf.x[s.xi][j];
            P.it.x_last[j] = (T)P.itf.x_last[j];
        }
        for (int i = gt; i < P.m; i += nt) {
            P.it.y[s.yi][i] = (T)P.itf.y[s.yi][i];
            P.it.y_last[i] = (T)P.itf.y_last[i];
        }
    }
    if (P.debug_delay_ns && blockIdx.x == 0 && tid == 0) {
        // test hook (bounded): hold CTA 0 back so the others' barrier wait runs out
        const unsigned long long t0 = gtimer();
        while (gtimer() - t0 < P.debug_delay_ns) __nanosleep(1000);
    }
    if (!grid_sync(sy)) return;
    {   // A x (and A^T y when resuming) at this precision
        const V* vb = vals<V>(P.A);
        T* ax = P.it.ax[s.ax_cur];
        for (int k = gw; k < P.A.n_slices; k += nw) {
            const int4 sl = __ldg(P.A.slice + k);
            const T acc = slice_dot<T, V, T>(P.A, vb, sl, lane, P.it.x[s.xi]);
            const int lg = (int)((uint32_t)sl.y >> kLenBits);
            const int i = sl.x + (lane >> lg);
            if ((lane & ((1 << lg) - 1)) == 0 && i < P.m) ax[i] = acc;
        }
        if (s.mode == MODE_RESUME) {
            const V* vt = vals<V>(P.AT);
            T* aty = P.it.aty[s.aty_cur];
            for (int k = gw; k < P.AT.n_slices; k += nw) {
                const int4 sl = __ldg(P.AT.slice + k);
                const T acc = slice_dot<T, V, T>(P.AT, vt, sl, lane, P.it.y[s.yi]);
                const int lg = (int)((uint32_t)sl.y >> kLenBits);
                const int j = sl.x + (lane >> lg);
                if ((lane & ((1 << lg) - 1)) == 0 && j < P.n) aty[j] = acc;
            }
        }
    }
    if (!grid_sync(sy)) return;
    {   // primal step of the first attempt
        double dx2[1] = {0.0};
        const double tau = s.eta / s.omega;
        for (int j = gt; j < P.n; j += nt)
            primal_col<T>(P, j, ld_it(P.it.x[s.xi] + j), (double)ld_it(P.it.aty[s.aty_cur] + j), tau,
                          P.it.x[1 - s.xi], dx2[0]);
        cta_partial<1>(dx2, P.part, SLOT_X, s_red);
    }
    if (!grid_sync(sy)) return;

    // --------------------------------------------------------- main loop
    bool check_pending = first_check;
    for (;;) {
        if (!check_pending) {
            // ---- rows pass of one attempt ----
            const bool poll = (s.attempts & 15) == 0;
            int hstop = 0;
            if (poll && blockIdx.x == 0 && tid == 0 && P.host_stop) hstop = *P.host_stop;
            {
                double v[2] = {0.0, 0.0};
                pass_rows_step<T, V>(P, s, gw, nw, lane, v);
                cta_partial<2>(v, P.part, SLOT_A, s_red);
            }
            if (poll && blockIdx.x == 0 && tid == 0) {
                P.bcast[0] = (double)hstop;
                P.bcast[1] = (P.time_limit_ns > 0 && (double)gtimer() - P.bcast[2] > P.time_limit_ns) ? 1.0 : 0.0;
            }
            if (!grid_sync(sy)) return;
            step_totals(P.part, s_tot);
            if (tid == 0) {
                // adaptive step size (pdlp_algo.hpp:107-131)
                s.attempts++;
                if (kFP32) s.fp32_attempts++;
                const double dy2 = s_tot[0], inter = s_tot[1], dx2 = s_tot[2];
                const double num = s.omega * dx2 + dy2 / s.omega;
                const double eta_bar = fabs(inter) > 0 ? num / (2.0 * fabs(inter)) : kInfD;
                const double k1 = s.accepted + 2.0;
                const double grow = (1.0 + pow(k1, -0.6)) * s.eta;
                const double eta_next = isfinite(eta_bar) ? fmin((1.0 - pow(k1, -0.3)) * eta_bar, grow) : grow;
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
                    if (__ldcg(&P.bcast[0]) != 0.0) s.stop_req = B2_EXIT_STOPPED;
                    else if (__ldcg(&P.bcast[1]) != 0.0) s.stop_req = B2_EXIT_TIME_LIMIT;
                }
                s_flag[0] = (s.last_accepted && (s.accepted % P.check_every) == 0) || s.attempts >= P.max_iterations;
            }
            __syncthreads();
            const bool check_due = s_flag[0] != 0;
            // ---- cols pass: A^T y' (if accepted) + next primal step ----
            {
                double dx2[1] = {0.0};
                pass_cols_step<T, V>(P, s, gw, nw, gt, nt, lane, dx2[0]);
                cta_partial<1>(dx2, P.part, SLOT_X, s_red);
            }
            if (tid == 0) {
                s.pend_x = 0.0;
                if (!check_due && s.stop_req) s.exit_reason = s.stop_req;
            }
            if (!grid_sync(sy)) return;
            if (!check_due) {
                if (s.exit_reason != 0) break;
                continue;
            }
        }
        check_pending = false;

        // ---- KKT check on the unscaled problem: current vs average ----
        {
            double v[10];
#pragma unroll
            for (int k = 0; k < 10; ++k) v[k] = 0.0;
            pass_rows_check<T, V>(P, s, gw, nw, lane, v);
            cta_partial<10>(v, P.part, SLOT_CK, s_red);
        }
        if (tid == 0) s.pend_y = 0.0;
        if (!grid_sync(sy)) return;
        {
            double v[12];
#pragma unroll
            for (int k = 0; k < 12; ++k) v[k] = 0.0;
            pass_cols_check<T, V>(P, s, gw, nw, lane, v);
            cta_partial_at<12>(v, P.part, SLOT_CK, 10, s_red);
        }
        if (!grid_sync(sy)) return;
        grid_totals<22>(P.part, SLOT_CK, s_tot);
        if (tid == 0) check_decision<kFP32>(P, s, s_tot, false, s_flag, &s_wsum_old);
        __syncthreads();
        if (s.exit_reason == B2_EXIT_CONVERGED) break;
        {
            const int best_sel = s_flag[0], restart = s_flag[1], use_avg = s_flag[2];
            if (best_sel != 0 || restart) {
                double dx2[1] = {0.0};
                pass_after_check<T>(P, s, best_sel, restart, use_avg, s_wsum_old, gt, nt, dx2[0]);
                if (restart) cta_partial<1>(dx2, P.part, SLOT_X, s_red);
                __syncthreads();
                if (tid == 0 && restart && use_avg) {
                    int t = s.ax_cur; s.ax_cur = s.ax_avg; s.ax_avg = t;
                    t = s.aty_cur; s.aty_cur = s.aty_avg; s.aty_avg = t;
                }
                if (!grid_sync(sy)) return;
            }
        }
        if (s.switch_req || s.exit_reason != 0) break;
    }

    // ------------------------------------------------------------- exit
    if (s.switch_req && s.exit_reason == 0) {
        // hand the state over to the FP64 kernel
        if (blockIdx.x == 0 && tid == 0) *P.ctl = s;
        return;
    }
    if (s.exit_reason != B2_EXIT_CONVERGED && !s.best_valid) {
        // no check has run yet: evaluate the current point to report it
        {
            double v[10];
#pragma unroll
            for (int k = 0; k < 10; ++k) v[k] = 0.0;
            pass_rows_check<T, V>(P, s, gw, nw, lane, v);
            cta_partial<10>(v, P.part, SLOT_CK, s_red);
        }
        if (tid == 0) s.pend_y = 0.0;
        if (!grid_sync(sy)) return;
        {
            double v[12];
#pragma unroll
            for (int k = 0; k < 12; ++k) v[k] = 0.0;
            pass_cols_check<T, V>(P, s, gw, nw, lane, v);
            cta_partial_at<12>(v, P.part, SLOT_CK, 10, s_red);
        }
        if (!grid_sync(sy)) return;
        grid_totals<22>(P.part, SLOT_CK, s_tot);
        if (tid == 0) check_decision<kFP32>(P, s, s_tot, true, s_flag, &s_wsum_old);
        __syncthreads();
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
        for (int j = gt; j < P.n; j += nt) {
            const double v = sel == SEL_CUR ? (double)ld_it(x + j)
                             : sel == SEL_AVG ? __ldcg(P.xsum + j) / wsum : __ldcg(P.best_x + j);
            P.out_x[P.perm_c[j]] = v;
        }
        for (int i = gt; i < P.m; i += nt) {
            const double v = sel == SEL_CUR ? (double)ld_it(y + i)
                             : sel == SEL_AVG ? __ldcg(P.ysum + i) / wsum : __ldcg(P.best_y + i);
            P.out_y[P.perm_r[i]] = v;
        }
        __syncthreads();
        if (blockIdx.x == 0 && tid == 0) { s.out_sel = sel; *P.ctl = s; }
    }
}

// Standalone SpMV of a sliced matrix (y = M x), for b2_engine_spmv and the
// bandwidth benchmark; the same slice_dot the solver uses.
template <class AccT, class V, class XT>
__global__ void __launch_bounds__(256) k_spmv(SellDev S, const XT* x, AccT* y) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const V* vb = vals<V>(S);
    for (int s = gw; s < S.n_slices; s += nw) {
        const int4 sl = __ldg(S.slice + s);
        const AccT acc = slice_dot<AccT, V, XT>(S, vb, sl, lane, x);
        const int lg = (int)((uint32_t)sl.y >> kLenBits);
        const int r = sl.x + (lane >> lg);
        if ((lane & ((1 << lg) - 1)) == 0 && r < S.n_rows) y[r] = acc;
    }
}

}  // namespace dev

// ===================================================================== host
namespace {

void cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) fail(B2_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        fail(B2_ERR_NO_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
    fail(B2_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
T* dalloc(size_t count, size_t& total) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cuda_ok(cudaMalloc(&p, bytes), "cudaMalloc");
    total += bytes;
    return static_cast<T*>(p);
}

template <class T>
T* upload(const std::vector<T>& h, size_t& total) {
    T* d = dalloc<T>(h.size(), total);
    if (!h.empty()) cuda_ok(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return d;
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
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    template <class T>
    T* alloc(size_t n) {
        T* p = dalloc<T>(n, bytes);
        allocs.push_back(p);
        return p;
    }
    template <class T>
    T* up(const std::vector<T>& h) {
        T* p = upload(h, bytes);
        allocs.push_back(p);
        return p;
    }

    ~EngineImpl() {
        for (void* p : allocs) cudaFree(p);
        if (h_stop) cudaFreeHost(h_stop);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }

    dev::SellDev upload_sell(const SellHost& S) {
        dev::SellDev d{};
        d.n_rows = S.n_rows;
        d.n_slices = (int)S.n_slices();
        d.slice = reinterpret_cast<const int4*>(up(S.slice));
        d.col = up(S.col);
        d.v32 = up(S.val32);
        d.v64 = S.val64.empty() ? nullptr : up(S.val64);
        return d;
    }

    template <class T>
    void alloc_bufs(dev::Bufs<T>& B) {
        for (auto& p : B.x) p = alloc<T>(L.n);
        for (auto& p : B.y) p = alloc<T>(L.m);
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
        build_layout(U, S, Dr, Dc, bp, L);
        int ndev = 0;
        cuda_ok(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
        if (ndev == 0) fail(B2_ERR_NO_DEVICE, "no CUDA device");
        cuda_ok(cudaGetDevice(&device), "cudaGetDevice");
        cuda_ok(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device), "attr");
        cuda_ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_ok(cudaEventCreate(&ev0), "event");
        cuda_ok(cudaEventCreate(&ev1), "event");
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
        part = alloc<double>((size_t)dev::NSLOTS * max_ctas * dev::kPartStride);
        cuda_ok(cudaDeviceSynchronize(), "create");
    }

    int pick_ctas(const b2_solve_opts& o) const {
        const int64_t work = L.A.padded + L.AT.padded + 4 * ((int64_t)L.m + L.n);
        int ctas = (int)std::min<int64_t>(max_ctas, std::max<int64_t>(1, work / 16384));
        if (o.max_ctas > 0) ctas = std::min(ctas, o.max_ctas);
        return std::max(1, ctas);
    }

    template <class T>
    dev::KParams<T> params(const b2_solve_opts& o, dev::Bufs<T>& B) {
        dev::KParams<T> P{};
        P.m = L.m; P.n = L.n;
        P.A = A; P.AT = AT;
        P.b = b; P.rU = rU; P.c = c; P.l = l; P.u = u; P.x0 = x0; P.dr2 = dr2; P.dc2 = dc2;
        P.it = B;
        P.itf = itf;
        P.xsum = xsum; P.ysum = ysum; P.best_x = best_x; P.best_y = best_y; P.out_x = out_x; P.out_y = out_y;
        P.perm_r = perm_r; P.perm_c = perm_c;
        P.part = part; P.bcast = bcast; P.bar = bar; P.abort = abort_flag; P.ctl = ctl;
        P.host_stop = d_stop;
        P.tol = o.tol;
        P.switch_tol = o.switch_tol;
        P.denom_p = L.denom_p; P.denom_d = L.denom_d;
        P.time_limit_ns = o.time_limit_s > 0 ? o.time_limit_s * 1e9 : 0.0;
        P.timeout_ns = (unsigned long long)((o.barrier_timeout_s > 0 ? o.barrier_timeout_s : 10.0) * 1e9);
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

    template <class T, class V>
    void launch(const dev::KParams<T>& P, int ctas, cudaStream_t st) {
        cuda_ok(cudaMemsetAsync(bar, 0, sizeof(unsigned), st), "memset");
        cuda_ok(cudaMemsetAsync(abort_flag, 0, sizeof(int), st), "memset");
        void* args[] = {(void*)&P};
        cuda_ok(cudaLaunchCooperativeKernel((const void*)dev::k_pdlp<T, V>, dim3(ctas), dim3(dev::kBlock), args, 0, st),
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
        *h_stop = stop_flag ? *stop_flag : 0;
        cuda_ok(cudaMemcpyAsync(ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st), "ctl upload");
        const int ctas = pick_ctas(o);
        const bool mixed = o.precision == B2_PREC_MIXED;
        const bool exact = L.exact32;
        cuda_ok(cudaEventRecord(ev0, st), "event");
        if (mixed) {
            auto P = params<float>(o, itf);
            launch<float, float>(P, ctas, st);
            cuda_ok(cudaEventRecord(ev1, st), "event");
            wait(stop_flag);
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
                if (exact) launch<double, float>(Q, ctas, st);
                else launch<double, double>(Q, ctas, st);
                cuda_ok(cudaEventRecord(ev1, st), "event");
                wait(stop_flag);
                check_abort();
            }
        } else {
            auto Q = params<double>(o, itd);
            if (exact) launch<double, float>(Q, ctas, st);
            else launch<double, double>(Q, ctas, st);
            cuda_ok(cudaEventRecord(ev1, st), "event");
            wait(stop_flag);
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
            res->objective = L.obj_offset;
            if (x_out) {
                // c'x in the caller's column order
                for (int32_t j = 0; j < L.n; ++j) res->objective += L.c[L.inv_c[j]] * x_out[j];
            }
            res->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
        }
    }

    // Waits for the persistent kernel while mirroring the caller's stop flag
    // into the mapped word the device polls.
    void wait(const volatile int32_t* stop_flag) {
        for (;;) {
            cudaError_t q = cudaEventQuery(ev1);
            if (q == cudaSuccess) return;
            if (q != cudaErrorNotReady) cuda_ok(q, "persistent kernel");
            if (stop_flag && *stop_flag) *(volatile int*)h_stop = 1;
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

void engine_destroy(EngineImpl* e) { delete e; }

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
