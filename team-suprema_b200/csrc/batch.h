// batch.h -- the queue-driven PDLP kernel shared by batches (batch.cu) and the
// served stream (serve.cu): its launch arguments and host-side launchers.
#pragma once
#include "device.cuh"

namespace b2 {
namespace dev {

constexpr int kMaxCluster = 16;  // CTAs per cluster (non-portable size: enabled per kernel)
constexpr int kClusterScratch = NSLOTS * kMaxCluster * kPartStride + 8;

struct BatchArgs {
    const LpDev* lps;                 // descriptors, indexed by LP id
    int n_inst;                       // single-CTA queue: LP ids in order, head counter
    const int* order;
    unsigned* next;
    int n_large;                      // cluster queue (large LPs)
    const int* order_large;
    unsigned* next_large;
    int* cl_slot;                     // per cluster: the LP it is on
    double* cl_scratch;               // per cluster: partial sums + broadcast words
    double* scratch;                  // per CTA: 8 broadcast words
    int* qstatus;                     // per queue position: exit reason, 0 = yielded
    const volatile int* host_stop;
    int* abort;
    unsigned long long *t_start, *t_end;  // per LP id: first start, finish (global timer)
    unsigned long long* t0;           // launch start, the base of the round deadline (host zeroes it)
    unsigned long long round_ns;      // groups yield this long after the launch starts; 0: never
    double tol, switch_tol, time_limit_ns;
    int max_iterations, check_every, stall_checks, mixed;
    int tail_attempts;                // > 0: LPs yield from this attempt on (the tail lane finishes them)
};

}  // namespace dev

// Co-resident CTAs (CL = 1) and clusters of kMaxCluster (CL = 16) of the
// batched kernel for CTAs of 128, 256 and 512 threads.
struct BatchShape {
    int max_ctas_nt[3];
    int max_clusters_nt[3];
};
void batch_kernel_shape(int sm_count, BatchShape& out);
// Launches the batched kernel on `st`: `units` CTAs (clusters == false) or
// `units` clusters of kMaxCluster CTAs.
void batch_kernel_launch(const dev::BatchArgs& B, bool clusters, int nt, int units, cudaStream_t st);
inline int batch_nt_index(int nt) { return nt == 128 ? 0 : nt == 256 ? 1 : 2; }

// Initial control state of an LP (pdlp_algo.hpp:67-102); fp64_only starts it
// in the FP64 phase.
void init_ctl(dev::Ctl& c, const Layout& l, bool fp64_only);
// Result fields that come from the control state.
void fill_result(const dev::Ctl& f, b2_result& r);
// y = M x through a device sliced matrix of an LP (FP64 accumulation); x, y
// in that LP's caller order; `which` 0: M = A, 1: M = A^T.
void spmv_sell(const dev::SellDev& S, const Layout& l, int which, bool exact32, cudaStream_t stream, const double* x,
               double* y);

}  // namespace b2
