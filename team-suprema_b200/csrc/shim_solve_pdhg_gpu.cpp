// shim_solve_pdhg_gpu.cpp -- the reference's GPU PDLP entry point, backed by
// the B200 engine's C ABI.
//
// Replaces gpu/pdlp_gpu_solve.cu:261-267 behind the unchanged declaration of
// include/pdlp_gpu.hpp:22-25, so src/solve.cpp (run_pdlp_stage :110, the
// --auto race :290, the concurrent portfolio :560) and tools/audit_lp.cpp:106
// link against this engine without a source change. Compile with the
// reference's headers and SOVEREIGN_WITH_CUDA=1, link with -lb200pdlp.
//
// Contract kept from the reference:
//   * same inputs, same PdlpResult fields (x, y in unscaled PDLP-form space,
//     iterations = attempts, restarts, converged, eps of the returned point);
//   * `eta` ignored (adaptive step size, gpu/pdlp_gpu_solve.cu:263);
//   * stop_flag: cooperative cancellation, answered with the best point so
//     far and converged = false (include/pdlp.hpp:30-34);
//   * errors are thrown as std::runtime_error (gpu/pdlp_gpu_solve.cu:32-38),
//     which every caller catches on its own thread (src/solve.cpp:108-122).
#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "b200_pdlp.h"
#include "pdlp_gpu.hpp"

namespace {

b2_lp_view view_of(const RangedLP& r) {
    b2_lp_view v;
    v.m = r.m();
    v.n = r.n();
    v.nnz = (int64_t)r.A.val.size();
    v.row_idx = r.A.row_idx.data();
    v.col_idx = r.A.col_idx.data();
    v.val = r.A.val.data();
    v.c = r.c.data();
    v.rL = r.rL.data();
    v.rU = r.rU.data();
    v.l = r.l.data();
    v.u = r.u.data();
    v.obj_offset = r.obj_offset;
    return v;
}

// The engine's wait loop calls this about every 20 us while the solve runs:
// a relaxed load of the caller's flag, as include/pdlp.hpp:30-34 polls it.
int32_t poll_stop(void* ctx) {
    return static_cast<const std::atomic<bool>*>(ctx)->load(std::memory_order_relaxed) ? 1 : 0;
}

}  // namespace

PdlpResult solve_pdhg_gpu(const RangedLP& unscaled_form, const RangedLP& scaled_form, const std::vector<double>& Dr,
                          const std::vector<double>& Dc, double eta, int max_iterations, int check_every, double tol,
                          std::atomic<bool>* stop_flag) {
    const b2_lp_view U = view_of(unscaled_form), S = view_of(scaled_form);
    if ((int)Dr.size() != U.m || (int)Dc.size() != U.n)
        throw std::runtime_error("solve_pdhg_gpu: Dr/Dc sizes do not match the PDLP form");
    b2_solve_opts o;
    b2_default_opts(&o);
    o.max_iterations = max_iterations;
    o.check_every = check_every;
    o.tol = tol;
    if (stop_flag) {
        o.stop_poll = poll_stop;
        o.stop_ctx = stop_flag;
    }
    (void)eta;  // adaptive step size (gpu/pdlp_gpu_solve.cu:263)
    PdlpResult res;
    res.x.assign(U.n, 0.0);
    res.y.assign(U.m, 0.0);
    b2_result r{};
    const int rc = b2_solve_pdhg_gpu_ex(&U, &S, Dr.data(), Dc.data(), &o, nullptr, res.x.data(), res.y.data(), &r);
    if (rc != B2_OK) throw std::runtime_error(std::string("b200 PDLP engine (code ") + std::to_string(rc) + "): " +
                                              b2_last_error());
    res.iterations = r.iterations;
    res.restarts = r.restarts;
    res.converged = r.converged != 0;
    res.eps_P = r.eps_P;
    res.eps_D = r.eps_D;
    res.eps_G = r.eps_G;
    return res;
}
