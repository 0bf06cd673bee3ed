// pool.cpp -- shares of a batch or a stream over several GPUs
// (b2_request_work, b2_shard_plan, b2_pool_*).
//
// The reference solves one LP on one device per call
// (gpu/pdlp_gpu_solve.cu:198-205); LPs of a batch or a stream are
// independent, so spreading them over GPUs needs no exchange at all: each GPU
// solves its own share with its own engine and nothing crosses NVLink on the
// data path.
//
//   one process per GPU  every rank runs b2_shard_plan on the same list of
//                        loads and takes the items of its own share; the plan
//                        is deterministic, so the ranks agree without talking.
//   one process          b2_pool keeps a server per GPU and routes each
//                        submitted LP to the member with the least unfinished
//                        work (its backlog, which drains as LPs finish).
#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <mutex>
#include <numeric>
#include <vector>

#include <cuda_runtime.h>

#include "internal.h"

namespace b2 {

void cuda_ok(cudaError_t e, const char* what);  // engine.cu

int64_t request_work(int32_t m, int32_t n, int64_t nnz) {
    return 2 * std::max<int64_t>(nnz, 0) + std::max<int32_t>(m, 0) + std::max<int32_t>(n, 0);
}

// Attempts to 1e-6 grow with the LP: on the 4,096 LPs of the uneven batch
// family (m 50..5,000) a least-squares fit of log(attempts) against log(m)
// gives attempts ~ 167 m^0.657 (R^2 0.83; 832 to 74,496 attempts), and the
// device time of an LP follows work x attempts (log correlation 0.98) more
// closely than work alone (0.95).
int64_t request_cost(int32_t m, int32_t n, int64_t nnz) {
    const double att = 167.0 * std::pow((double)std::max<int32_t>(m, 1), 0.657);
    return request_work(m, n, nnz) * (int64_t)std::llround(att);
}

void shard_plan(const int64_t* work, int64_t count, int32_t parts, bool online, int32_t* rank_of) {
    if (count < 0 || parts < 1) fail(B2_ERR_INVALID, "shard_plan: count < 0 or parts < 1");
    if (count > 0 && (!work || !rank_of)) fail(B2_ERR_INVALID, "null argument");
    for (int64_t i = 0; i < count; ++i)
        if (work[i] < 0) fail(B2_ERR_INVALID, "negative load at item " + std::to_string(i));
    std::vector<int64_t> order((size_t)count);
    std::iota(order.begin(), order.end(), int64_t(0));
    if (!online)
        std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return work[a] > work[b]; });
    std::vector<int64_t> load((size_t)parts, 0);
    for (int64_t i : order) {
        int32_t best = 0;
        for (int32_t r = 1; r < parts; ++r)
            if (load[r] < load[best]) best = r;
        load[best] += work[i];
        rank_of[i] = best;
    }
}

// Pool tickets carry the member in their low bits.
constexpr int kMemberBits = 8;
constexpr int32_t kMaxMembers = 1 << kMemberBits;

struct PoolImpl {
    std::vector<int32_t> devices;
    std::vector<ServerImpl*> members;
    std::mutex route_mu;  // route + submit as one step, so each submit sees the previous one's backlog

    ~PoolImpl() {
        for (ServerImpl* s : members) server_destroy(s);
    }

    int32_t route() const {
        int32_t best = 0;
        int64_t best_load = server_backlog(members[0]);
        for (int32_t k = 1; k < (int32_t)members.size(); ++k) {
            const int64_t w = server_backlog(members[k]);
            if (w < best_load) {
                best = k;
                best_load = w;
            }
        }
        return best;
    }

    static int64_t pack(int64_t inner, int32_t member) { return (inner << kMemberBits) | member; }

    ServerImpl* unpack(int64_t ticket, int64_t* inner, int32_t* member) const {
        if (ticket <= 0) fail(B2_ERR_INVALID, "unknown ticket");
        *member = (int32_t)(ticket & (kMaxMembers - 1));
        *inner = ticket >> kMemberBits;
        if (*member >= (int32_t)members.size()) fail(B2_ERR_INVALID, "unknown ticket");
        return members[*member];
    }
};

PoolImpl* pool_create(const int32_t* devices, int32_t count, const b2_server_opts& so, const b2_solve_opts& o) {
    if (!devices || count < 1) fail(B2_ERR_INVALID, "a pool needs at least one device");
    if (count > kMaxMembers) fail(B2_ERR_INVALID, "a pool holds at most 256 servers");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        fail(B2_ERR_NO_DEVICE, "no CUDA device");
    }
    for (int32_t k = 0; k < count; ++k)
        if (devices[k] < 0 || devices[k] >= ndev)
            fail(B2_ERR_INVALID, "device " + std::to_string(devices[k]) + " does not exist");
    int caller = 0;
    cuda_ok(cudaGetDevice(&caller), "cudaGetDevice");
    std::unique_ptr<PoolImpl> p(new PoolImpl());
    p->devices.assign(devices, devices + count);
    try {
        for (int32_t k = 0; k < count; ++k) {
            cuda_ok(cudaSetDevice(devices[k]), "cudaSetDevice");
            p->members.push_back(server_create(so, o));  // a server owns the current device
        }
    } catch (...) {
        cudaSetDevice(caller);
        throw;
    }
    cuda_ok(cudaSetDevice(caller), "cudaSetDevice");
    return p.release();
}

void pool_destroy(PoolImpl* p) { delete p; }

int64_t pool_submit(PoolImpl* p, const b2_lp_view& U) {
    std::lock_guard<std::mutex> lk(p->route_mu);
    const int32_t k = p->route();
    return PoolImpl::pack(server_submit(p->members[k], U), k);
}

int64_t pool_submit_file(PoolImpl* p, const std::string& path) {
    std::lock_guard<std::mutex> lk(p->route_mu);
    const int32_t k = p->route();
    return PoolImpl::pack(server_submit_file(p->members[k], path), k);
}

int pool_wait(PoolImpl* p, int64_t ticket, double timeout_s, double* x, double* y, b2_result* res,
              b2_request_info* info, int32_t* member) {
    int64_t inner = 0;
    int32_t k = 0;
    ServerImpl* s = p->unpack(ticket, &inner, &k);
    if (member) *member = k;
    return server_wait(s, inner, timeout_s, x, y, res, info);
}

void pool_stats(PoolImpl* p, int32_t member, b2_server_stats* out) {
    if (member < 0 || member >= (int32_t)p->members.size()) fail(B2_ERR_INVALID, "no such pool member");
    server_stats(p->members[member], out);
}

}  // namespace b2
