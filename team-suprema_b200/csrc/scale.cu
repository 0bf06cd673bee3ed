// scale.cu -- Ruiz + Pock-Chambolle scaling on the GPU (b2_scale_gpu).
//
// The same scaling as scale() in src/scaling.cpp:25-84 and as the host
// restatement scale_lp (host_prep.cpp), bit for bit: every value is touched by
// the same FP64 operations, and the two order-dependent reductions (the
// Pock-Chambolle row and column sums) add a row's (column's) entries in the
// order the COO lists them, as the sequential host loop does. Maxima and the
// elementwise products do not depend on order. The host only builds the two
// stable orderings of the entries (by row, by column; a counting sort) that
// give each row and column its entries in COO order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "device.cuh"

namespace b2 {
namespace dev {

// One thread per row (or column): the max of |val| over its entries, then
// the Ruiz factor 1/sqrt(max) (1 for an empty row), folded into D.
__global__ void k_ruiz_factor(int rows, const int64_t* __restrict__ ptr, const int64_t* __restrict__ ord,
                              const double* __restrict__ val, double* __restrict__ f, double* __restrict__ D) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        double mx = 0.0;
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) mx = fmax(mx, fabs(val[ord[p]]));
        const double s = mx > 0 ? 1.0 / sqrt(mx) : 1.0;
        f[i] = s;
        D[i] *= s;
    }
}

// val[k] *= f[key[k]] for every entry.
__global__ void k_scale_entries(int64_t nnz, const int32_t* __restrict__ key, const double* __restrict__ f,
                                double* __restrict__ val) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        val[k] = val[k] * f[key[k]];
}

// Pock-Chambolle (alpha = 1): sqrt(1 / sum |val|) per row / column, the sum
// taken in COO order; folded into D.
__global__ void k_pc_factor(int rows, const int64_t* __restrict__ ptr, const int64_t* __restrict__ ord,
                            const double* __restrict__ val, double* __restrict__ f, double* __restrict__ D) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) s += fabs(val[ord[p]]);
        const double g = sqrt(s > 0 ? 1.0 / s : 1.0);
        f[i] = g;
        D[i] *= g;
    }
}

// val[k] = val[k] * fr[row[k]] * fc[col[k]] (the final Pock-Chambolle step,
// one product after the other as the host loop forms it).
__global__ void k_scale_both(int64_t nnz, const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                             const double* __restrict__ fr, const double* __restrict__ fc, double* __restrict__ val) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        val[k] = val[k] * fr[row[k]] * fc[col[k]];
}

__global__ void k_fill(int n, double v, double* __restrict__ a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = v;
}

}  // namespace dev

namespace {

// Entries ordered by key, each key's entries in COO order (stable counting sort).
void stable_order(int rows, int64_t nnz, const int32_t* key, std::vector<int64_t>& ptr, std::vector<int64_t>& ord) {
    ptr.assign((size_t)rows + 1, 0);
    for (int64_t k = 0; k < nnz; ++k) ptr[key[k] + 1]++;
    for (int i = 0; i < rows; ++i) ptr[i + 1] += ptr[i];
    ord.resize((size_t)std::max<int64_t>(nnz, 1));
    std::vector<int64_t> cur(ptr.begin(), ptr.end() - 1);
    for (int64_t k = 0; k < nnz; ++k) ord[cur[key[k]]++] = k;
}

// Stream-ordered buffers: no device-wide synchronisation on free, so the
// served stream's preparation threads can scale while its rounds run.
struct DevBuf {
    cudaStream_t st;
    std::vector<void*> p;
    template <class T>
    T* get(size_t count) {
        void* q = nullptr;
        cuda_ok(cudaMallocAsync(&q, std::max<size_t>(count, 1) * sizeof(T), st), "cudaMallocAsync");
        p.push_back(q);
        return static_cast<T*>(q);
    }
    ~DevBuf() {
        for (void* q : p) cudaFreeAsync(q, st);
        cudaStreamSynchronize(st);
    }
};

template <class T>
void h2d(T* d, const T* h, size_t count, cudaStream_t st) {
    if (count) cuda_ok(cudaMemcpyAsync(d, h, count * sizeof(T), cudaMemcpyHostToDevice, st), "H2D");
}
template <class T>
void d2h(T* h, const T* d, size_t count, cudaStream_t st) {
    if (count) cuda_ok(cudaMemcpyAsync(h, d, count * sizeof(T), cudaMemcpyDeviceToHost, st), "D2H");
}

}  // namespace

void scale_lp_gpu(const b2_lp_view& lp, int ruiz_passes, double* val_s, double* c_s, double* rL_s, double* rU_s,
                  double* l_s, double* u_s, double* Dr, double* Dc) {
    const int32_t m = lp.m, n = lp.n;
    const int64_t nnz = lp.nnz;
    if (m < 0 || n < 0 || nnz < 0) fail(B2_ERR_INVALID, "negative size");
    if (nnz > 0 && (!lp.row_idx || !lp.col_idx || !lp.val)) fail(B2_ERR_INVALID, "null matrix arrays");
    for (int64_t k = 0; k < nnz; ++k)
        if (lp.row_idx[k] < 0 || lp.row_idx[k] >= m || lp.col_idx[k] < 0 || lp.col_idx[k] >= n)
            fail(B2_ERR_INVALID, "matrix index out of range");
    int ndev = 0;
    cuda_ok(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (ndev == 0) fail(B2_ERR_NO_DEVICE, "no CUDA device");
    std::vector<int64_t> rptr, rord, cptr, cord;
    stable_order(m, nnz, lp.row_idx, rptr, rord);
    stable_order(n, nnz, lp.col_idx, cptr, cord);

    cudaStream_t st = nullptr;
    cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    DevBuf B{st, {}};
    const size_t nz = (size_t)std::max<int64_t>(nnz, 1);
    int32_t* d_row = B.get<int32_t>(nz);
    int32_t* d_col = B.get<int32_t>(nz);
    double* d_val = B.get<double>(nz);
    int64_t* d_rptr = B.get<int64_t>((size_t)m + 1);
    int64_t* d_rord = B.get<int64_t>(nz);
    int64_t* d_cptr = B.get<int64_t>((size_t)n + 1);
    int64_t* d_cord = B.get<int64_t>(nz);
    double* d_fr = B.get<double>(std::max(m, 1));
    double* d_fc = B.get<double>(std::max(n, 1));
    double* d_Dr = B.get<double>(std::max(m, 1));
    double* d_Dc = B.get<double>(std::max(n, 1));
    h2d(d_row, lp.row_idx, (size_t)nnz, st);
    h2d(d_col, lp.col_idx, (size_t)nnz, st);
    h2d(d_val, lp.val, (size_t)nnz, st);
    h2d(d_rptr, rptr.data(), rptr.size(), st);
    h2d(d_rord, rord.data(), (size_t)nnz, st);
    h2d(d_cptr, cptr.data(), cptr.size(), st);
    h2d(d_cord, cord.data(), (size_t)nnz, st);
    auto grid = [](int64_t work) { return (int)std::max<int64_t>(1, std::min<int64_t>(148 * 16, (work + 255) / 256)); };
    if (m) dev::k_fill<<<grid(m), 256, 0, st>>>(m, 1.0, d_Dr);
    if (n) dev::k_fill<<<grid(n), 256, 0, st>>>(n, 1.0, d_Dc);
    for (int pass = 0; pass < ruiz_passes; ++pass) {
        if (m) dev::k_ruiz_factor<<<grid(m), 256, 0, st>>>(m, d_rptr, d_rord, d_val, d_fr, d_Dr);
        if (nnz) dev::k_scale_entries<<<grid(nnz), 256, 0, st>>>(nnz, d_row, d_fr, d_val);
        if (n) dev::k_ruiz_factor<<<grid(n), 256, 0, st>>>(n, d_cptr, d_cord, d_val, d_fc, d_Dc);
        if (nnz) dev::k_scale_entries<<<grid(nnz), 256, 0, st>>>(nnz, d_col, d_fc, d_val);
    }
    if (m) dev::k_pc_factor<<<grid(m), 256, 0, st>>>(m, d_rptr, d_rord, d_val, d_fr, d_Dr);
    if (n) dev::k_pc_factor<<<grid(n), 256, 0, st>>>(n, d_cptr, d_cord, d_val, d_fc, d_Dc);
    if (nnz) dev::k_scale_both<<<grid(nnz), 256, 0, st>>>(nnz, d_row, d_col, d_fr, d_fc, d_val);
    cuda_ok(cudaGetLastError(), "scaling kernels");
    d2h(val_s, d_val, (size_t)nnz, st);
    d2h(Dr, d_Dr, (size_t)m, st);
    d2h(Dc, d_Dc, (size_t)n, st);
    cuda_ok(cudaStreamSynchronize(st), "scaling");
    // bounds, costs and row sides as the host loop forms them
    for (int32_t j = 0; j < n; ++j) {
        c_s[j] = Dc[j] * lp.c[j];
        l_s[j] = lp.l[j] / Dc[j];
        u_s[j] = lp.u[j] / Dc[j];
    }
    for (int32_t i = 0; i < m; ++i) {
        rL_s[i] = Dr[i] * lp.rL[i];
        rU_s[i] = Dr[i] * lp.rU[i];
    }
}

}  // namespace b2
