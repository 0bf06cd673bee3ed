// pb_layout.cpp -- host side of the two-phase ("propagation-blocking")
// products of the whole-GPU engine: y = M v where every access is a
// coalesced stream instead of a random gather.
//
// A product of an R x C matrix M with a vector v is split between the CTAs of
// the cooperative launch: CTA k owns a chunk of the source dimension (the
// entries of v it produces) and a chunk of the destination dimension (the
// entries of y it finishes), and the destination chunk is cut into bins whose
// entries fit the CTA's shared memory.
//   * phase 1 (producer, the pass that computes v): CTA k multiplies each entry
//     of its source chunk by v (held in its shared memory) and writes each
//     product to its place in the product buffer; the chunk's entries are
//     stored in the order of those places, so consecutive threads write
//     consecutive places except where a destination bin ends.
//   * phase 2 (consumer, the next pass): CTA k streams the products of each of
//     its bins (a contiguous piece of the buffer), places each at its slot in
//     shared memory, and sums every destination row's products in the order of
//     the row's CSR entries (the order the entries were given in, as the
//     reference's CSR builders fill rows), then runs the row's epilogue.
// Every byte moves in coalesced streams; the summation order is fixed by the
// layout, so the result is the same bits on every run.
//
// Layout (all in the engine's device order of rows and columns):
//   product buffer : ordered by (bin t, source chunk p, CSR position q)
//   slot[pos]      : q - first CSR position of the bin (uint16)
//   producer list  : ordered by (source chunk p, bin t, q); src_first[p] its
//                    start; loc = source index within the chunk (uint16),
//                    val = the entry's value (FP32), dest = its place in the
//                    product buffer (int32)
//   dst_ptr        : CSR offsets of the destination rows
#include <algorithm>
#include <cstdint>
#include <vector>

#include "internal.h"

namespace b2 {

std::vector<int32_t> pb_split(const std::vector<int32_t>& w, int32_t parts, int32_t max_len) {
    const int32_t len = (int32_t)w.size();
    int64_t total = 0;
    for (int32_t v : w) total += v + 1;
    std::vector<int32_t> b(parts + 1, len);
    b[0] = 0;
    int64_t acc = 0;
    int32_t k = 1;
    for (int32_t i = 0; i < len && k < parts; ++i) {
        acc += w[i] + 1;
        if (acc * parts >= total * k || i + 1 - b[k - 1] >= max_len) b[k++] = i + 1;
    }
    for (; k < parts; ++k) b[k] = len;
    return b;
}

bool build_pb(int32_t n_dst, int32_t n_src, const std::vector<int32_t>& dst, const std::vector<int32_t>& src,
              const std::vector<float>& val, const std::vector<int32_t>& src_start,
              const std::vector<int32_t>& dst_start, int32_t bin_entries, PbHost& P) {
    const int64_t nnz = (int64_t)dst.size();
    const int32_t n_chunks = (int32_t)src_start.size() - 1;
    if (n_chunks < 1 || (int32_t)dst_start.size() != n_chunks + 1 || nnz == 0 || nnz >= (int64_t)INT32_MAX ||
        bin_entries > 65535)
        return false;
    P = PbHost();
    P.n_chunks = n_chunks;
    // destination CSR offsets
    std::vector<int32_t> dcnt(n_dst, 0);
    for (int64_t e = 0; e < nnz; ++e) dcnt[dst[e]]++;
    for (int32_t i = 0; i < n_dst; ++i)
        if (dcnt[i] > bin_entries) return false;  // a row must fit one bin
    P.dst_ptr.assign(n_dst + 1, 0);
    for (int32_t i = 0; i < n_dst; ++i) P.dst_ptr[i + 1] = P.dst_ptr[i] + dcnt[i];
    std::vector<int32_t> q_of(nnz);  // CSR position of entry e
    {
        // stable in the order the entries are given, as the reference's
        // to_csr / to_csc_as_transposed_csr fill (include/sparse.hpp:24-50)
        std::vector<int32_t> cur(P.dst_ptr.begin(), P.dst_ptr.end() - 1);
        for (int64_t e = 0; e < nnz; ++e) q_of[e] = cur[dst[e]]++;
    }
    P.src_start = src_start;
    P.dst_start = dst_start;
    // bins inside each destination chunk
    P.dst_bin.assign(n_chunks + 1, 0);
    for (int32_t k = 0; k < n_chunks; ++k) {
        P.dst_bin[k] = (int32_t)P.bin_first.size();
        int32_t i = P.dst_start[k];
        while (i < P.dst_start[k + 1]) {
            P.bin_first.push_back(i);
            int32_t ent = 0;
            while (i < P.dst_start[k + 1] && ent + dcnt[i] <= bin_entries) ent += dcnt[i++];
        }
    }
    P.dst_bin[n_chunks] = (int32_t)P.bin_first.size();
    P.bin_first.push_back(n_dst);
    const int32_t T = (int32_t)P.bin_first.size() - 1;
    P.n_bins = T;
    std::vector<int32_t> bin_of(n_dst), chunk_of(n_src);
    for (int32_t t = 0; t < T; ++t)
        for (int32_t i = P.bin_first[t]; i < P.bin_first[t + 1]; ++i) bin_of[i] = t;
    for (int32_t k = 0; k < n_chunks; ++k)
        for (int32_t j = P.src_start[k]; j < P.src_start[k + 1]; ++j) chunk_of[j] = k;
    for (int32_t k = 0; k < n_chunks; ++k) {
        P.max_src_chunk = std::max(P.max_src_chunk, P.src_start[k + 1] - P.src_start[k]);
        P.max_dst_chunk = std::max(P.max_dst_chunk, P.dst_start[k + 1] - P.dst_start[k]);
    }
    for (int32_t t = 0; t < T; ++t)
        P.max_bin_entries = std::max(P.max_bin_entries, P.dst_ptr[P.bin_first[t + 1]] - P.dst_ptr[P.bin_first[t]]);
    if (P.max_src_chunk > 65535) return false;  // local source indices are 16-bit
    // entries in CSR order
    std::vector<int32_t> e_at(nnz);
    for (int64_t e = 0; e < nnz; ++e) e_at[q_of[e]] = (int32_t)e;
    // run sizes (p, t)
    const size_t runs = (size_t)n_chunks * T;
    std::vector<int64_t> cnt(runs, 0);
    for (int32_t q = 0; q < (int32_t)nnz; ++q) {
        const int32_t e = e_at[q];
        cnt[(size_t)chunk_of[src[e]] * T + bin_of[dst[e]]]++;
    }
    // product buffer by (t, p, q): place of run (p, t); producer list by (p, t, q): start of run (p, t)
    std::vector<int64_t> run_place(runs, 0), run_first(runs, 0);
    {
        int64_t off = 0;
        for (int32_t t = 0; t < T; ++t)
            for (int32_t p = 0; p < n_chunks; ++p) {
                run_place[(size_t)p * T + t] = off;
                off += cnt[(size_t)p * T + t];
            }
        off = 0;
        P.src_first.assign(n_chunks + 1, 0);
        for (int32_t p = 0; p < n_chunks; ++p) {
            P.src_first[p] = (int32_t)off;
            for (int32_t t = 0; t < T; ++t) {
                run_first[(size_t)p * T + t] = off;
                off += cnt[(size_t)p * T + t];
            }
        }
        P.src_first[n_chunks] = (int32_t)off;
    }
    P.loc.resize(nnz);
    P.val.resize(nnz);
    P.dest.resize(nnz);
    P.slot.resize(nnz);
    std::vector<int64_t> fill(runs, 0);
    for (int32_t q = 0; q < (int32_t)nnz; ++q) {  // CSR order: q ascending inside every run
        const int32_t e = e_at[q];
        const int32_t p = chunk_of[src[e]], t = bin_of[dst[e]];
        const size_t r = (size_t)p * T + t;
        const int64_t k = fill[r]++;
        const int64_t at = run_first[r] + k, place = run_place[r] + k;
        P.loc[at] = (uint16_t)(src[e] - P.src_start[p]);
        P.val[at] = val[e];
        P.dest[at] = (int32_t)place;
        P.slot[place] = (uint16_t)(q - P.dst_ptr[P.bin_first[t]]);
    }
    return true;
}

// y = M x through the two-phase layout on the host, phase by phase as the
// device runs it (products placed by dest, bins summed from their slots in
// CSR order): the check of the layout that needs no GPU.
void pb_spmv_host(const PbHost& P, int32_t n_dst, const double* x, double* y) {
    std::vector<double> prod(P.dest.size());
    for (int32_t k = 0; k < P.n_chunks; ++k)
        for (int32_t i = P.src_first[k]; i < P.src_first[k + 1]; ++i)
            prod[P.dest[i]] = (double)P.val[i] * x[P.src_start[k] + P.loc[i]];
    std::vector<double> bin((size_t)std::max(P.max_bin_entries, 1));
    for (int32_t t = 0; t < P.n_bins; ++t) {
        const int32_t r0 = P.bin_first[t], r1 = P.bin_first[t + 1];
        const int32_t s = P.dst_ptr[r0], e = P.dst_ptr[r1];
        for (int32_t q = s; q < e; ++q) bin[P.slot[q]] = prod[q];
        for (int32_t i = r0; i < r1; ++i) {
            double acc = 0.0;
            for (int32_t z = P.dst_ptr[i] - s; z < P.dst_ptr[i + 1] - s; ++z) acc += bin[z];
            y[i] = acc;
        }
    }
    (void)n_dst;
}

}  // namespace b2
