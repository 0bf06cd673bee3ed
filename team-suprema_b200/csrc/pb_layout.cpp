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
//     of its source chunk by v (held in its shared memory) and writes the
//     products out in runs, one run per destination bin; each run is a
//     contiguous piece of the product buffer.
//   * phase 2 (consumer, the next pass): CTA k streams the products of each of
//     its bins (all runs of the bin are adjacent), places each at its slot in
//     shared memory, and sums every destination row's products in the order of
//     the row's CSR entries (ascending source index), then runs the row's
//     epilogue.
// Every byte moves in long coalesced runs; the summation order is fixed by the
// layout, so the result is the same bits on every run.
//
// Layout (all in the engine's device order of rows and columns):
//   product buffer : ordered by (bin t, source chunk p, CSR position q)
//   slot[pos]      : q - first CSR position of the bin (uint16)
//   producer list  : ordered by (source chunk p, bin t, q); loc = source index
//                    within its chunk (uint16), val = the entry's value (FP32)
//   run_start[p][t]: offset of run (p, t) in the producer list (T + 1 per p)
//   run_dest[p][t] : offset of run (p, t) in the product buffer
//   dst_ptr        : CSR offsets of the destination rows
#include <algorithm>
#include <cstdint>
#include <vector>

#include "internal.h"

namespace b2 {

namespace {

// Splits [0, len) into `parts` contiguous chunks of about equal weight
// (weight of index i: w[i] + 1), with no chunk above max_len indices.
std::vector<int32_t> balanced_split(const std::vector<int32_t>& w, int32_t parts, int32_t max_len) {
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

}  // namespace

bool build_pb(int32_t n_dst, int32_t n_src, const std::vector<int32_t>& dst, const std::vector<int32_t>& src,
              const std::vector<float>& val, int32_t n_chunks, int32_t bin_entries, PbHost& P) {
    const int64_t nnz = (int64_t)dst.size();
    if (n_chunks < 1 || nnz == 0 || nnz >= (int64_t)INT32_MAX || bin_entries > 65535) return false;
    P = PbHost();
    P.n_chunks = n_chunks;
    // destination CSR, entries in ascending source order inside a row
    std::vector<int32_t> dcnt(n_dst, 0), scnt(n_src, 0);
    for (int64_t e = 0; e < nnz; ++e) { dcnt[dst[e]]++; scnt[src[e]]++; }
    for (int32_t i = 0; i < n_dst; ++i)
        if (dcnt[i] > bin_entries) return false;  // a row must fit one bin
    P.dst_ptr.assign(n_dst + 1, 0);
    for (int32_t i = 0; i < n_dst; ++i) P.dst_ptr[i + 1] = P.dst_ptr[i] + dcnt[i];
    std::vector<int32_t> q_of(nnz);  // CSR position of entry e
    {
        // counting sort by source, then stable by destination: rows in ascending source order
        std::vector<int32_t> sp(n_src + 1, 0);
        for (int32_t j = 0; j < n_src; ++j) sp[j + 1] = sp[j] + scnt[j];
        std::vector<int32_t> by_src(nnz);
        for (int64_t e = 0; e < nnz; ++e) by_src[sp[src[e]]++] = (int32_t)e;
        std::vector<int32_t> cur(P.dst_ptr.begin(), P.dst_ptr.end() - 1);
        for (int32_t e : by_src) q_of[e] = cur[dst[e]]++;
    }
    // chunks: source and destination cut by entries, at most 65535 indices each
    P.src_start = balanced_split(scnt, n_chunks, 65535);
    P.dst_start = balanced_split(dcnt, n_chunks, 1 << 30);
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
    std::vector<int32_t> cnt(runs, 0);
    for (int32_t q = 0; q < (int32_t)nnz; ++q) {
        const int32_t e = e_at[q];
        cnt[(size_t)chunk_of[src[e]] * T + bin_of[dst[e]]]++;
    }
    // product buffer: by (t, p, q); run_dest[p][t]
    P.run_dest.assign(runs, 0);
    {
        int64_t off = 0;
        for (int32_t t = 0; t < T; ++t)
            for (int32_t p = 0; p < n_chunks; ++p) {
                P.run_dest[(size_t)p * T + t] = (int32_t)off;
                off += cnt[(size_t)p * T + t];
            }
    }
    // producer list: by (p, t, q); run_start[p][t]
    P.run_start.assign((size_t)n_chunks * (T + 1), 0);
    {
        int64_t off = 0;
        for (int32_t p = 0; p < n_chunks; ++p) {
            for (int32_t t = 0; t < T; ++t) {
                P.run_start[(size_t)p * (T + 1) + t] = (int32_t)off;
                off += cnt[(size_t)p * T + t];
            }
            P.run_start[(size_t)p * (T + 1) + T] = (int32_t)off;
        }
    }
    P.loc.resize(nnz);
    P.val.resize(nnz);
    P.slot.resize(nnz);
    std::vector<int32_t> fill(runs, 0);
    for (int32_t q = 0; q < (int32_t)nnz; ++q) {  // CSR order: q ascending inside every run
        const int32_t e = e_at[q];
        const int32_t p = chunk_of[src[e]], t = bin_of[dst[e]];
        const size_t r = (size_t)p * T + t;
        const int32_t k = fill[r]++;
        const int32_t at = P.run_start[(size_t)p * (T + 1) + t] + k;
        P.loc[at] = (uint16_t)(src[e] - P.src_start[p]);
        P.val[at] = val[e];
        P.slot[P.run_dest[r] + k] = (uint16_t)(q - P.dst_ptr[P.bin_first[t]]);
    }
    return true;
}

}  // namespace b2
