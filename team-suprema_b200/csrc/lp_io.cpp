// lp_io.cpp -- the binary LP request format (b2_lp_write / b2_lp_read*).
//
// The reference reads every LP from MPS text (src/mps_reader.cpp:66-308),
// which costs seconds for the large benchmark LPs; the served stream takes
// requests in this binary form instead (b2_server_submit_file), read on the
// server's preparation threads. Layout, little-endian, no padding:
//
//   char[8]  magic "B2LPCSR1"
//   int32    m, n
//   int64    nnz
//   double   obj_offset
//   int64    row_ptr[m + 1]        CSR of A: row_ptr[0] = 0, nondecreasing, row_ptr[m] = nnz
//   int32    col[nnz]              0 <= col < n
//   double   val[nnz]
//   double   c[n], l[n], u[n]
//   double   rL[m], rU[m]
//
// Reading checks the magic, the sizes against the file length, the row
// pointers and the column range, and reports a malformed file as
// B2_ERR_INVALID before anything else is done with it.
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "internal.h"

namespace b2 {
namespace {

constexpr char kMagic[8] = {'B', '2', 'L', 'P', 'C', 'S', 'R', '1'};

struct File {
    std::FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

void put(std::FILE* f, const void* p, size_t bytes, const std::string& path) {
    if (bytes && std::fwrite(p, 1, bytes, f) != bytes) fail(B2_ERR_INVALID, "write failed: " + path);
}

void get(std::FILE* f, void* p, size_t bytes, const std::string& path) {
    if (bytes && std::fread(p, 1, bytes, f) != bytes) fail(B2_ERR_INVALID, "truncated LP file: " + path);
}

}  // namespace

void lp_write(const std::string& path, const b2_lp_view& lp) {
    if (lp.m < 0 || lp.n < 0 || lp.nnz < 0) fail(B2_ERR_INVALID, "negative size");
    for (int64_t k = 0; k < lp.nnz; ++k)
        if (lp.row_idx[k] < 0 || lp.row_idx[k] >= lp.m || lp.col_idx[k] < 0 || lp.col_idx[k] >= lp.n)
            fail(B2_ERR_INVALID, "matrix index out of range at entry " + std::to_string(k));
    // CSR, entries of a row in COO order
    std::vector<int64_t> ptr((size_t)lp.m + 1, 0);
    for (int64_t k = 0; k < lp.nnz; ++k) ptr[lp.row_idx[k] + 1]++;
    for (int32_t i = 0; i < lp.m; ++i) ptr[i + 1] += ptr[i];
    std::vector<int32_t> col((size_t)lp.nnz);
    std::vector<double> val((size_t)lp.nnz);
    std::vector<int64_t> cur(ptr.begin(), ptr.end() - 1);
    for (int64_t k = 0; k < lp.nnz; ++k) {
        const int64_t p = cur[lp.row_idx[k]]++;
        col[p] = lp.col_idx[k];
        val[p] = lp.val[k];
    }
    File F;
    F.f = std::fopen(path.c_str(), "wb");
    if (!F.f) fail(B2_ERR_INVALID, "cannot open for writing: " + path);
    put(F.f, kMagic, 8, path);
    put(F.f, &lp.m, 4, path);
    put(F.f, &lp.n, 4, path);
    put(F.f, &lp.nnz, 8, path);
    put(F.f, &lp.obj_offset, 8, path);
    put(F.f, ptr.data(), ptr.size() * 8, path);
    put(F.f, col.data(), col.size() * 4, path);
    put(F.f, val.data(), val.size() * 8, path);
    put(F.f, lp.c, (size_t)lp.n * 8, path);
    put(F.f, lp.l, (size_t)lp.n * 8, path);
    put(F.f, lp.u, (size_t)lp.n * 8, path);
    put(F.f, lp.rL, (size_t)lp.m * 8, path);
    put(F.f, lp.rU, (size_t)lp.m * 8, path);
    if (std::fflush(F.f) != 0) fail(B2_ERR_INVALID, "write failed: " + path);
}

void lp_read_dims(const std::string& path, int32_t* m, int32_t* n, int64_t* nnz) {
    File F;
    F.f = std::fopen(path.c_str(), "rb");
    if (!F.f) fail(B2_ERR_INVALID, "cannot open: " + path);
    char magic[8];
    get(F.f, magic, 8, path);
    if (std::memcmp(magic, kMagic, 8) != 0) fail(B2_ERR_INVALID, "not a B2LPCSR1 file: " + path);
    int32_t mm = 0, nn = 0;
    int64_t zz = 0;
    get(F.f, &mm, 4, path);
    get(F.f, &nn, 4, path);
    get(F.f, &zz, 8, path);
    if (mm < 0 || nn < 0 || zz < 0) fail(B2_ERR_INVALID, "negative size in " + path);
    if (std::fseek(F.f, 0, SEEK_END) != 0) fail(B2_ERR_INVALID, "cannot seek: " + path);
    const long long len = std::ftell(F.f);
    const long long want = 32LL + 8LL * ((long long)mm + 1) + 12LL * zz + 24LL * nn + 16LL * mm;
    if (len != want)
        fail(B2_ERR_INVALID, "file length " + std::to_string(len) + " does not match its sizes (" + std::to_string(want) +
                                 "): " + path);
    *m = mm;
    *n = nn;
    *nnz = zz;
}

void lp_read(const std::string& path, LpArrays& out) {
    int32_t m = 0, n = 0;
    int64_t nnz = 0;
    lp_read_dims(path, &m, &n, &nnz);
    File F;
    F.f = std::fopen(path.c_str(), "rb");
    if (!F.f) fail(B2_ERR_INVALID, "cannot open: " + path);
    std::fseek(F.f, 24, SEEK_SET);
    out.m = m;
    out.n = n;
    get(F.f, &out.obj_offset, 8, path);
    std::vector<int64_t> ptr((size_t)m + 1);
    get(F.f, ptr.data(), ptr.size() * 8, path);
    if (ptr[0] != 0 || ptr[m] != nnz) fail(B2_ERR_INVALID, "row pointers do not span the entries: " + path);
    for (int32_t i = 0; i < m; ++i)
        if (ptr[i + 1] < ptr[i]) fail(B2_ERR_INVALID, "row pointers decrease at row " + std::to_string(i) + ": " + path);
    out.col.resize((size_t)nnz);
    out.val.resize((size_t)nnz);
    get(F.f, out.col.data(), (size_t)nnz * 4, path);
    get(F.f, out.val.data(), (size_t)nnz * 8, path);
    for (int64_t k = 0; k < nnz; ++k)
        if (out.col[k] < 0 || out.col[k] >= n) fail(B2_ERR_INVALID, "column index out of range at entry " + std::to_string(k));
    out.row.resize((size_t)nnz);
    for (int32_t i = 0; i < m; ++i)
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) out.row[p] = i;
    out.c.resize(n);
    out.l.resize(n);
    out.u.resize(n);
    out.rL.resize(m);
    out.rU.resize(m);
    get(F.f, out.c.data(), (size_t)n * 8, path);
    get(F.f, out.l.data(), (size_t)n * 8, path);
    get(F.f, out.u.data(), (size_t)n * 8, path);
    get(F.f, out.rL.data(), (size_t)m * 8, path);
    get(F.f, out.rU.data(), (size_t)m * 8, path);
}

}  // namespace b2
