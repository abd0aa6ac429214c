// mmio.cpp — Matrix Market reader: coordinate files to canonical CSR.
//
// The reference reads Matrix Market files with the NIST mmio routines
// (SparseBLAS/include/mmio.h, test/dspmv_test.cu:101-136) and then passes the
// COO arrays, in file order, to the drivers as if they were CSR arrays
// (dspmv_test.cu:228-251, 305-306): correct only for files whose entries are
// already sorted by row.  Symmetric files are used as stored (one triangle).
// This reader returns canonical CSR whatever the entry order:
//   * formats: coordinate; fields real / double / integer / pattern (complex
//     and the dense "array" format are rejected with an error);
//   * symmetry: general, symmetric (the mirror of every off-diagonal entry is
//     added), skew-symmetric (the mirror is negated); hermitian is complex-only
//     and rejected;
//   * rows sorted, columns sorted within a row, duplicate (row, col) entries
//     summed in file order; pattern entries get `pattern_value`;
//   * 1-based indices checked against the size line; every malformed line is
//     an error naming the line number.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../sbb_internal.h"

namespace {

struct MMData {
    int m = 0, n = 0;
    std::vector<long long> rowptr;
    std::vector<int> col;
    std::vector<double> val;
};

std::string lower(std::string s)
{
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// Parses the whole file; returns an error message or "" on success.
std::string parse(const char *path, double pattern_value, MMData &out)
{
    FILE *f = std::fopen(path, "rb");
    if (!f) return std::string("cannot open ") + path + ": " + std::strerror(errno);
    std::string buf;
    {
        char chunk[1 << 16];
        size_t k;
        while ((k = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.append(chunk, k);
        std::fclose(f);
    }
    const char *p = buf.c_str(), *end = p + buf.size();
    long long line = 0;
    auto next_line = [&](const char *&b, const char *&e) {
        if (p >= end) return false;
        b = p;
        const char *nl = static_cast<const char *>(std::memchr(p, '\n', end - p));
        e = nl ? nl : end;
        p = nl ? nl + 1 : end;
        ++line;
        return true;
    };
    const char *b, *e;
    // banner
    if (!next_line(b, e)) return "empty file";
    {
        char w[5][64] = {};
        std::string first(b, e);
        if (std::sscanf(first.c_str(), "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]) != 5 ||
            std::string(w[0]) != "%%MatrixMarket")
            return "line 1: not a Matrix Market banner";
        const std::string obj = lower(w[1]), fmt = lower(w[2]), field = lower(w[3]),
                          sym = lower(w[4]);
        if (obj != "matrix") return "line 1: object '" + obj + "' is not supported (matrix only)";
        if (fmt != "coordinate")
            return "line 1: format '" + fmt + "' is not supported (coordinate only)";
        if (field != "real" && field != "double" && field != "integer" && field != "pattern")
            return "line 1: field '" + field + "' is not supported (real, integer, pattern)";
        if (sym != "general" && sym != "symmetric" && sym != "skew-symmetric")
            return "line 1: symmetry '" + sym + "' is not supported (general, symmetric, "
                   "skew-symmetric)";
        const bool pattern = field == "pattern";
        const int mirror = sym == "general" ? 0 : (sym == "symmetric" ? 1 : -1);
        // size line (after comments and blank lines)
        long long M = -1, N = -1, L = -1;
        while (next_line(b, e)) {
            const char *q = b;
            while (q < e && (*q == ' ' || *q == '\t' || *q == '\r')) ++q;
            if (q == e || *q == '%') continue;
            std::string s(b, e);
            if (std::sscanf(s.c_str(), "%lld %lld %lld", &M, &N, &L) != 3)
                return "line " + std::to_string(line) + ": expected 'rows cols entries'";
            break;
        }
        if (M < 0 || N < 0 || L < 0) return "missing size line";
        if (M > 2147483647LL - 1 || N > 2147483647LL)
            return "matrix dimensions exceed the int32 row/column index range";
        // entries
        std::vector<int> ri, ci;
        std::vector<double> vv;
        const long long cap = L * (mirror ? 2 : 1);
        ri.reserve(cap);
        ci.reserve(cap);
        vv.reserve(cap);
        long long got = 0;
        while (got < L && next_line(b, e)) {
            const char *q = b;
            while (q < e && (*q == ' ' || *q == '\t' || *q == '\r')) ++q;
            if (q == e || *q == '%') continue;
            char *t;
            const long long i = std::strtoll(q, &t, 10);
            if (t == q) return "line " + std::to_string(line) + ": bad row index";
            q = t;
            const long long j = std::strtoll(q, &t, 10);
            if (t == q) return "line " + std::to_string(line) + ": bad column index";
            q = t;
            double v = pattern_value;
            if (!pattern) {
                v = std::strtod(q, &t);
                if (t == q) return "line " + std::to_string(line) + ": bad value";
            }
            if (i < 1 || i > M || j < 1 || j > N)
                return "line " + std::to_string(line) + ": entry (" + std::to_string(i) + ", " +
                       std::to_string(j) + ") outside " + std::to_string(M) + " x " +
                       std::to_string(N);
            ri.push_back((int)(i - 1));
            ci.push_back((int)(j - 1));
            vv.push_back(v);
            if (mirror && i != j) {
                ri.push_back((int)(j - 1));
                ci.push_back((int)(i - 1));
                vv.push_back(mirror > 0 ? v : -v);
            }
            ++got;
        }
        if (got < L)
            return "file ends after " + std::to_string(got) + " of " + std::to_string(L) +
                   " entries";
        // COO -> canonical CSR: stable counting sort by row, then by column
        // within each row, duplicates summed in file order
        const long long K = (long long)ri.size();
        std::vector<long long> start(M + 1, 0);
        for (long long k = 0; k < K; k++) start[ri[k] + 1]++;
        for (long long r = 0; r < M; r++) start[r + 1] += start[r];
        std::vector<long long> order(K);
        {
            std::vector<long long> fill(start.begin(), start.end() - 1);
            for (long long k = 0; k < K; k++) order[fill[ri[k]]++] = k;
        }
        out.m = (int)M;
        out.n = (int)N;
        out.rowptr.assign(M + 1, 0);
        out.col.clear();
        out.val.clear();
        out.col.reserve(K);
        out.val.reserve(K);
        for (long long r = 0; r < M; r++) {
            auto first = order.begin() + start[r], last = order.begin() + start[r + 1];
            std::stable_sort(first, last, [&](long long a, long long c) { return ci[a] < ci[c]; });
            for (auto it = first; it != last; ++it) {
                if (!out.col.empty() && (long long)out.col.size() > out.rowptr[r] &&
                    out.col.back() == ci[*it])
                    out.val.back() += vv[*it];
                else {
                    out.col.push_back(ci[*it]);
                    out.val.push_back(vv[*it]);
                }
            }
            out.rowptr[r + 1] = (long long)out.col.size();
        }
    }
    return "";
}

}  // namespace

extern "C" {

// Loads a Matrix Market coordinate file; *handle receives the CSR matrix
// (free with sbb_mm_free), *m, *n, *nnz its shape and stored entries.
int sbb_mm_load(const char *path, double pattern_value, void **handle, int *m, int *n,
                long long *nnz)
{
    if (!path || !handle || !m || !n || !nnz) {
        sbb::set_error("bad sbb_mm_load arguments");
        return SBB_ERR_ARG;
    }
    *handle = nullptr;
    auto *d = new MMData();
    std::string err;
    try {
        err = parse(path, pattern_value, *d);
    } catch (const std::bad_alloc &) {
        err = "out of host memory";
    }
    if (!err.empty()) {
        delete d;
        sbb::set_error(std::string(path) + ": " + err);
        return SBB_ERR_INPUT;
    }
    *handle = d;
    *m = d->m;
    *n = d->n;
    *nnz = (long long)d->col.size();
    return SBB_OK;
}

// Copies the loaded CSR arrays (m+1 row offsets, nnz columns, nnz values).
int sbb_mm_copy(void *handle, long long *rowptr, int *col, double *val)
{
    auto *d = static_cast<MMData *>(handle);
    if (!d || !rowptr || (!d->col.empty() && (!col || !val))) {
        sbb::set_error("bad sbb_mm_copy arguments");
        return SBB_ERR_ARG;
    }
    std::memcpy(rowptr, d->rowptr.data(), sizeof(long long) * d->rowptr.size());
    if (!d->col.empty()) {
        std::memcpy(col, d->col.data(), sizeof(int) * d->col.size());
        std::memcpy(val, d->val.data(), sizeof(double) * d->val.size());
    }
    return SBB_OK;
}

void sbb_mm_free(void *handle) { delete static_cast<MMData *>(handle); }

}  // extern "C"
