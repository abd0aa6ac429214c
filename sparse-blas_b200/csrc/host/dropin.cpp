// dropin.cpp — the reference's host-pointer entry points on one B200.
//
// spMV_mgpu_baseline / _v1 / _v2 keep the reference's contract bit for bit
// where it is observable: the partition (which rows and nnz each GPU/task
// covers, SparseBLAS/src/dspmv_mgpu_v1.cu:60-94, src/dspmv_mgpu_v2.cu:228-267,
// src/dspmv_mgpu_baseline.cu:60-87), which rows are written back, and the
// host fix-up of split rows (v1.cu:232-245, v2.cu:381-437).  The GPU count is
// pinned to 1, so there is one part (baseline, v1) or ceil(nnz/nb) tasks (v2).
//
// Device work per call:
//   rows covered by the partition are computed in one launch with their
//   natural extents; the few "special" rows (a split row, or a row whose
//   slice extent differs from its CSR extent because the bisection landed on
//   an empty row) get their slice sums from a small pieces kernel and are
//   merged on the host in the reference's order.  Rows the partition does not
//   cover keep their input y, as in the reference.
#include <cuda_runtime.h>
#include <sys/time.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "../sbb_internal.h"
#include "entry.h"

namespace sbb {

int plan_build_unchecked(Plan *p, const sbb_config *cfg, cudaStream_t s);
void plan_free_async(Plan *p, cudaStream_t s);

// Same bisection as src/spmv_helper.cu:16-39 (the partition must match the
// reference exactly, including which row of a run of empty rows it returns).
int row_from_index(int n, const long long *a, long long idx)
{
    int lo = 0, hi = n;
    while (lo < hi - 1) {
        int mid = lo + (hi - lo) / 2;
        if (idx < a[mid])
            hi = mid;
        else if (idx > a[mid])
            lo = mid;
        else
            return mid;
    }
    if (a[lo] == idx) return lo;
    if (a[hi] == idx) return hi;
    return lo;
}

namespace {

struct Slice {
    long long start_idx, end_idx;
    int start_row, end_row;
    bool start_flag, end_flag;
    double y2;
};

// v1 split, P parts (v1.cu:60-94): quotient in double, floor.
std::vector<Slice> v1_slices(int m, long long nnz, const long long *rp, const double *y, int P)
{
    std::vector<Slice> s(P);
    for (int i = 0; i < P; i++) {
        s[i].start_idx = (long long)std::floor((double)((long long)i * nnz) / P);
        s[i].end_idx = (long long)std::floor((double)((long long)(i + 1) * nnz) / P) - 1;
        s[i].start_row = row_from_index(m, rp, s[i].start_idx);
        s[i].start_flag = s[i].start_idx > rp[s[i].start_row];
        s[i].y2 = s[i].start_flag ? y[s[i].start_row] : 0.0;
        s[i].end_row = row_from_index(m, rp, s[i].end_idx);
        s[i].end_flag = s[i].end_idx < rp[s[i].end_row + 1] - 1;
    }
    return s;
}

// Baseline split (baseline.cu:60-87): even rows, nothing split.
std::vector<Slice> baseline_slices(int m, const long long *rp, int P)
{
    std::vector<Slice> s(P);
    for (int d = 0; d < P; d++) {
        s[d].start_row = d * m / P;
        s[d].end_row = (d + 1) * m / P - 1;
        s[d].start_idx = rp[s[d].start_row];
        s[d].end_idx = rp[s[d].end_row + 1] - 1;
        s[d].start_flag = s[d].end_flag = false;
        s[d].y2 = 0.0;
    }
    return s;
}

// v2 task table (v2.cu:218-273): integer quotient; y2 saved for a split
// start row and overwritten for a split end row.
std::vector<Slice> v2_slices(int m, long long nnz, const long long *rp, const double *y,
                             long long nb)
{
    int T = (int)((nnz + nb - 1) / nb);
    std::vector<Slice> s(T);
    for (int t = 0; t < T; t++) {
        s[t].start_idx = ((long long)t * nnz) / T;
        s[t].end_idx = ((long long)(t + 1) * nnz) / T - 1;
        s[t].y2 = 0.0;
    }
    for (int t = 0; t < T; t++) {
        s[t].start_row = row_from_index(m, rp, s[t].start_idx);
        s[t].start_flag = s[t].start_idx > rp[s[t].start_row];
        if (s[t].start_flag) s[t].y2 = y[s[t].start_row];
    }
    for (int t = 0; t < T; t++) {
        s[t].end_row = row_from_index(m, rp, s[t].end_idx);
        s[t].end_flag = s[t].end_idx < rp[s[t].end_row + 1] - 1;
        if (s[t].end_flag) s[t].y2 = y[s[t].end_row];
    }
    return s;
}

struct Piece {
    int row;
    long long lo, hi;
};

enum class Merge { V1, V2, NONE };

// Per-thread state of the drop-in calls: two streams per device and a few
// pinned status words, released when the thread ends (so callers that start
// a thread per call do not accumulate streams or pinned pages).
// Wall-clock marks of the calling thread's current host-pointer call; the
// phases between them are published when the call completes
// (sbb_last_call_phases).
struct CallTrace {
    std::chrono::steady_clock::time_point mark[SBB_TRACE_PHASES + 1];
    double ms[SBB_TRACE_PHASES] = {};
    int done = 0;  // phases of the last completed call
};
thread_local CallTrace g_trace;

void trace_mark(int k)
{
    g_trace.mark[k] = std::chrono::steady_clock::now();
    if (k == SBB_TRACE_PHASES) {
        for (int i = 0; i < SBB_TRACE_PHASES; ++i)
            g_trace.ms[i] =
                std::chrono::duration<double, std::milli>(g_trace.mark[i + 1] - g_trace.mark[i])
                    .count();
        g_trace.done = SBB_TRACE_PHASES;
    }
}

struct ThreadState {
    cudaStream_t s[2][64] = {};
    bool pool_set[64] = {};
    unsigned *words = nullptr;
    ~ThreadState()
    {
        for (auto &row : s)
            for (cudaStream_t st : row)
                if (st) cudaStreamDestroy(st);
        if (words) cudaFreeHost(words);
    }
};
ThreadState &thread_state()
{
    static thread_local ThreadState t;
    return t;
}

// Per-thread stream; device memory comes from the device's default pool,
// which keeps freed blocks for the next call.
cudaStream_t call_stream(int dev, int which = 0)
{
    ThreadState &t = thread_state();
    if (dev < 0 || dev >= 64) return 0;
    if (!t.pool_set[dev]) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            unsigned long long keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        t.pool_set[dev] = true;
    }
    if (!t.s[which][dev] &&
        cudaStreamCreateWithFlags(&t.s[which][dev], cudaStreamNonBlocking) != cudaSuccess)
        t.s[which][dev] = nullptr;
    return t.s[which][dev];
}

// A few pinned words per thread, so the status read-back is truly
// asynchronous and the large copies queued after it overlap the check.
unsigned *pinned_words()
{
    ThreadState &t = thread_state();
    if (!t.words && cudaMallocHost(reinterpret_cast<void **>(&t.words), 64) != cudaSuccess)
        t.words = nullptr;
    return t.words;
}

struct Buffers {
    cudaStream_t s;
    std::vector<void *> ptrs;
    bool ok = true;
    explicit Buffers(cudaStream_t st) : s(st) {}
    template <typename T>
    T *get(size_t count)
    {
        void *p = nullptr;
        if (dev_malloc_async(&p, std::max<size_t>(count, 1) * sizeof(T), s) != cudaSuccess) {
            ok = false;
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
    ~Buffers()
    {
        for (void *p : ptrs) cudaFreeAsync(p, s);
        cudaStreamSynchronize(s);
    }
};

double csrmv_value(double alpha, double sum, double beta, double y0)
{
    return beta == 0.0 ? alpha * sum : alpha * sum + beta * y0;
}

// The whole call.  Returns the reference's codes: 0, -1 (bad input, not
// enough memory, device error), 1 (allocation failure).
int run(int m, int n, long long nnz, double alpha, const double *val, const long long *rp,
        const int *col, const double *x, double beta, double *y, std::vector<Slice> &sl,
        Merge merge, int kernel, int q, long long queue_nnz = 0)
{
    // Slices that cover at least one row, and the hull of covered rows.
    int hr0 = INT_MAX, hr1 = -1;
    for (auto &t : sl)
        if (t.end_row >= t.start_row) {
            hr0 = std::min(hr0, t.start_row);
            hr1 = std::max(hr1, t.end_row);
        }
    if (hr1 < 0) return 0;  // nothing covered (e.g. nnz == 0 with a tie)
    trace_mark(0);

    // Special rows: slice extent != CSR extent, or split.
    std::vector<Piece> pieces;
    std::vector<int> first_piece(sl.size(), -1), last_piece(sl.size(), -1);
    std::vector<std::pair<int, int>> spans;  // covered row ranges [start_row, end_row]
    for (size_t t = 0; t < sl.size(); t++) {
        Slice &s = sl[t];
        int dev_m = s.end_row - s.start_row + 1;
        if (dev_m <= 0) continue;
        spans.push_back({s.start_row, s.end_row});
        long long lo = s.start_idx;
        long long hi = dev_m == 1 ? s.end_idx + 1 : rp[s.start_row + 1];
        if (s.start_flag || (dev_m == 1 && s.end_flag) || lo != rp[s.start_row] ||
            hi != rp[s.start_row + 1]) {
            first_piece[t] = (int)pieces.size();
            pieces.push_back({s.start_row, lo, hi});
        }
        if (dev_m >= 2) {
            lo = rp[s.end_row];
            hi = s.end_idx + 1;
            if (s.end_flag || hi != rp[s.end_row + 1]) {
                last_piece[t] = (int)pieces.size();
                pieces.push_back({s.end_row, lo, hi});
            }
        }
    }

    // Input y of every row the host will rewrite after the copy back: the
    // rows of the hull in the gaps between covered ranges (found from the
    // sorted ranges, not row by row), and the special rows.
    std::vector<std::pair<int, double>> saved;
    std::sort(spans.begin(), spans.end());
    int next = hr0;  // first row not yet known to be covered
    for (auto &sp : spans) {
        for (int r = next; r < sp.first; r++) saved.push_back({r, y[r]});
        next = std::max(next, sp.second + 1);
    }
    for (auto &p : pieces) saved.push_back({p.row, y[p.row]});

    // Memory pre-check as the reference does (0.8 x free memory, v1.cu:106-116).
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return -1;
    free_b = capped_free_bytes(free_b);
    const int hm = hr1 - hr0 + 1;
    double need = (double)nnz * 12.0 + ((double)m + 1.0) * 12.0 + (double)n * 8.0 + (double)hm * 8.0 +
                  (double)((long long)hm + nnz) / 256.0 * 24.0;
    if (need / 1e9 > 0.8 * ((double)free_b / 1e9)) return -1;

    int dev = 0;
    cudaGetDevice(&dev);
    cudaStream_t s = call_stream(dev);
    if (!s) return 1;  // library failure (no stream), as the reference's malloc failures
    Buffers B(s);
    long long *d_rp64 = B.get<long long>((size_t)m + 1);
    int *d_rp = B.get<int>((size_t)m + 1);
    int *d_col = B.get<int>((size_t)nnz);
    double *d_val = B.get<double>((size_t)nnz);
    double *d_x = B.get<double>((size_t)n);
    double *d_y = B.get<double>((size_t)hm);
    unsigned *d_st = B.get<unsigned>(4);
    if (!B.ok) return 1;
    cudaEvent_t ev;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return 1;

    bool cuda_ok = true;
    auto ck = [&](cudaError_t e) { cuda_ok = cuda_ok && e == cudaSuccess; };
    // Large calls run in kChunks nnz-balanced row chunks of the hull: chunk
    // k's kernels (on a second stream) and its y copy back overlap the
    // host-to-device copy of chunk k+1's columns and values.  Every row lies
    // in one chunk.
    const long long hnnz = rp[hr1 + 1] - rp[hr0];
    const int kChunks = hnnz >= (8LL << 20) && hm >= 4 * 1024 ? 4 : 1;
    std::vector<int> cr(kChunks + 1);  // chunk k: hull rows [cr[k], cr[k+1])
    cr[0] = hr0;
    cr[kChunks] = hr1 + 1;
    for (int k = 1; k < kChunks; k++) {
        const long long target = rp[hr0] + hnnz * k / kChunks;
        // first row whose nnz start at or after the target
        int r = (int)(std::lower_bound(rp + cr[k - 1], rp + hr1 + 1, target) - rp);
        cr[k] = std::min(std::max(r, cr[k - 1]), hr1 + 1);
    }
    cudaStream_t s2 = kChunks > 1 ? call_stream(dev, 1) : s;
    if (!s2) {
        cudaEventDestroy(ev);
        return 1;
    }
    std::vector<cudaEvent_t> ev_copy(kChunks, nullptr);
    cudaEvent_t ev_done = nullptr;
    auto destroy_events = [&]() {
        for (auto &e : ev_copy)
            if (e) cudaEventDestroy(e);
        if (ev_done) cudaEventDestroy(ev_done);
    };
    for (auto &e : ev_copy) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ck(cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
    if (!cuda_ok) {
        destroy_events();
        cudaEventDestroy(ev);
        return 1;
    }
    ck(cudaMemsetAsync(d_st, 0, 4 * sizeof(unsigned), s));
    ck(cudaMemcpyAsync(d_rp64, rp, sizeof(long long) * ((size_t)m + 1), cudaMemcpyHostToDevice, s));
    launch_rowptr_narrow(d_rp64, d_rp, m, nnz, d_st, s);
    unsigned *h_pin = pinned_words();
    if (!h_pin) {
        destroy_events();
        cudaEventDestroy(ev);
        return 1;
    }
    h_pin[0] = 0;
    ck(cudaMemcpyAsync(h_pin, d_st, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    ck(cudaEventRecord(ev, s));
    // The big copies queue behind the check and run while the host waits on it.
    ck(cudaMemcpyAsync(d_x, x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    for (int k = 0; k < kChunks; k++) {
        const long long lo = k == 0 ? 0 : rp[cr[k]], hi = k + 1 == kChunks ? nnz : rp[cr[k + 1]];
        ck(cudaMemcpyAsync(d_col + lo, col + lo, sizeof(int) * (hi - lo), cudaMemcpyHostToDevice, s));
        ck(cudaMemcpyAsync(d_val + lo, val + lo, sizeof(double) * (hi - lo), cudaMemcpyHostToDevice,
                           s));
        if (beta != 0.0 && cr[k + 1] > cr[k])
            ck(cudaMemcpyAsync(d_y + (cr[k] - hr0), y + cr[k], sizeof(double) * (cr[k + 1] - cr[k]),
                               cudaMemcpyHostToDevice, s));
        ck(cudaEventRecord(ev_copy[k], s));
    }
    trace_mark(1);
    ck(cudaEventSynchronize(ev));
    trace_mark(2);
    cudaEventDestroy(ev);
    const unsigned h_st = h_pin[0];
    if (!cuda_ok || (h_st & ST_BAD_ROWPTR)) {
        cudaStreamSynchronize(s);
        destroy_events();
        set_error(cuda_ok ? "row pointer is not monotone within [0, nnz]" : "CUDA copy failed");
        return -1;
    }

    // Natural-extent compute, chunk by chunk.
    std::vector<Plan> plans(kChunks);
    int rc = SBB_OK;
    unsigned *pst = h_pin + 1;  // pinned: the status reads stay asynchronous
    for (int k = 0; k <= kChunks; k++) pst[k] = 0;
    for (int k = 0; k < kChunks && rc == SBB_OK; k++) {
        if (cr[k + 1] <= cr[k]) continue;
        ck(cudaStreamWaitEvent(s2, ev_copy[k], 0));
        Plan &p = plans[k];
        p.m = cr[k + 1] - cr[k];
        p.n = n;
        p.nnz = (int)(rp[cr[k + 1]] - rp[cr[k]]);
        p.base = (int)rp[cr[k]];
        p.rowptr = d_rp + cr[k];
        p.col = d_col;
        p.val = d_val;
        p.status = nullptr;
        p.queue_nnz = queue_nnz;
        p.device_runs = true;  // no host synchronisation while the copies stream in
        sbb_config cfg{};
        cfg.kernel = kernel;
        cfg.persistent = q;
        rc = plan_build_unchecked(&p, &cfg, s2);
        if (rc == SBB_OK) rc = plan_run(&p, alpha, d_x, beta, d_y + (cr[k] - hr0), s2);
        if (rc == SBB_OK && kChunks > 1)  // this chunk's y goes back while the next computes
            ck(cudaMemcpyAsync(y + cr[k], d_y + (cr[k] - hr0), sizeof(double) * p.m,
                               cudaMemcpyDeviceToHost, s2));
        if (rc == SBB_OK && p.status)
            ck(cudaMemcpyAsync(&pst[k], p.status, sizeof(unsigned), cudaMemcpyDeviceToHost, s2));
    }
    if (rc != SBB_OK) {
        cudaStreamSynchronize(s2);
        cudaStreamSynchronize(s);
        for (auto &p : plans) plan_free_async(&p, s2);
        cudaStreamSynchronize(s2);
        destroy_events();
        return rc == SBB_ERR_NOMEM ? 1 : -1;
    }

    // Boundary pieces (after every chunk's copy: they read any columns).
    std::vector<double> psum(pieces.size(), 0.0);
    if (!pieces.empty()) {
        std::vector<long long> plo(pieces.size()), phi(pieces.size());
        for (size_t i = 0; i < pieces.size(); i++) {
            plo[i] = pieces[i].lo;
            phi[i] = pieces[i].hi;
        }
        long long *d_plo = B.get<long long>(pieces.size());
        long long *d_phi = B.get<long long>(pieces.size());
        double *d_ps = B.get<double>(pieces.size());
        if (!B.ok) {
            cudaStreamSynchronize(s2);
            for (auto &p : plans) plan_free_async(&p, s2);
            cudaStreamSynchronize(s2);
            destroy_events();
            return 1;
        }
        ck(cudaMemcpyAsync(d_plo, plo.data(), sizeof(long long) * plo.size(),
                           cudaMemcpyHostToDevice, s));
        ck(cudaMemcpyAsync(d_phi, phi.data(), sizeof(long long) * phi.size(),
                           cudaMemcpyHostToDevice, s));
        launch_pieces(d_plo, d_phi, (int)pieces.size(), d_col, d_val, d_x, n, d_ps, d_st, s);
        ck(cudaMemcpyAsync(psum.data(), d_ps, sizeof(double) * psum.size(),
                           cudaMemcpyDeviceToHost, s));
    }
    if (kChunks == 1)
        ck(cudaMemcpyAsync(y + hr0, d_y, sizeof(double) * hm, cudaMemcpyDeviceToHost, s2));
    ck(cudaMemcpyAsync(pst + kChunks, d_st, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    ck(cudaEventRecord(ev_done, s2));
    ck(cudaStreamWaitEvent(s, ev_done, 0));  // the frees below follow every chunk
    trace_mark(3);
    ck(cudaStreamSynchronize(s));
    trace_mark(4);
    ck(cudaGetLastError());
    for (auto &p : plans) plan_free_async(&p, s);
    destroy_events();
    if (!cuda_ok) return -1;
    // Restore the rows the reference never writes, and the special rows'
    // inputs for the merge.  This comes before the status check, so a call
    // that fails on bad column indices still leaves every row outside the
    // slices with its input value (the covered rows then hold partial sums).
    for (auto &sv : saved) y[sv.first] = sv.second;
    unsigned st2 = 0;
    for (int k = 0; k <= kChunks; k++) st2 |= pst[k];
    if (st2) {
        set_error("column index out of range (or corrupt tile)");
        return -1;
    }
    std::vector<double> y0(pieces.size());
    for (size_t i = 0; i < pieces.size(); i++) y0[i] = y[pieces[i].row];

    if (merge == Merge::V2) {
        // Pop order (back of the pool first) and the gather of v2.cu:381-437.
        std::vector<char> seen(hm, 0);
        for (int t = (int)sl.size() - 1; t >= 0; t--) {
            Slice &S = sl[t];
            int dev_m = S.end_row - S.start_row + 1;
            double first = 0, last = 0;
            if (first_piece[t] >= 0)
                first = csrmv_value(alpha, psum[first_piece[t]], beta, y0[first_piece[t]]);
            if (last_piece[t] >= 0)
                last = csrmv_value(alpha, psum[last_piece[t]], beta, y0[last_piece[t]]);
            auto fix = [&](int row, double &v) {
                char &f = seen[row - hr0];
                if (!f) {
                    f = 1;
                } else {
                    double cur = y[row];
                    v += cur;
                    v -= beta * S.y2;
                }
            };
            if (dev_m == 1 && S.start_flag && S.end_flag) {
                fix(S.start_row, first);
            } else {
                if (S.start_flag) fix(S.start_row, first);
                if (S.end_flag) {
                    if (dev_m == 1)
                        fix(S.end_row, first);
                    else
                        fix(S.end_row, last);
                }
            }
            if (first_piece[t] >= 0) y[S.start_row] = first;
            if (last_piece[t] >= 0) y[S.end_row] = last;
        }
    } else {
        // v1 / baseline: parts in order; a split start row adds the value
        // already written for it and removes the double-counted beta*y2.
        for (size_t t = 0; t < sl.size(); t++) {
            Slice &S = sl[t];
            if (S.end_row < S.start_row) continue;
            double prev = S.start_flag ? y[S.start_row] : 0.0;
            if (first_piece[t] >= 0)
                y[S.start_row] = csrmv_value(alpha, psum[first_piece[t]], beta, y0[first_piece[t]]);
            if (last_piece[t] >= 0)
                y[S.end_row] = csrmv_value(alpha, psum[last_piece[t]], beta, y0[last_piece[t]]);
            if (S.start_flag) {
                y[S.start_row] += prev;
                y[S.start_row] -= S.y2 * beta;
            }
        }
    }
    trace_mark(SBB_TRACE_PHASES);
    return 0;
}

bool basic_args_ok(int m, int n, long long nnz, const double *alpha, const double *val,
                   const long long *rp, const int *col, const double *x, const double *beta,
                   const double *y)
{
    if (m < 0 || n < 0 || nnz < 0 || nnz > INT_MAX || !alpha || !beta || !rp) return false;
    if (nnz > 0 && (!val || !col || !x)) return false;
    if (m > 0 && !y) return false;
    if (rp[0] != 0 || rp[m] != nnz) return false;
    return true;
}

}  // namespace

int dropin_baseline(int m, int n, long long nnz, double *alpha, double *val, long long *rp,
                    int *col, double *x, double *beta, double *y, int ngpu)
{
    if (ngpu <= 0 || !basic_args_ok(m, n, nnz, alpha, val, rp, col, x, beta, y)) return -1;
    if (m == 0) return 0;
    // one GPU: the calling thread's current device (device 0 unless the
    // caller selected another), as the reference with ngpu = 1 uses device 0
    auto sl = baseline_slices(m, rp, 1);
    // cusparseDcsrmv picks its own algorithm; the analogue here is the
    // automatic choice (vector CSR for even rows, merge path otherwise).
    return run(m, n, nnz, *alpha, val, rp, col, x, *beta, y, sl, Merge::NONE, SBB_KERNEL_AUTO, 0);
}

int dropin_v1(int m, int n, long long nnz, double *alpha, double *val, long long *rp, int *col,
              double *x, double *beta, double *y, int ngpu, int kernel)
{
    if (ngpu <= 0 || kernel < 1 || kernel > 3 ||
        !basic_args_ok(m, n, nnz, alpha, val, rp, col, x, beta, y))
        return -1;
    // With nnz == 0 the bisection gives rows [mid, 0]: row 0 alone for m == 1,
    // nothing for m >= 2 (the reference aborts for m >= 4, where dev_m < 0).
    if (m == 0) return 0;
    // one GPU: the calling thread's current device (device 0 unless the
    // caller selected another), as the reference with ngpu = 1 uses device 0
    auto sl = v1_slices(m, nnz, rp, y, 1);
    return run(m, n, nnz, *alpha, val, rp, col, x, *beta, y, sl, Merge::V1, kernel, 0);
}

int dropin_v2(int m, int n, long long nnz, double *alpha, double *val, long long *rp, int *col,
              double *x, double *beta, double *y, int ngpu, int kernel, long long nb, int q)
{
    if (ngpu <= 0 || q <= 0 || nb <= 0 || kernel < 1 || kernel > 3 ||
        !basic_args_ok(m, n, nnz, alpha, val, rp, col, x, beta, y))
        return -1;
    // one GPU: the calling thread's current device (device 0 unless the
    // caller selected another), as the reference with ngpu = 1 uses device 0
    // nb clamp of v2.cu:43: 0.8 x free memory / 16 B per nnz / q.
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return -1;
    free_b = capped_free_bytes(free_b);
    long long cap = (long long)(0.8 * ((double)free_b / 1e9) * 1e9 / 16.0) / q;
    nb = std::min(nb, cap);
    if (nb <= 0) return -1;
    if (m == 0 || nnz == 0) return 0;
    auto sl = v2_slices(m, nnz, rp, y, nb);
    // The task pool becomes the merge kernel's device work queue: q resident
    // CTAs per SM claim items of nb nnz (see merge_queue_item for the cap).
    return run(m, n, nnz, *alpha, val, rp, col, x, *beta, y, sl, Merge::V2,
               kernel == 2 ? SBB_KERNEL_MERGE : kernel, kernel == 2 ? q : 0, nb);
}

}  // namespace sbb

// ------------------------------------------------------------- C ABI
extern "C" {

int sbb_last_call_phases(double *ms, int n)
{
    const sbb::CallTrace &t = sbb::g_trace;
    const int k = ms && n > 0 ? std::min(n, t.done) : 0;
    for (int i = 0; i < k; ++i) ms[i] = t.ms[i];
    return k;
}

int spMV_mgpu_baseline(int m, int n, long long nnz, double *alpha, double *csrVal,
                       long long *csrRowPtr, int *csrColIndex, double *x, double *beta,
                       double *y, int ngpu)
{
    return sbb::dropin_baseline(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y,
                                ngpu);
}

int spMV_mgpu_v1(int m, int n, long long nnz, double *alpha, double *csrVal,
                 long long *csrRowPtr, int *csrColIndex, double *x, double *beta, double *y,
                 int ngpu, int kernel)
{
    return sbb::dropin_v1(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y, ngpu,
                          kernel);
}

int spMV_mgpu_v2(int m, int n, long long nnz, double *alpha, double *csrVal,
                 long long *csrRowPtr, int *csrColIndex, double *x, double *beta, double *y,
                 int ngpu, int kernel, long long nb, int q)
{
    return sbb::dropin_v2(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y, ngpu,
                          kernel, nb, q);
}

int get_row_from_index(int n, long long *a, long long idx)
{
    return sbb::row_from_index(n, a, idx);
}

double get_time(void) { return sbb::wall_time(); }
double get_gpu_availble_mem(int ngpu) { return sbb::min_free_gb(ngpu); }
int csr5_kernel(int m, int n, int nnz, double *alpha, double *csrVal, int *csrRowPtr,
                int *csrColIndex, double *x, double *beta, double *y)
{
    return sbb::csr5_entry(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y);
}

}  // extern "C"

namespace sbb {

double wall_time()
{
    struct timeval tp;
    gettimeofday(&tp, nullptr);
    return (double)tp.tv_sec + (double)tp.tv_usec * 1e-6;
}

double min_free_gb(int ngpu)
{
    int count = 0, prev = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return 0.0;
    cudaGetDevice(&prev);
    double best = std::numeric_limits<double>::max();
    int upto = std::min(std::max(ngpu, 1), count);
    for (int d = 0; d < upto; d++) {
        size_t f = 0, t = 0;
        cudaSetDevice(d);
        if (cudaMemGetInfo(&f, &t) == cudaSuccess) best = std::min(best, (double)f / 1e9);
    }
    cudaSetDevice(prev);
    return best;
}

int csr5_entry(int m, int n, int nnz, double *alpha, double *csrVal, int *csrRowPtr,
               int *csrColIndex, double *x, double *beta, double *y)
{
    if (!alpha || !beta) return -1;
    sbb_config cfg{};
    cfg.kernel = SBB_KERNEL_TILED;
    sbb_plan_t plan = nullptr;
    if (sbb_plan_create(&plan, m, n, nnz, csrRowPtr, csrColIndex, csrVal, &cfg, nullptr) != SBB_OK)
        return -1;
    int rc = sbb_spmv(plan, *alpha, x, *beta, y, nullptr);
    if (rc == SBB_OK) rc = sbb_plan_check(plan);
    sbb_plan_destroy(plan);
    return rc == SBB_OK ? 0 : -1;
}

}  // namespace sbb
