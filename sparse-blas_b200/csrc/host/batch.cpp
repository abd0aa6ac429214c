// batch.cpp — batched SpMV (one persistent kernel per kernel family, run as
// parallel branches of the caller's stream or of one CUDA graph) and the
// per-matrix class timer the autotuner uses.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../sbb_internal.h"

using namespace sbb;

struct sbb_batch_s {
    std::vector<Plan *> plans;
    std::vector<BatchMat> host_mats;
    BatchMat *d_mats = nullptr;              // every matrix (the fix-up's view)
    // per kernel family: its matrices, unit offsets, unit count, grid, bytes
    BatchMat *d_fmats[kBatchFamilies] = {};
    long long *d_unit0[kBatchFamilies] = {};
    int fcount[kBatchFamilies] = {};
    long long total[kBatchFamilies] = {};
    int grid[kBatchFamilies] = {};
    double fbytes[kBatchFamilies] = {};
    unsigned long long *d_queue = nullptr;  // [f]: family f's next claim of kBatchClaim units
    unsigned *d_status = nullptr;
    cudaStream_t side[kBatchFamilies - 1] = {};  // branches for the other families
    cudaEvent_t ev_fork = nullptr, ev_join[kBatchFamilies - 1] = {};
    // carry fix-up of the merge/tiled-class matrices, empty rows of tiled ones
    BatchFix fix{};
    long long fix_slots = 0;
    long long *d_tile0 = nullptr;
    int *d_fix_mat = nullptr, *d_run_mat = nullptr, *d_run_first = nullptr, *d_run_len = nullptr;
    int *d_empty_row = nullptr, *d_empty_mat = nullptr;
    int device = 0;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

static void batch_free(sbb_batch_s *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->cap) cudaStreamDestroy(b->cap);
    for (int f = 0; f < kBatchFamilies - 1; f++) {
        if (b->side[f]) cudaStreamDestroy(b->side[f]);
        if (b->ev_join[f]) cudaEventDestroy(b->ev_join[f]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    void *ptrs[] = {b->d_mats,    b->d_queue,     b->d_status,    b->d_tile0,
                    b->d_fix_mat, b->d_run_mat,   b->d_run_first, b->d_run_len,
                    b->d_empty_row, b->d_empty_mat};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (int f = 0; f < kBatchFamilies; f++) {
        if (b->d_fmats[f]) cudaFree(b->d_fmats[f]);
        if (b->d_unit0[f]) cudaFree(b->d_unit0[f]);
    }
    for (Plan *p : b->plans) {
        plan_free(p);
        delete p;
    }
    delete b;
}

// Families with work, largest (by bytes) first.
static std::vector<int> active_families(const sbb_batch_s *b)
{
    std::vector<int> fams;
    for (int f = 0; f < kBatchFamilies; f++)
        if (b->total[f] > 0) fams.push_back(f);
    std::stable_sort(fams.begin(), fams.end(),
                     [&](int a, int c) { return b->fbytes[a] > b->fbytes[c]; });
    return fams;
}

// The largest family's kernel runs on s, the others on side branches forked
// from s and joined back before the fix-up (also inside a stream capture).
static int enqueue(sbb_batch_s *b, cudaStream_t s)
{
    SBB_CUDA(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned long long) * kBatchFamilies, s));
    const std::vector<int> fams = active_families(b);
    if (fams.size() > 1) SBB_CUDA(cudaEventRecord(b->ev_fork, s));
    for (size_t j = 0; j < fams.size(); j++) {
        const int f = fams[j];
        cudaStream_t st = j == 0 ? s : b->side[j - 1];
        if (j > 0) SBB_CUDA(cudaStreamWaitEvent(st, b->ev_fork, 0));
        launch_batch(f, b->d_fmats[f], b->fcount[f], b->d_unit0[f], b->total[f], b->d_queue + f,
                     b->d_status, b->grid[f], st);
        if (j > 0) SBB_CUDA(cudaEventRecord(b->ev_join[j - 1], st));
    }
    for (size_t j = 1; j < fams.size(); j++) SBB_CUDA(cudaStreamWaitEvent(s, b->ev_join[j - 1], 0));
    launch_batch_fixup(b->d_mats, b->fix, b->fix_slots, s);
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}

extern "C" {

// The y arrays must not overlap one another or any item's x (a matrix's
// kernels write its y while the others read their x); x arrays may be
// shared.  Sorted y ranges, then one search per x: O(count log count).
static bool batch_ranges_ok(const sbb_batch_item *items, int count)
{
    std::vector<std::pair<uintptr_t, uintptr_t>> ys;  // [start, end) of each y
    for (int i = 0; i < count; i++)
        if (items[i].y && items[i].m > 0) {
            const auto a = reinterpret_cast<uintptr_t>(items[i].y);
            ys.push_back({a, a + 8 * (size_t)items[i].m});
        }
    std::sort(ys.begin(), ys.end());
    for (size_t j = 1; j < ys.size(); j++)
        if (ys[j].first < ys[j - 1].second) {
            set_error("batch: two items' y arrays overlap");
            return false;
        }
    // the y ranges are now disjoint and sorted, so their ends are sorted too
    for (int i = 0; i < count; i++) {
        if (!items[i].x || items[i].n <= 0) continue;
        const auto a = reinterpret_cast<uintptr_t>(items[i].x);
        const uintptr_t e = a + 8 * (size_t)items[i].n;
        auto k = std::lower_bound(ys.begin(), ys.end(), a,
                                  [](const std::pair<uintptr_t, uintptr_t> &iv, uintptr_t v) {
                                      return iv.second <= v;
                                  });
        if (k != ys.end() && k->first < e) {
            set_error("batch: item " + std::to_string(i) + "'s x overlaps a y array");
            return false;
        }
    }
    return true;
}

int sbb_batch_create(sbb_batch_t *out, const sbb_batch_item *items, int count, void *stream)
{
    if (!out || count < 0 || (count > 0 && !items)) {
        set_error("bad sbb_batch_create arguments");
        return SBB_ERR_ARG;
    }
    *out = nullptr;
    if (!batch_ranges_ok(items, count)) return SBB_ERR_ARG;
    auto s = static_cast<cudaStream_t>(stream);
    auto *b = new sbb_batch_s();
    cudaGetDevice(&b->device);
    std::vector<BatchMat> fmats[kBatchFamilies];
    std::vector<long long> funit0[kBatchFamilies];
    for (auto &u : funit0) u.push_back(0);
    std::vector<long long> tile0(1, 0);
    std::vector<int> fix_mat, run_mat, run_first, run_len, empty_row, empty_mat;
    // copies cnt ints from the device; false (error set) on failure
    auto fetch = [&](std::vector<int> &h, const int *d, int cnt) {
        h.resize(cnt);
        if (cnt == 0) return true;
        if (cudaMemcpyAsync(h.data(), d, sizeof(int) * cnt, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            set_error("batch: copy of plan metadata failed");
            return false;
        }
        return true;
    };
    // carries of one merge/tiled matrix: its slots and multi-slot runs
    auto add_carries = [&](int i, int slots, const CarryRuns &R) {
        if (slots <= 0) return true;
        fix_mat.push_back(i);
        tile0.push_back(tile0.back() + slots);
        std::vector<int> f, l;
        if (!fetch(f, R.run_first, R.n_runs) || !fetch(l, R.run_len, R.n_runs)) return false;
        for (int r = 0; r < R.n_runs; r++) {
            run_mat.push_back(i);
            run_first.push_back(f[r]);
            run_len.push_back(l[r]);
        }
        return true;
    };
    for (int i = 0; i < count; i++) {
        const sbb_batch_item &it = items[i];
        if (it.cls < 0 || it.cls >= SBB_NUM_CLASSES || it.m < 0 || it.n < 0 || it.nnz < 0 ||
            !it.rowptr || (it.nnz > 0 && (!it.col || !it.val || !it.x)) || (it.m > 0 && !it.y)) {
            set_error("bad batch item " + std::to_string(i));
            batch_free(b);
            return SBB_ERR_ARG;
        }
        auto *p = new Plan();
        p->m = it.m;
        p->n = it.n;
        p->nnz = it.nnz;
        p->rowptr = it.rowptr;
        p->col = it.col;
        p->val = it.val;
        b->plans.push_back(p);
        sbb_config c = batch_class_config(it.cls);
        int rc = plan_build(p, &c, s);
        if (rc != SBB_OK) {
            cudaStreamSynchronize(s);
            batch_free(b);
            return rc;
        }
        BatchMat M{};
        M.rowptr = it.rowptr;
        M.col = it.col;
        M.val = it.val;
        M.x = it.x;
        M.y = it.y;
        M.m = it.m;
        M.n = it.n;
        M.cls = it.cls;
        M.alpha = it.alpha;
        M.beta = it.beta;
        M.nnz = it.nnz;
        long long units;
        if (it.cls == kBatchMergeClass) {
            M.tile_row = p->tile_row;
            M.tile_nnz = p->tile_nnz;
            M.crow = p->tile_row + 1;  // segment t carries into the row it ends in
            M.carry_val = p->carry_val;
            M.tiles = p->tiles;
            units = p->tiles;
            if (!add_carries(i, p->tiles, p->runs)) {
                batch_free(b);
                return SBB_ERR_CUDA;
            }
        } else if (it.cls == kBatchTiledClass) {
            TiledView v{};
            if (!tiled_view(p, &v) || v.sigma != kBatchSigma) {
                set_error("batch: tiled plan missing");
                batch_free(b);
                return SBB_ERR_CUDA;
            }
            M.blob = v.blob;
            M.tile_seg = v.tile_seg;
            M.ne = v.ne;
            M.crow = v.carry_row;
            M.carry_val = v.carry_val;
            M.tiles = v.tiles;
            units = (v.tiles + kBatchTileGroup - 1) / kBatchTileGroup;
            std::vector<int> e;
            if (!add_carries(i, v.tiles, *v.runs) || !fetch(e, v.empty, v.n_empty)) {
                batch_free(b);
                return SBB_ERR_CUDA;
            }
            for (int r : e) {
                empty_row.push_back(r);
                empty_mat.push_back(i);
            }
        } else {
            // units of about kBatchVectorNnz nnz: vsteps chunks of cr rows
            const long long cr = vector_chunk_rows(4 << it.cls, kBatchVectorU);
            const double mean = it.m > 0 ? (double)it.nnz / it.m : 1.0;
            long long steps = (long long)(kBatchVectorNnz / (cr * std::max(mean, 1.0)) + 0.5);
            steps = std::min<long long>(64, std::max<long long>(1, steps));
            M.vsteps = (int)steps;
            const long long rows_per_unit = cr * steps;
            units = (it.m + rows_per_unit - 1) / rows_per_unit;
        }
        b->host_mats.push_back(M);
        const int f = batch_family(it.cls);
        fmats[f].push_back(M);
        funit0[f].push_back(funit0[f].back() + units);
        b->fbytes[f] += 12.0 * it.nnz + 4.0 * (it.m + 1) + 8.0 * it.n + 16.0 * it.m;
    }
    for (int f = 0; f < kBatchFamilies; f++) {
        b->fcount[f] = (int)fmats[f].size();
        b->total[f] = funit0[f].back();
    }
    auto fail = [&](cudaError_t e) {
        set_error(std::string("batch setup: ") + cudaGetErrorString(e));
        batch_free(b);
        return SBB_ERR_CUDA;
    };
    cudaError_t e;
    const int nfix = (int)fix_mat.size(), nruns = (int)run_mat.size();
    // long runs first: the fix-up gives them whole blocks, short runs a warp
    int n_long_runs = 0;
    {
        std::vector<int> order(nruns);
        for (int i = 0; i < nruns; ++i) order[i] = i;
        std::stable_partition(order.begin(), order.end(),
                              [&](int i) { return run_len[i] > kWarpRunMax; });
        std::vector<int> rm(nruns), rf(nruns), rl(nruns);
        for (int i = 0; i < nruns; ++i) {
            rm[i] = run_mat[order[i]];
            rf[i] = run_first[order[i]];
            rl[i] = run_len[order[i]];
            n_long_runs += rl[i] > kWarpRunMax;
        }
        run_mat.swap(rm);
        run_first.swap(rf);
        run_len.swap(rl);
    }
    const int nempty = (int)empty_row.size();
    for (int f = 0; f < kBatchFamilies; f++) {
        const size_t nf = fmats[f].size();
        if ((e = cudaMalloc(&b->d_fmats[f], sizeof(BatchMat) * std::max<size_t>(nf, 1))) ||
            (e = cudaMalloc(&b->d_unit0[f], sizeof(long long) * (nf + 1))) ||
            (nf && (e = cudaMemcpyAsync(b->d_fmats[f], fmats[f].data(), sizeof(BatchMat) * nf,
                                        cudaMemcpyHostToDevice, s))) ||
            (e = cudaMemcpyAsync(b->d_unit0[f], funit0[f].data(), sizeof(long long) * (nf + 1),
                                 cudaMemcpyHostToDevice, s)))
            return fail(e);
    }
    for (int f = 0; f < kBatchFamilies - 1; f++)
        if ((e = cudaStreamCreateWithFlags(&b->side[f], cudaStreamNonBlocking)) ||
            (e = cudaEventCreateWithFlags(&b->ev_join[f], cudaEventDisableTiming)))
            return fail(e);
    if ((e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming)) ||
        (e = cudaMalloc(&b->d_mats, sizeof(BatchMat) * std::max(count, 1))) ||
        (e = cudaMalloc(&b->d_queue, sizeof(unsigned long long) * kBatchFamilies)) ||
        (e = cudaMalloc(&b->d_status, sizeof(unsigned))) ||
        (e = cudaMalloc(&b->d_tile0, sizeof(long long) * (nfix + 1))) ||
        (e = cudaMalloc(&b->d_fix_mat, sizeof(int) * std::max(nfix, 1))) ||
        (e = cudaMalloc(&b->d_run_mat, sizeof(int) * std::max(nruns, 1))) ||
        (e = cudaMalloc(&b->d_run_first, sizeof(int) * std::max(nruns, 1))) ||
        (e = cudaMalloc(&b->d_run_len, sizeof(int) * std::max(nruns, 1))) ||
        (e = cudaMalloc(&b->d_empty_row, sizeof(int) * std::max(nempty, 1))) ||
        (e = cudaMalloc(&b->d_empty_mat, sizeof(int) * std::max(nempty, 1))))
        return fail(e);
    auto up = [&](void *dst, const void *src, size_t bytes) {
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
    };
    if ((e = up(b->d_tile0, tile0.data(), sizeof(long long) * (nfix + 1))) ||
        (e = up(b->d_fix_mat, fix_mat.data(), sizeof(int) * nfix)) ||
        (e = up(b->d_run_mat, run_mat.data(), sizeof(int) * nruns)) ||
        (e = up(b->d_run_first, run_first.data(), sizeof(int) * nruns)) ||
        (e = up(b->d_run_len, run_len.data(), sizeof(int) * nruns)) ||
        (e = up(b->d_empty_row, empty_row.data(), sizeof(int) * nempty)) ||
        (e = up(b->d_empty_mat, empty_mat.data(), sizeof(int) * nempty)) ||
        (e = up(b->d_mats, b->host_mats.data(), sizeof(BatchMat) * count)) ||
        (e = cudaMemsetAsync(b->d_status, 0, sizeof(unsigned), s)) ||
        (e = cudaStreamSynchronize(s)))
        return fail(e);
    b->fix = BatchFix{b->d_tile0,   b->d_fix_mat, nfix,        b->d_run_mat,   b->d_run_first,
                      b->d_run_len, nruns,        n_long_runs, b->d_empty_row, b->d_empty_mat,
                      nempty};
    b->fix_slots = tile0.back();
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    for (int f = 0; f < kBatchFamilies; f++)
        b->grid[f] = sms * std::max(batch_max_ctas_per_sm(f), 1);
    *out = b;
    return SBB_OK;
}

int sbb_batch_run(sbb_batch_t b, void *stream)
{
    if (!b) return SBB_ERR_ARG;
    return enqueue(b, static_cast<cudaStream_t>(stream));
}

int sbb_batch_run_graph(sbb_batch_t b, void *stream)
{
    if (!b) return SBB_ERR_ARG;
    if (!b->exec) {
        // capture on a private stream (the caller's may be the legacy default
        // stream, which cannot be captured), replay on the caller's
        if (!b->cap) SBB_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
        SBB_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue(b, b->cap);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->cap, &g);
        if (rc != SBB_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) {
            set_error(std::string("graph capture: ") + cudaGetErrorString(e));
            return SBB_ERR_CUDA;
        }
        b->graph = g;
        SBB_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    SBB_CUDA(cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)));
    return SBB_OK;
}

int sbb_batch_run_each(sbb_batch_t b, void *stream)
{
    if (!b) return SBB_ERR_ARG;
    auto s = static_cast<cudaStream_t>(stream);
    for (size_t i = 0; i < b->plans.size(); i++) {
        const BatchMat &M = b->host_mats[i];
        int rc = plan_run(b->plans[i], M.alpha, M.x, M.beta, M.y, s);
        if (rc != SBB_OK) return rc;
    }
    return SBB_OK;
}

int sbb_batch_launches(sbb_batch_t b, int per_matrix)
{
    if (!b) return 0;
    if (!per_matrix)
        return (int)active_families(b).size() + (b->fix_slots > 0 || b->fix.n_empty > 0 ? 1 : 0);
    int n = 0;
    for (Plan *p : b->plans) n += plan_launches(p);
    return n;
}

int sbb_batch_check(sbb_batch_t b)
{
    if (!b) return SBB_ERR_ARG;
    unsigned st = 0;
    SBB_CUDA(cudaMemcpy(&st, b->d_status, sizeof(st), cudaMemcpyDeviceToHost));
    for (Plan *p : b->plans) {
        unsigned q = 0;
        SBB_CUDA(cudaMemcpy(&q, p->status, sizeof(q), cudaMemcpyDeviceToHost));
        st |= q;
    }
    if (st) {
        set_error("batch: device status " + std::to_string(st) +
                  ((st & ST_TIMEOUT) ? " (a bounded wait on a tile copy gave up)" : ""));
        return SBB_ERR_INPUT;
    }
    return SBB_OK;
}

int sbb_batch_destroy(sbb_batch_t b)
{
    if (!b) return SBB_OK;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    batch_free(b);
    return SBB_OK;
}

int sbb_tune_classes(int m, int n, int nnz, const int *d_rowptr, const int *d_col,
                     const double *d_val, const double *d_x, double *d_y, double alpha,
                     double beta, int reps, float *ms, void *stream)
{
    if (!ms || reps <= 0 || m < 0 || n < 0 || nnz < 0 || !d_rowptr) {
        set_error("bad sbb_tune_classes arguments");
        return SBB_ERR_ARG;
    }
    auto s = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    SBB_CUDA(cudaEventCreate(&e0));
    SBB_CUDA(cudaEventCreate(&e1));
    int rc = SBB_OK;
    for (int cls = 0; cls < SBB_NUM_CLASSES && rc == SBB_OK; cls++) {
        Plan p;
        p.m = m;
        p.n = n;
        p.nnz = nnz;
        p.rowptr = d_rowptr;
        p.col = d_col;
        p.val = d_val;
        sbb_config c = batch_class_config(cls);
        rc = plan_build(&p, &c, s);
        if (rc == SBB_OK) rc = plan_run(&p, alpha, d_x, beta, d_y, s);  // warm-up
        if (rc == SBB_OK) {
            cudaEventRecord(e0, s);
            for (int r = 0; r < reps && rc == SBB_OK; r++) rc = plan_run(&p, alpha, d_x, beta, d_y, s);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            ms[cls] = t / reps;
        }
        cudaStreamSynchronize(s);
        plan_free(&p);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

}  // extern "C"
