// plan.cpp — device API: plans over device-resident CSR matrices.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <string>

#include "../sbb_internal.h"

namespace sbb {

static thread_local std::string g_error;
void set_error(const std::string &msg) { g_error = msg; }

TimingHooks &timing_hooks()
{
    static thread_local TimingHooks h;
    return h;
}

int plan_launches(const Plan *p)
{
    if (p->m == 0) return 0;
    switch (p->kernel) {
    case SBB_KERNEL_VECTOR: return 1;
    case SBB_KERNEL_MERGE: return p->tiles > 0 ? 2 : 0;
    case SBB_KERNEL_TILED: {
        extern int tiled_launches(const Plan *);
        return tiled_launches(p);
    }
    case SBB_KERNEL_ROWS: {
        extern int rows_launches(const Plan *);
        return rows_launches(p);
    }
    default: return 0;
    }
}

void launch_rowptr_check(const int *rp, int m, int nnz, unsigned *status, cudaStream_t s);

// Default (heuristic) kernel choice, the method without the learned selector:
// vector CSR when rows are short and even, 32x4 tiles otherwise (the fastest
// tile shape measured on the irregular benchmark matrices).
int default_kernel_choice(int m, int nnz, int max_row, int *vector_width, int *ipt, int *sigma)
{
    double mean = m > 0 ? (double)nnz / m : 0.0;
    int v = 2;
    while (v < 32 && v < mean) v <<= 1;
    *vector_width = v;
    *ipt = 6;
    *sigma = 4;
    if (m > 0 && max_row <= 4 * v && max_row <= 128) return SBB_KERNEL_VECTOR;
    return m > kTiledMaxRows ? SBB_KERNEL_MERGE : SBB_KERNEL_TILED;
}

sbb_config batch_class_config(int cls)
{
    sbb_config c{};
    if (cls == kBatchMergeClass) {
        c.kernel = SBB_KERNEL_MERGE;
        c.items_per_thread = kBatchIpt;
    } else if (cls == kBatchTiledClass) {
        c.kernel = SBB_KERNEL_TILED;
        c.tile_sigma = kBatchSigma;
    } else {
        c.kernel = SBB_KERNEL_VECTOR;
        c.vector_width = 4 << cls;
    }
    return c;
}

#include "mlp_params.inc"  // kLearnedParams: generated from the trained parameters

// The built-in selector parameters on device `dev` (copied once per device).
static const float *learned_params(int dev)
{
    static std::mutex mu;
    static float *ptr[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64) return nullptr;
    if (!ptr[dev]) {
        float *p = nullptr;
        if (cudaMalloc(&p, sizeof(kLearnedParams)) != cudaSuccess) return nullptr;
        if (cudaMemcpy(p, kLearnedParams, sizeof(kLearnedParams), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
            cudaFree(p);
            return nullptr;
        }
        ptr[dev] = p;
    }
    return ptr[dev];
}

static int sm_count(int dev)
{
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}

template <typename T>
static int dalloc(T **p, size_t count, cudaStream_t s, size_t *acc)
{
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = dev_malloc_async(reinterpret_cast<void **>(p), bytes, s);
    if (e != cudaSuccess) {
        *p = nullptr;
        set_error(std::string("device allocation failed: ") + cudaGetErrorString(e));
        return SBB_ERR_NOMEM;
    }
    *acc += bytes;
    return SBB_OK;
}

void plan_free_async(Plan *p, cudaStream_t s)
{
    void *ptrs[] = {p->tile_row, p->tile_nnz, p->carry_val, p->queue, p->status};
    for (void *q : ptrs)
        if (q) cudaFreeAsync(q, s);
    carry_runs_free(&p->runs, s, true);
    extern void tiled_free_async(Plan *, cudaStream_t);
    tiled_free_async(p, s);
    extern void rows_free_async(Plan *, cudaStream_t);
    rows_free_async(p, s);
    p->tile_row = p->tile_nnz = nullptr;
    p->carry_val = nullptr;
    p->queue = p->status = nullptr;
}

void plan_free(Plan *p)
{
    void *ptrs[] = {p->tile_row, p->tile_nnz, p->carry_val, p->queue, p->status};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    carry_runs_free(&p->runs, 0, false);
    extern void tiled_free(Plan *);
    tiled_free(p);
    extern void rows_free(Plan *);
    rows_free(p);
    p->tile_row = p->tile_nnz = nullptr;
    p->carry_val = nullptr;
    p->queue = p->status = nullptr;
}

extern int tiled_build(Plan *p, cudaStream_t s);
extern int tiled_run(Plan *p, double alpha, const void *x, double beta, double *y,
                     cudaStream_t s);
extern int rows_build(Plan *p, cudaStream_t s);
extern int rows_run(Plan *p, double alpha, const void *x, double beta, double *y,
                    cudaStream_t s);

// Build scratch for the resolved kernel.  Validation (one sync) only when
// `validate`; the drop-in validates while narrowing the row pointer instead.
static int plan_build_impl(Plan *p, const sbb_config *cfg, cudaStream_t s, bool validate)
{
    cudaGetDevice(&p->device);
    int rc;
    if ((rc = dalloc(&p->status, 4, s, &p->scratch_bytes))) return rc;
    SBB_CUDA(cudaMemsetAsync(p->status, 0, 4 * sizeof(unsigned), s));
    int *stats = reinterpret_cast<int *>(p->status + 2);
    bool want_stats = validate && (cfg == nullptr || cfg->kernel == SBB_KERNEL_AUTO);
    if (validate) {
        launch_rowptr_check(p->rowptr, p->m, p->nnz, p->status, s);
        if (want_stats) launch_row_stats(p->rowptr, p->m, stats, s);
        unsigned h[4];
        SBB_CUDA(cudaMemcpyAsync(h, p->status, sizeof(h), cudaMemcpyDeviceToHost, s));
        SBB_CUDA(cudaStreamSynchronize(s));
        if (h[0] & ST_BAD_ROWPTR) {
            set_error("row pointer is not monotone within [0, nnz] with rowptr[0] == 0 and "
                      "rowptr[m] == nnz");
            return SBB_ERR_INPUT;
        }
        p->max_row = (int)h[2];
        p->empty_rows = (int)h[3];
        SBB_CUDA(cudaMemsetAsync(p->status, 0, 4 * sizeof(unsigned), s));
    }
    sbb_config c{};
    if (cfg) c = *cfg;
    if (c.kernel == SBB_KERNEL_LEARNED) {
        // the row pointer was validated above, so the feature pass stays in range
        if (!validate) {
            set_error("SBB_KERNEL_LEARNED needs a validated plan");
            return SBB_ERR_ARG;
        }
        const float *params = learned_params(p->device);
        if (!params) {
            set_error("selector parameters: device copy failed");
            return SBB_ERR_CUDA;
        }
        int cls = -1;
        int rc2 = sbb_mlp_select(params, p->m, p->n, p->nnz, p->rowptr, p->col, &cls, s);
        if (rc2 != SBB_OK) return rc2;
        if (cls < 0 || cls >= SBB_NUM_CLASSES) {
            set_error("selector returned no class");
            return SBB_ERR_CUDA;
        }
        c = batch_class_config(cls);
        if (c.kernel == SBB_KERNEL_TILED && p->m > kTiledMaxRows)
            c = batch_class_config(kBatchMergeClass);
    }
    int vw = 0, ipt = 0, sigma = 0;
    int k = c.kernel;
    if (k == SBB_KERNEL_AUTO) {
        k = default_kernel_choice(p->m, p->nnz, want_stats ? p->max_row : INT_MAX, &vw, &ipt, &sigma);
        // FP32 storage: 32 x 8 tiles, which measured fastest for that form
        // (0.130 ms vs 0.166 ms for 32 x 4 on the 5.5M-row matrix)
        if (p->f32) sigma = 8;
    } else {
        default_kernel_choice(p->m, p->nnz, INT_MAX, &vw, &ipt, &sigma);
        sigma = 0;  // an explicit tiled request without a sigma uses the CSR5 rule
    }
    if (c.vector_width) vw = c.vector_width;
    if (c.items_per_thread) ipt = c.items_per_thread;
    if (c.tile_sigma) sigma = c.tile_sigma;
    if (p->lane32) {
        // FP32 lane sums exist in the tiled kernel only, for runs of at most
        // 8 products per lane (the error bound of the form)
        if (c.kernel == SBB_KERNEL_AUTO) k = SBB_KERNEL_TILED;
        if (!c.tile_sigma) sigma = 8;
        if (k != SBB_KERNEL_TILED || (sigma != 4 && sigma != 8) || p->m > kTiledMaxRows) {
            set_error("FP32 lane sums need the tiled kernel with tile_sigma 4 or 8 "
                      "(and at most 2^31 - 1025 rows)");
            return SBB_ERR_ARG;
        }
    }
    p->kernel = k;
    p->vector_width = vw;
    p->ipt = ipt;
    p->persistent = c.persistent;
    p->tile_sigma = sigma;
    if (k == SBB_KERNEL_VECTOR) {
        if (vw != 2 && vw != 4 && vw != 8 && vw != 16 && vw != 32) {
            set_error("vector_width must be 2, 4, 8, 16 or 32");
            return SBB_ERR_ARG;
        }
        return SBB_OK;
    }
    if (k == SBB_KERNEL_MERGE) {
        if (!merge_ipt_supported(ipt)) {
            set_error("items_per_thread must be 4, 6, 8 or 12");
            return SBB_ERR_ARG;
        }
        long long items = merge_items_per_tile(ipt);
        long long total = (long long)p->m + p->nnz;
        long long tiles = (total + items - 1) / items;
        if (tiles > INT_MAX - 1) {
            set_error("matrix too large for one merge-path plan");
            return SBB_ERR_ARG;
        }
        p->tiles = (int)tiles;
        if ((rc = dalloc(&p->tile_row, tiles + 1, s, &p->scratch_bytes))) return rc;
        if ((rc = dalloc(&p->tile_nnz, tiles + 1, s, &p->scratch_bytes))) return rc;
        if ((rc = dalloc(&p->carry_val, tiles, s, &p->scratch_bytes))) return rc;
        if ((rc = dalloc(&p->queue, 2, s, &p->scratch_bytes))) return rc;
        SBB_CUDA(cudaMemsetAsync(p->queue, 0, 2 * sizeof(unsigned), s));
        if (tiles > 0) {
            launch_merge_partition(p->rowptr, p->m, p->base, p->nnz, items, p->tiles, p->tile_row,
                                   p->tile_nnz, s);
            rc = p->device_runs
                     ? carry_runs_build_device(p->tile_row + 1, p->tiles, p->m, &p->runs, s)
                     : carry_runs_build(p->tile_row + 1, p->tiles, p->m, &p->runs, s);
            if (rc) return rc;
            p->scratch_bytes += p->runs.bytes;
        }
        if (p->persistent > 0) {
            int occ = merge_max_ctas_per_sm(ipt, p->f32);
            int per_sm = std::min(p->persistent, std::max(occ, 1));
            p->persistent_ctas = per_sm * sm_count(p->device);  // CTAs of kMergeThreads
        }
        SBB_CUDA(cudaGetLastError());
        return SBB_OK;
    }
    if (k == SBB_KERNEL_TILED) {
        rc = tiled_build(p, s);
        if (rc != SBB_OK) return rc;
        SBB_CUDA(cudaGetLastError());
        if (validate) {  // the tile copy range-checked every column
            unsigned st = 0;
            SBB_CUDA(cudaMemcpyAsync(&st, p->status, sizeof(st), cudaMemcpyDeviceToHost, s));
            SBB_CUDA(cudaStreamSynchronize(s));
            if (st & ST_BAD_COL) {
                set_error("column index out of range [0, n)");
                return SBB_ERR_INPUT;
            }
        }
        return SBB_OK;
    }
    if (k == SBB_KERNEL_ROWS) {
        rc = rows_build(p, s);
        if (rc != SBB_OK) return rc;
        SBB_CUDA(cudaGetLastError());
        if (validate) {  // the plan range-checked every column
            unsigned st = 0;
            SBB_CUDA(cudaMemcpyAsync(&st, p->status, sizeof(st), cudaMemcpyDeviceToHost, s));
            SBB_CUDA(cudaStreamSynchronize(s));
            if (st & ST_BAD_COL) {
                set_error("column index out of range [0, n)");
                return SBB_ERR_INPUT;
            }
        }
        return SBB_OK;
    }
    set_error("unknown kernel id");
    return SBB_ERR_ARG;
}

int plan_build(Plan *p, const sbb_config *cfg, cudaStream_t s)
{
    return plan_build_impl(p, cfg, s, true);
}

int plan_build_unchecked(Plan *p, const sbb_config *cfg, cudaStream_t s)
{
    return plan_build_impl(p, cfg, s, false);
}

// Segments a warp of the persistent merge form claims from the work queue at
// a time: queue_nnz rounded up to whole segments (one segment when unset),
// but at most a quarter of the segments per warp of the grid, so that every
// warp still claims several items (an item as large as a reference task,
// nnz / 8 for example, would leave most of the GPU idle).
int merge_queue_item(const Plan &p)
{
    const long long seg = 32LL * p.ipt;
    long long item = p.queue_nnz > 0 ? (p.queue_nnz + seg - 1) / seg : 1;
    const long long warps = (long long)p.persistent_ctas * (kMergeThreads / 32);
    const long long cap = warps > 0 ? p.tiles / (4 * warps) : 1;
    item = std::min(item, std::max(cap, 1LL));
    return (int)std::max(item, 1LL);
}

int plan_run(Plan *p, double alpha, const void *x, double beta, double *y, cudaStream_t s)
{
    CsrView A{p->m, p->n, p->rowptr, p->col, p->val};
    if (p->m == 0) return SBB_OK;
    switch (p->kernel) {
    case SBB_KERNEL_VECTOR:
        if (p->f32)
            launch_vector_f32(A, p->vector_width, alpha, static_cast<const float *>(x), beta, y,
                              p->status, s);
        else
            launch_vector(A, p->vector_width, alpha, static_cast<const double *>(x), beta, y,
                          p->status, s);
        break;
    case SBB_KERNEL_MERGE: {
        MergeScratch S{p->tile_row, p->tile_nnz, p->carry_val, &p->runs, p->runs.count, p->tiles,
                       p->queue, p->persistent_ctas, merge_queue_item(*p)};
        if (p->f32)
            launch_merge_f32(A, p->ipt, S, alpha, static_cast<const float *>(x), beta, y,
                             p->status, s);
        else
            launch_merge(A, p->ipt, S, alpha, static_cast<const double *>(x), beta, y,
                         p->status, s);
        break;
    }
    case SBB_KERNEL_TILED:
        return tiled_run(p, alpha, x, beta, y, s);
    case SBB_KERNEL_ROWS:
        return rows_run(p, alpha, x, beta, y, s);
    default:
        set_error("plan has no kernel");
        return SBB_ERR_ARG;
    }
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}

}  // namespace sbb

// ------------------------------------------------------------------ C ABI
using namespace sbb;

struct sbb_plan_s {
    Plan p;
};

static int create_common(sbb_plan_t *out, int m, int n, int nnz, const int *rp, const int *col,
                         const void *val, bool f32, const sbb_config *cfg, void *stream,
                         bool lane32 = false)
{
    if (!out) {
        set_error("plan pointer is NULL");
        return SBB_ERR_ARG;
    }
    *out = nullptr;
    if (m < 0 || n < 0 || nnz < 0 || !rp || (nnz > 0 && (!col || !val))) {
        set_error("bad matrix arguments");
        return SBB_ERR_ARG;
    }
    auto *h = new sbb_plan_s();
    h->p.m = m;
    h->p.n = n;
    h->p.nnz = nnz;
    h->p.rowptr = rp;
    h->p.col = col;
    h->p.val = val;
    h->p.f32 = f32;
    h->p.lane32 = lane32;
    int rc = plan_build(&h->p, cfg, static_cast<cudaStream_t>(stream));
    if (rc != SBB_OK) {
        cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
        plan_free(&h->p);
        delete h;
        return rc;
    }
    *out = h;
    return SBB_OK;
}

extern "C" {

int sbb_plan_create(sbb_plan_t *plan, int m, int n, int nnz, const int *d_rowptr,
                    const int *d_col, const double *d_val, const sbb_config *cfg, void *stream)
{
    return create_common(plan, m, n, nnz, d_rowptr, d_col, d_val, false, cfg, stream);
}

int sbb_plan_create_f32(sbb_plan_t *plan, int m, int n, int nnz, const int *d_rowptr,
                        const int *d_col, const float *d_val, const sbb_config *cfg,
                        void *stream)
{
    return create_common(plan, m, n, nnz, d_rowptr, d_col, d_val, true, cfg, stream);
}

int sbb_plan_create_f32_lanes(sbb_plan_t *plan, int m, int n, int nnz, const int *d_rowptr,
                              const int *d_col, const float *d_val, const sbb_config *cfg,
                              void *stream)
{
    return create_common(plan, m, n, nnz, d_rowptr, d_col, d_val, true, cfg, stream, true);
}

// x (n values) overlapping y (m doubles): an error, set here.
static bool xy_overlap(const sbb_plan_s *plan, const void *d_x, const double *d_y)
{
    const size_t xb = (size_t)plan->p.n * (plan->p.f32 ? 4 : 8), yb = (size_t)plan->p.m * 8;
    if (!ranges_overlap(d_x, xb, d_y, yb)) return false;
    set_error("x and y overlap (the kernels read x while they write y)");
    return true;
}

int sbb_spmv(sbb_plan_t plan, double alpha, const double *d_x, double beta, double *d_y,
             void *stream)
{
    if (!plan || plan->p.f32 || (plan->p.m > 0 && !d_y) || (plan->p.nnz > 0 && !d_x)) {
        set_error("bad sbb_spmv arguments (NULL pointer or an FP32 plan)");
        return SBB_ERR_ARG;
    }
    if (xy_overlap(plan, d_x, d_y)) return SBB_ERR_ARG;
    return plan_run(&plan->p, alpha, d_x, beta, d_y, static_cast<cudaStream_t>(stream));
}

int sbb_spmv_f32(sbb_plan_t plan, double alpha, const float *d_x, double beta, double *d_y,
                 void *stream)
{
    if (!plan || !plan->p.f32 || (plan->p.m > 0 && !d_y) || (plan->p.nnz > 0 && !d_x)) {
        set_error("bad sbb_spmv_f32 arguments (NULL pointer or an FP64 plan)");
        return SBB_ERR_ARG;
    }
    if (xy_overlap(plan, d_x, d_y)) return SBB_ERR_ARG;
    return plan_run(&plan->p, alpha, d_x, beta, d_y, static_cast<cudaStream_t>(stream));
}

int sbb_spmv_timed(sbb_plan_t plan, double alpha, const void *d_x, double beta, double *d_y,
                   void *stream, void *ev_start, void *ev_stop)
{
    if (!plan || (plan->p.m > 0 && !d_y) || (plan->p.nnz > 0 && !d_x)) {
        set_error("bad sbb_spmv_timed arguments");
        return SBB_ERR_ARG;
    }
    if (xy_overlap(plan, d_x, d_y)) return SBB_ERR_ARG;
    TimingHooks &h = timing_hooks();
    h.start = static_cast<cudaEvent_t>(ev_start);
    h.stop = static_cast<cudaEvent_t>(ev_stop);
    int rc = plan_run(&plan->p, alpha, d_x, beta, d_y, static_cast<cudaStream_t>(stream));
    h.start = h.stop = nullptr;
    return rc;
}

int sbb_plan_launches(sbb_plan_t plan) { return plan ? plan_launches(&plan->p) : 0; }

int sbb_plan_check(sbb_plan_t plan)
{
    if (!plan) return SBB_ERR_ARG;
    unsigned st = 0;
    cudaError_t e = cudaMemcpy(&st, plan->p.status, sizeof(st), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_error(cudaGetErrorString(e));
        return SBB_ERR_CUDA;
    }
    if (st) {
        set_error(std::string("device status ") + std::to_string(st) +
                  ((st & ST_BAD_COL) ? ": column index out of range" : "") +
                  ((st & ST_BAD_TILE) ? ": corrupt tile" : "") +
                  ((st & ST_BAD_QUEUE) ? ": work queue overflow" : "") +
                  ((st & ST_TIMEOUT) ? ": a bounded wait on a device copy gave up" : ""));
        return SBB_ERR_INPUT;
    }
    return SBB_OK;
}

int sbb_plan_info_get(sbb_plan_t plan, sbb_plan_info *info)
{
    if (!plan || !info) return SBB_ERR_ARG;
    const Plan &p = plan->p;
    info->kernel = p.kernel;
    info->vector_width = p.vector_width;
    info->items_per_thread = p.ipt;
    info->persistent = p.persistent_ctas;
    info->tile_sigma = p.tile_sigma;
    info->tiles = p.tiles;
    info->max_row_len = p.max_row;
    info->empty_rows = p.empty_rows;
    info->scratch_bytes = p.scratch_bytes;
    return SBB_OK;
}

int sbb_plan_partition(sbb_plan_t plan, int *h_row, int *h_nnz, int cap)
{
    if (!plan || !h_row || !h_nnz) return SBB_ERR_ARG;
    const Plan &p = plan->p;
    if (p.kernel != SBB_KERNEL_MERGE || !p.tile_row) {
        set_error("plan has no merge-path partition");
        return SBB_ERR_ARG;
    }
    int cnt = p.tiles + 1;
    if (cap < cnt) {
        set_error("partition buffer too small");
        return SBB_ERR_ARG;
    }
    if (cudaMemcpy(h_row, p.tile_row, sizeof(int) * cnt, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(h_nnz, p.tile_nnz, sizeof(int) * cnt, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("copy of the partition failed");
        return SBB_ERR_CUDA;
    }
    return cnt;
}

int sbb_plan_destroy(sbb_plan_t plan)
{
    if (!plan) return SBB_OK;
    cudaSetDevice(plan->p.device);
    cudaDeviceSynchronize();
    plan_free(&plan->p);
    delete plan;
    return SBB_OK;
}

const char *sbb_last_error(void) { return g_error.c_str(); }

}  // extern "C"
