// sbb_internal.h — shared declarations for libsbb (B200 FP64 CSR SpMV).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>

#include "sbb_spmv.h"

namespace sbb {

// ---- error plumbing --------------------------------------------------------
void set_error(const std::string &msg);
#define SBB_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) {                                              \
            ::sbb::set_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
            return SBB_ERR_CUDA;                                              \
        }                                                                     \
    } while (0)

// True when the byte ranges [a, a + abytes) and [b, b + bbytes) share a byte.
// x must not overlap y: the kernels read x while they write y (cuSPARSE's
// SpMV has the same rule).
inline bool ranges_overlap(const void *a, size_t abytes, const void *b, size_t bbytes)
{
    if (!a || !b || abytes == 0 || bbytes == 0) return false;
    const uintptr_t pa = reinterpret_cast<uintptr_t>(a), pb = reinterpret_cast<uintptr_t>(b);
    return pa < pb + bbytes && pb < pa + abytes;
}

// ---- test hooks (hooks.cpp; armed only by sbb_test_hook) -------------------
// cudaMallocAsync, except that an armed allocation-failure hook fails it.
cudaError_t dev_malloc_async(void **p, size_t bytes, cudaStream_t s);
// Free device memory as the drop-in memory pre-check sees it.
size_t capped_free_bytes(size_t free_b);
// -1, or the poll budget of the first tile-copy wait of a tiled launch's
// first warp.
int first_wait_budget();

// Device status word bits, written by kernels instead of trapping.
enum : unsigned {
    ST_BAD_ROWPTR = 1u << 0,   // non-monotone row pointer or out of [0, nnz]
    ST_BAD_COL = 1u << 1,      // column index outside [0, n)
    ST_BAD_TILE = 1u << 2,     // a merge-path tile with impossible extents
    ST_BAD_QUEUE = 1u << 3,    // work-queue index past its capacity
    ST_TIMEOUT = 1u << 4,      // a bounded wait on a copy gave up
};

// Resident CTAs per SM and SM count for a persistent kernel with the given
// block size and dynamic shared memory, on the current device.  The occupancy
// query runs once per device and kernel and later launches read the cache
// (the host work per launch otherwise shows up as idle GPU time between
// short SpMVs); the shared-memory attribute, which a new context would not
// have, is set on every launch that needs more than the default 48 KB.
struct LaunchShape {
    int sms, occ;
};
template <typename K>
LaunchShape cached_launch_shape(K kern, int threads, size_t smem)
{
    static std::atomic<long long> cache[64];  // sms << 32 | occ, 0 = not yet known
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    long long v = cache[dev].load(std::memory_order_acquire);
    if (v == 0) {  // racing first calls compute the same value
        int sms = 148, occ = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
        if (sms < 1) sms = 1;
        if (occ < 1) occ = 1;
        v = ((long long)sms << 32) | occ;
        cache[dev].store(v, std::memory_order_release);
    }
    return LaunchShape{(int)(v >> 32), (int)(v & 0xffffffff)};
}

// ---- kernel launchers (defined in the .cu files) ---------------------------
constexpr int kMergeThreads = 256;
// Tile plans take at most this many rows: row counts and segment ranks plus
// a tile's offsets stay in int.  The automatic and learned choices use the
// merge path above it.
constexpr int kTiledMaxRows = 2147483647 - 1024;

struct CsrView {          // rows [0, m) of a CSR matrix; offsets are absolute
    int m, n;
    const int *rowptr;    // m+1 entries; rowptr[0] may be non-zero
    const int *col;
    const void *val;      // double* (FP64 form) or float* (FP32 form)
};

// rowptr int64 -> int32 with validation (monotone, within [0, nnz]).
void launch_rowptr_narrow(const long long *src, int *dst, int m, long long nnz,
                          unsigned *status, cudaStream_t s);
void launch_rowptr_check(const int *rp, int m, int nnz, unsigned *status, cudaStream_t s);
// Row-length statistics: out[0] = max row length, out[1] = #empty rows.
void launch_row_stats(const int *rowptr, int m, int *out, cudaStream_t s);

// K1: vector CSR, V lanes per row.
void launch_vector(const CsrView &A, int V, double alpha, const double *x,
                   double beta, double *y, unsigned *status, cudaStream_t s);
void launch_vector_f32(const CsrView &A, int V, double alpha, const float *x,
                       double beta, double *y, unsigned *status, cudaStream_t s);

// Per-tile carries: carry_row[t] (static per plan; m = nothing carried) and
// carry_val[t] (written by the tiled kernel).  Runs of >= 2 tiles carrying
// the same row are listed once at plan time.
// Runs of at most this many carries are summed by one warp, longer ones by a
// block (spmv_device.cuh: fixup_run_warp, fixup_partial).
constexpr int kWarpRunMax = 1024;
struct CarryRuns {
    int *run_first = nullptr, *run_len = nullptr;
    int n_runs = 0;
    int n_long = 0;   // runs longer than kWarpRunMax, listed first
    int *count = nullptr;  // device-built lists: the run count, on the device only
    size_t bytes = 0;
};
int carry_runs_build(const int *carry_row, int T, int m, CarryRuns *R, cudaStream_t s);
// The same lists built without any host synchronisation: runs in the order
// the marking kernel found them, their count left on the device (R->count).
int carry_runs_build_device(const int *carry_row, int T, int m, CarryRuns *R, cudaStream_t s);
void carry_runs_free(CarryRuns *R, cudaStream_t s, bool async);
// Marks the runs on the device only; the count stays in *dev_count.
void launch_runs_mark(const int *carry_row, int T, int m, int *run_first, int *run_len,
                      int *dev_count, cudaStream_t s);
// Adds the carries to y in a fixed order; also rearms `queue` when non-null.
// dev_count non-null: the run count is read on the device (R.n_runs unused).
void launch_fixup(int m, const int *carry_row, const double *carry_val, int T,
                  const CarryRuns &R, double alpha, double *y, unsigned *queue, cudaStream_t s,
                  const int *dev_count = nullptr);

// K2: merge path.  One warp per segment of 32*IPT merge items.
int merge_ipt_supported(int ipt);
long long merge_items_per_tile(int ipt);
void launch_merge_partition(const int *rowptr, int m, int base, long long nnz, long long items,
                            int tiles, int *tile_row, int *tile_nnz, cudaStream_t s);
struct MergeScratch {
    const int *tile_row, *tile_nnz;   // tiles+1 coordinates; tile t carries row tile_row[t+1]
    double *carry_val;                // tiles
    const CarryRuns *runs;
    const int *runs_count;            // non-null: run count kept on the device
    int tiles;
    unsigned *queue;                  // persistent form: [0] = next segment to claim
    int persistent_ctas;              // 0 = one CTA per tile
    int queue_item;                   // persistent form: segments per claim (>= 1)
};
void launch_merge(const CsrView &A, int ipt, const MergeScratch &S, double alpha,
                  const double *x, double beta, double *y, unsigned *status,
                  cudaStream_t s);
void launch_merge_f32(const CsrView &A, int ipt, const MergeScratch &S,
                      double alpha, const float *x, double beta, double *y,
                      unsigned *status, cudaStream_t s);
int merge_max_ctas_per_sm(int ipt, bool f32);

// ---- batched form (k_batch.cu) ----------------------------------------------
constexpr int kBatchIpt = 6;        // merge-path class: items per lane (as its plain plan)
constexpr int kBatchMergeClass = 4; // classes 0..3: vector CSR with V = 4 << cls
constexpr int kBatchTiledClass = 5; // CSR5-style tiles, sigma = kBatchSigma
constexpr int kBatchSigma = 4;
constexpr int kBatchTileGroup = 2;  // tiled class: tiles per work unit (one bulk copy)
constexpr int kBatchClaim = 16;     // work units a warp claims per queue access
constexpr int kBatchVectorNnz = 1024; // vector classes: about this many nnz per work unit
constexpr int kBatchVectorU = 4;    // vector classes: rows of a lane group in flight together
// Rows per K1 chunk for V lanes per row and U rows in flight per lane group
// (VectorShape<V, U>::CR in spmv_device.cuh).
constexpr int vector_chunk_rows(int V, int U) { return (32 / V) * U < 32 ? (32 / V) * U : 32; }
struct BatchMat {                   // one matrix of a batch, as the kernel sees it
    const int *rowptr, *col;
    const void *val;
    const double *x;
    double *y;
    int m, n, cls;
    int vsteps;                      // vector classes: chunks per unit
    double alpha, beta;
    const int *tile_row, *tile_nnz;  // merge class: segment coordinates
    const int *crow;                 // merge/tiled: static carry row of each tile
    double *carry_val;
    int tiles;
    long long nnz;
    const unsigned char *blob;       // tiled class
    const int *tile_seg, *ne;
};
// Flat view of every merge/tiled matrix's carries (and of the tiled
// matrices' empty rows) for the batch fix-up.
struct BatchFix {
    const long long *tile0;          // nfix+1: first global carry slot of each matrix with slots
    const int *mat;                  // nfix: batch index of each such matrix
    int nfix;
    const int *run_mat, *run_first, *run_len;  // multi-slot runs (all matrices),
    int n_runs;                                // those longer than kWarpRunMax first
    int n_long_runs;
    const int *empty_row, *empty_mat;          // empty rows of tiled matrices: y = beta*y
    int n_empty;
};
// What the batch needs from a tiled plan.
struct Plan;
struct TiledView {
    const unsigned char *blob;
    const int *tile_seg, *ne, *empty, *carry_row;
    double *carry_val;
    int tiles, sigma, n_empty;
    const CarryRuns *runs;
};
bool tiled_view(const Plan *p, TiledView *v);
// The plain-plan configuration of batch class cls (0 .. SBB_NUM_CLASSES-1).
sbb_config batch_class_config(int cls);
// Kernel families of the batch: one persistent kernel each, compiled with
// only its family's code (so with that code's register budget): vector CSR
// with 4 or 8 lanes, with 16 or 32 lanes, the merge class, the tiled class.
enum { kFamVectorNarrow = 0, kFamVectorWide = 1, kFamMerge = 2, kFamTiled = 3,
       kBatchFamilies = 4 };
inline int batch_family(int cls)
{
    return cls < 2 ? kFamVectorNarrow
                   : (cls < kBatchMergeClass ? kFamVectorWide
                                             : (cls == kBatchMergeClass ? kFamMerge : kFamTiled));
}
int batch_max_ctas_per_sm(int fam);
// Units [0, total) of the family's matrices mats[0..nmat) (unit0: nmat+1
// prefix offsets), claimed from *queue.
void launch_batch(int fam, const BatchMat *mats, int nmat, const long long *unit0,
                  long long total, unsigned long long *queue, unsigned *status, int grid,
                  cudaStream_t s);
void launch_batch_fixup(const BatchMat *mats, const BatchFix &F, long long total_slots,
                        cudaStream_t s);

// ---- learned class selector (k_mlp.cu) -------------------------------------
constexpr int kMlpFeatures = 12, kMlpHidden = 64, kMlpClasses = SBB_NUM_CLASSES;
constexpr int kMlpParams = 2 * kMlpFeatures + kMlpHidden * kMlpFeatures + kMlpHidden +
                           kMlpHidden * kMlpHidden + kMlpHidden + kMlpClasses * kMlpHidden +
                           kMlpClasses;
// acc: 8 device words of scratch; feat: 12 floats (device).
void launch_features(const int *rp, const int *col, int m, int n, long long nnz,
                     unsigned long long *acc, float *feat, cudaStream_t s);
void launch_mlp_forward(const float *P, const float *X, int N, float *Xn, float *H1, float *H2,
                        float *Y, cudaStream_t s);
void launch_mlp_backward(const float *P, int N, const float *Xn, const float *H1,
                         const float *H2, const float *Y, const float *T, const float *W,
                         float inv_norm, float *dY, float *dZ2, float *dZ1, float *G,
                         float *loss, cudaStream_t s);
void launch_mlp_adam(float *P, const float *G, float *M, float *V, int step, float lr, float wd,
                     cudaStream_t s);
void launch_mlp_argmin(const float *Y, int N, int *cls, cudaStream_t s);

// Boundary pieces (drop-in): sum of val*x over [lo, hi) per piece.
void launch_pieces(const long long *lo, const long long *hi, int npieces,
                   const int *col, const double *val, const double *x, int n,
                   double *out, unsigned *status, cudaStream_t s);

// Plan object behind sbb_plan_t.
struct Plan {
    int m = 0, n = 0, nnz = 0;
    int base = 0;            // rowptr[0] (non-zero for a row range of a larger matrix)
    const int *rowptr = nullptr, *col = nullptr;
    const void *val = nullptr;
    bool f32 = false;
    bool lane32 = false;     // FP32 storage summed in FP32 lane runs (tiled, sigma <= 8)
    int kernel = 0;          // resolved SBB_KERNEL_*
    int vector_width = 0;    // K1
    int ipt = 0;             // K2
    int persistent = 0;      // K2 persistent CTAs per SM (0 = off)
    bool device_runs = false; // K2: carry runs built and counted on the device (no host sync)
    long long queue_nnz = 0; // K2 persistent form: nnz per queue item (0 = one segment)
    int tile_sigma = 0;      // K3
    int max_row = 0, empty_rows = 0;
    // device scratch owned by the plan
    int *tile_row = nullptr, *tile_nnz = nullptr;
    double *carry_val = nullptr;
    CarryRuns runs;
    unsigned *queue = nullptr;
    unsigned *status = nullptr;
    int tiles = 0, persistent_ctas = 0;
    void *tiled = nullptr;   // K3 tile plan (k_tiled.cu)
    void *rows = nullptr;    // K4 row-block plan (k_rows.cu)
    size_t scratch_bytes = 0;
    int device = 0;
};

int plan_build(Plan *p, const sbb_config *cfg, cudaStream_t s);
int plan_run(Plan *p, double alpha, const void *x, double beta, double *y,
             cudaStream_t s);
void plan_free(Plan *p);
int default_kernel_choice(int m, int nnz, int max_row, int *vector_width, int *ipt, int *sigma);
int plan_launches(const Plan *p);
// Optional timing hooks (set by sbb_spmv_timed for the calling thread): the
// launchers record them immediately before / after their main kernel.
struct TimingHooks {
    cudaEvent_t start = nullptr, stop = nullptr;
};
TimingHooks &timing_hooks();
inline void hook_start(cudaStream_t s)
{
    if (timing_hooks().start) cudaEventRecord(timing_hooks().start, s);
}
inline void hook_stop(cudaStream_t s)
{
    if (timing_hooks().stop) cudaEventRecord(timing_hooks().stop, s);
}

}  // namespace sbb
