/*
 * sbb_spmv.h — C ABI of libsbb: FP64 CSR SpMV  y = alpha*A*x + beta*y  on one
 * NVIDIA B200 (sm_100a).
 *
 * Part 1 is the drop-in boundary: the entry points of JieyangChen7/Sparse-BLAS
 * with their exact argument lists, meanings and return codes (citations are
 * to that project, paths relative to its root).  Part 2 is the device API
 * (device-resident arrays, reusable plans) the drop-in is built on.
 *
 * All functions are extern "C" and take plain pointers and sizes.  Return
 * codes of the drop-in entry points follow the reference: 0 success,
 * -1 bad argument / insufficient device memory / kernel failure,
 *  1 CUDA allocation failure.  Device-API functions return SBB_OK (0) or a
 * negative SBB_ERR_*; sbb_last_error() gives the message.
 */
#ifndef SBB_SPMV_H
#define SBB_SPMV_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================= Part 1: drop-in boundary ======================== */

/* The GPU count of these entry points is pinned to 1: a call runs on the
 * calling thread's current CUDA device (device 0 unless the caller selected
 * another, as with the reference's ngpu = 1) and returns when y is in host
 * memory.  nnz <= 2^31 - 1 (the reference casts a device's nnz to int,
 * SparseBLAS/src/dspmv_mgpu_v1.cu:119; larger calls return -1); kernel 3
 * takes at most 2^31 - 1025 rows. */

/* Replaces spMV_mgpu_baseline (SparseBLAS/include/spmv_kernel.h:9-13,
 * SparseBLAS/src/dspmv_mgpu_baseline.cu:14-213).  Host pointers; rows split
 * evenly over ngpu parts, which is pinned to 1 here (ngpu <= 0 -> -1). */
int spMV_mgpu_baseline(int m, int n, long long nnz, double *alpha,
                       double *csrVal, long long *csrRowPtr, int *csrColIndex,
                       double *x, double *beta, double *y, int ngpu);

/* Replaces spMV_mgpu_v1 (SparseBLAS/include/spmv_kernel.h:14-19,
 * SparseBLAS/src/dspmv_mgpu_v1.cu:16-277).  nnz-balanced split (pinned to one
 * part), kernel 1 = vector CSR, 2 = merge path, 3 = CSR5-style tiles. */
int spMV_mgpu_v1(int m, int n, long long nnz, double *alpha, double *csrVal,
                 long long *csrRowPtr, int *csrColIndex, double *x,
                 double *beta, double *y, int ngpu, int kernel);

/* Replaces spMV_mgpu_v2 (SparseBLAS/include/spmv_kernel.h:21-28,
 * SparseBLAS/src/dspmv_mgpu_v2.cu:33-207).  ceil(nnz/nb) tasks with the
 * reference's split-row merge.  With kernel 2 the task pool runs as one
 * persistent merge kernel: q resident CTAs per SM claim items of nb nnz
 * (capped so every warp gets several) from a device work queue.  Returns 0
 * on success (the reference returns no value, :207). */
int spMV_mgpu_v2(int m, int n, long long nnz, double *alpha, double *csrVal,
                 long long *csrRowPtr, int *csrColIndex, double *x,
                 double *beta, double *y, int ngpu, int kernel, long long nb,
                 int q);

/* Replaces csr5_kernel (SparseBLAS/include/spmv_kernel.h:4-7,
 * SparseBLAS/src/csr5_kernel.cu:12-32).  DEVICE pointers, int32 row pointer.
 * Unlike the reference, alpha and beta are honoured
 * (the reference drops them: include/detail/cuda/csr5_spmv_cuda.h:22,
 * include/anonymouslib_cuda.h:281) and the caller's col/val are not modified. */
int csr5_kernel(int m, int n, int nnz, double *alpha, double *csrVal,
                int *csrRowPtr, int *csrColIndex, double *x, double *beta,
                double *y);

/* Replaces get_row_from_index (SparseBLAS/src/spmv_helper.cu:16-39). */
int get_row_from_index(int n, long long *a, long long idx);
/* Replaces get_time (SparseBLAS/src/spmv_helper.cu:41-48): wall clock, s. */
double get_time(void);
/* Replaces get_gpu_availble_mem (SparseBLAS/src/spmv_helper.cu:51-76):
 * free memory in GB, minimum over the first ngpu devices that exist. */
double get_gpu_availble_mem(int ngpu);

/* ========================= Part 2: device API ============================ */

enum {
    SBB_OK = 0,
    SBB_ERR_ARG = -1,      /* bad argument                              */
    SBB_ERR_CUDA = -2,     /* CUDA runtime error                        */
    SBB_ERR_INPUT = -3,    /* malformed CSR found by a device check     */
    SBB_ERR_NOMEM = -4     /* allocation failed / would not fit          */
};

enum {
    SBB_KERNEL_AUTO = 0,
    SBB_KERNEL_VECTOR = 1, /* K1: V lanes per row, warp-shuffle reduce   */
    SBB_KERNEL_MERGE = 2,  /* K2: merge-path split of rows+nnz over CTAs */
    SBB_KERNEL_TILED = 3,  /* K3: CSR5-style 32 x sigma tiles            */
    SBB_KERNEL_LEARNED = 4,/* the trained selector (sbb_mlp_select, built-in
                              parameters) picks one of the SBB_NUM_CLASSES
                              batch classes' configurations on the GPU; the
                              parameters (21.6 KB) are copied to a device
                              the first time it is used and kept until exit */
    SBB_KERNEL_ROWS = 5    /* K4: blocks of <= 32 rows and <= 384 nnz (rows
                              longer than 384 nnz split into pieces), staged
                              into shared memory by TMA straight from the
                              caller's CSR arrays (no copy of the matrix),
                              one lane per row; no counterpart in the
                              reference.  Needs 4-byte-aligned int arrays and
                              an 8-byte-aligned (FP32: 4) value array. */
};

typedef struct {
    int kernel;            /* SBB_KERNEL_*                                  */
    int vector_width;      /* K1: 2,4,8,16,32 (0 = from mean row length)    */
    int items_per_thread;  /* K2: merge items per thread (0 = default)      */
    int persistent;        /* K2: >0 = persistent CTAs per SM with a device
                              work queue; 0 = one CTA per tile              */
    int tile_sigma;        /* K3: nnz per lane per tile (0 = CSR5 rule)     */
} sbb_config;

typedef struct sbb_plan_s *sbb_plan_t;

typedef struct {
    int kernel, vector_width, items_per_thread, persistent, tile_sigma;
    int tiles;             /* K2/K3 work tiles                               */
    int max_row_len, empty_rows;
    size_t scratch_bytes;  /* device memory the plan owns                    */
} sbb_plan_info;

/* Build a plan for an m x n CSR matrix resident on the current device
 * (int32 row pointer with rowptr[0] == 0 and rowptr[m] == nnz, int32 columns,
 * FP64 values).  The arrays must stay valid and unchanged while the plan
 * lives.  cfg may be NULL (automatic choice).  stream: a cudaStream_t or
 * NULL.  The row pointer is validated (one synchronisation). */
int sbb_plan_create(sbb_plan_t *plan, int m, int n, int nnz,
                    const int *d_rowptr, const int *d_col, const double *d_val,
                    const sbb_config *cfg, void *stream);
/* FP32-storage form: values (and x at run time) stored as float, halving
 * their bytes.  Each product of two floats is formed exactly in FP64 and the
 * row segments, carries and alpha/beta update are FP64, so the result differs
 * from the FP64 product of the rounded inputs only by FP64 summation error;
 * against the FP64 inputs the error is that of rounding val and x to float
 * (per row, about 1e-7 of sum_j |a_ij x_j|). */
int sbb_plan_create_f32(sbb_plan_t *plan, int m, int n, int nnz,
                        const int *d_rowptr, const int *d_col,
                        const float *d_val, const sbb_config *cfg, void *stream);
/* FP32-storage form with FP32 lane sums: the same storage, but each lane's
 * run of at most sigma (4 or 8) consecutive products of a row is summed by an
 * FP32 fused multiply-add chain and widened to FP64 once; the warp scan, the
 * carries and the alpha/beta update stay FP64.  Per row the error against the
 * FP64 inputs is at most about 10 * 2^-24 (6e-7) of sum_j |a_ij x_j|.  Tiled
 * kernel only (cfg NULL or kernel SBB_KERNEL_AUTO / SBB_KERNEL_TILED,
 * tile_sigma 0 = 8, or 4); anything else is SBB_ERR_ARG.  Run it with
 * sbb_spmv_f32.  No counterpart in the reference (it has no FP32 path). */
int sbb_plan_create_f32_lanes(sbb_plan_t *plan, int m, int n, int nnz,
                              const int *d_rowptr, const int *d_col,
                              const float *d_val, const sbb_config *cfg, void *stream);
/* y = alpha*A*x + beta*y on the stream (asynchronous).  y is not read when
 * beta == 0.  Out-of-range column indices are skipped and flagged; see
 * sbb_plan_check.  x (n values) and y (m values) must not overlap
 * (SBB_ERR_ARG): the kernels read x while they write y. */
int sbb_spmv(sbb_plan_t plan, double alpha, const double *d_x, double beta,
             double *d_y, void *stream);
int sbb_spmv_f32(sbb_plan_t plan, double alpha, const float *d_x, double beta,
                 double *d_y, void *stream);
/* sbb_spmv that also records ev_start / ev_stop (cudaEvent_t, may be NULL)
 * on the stream immediately before and after the plan's main kernel, so the
 * caller can time that kernel alone (the ordered carry fix-up and the
 * empty-row pass run after ev_stop). */
int sbb_spmv_timed(sbb_plan_t plan, double alpha, const void *d_x, double beta,
                   double *d_y, void *stream, void *ev_start, void *ev_stop);
/* Number of kernel launches one sbb_spmv of this plan makes. */
int sbb_plan_launches(sbb_plan_t plan);
/* Synchronise the plan's status word: SBB_OK or SBB_ERR_INPUT. */
int sbb_plan_check(sbb_plan_t plan);
int sbb_plan_info_get(sbb_plan_t plan, sbb_plan_info *info);
/* Copy the merge-path tile coordinates (tiles+1 rows and nnz offsets) to the
 * host; returns the number of entries written or a negative error. */
int sbb_plan_partition(sbb_plan_t plan, int *h_row, int *h_nnz, int cap);
int sbb_plan_destroy(sbb_plan_t plan);

/* ---- batched form: many matrices, a few persistent launches -------------- */

/* Kernel classes a matrix of a batch can use (the autotuner's and the
 * learned selector's choices; each computes the same SpMV):
 *   0..3: vector CSR with 4, 8, 16, 32 lanes per row;
 *   4:    merge path, 6 items per lane (192-item warp segments);
 *   5:    CSR5-style tiles of 32 x 4 nnz (sigma = 4).
 * No counterpart in the reference, whose v2 driver runs the tasks of ONE
 * matrix from a host pool (SparseBLAS/src/dspmv_mgpu_v2.cu:73-188). */
#define SBB_NUM_CLASSES 6

typedef struct {
    int m, n, nnz;
    const int *rowptr, *col;   /* device, int32, rowptr[0] == 0 */
    const double *val;         /* device, FP64 */
    const double *x;           /* device */
    double *y;                 /* device; y = alpha*A*x + beta*y */
    double alpha, beta;
    int cls;                   /* 0 .. SBB_NUM_CLASSES-1 */
} sbb_batch_item;

typedef struct sbb_batch_s *sbb_batch_t;

/* Builds one plan per matrix (validating each) and the device work list.
 * The arrays must stay valid while the batch lives. */
int sbb_batch_create(sbb_batch_t *batch, const sbb_batch_item *items, int count,
                     void *stream);
/* All SpMVs of the batch: one persistent kernel per kernel family present
 * (vector classes 0-1, vector classes 2-3, merge class 4, tiled class 5),
 * each taking work units
 * (row chunks, merge segments or tile groups) of all its matrices from its
 * own device queue; the kernels run as parallel branches forked from `stream`
 * and joined back, then one more launch adds the carries of every merge/tiled
 * matrix and finishes the empty rows of tiled ones.  Each matrix's y is
 * bit-identical to sbb_batch_run_each with the same classes.  The y arrays
 * must not overlap one another or any x (sbb_batch_create checks; x arrays
 * may be shared). */
int sbb_batch_run(sbb_batch_t batch, void *stream);
/* Same launches, captured once in a CUDA graph and replayed. */
int sbb_batch_run_graph(sbb_batch_t batch, void *stream);
/* The baseline: each matrix's own plain launch sequence, one after another. */
int sbb_batch_run_each(sbb_batch_t batch, void *stream);
/* Kernel launches of one run: per_matrix = 0 -> batched, 1 -> run_each. */
int sbb_batch_launches(sbb_batch_t batch, int per_matrix);
/* Synchronise the status words: SBB_OK or SBB_ERR_INPUT. */
int sbb_batch_check(sbb_batch_t batch);
int sbb_batch_destroy(sbb_batch_t batch);

/* Autotuner probe: mean time (ms, CUDA events, `reps` runs after one warm-up)
 * of each class on one matrix as a plain launch; d_y is overwritten.  ms has
 * SBB_NUM_CLASSES entries. */
int sbb_tune_classes(int m, int n, int nnz, const int *d_rowptr, const int *d_col,
                     const double *d_val, const double *d_x, double *d_y, double alpha,
                     double beta, int reps, float *ms, void *stream);

/* ---- learned class selector ---------------------------------------------- */

/* A small FP32 MLP (12 features -> 64 -> 64 -> SBB_NUM_CLASSES, ReLU) that
 * predicts, per kernel class, log2(t_class / t_best) of a plain launch; the
 * selector picks the class with the smallest prediction.  No counterpart in
 * the reference (its only tuner is the (ngpu, q) sweep of
 * test/dspmv_test.cu:314-332).  The parameters are one float array of
 * SBB_MLP_PARAMS entries: feature mean[12], feature std[12] (fixed input
 * normalisation), W1[64][12], b1[64], W2[64][64], b2[64], W3[6][64], b3[6]. */
#define SBB_MLP_FEATURES 12
#define SBB_MLP_PARAMS 5406

/* The 12 features of a device CSR matrix into d_feat (device, 12 floats):
 * log2(1+m), log2(1+n), log2(1+nnz), log2(1+mean row length), coefficient of
 * variation of the row lengths, log2(1+max row length), log2(1+max/mean),
 * fraction of empty rows, of rows with <= 4 nnz, of rows with > 32 nnz,
 * fraction of nnz in rows with > 128 nnz, mean column span of a row / n. */
int sbb_features(int m, int n, int nnz, const int *d_rowptr, const int *d_col, float *d_feat,
                 void *stream);
/* d_y[N][6] = MLP(d_x[N][12]) (device arrays). */
int sbb_mlp_forward(const float *d_params, const float *d_x, int N, float *d_y, void *stream);
/* Loss L = sum_n w_n sum_c (y[n][c] - t[n][c])^2 / (6 * sum_n w_n) and its
 * gradient d_grad[SBB_MLP_PARAMS] (zero for the normalisation entries);
 * d_w may be NULL (all weights 1).  d_loss: one device float or NULL.  Sums
 * over samples run in a fixed order (deterministic). */
int sbb_mlp_grad(const float *d_params, const float *d_x, const float *d_t, const float *d_w,
                 int N, float *d_grad, float *d_loss, void *stream);
/* `steps` full-batch Adam steps (lr, L2 weight decay wd) on device, updating
 * d_params in place; d_loss_hist (device, `steps` floats) or NULL. */
int sbb_mlp_train(float *d_params, const float *d_x, const float *d_t, const float *d_w, int N,
                  int steps, float lr, float wd, float *d_loss_hist, void *stream);
/* Features, forward pass and argmin on the GPU for one device CSR matrix;
 * *cls receives the chosen class (synchronises the stream). */
int sbb_mlp_select(const float *d_params, int m, int n, int nnz, const int *d_rowptr,
                   const int *d_col, int *cls, void *stream);

/* Merge-path y = alpha*A*x + beta*y on device arrays that allocates nothing:
 * no counterpart in the reference.  For callers that must not call cudaMalloc
 * (a memory-capped or pre-partitioned process, a callback or real-time path
 * that may not block on the allocator, a host framework that owns all device
 * memory), the scratch lives in a fixed 5 MiB __device__ array of the library,
 * held on every GPU that loads it until the process exits.  Limit:
 * m + nnz <= 100,663,296 (larger inputs return SBB_ERR_ARG); x and y must
 * not overlap (SBB_ERR_ARG).  All calls share
 * that array and it keeps the last call's contents, so calls that overlap on
 * the GPU race; serialise them.  The first call on a device looks up the
 * array's address; make it before any stream capture on that device.  The row
 * pointer must start at 0 and end at nnz; invalid indices are not reported by
 * this entry point (they cannot make it read out of range).  Asynchronous on
 * `stream` (a cudaStream_t or NULL). */
int sbb_spmv_merge_noalloc(int m, int n, int nnz, const int *d_rowptr,
                           const int *d_col, const double *d_val, double alpha,
                           const double *d_x, double beta, double *d_y,
                           void *stream);

/* ---- Matrix Market input ------------------------------------------------- */

/* Loads a Matrix Market coordinate file (fields real / integer / pattern,
 * symmetry general / symmetric / skew-symmetric) as canonical CSR: rows and
 * columns sorted, duplicates summed in file order, symmetric storage
 * expanded, pattern entries set to pattern_value.  Replaces the reader of the
 * reference's test driver (SparseBLAS/test/dspmv_test.cu:101-136, 228-251),
 * whose CSR is right only for files already sorted by row.  *handle receives
 * the matrix (host memory); copy it out with sbb_mm_copy (rowptr: m+1 int64
 * offsets, col: nnz int32, val: nnz doubles) and release it with
 * sbb_mm_free.  Errors name the offending line. */
int sbb_mm_load(const char *path, double pattern_value, void **handle, int *m, int *n,
                long long *nnz);
int sbb_mm_copy(void *handle, long long *rowptr, int *col, double *val);
void sbb_mm_free(void *handle);

const char *sbb_last_error(void);

/* ---- call trace ------------------------------------------------------------ */

/* Wall-clock phases of the calling thread's last host-pointer call
 * (spMV_mgpu_baseline / v1 / v2), in milliseconds, for finding where a slow
 * call spends its time: [0] host partition and copy enqueue, [1] wait for
 * the row-pointer check on the device, [2] plan building and launches of
 * every chunk, [3] wait for the kernels and the copy of y back, [4] host
 * merges and restores.  Writes min(n, SBB_TRACE_PHASES) values and returns
 * how many; 0 if the thread has made no call that got that far. */
#define SBB_TRACE_PHASES 5
int sbb_last_call_phases(double *ms, int n);

/* ---- test hooks ------------------------------------------------------------ */

/* Host-side fault injection for the library's own tests, so that the error
 * paths of the reference's contract run without faulting a GPU: the 1 a
 * drop-in call returns when a device allocation fails
 * (SparseBLAS/src/dspmv_mgpu_baseline.cu:99-135), the -1 of the 0.8 x
 * free-memory pre-check (SparseBLAS/src/dspmv_mgpu_v1.cu:104-116), and the
 * timeout status of the tiled kernel's bounded waits.  Process-wide; not for
 * production use.
 *   SBB_TEST_RESET        disarm every hook (value ignored);
 *   SBB_TEST_FAIL_ALLOC   value = k >= 1: the k-th device allocation the
 *                         library makes from now on fails, once (0 disarms);
 *   SBB_TEST_FREE_BYTES   value >= 0: the drop-in memory pre-check sees at
 *                         most this many free bytes (< 0 disarms);
 *   SBB_TEST_WAIT_BUDGET  value >= 0: in tiled-kernel launches the first wait
 *                         of the grid's first warp for its tile copy gives up
 *                         after `value` polls (0: at once); the kernel then
 *                         lets its copies in flight land, raises the timeout
 *                         status and stops, so sbb_plan_check reports
 *                         SBB_ERR_INPUT and drop-in calls return -1 (< 0
 *                         disarms). */
enum { SBB_TEST_RESET = 0, SBB_TEST_FAIL_ALLOC = 1, SBB_TEST_FREE_BYTES = 2,
       SBB_TEST_WAIT_BUDGET = 3 };
int sbb_test_hook(int what, long long value);

#ifdef __cplusplus
}
#endif
#endif /* SBB_SPMV_H */
