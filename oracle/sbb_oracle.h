/*
 * sbb_oracle.h — CPU oracle for the FP64 CSR SpMV path (y = alpha*A*x + beta*y).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the tests, the smoke
 * check and the CPU-baseline leg of bench.py call it; the product (libsbb.so)
 * never links, loads or calls it.
 *
 * Every function restates a piece of the reference (JieyangChen7/Sparse-BLAS)
 * and cites the file:line it follows.  Paths are relative to the reference
 * project root; a path with no directory prefix is under SparseBLAS/.
 */
#ifndef SBB_ORACLE_H
#define SBB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Bisection for the row that owns nnz index idx (src/spmv_helper.cu:16-39).
 * n is the row count, a[0..n] the int64 row pointer. */
int orc_get_row_from_index(int n, const long long *a, long long idx);

/* One row-slice of a partition: the unit the reference ships to one GPU (v1,
 * baseline) or one task (v2).  Row r of the slice, start_row <= r <= end_row,
 * covers nnz [r == start_row ? start_idx : rowptr[r],
 *             r == end_row   ? end_idx+1 : rowptr[r+1]).                   */
typedef struct {
    long long start_idx, end_idx;
    int start_row, end_row;
    int start_flag, end_flag; /* 1 = the row is split with a neighbour slice */
    double y2;                /* saved y of the split row (v2 only)          */
} orc_slice;

/* v1 nnz-balanced split into P parts (src/dspmv_mgpu_v1.cu:60-94). */
void orc_v1_partition(int m, long long nnz, const long long *rowptr, int P,
                      orc_slice *out);

/* Baseline even row split into P parts (src/dspmv_mgpu_baseline.cu:60-87). */
void orc_baseline_partition(int m, const long long *rowptr, int P,
                            orc_slice *out);

/* v2 task count ceil(nnz/nb) (src/dspmv_mgpu_v2.cu:218). */
int orc_v2_num_tasks(long long nnz, long long nb);

/* v2 task table (src/dspmv_mgpu_v2.cu:228-273), including the saved y2. */
void orc_v2_tasks(int m, long long nnz, const long long *rowptr,
                  const double *y, long long nb, int T, orc_slice *out);

/* Slice csrmv with the cuSPARSE csrmv contract (y = alpha*A*x + beta*y on the
 * slice; y is not read when beta == 0), plain FP64 running sum in nnz order.
 * csr5 != 0 models the vendored CSR5 instead: alpha and beta are dropped and
 * y = A*x (include/detail/cuda/csr5_spmv_cuda.h:22, include/anonymouslib_cuda.h:281).
 * y_slice holds end_row-start_row+1 values. */
void orc_slice_csrmv(const orc_slice *s, const long long *rowptr,
                     const int *col, const double *val, const double *x,
                     double alpha, double beta, int csr5, double *y_slice);

/* Whole drop-in entry points, host semantics included (partition, per-slice
 * device y, D2H order, boundary merges).  Return codes follow the reference:
 * 0 ok, -1 bad argument.  kernel: 1, 2 (same arithmetic here) or 3 (CSR5). */
int orc_dropin_baseline(int m, int n, long long nnz, double alpha,
                        const double *val, const long long *rowptr,
                        const int *col, const double *x, double beta,
                        double *y, int P);
int orc_dropin_v1(int m, int n, long long nnz, double alpha, const double *val,
                  const long long *rowptr, const int *col, const double *x,
                  double beta, double *y, int P, int kernel);
/* v2 with one GPU: tasks are popped from the back of the pool
 * (src/dspmv_mgpu_v2.cu:135-149) and merged in that order
 * (src/dspmv_mgpu_v2.cu:381-437). */
int orc_dropin_v2(int m, int n, long long nnz, double alpha, const double *val,
                  const long long *rowptr, const int *col, const double *x,
                  double beta, double *y, int kernel, long long nb, int q);

/* The reference's host CSR SpMV (main.cu:350-356: sum += x[col]*val*alpha,
 * row order) with the beta term added: y[i] = sum + beta*y[i].
 * nthreads > 1 runs rows in an OpenMP static schedule. */
void orc_spmv_host(int m, const long long *rowptr, const int *col,
                   const double *val, const double *x, double alpha,
                   double beta, double *y, int nthreads);

/* Same loop over int32 row pointers and FP32 values/x (the FP32-storage
 * form's inputs), FP64 accumulation. */
void orc_spmv_host_f32(int m, const int *rowptr, const int *col,
                       const float *val, const float *x, double alpha,
                       double beta, double *y, int nthreads);

/* Accurate oracle: double-double (TwoSum/TwoProd) accumulation of
 * alpha*sum(a_ij x_j) + beta*y_i per row, rounded once.  Also returns
 * scale_i = |alpha|*sum|a_ij x_j| + |beta*y_i| (the error-metric denominator).
 * rowptr is int64; rows with empty extents give beta*y_i. */
void orc_spmv_dd(int m, const long long *rowptr, const int *col,
                 const double *val, const double *x, double alpha, double beta,
                 const double *y_in, double *y_out, double *scale);

/* Merge-path split (Merrill & Garland, "Merge-based parallel sparse
 * matrix-vector multiplication", SC'16): for each of P+1 diagonals
 * d = min(p*items, m+nnz) find (rows consumed, nnz consumed) on the merge of
 * row ends rowptr[1..m] with nnz indices rowptr[0]..rowptr[m]-1.  This is the
 * CPU restatement of the device partition kernel; results are compared bit for
 * bit.  out_row/out_nnz have P+1 entries; nnz offsets are absolute. */
void orc_merge_path_split(int m, const int *rowptr, long long items_per_part,
                          int P, int *out_row, int *out_nnz);

/* CSR5 sigma rule (include/anonymouslib_cuda.h:296-313). */
int orc_csr5_sigma(int m, long long nnz);

#ifdef __cplusplus
}
#endif
#endif
