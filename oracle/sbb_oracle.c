/*
 * sbb_oracle.c — CPU oracle for the FP64 CSR SpMV path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for libsbb.so.  Only tests/, the smoke
 * check and bench.py's CPU-baseline leg load it; the product never does.
 *
 * Each function restates the reference (JieyangChen7/Sparse-BLAS) behaviour it
 * names, in code written for this oracle.  The partition and merge steps keep
 * the reference's exact arithmetic (integer/double floor, evaluation order of
 * the boundary fix-ups) because the drop-in must reproduce them bit for bit.
 */
#include "sbb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* --- partition ---------------------------------------------------------- */

/* src/spmv_helper.cu:16-39.  Bisection over a[0..n] keeping a[lo] <= idx <
 * a[hi]; an exact hit on a[mid] returns mid at once, which for runs of empty
 * rows is some row of the run rather than the row that owns idx. */
int orc_get_row_from_index(int n, const long long *a, long long idx)
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

/* Flags and row lookup shared by v1 (src/dspmv_mgpu_v1.cu:73-94) and v2
 * (src/dspmv_mgpu_v2.cu:242-267): a slice whose first nnz is past its start
 * row's first nnz has a split start row; one whose last nnz is before its end
 * row's last nnz has a split end row. */
static void slice_rows(int m, const long long *rowptr, orc_slice *s)
{
    s->start_row = orc_get_row_from_index(m, rowptr, s->start_idx);
    s->start_flag = s->start_idx > rowptr[s->start_row];
    s->end_row = orc_get_row_from_index(m, rowptr, s->end_idx);
    s->end_flag = s->end_idx < rowptr[s->end_row + 1] - 1;
}

/* src/dspmv_mgpu_v1.cu:60-94: part i gets nnz [floor(i*nnz/P),
 * floor((i+1)*nnz/P) - 1], the quotient taken in double. */
void orc_v1_partition(int m, long long nnz, const long long *rowptr, int P,
                      orc_slice *out)
{
    for (int i = 0; i < P; i++) {
        long long lo = (long long)i * nnz;
        long long hi = (long long)(i + 1) * nnz;
        out[i].start_idx = (long long)floor((double)lo / P);
        out[i].end_idx = (long long)floor((double)hi / P) - 1;
        out[i].y2 = 0.0;
        slice_rows(m, rowptr, &out[i]);
    }
}

/* src/dspmv_mgpu_baseline.cu:60-87: part d gets rows [d*m/P, (d+1)*m/P - 1]
 * (int arithmetic) and every nnz of those rows; nothing is split. */
void orc_baseline_partition(int m, const long long *rowptr, int P,
                            orc_slice *out)
{
    for (int d = 0; d < P; d++) {
        out[d].start_row = d * m / P;
        out[d].end_row = (d + 1) * m / P - 1;
        out[d].start_idx = rowptr[out[d].start_row];
        out[d].end_idx = rowptr[out[d].end_row + 1] - 1;
        out[d].start_flag = out[d].end_flag = 0;
        out[d].y2 = 0.0;
    }
}

int orc_v2_num_tasks(long long nnz, long long nb)
{
    return (int)((nnz + nb - 1) / nb);
}

/* src/dspmv_mgpu_v2.cu:228-273: task t gets nnz [t*nnz/T, (t+1)*nnz/T - 1]
 * with the quotient in integer arithmetic; y2 saves y of the split start row
 * and is then overwritten by y of the split end row when both are split. */
void orc_v2_tasks(int m, long long nnz, const long long *rowptr,
                  const double *y, long long nb, int T, orc_slice *out)
{
    (void)nb;
    for (int t = 0; t < T; t++) {
        long long lo = (long long)t * nnz;
        long long hi = (long long)(t + 1) * nnz;
        out[t].start_idx = lo / T;
        out[t].end_idx = hi / T - 1;
        out[t].y2 = 0.0;
    }
    for (int t = 0; t < T; t++) {
        out[t].start_row = orc_get_row_from_index(m, rowptr, out[t].start_idx);
        out[t].start_flag = out[t].start_idx > rowptr[out[t].start_row];
        if (out[t].start_flag) out[t].y2 = y[out[t].start_row];
    }
    for (int t = 0; t < T; t++) {
        out[t].end_row = orc_get_row_from_index(m, rowptr, out[t].end_idx);
        out[t].end_flag = out[t].end_idx < rowptr[out[t].end_row + 1] - 1;
        if (out[t].end_flag) out[t].y2 = y[out[t].end_row];
    }
}

/* --- slice compute ------------------------------------------------------ */

void orc_slice_csrmv(const orc_slice *s, const long long *rowptr,
                     const int *col, const double *val, const double *x,
                     double alpha, double beta, int csr5, double *y_slice)
{
    int dev_m = s->end_row - s->start_row + 1;
    for (int j = 0; j < dev_m; j++) {
        int r = s->start_row + j;
        long long lo = (j == 0) ? s->start_idx : rowptr[r];
        long long hi = (j == dev_m - 1) ? s->end_idx + 1 : rowptr[r + 1];
        double sum = 0.0;
        for (long long k = lo; k < hi; k++) sum += val[k] * x[col[k]];
        if (csr5)
            y_slice[j] = sum;
        else if (beta == 0.0)
            y_slice[j] = alpha * sum;
        else
            y_slice[j] = alpha * sum + beta * y_slice[j];
    }
}

static int valid_args(int m, int n, long long nnz)
{
    return m >= 0 && n >= 0 && nnz >= 0;
}

/* src/dspmv_mgpu_baseline.cu:14-213 with the GPU work done by
 * orc_slice_csrmv; parts are written back in order d = 0..P-1 (:184-187). */
int orc_dropin_baseline(int m, int n, long long nnz, double alpha,
                        const double *val, const long long *rowptr,
                        const int *col, const double *x, double beta,
                        double *y, int P)
{
    if (P <= 0 || !valid_args(m, n, nnz)) return -1;
    orc_slice *s = (orc_slice *)malloc(sizeof(orc_slice) * P);
    orc_baseline_partition(m, rowptr, P, s);
    double **dev_y = (double **)malloc(sizeof(double *) * P);
    for (int d = 0; d < P; d++) {
        int dev_m = s[d].end_row - s[d].start_row + 1;
        dev_y[d] = (double *)malloc(sizeof(double) * (dev_m > 0 ? dev_m : 1));
        if (dev_m > 0) memcpy(dev_y[d], y + s[d].start_row, sizeof(double) * dev_m);
    }
    for (int d = 0; d < P; d++)
        if (s[d].end_row >= s[d].start_row)
            orc_slice_csrmv(&s[d], rowptr, col, val, x, alpha, beta, 0, dev_y[d]);
    for (int d = 0; d < P; d++) {
        int dev_m = s[d].end_row - s[d].start_row + 1;
        if (dev_m > 0) memcpy(y + s[d].start_row, dev_y[d], sizeof(double) * dev_m);
        free(dev_y[d]);
    }
    free(dev_y);
    free(s);
    return 0;
}

/* src/dspmv_mgpu_v1.cu:16-277.  All device y slices are uploaded from the
 * original y before any compute (:176-184); results come back in order
 * d = 0..P-1 and a split start row is fixed up as y += previous; y -= y2*beta
 * (:232-245). */
int orc_dropin_v1(int m, int n, long long nnz, double alpha, const double *val,
                  const long long *rowptr, const int *col, const double *x,
                  double beta, double *y, int P, int kernel)
{
    if (P <= 0 || !valid_args(m, n, nnz) || kernel < 1 || kernel > 3) return -1;
    orc_slice *s = (orc_slice *)malloc(sizeof(orc_slice) * P);
    orc_v1_partition(m, nnz, rowptr, P, s);
    for (int d = 0; d < P; d++)
        if (s[d].start_flag) s[d].y2 = y[s[d].start_row];
    double **dev_y = (double **)malloc(sizeof(double *) * P);
    for (int d = 0; d < P; d++) {
        int dev_m = s[d].end_row - s[d].start_row + 1;
        dev_y[d] = (double *)malloc(sizeof(double) * (dev_m > 0 ? dev_m : 1));
        if (dev_m > 0) memcpy(dev_y[d], y + s[d].start_row, sizeof(double) * dev_m);
    }
    for (int d = 0; d < P; d++)
        if (s[d].end_row >= s[d].start_row)
            orc_slice_csrmv(&s[d], rowptr, col, val, x, alpha, beta,
                            kernel == 3, dev_y[d]);
    for (int d = 0; d < P; d++) {
        int dev_m = s[d].end_row - s[d].start_row + 1;
        if (dev_m <= 0) { free(dev_y[d]); continue; }
        double prev = s[d].start_flag ? y[s[d].start_row] : 0.0;
        memcpy(y + s[d].start_row, dev_y[d], sizeof(double) * dev_m);
        if (s[d].start_flag) {
            y[s[d].start_row] += prev;
            y[s[d].start_row] -= s[d].y2 * beta;
        }
        free(dev_y[d]);
    }
    free(dev_y);
    free(s);
    return 0;
}

/* One merge step of src/dspmv_mgpu_v2.cu:396-429: the first piece of a split
 * row seen in pop order is kept; every later piece adds the row's current y
 * and removes the beta*y2 it double counts. */
static void v2_merge_piece(char *seen, int row, double *piece, const double *y,
                           double beta, double y2)
{
    if (!seen[row]) {
        seen[row] = 1;
    } else {
        double cur = y[row];
        *piece += cur;
        *piece -= beta * y2;
    }
}

int orc_dropin_v2(int m, int n, long long nnz, double alpha, const double *val,
                  const long long *rowptr, const int *col, const double *x,
                  double beta, double *y, int kernel, long long nb, int q)
{
    if (nb <= 0 || q <= 0 || !valid_args(m, n, nnz) || kernel < 1 || kernel > 3)
        return -1;
    if (nnz == 0) return 0;
    int T = orc_v2_num_tasks(nnz, nb);
    orc_slice *s = (orc_slice *)malloc(sizeof(orc_slice) * T);
    orc_v2_tasks(m, nnz, rowptr, y, nb, T, s);
    double **local = (double **)malloc(sizeof(double *) * T);
    for (int t = 0; t < T; t++) {
        int dev_m = s[t].end_row - s[t].start_row + 1;
        local[t] = (double *)malloc(sizeof(double) * dev_m);
        memcpy(local[t], y + s[t].start_row, sizeof(double) * dev_m);
        orc_slice_csrmv(&s[t], rowptr, col, val, x, alpha, beta, kernel == 3,
                        local[t]);
    }
    char *seen = (char *)calloc(m > 0 ? m : 1, 1);
    for (int t = T - 1; t >= 0; t--) { /* pop order: back of the pool first */
        int dev_m = s[t].end_row - s[t].start_row + 1;
        if (dev_m == 1 && s[t].start_flag && s[t].end_flag) {
            v2_merge_piece(seen, s[t].start_row, &local[t][0], y, beta, s[t].y2);
        } else {
            if (s[t].start_flag)
                v2_merge_piece(seen, s[t].start_row, &local[t][0], y, beta, s[t].y2);
            if (s[t].end_flag)
                v2_merge_piece(seen, s[t].end_row, &local[t][dev_m - 1], y, beta,
                               s[t].y2);
        }
        memcpy(y + s[t].start_row, local[t], sizeof(double) * dev_m);
        free(local[t]);
    }
    free(seen);
    free(local);
    free(s);
    return 0;
}

/* --- host SpMV (CPU baseline) and accurate oracle ----------------------- */

void orc_spmv_host(int m, const long long *rowptr, const int *col,
                   const double *val, const double *x, double alpha,
                   double beta, double *y, int nthreads)
{
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1) if (nthreads > 1)
    for (int i = 0; i < m; i++) {
        double sum = 0.0;
        for (long long j = rowptr[i]; j < rowptr[i + 1]; j++)
            sum += x[col[j]] * val[j] * alpha;
        y[i] = sum + beta * y[i];
    }
}

void orc_spmv_host_f32(int m, const int *rowptr, const int *col,
                       const float *val, const float *x, double alpha,
                       double beta, double *y, int nthreads)
{
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1) if (nthreads > 1)
    for (int i = 0; i < m; i++) {
        double sum = 0.0;
        for (int j = rowptr[i]; j < rowptr[i + 1]; j++)
            sum += (double)x[col[j]] * (double)val[j] * alpha;
        y[i] = sum + beta * y[i];
    }
}

/* Error-free transforms (Knuth TwoSum; TwoProd through fma). */
static inline void two_sum(double a, double b, double *s, double *e)
{
    double t = a + b;
    double bb = t - a;
    *e = (a - (t - bb)) + (b - bb);
    *s = t;
}
static inline void two_prod(double a, double b, double *p, double *e)
{
    double t = a * b;
    *e = fma(a, b, -t);
    *p = t;
}
/* (hi, lo) += (p, pe) */
static inline void dd_add(double *hi, double *lo, double p, double pe)
{
    double s, e;
    two_sum(*hi, p, &s, &e);
    e += *lo + pe;
    two_sum(s, e, hi, lo);
}

void orc_spmv_dd(int m, const long long *rowptr, const int *col,
                 const double *val, const double *x, double alpha, double beta,
                 const double *y_in, double *y_out, double *scale)
{
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < m; i++) {
        double hi = 0.0, lo = 0.0, absum = 0.0;
        for (long long j = rowptr[i]; j < rowptr[i + 1]; j++) {
            double p, pe;
            two_prod(val[j], x[col[j]], &p, &pe);
            dd_add(&hi, &lo, p, pe);
            absum += fabs(p);
        }
        /* alpha * (hi + lo) in double-double */
        double ah, ahe;
        two_prod(alpha, hi, &ah, &ahe);
        ahe += alpha * lo;
        double rh = 0.0, rl = 0.0;
        dd_add(&rh, &rl, ah, ahe);
        double by = 0.0;
        if (beta != 0.0) {
            double bp, bpe;
            two_prod(beta, y_in[i], &bp, &bpe);
            dd_add(&rh, &rl, bp, bpe);
            by = fabs(beta * y_in[i]);
        }
        y_out[i] = rh + rl;
        if (scale) scale[i] = fabs(alpha) * absum + by;
    }
}

/* --- merge-path split --------------------------------------------------- */

void orc_merge_path_split(int m, const int *rowptr, long long items_per_part,
                          int P, int *out_row, int *out_nnz)
{
    long long base = rowptr[0];
    long long nnz = (long long)rowptr[m] - base;
    long long total = (long long)m + nnz;
    for (int p = 0; p <= P; p++) {
        long long d = (long long)p * items_per_part;
        if (d > total) d = total;
        long long lo = d - nnz > 0 ? d - nnz : 0;
        long long hi = d < m ? d : m;
        while (lo < hi) {
            long long pivot = (lo + hi) >> 1;
            if ((long long)rowptr[pivot + 1] - base <= d - pivot - 1)
                lo = pivot + 1;
            else
                hi = pivot;
        }
        out_row[p] = (int)lo;
        out_nnz[p] = (int)(base + d - lo);
    }
}

/* include/anonymouslib_cuda.h:296-313 */
int orc_csr5_sigma(int m, long long nnz)
{
    int per_row = m > 0 ? (int)(nnz / m) : 0;
    if (per_row <= 4) return 4;
    if (per_row <= 32) return per_row;
    if (per_row <= 256) return 32;
    return 6;
}
