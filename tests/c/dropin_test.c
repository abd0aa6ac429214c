/* dropin_test.c — a C program that calls libsbb's drop-in entry points the
 * way the reference's test driver calls the reference objects
 * (SparseBLAS/test/dspmv_test.cu): its generated matrix shape (:137-208),
 * x = 1, y = 0 and random alpha/beta (:268-282), then every version and
 * kernel (:305-383), each result checked against a host loop at the
 * reference test's own bar (absolute 1e-3, :390-401) and at the per-row
 * bar |y - y_ref| <= 1e-12 * (|alpha| sum_j |a_ij x_j| + |beta y_i|).  A
 * second round uses random x, y and beta != 0, which the reference test
 * never exercises.  Links against libsbb.so through include/sbb_spmv.h.
 *
 *   dropin_test --host-only   calls that do no device work (no GPU needed)
 *   dropin_test [n]           the full run (n a multiple of 8, default 4096)
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sbb_spmv.h"

static unsigned long long rng_state = 0x243F6A8885A308D3ull;

/* splitmix64, mapped to [0, 1) with 53 bits */
static double urand(void)
{
    unsigned long long z = (rng_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* The reference generator's shape ('g n'): m = n, eight row blocks of
 * nb = m/8 rows; rows of the first block hold ceil(0.9 n) nonzeros, the
 * others ceil(0.01 n), in columns 0, 1, ...; values uniform in [0, 1)
 * (seeded here).  m must be a multiple of 8: the reference's loop writes past
 * row m - 1 otherwise. */
static void gen_g(int n, long long **rp_out, int **col_out, double **val_out, long long *nnz_out)
{
    const int m = n, nb = m / 8;
    const int l1 = (int)ceil(0.9 * n), l2 = (int)ceil(0.01 * n);
    long long *rp = malloc(sizeof(long long) * (m + 1));
    long long nnz = 0;
    rp[0] = 0;
    for (int r = 0; r < m; r++) {
        nnz += r < nb ? l1 : l2;
        rp[r + 1] = nnz;
    }
    int *col = malloc(sizeof(int) * nnz);
    double *val = malloc(sizeof(double) * nnz);
    for (int r = 0; r < m; r++)
        for (long long k = rp[r]; k < rp[r + 1]; k++) {
            col[k] = (int)(k - rp[r]);
            val[k] = urand();
        }
    *rp_out = rp;
    *col_out = col;
    *val_out = val;
    *nnz_out = nnz;
}

/* Host loop (the reference's main.cu:350-356, with + beta*y), summed in long
 * double so its own rounding stays far below the bar, and both bars. */
static int check(const char *what, int m, const long long *rp, const int *col, const double *val,
                 const double *x, double alpha, double beta, const double *y_in,
                 const double *y_out)
{
    double worst = 0.0, worst_abs = 0.0;
    for (int r = 0; r < m; r++) {
        long double s = 0.0L, a = 0.0L;
        for (long long k = rp[r]; k < rp[r + 1]; k++) {
            const long double p = (long double)val[k] * x[col[k]];
            s += p;
            a += fabsl(p);
        }
        const double ref = (double)((long double)alpha * s + (long double)beta * y_in[r]);
        const double scale = (double)(fabsl((long double)alpha) * a + fabsl((long double)beta * y_in[r]));
        const double d = fabs(y_out[r] - ref);
        if (d > worst_abs) worst_abs = d;
        if (scale > 0.0 && d / scale > worst) worst = d / scale;
        if (scale == 0.0 && d != 0.0) worst = INFINITY;
    }
    if (!(worst <= 1e-12) || !(worst_abs < 1e-3)) {
        printf("FAIL %s: max scaled error %.3e, max absolute error %.3e\n", what, worst, worst_abs);
        return 1;
    }
    return 0;
}

static int host_only(void)
{
    int bad = 0;
    const double t0 = get_time();
    if (!(t0 > 0.0)) {
        printf("FAIL get_time\n");
        bad++;
    }
    long long a[6] = {0, 2, 2, 2, 5, 9};  /* 5 rows (n = 5), rows 1 and 2 empty */
    if (get_row_from_index(5, a, 0) != 0 || get_row_from_index(5, a, 4) != 3 ||
        get_row_from_index(5, a, 8) != 4) {
        printf("FAIL get_row_from_index\n");
        bad++;
    }
    /* argument checks return -1 before any device work */
    long long rp[2] = {0, 1};
    int col[1] = {0};
    double val[1] = {1.0}, x[1] = {1.0}, y[1] = {0.0}, al = 1.0, be = 0.0;
    if (spMV_mgpu_v1(1, 1, 1, &al, val, rp, col, x, &be, y, 0, 1) != -1 ||   /* ngpu <= 0 */
        spMV_mgpu_v1(1, 1, 1, &al, val, rp, col, x, &be, y, 1, 4) != -1 ||   /* kernel 4 */
        spMV_mgpu_v2(1, 1, 1, &al, val, rp, col, x, &be, y, 1, 1, 0, 1) != -1 || /* nb 0 */
        spMV_mgpu_baseline(1, 1, 1, NULL, val, rp, col, x, &be, y, 1) != -1) {
        printf("FAIL argument checks\n");
        bad++;
    }
    if (!bad) printf("host-only ok\n");
    return bad;
}

int main(int argc, char **argv)
{
    if (argc > 1 && strcmp(argv[1], "--host-only") == 0) return host_only();
    const int n = argc > 1 ? atoi(argv[1]) : 4096;
    if (n <= 0 || n % 8) {
        printf("n must be a positive multiple of 8\n");
        return 2;
    }
    long long *rp, nnz;
    int *col;
    double *val;
    gen_g(n, &rp, &col, &val, &nnz);
    const int m = n;
    double *x = malloc(sizeof(double) * n), *y0 = malloc(sizeof(double) * m),
           *y = malloc(sizeof(double) * m);
    int fails = 0, calls = 0;
    for (int round = 0; round < 2; round++) {
        double alpha = urand(), beta = urand();
        for (int i = 0; i < n; i++) x[i] = round == 0 ? 1.0 : 2.0 * urand() - 1.0;
        for (int i = 0; i < m; i++) y0[i] = round == 0 ? 0.0 : 2.0 * urand() - 1.0;
        if (round == 0) beta = 0.0 * beta;  /* y = 0 as in the reference test */
        const char *names[7] = {"baseline", "v1 kernel 1", "v1 kernel 2", "v1 kernel 3",
                                "v2 kernel 1", "v2 kernel 2", "v2 kernel 3"};
        for (int c = 0; c < 7; c++) {
            memcpy(y, y0, sizeof(double) * m);
            double al = alpha, be = beta;
            int rc;
            if (c == 0)
                rc = spMV_mgpu_baseline(m, n, nnz, &al, val, rp, col, x, &be, y, 1);
            else if (c <= 3)
                rc = spMV_mgpu_v1(m, n, nnz, &al, val, rp, col, x, &be, y, 1, c);
            else
                rc = spMV_mgpu_v2(m, n, nnz, &al, val, rp, col, x, &be, y, 1, c - 3, nnz / 8 + 1,
                                  2);
            calls++;
            if (rc != 0) {
                printf("FAIL %s (round %d): rc %d\n", names[c], round, rc);
                fails++;
                continue;
            }
            fails += check(names[c], m, rp, col, val, x, alpha, beta, y0, y);
        }
    }
    free(rp), free(col), free(val), free(x), free(y0), free(y);
    if (fails) return 1;
    printf("ok: %d calls, m = n = %d, nnz = %lld\n", calls, n, nnz);
    return 0;
}
