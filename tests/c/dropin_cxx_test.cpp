// dropin_cxx_test.cpp — a C++ caller compiled the way code that includes the
// reference's header is: the entry points declared with C++ linkage (the
// reference declares them without extern "C", SparseBLAS/include/spmv_kernel.h
// :4-34), so this program links to libsbb.so's C++-mangled names.  The
// declarations below are that interface, written out here.
//
//   dropin_cxx_test --host-only   calls that do no device work
//   dropin_cxx_test               also one spMV_mgpu_v1 call per kernel
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

int spMV_mgpu_baseline(int m, int n, long long nnz, double *alpha, double *csrVal,
                       long long *csrRowPtr, int *csrColIndex, double *x, double *beta,
                       double *y, int ngpu);
int spMV_mgpu_v1(int m, int n, long long nnz, double *alpha, double *csrVal,
                 long long *csrRowPtr, int *csrColIndex, double *x, double *beta, double *y,
                 int ngpu, int kernel);
int spMV_mgpu_v2(int m, int n, long long nnz, double *alpha, double *csrVal,
                 long long *csrRowPtr, int *csrColIndex, double *x, double *beta, double *y,
                 int ngpu, int kernel, long long nb, int q);
int get_row_from_index(int n, long long *a, long long idx);
double get_time();
double get_gpu_availble_mem(int ngpu);

int main(int argc, char **argv)
{
    const bool host_only = argc > 1 && std::strcmp(argv[1], "--host-only") == 0;
    int bad = 0;
    if (!(get_time() > 0.0)) bad++, std::printf("FAIL get_time\n");
    long long a[6] = {0, 2, 2, 2, 5, 9};  // 5 rows, rows 1 and 2 empty
    if (get_row_from_index(5, a, 4) != 3) bad++, std::printf("FAIL get_row_from_index\n");
    long long rp1[2] = {0, 1};
    int c1[1] = {0};
    double v1[1] = {1.0}, x1[1] = {1.0}, y1[1] = {0.0}, one = 1.0, zero = 0.0;
    if (spMV_mgpu_v1(1, 1, 1, &one, v1, rp1, c1, x1, &zero, y1, 0, 1) != -1)  // ngpu <= 0
        bad++, std::printf("FAIL ngpu check\n");
    if (host_only || bad) {
        if (!bad) std::printf("host-only ok\n");
        return bad;
    }
    if (!(get_gpu_availble_mem(1) > 0.0)) bad++, std::printf("FAIL get_gpu_availble_mem\n");

    // tridiagonal 1000 x 1000: a_ii = 2, a_i,i+-1 = -1; x_j = j; y_i = 1
    const int m = 1000;
    std::vector<long long> rp(m + 1, 0);
    std::vector<int> col;
    std::vector<double> val;
    for (int i = 0; i < m; i++) {
        for (int j = i - 1; j <= i + 1; j++)
            if (j >= 0 && j < m) {
                col.push_back(j);
                val.push_back(j == i ? 2.0 : -1.0);
            }
        rp[i + 1] = (long long)col.size();
    }
    std::vector<double> x(m);
    for (int j = 0; j < m; j++) x[j] = j;
    double alpha = 0.5, beta = 2.0;
    for (int kernel = 1; kernel <= 3; kernel++) {
        std::vector<double> y(m, 1.0);
        const int rc = spMV_mgpu_v1(m, m, (long long)col.size(), &alpha, val.data(), rp.data(),
                                    col.data(), x.data(), &beta, y.data(), 1, kernel);
        if (rc != 0) {
            bad++, std::printf("FAIL kernel %d: rc %d\n", kernel, rc);
            continue;
        }
        for (int i = 0; i < m; i++) {
            // (A x)_i = 2i - (i-1) - (i+1) = 0 inside; row 0: -1; row m-1: m
            const double ax = i == 0 ? -1.0 : (i == m - 1 ? (double)m : 0.0);
            if (y[i] != alpha * ax + beta * 1.0) {
                bad++, std::printf("FAIL kernel %d row %d: %.17g\n", kernel, i, y[i]);
                break;
            }
        }
    }
    if (!bad) std::printf("ok\n");
    return bad;
}
