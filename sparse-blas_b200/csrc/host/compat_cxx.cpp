// compat_cxx.cpp — C++-linkage copies of the reference's entry points.
//
// The reference declares them without extern "C" (SparseBLAS/include/spmv_kernel.h:4-34),
// so code compiled against that header links to the C++-mangled names.  These
// definitions give libsbb.so those names too; each forwards to the same
// implementation as the extern "C" entry point.
#include "entry.h"

int csr5_kernel(int m, int n, int nnz, double *alpha, double *csrVal, int *csrRowPtr,
                int *csrColIndex, double *x, double *beta, double *y)
{
    return sbb::csr5_entry(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y);
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
                 int ngpu, int kernel, long long nb, int copy_of_workspace)
{
    return sbb::dropin_v2(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y, ngpu,
                          kernel, nb, copy_of_workspace);
}

int get_row_from_index(int n, long long *a, long long idx) { return sbb::row_from_index(n, a, idx); }
double get_time() { return sbb::wall_time(); }
double get_gpu_availble_mem(int ngpu) { return sbb::min_free_gb(ngpu); }
