/*
 * ref_shim.cpp — CPU stand-ins that let the reference's own host drivers run
 * in this (GPU-less) container.  TEST INFRASTRUCTURE ONLY: the result,
 * oracle/_ref/libref.so, exists to pin the oracle against the reference's
 * partition / dispatch / merge code and to generate the golden fixtures under
 * tests/golden/.  It never ships with or runs inside the product.
 *
 * What is stood in for:
 *   - the CUDA runtime calls the drivers make (device memory becomes host
 *     memory, copies become memcpy, streams and syncs are no-ops);
 *   - cuSPARSE handles/descriptors and the removed legacy cusparseDcsrmv /
 *     cusparseDcsrmv_mp: y = alpha*A*x + beta*y with a plain FP64 running sum
 *     per row in nnz order (y is not read when beta == 0);
 *   - csr5_kernel (SparseBLAS/src/csr5_kernel.cu:12-32): y = A*x, alpha and
 *     beta dropped as the vendored CSR5 does
 *     (include/detail/cuda/csr5_spmv_cuda.h:22, include/anonymouslib_cuda.h:281).
 *     CSR5's handling of empty rows inside tiles is not modelled.
 * The csrmv arithmetic is therefore this file's, identical to the oracle's
 * orc_slice_csrmv; what the comparison pins is the reference's driver logic.
 */
#include <cuda_runtime_api.h>
#include <cusparse.h>
#include <cstdlib>
#include <cstring>

#include "ref_legacy.h"
#include "spmv_kernel.h" /* the reference's API header, C++ linkage */

struct CUstream_st { int unused; };
struct cusparseContext { int unused; };
struct cusparseMatDescr { int type, base; };

static size_t g_free_bytes = (size_t)180 * 1000 * 1000 * 1000;

extern "C" {

cudaError_t cudaSetDevice(int) { return cudaSuccess; }
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaStreamCreate(cudaStream_t *s)
{
    *s = new CUstream_st();
    return cudaSuccess;
}
cudaError_t cudaStreamDestroy(cudaStream_t s)
{
    delete s;
    return cudaSuccess;
}
cudaError_t cudaMalloc(void **p, size_t n)
{
    *p = std::malloc(n ? n : 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void *p)
{
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaMallocHost(void **p, size_t n) { return cudaMalloc(p, n); }
cudaError_t cudaFreeHost(void *p) { return cudaFree(p); }
cudaError_t cudaMemcpy(void *d, const void *s, size_t n, enum cudaMemcpyKind)
{
    if (n) std::memmove(d, s, n);
    return cudaSuccess;
}
cudaError_t cudaMemcpyAsync(void *d, const void *s, size_t n,
                            enum cudaMemcpyKind k, cudaStream_t)
{
    return cudaMemcpy(d, s, n, k);
}
cudaError_t cudaMemGetInfo(size_t *free_b, size_t *total_b)
{
    *free_b = g_free_bytes;
    *total_b = (size_t)192 * 1000 * 1000 * 1000;
    return cudaSuccess;
}

cusparseStatus_t cusparseCreate(cusparseHandle_t *h)
{
    *h = new cusparseContext();
    return CUSPARSE_STATUS_SUCCESS;
}
cusparseStatus_t cusparseDestroy(cusparseHandle_t h)
{
    delete h;
    return CUSPARSE_STATUS_SUCCESS;
}
cusparseStatus_t cusparseSetStream(cusparseHandle_t, cudaStream_t)
{
    return CUSPARSE_STATUS_SUCCESS;
}
cusparseStatus_t cusparseCreateMatDescr(cusparseMatDescr_t *d)
{
    *d = new cusparseMatDescr();
    return CUSPARSE_STATUS_SUCCESS;
}
cusparseStatus_t cusparseDestroyMatDescr(cusparseMatDescr_t d)
{
    delete d;
    return CUSPARSE_STATUS_SUCCESS;
}
cusparseStatus_t cusparseSetMatType(cusparseMatDescr_t d, cusparseMatrixType_t t)
{
    d->type = (int)t;
    return CUSPARSE_STATUS_SUCCESS;
}
cusparseStatus_t cusparseSetMatIndexBase(cusparseMatDescr_t d, cusparseIndexBase_t b)
{
    d->base = (int)b;
    return CUSPARSE_STATUS_SUCCESS;
}

static void csrmv_cpu(int m, const double *alpha, const double *val,
                      const int *rowptr, const int *col, const double *x,
                      const double *beta, double *y)
{
    for (int i = 0; i < m; i++) {
        double sum = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; k++) sum += val[k] * x[col[k]];
        y[i] = (*beta == 0.0) ? *alpha * sum : *alpha * sum + *beta * y[i];
    }
}

cusparseStatus_t cusparseDcsrmv(cusparseHandle_t, cusparseOperation_t, int m,
                                int, int, const double *alpha,
                                const cusparseMatDescr_t, const double *val,
                                const int *rowptr, const int *col,
                                const double *x, const double *beta, double *y)
{
    csrmv_cpu(m, alpha, val, rowptr, col, x, beta, y);
    return CUSPARSE_STATUS_SUCCESS;
}
cusparseStatus_t cusparseDcsrmv_mp(cusparseHandle_t, cusparseOperation_t, int m,
                                   int, int, const double *alpha,
                                   const cusparseMatDescr_t, const double *val,
                                   const int *rowptr, const int *col,
                                   const double *x, const double *beta, double *y)
{
    csrmv_cpu(m, alpha, val, rowptr, col, x, beta, y);
    return CUSPARSE_STATUS_SUCCESS;
}

} /* extern "C" */

int csr5_kernel(int m, int, int, double *, double *csrVal, int *csrRowPtr,
                int *csrColIndex, double *x, double *, double *y)
{
    for (int i = 0; i < m; i++) {
        double sum = 0.0;
        for (int k = csrRowPtr[i]; k < csrRowPtr[i + 1]; k++)
            sum += csrVal[k] * x[csrColIndex[k]];
        y[i] = sum;
    }
    return 0;
}

/* C entry points for ctypes. */
extern "C" {
void ref_set_free_bytes(unsigned long long b) { g_free_bytes = (size_t)b; }
int ref_get_row_from_index(int n, long long *a, long long idx)
{
    return get_row_from_index(n, a, idx);
}
int ref_spMV_mgpu_baseline(int m, int n, long long nnz, double *alpha,
                           double *val, long long *rowptr, int *col, double *x,
                           double *beta, double *y, int ngpu)
{
    return spMV_mgpu_baseline(m, n, nnz, alpha, val, rowptr, col, x, beta, y, ngpu);
}
int ref_spMV_mgpu_v1(int m, int n, long long nnz, double *alpha, double *val,
                     long long *rowptr, int *col, double *x, double *beta,
                     double *y, int ngpu, int kernel)
{
    return spMV_mgpu_v1(m, n, nnz, alpha, val, rowptr, col, x, beta, y, ngpu, kernel);
}
/* The reference's spMV_mgpu_v2 has no return statement
 * (SparseBLAS/src/dspmv_mgpu_v2.cu:207); its value is discarded here. */
void ref_spMV_mgpu_v2(int m, int n, long long nnz, double *alpha, double *val,
                      long long *rowptr, int *col, double *x, double *beta,
                      double *y, int ngpu, int kernel, long long nb, int q)
{
    (void)spMV_mgpu_v2(m, n, nnz, alpha, val, rowptr, col, x, beta, y, ngpu,
                       kernel, nb, q);
}
}
