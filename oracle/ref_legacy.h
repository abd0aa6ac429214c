/*
 * ref_legacy.h — force-included when the reference's host drivers are compiled
 * into oracle/_ref (TEST INFRASTRUCTURE ONLY).
 *
 * The reference calls the legacy cuSPARSE csrmv/csrmv_mp entry points
 * (SparseBLAS/src/dspmv_mgpu_v1.cu:200-210), which CUDA 11 removed from
 * cusparse.h.  This header only declares them, with the legacy signature,
 * so the unmodified driver sources compile; ref_shim.cpp defines them.
 */
#ifndef SBB_REF_LEGACY_H
#define SBB_REF_LEGACY_H
#include <cusparse.h>
#ifdef __cplusplus
extern "C" {
#endif
cusparseStatus_t cusparseDcsrmv(cusparseHandle_t handle, cusparseOperation_t op,
                                int m, int n, int nnz, const double *alpha,
                                const cusparseMatDescr_t descr,
                                const double *val, const int *rowptr,
                                const int *col, const double *x,
                                const double *beta, double *y);
cusparseStatus_t cusparseDcsrmv_mp(cusparseHandle_t handle, cusparseOperation_t op,
                                   int m, int n, int nnz, const double *alpha,
                                   const cusparseMatDescr_t descr,
                                   const double *val, const int *rowptr,
                                   const int *col, const double *x,
                                   const double *beta, double *y);
#ifdef __cplusplus
}
#endif
#endif
