// k_vector.cu — K1: vector CSR SpMV, V lanes per row (V = 2..32).
//
// Replaces cusparseDcsrmv (SparseBLAS/src/dspmv_mgpu_v1.cu:200-204,
// src/dspmv_mgpu_baseline.cu:163-167).  A warp takes chunks of rows; in a
// chunk a group of V lanes owns one row at a time, reads its col/val with
// coalesced streaming loads (V consecutive nnz per step), gathers x through
// the read-only path and reduces with warp shuffles (xor butterfly: the order
// is fixed for a given V), with several rows' loads in flight per group
// (vector_chunk).  Good for regular matrices whose row lengths are close to
// V; long rows serialise on one group.
#include "../sbb_internal.h"
#include "common.cuh"
#include "spmv_device.cuh"

namespace sbb {

namespace {

constexpr int VT = 256;  // threads per CTA

// Warp w of the grid takes chunks w, w + W, ... of CR rows (W = all warps).
template <typename PT, typename ACC, int V>
__global__ void __launch_bounds__(VT)
vector_kernel(int m, int n, const int *__restrict__ rowptr, const int *__restrict__ col,
              const typename PT::V *__restrict__ val, const typename PT::V *__restrict__ x,
              double *__restrict__ y, double alpha, double beta, unsigned *status)
{
    constexpr int CR = VectorShape<V>::CR;
    static_assert(CR == vector_chunk_rows(V, V < 4 ? V : 4), "host and device chunk sizes differ");
    const int warps = gridDim.x * (VT / 32);
    const int chunks = (int)(((long long)m + CR - 1) / CR);
    const uint64_t stream = l2_evict_first();
    unsigned bad = 0;
    for (int c = blockIdx.x * (VT / 32) + (threadIdx.x >> 5); c < chunks; c += warps)
        vector_chunk<PT, ACC, V>(c * CR, m, n, rowptr, col, val, x, y, alpha, beta, stream, bad);
    if (bad) atomicOr(status, ST_BAD_COL);
}

template <typename PT, typename ACC>
void launch_vector_t(const CsrView &A, int V, double alpha, const typename PT::V *x,
                     double beta, double *y, unsigned *status, cudaStream_t s)
{
    if (A.m <= 0) return;
    const auto *val = static_cast<const typename PT::V *>(A.val);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int CR = vector_chunk_rows(V, V < 4 ? V : 4);  // VectorShape<V>::CR
    long long need = (((long long)A.m + CR - 1) / CR * 32 + VT - 1) / VT;  // a warp per chunk
    int grid = (int)(need < (long long)sms * 64 ? need : (long long)sms * 64);
#define SBB_VL(W)                                                                     \
    case W:                                                                           \
        vector_kernel<PT, ACC, W><<<grid, VT, 0, s>>>(A.m, A.n, A.rowptr, A.col, val, \
                                                      x, y, alpha, beta, status);     \
        break;
    hook_start(s);
    switch (V) {
        SBB_VL(2) SBB_VL(4) SBB_VL(8) SBB_VL(16) SBB_VL(32)
    default: break;
    }
    hook_stop(s);
#undef SBB_VL
}

}  // namespace

void launch_vector(const CsrView &A, int V, double alpha, const double *x, double beta,
                   double *y, unsigned *status, cudaStream_t s)
{
    launch_vector_t<ProdF64, AccF64>(A, V, alpha, x, beta, y, status, s);
}

void launch_vector_f32(const CsrView &A, int V, double alpha, const float *x, double beta,
                       double *y, unsigned *status, cudaStream_t s)
{
    launch_vector_t<ProdF32, AccF32>(A, V, alpha, x, beta, y, status, s);
}

}  // namespace sbb
