// k_util.cu — small device kernels around the SpMV: row-pointer narrowing
// and validation, row-length statistics, and the boundary-piece sums used by
// the drop-in entry points.
#include "../sbb_internal.h"
#include "common.cuh"

namespace sbb {

namespace {

// int64 row pointer (the drop-in's host format) -> int32 device format
// (the reference rebases to int the same way, SparseBLAS/src/dspmv_mgpu_v1.cu:125-133).
// Flags a pointer that is not monotone, leaves [0, nnz], or does not start
// at 0 / end at nnz.
__global__ void rowptr_narrow_kernel(const long long *__restrict__ src, int *__restrict__ dst,
                                     int m, long long nnz, unsigned *status)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    bool bad = false;
    for (; i <= m; i += stride) {
        long long v = src[i];
        if (v < 0 || v > nnz) bad = true;
        if (i < m && v > src[i + 1]) bad = true;
        if (i == 0 && v != 0) bad = true;
        if (i == m && v != nnz) bad = true;
        dst[i] = (int)v;
    }
    if (bad) atomicOr(status, ST_BAD_ROWPTR);
}

__global__ void rowptr_check_kernel(const int *__restrict__ rp, int m, int nnz,
                                    unsigned *status)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    bool bad = false;
    for (; i <= m; i += stride) {
        int v = rp[i];
        if (v < 0 || v > nnz) bad = true;
        if (i < m && v > rp[i + 1]) bad = true;
        if (i == 0 && v != 0) bad = true;
        if (i == m && v != nnz) bad = true;
    }
    if (bad) atomicOr(status, ST_BAD_ROWPTR);
}

__global__ void row_stats_kernel(const int *__restrict__ rp, int m, int *out)
{
    int mx = 0, empty = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (long long)gridDim.x * blockDim.x) {
        int len = rp[i + 1] - rp[i];
        mx = max(mx, len);
        empty += (len == 0);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        empty += __shfl_xor_sync(0xffffffffu, empty, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, mx);
        if (empty) atomicAdd(out + 1, empty);
    }
}

// One CTA per boundary piece: sum of val*x over [lo, hi), tree-reduced in a
// fixed order.
__global__ void pieces_kernel(const long long *__restrict__ lo, const long long *__restrict__ hi,
                              const int *__restrict__ col, const double *__restrict__ val,
                              const double *__restrict__ x, int n, double *__restrict__ out,
                              unsigned *status)
{
    __shared__ double s[256];
    const int p = blockIdx.x;
    unsigned bad = 0;
    double sum = 0.0;
    for (long long k = lo[p] + threadIdx.x; k < hi[p]; k += 256)
        sum = __dadd_rn(sum, __dmul_rn(ld_stream(val + k), gather_x(x, ld_stream(col + k), n, bad)));
    s[threadIdx.x] = sum;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[p] = s[0];
    if (bad) atomicOr(status, ST_BAD_COL);
}

int grid_for(long long work, int tpb)
{
    long long g = (work + tpb - 1) / tpb;
    if (g < 1) g = 1;
    if (g > 148 * 16) g = 148 * 16;
    return (int)g;
}

}  // namespace

void launch_rowptr_narrow(const long long *src, int *dst, int m, long long nnz,
                          unsigned *status, cudaStream_t s)
{
    rowptr_narrow_kernel<<<grid_for((long long)m + 1, 256), 256, 0, s>>>(src, dst, m, nnz, status);
}

void launch_rowptr_check(const int *rp, int m, int nnz, unsigned *status, cudaStream_t s)
{
    rowptr_check_kernel<<<grid_for((long long)m + 1, 256), 256, 0, s>>>(rp, m, nnz, status);
}

void launch_row_stats(const int *rowptr, int m, int *out, cudaStream_t s)
{
    if (m <= 0) return;
    row_stats_kernel<<<grid_for(m, 256), 256, 0, s>>>(rowptr, m, out);
}

void launch_pieces(const long long *lo, const long long *hi, int npieces, const int *col,
                   const double *val, const double *x, int n, double *out, unsigned *status,
                   cudaStream_t s)
{
    if (npieces > 0) pieces_kernel<<<npieces, 256, 0, s>>>(lo, hi, col, val, x, n, out, status);
}

}  // namespace sbb
