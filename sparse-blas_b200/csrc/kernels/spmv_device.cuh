// spmv_device.cuh — per-row (K1) and per-segment (K2) device code shared by
// the standalone kernels and the batched persistent kernel, so a matrix gets
// bit-identical results whichever way it is run.
#pragma once
#include <climits>

#include "../sbb_internal.h"
#include "common.cuh"

namespace sbb {

constexpr int kLongRow = 32;  // K2: rows longer than this in a segment are summed by the warp

// One row per group of V lanes (K1).  All 32 lanes of the warp call this
// together (inactive groups pass active = false) so the full-mask shuffles
// see every lane; the reduction order is fixed for a given V.
template <typename PT, typename ACC, int V>
__device__ __forceinline__ void vector_row(int row, bool active, int n, const int *__restrict__ rowptr,
                                           const int *__restrict__ col,
                                           const typename PT::V *__restrict__ val,
                                           const typename PT::V *__restrict__ x,
                                           double *__restrict__ y, double alpha, double beta,
                                           unsigned &bad)
{
    const int lane = threadIdx.x & (V - 1);
    int lo = 0, hi = 0;
    if (active) {
        lo = __ldg(rowptr + row);
        hi = __ldg(rowptr + row + 1);
    }
    ACC acc;
    acc.zero();
    int k = lo + lane;
    // two independent loads in flight per lane
    for (; k + V < hi; k += 2 * V) {
        int c0 = ld_stream(col + k), c1 = ld_stream(col + k + V);
        auto v0 = ld_stream(val + k), v1 = ld_stream(val + k + V);
        auto x0 = gather_x(x, c0, n, bad), x1 = gather_x(x, c1, n, bad);
        acc.add(PT::make(v0, x0));
        acc.add(PT::make(v1, x1));
    }
    if (k < hi) acc.add(PT::make(ld_stream(val + k), gather_x(x, ld_stream(col + k), n, bad)));
    double sum = acc.get();
#pragma unroll
    for (int o = V / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, V);
    if (active && lane == 0) {
        double *yp = y + row;
        __stcs(yp, axpby(alpha, sum, beta, yp));
    }
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of the products s_p[lo..hi) by the whole warp (fixed order: lane-strided
// partial sums, then an xor butterfly).
template <typename ACC, typename P>
__device__ __forceinline__ double warp_range_sum(const P *s_p, int lo, int hi, int lane)
{
    ACC acc;
    acc.zero();
    for (int i = lo + lane; i < hi; i += 32) acc.add(s_p[i]);
    return warp_sum(acc.get());
}

template <typename PT, typename ACC, int IPT>
__device__ __forceinline__ void merge_segment(
    int w, int n, const int *__restrict__ rowptr, const int *__restrict__ col,
    const typename PT::V *__restrict__ val, const typename PT::V *__restrict__ x,
    double *__restrict__ y, double alpha, double beta, const int *__restrict__ tile_row,
    const int *__restrict__ tile_nnz, double *__restrict__ carry_val, unsigned *status,
    typename PT::P *s_p, int *s_re, uint64_t keep, uint64_t streaming)
{
    using P = typename PT::P;
    using V = typename PT::V;
    constexpr int SEG = 32 * IPT;
    const int lane = threadIdx.x & 31;
    const int r0 = __ldg(tile_row + w), r1 = __ldg(tile_row + w + 1);
    const int k0 = __ldg(tile_nnz + w), k1 = __ldg(tile_nnz + w + 1);
    const int nrows = r1 - r0, nz = k1 - k0;
    if (nrows < 0 || nz < 0 || nrows + nz > SEG) {  // corrupt coordinates
        if (lane == 0) atomicOr(status, ST_BAD_TILE);
        return;
    }
    unsigned bad = 0;
    // y of the first 32 rows, early: the beta*y read then is off the tail
    double ypre = 0.0;
    if (beta != 0.0 && lane < nrows) ypre = ld_y(y + r0 + lane, streaming);

    // 1. row ends and products (every load of the lane in flight together)
    int cc[IPT];
    V vv[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const int i = lane + 32 * j;
        if (i < nz) {
            cc[j] = ld_stream(col + k0 + i);
            vv[j] = ld_stream(val + k0 + i);
        }
    }
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const int i = lane + 32 * j;
        if (i < nrows) s_re[i] = __ldg(rowptr + r0 + 1 + i);
    }
    V xv[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const int i = lane + 32 * j;
        if (i < nz) {
            if ((unsigned)cc[j] < (unsigned)n) {
                xv[j] = ld_keep(x + cc[j], keep);
            } else {
                bad = 1u;
                xv[j] = V(0);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const int i = lane + 32 * j;
        if (i < nz) s_p[i] = PT::make(vv[j], xv[j]);
    }
    if (bad) atomicOr(status, ST_BAD_COL);
    __syncwarp();

    // 2. complete rows r0 .. r1-1: lane per row, long rows by the warp
    for (int b = 0; b < nrows; b += 32) {
        const int i = b + lane;
        int lo = 0, hi = 0;
        if (i < nrows) {
            lo = i == 0 ? 0 : s_re[i - 1] - k0;  // row r0 may have started before k0
            hi = s_re[i] - k0;
            // a valid row pointer keeps 0 <= lo <= hi <= nz; clamping makes a
            // corrupt one harmless (wrong sums, no out-of-range reads)
            lo = min(max(lo, 0), nz);
            hi = min(max(hi, lo), nz);
        }
        const bool is_long = hi - lo > kLongRow;
        if (i < nrows && !is_long) {
            ACC acc;
            acc.zero();
            for (int k = lo; k < hi; ++k) acc.add(s_p[k]);
            double *yp = y + r0 + i;
            double v = alpha * acc.get();
            if (beta != 0.0) v += beta * (b == 0 ? ypre : ld_y(yp, streaming));
            st_y(yp, v, streaming);
        }
        unsigned longs = __ballot_sync(0xffffffffu, i < nrows && is_long);
        while (longs) {
            const int src = __ffs(longs) - 1;
            longs &= longs - 1;
            const int llo = __shfl_sync(0xffffffffu, lo, src);
            const int lhi = __shfl_sync(0xffffffffu, hi, src);
            const double s = warp_range_sum<ACC>(s_p, llo, lhi, lane);
            if (lane == src) {
                double *yp = y + r0 + i;
                double v = alpha * s;
                if (beta != 0.0) v += beta * (b == 0 ? ypre : ld_y(yp, streaming));
                st_y(yp, v, streaming);
            }
        }
    }
    // 3. carry: the part of row r1 inside this segment
    const int clo = nrows > 0 ? min(max(s_re[nrows - 1] - k0, 0), nz) : 0;
    const double c = warp_range_sum<ACC>(s_p, clo, nz, lane);
    if (lane == 0) carry_val[w] = c;
    __syncwarp();  // shared memory is reused by this warp's next segment
}


}  // namespace sbb
