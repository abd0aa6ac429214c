// spmv_device.cuh — per-row (K1) and per-segment (K2) device code shared by
// the standalone kernels and the batched persistent kernel, so a matrix gets
// bit-identical results whichever way it is run.
#pragma once
#include <climits>

#include "../sbb_internal.h"
#include "common.cuh"

namespace sbb {

constexpr int kLongRow = 32;  // K2: rows longer than this in a segment are summed by the warp

// K1 chunk shape: 32/V rows per sub-step, U sub-steps in flight together, at
// most 32 rows (CR) per chunk.
template <int V, int U_ = (V < 4 ? V : 4)> struct VectorShape {
    static constexpr int RPW = 32 / V;
    static constexpr int U = U_;
    static constexpr int CR = RPW * U < 32 ? RPW * U : 32;
};

// K1: one chunk of CR consecutive rows [r0, r0 + CR) by one warp, V lanes per
// row.  Lane l first loads rowptr[r0+l], rowptr[r0+l+1] and y[r0+l]
// (coalesced, all in flight together).  Row q of the chunk is then reduced by
// lane group q % (32/V) in sub-step q / (32/V); the U sub-steps run together,
// their loads issued before any of them is summed, so a warp keeps U row
// fetches per group in flight instead of one (U = UU changes only which loads
// are in flight together, never a sum, so a caller picks it for its register
// budget).  Per row the order of the sum is fixed for a given V: lane i of
// the group adds the products of nnz lo+i, lo+i+V, lo+i+2V, ... in that order,
// then the group's partial sums meet in an xor butterfly.  Lane l ends with
// row r0+l's sum and writes y[r0+l] (one coalesced store per chunk).  All 32
// lanes call this together (the shuffles use the full mask).
template <typename PT, typename ACC, int V, int UU = (V < 4 ? V : 4)>
__device__ __forceinline__ void vector_chunk(int r0, int m, int n, const int *__restrict__ rowptr,
                                             const int *__restrict__ col,
                                             const typename PT::V *__restrict__ val,
                                             const typename PT::V *__restrict__ x,
                                             double *__restrict__ y, double alpha, double beta,
                                             uint64_t stream, unsigned &bad)
{
    using S = VectorShape<V, UU>;
    constexpr int RPW = S::RPW, U = S::U, CR = S::CR;
    const int lane = threadIdx.x & 31, g = lane / V, li = lane & (V - 1);
    const bool in = lane < CR && lane < m - r0;  // r0 < m: no overflow near INT_MAX
    int rlo = 0, rhi = 0;
    double yv = 0.0;
    if (in) {
        rlo = __ldg(rowptr + r0 + lane);
        rhi = __ldg(rowptr + r0 + lane + 1);
        if (beta != 0.0) yv = ld_y(y + r0 + lane, stream);
    }
    double out = 0.0;
    // nnz indices are unsigned: with nnz up to 2^31 - 1 a lane's index runs
    // to at most nnz - 1 + V (< 2^32), past the int range but never wrapping
#pragma unroll 1
    for (int j0 = 0; j0 * RPW < CR; j0 += U) {
        unsigned k[U], hi[U];
        ACC acc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int q = (j0 + u) * RPW + g;
            k[u] = (unsigned)__shfl_sync(0xffffffffu, rlo, q) + (unsigned)li;
            hi[u] = (unsigned)__shfl_sync(0xffffffffu, rhi, q);
            acc[u].zero();
        }
        for (;;) {
            bool any = false;
            int c[U];
            typename PT::V v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (k[u] < hi[u]) {
                    c[u] = ld_stream(col + k[u]);
                    v[u] = ld_stream(val + k[u]);
                    any = true;
                }
            }
            if (!any) break;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (k[u] < hi[u]) {
                    acc[u].mac(v[u], gather_x(x, c[u], n, bad));
                    k[u] += V;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            double sum = acc[u].get();
#pragma unroll
            for (int o = V / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, V);
            // row q = (j0+u)*RPW + g lands in lane q
            const double r = __shfl_sync(0xffffffffu, sum, (lane % RPW) * V);
            if (lane / RPW == j0 + u) out = r;
        }
    }
    if (in) st_y(y + r0 + lane, y_update(alpha, out, beta, yv), stream);
}

// Carry fix-up arithmetic shared by the standalone fix-up (k_fixup.cu) and
// the batch fix-up (k_batch.cu): a single carry is added as fma(alpha, c, y[r]); a
// run of at most kWarpRunMax carries is summed by one warp (lane i: slots i,
// i + 32, ... in order, then an xor butterfly); a longer run by kFixupThreads
// threads (thread i: slots i, i + kFixupThreads, ... in order) and then a
// shared-memory tree.  Which of the two a run gets depends only on its
// length, so both fix-ups sum every run in the same order.
constexpr int kFixupThreads = 256;
__device__ __forceinline__ void fixup_single(double *y, int r, double alpha, double c)
{
    y[r] = __fma_rn(alpha, c, y[r]);
}
__device__ __forceinline__ double fixup_partial(const double *cval, int first, int len, int i)
{
    double acc = 0.0;
    for (; i < len; i += kFixupThreads) acc += cval[first + i];
    return acc;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of a run of at most kWarpRunMax carries by the calling warp (every lane
// gets it).
__device__ __forceinline__ double fixup_run_warp(const double *cval, int first, int len)
{
    double acc = 0.0;
    for (int i = threadIdx.x & 31; i < len; i += 32) acc += cval[first + i];
    return warp_sum(acc);
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
            const double v = y_update(alpha, acc.get(), beta,
                                      beta == 0.0 ? 0.0 : (b == 0 ? ypre : ld_y(yp, streaming)));
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
                const double v = y_update(alpha, s, beta,
                                          beta == 0.0 ? 0.0 : (b == 0 ? ypre : ld_y(yp, streaming)));
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
