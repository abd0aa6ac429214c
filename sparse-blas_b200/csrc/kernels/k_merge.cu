// k_merge.cu — K2: merge-path CSR SpMV (FP64 and FP32-storage forms).
//
// The m row ends and the nnz values of A are merged into one list of m+nnz
// items (Merrill & Garland, SC'16) and cut into equal segments of 32*IPT
// items, one per warp, so every warp does the same amount of work whatever
// the row lengths.  This replaces the reference's across-GPU nnz split
// (SparseBLAS/src/dspmv_mgpu_v1.cu:60-94) and the cusparseDcsrmv_mp call
// (:206) with an across-warp split on one B200; the split is computed on the
// device (merge_partition_kernel) and is bit-identical to the CPU
// restatement.
//
// Per warp segment (rows r0..r1-1 complete, row r1 open, nnz k0..k1-1):
//   1. the row ends and the products val*x of the segment's nnz go to the
//      warp's shared memory: coalesced streaming loads of col/val, every
//      load of the lane issued before any is used, x gathered through the
//      read-only path with an L2 evict-last hint;
//   2. each lane sums one row at a time straight from shared memory
//      (consecutive lanes own consecutive rows, so the y writes coalesce);
//      rows with more than kLongRow nnz in the segment are summed by the
//      whole warp (strided partial sums, xor-butterfly reduction);
//   3. the part of row r1 inside the segment is the segment's carry, summed
//      by the whole warp and added afterwards in a fixed order (k_fixup.cu).
// The reduction order depends only on the matrix and IPT, never on timing.
#include <climits>

#include "../sbb_internal.h"
#include "common.cuh"
#include "spmv_device.cuh"

namespace sbb {

namespace {

constexpr int NT = kMergeThreads;  // threads per CTA
constexpr int WPB = NT / 32;       // warps (segments in flight) per CTA

// Merge-path search on the global row pointer for one diagonal.
__device__ __forceinline__ void path_search(const int *rowptr, int m, long long nnz,
                                            int base, long long d, int &row, int &nz)
{
    long long lo = d - nnz > 0 ? d - nnz : 0;
    long long hi = d < m ? d : m;
    while (lo < hi) {
        long long pivot = (lo + hi) >> 1;
        if ((long long)__ldg(rowptr + pivot + 1) - base <= d - pivot - 1)
            lo = pivot + 1;
        else
            hi = pivot;
    }
    row = (int)lo;
    nz = (int)(base + d - lo);
}

// base / nnz come from the host (rowptr[0] and rowptr[m] of a valid matrix),
// so even a corrupt row pointer cannot move a segment outside [base, base+nnz).
__global__ void merge_partition_kernel(const int *__restrict__ rowptr, int m, int base,
                                       long long nnz, long long items, int tiles,
                                       int *__restrict__ tile_row,
                                       int *__restrict__ tile_nnz)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > tiles) return;
    long long total = (long long)m + nnz;
    long long d = (long long)p * items;
    if (d > total) d = total;
    int r, z;
    path_search(rowptr, m, nnz, base, d, r, z);
    tile_row[p] = r;
    tile_nnz[p] = z;
}

// One warp per segment; in the persistent form (queue non-null) a fixed grid
// whose warps claim `item` consecutive segments at a time from a device work
// queue (queue[0], an atomicAdd head, zeroed again by the fix-up after the
// kernel) until the segments run out.  Which warp computes a segment does
// not change its arithmetic, so results are the same as one warp per
// segment.
template <int IPT> struct MergeShape {
    static constexpr int MINB = IPT <= 8 ? 4 : 2;  // CTAs per SM the launch bounds aim at
};

template <typename PT, typename ACC, int IPT>
__global__ void __launch_bounds__(NT, MergeShape<IPT>::MINB)
merge_kernel(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
             const typename PT::V *__restrict__ val, const typename PT::V *__restrict__ x,
             double *__restrict__ y, double alpha, double beta, const int *__restrict__ tile_row,
             const int *__restrict__ tile_nnz, double *__restrict__ carry_val, int tiles,
             unsigned *status, unsigned *queue, int item)
{
    using P = typename PT::P;
    constexpr int SEG = 32 * IPT;
    __shared__ P s_p[WPB][SEG];
    __shared__ int s_re[WPB][SEG + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t keep = l2_evict_last(), streaming = l2_evict_first();
    if (queue) {
        for (;;) {
            unsigned first = 0;
            if (lane == 0) first = atomicAdd(queue, (unsigned)item);
            first = __shfl_sync(0xffffffffu, first, 0);
            if (first >= (unsigned)tiles) break;
            const int end = (int)min((unsigned long long)first + item, (unsigned long long)tiles);
            for (int w = (int)first; w < end; ++w)
                merge_segment<PT, ACC, IPT>(w, n, rowptr, col, val, x, y, alpha, beta, tile_row,
                                            tile_nnz, carry_val, status, s_p[warp], s_re[warp],
                                            keep, streaming);
        }
        return;
    }
    for (int w = blockIdx.x * WPB + warp; w < tiles; w += gridDim.x * WPB)
        merge_segment<PT, ACC, IPT>(w, n, rowptr, col, val, x, y, alpha, beta, tile_row,
                                    tile_nnz, carry_val, status, s_p[warp], s_re[warp], keep,
                                    streaming);
}

template <typename PT, typename ACC, int IPT>
void launch_merge_t(const CsrView &A, const MergeScratch &S, double alpha,
                    const typename PT::V *x, double beta, double *y, unsigned *status,
                    cudaStream_t s)
{
    const auto *val = static_cast<const typename PT::V *>(A.val);
    if (S.tiles > 0) {
        long long blocks = (S.tiles + WPB - 1) / WPB;
        const bool queued = S.queue && S.persistent_ctas > 0 && S.persistent_ctas < blocks;
        int grid = (int)(queued ? S.persistent_ctas : blocks);
        hook_start(s);
        merge_kernel<PT, ACC, IPT><<<grid, NT, 0, s>>>(A.n, A.rowptr, A.col, val, x, y, alpha, beta,
                                                       S.tile_row, S.tile_nnz, S.carry_val,
                                                       S.tiles, status, queued ? S.queue : nullptr,
                                                       S.queue_item > 0 ? S.queue_item : 1);
        hook_stop(s);
        launch_fixup(A.m, S.tile_row + 1, S.carry_val, S.tiles, *S.runs, alpha, y,
                     queued ? S.queue : nullptr, s, S.runs_count);
    }
}

template <typename PT, typename ACC>
void dispatch_merge(const CsrView &A, int ipt, const MergeScratch &S, double alpha,
                    const typename PT::V *x, double beta, double *y, unsigned *status,
                    cudaStream_t s)
{
    switch (ipt) {
    case 4: launch_merge_t<PT, ACC, 4>(A, S, alpha, x, beta, y, status, s); break;
    case 6: launch_merge_t<PT, ACC, 6>(A, S, alpha, x, beta, y, status, s); break;
    case 8: launch_merge_t<PT, ACC, 8>(A, S, alpha, x, beta, y, status, s); break;
    case 12: launch_merge_t<PT, ACC, 12>(A, S, alpha, x, beta, y, status, s); break;
    default: break;
    }
}

template <typename PT, typename ACC, int IPT>
int occupancy_t()
{
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, merge_kernel<PT, ACC, IPT>, NT, 0);
    return blocks;
}

}  // namespace

int merge_ipt_supported(int ipt)
{
    return ipt == 4 || ipt == 6 || ipt == 8 || ipt == 12;
}

long long merge_items_per_tile(int ipt) { return 32LL * ipt; }

int merge_max_ctas_per_sm(int ipt, bool f32)
{
#define SBB_OCC(I)                                                              \
    case I:                                                                     \
        return f32 ? occupancy_t<ProdF32, AccF32, I>() : occupancy_t<ProdF64, AccF64, I>();
    switch (ipt) {
        SBB_OCC(4) SBB_OCC(6) SBB_OCC(8) SBB_OCC(12)
    default: return 0;
    }
#undef SBB_OCC
}

void launch_merge_partition(const int *rowptr, int m, int base, long long nnz, long long items,
                            int tiles, int *tile_row, int *tile_nnz, cudaStream_t s)
{
    int n = tiles + 1;
    merge_partition_kernel<<<(n + 255) / 256, 256, 0, s>>>(rowptr, m, base, nnz, items, tiles,
                                                           tile_row, tile_nnz);
}

void launch_merge(const CsrView &A, int ipt, const MergeScratch &S, double alpha,
                  const double *x, double beta, double *y, unsigned *status, cudaStream_t s)
{
    dispatch_merge<ProdF64, AccF64>(A, ipt, S, alpha, x, beta, y, status, s);
}

void launch_merge_f32(const CsrView &A, int ipt, const MergeScratch &S, double alpha,
                      const float *x, double beta, double *y, unsigned *status,
                      cudaStream_t s)
{
    dispatch_merge<ProdF32, AccF32>(A, ipt, S, alpha, x, beta, y, status, s);
}

}  // namespace sbb
