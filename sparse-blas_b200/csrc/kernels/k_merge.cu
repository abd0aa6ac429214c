// k_merge.cu — K2: merge-path CSR SpMV (FP64 and FP32-storage forms).
//
// The m row ends and the nnz values of A are merged into one list of m+nnz
// items (Merrill & Garland, SC'16) and cut into equal tiles of
// kMergeThreads*IPT items, so every CTA does the same work whatever the row
// lengths.  This replaces the reference's across-GPU nnz split
// (SparseBLAS/src/dspmv_mgpu_v1.cu:60-94) and the cusparseDcsrmv_mp call
// (:206) with an across-SM split on one B200.
//
// Per tile:
//   1. stage the row ends of the tile's rows and the products val*x of its
//      nnz in shared memory (coalesced 128-bit streaming loads of col/val,
//      x gathered through the read-only path);
//   2. each thread walks IPT merge items, closing rows as it meets their ends;
//   3. a block-wide segmented scan (keyed by row) hands each thread the
//      partial sum of the row it starts in;
//   4. completed rows are written with y = alpha*sum + beta*y, coalesced;
//   5. the partial sum of the row still open at the tile end is the tile's
//      carry, added by merge_fixup_kernel in tile order (deterministic).
// The reduction order depends only on the matrix and IPT, never on timing.
#include <climits>

#include "../sbb_internal.h"
#include "common.cuh"

namespace sbb {

namespace {

constexpr int NT = kMergeThreads;
constexpr int WARPS = NT / 32;

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

__global__ void merge_partition_kernel(const int *__restrict__ rowptr, int m,
                                       long long items, int tiles,
                                       int *__restrict__ tile_row,
                                       int *__restrict__ tile_nnz)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > tiles) return;
    int base = __ldg(rowptr);
    long long nnz = (long long)__ldg(rowptr + m) - base;
    long long total = (long long)m + nnz;
    long long d = (long long)p * items;
    if (d > total) d = total;
    int r, z;
    path_search(rowptr, m, nnz, base, d, r, z);
    tile_row[p] = r;
    tile_nnz[p] = z;
}

// Segmented inclusive scan over the CTA's threads, keyed by row.  Keys are
// non-decreasing in thread order, so equal neighbouring keys mean one run.
struct KeyVal {
    int k;
    double v;
};

__device__ __forceinline__ KeyVal block_seg_scan(KeyVal kv, KeyVal *s_warp)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int ku = __shfl_up_sync(0xffffffffu, kv.k, o);
        double vu = __shfl_up_sync(0xffffffffu, kv.v, o);
        if (lane >= o && ku == kv.k) kv.v += vu;
    }
    if (lane == 31) s_warp[warp] = kv;
    __syncthreads();
    if (warp == 0) {
        KeyVal w = lane < WARPS ? s_warp[lane] : KeyVal{INT_MAX, 0.0};
#pragma unroll
        for (int o = 1; o < WARPS; o <<= 1) {
            int ku = __shfl_up_sync(0xffffffffu, w.k, o);
            double vu = __shfl_up_sync(0xffffffffu, w.v, o);
            if (lane >= o && ku == w.k) w.v += vu;
        }
        if (lane < WARPS) s_warp[lane] = w;
    }
    __syncthreads();
    if (warp > 0) {
        KeyVal prev = s_warp[warp - 1];
        if (prev.k == kv.k) kv.v = prev.v + kv.v;
    }
    return kv;
}

template <typename PT, typename ACC, int IPT>
__device__ __forceinline__ void merge_tile(
    int tile, int m, int n, const int *__restrict__ rowptr,
    const int *__restrict__ col, const typename PT::V *__restrict__ val,
    const typename PT::V *__restrict__ x, double *__restrict__ y, double alpha,
    double beta, const int *__restrict__ tile_row, const int *__restrict__ tile_nnz,
    int *__restrict__ carry_row, double *__restrict__ carry_val, unsigned *status,
    bool vec_ok, unsigned char *smem)
{
    using P = typename PT::P;
    using V = typename PT::V;
    constexpr int ITEMS = NT * IPT;
    // shared layout: [ITEMS] 8-byte slots (products at [0, nnz), row sums at
    // [nnz, nnz+rows)), [ITEMS+1] row ends, [WARPS] scan partials,
    // [NT] thread carries.
    P *s_prod = reinterpret_cast<P *>(smem);
    double *s_slot = reinterpret_cast<double *>(smem);
    int *s_rowend = reinterpret_cast<int *>(smem + sizeof(double) * ITEMS);
    KeyVal *s_warp = reinterpret_cast<KeyVal *>(smem + sizeof(double) * ITEMS +
                                                sizeof(int) * (ITEMS + 1 + 1));
    double *s_carry = reinterpret_cast<double *>(s_warp + WARPS);

    const int tid = threadIdx.x;
    const int r0 = __ldg(tile_row + tile), r1 = __ldg(tile_row + tile + 1);
    const int k0 = __ldg(tile_nnz + tile), k1 = __ldg(tile_nnz + tile + 1);
    const int nrows = r1 - r0, nz = k1 - k0;
    if (nrows < 0 || nz < 0 || nrows + nz > ITEMS) {  // corrupt coordinates
        if (tid == 0) atomicOr(status, ST_BAD_TILE);
        return;
    }
    unsigned bad = 0;

    // 1a. row ends of rows r0 .. r1-1, sentinel after the last one
    for (int i = tid; i < nrows; i += NT) s_rowend[i] = __ldg(rowptr + r0 + 1 + i);
    if (tid == 0) s_rowend[nrows] = INT_MAX;

    // 1b. products of nnz k0 .. k1-1, in groups of 4 aligned to 16 bytes
    if (vec_ok) {
        const int g0 = k0 & ~3;
        for (int g = g0 + 4 * tid; g < k1; g += 4 * NT) {
            if (g >= k0 && g + 4 <= k1) {
                int4 c = ld_stream(reinterpret_cast<const int4 *>(col + g));
                V v[4];
                if constexpr (sizeof(V) == 8) {
                    double2 a = ld_stream(reinterpret_cast<const double2 *>(val + g));
                    double2 b = ld_stream(reinterpret_cast<const double2 *>(val + g + 2));
                    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
                } else {
                    float4 a = ld_stream(reinterpret_cast<const float4 *>(val + g));
                    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
                }
                V x0 = gather_x(x, c.x, n, bad), x1 = gather_x(x, c.y, n, bad);
                V x2 = gather_x(x, c.z, n, bad), x3 = gather_x(x, c.w, n, bad);
                P *dst = s_prod + (g - k0);
                dst[0] = PT::make(v[0], x0);
                dst[1] = PT::make(v[1], x1);
                dst[2] = PT::make(v[2], x2);
                dst[3] = PT::make(v[3], x3);
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    int k = g + j;
                    if (k >= k0 && k < k1) {
                        V xv = gather_x(x, ld_stream(col + k), n, bad);
                        s_prod[k - k0] = PT::make(ld_stream(val + k), xv);
                    }
                }
            }
        }
    } else {
        for (int k = k0 + tid; k < k1; k += NT) {
            V xv = gather_x(x, ld_stream(col + k), n, bad);
            s_prod[k - k0] = PT::make(ld_stream(val + k), xv);
        }
    }
    if (bad) atomicOr(status, ST_BAD_COL);
    __syncthreads();

    // 2. thread-level merge walk
    const int total = nrows + nz;
    const int dl = min(tid * IPT, total);
    const int dl_end = min(dl + IPT, total);
    int lo = max(dl - nz, 0), hi = min(dl, nrows);
    while (lo < hi) {
        int pivot = (lo + hi) >> 1;
        if (s_rowend[pivot] <= k0 + dl - pivot - 1)
            lo = pivot + 1;
        else
            hi = pivot;
    }
    int ri = lo, ki = dl - lo;
    const int ri_start = ri;
    // Products and row sums share s_slot: this thread's row sums go to
    // s_slot[nz + row], never over a product some thread still has to read.
    ACC acc;
    acc.zero();
#pragma unroll
    for (int it = 0; it < IPT; ++it) {
        if (dl + it < dl_end) {
            if (k0 + ki >= s_rowend[ri]) {  // row ri ends before nnz ki
                s_slot[nz + ri] = acc.get();
                acc.zero();
                ++ri;
            } else {
                acc.add(s_prod[ki]);
                ++ki;
            }
        }
    }
    __syncthreads();

    // 3. carry-in from the threads before (segmented scan keyed by row)
    KeyVal kv{r0 + ri, acc.get()};
    KeyVal inc = block_seg_scan(kv, s_warp);
    s_carry[tid] = inc.v;
    __syncthreads();
    if (ri > ri_start && tid > 0) s_slot[nz + ri_start] += s_carry[tid - 1];
    __syncthreads();

    // 4. completed rows r0 .. r1-1
    for (int i = tid; i < nrows; i += NT) {
        double *yp = y + r0 + i;
        __stcs(yp, axpby(alpha, s_slot[nz + i], beta, yp));
    }
    // 5. tile carry for row r1 (the row still open at the tile end)
    if (tid == NT - 1) {
        carry_row[tile] = inc.k;
        carry_val[tile] = inc.v;
    }
}

template <typename PT, typename ACC, int IPT>
__global__ void __launch_bounds__(NT)
merge_kernel(int m, int n, const int *__restrict__ rowptr, const int *__restrict__ col,
             const typename PT::V *__restrict__ val, const typename PT::V *__restrict__ x,
             double *__restrict__ y, double alpha, double beta,
             const int *__restrict__ tile_row, const int *__restrict__ tile_nnz,
             int *__restrict__ carry_row, double *__restrict__ carry_val, int tiles,
             unsigned *queue, unsigned *status, int vec_ok)
{
    extern __shared__ __align__(16) unsigned char smem[];
    if (queue == nullptr) {
        merge_tile<PT, ACC, IPT>(blockIdx.x, m, n, rowptr, col, val, x, y, alpha, beta,
                                 tile_row, tile_nnz, carry_row, carry_val, status,
                                 vec_ok != 0, smem);
        return;
    }
    // persistent form: tiles are taken from a device work queue
    __shared__ int s_next;
    for (;;) {
        if (threadIdx.x == 0) s_next = (int)atomicAdd(queue, 1u);
        __syncthreads();
        int tile = s_next;
        __syncthreads();
        if (tile >= tiles) break;
        merge_tile<PT, ACC, IPT>(tile, m, n, rowptr, col, val, x, y, alpha, beta,
                                 tile_row, tile_nnz, carry_row, carry_val, status,
                                 vec_ok != 0, smem);
        __syncthreads();
    }
}

// Adds the tile carries to the rows they belong to.  The carries of one row
// come from consecutive tiles; the first tile of each run sums the run in
// tile order and applies alpha once.  Also rearms the persistent work queue.
__global__ void merge_fixup_kernel(int m, const int *__restrict__ carry_row,
                                   const double *__restrict__ carry_val, int tiles,
                                   double alpha, double *__restrict__ y, unsigned *queue)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0 && queue != nullptr) queue[0] = 0u;
    if (t >= tiles) return;
    int r = carry_row[t];
    if (r >= m) return;
    if (t > 0 && carry_row[t - 1] == r) return;
    double s = carry_val[t];
    for (int u = t + 1; u < tiles && carry_row[u] == r; ++u) s += carry_val[u];
    y[r] += alpha * s;
}

template <int IPT>
constexpr size_t merge_smem_bytes()
{
    return sizeof(double) * NT * IPT + sizeof(int) * (NT * IPT + 2) + sizeof(KeyVal) * WARPS +
           sizeof(double) * NT;
}

template <typename PT, typename ACC, int IPT>
void launch_merge_t(const CsrView &A, const MergeScratch &S, double alpha,
                    const typename PT::V *x, double beta, double *y, unsigned *status,
                    cudaStream_t s)
{
    auto kern = merge_kernel<PT, ACC, IPT>;
    constexpr size_t smem = merge_smem_bytes<IPT>();
    // per function and device; cheap enough to set on every launch
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const auto *val = static_cast<const typename PT::V *>(A.val);
    int vec_ok = ((reinterpret_cast<uintptr_t>(A.col) | reinterpret_cast<uintptr_t>(val)) & 15) == 0;
    if (S.tiles > 0) {
        int grid = S.persistent_ctas > 0 ? S.persistent_ctas : S.tiles;
        hook_start(s);
        kern<<<grid, NT, smem, s>>>(A.m, A.n, A.rowptr, A.col, val, x, y, alpha, beta,
                                    S.tile_row, S.tile_nnz, S.carry_row, S.carry_val,
                                    S.tiles, S.persistent_ctas > 0 ? S.queue : nullptr,
                                    status, vec_ok);
        hook_stop(s);
        merge_fixup_kernel<<<(S.tiles + 255) / 256, 256, 0, s>>>(
            A.m, S.carry_row, S.carry_val, S.tiles, alpha, y,
            S.persistent_ctas > 0 ? S.queue : nullptr);
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
    case 16: launch_merge_t<PT, ACC, 16>(A, S, alpha, x, beta, y, status, s); break;
    default: break;
    }
}

template <typename PT, typename ACC, int IPT>
int occupancy_t()
{
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, merge_kernel<PT, ACC, IPT>, NT,
                                                  merge_smem_bytes<IPT>());
    return blocks;
}

}  // namespace

int merge_ipt_supported(int ipt)
{
    return ipt == 4 || ipt == 6 || ipt == 8 || ipt == 12 || ipt == 16;
}

int merge_max_ctas_per_sm(int ipt, bool f32)
{
    auto set = [](auto kern, size_t smem) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    };
#define SBB_OCC(I)                                                                    \
    case I:                                                                           \
        if (f32) {                                                                    \
            set(merge_kernel<ProdF32, AccF32, I>, merge_smem_bytes<I>());             \
            return occupancy_t<ProdF32, AccF32, I>();                                 \
        }                                                                             \
        set(merge_kernel<ProdF64, AccF64, I>, merge_smem_bytes<I>());                 \
        return occupancy_t<ProdF64, AccF64, I>();
    switch (ipt) {
        SBB_OCC(4) SBB_OCC(6) SBB_OCC(8) SBB_OCC(12) SBB_OCC(16)
    default: return 0;
    }
#undef SBB_OCC
}

void launch_carry_fixup(int m, const int *carry_row, const double *carry_val, int tiles,
                        double alpha, double *y, cudaStream_t s)
{
    if (tiles > 0)
        merge_fixup_kernel<<<(tiles + 255) / 256, 256, 0, s>>>(m, carry_row, carry_val, tiles,
                                                               alpha, y, nullptr);
}

void launch_merge_partition(const int *rowptr, int m, long long items, int tiles,
                            int *tile_row, int *tile_nnz, cudaStream_t s)
{
    int n = tiles + 1;
    merge_partition_kernel<<<(n + 255) / 256, 256, 0, s>>>(rowptr, m, items, tiles, tile_row,
                                                           tile_nnz);
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
