// k_batch.cu — many SpMVs of uneven sizes in a few persistent launches.
//
// The reference runs tasks from a host pool with an OpenMP thread per GPU
// and q streams each (SparseBLAS/src/dspmv_mgpu_v2.cu:73-188).  Here each
// kernel family of the batch (vector-CSR classes, the merge-path class, the
// tiled class) has one persistent kernel and one device work queue: every
// matrix of the family contributes work units - row chunks, warp segments or
// groups of kBatchTileGroup tiles - and the warps of the family's grid claim
// kBatchClaim consecutive units per queue access (one atomic on one counter)
// until the queue is empty.  The families' kernels run side by side (parallel
// branches of one stream or graph); a kernel holds only its family's code, so
// it gets the register budget and occupancy that code needs.  A unit runs
// exactly the device code the standalone kernel runs for it
// (spmv_device.cuh, tiled_device.cuh), and the carries and empty rows of every
// merge/tiled matrix are then finished by one fix-up launch with the
// standalone fix-up's arithmetic, so every matrix's y is bit-identical to a
// standalone launch with the same class.  A tiled unit is copied into shared
// memory with one TMA bulk copy; while a warp reduces a unit, the copy of the
// next unit of its claim is in flight, and the x values of each tile are
// gathered before the previous tile is reduced.
#include "../sbb_internal.h"
#include "common.cuh"
#include "spmv_device.cuh"
#include "tiled_device.cuh"

namespace sbb {

namespace {

constexpr int BT = 256;  // threads per CTA
constexpr int BW = BT / 32;
constexpr int SEG = 32 * kBatchIpt;
constexpr uint32_t TBB = (uint32_t)tile_bytes_of(kBatchSigma, 8);
constexpr int TG = kBatchTileGroup;
static_assert(TBB % 16 == 0, "bulk copies move multiples of 16 bytes");

// Per class kernel: dynamic shared memory per warp (merge: a segment's
// staging; tiled: two unit slots) and the CTAs per SM its register budget
// aims at.  The vector families spill a few dozen bytes at 64 registers;
// at 3 CTAs per SM they do not, but the 512-matrix batch ran slower (4.85
// vs 4.73 ms).
template <int FAM> struct FamShape {  // vector families
    static constexpr size_t kWarpBytes = 0;
    static constexpr int MINB = 4;
};
template <> struct FamShape<kFamMerge> {
    static constexpr size_t kWarpBytes =
        (sizeof(double) * SEG + sizeof(int) * (SEG + 1) + 127) / 128 * 128;
    static constexpr int MINB = 4;
};
template <> struct FamShape<kFamTiled> {
    static constexpr size_t kWarpBytes = 2 * (size_t)TG * TBB;
    static constexpr int MINB = 3;  // 80 registers: the tile path does not spill
};
template <int FAM> constexpr size_t fam_smem() { return BW * FamShape<FAM>::kWarpBytes; }

template <int FAM> __device__ __forceinline__ unsigned char *warp_smem()
{
    extern __shared__ __align__(128) unsigned char s_dyn[];
    return s_dyn + (size_t)(threadIdx.x >> 5) * FamShape<FAM>::kWarpBytes;
}

// A vector-class unit: vsteps consecutive chunks of CR rows (kBatchVectorU
// rows of each lane group in flight: the batch kernel's register budget).
template <int V>
__device__ __forceinline__ void vector_unit(const BatchMat &M, int local, unsigned &bad)
{
    constexpr int U = kBatchVectorU;
    constexpr int CR = VectorShape<V, U>::CR;
    static_assert(CR == vector_chunk_rows(V, U), "host and device chunk sizes differ");
    const uint64_t stream = l2_evict_first();
    const long long r0 = (long long)local * CR * M.vsteps;
    for (int s = 0; s < M.vsteps && r0 + (long long)CR * s < M.m; ++s)
        vector_chunk<ProdF64, AccF64, V, U>((int)(r0 + (long long)CR * s), M.m, M.n, M.rowptr,
                                            M.col, static_cast<const double *>(M.val), M.x, M.y,
                                            M.alpha, M.beta, stream, bad);
}

__device__ __forceinline__ int find_matrix(const long long *unit0, int nmat, long long u)
{
    int lo = 0, hi = nmat - 1;  // last i with unit0[i] <= u
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(unit0 + mid) <= u)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Units of matrix i relative to the claim start u0: first (negative when the
// matrix began before the claim) and last (clamped to the claim's n units).
// A matrix has fewer than 2^31 units, so both fit an int.
struct ClaimSpan {
    int first, last;
};
__device__ __forceinline__ ClaimSpan claim_span(const long long *unit0, int i, long long u0, int n)
{
    const long long a = __ldg(unit0 + i) - u0, b = __ldg(unit0 + i + 1) - u0;
    return ClaimSpan{(int)a, (int)(b < n ? b : n)};
}

template <int FAM>
__global__ void __launch_bounds__(BT, FamShape<FAM>::MINB)
batch_kernel(const BatchMat *__restrict__ mats, int nmat, const long long *__restrict__ unit0,
             long long total, unsigned long long *queue, unsigned *status)
{
    constexpr bool kTiled = FAM == kFamTiled;
    __shared__ __align__(8) uint64_t bars[kTiled ? BW : 1][2];
    const int lane = threadIdx.x & 31;
    uint32_t bar0 = 0;
    if constexpr (kTiled) {
        bar0 = smem_u32(&bars[threadIdx.x >> 5][0]);
        if (lane == 0) {
            mbar_init(bar0, 1);
            mbar_init(bar0 + 8, 1);
            mbar_fence_init();
        }
        __syncwarp();
    }
    // lane 0: copy the tiles of unit `unit` of MM into slot `sl`
    auto issue = [&](const BatchMat &MM, int unit, int sl) {
        if (lane == 0) {
            const int t0 = unit * TG;
            const int nt = MM.tiles - t0 < TG ? MM.tiles - t0 : TG;
            const uint32_t bytes = (uint32_t)nt * TBB;
            mbar_expect_tx(bar0 + 8 * sl, bytes);
            bulk_g2s(smem_u32(warp_smem<FAM>() + sl * TG * TBB), MM.blob + (size_t)t0 * TBB, bytes,
                     bar0 + 8 * sl, evict_first_policy());
        }
    };
    uint32_t phases = 0u;  // bit s: parity of slot s's next phase
    unsigned bad = 0, timeout = 0;
    int pre_k = -1;  // claim position whose tile copy is in flight (into slot pre_s)
    int pre_s = 0;
    while (!timeout) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(queue, 1ull);
        c = __shfl_sync(0xffffffffu, c, 0);
        const long long u0 = (long long)c * kBatchClaim;
        if (u0 >= total) break;
        const int n = (int)(total - u0 < kBatchClaim ? total - u0 : kBatchClaim);
        int i = find_matrix(unit0, nmat, u0);
        ClaimSpan sp = claim_span(unit0, i, u0, n);
        for (int k = 0; k < n; ++k) {
            while (k >= sp.last) {  // units are in matrix order
                ++i;
                sp = claim_span(unit0, i, u0, n);
            }
            const BatchMat &M = mats[i];
            const int local = k - sp.first;
            if constexpr (FAM == kFamVectorNarrow) {
                if (M.cls == 0)
                    vector_unit<4>(M, local, bad);
                else
                    vector_unit<8>(M, local, bad);
            } else if constexpr (FAM == kFamVectorWide) {
                if (M.cls == 2)
                    vector_unit<16>(M, local, bad);
                else
                    vector_unit<32>(M, local, bad);
            } else if constexpr (FAM == kFamMerge) {
                unsigned char *wsm = warp_smem<FAM>();
                merge_segment<ProdF64, AccF64, kBatchIpt>(
                    local, M.n, M.rowptr, M.col, static_cast<const double *>(M.val), M.x, M.y,
                    M.alpha, M.beta, M.tile_row, M.tile_nnz, M.carry_val, status,
                    reinterpret_cast<double *>(wsm),
                    reinterpret_cast<int *>(wsm + sizeof(double) * SEG), l2_evict_last(),
                    l2_evict_first());
            } else {
                int cur = 0;
                if (pre_k == k)
                    cur = pre_s;
                else
                    issue(M, local, 0);  // nothing is in flight here
                pre_k = -1;
                // start the copy of the claim's next unit
                if (k + 1 < n) {
                    int i2 = i;
                    ClaimSpan s2 = sp;
                    while (k + 1 >= s2.last) {
                        ++i2;
                        s2 = claim_span(unit0, i2, u0, n);
                    }
                    issue(mats[i2], k + 1 - s2.first, cur ^ 1);
                    pre_k = k + 1;
                    pre_s = cur ^ 1;
                }
                const int t0 = local * TG;
                const int nt = M.tiles - t0 < TG ? M.tiles - t0 : TG;
                if (!mbar_wait(bar0 + 8 * cur, (phases >> cur) & 1u)) {
                    // let the copies still in flight land (bounded) before the
                    // warp leaves: this unit's and, if started, the next one's
                    mbar_wait(bar0 + 8 * cur, (phases >> cur) & 1u);
                    if (pre_k >= 0) mbar_wait(bar0 + 8 * pre_s, (phases >> pre_s) & 1u);
                    timeout = 1;
                    break;
                }
                phases ^= 1u << cur;  // flips only once the copy has landed
                const uint64_t keep = l2_evict_last(), streaming = l2_evict_first();
                const unsigned char *tb = warp_smem<FAM>() + cur * TG * TBB;
                double xv[kBatchSigma], xn[kBatchSigma];
                tile_gather<ProdF64, kBatchSigma>(t0, M.tiles, M.nnz, tb, M.x, keep, xv);
#pragma unroll 1
                for (int j = 0; j < nt; ++j) {
                    const int t = t0 + j;
                    const unsigned char *tj = tb + j * TBB;
                    if (j + 1 < nt)  // the next tile's x, in flight during this reduce
                        tile_gather<ProdF64, kBatchSigma>(t + 1, M.tiles, M.nnz, tj + TBB, M.x,
                                                          keep, xn);
                    tile_reduce<ProdF64, AccF64, kBatchSigma>(t, tj, M.ne, xv, M.y, M.alpha,
                                                              M.beta, M.carry_val, streaming, 0.0,
                                                              0.0, nullptr);
#pragma unroll
                    for (int q = 0; q < kBatchSigma; ++q) xv[q] = xn[q];
                }
                __syncwarp();  // every lane is done with the slot before it is refilled
            }
        }
    }
    if constexpr (kTiled) {
        if (timeout && lane == 0) atomicOr(status, ST_TIMEOUT);
    }
    if (bad) atomicOr(status, ST_BAD_COL);
}

// The standalone fix-up (k_fixup.cu) and empty-row pass (k_tiled.cu) over
// every merge/tiled matrix of the batch at once, with the same arithmetic:
// blocks [0, short_blocks) take one global carry slot per thread (single
// carries), the next n_long_runs blocks one long run each (more than
// kWarpRunMax slots), the next warp_blocks eight short runs each (a warp a
// run), the rest the empty rows of tiled matrices.
__global__ void __launch_bounds__(kFixupThreads)
batch_fixup_kernel(const BatchMat *__restrict__ mats, BatchFix F, long long total_slots,
                   int short_blocks, int warp_blocks)
{
    if (blockIdx.x < short_blocks) {
        const long long g = (long long)blockIdx.x * kFixupThreads + threadIdx.x;
        if (g >= total_slots) return;
        const int k = find_matrix(F.tile0, F.nfix, g);
        const BatchMat &M = mats[__ldg(F.mat + k)];
        const int t = (int)(g - __ldg(F.tile0 + k)), T = M.tiles;
        const int *crow = M.crow;
        const int r = crow[t];
        if (r >= M.m) return;
        if ((t > 0 && crow[t - 1] == r) || (t + 1 < T && crow[t + 1] == r)) return;
        fixup_single(M.y, r, M.alpha, M.carry_val[t]);
        return;
    }
    const int j = blockIdx.x - short_blocks;
    if (j >= F.n_long_runs && j < F.n_long_runs + warp_blocks) {
        const int q = F.n_long_runs + (j - F.n_long_runs) * (kFixupThreads / 32) + (threadIdx.x >> 5);
        if (q >= F.n_runs) return;
        const BatchMat &M = mats[__ldg(F.run_mat + q)];
        const int first = __ldg(F.run_first + q), len = __ldg(F.run_len + q);
        const double sum = fixup_run_warp(M.carry_val, first, len);
        if ((threadIdx.x & 31) == 0) fixup_single(M.y, M.crow[first], M.alpha, sum);
        return;
    }
    if (j < F.n_long_runs) {
        __shared__ double s[kFixupThreads];
        const BatchMat &M = mats[__ldg(F.run_mat + j)];
        const int first = __ldg(F.run_first + j), len = __ldg(F.run_len + j);
        s[threadIdx.x] = fixup_partial(M.carry_val, first, len, threadIdx.x);
        __syncthreads();
        for (int w = kFixupThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) fixup_single(M.y, M.crow[first], M.alpha, s[0]);
        return;
    }
    const long long e = (long long)(j - F.n_long_runs - warp_blocks) * kFixupThreads + threadIdx.x;
    if (e >= F.n_empty) return;
    const BatchMat &M = mats[__ldg(F.empty_mat + e)];
    double *yp = M.y + __ldg(F.empty_row + e);
    *yp = M.beta == 0.0 ? 0.0 : M.beta * *yp;
}

}  // namespace

template <int FAM> static int max_ctas()
{
    int blocks = 0;
    cudaFuncSetAttribute(batch_kernel<FAM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)fam_smem<FAM>());
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, batch_kernel<FAM>, BT, fam_smem<FAM>());
    return blocks;
}

int batch_max_ctas_per_sm(int fam)
{
    switch (fam) {
    case 0: return max_ctas<0>();
    case 1: return max_ctas<1>();
    case 2: return max_ctas<2>();
    default: return max_ctas<3>();
    }
}

template <int FAM>
static void launch_fam(const BatchMat *mats, int nmat, const long long *unit0, long long total,
                       unsigned long long *queue, unsigned *status, int grid, cudaStream_t s)
{
    batch_kernel<FAM><<<grid, BT, fam_smem<FAM>(), s>>>(mats, nmat, unit0, total, queue, status);
}

void launch_batch(int fam, const BatchMat *mats, int nmat, const long long *unit0,
                  long long total, unsigned long long *queue, unsigned *status, int grid,
                  cudaStream_t s)
{
    if (total <= 0 || nmat <= 0) return;
    switch (fam) {
    case 0: launch_fam<0>(mats, nmat, unit0, total, queue, status, grid, s); break;
    case 1: launch_fam<1>(mats, nmat, unit0, total, queue, status, grid, s); break;
    case 2: launch_fam<2>(mats, nmat, unit0, total, queue, status, grid, s); break;
    default: launch_fam<3>(mats, nmat, unit0, total, queue, status, grid, s); break;
    }
}

void launch_batch_fixup(const BatchMat *mats, const BatchFix &F, long long total_slots,
                        cudaStream_t s)
{
    if (total_slots <= 0 && F.n_empty <= 0) return;
    const int short_blocks = (int)((total_slots + kFixupThreads - 1) / kFixupThreads);
    const int empty_blocks = (F.n_empty + kFixupThreads - 1) / kFixupThreads;
    const int warp_blocks = (F.n_runs - F.n_long_runs + kFixupThreads / 32 - 1) / (kFixupThreads / 32);
    batch_fixup_kernel<<<short_blocks + F.n_long_runs + warp_blocks + empty_blocks, kFixupThreads, 0, s>>>(
        mats, F, total_slots, short_blocks, warp_blocks);
}

}  // namespace sbb
