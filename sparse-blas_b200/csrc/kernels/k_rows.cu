// k_rows.cu — K4: CSR row blocks streamed into shared memory by TMA.
//
// A kernel of its own beside the three that replace the reference's
// cusparseDcsrmv / cusparseDcsrmv_mp / CSR5 calls (SparseBLAS/src/
// dspmv_mgpu_v1.cu:195-217): the rows are cut into blocks of at most 32
// consecutive rows and at most NMAX nnz (256 or 384, per plan), and a row
// longer than NMAX into pieces of NMAX nnz (the row-blocking idea of CSR-Adaptive,
// Greathouse & Daga, SC'14).  The blocks are fixed per plan and use the
// caller's CSR arrays as they are: there is no copy of the matrix.
//
// Per block, one warp:
//   * its columns, values and row pointers arrive in shared memory by 1-D TMA
//     bulk copies (cp.async.bulk + mbarrier, evict-first, bounded waits) of
//     the 16-byte-aligned middle of each range; the ragged ends (at most
//     three 4-byte or one 8-byte element per end) come by plain loads, so no
//     copy ever reads outside the ranges the matrix owns;
//   * products val*x are formed in nnz order, 32 consecutive nnz per warp
//     step (x gathered through the read-only path with an L2 evict-last hint,
//     every gather of a lane issued before any is used) and written back in
//     place (FP64) or beside the values (FP32 storage);
//   * lane i sums row i of the block from shared memory, left to right, and
//     writes y (one coalesced store per block); rows longer than kWarpRow
//     nnz are summed by the whole warp (lane-strided partial sums, then a
//     butterfly);
//   * a piece of a long row is summed by the whole warp; the last piece of a
//     row writes y, the others leave a carry that the ordered fix-up
//     (k_fixup.cu) adds afterwards - no atomics, bit-reproducible.
// Warps are persistent and take blocks round-robin, double-buffered: the
// copies of a warp's next block are in flight while it reduces the current
// one.
#include <stdint.h>
#include <stdlib.h>

#include <cub/cub.cuh>

#include "../sbb_internal.h"
#include "common.cuh"
#include "spmv_device.cuh"
#include "tiled_device.cuh"

namespace sbb {

namespace {

constexpr int RW = 4;              // warps per CTA
// Block shapes (nnz per block and per piece of a long row; CTAs per SM the
// launch bounds aim at): a plan picks one when it is built.
struct RowsShape {
    int nmax, minb;
};
constexpr RowsShape kRowsShapes[] = {{256, 8}, {384, 5}};
constexpr int kRowsDefaultShape = 1;
constexpr int kRowsPerBlock = 32;  // rows per block (one per lane)
constexpr int kWarpRow = 16;       // rows of a block longer than this: summed by the warp
constexpr int kNbuf = 2;           // blocks in shared memory per warp

// Shared-memory slot of one block.  Element k of a range sits at
// (its byte address mod 16) / size + (k - first), so the 16-byte-aligned
// middle of the range lands on a 16-byte boundary for the bulk copy.
template <typename V, int NMAX> struct RowsSlot {
    static constexpr int CI = NMAX + 4;                              // columns (int)
    static constexpr int VN = NMAX + 16 / (int)sizeof(V);            // values (V)
    static constexpr int RI = kRowsPerBlock + 1 + 3 + 4;             // row pointers (int)
    static constexpr int PN = sizeof(V) == 8 ? 0 : NMAX;             // FP32: products (double)
    static constexpr uint32_t C_OFF = 0;
    static constexpr uint32_t V_OFF = C_OFF + CI * 4;
    static constexpr uint32_t R_OFF = V_OFF + ((VN * (int)sizeof(V) + 15) / 16) * 16;
    static constexpr uint32_t P_OFF = R_OFF + RI * 4;
    static constexpr uint32_t BYTES = P_OFF + PN * 8;
    static_assert(C_OFF % 16 == 0 && V_OFF % 16 == 0 && R_OFF % 16 == 0 && P_OFF % 16 == 0 &&
                      BYTES % 16 == 0,
                  "16-byte aligned slot regions");
};

// The 16-byte-aligned middle [lo, hi) of the byte range of elements [k0, k1)
// of array a (element size e); lo >= hi when there is none.
struct Span {
    uintptr_t first;  // byte address of element k0
    uintptr_t lo, hi;
};
__device__ __forceinline__ Span span_of(const void *a, long long k0, long long k1, int e)
{
    Span s;
    s.first = reinterpret_cast<uintptr_t>(a) + (uintptr_t)k0 * e;
    const uintptr_t last = reinterpret_cast<uintptr_t>(a) + (uintptr_t)k1 * e;
    s.lo = (s.first + 15) & ~(uintptr_t)15;
    s.hi = last & ~(uintptr_t)15;
    return s;
}

// Block descriptor: x = first row, y = rows (>= 1), or 0 for the last piece
// of a long row (it writes y), or -1 for another piece (it leaves a carry);
// z, w = nnz range [k0, k1) (absolute offsets, as the row pointer holds them).
template <typename PT, int NMAX, int MINB>
__global__ void __launch_bounds__(RW * 32, MINB)
rows_kernel(int nblk, const int4 *__restrict__ desc, const int *__restrict__ rp,
            const int *__restrict__ col, const typename PT::V *__restrict__ val,
            const typename PT::V *__restrict__ x, double *__restrict__ y, double alpha,
            double beta, double *__restrict__ carry_val, unsigned *status, int first_wait,
            int m, int base, int nnz)
{
    using V = typename PT::V;
    using S = RowsSlot<V, NMAX>;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[RW][kNbuf];
    // columns were range-checked when the plan was built; a failed check
    // leaves the status bit set and no block runs
    if (*reinterpret_cast<volatile unsigned *>(status) & ST_BAD_COL) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *wbuf = smem + (size_t)warp * kNbuf * S::BYTES;
    const uint32_t bar_base = smem_u32(&bars[warp][0]);
    const int W = gridDim.x * RW;
    int b = blockIdx.x * RW + warp;
    uint64_t pol = 0;

    // The three ranges of block d as 4-byte words: g = 0 columns, 1 values,
    // 2 row pointers (none for a piece of a long row).
    struct Range {
        const unsigned *a;
        long long k0, n;
        uint32_t off;  // slot region
    };
    auto range_of = [&](int4 d, int g) {
        constexpr int VW = (int)sizeof(V) / 4;  // words per value
        Range r;
        r.a = g == 0 ? reinterpret_cast<const unsigned *>(col)
                     : (g == 1 ? reinterpret_cast<const unsigned *>(val)
                               : reinterpret_cast<const unsigned *>(rp));
        r.k0 = g == 0 ? (long long)d.z : (g == 1 ? (long long)d.z * VW : (long long)d.x);
        r.n = g == 0 ? (long long)d.w - d.z
                     : (g == 1 ? ((long long)d.w - d.z) * VW : (d.y > 0 ? (long long)d.y + 1 : 0));
        r.off = g == 0 ? S::C_OFF : (g == 1 ? S::V_OFF : S::R_OFF);
        return r;
    };
    // The range of the matrix's own words an array may be read in (the
    // view: nnz from `base`, rows 0..m), as byte addresses.
    auto view_of = [&](int g, uintptr_t &vlo, uintptr_t &vhi) {
        constexpr int VW = (int)sizeof(V) / 4;
        if (g == 0) {
            vlo = reinterpret_cast<uintptr_t>(col + base);
            vhi = reinterpret_cast<uintptr_t>(col + base + (long long)nnz);
        } else if (g == 1) {
            vlo = reinterpret_cast<uintptr_t>(val + base);
            vhi = vlo + (uintptr_t)nnz * VW * 4;
        } else {
            vlo = reinterpret_cast<uintptr_t>(rp);
            vhi = reinterpret_cast<uintptr_t>(rp + (long long)m + 1);
        }
    };
    // Whether range g of block d, widened outwards to 16-byte boundaries,
    // stays inside the view: then one bulk copy brings all of it (true for
    // every block but those at the ends of the matrix).
    auto widens = [&](const Range &r, const Span &sp, int g) {
        uintptr_t vlo, vhi;
        view_of(g, vlo, vhi);
        const uintptr_t last = sp.first + (uintptr_t)r.n * 4;
        return (sp.first & ~(uintptr_t)15) >= vlo && ((last + 15) & ~(uintptr_t)15) <= vhi;
    };
    // Lanes 0-2 each bulk-copy one range of block d into slot sl (widened to
    // 16-byte boundaries where it may be, else its aligned middle); lane 0
    // first arms the barrier with their total.  Called by the whole warp.
    auto issue = [&](int4 d, int sl) {
        const uint32_t bar = bar_base + 8 * sl;
        unsigned char *dst = wbuf + sl * S::BYTES;
        Range r{nullptr, 0, 0, 0};
        uintptr_t lo = 0;
        uint32_t bytes = 0;
        if (lane < 3) {
            r = range_of(d, lane);
            Span sp = span_of(r.a, r.k0, r.k0 + r.n, 4);
            if (r.n > 0 && widens(r, sp, lane)) {
                sp.lo = sp.first & ~(uintptr_t)15;
                sp.hi = (sp.first + (uintptr_t)r.n * 4 + 15) & ~(uintptr_t)15;
            }
            if (r.n > 0 && sp.hi > sp.lo) {
                bytes = (uint32_t)(sp.hi - sp.lo);
                lo = sp.lo;
            }
            r.off += (uint32_t)(sp.lo - (sp.first & ~(uintptr_t)15));
        }
        const uint32_t total = __shfl_sync(0xffffffffu, bytes, 0) +
                               __shfl_sync(0xffffffffu, bytes, 1) +
                               __shfl_sync(0xffffffffu, bytes, 2);
        if (lane == 0) mbar_expect_tx(bar, total);
        __syncwarp();  // armed before any copy can complete
        if (bytes)
            bulk_g2s(smem_u32(dst + r.off), reinterpret_cast<const void *>(lo), bytes, bar,
                     lane == 2 ? 0 : pol);
    };
    // Whether block d has a range that could not be widened (its ragged
    // ends then come by plain loads); uniform over the warp.
    auto needs_ragged = [&](int4 d) {
        bool need = false;
        if (lane < 3) {
            const Range r = range_of(d, lane);
            need = r.n > 0 && !widens(r, span_of(r.a, r.k0, r.k0 + r.n, 4), lane);
        }
        return __any_sync(0xffffffffu, need);
    };
    // Lanes 0-23: the words of block d outside the aligned middles (the
    // ragged ends), by plain loads into slot sl; eight lanes per range.
    // Lanes 0-3 of a group take the head (at most 3 words), lanes 4-7 the
    // tail; a range with no aligned middle (at most 7 words) is loaded by all
    // eight.
    auto ragged = [&](int4 d, int sl) {
        const int g = lane >> 3, l = lane & 7;
        if (g < 3) {
            const Range r = range_of(d, g);
            const Span sp = span_of(r.a, r.k0, r.k0 + r.n, 4);
            if (r.n > 0 && widens(r, sp, g)) return;  // the bulk copy brings all of it
            long long k = l;
            if (sp.hi > sp.lo) {
                const long long head = (long long)((sp.lo - sp.first) / 4);
                const long long tail0 = (long long)((sp.hi - sp.first) / 4);
                k = l >= 4 ? tail0 + (l - 4) : (l < head ? l : r.n);
            }
            if (k < r.n)
                reinterpret_cast<unsigned *>(wbuf + sl * S::BYTES + r.off)[(sp.first & 15) / 4 + k] =
                    __ldg(r.a + r.k0 + k);
        }
    };

    pol = evict_first_policy();
    if (lane == 0) {
        for (int sl = 0; sl < kNbuf; ++sl) mbar_init(bar_base + 8 * sl, 1);
        mbar_fence_init();
    }
    __syncwarp();
    for (int sl = 0; sl < kNbuf; ++sl)
        if (b + sl * W < nblk) issue(__ldg(desc + b + sl * W), sl);

    int polls = first_wait >= 0 && blockIdx.x == 0 && warp == 0 ? first_wait : kWaitPolls;
    uint32_t phases = 0u;
    const uint64_t keep = l2_evict_last(), streaming = l2_evict_first();
    int sl = 0;
    unsigned timeout = 0;
    int4 d = make_int4(0, 0, 0, 0);
    if (b < nblk) d = __ldg(desc + b);
    for (; b < nblk; b += W) {
        double yv = 0.0;
        if (beta != 0.0 && lane < d.y) yv = ld_y(y + d.x + lane, streaming);
        if (needs_ragged(d)) ragged(d, sl);
        int4 dn = make_int4(0, 0, 0, 0), df = make_int4(0, 0, 0, 0);
        if (b + W < nblk) dn = __ldg(desc + b + W);
        const bool more = b + kNbuf * W < nblk;
        if (more) df = __ldg(desc + b + kNbuf * W);
        if (!mbar_wait(bar_base + 8 * sl, (phases >> sl) & 1u, polls)) {
            timeout = 1;
            break;
        }
        polls = kWaitPolls;
        phases ^= 1u << sl;
        __syncwarp();  // the ragged ends written by other lanes are visible
        unsigned char *sb = wbuf + sl * S::BYTES;
        const int nz = d.w - d.z;
        const int *Cs = reinterpret_cast<const int *>(sb + S::C_OFF) +
                        (int)((reinterpret_cast<uintptr_t>(col + d.z) & 15) / 4);
        const V *Vs = reinterpret_cast<const V *>(sb + S::V_OFF) +
                      (int)((reinterpret_cast<uintptr_t>(val + d.z) & 15) / sizeof(V));
        double *Ps = sizeof(V) == 8 ? reinterpret_cast<double *>(const_cast<V *>(Vs))
                                    : reinterpret_cast<double *>(sb + S::P_OFF);
        // 1. products in nnz order: every x gather of the lane (up to
        // NMAX / 32) is issued before any product is formed
        constexpr int UM = NMAX / 32;
        int c[UM];
        V xv[UM];
#pragma unroll
        for (int u = 0; u < UM; ++u) {
            const int i = u * 32 + lane;
            if (i < nz) c[u] = Cs[i];
        }
#pragma unroll
        for (int u = 0; u < UM; ++u) {
            const int i = u * 32 + lane;
            if (i < nz) xv[u] = ld_keep(x + c[u], keep);
        }
#pragma unroll
        for (int u = 0; u < UM; ++u) {
            const int i = u * 32 + lane;
            if (i < nz) Ps[i] = PT::make(Vs[i], xv[u]);
        }
        __syncwarp();
        // 2. rows (lane i: row d.x + i) or the piece of a long row
        if (d.y > 0) {
            const int *Rs = reinterpret_cast<const int *>(sb + S::R_OFF) +
                            (int)((reinterpret_cast<uintptr_t>(rp + d.x) & 15) / 4);
            int lo = 0, hi = 0;
            if (lane < d.y) {
                lo = Rs[lane] - d.z;
                hi = Rs[lane + 1] - d.z;
            }
            const bool wide = hi - lo > kWarpRow;
            if (lane < d.y && !wide) {
                double acc = 0.0;
                for (int k = lo; k < hi; ++k) acc = __dadd_rn(acc, Ps[k]);
                st_y(y + d.x + lane, y_update(alpha, acc, beta, yv), streaming);
            }
            unsigned wides = __ballot_sync(0xffffffffu, lane < d.y && wide);
            while (wides) {
                const int src = __ffs(wides) - 1;
                wides &= wides - 1;
                const int llo = __shfl_sync(0xffffffffu, lo, src);
                const int lhi = __shfl_sync(0xffffffffu, hi, src);
                const double s = warp_range_sum<AccF64>(Ps, llo, lhi, lane);
                if (lane == src) st_y(y + d.x + lane, y_update(alpha, s, beta, yv), streaming);
            }
        } else {
            const double s = warp_range_sum<AccF64>(Ps, 0, nz, lane);
            if (lane == 0) {
                if (d.y == 0)
                    write_y(y + d.x, alpha, s, beta, streaming);
                else
                    carry_val[b] = s;
            }
        }
        // every lane is done with the slot, and its shared-memory writes are
        // ordered before the bulk copies that refill it
        fence_proxy_async();
        __syncwarp();
        if (more) issue(df, sl);
        sl = sl + 1 == kNbuf ? 0 : sl + 1;
        d = dn;
    }
    if (timeout) {
        // let every copy still in flight land (bounded) before the warp
        // leaves: block b in slot sl and the block queued after it
        for (int k = 0; k < kNbuf && b + k * W < nblk; ++k) {
            const int ss = (sl + k) % kNbuf;
            mbar_wait(bar_base + 8 * ss, (phases >> ss) & 1u);
        }
        if (lane == 0) atomicOr(status, ST_TIMEOUT);
    }
}

// ---- plan: the block list ---------------------------------------------------
// Rows are taken in groups of 32 (so blocks never straddle a group and the y
// stores of a block stay within one 256-byte row group); inside a group, rows
// are packed greedily into blocks of at most nmax nnz, and a row with
// more than nmax nnz becomes its own run of pieces.  One thread per
// group counts its blocks, a scan places them, a second pass writes them.
template <bool EMIT>
__global__ void rows_blocks_kernel(const int *__restrict__ rp, int m, int nmax,
                                   int *__restrict__ count,
                                   const int *__restrict__ offset, int4 *__restrict__ desc,
                                   int *__restrict__ carry_row)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long groups = ((long long)m + kRowsPerBlock - 1) / kRowsPerBlock;
    if (g >= groups) return;
    const int r0 = (int)(g * kRowsPerBlock);
    const int r1 = (int)min((long long)m, g * kRowsPerBlock + kRowsPerBlock);
    int out = EMIT ? offset[g] : 0;
    int start = r0, rows = 0, nz = 0;
    auto close = [&](int r_end) {
        if (EMIT) {
            desc[out] = make_int4(start, rows, rp[start], rp[r_end]);
            carry_row[out] = m;
        }
        ++out;
    };
    int lo = rp[r0];
    for (int r = r0; r < r1; ++r) {
        const int hi = rp[r + 1], len = hi - lo;
        if (len > nmax) {
            if (rows) close(r);
            for (long long k = lo; k < hi; k += nmax) {
                const long long k1 = min((long long)hi, k + nmax);
                if (EMIT) {
                    desc[out] = make_int4(r, k1 == hi ? 0 : -1, (int)k, (int)k1);
                    carry_row[out] = k1 == hi ? m : r;
                }
                ++out;
            }
            start = r + 1;
            rows = nz = 0;
        } else {
            if (rows && nz + len > nmax) {
                close(r);
                start = r;
                rows = nz = 0;
            }
            ++rows;
            nz += len;
        }
        lo = hi;
    }
    if (rows) close(r1);
    if (!EMIT) count[g] = out;
}

// Every column in [0, n): checked once when the plan is built.
__global__ void rows_col_check_kernel(const int *__restrict__ col, long long first, long long nnz,
                                      int n, unsigned *status)
{
    bool bad = false;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x)
        bad |= (unsigned)__ldg(col + first + k) >= (unsigned)n;
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status, ST_BAD_COL);
}

struct RowsPlan {
    int shape = kRowsDefaultShape;  // index into kRowsShapes
    int nblk = 0;
    int4 *desc = nullptr;
    int *carry_row = nullptr;
    double *carry_val = nullptr;
    CarryRuns runs;
};

int grid_of(long long work, int tpb)
{
    long long g = (work + tpb - 1) / tpb;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

template <typename PT, int NMAX, int MINB>
void launch_rows_n(const RowsPlan &R, const Plan *p, double alpha, const typename PT::V *x,
                   double beta, double *y, cudaStream_t s)
{
    using V = typename PT::V;
    auto kern = rows_kernel<PT, NMAX, MINB>;
    constexpr size_t smem = (size_t)RW * kNbuf * RowsSlot<V, NMAX>::BYTES;
    const LaunchShape ls = cached_launch_shape(kern, RW * 32, smem);
    const long long want = (R.nblk + RW - 1) / RW;
    const long long cap = (long long)ls.sms * ls.occ;
    const int grid = (int)(want < cap ? want : cap);
    hook_start(s);
    kern<<<grid, RW * 32, smem, s>>>(R.nblk, R.desc, p->rowptr, p->col,
                                     static_cast<const V *>(p->val), x, y, alpha, beta,
                                     R.carry_val, p->status, first_wait_budget(), p->m,
                                     p->base, p->nnz);
    hook_stop(s);
}

template <typename PT>
void launch_rows_t(const RowsPlan &R, const Plan *p, double alpha, const typename PT::V *x,
                   double beta, double *y, cudaStream_t s)
{
    static_assert(sizeof(kRowsShapes) / sizeof(kRowsShapes[0]) == 2, "one launch per shape");
    if (R.shape == 0)
        launch_rows_n<PT, kRowsShapes[0].nmax, kRowsShapes[0].minb>(R, p, alpha, x, beta, y, s);
    else
        launch_rows_n<PT, kRowsShapes[1].nmax, kRowsShapes[1].minb>(R, p, alpha, x, beta, y, s);
    launch_fixup(p->m, R.carry_row, R.carry_val, R.nblk, R.runs, alpha, y, nullptr, s);
}

}  // namespace

int rows_build(Plan *p, cudaStream_t s)
{
    auto *R = new RowsPlan();
    p->rows = R;
    // SBB_ROWS_SHAPE (0 or 1) overrides the default block shape
    if (const char *e = getenv("SBB_ROWS_SHAPE")) {
        const int v = atoi(e);
        if (v == 0 || v == 1) R->shape = v;
    }
    const int m = p->m;
    const long long groups = ((long long)m + kRowsPerBlock - 1) / kRowsPerBlock;
    auto al = [&](void **ptr, size_t bytes) {
        bytes = bytes ? bytes : 16;
        p->scratch_bytes += bytes;
        return dev_malloc_async(ptr, bytes, s) == cudaSuccess;
    };
    int *count = nullptr, *offset = nullptr;
    if (!al((void **)&count, sizeof(int) * (groups + 1)) ||
        !al((void **)&offset, sizeof(int) * (groups + 1))) {
        set_error("row-block plan: device allocation failed");
        return SBB_ERR_NOMEM;
    }
    // the columns are checked here, not in every SpMV
    if (p->nnz > 0)
        rows_col_check_kernel<<<grid_of(p->nnz, 256), 256, 0, s>>>(p->col, p->base, p->nnz, p->n,
                                                                   p->status);
    SBB_CUDA(cudaMemsetAsync(count + groups, 0, sizeof(int), s));
    if (groups > 0)
        rows_blocks_kernel<false><<<(int)((groups + 255) / 256), 256, 0, s>>>(
            p->rowptr, m, kRowsShapes[R->shape].nmax, count, nullptr, nullptr, nullptr);
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, count, offset, groups + 1, s);
    void *tmp = nullptr;
    if (!al(&tmp, tmp_bytes)) {
        set_error("row-block plan: device allocation failed");
        return SBB_ERR_NOMEM;
    }
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, count, offset, groups + 1, s);
    int nblk = 0;
    SBB_CUDA(cudaMemcpyAsync(&nblk, offset + groups, sizeof(int), cudaMemcpyDeviceToHost, s));
    SBB_CUDA(cudaStreamSynchronize(s));
    R->nblk = nblk;
    if (!al((void **)&R->desc, sizeof(int4) * (size_t)nblk) ||
        !al((void **)&R->carry_row, sizeof(int) * (size_t)nblk) ||
        !al((void **)&R->carry_val, sizeof(double) * (size_t)nblk)) {
        set_error("row-block plan: device allocation failed");
        return SBB_ERR_NOMEM;
    }
    if (groups > 0)
        rows_blocks_kernel<true><<<(int)((groups + 255) / 256), 256, 0, s>>>(
            p->rowptr, m, kRowsShapes[R->shape].nmax, nullptr, offset, R->desc, R->carry_row);
    if (nblk > 0) {
        int rc = carry_runs_build(R->carry_row, nblk, m, &R->runs, s);
        if (rc) return rc;
        p->scratch_bytes += R->runs.bytes;
    }
    p->tiles = nblk;
    SBB_CUDA(cudaFreeAsync(tmp, s));
    SBB_CUDA(cudaFreeAsync(count, s));
    SBB_CUDA(cudaFreeAsync(offset, s));
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}

int rows_run(Plan *p, double alpha, const void *x, double beta, double *y, cudaStream_t s)
{
    auto *R = static_cast<RowsPlan *>(p->rows);
    if (!R) {
        set_error("row-block plan missing");
        return SBB_ERR_ARG;
    }
    if (R->nblk > 0) {
        if (p->f32)
            launch_rows_t<ProdF32>(*R, p, alpha, static_cast<const float *>(x), beta, y, s);
        else
            launch_rows_t<ProdF64>(*R, p, alpha, static_cast<const double *>(x), beta, y, s);
    }
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}

static void rows_release(Plan *p, cudaStream_t s, bool async)
{
    auto *R = static_cast<RowsPlan *>(p->rows);
    if (!R) return;
    void *ptrs[] = {R->desc, R->carry_row, R->carry_val};
    for (void *q : ptrs)
        if (q) {
            if (async)
                cudaFreeAsync(q, s);
            else
                cudaFree(q);
        }
    carry_runs_free(&R->runs, s, async);
    delete R;
    p->rows = nullptr;
}

void rows_free(Plan *p) { rows_release(p, 0, false); }
void rows_free_async(Plan *p, cudaStream_t s) { rows_release(p, s, true); }

int rows_launches(const Plan *p)
{
    auto *R = static_cast<const RowsPlan *>(p->rows);
    return R && R->nblk > 0 ? 2 : 0;
}

}  // namespace sbb
