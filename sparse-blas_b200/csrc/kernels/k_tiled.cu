// k_tiled.cu — K3: CSR5-style tiled segmented reduction.
//
// Replaces the reference's vendored CSR5 (SparseBLAS/src/csr5_kernel.cu:12-32,
// include/anonymouslib_cuda.h, include/detail/cuda/{format,csr5_spmv}_cuda.h)
// with a design of its own for one B200:
//
//   * Tile = 32 lanes x sigma nnz; lane l owns sigma consecutive nnz.  sigma
//     follows the CSR5 rule (include/anonymouslib_cuda.h:296-313) rounded up
//     to a power of two in {4, 8, 16, 32}.
//   * The plan keeps a COPY of the matrix as one blob per tile (the reference
//     transposes the caller's arrays in place, format_cuda.h:525-744):
//         [int cols[TILE] | V vals[TILE] | uint32 row-start bitmap[sigma] |
//          header: segment rank, closing / row-start flags, per-lane counts
//          of earlier row starts]
//     Inside a tile, nnz go in groups of 4 per lane, laid out so every
//     shared-memory read is 16 contiguous bytes per lane (no bank conflicts).
//   * One bit per nnz marks row starts (CSR5's bit-flag descriptor,
//     format_cuda.h:129-360).  The header plays the part of CSR5's tile
//     pointer and per-lane y offsets (format_cuda.h:362-523) in a layout of
//     its own: it arrives with the tile's bulk copy, so a tile needs no
//     metadata loads and no prefix scan of row starts.
//   * Persistent warps take tiles round-robin.  Each warp double-buffers tiles
//     in shared memory with one TMA bulk copy per tile (cp.async.bulk +
//     mbarrier, evict-first so x stays in L2; every wait is bounded).  All x
//     gathers of a lane are issued before any is used.
//   * Rows ending inside a lane are written at once; a warp segmented scan
//     (reset at lanes that start a row) joins segments across lanes; the row
//     open at the tile end is the tile's carry (CSR5's calibrator,
//     csr5_spmv_cuda.h:313-382) added afterwards in a fixed order
//     (k_fixup.cu) - no atomics, bit-reproducible.
//   * Empty rows (CSR5's descriptor-offset table, format_cuda.h:362-523): a
//     compact list of non-empty rows maps segments to rows, and a list of
//     empty rows gets y = beta*y.
//   * Unlike the reference, alpha and beta are applied (csr5_spmv_cuda.h:22
//     and anonymouslib_cuda.h:281 drop them); the last partial tile is padded
//     instead of taking a CSR-vector pass (csr5_spmv_cuda.h:384-419).
#include <stdint.h>
#include <stdlib.h>

#include <type_traits>

#include <cub/cub.cuh>

#include "../sbb_internal.h"
#include "common.cuh"
#include "tiled_device.cuh"

namespace sbb {

namespace {

constexpr int TW = 4;  // warps per CTA

struct TiledPlan {
    int sigma = 0, tiles = 0;
    size_t tile_bytes = 0;        // one tile blob
    unsigned char *blob = nullptr;
    int *tile_seg = nullptr;      // segment rank of the row holding each tile's first nnz
    int *ne = nullptr;            // non-empty rows (segment rank -> row); null if none empty
    int *empty = nullptr;         // empty rows
    int n_empty = 0;
    int *carry_row = nullptr;     // static: row carried out of each tile, m if none
    double *carry_val = nullptr;
    CarryRuns runs;
};

// Slot of nnz (lane, j) of group g inside a tile, for columns / FP32 values
// and for FP64 values.
__device__ __forceinline__ long long slot4(int g, int lane, int j) { return g * 128 + lane * 4 + j; }
__device__ __forceinline__ long long slot2(int g, int lane, int j)
{
    return g * 128 + (j >> 1) * 64 + lane * 2 + (j & 1);
}

// One thread per tile slot, in original nnz order: the column and value of
// the slot (zeros past nnz), and for the first slots of each tile a zero
// word of its row-start bits and header, which the later plan kernels OR
// into and write.  Sigma and the value width are compile-time, so the slot
// arithmetic is shifts and masks.
template <int SIGMA, int VB>
__global__ void blob_fill_kernel(const int *__restrict__ rp, const int *__restrict__ col,
                                 const void *__restrict__ val, long long nnz, int n, int tiles,
                                 unsigned char *__restrict__ blob, unsigned *status)
{
    constexpr long long TILE = 32LL * SIGMA;
    constexpr size_t TB = tile_bytes_of(SIGMA, VB);
    constexpr size_t DATA = (size_t)TILE * (4 + VB);
    constexpr int META_WORDS = (int)((TB - DATA) / 4);  // row-start bits and header
    static_assert((TB - DATA) % 4 == 0 && META_WORDS <= TILE, "tile layout");
    bool bad = false;
    const long long first = rp[0];  // the view's nnz start at rowptr[0]
    const long long total = (long long)tiles * TILE;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        // e enumerates (tile, lane, group, j) in original nnz order
        const long long t = e / TILE;
        const int q = (int)(e % TILE);
        const int lane = q / SIGMA, sl = q % SIGMA, g = sl >> 2, j = sl & 3;
        const bool in = e < nnz;
        unsigned char *tb = blob + (size_t)t * TB;
        int c = in ? col[first + e] : 0;
        if ((unsigned)c >= (unsigned)n) {  // checked once here: the kernel trusts the copy
            bad |= in;
            c = 0;
        }
        reinterpret_cast<int *>(tb)[slot4(g, lane, j)] = c;
        if (VB == 8)
            reinterpret_cast<double *>(tb + TILE * 4)[slot2(g, lane, j)] =
                in ? static_cast<const double *>(val)[first + e] : 0.0;
        else
            reinterpret_cast<float *>(tb + TILE * 4)[slot4(g, lane, j)] =
                in ? static_cast<const float *>(val)[first + e] : 0.f;
        if (q < META_WORDS) reinterpret_cast<unsigned *>(tb + DATA)[q] = 0u;
    }
    if (bad) atomicOr(status, ST_BAD_COL);
}

int grid_for(long long work, int tpb);

template <int VB>
void launch_blob_fill(int sigma, const int *rp, const int *col, const void *val, long long nnz,
                      int n, int tiles, unsigned char *blob, unsigned *status, cudaStream_t s)
{
    const int grid = grid_for((long long)tiles * 32 * sigma, 256);
    switch (sigma) {
    case 4: blob_fill_kernel<4, VB><<<grid, 256, 0, s>>>(rp, col, val, nnz, n, tiles, blob, status); break;
    case 8: blob_fill_kernel<8, VB><<<grid, 256, 0, s>>>(rp, col, val, nnz, n, tiles, blob, status); break;
    case 16: blob_fill_kernel<16, VB><<<grid, 256, 0, s>>>(rp, col, val, nnz, n, tiles, blob, status); break;
    case 32: blob_fill_kernel<32, VB><<<grid, 256, 0, s>>>(rp, col, val, nnz, n, tiles, blob, status); break;
    default: break;
    }
}

// Row-start bits (one per nnz, original order within the tile) and
// non-empty flags.
__global__ void starts_kernel(const int *__restrict__ rp, int m, int sigma, int vbytes,
                              unsigned char *__restrict__ blob, int *__restrict__ nonempty)
{
    const long long TILE = 32LL * sigma;
    const size_t TB = tile_bytes_of(sigma, vbytes);
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < m;
         r += (long long)gridDim.x * blockDim.x) {
        int lo = rp[r], hi = rp[r + 1];
        int ne = hi > lo;
        nonempty[r] = ne;
        if (ne) {
            long long k = lo - rp[0];
            long long t = k / TILE, q = k % TILE;
            unsigned *bits = reinterpret_cast<unsigned *>(blob + (size_t)t * TB + TILE * (4 + vbytes));
            atomicOr(bits + q / 32, 1u << (q % 32));
        }
    }
}

__global__ void compact_kernel(const int *__restrict__ flag, const int *__restrict__ rank, int m,
                               int *__restrict__ ne, int *__restrict__ empty)
{
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < m;
         r += (long long)gridDim.x * blockDim.x) {
        if (flag[r])
            ne[rank[r]] = (int)r;
        else
            empty[r - rank[r]] = (int)r;
    }
}

// Segment rank of the row owning the first nnz of each tile: the last row r
// with rp[r] <= k (that row is non-empty), mapped through the non-empty rank.
__global__ void tile_seg_kernel(const int *__restrict__ rp, int m, int sigma, int tiles,
                                const int *__restrict__ rank, int nonempty,
                                int *__restrict__ tile_seg)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == tiles) tile_seg[t] = nonempty;  // sentinel: one past the last segment
    if (t >= tiles) return;
    long long k = (long long)rp[0] + (long long)t * 32 * sigma;
    int lo = 0, hi = m;  // last r in [0, m) with rp[r] <= k
    while (lo < hi) {
        int mid = lo + ((hi - lo + 1) >> 1);
        if (rp[mid] <= k)
            lo = mid;
        else
            hi = mid - 1;
    }
    tile_seg[t] = rank ? rank[lo] : lo;
}

// Tile headers (tiled_device.cuh): segment rank, closing and row-start
// flags, and each lane's count of earlier row starts.  One warp per tile:
// lane l counts its own row starts, a warp scan gives the offsets.
__global__ void tile_header_kernel(const int *__restrict__ tile_seg, int sigma, int vbytes,
                                   int tiles, unsigned char *__restrict__ blob)
{
    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= tiles) return;  // whole warps leave together
    const long long TILE = 32LL * sigma;
    const size_t TB = tile_bytes_of(sigma, vbytes);
    unsigned char *tb = blob + (size_t)t * TB;
    const unsigned *bits = reinterpret_cast<const unsigned *>(tb + TILE * (4 + vbytes));
    unsigned char *hdr = tb + tile_hdr_offset(sigma, vbytes);
    const unsigned lb = sigma == 32 ? bits[lane]
                                    : (bits[(lane * sigma) >> 5] >> ((lane * sigma) & 31)) &
                                          ((1u << sigma) - 1u);
    const int cnt = __popc(lb);
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (sigma <= 8)
        hdr[16 + lane] = (unsigned char)(incl - cnt);
    else
        reinterpret_cast<unsigned short *>(hdr + 16)[lane] = (unsigned short)(incl - cnt);
    if (lane == 0) {
        const unsigned next0 =
            t + 1 < tiles ? *reinterpret_cast<const unsigned *>(blob + (size_t)(t + 1) * TB +
                                                                TILE * (4 + vbytes)) & 1u
                          : 1u;  // the last tile closes its open row
        reinterpret_cast<int *>(hdr)[0] = tile_seg[t];
        reinterpret_cast<int *>(hdr)[1] =
            (int)((next0 ? kTileCloses : 0u) | ((bits[0] & 1u) ? kTileStartsRow : 0u));
    }
}

__device__ __forceinline__ unsigned first_bit_of_tile(const unsigned char *blob, size_t TB,
                                                      long long TILE, int vbytes, int t)
{
    return *reinterpret_cast<const unsigned *>(blob + (size_t)t * TB + TILE * (4 + vbytes)) & 1u;
}

// Row carried out of tile t: the row holding its last nnz, when that row goes
// on into tile t+1 (whose first nnz then starts no row); m otherwise.
__global__ void carry_rows_kernel(const unsigned char *__restrict__ blob, int sigma, int vbytes,
                                  const int *__restrict__ tile_seg, const int *__restrict__ ne,
                                  int tiles, int m, int *__restrict__ carry_row)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tiles) return;
    const long long TILE = 32LL * sigma;
    const size_t TB = tile_bytes_of(sigma, vbytes);
    int r = m;
    if (t + 1 < tiles && !first_bit_of_tile(blob, TB, TILE, vbytes, t + 1)) {
        int seg = tile_seg[t + 1];
        r = ne ? ne[seg] : seg;
    }
    carry_row[t] = r;
}

__global__ void empty_rows_kernel(const int *__restrict__ empty, int n_empty, double beta,
                                  double *__restrict__ y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_empty; i += gridDim.x * blockDim.x) {
        double *yp = y + empty[i];
        *yp = beta == 0.0 ? 0.0 : beta * *yp;
    }
}

// CTAs per SM the launch bounds aim at.
template <int SIGMA> struct TiledShape {
    static constexpr int MINB = SIGMA <= 4 ? 12 : (SIGMA <= 8 ? 8 : 1);
};

// Persistent: warp w of the grid takes tiles w, w + W, w + 2W, ... (W = all
// warps), fixed per launch shape, so results do not depend on timing.  Each
// warp keeps a ring of NBUF tile blobs in shared memory: lane 0 issues the
// bulk copy of tile i+NBUF as soon as tile i is reduced.
template <typename PT, typename ACC, int SIGMA, int NBUF, bool NE>
__global__ void __launch_bounds__(TW * 32, TiledShape<SIGMA>::MINB)
tiled_kernel(int m, int n, long long nnz, int tiles, const unsigned char *__restrict__ blob,
             const int *__restrict__ tile_seg, const int *__restrict__ ne,
             const typename PT::V *__restrict__ x, double *__restrict__ y, double alpha,
             double beta, double *__restrict__ carry_val, unsigned *status, int evict_first,
             int first_wait)
{
    using V = typename PT::V;
    constexpr uint32_t TB = (uint32_t)tile_bytes_of(SIGMA, sizeof(V));
    constexpr uint32_t SB = (uint32_t)sum_bytes_of(SIGMA);
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[TW][NBUF];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *wbuf = smem + (size_t)warp * (NBUF * TB + SB);
    double *s_sum = reinterpret_cast<double *>(wbuf + NBUF * TB);
    const uint32_t bar_base = smem_u32(&bars[warp][0]);
    const int W = gridDim.x * TW;
    int t = blockIdx.x * TW + warp;
    (void)m;
    (void)n;

    uint64_t pol = 0;
    auto issue = [&](int tt, int b) {  // lane 0 only
        const uint32_t bar = bar_base + 8 * b;
        mbar_expect_tx(bar, TB);
        bulk_g2s(smem_u32(wbuf + b * TB), blob + (size_t)tt * TB, TB, bar, pol);
    };
    if (lane == 0) {
        pol = evict_first ? evict_first_policy() : 0;
#pragma unroll
        for (int b = 0; b < NBUF; ++b) mbar_init(bar_base + 8 * b, 1);
        mbar_fence_init();
#pragma unroll
        for (int b = 0; b < NBUF; ++b)
            if (t + b * W < tiles) issue(t + b * W, b);
    }
    __syncwarp();
    // The carry fix-up after this kernel is a programmatic dependent launch:
    // its blocks may take the SM slots this grid frees while it drains.
    allow_dependent_launch();

    unsigned timeout = 0;
    uint32_t phases = 0u;  // bit b: parity of buffer b's next phase
    const uint64_t keep = l2_evict_last(), streaming = l2_evict_first();
    // first_wait >= 0 (a test hook): the grid's first warp gives up its first
    // wait after that many polls and takes the timeout path below.
    int polls = first_wait >= 0 && blockIdx.x == 0 && warp == 0 ? first_wait : kWaitPolls;
    auto wait_buf = [&](int bb) {  // the phase bit flips only once the copy has landed
        const bool ok = mbar_wait(bar_base + 8 * bb, (phases >> bb) & 1u, polls);
        polls = kWaitPolls;
        if (ok) phases ^= 1u << bb;
        return ok;
    };
    int b = 0;
    // Tiles of sigma >= 16 load y of the segments they can write before the
    // tile arrives, from the segment ranks of this tile and the next one.
    int tseg = 0, tseg1 = 0;
    if (SIGMA >= kTileStagedSigma && t < tiles) {
        tseg = __ldg(tile_seg + t);
        tseg1 = __ldg(tile_seg + t + 1);
    }
    for (; t < tiles; t += W) {
        double ya = 0.0, yb = 0.0;
        int tseg_n = 0, tseg1_n = 0;
        if (SIGMA >= kTileStagedSigma) {
            if (beta != 0.0) {
                const int lim = tseg1 + (t + 1 < tiles ? 1 : 0);
                if (tseg + lane < lim)
                    ya = ld_y(y + (NE && ne ? __ldg(ne + tseg + lane) : tseg + lane), streaming);
                if (tseg + 32 + lane < lim)
                    yb = ld_y(y + (NE && ne ? __ldg(ne + tseg + 32 + lane) : tseg + 32 + lane),
                              streaming);
            }
            const int tn = t + W;  // segment ranks of the next tile, in flight meanwhile
            if (tn < tiles) {
                tseg_n = __ldg(tile_seg + tn);
                tseg1_n = __ldg(tile_seg + tn + 1);
            }
        }
        if (!wait_buf(b)) {
            timeout = 1;
            break;
        }
        V xv[SIGMA];
        tile_gather<PT, SIGMA>(t, tiles, nnz, wbuf + b * TB, x, keep, xv);
        tile_reduce<PT, ACC, SIGMA, NE>(t, wbuf + b * TB, ne, xv, y, alpha, beta, carry_val, streaming,
                                    ya, yb, s_sum);
        __syncwarp();  // every lane is done with buffer b before it is refilled
        if (lane == 0 && t + NBUF * W < tiles) issue(t + NBUF * W, b);
        b = b + 1 == NBUF ? 0 : b + 1;
        tseg = tseg_n;
        tseg1 = tseg1_n;
    }
    if (timeout) {
        // Let every copy still in flight land (bounded) before the warp
        // leaves: tile t in buffer b and the tiles t + k*W queued after it.
        for (int k = 0; k < NBUF && t + k * W < tiles; ++k) {
            const int bb = (b + k) % NBUF;
            mbar_wait(bar_base + 8 * bb, (phases >> bb) & 1u);
        }
        if (lane == 0) atomicOr(status, ST_TIMEOUT);
    }
    (void)status;
}

int grid_for(long long work, int tpb)
{
    long long g = (work + tpb - 1) / tpb;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

// L2 policy of the bulk copies (SBB_TILED_EVICT_FIRST=0 turns the
// evict-first hint off), read once per process.  Deeper copy rings (3-4
// tiles per warp) measured slower and are not built.
static int tiled_evict_first()
{
    static const int v = [] {
        const char *e = getenv("SBB_TILED_EVICT_FIRST");
        return e ? atoi(e) : 1;
    }();
    return v;
}

template <typename PT, typename ACC, int SIGMA, bool NE>
void launch_tiled_n(const TiledPlan &T, int m, int n, long long nnz, double alpha,
                    const typename PT::V *x, double beta, double *y, unsigned *status,
                    cudaStream_t s)
{
    auto kern = tiled_kernel<PT, ACC, SIGMA, 2, NE>;
    constexpr size_t smem =
        (size_t)TW * (2 * tile_bytes_of(SIGMA, sizeof(typename PT::V)) + sum_bytes_of(SIGMA));
    const LaunchShape ls = cached_launch_shape(kern, TW * 32, smem);
    long long want = (T.tiles + TW - 1) / TW;
    long long cap = (long long)ls.sms * ls.occ;
    int grid = (int)(want < cap ? want : cap);
    hook_start(s);
    kern<<<grid, TW * 32, smem, s>>>(m, n, nnz, T.tiles, T.blob, T.tile_seg, T.ne, x, y, alpha,
                                     beta, T.carry_val, status, tiled_evict_first(),
                                     first_wait_budget());
    hook_stop(s);
}

template <typename PT, typename ACC, int SIGMA>
void launch_tiled_s(const TiledPlan &T, int m, int n, long long nnz, double alpha,
                    const typename PT::V *x, double beta, double *y, unsigned *status,
                    cudaStream_t s)
{
    if (T.ne)
        launch_tiled_n<PT, ACC, SIGMA, true>(T, m, n, nnz, alpha, x, beta, y, status, s);
    else
        launch_tiled_n<PT, ACC, SIGMA, false>(T, m, n, nnz, alpha, x, beta, y, status, s);
}

template <typename PT, typename ACC>
void launch_tiled_t(const TiledPlan &T, int m, int n, long long nnz, double alpha,
                    const typename PT::V *x, double beta, double *y, unsigned *status,
                    cudaStream_t s)
{
    if (T.tiles > 0) {
        switch (T.sigma) {
        case 4: launch_tiled_s<PT, ACC, 4>(T, m, n, nnz, alpha, x, beta, y, status, s); break;
        case 8: launch_tiled_s<PT, ACC, 8>(T, m, n, nnz, alpha, x, beta, y, status, s); break;
        case 16:
        case 32:
            // FP32 lane sums are built for runs of at most 8 products
            if constexpr (!std::is_same<ACC, AccF32Lane>::value) {
                if (T.sigma == 16)
                    launch_tiled_s<PT, ACC, 16>(T, m, n, nnz, alpha, x, beta, y, status, s);
                else
                    launch_tiled_s<PT, ACC, 32>(T, m, n, nnz, alpha, x, beta, y, status, s);
            }
            break;
        default: break;
        }
        launch_fixup(m, T.carry_row, T.carry_val, T.tiles, T.runs, alpha, y, nullptr, s);
    }
    if (T.n_empty > 0)
        empty_rows_kernel<<<grid_for(T.n_empty, 256), 256, 0, s>>>(T.empty, T.n_empty, beta, y);
}

}  // namespace

bool tiled_view(const Plan *p, TiledView *v)
{
    auto *T = static_cast<const TiledPlan *>(p->tiled);
    if (!T) return false;
    *v = TiledView{T->blob, T->tile_seg, T->ne, T->empty, T->carry_row, T->carry_val,
                   T->tiles, T->sigma, T->n_empty, &T->runs};
    return true;
}

// CSR5 sigma rule (include/anonymouslib_cuda.h:296-313), then rounded up to a
// power of two in {4, 8, 16, 32} so a lane's row-start bits sit in one word.
int tiled_sigma(int m, long long nnz, int requested)
{
    int s = requested;
    if (s <= 0) {
        long long per_row = m > 0 ? nnz / m : 0;
        if (per_row <= 4)
            s = 4;
        else if (per_row <= 32)
            s = (int)per_row;
        else if (per_row <= 256)
            s = 32;
        else
            s = 6;
    }
    int p = 4;
    while (p < s && p < 32) p <<= 1;
    return p;
}

int tiled_build(Plan *p, cudaStream_t s)
{
    // row counts and segment ranks (plus a tile's few dozen) stay in int
    if (p->m > kTiledMaxRows) {
        set_error("tiled plan: at most 2^31 - 1025 rows (use the merge or vector kernel)");
        return SBB_ERR_ARG;
    }
    auto *T = new TiledPlan();
    p->tiled = T;
    T->sigma = tiled_sigma(p->m, p->nnz, p->tile_sigma);
    p->tile_sigma = T->sigma;
    const int vbytes = p->f32 ? 4 : 8;
    const long long TILE = 32LL * T->sigma;
    const long long tiles = (p->nnz + TILE - 1) / TILE;
    T->tiles = (int)tiles;
    p->tiles = T->tiles;
    T->tile_bytes = tile_bytes_of(T->sigma, vbytes);
    auto al = [&](void **ptr, size_t bytes) {
        bytes = bytes ? bytes : 16;
        p->scratch_bytes += bytes;
        return dev_malloc_async(ptr, bytes, s) == cudaSuccess;
    };
    const int m = p->m;
    int *flag = nullptr, *rank = nullptr;
    bool ok = al((void **)&T->blob, T->tile_bytes * (size_t)tiles) &&
              al((void **)&T->tile_seg, sizeof(int) * (tiles + 1)) &&
              al((void **)&T->carry_row, sizeof(int) * tiles) &&
              al((void **)&T->carry_val, sizeof(double) * tiles) &&
              al((void **)&flag, sizeof(int) * (m + 1)) && al((void **)&rank, sizeof(int) * (m + 1));
    if (!ok) {
        set_error("tiled plan: device allocation failed");
        return SBB_ERR_NOMEM;
    }
    if (tiles > 0) {  // every byte of the blob: slots here, bits and headers zeroed here too
        if (vbytes == 8)
            launch_blob_fill<8>(T->sigma, p->rowptr, p->col, p->val, p->nnz, p->n, T->tiles,
                                T->blob, p->status, s);
        else
            launch_blob_fill<4>(T->sigma, p->rowptr, p->col, p->val, p->nnz, p->n, T->tiles,
                                T->blob, p->status, s);
    }
    if (m > 0)
        starts_kernel<<<grid_for(m, 256), 256, 0, s>>>(p->rowptr, m, T->sigma, vbytes, T->blob, flag);
    // rank[r] = number of non-empty rows before r (rank[m] = count)
    SBB_CUDA(cudaMemsetAsync(flag + m, 0, sizeof(int), s));
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flag, rank, m + 1, s);
    void *tmp = nullptr;
    if (!al(&tmp, tmp_bytes)) return SBB_ERR_NOMEM;
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flag, rank, m + 1, s);
    int count = 0;
    SBB_CUDA(cudaMemcpyAsync(&count, rank + m, sizeof(int), cudaMemcpyDeviceToHost, s));
    SBB_CUDA(cudaStreamSynchronize(s));
    T->n_empty = m - count;
    if (T->n_empty > 0) {
        if (!al((void **)&T->ne, sizeof(int) * (count + 1)) ||
            !al((void **)&T->empty, sizeof(int) * T->n_empty))
            return SBB_ERR_NOMEM;
        compact_kernel<<<grid_for(m, 256), 256, 0, s>>>(flag, rank, m, T->ne, T->empty);
    }
    if (tiles > 0) {
        tile_seg_kernel<<<(T->tiles + 256) / 256, 256, 0, s>>>(
            p->rowptr, m, T->sigma, T->tiles, T->n_empty > 0 ? rank : nullptr, count,
            T->tile_seg);
        carry_rows_kernel<<<(T->tiles + 255) / 256, 256, 0, s>>>(
            T->blob, T->sigma, vbytes, T->tile_seg, T->ne, T->tiles, m, T->carry_row);
        tile_header_kernel<<<(int)(((long long)T->tiles * 32 + 255) / 256), 256, 0, s>>>(
            T->tile_seg, T->sigma, vbytes, T->tiles, T->blob);
        int rc = carry_runs_build(T->carry_row, T->tiles, m, &T->runs, s);
        if (rc) return rc;
        p->scratch_bytes += T->runs.bytes;
    }
    SBB_CUDA(cudaFreeAsync(tmp, s));
    SBB_CUDA(cudaFreeAsync(flag, s));
    SBB_CUDA(cudaFreeAsync(rank, s));
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}

int tiled_run(Plan *p, double alpha, const void *x, double beta, double *y, cudaStream_t s)
{
    auto *T = static_cast<TiledPlan *>(p->tiled);
    if (!T) {
        set_error("tiled plan missing");
        return SBB_ERR_ARG;
    }
    if (p->f32 && p->lane32)
        launch_tiled_t<ProdF32, AccF32Lane>(*T, p->m, p->n, p->nnz, alpha,
                                            static_cast<const float *>(x), beta, y, p->status, s);
    else if (p->f32)
        launch_tiled_t<ProdF32, AccF32>(*T, p->m, p->n, p->nnz, alpha,
                                        static_cast<const float *>(x), beta, y, p->status, s);
    else
        launch_tiled_t<ProdF64, AccF64>(*T, p->m, p->n, p->nnz, alpha,
                                        static_cast<const double *>(x), beta, y, p->status, s);
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}

static void tiled_release(Plan *p, cudaStream_t s, bool async)
{
    auto *T = static_cast<TiledPlan *>(p->tiled);
    if (!T) return;
    void *ptrs[] = {T->blob, T->tile_seg, T->ne, T->empty, T->carry_row, T->carry_val};
    for (void *q : ptrs)
        if (q) {
            if (async)
                cudaFreeAsync(q, s);
            else
                cudaFree(q);
        }
    carry_runs_free(&T->runs, s, async);
    delete T;
    p->tiled = nullptr;
}

void tiled_free(Plan *p) { tiled_release(p, 0, false); }
void tiled_free_async(Plan *p, cudaStream_t s) { tiled_release(p, s, true); }

int tiled_launches(const Plan *p)
{
    auto *T = static_cast<const TiledPlan *>(p->tiled);
    if (!T) return 0;
    return (T->tiles > 0 ? 2 : 0) + (T->n_empty > 0 ? 1 : 0);
}

}  // namespace sbb
