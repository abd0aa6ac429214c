// k_tiled.cu — K3: CSR5-style tiled segmented reduction.
//
// Replaces the reference's vendored CSR5 (SparseBLAS/src/csr5_kernel.cu:12-32,
// include/anonymouslib_cuda.h, include/detail/cuda/{format,csr5_spmv}_cuda.h)
// with a design of its own for one B200:
//
//   * Tile = 32 lanes x sigma nnz (sigma from the CSR5 rule of
//     include/anonymouslib_cuda.h:296-313, rounded up to a multiple of 4).
//     Lane l owns sigma consecutive nnz of the tile.
//   * The plan keeps a tile-transposed COPY of col/val (the reference
//     transposes the caller's arrays in place, format_cuda.h:525-744): within
//     a tile, groups of 4 consecutive nnz of a lane are stored together and the
//     32 lanes' groups side by side, so every load is a coalesced 128-bit
//     load (int4 of columns, 2 x double2 / float4 of values).
//   * Per lane a sigma-bit mask marks which of its nnz start a row
//     (CSR5's bit-flag descriptor, format_cuda.h:129-360, without the packed
//     y/scan offsets: the row of each segment comes from a warp scan of the
//     masks' popcounts instead).
//   * One warp per tile: each lane sums its segments; rows that end inside the
//     lane are written at once; a warp segmented scan (reset at lanes that
//     start a row) joins segments across lanes; the row still open at the tile
//     end becomes the tile's carry (CSR5's calibrator, csr5_spmv_cuda.h:313-382)
//     added by the same ordered fix-up as the merge-path kernel - no atomics,
//     so results are bit-reproducible.
//   * Empty rows (CSR5's descriptor-offset table, format_cuda.h:362-523) are
//     handled by a compact list of non-empty rows (segment -> row) and a list
//     of empty rows that get y = beta*y.
//   * Unlike the reference, alpha and beta are applied (csr5_spmv_cuda.h:22
//     and anonymouslib_cuda.h:281 drop them) and the last partial tile needs no
//     separate CSR-vector pass (csr5_spmv_cuda.h:384-419): it is padded.
#include <cub/cub.cuh>

#include "../sbb_internal.h"
#include "common.cuh"

namespace sbb {

namespace {

constexpr int TW = 4;  // warps (tiles) per CTA

struct TiledPlan {
    int sigma = 0, tiles = 0;
    int *col_t = nullptr;
    void *val_t = nullptr;
    unsigned *bits = nullptr;     // tiles*32 masks
    int *tile_seg = nullptr;      // tiles: segment rank of the row holding the tile's first nnz
    int *ne = nullptr;            // non-empty rows (segment rank -> row), null if none empty
    int *empty = nullptr;         // empty rows
    int n_empty = 0;
    int *carry_row = nullptr;
    double *carry_val = nullptr;
};

__global__ void transpose_kernel(const int *__restrict__ rp, const int *__restrict__ col,
                                 const void *__restrict__ val, int vbytes, long long nnz,
                                 int sigma, long long total, int *__restrict__ col_t,
                                 void *__restrict__ val_t)
{
    const long long TILE = 32LL * sigma;
    const long long first = rp[0];  // the view's nnz start at rowptr[0]
    for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < total;
         o += (long long)gridDim.x * blockDim.x) {
        long long t = o / TILE, q = o % TILE;
        long long g = q / 128, w = q % 128;  // group of 4 steps, then lane*4 + j
        long long lane = w / 4, j = w % 4;
        long long k = t * TILE + lane * sigma + g * 4 + j;  // original nnz index
        bool in = k < nnz;
        col_t[o] = in ? col[first + k] : 0;
        if (vbytes == 8)
            static_cast<double *>(val_t)[o] = in ? static_cast<const double *>(val)[first + k] : 0.0;
        else
            static_cast<float *>(val_t)[o] = in ? static_cast<const float *>(val)[first + k] : 0.f;
    }
}

// Row-start bits, non-empty flags.
__global__ void starts_kernel(const int *__restrict__ rp, int m, int sigma,
                              unsigned *__restrict__ bits, int *__restrict__ nonempty)
{
    const long long TILE = 32LL * sigma;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < m;
         r += (long long)gridDim.x * blockDim.x) {
        int lo = rp[r], hi = rp[r + 1];
        int ne = hi > lo;
        nonempty[r] = ne;
        if (ne) {
            long long k = lo - rp[0];
            long long t = k / TILE, q = k % TILE;
            atomicOr(bits + t * 32 + q / sigma, 1u << (q % sigma));
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
                                const int *__restrict__ rank, int *__restrict__ tile_seg)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tiles) return;
    long long k = (long long)rp[0] + (long long)t * 32 * sigma;
    int lo = 0, hi = m;  // find last r in [0, m) with rp[r] <= k
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (rp[mid] <= k)
            lo = mid;
        else
            hi = mid - 1;
    }
    tile_seg[t] = rank ? rank[lo] : lo;
}

__global__ void empty_rows_kernel(const int *__restrict__ empty, int n_empty, double beta,
                                  double *__restrict__ y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_empty; i += gridDim.x * blockDim.x) {
        double *yp = y + empty[i];
        *yp = beta == 0.0 ? 0.0 : beta * *yp;
    }
}

template <typename PT>
__device__ __forceinline__ void load4(const int *col_t, const typename PT::V *val_t, long long o,
                                      int4 &c, typename PT::V (&v)[4])
{
    c = ld_stream(reinterpret_cast<const int4 *>(col_t + o));
    if constexpr (sizeof(typename PT::V) == 8) {
        double2 a = ld_stream(reinterpret_cast<const double2 *>(val_t + o));
        double2 b = ld_stream(reinterpret_cast<const double2 *>(val_t + o + 2));
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else {
        float4 a = ld_stream(reinterpret_cast<const float4 *>(val_t + o));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
}

template <typename PT, typename ACC, int SIGMA>
__global__ void __launch_bounds__(TW * 32)
tiled_kernel(int m, int n, long long nnz, int tiles, const int *__restrict__ col_t,
             const typename PT::V *__restrict__ val_t, const unsigned *__restrict__ bits_arr,
             const int *__restrict__ tile_seg, const int *__restrict__ ne,
             const typename PT::V *__restrict__ x, double *__restrict__ y, double alpha,
             double beta, int *__restrict__ carry_row, double *__restrict__ carry_val,
             unsigned *status)
{
    constexpr int TILE = 32 * SIGMA;
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * TW + (threadIdx.x >> 5);
    if (t >= tiles) return;  // warp-uniform
    const long long base = (long long)t * TILE;
    const unsigned bits = __ldg(bits_arr + (long long)t * 32 + lane);
    const unsigned b0 = __shfl_sync(0xffffffffu, bits, 0) & 1u;
    const int cnt = __popc(bits);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    const int seg0 = __ldg(tile_seg + t) - (int)b0;
    const int head_seg = seg0 + incl - cnt;  // segment open before this lane's first nnz
    auto row_of = [&](int seg) { return ne ? __ldg(ne + seg) : seg; };

    unsigned bad = 0;
    const bool last = t == tiles - 1;
    ACC acc;
    acc.zero();
    double head = 0.0;
    bool started = false;
    int seg = head_seg;
#pragma unroll
    for (int g = 0; g < SIGMA / 4; ++g) {
        int4 c;
        typename PT::V v[4];
        load4<PT>(col_t, val_t, base + g * 128 + lane * 4, c, v);
        const int cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int s = g * 4 + j;
            if ((bits >> s) & 1u) {
                if (!started) {
                    head = acc.get();
                    started = true;
                } else {  // a whole row inside this lane
                    double *yp = y + row_of(seg);
                    *yp = axpby(alpha, acc.get(), beta, yp);
                }
                acc.zero();
                ++seg;
            }
            const bool live = !last || base + lane * SIGMA + s < nnz;
            if (live) acc.add(PT::make(v[j], gather_x(x, cc[j], n, bad)));
        }
    }
    // Warp segmented scan of lane carries, reset at lanes that start a row.
    double cv = acc.get();  // tail (or whole lane when no row starts here)
    unsigned f = started;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double vu = __shfl_up_sync(0xffffffffu, cv, o);
        unsigned fu = __shfl_up_sync(0xffffffffu, f, o);
        if (lane >= o) {
            if (!f) cv += vu;
            f |= fu;
        }
    }
    double incoming = __shfl_up_sync(0xffffffffu, cv, 1);
    if (lane == 0) incoming = 0.0;
    // The row open when this lane began ends at its first row start.  For
    // lane 0 with a start on its first nnz that row ended with the previous
    // tile, which wrote it.
    if (started && !(lane == 0 && b0)) {
        double *yp = y + row_of(head_seg);
        *yp = axpby(alpha, incoming + head, beta, yp);
    }
    if (lane == 31) {
        const bool closes = last || (__ldg(bits_arr + (long long)(t + 1) * 32) & 1u);
        const int r = row_of(seg);
        if (closes) {
            double *yp = y + r;
            *yp = axpby(alpha, cv, beta, yp);
            carry_row[t] = m;  // nothing to carry
            carry_val[t] = 0.0;
        } else {
            carry_row[t] = r;
            carry_val[t] = cv;
        }
    }
    if (bad) atomicOr(status, ST_BAD_COL);
}

int grid_for(long long work, int tpb)
{
    long long g = (work + tpb - 1) / tpb;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

template <typename PT, typename ACC>
void launch_tiled_t(const TiledPlan &T, int m, int n, long long nnz, double alpha,
                    const typename PT::V *x, double beta, double *y, unsigned *status,
                    cudaStream_t s)
{
    if (T.tiles > 0) {
        const auto *val_t = static_cast<const typename PT::V *>(T.val_t);
        int grid = (T.tiles + TW - 1) / TW;
        hook_start(s);
#define SBB_TL(S)                                                                          \
    case S:                                                                                \
        tiled_kernel<PT, ACC, S><<<grid, TW * 32, 0, s>>>(m, n, nnz, T.tiles, T.col_t, val_t, \
                                                          T.bits, T.tile_seg, T.ne, x, y,  \
                                                          alpha, beta, T.carry_row,        \
                                                          T.carry_val, status);            \
        break;
        switch (T.sigma) {
            SBB_TL(4) SBB_TL(8) SBB_TL(12) SBB_TL(16) SBB_TL(20) SBB_TL(24) SBB_TL(28) SBB_TL(32)
        default: break;
        }
#undef SBB_TL
        hook_stop(s);
        launch_carry_fixup(m, T.carry_row, T.carry_val, T.tiles, alpha, y, s);
    }
    if (T.n_empty > 0)
        empty_rows_kernel<<<grid_for(T.n_empty, 256), 256, 0, s>>>(T.empty, T.n_empty, beta, y);
}

}  // namespace

// CSR5 sigma rule (include/anonymouslib_cuda.h:296-313), then rounded up to a
// multiple of 4 for the 128-bit tile layout.
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
    s = ((s + 3) / 4) * 4;
    return s < 4 ? 4 : (s > 32 ? 32 : s);
}

int tiled_build(Plan *p, cudaStream_t s)
{
    auto *T = new TiledPlan();
    p->tiled = T;
    T->sigma = tiled_sigma(p->m, p->nnz, p->tile_sigma);
    p->tile_sigma = T->sigma;
    const long long TILE = 32LL * T->sigma;
    const long long tiles = (p->nnz + TILE - 1) / TILE;
    T->tiles = (int)tiles;
    p->tiles = T->tiles;
    const long long total = tiles * TILE;
    const int vbytes = p->f32 ? 4 : 8;
    auto al = [&](void **ptr, size_t bytes) {
        bytes = bytes ? bytes : 16;
        p->scratch_bytes += bytes;
        return cudaMallocAsync(ptr, bytes, s) == cudaSuccess;
    };
    const int m = p->m;
    int *flag = nullptr, *rank = nullptr;
    bool ok = al((void **)&T->col_t, sizeof(int) * total) && al(&T->val_t, (size_t)vbytes * total) &&
              al((void **)&T->bits, sizeof(unsigned) * (tiles + 1) * 32) &&
              al((void **)&T->tile_seg, sizeof(int) * tiles) &&
              al((void **)&T->carry_row, sizeof(int) * tiles) &&
              al((void **)&T->carry_val, sizeof(double) * tiles) &&
              al((void **)&flag, sizeof(int) * (m + 1)) && al((void **)&rank, sizeof(int) * (m + 1));
    if (!ok) {
        set_error("tiled plan: device allocation failed");
        return SBB_ERR_NOMEM;
    }
    if (total > 0)
        transpose_kernel<<<grid_for(total, 256), 256, 0, s>>>(p->rowptr, p->col, p->val, vbytes, p->nnz,
                                                              T->sigma, total, T->col_t, T->val_t);
    SBB_CUDA(cudaMemsetAsync(T->bits, 0, sizeof(unsigned) * (tiles + 1) * 32, s));
    if (m > 0) starts_kernel<<<grid_for(m, 256), 256, 0, s>>>(p->rowptr, m, T->sigma, T->bits, flag);
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
    if (tiles > 0)
        tile_seg_kernel<<<(T->tiles + 255) / 256, 256, 0, s>>>(p->rowptr, m, T->sigma, T->tiles,
                                                              T->n_empty > 0 ? rank : nullptr,
                                                              T->tile_seg);
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
    if (p->f32)
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
    void *ptrs[] = {T->col_t, T->val_t, T->bits, T->tile_seg, T->ne, T->empty, T->carry_row,
                    T->carry_val};
    for (void *q : ptrs)
        if (q) {
            if (async)
                cudaFreeAsync(q, s);
            else
                cudaFree(q);
        }
    delete T;
    p->tiled = nullptr;
}

void tiled_free(Plan *p) { tiled_release(p, 0, false); }

int tiled_launches(const Plan *p)
{
    auto *T = static_cast<const TiledPlan *>(p->tiled);
    if (!T) return 0;
    return (T->tiles > 0 ? 2 : 0) + (T->n_empty > 0 ? 1 : 0);
}
void tiled_free_async(Plan *p, cudaStream_t s) { tiled_release(p, s, true); }

}  // namespace sbb
