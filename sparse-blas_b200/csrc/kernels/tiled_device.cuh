// tiled_device.cuh — tile layout, TMA helpers and the per-tile device code of
// K3, shared by the standalone tiled kernel (k_tiled.cu) and the batched
// kernel (k_batch.cu), so a matrix gets bit-identical results either way.
#pragma once
#include <stdint.h>

#include <type_traits>

#include "../sbb_internal.h"
#include "common.cuh"

namespace sbb {

// A tile blob:
//   [int cols[TILE] | V vals[TILE] | uint32 row-start bits[sigma] | header]
// The header holds what the reduction of a tile needs beyond its nnz, so it
// arrives with the same bulk copy instead of costing loads and scans:
//   int seg    segment rank (row, when no row is empty) of the row holding
//              the tile's first nnz;
//   int flags  bit 0: the row open at the tile's end closes in it (the next
//              tile starts a row, or this is the last tile); bit 1: the
//              tile's first nnz starts a row;
//   8 bytes of padding, then per lane the number of row starts in the lanes
//   before it (uint8 for sigma <= 8, uint16 above).
__host__ __device__ constexpr size_t tile_hdr_offset(int sigma, int vbytes)
{
    return (size_t)32 * sigma * (4 + vbytes) + 4 * (size_t)sigma;
}
__host__ __device__ constexpr size_t tile_hdr_bytes(int sigma)
{
    return 16 + 32 * (sigma <= 8 ? 1 : 2);
}
__host__ __device__ constexpr size_t tile_bytes_of(int sigma, int vbytes)
{
    return tile_hdr_offset(sigma, vbytes) + tile_hdr_bytes(sigma);
}
constexpr unsigned kTileCloses = 1u, kTileStartsRow = 2u;
// Tiles of at least this sigma stage their row sums in shared memory and
// write them in one coalesced pass; smaller tiles write each row as it
// completes.
constexpr int kTileStagedSigma = 16;
// Per-warp staging of a tile's row sums: up to 32*sigma + 1 segments.
__host__ __device__ constexpr size_t sum_bytes_of(int sigma)
{
    return sigma < kTileStagedSigma ? 0 : ((size_t)(32 * sigma + 1) * 8 + 127) / 128 * 128;
}

// ---- TMA (1-D bulk async copy) helpers ------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ uint64_t evict_first_policy()
{
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// pol == 0: default L2 policy; otherwise an L2 cache-hint policy.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar,
                                         uint64_t pol)
{
    if (pol)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
            " [%0], [%1], %2, [%3], %4;" ::"r"(dst),
            "l"(src), "r"(bytes), "r"(bar), "l"(pol)
            : "memory");
    else
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
            " [%0], [%1], %2, [%3];" ::"r"(dst),
            "l"(src), "r"(bytes), "r"(bar)
            : "memory");
}
// Bounded wait for the phase with the given parity; false if it never came
// within `polls` tries (the caller raises ST_TIMEOUT and stops instead of
// spinning for ever).
constexpr int kWaitPolls = 1 << 22;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int polls = kWaitPolls)
{
    for (int i = 0; i < polls; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

// One tile from shared memory.
// Columns in the blob were range-checked when the plan copied them, so x is
// gathered without a per-element check; the final tile masks its padding.
template <typename PT, int SIGMA>
__device__ __forceinline__ void tile_gather(int t, int tiles, long long nnz, const unsigned char *tb,
                                            const typename PT::V *__restrict__ x, uint64_t keep,
                                            typename PT::V (&xv)[SIGMA])
{
    using V = typename PT::V;
    constexpr int TILE = 32 * SIGMA;
    const int lane = threadIdx.x & 31;
    const int *s_col = reinterpret_cast<const int *>(tb);
    const long long base = (long long)t * TILE;
    const bool last = t == tiles - 1;
#pragma unroll
    for (int g = 0; g < SIGMA / 4; ++g) {
        const int4 c = *reinterpret_cast<const int4 *>(s_col + g * 128 + lane * 4);
        const int cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (last)
                xv[g * 4 + j] = base + lane * SIGMA + g * 4 + j < nnz ? ld_keep(x + cc[j], keep) : V(0);
            else
                xv[g * 4 + j] = ld_keep(x + cc[j], keep);
        }
    }
}

// Reduces one tile whose x values are already gathered (xv).  The tile's
// segment rank, closing flag and each lane's count of earlier row starts come
// from its header.  Tiles of sigma >= 16 stage row sums in the warp's s_sum
// (index = segment - tseg) and write them to y in one coalesced pass at the
// end, so the divergent per-nnz loop touches no global memory; ya/yb hold y
// of segments tseg+lane and tseg+32+lane, loaded when the tile started.
// Tiles of sigma 4 and 8 write each row as it completes.
// NE = false: the matrix has no empty rows (ne is null), segment = row.
template <typename PT, typename ACC, int SIGMA, bool NE = true>
__device__ __forceinline__ void tile_reduce(int t, const unsigned char *tb,
                                            const int *__restrict__ ne,
                                            const typename PT::V (&xv)[SIGMA],
                                            double *__restrict__ y, double alpha, double beta,
                                            double *__restrict__ carry_val, uint64_t stream,
                                            double ya, double yb, double *s_sum)
{
    using V = typename PT::V;
    constexpr int TILE = 32 * SIGMA;
    constexpr int G = SIGMA / 4;
    constexpr size_t HDR = tile_hdr_offset(SIGMA, sizeof(V));
    const int lane = threadIdx.x & 31;
    const V *s_val = reinterpret_cast<const V *>(tb + TILE * 4);
    const unsigned *s_bits = reinterpret_cast<const unsigned *>(tb + TILE * (4 + sizeof(V)));

    // this lane's sigma row-start bits and the tile's header
    unsigned bits;
    if constexpr (SIGMA == 32)
        bits = s_bits[lane];
    else
        bits = (s_bits[(lane * SIGMA) >> 5] >> ((lane * SIGMA) & 31)) & ((1u << SIGMA) - 1u);
    const int2 hdr = *reinterpret_cast<const int2 *>(tb + HDR);
    const int tseg = hdr.x;
    const bool closes = hdr.y & kTileCloses;  // the row open at the end ends here
    const unsigned b0 = (hdr.y & kTileStartsRow) ? 1u : 0u;
    int excl;  // row starts in the lanes before this one
    if constexpr (SIGMA <= 8)
        excl = tb[HDR + 16 + lane];
    else
        excl = reinterpret_cast<const unsigned short *>(tb + HDR + 16)[lane];

    // 2. segment rows of this lane.  Tiles of sigma >= 16 stage row sums and
    // write them in one coalesced pass; sigma 4 and 8 tiles (few rows per
    // lane, tight register budgets) write each row as it completes, which
    // measured faster for them (sigma 8: 0.130 vs 0.196 ms, FP32 storage, on
    // the 5.5M-row matrix).
    constexpr bool kStaged = SIGMA >= kTileStagedSigma;
    auto put = [&](int sg, double sum) {
        if (kStaged) {
            s_sum[sg - tseg] = sum;
        } else {
            write_y(y + (NE && ne ? __ldg(ne + sg) : sg), alpha, sum, beta, stream);
        }
    };
    const int head_seg = tseg - (int)b0 + excl;  // segment open before this lane's first nnz

    // 3. products and lane-local segmented sums
    ACC acc;
    acc.zero();
    double head = 0.0;
    bool started = false;
    int seg = head_seg;
    // The general loop: any number of row starts per lane.
#define SBB_TILE_GENERAL_LOOP()                                                                   \
    _Pragma("unroll") for (int g = 0; g < G; ++g)                                                 \
    {                                                                                             \
        V v[4];                                                                                   \
        if constexpr (sizeof(V) == 8) {                                                           \
            double2 a = *reinterpret_cast<const double2 *>(s_val + g * 128 + lane * 2);           \
            double2 b = *reinterpret_cast<const double2 *>(s_val + g * 128 + 64 + lane * 2);      \
            v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;                                       \
        } else {                                                                                  \
            float4 a = *reinterpret_cast<const float4 *>(s_val + g * 128 + lane * 4);             \
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;                                       \
        }                                                                                         \
        _Pragma("unroll") for (int j = 0; j < 4; ++j)                                             \
        {                                                                                         \
            const int s = g * 4 + j;                                                              \
            if ((bits >> s) & 1u) {                                                               \
                if (!started) {                                                                   \
                    head = acc.get();                                                             \
                    started = true;                                                               \
                } else { /* a whole row inside this lane */                                       \
                    put(seg, acc.get());                                                          \
                }                                                                                 \
                acc.zero();                                                                       \
                ++seg;                                                                            \
            }                                                                                     \
            acc.mac(v[j], xv[s]);                                                                 \
        }                                                                                         \
    }
    // FP32 storage with exact FP64 products: when no lane of the warp starts
    // two rows (every row here is longer than sigma, as in banded matrices),
    // a lane's products before its row start (if any) go to h and the rest
    // to acc, each summed from zero in nnz order - the same operations as
    // the general loop, without its per-nnz branches.  Measured on the
    // 5.5M-row matrix: 0.1273 vs 0.1299 ms for this form; the same path made
    // the FP64 (0.180 vs 0.174 ms) and FP32-lane-sum (0.141 vs 0.129 ms)
    // kernels slower, so they keep the general loop.
    if constexpr (std::is_same<ACC, AccF32>::value) {
        if (!__any_sync(0xffffffffu, (bits & (bits - 1u)) != 0u)) {
            const int p1 = bits ? __ffs(bits) - 1 : SIGMA;
            ACC h;
            h.zero();
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const float4 a = *reinterpret_cast<const float4 *>(s_val + g * 128 + lane * 4);
                const float v[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (g * 4 + j < p1)
                        h.mac(v[j], xv[g * 4 + j]);
                    else
                        acc.mac(v[j], xv[g * 4 + j]);
                }
            }
            started = bits != 0u;
            if (started) {
                head = h.get();
                seg = head_seg + 1;
            } else {
                acc = h;
            }
        } else {
            SBB_TILE_GENERAL_LOOP()
        }
    } else {
        SBB_TILE_GENERAL_LOOP()
    }
#undef SBB_TILE_GENERAL_LOOP

    // 4. warp segmented scan of lane carries, reset at lanes that start a row
    // A lane adds the partial scan from o lanes back while no row starts in
    // the o lanes ending at it: o <= d, d = distance to the last lane at or
    // before it that starts a row (its own index when none does).  These are
    // exactly the additions of the flag-carrying segmented scan, in the same
    // order, without shuffling the flags.
    double cv = acc.get();  // tail (or whole lane when no row starts here)
    {
        const unsigned below = __ballot_sync(0xffffffffu, started) & (0xffffffffu >> (31 - lane));
        const int d = below ? lane - (31 - __clz(below)) : lane;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double vu = __shfl_up_sync(0xffffffffu, cv, o);
            if (o <= d) cv += vu;
        }
    }
    double incoming = __shfl_up_sync(0xffffffffu, cv, 1);
    if (lane == 0) incoming = 0.0;
    // The row open when this lane began ends at its first row start.  For
    // lane 0 with a start on its first nnz that row ended with the previous
    // tile, which wrote it.
    if (started && !(lane == 0 && b0)) put(head_seg, incoming + head);
    if (lane == 31) {
        if (closes)
            put(seg, cv);        // carry_row[t] == m: no carry is read for this tile
        else
            carry_val[t] = cv;   // carried into row_of(seg) == carry_row[t]
    }
    if (!kStaged) return;
    // 5. rows completed here: segments tseg .. tseg+nwrite-1, coalesced
    const int total = __shfl_sync(0xffffffffu, excl + __popc(bits), 31);
    const int nwrite = total + (closes ? 1 : 0) - (int)b0;
    __syncwarp();
    for (int i = lane; i < nwrite; i += 32) {
        double *yp = y + (NE && ne ? __ldg(ne + tseg + i) : tseg + i);
        const double yv = beta == 0.0 ? 0.0 : (i < 32 ? ya : (i < 64 ? yb : ld_y(yp, stream)));
        st_y(yp, y_update(alpha, s_sum[i], beta, yv), stream);
    }
    __syncwarp();  // s_sum is reused by the next tile
}

}  // namespace sbb
