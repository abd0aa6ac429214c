// k_fixup.cu — ordered combination of per-tile carries (K2 and K3).
//
// A tiled kernel leaves, for every tile t, the partial sum carry_val[t] of the
// row still open at the tile's end; the tile where that row ends has already
// written y = alpha*sum + beta*y for its own part.  Which row each tile
// carries (carry_row[t], or m for none) depends only on the matrix and the
// tiling, so it is fixed when the plan is built; so are the runs of
// consecutive tiles carrying the same row (a long row spans many tiles).
//
// Run time: one launch.  The first blocks take one long run each (more than
// kWarpRunMax carries: per-thread strided sums, then a shared-memory tree),
// the next take eight short runs each (one warp a run: lane-strided sums,
// then a butterfly), the others stride over the tiles and add single-tile
// carries.  Each row is updated by one thread, so results are
// bit-reproducible.
#include <algorithm>
#include <vector>

#include "../sbb_internal.h"
#include "spmv_device.cuh"

namespace sbb {

namespace {

constexpr int FT = kFixupThreads;

__global__ void runs_mark_kernel(const int *__restrict__ crow, int T, int m,
                                 int *__restrict__ run_first, int *__restrict__ run_len,
                                 int *__restrict__ count)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    int r = crow[t];
    if (r >= m) return;
    bool head = t == 0 || crow[t - 1] != r;
    bool multi = t + 1 < T && crow[t + 1] == r;
    if (!(head && multi)) return;
    // Run end (equal values are contiguous): exponential probe from t+1, then
    // bisection between the last index known to carry r and the first known
    // not to (or T).
    int lo = t + 1, hi = T, step = 1;
    for (;;) {
        int probe = lo + step;
        if (probe >= T) break;
        if (crow[probe] != r) {
            hi = probe;
            break;
        }
        lo = probe;
        step <<= 1;
    }
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (crow[mid] == r)
            lo = mid;
        else
            hi = mid;
    }
    int j = atomicAdd(count, 1);
    run_first[j] = t;
    run_len[j] = lo - t + 1;
}

// Blocks [0, long_blocks) take the long runs (launched first: they are the
// longest), the next warp_blocks the short runs, eight per block; the rest
// stride over the tiles for single carries.  With a device-side run count
// (dev_count), the long_blocks stride over every run.
__global__ void __launch_bounds__(FT)
fixup_kernel(int m, const int *__restrict__ crow, const double *__restrict__ cval, int T,
             const int *__restrict__ run_first, const int *__restrict__ run_len, int long_blocks,
             int n_long, int n_runs_host, int warp_blocks, double alpha, double *__restrict__ y,
             unsigned *queue, const int *dev_count)
{
    // Launched as a programmatic dependent of the kernel before it: nothing
    // is read before that grid has completed and its writes are visible.
    grid_dependency_wait();
    if (blockIdx.x >= long_blocks && blockIdx.x < long_blocks + warp_blocks) {
        const int j = n_long + (blockIdx.x - long_blocks) * (FT / 32) + (threadIdx.x >> 5);
        if (j >= n_runs_host) return;
        const int first = run_first[j], len = run_len[j];
        const double sum = fixup_run_warp(cval, first, len);
        if ((threadIdx.x & 31) == 0) fixup_single(y, crow[first], alpha, sum);
        return;
    }
    if (blockIdx.x >= long_blocks) {
        const int sb = blockIdx.x - long_blocks - warp_blocks,
                  nsb = gridDim.x - long_blocks - warp_blocks;
        if (sb == 0 && threadIdx.x == 0 && queue != nullptr) queue[0] = 0u;  // rearm a work queue
        for (int t = sb * FT + threadIdx.x; t < T; t += nsb * FT) {
            const int r = crow[t];
            if (r >= m) continue;
            if ((t > 0 && crow[t - 1] == r) || (t + 1 < T && crow[t + 1] == r)) continue;
            fixup_single(y, r, alpha, cval[t]);
        }
        return;
    }
    __shared__ double s[FT];
    // With a device-side count, a fixed set of blocks goes over all the runs
    // twice: every warp takes runs of at most kWarpRunMax carries (the same
    // warp sum as above), then every block the longer ones.
    if (dev_count) {
        const int n_all = *dev_count, nw = long_blocks * (FT / 32);
        for (int j = blockIdx.x * (FT / 32) + (threadIdx.x >> 5); j < n_all; j += nw) {
            const int first = run_first[j], len = run_len[j];
            if (len > kWarpRunMax) continue;
            const double sum = fixup_run_warp(cval, first, len);
            if ((threadIdx.x & 31) == 0) fixup_single(y, crow[first], alpha, sum);
        }
    }
    const int n_runs = dev_count ? *dev_count : n_long;
    for (int j = blockIdx.x; j < n_runs; j += long_blocks) {
        const int first = run_first[j], len = run_len[j];
        if (dev_count && len <= kWarpRunMax) continue;  // block-uniform: summed above
        s[threadIdx.x] = fixup_partial(cval, first, len, threadIdx.x);
        __syncthreads();
        for (int w = FT / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) fixup_single(y, crow[first], alpha, s[0]);
        __syncthreads();
    }
}

}  // namespace

int carry_runs_build(const int *crow, int T, int m, CarryRuns *R, cudaStream_t s)
{
    R->n_runs = 0;
    R->run_first = R->run_len = nullptr;
    if (T <= 0) return SBB_OK;
    int cap = T / 2 + 1;
    int *count = nullptr;
    if (dev_malloc_async((void **)&R->run_first, sizeof(int) * cap, s) != cudaSuccess ||
        dev_malloc_async((void **)&R->run_len, sizeof(int) * cap, s) != cudaSuccess ||
        dev_malloc_async((void **)&count, sizeof(int), s) != cudaSuccess) {
        set_error("carry runs: device allocation failed");
        return SBB_ERR_NOMEM;
    }
    R->bytes = 2 * sizeof(int) * (size_t)cap;
    SBB_CUDA(cudaMemsetAsync(count, 0, sizeof(int), s));
    runs_mark_kernel<<<(T + FT - 1) / FT, FT, 0, s>>>(crow, T, m, R->run_first, R->run_len, count);
    int h = 0;
    SBB_CUDA(cudaMemcpyAsync(&h, count, sizeof(int), cudaMemcpyDeviceToHost, s));
    SBB_CUDA(cudaStreamSynchronize(s));
    SBB_CUDA(cudaFreeAsync(count, s));
    R->n_runs = h;
    R->n_long = 0;
    if (h > 0) {  // long runs first (the fix-up gives them whole blocks)
        std::vector<int> f(h), l(h);
        SBB_CUDA(cudaMemcpyAsync(f.data(), R->run_first, sizeof(int) * h, cudaMemcpyDeviceToHost, s));
        SBB_CUDA(cudaMemcpyAsync(l.data(), R->run_len, sizeof(int) * h, cudaMemcpyDeviceToHost, s));
        SBB_CUDA(cudaStreamSynchronize(s));
        std::vector<int> order(h);
        for (int i = 0; i < h; ++i) order[i] = i;
        std::stable_partition(order.begin(), order.end(),
                              [&](int i) { return l[i] > kWarpRunMax; });
        std::vector<int> f2(h), l2(h);
        for (int i = 0; i < h; ++i) {
            f2[i] = f[order[i]];
            l2[i] = l[order[i]];
            R->n_long += l2[i] > kWarpRunMax;
        }
        SBB_CUDA(cudaMemcpyAsync(R->run_first, f2.data(), sizeof(int) * h, cudaMemcpyHostToDevice, s));
        SBB_CUDA(cudaMemcpyAsync(R->run_len, l2.data(), sizeof(int) * h, cudaMemcpyHostToDevice, s));
        SBB_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
    }
    return SBB_OK;
}

int carry_runs_build_device(const int *crow, int T, int m, CarryRuns *R, cudaStream_t s)
{
    R->n_runs = 0;
    R->n_long = 0;
    R->run_first = R->run_len = R->count = nullptr;
    if (T <= 0) return SBB_OK;
    const int cap = T / 2 + 1;
    if (dev_malloc_async((void **)&R->run_first, sizeof(int) * cap, s) != cudaSuccess ||
        dev_malloc_async((void **)&R->run_len, sizeof(int) * cap, s) != cudaSuccess ||
        dev_malloc_async((void **)&R->count, sizeof(int), s) != cudaSuccess) {
        set_error("carry runs: device allocation failed");
        return SBB_ERR_NOMEM;
    }
    R->bytes = 2 * sizeof(int) * (size_t)cap + sizeof(int);
    SBB_CUDA(cudaMemsetAsync(R->count, 0, sizeof(int), s));
    runs_mark_kernel<<<(T + FT - 1) / FT, FT, 0, s>>>(crow, T, m, R->run_first, R->run_len,
                                                      R->count);
    return SBB_OK;
}

void carry_runs_free(CarryRuns *R, cudaStream_t s, bool async)
{
    for (int *p : {R->run_first, R->run_len, R->count})
        if (p) {
            if (async)
                cudaFreeAsync(p, s);
            else
                cudaFree(p);
        }
    R->count = nullptr;
    R->run_first = R->run_len = nullptr;
    R->n_runs = 0;
    R->n_long = 0;
}

void launch_runs_mark(const int *crow, int T, int m, int *run_first, int *run_len,
                      int *dev_count, cudaStream_t s)
{
    if (T > 0)
        runs_mark_kernel<<<(T + FT - 1) / FT, FT, 0, s>>>(crow, T, m, run_first, run_len, dev_count);
}

void launch_fixup(int m, const int *crow, const double *cval, int T, const CarryRuns &R,
                  double alpha, double *y, unsigned *queue, cudaStream_t s, const int *dev_count)
{
    if (T <= 0) return;
    // single carries: one wave of blocks at most, each thread striding over tiles
    int short_blocks = (T + FT - 1) / FT;
    if (short_blocks > 148 * 8) short_blocks = 148 * 8;
    const int long_blocks = dev_count ? 148 : R.n_long;
    const int warp_blocks = dev_count ? 0 : (R.n_runs - R.n_long + FT / 32 - 1) / (FT / 32);
    // Programmatic dependent launch: the fix-up's blocks are placed while the
    // producing kernel drains and wait in grid_dependency_wait(), which hides
    // the launch gap between the two kernels.
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(short_blocks + long_blocks + warp_blocks);
    cfg.blockDim = dim3(FT);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, fixup_kernel, m, crow, cval, T, (const int *)R.run_first,
                       (const int *)R.run_len, long_blocks, R.n_long, R.n_runs, warp_blocks, alpha,
                       y, queue, dev_count);
}

}  // namespace sbb
