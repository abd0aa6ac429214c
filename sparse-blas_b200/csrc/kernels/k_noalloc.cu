// k_noalloc.cu — merge-path SpMV for callers that cannot allocate device
// memory.
//
// Some callers must not call cudaMalloc at all: code that runs where the
// device allocator is off limits (inside a memory-capped or pre-partitioned
// process, from a callback or real-time path that may not block on the
// allocator, or next to a framework that owns every byte of the device).  This
// entry point runs the same merge-path kernel as sbb_spmv with a merge plan,
// but its scratch (segment coordinates, per-segment carries, the carry-run
// list and a status word) lives in one file-scope __device__ array of fixed
// size, so the call allocates nothing: no cudaMalloc, no cudaFree, no
// allocating library routine.
//
// Limits and sharing:
//   * capacity: kMaxSegments warp segments of 32*kIpt merge items, i.e.
//     m + nnz <= 262,144 * 384 = 100,663,296; larger inputs are rejected;
//   * the array (about 5 MiB) is held by every GPU that loads the library,
//     until the process exits;
//   * every call shares it and it keeps the last call's contents: calls whose
//     work overlaps on the GPU (different streams or threads) race on it and
//     give wrong results - serialise them;
//   * the first call on a device looks up the array's device address (an
//     ordinary host-side step); make that first call before any stream
//     capture on that device.  The address is kept per device together with
//     the identity of the context it was found in, and looked up again when
//     that context has been replaced (after cudaDeviceReset, for example).
#include <cuda.h>  // driver types only; the entry points are fetched at run time

#include <mutex>

#include "../sbb_internal.h"

namespace sbb {

namespace {

constexpr int kIpt = 12;                       // merge items per lane
constexpr long long kItems = 32LL * kIpt;      // 384 merge items per warp segment
constexpr long long kMaxSegments = 1LL << 18;  // 262,144 segments

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kCoordBytes = align256(sizeof(int) * (kMaxSegments + 1));
constexpr size_t kCarryBytes = align256(sizeof(double) * kMaxSegments);
constexpr size_t kRunBytes = align256(sizeof(int) * (kMaxSegments / 2 + 1));
constexpr size_t kWordBytes = 256;  // run count, status
constexpr size_t kScratchBytes = 2 * kCoordBytes + kCarryBytes + 2 * kRunBytes + kWordBytes;

// The scratch.  In host code this name is only a host-side stand-in: kernels
// get its device address from cudaGetSymbolAddress (scratch_on_device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
struct ScratchAddr {
    void *ptr = nullptr;
    unsigned long long ctx = 0;  // identity of the context the address belongs to
};
ScratchAddr g_scratch_addr[64];

// Unique id of the calling thread's current context, or 0 when there is none
// or the driver cannot tell (cuCtxGetId, CUDA 12.0+).  The driver entry
// points are fetched through the runtime, so the library does not link
// libcuda itself.
unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    if (get_current(&c) != CUDA_SUCCESS || !c) return 0;
    unsigned long long id = 0;
    return get_id(c, &id) == CUDA_SUCCESS ? id : 0;
}

// Device address of the scratch on device `dev` (the current device): looked
// up with that device current the first time, and again whenever the
// device's context is not the one the cached address was found in.  When the
// context id is unknown the address is looked up on every call.
void *scratch_on_device(int dev)
{
    std::lock_guard<std::mutex> lock(g_mu);
    if (dev < 0 || dev >= 64) return nullptr;
    ScratchAddr &a = g_scratch_addr[dev];
    const unsigned long long ctx = current_context_id();
    if (a.ptr && ctx != 0 && a.ctx == ctx) return a.ptr;
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
        set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return nullptr;
    }
    a.ptr = p;
    a.ctx = current_context_id();  // the lookup made the primary context current
    return p;
}

}  // namespace

size_t noalloc_scratch_bytes() { return kScratchBytes; }
long long noalloc_max_items() { return kMaxSegments * kItems; }

}  // namespace sbb

using namespace sbb;

extern "C" int sbb_spmv_merge_noalloc(int m, int n, int nnz, const int *d_rowptr, const int *d_col,
                                      const double *d_val, double alpha, const double *d_x,
                                      double beta, double *d_y, void *stream)
{
    if (m < 0 || n < 0 || nnz < 0 || !d_rowptr || (nnz > 0 && (!d_col || !d_val || !d_x)) ||
        (m > 0 && !d_y)) {
        set_error("sbb_spmv_merge_noalloc: bad arguments");
        return SBB_ERR_ARG;
    }
    const long long items = (long long)m + nnz;
    if (items > kMaxSegments * kItems) {
        set_error("sbb_spmv_merge_noalloc: m + nnz = " + std::to_string(items) +
                  " exceeds the fixed scratch capacity of " +
                  std::to_string(kMaxSegments * kItems) + " merge items");
        return SBB_ERR_ARG;
    }
    if (ranges_overlap(d_x, (size_t)n * 8, d_y, (size_t)m * 8)) {
        set_error("sbb_spmv_merge_noalloc: x and y overlap");
        return SBB_ERR_ARG;
    }
    if (m == 0) return SBB_OK;
    int dev = 0;
    SBB_CUDA(cudaGetDevice(&dev));
    auto *base = static_cast<unsigned char *>(scratch_on_device(dev));
    if (!base) return SBB_ERR_CUDA;
    auto s = static_cast<cudaStream_t>(stream);
    int *tile_row = reinterpret_cast<int *>(base);
    int *tile_nnz = reinterpret_cast<int *>(base + kCoordBytes);
    double *carry_val = reinterpret_cast<double *>(base + 2 * kCoordBytes);
    int *run_first = reinterpret_cast<int *>(base + 2 * kCoordBytes + kCarryBytes);
    int *run_len = reinterpret_cast<int *>(base + 2 * kCoordBytes + kCarryBytes + kRunBytes);
    int *words = reinterpret_cast<int *>(base + 2 * kCoordBytes + kCarryBytes + 2 * kRunBytes);
    int *run_count = words;
    unsigned *status = reinterpret_cast<unsigned *>(words + 1);
    const int tiles = (int)((items + kItems - 1) / kItems);

    // The array keeps the previous call's contents: clear what must start at 0.
    SBB_CUDA(cudaMemsetAsync(words, 0, kWordBytes, s));
    launch_merge_partition(d_rowptr, m, 0, nnz, kItems, tiles, tile_row, tile_nnz, s);
    launch_runs_mark(tile_row + 1, tiles, m, run_first, run_len, run_count, s);
    CsrView A{m, n, d_rowptr, d_col, d_val};
    CarryRuns runs;
    runs.run_first = run_first;
    runs.run_len = run_len;
    MergeScratch S{tile_row, tile_nnz, carry_val, &runs, run_count, tiles, nullptr, 0, 1};
    launch_merge(A, kIpt, S, alpha, d_x, beta, d_y, status, s);
    SBB_CUDA(cudaGetLastError());
    return SBB_OK;
}
