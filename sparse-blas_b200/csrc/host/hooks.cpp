// hooks.cpp — host-side fault injection for the library's own tests.
//
// The reference's entry points return 1 when a device allocation fails
// (SparseBLAS/src/dspmv_mgpu_baseline.cu:99-135) and -1 when the memory
// pre-check finds too little free memory (SparseBLAS/src/dspmv_mgpu_v1.cu:
// 104-116); the tiled kernel gives up a bounded wait with a timeout status.
// None of these happen on a healthy GPU with test-sized inputs, so the tests
// arm one of these hooks instead: every fault is made on the host (or by a
// wait budget of zero polls), never by faulting the GPU.
#include <atomic>

#include "../sbb_internal.h"

namespace sbb {

namespace {
std::atomic<long long> g_fail_alloc{0};    // k > 0: the k-th allocation from now fails
std::atomic<long long> g_free_cap{-1};     // >= 0: the pre-check sees at most this
std::atomic<int> g_first_wait{-1};         // >= 0: budget of the first tile-copy wait
}  // namespace

cudaError_t dev_malloc_async(void **p, size_t bytes, cudaStream_t s)
{
    long long k = g_fail_alloc.load();
    while (k > 0 && !g_fail_alloc.compare_exchange_weak(k, k - 1)) {
    }
    if (k == 1) {  // this is the armed allocation
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMallocAsync(p, bytes, s);
}

size_t capped_free_bytes(size_t free_b)
{
    const long long cap = g_free_cap.load();
    return cap >= 0 && (size_t)cap < free_b ? (size_t)cap : free_b;
}

int first_wait_budget() { return g_first_wait.load(); }

}  // namespace sbb

extern "C" int sbb_test_hook(int what, long long value)
{
    using namespace sbb;
    switch (what) {
    case SBB_TEST_RESET:
        g_fail_alloc = 0;
        g_free_cap = -1;
        g_first_wait = -1;
        return SBB_OK;
    case SBB_TEST_FAIL_ALLOC:
        if (value < 0) break;
        g_fail_alloc = value;
        return SBB_OK;
    case SBB_TEST_FREE_BYTES:
        g_free_cap = value < 0 ? -1 : value;
        return SBB_OK;
    case SBB_TEST_WAIT_BUDGET:
        if (value > (1 << 30)) break;
        g_first_wait = value < 0 ? -1 : (int)value;
        return SBB_OK;
    default:
        break;
    }
    set_error("sbb_test_hook: unknown hook or bad value");
    return SBB_ERR_ARG;
}
