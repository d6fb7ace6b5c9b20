// Fault injection for the failure-detection tests. Neither hook faults, traps
// or hangs a GPU:
//
//  * sift_test_inject_wait_expiry(n): the next n exact searches (sift2nn_match
//    and its reference-named callers, sift2nn_match_noalloc) first launch a
//    one-thread probe kernel that waits, through the same bounded mbarrier
//    wait every pipeline stage of the search kernels uses, on a barrier that
//    nothing ever completes. The wait runs out after kProbeLimitNs, raises the
//    probe's abort flag and records kErrWaitProbe in the call's device status
//    word -- exactly what an expired wait inside a search kernel records -- and
//    the probe returns. The search itself then runs normally; the host sees
//    the error through the status paths (sift_stream_status,
//    sift2nn_noalloc_status) and the context stays usable.
//  * sift_test_fail_arena(n): the next n calls that need the scratch arena get
//    SIFT_ERR_ALLOC from it as if cudaMalloc had failed (host side only).
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>
#include "sift2nn.h"
#include "context.h"
#include "exact2nn.cuh"
#include "ptx.cuh"

namespace sift {
namespace {

constexpr uint64_t kProbeLimitNs = 1000000ull;  // 1 ms

std::atomic<int> g_inject_waits{0};
std::atomic<int> g_fail_arena{0};

__global__ void wait_probe_kernel(int* err, uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_flag;
    const uint32_t b = ptx::smem_u32(&bar);
    ptx::mbar_init(b, 1);
    abort_flag = 0;
    ptx::fence_mbar_init();
    // Phase 0 needs one arrival that never comes: the wait can only expire.
    ptx::mbar_wait_limit(b, 0, &abort_flag, err, kErrWaitProbe, limit_ns);
}

// Takes one unit from an armed counter; false when it is not armed.
bool take(std::atomic<int>& counter) {
    int v = counter.load();
    while (v > 0)
        if (counter.compare_exchange_weak(v, v - 1)) return true;
    return false;
}

}  // namespace

namespace detail {

cudaError_t maybe_inject_wait_expiry(int* err, cudaStream_t st) {
    if (!take(g_inject_waits)) return cudaSuccess;
    wait_probe_kernel<<<1, 1, 0, st>>>(err, kProbeLimitNs);
    ++g_launches;
    return cudaGetLastError();
}

bool arena_fault() { return take(g_fail_arena); }

}  // namespace detail
}  // namespace sift

extern "C" {

SIFT_API int sift_test_inject_wait_expiry(int calls) {
    if (calls < 0) return SIFT_ERR_INVALID_ARG;
    sift::g_inject_waits.store(calls);
    return SIFT_OK;
}

SIFT_API int sift_test_fail_arena(int calls) {
    if (calls < 0) return SIFT_ERR_INVALID_ARG;
    sift::g_fail_arena.store(calls);
    return SIFT_OK;
}

}  // extern "C"
