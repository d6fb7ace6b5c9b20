// Exact 2-NN entry point that allocates no memory.
//
// Some callers cannot allocate device memory at call time: code running under
// a custom allocator or a memory pool that owns all device memory, real-time
// loops where cudaMalloc's implicit synchronisation is not acceptable, and
// hosts that hand this library a fixed memory budget up front. For them,
// sift2nn_match_noalloc runs the same search as sift2nn_match with every piece
// of scratch memory (base norm records, per-query norms and shared bounds,
// partial top-2 lists, the device status word) taken from one statically
// sized __device__ array of this library. The caller supplies the inputs and
// outputs; nothing is allocated, not even by the first call.
//
// Consequences for the caller:
//   * every GPU that loads the library holds the array (kNoAllocScratchBytes)
//     until the process exits;
//   * sizes are bounded: q_n <= kNoAllocMaxQueries, r_n <= kNoAllocMaxBase;
//     larger requests return SIFT_ERR_INVALID_ARG without launching anything;
//   * all calls on a device share the array, so calls whose kernels overlap
//     on the GPU (different streams, or different host threads) race on it:
//     serialise them (one stream, or events);
//   * the first call on a device resolves the array's device address with
//     cudaGetSymbolAddress (with that device current); make that first call
//     before any stream capture;
//   * a bounded wait that expires inside a call's search kernel (an error no
//     correct run produces) leaves that call's outputs marked "no result"
//     (UINT32_MAX, -1, FLT_MAX) rather than half written, and is reported by
//     sift2nn_noalloc_status, which reads a word in the same array (no
//     allocation there either).
#include <cfloat>
#include <climits>
#include <cstdint>
#include <functional>
#include <mutex>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include "sift2nn.h"
#include "context.h"
#include "exact2nn.cuh"

namespace sift {
namespace {

// Layout of the array: [0] this call's device error word (cleared by every
// call), [1] the sticky status word (set by any call whose search reported an
// error, cleared by sift2nn_noalloc_status), then 256-byte aligned regions.
constexpr size_t kNoAllocErrOff = 0;
constexpr size_t kNoAllocStickyOff = sizeof(int);
constexpr size_t kNoAllocHeader = 256;

// After the merge: if this call's search reported an error, its partial lists
// may be stale, so every output row is overwritten with "no result" and the
// error is recorded in the sticky word.
__global__ void noalloc_invalidate_kernel(const int* __restrict__ err, int* __restrict__ sticky, int q_n,
                                          uint32_t* __restrict__ matches, int32_t* __restrict__ nn_idx,
                                          float* __restrict__ nn_dist) {
    const int code = *err;
    if (code == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) atomicCAS(sticky, 0, code);
    if (i >= q_n) return;
    if (matches) matches[i] = UINT32_MAX;
    if (nn_idx) {
        nn_idx[2 * i] = -1;
        nn_idx[2 * i + 1] = -1;
    }
    if (nn_dist) {
        nn_dist[2 * i] = FLT_MAX;
        nn_dist[2 * i + 1] = FLT_MAX;
    }
}

constexpr uint32_t kNoAllocMaxQueries = 16384;
constexpr uint32_t kNoAllocMaxBase = 1u << 20;
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB per device
constexpr int kNoAllocMaxDevices = 64;

// The scratch. Host code must not use its name as an address: the device
// address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocDevice {
    std::once_flag once;
    int status = SIFT_ERR_NO_DEVICE;
    unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
    int num_sms = 0;
    PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
};
NoAllocDevice g_noalloc[kNoAllocMaxDevices];

void noalloc_setup(NoAllocDevice& d, int dev) {
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) { d.status = SIFT_ERR_CUDA; return; }
    if (prop.major != 10) { d.status = SIFT_ERR_UNSUPPORTED; return; }
    void* sym = nullptr;
    if (cudaGetSymbolAddress(&sym, g_noalloc_scratch) != cudaSuccess || !sym) {
        cudaGetLastError();
        d.status = SIFT_ERR_CUDA;
        return;
    }
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
        d.status = SIFT_ERR_CUDA;
        return;
    }
    d.scratch = static_cast<unsigned char*>(sym);
    d.num_sms = prop.multiProcessorCount;
    d.encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    d.status = SIFT_OK;
}

int encode_rows(const NoAllocDevice& d, CUtensorMap* m, const void* base, uint64_t rows, uint32_t box_rows) {
    cuuint64_t dims[2] = {static_cast<cuuint64_t>(kDim), static_cast<cuuint64_t>(rows)};
    cuuint64_t strides[1] = {static_cast<cuuint64_t>(kDim)};
    cuuint32_t box[2] = {static_cast<cuuint32_t>(kDim), box_rows};
    cuuint32_t estr[2] = {1, 1};
    return d.encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS
               ? SIFT_OK
               : SIFT_ERR_CUDA;
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

}  // namespace
}  // namespace sift

extern "C" SIFT_API int sift2nn_match_noalloc(const uint8_t* q, const uint8_t* r, uint32_t q_n, uint32_t r_n,
                                              float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist,
                                              void* stream) {
    using namespace sift;
    if (q_n > kNoAllocMaxQueries || r_n > kNoAllocMaxBase) return SIFT_ERR_INVALID_ARG;
    if ((q_n && !q) || (r_n && !r)) return SIFT_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(q) & 15) || (reinterpret_cast<uintptr_t>(r) & 15)) return SIFT_ERR_INVALID_ARG;
    if (q_n == 0) return SIFT_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
        cudaGetLastError();
        return SIFT_ERR_NO_DEVICE;
    }
    // Inputs and outputs must be memory the GPU reads and writes directly: a
    // host pointer would reach the tensor map or the kernel stores.
    // (cudaPointerGetAttributes allocates nothing.)
    using detail::is_device_accessible;
    if (!is_device_accessible(q) || (r_n && !is_device_accessible(r)) ||
        (matches && !is_device_accessible(matches)) || (nn_idx && !is_device_accessible(nn_idx)) ||
        (nn_dist && !is_device_accessible(nn_dist)))
        return SIFT_ERR_INVALID_ARG;
    NoAllocDevice& d = g_noalloc[dev];
    std::call_once(d.once, noalloc_setup, std::ref(d), dev);
    if (d.status != SIFT_OK) return d.status;

    const ExactPlan plan = make_exact_plan(static_cast<int>(q_n), static_cast<int>(r_n), d.num_sms / 2, 2);
    const size_t o_err = kNoAllocErrOff;
    size_t off = kNoAllocHeader;
    const size_t o_rec = off;
    off = align256(off + static_cast<size_t>(plan.base_tiles) * kRecInts * 4 + 16);
    const size_t o_qnorm = off;
    off = align256(off + static_cast<size_t>(plan.q_pad) * 4);
    const size_t o_thr = off;
    off = align256(off + static_cast<size_t>(plan.q_pad) * 4);
    const size_t o_part = off;
    off = align256(off + static_cast<size_t>(plan.max_splits) * plan.parts * plan.q_pad * sizeof(int4));
    if (off > kNoAllocScratchBytes) return SIFT_ERR_INVALID_ARG;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* S = d.scratch;
    int* err = reinterpret_cast<int*>(S + o_err);
    int32_t* rec = reinterpret_cast<int32_t*>(S + o_rec);
    int32_t* qnorm = reinterpret_cast<int32_t*>(S + o_qnorm);
    int32_t* thresh = reinterpret_cast<int32_t*>(S + o_thr);
    int4* partial = reinterpret_cast<int4*>(S + o_part);
    // The status word is the only scratch that must start at zero; every other
    // region is fully written by the kernels before it is read.
    if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return SIFT_ERR_CUDA;
    if (detail::maybe_inject_wait_expiry(err, st) != cudaSuccess) return SIFT_ERR_CUDA;
    if (launch_row_norms_u8(r, static_cast<int>(r_n), plan.r_pad, kMetricL2, nullptr, rec, nullptr, st) != cudaSuccess ||
        launch_row_norms_u8(q, static_cast<int>(q_n), plan.q_pad, kMetricL2, qnorm, nullptr, thresh, st) != cudaSuccess)
        return SIFT_ERR_CUDA;
    if (r_n > 0) {
        CUtensorMap qmap, bmap;
        if (encode_rows(d, &qmap, q, q_n, kBM) != SIFT_OK || encode_rows(d, &bmap, r, r_n, kBN / 2) != SIFT_OK)
            return SIFT_ERR_CUDA;
        if (launch_exact2nn_u8_pair(qmap, bmap, rec, plan, partial, thresh, err, st) != cudaSuccess)
            return SIFT_ERR_CUDA;
    }
    if (launch_merge2nn(partial, plan, qnorm, kMetricL2, threshold, 1.0f, matches, nullptr, nn_idx, nn_dist, st) !=
        cudaSuccess)
        return SIFT_ERR_CUDA;
    noalloc_invalidate_kernel<<<(q_n + 255) / 256, 256, 0, st>>>(err, reinterpret_cast<int*>(S + kNoAllocStickyOff),
                                                                 static_cast<int>(q_n), matches, nn_idx, nn_dist);
    if (cudaGetLastError() != cudaSuccess) return SIFT_ERR_CUDA;
    return SIFT_OK;
}

// Synchronises `stream` and reports whether a search of sift2nn_match_noalloc
// on the current device hit an expired bounded wait since the last check
// (SIFT_ERR_DEVICE_TIMEOUT; SIFT_OK otherwise), clearing the record. Reads the
// word through the array's device address: no allocation.
extern "C" SIFT_API int sift2nn_noalloc_status(void* stream) {
    using namespace sift;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
        cudaGetLastError();
        return SIFT_ERR_NO_DEVICE;
    }
    NoAllocDevice& d = g_noalloc[dev];
    std::call_once(d.once, noalloc_setup, std::ref(d), dev);
    if (d.status != SIFT_OK) return d.status;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int* sticky = reinterpret_cast<int*>(d.scratch + kNoAllocStickyOff);
    int word = 0;
    if (cudaStreamSynchronize(st) != cudaSuccess ||
        cudaMemcpyAsync(&word, sticky, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return SIFT_ERR_CUDA;
    if (word == 0) return SIFT_OK;
    if (cudaMemsetAsync(sticky, 0, sizeof(int), st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
        return SIFT_ERR_CUDA;
    return SIFT_ERR_DEVICE_TIMEOUT;
}
