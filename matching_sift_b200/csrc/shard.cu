// Merge of 2-NN results searched over disjoint base shards (one per rank of a
// base-sharded search): per query the lexicographic (distance, global index)
// top-2 of the shards' top-2 lists, then the ratio test -- the same order and
// test as the single-search merge (merge2nn_kernel), so a base split over G
// searches gives the unsplit result. The reference has no multi-GPU path.
#include <cfloat>
#include <climits>
#include <cmath>
#include "api_internal.h"
#include "context.h"

namespace sift {
namespace {

using detail::DeviceCtx;
constexpr int kMaxParts = 64;
struct PartOffsets {
    int off[kMaxParts];
};

__global__ void __launch_bounds__(256) merge_parts_kernel(const float* __restrict__ dist,
                                                          const int32_t* __restrict__ idx, PartOffsets po, int parts,
                                                          int q_n, float thr, uint32_t* __restrict__ matches,
                                                          int32_t* __restrict__ nn_idx, float* __restrict__ nn_dist) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= q_n) return;
    float d1 = FLT_MAX, d2 = FLT_MAX;
    int j1 = -1, j2 = -1;
    auto less = [](float da, int ia, float db, int ib) { return da < db || (da == db && ia < ib); };
    for (int p = 0; p < parts; ++p) {
        const size_t base = (static_cast<size_t>(p) * q_n + q) * 2;
        #pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int li = idx[base + e];
            if (li < 0) continue;
            const int gi = li + po.off[p];
            const float d = dist[base + e];
            if (j1 < 0 || less(d, gi, d1, j1)) {
                d2 = d1; j2 = j1;
                d1 = d; j1 = gi;
            } else if (j2 < 0 || less(d, gi, d2, j2)) {
                d2 = d; j2 = gi;
            }
        }
    }
    if (matches) {
        bool pass = false;
        if (j1 >= 0) {
            const float f1 = sqrtf(d1);
            const float f2 = j2 >= 0 ? sqrtf(d2) : INFINITY;
            pass = (f1 / f2) < thr;
        }
        matches[q] = pass ? static_cast<uint32_t>(j1) : UINT32_MAX;
    }
    if (nn_idx) {
        nn_idx[2 * static_cast<size_t>(q)] = j1;
        nn_idx[2 * static_cast<size_t>(q) + 1] = j2;
    }
    if (nn_dist) {
        nn_dist[2 * static_cast<size_t>(q)] = j1 >= 0 ? d1 : FLT_MAX;
        nn_dist[2 * static_cast<size_t>(q) + 1] = j2 >= 0 ? d2 : FLT_MAX;
    }
}

}  // namespace

int merge_top2_parts(const float* dist, const int32_t* idx, const int32_t* offsets, int parts, uint32_t q_n,
                     float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist, void* stream) {
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    if (parts < 1 || parts > kMaxParts || q_n > 0x7fffffffu || (parts > 0 && !offsets)) return SIFT_ERR_INVALID_ARG;
    if (q_n == 0) return SIFT_OK;
    if (!dist || !idx || !detail::is_device_accessible(dist) || !detail::is_device_accessible(idx))
        return SIFT_ERR_INVALID_ARG;
    for (const void* o : {static_cast<const void*>(matches), static_cast<const void*>(nn_idx),
                          static_cast<const void*>(nn_dist)})
        if (o && !detail::is_device_accessible(o)) return SIFT_ERR_INVALID_ARG;
    PartOffsets po{};
    for (int p = 0; p < parts; ++p) {
        if (offsets[p] < 0) return SIFT_ERR_INVALID_ARG;
        po.off[p] = offsets[p];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    merge_parts_kernel<<<(q_n + 255) / 256, 256, 0, st>>>(dist, idx, po, parts, static_cast<int>(q_n), threshold,
                                                          matches, nn_idx, nn_dist);
    SIFT_CUDA(cudaGetLastError());
    ++detail::g_launches;
    return SIFT_OK;
}

}  // namespace sift

extern "C" {

int sift_merge_top2(const float* nn_dist_parts, const int32_t* nn_idx_parts, const int32_t* offsets, int parts,
                    uint32_t q_n, float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist, void* stream) {
    return sift::merge_top2_parts(nn_dist_parts, nn_idx_parts, offsets, parts, q_n, threshold, matches, nn_idx,
                                  nn_dist, stream);
}

}  // extern "C"
