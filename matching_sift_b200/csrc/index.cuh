// Exact fallback of the hash searches (index.cu), shared by the persistent
// indexes and sift_mlp_match.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include "context.h"

namespace sift {

// Arena offsets of the fallback's scratch for at most q_n queries.
struct FallbackScratch {
    size_t o_fidx = 0, o_frows = 0, o_fm = 0, o_fi = 0, o_fd = 0, o_brec = 0, o_fqn = 0, o_fthr = 0, o_fpart = 0;
    size_t fb_part = 0;
    bool own_brec = false;
};
// Appends the fallback's regions to L. own_brec: also room for the base's
// tile records (when the caller has none precomputed).
void fallback_layout(detail::Layout& L, int q_n, int r_n, int num_workers, bool own_brec, FallbackScratch& fs);

// Flags the queries with fewer than min_cand candidates (counts) or, when
// max_dist > 0, a nearest candidate farther than max_dist (dist[2 q]), searches
// them exactly against r (records brec, or computed when null) and writes
// their results over the outputs. Synchronises `st` once (the flag count).
int exact_fallback(detail::DeviceCtx& c, char* A, const FallbackScratch& fs, const uint8_t* q, const uint8_t* r,
                   int q_n, int r_n, const int32_t* brec, const uint32_t* counts, const float* dist, int min_cand,
                   float max_dist, float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist,
                   uint32_t* fallback_count, cudaStream_t st);

}  // namespace sift
