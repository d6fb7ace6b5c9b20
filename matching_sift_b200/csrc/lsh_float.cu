// Random-hyperplane LSH for general float / half descriptors (values that are
// not integers times one power of two, e.g. the reference benchmark's
// unit-normalised rand() vectors, src/helper.cu:40-58). The u8 path's hash
// (exact int8 dot products on the tensor cores) and candidate scan (exact
// integer distances) need integer rows; these CUDA-core kernels do the same
// work in FP32 on the caller's rows:
//
//   lsh_hash_float_kernel   bit j of a point's code is set when its FP32 dot
//                           product with hyperplane j is negative (set_bit_h,
//                           src/lsh_h.cu:302-309; the reference forms the dot
//                           products in FP16 with cublasHgemm, :909, so the two
//                           agree except on points with a dot product near 0)
//   lsh_scan_float_kernel   exact-arithmetic-order FP32 squared distances to
//                           the members of the query's buckets, lexicographic
//                           (distance, index) top-2 as the u8 scan
//
// Buckets are the u8 path's (lsh.cu counting sort on the codes).
#include <cfloat>
#include <climits>
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include "exact2nn.cuh"
#include "lsh.cuh"

namespace sift {
namespace {

__device__ __forceinline__ void load4(const float* x, size_t off, float (&v)[4]) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(x + off));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void load4(const __half* x, size_t off, float (&v)[4]) {
    const uint2 a = __ldg(reinterpret_cast<const uint2*>(x + off));
    const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&a.x));
    const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&a.y));
    v[0] = lo.x; v[1] = lo.y; v[2] = hi.x; v[3] = hi.y;
}

// One warp per row (8 rows per block of 256): lane l holds elements
// [4 l, 4 l + 4); per hyperplane a partial dot and a 5-step shuffle sum (fixed
// order: deterministic). planes: [L * k][128] int8, staged in shared memory.
template <typename T>
__global__ void __launch_bounds__(256) lsh_hash_float_kernel(const T* __restrict__ x, int n,
                                                             const int8_t* __restrict__ planes, int L, int k,
                                                             uint32_t* __restrict__ codes, float* __restrict__ z) {
    extern __shared__ int8_t p_s[];
    const int np = L * k;
    for (int i = threadIdx.x; i < np * kDim / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(p_s)[i] = reinterpret_cast<const uint4*>(planes)[i];
    __syncthreads();
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    float v[4];
    load4(x, static_cast<size_t>(row) * kDim + 4 * lane, v);
    uint32_t code = 0;
    for (int j = 0; j < np; ++j) {
        const char4 p = *reinterpret_cast<const char4*>(p_s + j * kDim + 4 * lane);
        float d = v[0] * static_cast<float>(p.x);
        d = fmaf(v[1], static_cast<float>(p.y), d);
        d = fmaf(v[2], static_cast<float>(p.z), d);
        d = fmaf(v[3], static_cast<float>(p.w), d);
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        const int t = j / k, b = j - t * k;
        if (d < 0.0f) code |= 1u << b;
        if (z && lane == 0) z[(static_cast<size_t>(t) * n + row) * k + b] = d;
        if (b == k - 1) {
            if (lane == 0) codes[static_cast<size_t>(t) * n + row] = code;
            code = 0;
        }
    }
}

__device__ __forceinline__ bool lex_lt(int da, int ia, int db, int ib) { return da < db || (da == db && ia < ib); }

__device__ __forceinline__ void push_dedup(int d, int i, int& d1, int& i1, int& d2, int& i2) {
    if (i < 0 || i == i1 || i == i2) return;
    if (i1 < 0 || lex_lt(d, i, d1, i1)) {
        d2 = d1; i2 = i1;
        d1 = d; i1 = i;
    } else if (i2 < 0 || lex_lt(d, i, d2, i2)) {
        d2 = d; i2 = i;
    }
}

// One warp per query, buckets walked 32 positions at a time as in the u8
// scan; every 8 lanes score one candidate (lane part p: elements
// [16 p, 16 p + 16)), 4 candidates per step; squared distances in FP32 with
// a fixed summation order, compared as float_key images (distances are >= 0).
template <typename T>
__global__ void __launch_bounds__(256) lsh_scan_float_kernel(
    const T* __restrict__ q, const T* __restrict__ r, int q_n, int r_n, int L, int probes, int shift, int nbins,
    const uint32_t* __restrict__ qcodes, const int* __restrict__ start, const int* __restrict__ order,
    const uint32_t* __restrict__ ocode, float thr, int ratio, uint32_t* __restrict__ matches,
    uint32_t* __restrict__ counts, int32_t* __restrict__ nn_idx, float* __restrict__ nn_dist) {
    __shared__ int s_ids[8][32];
    const int wq = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int sub = lane >> 3, part = lane & 7;
    if (wq >= q_n) return;
    int* ids = s_ids[threadIdx.x >> 5];
    float qv[16];
    #pragma unroll
    for (int c = 0; c < 4; ++c) {
        float t4[4];
        load4(q, static_cast<size_t>(wq) * kDim + 16 * part + 4 * c, t4);
        #pragma unroll
        for (int e = 0; e < 4; ++e) qv[4 * c + e] = t4[e];
    }
    const bool whole_bins = shift == 0;
    int d1 = INT_MAX, i1 = -1, d2 = INT_MAX, i2 = -1;
    uint32_t seen = 0;
    for (int t = 0; t < L; ++t) {
        // The table's probe codes and bucket bounds, one probe per lane
        // (probes <= 64: two per lane), fetched in parallel.
        const int* st = start + static_cast<size_t>(t) * (nbins + 1);
        const uint32_t* tq = qcodes + static_cast<size_t>(t) * probes * q_n + wq;
        uint32_t pc0 = 0, pc1 = 0;
        int ps0 = 0, pe0 = 0, ps1 = 0, pe1 = 0;
        if (lane < probes) pc0 = tq[static_cast<size_t>(lane) * q_n];
        if (lane + 32 < probes) pc1 = tq[static_cast<size_t>(lane + 32) * q_n];
        if (lane < probes) {
            const int b = static_cast<int>(pc0 >> shift);
            ps0 = st[b];
            pe0 = st[b + 1];
        }
        if (lane + 32 < probes) {
            const int b = static_cast<int>(pc1 >> shift);
            ps1 = st[b];
            pe1 = st[b + 1];
        }
        for (int pi = 0; pi < probes; ++pi) {
            const bool lo = pi < 32;
            const uint32_t code = __shfl_sync(0xffffffffu, lo ? pc0 : pc1, pi & 31);
            // A repeated probe code (fewer distinct probes than requested) is skipped.
            if (__any_sync(0xffffffffu, (lane < pi && pc0 == code) || (lane + 32 < pi && pc1 == code))) continue;
            const int s = __shfl_sync(0xffffffffu, lo ? ps0 : ps1, pi & 31);
            const int e = __shfl_sync(0xffffffffu, lo ? pe0 : pe1, pi & 31);
            const int* ord = order + static_cast<size_t>(t) * r_n;
            const uint32_t* oc = ocode + static_cast<size_t>(t) * r_n;
            for (int p0 = s; p0 < e; p0 += 32) {
                const int p = p0 + lane;
                const bool hit = p < e && (whole_bins || oc[p] == code);
                const uint32_t mask = __ballot_sync(0xffffffffu, hit);
                const int nm = __popc(mask);
                if (nm == 0) continue;
                seen += nm;
                if (hit) ids[__popc(mask & ((1u << lane) - 1u))] = ord[p];
                __syncwarp();
                for (int j = 0; 4 * j < nm; ++j) {
                    const int rank = 4 * j + sub;
                    const int cid = rank < nm ? ids[rank] : -1;
                    float dist = 0.0f;
                    if (cid >= 0) {
                        #pragma unroll
                        for (int cc = 0; cc < 4; ++cc) {
                            float b4[4];
                            load4(r, static_cast<size_t>(cid) * kDim + 16 * part + 4 * cc, b4);
                            #pragma unroll
                            for (int ee = 0; ee < 4; ++ee) {
                                const float df = qv[4 * cc + ee] - b4[ee];
                                dist = fmaf(df, df, dist);
                            }
                        }
                    }
                    dist += __shfl_xor_sync(0xffffffffu, dist, 1);
                    dist += __shfl_xor_sync(0xffffffffu, dist, 2);
                    dist += __shfl_xor_sync(0xffffffffu, dist, 4);
                    if (part == 0 && cid >= 0) push_dedup(float_key(dist), cid, d1, i1, d2, i2);
                }
                __syncwarp();
            }
        }
    }
    #pragma unroll
    for (int o = 8; o < 32; o <<= 1) {
        const int od1 = __shfl_xor_sync(0xffffffffu, d1, o), oi1 = __shfl_xor_sync(0xffffffffu, i1, o);
        const int od2 = __shfl_xor_sync(0xffffffffu, d2, o), oi2 = __shfl_xor_sync(0xffffffffu, i2, o);
        push_dedup(od1, oi1, d1, i1, d2, i2);
        push_dedup(od2, oi2, d1, i1, d2, i2);
    }
    if (lane == 0) {
        if (counts) counts[wq] = seen;
        const bool v1 = i1 >= 0, v2 = i2 >= 0;
        const float f1 = v1 ? key_float(d1) : FLT_MAX;
        const float f2 = v2 ? key_float(d2) : FLT_MAX;
        if (matches) {
            bool pass = v1;
            if (v1 && ratio) pass = (sqrtf(f1) / (v2 ? sqrtf(f2) : INFINITY)) < thr;
            matches[wq] = pass ? static_cast<uint32_t>(i1) : UINT32_MAX;
        }
        if (nn_idx) {
            nn_idx[2 * wq] = i1;
            nn_idx[2 * wq + 1] = i2;
        }
        if (nn_dist) {
            nn_dist[2 * wq] = f1;
            nn_dist[2 * wq + 1] = f2;
        }
    }
}

}  // namespace

cudaError_t launch_lsh_hash_float(const void* x, bool half, int n, const int8_t* planes, int L, int k,
                                  uint32_t* codes, float* z, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const size_t smem = static_cast<size_t>(L) * k * kDim;
    const unsigned blocks = static_cast<unsigned>((n + 7) / 8);
    if (half)
        lsh_hash_float_kernel<__half><<<blocks, 256, smem, stream>>>(static_cast<const __half*>(x), n, planes, L, k,
                                                                     codes, z);
    else
        lsh_hash_float_kernel<float><<<blocks, 256, smem, stream>>>(static_cast<const float*>(x), n, planes, L, k,
                                                                    codes, z);
    return cudaGetLastError();
}

cudaError_t launch_lsh_scan_float(const void* q, const void* r, bool half, int q_n, int r_n, int L, int probes,
                                  int shift, int nbins, const uint32_t* qcodes, const int* start, const int* order,
                                  const uint32_t* ocode, float thr, int ratio, uint32_t* matches, uint32_t* counts,
                                  int32_t* nn_idx, float* nn_dist, cudaStream_t stream) {
    if (q_n <= 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((static_cast<long long>(q_n) * 32 + 255) / 256);
    if (half)
        lsh_scan_float_kernel<__half><<<blocks, 256, 0, stream>>>(
            static_cast<const __half*>(q), static_cast<const __half*>(r), q_n, r_n, L, probes, shift, nbins, qcodes,
            start, order, ocode, thr, ratio, matches, counts, nn_idx, nn_dist);
    else
        lsh_scan_float_kernel<float><<<blocks, 256, 0, stream>>>(
            static_cast<const float*>(q), static_cast<const float*>(r), q_n, r_n, L, probes, shift, nbins, qcodes,
            start, order, ocode, thr, ratio, matches, counts, nn_idx, nn_dist);
    return cudaGetLastError();
}

}  // namespace sift
