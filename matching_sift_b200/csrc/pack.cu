// Input conversion kernels: float / half descriptors -> u8 (with an exactness
// flag). Replaces the reference's float2half (src/knn_brute.cu:315-338), which
// converted every batch to FP16; here descriptors whose values are integers in
// [0, 255], or such integers times one common power of two (the reference's
// own benchmark divides SIFT1M's integer components by 512, src/test.cu:99-103),
// are packed once to u8, the format the tensor-core kernel consumes.
#include <cuda_fp16.h>
#include "pack.cuh"

namespace sift {
namespace {

// v * mul (mul a power of two, so the product is exact) as u8; bad when it is
// not an integer in [0, 255].
__device__ __forceinline__ uint32_t to_u8(float v, float mul, bool& bad) {
    v *= mul;
    const float r = rintf(v);
    bad |= !(v >= 0.0f && v <= 255.0f && r == v);
    return static_cast<uint32_t>(fminf(fmaxf(r, 0.0f), 255.0f));
}

// n4: number of 4-element groups (n_elems / 4; n_elems is a multiple of 128).
__global__ void pack_f32_u8_kernel(const float4* __restrict__ x, size_t n4, float mul, uchar4* __restrict__ out,
                                   int* __restrict__ flag) {
    bool bad = false;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float4 v = x[i];
        uchar4 o;
        o.x = static_cast<unsigned char>(to_u8(v.x, mul, bad));
        o.y = static_cast<unsigned char>(to_u8(v.y, mul, bad));
        o.z = static_cast<unsigned char>(to_u8(v.z, mul, bad));
        o.w = static_cast<unsigned char>(to_u8(v.w, mul, bad));
        out[i] = o;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// n8: number of 8-element groups.
__global__ void pack_f16_u8_kernel(const uint4* __restrict__ x, size_t n8, float mul, uint2* __restrict__ out,
                                   int* __restrict__ flag) {
    bool bad = false;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n8;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint4 v = x[i];
        const __half2* h = reinterpret_cast<const __half2*>(&v);
        uint32_t b[8];
        #pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 f = __half22float2(h[k]);
            b[2 * k] = to_u8(f.x, mul, bad);
            b[2 * k + 1] = to_u8(f.y, mul, bad);
        }
        out[i] = make_uint2(b[0] | (b[1] << 8) | (b[2] << 16) | (b[3] << 24),
                            b[4] | (b[5] << 8) | (b[6] << 16) | (b[7] << 24));
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// Smallest s >= 0 with v * 2^s an integer, for finite v >= 0 (0 for v = 0).
__device__ __forceinline__ int int_shift(float v) {
    const uint32_t b = __float_as_uint(v);
    const int e = static_cast<int>((b >> 23) & 0xff);
    uint32_t m = b & 0x7fffffu;
    if (m == 0 && e == 0) return 0;
    int ex = e == 0 ? -149 : e - 150;  // v = m * 2^ex
    if (e != 0) m |= 0x800000u;
    ex += __ffs(static_cast<int>(m)) - 1;  // strip trailing zero bits of m
    return ex < 0 ? -ex : 0;
}

__device__ __forceinline__ void stat_one(float v, bool& bad, int& sh, float& mx) {
    bad |= !(v >= 0.0f && v <= 3.0e38f);
    if (v >= 0.0f && v <= 3.0e38f) {
        sh = max(sh, int_shift(v));
        mx = fmaxf(mx, v);
    }
}

// stats[0] |= 1 if any value is negative or not finite; stats[1] = max over
// values of int_shift; stats[2] = bit pattern of the largest value (the bit
// patterns of non-negative floats order like the values).
__device__ __forceinline__ void stats_flush(bool bad, int sh, float mx, int* stats) {
    const unsigned full = 0xffffffffu;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sh = max(sh, __shfl_xor_sync(full, sh, o));
        mx = fmaxf(mx, __shfl_xor_sync(full, mx, o));
    }
    bad = __any_sync(full, bad);
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicOr(stats, 1);
        atomicMax(stats + 1, sh);
        atomicMax(stats + 2, __float_as_int(mx));
    }
}

__global__ void stats_f32_kernel(const float4* __restrict__ x, size_t n4, int* __restrict__ stats) {
    bool bad = false;
    int sh = 0;
    float mx = 0.0f;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float4 v = x[i];
        stat_one(v.x, bad, sh, mx);
        stat_one(v.y, bad, sh, mx);
        stat_one(v.z, bad, sh, mx);
        stat_one(v.w, bad, sh, mx);
    }
    stats_flush(bad, sh, mx, stats);
}

__global__ void stats_f16_kernel(const uint4* __restrict__ x, size_t n8, int* __restrict__ stats) {
    bool bad = false;
    int sh = 0;
    float mx = 0.0f;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n8;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint4 v = x[i];
        const __half2* h = reinterpret_cast<const __half2*>(&v);
        #pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 f = __half22float2(h[k]);
            stat_one(f.x, bad, sh, mx);
            stat_one(f.y, bad, sh, mx);
        }
    }
    stats_flush(bad, sh, mx, stats);
}

// General (non-integer) descriptors: stats[0] |= 1 if a value is not finite,
// stats[1] = bit pattern of the largest |value|.
__device__ __forceinline__ void abs_one(float v, bool& bad, float& mx) {
    const float a = fabsf(v);
    bad |= !(a <= 3.0e38f);
    if (a <= 3.0e38f) mx = fmaxf(mx, a);
}

__device__ __forceinline__ void abs_flush(bool bad, float mx, int* stats) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    bad = __any_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicOr(stats, 1);
        atomicMax(stats + 1, __float_as_int(mx));
    }
}

__global__ void abs_stats_f32_kernel(const float4* __restrict__ x, size_t n4, int* __restrict__ stats) {
    bool bad = false;
    float mx = 0.0f;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float4 v = x[i];
        abs_one(v.x, bad, mx);
        abs_one(v.y, bad, mx);
        abs_one(v.z, bad, mx);
        abs_one(v.w, bad, mx);
    }
    abs_flush(bad, mx, stats);
}

__global__ void abs_stats_f16_kernel(const uint4* __restrict__ x, size_t n8, int* __restrict__ stats) {
    bool bad = false;
    float mx = 0.0f;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n8;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint4 v = x[i];
        const __half2* h = reinterpret_cast<const __half2*>(&v);
        #pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 f = __half22float2(h[k]);
            abs_one(f.x, bad, mx);
            abs_one(f.y, bad, mx);
        }
    }
    abs_flush(bad, mx, stats);
}

// Float rows -> split FP16 rows [n][256]: halves [0, 128) hold hi = fp16(x * mul)
// and [128, 256) lo = fp16(x * mul - hi), so hi + lo carries 22 significant
// bits of x * mul (mul a power of two: exact). Each thread converts 4
// consecutive elements of one row.
__global__ void pack_split_f16_kernel(const float4* __restrict__ x, size_t n4, float mul, __half* __restrict__ out) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float4 v = x[i];
        const size_t row = i >> 5, col = (i & 31) * 4;
        const float s[4] = {v.x * mul, v.y * mul, v.z * mul, v.w * mul};
        __half hi[4], lo[4];
        #pragma unroll
        for (int k = 0; k < 4; ++k) {
            hi[k] = __float2half_rn(s[k]);
            lo[k] = __float2half_rn(s[k] - __half2float(hi[k]));
        }
        __half* o = out + row * 256 + col;
        *reinterpret_cast<uint2*>(o) = *reinterpret_cast<const uint2*>(hi);
        *reinterpret_cast<uint2*>(o + 128) = *reinterpret_cast<const uint2*>(lo);
    }
}

unsigned grid_for(size_t items, int num_sms) {
    size_t blocks = (items + 255) / 256;
    const size_t cap = static_cast<size_t>(num_sms) * 8;
    if (blocks > cap) blocks = cap;
    return static_cast<unsigned>(blocks);
}

}  // namespace

cudaError_t launch_value_stats(const void* x, bool half, size_t n_rows, int* stats, int num_sms, cudaStream_t stream) {
    if (n_rows == 0) return cudaSuccess;
    if (half) {
        const size_t n8 = n_rows * 16;
        stats_f16_kernel<<<grid_for(n8, num_sms), 256, 0, stream>>>(reinterpret_cast<const uint4*>(x), n8, stats);
    } else {
        const size_t n4 = n_rows * 32;
        stats_f32_kernel<<<grid_for(n4, num_sms), 256, 0, stream>>>(reinterpret_cast<const float4*>(x), n4, stats);
    }
    return cudaGetLastError();
}

cudaError_t launch_abs_stats(const void* x, bool half, size_t n_rows, int* stats, int num_sms, cudaStream_t stream) {
    if (n_rows == 0) return cudaSuccess;
    if (half) {
        const size_t n8 = n_rows * 16;
        abs_stats_f16_kernel<<<grid_for(n8, num_sms), 256, 0, stream>>>(reinterpret_cast<const uint4*>(x), n8, stats);
    } else {
        const size_t n4 = n_rows * 32;
        abs_stats_f32_kernel<<<grid_for(n4, num_sms), 256, 0, stream>>>(reinterpret_cast<const float4*>(x), n4, stats);
    }
    return cudaGetLastError();
}

cudaError_t launch_pack_split_f16(const float* x, size_t n_rows, float mul, void* out, int num_sms,
                                  cudaStream_t stream) {
    const size_t n4 = n_rows * 32;
    if (n4 == 0) return cudaSuccess;
    pack_split_f16_kernel<<<grid_for(n4, num_sms), 256, 0, stream>>>(reinterpret_cast<const float4*>(x), n4, mul,
                                                                     static_cast<__half*>(out));
    return cudaGetLastError();
}

cudaError_t launch_pack_f32_u8(const float* x, size_t n_rows, float mul, uint8_t* out, int* flag, int num_sms,
                               cudaStream_t stream) {
    const size_t n4 = n_rows * 32;
    if (n4 == 0) return cudaSuccess;
    size_t blocks = (n4 + 255) / 256;
    const size_t cap = static_cast<size_t>(num_sms) * 8;
    if (blocks > cap) blocks = cap;
    pack_f32_u8_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(reinterpret_cast<const float4*>(x), n4,
                                                                         mul, reinterpret_cast<uchar4*>(out), flag);
    return cudaGetLastError();
}

cudaError_t launch_pack_f16_u8(const void* x, size_t n_rows, float mul, uint8_t* out, int* flag, int num_sms,
                               cudaStream_t stream) {
    const size_t n8 = n_rows * 16;
    if (n8 == 0) return cudaSuccess;
    size_t blocks = (n8 + 255) / 256;
    const size_t cap = static_cast<size_t>(num_sms) * 8;
    if (blocks > cap) blocks = cap;
    pack_f16_u8_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(reinterpret_cast<const uint4*>(x), n8,
                                                                         mul, reinterpret_cast<uint2*>(out), flag);
    return cudaGetLastError();
}

}  // namespace sift
