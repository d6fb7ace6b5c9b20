// Input conversion kernels: float / half descriptors -> u8 (with an exactness
// flag). Replaces the reference's float2half (src/knn_brute.cu:315-338), which
// converted every batch to FP16; here integer-valued descriptors in [0, 255]
// are packed once to u8, the format the tensor-core kernel consumes.
#include <cuda_fp16.h>
#include "pack.cuh"

namespace sift {
namespace {

__device__ __forceinline__ uint32_t to_u8(float v, bool& bad) {
    const float r = rintf(v);
    bad |= !(v >= 0.0f && v <= 255.0f && r == v);
    return static_cast<uint32_t>(fminf(fmaxf(r, 0.0f), 255.0f));
}

// n4: number of 4-element groups (n_elems / 4; n_elems is a multiple of 128).
__global__ void pack_f32_u8_kernel(const float4* __restrict__ x, size_t n4, uchar4* __restrict__ out,
                                   int* __restrict__ flag) {
    bool bad = false;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float4 v = x[i];
        uchar4 o;
        o.x = static_cast<unsigned char>(to_u8(v.x, bad));
        o.y = static_cast<unsigned char>(to_u8(v.y, bad));
        o.z = static_cast<unsigned char>(to_u8(v.z, bad));
        o.w = static_cast<unsigned char>(to_u8(v.w, bad));
        out[i] = o;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// n8: number of 8-element groups.
__global__ void pack_f16_u8_kernel(const uint4* __restrict__ x, size_t n8, uint2* __restrict__ out,
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
            b[2 * k] = to_u8(f.x, bad);
            b[2 * k + 1] = to_u8(f.y, bad);
        }
        out[i] = make_uint2(b[0] | (b[1] << 8) | (b[2] << 16) | (b[3] << 24),
                            b[4] | (b[5] << 8) | (b[6] << 16) | (b[7] << 24));
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

}  // namespace

cudaError_t launch_pack_f32_u8(const float* x, size_t n_rows, uint8_t* out, int* flag, int num_sms,
                               cudaStream_t stream) {
    const size_t n4 = n_rows * 32;
    if (n4 == 0) return cudaSuccess;
    size_t blocks = (n4 + 255) / 256;
    const size_t cap = static_cast<size_t>(num_sms) * 8;
    if (blocks > cap) blocks = cap;
    pack_f32_u8_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(reinterpret_cast<const float4*>(x), n4,
                                                                         reinterpret_cast<uchar4*>(out), flag);
    return cudaGetLastError();
}

cudaError_t launch_pack_f16_u8(const void* x, size_t n_rows, uint8_t* out, int* flag, int num_sms,
                               cudaStream_t stream) {
    const size_t n8 = n_rows * 16;
    if (n8 == 0) return cudaSuccess;
    size_t blocks = (n8 + 255) / 256;
    const size_t cap = static_cast<size_t>(num_sms) * 8;
    if (blocks > cap) blocks = cap;
    pack_f16_u8_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(reinterpret_cast<const uint4*>(x), n8,
                                                                         reinterpret_cast<uint2*>(out), flag);
    return cudaGetLastError();
}

}  // namespace sift
