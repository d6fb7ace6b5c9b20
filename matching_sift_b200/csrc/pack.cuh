#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace sift {

// Convert n_rows x 128 float (resp. __half) descriptors to u8. *flag |= 1 when
// any element is not an integer in [0, 255] (the u8 output is then clamped and
// must not be used for an exact search). x must be 16-byte aligned.
cudaError_t launch_pack_f32_u8(const float* x, size_t n_rows, uint8_t* out, int* flag, int num_sms,
                               cudaStream_t stream);
cudaError_t launch_pack_f16_u8(const void* x, size_t n_rows, uint8_t* out, int* flag, int num_sms,
                               cudaStream_t stream);

}  // namespace sift
