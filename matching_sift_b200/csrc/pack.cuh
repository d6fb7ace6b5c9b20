#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace sift {

// Convert n_rows x 128 float (resp. __half) descriptors times mul (a power of
// two) to u8. *flag |= 1 when any product is not an integer in [0, 255] (the
// u8 output is then clamped and must not be used for an exact search). x must
// be 16-byte aligned.
cudaError_t launch_pack_f32_u8(const float* x, size_t n_rows, float mul, uint8_t* out, int* flag, int num_sms,
                               cudaStream_t stream);
cudaError_t launch_pack_f16_u8(const void* x, size_t n_rows, float mul, uint8_t* out, int* flag, int num_sms,
                               cudaStream_t stream);

// Value statistics of n_rows x 128 float (half = false) or __half values,
// accumulated into stats[0..2] (caller zeroes them first):
//   stats[0] |= 1   some value is negative, infinite or NaN
//   stats[1]        max over values of the smallest s >= 0 making v * 2^s an integer
//   stats[2]        bit pattern of the largest value (as a float)
// The inputs are exact for the integer kernels with shift s = stats[1] when
// stats[0] == 0 and (largest value) * 2^s <= 255.
cudaError_t launch_value_stats(const void* x, bool half, size_t n_rows, int* stats, int num_sms, cudaStream_t stream);

// General descriptors (any finite float / half values), accumulated into
// stats[0..1] (caller zeroes them first): stats[0] |= 1 when a value is
// infinite or NaN, stats[1] = bit pattern of the largest |value|.
cudaError_t launch_abs_stats(const void* x, bool half, size_t n_rows, int* stats, int num_sms, cudaStream_t stream);

// Float rows -> split FP16 rows out[n_rows][256] (16-byte aligned): halves
// [0, 128) = hi = fp16(x * mul), [128, 256) = lo = fp16(x * mul - hi); mul is a
// power of two chosen so that the largest |x * mul| stays below the FP16 range.
cudaError_t launch_pack_split_f16(const float* x, size_t n_rows, float mul, void* out, int num_sms,
                                  cudaStream_t stream);

}  // namespace sift
