// LSH kernels (lsh.cu): hashing on the tensor cores, bucket build, candidate scan.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>
#include "exact2nn.cuh"

namespace sift {

constexpr int kLshMaxPlanes = 256;  // L * k (hash bits over all tables)
constexpr int kLshMaxTopBits = 16;  // bucket groups: top min(k, 16) code bits

// Hyperplane rows padded to a multiple of 32 (the MMA N and the TMEM slot).
int lsh_planes_padded(int L, int k);
size_t lsh_hash_smem(int P);

// codes[t][i] (t < L, i < n): bit j set when x_i . planes[t * k + j] < 0.
// xmap: u8 rows [n][128], box 128 rows; pmap: s8 rows [L * k][128], box P rows.
// z (optional): the dot products themselves, z[t][i][j] as floats (exact), the
// margins that multi-probe ranks bits by.
cudaError_t launch_lsh_hash(const CUtensorMap& xmap, const CUtensorMap& pmap, int n, int P, int L, int k,
                            uint32_t* codes, float* z, int* err, int num_sms, cudaStream_t stream);

// Groups the n base points of every table by the top code bits
// (bin = code >> shift, nbins = 2^(k - shift)): start[t][0..nbins] offsets,
// order[t][pos] point ids, ocode[t][pos] their codes. hist: [L][nbins] scratch.
cudaError_t launch_lsh_buckets(const uint32_t* codes, int n, int L, int shift, int nbins, int* hist, int* start,
                               int* order, uint32_t* ocode, int num_sms, cudaStream_t stream);

// Exact 2-NN of every query over the union of its buckets: qcodes[L * probes][q_n],
// code c of a query searching table c / probes (probes = 1: its own code in
// every table). ratio != 0 applies the Lowe test with `thr` to `matches`;
// otherwise matches = nearest. dist_scale multiplies the distances (2^-2s for
// inputs scaled by 2^-s). counts (optional): candidates compared per query.
cudaError_t launch_lsh_scan(const uint8_t* q, const uint8_t* r, int q_n, int r_n, int L, int probes, int shift,
                            int nbins, const uint32_t* qcodes, const int* start, const int* order,
                            const uint32_t* ocode, float thr, int ratio, float dist_scale, uint32_t* matches,
                            uint32_t* counts, int32_t* nn_idx, float* nn_dist, cudaStream_t stream);

// General float (half = false) or half rows (lsh_float.cu): codes[t][i] bit j
// set when the FP32 dot product of row i with planes[t * k + j] (int8,
// [L * k][128] device, 16-byte aligned) is negative; z (optional) the dot
// products [t][i][j].
cudaError_t launch_lsh_hash_float(const void* x, bool half, int n, const int8_t* planes, int L, int k,
                                  uint32_t* codes, float* z, cudaStream_t stream);
// The candidate scan of launch_lsh_scan on float / half rows (FP32 squared
// distances).
cudaError_t launch_lsh_scan_float(const void* q, const void* r, bool half, int q_n, int r_n, int L, int probes,
                                  int shift, int nbins, const uint32_t* qcodes, const int* start, const int* order,
                                  const uint32_t* ocode, float thr, int ratio, uint32_t* matches, uint32_t* counts,
                                  int32_t* nn_idx, float* nn_dist, cudaStream_t stream);

}  // namespace sift
