// Learned hash: a small MLP 128 -> 256 -> k (BF16 weights, FP32 accumulate)
// whose output signs replace random hyperplanes in the bucketing. Inference
// (fused with code packing) runs on the tensor cores; training kernels are in
// learned_train.cu. No counterpart in the reference, whose only hash is the
// random-hyperplane family of src/lsh_h.cu:88-100.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace sift {

constexpr int kMlpIn = 128;
constexpr int kMlpHidden = 256;
constexpr int kMlpMaxBits = 32;
constexpr int kMlpOutRows = 32;          // layer-2 rows as loaded (k padded with zeros)
constexpr float kMlpInScale = 1.0f / 64;  // inputs are u8 / 64 (exact in BF16)

// Model in device memory: z = W2 relu(W1 (x / 64) + b1) + b2, bit j of the
// code set when z_j > 0. The hidden activations are rounded to BF16 before
// layer 2 (the tensor-core operand type), in training as in inference.
struct MlpModel {
    const __nv_bfloat16* w1;  // [256][128]
    const float* b1;          // [256]
    const __nv_bfloat16* w2;  // [k][256]
    const float* b2;          // [k]
    int k;
};

// Codes (and optionally z, [n][k] floats) of n u8 rows. xmap: the rows (u8,
// box 128 x 128, 128-byte swizzle); w1map: the W1 tensor map (dims {128, 256},
// box {64, 256}); w2map: W2 (dims {256, k}, box {64, 32}).
cudaError_t launch_mlp_hash(const CUtensorMap& xmap, int n, const CUtensorMap& w1map, const CUtensorMap& w2map,
                            const float* b1, const float* b2, int k, uint32_t* codes, float* z, int* err,
                            int num_sms, cudaStream_t stream);
size_t mlp_hash_smem_bytes();

// Query-directed multi-probe: probe p of query i is codes[i] with the bits of
// the p-th lightest subset of its `flip` smallest-|z| bits flipped (subsets
// ordered by the sum of their |z|; probe 0 is the code itself). Writes
// probe_codes[p][n] for p < n_probes (n_probes <= 64, flip <= 6).
cudaError_t launch_probe_codes(const uint32_t* codes, const float* z, int n, int k, int flip, int n_probes,
                               uint32_t* probe_codes, cudaStream_t stream);

// ---- training (learned_train.cu)
// One training step's data: R = 3B gathered rows [queries | their exact
// nearest neighbours | random base rows].
struct MlpTrainBufs {
    float* h;        // [R][256] hidden (BF16-rounded, post-ReLU)
    float* t;        // [R][32] tanh(z)
    float* dz;       // [R][32]
    float* da1;      // [R][256] gradient at the hidden pre-activation
    float* colsum;   // [32] column sums of t
    float* loss;     // [4] total, positive, negative, balance
};
struct MlpParams {  // FP32 master copies (+ gradients, Adam moments: same layout)
    float* w1;  // [256][128]
    float* b1;  // [256]
    float* w2;  // [32][256] (rows >= k stay zero)
    float* b2;  // [32]
};
constexpr size_t kMlpParamCount = 256 * 128 + 256 + 32 * 256 + 32;
MlpParams mlp_params_at(float* base);

struct MlpLossWeights {
    float neg;      // weight of the negative-pair term mean(s_qn^2)
    float balance;  // weight of sum_j mean_i(t_ij)^2
};

// Forward, loss and gradients for rows x[R][128] (R = 3B), weights from the
// FP32 masters rounded to BF16 (w1b, w2b). Gradients are written (not
// accumulated) into g; deterministic (no atomics on parameters).
cudaError_t launch_mlp_loss_grad(const uint8_t* x, int B, int k, const MlpParams& p, const __nv_bfloat16* w1b,
                                 const __nv_bfloat16* w2b, const MlpLossWeights& lw, MlpTrainBufs& tb,
                                 const MlpParams& g, cudaStream_t stream);
// Adam step on every parameter; refreshes the BF16 copies. step starts at 1.
cudaError_t launch_mlp_adam(const MlpParams& p, const MlpParams& g, const MlpParams& m, const MlpParams& v, int k,
                            int step, float lr, __nv_bfloat16* w1b, __nv_bfloat16* w2b, cudaStream_t stream);
// FP32 masters -> BF16 copies (W1, W2 rows < k) and, when given, b1 / b2 (k entries).
cudaError_t launch_mlp_export(const MlpParams& p, int k, __nv_bfloat16* w1b, __nv_bfloat16* w2b, float* b1_out,
                              float* b2_out, cudaStream_t stream);
// Gathers the training rows of one step: for i < B with seed-derived choices
// qi in [0, t_n), rows q[qi], base[nn[2 qi]], base[ri] (ri in [0, r_n)).
cudaError_t launch_mlp_gather(const uint8_t* tq, int t_n, const int32_t* nn, const uint8_t* base, int r_n, int B,
                              unsigned long long seed, int step, uint8_t* x, cudaStream_t stream);

}  // namespace sift
