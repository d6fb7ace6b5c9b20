// Training kernels of the learned hash (forward, loss, backward, Adam).
//
// Model (learned.cuh): a1 = W1 (x / 64) + b1, h = bf16(relu(a1)),
// z = W2 h + b2, t = tanh(z) (the sign surrogate; codes use sign(z)).
// One step sees R = 3B rows: B training queries, their exact nearest
// neighbours (labelled by the exact search kernel) and B random base rows.
// With s(a, b) = (1/k) sum_j t_aj t_bj and m_j = mean over the R rows of t_j:
//   loss = mean_i (1 - s(q_i, p_i)) + neg * mean_i s(q_i, n_i)^2 + balance * sum_j m_j^2
// (neighbours agree bit by bit, random pairs decorrelate, every bit splits
// the data evenly). Gradients pass straight through the BF16 roundings of the
// weights and of h. Every reduction runs in a fixed order, so a step is
// deterministic.
#include <cmath>
#include <cstdint>
#include <cuda_bf16.h>
#include "learned.cuh"

namespace sift {
namespace {

constexpr int kFwdRows = 32;
constexpr size_t kFwdSmem = kMlpIn * kMlpHidden * 2 + kMlpHidden * kMlpOutRows * 4 + kFwdRows * kMlpIn * 4 +
                            kFwdRows * kMlpHidden * 4;

// Block of 256 threads per 32 rows. Thread j: hidden unit j of the 32 rows;
// then 4 (row, output) pairs of layer 2.
__global__ void __launch_bounds__(256) mlp_fwd_kernel(const uint8_t* __restrict__ x, int R,
                                                      const __nv_bfloat16* __restrict__ w1b,
                                                      const float* __restrict__ b1,
                                                      const __nv_bfloat16* __restrict__ w2b,
                                                      const float* __restrict__ b2, int k, float* __restrict__ h_out,
                                                      float* __restrict__ t_out) {
    extern __shared__ uint8_t smem[];
    __nv_bfloat16* w1t = reinterpret_cast<__nv_bfloat16*>(smem);                 // [128][256]
    float* w2t = reinterpret_cast<float*>(smem + kMlpIn * kMlpHidden * 2);          // [256][32]
    float* xs = w2t + kMlpHidden * kMlpOutRows;                                     // [32][128]
    float* hs = xs + kFwdRows * kMlpIn;                                             // [32][256]
    const int tid = threadIdx.x;
    for (int e = tid; e < kMlpIn * kMlpHidden; e += 256) {
        const int j = e / kMlpIn, i = e % kMlpIn;
        w1t[i * kMlpHidden + j] = w1b[e];
    }
    for (int e = tid; e < kMlpOutRows * kMlpHidden; e += 256) {
        const int m = e / kMlpHidden, j = e % kMlpHidden;
        w2t[j * kMlpOutRows + m] = m < k ? __bfloat162float(w2b[e]) : 0.0f;
    }
    const int row0 = blockIdx.x * kFwdRows;
    for (int e = tid; e < kFwdRows * kMlpIn; e += 256) {
        const int r = e / kMlpIn;
        xs[e] = row0 + r < R ? static_cast<float>(x[static_cast<size_t>(row0) * kMlpIn + e]) * kMlpInScale : 0.0f;
    }
    __syncthreads();
    {
        const int j = tid;
        float acc[kFwdRows];
        #pragma unroll
        for (int r = 0; r < kFwdRows; ++r) acc[r] = 0.0f;
        for (int i = 0; i < kMlpIn; ++i) {
            const float w = __bfloat162float(w1t[i * kMlpHidden + j]);
            #pragma unroll
            for (int r = 0; r < kFwdRows; ++r) acc[r] = fmaf(xs[r * kMlpIn + i], w, acc[r]);
        }
        const float bj = b1[j];
        #pragma unroll
        for (int r = 0; r < kFwdRows; ++r) {
            const float hv = __bfloat162float(__float2bfloat16_rn(fmaxf(acc[r] + bj, 0.0f)));
            hs[r * kMlpHidden + j] = hv;
            if (row0 + r < R) h_out[static_cast<size_t>(row0 + r) * kMlpHidden + j] = hv;
        }
    }
    __syncthreads();
    const int m = tid & 31;
    for (int r = tid >> 5; r < kFwdRows; r += 8) {
        float acc = 0.0f;
        for (int j = 0; j < kMlpHidden; ++j) acc = fmaf(hs[r * kMlpHidden + j], w2t[j * kMlpOutRows + m], acc);
        if (row0 + r < R)
            t_out[static_cast<size_t>(row0 + r) * kMlpOutRows + m] = m < k ? tanhf(acc + b2[m]) : 0.0f;
    }
}

// colsum[m] = sum over rows of a[row][m] (width 32), one block, fixed order.
__global__ void __launch_bounds__(1024) colsum32_kernel(const float* __restrict__ a, int R, float* __restrict__ out) {
    __shared__ float part[32][33];
    const int m = threadIdx.x & 31, p = threadIdx.x >> 5;
    float s = 0.0f;
    for (int r = p; r < R; r += 32) s += a[static_cast<size_t>(r) * kMlpOutRows + m];
    part[p][m] = s;
    __syncthreads();
    if (p == 0) {
        float t = 0.0f;
        for (int q = 0; q < 32; ++q) t += part[q][m];
        out[m] = t;
    }
}

// One thread per pair i: dz of rows q_i, p_i, n_i and the pair's loss terms.
__global__ void mlp_dz_kernel(const float* __restrict__ t, int B, int k, const float* __restrict__ colsum,
                              MlpLossWeights lw, float* __restrict__ dz, float* __restrict__ terms) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const float* tq = t + static_cast<size_t>(i) * kMlpOutRows;
    const float* tp = t + static_cast<size_t>(B + i) * kMlpOutRows;
    const float* tn = t + static_cast<size_t>(2 * B + i) * kMlpOutRows;
    float sqp = 0.0f, sqn = 0.0f;
    for (int j = 0; j < k; ++j) {
        sqp += tq[j] * tp[j];
        sqn += tq[j] * tn[j];
    }
    sqp /= k;
    sqn /= k;
    const float rows = 3.0f * B;
    const float cp = -1.0f / (k * static_cast<float>(B));
    const float cn = lw.neg * 2.0f * sqn / (k * static_cast<float>(B));
    float* dq = dz + static_cast<size_t>(i) * kMlpOutRows;
    float* dp = dz + static_cast<size_t>(B + i) * kMlpOutRows;
    float* dn = dz + static_cast<size_t>(2 * B + i) * kMlpOutRows;
    for (int j = 0; j < kMlpOutRows; ++j) {
        if (j < k) {
            const float bal = lw.balance * 2.0f * (colsum[j] / rows) / rows;
            const float gq = cp * tp[j] + cn * tn[j] + bal;
            const float gp = cp * tq[j] + bal;
            const float gn = cn * tq[j] + bal;
            dq[j] = gq * (1.0f - tq[j] * tq[j]);
            dp[j] = gp * (1.0f - tp[j] * tp[j]);
            dn[j] = gn * (1.0f - tn[j] * tn[j]);
        } else {
            dq[j] = dp[j] = dn[j] = 0.0f;
        }
    }
    terms[2 * i] = 1.0f - sqp;
    terms[2 * i + 1] = sqn * sqn;
}

// loss[0..3] = total, positive, negative, balance (one block, fixed order).
__global__ void __launch_bounds__(256) mlp_loss_kernel(const float* __restrict__ terms, int B, int k,
                                                       const float* __restrict__ colsum, MlpLossWeights lw,
                                                       float* __restrict__ loss) {
    __shared__ float sp[256], sn[256];
    float a = 0.0f, b = 0.0f;
    for (int i = threadIdx.x; i < B; i += 256) {
        a += terms[2 * i];
        b += terms[2 * i + 1];
    }
    sp[threadIdx.x] = a;
    sn[threadIdx.x] = b;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sp[threadIdx.x] += sp[threadIdx.x + s];
            sn[threadIdx.x] += sn[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        float bal = 0.0f;
        const float rows = 3.0f * B;
        for (int j = 0; j < k; ++j) bal += (colsum[j] / rows) * (colsum[j] / rows);
        const float pos = sp[0] / B, neg = sn[0] / B;
        loss[0] = pos + lw.neg * neg + lw.balance * bal;
        loss[1] = pos;
        loss[2] = neg;
        loss[3] = bal;
    }
}

// da1[row][j] = (sum_m dz[row][m] W2[m][j]) * (h[row][j] > 0); one block per row.
__global__ void __launch_bounds__(256) mlp_dh_kernel(const float* __restrict__ dz, const float* __restrict__ h,
                                                     const __nv_bfloat16* __restrict__ w2b, int k,
                                                     float* __restrict__ da1) {
    __shared__ float d[kMlpOutRows];
    const size_t row = blockIdx.x;
    if (threadIdx.x < kMlpOutRows) d[threadIdx.x] = dz[row * kMlpOutRows + threadIdx.x];
    __syncthreads();
    const int j = threadIdx.x;
    float s = 0.0f;
    for (int m = 0; m < k; ++m) s = fmaf(d[m], __bfloat162float(w2b[static_cast<size_t>(m) * kMlpHidden + j]), s);
    da1[row * kMlpHidden + j] = h[row * kMlpHidden + j] > 0.0f ? s : 0.0f;
}

// out[a][b] = sum over rows of A[row][a] * Bm[row][b] * bscale (A: float
// [R][wa]; Bm: float or u8 [R][wb]); 32 x 32 output tile per block, rows in
// chunks of 32, fixed order. Also colA[a] = sum over rows of A[row][a] when
// colA is given (from the blocks with blockIdx.y == 0).
template <typename TB>
__global__ void __launch_bounds__(256) wgrad_kernel(const float* __restrict__ A, int wa, const TB* __restrict__ Bm,
                                                    int wb, float bscale, int R, float* __restrict__ out,
                                                    float* __restrict__ colA) {
    __shared__ float as[32][33], bs[32][33];
    const int a0 = blockIdx.x * 32, b0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 row groups of 4 outputs
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    float csum = 0.0f;
    for (int r0 = 0; r0 < R; r0 += 32) {
        for (int e = threadIdx.x; e < 32 * 32; e += 256) {
            const int rr = e >> 5, cc = e & 31;
            const int row = r0 + rr;
            as[rr][cc] = row < R ? A[static_cast<size_t>(row) * wa + a0 + cc] : 0.0f;
            bs[rr][cc] = row < R ? static_cast<float>(Bm[static_cast<size_t>(row) * wb + b0 + cc]) * bscale : 0.0f;
        }
        __syncthreads();
        #pragma unroll 4
        for (int rr = 0; rr < 32; ++rr) {
            const float bv = bs[rr][tx];
            #pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] = fmaf(as[rr][ty * 4 + q], bv, acc[q]);
        }
        if (colA && blockIdx.y == 0 && threadIdx.x < 32)
            for (int rr = 0; rr < 32; ++rr) csum += as[rr][threadIdx.x];
        __syncthreads();
    }
    #pragma unroll
    for (int q = 0; q < 4; ++q) out[static_cast<size_t>(a0 + ty * 4 + q) * wb + b0 + tx] = acc[q];
    if (colA && blockIdx.y == 0 && threadIdx.x < 32) colA[a0 + threadIdx.x] = csum;
}

__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, int n, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

__global__ void mlp_export_kernel(const float* __restrict__ w1, const float* __restrict__ b1,
                                  const float* __restrict__ w2, const float* __restrict__ b2, int k,
                                  __nv_bfloat16* __restrict__ w1b, __nv_bfloat16* __restrict__ w2b,
                                  float* __restrict__ b1o, float* __restrict__ b2o) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kMlpHidden * kMlpIn) w1b[i] = __float2bfloat16_rn(w1[i]);
    if (i < k * kMlpHidden) w2b[i] = __float2bfloat16_rn(w2[i]);
    if (b1o && i < kMlpHidden) b1o[i] = b1[i];
    if (b2o && i < k) b2o[i] = b2[i];
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Thread per 16-byte chunk of the 3B gathered rows.
__global__ void mlp_gather_kernel(const uint8_t* __restrict__ tq, int t_n, const int32_t* __restrict__ nn,
                                  const uint8_t* __restrict__ base, int r_n, int B, unsigned long long seed, int step,
                                  uint8_t* __restrict__ x) {
    const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (e >= 3LL * B * 8) return;
    const int row = static_cast<int>(e >> 3), c = static_cast<int>(e & 7);
    const int i = row % B, part = row / B;
    const unsigned long long h = mix64(seed ^ (static_cast<unsigned long long>(step) << 32) ^
                                       (static_cast<unsigned long long>(i) * 0x632BE59BD9B4E019ull));
    const int qi = static_cast<int>(h % static_cast<unsigned long long>(t_n));
    const uint8_t* src;
    if (part == 0) {
        src = tq + static_cast<size_t>(qi) * kMlpIn;
    } else if (part == 1) {
        src = base + static_cast<size_t>(nn[2 * qi]) * kMlpIn;
    } else {
        const int ri = static_cast<int>(mix64(h) % static_cast<unsigned long long>(r_n));
        src = base + static_cast<size_t>(ri) * kMlpIn;
    }
    reinterpret_cast<uint4*>(x + static_cast<size_t>(row) * kMlpIn)[c] = reinterpret_cast<const uint4*>(src)[c];
}

}  // namespace

MlpParams mlp_params_at(float* base) {
    MlpParams p;
    p.w1 = base;
    p.b1 = p.w1 + kMlpHidden * kMlpIn;
    p.w2 = p.b1 + kMlpHidden;
    p.b2 = p.w2 + kMlpOutRows * kMlpHidden;
    return p;
}

cudaError_t launch_mlp_loss_grad(const uint8_t* x, int B, int k, const MlpParams& p, const __nv_bfloat16* w1b,
                                 const __nv_bfloat16* w2b, const MlpLossWeights& lw, MlpTrainBufs& tb,
                                 const MlpParams& g, cudaStream_t stream) {
    if (B <= 0 || k < 1 || k > kMlpMaxBits) return cudaErrorInvalidValue;
    const int R = 3 * B;
    cudaError_t e = cudaFuncSetAttribute(mlp_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kFwdSmem));
    if (e != cudaSuccess) return e;
    mlp_fwd_kernel<<<(R + kFwdRows - 1) / kFwdRows, 256, kFwdSmem, stream>>>(x, R, w1b, p.b1, w2b, p.b2, k, tb.h,
                                                                             tb.t);
    colsum32_kernel<<<1, 1024, 0, stream>>>(tb.t, R, tb.colsum);
    // per-pair loss terms use the first 2B floats of da1 (written later)
    float* terms = tb.da1;
    mlp_dz_kernel<<<(B + 127) / 128, 128, 0, stream>>>(tb.t, B, k, tb.colsum, lw, tb.dz, terms);
    mlp_loss_kernel<<<1, 256, 0, stream>>>(terms, B, k, tb.colsum, lw, tb.loss);
    mlp_dh_kernel<<<R, 256, 0, stream>>>(tb.dz, tb.h, w2b, k, tb.da1);
    // dW2 = dz^T h, db2 = colsum(dz); dW1 = da1^T (x / 64), db1 = colsum(da1)
    wgrad_kernel<float><<<dim3(kMlpOutRows / 32, kMlpHidden / 32), 256, 0, stream>>>(
        tb.dz, kMlpOutRows, tb.h, kMlpHidden, 1.0f, R, g.w2, g.b2);
    wgrad_kernel<uint8_t><<<dim3(kMlpHidden / 32, kMlpIn / 32), 256, 0, stream>>>(
        tb.da1, kMlpHidden, x, kMlpIn, kMlpInScale, R, g.w1, g.b1);
    return cudaGetLastError();
}

cudaError_t launch_mlp_adam(const MlpParams& p, const MlpParams& g, const MlpParams& m, const MlpParams& v, int k,
                            int step, float lr, __nv_bfloat16* w1b, __nv_bfloat16* w2b, cudaStream_t stream) {
    const int n = static_cast<int>(kMlpParamCount);
    const float c1 = 1.0f - powf(0.9f, static_cast<float>(step));
    const float c2 = 1.0f - powf(0.999f, static_cast<float>(step));
    mlp_adam_kernel<<<(n + 255) / 256, 256, 0, stream>>>(p.w1, g.w1, m.w1, v.w1, n, lr, c1, c2);
    mlp_export_kernel<<<(kMlpHidden * kMlpIn + 255) / 256, 256, 0, stream>>>(p.w1, p.b1, p.w2, p.b2, k, w1b, w2b,
                                                                          nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_mlp_export(const MlpParams& p, int k, __nv_bfloat16* w1b, __nv_bfloat16* w2b, float* b1_out,
                              float* b2_out, cudaStream_t stream) {
    mlp_export_kernel<<<(kMlpHidden * kMlpIn + 255) / 256, 256, 0, stream>>>(p.w1, p.b1, p.w2, p.b2, k, w1b, w2b,
                                                                          b1_out, b2_out);
    return cudaGetLastError();
}

cudaError_t launch_mlp_gather(const uint8_t* tq, int t_n, const int32_t* nn, const uint8_t* base, int r_n, int B,
                              unsigned long long seed, int step, uint8_t* x, cudaStream_t stream) {
    const long long items = 3LL * B * 8;
    mlp_gather_kernel<<<static_cast<unsigned>((items + 255) / 256), 256, 0, stream>>>(tq, t_n, nn, base, r_n, B, seed,
                                                                                    step, x);
    return cudaGetLastError();
}

}  // namespace sift
