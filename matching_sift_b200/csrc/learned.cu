// Learned-hash inference on sm_100a: both MLP layers on the tensor cores
// (tcgen05 kind::f16, BF16 operands, FP32 accumulators in TMEM), fused with
// the conversion of the u8 descriptors to BF16 and the packing of the output
// signs into bucket codes; plus query-directed probe generation.
//
// Per CTA (persistent over 128-row tiles), shared memory holds W1 (256 x 128)
// and W2 (32 x 256, rows >= k zero) for the whole launch, one BF16 input tile
// (128 x 128) and one BF16 hidden tile (128 x 256), all K-major with the
// 128-byte swizzle (the layout TMA writes for the weights; the epilogue warps
// write the activations in the same layout themselves).
//
// Warps: 0 = weight and input-tile TMA, TMEM allocation, MMA issue (one
//            thread); the u8 input tiles stream through a 2-stage ring,
//            loaded two tiles ahead;
//        1..8 = conversion and epilogue, two warps per TMEM lane quarter:
//            thread = tile row (TMEM lane), warp half h converts K block h of
//            the input row and applies layer 1's epilogue to hidden columns
//            [128 h, 128 h + 128); half 0 also forms the codes.
// Per tile i (epilogue threads):
//   convert x(i) -> x_s      [x_ready]     MMA1: TMEM[0,256) = x W1^T
//   epi1: h = bf16(relu(acc / 64 + b1)) -> h_s   [h_ready]   MMA2: TMEM[256,288) = h W2^T
//   convert x(i+1) (x_s is free once MMA1(i) completed) while MMA2(i) runs
//   epi2: z = acc + b2 -> code bits (and z)
// Every wait is bounded (2 s) and reports through `err`.
#include <climits>
#include <cuda_bf16.h>
#include "exact2nn.cuh"
#include "learned.cuh"
#include "ptx.cuh"

namespace sift {
namespace {

constexpr int kLEpiWarps = 8;  // two per TMEM lane quarter
constexpr int kLThreads = 32 * (1 + kLEpiWarps);
constexpr int kXKBlock = 128 * 128;                     // bytes of one K block of a 128-row BF16 tile
constexpr int kW1Bytes = kMlpHidden * kMlpIn * 2;       // 64 KB
constexpr int kW2Bytes = kMlpOutRows * kMlpHidden * 2;  // 16 KB
constexpr int kXBytes = 128 * kMlpIn * 2;               // 32 KB
constexpr int kHBytes = 128 * kMlpHidden * 2;           // 64 KB
constexpr uint32_t kLTmemCols = 512;
constexpr int kXStages = 2;                             // u8 input tile ring
constexpr int kXTileBytes = 128 * kMlpIn;               // 16 KB

struct __align__(8) MlpCtl {
    uint64_t w_full, x_ready, h_ready, m1, m2, drain;
    uint64_t xfull[kXStages];
    uint32_t tmem_base;
    int abort_flag, no_abort;
    float b1[kMlpHidden];
    float b2[kMlpOutRows];
};

constexpr size_t kLSmemBytes = 1024 + kW1Bytes + kW2Bytes + kXBytes + kHBytes + kXStages * kXTileBytes + sizeof(MlpCtl);
static_assert(kLSmemBytes <= 227 * 1024, "MLP hash shared memory");

// Byte offset of the 16-byte chunk `ch` (0..7) of row r in a K block of a
// SW128 K-major tile (rows of 128 bytes, 8-row atoms).
__device__ __forceinline__ uint32_t sw128_off(int r, int ch) {
    return static_cast<uint32_t>(r * 128 + ((ch ^ (r & 7)) << 4));
}

__device__ __forceinline__ uint32_t bf16x2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Half h of row r of a u8 tile in shared memory (TMA, 128-byte swizzle; rows
// past the end of the input are zeros) -> BF16 K block h of x_s.
__device__ __forceinline__ void convert_row(const uint8_t* u8_tile, int r, uint8_t* x_s, int h) {
    #pragma unroll
    for (int c = 4 * h; c < 4 * h + 4; ++c) {
        const uint4 v = *reinterpret_cast<const uint4*>(u8_tile + sw128_off(r, c));
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
        uint32_t o[8];
        #pragma unroll
        for (int q = 0; q < 4; ++q) {
            o[2 * q] = bf16x2(static_cast<float>(w[q] & 0xff), static_cast<float>((w[q] >> 8) & 0xff));
            o[2 * q + 1] = bf16x2(static_cast<float>((w[q] >> 16) & 0xff), static_cast<float>(w[q] >> 24));
        }
        // elements 16c .. 16c + 15: K block c / 4, chunks 2 (c % 4) and 2 (c % 4) + 1
        uint8_t* blk = x_s + (c >> 2) * kXKBlock;
        const int ch = 2 * (c & 3);
        *reinterpret_cast<uint4*>(blk + sw128_off(r, ch)) = make_uint4(o[0], o[1], o[2], o[3]);
        *reinterpret_cast<uint4*>(blk + sw128_off(r, ch + 1)) = make_uint4(o[4], o[5], o[6], o[7]);
    }
}

__global__ void __launch_bounds__(kLThreads, 1)
    mlp_hash_kernel(const __grid_constant__ CUtensorMap xmap, int n, const __grid_constant__ CUtensorMap w1map,
                    const __grid_constant__ CUtensorMap w2map, const float* __restrict__ b1,
                    const float* __restrict__ b2, int k, uint32_t* __restrict__ codes, float* __restrict__ zout,
                    int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = ptx::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
    uint8_t* w1_s = smem;
    uint8_t* w2_s = w1_s + kW1Bytes;
    uint8_t* x_s = w2_s + kW2Bytes;
    uint8_t* h_s = x_s + kXBytes;
    uint8_t* xr_s = h_s + kHBytes;  // u8 tile ring
    MlpCtl* ctl = reinterpret_cast<MlpCtl*>(xr_s + kXStages * kXTileBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles = (n + 127) / 128;
    const int bx = static_cast<int>(blockIdx.x), gx = static_cast<int>(gridDim.x);
    const int my_tiles = bx < tiles ? (tiles - 1 - bx) / gx + 1 : 0;

    const uint32_t bar_w = ptx::smem_u32(&ctl->w_full), bar_x = ptx::smem_u32(&ctl->x_ready);
    const uint32_t bar_h = ptx::smem_u32(&ctl->h_ready), bar_m1 = ptx::smem_u32(&ctl->m1);
    const uint32_t bar_m2 = ptx::smem_u32(&ctl->m2), bar_drain = ptx::smem_u32(&ctl->drain);
    if (threadIdx.x == 0) {
        ptx::mbar_init(bar_w, 1);
        ptx::mbar_init(bar_x, 32 * kLEpiWarps);
        ptx::mbar_init(bar_h, 32 * kLEpiWarps);
        ptx::mbar_init(bar_m1, 1);
        ptx::mbar_init(bar_m2, 1);
        ptx::mbar_init(bar_drain, 1);
        for (int s = 0; s < kXStages; ++s) ptx::mbar_init(ptx::smem_u32(&ctl->xfull[s]), 1);
        ctl->abort_flag = 0;
        ctl->no_abort = 0;
        ptx::fence_mbar_init();
    }
    for (int j = threadIdx.x; j < kMlpHidden; j += kLThreads) ctl->b1[j] = b1[j];
    for (int j = threadIdx.x; j < kMlpOutRows; j += kLThreads) ctl->b2[j] = j < k ? b2[j] : 0.0f;
    if (warp == 0) {
        ptx::tmem_alloc(ptx::smem_u32(&ctl->tmem_base), kLTmemCols);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;
    volatile int* abort_flag = &ctl->abort_flag;
    volatile int* never = &ctl->no_abort;
    const uint32_t w1_a = ptx::smem_u32(w1_s), w2_a = ptx::smem_u32(w2_s);
    const uint32_t x_a = ptx::smem_u32(x_s), h_a = ptx::smem_u32(h_s);
    const uint32_t xr_a = ptx::smem_u32(xr_s), bar_xf = ptx::smem_u32(&ctl->xfull[0]);

    if (warp == 0) {
        if (lane == 0 && my_tiles > 0) {
            ptx::tma_prefetch_desc(&w1map);
            ptx::tma_prefetch_desc(&w2map);
            ptx::tma_prefetch_desc(&xmap);
            int issued = 0;  // input tiles whose TMA load has been issued
            for (; issued < kXStages && issued < my_tiles; ++issued) {
                ptx::mbar_arrive_expect_tx(bar_xf + 8 * issued, kXTileBytes);
                ptx::tma_load_2d(xr_a + issued * kXTileBytes, &xmap, 0, (bx + issued * gx) * 128, bar_xf + 8 * issued);
            }
            ptx::mbar_arrive_expect_tx(bar_w, kW1Bytes + kW2Bytes);
            for (int kb = 0; kb < 2; ++kb) ptx::tma_load_2d(w1_a + kb * (kMlpHidden * 128), &w1map, kb * 64, 0, bar_w);
            for (int kb = 0; kb < 4; ++kb) ptx::tma_load_2d(w2_a + kb * (kMlpOutRows * 128), &w2map, kb * 64, 0, bar_w);
            // layer 1: M = 128, N = 256, K = 16 per MMA; layer 2: M = 128, N = 32
            constexpr uint32_t idesc1 = ptx::idesc_make(1 /*F32*/, 1 /*BF16*/, 1 /*BF16*/, 128, kMlpHidden);
            constexpr uint32_t idesc2 = ptx::idesc_make(1 /*F32*/, 1 /*BF16*/, 1 /*BF16*/, 128, kMlpOutRows);
            const bool ok = ptx::mbar_wait(bar_w, 0, abort_flag, err, kErrWaitMmaFull);
            for (int i = 0; i < my_tiles && ok; ++i) {
                if (!ptx::mbar_wait(bar_x, i & 1, abort_flag, err, kErrWaitMmaFull)) break;
                ptx::tc_fence_after();
                #pragma unroll
                for (int kb = 0; kb < 2; ++kb) {
                    #pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                        ptx::mma_f16(tmem, ptx::sdesc_sw128(x_a + kb * kXKBlock + kk * 32),
                                     ptx::sdesc_sw128(w1_a + kb * (kMlpHidden * 128) + kk * 32), idesc1,
                                     (kb | kk) ? 1u : 0u);
                }
                ptx::tc_commit(bar_m1);
                // Tile i's u8 stage was converted (x_ready): reuse it for tile i + 2.
                if (issued < my_tiles) {
                    const int st = issued % kXStages;
                    ptx::mbar_arrive_expect_tx(bar_xf + 8 * st, kXTileBytes);
                    ptx::tma_load_2d(xr_a + st * kXTileBytes, &xmap, 0, (bx + issued * gx) * 128, bar_xf + 8 * st);
                    ++issued;
                }
                if (!ptx::mbar_wait(bar_h, i & 1, abort_flag, err, kErrWaitMmaTmem)) break;
                ptx::tc_fence_after();
                #pragma unroll
                for (int kb = 0; kb < 4; ++kb) {
                    #pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                        ptx::mma_f16(tmem + kMlpHidden, ptx::sdesc_sw128(h_a + kb * kXKBlock + kk * 32),
                                     ptx::sdesc_sw128(w2_a + kb * (kMlpOutRows * 128) + kk * 32), idesc2,
                                     (kb | kk) ? 1u : 0u);
                }
                ptx::tc_commit(bar_m2);
            }
            if (!ok) ptx::mbar_wait(bar_w, 0, never, err, kErrWaitDrain);  // weights landed before exit
            // Input tiles in flight land before exit (the last kXStages issued).
            for (int t = (issued > kXStages ? issued - kXStages : 0); t < issued; ++t)
                ptx::mbar_wait(bar_xf + 8 * (t % kXStages), (t / kXStages) & 1, never, err, kErrWaitDrain);
            ptx::tc_commit(bar_drain);
            ptx::mbar_wait(bar_drain, 0, never, err, kErrWaitDrain);
        }
        __syncwarp();
    } else {
        const int quarter = warp & 3;
        const int half = (warp - 1) >> 2;   // which K block / hidden half this warp handles
        const int r = quarter * 32 + lane;  // tile row = TMEM lane
        const uint32_t lane_base = static_cast<uint32_t>(quarter * 32) << 16;
        bool conv_ok = true;
        if (my_tiles > 0) {
            conv_ok = ptx::mbar_wait(bar_xf, 0, abort_flag, err, kErrWaitEpilogue);
            if (conv_ok) convert_row(xr_s, r, x_s, half);
            ptx::fence_proxy_async();
            ptx::mbar_arrive(bar_x);
        }
        for (int i = 0; i < my_tiles && __all_sync(0xffffffffu, conv_ok); ++i) {
            const int g0 = (bx + i * gx) * 128;
            bool waited = ptx::mbar_wait(bar_m1, i & 1, abort_flag, err, kErrWaitEpilogue);
            if (!__all_sync(0xffffffffu, waited)) break;
            ptx::tc_fence_after();
            #pragma unroll 1
            for (int m = 4 * half; m < 4 * half + 4; ++m) {
                uint32_t v[32];
                ptx::tmem_ld32(tmem + lane_base + m * 32, v);
                ptx::tmem_ld_wait(v);
                uint8_t* blk = h_s + (m >> 1) * kXKBlock;
                #pragma unroll
                for (int c8 = 0; c8 < 4; ++c8) {
                    uint32_t o[4];
                    #pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int j = m * 32 + c8 * 8 + 2 * e;
                        const float a = fmaxf(fmaf(__uint_as_float(v[c8 * 8 + 2 * e]), kMlpInScale, ctl->b1[j]), 0.0f);
                        const float b =
                            fmaxf(fmaf(__uint_as_float(v[c8 * 8 + 2 * e + 1]), kMlpInScale, ctl->b1[j + 1]), 0.0f);
                        o[e] = bf16x2(a, b);
                    }
                    *reinterpret_cast<uint4*>(blk + sw128_off(r, 4 * (m & 1) + c8)) = make_uint4(o[0], o[1], o[2], o[3]);
                }
            }
            ptx::tc_fence_before();
            ptx::fence_proxy_async();
            ptx::mbar_arrive(bar_h);
            if (i + 1 < my_tiles) {
                const int st = (i + 1) % kXStages;
                conv_ok = ptx::mbar_wait(bar_xf + 8 * st, ((i + 1) / kXStages) & 1, abort_flag, err, kErrWaitEpilogue);
                if (conv_ok) convert_row(xr_s + st * kXTileBytes, r, x_s, half);
                ptx::fence_proxy_async();
                ptx::mbar_arrive(bar_x);
            }
            if (half) continue;  // layer 2's 32 columns: half 0
            waited = ptx::mbar_wait(bar_m2, i & 1, abort_flag, err, kErrWaitEpilogue);
            if (!__all_sync(0xffffffffu, waited)) break;
            ptx::tc_fence_after();
            uint32_t v[32];
            ptx::tmem_ld32(tmem + lane_base + kMlpHidden, v);
            ptx::tmem_ld_wait(v);
            ptx::tc_fence_before();
            const int g = g0 + r;
            if (g < n) {
                uint32_t code = 0;
                #pragma unroll
                for (int j = 0; j < kMlpMaxBits; ++j) {
                    if (j < k) {
                        const float z = __uint_as_float(v[j]) + ctl->b2[j];
                        code |= (z > 0.0f ? 1u : 0u) << j;
                        if (zout) zout[static_cast<size_t>(g) * k + j] = z;
                    }
                }
                codes[g] = code;
            }
        }
    }
    ptx::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc(tmem, kLTmemCols);
    }
}

// One thread per query: the `flip` smallest-|z| bits, all their subsets
// ordered by summed |z| (ties by subset mask), the first n_probes applied.
__global__ void probe_codes_kernel(const uint32_t* __restrict__ codes, const float* __restrict__ z, int n, int k,
                                   int flip, int n_probes, uint32_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int bit[6];
    float mag[6];
    int m = 0;
    for (int j = 0; j < k; ++j) {
        const float a = fabsf(z[static_cast<size_t>(i) * k + j]);
        int p;  // kept bits sorted by |z|, ties by bit index (earlier bits stay first)
        if (m < flip) p = m++;
        else if (flip > 0 && a < mag[flip - 1]) p = flip - 1;
        else continue;
        while (p > 0 && mag[p - 1] > a) {
            mag[p] = mag[p - 1];
            bit[p] = bit[p - 1];
            --p;
        }
        mag[p] = a;
        bit[p] = j;
    }
    const uint32_t code = codes[i];
    // Selection of the n_probes lightest subsets of the m kept bits.
    const int subsets = 1 << m;
    uint32_t taken[2] = {0u, 0u};  // bitmap over subset ids (m <= 6: 64 subsets)
    for (int p = 0; p < n_probes; ++p) {
        int best = -1;
        float bs = 0.0f;
        for (int s = 0; s < subsets; ++s) {
            if ((taken[s >> 5] >> (s & 31)) & 1u) continue;
            float sc = 0.0f;
            for (int b = 0; b < m; ++b)
                if ((s >> b) & 1) sc += mag[b];
            if (best < 0 || sc < bs) { best = s; bs = sc; }
        }
        uint32_t c = code;
        if (best >= 0) {
            taken[best >> 5] |= 1u << (best & 31);
            for (int b = 0; b < m; ++b)
                if ((best >> b) & 1) c ^= 1u << bit[b];
        }
        out[static_cast<size_t>(p) * n + i] = c;  // past the subsets: repeats the code (skipped by the scan)
    }
}

}  // namespace

size_t mlp_hash_smem_bytes() { return kLSmemBytes; }

cudaError_t launch_mlp_hash(const CUtensorMap& xmap, int n, const CUtensorMap& w1map, const CUtensorMap& w2map,
                            const float* b1, const float* b2, int k, uint32_t* codes, float* z, int* err,
                            int num_sms, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(mlp_hash_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kLSmemBytes));
    if (e != cudaSuccess) return e;
    const int tiles = (n + 127) / 128;
    const int grid = tiles < num_sms ? tiles : num_sms;
    mlp_hash_kernel<<<grid, kLThreads, kLSmemBytes, stream>>>(xmap, n, w1map, w2map, b1, b2, k, codes, z, err);
    return cudaGetLastError();
}

cudaError_t launch_probe_codes(const uint32_t* codes, const float* z, int n, int k, int flip, int n_probes,
                               uint32_t* probe_codes, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    if (flip < 0 || flip > 6 || n_probes < 1 || n_probes > 64 || flip > k) return cudaErrorInvalidValue;
    probe_codes_kernel<<<(n + 127) / 128, 128, 0, stream>>>(codes, z, n, k, flip, n_probes, probe_codes);
    return cudaGetLastError();
}

}  // namespace sift
