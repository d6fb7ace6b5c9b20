// Exact 2-NN of u8 SIFT descriptors on sm_100a: one persistent, warp-
// specialised kernel computes q.b on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, u8 x u8 -> s32, accumulators in TMEM, operands
// staged by TMA) and reduces every accumulator tile to a per-query top-2 in
// the epilogue, so the queries x base distance matrix never reaches HBM.
//
// Replaces the reference's GEMM + scan pairs:
//   cublasHgemm / cublasGemmEx   src/knn_brute.cu:244, :592   (dist = -2 q.r to HBM)
//   find_matches / min_dist_f    src/knn_brute.cu:340-448, :726-796 (scan of dist)
//   sqrEuclidianDist             src/knn_brute.cu:671-691     (full squared L2)
//
// Ranking key. For query q and base row b the kernel ranks by
//     key(b) = norm(b) - 2 q.b        (norm(b) = |b|^2 for kMetricL2, 0 for kMetricDot)
// which orders candidates exactly like |q - b|^2 = |q|^2 + key (resp. -2 q.b).
// All values are exact integers: |key| <= 2 * 128 * 255^2 < 2^25.
// Ties are broken by the lower base index (lexicographic (key, index) order),
// which is the order of the reference's host_brute (src/knn_brute.cu:816-831).
//
// Work decomposition. A CTA holds kQT = 4 query tiles (512 queries) in shared
// memory and streams base tiles of kBN = 128 rows; a unit = (query group,
// base tile). Units are split evenly over a persistent grid of one CTA per SM.
//
// Warp roles (kThreads = 576):
//   warp 0       TMA producer: the query tiles of the current group and a
//                kStages ring of base tiles
//   warp 1       TMEM allocator + single-thread MMA issuer: per base tile one
//                128 x 128 x 128 product per query tile into that tile's
//                TMEM slot (4 slots x 128 columns)
//   warps 2..17  epilogue: warp w owns query tile (w - 2) / 4 and TMEM lane
//                quarter w % 4, i.e. 32 query rows, one thread per row
//
// Epilogue pruning. Per 8-row subgroup of base rows a thread takes the largest
// dot product m of its query row; with n_min the smallest norm of the subgroup
// (precomputed), n_min - 2 m is a lower bound of every key in it. A group of
// 32 rows (four subgroups, one vote) whose four bounds all exceed the thread's
// threshold is skipped (~0.8 instruction per element); otherwise only the
// passing subgroups form exact keys. The threshold is the thread's own
// second-best key and an upper bound of the final second-best key that the
// CTAs splitting the same query group share through global memory (atomicMin).
#include <cfloat>
#include <climits>
#include <algorithm>
#include <cuda_fp16.h>
#include "exact2nn.cuh"
#include "ptx.cuh"
#include "epilogue.cuh"

namespace sift {

namespace {

constexpr int kQTileBytes = kBM * kDim;           // 16 KB: one query tile (u8)
constexpr int kBTileBytes = kBN * kDim;           // 16 KB: one base tile (u8)
constexpr int kRecBytes = kRecInts * 4;           // 640 B: norms record of one base tile

struct __align__(8) SmemCtl {
    uint64_t full[kStages];    // base tile + norms record landed (TMA)
    uint64_t empty[kStages];   // MMAs reading the base tile done (tcgen05.commit)
    uint64_t nempty[kStages];  // all epilogue warps done with the norms record
    uint64_t qfull, qempty;
    uint64_t tfull[kQT], tempty[kQT];
    uint64_t drain;
    uint32_t tmem_base;
    int abort_flag;
    int no_abort;
};

constexpr size_t kSmemBytes =
    1024 + kQT * kQTileBytes + kStages * kBTileBytes + kStages * kRecBytes + sizeof(SmemCtl);

// 16 consecutive elements of a row as u8 (FP16: value * mul, exact by contract).
__device__ __forceinline__ uint4 load16_u8(const uint8_t* x, int row, int sub, float) {
    return reinterpret_cast<const uint4*>(x + static_cast<size_t>(row) * kDim)[sub];
}
__device__ __forceinline__ uint4 load16_u8(const __half* x, int row, int sub, float mul) {
    const uint4* p = reinterpret_cast<const uint4*>(x + static_cast<size_t>(row) * kDim) + 2 * sub;
    uint32_t w[4];
    #pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint4 v = p[h];
        const __half2* hv = reinterpret_cast<const __half2*>(&v);
        #pragma unroll
        for (int k = 0; k < 2; ++k) {
            const float2 a = __half22float2(hv[2 * k]), b = __half22float2(hv[2 * k + 1]);
            w[2 * h + k] = static_cast<uint32_t>(__float2int_rn(a.x * mul)) |
                           (static_cast<uint32_t>(__float2int_rn(a.y * mul)) << 8) |
                           (static_cast<uint32_t>(__float2int_rn(b.x * mul)) << 16) |
                           (static_cast<uint32_t>(__float2int_rn(b.y * mul)) << 24);
        }
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

template <typename T>
__global__ void __launch_bounds__(256) row_norms_kernel(const T* __restrict__ x, int n, int n_pad, float mul,
                                                        int metric, int32_t* __restrict__ norm,
                                                        int32_t* __restrict__ rec,
                                                        int32_t* __restrict__ thresh) {
    // 32 rows per block, 8 threads per row, 16 elements per thread.
    const int row = blockIdx.x * 32 + (threadIdx.x >> 3);
    const int sub = threadIdx.x & 7;
    uint32_t s = 0;
    if (row < n) {
        const uint4 w = load16_u8(x, row, sub, mul);
        s = __dp4a(w.x, w.x, 0u);
        s = __dp4a(w.y, w.y, s);
        s = __dp4a(w.z, w.z, s);
        s = __dp4a(w.w, w.w, s);
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    const int32_t v = row < n ? (metric == kMetricL2 ? static_cast<int32_t>(s) : 0) : kKeyPad;
    __shared__ int32_t nrm[32];
    // Record of base tile (row / kBN): [0, 128) norms, [128, 144) 8-row minima.
    int32_t* r = rec ? rec + static_cast<size_t>(blockIdx.x / 4) * kRecInts : nullptr;
    const int part = blockIdx.x & 3;  // which 32-row quarter of the tile
    if (sub == 0) {
        nrm[threadIdx.x >> 3] = v;
        if (norm) norm[row] = v;
        if (r) r[part * 32 + (threadIdx.x >> 3)] = v;
        if (thresh) thresh[row] = INT_MAX;
    }
    __syncthreads();
    if (threadIdx.x < 4 && r) {
        int m = nrm[8 * threadIdx.x];
        #pragma unroll
        for (int i = 1; i < 8; ++i) m = min(m, nrm[8 * threadIdx.x + i]);
        r[128 + part * 4 + threadIdx.x] = m;
    }
}

// Norm folding (the fold variant of the u8 pair kernel). A fifth MMA per tile
// product multiplies a constant query-side row a[32] (u8) with 32 signed
// digits d[32] per base row (s8) so that the accumulator holds
// q.b - c with c = min(ceil(|b|^2 / 2), kFoldMax) and a.d = -c:
//   a = {1, 16, 255 x 30}, c = 255 h + l (0 <= l < 255),
//   d[0] = -(l & 15), d[1] = -(l >> 4), d[2..31] = -h in parts of at most 128.
// The key |b|^2 - 2 q.b = r - 2 acc with the residual r = |b|^2 - 2 c >= -1,
// so every key of a row set is at least -1 - 2 max(acc): one max tree per
// row set bounds its keys exactly up to that 1 (rows whose c was clamped
// only make the bound looser). Records hold the residuals.
//
// fold[] layout: per base tile, per half of 64 rows, 2048 bytes in the
// tensor cores' no-swizzle K-major layout (8-row groups of 256 bytes, two
// 16-byte K chunks of 128 bytes each, 16 bytes per row), so one 2-D TMA box
// of 8 x 256 bytes lands a half tile ready as an MMA operand.
//
// One block per base tile: 8 threads per row, the 4 rows of a thread's
// 32-row parts loaded up front (64 bytes in flight per thread), then per row
// the norm, the folded half-norm c, its digits and the residual.
__global__ void __launch_bounds__(256) fold_records_kernel(const uint8_t* __restrict__ x, int n, int n_pad,
                                                           int metric, int32_t* __restrict__ rec,
                                                           uint32_t* __restrict__ fold) {
    const int t = blockIdx.x;
    const int sub = threadIdx.x & 7;
    const int lrow = threadIdx.x >> 3;
    uint4 w[4];
    #pragma unroll
    for (int part = 0; part < 4; ++part) {
        const int row = t * kBN + part * 32 + lrow;
        w[part] = row < n ? load16_u8(x, row, sub, 1.0f) : make_uint4(0u, 0u, 0u, 0u);
    }
    __shared__ int32_t res[kBN];
    int32_t* r = rec + static_cast<size_t>(t) * kRecInts;
    #pragma unroll
    for (int part = 0; part < 4; ++part) {
        const int wr = part * 32 + lrow;  // row within the tile
        const bool live = t * kBN + wr < n;
        uint32_t s = __dp4a(w[part].x, w[part].x, 0u);
        s = __dp4a(w[part].y, w[part].y, s);
        s = __dp4a(w[part].z, w[part].z, s);
        s = __dp4a(w[part].w, w[part].w, s);
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        s += __shfl_xor_sync(0xffffffffu, s, 4);
        const int32_t norm = live ? (metric == kMetricL2 ? static_cast<int32_t>(s) : 0) : kKeyPad;
        const int32_t c = live ? min((norm + 1) >> 1, kFoldMax) : 0;
        const int32_t resid = norm - 2 * c;
        // This thread's 4 digits k = 4 sub .. 4 sub + 3.
        const int l = c % 255, h = c / 255;
        uint32_t word = 0;
        #pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int k = 4 * sub + b;
            const int d = k == 0 ? -(l & 15) : (k == 1 ? -(l >> 4) : -min(128, max(0, h - 128 * (k - 2))));
            word |= (static_cast<uint32_t>(d) & 0xFFu) << (8 * b);
        }
        const size_t off = (static_cast<size_t>(t) * 2 + (wr >> 6)) * kFoldHalfBytes + ((wr & 63) >> 3) * 256 +
                           (sub >> 2) * 128 + (wr & 7) * 16 + 4 * (sub & 3);
        fold[off / 4] = word;
        if (sub == 0) {
            res[wr] = resid;
            r[wr] = resid;
        }
    }
    __syncthreads();
    if (threadIdx.x < 16) {
        int m = res[8 * threadIdx.x];
        #pragma unroll
        for (int i = 1; i < 8; ++i) m = min(m, res[8 * threadIdx.x + i]);
        r[128 + threadIdx.x] = m;
    } else if (threadIdx.x < 24) {
        const int hh = threadIdx.x - 16;
        int m = res[16 * hh];
        #pragma unroll
        for (int i = 1; i < 16; ++i) m = min(m, res[16 * hh + i]);
        r[144 + hh] = m;
    }
}

// 16 consecutive elements of a row, times mul, as floats.
__device__ __forceinline__ void load16_f32(const float* x, int row, int sub, float mul, float (&f)[16]) {
    const float4* p = reinterpret_cast<const float4*>(x + static_cast<size_t>(row) * kDim) + 4 * sub;
    #pragma unroll
    for (int h = 0; h < 4; ++h) {
        const float4 v = p[h];
        f[4 * h] = v.x * mul;
        f[4 * h + 1] = v.y * mul;
        f[4 * h + 2] = v.z * mul;
        f[4 * h + 3] = v.w * mul;
    }
}
__device__ __forceinline__ void load16_f32(const __half* x, int row, int sub, float mul, float (&f)[16]) {
    const uint4* p = reinterpret_cast<const uint4*>(x + static_cast<size_t>(row) * kDim) + 2 * sub;
    #pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint4 v = p[h];
        const __half2* hv = reinterpret_cast<const __half2*>(&v);
        #pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 a = __half22float2(hv[k]);
            f[8 * h + 2 * k] = a.x * mul;
            f[8 * h + 2 * k + 1] = a.y * mul;
        }
    }
}

// Squared norms of general (non-integer) float / half rows times mul, in FP32,
// stored as float bit patterns in the int32 slots of the integer path (norm,
// record norms and 8-row minima); padding rows get kFloatKeyPad. thresh is set
// to INT_MAX (the largest ordered key, see float_key).
template <typename T>
__global__ void __launch_bounds__(256) row_norms_float_kernel(const T* __restrict__ x, int n, int n_pad, float mul,
                                                              int metric, int32_t* __restrict__ norm,
                                                              int32_t* __restrict__ rec,
                                                              int32_t* __restrict__ thresh) {
    const int row = blockIdx.x * 32 + (threadIdx.x >> 3);
    const int sub = threadIdx.x & 7;
    float s = 0.0f;
    if (row < n) {
        float f[16];
        load16_f32(x, row, sub, mul, f);
        #pragma unroll
        for (int i = 0; i < 16; ++i) s = fmaf(f[i], f[i], s);
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    const float v = row < n ? (metric == kMetricL2 ? s : 0.0f) : kFloatKeyPad;
    __shared__ float nrm[32];
    int32_t* r = rec ? rec + static_cast<size_t>(blockIdx.x / 4) * kRecInts : nullptr;
    const int part = blockIdx.x & 3;
    if (sub == 0) {
        nrm[threadIdx.x >> 3] = v;
        if (norm) norm[row] = __float_as_int(v);
        if (r) r[part * 32 + (threadIdx.x >> 3)] = __float_as_int(v);
        if (thresh) thresh[row] = INT_MAX;
    }
    __syncthreads();
    if (threadIdx.x < 4 && r) {
        float m = nrm[8 * threadIdx.x];
        #pragma unroll
        for (int i = 1; i < 8; ++i) m = fminf(m, nrm[8 * threadIdx.x + i]);
        r[128 + part * 4 + threadIdx.x] = __float_as_int(m);
    }
}

// Largest k with key(items[k]) <= v over a non-decreasing key; empty
// problems share the key of the problem after them, so the match is the
// problem that owns v.
template <typename F>
__device__ __forceinline__ int find_item(int n_items, long long v, F key) {
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (key(mid) <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Base-tile records of a batch: block b fills quarter b % 4 of record b / 4;
// the record belongs to the problem whose record range holds it, and rows of
// its base set past n_b are padding (norm kKeyPad).
__global__ void __launch_bounds__(256) batch_records_kernel(const uint8_t* __restrict__ x,
                                                            const WorkItem* __restrict__ items, int n_items,
                                                            int metric, int32_t* __restrict__ rec) {
    const int T = blockIdx.x >> 2, part = blockIdx.x & 3;
    const int p = find_item(n_items, T, [&](int k) { return static_cast<long long>(items[k].rec_off); });
    const WorkItem it = items[p];
    const int local = (T - it.rec_off) * kBN + part * 32 + (threadIdx.x >> 3);
    const int sub = threadIdx.x & 7;
    uint32_t s = 0;
    if (local < it.n_b) {
        const uint4 w = reinterpret_cast<const uint4*>(x + static_cast<size_t>(it.b_off + local) * kDim)[sub];
        s = __dp4a(w.x, w.x, 0u);
        s = __dp4a(w.y, w.y, s);
        s = __dp4a(w.z, w.z, s);
        s = __dp4a(w.w, w.w, s);
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    const int32_t v = local < it.n_b ? (metric == kMetricL2 ? static_cast<int32_t>(s) : 0) : kKeyPad;
    __shared__ int32_t nrm[32];
    int32_t* r = rec + static_cast<size_t>(T) * kRecInts;
    if (sub == 0) {
        nrm[threadIdx.x >> 3] = v;
        r[part * 32 + (threadIdx.x >> 3)] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        int m = nrm[8 * threadIdx.x];
        #pragma unroll
        for (int i = 1; i < 8; ++i) m = min(m, nrm[8 * threadIdx.x + i]);
        r[128 + part * 4 + threadIdx.x] = m;
    }
}

__global__ void __launch_bounds__(kThreads, 1)
    exact2nn_u8_kernel(const __grid_constant__ CUtensorMap qmap, const __grid_constant__ CUtensorMap bmap,
                       const int32_t* __restrict__ brec, const ExactPlan plan, int4* __restrict__ partial,
                       int32_t* __restrict__ thresh, int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte alignment for the 128-byte swizzle atoms.
    const uint32_t raw_u32 = ptx::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (raw_u32 & 1023u)) & 1023u);
    uint8_t* q_smem = smem;
    uint8_t* b_smem = smem + kQT * kQTileBytes;
    int32_t* r_smem = reinterpret_cast<int32_t*>(b_smem + kStages * kBTileBytes);
    SmemCtl* ctl = reinterpret_cast<SmemCtl*>(r_smem + kStages * kRecInts);
    const uint32_t q_s = ptx::smem_u32(q_smem);
    const uint32_t b_s = ptx::smem_u32(b_smem);
    const uint32_t r_s = ptx::smem_u32(r_smem);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const long long W = plan.units;
    const long long G = plan.grid;
    const long long w_begin = plan_w0(blockIdx.x, W, G);
    const int n_units = static_cast<int>(plan_w0(blockIdx.x + 1, W, G) - w_begin);
    const int BT = plan.base_tiles;
    const int g_begin = static_cast<int>(w_begin / BT);
    const int j_begin = static_cast<int>(w_begin - static_cast<long long>(g_begin) * BT);

    const uint32_t bar_full = ptx::smem_u32(&ctl->full[0]);
    const uint32_t bar_empty = ptx::smem_u32(&ctl->empty[0]);
    const uint32_t bar_nempty = ptx::smem_u32(&ctl->nempty[0]);
    const uint32_t bar_qfull = ptx::smem_u32(&ctl->qfull);
    const uint32_t bar_qempty = ptx::smem_u32(&ctl->qempty);
    const uint32_t bar_tfull = ptx::smem_u32(&ctl->tfull[0]);
    const uint32_t bar_tempty = ptx::smem_u32(&ctl->tempty[0]);
    const uint32_t bar_drain = ptx::smem_u32(&ctl->drain);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            ptx::mbar_init(bar_full + 8 * s, 1);
            ptx::mbar_init(bar_empty + 8 * s, 1);
            ptx::mbar_init(bar_nempty + 8 * s, kEpiWarps);
        }
        ptx::mbar_init(bar_qfull, 1);
        ptx::mbar_init(bar_qempty, 1);
        for (int i = 0; i < kQT; ++i) {
            ptx::mbar_init(bar_tfull + 8 * i, 1);
            ptx::mbar_init(bar_tempty + 8 * i, 4);  // the four lane-quarter warps of tile i
        }
        ptx::mbar_init(bar_drain, 1);
        ctl->abort_flag = 0;
        ctl->no_abort = 0;
        ptx::fence_mbar_init();
    }
    if (warp == 1) {
        ptx::tmem_alloc(ptx::smem_u32(&ctl->tmem_base), kTmemCols);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;
    volatile int* abort_flag = &ctl->abort_flag;
    volatile int* never = &ctl->no_abort;  // drain waits: time-bounded, never aborted early

    if (warp == 0) {
        if (lane == 0) {
            // ------------------------------------------------ TMA producer
            ptx::tma_prefetch_desc(&qmap);
            ptx::tma_prefetch_desc(&bmap);
            int cur_g = -1, ngroups = 0;
            int g = g_begin, j = j_begin;
            int n = 0;
            for (; n < n_units; ++n) {
                if (g != cur_g) {
                    if (ngroups > 0 &&
                        !ptx::mbar_wait(bar_qempty, (ngroups - 1) & 1, abort_flag, err, kErrWaitQuery))
                        break;
                    const int t0 = g * kQT;
                    const int nqt = min(kQT, plan.q_tiles - t0);
                    ptx::mbar_arrive_expect_tx(bar_qfull, nqt * kQTileBytes);
                    for (int t = 0; t < nqt; ++t)
                        ptx::tma_load_2d(q_s + t * kQTileBytes, &qmap, 0, (t0 + t) * kBM, bar_qfull);
                    cur_g = g;
                    ++ngroups;
                }
                const int s = n % kStages;
                const uint32_t par = ((n / kStages) & 1) ^ 1;
                if (!ptx::mbar_wait(bar_empty + 8 * s, par, abort_flag, err, kErrWaitProducer)) break;
                if (!ptx::mbar_wait(bar_nempty + 8 * s, par, abort_flag, err, kErrWaitProducer)) break;
                ptx::mbar_arrive_expect_tx(bar_full + 8 * s, kBTileBytes + kRecBytes);
                ptx::tma_load_2d(b_s + s * kBTileBytes, &bmap, 0, j * kBN, bar_full + 8 * s);
                ptx::bulk_load(r_s + s * kRecBytes, brec + static_cast<size_t>(j) * kRecInts, kRecBytes,
                               bar_full + 8 * s);
                if (++j == BT) { j = 0; ++g; }
            }
            // Drain: every issued copy lands before the CTA may exit.
            for (int k = (n > kStages ? n - kStages : 0); k < n; ++k)
                ptx::mbar_wait(bar_full + 8 * (k % kStages), (k / kStages) & 1, never, err, kErrWaitDrain);
            if (ngroups > 0) ptx::mbar_wait(bar_qfull, (ngroups - 1) & 1, never, err, kErrWaitDrain);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // -------------------------------------------------- MMA issuer
            constexpr uint32_t idesc = ptx::idesc_make(2 /*S32*/, 0 /*u8*/, 0 /*u8*/, kBM, kBN);
            int cur_g = -1, ngroups = 0, nqt = 0;
            int g = g_begin, j = j_begin;
            uint32_t use_parity = 0;  // bit t: parity of the accumulator uses of tile t so far
            bool ok = true;
            for (int n = 0; n < n_units && ok; ++n) {
                if (g != cur_g) {
                    if (!ptx::mbar_wait(bar_qfull, ngroups & 1, abort_flag, err, kErrWaitQuery)) break;
                    cur_g = g;
                    ++ngroups;
                    nqt = min(kQT, plan.q_tiles - g * kQT);
                }
                const int s = n % kStages;
                if (!ptx::mbar_wait(bar_full + 8 * s, (n / kStages) & 1, abort_flag, err, kErrWaitMmaFull)) break;
                ptx::tc_fence_after();
                const uint32_t b0 = b_s + s * kBTileBytes;
                #pragma unroll
                for (int t = 0; t < kQT; ++t) {
                    if (t < nqt && ok) {
                        if (!ptx::mbar_wait(bar_tempty + 8 * t, ((use_parity >> t) & 1) ^ 1, abort_flag, err,
                                            kErrWaitMmaTmem)) {
                            ok = false;
                        } else {
                            ptx::tc_fence_after();
                            const uint32_t d = tmem + t * kBN;
                            const uint32_t a0 = q_s + t * kQTileBytes;
                            #pragma unroll
                            for (int kk = 0; kk < kDim / 32; ++kk)
                                ptx::mma_i8(d, ptx::sdesc_sw128(a0 + kk * 32), ptx::sdesc_sw128(b0 + kk * 32), idesc,
                                            kk > 0 ? 1u : 0u);
                            ptx::tc_commit(bar_tfull + 8 * t);
                            use_parity ^= 1u << t;
                        }
                    }
                }
                if (!ok) break;
                ptx::tc_commit(bar_empty + 8 * s);
                const bool last_of_group = (n + 1 == n_units) || (j + 1 == BT);
                if (last_of_group) ptx::tc_commit(bar_qempty);
                if (++j == BT) { j = 0; ++g; }
            }
            // Drain: all issued MMAs complete before TMEM is released.
            ptx::tc_commit(bar_drain);
            ptx::mbar_wait(bar_drain, 0, never, err, kErrWaitDrain);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------ epilogue
        const int e = warp - 2;
        const int t = e >> 2;          // query tile of this warp
        const int quarter = warp & 3;  // TMEM lane quarter this warp may access
        const uint32_t taddr0 = tmem + (static_cast<uint32_t>(quarter * 32) << 16) + t * kBN;
        Top2 st{INT_MAX, -1, INT_MAX, -1, INT_MAX};
        int published = INT_MAX;
        int cur_g = -1, nqt = 0, split = 0, q = 0;
        int g = g_begin, j = j_begin;
        uint32_t use = 0;

        for (int n = 0; n < n_units; ++n) {
            if (g != cur_g) {
                if (cur_g >= 0 && t < nqt)
                    partial[static_cast<size_t>(split) * plan.q_pad + q] = make_int4(st.k1, st.i1, st.k2, st.i2);
                st = Top2{INT_MAX, -1, INT_MAX, -1, INT_MAX};
                published = INT_MAX;
                cur_g = g;
                nqt = min(kQT, plan.q_tiles - g * kQT);
                split = static_cast<int>(blockIdx.x) - plan_cta_of(static_cast<long long>(g) * BT, W, G);
                q = (g * kQT + t) * kBM + quarter * 32 + lane;
            }
            const bool active = t < nqt;
            // Bound shared with the other CTAs that scan this query's group;
            // loaded before the waits so its latency hides behind them.
            const int shared_thr = active ? __ldcg(thresh + q) : INT_MAX;
            const int s = n % kStages;
            bool waited = ptx::mbar_wait(bar_full + 8 * s, (n / kStages) & 1, abort_flag, err, kErrWaitEpilogue);
            if (active && waited)
                waited = ptx::mbar_wait(bar_tfull + 8 * t, use & 1, abort_flag, err, kErrWaitEpilogue);
            if (!__all_sync(0xffffffffu, waited)) break;
            if (active) {
                ++use;
                ptx::tc_fence_after();
                st.thr = min(st.thr, shared_thr);
                const int32_t* rec = r_smem + s * kRecInts;
                const int row0 = j * kBN;
                uint32_t va[32];
                ptx::tmem_ld32(taddr0, va);
                ptx::tmem_ld_wait(va);
                scan_group(va, row0, rec, rec + 128, st);
                ptx::tmem_ld32(taddr0 + 32, va);
                ptx::tmem_ld_wait(va);
                scan_group(va, row0 + 32, rec + 32, rec + 132, st);
                ptx::tmem_ld32(taddr0 + 64, va);
                ptx::tmem_ld_wait(va);
                scan_group(va, row0 + 64, rec + 64, rec + 136, st);
                ptx::tmem_ld32(taddr0 + 96, va);
                ptx::tmem_ld_wait(va);
                ptx::tc_fence_before();
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(bar_tempty + 8 * t);
                scan_group(va, row0 + 96, rec + 96, rec + 140, st);
                if (st.k2 < published) {
                    atomicMin(thresh + q, st.k2);
                    published = st.k2;
                }
            }
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(bar_nempty + 8 * s);
            if (++j == BT) { j = 0; ++g; }
        }
        if (cur_g >= 0 && t < nqt)
            partial[static_cast<size_t>(split) * plan.q_pad + q] = make_int4(st.k1, st.i1, st.k2, st.i2);
    }

    ptx::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc(tmem, kTmemCols);
    }
}

__device__ __forceinline__ bool lex_less(int ka, int ia, int kb, int ib) {
    return ka < kb || (ka == kb && ia < ib);
}

// FLOATKEY: the keys are ordered images of float keys (float_key) and the
// query norms float bit patterns (the general float path); else integers.
template <bool FLOATKEY>
__global__ void __launch_bounds__(256) merge2nn_kernel(const int4* __restrict__ partial, const ExactPlan plan,
                                                       const WorkItem* __restrict__ items, int n_items,
                                                       const WorkItem single, int group_rows, int total_q,
                                                       const int32_t* __restrict__ qnorm, int metric, float thr,
                                                       float dscale,
                                                       uint32_t* __restrict__ matches, float4* __restrict__ sorted,
                                                       int32_t* __restrict__ nn_idx, float* __restrict__ nn_dist) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= total_q) return;
    const long long W = plan.units, G = plan.grid;
    const WorkItem it =
        items ? items[find_item(n_items, q, [&](int k) { return static_cast<long long>(items[k].a_off); })] : single;
    int a1 = INT_MAX, j1 = -1, a2 = INT_MAX, j2 = -1;
    auto push = [&](int k, int i) {
        if (i < 0) return;
        if (lex_less(k, i, a1, j1) || j1 < 0) {
            a2 = a1; j2 = j1;
            a1 = k; j1 = i;
        } else if (lex_less(k, i, a2, j2) || j2 < 0) {
            a2 = k; j2 = i;
        }
    };
    // No base rows: no CTA scanned this query and every neighbour is absent.
    if (W > 0 && it.tiles > 0) {
        const long long first = it.u_begin + static_cast<long long>((q - it.a_off) / group_rows) * it.tiles;
        const int c0 = plan_cta_of(first, W, G);
        const int c1 = plan_cta_of(first + it.tiles - 1, W, G);
        for (int s = 0; s < (c1 - c0 + 1) * plan.parts; ++s) {
            const int4 p = partial[static_cast<size_t>(s) * plan.q_pad + q];
            push(p.x, p.y);
            push(p.z, p.w);
        }
    }
    // Rows past the problem's base set are padding (they may hold another
    // problem's rows, but only enter a top-2 when fewer real rows exist).
    bool v1, v2;
    float d1, d2;
    if constexpr (FLOATKEY) {
        // Squared distances |b|^2 - 2 q.b + |q|^2 can round a little below
        // zero for (near-)identical rows: clamped at 0.
        v1 = j1 >= 0 && j1 < it.n_b;
        v2 = j2 >= 0 && j2 < it.n_b;
        const float qn = metric == kMetricL2 ? __int_as_float(qnorm[q]) : 0.0f;
        const float lo = metric == kMetricL2 ? 0.0f : -FLT_MAX;
        d1 = v1 ? fmaxf((key_float(a1) + qn) * dscale, lo) : FLT_MAX;
        d2 = v2 ? fmaxf((key_float(a2) + qn) * dscale, lo) : FLT_MAX;
    } else {
        v1 = j1 >= 0 && j1 < it.n_b && a1 < kKeyPad;
        v2 = j2 >= 0 && j2 < it.n_b && a2 < kKeyPad;
        const int qn = metric == kMetricL2 ? qnorm[q] : 0;
        d1 = v1 ? static_cast<float>(a1 + qn) * dscale : FLT_MAX;
        d2 = v2 ? static_cast<float>(a2 + qn) * dscale : FLT_MAX;
    }
    if (matches) {
        bool pass = false;
        if (v1) {
            float f1, f2;
            if (metric == kMetricL2) {
                f1 = sqrtf(d1);
                f2 = v2 ? sqrtf(d2) : INFINITY;
            } else {
                f1 = sqrtf(d1 + 2.0f);
                f2 = v2 ? sqrtf(d2 + 2.0f) : INFINITY;
            }
            pass = (f1 / f2) < thr;
        }
        matches[q] = pass ? static_cast<uint32_t>(j1) : UINT32_MAX;
    }
    if (sorted)
        sorted[q] = make_float4(d1, d2, v1 ? static_cast<float>(j1) : FLT_MAX, v2 ? static_cast<float>(j2) : FLT_MAX);
    if (nn_idx) {
        nn_idx[2 * q] = v1 ? j1 : -1;
        nn_idx[2 * q + 1] = v2 ? j2 : -1;
    }
    if (nn_dist) {
        nn_dist[2 * q] = d1;
        nn_dist[2 * q + 1] = d2;
    }
}

// Merge of a search split over base chunks (indices already global). A
// query row has a partial list per (chunk, CTA pair of its group, buffer),
// ~90 for 10,000 x 1,000,000 in 9 chunks: kMergeLanes threads per row read
// every kMergeLanes-th list (independent loads instead of one dependent
// chain), and their top-2s are merged by shuffles. Every row of the base is
// in exactly one list and (key, index) is a total order, so the top-2 does
// not depend on the order of the merges.
constexpr int kMergeLanes = 8;
__global__ void __launch_bounds__(256) merge2nn_chunks_kernel(const int4* __restrict__ partial, const ChunkSet cs,
                                                              int q_n, const int32_t* __restrict__ qnorm, int metric,
                                                              float thr, float dscale, uint32_t* __restrict__ matches,
                                                              float4* __restrict__ sorted,
                                                              int32_t* __restrict__ nn_idx,
                                                              float* __restrict__ nn_dist) {
    const long long tid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int q = static_cast<int>(tid / kMergeLanes), sub = static_cast<int>(tid % kMergeLanes);
    int a1 = INT_MAX, j1 = -1, a2 = INT_MAX, j2 = -1;
    auto push = [&](int k, int i) {
        if (i < 0) return;
        if (lex_less(k, i, a1, j1) || j1 < 0) {
            a2 = a1; j2 = j1;
            a1 = k; j1 = i;
        } else if (lex_less(k, i, a2, j2) || j2 < 0) {
            a2 = k; j2 = i;
        }
    };
    if (q < q_n) {
        const int g = q / (kQT * kBM);
        int done = 0;  // lists of the earlier chunks
        for (int c = 0; c < cs.n; ++c) {
            if (cs.W[c] <= 0 || cs.tiles[c] <= 0) continue;
            const long long first = static_cast<long long>(g) * cs.tiles[c];
            const int c0 = plan_cta_of(first, cs.W[c], cs.G[c]);
            const int c1 = plan_cta_of(first + cs.tiles[c] - 1, cs.W[c], cs.G[c]);
            const int4* pc = partial + c * cs.slot_stride;
            const int n_lists = (c1 - c0 + 1) * cs.parts;
            for (int s = (sub - done % kMergeLanes + kMergeLanes) % kMergeLanes; s < n_lists; s += kMergeLanes) {
                const int4 p = pc[static_cast<size_t>(s) * cs.q_pad + q];
                push(p.x, p.y);
                push(p.z, p.w);
            }
            done += n_lists;
        }
    }
    // The kMergeLanes threads of a row are consecutive lanes of one warp.
    #pragma unroll
    for (int off = 1; off < kMergeLanes; off <<= 1) {
        const int b1 = __shfl_xor_sync(0xffffffffu, a1, off), i1 = __shfl_xor_sync(0xffffffffu, j1, off);
        const int b2 = __shfl_xor_sync(0xffffffffu, a2, off), i2 = __shfl_xor_sync(0xffffffffu, j2, off);
        push(b1, i1);
        push(b2, i2);
    }
    if (q >= q_n || sub != 0) return;
    const bool v1 = j1 >= 0 && j1 < cs.r_n && a1 < kKeyPad;
    const bool v2 = j2 >= 0 && j2 < cs.r_n && a2 < kKeyPad;
    const int qn = metric == kMetricL2 ? qnorm[q] : 0;
    const float d1 = v1 ? static_cast<float>(a1 + qn) * dscale : FLT_MAX;
    const float d2 = v2 ? static_cast<float>(a2 + qn) * dscale : FLT_MAX;
    if (matches) {
        bool pass = false;
        if (v1) {
            const float f1 = metric == kMetricL2 ? sqrtf(d1) : sqrtf(d1 + 2.0f);
            const float f2 = v2 ? (metric == kMetricL2 ? sqrtf(d2) : sqrtf(d2 + 2.0f)) : INFINITY;
            pass = (f1 / f2) < thr;
        }
        matches[q] = pass ? static_cast<uint32_t>(j1) : UINT32_MAX;
    }
    if (sorted)
        sorted[q] = make_float4(d1, d2, v1 ? static_cast<float>(j1) : FLT_MAX, v2 ? static_cast<float>(j2) : FLT_MAX);
    if (nn_idx) {
        nn_idx[2 * q] = v1 ? j1 : -1;
        nn_idx[2 * q + 1] = v2 ? j2 : -1;
    }
    if (nn_dist) {
        nn_dist[2 * q] = d1;
        nn_dist[2 * q + 1] = d2;
    }
}

}  // namespace

cudaError_t launch_merge2nn_chunks(const int4* partial, const ChunkSet& cs, int q_n, const int32_t* qnorm, int metric,
                                   float threshold, float dist_scale, uint32_t* matches, float4* sorted,
                                   int32_t* nn_idx, float* nn_dist, cudaStream_t stream) {
    if (q_n <= 0) return cudaSuccess;
    const long long threads = static_cast<long long>(q_n) * kMergeLanes;
    merge2nn_chunks_kernel<<<static_cast<unsigned>((threads + 255) / 256), 256, 0, stream>>>(
        partial, cs, q_n, qnorm, metric, threshold, dist_scale, matches, sorted, nn_idx, nn_dist);
    return cudaGetLastError();
}

ExactPlan make_exact_plan(int q_n, int r_n, int num_sms, int parts, int group_tiles) {
    ExactPlan p{};
    p.parts = parts;
    p.q_n = q_n;
    p.r_n = r_n;
    p.q_tiles = (q_n + kBM - 1) / kBM;
    p.q_groups = (p.q_tiles + group_tiles - 1) / group_tiles;
    p.q_pad = p.q_tiles * kBM;
    p.base_tiles = (r_n + kBN - 1) / kBN;
    p.r_pad = p.base_tiles * kBN;
    p.units = static_cast<long long>(p.q_groups) * p.base_tiles;
    p.grid = static_cast<int>(std::min<long long>(num_sms, p.units));
    int ms = 1;
    if (p.grid > 0) {
        for (int g = 0; g < p.q_groups; ++g) {
            const long long BT = p.base_tiles;
            const int c0 = plan_cta_of(g * BT, p.units, p.grid);
            const int c1 = plan_cta_of((g + 1) * BT - 1, p.units, p.grid);
            ms = std::max(ms, c1 - c0 + 1);
        }
    }
    p.max_splits = ms;
    return p;
}

size_t exact2nn_smem_bytes() { return kSmemBytes; }

cudaError_t launch_row_norms_u8(const uint8_t* x, int n, int n_pad, int metric, int32_t* norm, int32_t* rec,
                                int32_t* thresh, cudaStream_t stream) {
    if (n_pad <= 0) return cudaSuccess;
    row_norms_kernel<uint8_t><<<n_pad / 32, 256, 0, stream>>>(x, n, n_pad, 1.0f, metric, norm, rec, thresh);
    return cudaGetLastError();
}

cudaError_t launch_fold_records_u8(const uint8_t* x, int n, int n_pad, int metric, int32_t* rec, uint32_t* fold,
                                   cudaStream_t stream) {
    if (n_pad <= 0) return cudaSuccess;
    fold_records_kernel<<<n_pad / kBN, 256, 0, stream>>>(x, n, n_pad, metric, rec, fold);
    return cudaGetLastError();
}

cudaError_t launch_row_norms_f16(const void* x, int n, int n_pad, float mul, int metric, int32_t* norm, int32_t* rec,
                                 int32_t* thresh, cudaStream_t stream) {
    if (n_pad <= 0) return cudaSuccess;
    row_norms_kernel<__half><<<n_pad / 32, 256, 0, stream>>>(static_cast<const __half*>(x), n, n_pad, mul, metric,
                                                             norm, rec, thresh);
    return cudaGetLastError();
}

cudaError_t launch_row_norms_float(const void* x, bool half, int n, int n_pad, float mul, int metric, int32_t* norm,
                                   int32_t* rec, int32_t* thresh, cudaStream_t stream) {
    if (n_pad <= 0) return cudaSuccess;
    if (half)
        row_norms_float_kernel<__half><<<n_pad / 32, 256, 0, stream>>>(static_cast<const __half*>(x), n, n_pad, mul,
                                                                       metric, norm, rec, thresh);
    else
        row_norms_float_kernel<float><<<n_pad / 32, 256, 0, stream>>>(static_cast<const float*>(x), n, n_pad, mul,
                                                                      metric, norm, rec, thresh);
    return cudaGetLastError();
}

cudaError_t launch_exact2nn_u8(const CUtensorMap& qmap, const CUtensorMap& bmap, const int32_t* brec,
                               const ExactPlan& plan, int4* partial, int32_t* thresh, int* err, cudaStream_t stream) {
    // The shared-memory opt-in is per device; the host API serialises calls per device.
    static bool attr_set[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        e = cudaFuncSetAttribute(exact2nn_u8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kSmemBytes));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
    if (plan.grid <= 0) return cudaSuccess;
    exact2nn_u8_kernel<<<plan.grid, kThreads, kSmemBytes, stream>>>(qmap, bmap, brec, plan, partial, thresh, err);
    return cudaGetLastError();
}

cudaError_t launch_merge2nn(const int4* partial, const ExactPlan& plan, const int32_t* qnorm, int metric,
                            float threshold, float dist_scale, uint32_t* matches, float4* sorted, int32_t* nn_idx,
                            float* nn_dist, cudaStream_t stream) {
    if (plan.q_n <= 0) return cudaSuccess;
    WorkItem single{};
    single.n_a = plan.q_n;
    single.n_b = plan.r_n;
    single.groups = plan.q_groups;
    single.tiles = plan.base_tiles;
    merge2nn_kernel<false><<<(plan.q_n + 255) / 256, 256, 0, stream>>>(partial, plan, nullptr, 1, single, kQT * kBM,
                                                                      plan.q_n, qnorm, metric, threshold, dist_scale,
                                                                      matches, sorted, nn_idx, nn_dist);
    return cudaGetLastError();
}

cudaError_t launch_merge2nn_float(const int4* partial, const ExactPlan& plan, int group_rows, const int32_t* qnorm,
                                  int metric, float threshold, float dist_scale, uint32_t* matches, float4* sorted,
                                  int32_t* nn_idx, float* nn_dist, cudaStream_t stream) {
    if (plan.q_n <= 0) return cudaSuccess;
    WorkItem single{};
    single.n_a = plan.q_n;
    single.n_b = plan.r_n;
    single.groups = plan.q_groups;
    single.tiles = plan.base_tiles;
    merge2nn_kernel<true><<<(plan.q_n + 255) / 256, 256, 0, stream>>>(partial, plan, nullptr, 1, single, group_rows,
                                                                     plan.q_n, qnorm, metric, threshold, dist_scale,
                                                                     matches, sorted, nn_idx, nn_dist);
    return cudaGetLastError();
}

cudaError_t launch_merge2nn_batch(const int4* partial, const BatchPlan& bp, int total_queries, const int32_t* qnorm,
                                  int metric, float threshold, float dist_scale, uint32_t* matches, float4* sorted,
                                  int32_t* nn_idx, float* nn_dist, cudaStream_t stream) {
    if (total_queries <= 0) return cudaSuccess;
    merge2nn_kernel<false><<<(total_queries + 255) / 256, 256, 0, stream>>>(
        partial, bp.plan, bp.items, bp.n_items, WorkItem{}, bp.group_rows, total_queries, qnorm, metric, threshold,
        dist_scale, matches, sorted, nn_idx, nn_dist);
    return cudaGetLastError();
}

cudaError_t launch_batch_records(const uint8_t* base, int, const BatchPlan& bp, int metric, int32_t* rec,
                                 cudaStream_t stream) {
    if (bp.total_tiles <= 0) return cudaSuccess;
    batch_records_kernel<<<bp.total_tiles * 4, 256, 0, stream>>>(base, bp.items, bp.n_items, metric, rec);
    return cudaGetLastError();
}

long long make_batch_items(int n_items, const int* n_a, const int* n_b, const int* b_off, int group_rows,
                           WorkItem* items, int* total_tiles, int* total_queries) {
    long long u = 0;
    int a = 0, rec = 0;
    for (int p = 0; p < n_items; ++p) {
        WorkItem& it = items[p];
        it = WorkItem{};
        it.a_off = a;
        it.n_a = n_a[p];
        it.b_off = b_off[p];
        it.n_b = n_b[p];
        it.groups = (n_a[p] + group_rows - 1) / group_rows;
        it.tiles = (n_b[p] + kBN - 1) / kBN;
        it.u_begin = u;
        it.rec_off = rec;
        u += static_cast<long long>(it.groups) * it.tiles;
        rec += it.tiles;
        a += n_a[p];
    }
    if (total_tiles) *total_tiles = rec;
    if (total_queries) *total_queries = a;
    return u;
}

ExactPlan make_batch_plan(const WorkItem* items, int n_items, long long units, int total_queries, int num_workers,
                          int parts) {
    ExactPlan p{};
    p.parts = parts;
    p.q_n = total_queries;
    p.r_n = 0;
    p.q_tiles = (total_queries + kBM - 1) / kBM;
    p.q_pad = p.q_tiles * kBM;
    p.units = units;
    p.grid = static_cast<int>(std::min<long long>(num_workers, units));
    int ms = 1;
    if (p.grid > 0) {
        for (int k = 0; k < n_items; ++k) {
            const WorkItem& it = items[k];
            for (int g = 0; g < it.groups && it.tiles > 0; ++g) {
                const long long first = it.u_begin + static_cast<long long>(g) * it.tiles;
                const int c0 = plan_cta_of(first, units, p.grid);
                const int c1 = plan_cta_of(first + it.tiles - 1, units, p.grid);
                ms = std::max(ms, c1 - c0 + 1);
            }
        }
    }
    p.max_splits = ms;
    return p;
}

}  // namespace sift
