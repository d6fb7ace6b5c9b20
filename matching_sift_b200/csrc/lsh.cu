// Random-hyperplane LSH for u8 SIFT descriptors on sm_100a.
//
// Replaces the reference's LSH pipeline (src/lsh_h.cu):
//   hash GEMM cublasHgemm(H, X)            :909, :914   -> lsh_hash_kernel (tcgen05 kind::i8)
//   set_bit_h sign packing                 :265-317     -> fused into lsh_hash_kernel's epilogue
//   thrust::sort by code + host run-length :565-629     -> bucket histogram / scan / scatter kernels
//   host merge-join of Q and R buckets     :657-681     -> the query code indexes the bucket table
//   brute_2nn_h + atomic_min2_update       :441-562     -> lsh_scan_kernel (warp per query)
//
// Codes. Table t of L uses k hyperplanes; bit j of a point's code is set when
// its dot product with hyperplane j is negative (set_bit_h, src/lsh_h.cu:302-309).
// Hyperplanes are int8, so the dot products are exact integers computed on
// the tensor cores (u8 x s8 -> s32), and a code is a pure function of the
// point and the hyperplanes.
//
// Buckets. Per table, base points are grouped by the top B = min(k, 16) bits
// of their code (counting sort: histogram, exclusive scan, scatter). A query
// scans the group of its own top bits and keeps the members whose full code
// equals its own, so every table contributes exactly the bucket of the
// query's code (the reference scans sorted positions starting at a point id
// instead, src/lsh_h.cu:599,617 vs :469,482, which is not the bucket).
//
// Candidate scan. One warp per query over its L buckets (L x P with P probe
// codes per table: multi-probe); candidate rows are fetched by groups of 8
// lanes with coalesced 16-byte loads (4 rows per warp-wide load) and scored
// as the exact |q - b|^2 (byte-wise absolute differences squared and summed
// by dp4a); the per-query top-2 is lexicographic in (distance, index) and
// counts a base point found in several tables once.
#include <climits>
#include <cfloat>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>
#include "lsh.cuh"
#include "ptx.cuh"

namespace sift {
namespace {

// ------------------------------------------------------------ hash kernel
constexpr int kHStages = 6;
constexpr int kHTileBytes = 128 * 128;  // 128 points x 128 u8
constexpr int kHThreads = 64 + 4 * 32;  // producer, MMA, 4 epilogue warps

struct __align__(8) HashCtl {
    uint64_t full[kHStages], empty[kHStages];
    uint64_t pfull;
    uint64_t tfull[4], tempty[4];
    uint64_t drain;
    uint32_t tmem_base;
    int abort_flag, no_abort;
};

__host__ __device__ constexpr size_t hash_smem_bytes(int P) {
    return 1024 + static_cast<size_t>(P) * 128 + kHStages * kHTileBytes + sizeof(HashCtl);
}

// P = number of hyperplane rows padded to a multiple of 32 (<= 256). TMEM:
// nbuf accumulator buffers of slot_cols columns (P rounded up to a power of
// two; nbuf = 4 for P <= 128, else 2), so the MMA of tile i + nbuf - 1 can run
// while the epilogue still reads tile i.
__global__ void __launch_bounds__(kHThreads, 1)
    lsh_hash_kernel(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap pmap, int n, int P,
                    int L, int k, int nbuf, uint32_t slot_cols, uint32_t* __restrict__ codes,
                    float* __restrict__ z, int* __restrict__ err) {
    const uint32_t tmem_cols = static_cast<uint32_t>(nbuf) * slot_cols;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = ptx::smem_u32(smem_raw);
    uint8_t* smem = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
    uint8_t* p_smem = smem;                                   // P x 128 planes (s8)
    uint8_t* x_smem = smem + static_cast<size_t>(P) * 128;    // point tile ring (P*128 is a multiple of 1024)
    HashCtl* ctl = reinterpret_cast<HashCtl*>(x_smem + kHStages * kHTileBytes);
    const uint32_t p_s = ptx::smem_u32(p_smem), x_s = ptx::smem_u32(x_smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles = (n + 127) / 128;
    const int my_tiles = blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    const uint32_t bar_full = ptx::smem_u32(&ctl->full[0]), bar_empty = ptx::smem_u32(&ctl->empty[0]);
    const uint32_t bar_pfull = ptx::smem_u32(&ctl->pfull), bar_drain = ptx::smem_u32(&ctl->drain);
    const uint32_t bar_tfull = ptx::smem_u32(&ctl->tfull[0]), bar_tempty = ptx::smem_u32(&ctl->tempty[0]);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kHStages; ++s) {
            ptx::mbar_init(bar_full + 8 * s, 1);
            ptx::mbar_init(bar_empty + 8 * s, 1);
        }
        ptx::mbar_init(bar_pfull, 1);
        for (int b = 0; b < nbuf; ++b) {
            ptx::mbar_init(bar_tfull + 8 * b, 1);
            ptx::mbar_init(bar_tempty + 8 * b, 4);
        }
        ptx::mbar_init(bar_drain, 1);
        ctl->abort_flag = 0;
        ctl->no_abort = 0;
        ptx::fence_mbar_init();
    }
    if (warp == 1) {
        ptx::tmem_alloc(ptx::smem_u32(&ctl->tmem_base), tmem_cols);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;
    volatile int* abort_flag = &ctl->abort_flag;
    volatile int* never = &ctl->no_abort;

    if (warp == 0) {
        if (lane == 0) {
            ptx::tma_prefetch_desc(&xmap);
            ptx::tma_prefetch_desc(&pmap);
            // One box of all P hyperplane rows (the map's box is P rows, P <= 256).
            ptx::mbar_arrive_expect_tx(bar_pfull, P * 128);
            ptx::tma_load_2d(p_s, &pmap, 0, 0, bar_pfull);
            int i = 0;
            for (; i < my_tiles; ++i) {
                const int s = i % kHStages;
                if (!ptx::mbar_wait(bar_empty + 8 * s, ((i / kHStages) & 1) ^ 1, abort_flag, err, kErrWaitProducer))
                    break;
                ptx::mbar_arrive_expect_tx(bar_full + 8 * s, kHTileBytes);
                ptx::tma_load_2d(x_s + s * kHTileBytes, &xmap, 0, (blockIdx.x + i * gridDim.x) * 128, bar_full + 8 * s);
            }
            for (int kk = (i > kHStages ? i - kHStages : 0); kk < i; ++kk)
                ptx::mbar_wait(bar_full + 8 * (kk % kHStages), (kk / kHStages) & 1, never, err, kErrWaitDrain);
            ptx::mbar_wait(bar_pfull, 0, never, err, kErrWaitDrain);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // u8 points (A) x s8 hyperplanes (B) -> s32, in MMAs of at most
            // 128 hyperplane columns: P > 128 is split into two equal chunks
            // of P/2 columns (a multiple of 16; each chunk starts on a
            // 1024-byte swizzle atom) written to adjacent TMEM columns.
            const int nchunk = (P + 127) / 128;
            const uint32_t nc = static_cast<uint32_t>(P / nchunk);
            const uint32_t idesc = ptx::idesc_make(2 /*S32*/, 0 /*u8*/, 1 /*s8*/, 128, nc);
            bool ok = ptx::mbar_wait(bar_pfull, 0, abort_flag, err, kErrWaitMmaFull);
            for (int i = 0; i < my_tiles && ok; ++i) {
                const int s = i % kHStages, b = i % nbuf;
                if (!ptx::mbar_wait(bar_full + 8 * s, (i / kHStages) & 1, abort_flag, err, kErrWaitMmaFull)) break;
                if (!ptx::mbar_wait(bar_tempty + 8 * b, ((i / nbuf) & 1) ^ 1, abort_flag, err, kErrWaitMmaTmem))
                    break;
                ptx::tc_fence_after();
                const uint32_t d = tmem + b * slot_cols;
                for (int ch = 0; ch < nchunk; ++ch) {
                    #pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                        ptx::mma_i8(d + ch * nc, ptx::sdesc_sw128(x_s + s * kHTileBytes + kk * 32),
                                    ptx::sdesc_sw128(p_s + ch * nc * 128 + kk * 32), idesc, kk > 0 ? 1u : 0u);
                }
                ptx::tc_commit(bar_tfull + 8 * b);
                ptx::tc_commit(bar_empty + 8 * s);
            }
            ptx::tc_commit(bar_drain);
            ptx::mbar_wait(bar_drain, 0, never, err, kErrWaitDrain);
        }
        __syncwarp();
    } else {
        const int quarter = warp & 3;
        for (int i = 0; i < my_tiles; ++i) {
            const int b = i % nbuf;
            const bool waited = ptx::mbar_wait(bar_tfull + 8 * b, (i / nbuf) & 1, abort_flag, err, kErrWaitEpilogue);
            if (!__all_sync(0xffffffffu, waited)) break;
            ptx::tc_fence_after();
            const uint32_t taddr = tmem + (static_cast<uint32_t>(quarter * 32) << 16) + b * slot_cols;
            const int point = (blockIdx.x + i * gridDim.x) * 128 + quarter * 32 + lane;
            uint32_t mask[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            // Up to 4 loads of 32 columns in flight per wait (one TMEM round
            // trip for P <= 128 hyperplanes instead of one per 32 columns).
            #pragma unroll
            for (int w0 = 0; w0 < 8; w0 += 4) {
                if (w0 * 32 < P) {
                    uint32_t v[4][32];
                    #pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if ((w0 + u) * 32 < P) ptx::tmem_ld32(taddr + (w0 + u) * 32, v[u]);
                    ptx::tmem_ld_wait(v[0]);
                    ptx::tmem_ld_wait(v[1]);
                    ptx::tmem_ld_wait(v[2]);
                    ptx::tmem_ld_wait(v[3]);
                    #pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int w = w0 + u;
                        if (w * 32 < P) {
                            uint32_t m = 0;
                            #pragma unroll
                            for (int c = 0; c < 32; ++c) m |= (v[u][c] >> 31) << c;
                            mask[w] = m;
                            if (z && point < n) {
                                // Dot products of the point with each hyperplane (multi-probe margins).
                                #pragma unroll
                                for (int c = 0; c < 32; ++c) {
                                    const int col = w * 32 + c;
                                    if (col < L * k)
                                        z[(static_cast<size_t>(col / k) * n + point) * k + col % k] =
                                            static_cast<float>(static_cast<int>(v[u][c]));
                                }
                            }
                        }
                    }
                }
            }
            ptx::tc_fence_before();
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(bar_tempty + 8 * b);
            if (point < n) {
                for (int t = 0; t < L; ++t) {
                    const int bit0 = t * k;
                    const int w = bit0 >> 5, sh = bit0 & 31;
                    // mask[w], mask[w + 1] by selects (register-resident, no indexed access)
                    uint32_t lo = mask[0], hi = mask[1];
                    #pragma unroll
                    for (int u = 1; u < 8; ++u) {
                        lo = w == u ? mask[u] : lo;
                        hi = w + 1 == u ? mask[u] : hi;
                    }
                    if (w + 1 >= 8) hi = 0;
                    const uint64_t pair = static_cast<uint64_t>(lo) | (static_cast<uint64_t>(hi) << 32);
                    const uint32_t code = static_cast<uint32_t>(pair >> sh) & (k == 32 ? 0xffffffffu : ((1u << k) - 1));
                    codes[static_cast<size_t>(t) * n + point] = code;
                }
            }
        }
    }
    ptx::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc(tmem, tmem_cols);
    }
}

// --------------------------------------------------------------- buckets
// hist[t][bin] counts the points of table t whose code's top bits are bin.
__global__ void lsh_hist_kernel(const uint32_t* __restrict__ codes, int n, int L, int shift, int nbins,
                                int* __restrict__ hist) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < static_cast<size_t>(n) * L;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int t = static_cast<int>(i / n);
        atomicAdd(&hist[static_cast<size_t>(t) * nbins + (codes[i] >> shift)], 1);
    }
}

// Exclusive scan of hist[t][0..nbins) into start[t][0..nbins] (one block per table).
__global__ void __launch_bounds__(1024) lsh_scan_bins_kernel(const int* __restrict__ hist, int nbins,
                                                             int* __restrict__ start) {
    const int t = blockIdx.x;
    const int* h = hist + static_cast<size_t>(t) * nbins;
    int* st = start + static_cast<size_t>(t) * (nbins + 1);
    const int per = (nbins + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * per, b1 = min(b0 + per, nbins);
    int local = 0;
    for (int b = b0; b < b1; ++b) local += h[b];
    __shared__ int warp_sums[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = local;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0) {
        int v = lane < (blockDim.x >> 5) ? warp_sums[lane] : 0;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        warp_sums[lane] = v;
    }
    __syncthreads();
    int run = incl - local + (w > 0 ? warp_sums[w - 1] : 0);
    for (int b = b0; b < b1; ++b) {
        st[b] = run;
        run += h[b];
    }
    if (threadIdx.x == blockDim.x - 1) st[nbins] = run;
}

// order[t][pos] = point id, ocode[t][pos] = its code, grouped by top bits.
// hist is consumed (counted down to zero).
__global__ void lsh_scatter_kernel(const uint32_t* __restrict__ codes, int n, int L, int shift, int nbins,
                                   const int* __restrict__ start, int* __restrict__ hist, int* __restrict__ order,
                                   uint32_t* __restrict__ ocode) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < static_cast<size_t>(n) * L;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int t = static_cast<int>(i / n);
        const int id = static_cast<int>(i - static_cast<size_t>(t) * n);
        const uint32_t c = codes[i];
        const int bin = static_cast<int>(c >> shift);
        const int pos = start[static_cast<size_t>(t) * (nbins + 1) + bin] +
                        atomicSub(&hist[static_cast<size_t>(t) * nbins + bin], 1) - 1;
        order[static_cast<size_t>(t) * n + pos] = id;
        ocode[static_cast<size_t>(t) * n + pos] = c;
    }
}

// ---------------------------------------------------------- candidate scan
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

// One warp per query, its buckets walked 32 positions at a time. The ids and
// codes of a chunk are one coalesced 128-byte load each (the next chunk's are
// fetched while the current chunk's rows load); members whose full code
// matches are compacted through shared memory; then every 8 lanes fetch one
// candidate row with coalesced 16-byte loads (4 rows per warp-wide load, up
// to 8 loads = 32 rows in flight per lane before any arithmetic), each lane
// forms the squared distance of its 16 bytes (byte-wise absolute difference,
// then dp4a) and 3 shuffles sum them: exact integers, no norms needed. The
// lane leading each group of 8 keeps a lexicographic (distance, index)
// top-2; the four lists are merged at the end. A base row found in several
// tables (or probes) is compared each time but enters a list once.
constexpr int kScanThreads = 256;

__global__ void __launch_bounds__(kScanThreads) lsh_scan_kernel(
    const uint8_t* __restrict__ q, const uint8_t* __restrict__ r, int q_n, int r_n, int L, int probes, int shift,
    int nbins, const uint32_t* __restrict__ qcodes, const int* __restrict__ start, const int* __restrict__ order,
    const uint32_t* __restrict__ ocode, float thr, int ratio, float dscale, uint32_t* __restrict__ matches,
    uint32_t* __restrict__ counts, int32_t* __restrict__ nn_idx, float* __restrict__ nn_dist) {
    __shared__ int s_ids[kScanThreads / 32][32];
    const int wq = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int sub = lane >> 3, part = lane & 7;  // row slot of a 4-row load, 16-byte chunk of the row
    if (wq >= q_n) return;
    int* ids = s_ids[threadIdx.x >> 5];
    const uint4 qv = __ldg(reinterpret_cast<const uint4*>(q + static_cast<size_t>(wq) * 128) + part);
    const bool whole_bins = shift == 0;  // a group holds exactly one code
    int d1 = INT_MAX, i1 = -1, d2 = INT_MAX, i2 = -1;
    uint32_t seen = 0;  // candidates compared (bucket members)
    for (int t = 0; t < L; ++t) {
        // The table's probe codes and their bucket bounds, one probe per lane
        // (probes <= 64: two per lane), fetched in parallel: two round trips per
        // table instead of two per probe.
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
            int nid = -1;
            uint32_t ncode = ~code;
            if (s + lane < e) {
                nid = ord[s + lane];
                ncode = whole_bins ? code : oc[s + lane];
            }
            for (int p0 = s; p0 < e; p0 += 32) {
                const int id = nid;
                const bool hit = id >= 0 && ncode == code;
                const int pn = p0 + 32 + lane;
                nid = -1;
                ncode = ~code;
                if (pn < e) {
                    nid = ord[pn];
                    ncode = whole_bins ? code : oc[pn];
                }
                const uint32_t mask = __ballot_sync(0xffffffffu, hit);
                const int nm = __popc(mask);
                if (nm == 0) continue;
                seen += nm;
                if (hit) ids[__popc(mask & ((1u << lane) - 1u))] = id;
                __syncwarp();
                // The hits in two rounds of 16 (4 rows per lane in flight):
                // fewer registers than one round of 32, so more queries (warps)
                // share an SM and hide each other's load latency.
                #pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (16 * h >= nm) break;
                    uint4 rv[4];
                    int cid[4];
                    #pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int rank = 16 * h + 4 * j + sub;
                        cid[j] = rank < nm ? ids[rank] : -1;
                        if (cid[j] >= 0)
                            rv[j] = __ldg(reinterpret_cast<const uint4*>(r + static_cast<size_t>(cid[j]) * 128) + part);
                    }
                    #pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        if (16 * h + 4 * j >= nm) break;
                        // |q - b|^2 of this lane's 16 bytes: byte-wise |q - b| (SIMD
                        // absolute difference), then the sum of their squares by dp4a.
                        uint32_t dist = 0;
                        if (cid[j] >= 0) {
                            uint32_t a = __vabsdiffu4(qv.x, rv[j].x);
                            dist = __dp4a(a, a, dist);
                            a = __vabsdiffu4(qv.y, rv[j].y);
                            dist = __dp4a(a, a, dist);
                            a = __vabsdiffu4(qv.z, rv[j].z);
                            dist = __dp4a(a, a, dist);
                            a = __vabsdiffu4(qv.w, rv[j].w);
                            dist = __dp4a(a, a, dist);
                        }
                        dist += __shfl_xor_sync(0xffffffffu, dist, 1);
                        dist += __shfl_xor_sync(0xffffffffu, dist, 2);
                        dist += __shfl_xor_sync(0xffffffffu, dist, 4);
                        if (part == 0 && cid[j] >= 0) push_dedup(static_cast<int>(dist), cid[j], d1, i1, d2, i2);
                    }
                }
                __syncwarp();  // ids is rewritten by the next 32 positions
            }
        }
    }
    // Merge the four group lists (lexicographic, duplicates counted once).
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
        const float f1 = v1 ? static_cast<float>(d1) * dscale : FLT_MAX;
        const float f2 = v2 ? static_cast<float>(d2) * dscale : FLT_MAX;
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

int lsh_planes_padded(int L, int k) { return ((L * k + 31) / 32) * 32; }

size_t lsh_hash_smem(int P) { return hash_smem_bytes(P); }

cudaError_t launch_lsh_hash(const CUtensorMap& xmap, const CUtensorMap& pmap, int n, int P, int L, int k,
                            uint32_t* codes, float* z, int* err, int num_sms, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const size_t smem = hash_smem_bytes(P);
    cudaError_t e = cudaFuncSetAttribute(lsh_hash_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    uint32_t slot = 32;
    while (slot < static_cast<uint32_t>(P)) slot <<= 1;
    const int nbuf = slot <= 128 ? 4 : 2;  // 512 TMEM columns
    const int tiles = (n + 127) / 128;
    const int grid = tiles < num_sms ? tiles : num_sms;
    lsh_hash_kernel<<<grid, kHThreads, smem, stream>>>(xmap, pmap, n, P, L, k, nbuf, slot, codes, z, err);
    return cudaGetLastError();
}

cudaError_t launch_lsh_buckets(const uint32_t* codes, int n, int L, int shift, int nbins, int* hist, int* start,
                               int* order, uint32_t* ocode, int num_sms, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(int) * static_cast<size_t>(L) * nbins, stream);
    if (e != cudaSuccess) return e;
    if (n <= 0) {
        e = cudaMemsetAsync(start, 0, sizeof(int) * static_cast<size_t>(L) * (nbins + 1), stream);
        return e;
    }
    const int blocks = num_sms * 8;
    lsh_hist_kernel<<<blocks, 256, 0, stream>>>(codes, n, L, shift, nbins, hist);
    lsh_scan_bins_kernel<<<L, 1024, 0, stream>>>(hist, nbins, start);
    lsh_scatter_kernel<<<blocks, 256, 0, stream>>>(codes, n, L, shift, nbins, start, hist, order, ocode);
    return cudaGetLastError();
}

cudaError_t launch_lsh_scan(const uint8_t* q, const uint8_t* r, int q_n, int r_n, int L, int probes, int shift,
                            int nbins, const uint32_t* qcodes, const int* start, const int* order,
                            const uint32_t* ocode, float thr, int ratio, float dist_scale, uint32_t* matches,
                            uint32_t* counts, int32_t* nn_idx, float* nn_dist, cudaStream_t stream) {
    if (q_n <= 0) return cudaSuccess;
    const long long blocks = (static_cast<long long>(q_n) * 32 + kScanThreads - 1) / kScanThreads;
    lsh_scan_kernel<<<static_cast<unsigned>(blocks), kScanThreads, 0, stream>>>(
        q, r, q_n, r_n, L, probes, shift, nbins, qcodes, start, order, ocode, thr, ratio, dist_scale, matches, counts,
        nn_idx, nn_dist);
    return cudaGetLastError();
}

}  // namespace sift
