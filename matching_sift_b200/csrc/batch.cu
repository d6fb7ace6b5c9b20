// Batched exact 2-NN: many (query set, base set) problems -- e.g. the two
// keypoint sets of many image pairs, of uneven sizes -- in ONE persistent
// launch of the CTA-pair kernel driven by a device work list (WorkItem per
// problem). The reference matches one image pair per call (cublas_2nn_sift,
// src/knn_brute.cu:24; its benchmark loops over calls, src/test.cu:194-216);
// this has no counterpart there.
//
// Sequence per batch (one stream): query norms + bounds, base-tile records of
// every problem, the search kernel over all units, the merge. A plan
// (sift_batch_plan) owns its device memory, picks the kernel shape with a
// small autotuner (times each shape on the batch itself) and captures the
// sequence in a CUDA graph, so a repeated batch of the same sizes (new
// descriptor values in the same buffers) costs one graph launch.
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>
#include "api_internal.h"
#include "context.h"
#include "exact2nn.cuh"

struct sift_batch_plan {
    int dev = 0;
    sift::detail::DeviceCtx* ctx = nullptr;
    int shape = 0;
    float tuned_ms[3] = {-1.f, -1.f, -1.f};
    sift::WorkItem* d_items = nullptr;
    char* mem = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace sift {
namespace {

using detail::DeviceCtx;

struct Shape {
    int qpt, qbuf;
};
// Kernel shapes the autotuner chooses from: query tiles per CTA (groups of
// 512 or 256 queries) and query buffers (2: next group's queries load during
// the current group's MMAs).
constexpr Shape kShapes[3] = {{2, 1}, {2, 2}, {1, 2}};
constexpr int kNumShapes = 3;
constexpr int kDefaultShape = 1;

std::mutex g_tune_mu;
std::map<std::array<long long, 4>, int> g_tune_cache;

struct Built {
    std::vector<WorkItem> items;
    long long units = 0;
    int total_tiles = 0, total_q = 0, group_rows = 0;
    ExactPlan plan{};
};

int build(const sift_pair* pairs, int n_pairs, uint32_t r_rows, int qpt, int workers, Built& b) {
    if (n_pairs < 0 || (n_pairs > 0 && !pairs)) return SIFT_ERR_INVALID_ARG;
    std::vector<int> na(n_pairs), nb(n_pairs), off(n_pairs);
    long long tq = 0;
    for (int p = 0; p < n_pairs; ++p) {
        const sift_pair& s = pairs[p];
        if (static_cast<uint64_t>(s.r_off) + s.n_r > r_rows) return SIFT_ERR_INVALID_ARG;
        tq += s.n_q;
        if (tq > 0x7fffffffLL - 1024 || s.n_r > 0x7fffffffu - 1024) return SIFT_ERR_INVALID_ARG;
        na[p] = static_cast<int>(s.n_q);
        nb[p] = static_cast<int>(s.n_r);
        off[p] = static_cast<int>(s.r_off);
    }
    if (r_rows > 0x7fffffffu - 1024) return SIFT_ERR_INVALID_ARG;
    b.group_rows = 2 * qpt * kBM;
    b.items.resize(n_pairs);
    b.units = make_batch_items(n_pairs, na.data(), nb.data(), off.data(), b.group_rows, b.items.data(),
                               &b.total_tiles, &b.total_q);
    b.plan = make_batch_plan(b.items.data(), n_pairs, b.units, b.total_q, workers, 2);
    return SIFT_OK;
}

std::array<long long, 4> signature(const Built& b) {
    return {static_cast<long long>(b.items.size()), b.total_q, b.units, b.total_tiles};
}

struct Buffers {
    WorkItem* items = nullptr;
    int32_t* rec = nullptr;
    int32_t* qnorm = nullptr;
    int32_t* thresh = nullptr;
    int4* partial = nullptr;
};

size_t partial_bytes(const Built& b) {
    return static_cast<size_t>(b.plan.max_splits) * b.plan.parts * b.plan.q_pad * sizeof(int4);
}

// Layout of a batch's scratch for the largest of `builds`.
struct BatchLayout {
    size_t o_items, o_rec, o_qn, o_thr, o_part, bytes;
};
BatchLayout layout_for(const Built* builds, int n) {
    size_t part = 0;
    for (int k = 0; k < n; ++k) part = std::max(part, partial_bytes(builds[k]));
    const Built& b = builds[0];
    detail::Layout L;
    BatchLayout o{};
    o.o_items = L.take(sizeof(WorkItem) * (b.items.size() + 1));
    o.o_rec = L.take(static_cast<size_t>(b.total_tiles) * kRecInts * 4 + 16);
    o.o_qn = L.take(static_cast<size_t>(b.plan.q_pad) * 4 + 16);
    o.o_thr = L.take(static_cast<size_t>(b.plan.q_pad) * 4 + 16);
    o.o_part = L.take(part + 16);
    o.bytes = L.off;
    return o;
}
Buffers buffers_at(char* base, const BatchLayout& o) {
    Buffers m;
    m.items = reinterpret_cast<WorkItem*>(base + o.o_items);
    m.rec = reinterpret_cast<int32_t*>(base + o.o_rec);
    m.qnorm = reinterpret_cast<int32_t*>(base + o.o_qn);
    m.thresh = reinterpret_cast<int32_t*>(base + o.o_thr);
    m.partial = reinterpret_cast<int4*>(base + o.o_part);
    return m;
}

int enqueue(DeviceCtx& c, const uint8_t* q, const uint8_t* r, uint32_t r_rows, const Built& b, const Buffers& m,
            Shape sh, float thr, uint32_t* matches, int32_t* nn_idx, float* nn_dist, cudaStream_t st) {
    if (b.total_q == 0) return SIFT_OK;
    BatchPlan bp{b.plan, m.items, static_cast<int>(b.items.size()), b.total_tiles, b.group_rows};
    SIFT_CUDA(launch_row_norms_u8(q, b.total_q, b.plan.q_pad, kMetricL2, m.qnorm, nullptr, m.thresh, st));
    int launches = 2;
    if (b.units > 0) {
        SIFT_CUDA(launch_batch_records(r, static_cast<int>(r_rows), bp, kMetricL2, m.rec, st));
        CUtensorMap qmap, rmap;
        SIFT_TRY(detail::encode_u8_rows(&qmap, q, static_cast<uint64_t>(b.total_q), kBM));
        SIFT_TRY(detail::encode_u8_rows(&rmap, r, r_rows, kBN / 2));
        SIFT_CUDA(launch_exact2nn_u8_pair_batch(qmap, rmap, m.rec, bp, m.partial, m.thresh, c.d_status, sh.qpt,
                                                sh.qbuf, st));
        launches += 2;
    }
    SIFT_CUDA(launch_merge2nn_batch(m.partial, bp, b.total_q, m.qnorm, kMetricL2, thr, 1.0f, matches, nullptr, nn_idx,
                                    nn_dist, st));
    detail::g_launches += launches;
    return SIFT_OK;
}

int check_io(const uint8_t* q, const uint8_t* r, uint32_t r_rows, long long total_q, uint32_t* matches,
             int32_t* nn_idx, float* nn_dist) {
    if (total_q > 0 && (!q || (reinterpret_cast<uintptr_t>(q) & 15) || !detail::is_device_accessible(q)))
        return SIFT_ERR_INVALID_ARG;
    if (r_rows > 0 && (!r || (reinterpret_cast<uintptr_t>(r) & 15) || !detail::is_device_accessible(r)))
        return SIFT_ERR_INVALID_ARG;
    for (const void* o : {static_cast<const void*>(matches), static_cast<const void*>(nn_idx),
                          static_cast<const void*>(nn_dist)})
        if (o && total_q > 0 && !detail::is_device_accessible(o)) return SIFT_ERR_INVALID_ARG;
    return SIFT_OK;
}

int cached_shape(const Built& b) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(signature(b));
    return it == g_tune_cache.end() ? kDefaultShape : it->second;
}

}  // namespace

int match_batch(const uint8_t* q, const uint8_t* r, uint32_t r_rows, const sift_pair* pairs, int n_pairs,
                float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist, void* stream) {
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    DeviceCtx& c = *cp;
    Built probe;
    SIFT_TRY(build(pairs, n_pairs, r_rows, 2, c.num_sms / 2, probe));
    const int shape = cached_shape(probe);
    Built b;
    SIFT_TRY(build(pairs, n_pairs, r_rows, kShapes[shape].qpt, c.num_sms / 2, b));
    SIFT_TRY(check_io(q, r, r_rows, b.total_q, matches, nn_idx, nn_dist));
    if (b.total_q == 0) return SIFT_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    detail::ArenaLock lk(c, st);
    const BatchLayout o = layout_for(&b, 1);
    SIFT_TRY(detail::ensure_arena(c, o.bytes));
    const Buffers m = buffers_at(c.arena, o);
    if (!b.items.empty())
        SIFT_CUDA(cudaMemcpyAsync(m.items, b.items.data(), sizeof(WorkItem) * b.items.size(), cudaMemcpyHostToDevice,
                                  st));
    return enqueue(c, q, r, r_rows, b, m, kShapes[shape], threshold, matches, nn_idx, nn_dist, st);
}

// Largest p with off[p] <= i over a non-decreasing off[0..n) (empty
// problems share the offset of the next one, so p is the problem owning row i).
__device__ __forceinline__ int owner_of(const int* __restrict__ off, int n, int i) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Rows of every problem's base set, in problem order, as one query array of
// the reverse search: row k of the output is row k - b_row[p] of set p.
__global__ void gather_sets_kernel(const uint8_t* __restrict__ b, const int* __restrict__ b_row,
                                   const int* __restrict__ r_off, int n_pairs, int total, uint8_t* __restrict__ out) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int k = static_cast<int>(t >> 3), part = static_cast<int>(t & 7);
    if (k >= total) return;
    const int p = owner_of(b_row, n_pairs, k);
    const size_t src = static_cast<size_t>(r_off[p]) + (k - b_row[p]);
    reinterpret_cast<uint4*>(out + static_cast<size_t>(k) * kDim)[part] =
        reinterpret_cast<const uint4*>(b + src * kDim)[part];
}

// Mutual check: row i of a (problem p, local row li = i - a_off[p]) keeps its
// nearest base row j (local to set p) when the reverse search of row j of set
// p found li as its nearest row, and (ratio) the forward ratio test passed.
__global__ void cross_check_kernel(const int32_t* __restrict__ nn_fwd, const uint32_t* __restrict__ m_fwd,
                                   const int32_t* __restrict__ nn_rev, const int* __restrict__ a_off,
                                   const int* __restrict__ b_row, int n_pairs, int total_a, int ratio,
                                   uint32_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total_a) return;
    const int p = owner_of(a_off, n_pairs, i);
    const int j = nn_fwd[2 * static_cast<size_t>(i)];
    uint32_t res = 0xffffffffu;
    if (j >= 0 && (!ratio || m_fwd[i] != 0xffffffffu) &&
        nn_rev[2 * (static_cast<size_t>(b_row[p]) + j)] == i - a_off[p])
        res = static_cast<uint32_t>(j);
    out[i] = res;
}

int match_mutual_batch(const uint8_t* a, const uint8_t* b, uint32_t b_rows, const sift_pair* pairs, int n_pairs,
                       float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist, void* stream) {
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    DeviceCtx& c = *cp;
    if (!matches || n_pairs < 0 || (n_pairs > 0 && !pairs)) return SIFT_ERR_INVALID_ARG;
    // Reverse problems: set p of b searched against rows of problem p of a.
    std::vector<sift_pair> rev(n_pairs);
    std::vector<int> a_off(n_pairs + 1), b_row(n_pairs), r_off(n_pairs);
    long long arow = 0, brow = 0;
    bool contiguous = true;
    for (int p = 0; p < n_pairs; ++p) {
        if (brow > 0x7fffffffLL - 1024 || arow > 0x7fffffffLL - 1024) return SIFT_ERR_INVALID_ARG;
        rev[p] = sift_pair{pairs[p].n_r, pairs[p].n_q, static_cast<uint32_t>(arow)};
        a_off[p] = static_cast<int>(arow);
        b_row[p] = static_cast<int>(brow);
        r_off[p] = static_cast<int>(pairs[p].r_off);
        if (pairs[p].r_off != brow) contiguous = false;
        arow += pairs[p].n_q;
        brow += pairs[p].n_r;
    }
    if (brow > 0x7fffffffLL - 1024 || arow > 0x7fffffffLL - 1024) return SIFT_ERR_INVALID_ARG;
    a_off[n_pairs] = static_cast<int>(arow);
    const int workers = c.num_sms / 2;
    Built probe_f, bf, probe_r, br;
    SIFT_TRY(build(pairs, n_pairs, b_rows, 2, workers, probe_f));
    const int shape_f = cached_shape(probe_f);
    SIFT_TRY(build(pairs, n_pairs, b_rows, kShapes[shape_f].qpt, workers, bf));
    SIFT_TRY(build(rev.data(), n_pairs, static_cast<uint32_t>(arow), 2, workers, probe_r));
    const int shape_r = cached_shape(probe_r);
    SIFT_TRY(build(rev.data(), n_pairs, static_cast<uint32_t>(arow), kShapes[shape_r].qpt, workers, br));
    SIFT_TRY(check_io(a, b, b_rows, bf.total_q, matches, nn_idx, nn_dist));
    if (bf.total_q == 0) return SIFT_OK;
    const int total_a = bf.total_q, total_b = static_cast<int>(brow);

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    detail::ArenaLock lk(c, st);
    const BatchLayout lf = layout_for(&bf, 1), lr = layout_for(&br, 1);
    detail::Layout L;
    const size_t o_f = L.take(lf.bytes), o_r = L.take(lr.bytes);
    const size_t o_nnf = L.take(static_cast<size_t>(total_a) * 8);
    const size_t o_mf = L.take(static_cast<size_t>(total_a) * 4);
    const size_t o_nnr = L.take(static_cast<size_t>(total_b) * 8 + 16);
    const size_t o_rows = L.take(contiguous ? 0 : static_cast<size_t>(total_b) * kDim + 16);
    const size_t o_off = L.take(sizeof(int) * (3 * static_cast<size_t>(n_pairs) + 1));
    SIFT_TRY(detail::ensure_arena(c, L.off));
    char* A = c.arena;
    const Buffers mf = buffers_at(A + o_f, lf), mr = buffers_at(A + o_r, lr);
    int32_t* nn_f = nn_idx ? nn_idx : reinterpret_cast<int32_t*>(A + o_nnf);
    uint32_t* m_f = reinterpret_cast<uint32_t*>(A + o_mf);
    int32_t* nn_r = reinterpret_cast<int32_t*>(A + o_nnr);
    int* d_aoff = reinterpret_cast<int*>(A + o_off);
    int* d_brow = d_aoff + n_pairs + 1;
    int* d_roff = d_brow + n_pairs;
    std::vector<int> offs(a_off);
    offs.insert(offs.end(), b_row.begin(), b_row.end());
    offs.insert(offs.end(), r_off.begin(), r_off.end());
    SIFT_CUDA(cudaMemcpyAsync(d_aoff, offs.data(), sizeof(int) * offs.size(), cudaMemcpyHostToDevice, st));
    if (!bf.items.empty())
        SIFT_CUDA(cudaMemcpyAsync(mf.items, bf.items.data(), sizeof(WorkItem) * bf.items.size(),
                                  cudaMemcpyHostToDevice, st));
    if (!br.items.empty())
        SIFT_CUDA(cudaMemcpyAsync(mr.items, br.items.data(), sizeof(WorkItem) * br.items.size(),
                                  cudaMemcpyHostToDevice, st));
    const uint8_t* qrev = b;
    if (!contiguous && total_b > 0) {
        uint8_t* rows = reinterpret_cast<uint8_t*>(A + o_rows);
        gather_sets_kernel<<<static_cast<unsigned>((static_cast<long long>(total_b) * 8 + 255) / 256), 256, 0, st>>>(
            b, d_brow, d_roff, n_pairs, total_b, rows);
        SIFT_CUDA(cudaGetLastError());
        ++detail::g_launches;
        qrev = rows;
    }
    SIFT_TRY(enqueue(c, a, b, b_rows, bf, mf, kShapes[shape_f], threshold, m_f, nn_f, nn_dist, st));
    SIFT_TRY(enqueue(c, qrev, a, static_cast<uint32_t>(total_a), br, mr, kShapes[shape_r], 0.0f, nullptr, nn_r,
                     nullptr, st));
    cross_check_kernel<<<(total_a + 255) / 256, 256, 0, st>>>(nn_f, m_f, nn_r, d_aoff, d_brow, n_pairs, total_a,
                                                               threshold > 0.0f ? 1 : 0, matches);
    SIFT_CUDA(cudaGetLastError());
    ++detail::g_launches;
    return SIFT_OK;
}

// ---- match lists for geometric verification ---------------------------
// Deterministic stream compaction of the rows with a match, 1024 rows per
// block: block counts, one scan of them, then each block's rows placed by
// warp ballots. The lists come out grouped by problem, rows in order.
constexpr int kCompactRows = 1024;

__global__ void __launch_bounds__(kCompactRows) count_matches_kernel(const uint32_t* __restrict__ matches, int rows,
                                                                       int* __restrict__ block_counts) {
    const int i = blockIdx.x * kCompactRows + threadIdx.x;
    const bool v = i < rows && matches[i] != 0xffffffffu;
    const int c = __syncthreads_count(v);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = c;
}

// Exclusive prefix of the block counts (one block, chunks of 1024 with a
// running carry); offsets[n_blocks] = total.
__global__ void __launch_bounds__(1024) scan_counts_kernel(const int* __restrict__ counts, int n_blocks,
                                                           int* __restrict__ offsets) {
    __shared__ int warp_sum[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n_blocks; base += 1024) {
        const int i = base + threadIdx.x;
        const int c = i < n_blocks ? counts[i] : 0;
        int x = c;  // inclusive warp scan
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int w = warp_sum[lane];
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sum[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        const int before = carry + (warp > 0 ? warp_sum[warp - 1] : 0) + x - c;
        if (i < n_blocks) offsets[i] = before;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_sum[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) offsets[n_blocks] = carry;
}

// Position of row i among the matched rows: its block's offset plus the
// matched rows before it in the block (ballots).
__global__ void __launch_bounds__(kCompactRows) scatter_matches_kernel(
    const uint32_t* __restrict__ matches, const float* __restrict__ nn_dist, int rows, const int* __restrict__ offsets,
    const int* __restrict__ a_off, int n_pairs, sift_match* __restrict__ out, uint32_t capacity) {
    __shared__ int warp_count[32];
    const int i = blockIdx.x * kCompactRows + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool v = i < rows && matches[i] != 0xffffffffu;
    const unsigned bal = __ballot_sync(0xffffffffu, v);
    if (lane == 0) warp_count[warp] = __popc(bal);
    __syncthreads();
    if (!v) return;
    int pos = offsets[blockIdx.x] + __popc(bal & ((1u << lane) - 1u));
    for (int w = 0; w < warp; ++w) pos += warp_count[w];
    if (static_cast<uint32_t>(pos) >= capacity) return;
    const int p = owner_of(a_off, n_pairs, i);
    sift_match m;
    m.pair = static_cast<uint32_t>(p);
    m.a = static_cast<uint32_t>(i - a_off[p]);
    m.b = matches[i];
    m.d1 = nn_dist ? nn_dist[2 * static_cast<size_t>(i)] : 0.0f;
    m.d2 = nn_dist ? nn_dist[2 * static_cast<size_t>(i) + 1] : 0.0f;
    out[pos] = m;
}

// pair_offsets[p] = matched rows before problem p's first row (one warp per
// problem: the block offset plus ballots over the block's earlier rows).
__global__ void pair_offsets_kernel(const uint32_t* __restrict__ matches, const int* __restrict__ offsets,
                                    const int* __restrict__ a_off, int n_pairs, int n_blocks,
                                    uint32_t* __restrict__ pair_offsets) {
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p > n_pairs) return;
    if (p == n_pairs) {
        if (lane == 0) pair_offsets[p] = static_cast<uint32_t>(offsets[n_blocks]);
        return;
    }
    const int row = a_off[p];
    const int blk = row / kCompactRows;
    if (blk >= n_blocks) {  // no rows from here on
        if (lane == 0) pair_offsets[p] = static_cast<uint32_t>(offsets[n_blocks]);
        return;
    }
    int before = 0;
    for (int r0 = blk * kCompactRows; r0 < row; r0 += 32) {
        const int r = r0 + lane;
        before += __popc(__ballot_sync(0xffffffffu, r < row && matches[r] != 0xffffffffu));
    }
    if (lane == 0) pair_offsets[p] = static_cast<uint32_t>(offsets[blk] + before);
}

int compact_matches(const uint32_t* matches, const float* nn_dist, uint32_t rows, const sift_pair* pairs, int n_pairs,
                    sift_match* out, uint32_t capacity, uint32_t* pair_offsets, void* stream) {
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    DeviceCtx& c = *cp;
    if (n_pairs < 0 || (n_pairs > 0 && !pairs) || !pair_offsets || rows > 0x7fffffffu - kCompactRows)
        return SIFT_ERR_INVALID_ARG;
    std::vector<int> a_off(n_pairs + 1);
    long long row = 0;
    for (int p = 0; p < n_pairs; ++p) {
        a_off[p] = static_cast<int>(row);
        row += pairs[p].n_q;
        if (row > static_cast<long long>(rows)) return SIFT_ERR_INVALID_ARG;
    }
    if (row != static_cast<long long>(rows)) return SIFT_ERR_INVALID_ARG;
    a_off[n_pairs] = static_cast<int>(row);
    if (!detail::is_device_accessible(pair_offsets) || (rows > 0 && (!matches || !detail::is_device_accessible(matches))) ||
        (nn_dist && !detail::is_device_accessible(nn_dist)) ||
        (capacity > 0 && (!out || !detail::is_device_accessible(out))))
        return SIFT_ERR_INVALID_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    detail::ArenaLock lk(c, st);
    const int n_blocks = static_cast<int>((rows + kCompactRows - 1) / kCompactRows);
    detail::Layout L;
    const size_t o_cnt = L.take(sizeof(int) * (static_cast<size_t>(n_blocks) + 1));
    const size_t o_off = L.take(sizeof(int) * (static_cast<size_t>(n_blocks) + 1));
    const size_t o_aoff = L.take(sizeof(int) * (static_cast<size_t>(n_pairs) + 1));
    SIFT_TRY(detail::ensure_arena(c, L.off));
    int* d_cnt = reinterpret_cast<int*>(c.arena + o_cnt);
    int* d_off = reinterpret_cast<int*>(c.arena + o_off);
    int* d_aoff = reinterpret_cast<int*>(c.arena + o_aoff);
    SIFT_CUDA(cudaMemcpyAsync(d_aoff, a_off.data(), sizeof(int) * a_off.size(), cudaMemcpyHostToDevice, st));
    if (n_blocks > 0) {
        count_matches_kernel<<<n_blocks, kCompactRows, 0, st>>>(matches, static_cast<int>(rows), d_cnt);
        SIFT_CUDA(cudaGetLastError());
    }
    scan_counts_kernel<<<1, 1024, 0, st>>>(d_cnt, n_blocks, d_off);
    SIFT_CUDA(cudaGetLastError());
    if (n_blocks > 0) {
        scatter_matches_kernel<<<n_blocks, kCompactRows, 0, st>>>(matches, nn_dist, static_cast<int>(rows), d_off,
                                                                  d_aoff, n_pairs, out, capacity);
        SIFT_CUDA(cudaGetLastError());
    }
    const long long threads = 32LL * (n_pairs + 1);
    pair_offsets_kernel<<<static_cast<unsigned>((threads + 255) / 256), 256, 0, st>>>(matches, d_off, d_aoff, n_pairs,
                                                                                     n_blocks, pair_offsets);
    SIFT_CUDA(cudaGetLastError());
    detail::g_launches += 2 + (n_blocks > 0 ? 2 : 0);
    return SIFT_OK;
}

int batch_plan_create(const uint8_t* q, const uint8_t* r, uint32_t r_rows, const sift_pair* pairs, int n_pairs,
                      float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist, int flags,
                      sift_batch_plan** out) {
    if (!out) return SIFT_ERR_INVALID_ARG;
    *out = nullptr;
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    DeviceCtx& c = *cp;
    Built builds[kNumShapes];
    for (int k = 0; k < kNumShapes; ++k)
        SIFT_TRY(build(pairs, n_pairs, r_rows, kShapes[k].qpt, c.num_sms / 2, builds[k]));
    SIFT_TRY(check_io(q, r, r_rows, builds[0].total_q, matches, nn_idx, nn_dist));
    const int forced = (flags >> 4) & 0xf;  // SIFT_BATCH_SHAPE(k) = (k + 1) << 4
    if (forced > kNumShapes) return SIFT_ERR_INVALID_ARG;

    sift_batch_plan* P = new (std::nothrow) sift_batch_plan();
    if (!P) return SIFT_ERR_ALLOC;
    P->dev = dev;
    P->ctx = cp;
    auto fail = [&](int rc) {
        if (P->exec) cudaGraphExecDestroy(P->exec);
        if (P->graph) cudaGraphDestroy(P->graph);
        if (P->mem) cudaFree(P->mem);
        delete P;
        return rc;
    };
    const BatchLayout o = layout_for(builds, kNumShapes);
    if (cudaMalloc(&P->mem, o.bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(SIFT_ERR_ALLOC);
    }
    const Buffers m = buffers_at(P->mem, o);
    cudaStream_t cs = nullptr;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return fail(SIFT_ERR_CUDA);
    auto run_shape = [&](int k) -> int {
        const Built& b = builds[k];
        if (!b.items.empty())
            SIFT_CUDA(cudaMemcpyAsync(m.items, b.items.data(), sizeof(WorkItem) * b.items.size(),
                                      cudaMemcpyHostToDevice, cs));
        return enqueue(c, q, r, r_rows, b, m, kShapes[k], threshold, matches, nn_idx, nn_dist, cs);
    };
    int rc = SIFT_OK;
    int shape = forced > 0 ? forced - 1 : cached_shape(builds[0]);
    if ((flags & SIFT_BATCH_TUNE) && forced == 0 && builds[0].units > 0) {
        // Autotune: each shape once to warm up, then the best of three timed runs.
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = SIFT_ERR_CUDA;
        float best = 0.f;
        for (int k = 0; k < kNumShapes && rc == SIFT_OK; ++k) {
            rc = run_shape(k);
            float t_min = 1e30f;
            for (int rep = 0; rep < 3 && rc == SIFT_OK; ++rep) {
                if (cudaEventRecord(e0, cs) != cudaSuccess) rc = SIFT_ERR_CUDA;
                if (rc == SIFT_OK) rc = run_shape(k);
                float ms = 0.f;
                if (rc == SIFT_OK && (cudaEventRecord(e1, cs) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                                      cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
                    rc = SIFT_ERR_CUDA;
                t_min = std::min(t_min, ms);
            }
            if (rc == SIFT_OK) {
                P->tuned_ms[k] = t_min;
                if (k == 0 || t_min < best) {
                    best = t_min;
                    shape = k;
                }
            }
        }
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (rc == SIFT_OK) {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune_cache[signature(builds[0])] = shape;
        }
    }
    // One plain run of the chosen shape (sets kernel attributes, checks the
    // device status), then the capture.
    if (rc == SIFT_OK) rc = run_shape(shape);
    if (rc == SIFT_OK && cudaStreamSynchronize(cs) != cudaSuccess) rc = SIFT_ERR_CUDA;
    if (rc == SIFT_OK) {
        std::lock_guard<std::mutex> lk(c.mu);
        rc = detail::collect_device_status(c, cs);
    }
    if (rc == SIFT_OK) {
        if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            rc = SIFT_ERR_CUDA;
        } else {
            const int erc = enqueue(c, q, r, r_rows, builds[shape], m, kShapes[shape], threshold, matches, nn_idx,
                                    nn_dist, cs);
            const cudaError_t ce = cudaStreamEndCapture(cs, &P->graph);
            rc = erc != SIFT_OK ? erc : detail::map_cuda(ce);
        }
    }
    if (rc == SIFT_OK && cudaGraphInstantiate(&P->exec, P->graph, 0) != cudaSuccess) rc = SIFT_ERR_CUDA;
    cudaStreamDestroy(cs);
    if (rc != SIFT_OK) {
        cudaGetLastError();
        return fail(rc);
    }
    P->shape = shape;
    *out = P;
    return SIFT_OK;
}

int batch_plan_run(sift_batch_plan* P, void* stream) {
    if (!P || !P->exec) return SIFT_ERR_INVALID_ARG;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != P->dev) return SIFT_ERR_INVALID_ARG;
    SIFT_CUDA(cudaGraphLaunch(P->exec, static_cast<cudaStream_t>(stream)));
    return SIFT_OK;
}

int batch_plan_info(const sift_batch_plan* P, int* qpt, int* qbuf, float* tuned_ms) {
    if (!P) return SIFT_ERR_INVALID_ARG;
    if (qpt) *qpt = kShapes[P->shape].qpt;
    if (qbuf) *qbuf = kShapes[P->shape].qbuf;
    if (tuned_ms) std::memcpy(tuned_ms, P->tuned_ms, sizeof(P->tuned_ms));
    return SIFT_OK;
}

void batch_plan_destroy(sift_batch_plan* P) {
    if (!P) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(P->dev);
    cudaDeviceSynchronize();
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    if (P->mem) cudaFree(P->mem);
    cudaSetDevice(cur);
    delete P;
}

int batch_describe(const sift_pair* pairs, int n_pairs, uint32_t r_rows, int qpt, int workers, long long* out) {
    if (!out || workers < 1 || (qpt != 1 && qpt != 2)) return SIFT_ERR_INVALID_ARG;
    Built b;
    SIFT_TRY(build(pairs, n_pairs, r_rows, qpt, workers, b));
    out[0] = b.units;
    out[1] = b.total_tiles;
    out[2] = b.total_q;
    out[3] = b.plan.max_splits;
    out[4] = b.plan.grid;
    out[5] = b.group_rows;
    return SIFT_OK;
}

}  // namespace sift

extern "C" {

int sift_compact_matches(const uint32_t* matches, const float* nn_dist, uint32_t rows, const sift_pair* pairs,
                         int n_pairs, sift_match* out, uint32_t capacity, uint32_t* pair_offsets, void* stream) {
    return sift::compact_matches(matches, nn_dist, rows, pairs, n_pairs, out, capacity, pair_offsets, stream);
}

int sift2nn_match_mutual_batch(const uint8_t* a, const uint8_t* b, uint32_t b_rows, const sift_pair* pairs,
                               int n_pairs, float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist,
                               void* stream) {
    return sift::match_mutual_batch(a, b, b_rows, pairs, n_pairs, threshold, matches, nn_idx, nn_dist, stream);
}

int sift2nn_match_batch(const uint8_t* q, const uint8_t* r, uint32_t r_rows, const sift_pair* pairs, int n_pairs,
                        float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist, void* stream) {
    return sift::match_batch(q, r, r_rows, pairs, n_pairs, threshold, matches, nn_idx, nn_dist, stream);
}

int sift_batch_plan_create(const uint8_t* q, const uint8_t* r, uint32_t r_rows, const sift_pair* pairs, int n_pairs,
                           float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist, int flags,
                           sift_batch_plan** plan) {
    return sift::batch_plan_create(q, r, r_rows, pairs, n_pairs, threshold, matches, nn_idx, nn_dist, flags, plan);
}

int sift_batch_plan_run(sift_batch_plan* plan, void* stream) { return sift::batch_plan_run(plan, stream); }

int sift_batch_plan_info(const sift_batch_plan* plan, int* qpt, int* qbuf, float* tuned_ms) {
    return sift::batch_plan_info(plan, qpt, qbuf, tuned_ms);
}

void sift_batch_plan_destroy(sift_batch_plan* plan) { sift::batch_plan_destroy(plan); }

int sift_batch_describe(const sift_pair* pairs, int n_pairs, uint32_t r_rows, int qpt, int workers, long long* out) {
    return sift::batch_describe(pairs, n_pairs, r_rows, qpt, workers, out);
}

}  // extern "C"
