// Exact 2-NN over 128-d descriptors: shared declarations between the kernels
// (exact2nn.cu) and the host entry points (api.cu).
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace sift {

constexpr int kDim = 128;            // descriptor length (elements)
constexpr int kBM = 128;             // queries per tile = TMEM lanes = MMA M
constexpr int kQT = 4;               // query tiles held by one CTA at a time
constexpr int kBN = 128;             // base rows per unit = MMA N
constexpr int kStages = 8;           // base-tile ring depth
constexpr int kEpiWarps = 4 * kQT;   // one epilogue warp per (query tile, TMEM lane quarter)
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr int kTmemCols = kQT * kBN; // one accumulator slot of kBN columns per query tile
constexpr int32_t kKeyPad = 1 << 30; // ranking key of padding rows (never a real key)
constexpr int32_t kFoldMax = 30 * 128 * 255 + 254;  // largest folded half-norm (norms up to ~1.96e6 fold exactly)
constexpr int kFoldHalfBytes = 2048;                // folding digits of 64 base rows (32 s8 each)
constexpr int kRecInts = 160;        // per-base-tile record: 128 norms, 16 8-row minima, pad

// Distance definitions of the exact path.
enum Metric : int {
    kMetricL2 = 0,   // full squared Euclidean distance (host_brute / device_brute)
    kMetricDot = 1,  // -2 q.r (the ranking of cublas_2nn_f / cublas_2nn_sift)
};

// Device error codes written by bounded waits (first one wins).
enum DeviceError : int {
    kErrNone = 0,
    kErrWaitProducer = 1,
    kErrWaitMmaFull = 2,
    kErrWaitMmaTmem = 3,
    kErrWaitEpilogue = 4,
    kErrWaitQuery = 5,
    kErrWaitDrain = 6,
    kErrWaitProbe = 7,  // the fault-injection probe (faults.cu) let its wait expire
};

// Work decomposition of one exact search. A "unit" is (query group g, base
// tile j); units are numbered w = g * base_tiles + j and every CTA of the
// persistent grid owns the contiguous range [w0(c), w0(c+1)), w0(c) =
// floor(c * W / G). cta_of(w) = floor(((w + 1) * G - 1) / W) inverts that.
struct ExactPlan {
    int q_n, r_n;
    int q_tiles, q_groups, q_pad;   // q_pad = q_tiles * kBM
    int base_tiles, r_pad;          // r_pad = base_tiles * kBN
    long long units;                // q_groups * base_tiles
    int grid;                       // persistent CTAs (CTA pairs for the pair kernel)
    int max_splits;                 // max CTAs covering one query group
    int parts;                      // partial top-2 lists per (split, query): column slices
};

__host__ __device__ inline long long plan_w0(long long c, long long W, long long G) { return (c * W) / G; }
__host__ __device__ inline int plan_cta_of(long long w, long long W, long long G) {
    return static_cast<int>(((w + 1) * G - 1) / W);
}

// One (query set, base set) problem of a batch searched by one launch of the
// CTA-pair kernels. Query sets are consecutive row ranges of one query tensor
// (a_off = rows of the problems before it); base sets are any row ranges of
// one base tensor. Units of problem p: groups x tiles, numbered from u_begin;
// its base-tile records start at rec_off. A single search is the batch of one
// problem {0, q_n, 0, r_n, 0, q_groups, base_tiles, 0, 0}. idx_base is added
// to every base index the kernel reports (0 for batches, whose indices are
// local to the problem; the first row of a chunk when one base is searched
// chunk by chunk).
struct WorkItem {
    int a_off, n_a;
    int b_off, n_b;
    long long u_begin;
    int groups, tiles;
    int rec_off;
    int idx_base;
};
static_assert(sizeof(WorkItem) == 40, "WorkItem layout");

// Batch plan: items[] in device memory, plan.units = sum of all units,
// plan.q_pad = query capacity (>= total query rows, multiple of kBM),
// plan.max_splits over every query group of every problem.
struct BatchPlan {
    ExactPlan plan;
    const WorkItem* items;   // device
    int n_items;
    int total_tiles;         // records
    int group_rows;          // queries per query group
};

// Builds the work items of a batch on the host. n_a[p], n_b[p], b_off[p]:
// sizes and base-row offsets of the problems (a_off is the sum of the n_a
// before p); group_rows: queries per group (512 or 256). Returns total units.
long long make_batch_items(int n_items, const int* n_a, const int* n_b, const int* b_off, int group_rows,
                           WorkItem* items, int* total_tiles, int* total_queries);
// The plan of a batch: units, grid, q_pad (query capacity) and max_splits over
// every query group of every problem.
ExactPlan make_batch_plan(const WorkItem* items, int n_items, long long units, int total_queries, int num_workers,
                          int parts);

// num_workers: persistent CTAs (or CTA pairs); parts: partial top-2 lists
// each worker writes per query (one per disjoint column slice it scans).
// group_tiles: 128-row query tiles per query group (kQT: groups of 512 rows
// for the u8 / FP16 kernels; 2: groups of 256 for the general-float kernel).
ExactPlan make_exact_plan(int q_n, int r_n, int num_workers, int parts, int group_tiles = kQT);

// ---- general (non-integer) float / half descriptors
// Keys of the float path are floats mapped to int32 so that signed integer
// order is float order (the integer top-2, shared bounds and merge machinery
// then apply unchanged): non-negative floats keep their bit pattern, negative
// ones have their magnitude bits flipped. -0.0 is folded into +0.0.
__device__ __forceinline__ int32_t float_key(float x) {
    const int32_t i = __float_as_int(x + 0.0f);
    return i >= 0 ? i : (i ^ 0x7fffffff);
}
__device__ __forceinline__ float key_float(int32_t k) { return __int_as_float(k >= 0 ? k : (k ^ 0x7fffffff)); }
constexpr float kFloatKeyPad = 3.0e38f;  // norm of padding rows (never a real key)

// Squared norms (float bit patterns) of n float or half rows times mul, laid
// out as launch_row_norms_u8's outputs (norm / rec / thresh, each optional).
cudaError_t launch_row_norms_float(const void* x, bool half, int n, int n_pad, float mul, int metric, int32_t* norm,
                                   int32_t* rec, int32_t* thresh, cudaStream_t stream);
// The CTA-pair search on FP16 rows with float keys: query and base rows are
// [hi | lo] split rows of 256 halves (qmap / bmap_half: dims {256, rows}, box
// {64, 128 / 64}) when has_lo, else plain FP16 rows of 128 halves (the lo
// products are skipped). dot = hi.hi' + hi.lo' + lo.hi' in f32 (kind::f16).
// Query groups of 256 rows (plan made with group_tiles = 2).
cudaError_t launch_exact2nn_float_pair(const CUtensorMap& qmap, const CUtensorMap& bmap_half, const int32_t* brec,
                                       const ExactPlan& plan, int4* partial, int32_t* thresh, int* err, bool has_lo,
                                       cudaStream_t stream);
// Merge of the float path (float keys, float query norms); group_rows = 256.
cudaError_t launch_merge2nn_float(const int4* partial, const ExactPlan& plan, int group_rows, const int32_t* qnorm,
                                  int metric, float threshold, float dist_scale, uint32_t* matches, float4* sorted,
                                  int32_t* nn_idx, float* nn_dist, cudaStream_t stream);

// Per-row squared norms of u8 descriptors (or zeros for kMetricDot), padded
// to n_pad rows (a multiple of kBN) with kKeyPad. Outputs (each optional):
//   norm[n_pad]                       plain per-row norms
//   rec[n_pad / kBN][kRecInts]        per base tile of kBN rows: the 128 norms
//                                     and the 16 minima over 8-row groups
//   thresh[n_pad]                     set to INT_MAX (the per-query shared
//                                     pruning bound of the search kernel)
cudaError_t launch_row_norms_u8(const uint8_t* x, int n, int n_pad, int metric, int32_t* norm, int32_t* rec,
                                int32_t* thresh, cudaStream_t stream);
// Records of the fold variant: residuals |b|^2 - 2 c (c = the folded
// half-norm) in place of the norms, their 8- and 16-row minima, and the
// folding digits of every row, n_pad / kBN tiles x 2 x kFoldHalfBytes bytes.
cudaError_t launch_fold_records_u8(const uint8_t* x, int n, int n_pad, int metric, int32_t* rec, uint32_t* fold,
                                   cudaStream_t stream);
// The same for FP16 rows whose values times mul (a power of two) are
// integers in [0, 255].
cudaError_t launch_row_norms_f16(const void* x, int n, int n_pad, float mul, int metric, int32_t* norm, int32_t* rec,
                                 int32_t* thresh, cudaStream_t stream);

// The fused GEMM + top-2 kernel. partial: [max_splits][parts][q_pad] int4
// {key1, idx1, key2, idx2} with key = norm(b) - 2 q.b. brec: base records
// (see launch_row_norms_u8). thresh: [q_pad] per-query upper bounds of the
// second-best key shared by the CTAs that split one query group.
cudaError_t launch_exact2nn_u8(const CUtensorMap& qmap, const CUtensorMap& bmap, const int32_t* brec,
                               const ExactPlan& plan, int4* partial, int32_t* thresh, int* err, cudaStream_t stream);

// The same search on CTA pairs (tcgen05 cta_group::2, exact2nn_pair.cu).
// plan.grid counts pairs; bmap_half must use a box of kBN / 2 rows.
cudaError_t launch_exact2nn_u8_pair(const CUtensorMap& qmap, const CUtensorMap& bmap_half, const int32_t* brec,
                                    const ExactPlan& plan, int4* partial, int32_t* thresh, int* err,
                                    cudaStream_t stream);
// The same kernel over a batch (items in device memory). qpt: query tiles per
// CTA (2: query groups of 512 rows, 1: groups of 256 rows; the items must be
// made with the same group size); qbuf: query buffers (1 or 2). Shapes built:
// (2, 1), (2, 2), (1, 2).
cudaError_t launch_exact2nn_u8_pair_batch(const CUtensorMap& qmap, const CUtensorMap& bmap_half, const int32_t* brec,
                                          const BatchPlan& bp, int4* partial, int32_t* thresh, int* err, int qpt,
                                          int qbuf, cudaStream_t stream);
// One search split over base chunks (launched chunk by chunk while later
// chunks are still being copied in): chunk c's partial lists start at
// partial + c * slot_stride, laid out by its own plan (W, G, tiles); indices
// in them are global base rows.
constexpr int kMaxChunks = 16;
struct ChunkSet {
    int n;
    int r_n;
    int parts;
    int q_pad;
    long long slot_stride;
    long long W[kMaxChunks];
    int G[kMaxChunks];
    int tiles[kMaxChunks];
};
// The fold variant of launch_exact2nn_u8_pair: brec from launch_fold_records_u8
// (residual records) and fmap a 2-D u8 tensor map of its folding digits
// (rows of 256 bytes, box 256 x 8: one half tile).
cudaError_t launch_exact2nn_u8fold_pair(const CUtensorMap& qmap, const CUtensorMap& bmap_half,
                                        const CUtensorMap& fmap, const int32_t* brec, const ExactPlan& plan,
                                        int4* partial, int32_t* thresh, int* err, cudaStream_t stream);
// The fold variant over one explicit work item (the item's rec_off indexes
// both the residual records and the folding digits).
cudaError_t launch_exact2nn_u8fold_pair_item(const CUtensorMap& qmap, const CUtensorMap& bmap_half,
                                             const CUtensorMap& fmap, const int32_t* brec, const ExactPlan& plan,
                                             const WorkItem& item, int4* partial, int32_t* thresh, int* err,
                                             cudaStream_t stream);
// The pair kernel over one explicit work item (a chunk of the base).
cudaError_t launch_exact2nn_u8_pair_item(const CUtensorMap& qmap, const CUtensorMap& bmap_half, const int32_t* brec,
                                         const ExactPlan& plan, const WorkItem& item, int4* partial, int32_t* thresh,
                                         int* err, cudaStream_t stream);
cudaError_t launch_merge2nn_chunks(const int4* partial, const ChunkSet& cs, int q_n, const int32_t* qnorm, int metric,
                                   float threshold, float dist_scale, uint32_t* matches, float4* sorted,
                                   int32_t* nn_idx, float* nn_dist, cudaStream_t stream);

// Base-tile records of every problem of a batch (rows of base set p past
// n_b[p] are padding), total_tiles records.
cudaError_t launch_batch_records(const uint8_t* base, int base_rows, const BatchPlan& bp, int metric, int32_t* rec,
                                 cudaStream_t stream);
// Merge for a batch: query row q belongs to the problem whose range holds it;
// indices are local to the problem's base set.
cudaError_t launch_merge2nn_batch(const int4* partial, const BatchPlan& bp, int total_queries, const int32_t* qnorm,
                                  int metric, float threshold, float dist_scale, uint32_t* matches, float4* sorted,
                                  int32_t* nn_idx, float* nn_dist, cudaStream_t stream);
// FP16 rows (bmap_half / qmap: half tensor maps with boxes of 64 elements):
// values are integers times 2^-s and dscale = 2^(2s) turns the f32 dot
// products back into integers (brec built from the same integers).
cudaError_t launch_exact2nn_f16_pair(const CUtensorMap& qmap, const CUtensorMap& bmap_half, const int32_t* brec,
                                     const ExactPlan& plan, int4* partial, int32_t* thresh, int* err, float dscale,
                                     cudaStream_t stream);
size_t exact2nn_pair_smem_bytes();

// Merge of the per-CTA partial top-2 lists, distances, ratio test and output.
// Any output pointer may be null.
//   matches[q]   idx1 if the ratio test passes else UINT32_MAX
//   sorted[q]    {d1, d2, i1, i2} as floats (FLT_MAX where absent)
//   nn_idx[2q..] int32 indices (-1 where absent)
//   nn_dist[2q..] float distances (FLT_MAX where absent)
// dist_scale multiplies every distance (2^-2s for inputs that were integers
// times 2^-s; 1 otherwise) before the ratio test and the outputs.
cudaError_t launch_merge2nn(const int4* partial, const ExactPlan& plan, const int32_t* qnorm, int metric,
                            float threshold, float dist_scale, uint32_t* matches, float4* sorted, int32_t* nn_idx,
                            float* nn_dist, cudaStream_t stream);

size_t exact2nn_smem_bytes();

}  // namespace sift
