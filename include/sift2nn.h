/*
 * sift2nn.h - C ABI of the B200-native 2-NN SIFT descriptor matcher.
 *
 * Part 1 keeps the reference's entry points, with the reference's names and
 * argument lists, so existing callers (C via this header, cgo, ctypes, or C++
 * through the mangled forwarders also exported by libsift2nn.so) switch by
 * relinking. Part 2 is the native interface: u8 descriptors, explicit
 * streams, all four outputs.
 *
 * Conventions shared by every entry point
 *  - Descriptors are row-major [n][128] (des_t_f = float[128] in the
 *    reference, include/knn_brute.h:5; des_t_h2 = __half2[64], :6).
 *  - Distances are squared Euclidean unless stated otherwise; nearest and
 *    second-nearest are taken in lexicographic (distance, index) order, so a
 *    tie goes to the lower base index (the order of the reference host_brute,
 *    src/knn_brute.cu:816-831).
 *  - The Lowe ratio test passes when sqrtf(d1) / sqrtf(d2) < threshold in
 *    single precision. For unit-norm inputs this is the reference's
 *    sqrt(d + 2) form of src/knn_brute.cu:430-442, whose d = -2 q.r.
 *  - Results are exact for integer-valued descriptors in [0, 255] (computed
 *    on the tensor cores as u8 x u8 -> s32).
 *  - The library allocates nothing per call after warm-up: scratch lives in a
 *    per-device arena that grows on demand and is reused.
 *  - int-returning functions return SIFT_OK (0) or a negative SIFT_ERR_*;
 *    void compatibility functions record their status for sift_last_status().
 *  - Nothing here falls back to the CPU: without a usable CUDA device every
 *    call returns SIFT_ERR_NO_DEVICE.
 */
#ifndef SIFT2NN_H_
#define SIFT2NN_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SIFT_API __attribute__((visibility("default")))
#else
#define SIFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Input memory types: 0..2 as in the reference (src/knn_brute.cu:15-19,
   src/lsh_h.cu:710-714); 3 and 4 are extensions for u8 descriptors. A host
   pointer given with a device type returns SIFT_ERR_INVALID_ARG. */
enum sift_mem_type {
    SIFT_FLOAT_HOST = 0,   /* float[n][128] in mapped pinned host memory (read zero-copy) */
    SIFT_FLOAT_DEVICE = 1, /* float[n][128] in device memory */
    SIFT_HALF_DEVICE = 2,  /* __half[n][128] in device memory */
    SIFT_U8_DEVICE = 3,    /* uint8[n][128] in device memory (16-byte aligned) */
    SIFT_U8_HOST = 4       /* uint8[n][128] in host memory (pinned is fastest) */
};

/* Metrics of the native interface. */
enum sift_metric {
    SIFT_METRIC_L2 = 0, /* squared Euclidean distance */
    SIFT_METRIC_DOT = 1 /* -2 q.r, the ranking of the reference cublas_2nn_f (src/knn_brute.cu:579-592) */
};

#define SIFT_OK 0
#define SIFT_ERR_INVALID_ARG (-1)
#define SIFT_ERR_CUDA (-2)
#define SIFT_ERR_NOT_INTEGER (-3)
#define SIFT_ERR_DEVICE_TIMEOUT (-4)
#define SIFT_ERR_NO_DEVICE (-5)
#define SIFT_ERR_UNSUPPORTED (-6)
#define SIFT_ERR_ALLOC (-7)

typedef struct cublasContext* cublasHandle_t; /* accepted and ignored: no cuBLAS inside */
typedef float des_t_f[128];
typedef struct {
    float x, y, z, w;
} sift_float4; /* layout of CUDA float4: {d1, d2, i1, i2} */

/* ---------------------------------------------------------------------
 * Part 1: reference entry points (same names and arguments)
 * ------------------------------------------------------------------- */

/* Exact 2-NN + Lowe ratio test. Replaces cublas_2nn_sift,
   include/knn_brute.h:22 / src/knn_brute.cu:24. matches[q] = index of the
   nearest base row if the ratio test passes, else UINT32_MAX. `matches` may be
   device, managed or host memory. handle, stream_n, use and warps (the
   reference's cuBLAS handle, stream count, batch byte budget and scan block
   size) are accepted and ignored: the fused kernel needs no distance batches.
   Synchronises before returning (the reference's trailing cudaFree did). */
SIFT_API int cublas_2nn_sift(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n, uint32_t* matches,
                    float threshold, cublasHandle_t handle, int stream_n, size_t use, int warps);

/* FP32-interface 2-NN ranked by -2 q.r. Replaces cublas_2nn_f,
   include/knn_brute.h:18 / src/knn_brute.cu:523. sorted[q] = {d1, d2, i1, i2}
   with d = -2 q.r as the reference computes it (norms are not added).
   q/r/sorted: device or managed memory. Synchronises. */
SIFT_API void cublas_2nn_f(des_t_f* q_points, des_t_f* r_points, int q_n, int r_n, sift_float4* sorted,
                  cublasHandle_t handle);

/* Exact 2-NN with full squared distances. Replaces device_brute,
   include/knn_brute.h:14 / src/knn_brute.cu:619. sorted[q] = {d1, d2, i1, i2};
   absent neighbours are FLT_MAX. q/r/sorted: device or managed memory.
   Synchronises. */
SIFT_API void device_brute(des_t_f* q_points, des_t_f* r_points, int q_n, int r_n, sift_float4* sorted);

/* Same contract as device_brute for host arrays. Replaces host_brute,
   include/knn_brute.h:29 / src/knn_brute.cu:801; the search runs on the GPU
   (there is no CPU path in this library). */
SIFT_API void host_brute(des_t_f* q_points, des_t_f* r_points, int q_points_size, int r_points_size, sift_float4* sorted);

/* Random-hyperplane LSH 2-NN. Replaces lsh_gpu, include/lsh_h.h:69 /
   src/lsh_h.cu:722. Hyperplanes: l tables of nbits +/-1 planes drawn with the C
   library's rand() in the reference's order (make_vec_h, src/lsh_h.cu:88-100),
   so a caller that seeds rand() identically gets the reference's hash family.
   matches[q] = nearest base row among the members of the query's bucket in
   any table (exact squared distance, lower index on ties), UINT32_MAX when no
   bucket holds a candidate. threshold, handle, stream_n and lsh_type are
   accepted and ignored, as in the reference. Unlike the reference, the
   caller's buffers are not freed. Synchronises. */
SIFT_API int lsh_gpu(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n, uint32_t* matches,
                     float threshold, cublasHandle_t handle, int stream_n, int l, int lsh_type, int nbits);

/* Status of the last void call above on this thread (SIFT_OK or SIFT_ERR_*). */
SIFT_API int sift_last_status(void);

/* ---------------------------------------------------------------------
 * Part 2: native interface
 * ------------------------------------------------------------------- */

/* Exact 2-NN of q against r. q, r: descriptors of memory type `type` (the same
   for both). Outputs (device, managed or host memory; any may be NULL):
     matches[q_n]    nearest index if the ratio test passes, else UINT32_MAX
     sorted[q_n]     {d1, d2, i1, i2} as floats, FLT_MAX where absent
     nn_idx[2*q_n]   int32 nearest / second indices, -1 where absent
     nn_dist[2*q_n]  float distances under `metric`, FLT_MAX where absent
   Float and half values that are integers in [0, 255] times one common power
   of two 2^-s, s <= 24 (raw SIFT components, or the reference benchmark's
   components / 512, src/test.cu:99-103) are searched exactly, distances in
   the caller's units (the integer results times 2^-2s): SIFT_HALF_DEVICE
   rows in place by the FP16 tensor-core kernel (kind::f16, f32
   accumulation, exact for such values), float rows packed to u8 for the u8
   kernel. Any other finite values (e.g. the reference benchmark's default
   unit-normalised rand() vectors) take the general float path: float rows
   split into FP16 hi + lo parts, half rows in place, f32 accumulation on the
   tensor cores; distances within 2^-16 (|q|^2 + |r|^2) of FP64 and index
   swaps only among rows that close. Infinite or NaN values return
   SIFT_ERR_INVALID_ARG.
   stream: a cudaStream_t (NULL = legacy default stream). With u8 device
   inputs and device outputs the call is asynchronous on `stream`; device-side
   problems are then reported by sift_stream_status(stream). Float / half
   inputs synchronise once (value check); any host input or host output makes
   the call synchronous. */
SIFT_API int sift2nn_match(const void* q, const void* r, int type, uint32_t q_n, uint32_t r_n, int metric, float threshold,
                  uint32_t* matches, sift_float4* sorted, int32_t* nn_idx, float* nn_dist, void* stream);

/* LSH codes of n u8 descriptors (device memory, 16-byte aligned):
   codes[t * n + i] bit j is set when x_i . planes[t][j] < 0, for L tables of
   k bits (k <= 32, L * k <= 256). planes: int8 [L][k][128] in device memory.
   The dot products are exact (u8 x s8 -> s32 on the tensor cores). */
SIFT_API int sift_lsh_hash(const uint8_t* x, uint32_t n, const int8_t* planes, int L, int k, uint32_t* codes,
                           void* stream);

/* Bucket table of LSH codes (codes[t * n + i], t < L, as sift_lsh_hash writes
   them; device memory): per table the n points grouped by the top
   B = min(k, 16) code bits, the grouping the LSH search scans. Replaces the
   reference's thrust sort by code + host run-length encoding
   (lsh_thread_sort_reduce, src/lsh_h.cu:565-629). Outputs (device):
   start[t * (2^B + 1) + b] .. start[t * (2^B + 1) + b + 1] are the positions
   of group b, order[t * n + pos] the point id at a position and
   ocode[t * n + pos] its code. Within a group, positions are in no fixed
   order (the groups themselves are). Asynchronous on `stream`. */
SIFT_API int sift_lsh_buckets(const uint32_t* codes, uint32_t n, int L, int k, int* start, int* order,
                              uint32_t* ocode, void* stream);

/* LSH 2-NN with caller-given int8 hyperplanes [L][k][128] (host or device
   memory): each query is compared exactly with the base rows that share its
   code in at least one table. Outputs as sift2nn_match (nn_dist = squared
   distances; -1 / FLT_MAX where fewer than 1 / 2 candidates); matches applies
   the ratio test when threshold > 0, else holds the nearest candidate.
   Integer-valued rows (as sift2nn_match) are hashed and scanned exactly;
   other finite float / half rows are hashed and scanned in FP32 on the
   CUDA cores (a point whose dot product with a plane lies within FP32
   rounding of 0 may land in the neighbouring bucket). */
SIFT_API int sift_lsh_match(const void* q, const void* r, int type, uint32_t q_n, uint32_t r_n, const int8_t* planes,
                            int L, int k, float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist,
                            void* stream);

/* sift_lsh_match with query-directed multi-probe (the reference declares but
   never implements neighbouring-bucket search, include/lsh_h.h:71 /
   src/lsh_h.cu:393-407): per table the query also searches the buckets of
   its code with subsets of its min(6, k) lowest-margin bits flipped (margin =
   |q . plane|), the `probes` lightest subsets by summed margin, probe 0 the
   code itself; 1 <= probes <= 2^min(6, k). candidates (optional device
   [q_n]) receives the number of base rows compared per query (duplicates
   across tables counted once per table). */
SIFT_API int sift_lsh_match_probes(const void* q, const void* r, int type, uint32_t q_n, uint32_t r_n,
                                   const int8_t* planes, int L, int k, int probes, float threshold,
                                   uint32_t* matches, int32_t* nn_idx, float* nn_dist, uint32_t* candidates,
                                   void* stream);

/* Exact 2-NN that allocates no memory at all (no counterpart in the
   reference). For callers that cannot allocate device memory at call time:
   code whose device memory is owned by a custom allocator or pool, real-time
   loops that cannot take cudaMalloc's implicit synchronisation, hosts that
   give the library a fixed memory budget up front. The search and results
   are those of sift2nn_match with type SIFT_U8_DEVICE and SIFT_METRIC_L2;
   q, r (16-byte aligned uint8 [n][128]) and the outputs (matches[q_n],
   nn_idx[2*q_n], nn_dist[2*q_n]; any may be NULL) are device memory the
   caller owns. All scratch lives in one 8 MiB __device__ array of the library
   (held by every GPU that loads it, until exit), which limits q_n to 16384 and
   r_n to 1048576: larger sizes return SIFT_ERR_INVALID_ARG. Calls on one
   device share that array, so calls that overlap on the GPU race: serialise
   them. The first call on a device looks the array's address up with
   cudaGetSymbolAddress; make it before any stream capture. Asynchronous on
   `stream` (NULL = legacy default stream). q, r and the outputs must be
   device or managed memory (host pointers return SIFT_ERR_INVALID_ARG). If a
   bounded wait inside the search expires (no correct run does this), every
   output row of that call is written as "no result" (UINT32_MAX, -1,
   FLT_MAX) and sift2nn_noalloc_status reports it. */
SIFT_API int sift2nn_match_noalloc(const uint8_t* q, const uint8_t* r, uint32_t q_n, uint32_t r_n, float threshold,
                                   uint32_t* matches, int32_t* nn_idx, float* nn_dist, void* stream);

/* Device status of sift2nn_match_noalloc (no counterpart in the reference):
   synchronises `stream` and returns SIFT_ERR_DEVICE_TIMEOUT if a call on the
   current device hit an expired bounded wait since the last check (then
   clears the record), else SIFT_OK. Reads a word of the library's own array;
   allocates nothing. */
SIFT_API int sift2nn_noalloc_status(void* stream);

/* Batched exact 2-NN of many independent (query set, base set) problems,
   e.g. the keypoint descriptors of many image pairs of uneven sizes, in one
   persistent launch driven by a device work list (no counterpart in the
   reference, which matches one pair per call). q: the query sets of all
   problems concatenated in problem order (sum of n_q rows); r: r_rows base
   rows, problem p using rows [r_off, r_off + n_r) (problems may share rows).
   Both uint8 [rows][128], 16-byte aligned device memory. Outputs are per
   query row of q (device memory; any may be NULL), indices local to the
   problem's base set: matches (ratio test at `threshold`, else UINT32_MAX),
   nn_idx[2*row] (-1 absent), nn_dist[2*row] (squared L2, FLT_MAX absent).
   Asynchronous on `stream`; the kernel shape is the one last tuned for a
   batch of the same sizes, else the default. */
typedef struct sift_pair {
    uint32_t n_q;   /* query rows of the problem (consecutive in q) */
    uint32_t n_r;   /* base rows of the problem */
    uint32_t r_off; /* first base row of the problem in r */
} sift_pair;
SIFT_API int sift2nn_match_batch(const uint8_t* q, const uint8_t* r, uint32_t r_rows, const sift_pair* pairs,
                                 int n_pairs, float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist,
                                 void* stream);

/* Mutual nearest neighbours (cross-check) of the problems of a batch, e.g.
   the two keypoint sets of each image pair: a holds every problem's first set
   (consecutive, in problem order; `pairs` as in sift2nn_match_batch with
   n_q = rows of the set in a), b the second sets at r_off. Both directions
   run through the batched exact search; matches[row] (required) = j, local to
   the problem's set in b, when j is the nearest row of b for that row of a,
   that row is the nearest row of a for row j of b, and -- when threshold > 0
   -- the forward ratio test passes; else UINT32_MAX. nn_idx / nn_dist
   (optional) receive the forward 2-NN as in sift2nn_match_batch. Sets of b
   that are not stored consecutively in problem order are gathered first.
   No counterpart in the reference (which matches one direction per call). */
SIFT_API int sift2nn_match_mutual_batch(const uint8_t* a, const uint8_t* b, uint32_t b_rows, const sift_pair* pairs,
                                        int n_pairs, float threshold, uint32_t* matches, int32_t* nn_idx,
                                        float* nn_dist, void* stream);

/* Match lists for geometric verification (e.g. RANSAC on each image pair):
   the rows of a batch whose matches[row] is not UINT32_MAX (matches and
   nn_dist as sift2nn_match_batch / sift2nn_match_mutual_batch write them,
   device memory, `rows` = sum of pairs[].n_q) as records grouped by problem,
   rows in order. pair_offsets (device, [n_pairs + 1]) receives the first
   record of each problem and, last, the number of matches; records past
   `capacity` are not written (compare the count with it). nn_dist may be
   NULL (d1 = d2 = 0). Asynchronous on `stream`. */
typedef struct sift_match {
    uint32_t pair; /* problem */
    uint32_t a;    /* row within the problem's first set */
    uint32_t b;    /* matched row within its second set */
    float d1, d2;  /* squared distances to the nearest and second nearest */
} sift_match;
SIFT_API int sift_compact_matches(const uint32_t* matches, const float* nn_dist, uint32_t rows, const sift_pair* pairs,
                                  int n_pairs, sift_match* out, uint32_t capacity, uint32_t* pair_offsets,
                                  void* stream);

/* Merge of 2-NN results searched over `parts` disjoint base shards (e.g. one
   per rank of a base-sharded search, after an all-gather): nn_dist_parts /
   nn_idx_parts are [parts][q_n][2] device arrays as sift2nn_match writes them
   (indices local to the shard, -1 / FLT_MAX absent), offsets[parts] (host)
   the first base row of each shard. Writes the lexicographic (distance,
   global index) top-2 of every query and the ratio test at `threshold`, the
   same result as one search over the whole base. parts <= 64. */
SIFT_API int sift_merge_top2(const float* nn_dist_parts, const int32_t* nn_idx_parts, const int32_t* offsets,
                             int parts, uint32_t q_n, float threshold, uint32_t* matches, int32_t* nn_idx,
                             float* nn_dist, void* stream);

/* A batch bound to fixed buffers, replayed as one CUDA graph: create times
   the kernel shapes on this batch when flags has SIFT_BATCH_TUNE (the choice
   is remembered for batches of the same sizes), or takes shape k with
   SIFT_BATCH_SHAPE(k), k in 0..2 (0: 512-query groups, one query buffer;
   1: 512-query groups, two buffers; 2: 256-query groups, two buffers). The
   plan owns its scratch memory; run launches the graph on `stream` (the
   results follow the current contents of q and r). Create synchronises. */
typedef struct sift_batch_plan sift_batch_plan;
#define SIFT_BATCH_TUNE 1
#define SIFT_BATCH_SHAPE(k) (((k) + 1) << 4)
SIFT_API int sift_batch_plan_create(const uint8_t* q, const uint8_t* r, uint32_t r_rows, const sift_pair* pairs,
                                    int n_pairs, float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist,
                                    int flags, sift_batch_plan** plan);
SIFT_API int sift_batch_plan_run(sift_batch_plan* plan, void* stream);
/* Chosen shape (query tiles per CTA, query buffers) and, after tuning, the
   measured milliseconds of each shape (tuned_ms[3], -1 when not timed). */
SIFT_API int sift_batch_plan_info(const sift_batch_plan* plan, int* qpt, int* qbuf, float* tuned_ms);
SIFT_API void sift_batch_plan_destroy(sift_batch_plan* plan);

/* Synchronises `stream` and returns the device status of the calls issued on
   the current device since the last check (SIFT_OK, SIFT_ERR_DEVICE_TIMEOUT
   when a bounded wait inside a kernel expired, SIFT_ERR_CUDA). */
SIFT_API int sift_stream_status(void* stream);

/* Human-readable name of a status code. */
SIFT_API const char* sift_status_string(int status);

/* Library version string. */
SIFT_API const char* sift_version(void);

/* ---------------------------------------------------------------------
 * Part 3: instrumentation (used by the benchmark)
 * ------------------------------------------------------------------- */

/* ---------------------------------------------------------------------
 * Learned hash (no counterpart in the reference, whose only hash is the
 * random-hyperplane family of src/lsh_h.cu:88-100): an MLP 128 -> 256 -> k,
 * z = W2 h + b2, h = bf16(relu(W1 (x / 64) + b1)), BF16 weights, FP32
 * accumulation; bit j of a descriptor's bucket code is set when z_j > 0.
 * ------------------------------------------------------------------- */
typedef struct sift_mlp {
    const void* w1;  /* bf16 [256][128], device, 16-byte aligned */
    const float* b1; /* [256] */
    const void* w2;  /* bf16 [k][256] */
    const float* b2; /* [k] */
    int k;           /* code bits, 1..32 */
} sift_mlp;

/* Trains a model on neighbour pairs labelled by the exact search: each of
   `steps` Adam steps (learning rate lr) draws `batch` (multiple of 32)
   training queries from train_q, their exact nearest base rows and `batch`
   random base rows, and minimises
     mean(1 - s(q, nn)) + neg_weight * mean(s(q, random)^2)
       + balance_weight * sum_j mean(t_j)^2,
   t = tanh(z), s(a, b) = mean_j t_aj t_bj. base, train_q: uint8 [n][128]
   device rows. Outputs: the model (w1, b1, w2, b2 as in sift_mlp, device),
   optionally the FP32 parameters (params_out, device, SIFT_MLP_PARAMS
   floats: W1, b1, W2 padded to 32 rows, b2 padded to 32) and the loss of
   every step (loss_curve, host). Deterministic for a given seed.
   Synchronises. */
#define SIFT_MLP_PARAMS (256 * 128 + 256 + 32 * 256 + 32)
SIFT_API int sift_mlp_train(const uint8_t* base, uint32_t r_n, const uint8_t* train_q, uint32_t t_n, int k, int steps,
                            int batch, float lr, float neg_weight, float balance_weight, unsigned long long seed,
                            void* w1, float* b1, void* w2, float* b2, float* params_out, float* loss_curve);

/* Bucket codes of n uint8 rows (device) on the tensor cores; z (optional,
   device [n][k]) receives the outputs. Asynchronous on `stream`. */
SIFT_API int sift_mlp_hash(const uint8_t* x, uint32_t n, const sift_mlp* model, uint32_t* codes, float* z,
                           void* stream);

/* Approximate 2-NN with the learned hash: base rows are bucketed by code;
   each query scans n_probes buckets (its code, then codes with its
   smallest-|z| bits flipped, lightest flips first; n_probes <= 64) with
   exact distances; queries whose buckets held fewer than min_candidates rows,
   or (max_dist > 0) whose nearest candidate lies farther than max_dist
   (squared L2; none found counts as farther), are searched exactly (the
   exact kernel) instead. Outputs as sift2nn_match
   for uint8 device rows (matches: ratio test when threshold > 0, else the
   nearest candidate); candidates (device [q_n], optional) receives the number
   of base rows each query compared in its buckets; fallback_count (host,
   optional) the number of queries searched exactly. Synchronises when
   min_candidates > 0 or max_dist > 0. */
SIFT_API int sift_mlp_match(const uint8_t* q, const uint8_t* r, uint32_t q_n, uint32_t r_n, const sift_mlp* model,
                            int n_probes, int min_candidates, float max_dist, float threshold, uint32_t* matches,
                            int32_t* nn_idx, float* nn_dist, uint32_t* candidates, uint32_t* fallback_count,
                            void* stream);

/* Persistent hash index of a base (no counterpart in the reference, whose
   lsh_gpu hashes and sorts the base again on every call, src/lsh_h.cu:894-972):
   the base is hashed and bucketed once at creation and searched any number
   of times. The index keeps its own bucket table, base-tile records and a
   copy of the hash (hyperplanes or model); it reads the base rows `r` (uint8
   [r_n][128], 16-byte aligned device memory) by reference, so they must stay
   valid and unchanged while the index lives. Creation synchronises.
     sift_lsh_index_create: random-hyperplane hash with int8 planes
       [L][k][128] (host or device memory), as sift_lsh_match.
     sift_mlp_index_create: the learned hash `model` (L = 1 table).
   sift_index_search: 2-NN of q_n uint8 device queries as sift_lsh_match
   (probes: 1..2^min(6, k) buckets per table, query-directed multi-probe), with
   the exact fallback of sift_mlp_match when min_candidates > 0 or
   max_dist > 0 (then it synchronises once). Outputs as sift_mlp_match.
   sift_index_buckets: copies the bucket table into caller device buffers
   (start, order, ocode laid out as sift_lsh_buckets writes them; any may be
   NULL) on `stream`, and returns its group bits B in top_bits. */
typedef struct sift_code_index sift_code_index;
SIFT_API int sift_lsh_index_create(const uint8_t* r, uint32_t r_n, const int8_t* planes, int L, int k,
                                   sift_code_index** index);
SIFT_API int sift_mlp_index_create(const uint8_t* r, uint32_t r_n, const sift_mlp* model, sift_code_index** index);
SIFT_API int sift_index_search(const sift_code_index* index, const uint8_t* q, uint32_t q_n, int probes,
                               int min_candidates, float max_dist, float threshold, uint32_t* matches,
                               int32_t* nn_idx, float* nn_dist, uint32_t* candidates, uint32_t* fallback_count,
                               void* stream);
SIFT_API int sift_index_buckets(const sift_code_index* index, int* start, int* order, uint32_t* ocode, int* top_bits,
                                void* stream);
SIFT_API void sift_index_destroy(sift_code_index* index);

/* Loss and gradients of one training step, for checking the training
   kernels: x = [3 * batch][128] uint8 device rows (queries, their
   neighbours, random rows), params / grads = SIFT_MLP_PARAMS device floats
   (weights are rounded to BF16 for the forward pass; gradients pass straight
   through the roundings), loss (host [4]) = total, positive, negative,
   balance terms. Synchronises. */
SIFT_API int sift_mlp_loss_grad(const uint8_t* x, int batch, int k, const float* params, float neg_weight,
                                float balance_weight, float* grads, float* loss);

/* Host-side work decomposition of a batch (no GPU needed): out[0..5] =
   units, base-tile records, query rows, max CTA pairs sharing one query
   group, CTA pairs launched, queries per group; for `workers` CTA pairs and
   qpt query tiles per CTA (1 or 2). */
SIFT_API int sift_batch_describe(const sift_pair* pairs, int n_pairs, uint32_t r_rows, int qpt, int workers,
                                 long long* out);

/* Number of kernels this library has launched in the process so far. */
SIFT_API long long sift_launch_count(void);

/* When enabled, the timed kernels of every call are bracketed by CUDA events
   recorded on the stream they are launched on: the exact search kernel
   (SIFT_PROF_SEARCH), the query hash of the hash searches (SIFT_PROF_HASH)
   and their candidate scan (SIFT_PROF_SCAN). */
#define SIFT_PROF_SEARCH 0
#define SIFT_PROF_HASH 1
#define SIFT_PROF_SCAN 2
SIFT_API void sift_profile_enable(int on);

/* Synchronises the recorded events and returns (and clears) the summed search
   kernel time in milliseconds and the number of timed launches. */
SIFT_API int sift_profile_collect(double* total_ms, int* launches);
/* The same for one kernel kind (SIFT_PROF_*). */
SIFT_API int sift_profile_collect_kernel(int kernel, double* total_ms, int* launches);

/* Selects the exact-search kernel for subsequent calls in this process:
   0 (default) the CTA-pair kernels (tcgen05 cta_group::2): u8 rows on the
   kernel that folds the base norms into a fifth MMA per tile, half inputs on
   the FP16 kernel; 1 the single-CTA u8 kernel; 2 the CTA-pair u8 kernel
   without folding for every input type (half inputs packed to u8); 3 as 0
   but without folding. All return identical results. */
SIFT_API int sift_set_kernel_variant(int variant);

/* Fault injection for failure-detection tests (no counterpart in the
   reference, which checks no errors, src/knn_brute.cu:254-275). Neither hook
   faults, traps or hangs the GPU.
   sift_test_inject_wait_expiry(n): the next n exact searches first run a
   one-thread probe whose bounded mbarrier wait (the wait every pipeline stage
   of the search kernels uses) can never complete; it expires after 1 ms and
   records the same device error an expired wait in a search records, so
   sift_stream_status / sift2nn_noalloc_status report SIFT_ERR_DEVICE_TIMEOUT.
   sift_test_fail_arena(n): the next n calls that request the scratch arena
   fail with SIFT_ERR_ALLOC as if the allocation had failed. n = 0 disarms. */
SIFT_API int sift_test_inject_wait_expiry(int calls);
SIFT_API int sift_test_fail_arena(int calls);

#ifdef __cplusplus
}
#endif

#endif /* SIFT2NN_H_ */
