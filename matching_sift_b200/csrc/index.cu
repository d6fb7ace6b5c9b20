// Persistent hash indexes of a base: the base is hashed and bucketed once
// (sift_lsh_index_create / sift_mlp_index_create) and searched any number of
// times (sift_index_search). The reference re-hashes and re-sorts the base on
// every lsh_gpu call (src/lsh_h.cu:894-972); here that work leaves the query
// path, which is then: hash the queries (+ their margins for multi-probe),
// probe codes, candidate scan, and optionally the exact fallback for queries
// whose buckets held too few candidates.
//
// Also the exact fallback shared with sift_mlp_match: the flagged queries are
// gathered, searched by the exact CTA-pair kernel and their results scattered
// back over the hash results.
#include <cstring>
#include <new>
#include <tuple>
#include "api_internal.h"
#include "context.h"
#include "exact2nn.cuh"
#include "index.cuh"
#include "learned.cuh"
#include "lsh.cuh"

struct sift_code_index {
    int dev = -1;
    int kind = 0;  // 1: random hyperplanes (int8), 2: learned hash (MLP)
    const uint8_t* r = nullptr;  // the caller's base rows (device), used by reference
    int r_n = 0, L = 1, k = 0, top = 0, shift = 0, nbins = 0, P = 0;
    char* mem = nullptr;
    int* start = nullptr;       // [L][nbins + 1]
    int* order = nullptr;       // [L][r_n]
    uint32_t* ocode = nullptr;  // [L][r_n]
    int32_t* brec = nullptr;    // base-tile records of the exact fallback
    int8_t* planes = nullptr;   // kind 1: [L][k][128]
    __nv_bfloat16* w1 = nullptr;  // kind 2: copies of the model
    float* b1 = nullptr;
    __nv_bfloat16* w2 = nullptr;
    float* b2 = nullptr;
};

namespace sift {
namespace {

using detail::DeviceCtx;

// Queries whose probed buckets compared fewer than min_cand candidates, or
// (max_dist > 0) whose nearest candidate lies farther than max_dist.
__global__ void flag_kernel(const uint32_t* __restrict__ counts, const float* __restrict__ dist, int n,
                            uint32_t min_cand, float max_dist, int* __restrict__ idx, int* __restrict__ n_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool far = max_dist > 0.0f && !(dist[2 * i] <= max_dist);
    if (counts[i] < min_cand || far) idx[atomicAdd(n_out, 1)] = i;
}

__global__ void gather_rows_kernel(const uint8_t* __restrict__ q, const int* __restrict__ idx, int n,
                                   uint8_t* __restrict__ out) {
    const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (e >= static_cast<long long>(n) * 8) return;
    const int f = static_cast<int>(e >> 3), c = static_cast<int>(e & 7);
    reinterpret_cast<uint4*>(out + static_cast<size_t>(f) * kDim)[c] =
        reinterpret_cast<const uint4*>(q + static_cast<size_t>(idx[f]) * kDim)[c];
}

__global__ void scatter_results_kernel(const int* __restrict__ idx, int n, const uint32_t* __restrict__ m_in,
                                       const int32_t* __restrict__ i_in, const float* __restrict__ d_in,
                                       uint32_t* __restrict__ matches, int32_t* __restrict__ nn_idx,
                                       float* __restrict__ nn_dist) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    const int q = idx[f];
    if (matches) matches[q] = m_in[f];
    if (nn_idx) {
        nn_idx[2 * q] = i_in[2 * f];
        nn_idx[2 * q + 1] = i_in[2 * f + 1];
    }
    if (nn_dist) {
        nn_dist[2 * q] = d_in[2 * f];
        nn_dist[2 * q + 1] = d_in[2 * f + 1];
    }
}

bool aligned_dev(const void* p) {
    return p && !(reinterpret_cast<uintptr_t>(p) & 15) && detail::is_device_accessible(p);
}

}  // namespace

void fallback_layout(detail::Layout& L, int q_n, int r_n, int num_workers, bool own_brec, FallbackScratch& fs) {
    // A group of 512 queries spans at most grid / groups + 2 workers.
    const ExactPlan worst = make_exact_plan(q_n, r_n, num_workers, 2);
    fs.fb_part = static_cast<size_t>(worst.grid + 2 * worst.q_groups + 2) * (kQT * kBM) * 2 * sizeof(int4);
    fs.o_fidx = L.take(static_cast<size_t>(q_n) * 4 + 16);
    fs.o_frows = L.take(static_cast<size_t>(q_n) * kDim + 16);
    fs.o_fm = L.take(static_cast<size_t>(q_n) * 4);
    fs.o_fi = L.take(static_cast<size_t>(q_n) * 8);
    fs.o_fd = L.take(static_cast<size_t>(q_n) * 8);
    fs.o_brec = own_brec ? L.take(static_cast<size_t>(worst.base_tiles) * kRecInts * 4 + 16) : 0;
    fs.o_fqn = L.take(static_cast<size_t>(worst.q_pad) * 4);
    fs.o_fthr = L.take(static_cast<size_t>(worst.q_pad) * 4);
    fs.o_fpart = L.take(fs.fb_part);
    fs.own_brec = own_brec;
}

int exact_fallback(DeviceCtx& c, char* A, const FallbackScratch& fs, const uint8_t* q, const uint8_t* r, int q_n,
                   int r_n, const int32_t* brec_in, const uint32_t* counts, const float* dist, int min_cand,
                   float max_dist, float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist,
                   uint32_t* fallback_count, cudaStream_t st) {
    auto I32 = [&](size_t o) { return reinterpret_cast<int32_t*>(A + o); };
    int* fidx = I32(fs.o_fidx);
    int* fcount = fidx + q_n;  // the 16 bytes past the index list
    SIFT_CUDA(cudaMemsetAsync(fcount, 0, sizeof(int), st));
    flag_kernel<<<(q_n + 255) / 256, 256, 0, st>>>(counts, dist, q_n, static_cast<uint32_t>(min_cand), max_dist,
                                                    fidx, fcount);
    SIFT_CUDA(cudaGetLastError());
    SIFT_CUDA(cudaMemcpyAsync(c.h_status + 1, fcount, sizeof(int), cudaMemcpyDeviceToHost, st));
    SIFT_CUDA(cudaStreamSynchronize(st));
    const int nf = c.h_status[1];
    if (fallback_count) *fallback_count = static_cast<uint32_t>(nf);
    ++detail::g_launches;
    if (nf == 0) return SIFT_OK;
    uint8_t* frows = reinterpret_cast<uint8_t*>(A + fs.o_frows);
    gather_rows_kernel<<<static_cast<unsigned>((static_cast<long long>(nf) * 8 + 255) / 256), 256, 0, st>>>(
        q, fidx, nf, frows);
    SIFT_CUDA(cudaGetLastError());
    const ExactPlan plan = make_exact_plan(nf, r_n, c.num_sms / 2, 2);
    if (static_cast<size_t>(plan.max_splits) * plan.parts * plan.q_pad * sizeof(int4) > fs.fb_part)
        return SIFT_ERR_INVALID_ARG;  // guard: fb_part bounds every plan of <= q_n queries
    const int32_t* brec = brec_in;
    int launches = 6;
    if (!brec) {
        SIFT_CUDA(launch_row_norms_u8(r, r_n, plan.r_pad, kMetricL2, nullptr, I32(fs.o_brec), nullptr, st));
        brec = I32(fs.o_brec);
        ++launches;
    }
    SIFT_CUDA(launch_row_norms_u8(frows, nf, plan.q_pad, kMetricL2, I32(fs.o_fqn), nullptr, I32(fs.o_fthr), st));
    CUtensorMap qmap, bmap;
    SIFT_TRY(detail::encode_u8_rows(&qmap, frows, nf, kBM));
    SIFT_TRY(detail::encode_u8_rows(&bmap, r, r_n, kBN / 2));
    int4* part = reinterpret_cast<int4*>(A + fs.o_fpart);
    SIFT_CUDA(launch_exact2nn_u8_pair(qmap, bmap, brec, plan, part, I32(fs.o_fthr), c.d_status, st));
    uint32_t* fm = reinterpret_cast<uint32_t*>(A + fs.o_fm);
    int32_t* fi = I32(fs.o_fi);
    float* fd = reinterpret_cast<float*>(A + fs.o_fd);
    SIFT_CUDA(launch_merge2nn(part, plan, I32(fs.o_fqn), kMetricL2, threshold, 1.0f, fm, nullptr, fi, fd, st));
    scatter_results_kernel<<<(nf + 255) / 256, 256, 0, st>>>(fidx, nf, fm, fi, fd, matches, nn_idx, nn_dist);
    SIFT_CUDA(cudaGetLastError());
    detail::g_launches += launches;
    return SIFT_OK;
}

namespace {

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Device memory of an index: bucket table, base records, the hash's parameters.
int index_alloc(sift_code_index& ix, size_t param_bytes) {
    const size_t n_start = static_cast<size_t>(ix.L) * (ix.nbins + 1) * 4;
    const size_t n_order = static_cast<size_t>(ix.L) * ix.r_n * 4 + 16;
    const int base_tiles = (ix.r_n + kBN - 1) / kBN;
    const size_t n_brec = static_cast<size_t>(base_tiles) * kRecInts * 4 + 16;
    const size_t total = align256(n_start) + 2 * align256(n_order) + align256(n_brec) + align256(param_bytes);
    if (cudaMalloc(&ix.mem, total) != cudaSuccess) {
        cudaGetLastError();
        ix.mem = nullptr;
        return SIFT_ERR_ALLOC;
    }
    size_t off = 0;
    auto take = [&](size_t b) {
        char* p = ix.mem + off;
        off += align256(b);
        return p;
    };
    ix.start = reinterpret_cast<int*>(take(n_start));
    ix.order = reinterpret_cast<int*>(take(n_order));
    ix.ocode = reinterpret_cast<uint32_t*>(take(n_order));
    ix.brec = reinterpret_cast<int32_t*>(take(n_brec));
    char* params = take(param_bytes);
    if (ix.kind == 1) {
        ix.planes = reinterpret_cast<int8_t*>(params);
    } else {
        ix.w1 = reinterpret_cast<__nv_bfloat16*>(params);
        ix.b1 = reinterpret_cast<float*>(params + align256(kMlpHidden * kMlpIn * 2));
        ix.w2 = reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(ix.b1) + align256(kMlpHidden * 4));
        ix.b2 = reinterpret_cast<float*>(reinterpret_cast<char*>(ix.w2) + align256(kMlpOutRows * kMlpHidden * 2));
    }
    return SIFT_OK;
}

size_t mlp_param_bytes() {
    return align256(kMlpHidden * kMlpIn * 2) + align256(kMlpHidden * 4) + align256(kMlpOutRows * kMlpHidden * 2) +
           align256(kMlpOutRows * 4);
}

MlpModel index_model(const sift_code_index& ix) {
    MlpModel m;
    m.w1 = ix.w1;
    m.b1 = ix.b1;
    m.w2 = ix.w2;
    m.b2 = ix.b2;
    m.k = ix.k;
    return m;
}

int encode_model(const MlpModel& m, CUtensorMap* w1map, CUtensorMap* w2map) {
    SIFT_TRY(detail::encode_bf16_2d(w1map, m.w1, kMlpIn, kMlpHidden, 64, kMlpHidden));
    SIFT_TRY(detail::encode_bf16_2d(w2map, m.w2, kMlpHidden, static_cast<uint64_t>(m.k), 64, kMlpOutRows));
    return SIFT_OK;
}

// Codes of n rows into codes[L][n] (and the margins z[L][n][k] when z is
// given) with the index's hash.
int index_hash(DeviceCtx& c, const sift_code_index& ix, const uint8_t* x, int n, uint32_t* codes, float* z,
               cudaStream_t st) {
    if (n <= 0) return SIFT_OK;
    CUtensorMap xmap;
    SIFT_TRY(detail::encode_u8_rows(&xmap, x, static_cast<uint64_t>(n), 128));
    if (ix.kind == 1) {
        CUtensorMap pmap;
        SIFT_TRY(detail::encode_u8_rows(&pmap, ix.planes, static_cast<uint64_t>(ix.L) * ix.k,
                                        static_cast<uint32_t>(ix.P)));
        SIFT_CUDA(launch_lsh_hash(xmap, pmap, n, ix.P, ix.L, ix.k, codes, z, c.d_status, c.num_sms, st));
    } else {
        CUtensorMap w1map, w2map;
        const MlpModel m = index_model(ix);
        SIFT_TRY(encode_model(m, &w1map, &w2map));
        SIFT_CUDA(launch_mlp_hash(xmap, n, w1map, w2map, m.b1, m.b2, m.k, codes, z, c.d_status, c.num_sms, st));
    }
    ++detail::g_launches;
    return SIFT_OK;
}

// Hashes and buckets the base (one-off, synchronous on the legacy stream).
int index_build(sift_code_index& ix) {
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    DeviceCtx& c = *cp;
    ix.dev = dev;
    cudaStream_t st = nullptr;
    detail::ArenaLock lk(c, st);
    detail::Layout L;
    const size_t o_codes = L.take(static_cast<size_t>(ix.L) * ix.r_n * 4 + 16);
    const size_t o_hist = L.take(static_cast<size_t>(ix.L) * ix.nbins * 4);
    SIFT_TRY(detail::ensure_arena(c, L.off));
    uint32_t* codes = reinterpret_cast<uint32_t*>(c.arena + o_codes);
    SIFT_TRY(index_hash(c, ix, ix.r, ix.r_n, codes, nullptr, st));
    SIFT_CUDA(launch_lsh_buckets(codes, ix.r_n, ix.L, ix.shift, ix.nbins, reinterpret_cast<int*>(c.arena + o_hist),
                                 ix.start, ix.order, ix.ocode, c.num_sms, st));
    const int r_pad = (ix.r_n + kBN - 1) / kBN * kBN;
    SIFT_CUDA(launch_row_norms_u8(ix.r, ix.r_n, r_pad, kMetricL2, nullptr, ix.brec, nullptr, st));
    detail::g_launches += (ix.r_n > 0 ? 3 : 0) + (r_pad > 0 ? 1 : 0);
    SIFT_CUDA(cudaStreamSynchronize(st));
    return detail::collect_device_status(c, st);
}

void set_bins(sift_code_index& ix) {
    ix.top = ix.k < kLshMaxTopBits ? ix.k : kLshMaxTopBits;
    ix.shift = ix.k - ix.top;
    ix.nbins = 1 << ix.top;
}

int finish_create(sift_code_index* ix, sift_code_index** out) {
    const int rc = index_build(*ix);
    if (rc != SIFT_OK) {
        cudaFree(ix->mem);
        delete ix;
        return rc;
    }
    *out = ix;
    return SIFT_OK;
}

}  // namespace

int lsh_index_create(const uint8_t* r, uint32_t r_n, const int8_t* planes, int L_, int k, sift_code_index** out) {
    if (!out) return SIFT_ERR_INVALID_ARG;
    *out = nullptr;
    if (L_ < 1 || k < 1 || k > 32 || L_ * k > kLshMaxPlanes || !planes) return SIFT_ERR_INVALID_ARG;
    if (r_n > 0x7fffffffu / 32 || (r_n > 0 && !aligned_dev(r))) return SIFT_ERR_INVALID_ARG;
    auto* ix = new (std::nothrow) sift_code_index;
    if (!ix) return SIFT_ERR_ALLOC;
    ix->kind = 1;
    ix->r = r;
    ix->r_n = static_cast<int>(r_n);
    ix->L = L_;
    ix->k = k;
    ix->P = lsh_planes_padded(L_, k);
    set_bins(*ix);
    int rc = index_alloc(*ix, static_cast<size_t>(L_) * k * kDim);
    if (rc == SIFT_OK &&
        cudaMemcpy(ix->planes, planes, static_cast<size_t>(L_) * k * kDim, cudaMemcpyDefault) != cudaSuccess)
        rc = SIFT_ERR_CUDA;
    if (rc != SIFT_OK) {
        cudaGetLastError();
        cudaFree(ix->mem);
        delete ix;
        return rc;
    }
    return finish_create(ix, out);
}

int mlp_index_create(const uint8_t* r, uint32_t r_n, const sift_mlp* model, sift_code_index** out) {
    if (!out) return SIFT_ERR_INVALID_ARG;
    *out = nullptr;
    if (!model || model->k < 1 || model->k > kMlpMaxBits || !model->w1 || !model->b1 || !model->w2 || !model->b2)
        return SIFT_ERR_INVALID_ARG;
    if (r_n > 0x7fffffffu / 64 || (r_n > 0 && !aligned_dev(r))) return SIFT_ERR_INVALID_ARG;
    auto* ix = new (std::nothrow) sift_code_index;
    if (!ix) return SIFT_ERR_ALLOC;
    ix->kind = 2;
    ix->r = r;
    ix->r_n = static_cast<int>(r_n);
    ix->L = 1;
    ix->k = model->k;
    set_bins(*ix);
    int rc = index_alloc(*ix, mlp_param_bytes());
    if (rc == SIFT_OK) {
        // The index keeps its own copy of the model (W2 rows past k are zero).
        const int k = model->k;
        if (cudaMemset(ix->w2, 0, kMlpOutRows * kMlpHidden * 2) != cudaSuccess ||
            cudaMemset(ix->b2, 0, kMlpOutRows * 4) != cudaSuccess ||
            cudaMemcpy(ix->w1, model->w1, kMlpHidden * kMlpIn * 2, cudaMemcpyDefault) != cudaSuccess ||
            cudaMemcpy(ix->b1, model->b1, kMlpHidden * 4, cudaMemcpyDefault) != cudaSuccess ||
            cudaMemcpy(ix->w2, model->w2, static_cast<size_t>(k) * kMlpHidden * 2, cudaMemcpyDefault) != cudaSuccess ||
            cudaMemcpy(ix->b2, model->b2, static_cast<size_t>(k) * 4, cudaMemcpyDefault) != cudaSuccess)
            rc = SIFT_ERR_CUDA;
    }
    if (rc != SIFT_OK) {
        cudaGetLastError();
        cudaFree(ix->mem);
        delete ix;
        return rc;
    }
    return finish_create(ix, out);
}

int index_search(const sift_code_index* ix, const uint8_t* q, uint32_t q_n_, int probes, int min_cand,
                 float max_dist, float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist,
                 uint32_t* candidates, uint32_t* fallback_count, void* stream) {
    if (!ix) return SIFT_ERR_INVALID_ARG;
    const int flip = ix->k < 6 ? ix->k : 6;
    if (probes < 1 || probes > (1 << flip) || min_cand < 0 || !(max_dist >= 0.0f)) return SIFT_ERR_INVALID_ARG;
    if (q_n_ > 0x7fffffffu / 64 || static_cast<long long>(q_n_) * ix->L * (ix->k + probes) > 0x7fffffffLL)
        return SIFT_ERR_INVALID_ARG;
    if (fallback_count) *fallback_count = 0;
    if (q_n_ == 0) return SIFT_OK;
    if (!aligned_dev(q)) return SIFT_ERR_INVALID_ARG;
    for (const void* o : {static_cast<const void*>(matches), static_cast<const void*>(nn_idx),
                          static_cast<const void*>(nn_dist), static_cast<const void*>(candidates)})
        if (o && !detail::is_device_accessible(o)) return SIFT_ERR_INVALID_ARG;
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    if (dev != ix->dev) return SIFT_ERR_INVALID_ARG;
    DeviceCtx& c = *cp;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    detail::ArenaLock lk(c, st);
    const int q_n = static_cast<int>(q_n_), L_ = ix->L, k = ix->k;
    const bool multi = probes > 1;
    const bool fallback = (min_cand > 0 || max_dist > 0.0f) && ix->r_n > 0;

    detail::Layout L;
    const size_t o_cq = L.take(static_cast<size_t>(L_) * q_n * 4);
    const size_t o_z = multi ? L.take(static_cast<size_t>(L_) * q_n * k * 4) : 0;
    const size_t o_pc = multi ? L.take(static_cast<size_t>(L_) * probes * q_n * 4) : 0;
    const size_t o_cnt = L.take(static_cast<size_t>(q_n) * 4);
    const size_t o_dist = L.take(static_cast<size_t>(q_n) * 8);
    FallbackScratch fs{};
    if (fallback) fallback_layout(L, q_n, ix->r_n, c.num_sms / 2, false, fs);
    SIFT_TRY(detail::ensure_arena(c, L.off));
    char* A = c.arena;
    uint32_t* codes_q = reinterpret_cast<uint32_t*>(A + o_cq);
    float* z = multi ? reinterpret_cast<float*>(A + o_z) : nullptr;
    uint32_t* counts = candidates ? candidates : reinterpret_cast<uint32_t*>(A + o_cnt);
    float* dist = nn_dist ? nn_dist : reinterpret_cast<float*>(A + o_dist);

    {
        detail::ProfSpan span(st, detail::kProfHash);
        SIFT_TRY(index_hash(c, *ix, q, q_n, codes_q, z, st));
        span.end();
    }
    const uint32_t* probe_codes = codes_q;
    if (multi) {
        uint32_t* pc = reinterpret_cast<uint32_t*>(A + o_pc);
        for (int t = 0; t < L_; ++t)
            SIFT_CUDA(launch_probe_codes(codes_q + static_cast<size_t>(t) * q_n, z + static_cast<size_t>(t) * q_n * k,
                                         q_n, k, flip, probes, pc + static_cast<size_t>(t) * probes * q_n, st));
        detail::g_launches += L_;
        probe_codes = pc;
    }
    {
        detail::ProfSpan span(st, detail::kProfScan);
        SIFT_CUDA(launch_lsh_scan(q, ix->r, q_n, ix->r_n, L_, probes, ix->shift, ix->nbins, probe_codes, ix->start,
                                  ix->order, ix->ocode, threshold, threshold > 0.0f ? 1 : 0, 1.0f, matches, counts,
                                  nn_idx, dist, st));
        span.end();
    }
    ++detail::g_launches;
    if (!fallback) return SIFT_OK;
    SIFT_TRY(exact_fallback(c, A, fs, q, ix->r, q_n, ix->r_n, ix->brec, counts, dist, min_cand, max_dist, threshold,
                            matches, nn_idx, nn_dist, fallback_count, st));
    return SIFT_OK;
}

}  // namespace sift

extern "C" {

SIFT_API int sift_lsh_index_create(const uint8_t* r, uint32_t r_n, const int8_t* planes, int L, int k,
                                   sift_code_index** index) {
    return sift::lsh_index_create(r, r_n, planes, L, k, index);
}

SIFT_API int sift_mlp_index_create(const uint8_t* r, uint32_t r_n, const sift_mlp* model, sift_code_index** index) {
    return sift::mlp_index_create(r, r_n, model, index);
}

SIFT_API int sift_index_search(const sift_code_index* index, const uint8_t* q, uint32_t q_n, int probes,
                               int min_candidates, float max_dist, float threshold, uint32_t* matches,
                               int32_t* nn_idx, float* nn_dist, uint32_t* candidates, uint32_t* fallback_count,
                               void* stream) {
    return sift::index_search(index, q, q_n, probes, min_candidates, max_dist, threshold, matches, nn_idx, nn_dist,
                              candidates, fallback_count, stream);
}

SIFT_API int sift_index_buckets(const sift_code_index* index, int* start, int* order, uint32_t* ocode, int* top_bits,
                                void* stream) {
    if (!index) return SIFT_ERR_INVALID_ARG;
    if (top_bits) *top_bits = index->top;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n_start = static_cast<size_t>(index->L) * (index->nbins + 1) * 4;
    const size_t n_pos = static_cast<size_t>(index->L) * index->r_n * 4;
    for (auto [dst, src, bytes] : {std::tuple<void*, const void*, size_t>{start, index->start, n_start},
                                   {order, index->order, n_pos},
                                   {ocode, index->ocode, n_pos}}) {
        if (!dst || bytes == 0) continue;
        if (!sift::detail::is_device_accessible(dst)) return SIFT_ERR_INVALID_ARG;
        if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return SIFT_ERR_CUDA;
    }
    return SIFT_OK;
}

SIFT_API void sift_index_destroy(sift_code_index* index) {
    if (!index) return;
    int cur = 0;
    const bool switch_dev = cudaGetDevice(&cur) == cudaSuccess && index->dev >= 0 && cur != index->dev;
    if (switch_dev) cudaSetDevice(index->dev);
    cudaDeviceSynchronize();
    cudaFree(index->mem);
    if (switch_dev) cudaSetDevice(cur);
    delete index;
}

}  // extern "C"
