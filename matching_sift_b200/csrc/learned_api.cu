// Host entry points of the learned hash: training (labels from the exact
// search kernel), hashing, and matching (bucket build, query-directed
// multi-probe, candidate scan, exact fallback for queries whose probed
// buckets hold too few candidates).
#include <cmath>
#include <cstring>
#include <random>
#include <vector>
#include "api_internal.h"
#include "context.h"
#include "exact2nn.cuh"
#include "index.cuh"
#include "learned.cuh"
#include "lsh.cuh"

namespace sift {
namespace {

using detail::DeviceCtx;

int encode_model(const MlpModel& m, CUtensorMap* w1map, CUtensorMap* w2map) {
    SIFT_TRY(detail::encode_bf16_2d(w1map, m.w1, kMlpIn, kMlpHidden, 64, kMlpHidden));
    SIFT_TRY(detail::encode_bf16_2d(w2map, m.w2, kMlpHidden, static_cast<uint64_t>(m.k), 64, kMlpOutRows));
    return SIFT_OK;
}

int check_model(const sift_mlp* m) {
    if (!m || m->k < 1 || m->k > kMlpMaxBits || !m->w1 || !m->b1 || !m->w2 || !m->b2) return SIFT_ERR_INVALID_ARG;
    for (const void* p : {m->w1, static_cast<const void*>(m->b1), m->w2, static_cast<const void*>(m->b2)})
        if (!detail::is_device_accessible(p) || (reinterpret_cast<uintptr_t>(p) & 15)) return SIFT_ERR_INVALID_ARG;
    return SIFT_OK;
}

MlpModel to_model(const sift_mlp* m) {
    MlpModel mm;
    mm.w1 = static_cast<const __nv_bfloat16*>(m->w1);
    mm.b1 = m->b1;
    mm.w2 = static_cast<const __nv_bfloat16*>(m->w2);
    mm.b2 = m->b2;
    mm.k = m->k;
    return mm;
}

bool aligned_dev(const void* p) {
    return p && !(reinterpret_cast<uintptr_t>(p) & 15) && detail::is_device_accessible(p);
}

}  // namespace

int mlp_hash(const uint8_t* x, uint32_t n, const sift_mlp* model, uint32_t* codes, float* z, void* stream) {
    SIFT_TRY(check_model(model));
    if (n == 0) return SIFT_OK;
    if (!aligned_dev(x) || !codes || !detail::is_device_accessible(codes) || (z && !detail::is_device_accessible(z)) ||
        n > 0x7fffffffu)
        return SIFT_ERR_INVALID_ARG;
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    const MlpModel m = to_model(model);
    CUtensorMap w1map, w2map;
    SIFT_TRY(encode_model(m, &w1map, &w2map));
    CUtensorMap xmap;
    SIFT_TRY(detail::encode_u8_rows(&xmap, x, n, 128));
    SIFT_CUDA(launch_mlp_hash(xmap, static_cast<int>(n), w1map, w2map, m.b1, m.b2, m.k, codes, z, cp->d_status,
                              cp->num_sms, static_cast<cudaStream_t>(stream)));
    ++detail::g_launches;
    return SIFT_OK;
}

int mlp_match(const uint8_t* q, const uint8_t* r, uint32_t q_n_, uint32_t r_n_, const sift_mlp* model, int n_probes,
              int min_candidates, float max_dist, float threshold, uint32_t* matches, int32_t* nn_idx,
              float* nn_dist, uint32_t* candidates, uint32_t* fallback_count, void* stream) {
    SIFT_TRY(check_model(model));
    if (q_n_ > 0x7fffffffu / 64 || r_n_ > 0x7fffffffu / 64 || n_probes < 1 || n_probes > 64 || min_candidates < 0 ||
        !(max_dist >= 0.0f))
        return SIFT_ERR_INVALID_ARG;
    if (fallback_count) *fallback_count = 0;
    if (q_n_ == 0) return SIFT_OK;
    if (!aligned_dev(q) || (r_n_ > 0 && !aligned_dev(r))) return SIFT_ERR_INVALID_ARG;
    for (const void* o : {static_cast<const void*>(matches), static_cast<const void*>(nn_idx),
                          static_cast<const void*>(nn_dist), static_cast<const void*>(candidates)})
        if (o && !detail::is_device_accessible(o)) return SIFT_ERR_INVALID_ARG;
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    DeviceCtx& c = *cp;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    detail::ArenaLock lk(c, st);
    const int q_n = static_cast<int>(q_n_), r_n = static_cast<int>(r_n_);
    const MlpModel m = to_model(model);
    const int k = m.k;
    const int top = k < kLshMaxTopBits ? k : kLshMaxTopBits;
    const int shift = k - top, nbins = 1 << top;
    const int flip = k < 6 ? k : 6;
    detail::Layout L;
    const size_t o_cr = L.take(static_cast<size_t>(r_n) * 4 + 16);
    const size_t o_cq = L.take(static_cast<size_t>(q_n) * 4);
    const size_t o_z = L.take(static_cast<size_t>(q_n) * k * 4);
    const size_t o_pc = L.take(static_cast<size_t>(n_probes) * q_n * 4);
    const size_t o_hist = L.take(static_cast<size_t>(nbins) * 4);
    const size_t o_start = L.take(static_cast<size_t>(nbins + 1) * 4);
    const size_t o_order = L.take(static_cast<size_t>(r_n) * 4 + 16);
    const size_t o_ocode = L.take(static_cast<size_t>(r_n) * 4 + 16);
    const size_t o_cnt = L.take(static_cast<size_t>(q_n) * 4);
    const size_t o_dist = L.take(static_cast<size_t>(q_n) * 8);  // distances when the caller takes none
    FallbackScratch fs{};
    fallback_layout(L, q_n, r_n, c.num_sms / 2, true, fs);
    SIFT_TRY(detail::ensure_arena(c, L.off));
    char* A = c.arena;
    auto U32 = [&](size_t o) { return reinterpret_cast<uint32_t*>(A + o); };
    auto I32 = [&](size_t o) { return reinterpret_cast<int32_t*>(A + o); };
    uint32_t* counts = candidates ? candidates : U32(o_cnt);
    float* dist = nn_dist ? nn_dist : reinterpret_cast<float*>(A + o_dist);

    CUtensorMap w1map, w2map;
    SIFT_TRY(encode_model(m, &w1map, &w2map));
    int launches = 0;
    if (r_n > 0) {
        CUtensorMap rmap;
        SIFT_TRY(detail::encode_u8_rows(&rmap, r, r_n, 128));
        SIFT_CUDA(launch_mlp_hash(rmap, r_n, w1map, w2map, m.b1, m.b2, k, U32(o_cr), nullptr, c.d_status, c.num_sms,
                                  st));
        SIFT_CUDA(launch_lsh_buckets(U32(o_cr), r_n, 1, shift, nbins, I32(o_hist), I32(o_start), I32(o_order),
                                     U32(o_ocode), c.num_sms, st));
        launches += 4;
    } else {
        SIFT_CUDA(cudaMemsetAsync(I32(o_start), 0, static_cast<size_t>(nbins + 1) * 4, st));
    }
    CUtensorMap qmap_h;
    SIFT_TRY(detail::encode_u8_rows(&qmap_h, q, q_n, 128));
    SIFT_CUDA(launch_mlp_hash(qmap_h, q_n, w1map, w2map, m.b1, m.b2, k, U32(o_cq), reinterpret_cast<float*>(A + o_z),
                              c.d_status, c.num_sms, st));
    SIFT_CUDA(launch_probe_codes(U32(o_cq), reinterpret_cast<float*>(A + o_z), q_n, k, flip, n_probes, U32(o_pc), st));
    SIFT_CUDA(launch_lsh_scan(q, r, q_n, r_n, 1, n_probes, shift, nbins, U32(o_pc), I32(o_start), I32(o_order),
                              U32(o_ocode), threshold, threshold > 0.f ? 1 : 0, 1.0f, matches, counts, nn_idx, dist,
                              st));
    launches += 3;
    detail::g_launches += launches;
    if ((min_candidates <= 0 && max_dist <= 0.0f) || r_n == 0) return SIFT_OK;

    // ---- exact fallback for queries with too few candidates
    return exact_fallback(c, A, fs, q, r, q_n, r_n, nullptr, counts, dist, min_candidates, max_dist, threshold,
                          matches, nn_idx, nn_dist, fallback_count, st);
}

int mlp_loss_grad(const uint8_t* x, int B, int k, const float* params, float neg_w, float bal_w, float* grads,
                  float* loss_host) {
    if (B < 1 || k < 1 || k > kMlpMaxBits || !loss_host || !aligned_dev(x) || !aligned_dev(params) ||
        !aligned_dev(grads))
        return SIFT_ERR_INVALID_ARG;
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    DeviceCtx& c = *cp;
    detail::ArenaLock lk(c, nullptr);
    const int R = 3 * B;
    detail::Layout L;
    const size_t o_w1b = L.take(kMlpHidden * kMlpIn * 2);
    const size_t o_w2b = L.take(kMlpOutRows * kMlpHidden * 2);
    const size_t o_h = L.take(static_cast<size_t>(R) * kMlpHidden * 4);
    const size_t o_t = L.take(static_cast<size_t>(R) * kMlpOutRows * 4);
    const size_t o_dz = L.take(static_cast<size_t>(R) * kMlpOutRows * 4);
    const size_t o_da = L.take(static_cast<size_t>(R) * kMlpHidden * 4);
    const size_t o_cs = L.take(kMlpOutRows * 4);
    const size_t o_loss = L.take(16);
    SIFT_TRY(detail::ensure_arena(c, L.off));
    char* A = c.arena;
    cudaStream_t st = nullptr;
    const MlpParams p = mlp_params_at(const_cast<float*>(params));
    const MlpParams g = mlp_params_at(grads);
    auto* w1b = reinterpret_cast<__nv_bfloat16*>(A + o_w1b);
    auto* w2b = reinterpret_cast<__nv_bfloat16*>(A + o_w2b);
    SIFT_CUDA(cudaMemsetAsync(w2b, 0, kMlpOutRows * kMlpHidden * 2, st));
    SIFT_CUDA(launch_mlp_export(p, k, w1b, w2b, nullptr, nullptr, st));
    MlpTrainBufs tb{reinterpret_cast<float*>(A + o_h), reinterpret_cast<float*>(A + o_t),
                    reinterpret_cast<float*>(A + o_dz), reinterpret_cast<float*>(A + o_da),
                    reinterpret_cast<float*>(A + o_cs), reinterpret_cast<float*>(A + o_loss)};
    SIFT_CUDA(launch_mlp_loss_grad(x, B, k, p, w1b, w2b, MlpLossWeights{neg_w, bal_w}, tb, g, st));
    SIFT_CUDA(cudaMemcpyAsync(loss_host, tb.loss, 4 * sizeof(float), cudaMemcpyDeviceToHost, st));
    SIFT_CUDA(cudaStreamSynchronize(st));
    detail::g_launches += 9;
    return detail::collect_device_status(c, st);
}

int mlp_train(const uint8_t* base, uint32_t r_n, const uint8_t* tq, uint32_t t_n, int k, int steps, int batch,
              float lr, float neg_w, float bal_w, unsigned long long seed, void* w1_out, float* b1_out, void* w2_out,
              float* b2_out, float* params_out, float* loss_curve) {
    if (k < 1 || k > kMlpMaxBits || steps < 0 || batch < 32 || batch % 32 || r_n == 0 || t_n == 0 ||
        r_n > 0x7fffffffu / 64 || t_n > 0x7fffffffu / 64 || !aligned_dev(base) || !aligned_dev(tq))
        return SIFT_ERR_INVALID_ARG;
    for (const void* o : {w1_out, static_cast<void*>(b1_out), w2_out, static_cast<void*>(b2_out)})
        if (!aligned_dev(o)) return SIFT_ERR_INVALID_ARG;
    if (params_out && !aligned_dev(params_out)) return SIFT_ERR_INVALID_ARG;
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(detail::ensure_ready(cp, dev));
    // Labels: exact nearest neighbour of every training query (the exact kernel).
    int32_t* nn = nullptr;
    SIFT_CUDA(cudaMalloc(&nn, static_cast<size_t>(t_n) * 8));
    MatchArgs ma;
    ma.q = tq;
    ma.r = base;
    ma.type = SIFT_U8_DEVICE;
    ma.q_n = t_n;
    ma.r_n = r_n;
    ma.nn_idx = nn;
    ma.sync = true;
    int rc = exact_match(ma);
    if (rc != SIFT_OK) {
        cudaFree(nn);
        return rc;
    }
    // Training buffers (one-off allocations: training is not on the search path).
    const int R = 3 * batch;
    const size_t np = kMlpParamCount;
    std::vector<void*> owned;
    auto alloc = [&](size_t bytes) -> char* {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        owned.push_back(p);
        return static_cast<char*>(p);
    };
    char* pm = alloc(4 * np * sizeof(float));
    char* w1b = alloc(kMlpHidden * kMlpIn * 2);
    char* w2b = alloc(kMlpOutRows * kMlpHidden * 2);
    char* xb = alloc(static_cast<size_t>(R) * kMlpIn);
    char* h = alloc(static_cast<size_t>(R) * kMlpHidden * 4);
    char* t = alloc(static_cast<size_t>(R) * kMlpOutRows * 4);
    char* dz = alloc(static_cast<size_t>(R) * kMlpOutRows * 4);
    char* da = alloc(static_cast<size_t>(R) * kMlpHidden * 4);
    char* cs = alloc(kMlpOutRows * 4);
    char* losses = alloc(static_cast<size_t>(steps + 1) * 4 * sizeof(float));
    auto release = [&]() {
        for (void* p : owned) cudaFree(p);
        cudaFree(nn);
    };
    if (owned.size() != 10) {
        release();
        return SIFT_ERR_ALLOC;
    }
    float* P = reinterpret_cast<float*>(pm);
    const MlpParams p = mlp_params_at(P), g = mlp_params_at(P + np), mo = mlp_params_at(P + 2 * np),
                    vo = mlp_params_at(P + 3 * np);
    // Initial weights: W1 ~ N(0, 1/64) (pre-activations ~ N(0, 1) for inputs
    // of norm 512 / 64), W2 rows < k ~ N(0, 1/128), biases 0.
    std::vector<float> init(np, 0.0f);
    std::mt19937_64 gen(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    for (int e = 0; e < kMlpHidden * kMlpIn; ++e) init[e] = nd(gen) * 0.125f;
    float* w2i = init.data() + kMlpHidden * kMlpIn + kMlpHidden;
    for (int mrow = 0; mrow < k; ++mrow)
        for (int j = 0; j < kMlpHidden; ++j) w2i[mrow * kMlpHidden + j] = nd(gen) * 0.0884f;
    cudaStream_t st = nullptr;
    rc = SIFT_OK;
    auto step_rc = [&](cudaError_t e) {
        if (rc == SIFT_OK && e != cudaSuccess) rc = detail::map_cuda(e);
    };
    step_rc(cudaMemcpy(P, init.data(), np * sizeof(float), cudaMemcpyHostToDevice));
    step_rc(cudaMemset(P + np, 0, 3 * np * sizeof(float)));
    step_rc(cudaMemset(w2b, 0, kMlpOutRows * kMlpHidden * 2));
    step_rc(launch_mlp_export(p, k, reinterpret_cast<__nv_bfloat16*>(w1b), reinterpret_cast<__nv_bfloat16*>(w2b),
                              nullptr, nullptr, st));
    MlpTrainBufs tb{reinterpret_cast<float*>(h), reinterpret_cast<float*>(t), reinterpret_cast<float*>(dz),
                    reinterpret_cast<float*>(da), reinterpret_cast<float*>(cs), nullptr};
    const MlpLossWeights lw{neg_w, bal_w};
    for (int s = 0; s < steps && rc == SIFT_OK; ++s) {
        tb.loss = reinterpret_cast<float*>(losses) + 4 * s;
        step_rc(launch_mlp_gather(tq, static_cast<int>(t_n), nn, base, static_cast<int>(r_n), batch, seed, s,
                                  reinterpret_cast<uint8_t*>(xb), st));
        step_rc(launch_mlp_loss_grad(reinterpret_cast<uint8_t*>(xb), batch, k, p,
                                     reinterpret_cast<__nv_bfloat16*>(w1b), reinterpret_cast<__nv_bfloat16*>(w2b), lw,
                                     tb, g, st));
        step_rc(launch_mlp_adam(p, g, mo, vo, k, s + 1, lr, reinterpret_cast<__nv_bfloat16*>(w1b),
                                reinterpret_cast<__nv_bfloat16*>(w2b), st));
        detail::g_launches += 12;
    }
    step_rc(launch_mlp_export(p, k, static_cast<__nv_bfloat16*>(w1_out), static_cast<__nv_bfloat16*>(w2_out), b1_out,
                              b2_out, st));
    if (params_out) step_rc(cudaMemcpyAsync(params_out, P, np * sizeof(float), cudaMemcpyDeviceToDevice, st));
    if (loss_curve && steps > 0) {
        std::vector<float> lv(static_cast<size_t>(steps) * 4);
        step_rc(cudaMemcpy(lv.data(), losses, lv.size() * sizeof(float), cudaMemcpyDeviceToHost));
        for (int s = 0; s < steps; ++s) loss_curve[s] = lv[4 * static_cast<size_t>(s)];
    }
    step_rc(cudaDeviceSynchronize());
    release();
    if (rc == SIFT_OK) {
        std::lock_guard<std::mutex> lk(cp->mu);
        rc = detail::collect_device_status(*cp, st);
    }
    return rc;
}

}  // namespace sift

extern "C" {

int sift_mlp_hash(const uint8_t* x, uint32_t n, const sift_mlp* model, uint32_t* codes, float* z, void* stream) {
    return sift::mlp_hash(x, n, model, codes, z, stream);
}

int sift_mlp_match(const uint8_t* q, const uint8_t* r, uint32_t q_n, uint32_t r_n, const sift_mlp* model,
                   int n_probes, int min_candidates, float max_dist, float threshold, uint32_t* matches,
                   int32_t* nn_idx, float* nn_dist, uint32_t* candidates, uint32_t* fallback_count, void* stream) {
    return sift::mlp_match(q, r, q_n, r_n, model, n_probes, min_candidates, max_dist, threshold, matches, nn_idx,
                           nn_dist, candidates, fallback_count, stream);
}

int sift_mlp_train(const uint8_t* base, uint32_t r_n, const uint8_t* train_q, uint32_t t_n, int k, int steps,
                   int batch, float lr, float neg_weight, float balance_weight, unsigned long long seed, void* w1,
                   float* b1, void* w2, float* b2, float* params_out, float* loss_curve) {
    return sift::mlp_train(base, r_n, train_q, t_n, k, steps, batch, lr, neg_weight, balance_weight, seed, w1, b1, w2,
                           b2, params_out, loss_curve);
}

int sift_mlp_loss_grad(const uint8_t* x, int batch, int k, const float* params, float neg_weight,
                       float balance_weight, float* grads, float* loss) {
    return sift::mlp_loss_grad(x, batch, k, params, neg_weight, balance_weight, grads, loss);
}

}  // extern "C"
