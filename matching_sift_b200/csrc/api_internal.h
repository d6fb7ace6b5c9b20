// Internal interface between the C ABI entry points and the implementation.
#pragma once
#include <cstdint>
#include "sift2nn.h"

namespace sift {

struct MatchArgs {
    const void* q = nullptr;
    const void* r = nullptr;
    int type = SIFT_U8_DEVICE;
    uint32_t q_n = 0, r_n = 0;
    int metric = SIFT_METRIC_L2;
    float threshold = 0.8f;
    uint32_t* matches = nullptr;
    sift_float4* sorted = nullptr;
    int32_t* nn_idx = nullptr;
    float* nn_dist = nullptr;
    void* stream = nullptr;
    bool sync = false;  // synchronise and collect the device status before returning
};

int exact_match(const MatchArgs& a);

struct LshArgs {
    const void* q = nullptr;
    const void* r = nullptr;
    int type = SIFT_U8_DEVICE;
    uint32_t q_n = 0, r_n = 0;
    const int8_t* planes = nullptr;  // [L][k][128] int8, host or device
    int L = 1, k = 16;
    float threshold = 0.8f;
    bool ratio = false;  // apply the ratio test to `matches`
    int probes = 1;      // buckets searched per table (query-directed multi-probe when > 1)
    uint32_t* candidates = nullptr;  // optional device [q_n]: base rows compared per query
    uint32_t* matches = nullptr;
    int32_t* nn_idx = nullptr;
    float* nn_dist = nullptr;
    void* stream = nullptr;
    bool sync = false;
};
int lsh_match(const LshArgs& a);
int mlp_train(const uint8_t* base, uint32_t r_n, const uint8_t* tq, uint32_t t_n, int k, int steps, int batch,
              float lr, float neg_w, float bal_w, unsigned long long seed, void* w1_out, float* b1_out, void* w2_out,
              float* b2_out, float* params_out, float* loss_curve);
int lsh_hash(const uint8_t* x, uint32_t n, const int8_t* planes, int L, int k, uint32_t* codes, void* stream);
int lsh_buckets(const uint32_t* codes, uint32_t n, int L, int k, int* start, int* order, uint32_t* ocode,
                void* stream);
void reference_planes(int L, int nbits, int8_t* out);
int stream_status(void* stream);
void set_last_status(int s);
int profile_collect(int tag, double* total_ms, int* launches);
long long launch_count();
void profile_enable(bool on);
int set_variant(int v);
int last_status();

}  // namespace sift

// C-linkage implementations used by the mangled C++ forwarders (compat_cxx.cpp).
extern "C" {
int sift_impl_cublas_2nn_sift(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n,
                              uint32_t* matches, float threshold);
void sift_impl_cublas_2nn_f(void* q_points, void* r_points, int q_n, int r_n, void* sorted);
void sift_impl_device_brute(void* q_points, void* r_points, int q_n, int r_n, void* sorted);
void sift_impl_host_brute(void* q_points, void* r_points, int q_n, int r_n, void* sorted);
int sift_impl_lsh_gpu(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n, uint32_t* matches, int l,
                      int nbits);
}
