// Test program (not product code): a C++ caller compiled against the
// reference's own headers (include/knn_brute.h, include/lsh_h.h) and linked to
// libsift2nn.so. It calls the reference entry points by their C++ (mangled)
// names -- cublas_2nn_sift, cublas_2nn_f, device_brute, host_brute, lsh_gpu
// (include/knn_brute.h:14,18,22,29, include/lsh_h.h:69) -- which resolve to
// the library's forwarders (matching_sift_b200/csrc/compat_cxx.cpp), and
// writes every output for tests/test_cxx_callers_gpu.py to check.
//
// Usage: reference_caller DIR Q_N R_N
//   DIR/q.f32, DIR/r.f32: float [n][128] inputs; writes DIR/sift.u32,
//   DIR/f.f32, DIR/device_brute.f32, DIR/host_brute.f32, DIR/lsh.u32 and
//   DIR/status.txt (the return codes).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "knn_brute.h"
#include "lsh_h.h"

static bool read_file(const std::string& path, void* p, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    const bool ok = std::fread(p, 1, bytes, f) == bytes;
    std::fclose(f);
    return ok;
}

static bool write_file(const std::string& path, const void* p, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(p, 1, bytes, f) == bytes;
    std::fclose(f);
    return ok;
}

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s DIR Q_N R_N\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const int q_n = std::atoi(argv[2]), r_n = std::atoi(argv[3]);
    std::vector<float> q(static_cast<size_t>(q_n) * 128), r(static_cast<size_t>(r_n) * 128);
    if (!read_file(dir + "/q.f32", q.data(), q.size() * 4) || !read_file(dir + "/r.f32", r.data(), r.size() * 4))
        return 3;
    des_t_f *qd = nullptr, *rd = nullptr;
    uint32_t* matches = nullptr;
    float4* sorted = nullptr;
    if (cudaMalloc(&qd, q.size() * 4) != cudaSuccess || cudaMalloc(&rd, r.size() * 4) != cudaSuccess ||
        cudaMallocManaged(&matches, q_n * sizeof(uint32_t)) != cudaSuccess ||
        cudaMallocManaged(&sorted, q_n * sizeof(float4)) != cudaSuccess)
        return 4;
    cudaMemcpy(qd, q.data(), q.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(rd, r.data(), r.size() * 4, cudaMemcpyHostToDevice);
    cublasHandle_t handle = nullptr;  // the library uses no cuBLAS; the reference's callers pass theirs

    // FLOAT_DEVICE (type 1) as in the reference's enum (src/knn_brute.cu:15-19).
    const int rc_sift = cublas_2nn_sift(qd, rd, 1, q_n, r_n, matches, 0.8f, handle, 1, 0, 17);
    cudaDeviceSynchronize();
    bool ok = write_file(dir + "/sift.u32", matches, q_n * sizeof(uint32_t));
    cublas_2nn_f(qd, rd, q_n, r_n, sorted, handle);
    cudaDeviceSynchronize();
    ok &= write_file(dir + "/f.f32", sorted, q_n * sizeof(float4));
    device_brute(qd, rd, q_n, r_n, sorted);
    cudaDeviceSynchronize();
    ok &= write_file(dir + "/device_brute.f32", sorted, q_n * sizeof(float4));
    std::vector<float4> hs(q_n);
    host_brute(reinterpret_cast<des_t_f*>(q.data()), reinterpret_cast<des_t_f*>(r.data()), q_n, r_n, hs.data());
    ok &= write_file(dir + "/host_brute.f32", hs.data(), q_n * sizeof(float4));
    // lsh_gpu draws its +/-1 hyperplanes with rand(): seed it as a caller would.
    std::srand(1234);
    const int rc_lsh = lsh_gpu(qd, rd, 1, q_n, r_n, matches, 0.8f, handle, 2, 3, 0, 10);
    cudaDeviceSynchronize();
    ok &= write_file(dir + "/lsh.u32", matches, q_n * sizeof(uint32_t));
    FILE* f = std::fopen((dir + "/status.txt").c_str(), "w");
    if (!f) return 5;
    std::fprintf(f, "%d %d\n", rc_sift, rc_lsh);
    std::fclose(f);
    cudaFree(qd);
    cudaFree(rd);
    cudaFree(matches);
    cudaFree(sorted);
    return ok ? 0 : 6;
}
