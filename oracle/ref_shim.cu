// Test-infrastructure shim: exposes the reference implementation's own
// functions (compiled unmodified from the reference sources by oracle/Makefile)
// under C linkage so that Python tests can call them through ctypes.
//
// This file is the checker, never the product: only tests/, the smoke check and
// bench.py's CPU-baseline / reference legs load the library built from it.
//
// Every wrapper forwards to a reference function with the reference's own
// argument conventions:
//   host_brute            src/knn_brute.cu:801   (CPU brute-force 2-NN, float4 {d1,d2,i1,i2})
//   device_brute          src/knn_brute.cu:619   (naive CUDA brute force)
//   cublas_2nn_f          src/knn_brute.cu:523   (FP32 cuBLAS GEMM + min_dist_f)
//   cublas_2nn_sift       src/knn_brute.cu:24    (FP16 cuBLAS GEMM + find_matches ratio test)
//   lsh_thread_sort_reduce src/lsh_h.cu:565      (sign-bit hash codes, thrust sort, host RLE)
// The hash-dot GEMM in ref_lsh_buckets is issued exactly as src/lsh_h.cu:909
// issues it (cublasHgemm, OP_T/OP_N, alpha=1, beta=0, FP16 in/out).
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "cublas_v2.h"
#include "knn_brute.h"
#include "lsh_h.h"

extern "C" {

// CPU brute force over query rows [q_begin, q_end), calling the unmodified
// reference host_brute on each thread's slice. nthreads <= 1 runs inline.
void ref_host_brute_mt(float* q, float* r, int q_n, int r_n, float4* sorted, int nthreads) {
    if (nthreads <= 1 || q_n < 2) {
        host_brute((des_t_f*)q, (des_t_f*)r, q_n, r_n, sorted);
        return;
    }
    std::vector<std::thread> th;
    int per = (q_n + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; ++t) {
        int b = t * per, e = b + per < q_n ? b + per : q_n;
        if (b >= e) break;
        th.emplace_back([=]() { host_brute((des_t_f*)q + b, (des_t_f*)r, e - b, r_n, sorted + b); });
    }
    for (auto& x : th) x.join();
}

// Device-side reference calls. All pointers are device (or managed) memory
// except where noted; the call synchronises before returning.
int ref_device_brute(float* q_dev, float* r_dev, int q_n, int r_n, float4* sorted_dev) {
    device_brute((des_t_f*)q_dev, (des_t_f*)r_dev, q_n, r_n, sorted_dev);
    return (int)cudaDeviceSynchronize();
}

int ref_cublas_2nn_f(float* q_dev, float* r_dev, int q_n, int r_n, float4* sorted_dev) {
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return -1;
    cublas_2nn_f((des_t_f*)q_dev, (des_t_f*)r_dev, q_n, r_n, sorted_dev, h);
    int rc = (int)cudaDeviceSynchronize();
    cublasDestroy(h);
    return rc;
}

// type must be 1 (FLOAT_DEVICE); type 2 frees an uninitialised pointer in the
// reference (src/knn_brute.cu:148-151,195) and is never used here.
int ref_cublas_2nn_sift(float* q_dev, float* r_dev, uint32_t q_n, uint32_t r_n, uint32_t* matches_dev,
                        float threshold, int stream_n, size_t use, int warps) {
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return -1;
    cublas_2nn_sift(q_dev, r_dev, 1, q_n, r_n, matches_dev, threshold, h, stream_n, use, warps);
    int rc = (int)cudaDeviceSynchronize();
    cublasDestroy(h);
    return rc;
}

// Hash codes and buckets of the reference LSH for n FP16 points and given FP16
// hyperplanes (nbits rows of 128 halves, nbits even). Outputs (host arrays):
// code[n] (bit j set when dot_j < 0), index[n] (point ids sorted by code),
// buckets[2*n] ({first id, count} pairs as produced by the host RLE) and the
// bucket count. Points and planes are host arrays copied to the device here.
int ref_lsh_buckets(const uint16_t* points_h, uint32_t n, const uint16_t* planes_h, int nbits,
                    int* code_h, int* index_h, int* buckets_h, int* n_buckets) {
    if (nbits % 2) return -2;
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return -1;
    cudaStream_t st;
    cudaStreamCreate(&st);
    half *pts, *planes, *dot;
    int *code_d, *index_d;
    cudaMalloc(&pts, sizeof(half) * 128 * (size_t)n);
    cudaMalloc(&planes, sizeof(half) * 128 * (size_t)nbits);
    cudaMalloc(&dot, sizeof(half) * (size_t)nbits * n);
    cudaMalloc(&code_d, sizeof(int) * (size_t)n);
    cudaMalloc(&index_d, sizeof(int) * (size_t)n);
    cudaMemcpy(pts, points_h, sizeof(half) * 128 * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(planes, planes_h, sizeof(half) * 128 * (size_t)nbits, cudaMemcpyHostToDevice);
    half a = 1.0f, b = 0.0f;
    cublasSetStream(h, st);
    cublasHgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, nbits, n, 128, &a, planes, 128, pts, 128, &b, dot, nbits);
    int* code_pinned;
    int* index_pinned;
    int2* buckets_pinned;
    cudaMallocHost(&code_pinned, sizeof(int) * (size_t)n);
    cudaMallocHost(&index_pinned, sizeof(int) * (size_t)n);
    cudaMallocHost(&buckets_pinned, sizeof(int2) * (size_t)n);
    int nb = 0;
    lsh_thread_sort_reduce((des_t_h2*)pts, n, (des_t_h2*)planes, nbits, (half2*)dot, code_pinned, code_d,
                           index_pinned, index_d, buckets_pinned, st, nb);
    int rc = (int)cudaStreamSynchronize(st);
    memcpy(code_h, code_pinned, sizeof(int) * (size_t)n);
    memcpy(index_h, index_pinned, sizeof(int) * (size_t)n);
    memcpy(buckets_h, buckets_pinned, sizeof(int2) * (size_t)nb);
    *n_buckets = nb;
    cudaFreeHost(code_pinned);
    cudaFreeHost(index_pinned);
    cudaFreeHost(buckets_pinned);
    cudaFree(pts);
    cudaFree(planes);
    cudaFree(dot);
    cudaFree(code_d);
    cudaFree(index_d);
    cudaStreamDestroy(st);
    cublasDestroy(h);
    return rc;
}

}  // extern "C"
