// C++-linkage forwarders with the reference's exact signatures, so C++ code
// compiled against the reference headers (include/knn_brute.h,
// include/lsh_h.h) links against libsift2nn.so unchanged: the mangled symbols
// below are the ones such callers reference (e.g.
// _Z15cublas_2nn_siftPvS_ijjPjfP13cublasContextimi). This translation unit
// must not see the extern "C" declarations of the same names.
#include <cstddef>
#include <cstdint>
#include <vector_types.h>  // float4

struct cublasContext;
typedef struct cublasContext* cublasHandle_t;
typedef float des_t_f[128];
#define SIFT_CXX_API __attribute__((visibility("default")))

extern "C" {
int sift_impl_cublas_2nn_sift(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n,
                              uint32_t* matches, float threshold);
void sift_impl_cublas_2nn_f(void* q_points, void* r_points, int q_n, int r_n, void* sorted);
void sift_impl_device_brute(void* q_points, void* r_points, int q_n, int r_n, void* sorted);
void sift_impl_host_brute(void* q_points, void* r_points, int q_n, int r_n, void* sorted);
int sift_impl_lsh_gpu(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n, uint32_t* matches, int l,
                      int nbits);
}

// include/knn_brute.h:22
SIFT_CXX_API int cublas_2nn_sift(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n, uint32_t* matches,
                    float threshold, cublasHandle_t, int, size_t, int) {
    return sift_impl_cublas_2nn_sift(q_points, r_points, type, q_n, r_n, matches, threshold);
}

// include/knn_brute.h:18
SIFT_CXX_API void cublas_2nn_f(des_t_f* q_points, des_t_f* r_points, int q_n, int r_n, float4* sorted, cublasHandle_t) {
    sift_impl_cublas_2nn_f(q_points, r_points, q_n, r_n, sorted);
}

// include/knn_brute.h:14
SIFT_CXX_API void device_brute(des_t_f* q_points, des_t_f* r_points, int q_n, int r_n, float4* sorted) {
    sift_impl_device_brute(q_points, r_points, q_n, r_n, sorted);
}

// include/knn_brute.h:29
SIFT_CXX_API void host_brute(des_t_f* q_points, des_t_f* r_points, int q_points_size, int r_points_size, float4* sorted) {
    sift_impl_host_brute(q_points, r_points, q_points_size, r_points_size, sorted);
}

// include/lsh_h.h:69
SIFT_CXX_API int lsh_gpu(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n, uint32_t* matches,
                         float, cublasHandle_t, int, int l, int, int nbits) {
    return sift_impl_lsh_gpu(q_points, r_points, type, q_n, r_n, matches, l, nbits);
}
