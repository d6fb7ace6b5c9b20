// TMEM -> register read throughput of this GPU (the rate at which an
// epilogue can drain tcgen05 accumulators), per SM and per warp.
//
// One CTA per SM (200 KB of dynamic shared memory keeps a second one out),
// 512 TMEM columns allocated; WARPS warps, warp w reading lane quarter w % 4.
// Each iteration issues L loads of tcgen05.ld.32x32b.x32 (4 KB per warp) or
// one x64 load, then one tcgen05.wait::ld, then folds the values into a
// checksum so nothing is dead. Cycles from clock64 per warp.
//
//   make -C matching_sift_b200 tmem_bw && matching_sift_b200/tmem_bw
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>
#include "csrc/ptx.cuh"

using namespace sift;

namespace {

// Redefines the registers in place (no instruction): uses of v cannot move
// above the preceding volatile asm (the tcgen05.wait::ld).
__device__ __forceinline__ void reg_pin(uint32_t (&v)[32]) {
    asm volatile(""
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                   "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),
                   "+r"(v[15]), "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]),
                   "+r"(v[22]), "+r"(v[23]), "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]),
                   "+r"(v[29]), "+r"(v[30]), "+r"(v[31])
                 :
                 : "memory");
}

template <int WARPS, int L>
__global__ void __launch_bounds__(WARPS * 32, 1) read_x32(int iters, unsigned long long* cycles, unsigned* sink) {
    __shared__ uint32_t tbase;
    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        ptx::tmem_alloc(ptx::smem_u32(&tbase), 512);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t t0 = tbase + (static_cast<uint32_t>((warp & 3) * 32) << 16);
    uint32_t acc = 0;
    uint32_t v[L][32];
    const unsigned long long c0 = clock64();
    for (int i = 0; i < iters; ++i) {
        // columns (multiple of 32) + 32 <= 512
        #pragma unroll
        for (int j = 0; j < L; ++j) ptx::tmem_ld32(t0 + (((i * L + j) * 32 + (warp >> 2) * 128) & 511), v[j]);
        ptx::tmem_ld_wait(v[0]);
        #pragma unroll
        for (int j = 1; j < L; ++j) reg_pin(v[j]);
        #pragma unroll
        for (int j = 0; j < L; ++j)
            #pragma unroll
            for (int c = 0; c < 32; ++c) acc ^= v[j][c];
    }
    const unsigned long long c1 = clock64();
    ptx::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc(tbase, 512);
    }
    if ((threadIdx.x & 31) == 0) atomicMax(cycles + blockIdx.x, c1 - c0);
    if (acc == 0x12345678u) sink[0] = acc;
}

template <int WARPS>
void run(unsigned long long* d_cycles, unsigned* sink, int nsm, auto kernel, double bytes_per_iter_warp,
         const char* label, int loads) {
    const int iters = 4096;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    for (int rep = 0; rep < 2; ++rep) {  // the first run warms up
        cudaMemset(d_cycles, 0, nsm * sizeof(unsigned long long));
        kernel<<<nsm, WARPS * 32, 200 * 1024>>>(iters, d_cycles, sink);
        const cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            std::printf("error: %s\n", cudaGetErrorString(e));
            return;
        }
    }
    unsigned long long h[1024];
    cudaMemcpy(h, d_cycles, nsm * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    double sum = 0;
    for (int i = 0; i < nsm; ++i) sum += static_cast<double>(h[i]);
    const double cyc = sum / nsm;
    const double bytes = WARPS * iters * bytes_per_iter_warp;
    std::printf("%-4s warps %2d loads/wait %d: %6.1f B/clk/SM  %5.1f B/clk/warp\n", label, WARPS, loads,
                bytes / cyc, bytes / cyc / WARPS);
}

}  // namespace

int main() {
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
    if (nsm <= 0 || nsm > 1024) return 1;
    unsigned long long* d_cycles = nullptr;
    unsigned* sink = nullptr;
    cudaMalloc(&d_cycles, 1024 * sizeof(unsigned long long));
    cudaMalloc(&sink, 4);
    run<4>(d_cycles, sink, nsm, read_x32<4, 1>, 4096.0, "x32", 1);
    run<4>(d_cycles, sink, nsm, read_x32<4, 4>, 4 * 4096.0, "x32", 4);
    run<8>(d_cycles, sink, nsm, read_x32<8, 1>, 4096.0, "x32", 1);
    run<8>(d_cycles, sink, nsm, read_x32<8, 2>, 2 * 4096.0, "x32", 2);
    run<16>(d_cycles, sink, nsm, read_x32<16, 1>, 4096.0, "x32", 1);
    run<16>(d_cycles, sink, nsm, read_x32<16, 2>, 2 * 4096.0, "x32", 2);
    cudaFree(d_cycles);
    cudaFree(sink);
    return 0;
}
