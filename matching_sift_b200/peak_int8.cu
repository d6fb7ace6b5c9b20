// Dense int8 tensor-core peak of this GPU, and the issue cost of the
// synchronisation the search kernels put between MMAs.
//
// One CTA per SM (or one CTA pair per TPC for cta_group::2), operands resident
// in shared memory, one thread issuing back-to-back tcgen05.mma.kind::i8 with
// K = 32 into TMEM, then one commit + bounded wait. MODE adds, per group of 4
// MMAs: 1 = a tcgen05.commit, 2 = + tcgen05.fence::after_thread_sync,
// 3 = + an mbarrier.try_wait on an already completed phase. ISSUERS = 2 splits
// the same MMAs between two threads (lane 0 of warps 0 and 1, each with its
// own half of TMEM and its own barriers): whether a second issuing thread
// hides the first one's synchronisation.
// The MAC/clk/SM figure of MODE 0 is the roofline denominator bench.py uses.
//
// chain_kernel below measures the accumulator hand-off between the MMA issuer
// and the epilogue warps.
//
//   make -C matching_sift_b200 peak && matching_sift_b200/peak_int8
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "csrc/ptx.cuh"

using namespace sift;

template <int M, int N, bool PAIR, int MODE, int ISSUERS>
__global__ void __launch_bounds__(128, 1) bench_kernel(int iters, unsigned long long* cycles) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t* base = sm + ((1024 - (ptx::smem_u32(sm) & 1023)) & 1023);
    __shared__ uint64_t bar[2];
    __shared__ uint64_t side[2][4];
    __shared__ uint32_t tbase;
    __shared__ int flag_abort, flag_err;
    const int warp = threadIdx.x >> 5;
    // zero operands
    for (int i = threadIdx.x; i < (128 * 128 + 256 * 128) / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(base)[i] = make_uint4(0, 0, 0, 0);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (threadIdx.x == 0) {
        for (int w = 0; w < 2; ++w) {
            ptx::mbar_init(ptx::smem_u32(&bar[w]), 1);
            for (int i = 0; i < 4; ++i) ptx::mbar_init(ptx::smem_u32(&side[w][i]), 1);
        }
        ptx::fence_mbar_init(); flag_abort = 0; flag_err = 0;
    }
    if (warp == 0) {
        if (PAIR) { ptx::tmem_alloc_pair(ptx::smem_u32(&tbase), 512); ptx::tmem_relinquish_pair(); }
        else { ptx::tmem_alloc(ptx::smem_u32(&tbase), 512); ptx::tmem_relinquish(); }
    }
    ptx::tc_fence_before();
    __syncthreads();
    if (PAIR) ptx::cluster_sync();
    ptx::tc_fence_after();
    const uint32_t tmem = tbase;
    const uint32_t rank = PAIR ? ptx::cluster_ctarank() : 0;
    unsigned long long t0 = clock64();
    if ((threadIdx.x & 31) == 0 && warp < ISSUERS && rank == 0) {
        const uint32_t a0 = ptx::smem_u32(base), b0 = a0 + 128 * 128;
        const uint64_t ad = ptx::sdesc_sw128(a0), bd = ptx::sdesc_sw128(b0);
        constexpr uint32_t idesc = ptx::idesc_make(2, 0, 0, M, N);
        constexpr uint32_t width = 512 / ISSUERS;  // TMEM columns of this issuer
        static_assert(N <= width, "accumulator wider than the issuer's TMEM share");
        const uint32_t col0 = warp * width;
        for (int i = 0; i < iters / ISSUERS; ++i) {
            const uint32_t k = i & 3;
            const uint32_t d = tmem + col0 + (((i >> 2) & 1) ? (width - N) : 0);
            if (MODE >= 3 && k == 0) (void)ptx::mbar_try_wait(ptx::smem_u32(&side[warp][(i >> 2) & 3]), 1);  // a completed phase
            if (MODE >= 2 && k == 0) ptx::tc_fence_after();
            if (PAIR) ptx::mma_i8_pair(d, ad + 2 * k, bd + 2 * k, idesc, k > 0);
            else ptx::mma_i8(d, ad + 2 * k, bd + 2 * k, idesc, k > 0);
            if (MODE >= 1 && k == 3) {
                if (PAIR) ptx::tc_commit_pair(ptx::smem_u32(&side[warp][(i >> 2) & 3]));
                else ptx::tc_commit(ptx::smem_u32(&side[warp][(i >> 2) & 3]));
            }
        }
        if (PAIR) ptx::tc_commit_pair(ptx::smem_u32(&bar[warp])); else ptx::tc_commit(ptx::smem_u32(&bar[warp]));
        ptx::mbar_wait(ptx::smem_u32(&bar[warp]), 0, &flag_abort, &flag_err, 1);
    }
    __syncthreads();
    unsigned long long t1 = clock64();
    if (threadIdx.x == 0 && rank == 0) atomicAdd(cycles, t1 - t0);
    ptx::tc_fence_before();
    __syncthreads();
    if (PAIR) ptx::cluster_sync();
    if (warp == 0) {
        ptx::tc_fence_after();
        if (PAIR) ptx::tmem_dealloc_pair(tmem, 512); else ptx::tmem_dealloc(tmem, 512);
    }
}

template <int M, int N, bool PAIR, int MODE = 0, int ISSUERS = 1>
void run(const char* name, int sms) {
    auto k = bench_kernel<M, N, PAIR, MODE, ISSUERS>;
    size_t smem = 1024 + 128 * 128 + 256 * 128;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    unsigned long long* d; cudaMalloc(&d, 8);
    const int iters = 40000;
    int grid = sms;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(grid); cfg.blockDim = dim3(128); cfg.dynamicSmemBytes = smem;
    if (PAIR) { attr[0].id = cudaLaunchAttributeClusterDimension; attr[0].val.clusterDim.x = 2; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1; cfg.attrs = attr; cfg.numAttrs = 1; }
    for (int rep = 0; rep < 3; ++rep) {
        cudaMemset(d, 0, 8);
        cudaEvent_t e0, e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
        cudaEventRecord(e0);
        cudaError_t e = cudaLaunchKernelEx(&cfg, k, iters, d);
        cudaEventRecord(e1); cudaEventSynchronize(e1);
        if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) { printf("%s launch error\n", name); return; }
        float ms; cudaEventElapsedTime(&ms, e0, e1);
        unsigned long long cyc; cudaMemcpy(&cyc, d, 8, cudaMemcpyDeviceToHost);
        const int issuers = PAIR ? grid / 2 : grid;
        double macs = (double)M * N * 32 * iters * issuers;   // M counts both CTAs for a pair
        double avg_cyc = (double)cyc / issuers;
        double mac_per_clk_sm = (double)M * N * 32 * iters / avg_cyc / (PAIR ? 2 : 1);
        printf("%-22s %8.3f ms  %7.1f TOP/s  cycles/MMA %6.1f  MAC/clk/SM %7.0f\n", name, ms, 2 * macs / (ms * 1e-3) / 1e12,
               avg_cyc / iters, mac_per_clk_sm);
    }
}

// Accumulator hand-off chain of the search kernels: one MMA issuer (lane 0
// of warp 0 of the leader CTA) and EW epilogue warps in each CTA of a pair,
// NB TMEM slots of 128 columns used round robin. Per step the issuer waits
// for the slot's free barrier, issues 4 MMAs (M256 N128 K32, 256 cycles of
// tensor work) and commits to the slot's ready barrier in both CTAs; each
// epilogue warp waits for ready, reads its lane quarter of the slot (READ:
// 8 loads of 16 columns) and arrives on the leader's free barrier. Cycles
// per step = max(256, hand-off latency / NB). CTA_WAIT: waits with CTA scope
// instead of cluster scope. ISSUERS = 2: lane 0 of warp 1 issues the odd
// steps (slots of odd index). HOLD: cycles an epilogue warp spends after its
// reads before handing the slot back (the scan of a search kernel).
template <int NB, int EW, bool READ, bool CTA_WAIT, int ISSUERS = 1, int HOLD = 0>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(192, 1)
    chain_kernel(int iters, unsigned long long* cycles, unsigned* sink) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t* base = sm + ((1024 - (ptx::smem_u32(sm) & 1023)) & 1023);
    __shared__ uint64_t ready[NB], freeb[NB], drain[2];
    __shared__ uint32_t tbase;
    __shared__ int flag_abort, flag_err;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < (128 * 128 + 64 * 128) / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(base)[i] = make_uint4(0, 0, 0, 0);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (threadIdx.x == 0) {
        for (int b = 0; b < NB; ++b) {
            ptx::mbar_init(ptx::smem_u32(&ready[b]), 1);
            ptx::mbar_init(ptx::smem_u32(&freeb[b]), 2 * EW);
        }
        ptx::mbar_init(ptx::smem_u32(&drain[0]), 1);
        ptx::mbar_init(ptx::smem_u32(&drain[1]), 1);
        ptx::fence_mbar_init();
        flag_abort = 0;
        flag_err = 0;
    }
    if (warp == 0) {
        ptx::tmem_alloc_pair(ptx::smem_u32(&tbase), 512);
        ptx::tmem_relinquish_pair();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::cluster_sync();
    ptx::tc_fence_after();
    const uint32_t tmem = tbase;
    const uint32_t rank = ptx::cluster_ctarank();
    auto wait = [&](uint32_t bar, uint32_t par) {
        return CTA_WAIT ? ptx::mbar_wait(bar, par, &flag_abort, &flag_err, 1)
                        : ptx::mbar_wait_cluster(bar, par, &flag_abort, &flag_err, 1);
    };
    const unsigned long long t0 = clock64();
    if (warp < ISSUERS && lane == 0 && rank == 0) {
        const uint32_t a0 = ptx::smem_u32(base), b0 = a0 + 128 * 128;
        const uint64_t ad = ptx::sdesc_sw128(a0), bd = ptx::sdesc_sw128(b0);
        constexpr uint32_t idesc = ptx::idesc_make(2, 0, 0, 256, 128);
        for (int i = warp; i < iters; i += ISSUERS) {
            const int b = i % NB, k = i / NB;
            if (k > 0 && !wait(ptx::smem_u32(&freeb[b]), (k - 1) & 1)) break;
            ptx::tc_fence_after();
            for (int kk = 0; kk < 4; ++kk) ptx::mma_i8_pair(tmem + b * 128, ad + 2 * kk, bd + 2 * kk, idesc, kk > 0);
            ptx::tc_commit_pair_mc(ptx::smem_u32(&ready[b]), 0x3);
        }
        ptx::tc_commit_pair(ptx::smem_u32(&drain[warp]));
        ptx::mbar_wait(ptx::smem_u32(&drain[warp]), 0, &flag_abort, &flag_err, 1);
    } else if (warp >= 2 && warp < 2 + EW) {
        const uint32_t quarter = warp & 3;
        unsigned acc = 0;
        for (int i = 0; i < iters; ++i) {
            const int b = i % NB, k = i / NB;
            if (!__all_sync(0xffffffffu, wait(ptx::smem_u32(&ready[b]), k & 1))) break;
            ptx::tc_fence_after();
            if (READ) {
                uint32_t v[16];
                for (int c = 0; c < 8; ++c) {
                    ptx::tmem_ld16(tmem + (quarter * 32 << 16) + b * 128 + 16 * c, v);
                    ptx::tmem_ld_wait(v);
                    acc ^= v[0] ^ v[15];
                }
            }
            if (HOLD > 0) {
                const long long h0 = clock64();
                while (clock64() - h0 < HOLD) {}
            }
            ptx::tc_fence_before();
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive_cluster_relaxed(ptx::mapa(ptx::smem_u32(&freeb[b]), 0));
        }
        if (acc == 0x12345678u) sink[0] = acc;
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::cluster_sync();
    const unsigned long long t1 = clock64();
    if (threadIdx.x == 0 && rank == 0) atomicAdd(cycles, t1 - t0);
    if (threadIdx.x == 0 && flag_err) atomicAdd(cycles + 1, 1ull);
    if (warp == 0) {
        ptx::tc_fence_after();
        ptx::tmem_dealloc_pair(tmem, 512);
    }
}

template <int NB, int EW, bool READ, bool CTA_WAIT, int ISSUERS = 1, int HOLD = 0>
void run_chain(const char* name, int sms) {
    auto k = chain_kernel<NB, EW, READ, CTA_WAIT, ISSUERS, HOLD>;
    const size_t smem = 1024 + 128 * 128 + 64 * 128;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    unsigned long long* d;
    unsigned* sink;
    cudaMalloc(&d, 16);
    cudaMalloc(&sink, 4);
    const int iters = 20000;
    for (int rep = 0; rep < 2; ++rep) {
        cudaMemset(d, 0, 16);
        k<<<sms, 192, smem>>>(iters, d, sink);
        if (cudaDeviceSynchronize() != cudaSuccess) { printf("%s launch error\n", name); return; }
        unsigned long long c[2];
        cudaMemcpy(c, d, 16, cudaMemcpyDeviceToHost);
        printf("%-34s cycles/step %7.1f (MMA work 256)  timeouts %llu\n", name, (double)c[0] / (sms / 2) / iters, c[1]);
    }
    cudaFree(d);
    cudaFree(sink);
}

int main() {
    int sms; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    run<128, 64, false, 0>("1cta M128 N64", sms);
    run<128, 128, false, 0>("1cta M128 N128", sms);
    run<128, 256, false, 0>("1cta M128 N256", sms);
    run<256, 128, true, 0>("pair M256 N128", sms);
    run<256, 256, true, 0>("pair M256 N256", sms);
    run<128, 128, false, 1>("1cta N128 +commit", sms);
    run<128, 128, false, 2>("1cta N128 +fence", sms);
    run<128, 128, false, 3>("1cta N128 +trywait", sms);
    run<256, 128, true, 1>("pair N128 +commit", sms);
    run<256, 128, true, 3>("pair N128 +all", sms);
    run<256, 128, true, 1, 2>("pair N128 +commit x2", sms);
    run<256, 128, true, 3, 2>("pair N128 +all x2", sms);
    run<128, 128, false, 3, 2>("1cta N128 +all x2", sms);
    run_chain<2, 1, false, false>("chain NB2 1 warp, no read", sms);
    run_chain<2, 4, false, false>("chain NB2 4 warps, no read", sms);
    run_chain<2, 4, false, true>("chain NB2 4 warps, no read, cta", sms);
    run_chain<2, 4, true, false>("chain NB2 4 warps, read", sms);
    run_chain<2, 4, true, true>("chain NB2 4 warps, read, cta", sms);
    run_chain<4, 4, true, false>("chain NB4 4 warps, read", sms);
    run_chain<3, 4, true, false>("chain NB3 4 warps, read", sms);
    run_chain<2, 4, true, false, 2>("chain NB2 read, 2 issuers", sms);
    run_chain<4, 4, true, false, 2>("chain NB4 read, 2 issuers", sms);
    run_chain<4, 4, true, false, 2, 400>("chain NB4 read, 2 issuers, hold 400", sms);
    run_chain<4, 4, true, false, 2, 800>("chain NB4 read, 2 issuers, hold 800", sms);
    run_chain<4, 4, true, false, 2, 1200>("chain NB4 read, 2 issuers, hold 1200", sms);
    return 0;
}
