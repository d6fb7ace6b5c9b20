// C ABI of the matcher (include/sift2nn.h): per-device context, scratch arena,
// input staging, TMA descriptor construction and the launch sequence
//   [pack f32/f16 -> u8] -> row norms -> exact2nn (tcgen05) -> merge.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include "sift2nn.h"
#include "api_internal.h"
#include "context.h"
#include "exact2nn.cuh"
#include "pack.cuh"
#include "lsh.cuh"
#include "learned.cuh"
#include <cstdlib>

namespace sift {

namespace detail {



DeviceCtx g_ctx[kMaxDevices];
std::mutex g_init_mu;
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
thread_local int t_last_status = SIFT_OK;
std::atomic<long long> g_launches{0};  // kernels launched by this library
// 0: CTA-pair kernels (half inputs searched by the FP16 kernel),
// 1: single-CTA u8 kernel, 2: CTA-pair u8 kernel for every input type.
std::atomic<int> g_variant{0};
std::atomic<bool> g_profile{false};
std::mutex g_prof_mu;
struct ProfRecord {
    int tag;
    cudaEvent_t e0, e1;
};
std::vector<ProfRecord> g_prof_events;

ProfSpan::ProfSpan(cudaStream_t st, int tag) : st_(st), tag_(tag) {
    if (!g_profile.load()) return;
    if (cudaEventCreate(&e0_) != cudaSuccess || cudaEventRecord(e0_, st) != cudaSuccess) {
        cudaGetLastError();
        if (e0_) cudaEventDestroy(e0_);
        e0_ = nullptr;
    }
}

void ProfSpan::end() {
    if (!e0_) return;
    cudaEvent_t e1 = nullptr;
    if (cudaEventCreate(&e1) == cudaSuccess && cudaEventRecord(e1, st_) == cudaSuccess) {
        std::lock_guard<std::mutex> pl(g_prof_mu);
        g_prof_events.push_back({tag_, e0_, e1});
    } else {
        cudaGetLastError();
        cudaEventDestroy(e0_);
        if (e1) cudaEventDestroy(e1);
    }
    e0_ = nullptr;
}

ProfSpan::~ProfSpan() {
    if (e0_) cudaEventDestroy(e0_);
}


int ensure_ready(DeviceCtx*& out, int& dev) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return SIFT_ERR_NO_DEVICE;
    }
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SIFT_ERR_NO_DEVICE;
    DeviceCtx& c = g_ctx[dev];
    {
        std::lock_guard<std::mutex> lk(g_init_mu);
        if (!g_encode) {
            void* fn = nullptr;
            cudaDriverEntryPointQueryResult q{};
            if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) !=
                    cudaSuccess ||
                q != cudaDriverEntryPointSuccess || !fn)
                return SIFT_ERR_CUDA;
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        }
        if (!c.ready) {
            cudaDeviceProp prop{};
            if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return SIFT_ERR_CUDA;
            if (prop.major != 10) return SIFT_ERR_UNSUPPORTED;  // sm_100a code only
            c.num_sms = prop.multiProcessorCount;
            if (cudaMalloc(&c.d_status, 4 * sizeof(int)) != cudaSuccess) return SIFT_ERR_ALLOC;
            if (cudaMemset(c.d_status, 0, 4 * sizeof(int)) != cudaSuccess) return SIFT_ERR_CUDA;
            if (cudaMallocHost(&c.h_status, 4 * sizeof(int)) != cudaSuccess) return SIFT_ERR_ALLOC;
            if (cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking) != cudaSuccess) return SIFT_ERR_CUDA;
            for (auto& e : c.chunk_ev)
                if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return SIFT_ERR_CUDA;
            if (cudaEventCreateWithFlags(&c.arena_ev, cudaEventDisableTiming) != cudaSuccess) return SIFT_ERR_CUDA;
            if (cudaDeviceSynchronize() != cudaSuccess) return SIFT_ERR_CUDA;
            c.ready = true;
        }
    }
    out = &c;
    return SIFT_OK;
}

int ensure_arena(DeviceCtx& c, size_t bytes) {
    if (arena_fault()) return SIFT_ERR_ALLOC;
    if (bytes <= c.arena_bytes) return SIFT_OK;
    if (c.arena) {
        cudaDeviceSynchronize();
        cudaFree(c.arena);
        c.arena = nullptr;
        c.arena_bytes = 0;
    }
    size_t cap = bytes + bytes / 8 + (1 << 20);
    if (cudaMalloc(&c.arena, cap) != cudaSuccess) {
        cudaGetLastError();
        return SIFT_ERR_ALLOC;
    }
    c.arena_bytes = cap;
    return SIFT_OK;
}

bool is_device_accessible(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int encode_u8_rows(CUtensorMap* m, const void* base, uint64_t rows, uint32_t box_rows) {
    cuuint64_t dims[2] = {static_cast<cuuint64_t>(kDim), static_cast<cuuint64_t>(rows)};
    cuuint64_t strides[1] = {static_cast<cuuint64_t>(kDim)};
    cuuint32_t box[2] = {static_cast<cuuint32_t>(kDim), box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? SIFT_OK : SIFT_ERR_CUDA;
}

// The folding digits of fold_records_kernel as a 2-D u8 tensor of 256-byte
// rows (8 rows = one half tile, copied as is: no swizzle).
int encode_fold_map(CUtensorMap* m, const void* base, uint64_t tiles) {
    cuuint64_t dims[2] = {256, static_cast<cuuint64_t>(tiles) * 16};
    cuuint64_t strides[1] = {256};
    cuuint32_t box[2] = {256, 8};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? SIFT_OK : SIFT_ERR_CUDA;
}

int encode_bf16_2d(CUtensorMap* m, const void* base, uint64_t inner, uint64_t rows, uint32_t box_inner,
                   uint32_t box_rows) {
    cuuint64_t dims[2] = {static_cast<cuuint64_t>(inner), static_cast<cuuint64_t>(rows)};
    cuuint64_t strides[1] = {static_cast<cuuint64_t>(inner) * 2};
    cuuint32_t box[2] = {box_inner, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? SIFT_OK : SIFT_ERR_CUDA;
}

// FP16 rows of `width` halves (128, or 256 for split [hi | lo] rows): dims
// {width, rows}, box {64, box_rows} (one 128-byte K block per load, the widest
// SWIZZLE_128B box).
int encode_f16_rows(CUtensorMap* m, const void* base, uint64_t rows, uint32_t box_rows, uint64_t width = kDim) {
    cuuint64_t dims[2] = {static_cast<cuuint64_t>(width), static_cast<cuuint64_t>(rows)};
    cuuint64_t strides[1] = {static_cast<cuuint64_t>(width) * 2};
    cuuint32_t box[2] = {static_cast<cuuint32_t>(kDim / 2), box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? SIFT_OK : SIFT_ERR_CUDA;
}

int map_cuda(cudaError_t e) {
    if (e == cudaSuccess) return SIFT_OK;
    if (e == cudaErrorMemoryAllocation) return SIFT_ERR_ALLOC;
    return SIFT_ERR_CUDA;
}


// Reads and clears the device status words: one copy on `st` and one
// synchronisation, which also waits for all the work enqueued on `st` before.
int collect_device_status(DeviceCtx& c, cudaStream_t st) {
    SIFT_CUDA(cudaMemcpyAsync(c.h_status, c.d_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    SIFT_CUDA(cudaStreamSynchronize(st));
    const int code = c.h_status[0];
    if (code != 0) {
        SIFT_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(int), st));
        SIFT_CUDA(cudaStreamSynchronize(st));
        return SIFT_ERR_DEVICE_TIMEOUT;
    }
    return SIFT_OK;
}

}  // namespace detail

using namespace detail;

// Largest power-of-two shift needed to make every q and r value (float or
// half, device-readable) an integer, checked to keep them in [0, 255].
int common_shift(DeviceCtx& c, const void* q, const void* r, bool half, int q_n, int r_n, cudaStream_t st,
                 int& shift) {
    SIFT_CUDA(cudaMemsetAsync(c.d_status + 1, 0, 3 * sizeof(int), st));
    SIFT_CUDA(launch_value_stats(q, half, q_n, c.d_status + 1, c.num_sms, st));
    SIFT_CUDA(launch_value_stats(r, half, r_n, c.d_status + 1, c.num_sms, st));
    SIFT_CUDA(cudaMemcpyAsync(c.h_status + 1, c.d_status + 1, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
    SIFT_CUDA(cudaStreamSynchronize(st));
    const int bad = c.h_status[1], s = c.h_status[2];
    float mx = 0.0f;
    std::memcpy(&mx, &c.h_status[3], sizeof(float));
    if (bad || s > kMaxShift || ldexpf(mx, s) > 255.0f) return SIFT_ERR_NOT_INTEGER;
    shift = s;
    return SIFT_OK;
}

// Where the u8 descriptors a kernel reads come from, for every memory type.
struct InputPlan {
    const void* q_src = nullptr;
    const void* r_src = nullptr;
    bool need_pack = false;  // float / half -> u8 conversion
    bool stage_u8 = false;   // copy u8 rows into the arena
    bool stage_f32 = false;  // copy host float rows into the arena first
    size_t o_qu8 = 0, o_ru8 = 0, o_qf = 0, o_rf = 0;
};

// type -1: FP16 device rows read in place by the FP16 kernel (checked only).
int plan_inputs(const void* q, const void* r, int type, int q_n, int r_n, Layout& L, InputPlan& ip) {
    if (q_n > 0 && !q) return SIFT_ERR_INVALID_ARG;
    if (r_n > 0 && !r) return SIFT_ERR_INVALID_ARG;
    // Device types must be device (or managed) memory: a host pointer would
    // reach a tensor map or a kernel and fault instead of being refused.
    if (type == -1 || type == SIFT_FLOAT_DEVICE || type == SIFT_HALF_DEVICE || type == SIFT_U8_DEVICE) {
        if ((q_n > 0 && !is_device_accessible(q)) || (r_n > 0 && !is_device_accessible(r)))
            return SIFT_ERR_INVALID_ARG;
    }
    if (type == -1)
        return ((reinterpret_cast<uintptr_t>(q) & 15) || (reinterpret_cast<uintptr_t>(r) & 15)) ? SIFT_ERR_INVALID_ARG
                                                                                                : SIFT_OK;
    if (type < SIFT_FLOAT_HOST || type > SIFT_U8_HOST) return SIFT_ERR_INVALID_ARG;
    ip.q_src = q;
    ip.r_src = r;
    ip.need_pack = type != SIFT_U8_DEVICE && type != SIFT_U8_HOST;
    ip.stage_u8 = type == SIFT_U8_HOST;
    if (type == SIFT_U8_DEVICE) {
        // TMA needs 16-byte aligned rows; unaligned device input is copied.
        ip.stage_u8 = (reinterpret_cast<uintptr_t>(q) & 15) || (reinterpret_cast<uintptr_t>(r) & 15);
    }
    if (type == SIFT_FLOAT_HOST) {
        // Zero-copy like the reference (src/knn_brute.cu:58, :223) when the
        // memory is mapped pinned memory; otherwise stage it.
        void* qm = nullptr;
        void* rm = nullptr;
        if (cudaHostGetDevicePointer(&qm, const_cast<void*>(q), 0) == cudaSuccess &&
            (r_n == 0 || cudaHostGetDevicePointer(&rm, const_cast<void*>(r), 0) == cudaSuccess) &&
            !(reinterpret_cast<uintptr_t>(qm) & 15) && !(reinterpret_cast<uintptr_t>(rm) & 15)) {
            ip.q_src = qm;
            ip.r_src = rm;
        } else {
            cudaGetLastError();
            ip.stage_f32 = true;
        }
    }
    if ((type == SIFT_FLOAT_DEVICE || type == SIFT_HALF_DEVICE) &&
        ((reinterpret_cast<uintptr_t>(q) & 15) || (reinterpret_cast<uintptr_t>(r) & 15)))
        return SIFT_ERR_INVALID_ARG;
    if (ip.need_pack || ip.stage_u8) {
        ip.o_qu8 = L.take(static_cast<size_t>(q_n) * kDim);
        ip.o_ru8 = L.take(static_cast<size_t>(r_n) * kDim + 16);
    }
    if (ip.stage_f32) {
        ip.o_qf = L.take(static_cast<size_t>(q_n) * kDim * 4);
        ip.o_rf = L.take(static_cast<size_t>(r_n) * kDim * 4 + 16);
    }
    return SIFT_OK;
}

// Produces 16-byte aligned device u8 rows for both sides (arena A laid out by plan_inputs).
// shift: the inputs were integers times 2^-shift (0 for integer inputs); the
// u8 rows hold the integers, so distances scale by 2^(-2 shift).
int stage_inputs(DeviceCtx& c, char* A, const InputPlan& ip, int type, const void* q, const void* r, int q_n,
                 int r_n, cudaStream_t st, const uint8_t*& qd, const uint8_t*& rd, int& shift) {
    shift = 0;
    if (type == SIFT_U8_DEVICE && !ip.stage_u8) {
        qd = static_cast<const uint8_t*>(q);
        rd = static_cast<const uint8_t*>(r);
        return SIFT_OK;
    }
    if (ip.stage_u8) {
        const cudaMemcpyKind k = type == SIFT_U8_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
        SIFT_CUDA(cudaMemcpyAsync(A + ip.o_qu8, q, static_cast<size_t>(q_n) * kDim, k, st));
        if (r_n) SIFT_CUDA(cudaMemcpyAsync(A + ip.o_ru8, r, static_cast<size_t>(r_n) * kDim, k, st));
        qd = reinterpret_cast<uint8_t*>(A + ip.o_qu8);
        rd = reinterpret_cast<uint8_t*>(A + ip.o_ru8);
        return SIFT_OK;
    }
    const void* q_src = ip.q_src;
    const void* r_src = ip.r_src;
    if (ip.stage_f32) {
        SIFT_CUDA(cudaMemcpyAsync(A + ip.o_qf, q, static_cast<size_t>(q_n) * kDim * 4, cudaMemcpyHostToDevice, st));
        if (r_n)
            SIFT_CUDA(cudaMemcpyAsync(A + ip.o_rf, r, static_cast<size_t>(r_n) * kDim * 4, cudaMemcpyHostToDevice, st));
        q_src = A + ip.o_qf;
        r_src = A + ip.o_rf;
    }
    SIFT_CUDA(cudaMemsetAsync(c.d_status + 1, 0, sizeof(int), st));
    uint8_t* qo = reinterpret_cast<uint8_t*>(A + ip.o_qu8);
    uint8_t* ro = reinterpret_cast<uint8_t*>(A + ip.o_ru8);
    g_launches += r_n > 0 ? 2 : 1;
    const bool half = type == SIFT_HALF_DEVICE;
    auto pack = [&](float mul) -> int {
        SIFT_CUDA(cudaMemsetAsync(c.d_status + 1, 0, sizeof(int), st));
        if (half) {
            SIFT_CUDA(launch_pack_f16_u8(q_src, q_n, mul, qo, c.d_status + 1, c.num_sms, st));
            SIFT_CUDA(launch_pack_f16_u8(r_src, r_n, mul, ro, c.d_status + 1, c.num_sms, st));
        } else {
            SIFT_CUDA(launch_pack_f32_u8(static_cast<const float*>(q_src), q_n, mul, qo, c.d_status + 1, c.num_sms, st));
            SIFT_CUDA(launch_pack_f32_u8(static_cast<const float*>(r_src), r_n, mul, ro, c.d_status + 1, c.num_sms, st));
        }
        SIFT_CUDA(cudaMemcpyAsync(c.h_status + 1, c.d_status + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        SIFT_CUDA(cudaStreamSynchronize(st));
        return c.h_status[1] != 0 ? SIFT_ERR_NOT_INTEGER : SIFT_OK;
    };
    if (pack(1.0f) != SIFT_OK) {
        // Not plain integers: look for one power-of-two scale of all values.
        int s = 0;
        SIFT_TRY(common_shift(c, q_src, r_src, half, q_n, r_n, st, s));
        g_launches += 2;
        SIFT_TRY(pack(ldexpf(1.0f, s)));
        shift = s;
    }
    qd = qo;
    rd = ro;
    return SIFT_OK;
}

// Host u8 inputs (U8_HOST) with a large base: the base is copied to the
// device in chunks on the copy stream while the search kernel runs on the
// chunks that have landed (records, then one persistent pair-kernel launch
// per chunk); the per-query pruning bounds carry over from chunk to chunk
// and one merge combines every chunk's partial lists. Same results as the
// single-launch path. Caller holds c.mu.
constexpr int kChunkMinRows = 1 << 16;
constexpr int kChunks = 8;

// Base tiles per chunk, in base order (returns the number of chunks).
// The pinned copy moves a 128-byte row in ~2.3 ns (~55 GB/s of PCIe), and
// the search kernel spends ~0.128 ps per query x row (10,000 x 1,000,000 in
// ~1.28 ms), so with q_n queries a chunk's search takes beta = q_n x 5.5e-5
// of its copy time. When beta is small the copy sets the pace and only the
// last chunk's search (plus the merge) runs after the last byte lands: the
// chunks then shrink geometrically toward the end of the base, each one
// 1 / (1.25 beta) of the size of the chunk after it (between 1.25 and 4
// times, the 1.25 covering the launches of a chunk), from a last chunk of 128
// tiles (or 1/64 of the base), so that every chunk's search ends about when
// the next chunk lands. Otherwise (the search sets the pace) the base goes in
// kChunks equal chunks.
int plan_chunk_tiles(int q_n, int tiles, int (&out)[kMaxChunks]) {
    const double beta = 5.5e-5 * q_n, paced = 1.25 * beta;
    if (paced > 1.0) {
        const int per = (tiles + kChunks - 1) / kChunks;
        int n = 0;
        for (int t = 0; t < tiles; t += per) out[n++] = std::min(per, tiles - t);
        return n;
    }
    const double grow = std::min(4.0, std::max(1.25, 1.0 / paced));
    int rev[kMaxChunks];
    int n = 0, left = tiles;
    double size = std::max(128.0, tiles / 64.0);
    while (left > 0) {
        const int t = (n + 1 == kMaxChunks) ? left : std::min(left, static_cast<int>(size));
        rev[n++] = t;
        left -= t;
        size *= grow;
    }
    for (int k = 0; k < n; ++k) out[k] = rev[n - 1 - k];
    return n;
}

// fold: the search kernel with the norms folded into the MMAs (the default
// for u8 rows), else the pair kernel without folding.
int exact_match_chunked(const MatchArgs& a, DeviceCtx& c, cudaStream_t st, bool fold) {
    const int q_n = static_cast<int>(a.q_n), r_n = static_cast<int>(a.r_n);
    const int workers = c.num_sms / 2;
    const ExactPlan whole = make_exact_plan(q_n, r_n, workers, 2);
    int chunk_tiles[kMaxChunks];
    const int n_chunks = plan_chunk_tiles(q_n, whole.base_tiles, chunk_tiles);
    int chunk_off[kMaxChunks];  // first base row of each chunk (a multiple of kBN)
    ChunkSet cs{};
    cs.n = n_chunks;
    cs.r_n = r_n;
    cs.parts = 2;
    cs.q_pad = whole.q_pad;
    ExactPlan plans[kMaxChunks];
    long long slots = 1;
    for (int ch = 0, off = 0; ch < n_chunks; ++ch) {
        chunk_off[ch] = off;
        const int rows = std::min(chunk_tiles[ch] * kBN, r_n - off);
        off += rows;
        plans[ch] = make_exact_plan(q_n, rows, workers, 2);
        cs.W[ch] = plans[ch].units;
        cs.G[ch] = plans[ch].grid;
        cs.tiles[ch] = plans[ch].base_tiles;
        slots = std::max<long long>(slots, static_cast<long long>(plans[ch].max_splits) * plans[ch].parts);
    }
    cs.slot_stride = slots * whole.q_pad;

    const bool m_dev = !a.matches || is_device_accessible(a.matches);
    const bool s_dev = !a.sorted || is_device_accessible(a.sorted);
    const bool i_dev = !a.nn_idx || is_device_accessible(a.nn_idx);
    const bool d_dev = !a.nn_dist || is_device_accessible(a.nn_dist);
    Layout L;
    const size_t o_q = L.take(static_cast<size_t>(q_n) * kDim);
    const size_t o_r = L.take(static_cast<size_t>(r_n) * kDim + 16);
    const size_t o_brec = L.take(static_cast<size_t>(whole.base_tiles) * kRecInts * 4 + 16);
    const size_t o_qnorm = L.take(static_cast<size_t>(whole.q_pad) * 4);
    const size_t o_thr = L.take(static_cast<size_t>(whole.q_pad) * 4);
    const size_t o_part = L.take(static_cast<size_t>(n_chunks) * cs.slot_stride * sizeof(int4));
    const size_t o_fold = fold ? L.take(static_cast<size_t>(whole.base_tiles) * 2 * kFoldHalfBytes) : 0;
    const size_t o_m = (a.matches && !m_dev) ? L.take(static_cast<size_t>(q_n) * 4) : 0;
    const size_t o_s = (a.sorted && !s_dev) ? L.take(static_cast<size_t>(q_n) * 16) : 0;
    const size_t o_i = (a.nn_idx && !i_dev) ? L.take(static_cast<size_t>(q_n) * 8) : 0;
    const size_t o_d = (a.nn_dist && !d_dev) ? L.take(static_cast<size_t>(q_n) * 8) : 0;
    SIFT_TRY(ensure_arena(c, L.off));
    char* A = c.arena;
    uint8_t* qd = reinterpret_cast<uint8_t*>(A + o_q);
    uint8_t* rd = reinterpret_cast<uint8_t*>(A + o_r);
    int32_t* brec = reinterpret_cast<int32_t*>(A + o_brec);
    int32_t* qnorm = reinterpret_cast<int32_t*>(A + o_qnorm);
    int32_t* thresh = reinterpret_cast<int32_t*>(A + o_thr);
    int4* partial = reinterpret_cast<int4*>(A + o_part);
    uint32_t* fold_digits = reinterpret_cast<uint32_t*>(A + o_fold);
    const uint8_t* rh = static_cast<const uint8_t*>(a.r);

    // The base chunks on the copy stream once every earlier use of the arena
    // on the search stream is done; the queries meanwhile on the search stream.
    SIFT_CUDA(cudaEventRecord(c.chunk_ev[kMaxChunks], st));
    SIFT_CUDA(cudaStreamWaitEvent(c.copy_stream, c.chunk_ev[kMaxChunks], 0));
    SIFT_CUDA(cudaMemcpyAsync(qd, a.q, static_cast<size_t>(q_n) * kDim, cudaMemcpyHostToDevice, st));
    SIFT_CUDA(launch_row_norms_u8(qd, q_n, whole.q_pad, kMetricL2, qnorm, nullptr, thresh, st));
    for (int ch = 0; ch < n_chunks; ++ch) {
        const size_t off = static_cast<size_t>(chunk_off[ch]);
        SIFT_CUDA(cudaMemcpyAsync(rd + off * kDim, rh + off * kDim, static_cast<size_t>(plans[ch].r_n) * kDim,
                                  cudaMemcpyHostToDevice, c.copy_stream));
        SIFT_CUDA(cudaEventRecord(c.chunk_ev[ch], c.copy_stream));
    }
    CUtensorMap qmap, bmap, fmap;
    SIFT_TRY(encode_u8_rows(&qmap, qd, q_n, kBM));
    SIFT_TRY(encode_u8_rows(&bmap, rd, r_n, kBN / 2));
    if (fold) SIFT_TRY(encode_fold_map(&fmap, fold_digits, whole.base_tiles));
    for (int ch = 0; ch < n_chunks; ++ch) {
        const int off = chunk_off[ch];
        const uint8_t* rows = rd + static_cast<size_t>(off) * kDim;
        int32_t* rec = brec + static_cast<size_t>(off / kBN) * kRecInts;
        SIFT_CUDA(cudaStreamWaitEvent(st, c.chunk_ev[ch], 0));
        if (fold)
            SIFT_CUDA(launch_fold_records_u8(rows, plans[ch].r_n, plans[ch].r_pad, a.metric, rec,
                                             fold_digits + static_cast<size_t>(off / kBN) * 2 * kFoldHalfBytes / 4,
                                             st));
        else
            SIFT_CUDA(launch_row_norms_u8(rows, plans[ch].r_n, plans[ch].r_pad, a.metric, nullptr, rec, nullptr, st));
        WorkItem it{};
        it.n_a = q_n;
        it.b_off = off;
        it.n_b = plans[ch].r_n;
        it.groups = plans[ch].q_groups;
        it.tiles = plans[ch].base_tiles;
        it.rec_off = off / kBN;
        it.idx_base = off;
        if (fold)
            SIFT_CUDA(launch_exact2nn_u8fold_pair_item(qmap, bmap, fmap, brec, plans[ch], it,
                                                       partial + ch * cs.slot_stride, thresh, c.d_status, st));
        else
            SIFT_CUDA(launch_exact2nn_u8_pair_item(qmap, bmap, brec, plans[ch], it, partial + ch * cs.slot_stride,
                                                   thresh, c.d_status, st));
    }
    g_launches += 1 + 2 * n_chunks + 1;

    uint32_t* m_out = (a.matches && !m_dev) ? reinterpret_cast<uint32_t*>(A + o_m) : a.matches;
    float4* s_out = (a.sorted && !s_dev) ? reinterpret_cast<float4*>(A + o_s) : reinterpret_cast<float4*>(a.sorted);
    int32_t* i_out = (a.nn_idx && !i_dev) ? reinterpret_cast<int32_t*>(A + o_i) : a.nn_idx;
    float* d_out = (a.nn_dist && !d_dev) ? reinterpret_cast<float*>(A + o_d) : a.nn_dist;
    SIFT_CUDA(launch_merge2nn_chunks(partial, cs, q_n, qnorm, a.metric, a.threshold, 1.0f, m_out, s_out, i_out, d_out,
                                     st));
    if (a.matches && !m_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.matches, m_out, static_cast<size_t>(q_n) * 4, cudaMemcpyDeviceToHost, st));
    if (a.sorted && !s_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.sorted, s_out, static_cast<size_t>(q_n) * 16, cudaMemcpyDeviceToHost, st));
    if (a.nn_idx && !i_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.nn_idx, i_out, static_cast<size_t>(q_n) * 8, cudaMemcpyDeviceToHost, st));
    if (a.nn_dist && !d_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.nn_dist, d_out, static_cast<size_t>(q_n) * 8, cudaMemcpyDeviceToHost, st));
    return collect_device_status(c, st);
}

// General float / half descriptors (values that are not integers times one
// power of two, e.g. the unit-normalised rand() vectors of the reference
// benchmark, src/helper.cu:40-58): searched on the tensor cores with f32
// accumulation and float keys. Half rows are read in place (exact products);
// float rows are first split into FP16 hi + lo parts after scaling by a power
// of two 2^e that puts the largest |value| in [2^14, 2^15), and the dot
// product is hi.hi' + hi.lo' + lo.hi' (22 significant bits per value, the
// f32 accumulation of the tensor cores). Norms are f32 sums of the scaled
// values. Distances come back in the caller's units (x 2^-2e). Caller holds
// the arena lock.
int exact_match_float(const MatchArgs& a, DeviceCtx& c, cudaStream_t st) {
    const int q_n = static_cast<int>(a.q_n), r_n = static_cast<int>(a.r_n);
    const bool half = a.type == SIFT_HALF_DEVICE;
    const bool host_in = a.type == SIFT_FLOAT_HOST;
    const bool has_lo = !half;
    constexpr int kGroupTiles = 2;  // query groups of 256 rows (one 128-row tile per CTA of a pair)
    const ExactPlan plan = make_exact_plan(q_n, r_n, c.num_sms / 2, 2, kGroupTiles);
    if (!host_in && ((reinterpret_cast<uintptr_t>(a.q) & 15) || (r_n && (reinterpret_cast<uintptr_t>(a.r) & 15))))
        return SIFT_ERR_INVALID_ARG;
    const bool m_dev = !a.matches || is_device_accessible(a.matches);
    const bool s_dev = !a.sorted || is_device_accessible(a.sorted);
    const bool i_dev = !a.nn_idx || is_device_accessible(a.nn_idx);
    const bool d_dev = !a.nn_dist || is_device_accessible(a.nn_dist);
    const bool host_out = !(m_dev && s_dev && i_dev && d_dev);

    Layout L;
    const size_t o_qf = host_in ? L.take(static_cast<size_t>(q_n) * kDim * 4) : 0;
    const size_t o_rf = host_in ? L.take(static_cast<size_t>(r_n) * kDim * 4 + 16) : 0;
    const size_t o_qs = has_lo ? L.take(static_cast<size_t>(q_n) * 512) : 0;
    const size_t o_rs = has_lo ? L.take(static_cast<size_t>(r_n) * 512 + 16) : 0;
    const size_t o_brec = L.take(static_cast<size_t>(plan.base_tiles) * kRecInts * 4 + 16);
    const size_t o_qnorm = L.take(static_cast<size_t>(plan.q_pad) * 4);
    const size_t o_thr = L.take(static_cast<size_t>(plan.q_pad) * 4);
    const size_t o_part = L.take(static_cast<size_t>(plan.max_splits) * plan.parts * plan.q_pad * sizeof(int4));
    const size_t o_m = (a.matches && !m_dev) ? L.take(static_cast<size_t>(q_n) * 4) : 0;
    const size_t o_s = (a.sorted && !s_dev) ? L.take(static_cast<size_t>(q_n) * 16) : 0;
    const size_t o_i = (a.nn_idx && !i_dev) ? L.take(static_cast<size_t>(q_n) * 8) : 0;
    const size_t o_d = (a.nn_dist && !d_dev) ? L.take(static_cast<size_t>(q_n) * 8) : 0;
    SIFT_TRY(ensure_arena(c, L.off));
    char* A = c.arena;

    const void* q_src = a.q;
    const void* r_src = a.r;
    if (host_in) {
        SIFT_CUDA(cudaMemcpyAsync(A + o_qf, a.q, static_cast<size_t>(q_n) * kDim * 4, cudaMemcpyHostToDevice, st));
        if (r_n)
            SIFT_CUDA(cudaMemcpyAsync(A + o_rf, a.r, static_cast<size_t>(r_n) * kDim * 4, cudaMemcpyHostToDevice, st));
        q_src = A + o_qf;
        r_src = A + o_rf;
    }
    // Largest |value| of both sets (and a finiteness check) for the scale.
    SIFT_CUDA(cudaMemsetAsync(c.d_status + 1, 0, 2 * sizeof(int), st));
    SIFT_CUDA(launch_abs_stats(q_src, half, q_n, c.d_status + 1, c.num_sms, st));
    SIFT_CUDA(launch_abs_stats(r_src, half, r_n, c.d_status + 1, c.num_sms, st));
    SIFT_CUDA(cudaMemcpyAsync(c.h_status + 1, c.d_status + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    SIFT_CUDA(cudaStreamSynchronize(st));
    if (c.h_status[1] != 0) return SIFT_ERR_INVALID_ARG;  // infinite or NaN values
    float mx = 0.0f;
    std::memcpy(&mx, &c.h_status[2], sizeof(float));
    int e = 0;
    if (has_lo && mx > 0.0f) {
        int ex = 0;
        std::frexp(mx, &ex);  // mx in [2^(ex-1), 2^ex)
        e = 15 - ex;          // mx * 2^e in [2^14, 2^15)
    }
    const float mul = ldexpf(1.0f, e);
    g_launches += (r_n > 0 ? 2 : 1);

    const void* q_rows = q_src;
    const void* r_rows = r_src;
    if (has_lo) {
        SIFT_CUDA(launch_pack_split_f16(static_cast<const float*>(q_src), q_n, mul, A + o_qs, c.num_sms, st));
        SIFT_CUDA(launch_pack_split_f16(static_cast<const float*>(r_src), r_n, mul, A + o_rs, c.num_sms, st));
        q_rows = A + o_qs;
        r_rows = A + o_rs;
        g_launches += (r_n > 0 ? 2 : 1);
    }
    int32_t* brec = reinterpret_cast<int32_t*>(A + o_brec);
    int32_t* qnorm = reinterpret_cast<int32_t*>(A + o_qnorm);
    int32_t* thresh = reinterpret_cast<int32_t*>(A + o_thr);
    SIFT_CUDA(launch_row_norms_float(r_src, half, r_n, plan.r_pad, mul, a.metric, nullptr, brec, nullptr, st));
    SIFT_CUDA(launch_row_norms_float(q_src, half, q_n, plan.q_pad, mul, kMetricL2, qnorm, nullptr, thresh, st));
    g_launches += (plan.r_pad > 0 ? 1 : 0) + 1;
    int4* partial = reinterpret_cast<int4*>(A + o_part);
    if (r_n > 0) {
        const uint64_t width = has_lo ? 2 * kDim : kDim;
        CUtensorMap qmap, bmap;
        SIFT_TRY(encode_f16_rows(&qmap, q_rows, q_n, kBM, width));
        SIFT_TRY(encode_f16_rows(&bmap, r_rows, r_n, kBN / 2, width));
        SIFT_CUDA(maybe_inject_wait_expiry(c.d_status, st));
        ProfSpan span(st, kProfSearch);
        SIFT_CUDA(launch_exact2nn_float_pair(qmap, bmap, brec, plan, partial, thresh, c.d_status, has_lo, st));
        span.end();
        ++g_launches;
    }
    uint32_t* m_out = (a.matches && !m_dev) ? reinterpret_cast<uint32_t*>(A + o_m) : a.matches;
    float4* s_out = (a.sorted && !s_dev) ? reinterpret_cast<float4*>(A + o_s) : reinterpret_cast<float4*>(a.sorted);
    int32_t* i_out = (a.nn_idx && !i_dev) ? reinterpret_cast<int32_t*>(A + o_i) : a.nn_idx;
    float* d_out = (a.nn_dist && !d_dev) ? reinterpret_cast<float*>(A + o_d) : a.nn_dist;
    SIFT_CUDA(launch_merge2nn_float(partial, plan, kGroupTiles * kBM, qnorm, a.metric, a.threshold,
                                    ldexpf(1.0f, -2 * e), m_out, s_out, i_out, d_out, st));
    ++g_launches;
    if (a.matches && !m_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.matches, m_out, static_cast<size_t>(q_n) * 4, cudaMemcpyDeviceToHost, st));
    if (a.sorted && !s_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.sorted, s_out, static_cast<size_t>(q_n) * 16, cudaMemcpyDeviceToHost, st));
    if (a.nn_idx && !i_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.nn_idx, i_out, static_cast<size_t>(q_n) * 8, cudaMemcpyDeviceToHost, st));
    if (a.nn_dist && !d_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.nn_dist, d_out, static_cast<size_t>(q_n) * 8, cudaMemcpyDeviceToHost, st));
    if (a.sync || host_out || host_in) {
        return collect_device_status(c, st);
    }
    return SIFT_OK;
}

// Core of every exact entry point.
int exact_match(const MatchArgs& a) {
    if (a.q_n > 0 && !a.q) return SIFT_ERR_INVALID_ARG;
    if (a.r_n > 0 && !a.r) return SIFT_ERR_INVALID_ARG;
    if (a.type < SIFT_FLOAT_HOST || a.type > SIFT_U8_HOST) return SIFT_ERR_INVALID_ARG;
    if (a.metric != SIFT_METRIC_L2 && a.metric != SIFT_METRIC_DOT) return SIFT_ERR_INVALID_ARG;
    if (a.q_n > 0x7fffffffu - 256 || a.r_n > 0x7fffffffu - 256) return SIFT_ERR_INVALID_ARG;
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(ensure_ready(cp, dev));
    DeviceCtx& c = *cp;
    cudaStream_t st = static_cast<cudaStream_t>(a.stream);
    ArenaLock lk(c, st);
    const int q_n = static_cast<int>(a.q_n), r_n = static_cast<int>(a.r_n);
    if (q_n == 0) return SIFT_OK;

    const int variant = g_variant.load();
    const bool use_pair = variant != 1;
    // Half inputs are searched as FP16 by the FP16 tensor-core kernel in place.
    const bool use_f16 = (variant == 0 || variant == 3) && a.type == SIFT_HALF_DEVICE;
    // The default for u8 rows: the pair kernel with the norms folded into the
    // MMAs; variant 3 keeps the pair kernel without folding.
    const bool use_fold = variant == 0 && a.type != SIFT_HALF_DEVICE;
    if (use_pair && a.type == SIFT_U8_HOST && r_n >= kChunkMinRows) return exact_match_chunked(a, c, st, use_fold);
    const ExactPlan plan = use_pair ? make_exact_plan(q_n, r_n, c.num_sms / 2, 2) : make_exact_plan(q_n, r_n, c.num_sms, 1);

    // Output placement: direct when the device can write the pointer, else staged.
    const bool m_dev = !a.matches || is_device_accessible(a.matches);
    const bool s_dev = !a.sorted || is_device_accessible(a.sorted);
    const bool i_dev = !a.nn_idx || is_device_accessible(a.nn_idx);
    const bool d_dev = !a.nn_dist || is_device_accessible(a.nn_dist);
    const bool host_out = !(m_dev && s_dev && i_dev && d_dev);

    Layout L;
    InputPlan ip;
    SIFT_TRY(plan_inputs(a.q, a.r, use_f16 ? -1 : a.type, q_n, r_n, L, ip));
    const size_t o_brec = L.take(static_cast<size_t>(plan.base_tiles) * kRecInts * 4 + 16);
    const size_t o_qnorm = L.take(static_cast<size_t>(plan.q_pad) * 4);
    const size_t o_thr = L.take(static_cast<size_t>(plan.q_pad) * 4);
    const size_t o_part = L.take(static_cast<size_t>(plan.max_splits) * plan.parts * plan.q_pad * sizeof(int4));
    const size_t o_m = (a.matches && !m_dev) ? L.take(static_cast<size_t>(q_n) * 4) : 0;
    const size_t o_s = (a.sorted && !s_dev) ? L.take(static_cast<size_t>(q_n) * 16) : 0;
    const size_t o_i = (a.nn_idx && !i_dev) ? L.take(static_cast<size_t>(q_n) * 8) : 0;
    const size_t o_d = (a.nn_dist && !d_dev) ? L.take(static_cast<size_t>(q_n) * 8) : 0;
    const size_t o_fold = use_fold ? L.take(static_cast<size_t>(plan.base_tiles) * 2 * kFoldHalfBytes) : 0;
    SIFT_TRY(ensure_arena(c, L.off));
    char* A = c.arena;

    // ---- inputs: u8 rows (packed from float / half when needed), or the
    // caller's FP16 rows for the FP16 kernel.
    const uint8_t* qd = nullptr;
    const uint8_t* rd = nullptr;
    int shift = 0;
    // Values that are not integers times one power of two take the general
    // float path (float keys on the FP16 tensor cores).
    if (use_f16) {
        const int rc = common_shift(c, a.q, a.r, true, q_n, r_n, st, shift);
        g_launches += r_n > 0 ? 2 : 1;
        if (rc == SIFT_ERR_NOT_INTEGER) return exact_match_float(a, c, st);
        SIFT_TRY(rc);
    } else {
        const int rc = stage_inputs(c, A, ip, a.type, a.q, a.r, q_n, r_n, st, qd, rd, shift);
        if (rc == SIFT_ERR_NOT_INTEGER && a.type != SIFT_U8_DEVICE && a.type != SIFT_U8_HOST)
            return exact_match_float(a, c, st);
        SIFT_TRY(rc);
    }

    // ---- norms
    int32_t* brec = reinterpret_cast<int32_t*>(A + o_brec);
    int32_t* qnorm = reinterpret_cast<int32_t*>(A + o_qnorm);
    int32_t* thresh = reinterpret_cast<int32_t*>(A + o_thr);
    if (use_f16) {
        const float mul = ldexpf(1.0f, shift);
        SIFT_CUDA(launch_row_norms_f16(a.r, r_n, plan.r_pad, mul, a.metric, nullptr, brec, nullptr, st));
        SIFT_CUDA(launch_row_norms_f16(a.q, q_n, plan.q_pad, mul, kMetricL2, qnorm, nullptr, thresh, st));
    } else {
        if (use_fold)
            SIFT_CUDA(launch_fold_records_u8(rd, r_n, plan.r_pad, a.metric, brec,
                                             reinterpret_cast<uint32_t*>(A + o_fold), st));
        else
            SIFT_CUDA(launch_row_norms_u8(rd, r_n, plan.r_pad, a.metric, nullptr, brec, nullptr, st));
        SIFT_CUDA(launch_row_norms_u8(qd, q_n, plan.q_pad, kMetricL2, qnorm, nullptr, thresh, st));
    }
    g_launches += (plan.r_pad > 0 ? 1 : 0) + 1;

    // ---- fused GEMM + top-2
    int4* partial = reinterpret_cast<int4*>(A + o_part);
    if (r_n > 0) {
        CUtensorMap qmap, bmap;
        if (use_f16) {
            SIFT_TRY(encode_f16_rows(&qmap, a.q, q_n, kBM));
            SIFT_TRY(encode_f16_rows(&bmap, a.r, r_n, kBN / 2));
        } else {
            SIFT_TRY(encode_u8_rows(&qmap, qd, q_n, kBM));
            SIFT_TRY(encode_u8_rows(&bmap, rd, r_n, use_pair ? kBN / 2 : kBN));
        }
        SIFT_CUDA(maybe_inject_wait_expiry(c.d_status, st));
        ProfSpan span(st, kProfSearch);
        if (use_f16)
            SIFT_CUDA(launch_exact2nn_f16_pair(qmap, bmap, brec, plan, partial, thresh, c.d_status,
                                               ldexpf(1.0f, 2 * shift), st));
        else if (use_fold) {
            CUtensorMap fmap;
            SIFT_TRY(encode_fold_map(&fmap, A + o_fold, plan.base_tiles));
            SIFT_CUDA(launch_exact2nn_u8fold_pair(qmap, bmap, fmap, brec, plan, partial, thresh, c.d_status, st));
        } else if (use_pair)
            SIFT_CUDA(launch_exact2nn_u8_pair(qmap, bmap, brec, plan, partial, thresh, c.d_status, st));
        else
            SIFT_CUDA(launch_exact2nn_u8(qmap, bmap, brec, plan, partial, thresh, c.d_status, st));
        ++g_launches;
        span.end();
    }

    // ---- merge + outputs
    uint32_t* m_out = (a.matches && !m_dev) ? reinterpret_cast<uint32_t*>(A + o_m) : a.matches;
    float4* s_out = (a.sorted && !s_dev) ? reinterpret_cast<float4*>(A + o_s) : reinterpret_cast<float4*>(a.sorted);
    int32_t* i_out = (a.nn_idx && !i_dev) ? reinterpret_cast<int32_t*>(A + o_i) : a.nn_idx;
    float* d_out = (a.nn_dist && !d_dev) ? reinterpret_cast<float*>(A + o_d) : a.nn_dist;
    SIFT_CUDA(launch_merge2nn(partial, plan, qnorm, a.metric, a.threshold, ldexpf(1.0f, -2 * shift), m_out, s_out,
                              i_out, d_out, st));
    ++g_launches;
    if (a.matches && !m_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.matches, m_out, static_cast<size_t>(q_n) * 4, cudaMemcpyDeviceToHost, st));
    if (a.sorted && !s_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.sorted, s_out, static_cast<size_t>(q_n) * 16, cudaMemcpyDeviceToHost, st));
    if (a.nn_idx && !i_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.nn_idx, i_out, static_cast<size_t>(q_n) * 8, cudaMemcpyDeviceToHost, st));
    if (a.nn_dist && !d_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.nn_dist, d_out, static_cast<size_t>(q_n) * 8, cudaMemcpyDeviceToHost, st));

    const bool host_in = a.type == SIFT_U8_HOST || a.type == SIFT_FLOAT_HOST;
    if (a.sync || host_out || host_in) {
        return collect_device_status(c, st);
    }
    return SIFT_OK;
}


// Hyperplane rows are int8: dims {128, rows}, box {128, box_rows}.
int encode_i8_rows(CUtensorMap* m, const void* base, uint64_t rows, uint32_t box_rows) {
    return encode_u8_rows(m, base, rows, box_rows);
}

// LSH of general float / half rows (values that are not integers times one
// power of two): FP32 hash and scan on the CUDA cores over the caller's rows
// (host float rows are copied to the device first); the bucketing is the u8
// path's. Caller holds the arena lock and has checked the arguments.
int lsh_match_float(const LshArgs& a, DeviceCtx& c, cudaStream_t st) {
    const int q_n = static_cast<int>(a.q_n), r_n = static_cast<int>(a.r_n);
    const int L_ = a.L, k = a.k;
    const int top = k < kLshMaxTopBits ? k : kLshMaxTopBits;
    const int shift = k - top, nbins = 1 << top;
    const int flip = k < 6 ? k : 6;
    const bool half = a.type == SIFT_HALF_DEVICE;
    const bool host_in = a.type == SIFT_FLOAT_HOST;
    if (!host_in && ((reinterpret_cast<uintptr_t>(a.q) & 15) || (r_n && (reinterpret_cast<uintptr_t>(a.r) & 15))))
        return SIFT_ERR_INVALID_ARG;
    const bool m_dev = !a.matches || is_device_accessible(a.matches);
    const bool i_dev = !a.nn_idx || is_device_accessible(a.nn_idx);
    const bool d_dev = !a.nn_dist || is_device_accessible(a.nn_dist);
    const bool host_out = !(m_dev && i_dev && d_dev);
    const bool multi = a.probes > 1;
    Layout L;
    const size_t o_qf = host_in ? L.take(static_cast<size_t>(q_n) * kDim * 4) : 0;
    const size_t o_rf = host_in ? L.take(static_cast<size_t>(r_n) * kDim * 4 + 16) : 0;
    const size_t o_pl = L.take(static_cast<size_t>(L_) * k * kDim);
    const size_t o_cr = L.take(static_cast<size_t>(L_) * r_n * 4 + 16);
    const size_t o_cq = L.take(static_cast<size_t>(L_) * q_n * 4);
    const size_t o_z = multi ? L.take(static_cast<size_t>(L_) * q_n * k * 4) : 0;
    const size_t o_pc = multi ? L.take(static_cast<size_t>(L_) * a.probes * q_n * 4) : 0;
    const size_t o_hist = L.take(static_cast<size_t>(L_) * nbins * 4);
    const size_t o_start = L.take(static_cast<size_t>(L_) * (nbins + 1) * 4);
    const size_t o_order = L.take(static_cast<size_t>(L_) * r_n * 4 + 16);
    const size_t o_ocode = L.take(static_cast<size_t>(L_) * r_n * 4 + 16);
    const size_t o_m = (a.matches && !m_dev) ? L.take(static_cast<size_t>(q_n) * 4) : 0;
    const size_t o_i = (a.nn_idx && !i_dev) ? L.take(static_cast<size_t>(q_n) * 8) : 0;
    const size_t o_d = (a.nn_dist && !d_dev) ? L.take(static_cast<size_t>(q_n) * 8) : 0;
    SIFT_TRY(ensure_arena(c, L.off));
    char* A = c.arena;
    const void* q_src = a.q;
    const void* r_src = a.r;
    if (host_in) {
        SIFT_CUDA(cudaMemcpyAsync(A + o_qf, a.q, static_cast<size_t>(q_n) * kDim * 4, cudaMemcpyHostToDevice, st));
        if (r_n)
            SIFT_CUDA(cudaMemcpyAsync(A + o_rf, a.r, static_cast<size_t>(r_n) * kDim * 4, cudaMemcpyHostToDevice, st));
        q_src = A + o_qf;
        r_src = A + o_rf;
    }
    // Finite values only (the same check as the exact float path).
    SIFT_CUDA(cudaMemsetAsync(c.d_status + 1, 0, 2 * sizeof(int), st));
    SIFT_CUDA(launch_abs_stats(q_src, half, q_n, c.d_status + 1, c.num_sms, st));
    SIFT_CUDA(launch_abs_stats(r_src, half, r_n, c.d_status + 1, c.num_sms, st));
    SIFT_CUDA(cudaMemcpyAsync(c.h_status + 1, c.d_status + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SIFT_CUDA(cudaStreamSynchronize(st));
    if (c.h_status[1] != 0) return SIFT_ERR_INVALID_ARG;
    int8_t* pl = reinterpret_cast<int8_t*>(A + o_pl);
    SIFT_CUDA(cudaMemcpyAsync(pl, a.planes, static_cast<size_t>(L_) * k * kDim, cudaMemcpyDefault, st));
    uint32_t* codes_r = reinterpret_cast<uint32_t*>(A + o_cr);
    uint32_t* codes_q = reinterpret_cast<uint32_t*>(A + o_cq);
    float* zq = multi ? reinterpret_cast<float*>(A + o_z) : nullptr;
    SIFT_CUDA(launch_lsh_hash_float(r_src, half, r_n, pl, L_, k, codes_r, nullptr, st));
    SIFT_CUDA(launch_lsh_hash_float(q_src, half, q_n, pl, L_, k, codes_q, zq, st));
    const uint32_t* probe_codes = codes_q;
    if (multi) {
        uint32_t* pc = reinterpret_cast<uint32_t*>(A + o_pc);
        for (int t = 0; t < L_; ++t)
            SIFT_CUDA(launch_probe_codes(codes_q + static_cast<size_t>(t) * q_n, zq + static_cast<size_t>(t) * q_n * k,
                                         q_n, k, flip, a.probes, pc + static_cast<size_t>(t) * a.probes * q_n, st));
        g_launches += L_;
        probe_codes = pc;
    }
    int* start = reinterpret_cast<int*>(A + o_start);
    int* order = reinterpret_cast<int*>(A + o_order);
    uint32_t* ocode = reinterpret_cast<uint32_t*>(A + o_ocode);
    SIFT_CUDA(launch_lsh_buckets(codes_r, r_n, L_, shift, nbins, reinterpret_cast<int*>(A + o_hist), start, order,
                                 ocode, c.num_sms, st));
    uint32_t* m_out = (a.matches && !m_dev) ? reinterpret_cast<uint32_t*>(A + o_m) : a.matches;
    int32_t* i_out = (a.nn_idx && !i_dev) ? reinterpret_cast<int32_t*>(A + o_i) : a.nn_idx;
    float* d_out = (a.nn_dist && !d_dev) ? reinterpret_cast<float*>(A + o_d) : a.nn_dist;
    SIFT_CUDA(launch_lsh_scan_float(q_src, r_src, half, q_n, r_n, L_, a.probes, shift, nbins, probe_codes, start,
                                    order, ocode, a.threshold, a.ratio ? 1 : 0, m_out, a.candidates, i_out, d_out, st));
    g_launches += 2 + (r_n > 0 ? 1 : 0) + (r_n > 0 ? 3 : 0) + 1;
    if (a.matches && !m_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.matches, m_out, static_cast<size_t>(q_n) * 4, cudaMemcpyDeviceToHost, st));
    if (a.nn_idx && !i_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.nn_idx, i_out, static_cast<size_t>(q_n) * 8, cudaMemcpyDeviceToHost, st));
    if (a.nn_dist && !d_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.nn_dist, d_out, static_cast<size_t>(q_n) * 8, cudaMemcpyDeviceToHost, st));
    if (a.sync || host_out || host_in) {
        return collect_device_status(c, st);
    }
    return SIFT_OK;
}

int lsh_match(const LshArgs& a) {
    if (a.L < 1 || a.k < 1 || a.k > 32 || a.L * a.k > kLshMaxPlanes || !a.planes) return SIFT_ERR_INVALID_ARG;
    if (a.q_n > 0x7fffffffu / 32 || a.r_n > 0x7fffffffu / 32) return SIFT_ERR_INVALID_ARG;
    // Multi-probe flips subsets of the min(6, k) lowest-margin bits: at most 2^flip distinct codes.
    const int flip = a.k < 6 ? a.k : 6;
    if (a.probes < 1 || a.probes > (1 << flip)) return SIFT_ERR_INVALID_ARG;
    if (a.candidates && !is_device_accessible(a.candidates)) return SIFT_ERR_INVALID_ARG;
    if (static_cast<long long>(a.q_n) * a.L * (a.k + a.probes) > 0x7fffffffLL) return SIFT_ERR_INVALID_ARG;
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(ensure_ready(cp, dev));
    DeviceCtx& c = *cp;
    cudaStream_t st = static_cast<cudaStream_t>(a.stream);
    ArenaLock lk(c, st);
    const int q_n = static_cast<int>(a.q_n), r_n = static_cast<int>(a.r_n);
    if (q_n == 0) return SIFT_OK;
    const int L_ = a.L, k = a.k, P = lsh_planes_padded(L_, k);
    const int top = k < kLshMaxTopBits ? k : kLshMaxTopBits;
    const int shift = k - top, nbins = 1 << top;

    const bool m_dev = !a.matches || is_device_accessible(a.matches);
    const bool i_dev = !a.nn_idx || is_device_accessible(a.nn_idx);
    const bool d_dev = !a.nn_dist || is_device_accessible(a.nn_dist);
    const bool host_out = !(m_dev && i_dev && d_dev);
    const bool planes_dev = is_device_accessible(a.planes) && !(reinterpret_cast<uintptr_t>(a.planes) & 15);

    Layout L;
    InputPlan ip;
    SIFT_TRY(plan_inputs(a.q, a.r, a.type, q_n, r_n, L, ip));
    const size_t o_pl = planes_dev ? 0 : L.take(static_cast<size_t>(L_) * k * kDim);
    const size_t o_cr = L.take(static_cast<size_t>(L_) * r_n * 4 + 16);
    const size_t o_cq = L.take(static_cast<size_t>(L_) * q_n * 4);
    const bool multi = a.probes > 1;
    const size_t o_z = multi ? L.take(static_cast<size_t>(L_) * q_n * k * 4) : 0;
    const size_t o_pc = multi ? L.take(static_cast<size_t>(L_) * a.probes * q_n * 4) : 0;
    const size_t o_hist = L.take(static_cast<size_t>(L_) * nbins * 4);
    const size_t o_start = L.take(static_cast<size_t>(L_) * (nbins + 1) * 4);
    const size_t o_order = L.take(static_cast<size_t>(L_) * r_n * 4 + 16);
    const size_t o_ocode = L.take(static_cast<size_t>(L_) * r_n * 4 + 16);
    const size_t o_m = (a.matches && !m_dev) ? L.take(static_cast<size_t>(q_n) * 4) : 0;
    const size_t o_i = (a.nn_idx && !i_dev) ? L.take(static_cast<size_t>(q_n) * 8) : 0;
    const size_t o_d = (a.nn_dist && !d_dev) ? L.take(static_cast<size_t>(q_n) * 8) : 0;
    SIFT_TRY(ensure_arena(c, L.off));
    char* A = c.arena;

    const uint8_t* qd = nullptr;
    const uint8_t* rd = nullptr;
    int vshift = 0;  // inputs were integers times 2^-vshift
    {
        const int rc = stage_inputs(c, A, ip, a.type, a.q, a.r, q_n, r_n, st, qd, rd, vshift);
        // General float values: the same hash and scan in FP32 on the caller's rows.
        if (rc == SIFT_ERR_NOT_INTEGER && a.type != SIFT_U8_DEVICE && a.type != SIFT_U8_HOST)
            return lsh_match_float(a, c, st);
        SIFT_TRY(rc);
    }
    const int8_t* pl = a.planes;
    if (!planes_dev) {
        SIFT_CUDA(cudaMemcpyAsync(A + o_pl, a.planes, static_cast<size_t>(L_) * k * kDim, cudaMemcpyDefault, st));
        pl = reinterpret_cast<const int8_t*>(A + o_pl);
    }
    uint32_t* codes_r = reinterpret_cast<uint32_t*>(A + o_cr);
    uint32_t* codes_q = reinterpret_cast<uint32_t*>(A + o_cq);
    int* hist = reinterpret_cast<int*>(A + o_hist);
    int* start = reinterpret_cast<int*>(A + o_start);
    int* order = reinterpret_cast<int*>(A + o_order);
    uint32_t* ocode = reinterpret_cast<uint32_t*>(A + o_ocode);

    CUtensorMap pmap, qmap, rmap;
    SIFT_TRY(encode_i8_rows(&pmap, pl, static_cast<uint64_t>(L_) * k, static_cast<uint32_t>(P)));
    SIFT_TRY(encode_u8_rows(&qmap, qd, q_n, 128));
    if (r_n > 0) {
        SIFT_TRY(encode_u8_rows(&rmap, rd, r_n, 128));
        SIFT_CUDA(launch_lsh_hash(rmap, pmap, r_n, P, L_, k, codes_r, nullptr, c.d_status, c.num_sms, st));
        ++g_launches;
    }
    float* zq = multi ? reinterpret_cast<float*>(A + o_z) : nullptr;
    SIFT_CUDA(launch_lsh_hash(qmap, pmap, q_n, P, L_, k, codes_q, zq, c.d_status, c.num_sms, st));
    const uint32_t* probe_codes = codes_q;
    if (multi) {
        // Per table: the query's code with the lightest subsets of its
        // lowest-margin bits flipped, [t][probe][query] as the scan reads them.
        uint32_t* pc = reinterpret_cast<uint32_t*>(A + o_pc);
        for (int t = 0; t < L_; ++t)
            SIFT_CUDA(launch_probe_codes(codes_q + static_cast<size_t>(t) * q_n, zq + static_cast<size_t>(t) * q_n * k,
                                         q_n, k, flip, a.probes, pc + static_cast<size_t>(t) * a.probes * q_n, st));
        g_launches += L_;
        probe_codes = pc;
    }
    SIFT_CUDA(launch_lsh_buckets(codes_r, r_n, L_, shift, nbins, hist, start, order, ocode, c.num_sms, st));
    uint32_t* m_out = (a.matches && !m_dev) ? reinterpret_cast<uint32_t*>(A + o_m) : a.matches;
    int32_t* i_out = (a.nn_idx && !i_dev) ? reinterpret_cast<int32_t*>(A + o_i) : a.nn_idx;
    float* d_out = (a.nn_dist && !d_dev) ? reinterpret_cast<float*>(A + o_d) : a.nn_dist;
    SIFT_CUDA(launch_lsh_scan(qd, rd, q_n, r_n, L_, a.probes, shift, nbins, probe_codes, start, order, ocode,
                              a.threshold, a.ratio ? 1 : 0, ldexpf(1.0f, -2 * vshift), m_out, a.candidates, i_out,
                              d_out, st));
    g_launches += 1 + (r_n > 0 ? 3 : 0) + 1;
    if (a.matches && !m_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.matches, m_out, static_cast<size_t>(q_n) * 4, cudaMemcpyDeviceToHost, st));
    if (a.nn_idx && !i_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.nn_idx, i_out, static_cast<size_t>(q_n) * 8, cudaMemcpyDeviceToHost, st));
    if (a.nn_dist && !d_dev)
        SIFT_CUDA(cudaMemcpyAsync(a.nn_dist, d_out, static_cast<size_t>(q_n) * 8, cudaMemcpyDeviceToHost, st));
    const bool host_in = a.type == SIFT_U8_HOST || a.type == SIFT_FLOAT_HOST || !planes_dev;
    if (a.sync || host_out || host_in) {
        return collect_device_status(c, st);
    }
    return SIFT_OK;
}

int lsh_hash(const uint8_t* x, uint32_t n, const int8_t* planes, int L_, int k, uint32_t* codes, void* stream) {
    if (L_ < 1 || k < 1 || k > 32 || L_ * k > kLshMaxPlanes || !planes || (n && (!x || !codes)))
        return SIFT_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(x) & 15) || (reinterpret_cast<uintptr_t>(planes) & 15) ||
        !is_device_accessible(planes) || (n && !is_device_accessible(x)) || (n && !is_device_accessible(codes)))
        return SIFT_ERR_INVALID_ARG;
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(ensure_ready(cp, dev));
    std::lock_guard<std::mutex> lk(cp->mu);
    if (n == 0) return SIFT_OK;
    const int P = lsh_planes_padded(L_, k);
    CUtensorMap pmap, xmap;
    SIFT_TRY(encode_i8_rows(&pmap, planes, static_cast<uint64_t>(L_) * k, static_cast<uint32_t>(P)));
    SIFT_TRY(encode_u8_rows(&xmap, x, n, 128));
    SIFT_CUDA(launch_lsh_hash(xmap, pmap, static_cast<int>(n), P, L_, k, codes, nullptr, cp->d_status, cp->num_sms,
                              static_cast<cudaStream_t>(stream)));
    ++g_launches;
    return SIFT_OK;
}

// Bucket table of given codes (the counting sort lsh_match runs on the base):
// per table, points grouped by the top min(k, 16) code bits. Replaces the
// reference's thrust sort + host run-length loop (lsh_thread_sort_reduce,
// src/lsh_h.cu:587-620) and exposes the grouping for inspection.
int lsh_buckets(const uint32_t* codes, uint32_t n, int L_, int k, int* start, int* order, uint32_t* ocode,
                void* stream) {
    if (L_ < 1 || k < 1 || k > 32 || L_ * k > kLshMaxPlanes || !start) return SIFT_ERR_INVALID_ARG;
    if (n > 0x7fffffffu / static_cast<uint32_t>(L_)) return SIFT_ERR_INVALID_ARG;
    if (n && (!codes || !order || !ocode)) return SIFT_ERR_INVALID_ARG;
    if (!is_device_accessible(start) || (n && (!is_device_accessible(codes) || !is_device_accessible(order) ||
                                               !is_device_accessible(ocode))))
        return SIFT_ERR_INVALID_ARG;
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(ensure_ready(cp, dev));
    DeviceCtx& c = *cp;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ArenaLock lk(c, st);
    const int top = k < kLshMaxTopBits ? k : kLshMaxTopBits;
    const int nbins = 1 << top;
    Layout L;
    const size_t o_hist = L.take(static_cast<size_t>(L_) * nbins * 4);
    SIFT_TRY(ensure_arena(c, L.off));
    int* hist = reinterpret_cast<int*>(c.arena + o_hist);
    SIFT_CUDA(launch_lsh_buckets(codes, static_cast<int>(n), L_, k - top, nbins, hist, start, order, ocode, c.num_sms,
                                 st));
    g_launches += n > 0 ? 3 : 0;
    return SIFT_OK;
}

// The reference draws each hyperplane component as +1 / -1 from the C
// library's rand() (make_vector_h_sum_1, src/lsh_h.cu:61-83), nbits planes per
// table in table order (make_vec_h, src/lsh_h.cu:89-100).
void reference_planes(int L_, int nbits, int8_t* out) {
    for (int t = 0; t < L_; ++t)
        for (int j = 0; j < nbits; ++j)
            for (int d = 0; d < kDim; ++d)
                out[(static_cast<size_t>(t) * nbits + j) * kDim + d] =
                    ((static_cast<float>(rand()) / static_cast<float>(RAND_MAX)) - 0.5f) >= 0 ? 1 : -1;
}

int stream_status(void* stream) {
    DeviceCtx* cp = nullptr;
    int dev = 0;
    SIFT_TRY(ensure_ready(cp, dev));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SIFT_CUDA(cudaStreamSynchronize(st));
    std::lock_guard<std::mutex> lk(cp->mu);
    return collect_device_status(*cp, st);
}

int profile_collect(int tag, double* total_ms, int* launches) {
    if (tag < 0 || tag >= kProfTags) return SIFT_ERR_INVALID_ARG;
    std::vector<ProfRecord> ev;
    {
        std::lock_guard<std::mutex> pl(g_prof_mu);
        std::vector<ProfRecord> keep;
        for (auto& p : g_prof_events) (p.tag == tag ? ev : keep).push_back(p);
        g_prof_events.swap(keep);
    }
    double tot = 0.0;
    int rc = SIFT_OK;
    for (auto& p : ev) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.e1) != cudaSuccess || cudaEventElapsedTime(&ms, p.e0, p.e1) != cudaSuccess)
            rc = SIFT_ERR_CUDA;
        tot += ms;
        cudaEventDestroy(p.e0);
        cudaEventDestroy(p.e1);
    }
    if (total_ms) *total_ms = tot;
    if (launches) *launches = static_cast<int>(ev.size());
    return rc;
}

long long launch_count() { return g_launches.load(); }
int set_variant(int v) {
    if (v < 0 || v > 3) return SIFT_ERR_INVALID_ARG;
    g_variant.store(v);
    return SIFT_OK;
}
void profile_enable(bool on) { g_profile.store(on); }

void set_last_status(int s) { t_last_status = s; }
int last_status() { return t_last_status; }

}  // namespace sift

// ------------------------------------------------------------------ C ABI --
using sift::MatchArgs;

extern "C" {

int sift_impl_cublas_2nn_sift(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n,
                              uint32_t* matches, float threshold) {
    if (!matches && q_n) return SIFT_ERR_INVALID_ARG;
    MatchArgs a{};
    a.q = q_points; a.r = r_points; a.type = type; a.q_n = q_n; a.r_n = r_n;
    a.metric = SIFT_METRIC_L2; a.threshold = threshold; a.matches = matches; a.sync = true;
    return sift::exact_match(a);
}

void sift_impl_cublas_2nn_f(void* q_points, void* r_points, int q_n, int r_n, void* sorted) {
    if (q_n < 0 || r_n < 0 || (q_n && !sorted)) { sift::set_last_status(SIFT_ERR_INVALID_ARG); return; }
    MatchArgs a{};
    a.q = q_points; a.r = r_points; a.type = SIFT_FLOAT_DEVICE; a.q_n = q_n; a.r_n = r_n;
    a.metric = SIFT_METRIC_DOT; a.threshold = 0.8f; a.sorted = static_cast<sift_float4*>(sorted); a.sync = true;
    sift::set_last_status(sift::exact_match(a));
}

void sift_impl_device_brute(void* q_points, void* r_points, int q_n, int r_n, void* sorted) {
    if (q_n < 0 || r_n < 0 || (q_n && !sorted)) { sift::set_last_status(SIFT_ERR_INVALID_ARG); return; }
    MatchArgs a{};
    a.q = q_points; a.r = r_points; a.type = SIFT_FLOAT_DEVICE; a.q_n = q_n; a.r_n = r_n;
    a.metric = SIFT_METRIC_L2; a.threshold = 0.8f; a.sorted = static_cast<sift_float4*>(sorted); a.sync = true;
    sift::set_last_status(sift::exact_match(a));
}

void sift_impl_host_brute(void* q_points, void* r_points, int q_n, int r_n, void* sorted) {
    if (q_n < 0 || r_n < 0 || (q_n && !sorted)) { sift::set_last_status(SIFT_ERR_INVALID_ARG); return; }
    MatchArgs a{};
    a.q = q_points; a.r = r_points; a.type = SIFT_FLOAT_HOST; a.q_n = q_n; a.r_n = r_n;
    a.metric = SIFT_METRIC_L2; a.threshold = 0.8f; a.sorted = static_cast<sift_float4*>(sorted); a.sync = true;
    sift::set_last_status(sift::exact_match(a));
}

int cublas_2nn_sift(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n, uint32_t* matches,
                    float threshold, cublasHandle_t, int, size_t, int) {
    return sift_impl_cublas_2nn_sift(q_points, r_points, type, q_n, r_n, matches, threshold);
}

void cublas_2nn_f(des_t_f* q_points, des_t_f* r_points, int q_n, int r_n, sift_float4* sorted, cublasHandle_t) {
    sift_impl_cublas_2nn_f(q_points, r_points, q_n, r_n, sorted);
}

void device_brute(des_t_f* q_points, des_t_f* r_points, int q_n, int r_n, sift_float4* sorted) {
    sift_impl_device_brute(q_points, r_points, q_n, r_n, sorted);
}

void host_brute(des_t_f* q_points, des_t_f* r_points, int q_points_size, int r_points_size, sift_float4* sorted) {
    sift_impl_host_brute(q_points, r_points, q_points_size, r_points_size, sorted);
}

int sift_last_status(void) { return sift::last_status(); }

int sift2nn_match(const void* q, const void* r, int type, uint32_t q_n, uint32_t r_n, int metric, float threshold,
                  uint32_t* matches, sift_float4* sorted, int32_t* nn_idx, float* nn_dist, void* stream) {
    MatchArgs a{};
    a.q = q; a.r = r; a.type = type; a.q_n = q_n; a.r_n = r_n; a.metric = metric; a.threshold = threshold;
    a.matches = matches; a.sorted = sorted; a.nn_idx = nn_idx; a.nn_dist = nn_dist; a.stream = stream;
    a.sync = false;
    return sift::exact_match(a);
}

int sift_stream_status(void* stream) { return sift::stream_status(stream); }

int sift_lsh_hash(const uint8_t* x, uint32_t n, const int8_t* planes, int L, int k, uint32_t* codes, void* stream) {
    return sift::lsh_hash(x, n, planes, L, k, codes, stream);
}

int sift_lsh_buckets(const uint32_t* codes, uint32_t n, int L, int k, int* start, int* order, uint32_t* ocode,
                     void* stream) {
    return sift::lsh_buckets(codes, n, L, k, start, order, ocode, stream);
}

int sift_lsh_match_probes(const void* q, const void* r, int type, uint32_t q_n, uint32_t r_n, const int8_t* planes,
                          int L, int k, int probes, float threshold, uint32_t* matches, int32_t* nn_idx,
                          float* nn_dist, uint32_t* candidates, void* stream) {
    sift::LshArgs a{};
    a.q = q; a.r = r; a.type = type; a.q_n = q_n; a.r_n = r_n; a.planes = planes; a.L = L; a.k = k;
    a.probes = probes; a.candidates = candidates;
    a.threshold = threshold; a.ratio = threshold > 0.0f; a.matches = matches; a.nn_idx = nn_idx; a.nn_dist = nn_dist;
    a.stream = stream; a.sync = false;
    return sift::lsh_match(a);
}

int sift_lsh_match(const void* q, const void* r, int type, uint32_t q_n, uint32_t r_n, const int8_t* planes, int L,
                   int k, float threshold, uint32_t* matches, int32_t* nn_idx, float* nn_dist, void* stream) {
    sift::LshArgs a{};
    a.q = q; a.r = r; a.type = type; a.q_n = q_n; a.r_n = r_n; a.planes = planes; a.L = L; a.k = k;
    a.threshold = threshold; a.ratio = threshold > 0.0f; a.matches = matches; a.nn_idx = nn_idx; a.nn_dist = nn_dist;
    a.stream = stream; a.sync = false;
    return sift::lsh_match(a);
}

int sift_impl_lsh_gpu(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n, uint32_t* matches, int l,
                      int nbits) {
    if (l < 1 || nbits < 1 || nbits > 32 || l * nbits > sift::kLshMaxPlanes || (q_n && !matches))
        return SIFT_ERR_INVALID_ARG;
    int8_t* planes = static_cast<int8_t*>(malloc(static_cast<size_t>(l) * nbits * sift::kDim));
    if (!planes) return SIFT_ERR_ALLOC;
    sift::reference_planes(l, nbits, planes);
    sift::LshArgs a{};
    a.q = q_points; a.r = r_points; a.type = type; a.q_n = q_n; a.r_n = r_n; a.planes = planes; a.L = l;
    a.k = nbits; a.threshold = 0.0f; a.ratio = false; a.matches = matches; a.sync = true;
    const int rc = sift::lsh_match(a);
    free(planes);
    return rc;
}

int lsh_gpu(void* q_points, void* r_points, int type, uint32_t q_n, uint32_t r_n, uint32_t* matches, float,
            cublasHandle_t, int, int l, int, int nbits) {
    return sift_impl_lsh_gpu(q_points, r_points, type, q_n, r_n, matches, l, nbits);
}

const char* sift_status_string(int s) {
    switch (s) {
        case SIFT_OK: return "ok";
        case SIFT_ERR_INVALID_ARG: return "invalid argument";
        case SIFT_ERR_CUDA: return "CUDA error";
        case SIFT_ERR_NOT_INTEGER: return "descriptor values are not integers in [0, 255]";
        case SIFT_ERR_DEVICE_TIMEOUT: return "a bounded wait inside a kernel expired";
        case SIFT_ERR_NO_DEVICE: return "no usable CUDA device";
        case SIFT_ERR_UNSUPPORTED: return "unsupported device or input";
        case SIFT_ERR_ALLOC: return "device allocation failed";
        default: return "unknown status";
    }
}

const char* sift_version(void) { return "sift2nn-b200 0.1.0 (sm_100a)"; }

long long sift_launch_count(void) { return sift::launch_count(); }
void sift_profile_enable(int on) { sift::profile_enable(on != 0); }
int sift_set_kernel_variant(int variant) { return sift::set_variant(variant); }
int sift_profile_collect(double* total_ms, int* launches) { return sift::profile_collect(0, total_ms, launches); }
int sift_profile_collect_kernel(int kernel, double* total_ms, int* launches) {
    return sift::profile_collect(kernel, total_ms, launches);
}

}  // extern "C"
