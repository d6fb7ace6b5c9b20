// Per-device runtime state shared by the host entry points (api.cu,
// batch.cu): readiness, scratch arena, status words, tensor-map encoding.
#pragma once
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include "sift2nn.h"

namespace sift {
namespace detail {

constexpr int kMaxDevices = 64;
// Largest power-of-two scale 2^-s of descriptor values the exact kernels take.
constexpr int kMaxShift = 24;

struct DeviceCtx {
    std::mutex mu;            // serialises the calls that use the arena
    bool ready = false;
    int num_sms = 0;
    char* arena = nullptr;    // scratch, grown on demand, reused across calls
    size_t arena_bytes = 0;
    int* d_status = nullptr;  // [0] device error code, [1] pack flag / value stats [1..3]
    int* h_status = nullptr;  // pinned mirror of d_status
    cudaStream_t copy_stream = nullptr;  // host->device chunk copies that overlap the search
    cudaEvent_t chunk_ev[17] = {};       // per-chunk "landed" events + one "arena free" event
    cudaEvent_t arena_ev = nullptr;      // recorded after the last call's arena work
    bool arena_used = false;
};

// Holds the device's mutex for one call that uses the arena and orders the
// call's GPU work after the previous call's: the mutex only orders when work
// is enqueued, so two calls on different streams would otherwise run at the
// same time on the GPU over the same scratch. The constructor makes `st` wait
// for the event recorded by the previous call; the destructor records it on
// `st` after this call's work. Streams being captured into a graph neither
// wait nor record (a captured call is ordered by the graph's launch).
class ArenaLock {
public:
    ArenaLock(DeviceCtx& c, cudaStream_t st) : c_(c), lk_(c.mu), st_(st) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
            cudaGetLastError();
            cs = cudaStreamCaptureStatusActive;
        }
        capturing_ = cs != cudaStreamCaptureStatusNone;
        if (!capturing_ && c.arena_used && cudaStreamWaitEvent(st, c.arena_ev, 0) != cudaSuccess) cudaGetLastError();
    }
    ~ArenaLock() {
        if (capturing_) return;
        if (cudaEventRecord(c_.arena_ev, st_) == cudaSuccess)
            c_.arena_used = true;
        else
            cudaGetLastError();
    }
    ArenaLock(const ArenaLock&) = delete;
    ArenaLock& operator=(const ArenaLock&) = delete;

private:
    DeviceCtx& c_;
    std::lock_guard<std::mutex> lk_;
    cudaStream_t st_;
    bool capturing_ = false;
};

// 256-byte aligned bump layout over the arena.
struct Layout {
    size_t off = 0;
    size_t take(size_t bytes) {
        off = (off + 255) & ~static_cast<size_t>(255);
        const size_t o = off;
        off += bytes;
        return o;
    }
};

extern std::atomic<long long> g_launches;

// Context of the current device (initialised on first use; sm_100 only).
int ensure_ready(DeviceCtx*& out, int& dev);
// Grows c's arena to at least `bytes` (synchronises the device when it grows).
int ensure_arena(DeviceCtx& c, size_t bytes);
bool is_device_accessible(const void* p);
// u8 rows of 128 bytes: dims {128, rows}, box {128, box_rows}, SWIZZLE_128B.
int encode_u8_rows(CUtensorMap* m, const void* base, uint64_t rows, uint32_t box_rows);
// BF16 matrix [rows][inner] (row pitch inner * 2 bytes): box {box_inner, box_rows},
// SWIZZLE_128B (box_inner * 2 <= 128), rows past the end read as zeros.
int encode_bf16_2d(CUtensorMap* m, const void* base, uint64_t inner, uint64_t rows, uint32_t box_inner,
                   uint32_t box_rows);
int map_cuda(cudaError_t e);
// Reads and clears the device status words. Caller has synchronised `st`.
int collect_device_status(DeviceCtx& c, cudaStream_t st);
// Benchmark timing of one kernel launch on `st` (CUDA events recorded on the
// launching stream when profiling is enabled; collected by tag).
enum ProfTag : int { kProfSearch = 0, kProfHash = 1, kProfScan = 2, kProfTags = 3 };
class ProfSpan {
public:
    ProfSpan(cudaStream_t st, int tag);
    void end();
    ~ProfSpan();
    ProfSpan(const ProfSpan&) = delete;
    ProfSpan& operator=(const ProfSpan&) = delete;

private:
    cudaStream_t st_;
    int tag_;
    cudaEvent_t e0_ = nullptr;
};

// Fault injection for the failure-detection tests (faults.cu): launches the
// wait-expiry probe on `st` when armed, recording into *err.
cudaError_t maybe_inject_wait_expiry(int* err, cudaStream_t st);
// True when the next arena request is armed to fail.
bool arena_fault();

}  // namespace detail
}  // namespace sift

#define SIFT_TRY(expr)                  \
    do {                                \
        int _rc = (expr);               \
        if (_rc != SIFT_OK) return _rc; \
    } while (0)
#define SIFT_CUDA(expr) SIFT_TRY(::sift::detail::map_cuda(expr))
