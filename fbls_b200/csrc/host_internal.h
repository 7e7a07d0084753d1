// Internal to the library's host code (host.cu, host_maps.cu, host_next.cu):
// the context and family handles behind the C ABI's opaque types, and the
// helpers every host file uses (error reporting, workspace growth, page-locked
// staging, a small host thread pool).
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/fbls_b200.h"

namespace fbls {

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct PinBuf {  // page-locked host memory
    void* ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace fbls

struct fbls_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::string error;
    bool profile = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool kernel_timing = false;
    cudaEvent_t timer[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> pool;  // per-launch timing events
    fbls_counters counters{};
    // Workspace, grown on demand and reused across bands and calls.
    fbls::DevBuf cum, cum32, hist, parts, keys, tflags;  // per launch
    fbls::DevBuf pass_in, pass_out;  // per session: every pass's inputs and outputs
    fbls::DevBuf evidence, fault;
    fbls::DevBuf steal;   // the work counter of a persistent fold grid
    fbls::DevBuf family;  // observations of the star a batch worker is searching
    fbls::DevBuf mapbin;  // time-binned observations of a coarse map
    fbls::DevBuf feat;    // the proposal network's input made from coarse maps
    fbls::DevBuf rescore; // peak-selection rescoring: rows, masks, times and results
    fbls::PinBuf pin_up, pin_down, pin_down2;  // staging of a session's upload and download (two sessions in flight)
    std::vector<fbls_ctx*> workers;  // fbls_search_batch worker contexts, kept for reuse
};

struct fbls_ready {
    fbls_ctx* ctx = nullptr;
    int device = 0;          // the device holding time/v/w; fbls_free_ready reads it, not ctx, which may be gone
    double* time = nullptr;  // n
    double* v = nullptr;     // n
    double* w = nullptr;     // n
    uint32_t n = 0;
    double baseline_norm = 0.0;
    double origin = 0.0;
    double residual_energy = 0.0;
    double t_last = 0.0;
    std::vector<double> time_host;  // for the fold's chunk boundaries
    bool owned = true;              // time/v/w allocated for this handle (else a context's buffer)
};

namespace fbls {

// The tile scan's mode for a precision_mode of the C ABI: 0 (the reference's
// f32 pre-rank, f64 rescans and winner) -> 1, 1 (f64 ranking) -> 0, 2 (the
// f32 form: f32 ranking and winner, no f64 rows) -> 2.
inline int scan_mode(uint32_t precision_mode) { return precision_mode == 0 ? 1 : precision_mode == 1 ? 0 : 2; }

inline int fail(fbls_ctx* ctx, int status, const std::string& message) {
    if (ctx) ctx->error = message;
    return status;
}

inline int cuda_fail(fbls_ctx* ctx, cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    return fail(ctx, FBLS_ERR_CUDA, m);
}

#define CK(call, where)                                   \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
    } while (0)

inline cudaError_t ensure(DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return cudaSuccess;
    if (b.ptr) {
        cudaError_t e = cudaFree(b.ptr);
        if (e != cudaSuccess) return e;
        b.ptr = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes + bytes / 4;
    cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) return e;
    b.bytes = want;
    return cudaSuccess;
}

inline void release(DevBuf& b) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
}

template <typename T>
inline T* as(DevBuf& b) {
    return reinterpret_cast<T*>(b.ptr);
}

// Fold budget in MiB: the configured value capped at half of the free device
// memory (Gpu::fold_budget_mib, scan.rs:93-98).
inline double fold_budget_mib(double configured) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return configured;
    double cap = (double)free_b / 1048576.0 / 2.0;
    return configured < cap ? configured : cap;
}

inline double now_seconds() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

inline cudaError_t ensure_pinned(PinBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 256;
    if (b.bytes >= bytes) return cudaSuccess;
    if (b.ptr) {
        cudaError_t e = cudaFreeHost(b.ptr);
        if (e != cudaSuccess) return e;
        b.ptr = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes + bytes / 4;
    cudaError_t e = cudaHostAlloc(&b.ptr, want, cudaHostAllocDefault);
    if (e != cudaSuccess) return e;
    b.bytes = want;
    return cudaSuccess;
}

// Runs f(i) for i in [0, n) on up to 16 host threads, the caller's included.
// Fewer than PARALLEL_MIN items run on the caller's thread: a single star's
// few passes plan in milliseconds, and starting threads for them only adds
// the risk of waiting on a descheduled one when the host's cores are busy.
constexpr size_t PARALLEL_MIN = 32;
template <typename F>
void parallel_for(size_t n, F f) {
    const size_t threads = std::min<size_t>(n, std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
    if (threads <= 1 || n < PARALLEL_MIN) {
        for (size_t i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t i; (i = next.fetch_add(1)) < n;) f(i);
    };
    std::vector<std::thread> pool;
    for (size_t k = 1; k < threads; k++) pool.emplace_back(work);
    work();
    for (std::thread& t : pool) t.join();
}

}  // namespace fbls
