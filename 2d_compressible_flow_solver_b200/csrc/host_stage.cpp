// Chunked, threaded copies between pageable host arrays and device memory
// through a pinned staging buffer (host_stage.h).
#include "host_stage.h"

#include <sched.h>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace cfs {

namespace {

constexpr int kChunks = 16;       // DMA chunks per copy
constexpr int kMaxWorkers = 16;   // host copy threads (memory-bound past this)

size_t ceil_div(size_t a, size_t b) { return (a + b - 1) / b; }
size_t round_up(size_t a, size_t b) { return ceil_div(a, b) * b; }

int worker_count() {
    cpu_set_t set;
    int n = 1;
    if (sched_getaffinity(0, sizeof(set), &set) == 0) n = CPU_COUNT(&set);
    return std::max(1, std::min(n, kMaxWorkers));
}

// Byte range [a0, a1) of worker t's stripe of chunk c.
struct Plan {
    size_t bytes, chunk;
    int nch, workers;
    Plan(size_t b, int w) : bytes(b), chunk(round_up(ceil_div(b, kChunks), 4096)), nch(0), workers(w) {
        nch = static_cast<int>(ceil_div(bytes, chunk));
    }
    void chunk_range(int c, size_t& c0, size_t& c1) const {
        c0 = static_cast<size_t>(c) * chunk;
        c1 = std::min(bytes, c0 + chunk);
    }
    void stripe(int c, int t, size_t& a0, size_t& a1) const {
        size_t c0, c1;
        chunk_range(c, c0, c1);
        const size_t per = round_up(ceil_div(c1 - c0, static_cast<size_t>(workers)), 64);
        a0 = std::min(c1, c0 + static_cast<size_t>(t) * per);
        a1 = std::min(c1, a0 + per);
    }
};

// memcpy with streaming (non-temporal) stores: the destination's cache lines
// are written without being read first, so a copy moves its bytes through
// host memory twice rather than three times.  The fence orders the stores
// before the caller publishes the stripe as done.
void stream_copy(void* dst, const void* src, size_t n) {
#if defined(__SSE2__)
    char* d = static_cast<char*>(dst);
    const char* s = static_cast<const char*>(src);
    const size_t head = std::min(n, (16 - (reinterpret_cast<uintptr_t>(d) & 15)) & 15);
    std::memcpy(d, s, head);
    d += head;
    s += head;
    n -= head;
    const size_t blocks = n / 64;
    for (size_t b = 0; b < blocks; ++b, d += 64, s += 64) {
        const __m128i x0 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s));
        const __m128i x1 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + 16));
        const __m128i x2 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + 32));
        const __m128i x3 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + 48));
        _mm_stream_si128(reinterpret_cast<__m128i*>(d), x0);
        _mm_stream_si128(reinterpret_cast<__m128i*>(d + 16), x1);
        _mm_stream_si128(reinterpret_cast<__m128i*>(d + 32), x2);
        _mm_stream_si128(reinterpret_cast<__m128i*>(d + 48), x3);
    }
    std::memcpy(d, s, n - blocks * 64);
    _mm_sfence();
#else
    std::memcpy(dst, src, n);
#endif
}

// Starts work(t) on a thread for t = 0..n-1 and returns how many started; a
// thread the system refuses has its share run by the caller (nothing here
// throws past the C ABI).
template <class F>
int spawn(std::vector<std::thread>& pool, int n, F& work) {
    int made = 0;
    try {
        pool.reserve(static_cast<size_t>(n));
        for (; made < n; ++made) pool.emplace_back(work, made);
    } catch (...) {
    }
    return made;
}

}  // namespace

bool host_is_pageable(const void* p) {
    cudaPointerAttributes at{};
    const cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();  // this query's own error only
        return false;
    }
    return at.type == cudaMemoryTypeUnregistered;
}

cudaError_t upload_staged(void* dst, const void* src, size_t bytes, void* stage, cudaStream_t stream, int device) {
    (void)device;
    const Plan P(bytes, worker_count());
    std::array<std::atomic<int>, kChunks> done;
    for (auto& d : done) d.store(0, std::memory_order_relaxed);
    auto work = [&](int t) {
        for (int c = 0; c < P.nch; ++c) {
            size_t a0, a1;
            P.stripe(c, t, a0, a1);
            if (a1 > a0) stream_copy(static_cast<char*>(stage) + a0, static_cast<const char*>(src) + a0, a1 - a0);
            done[static_cast<size_t>(c)].fetch_add(1, std::memory_order_release);
        }
    };
    std::vector<std::thread> pool;
    for (int t = spawn(pool, P.workers, work); t < P.workers; ++t) work(t);
    // this thread issues each chunk's copy once every worker has staged its
    // stripe of it (the workers always finish: plain host copies)
    cudaError_t err = cudaSuccess;
    for (int c = 0; c < P.nch; ++c) {
        while (done[static_cast<size_t>(c)].load(std::memory_order_acquire) < P.workers) std::this_thread::yield();
        if (err != cudaSuccess) continue;
        size_t c0, c1;
        P.chunk_range(c, c0, c1);
        err = cudaMemcpyAsync(static_cast<char*>(dst) + c0, static_cast<const char*>(stage) + c0, c1 - c0,
                              cudaMemcpyHostToDevice, stream);
    }
    for (auto& th : pool) th.join();
    return err;
}

cudaError_t download_staged(void* dst, const void* src, size_t bytes, void* stage, cudaStream_t stream, int device) {
    const Plan P(bytes, worker_count());
    std::array<cudaEvent_t, kChunks> ev{};
    cudaError_t err = cudaSuccess;
    for (int c = 0; c < P.nch && err == cudaSuccess; ++c)
        err = cudaEventCreateWithFlags(&ev[static_cast<size_t>(c)], cudaEventDisableTiming);
    for (int c = 0; c < P.nch && err == cudaSuccess; ++c) {
        size_t c0, c1;
        P.chunk_range(c, c0, c1);
        err = cudaMemcpyAsync(static_cast<char*>(stage) + c0, static_cast<const char*>(src) + c0, c1 - c0,
                              cudaMemcpyDeviceToHost, stream);
        if (err == cudaSuccess) err = cudaEventRecord(ev[static_cast<size_t>(c)], stream);
    }
    if (err == cudaSuccess) {
        // each worker waits for a chunk's copy, then moves its stripe of it
        std::atomic<int> werr{static_cast<int>(cudaSuccess)};
        auto work = [&](int t) {
            if (cudaSetDevice(device) != cudaSuccess) {
                werr.store(static_cast<int>(cudaErrorInvalidDevice));
                return;
            }
            for (int c = 0; c < P.nch; ++c) {
                const cudaError_t e = cudaEventSynchronize(ev[static_cast<size_t>(c)]);
                if (e != cudaSuccess) {
                    werr.store(static_cast<int>(e));
                    return;
                }
                size_t a0, a1;
                P.stripe(c, t, a0, a1);
                if (a1 > a0) stream_copy(static_cast<char*>(dst) + a0, static_cast<const char*>(stage) + a0, a1 - a0);
            }
        };
        std::vector<std::thread> pool;
        for (int t = spawn(pool, P.workers, work); t < P.workers; ++t) work(t);
        for (auto& th : pool) th.join();
        err = static_cast<cudaError_t>(werr.load());
    } else {
        (void)cudaStreamSynchronize(stream);  // the staging buffer is free again before an error returns
    }
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    return err;
}

}  // namespace cfs
