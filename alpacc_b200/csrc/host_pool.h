// Host-side widening of 32-bit values into 64-bit arrays, and the thread pool
// that runs it (host code only, no CUDA): alp_parse_host and the other host
// entry points of capi.cu hand it each chunk of parents and spans as the chunk
// lands from the device.  Kept apart from capi.cu so that the CPU tests can
// compile and check it on its own (tests/host_pool_check.cpp).
#pragma once

#include <immintrin.h>
#include <sched.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

namespace alp_host {

constexpr size_t WIDEN_SLICE = (size_t)1 << 18;  // values per widening task
constexpr int HOST_WORKERS = 8;                  // default cap on the pool's threads

// n int32 values sign-extended into int64 (AVX2, streaming stores once the
// destination is 32-byte aligned).
__attribute__((target("avx2"))) inline void widen_avx2(const int32_t* s, int64_t* d, size_t n) {
    size_t i = 0;
    for (; i < n && ((uintptr_t)(d + i) & 31); ++i) d[i] = s[i];
    for (; i + 4 <= n; i += 4) {
        const __m128i x = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i));
        _mm256_stream_si256(reinterpret_cast<__m256i*>(d + i), _mm256_cvtepi32_epi64(x));
    }
    for (; i < n; ++i) d[i] = s[i];
    _mm_sfence();
}

inline void widen(const int32_t* s, int64_t* d, size_t n) {
    static const bool avx2 = [] {
        __builtin_cpu_init();
        return __builtin_cpu_supports("avx2") != 0;
    }();
    if (avx2 && ((uintptr_t)d & 7) == 0) {
        widen_avx2(s, d, n);
        return;
    }
    for (size_t i = 0; i < n; ++i) d[i] = s[i];
}

// Worker threads for widen(): the host's CPUs this process may run on, less the
// calling thread, at most HOST_WORKERS (ALP_HOST_THREADS sets the count).
inline int host_workers() {
    if (const char* e = getenv("ALP_HOST_THREADS")) {
        const int v = atoi(e);
        if (v >= 1) return std::min(v, 256);
    }
    cpu_set_t set;
    int n = 1;
    if (sched_getaffinity(0, sizeof set, &set) == 0) n = CPU_COUNT(&set);
    return std::max(1, std::min(n - 1, HOST_WORKERS));
}

class HostPool {
  public:
    // As many of `workers` threads as the system grants; with none, the calling
    // thread widens every slice itself (help / wait).
    explicit HostPool(int workers) {
        for (int i = 0; i < workers; ++i) {
            try {
                th_.emplace_back([this] { run(); });
            } catch (...) {
                break;
            }
        }
    }
    ~HostPool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    static int slices(size_t n) { return (int)((n + WIDEN_SLICE - 1) / WIDEN_SLICE); }
    // Queue the widening of n values; *left (set to slices(n) by the caller) counts
    // the slices not yet written.
    void push(const int32_t* s, int64_t* d, size_t n, std::atomic<int>* left) {
        {
            std::lock_guard<std::mutex> lk(m_);
            for (size_t o = 0; o < n; o += WIDEN_SLICE)
                q_.push_back({s + o, d + o, std::min(WIDEN_SLICE, n - o), left});
        }
        cv_.notify_all();
    }
    // Widen one queued slice on the calling thread; false when none is queued.
    bool help() {
        Slice x;
        {
            std::lock_guard<std::mutex> lk(m_);
            if (q_.empty()) return false;
            x = q_.front();
            q_.pop_front();
            ++busy_;
        }
        finish(x);
        return true;
    }
    // Every pushed slice written.
    void wait() {
        while (help()) {
        }
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return q_.empty() && busy_ == 0; });
    }

  private:
    struct Slice {
        const int32_t* s;
        int64_t* d;
        size_t n;
        std::atomic<int>* left;
    };
    void finish(const Slice& x) {
        widen(x.s, x.d, x.n);
        x.left->fetch_sub(1, std::memory_order_release);
        std::lock_guard<std::mutex> lk(m_);
        if (--busy_ == 0 && q_.empty()) done_.notify_all();
    }
    void run() {
        for (;;) {
            Slice x;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || !q_.empty(); });
                if (q_.empty()) return;  // stopping
                x = q_.front();
                q_.pop_front();
                ++busy_;
            }
            finish(x);
        }
    }
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    std::deque<Slice> q_;
    size_t busy_ = 0;
    bool stop_ = false;
};

}  // namespace alp_host
