// Parallel host memcpy for staging pageable buffers through pinned memory.
//
// On the B200 hosts a single thread copies pageable -> pinned at ~21 GB/s and
// eight or more threads at ~70 GB/s, against ~55 GB/s for the PCIe DMA, so the
// staging copy of chunk k + 1 (done here) hides behind the DMA of chunk k.
// (Reference counterpart: CopyPool, solve.cu:312-415.)
//
// copy() splits a job into pieces that the calling thread and the workers
// claim from an atomic counter; it returns when every piece is done.  Workers
// spin for a short while after each job (jobs come every few hundred
// microseconds during a call) and then sleep on a condition variable.
#pragma once

#include <atomic>
#include <cstdint>
#include <condition_variable>
#include <cstddef>
#include <mutex>
#include <thread>
#include <vector>

namespace fpm {

class CopyPool {
public:
    // threads: total copying threads including the caller (>= 1).
    explicit CopyPool(int threads, int spin_us = 2000);
    ~CopyPool();
    CopyPool(const CopyPool&) = delete;
    CopyPool& operator=(const CopyPool&) = delete;

    void copy(void* dst, const void* src, size_t bytes);
    int threads() const { return static_cast<int>(workers_.size()) + 1; }

private:
    struct Job {
        char* dst = nullptr;
        const char* src = nullptr;
        size_t bytes = 0, piece = 0, pieces = 0;
        uint64_t gen = 0;
    };
    void worker();
    void run_pieces(const Job& j);

    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_;
    Job job_;                               // guarded by mu_
    std::atomic<uint64_t> gen_{0};
    std::atomic<bool> stop_{false};
    // (generation << 32) | next piece: a stale worker's claim fails the
    // generation check, so it can never touch a newer job.
    std::atomic<uint64_t> claim_{0};
    std::atomic<uint64_t> finished_{0};     // pieces done in the current job
    int spin_us_;
};

// Threads for the pool: the hardware threads, capped at 16 (the memcpy rate
// saturates there).
int default_copy_threads();

}  // namespace fpm
