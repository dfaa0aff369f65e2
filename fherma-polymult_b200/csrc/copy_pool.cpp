#include "copy_pool.h"

#include <chrono>
#include <cstdlib>
#include <cstring>

namespace fpm {

int default_copy_threads() {
    if (const char* v = std::getenv("FPM_COPY_THREADS")) {
        const int t = std::atoi(v);
        if (t >= 1) return t;
    }
    const unsigned hw = std::thread::hardware_concurrency();
    return hw == 0 ? 4 : static_cast<int>(hw < 16 ? hw : 16);
}

CopyPool::CopyPool(int threads, int spin_us) : spin_us_(spin_us) {
    for (int i = 1; i < threads; ++i) workers_.emplace_back([this] { worker(); });
}

CopyPool::~CopyPool() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        stop_.store(true);
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
}

void CopyPool::run_pieces(const Job& j) {
    for (;;) {
        uint64_t c = claim_.load(std::memory_order_acquire);
        do {
            if ((c >> 32) != (j.gen & 0xFFFFFFFFu) || (c & 0xFFFFFFFFu) >= j.pieces) return;
        } while (!claim_.compare_exchange_weak(c, c + 1, std::memory_order_acq_rel));
        const size_t at = (c & 0xFFFFFFFFu) * j.piece;
        const size_t n = at + j.piece <= j.bytes ? j.piece : j.bytes - at;
        std::memcpy(j.dst + at, j.src + at, n);
        finished_.fetch_add(1, std::memory_order_acq_rel);
    }
}

void CopyPool::worker() {
    uint64_t seen = 0;
    for (;;) {
        // Spin for a while, then sleep until the next job.
        const auto t0 = std::chrono::steady_clock::now();
        while (gen_.load(std::memory_order_acquire) == seen && !stop_.load()) {
            if (std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(spin_us_)) {
                std::unique_lock<std::mutex> lock(mu_);
                cv_.wait(lock, [&] { return gen_.load(std::memory_order_acquire) != seen || stop_.load(); });
                break;
            }
        }
        if (stop_.load()) return;
        Job j;
        {
            std::lock_guard<std::mutex> lock(mu_);
            j = job_;
        }
        seen = j.gen;
        run_pieces(j);
    }
}

void CopyPool::copy(void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return;
    const size_t min_piece = 256 << 10;
    if (workers_.empty() || bytes <= min_piece) {
        std::memcpy(dst, src, bytes);
        return;
    }
    Job j;
    j.dst = static_cast<char*>(dst);
    j.src = static_cast<const char*>(src);
    j.bytes = bytes;
    const size_t want = bytes / (4 * static_cast<size_t>(threads()));
    j.piece = want > min_piece ? (want + 4095) / 4096 * 4096 : min_piece;
    j.pieces = (bytes + j.piece - 1) / j.piece;
    {
        std::lock_guard<std::mutex> lock(mu_);
        j.gen = gen_.load() + 1;
        job_ = j;
        finished_.store(0, std::memory_order_relaxed);
        claim_.store((j.gen & 0xFFFFFFFFu) << 32, std::memory_order_release);
        gen_.store(j.gen, std::memory_order_release);
    }
    cv_.notify_all();
    run_pieces(j);
    while (finished_.load(std::memory_order_acquire) < j.pieces) {
    }
}

}  // namespace fpm
