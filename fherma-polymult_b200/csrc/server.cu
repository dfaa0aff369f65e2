// Serving loop (server.h).
#include "server.h"
#include "kernels.h"

#include <algorithm>
#include <stdexcept>
#include <string>

namespace fpm {

namespace {

constexpr size_t kUnit = 256;

size_t round_up(size_t x) { return (x + kUnit - 1) / kUnit * kUnit; }

}  // namespace

// ---------------------------------------------------------------------------

Arena::Arena(size_t size) : size_(size / kUnit * kUnit) {
    if (size_) free_[0] = size_;
}

size_t Arena::take(size_t bytes) {
    bytes = round_up(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second < bytes) continue;
        const size_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > bytes) free_[off + bytes] = len - bytes;
        used_ += bytes;
        return off;
    }
    return SIZE_MAX;
}

void Arena::give(size_t offset, size_t bytes) {
    bytes = round_up(bytes);
    used_ -= bytes;
    auto it = free_.emplace(offset, bytes).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
        it->second += next->second;
        free_.erase(next);
    }
    if (it != free_.begin()) {
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
            prev->second += it->second;
            free_.erase(it);
        }
    }
}

// ---------------------------------------------------------------------------

Server::Server(const std::vector<Engine*>& points, const ServerConfig& cfg)
    : points_(points), cfg_(cfg), arena_(cfg.budget_bytes) {
    if (points_.empty()) throw std::runtime_error("server: no points");
    if (cfg_.lanes < 1 || cfg_.lanes > 64) throw std::runtime_error("server: lanes must be in [1, 64]");
    if (cfg_.max_batch < 1 || cfg_.max_batch > kGroupMax)
        throw std::runtime_error("server: max_batch must be in [1, " + std::to_string(kGroupMax) + "]");
    int dev = -1;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    device_ = dev;
    for (Engine* e : points_) {
        if (!e) throw std::runtime_error("server: null point");
        if (e->device() != dev) throw std::runtime_error("server: every point must live on the current device");
        footprint_.push_back(3 * round_up(e->words() * 4) + 2 * round_up(e->residues() * 4));
    }
    try {
        if (arena_.size()) check(cudaMalloc(&base_, arena_.size()), "cudaMalloc (server arena)");
        check(cudaMalloc(&words_, kUnit * cfg_.lanes), "cudaMalloc (server)");
        check(cudaMemset(words_, 0, kUnit * cfg_.lanes), "memset");
        lanes_.resize(cfg_.lanes);
        for (int i = 0; i < cfg_.lanes; ++i) {
            Lane& l = lanes_[i];
            check(cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking), "stream");
            check(cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming), "event");
            l.err = reinterpret_cast<uint32_t*>(words_ + kUnit * i);
            check(cudaHostAlloc(reinterpret_cast<void**>(&l.herr), sizeof(uint32_t), cudaHostAllocDefault),
                  "cudaHostAlloc");
            *l.herr = 0;
        }
    } catch (...) {
        for (Lane& l : lanes_) {
            if (l.stream) cudaStreamDestroy(l.stream);
            if (l.done) cudaEventDestroy(l.done);
            if (l.herr) cudaFreeHost(l.herr);
        }
        if (words_) cudaFree(words_);
        if (base_) cudaFree(base_);
        throw;
    }
    thread_ = std::thread([this, dev] {
        cudaSetDevice(dev);
        loop();
    });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    work_.notify_all();
    if (thread_.joinable()) thread_.join();
    for (Lane& l : lanes_) {
        cudaStreamSynchronize(l.stream);
        cudaStreamDestroy(l.stream);
        cudaEventDestroy(l.done);
        cudaFreeHost(l.herr);
    }
    if (words_) cudaFree(words_);
    if (base_) cudaFree(base_);
}

size_t Server::footprint(uint32_t point) const {
    std::lock_guard<std::mutex> lk(mu_);
    return footprint_.at(point);
}

uint32_t Server::add_point(Engine* e) {
    if (!e) throw std::runtime_error("server: null point");
    if (e->device() != device_) throw std::runtime_error("server: every point must live on the server's device");
    std::lock_guard<std::mutex> lk(mu_);
    points_.push_back(e);
    footprint_.push_back(3 * round_up(e->words() * 4) + 2 * round_up(e->residues() * 4));
    return static_cast<uint32_t>(points_.size() - 1);
}

uint64_t Server::submit(uint32_t point, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    if (!a || !b || !c) throw std::runtime_error("server: NULL buffer");
    uint64_t t;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (point >= points_.size()) throw std::runtime_error("server: point index out of range");
        if (footprint_[point] > arena_.size()) {
            throw std::runtime_error("server: a request on point " + std::to_string(point) + " needs " +
                                     std::to_string(footprint_[point]) + " bytes of device memory; the budget is " +
                                     std::to_string(arena_.size()));
        }
        t = reqs_.size();
        Request r;
        r.point = point;
        r.a = a;
        r.b = b;
        r.c = c;
        r.arrival = Clock::now();
        reqs_.push_back(r);
        queue_.push_back(t);
    }
    work_.notify_one();
    return t;
}

double Server::wait(uint64_t ticket) {
    std::unique_lock<std::mutex> lk(mu_);
    if (ticket >= reqs_.size()) throw std::runtime_error("server: unknown ticket");
    cv_.wait(lk, [&] { return reqs_[ticket].state >= 2; });
    const Request& r = reqs_[ticket];
    if (r.state == 3) throw std::runtime_error("server: request failed on the device");
    return std::chrono::duration<double, std::micro>(r.done - r.arrival).count();
}

void Server::replay(uint32_t n, const uint32_t* point, const double* arrival_us, const uint32_t* const* a,
                    const uint32_t* const* b, uint32_t* const* c, double* latency_us) {
    std::vector<uint64_t> tickets(n);
    const Clock::time_point t0 = Clock::now();
    for (uint32_t i = 0; i < n; ++i) {
        const auto at = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(
                                 arrival_us[i]));
        // Sleep to within ~100 us of the arrival, then spin.
        const auto early = at - std::chrono::microseconds(100);
        if (Clock::now() < early) std::this_thread::sleep_until(early);
        while (Clock::now() < at) {
        }
        tickets[i] = submit(point[i], a[i], b[i], c[i]);
    }
    std::string failed;
    for (uint32_t i = 0; i < n; ++i) {
        try {
            latency_us[i] = wait(tickets[i]);
        } catch (const std::runtime_error& e) {
            latency_us[i] = -1;
            if (failed.empty()) failed = "request " + std::to_string(i) + ": " + e.what();
        }
    }
    if (!failed.empty()) throw std::runtime_error(failed);
}

ServerStats Server::stats() const {
    std::lock_guard<std::mutex> lk(mu_);
    return stats_;
}

void Server::loop() {
    std::unique_lock<std::mutex> lk(mu_);
    while (true) {
        const bool reaped = reap();
        const bool admitted = admit_locked();
        bool busy = false;
        for (const Lane& l : lanes_) busy = busy || l.busy;
        if (stop_ && !busy) break;
        if (!busy && queue_.empty()) {
            work_.wait(lk, [&] { return stop_ || !queue_.empty(); });
            continue;
        }
        if (!reaped && !admitted) {
            // Work is on the GPU: poll its completion without holding the lock.
            lk.unlock();
            std::this_thread::yield();
            lk.lock();
        }
    }
}

bool Server::reap() {
    bool any = false;
    for (Lane& l : lanes_) {
        if (!l.busy) continue;
        const cudaError_t r = cudaEventQuery(l.done);
        if (r == cudaErrorNotReady) continue;
        const auto now = Clock::now();
        const bool failed = r != cudaSuccess || *l.herr != 0;
        if (r != cudaSuccess) cudaGetLastError();
        for (uint64_t t : l.tickets) {
            Request& q = reqs_[t];
            q.done = now;
            q.state = failed ? 3 : 2;
            arena_.give(q.offset, q.bytes);
            if (failed) {
                ++stats_.failed;
            } else {
                ++stats_.completed;
            }
        }
        l.tickets.clear();
        l.busy = false;
        any = true;
    }
    if (any) cv_.notify_all();
    return any;
}

bool Server::admit_locked() {
    bool any = false;
    for (Lane& l : lanes_) {
        if (queue_.empty()) break;
        if (l.busy) continue;
        // First come, first served: take the head while it fits.
        while (!queue_.empty() && l.tickets.size() < static_cast<size_t>(cfg_.max_batch)) {
            Request& q = reqs_[queue_.front()];
            const size_t off = arena_.take(footprint_[q.point]);
            if (off == SIZE_MAX) break;
            q.offset = off;
            q.bytes = footprint_[q.point];
            q.state = 1;
            l.tickets.push_back(queue_.front());
            queue_.pop_front();
        }
        if (l.tickets.empty()) break;   // the head waits for memory
        stats_.peak_bytes = std::max(stats_.peak_bytes, arena_.used());
        launch(l);
        any = true;
    }
    uint32_t busy = 0;
    for (const Lane& l : lanes_) busy += l.busy ? 1 : 0;
    stats_.max_lanes_busy = std::max(stats_.max_lanes_busy, busy);
    return any;
}

void Server::launch(Lane& l) {
    try {
        std::vector<GroupedProduct> prods;
        check(cudaMemsetAsync(l.err, 0, sizeof(uint32_t), l.stream), "clear error word");
        for (uint64_t t : l.tickets) {
            const Request& q = reqs_[t];
            Engine* e = points_[q.point];
            uint8_t* at = base_ + q.offset;
            auto take = [&](size_t words) {
                uint32_t* p = reinterpret_cast<uint32_t*>(at);
                at += round_up(words * 4);
                return p;
            };
            GroupedProduct p{};
            p.e = e;
            p.d = e->point();
            p.d.err = l.err;
            p.a = take(e->words());
            p.b = take(e->words());
            p.c = take(e->words());
            p.A = take(e->residues());
            p.B = take(e->residues());
            const HostPlan& pl = e->plan();
            p.cost = static_cast<double>(pl.K) * pl.N * (pl.g.logN + 0.5 * pl.L);
            check(cudaMemcpyAsync(p.a, q.a, e->words() * 4, cudaMemcpyHostToDevice, l.stream), "copy a");
            check(cudaMemcpyAsync(p.b, q.b, e->words() * 4, cudaMemcpyHostToDevice, l.stream), "copy b");
            prods.push_back(p);
        }
        enqueue_grouped(prods, BatchSchedule{0, 1, 0, 0}, l.stream, GroupedLaunchEnv{});
        for (size_t i = 0; i < prods.size(); ++i) {
            const Request& q = reqs_[l.tickets[i]];
            check(cudaMemcpyAsync(q.c, prods[i].c, prods[i].e->words() * 4, cudaMemcpyDeviceToHost, l.stream),
                  "copy c");
        }
        check(cudaMemcpyAsync(l.herr, l.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, l.stream), "copy error word");
        check(cudaEventRecord(l.done, l.stream), "event record");
        l.busy = true;
        ++stats_.batches;
    } catch (const std::exception&) {
        // The launch never completed: let what was enqueued drain, then fail
        // its requests and free their memory.
        cudaStreamSynchronize(l.stream);
        cudaGetLastError();
        const auto now = Clock::now();
        for (uint64_t t : l.tickets) {
            Request& q = reqs_[t];
            q.done = now;
            q.state = 3;
            arena_.give(q.offset, q.bytes);
            ++stats_.failed;
        }
        l.tickets.clear();
        l.busy = false;
        cv_.notify_all();
    }
}

}  // namespace fpm
