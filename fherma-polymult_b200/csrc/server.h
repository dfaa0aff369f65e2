// Serving loop: requests for products on resident points, admitted by their
// device-memory footprint and batched as they arrive.
//
// The points (Engines from fpm_init) keep their plan tables resident.  The
// server owns one device arena of a fixed budget; a request needs its
// operands, result and residue workspaces there (3 N L + 2 K N words, rounded
// to 256 bytes) and is admitted, in arrival order, once that much is free and
// a lane is idle.  A lane is a CUDA stream running one micro-batch at a time:
// the host-to-device copies of every request it took, one grouped launch per
// stage over all of them, the device-to-host copies.  Lanes run concurrently,
// so requests that arrive while others are on the GPU start as soon as a lane
// and memory free up, and their work overlaps on the device (continuous
// batching).  A server thread does the admission and polls the lanes'
// completion events; latency is measured from a request's arrival (submit)
// to the host seeing its result written.
//
// Host buffers should be pinned for the copies to run asynchronously.
#pragma once

#include "batch.h"
#include "engine.h"

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

namespace fpm {

struct ServerConfig {
    size_t budget_bytes = size_t(8) << 30;   // device arena for requests
    int lanes = 4;                           // micro-batches in flight
    int max_batch = 16;                      // requests per micro-batch
};

struct ServerStats {
    uint64_t completed = 0, failed = 0, batches = 0;
    uint32_t max_lanes_busy = 0;
    size_t peak_bytes = 0;
};

// First-fit allocator over [0, size) in 256-byte units; host bookkeeping only.
class Arena {
public:
    explicit Arena(size_t size);
    // Offset of a free range of `bytes`, or SIZE_MAX when none is large enough.
    size_t take(size_t bytes);
    void give(size_t offset, size_t bytes);
    size_t used() const { return used_; }
    size_t size() const { return size_; }

private:
    std::map<size_t, size_t> free_;   // offset -> length, coalesced
    size_t size_, used_ = 0;
};

class Server {
public:
    Server(const std::vector<Engine*>& points, const ServerConfig& cfg);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // Queues c = a b on point `point`; returns a ticket.  Thread-safe.  Throws
    // std::runtime_error when the request can never fit the arena.
    uint64_t submit(uint32_t point, const uint32_t* a, const uint32_t* b, uint32_t* c);
    // Blocks until the ticket's result is written; returns its latency in us.
    // Throws if it failed.
    double wait(uint64_t ticket);
    // Submits request i at arrival_us[i] (microseconds after the call starts),
    // waits for all, and fills latency_us[i].
    void replay(uint32_t n, const uint32_t* point, const double* arrival_us, const uint32_t* const* a,
                const uint32_t* const* b, uint32_t* const* c, double* latency_us);

    // Adds a point while the server runs (thread-safe); returns its index.
    // Requests on it may be submitted as soon as this returns.
    uint32_t add_point(Engine* e);

    ServerStats stats() const;
    size_t footprint(uint32_t point) const;
    size_t budget() const { return arena_.size(); }

private:
    using Clock = std::chrono::steady_clock;
    struct Request {
        uint32_t point;
        const uint32_t* a;
        const uint32_t* b;
        uint32_t* c;
        Clock::time_point arrival, done;
        size_t offset = SIZE_MAX, bytes = 0;
        int state = 0;   // 0 queued, 1 running, 2 done, 3 failed
    };
    struct Lane {
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
        uint32_t* err = nullptr;       // device error word of the lane's launches
        uint32_t* herr = nullptr;      // pinned copy, read after `done`
        std::vector<uint64_t> tickets;
        bool busy = false;
    };
    void loop();
    bool admit_locked();
    bool reap();
    void launch(Lane& lane);

    std::vector<Engine*> points_;      // guarded by mu_ (add_point appends)
    std::vector<size_t> footprint_;
    int device_ = -1;
    ServerConfig cfg_;
    Arena arena_;
    uint8_t* base_ = nullptr;          // device arena
    uint8_t* words_ = nullptr;         // lanes' error words
    std::vector<Lane> lanes_;
    std::vector<Request> reqs_;        // by ticket
    std::deque<uint64_t> queue_;       // arrived, not yet admitted
    mutable std::mutex mu_;
    std::condition_variable cv_;       // a request finished
    std::condition_variable work_;     // a request arrived
    std::atomic<bool> stop_{false};
    ServerStats stats_;
    std::thread thread_;
};

}  // namespace fpm
