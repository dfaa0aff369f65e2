// Batched products: many points of uneven N and q width in one graph of
// grouped launches.
//
// Each product keeps its own resident plan (an Engine from fpm_init).  The
// batch owns one device slab with every product's operands, result and residue
// workspaces, so its launch graph is fixed: one grouped decompose launch for
// all products, per transform geometry (logR, logS) a grouped column / row /
// inverse-column chain whose items are groups of a product's primes, and one
// grouped CRT launch, all captured once as a CUDA graph and replayed.
//
// The schedule -- whether the geometry chains run as parallel graph branches,
// the order of the items, how many primes one transform item carries,
// whether the transform grids are persistent, and from which size a product
// takes the one-product pipelines for decompose and CRT -- is chosen by Batch::tune,
// which times every candidate on this batch and keeps the fastest.
#pragma once

#include "engine.h"
#include "group.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <vector>

namespace fpm {

struct BatchSchedule {
    int layout = 1;        // 0 one stream; 1 geometry chains as branches between the shared
                           // decompose and CRT; 2 a whole branch (decompose .. CRT) per geometry;
                           // 3 one launch per stage: each transform pass covers every R = 64
                           // product whatever its row length (mixed-geometry kernels)
    int order = 1;         // 0 products as given; 1 largest first
    int prime_group = 0;   // primes per transform item; 0 = all of a product's primes
    int grid = 0;          // transform grids: 0 one block per tile; k > 0 persistent,
                           // k x (resident blocks per SM) x SMs
    int pipe_min_log_n = 0;   // products with logN >= this (0: none) take the pipelined
                              // decompose and CRT, one launch each, instead of the grouped ones
};

// One product of a grouped launch sequence: its point (with the error word
// the launches should report to) and its device buffers.
struct GroupedProduct {
    const Engine* e;
    DevPoint d;
    uint32_t *a, *b, *c, *A, *B;   // limbs N x L (a, b in; c out), residues K x N
    double cost;                   // relative work, for ordering
};

// Streams and events a layout with branches uses (created beforehand, so the
// sequence can be captured), and the resident blocks per SM of the grouped
// transform kernels (persistent grids).
struct GroupedLaunchEnv {
    std::vector<cudaStream_t> branches;   // one per transform geometry
    std::vector<cudaEvent_t> events;      // two per geometry
    const std::map<uint64_t, int>* occupancy = nullptr;
    int sms = 0;
};

uint64_t occupancy_key(int pass, uint32_t logR, uint32_t logS, bool lazy);

// Enqueues every product's decompose, transform chain and CRT as grouped
// launches on st (and, for layouts 1 and 2, the branches); returns the number
// of kernel launches.
int enqueue_grouped(const std::vector<GroupedProduct>& prods, const BatchSchedule& s, cudaStream_t st,
                    const GroupedLaunchEnv& env);

class Batch {
public:
    // All engines on the current device; the batch does not own them, and
    // they must outlive it.
    explicit Batch(const std::vector<Engine*>& engines);
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    size_t size() const { return prods_.size(); }
    // Device limbs of product i (N_i x L_i u32 each): write a and b, read c.
    uint32_t* a(size_t i) const { return prods_.at(i).a; }
    uint32_t* b(size_t i) const { return prods_.at(i).b; }
    uint32_t* c(size_t i) const { return prods_.at(i).c; }
    size_t device_bytes() const { return slab_bytes_; }

    const BatchSchedule& schedule() const { return sched_; }
    void set_schedule(const BatchSchedule& s);   // recaptures the graph

    // Every product of the batch on its device buffers: one graph launch on st.
    void run_device(cudaStream_t st);
    // The same from host arrays (a[i], b[i] in, c[i] out); returns when every
    // c[i] is written.  The products run as up to four sub-batches (separate
    // graphs) so each one's copies overlap the others' kernels.
    void run_host(const uint32_t* const* a, const uint32_t* const* b, uint32_t* const* c);

    // Times each candidate schedule (one warm-up and `reps` timed graph
    // replays, minimum kept) and keeps the fastest; returns its time in us.
    double tune(int reps);

    // Launches in one replay of the graph (kernel nodes).
    int launches() const { return launches_; }

    // Reads and clears the batch's error word (nonzero: a pipeline wait in a
    // tensor-core kernel timed out); synchronous.
    uint32_t take_error();

private:
    void build_graph();
    void build_io_graphs();
    cudaGraphExec_t capture(const std::vector<GroupedProduct>& prods, int* launches);
    void release_graph();
    cudaStream_t branch(size_t i);

    std::vector<GroupedProduct> prods_;
    BatchSchedule sched_{};
    void* slab_ = nullptr;
    size_t slab_bytes_ = 0;
    uint32_t* err_ = nullptr;
    int sms_ = 0;
    int launches_ = 0;
    cudaStream_t stream_ = nullptr;   // capture origin and host-path copies
    std::vector<cudaStream_t> branches_;
    std::vector<cudaEvent_t> events_;
    std::map<uint64_t, int> occupancy_;   // resident blocks per SM, per grouped transform kernel
    cudaGraphExec_t exec_ = nullptr;
    // Host path: sub-batches, their graphs, copy streams and events.
    static constexpr size_t kIoGroups = 4;
    std::vector<std::vector<size_t>> io_groups_;
    std::vector<cudaGraphExec_t> io_exec_;
    std::vector<cudaEvent_t> io_events_;
    cudaStream_t copy_ = nullptr;
    cudaStream_t out_ = nullptr;
};

}  // namespace fpm
