// Batched products: grouped launches captured as one CUDA graph (batch.h).
#include "batch.h"
#include "kernels.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <tuple>

namespace fpm {

namespace {

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Fills GroupTables item by item and launches each when it is full.
struct TableFill {
    std::unique_ptr<GroupTable> t{new GroupTable};
    TableFill() { reset(); }
    void reset() {
        std::memset(t.get(), 0, sizeof(GroupTable));
    }
    bool full() const { return t->count == static_cast<uint32_t>(kGroupMax); }
    void add(const DevPoint& d, uint32_t* a, uint32_t* b, uint32_t* A, uint32_t* B, uint32_t* c, uint32_t j0,
             uint32_t blocks) {
        GroupItem& it = t->item[t->count];
        it.d = d;
        it.a = a;
        it.b = b;
        it.A = A;
        it.B = B;
        it.c = c;
        it.j0 = j0;
        t->total += blocks;
        t->count += 1;
        t->first[t->count] = t->total;
    }
};

struct TransformClass {
    uint32_t logR, logS;
    bool lazy;
    bool operator<(const TransformClass& o) const {
        return std::tie(logR, logS, lazy) < std::tie(o.logR, o.logS, o.lazy);
    }
};

}  // namespace

uint64_t occupancy_key(int pass, uint32_t logR, uint32_t logS, bool lazy) {
    return (static_cast<uint64_t>(pass) << 32) | (logR << 16) | (logS << 1) | (lazy ? 1u : 0u);
}

int enqueue_grouped(const std::vector<GroupedProduct>& prods_, const BatchSchedule& sched_, cudaStream_t st,
                    const GroupedLaunchEnv& env) {
    int launches_ = 0;
    std::vector<size_t> ord(prods_.size());
    std::iota(ord.begin(), ord.end(), size_t(0));
    if (sched_.order == 1) {
        std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return prods_[x].cost > prods_[y].cost; });
    }
    // Products by transform geometry; N <= 1024 runs the one-block-per-prime
    // kernel, product by product.
    std::map<TransformClass, std::vector<size_t>> classes;
    std::vector<size_t> small;
    for (size_t i : ord) {
        const DevPoint& d = prods_[i].d;
        if (d.logN <= kSmallLogN) {
            small.push_back(i);
        } else {
            classes[TransformClass{d.logR, d.logS, d.lazy != 0}].push_back(i);
        }
    }
    TableFill fill;
    // Large products may take the one-product pipelines for decompose and CRT.
    auto piped = [&](const GroupedProduct& p) {
        return sched_.pipe_min_log_n > 0 && static_cast<int>(p.d.logN) >= sched_.pipe_min_log_n &&
               p.e->dec_consts() != nullptr;
    };

    auto decompose = [&](const std::vector<size_t>& list, cudaStream_t s) {
        fill.reset();
        auto flush = [&] {
            if (fill.t->count) {
                launch_decompose_tc_group(*fill.t, s);
                ++launches_;
            }
            fill.reset();
        };
        for (size_t i : list) {
            const GroupedProduct& p = prods_[i];
            if (p.e->simt()) {
                launch_decompose(p.d, p.a, p.A, 0, 0, p.d.N, s);
                launch_decompose(p.d, p.b, p.B, 1, 0, p.d.N, s);
                launches_ += 2;
                continue;
            }
            if (piped(p)) {
                launch_decompose_pipe(p.d, *p.e->dec_consts(), p.a, p.b, p.A, p.B, 0, 0, p.d.N, p.e->sms(), s);
                ++launches_;
                continue;
            }
            if (fill.full()) flush();
            fill.add(p.d, p.a, p.b, p.A, p.B, p.c, 0, decompose_tc_group_blocks(p.d.N));
        }
        flush();
    };
    auto crt = [&](const std::vector<size_t>& list, cudaStream_t s) {
        fill.reset();
        auto flush = [&] {
            if (fill.t->count) {
                launch_crt_tc_group(*fill.t, s);
                ++launches_;
            }
            fill.reset();
        };
        for (size_t i : list) {
            const GroupedProduct& p = prods_[i];
            if (p.e->simt() || !crt_uses_tc(p.e->plan())) {
                launch_crt(p.d, p.A, p.c, 0, p.d.N, s);
                ++launches_;
                continue;
            }
            if (piped(p) && p.e->crt_consts() && crt_pipe_supported(p.d, *p.e->crt_consts(), p.A, 0, p.d.N)) {
                launch_crt_pipe(p.d, *p.e->crt_consts(), p.A, p.c, 0, p.d.N, p.e->sms(), s);
                ++launches_;
                continue;
            }
            if (fill.full()) flush();
            fill.add(p.d, p.a, p.b, p.A, p.B, p.c, 0, crt_tc_group_blocks(p.d.N));
        }
        flush();
    };
    auto small_ntt = [&](const std::vector<size_t>& list, cudaStream_t s) {
        for (size_t i : list) {
            launch_ntt(prods_[i].d, prods_[i].A, prods_[i].B, kRowProduct, s);
            ++launches_;
        }
    };
    // One geometry's chain: every item (a group of one product's primes)
    // through the column pass, the fused row pass, the inverse column pass.
    auto transform = [&](const TransformClass& g, const std::vector<size_t>& list, cudaStream_t s) {
        struct Item {
            size_t p;
            uint32_t j0, nj;
        };
        std::vector<Item> items;
        if (sched_.prime_group <= 0) {
            for (size_t i : list) items.push_back({i, 0, static_cast<uint32_t>(prods_[i].d.K)});
        } else {
            // Round robin over the products, prime group by prime group.
            const uint32_t grp = static_cast<uint32_t>(sched_.prime_group);
            for (uint32_t r = 0;; ++r) {
                bool any = false;
                for (size_t i : list) {
                    const uint32_t K = static_cast<uint32_t>(prods_[i].d.K), j0 = r * grp;
                    if (j0 >= K) continue;
                    items.push_back({i, j0, std::min(grp, K - j0)});
                    any = true;
                }
                if (!any) break;
            }
        }
        for (int pass : {int(kPassColFwd), int(kPassRow), int(kPassColInv)}) {
            if (pass != kPassRow && g.logR == 0) continue;
            const uint32_t per = ntt_blocks_per_prime(pass, g.logR, g.logS);
            uint32_t grid = 0;
            if (sched_.grid > 0) {
                grid = static_cast<uint32_t>(sched_.grid) * static_cast<uint32_t>(env.sms) *
                       static_cast<uint32_t>(std::max(1, env.occupancy->at(occupancy_key(pass, g.logR, g.logS, g.lazy))));
            }
            fill.reset();
            auto flush = [&] {
                if (fill.t->count) {
                    launch_ntt_group(*fill.t, pass, g.logR, g.logS, g.lazy, grid, s);
                    ++launches_;
                }
                fill.reset();
            };
            for (const Item& it : items) {
                if (fill.full()) flush();
                const GroupedProduct& p = prods_[it.p];
                fill.add(p.d, p.a, p.b, p.A, p.B, p.c, it.j0, it.nj * per);
            }
            flush();
        }
    };

    // Every product of mixed-row-length geometry (R = 64) through each pass in
    // one launch (layout 3): items as in transform(), any row length.
    auto transform_mixed = [&](const std::vector<size_t>& list, bool lazy, cudaStream_t s) {
        struct Item {
            size_t p;
            uint32_t j0, nj;
        };
        std::vector<Item> items;
        uint32_t max_log_s = 6;
        for (size_t i : list) max_log_s = std::max(max_log_s, prods_[i].d.logS);
        if (sched_.prime_group <= 0) {
            for (size_t i : list) items.push_back({i, 0, static_cast<uint32_t>(prods_[i].d.K)});
        } else {
            const uint32_t grp = static_cast<uint32_t>(sched_.prime_group);
            for (uint32_t r = 0;; ++r) {
                bool any = false;
                for (size_t i : list) {
                    const uint32_t K = static_cast<uint32_t>(prods_[i].d.K), j0 = r * grp;
                    if (j0 >= K) continue;
                    items.push_back({i, j0, std::min(grp, K - j0)});
                    any = true;
                }
                if (!any) break;
            }
        }
        for (int pass : {int(kPassColFwd), int(kPassRow), int(kPassColInv)}) {
            uint32_t grid = 0;
            if (sched_.grid > 0) {
                // (Sub-batches of the host path may have a smaller largest row.)
                const auto it = env.occupancy->find(occupancy_key(pass, 63, max_log_s, lazy));
                const int occ = it != env.occupancy->end() ? it->second : ntt_mixed_occupancy(pass, lazy, max_log_s);
                grid = static_cast<uint32_t>(sched_.grid) * static_cast<uint32_t>(env.sms) *
                       static_cast<uint32_t>(std::max(1, occ));
            }
            fill.reset();
            auto flush = [&] {
                if (fill.t->count) {
                    launch_ntt_mixed(*fill.t, pass, lazy, max_log_s, grid, s);
                    ++launches_;
                }
                fill.reset();
            };
            for (const Item& it : items) {
                if (fill.full()) flush();
                const GroupedProduct& p = prods_[it.p];
                fill.add(p.d, p.a, p.b, p.A, p.B, p.c, it.j0, ntt_mixed_blocks(pass, p.d.logS, it.nj));
            }
            flush();
        }
    };

    size_t ev = 0;
    auto fork = [&](cudaStream_t from, cudaStream_t to) {
        check(cudaEventRecord(env.events.at(ev), from), "event record");
        check(cudaStreamWaitEvent(to, env.events.at(ev), 0), "stream wait");
        ++ev;
    };
    std::vector<size_t> all(ord);
    if (sched_.layout == 0) {
        decompose(all, st);
        for (auto& kv : classes) transform(kv.first, kv.second, st);
        small_ntt(small, st);
        crt(all, st);
    } else if (sched_.layout == 1) {
        decompose(all, st);
        size_t b = 0;
        std::vector<cudaStream_t> used;
        for (auto& kv : classes) {
            cudaStream_t s = env.branches.at(b++);
            fork(st, s);
            transform(kv.first, kv.second, s);
            used.push_back(s);
        }
        small_ntt(small, st);
        for (cudaStream_t s : used) fork(s, st);
        crt(all, st);
    } else if (sched_.layout == 3) {
        // One launch per stage: grouped decompose, the three transform passes
        // over every R = 64 product at once (per prime window), grouped CRT.
        // Other geometries (N <= 2048, N >= 2^18) keep their own launches.
        decompose(all, st);
        std::vector<size_t> mixed[2];
        for (auto& kv : classes) {
            bool ok = true;
            for (size_t i : kv.second) ok = ok && ntt_mixed_ok(prods_[i].d);
            if (ok) {
                mixed[kv.first.lazy ? 1 : 0].insert(mixed[kv.first.lazy ? 1 : 0].end(), kv.second.begin(),
                                                    kv.second.end());
            } else {
                transform(kv.first, kv.second, st);
            }
        }
        for (int lz = 0; lz < 2; ++lz) {
            if (mixed[lz].empty()) continue;
            // Keep the schedule's product order (classes regrouped them).
            std::vector<size_t> list;
            for (size_t i : ord)
                if (std::find(mixed[lz].begin(), mixed[lz].end(), i) != mixed[lz].end()) list.push_back(i);
            transform_mixed(list, lz == 1, st);
        }
        small_ntt(small, st);
        crt(all, st);
    } else {
        size_t b = 0;
        std::vector<cudaStream_t> used;
        for (auto& kv : classes) {
            cudaStream_t s = env.branches.at(b++);
            fork(st, s);
            decompose(kv.second, s);
            transform(kv.first, kv.second, s);
            crt(kv.second, s);
            used.push_back(s);
        }
        decompose(small, st);
        small_ntt(small, st);
        crt(small, st);
        for (cudaStream_t s : used) fork(s, st);
    }
    check(cudaGetLastError(), "batch launch");
    return launches_;
}


Batch::Batch(const std::vector<Engine*>& engines) {
    if (engines.empty()) throw std::runtime_error("batch: no products");
    int dev = -1;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    size_t bytes = 0;
    for (Engine* e : engines) {
        if (!e) throw std::runtime_error("batch: null context");
        if (e->device() != dev) throw std::runtime_error("batch: every context must live on the current device");
        bytes += 3 * align256(e->words() * 4) + 2 * align256(e->residues() * 4);
    }
    bytes += 256;   // error word
    try {
        check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev), "SM count");
        check(cudaMalloc(&slab_, bytes), "cudaMalloc (batch)");
        slab_bytes_ = bytes;
        check(cudaMemset(slab_, 0, bytes), "memset (batch)");
        uint8_t* at = static_cast<uint8_t*>(slab_);
        auto take = [&](size_t n) {
            uint32_t* p = reinterpret_cast<uint32_t*>(at);
            at += align256(n * 4);
            return p;
        };
        err_ = take(1);
        for (Engine* e : engines) {
            GroupedProduct p{};
            p.e = e;
            p.d = e->point();
            p.d.err = err_;
            p.a = take(e->words());
            p.b = take(e->words());
            p.c = take(e->words());
            p.A = take(e->residues());
            p.B = take(e->residues());
            const HostPlan& pl = e->plan();
            p.cost = static_cast<double>(pl.K) * pl.N * (pl.g.logN + 0.5 * pl.L);
            prods_.push_back(p);
        }
        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
        check(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking), "stream");
        check(cudaStreamCreateWithFlags(&out_, cudaStreamNonBlocking), "stream");
        build_graph();
    } catch (...) {
        release_graph();
        for (auto s : branches_) cudaStreamDestroy(s);
        for (auto ev : events_) cudaEventDestroy(ev);
        for (cudaStream_t x : {copy_, out_})
            if (x) cudaStreamDestroy(x);
        if (stream_) cudaStreamDestroy(stream_);
        if (slab_) cudaFree(slab_);
        throw;
    }
}

Batch::~Batch() {
    for (cudaStream_t x : {copy_, out_, stream_})
        if (x) cudaStreamSynchronize(x);
    release_graph();
    for (auto s : branches_) cudaStreamDestroy(s);
    for (auto ev : events_) cudaEventDestroy(ev);
    for (auto ev : io_events_) cudaEventDestroy(ev);
    for (cudaStream_t x : {copy_, out_})
        if (x) cudaStreamDestroy(x);
    if (stream_) cudaStreamDestroy(stream_);
    if (slab_) cudaFree(slab_);
}

void Batch::release_graph() {
    if (exec_) cudaGraphExecDestroy(exec_);
    exec_ = nullptr;
    for (cudaGraphExec_t e : io_exec_) cudaGraphExecDestroy(e);
    io_exec_.clear();
    io_groups_.clear();
}

cudaStream_t Batch::branch(size_t i) {
    while (branches_.size() <= i) {
        cudaStream_t s = nullptr;
        check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        branches_.push_back(s);
    }
    return branches_[i];
}

void Batch::set_schedule(const BatchSchedule& s) {
    if (s.layout < 0 || s.layout > 3 || s.order < 0 || s.order > 1 || s.prime_group < 0 || s.grid < 0 ||
        s.pipe_min_log_n < 0 || s.pipe_min_log_n > 22)
        throw std::runtime_error("batch: invalid schedule");
    sched_ = s;
    build_graph();
}

void Batch::build_graph() {
    check(cudaStreamSynchronize(stream_), "batch sync");
    release_graph();
    // Events and branch streams used by the capture, created outside it.
    const size_t need = 2 * (prods_.size() + 8);
    while (events_.size() < need) {
        cudaEvent_t ev = nullptr;
        check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
        events_.push_back(ev);
    }
    // One branch stream per transform geometry, and the resident blocks per SM
    // of every grouped transform kernel (persistent grids).
    size_t classes = 0;
    std::vector<uint32_t> seen;
    for (const GroupedProduct& p : prods_) {
        if (p.d.logN <= kSmallLogN) continue;
        const uint32_t key = p.d.logR * 64 + p.d.logS * 2 + (p.d.lazy ? 1 : 0);
        if (std::find(seen.begin(), seen.end(), key) != seen.end()) continue;
        seen.push_back(key);
        ++classes;
        for (int pass : {int(kPassColFwd), int(kPassRow), int(kPassColInv)}) {
            if (pass != kPassRow && p.d.logR == 0) continue;
            const uint64_t k = occupancy_key(pass, p.d.logR, p.d.logS, p.d.lazy != 0);
            if (!occupancy_.count(k)) occupancy_[k] = ntt_group_occupancy(pass, p.d.logR, p.d.logS, p.d.lazy != 0);
        }
    }
    // The mixed-geometry kernels (layout 3), keyed by the largest row length.
    uint32_t max_log_s[2] = {0, 0};
    for (const GroupedProduct& p : prods_)
        if (ntt_mixed_ok(p.d)) max_log_s[p.d.lazy ? 1 : 0] = std::max(max_log_s[p.d.lazy ? 1 : 0], p.d.logS);
    for (int lz = 0; lz < 2; ++lz) {
        if (!max_log_s[lz]) continue;
        for (int pass : {int(kPassColFwd), int(kPassRow), int(kPassColInv)}) {
            const uint64_t k = occupancy_key(pass, 63, max_log_s[lz], lz == 1);
            if (!occupancy_.count(k)) occupancy_[k] = ntt_mixed_occupancy(pass, lz == 1, max_log_s[lz]);
        }
    }
    for (size_t i = 0; i < classes; ++i) branch(i);
    exec_ = capture(prods_, &launches_);
}

cudaGraphExec_t Batch::capture(const std::vector<GroupedProduct>& prods, int* launches) {
    GroupedLaunchEnv env;
    env.branches = branches_;
    env.events = events_;
    env.occupancy = &occupancy_;
    env.sms = sms_;
    cudaGraph_t graph = nullptr;
    check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        const int n = enqueue_grouped(prods, sched_, stream_, env);
        if (launches) *launches = n;
    } catch (...) {
        cudaStreamEndCapture(stream_, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        throw;
    }
    check(cudaStreamEndCapture(stream_, &graph), "end capture");
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    check(e, "graph instantiate");
    return exec;
}

// Sub-batches for the host path: the products in schedule order, cut into up
// to kIoGroups runs of about equal work, each captured as its own graph.
void Batch::build_io_graphs() {
    if (!io_exec_.empty()) return;
    std::vector<size_t> ord(prods_.size());
    std::iota(ord.begin(), ord.end(), size_t(0));
    if (sched_.order == 1) {
        std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return prods_[x].cost > prods_[y].cost; });
    }
    double total = 0;
    for (const GroupedProduct& p : prods_) total += p.cost;
    const size_t groups = std::min<size_t>(kIoGroups, prods_.size());
    io_groups_.assign(1, {});
    double acc = 0;
    for (size_t k = 0; k < ord.size(); ++k) {
        io_groups_.back().push_back(ord[k]);
        acc += prods_[ord[k]].cost;
        const size_t left = ord.size() - k - 1;
        if (io_groups_.size() < groups && left > 0 && acc >= total * io_groups_.size() / groups)
            io_groups_.emplace_back();
    }
    for (const std::vector<size_t>& g : io_groups_) {
        std::vector<GroupedProduct> sub;
        for (size_t i : g) sub.push_back(prods_[i]);
        io_exec_.push_back(capture(sub, nullptr));
    }
    while (io_events_.size() < 2 * io_groups_.size()) {
        cudaEvent_t ev = nullptr;
        check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
        io_events_.push_back(ev);
    }
}

void Batch::run_device(cudaStream_t st) { check(cudaGraphLaunch(exec_, st), "graph launch"); }

void Batch::run_host(const uint32_t* const* a, const uint32_t* const* b, uint32_t* const* c) {
    build_io_graphs();
    // Sub-batch s: its copies in (copy stream), its graph (compute stream),
    // its copies out (out stream); s + 1 moves in while s computes and s - 1
    // moves out.
    for (size_t s = 0; s < io_groups_.size(); ++s) {
        for (size_t i : io_groups_[s]) {
            const size_t bytes = prods_[i].e->words() * 4;
            check(cudaMemcpyAsync(prods_[i].a, a[i], bytes, cudaMemcpyHostToDevice, copy_), "copy a");
            check(cudaMemcpyAsync(prods_[i].b, b[i], bytes, cudaMemcpyHostToDevice, copy_), "copy b");
        }
        check(cudaEventRecord(io_events_[2 * s], copy_), "event record");
        check(cudaStreamWaitEvent(stream_, io_events_[2 * s], 0), "stream wait");
        check(cudaGraphLaunch(io_exec_[s], stream_), "graph launch");
        check(cudaEventRecord(io_events_[2 * s + 1], stream_), "event record");
        check(cudaStreamWaitEvent(out_, io_events_[2 * s + 1], 0), "stream wait");
        for (size_t i : io_groups_[s]) {
            const size_t bytes = prods_[i].e->words() * 4;
            check(cudaMemcpyAsync(c[i], prods_[i].c, bytes, cudaMemcpyDeviceToHost, out_), "copy c");
        }
    }
    check(cudaStreamSynchronize(out_), "batch sync");
    check(cudaStreamSynchronize(stream_), "batch sync");
    if (take_error()) throw std::runtime_error("batch: a tensor-core pipeline wait timed out");
}

uint32_t Batch::take_error() {
    uint32_t e = 0;
    check(cudaMemcpy(&e, err_, sizeof(e), cudaMemcpyDeviceToHost), "read error word");
    if (e) check(cudaMemset(err_, 0, sizeof(e)), "clear error word");
    return e;
}

double Batch::tune(int reps) {
    if (reps < 1) reps = 1;
    std::vector<BatchSchedule> cands;
    for (int layout : {0, 1, 2, 3})
        for (int grp : {0, 16})
            for (int grid : {0, 1})
                for (int pipe : {0, 14, 16}) cands.push_back(BatchSchedule{layout, 1, grp, grid, pipe});
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    check(cudaEventCreate(&t0), "event");
    check(cudaEventCreate(&t1), "event");
    auto time_current = [&]() {
        run_device(stream_);   // warm-up
        float best = 1e30f;
        for (int r = 0; r < reps; ++r) {
            check(cudaEventRecord(t0, stream_), "event");
            run_device(stream_);
            check(cudaEventRecord(t1, stream_), "event");
            check(cudaEventSynchronize(t1), "event sync");
            float ms = 0;
            check(cudaEventElapsedTime(&ms, t0, t1), "elapsed");
            best = std::min(best, ms);
        }
        return best;
    };
    BatchSchedule best_s = sched_;
    float best = 1e30f;
    try {
        for (const BatchSchedule& s : cands) {
            set_schedule(s);
            const float ms = time_current();
            if (ms < best) {
                best = ms;
                best_s = s;
            }
        }
        // The given order against the best schedule found.
        BatchSchedule s = best_s;
        s.order = 0;
        set_schedule(s);
        const float ms = time_current();
        if (ms < best) {
            best = ms;
            best_s = s;
        }
        set_schedule(best_s);
    } catch (...) {
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        throw;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (take_error()) throw std::runtime_error("batch: a tensor-core pipeline wait timed out while tuning");
    return best * 1000.0;
}

}  // namespace fpm
