// C ABI (include/fherma_polymult.h) and the reference's C++ entry points
// (include/fherma_abi.h) over fpm::Engine.
#include "fherma_abi.h"
#include "fherma_polymult.h"

#include "batch.h"
#include "engine.h"
#include "kernels.h"
#include "server.h"

#include <cuda_runtime.h>

#include <cstdlib>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

struct fpm_ctx {
    fpm::Engine* engine;
    uint32_t W;
};

struct fpm_batch {
    fpm::Batch* batch;
    double tuned_us;
};

struct fpm_server {
    fpm::Server* server;
    int lanes;
};

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

// Runs f, mapping exceptions to error codes.
template <class F>
int guarded(F&& f) {
    try {
        f();
        return FPM_OK;
    } catch (const std::bad_alloc&) {
        return fail(FPM_ENOMEM, "out of host memory");
    } catch (const fpm::PipelineTimeout& e) {
        return fail(FPM_ETIMEOUT, e.what());
    } catch (const fpm::CudaError& e) {
        return fail(e.code == cudaErrorMemoryAllocation ? FPM_ENOMEM : FPM_ECUDA, e.what());
    } catch (const std::runtime_error& e) {
        return fail(FPM_EINVAL, e.what());
    } catch (const std::exception& e) {
        return fail(FPM_EINTERNAL, e.what());
    }
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

int resolve_prime_bits(int prime_bits) {
    if (prime_bits) return prime_bits;
    if (const char* v = std::getenv("FPM_PRIME_BITS")) return std::atoi(v);
    return fpm::kDefaultPrimeBits;
}

void fill_info(const fpm::HostPlan& pl, uint32_t W, int device, size_t device_bytes, fpm_info* out) {
    out->N = pl.N;
    out->W = W;
    out->L = static_cast<uint32_t>(pl.L);
    out->K = static_cast<uint32_t>(pl.K);
    out->logN = pl.g.logN;
    out->logR = pl.g.logR;
    out->logS = pl.g.logS;
    out->device = device;
    out->device_bytes = device_bytes;
    out->prime_bits = static_cast<uint32_t>(pl.pmax_log2);
}

}  // namespace

extern "C" {

const char* fpm_last_error(void) { return g_error.c_str(); }

int fpm_init(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, fpm_ctx** out) {
    return fpm_init_ex(N, W, L, q, 0, out);
}

int fpm_init_ex(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int prime_bits, fpm_ctx** out) {
    if (!out) return fail(FPM_EINVAL, "fpm_init: out is NULL");
    *out = nullptr;
    if (!q) return fail(FPM_EINVAL, "fpm_init: q is NULL");
    if (L < 1 || L > static_cast<uint32_t>(fpm::kMaxL)) {
        return fail(FPM_EINVAL, "unsupported limb count L = " + std::to_string(L) + ": expected 1 to " +
                                    std::to_string(fpm::kMaxL));
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(FPM_ECUDA, "no CUDA device: this library has no CPU fallback");
    }
    fpm::Engine* e = nullptr;
    const int bits = resolve_prime_bits(prime_bits);
    if (bits != 30 && bits != 31) return fail(FPM_EINVAL, "prime_bits must be 30 or 31");
    const int rc = guarded([&] { e = new fpm::Engine(N, W, q, static_cast<int>(L), bits); });
    if (rc) return rc;
    *out = new fpm_ctx{e, W};
    return FPM_OK;
}

int fpm_run(fpm_ctx* ctx, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    if (!ctx || !a || !b || !c) return fail(FPM_EINVAL, "fpm_run: NULL argument");
    return guarded([&] { ctx->engine->run_host(a, b, c); });
}

int fpm_run_device(fpm_ctx* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, void* stream) {
    if (!ctx || !d_a || !d_b || !d_c) return fail(FPM_EINVAL, "fpm_run_device: NULL argument");
    return guarded([&] { ctx->engine->run_device(d_a, d_b, d_c, as_stream(stream)); });
}

int fpm_run_device_noalloc(fpm_ctx* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, void* stream) {
    if (!ctx || !d_a || !d_b || !d_c) return fail(FPM_EINVAL, "fpm_run_device_noalloc: NULL argument");
    return guarded([&] { ctx->engine->run_device_static(d_a, d_b, d_c, as_stream(stream)); });
}

namespace {

int timeout_status(uint32_t word, const char* where) {
    if (!word) return FPM_OK;
    return fail(FPM_ETIMEOUT, std::string(where) + ": a kernel pipeline wait ran out of time (error word " +
                                  std::to_string(word) + "); the products enqueued since the last check are not "
                                  "valid");
}

}  // namespace

int fpm_get_error(fpm_ctx* ctx, void* stream) {
    if (!ctx) return fail(FPM_EINVAL, "fpm_get_error: NULL context");
    uint32_t word = 0;
    const int rc = guarded([&] { word = ctx->engine->take_error(as_stream(stream)); });
    return rc ? rc : timeout_status(word, "fpm_get_error");
}

int fpm_noalloc_get_error(void* stream) {
    uint32_t word = 0;
    const int rc = guarded([&] { word = fpm::Engine::take_static_error(as_stream(stream)); });
    return rc ? rc : timeout_status(word, "fpm_noalloc_get_error");
}

int fpm_set_wait_limit(fpm_ctx* ctx, uint64_t ns) {
    if (!ctx) return fail(FPM_EINVAL, "fpm_set_wait_limit: NULL context");
    if (ns == 0) return fail(FPM_EINVAL, "fpm_set_wait_limit: the limit must be positive");
    ctx->engine->set_wait_limit(ns);
    return FPM_OK;
}

int fpm_debug_inject_stall(fpm_ctx* ctx, uint32_t mask) {
    if (!ctx) return fail(FPM_EINVAL, "fpm_debug_inject_stall: NULL context");
    if (mask & ~3u) return fail(FPM_EINVAL, "fpm_debug_inject_stall: mask bits are 1 (decompose) and 2 (CRT)");
    ctx->engine->set_fault(mask);
    return FPM_OK;
}

void fpm_free(fpm_ctx* ctx) {
    if (!ctx) return;
    delete ctx->engine;
    delete ctx;
}

int fpm_get_info(const fpm_ctx* ctx, fpm_info* out) {
    if (!ctx || !out) return fail(FPM_EINVAL, "fpm_get_info: NULL argument");
    fill_info(ctx->engine->plan(), ctx->W, ctx->engine->device(), ctx->engine->device_bytes(), out);
    return FPM_OK;
}

int fpm_plan_info(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, fpm_info* out, uint32_t* primes) {
    return fpm_plan_info_ex(N, W, L, q, 0, out, primes);
}

int fpm_plan_info_ex(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int prime_bits, fpm_info* out,
                     uint32_t* primes) {
    if (!q || !out) return fail(FPM_EINVAL, "fpm_plan_info: NULL argument");
    const int bits = resolve_prime_bits(prime_bits);
    if (bits != 30 && bits != 31) return fail(FPM_EINVAL, "prime_bits must be 30 or 31");
    return guarded([&] {
        const fpm::HostPlan pl = fpm::make_plan(N, W, q, static_cast<int>(L), bits);
        fill_info(pl, W, -1, fpm::device_footprint(pl), out);
        if (primes) {
            for (int j = 0; j < pl.K; ++j) primes[j] = pl.primes[j];
        }
    });
}

int fpm_get_primes(const fpm_ctx* ctx, uint32_t* out) {
    if (!ctx || !out) return fail(FPM_EINVAL, "fpm_get_primes: NULL argument");
    const auto& p = ctx->engine->plan().primes;
    for (size_t i = 0; i < p.size(); ++i) out[i] = p[i];
    return FPM_OK;
}

int fpm_tune_host_path(fpm_ctx* ctx, int* chunks) {
    if (!ctx) return fail(FPM_EINVAL, "fpm_tune_host_path: NULL context");
    return guarded([&] {
        const int n = ctx->engine->tune_host_path();
        if (chunks) *chunks = n;
    });
}

int fpm_get_crt_tables(const fpm_ctx* ctx, uint32_t* M, uint32_t* negvP) {
    if (!ctx || !M || !negvP) return fail(FPM_EINVAL, "fpm_get_crt_tables: NULL argument");
    return guarded([&] { ctx->engine->crt_tables(M, negvP); });
}

int fpm_stage_decompose(fpm_ctx* ctx, const uint32_t* d_limbs, uint32_t* d_res, int operand, void* stream) {
    if (!ctx || !d_limbs || !d_res || operand < 0 || operand > 2)
        return fail(FPM_EINVAL, "fpm_stage_decompose: bad argument");
    if (operand == 2) return guarded([&] { ctx->engine->decompose_pair(d_limbs, d_res, as_stream(stream)); });
    return guarded([&] { ctx->engine->decompose(d_limbs, d_res, operand, as_stream(stream)); });
}

int fpm_stage_transform(fpm_ctx* ctx, uint32_t* d_A, uint32_t* d_B, int mode, void* stream) {
    if (!ctx || !d_A || !d_B || mode < 0 || mode > 4)
        return fail(FPM_EINVAL, "fpm_stage_transform: bad argument");
    return guarded([&] { ctx->engine->transform(d_A, d_B, mode, as_stream(stream)); });
}

int fpm_stage_crt(fpm_ctx* ctx, const uint32_t* d_y, uint32_t* d_c, void* stream) {
    if (!ctx || !d_y || !d_c) return fail(FPM_EINVAL, "fpm_stage_crt: bad argument");
    return guarded([&] { ctx->engine->crt(d_y, d_c, as_stream(stream)); });
}

int fpm_batch_create(fpm_ctx* const* ctxs, uint32_t count, fpm_batch** out) {
    if (!ctxs || !out || count == 0) return fail(FPM_EINVAL, "fpm_batch_create: bad argument");
    *out = nullptr;
    fpm::Batch* b = nullptr;
    const int rc = guarded([&] {
        std::vector<fpm::Engine*> engines;
        for (uint32_t i = 0; i < count; ++i) {
            if (!ctxs[i]) throw std::runtime_error("fpm_batch_create: NULL context");
            engines.push_back(ctxs[i]->engine);
        }
        b = new fpm::Batch(engines);
    });
    if (rc) return rc;
    *out = new fpm_batch{b, 0.0};
    return FPM_OK;
}

int fpm_batch_buffers(fpm_batch* batch, uint32_t i, uint32_t** d_a, uint32_t** d_b, uint32_t** d_c) {
    if (!batch || i >= batch->batch->size()) return fail(FPM_EINVAL, "fpm_batch_buffers: bad argument");
    if (d_a) *d_a = batch->batch->a(i);
    if (d_b) *d_b = batch->batch->b(i);
    if (d_c) *d_c = batch->batch->c(i);
    return FPM_OK;
}

int fpm_batch_run_device(fpm_batch* batch, void* stream) {
    if (!batch) return fail(FPM_EINVAL, "fpm_batch_run_device: NULL argument");
    return guarded([&] { batch->batch->run_device(as_stream(stream)); });
}

int fpm_batch_run(fpm_batch* batch, const uint32_t* const* a, const uint32_t* const* b, uint32_t* const* c) {
    if (!batch || !a || !b || !c) return fail(FPM_EINVAL, "fpm_batch_run: NULL argument");
    for (size_t i = 0; i < batch->batch->size(); ++i) {
        if (!a[i] || !b[i] || !c[i]) return fail(FPM_EINVAL, "fpm_batch_run: NULL buffer");
    }
    return guarded([&] { batch->batch->run_host(a, b, c); });
}

int fpm_batch_get_info(const fpm_batch* batch, fpm_batch_info* out) {
    if (!batch || !out) return fail(FPM_EINVAL, "fpm_batch_get_info: NULL argument");
    const fpm::BatchSchedule& s = batch->batch->schedule();
    out->count = static_cast<uint32_t>(batch->batch->size());
    out->layout = s.layout;
    out->order = s.order;
    out->prime_group = s.prime_group;
    out->grid = s.grid;
    out->pipe_min_log_n = s.pipe_min_log_n;
    out->launches = batch->batch->launches();
    out->device_bytes = batch->batch->device_bytes();
    out->tuned_us = batch->tuned_us;
    return FPM_OK;
}

int fpm_batch_tune(fpm_batch* batch, int reps, fpm_batch_info* info) {
    if (!batch) return fail(FPM_EINVAL, "fpm_batch_tune: NULL argument");
    const int rc = guarded([&] { batch->tuned_us = batch->batch->tune(reps); });
    if (rc) return rc;
    return info ? fpm_batch_get_info(batch, info) : FPM_OK;
}

int fpm_batch_set_schedule(fpm_batch* batch, int layout, int order, int prime_group, int grid,
                           int pipe_min_log_n) {
    if (!batch) return fail(FPM_EINVAL, "fpm_batch_set_schedule: NULL argument");
    return guarded([&] {
        batch->batch->set_schedule(fpm::BatchSchedule{layout, order, prime_group, grid, pipe_min_log_n});
    });
}

void fpm_batch_free(fpm_batch* batch) {
    if (!batch) return;
    delete batch->batch;
    delete batch;
}

int fpm_server_create(fpm_ctx* const* points, uint32_t count, uint64_t budget_bytes, int lanes, int max_batch,
                      fpm_server** out) {
    if (!points || !out || count == 0) return fail(FPM_EINVAL, "fpm_server_create: bad argument");
    *out = nullptr;
    fpm::Server* srv = nullptr;
    const int rc = guarded([&] {
        std::vector<fpm::Engine*> engines;
        for (uint32_t i = 0; i < count; ++i) {
            if (!points[i]) throw std::runtime_error("fpm_server_create: NULL context");
            engines.push_back(points[i]->engine);
        }
        fpm::ServerConfig cfg;
        cfg.budget_bytes = budget_bytes;
        cfg.lanes = lanes;
        cfg.max_batch = max_batch;
        srv = new fpm::Server(engines, cfg);
    });
    if (rc) return rc;
    *out = new fpm_server{srv, lanes};
    return FPM_OK;
}

int fpm_server_add_point(fpm_server* srv, fpm_ctx* point, uint32_t* index) {
    if (!srv || !point || !index) return fail(FPM_EINVAL, "fpm_server_add_point: NULL argument");
    return guarded([&] { *index = srv->server->add_point(point->engine); });
}

int fpm_server_footprint(const fpm_server* srv, uint32_t point, uint64_t* bytes) {
    if (!srv || !bytes) return fail(FPM_EINVAL, "fpm_server_footprint: NULL argument");
    return guarded([&] { *bytes = srv->server->footprint(point); });
}

int fpm_server_submit(fpm_server* srv, uint32_t point, const uint32_t* a, const uint32_t* b, uint32_t* c,
                      uint64_t* ticket) {
    if (!srv || !a || !b || !c || !ticket) return fail(FPM_EINVAL, "fpm_server_submit: NULL argument");
    return guarded([&] { *ticket = srv->server->submit(point, a, b, c); });
}

int fpm_server_wait(fpm_server* srv, uint64_t ticket, double* latency_us) {
    if (!srv) return fail(FPM_EINVAL, "fpm_server_wait: NULL argument");
    return guarded([&] {
        const double us = srv->server->wait(ticket);
        if (latency_us) *latency_us = us;
    });
}

int fpm_server_replay(fpm_server* srv, uint32_t n, const uint32_t* point, const double* arrival_us,
                      const uint32_t* const* a, const uint32_t* const* b, uint32_t* const* c, double* latency_us) {
    if (!srv || !point || !arrival_us || !a || !b || !c || !latency_us)
        return fail(FPM_EINVAL, "fpm_server_replay: NULL argument");
    return guarded([&] { srv->server->replay(n, point, arrival_us, a, b, c, latency_us); });
}

int fpm_server_get_stats(const fpm_server* srv, fpm_server_stats* out) {
    if (!srv || !out) return fail(FPM_EINVAL, "fpm_server_get_stats: NULL argument");
    const fpm::ServerStats s = srv->server->stats();
    out->completed = s.completed;
    out->failed = s.failed;
    out->batches = s.batches;
    out->lanes = static_cast<uint32_t>(srv->lanes);
    out->max_lanes_busy = s.max_lanes_busy;
    out->budget_bytes = srv->server->budget();
    out->peak_bytes = s.peak_bytes;
    return FPM_OK;
}

void fpm_server_free(fpm_server* srv) {
    if (!srv) return;
    delete srv->server;
    delete srv;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The reference's C++ entry points (fherma.h:46-48).

void* fherma_init(const fherma::Point& p) {
    if (p.q.data.size() != p.L) {
        throw std::runtime_error("q has " + std::to_string(p.q.data.size()) + " limbs, expected L = " +
                                 std::to_string(p.L));
    }
    fpm_ctx* ctx = nullptr;
    if (fpm_init(p.N, p.W, p.L, p.q.data.data(), &ctx) != FPM_OK) throw std::runtime_error(fpm_last_error());
    // As the reference's init measures its copy modes, set-up measures the
    // host path's chunking here, outside the timed fherma_run calls.
    if (fpm_tune_host_path(ctx, nullptr) != FPM_OK) {
        const std::string msg = fpm_last_error();
        fpm_free(ctx);
        throw std::runtime_error(msg);
    }
    return ctx;
}

fherma::Outputs fherma_run(void* state, const fherma::Inputs& in) {
    auto* ctx = static_cast<fpm_ctx*>(state);
    if (!ctx) throw std::runtime_error("fherma_run: null state");
    const fpm::HostPlan& pl = ctx->engine->plan();
    const size_t words = static_cast<size_t>(pl.N) * pl.L;
    if (in.a.data.size() != words || in.b.data.size() != words) {
        throw std::runtime_error("operand size does not match the point");
    }
    fherma::Outputs out;
    out.c.shape = {static_cast<int64_t>(pl.N), static_cast<int64_t>(pl.L)};
    // The answer's vector is sized (a zero fill of N L words) on a helper
    // thread while the GPU works; run_host asks for it only when the first
    // result chunk is ready to be copied out.
    struct Filler {
        std::vector<uint32_t>* v;
        size_t n;
        std::thread t;
        ~Filler() {
            if (t.joinable()) t.join();
        }
    } filler{&out.c.data, words, {}};
    filler.t = std::thread([&filler] { filler.v->resize(filler.n); });
    const int rc = guarded([&] {
        ctx->engine->run_host(in.a.data.data(), in.b.data.data(), nullptr,
                              [](void* p) -> uint32_t* {
                                  auto* f = static_cast<Filler*>(p);
                                  f->t.join();
                                  return f->v->data();
                              },
                              &filler);
    });
    if (rc != FPM_OK) throw std::runtime_error(fpm_last_error());
    return out;
}

void fherma_free(void* state) { fpm_free(static_cast<fpm_ctx*>(state)); }
