// Engine: plan upload, buffers, and the launch sequence of one product.
//
// Reference counterpart: fherma_init / fherma_run / fherma_free,
// solve.cu:710-1083.  The product is four launches on one stream: decompose a,
// decompose b (scaled), the transform chain (column pass, fused row pass,
// inverse column pass), CRT.  The host path stages the caller's buffers
// through pinned memory in chunks so the copies overlap the host-side memcpys.
#include "engine.h"
#include "kernels.h"

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <tuple>

namespace fpm {

void ensure_kernel_attributes(int device) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    for (int d : done) {
        if (d == device) return;
    }
    ntt_init_attributes();
    decompose_init_attributes();
    crt_init_attributes();
    decompose_tc_init_attributes();
    crt_tc_init_attributes();
    crt_pipe_init_attributes();
    decompose_pipe_init_attributes();
    done.push_back(device);
}

namespace {

// Device allocations of a shared prime basis.
struct DeviceBlocks {
    std::vector<void*> ptrs;
    size_t bytes = 0;
    template <class T>
    T* alloc(size_t count) {
        void* p = nullptr;
        const size_t b = std::max<size_t>(count, 1) * sizeof(T);
        check(cudaMalloc(&p, b), "cudaMalloc");
        ptrs.push_back(p);
        bytes += b;
        return static_cast<T*>(p);
    }
    template <class T>
    const T* upload(const std::vector<T>& v) {
        if (v.empty()) return nullptr;
        T* d = alloc<T>(v.size());
        check(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
        return d;
    }
    void release() {
        for (void* p : ptrs) cudaFree(p);
        ptrs.clear();
        bytes = 0;
    }
};

template <class T>
void drop(std::vector<T>& v) {
    std::vector<T>().swap(v);
}

}  // namespace

// The tables of one prime basis on one device: everything a point's kernels
// read that depends on q only through its bit length (make_plan_basis), among
// them the row pass's K x N twiddle tables.  Every Engine on the device whose
// (N, L, bits of q, prime window) match shares one Basis, so a context for a
// new modulus of a width already in use uploads nothing but q and builds its
// CRT tables on the device.
struct Engine::Basis {
    HostPlan plan;            // no modulus; the big host tables are dropped after upload
    DevPoint dp{};            // the basis tables' device pointers
    DeviceBlocks mem;
    std::shared_ptr<const DecConsts> dec;
    ~Basis() { mem.release(); }

    static std::shared_ptr<Basis> get(int device, uint32_t N, uint32_t W, int L, int qbits, int pmax_log2) {
        static std::mutex mu;
        static std::map<std::tuple<int, uint32_t, int, int, int>, std::weak_ptr<Basis>> cache;
        const auto key = std::make_tuple(device, N, L, qbits, pmax_log2);
        std::lock_guard<std::mutex> lock(mu);
        if (auto b = cache[key].lock()) return b;
        std::shared_ptr<Basis> b(new Basis());
        b->build(make_plan_basis(N, W, L, qbits, pmax_log2));
        cache[key] = b;
        return b;
    }

private:
    void build(HostPlan pl) {
        DevPoint& d = dp;
        d.N = pl.N;
        d.logN = pl.g.logN;
        d.logR = pl.g.logR;
        d.logS = pl.g.logS;
        d.L = pl.L;
        d.K = pl.K;
        d.lazy = pl.lazy ? 1 : 0;
        d.pc = mem.upload(pl.pc);
        d.dec_a = mem.upload(pl.dec_a);
        d.dec_b = mem.upload(pl.dec_b);
        d.col_f = mem.upload(pl.col_f);
        d.col_i = mem.upload(pl.col_i);
        d.row_u_f = mem.upload(pl.row_u_f);
        d.row_q_f = mem.upload(pl.row_q_f);
        d.row_tw = nullptr;
        d.full_f = mem.upload(pl.full_f);
        d.full_i = mem.upload(pl.full_i);
        d.p_recip = mem.upload(pl.p_recip);
        d.dec_kb = pl.dec_kb;
        d.dec_chunks = static_cast<int>(pl.dec_chunks);
        d.dec_img_a = mem.upload(pl.dec_img_a);
        d.dec_img_b = mem.upload(pl.dec_img_b);
        d.dec_fold = mem.upload(pl.dec_fold);
        d.crt_u = pl.crt_u;
        d.crt_tmem_cols = pl.crt_tmem_cols;
        d.wait_ns = kDefaultWaitNs;
        d.fault = 0;
        if (decompose_pipe_supported(pl)) {
            const uint8_t* wa = mem.upload(pl.dec_wimg_a);
            const uint8_t* wb = mem.upload(pl.dec_wimg_b);
            dec.reset(new DecConsts(make_dec_consts(pl, wa, wb)));
        }
        if (!pl.g.small) {
            uint2* tw = mem.alloc<uint2>(static_cast<size_t>(pl.K) * pl.N);
            build_row_tables(d, tw, nullptr);
            check(cudaDeviceSynchronize(), "row tables");
            d.row_tw = tw;
        }
        for (auto* v : {&pl.dec_a, &pl.dec_b, &pl.col_f, &pl.col_i, &pl.row_u_f, &pl.row_q_f, &pl.full_f, &pl.full_i})
            drop(*v);
        for (auto* v : {&pl.dec_img_a, &pl.dec_img_b, &pl.dec_wimg_a, &pl.dec_wimg_b}) drop(*v);
        plan = std::move(pl);
    }
};

template <class T>
T* Engine::dalloc(size_t count) {
    void* p = nullptr;
    const size_t b = std::max<size_t>(count, 1) * sizeof(T);
    check(cudaMalloc(&p, b), "cudaMalloc");
    dmem_.push_back(p);
    own_bytes_ += b;
    return static_cast<T*>(p);
}

template <class T>
const T* Engine::upload(const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    T* d = dalloc<T>(v.size());
    check(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return d;
}

Engine::Engine(uint32_t N, uint32_t W, const uint32_t* q, int L, int pmax_log2) {
    try {
        check(cudaGetDevice(&device_), "cudaGetDevice");
        check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_), "SM count");
        ensure_kernel_attributes(device_);
        // The point is checked before any device work (N first, as make_plan does).
        check_length(N);
        const int qbits = modulus_bits(q, L);
        basis_ = Basis::get(device_, N, W, L, qbits, pmax_log2);
        plan_ = basis_->plan;
        plan_.W = W;
        set_modulus_limbs(plan_, q);
        const HostPlan& pl = plan_;
        const int K = pl.K;
        dp_ = basis_->dp;
        dec_consts_ = basis_->dec;
        dp_.q = upload(pl.q);
        dp_.q_top = pl.q_top;
        dp_.q_top_inv = 1.0 / pl.q_top;
        // The modulus tables, built on the device from the basis's primes.
        uint32_t* M = dalloc<uint32_t>(static_cast<size_t>(K) * L);
        uint32_t* negvP = dalloc<uint32_t>(static_cast<size_t>(K + 1) * L);
        uint32_t* Pq = dalloc<uint32_t>(static_cast<size_t>(L));
        uint8_t* img = nullptr;
        uint8_t* img_v = nullptr;
        if (crt_uses_tc(pl)) {
            img = dalloc<uint8_t>(crt_image_bytes(pl, K));
            img_v = dalloc<uint8_t>(crt_image_bytes(pl, K + 1));
        }
        build_crt_tables(pl, dp_.pc, dp_.q, M, negvP, Pq, img, img_v, nullptr);
        dp_.M = M;
        dp_.negvP = negvP;
        dp_.crt_img = img;
        dp_.crt_img_v = img_v;
        if (crt_uses_tc(pl)) {
            // The CRT pipeline's parameters need the constants' top limbs.
            std::vector<uint32_t> tops(static_cast<size_t>(K) + 1);
            check(cudaMemcpy2D(tops.data(), sizeof(uint32_t), M + (L - 1), static_cast<size_t>(L) * 4,
                               sizeof(uint32_t), static_cast<size_t>(K), cudaMemcpyDeviceToHost),
                  "CRT top limbs");
            check(cudaMemcpy(&tops[K], negvP + L + (L - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost),
                  "CRT top limb");
            plan_.negp_top = tops[K];
            dp_.negp_top = tops[K];
            crt_consts_.reset(new CrtConsts(make_crt_consts(plan_, tops.data())));
        } else {
            check(cudaDeviceSynchronize(), "CRT tables");
        }
        dp_.err = dalloc<uint32_t>(1);
        check(cudaMemset(dp_.err, 0, sizeof(uint32_t)), "memset");
        if (const char* k = std::getenv("FPM_KERNELS")) simt_ = std::strcmp(k, "simt") == 0;
        A_ = dalloc<uint32_t>(residues());
        B_ = dalloc<uint32_t>(residues());
        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
        check(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking), "stream");
        check(cudaStreamCreateWithFlags(&out_, cudaStreamNonBlocking), "stream");
    } catch (...) {
        release();
        throw;
    }
}

size_t Engine::device_bytes() const { return own_bytes_ + (basis_ ? basis_->mem.bytes : 0); }

uint32_t Engine::crt_tables(uint32_t* M, uint32_t* negvP) const {
    const size_t K = static_cast<size_t>(plan_.K), L = static_cast<size_t>(plan_.L);
    check(cudaMemcpy(M, dp_.M, K * L * 4, cudaMemcpyDeviceToHost), "read M");
    check(cudaMemcpy(negvP, dp_.negvP, (K + 1) * L * 4, cudaMemcpyDeviceToHost), "read negvP");
    return static_cast<uint32_t>(K);
}

Engine::~Engine() { release(); }

void Engine::release() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (copy_) cudaStreamSynchronize(copy_);
    for (auto e : events_) cudaEventDestroy(e);
    events_.clear();
    if (out_) cudaStreamSynchronize(out_);
    if (stream_) cudaStreamDestroy(stream_);
    if (copy_) cudaStreamDestroy(copy_);
    if (out_) cudaStreamDestroy(out_);
    stream_ = copy_ = out_ = nullptr;
    pool_.reset();
    for (void* p : dmem_) cudaFree(p);
    dmem_.clear();
    for (uint32_t* h : {ha_, hb_, hc_}) {
        if (h) cudaFreeHost(h);
    }
    ha_ = hb_ = hc_ = nullptr;
}

void Engine::launch_dec(const uint32_t* d_limbs, uint32_t* d_res, int operand, uint32_t n0, uint32_t n1,
                        cudaStream_t st) {
    if (simt_) {
        launch_decompose(dp_, d_limbs, d_res, operand, n0, n1, st);
    } else if (dec_consts_) {
        launch_decompose_pipe(dp_, *dec_consts_, d_limbs, nullptr, d_res, nullptr, operand, n0, n1, sms_, st);
    } else {
        launch_decompose_tc(dp_, d_limbs, d_res, operand, n0, n1, st);
    }
}

void Engine::launch_crt_any(const DevPoint& d, const uint32_t* d_y, uint32_t* d_c, uint32_t n0, uint32_t n1,
                            cudaStream_t st) {
    if (simt_ || !crt_uses_tc(plan_)) {
        launch_crt(d, d_y, d_c, n0, n1, st);
    } else if (crt_consts_ && crt_pipe_supported(d, *crt_consts_, d_y, n0, n1)) {
        launch_crt_pipe(d, *crt_consts_, d_y, d_c, n0, n1, sms_, st);
    } else {
        launch_crt_tc(d, d_y, d_c, n0, n1, st);
    }
}

uint32_t Engine::take_error() {
    uint32_t e = 0;
    check(cudaMemcpy(&e, dp_.err, sizeof(e), cudaMemcpyDeviceToHost), "read error word");
    if (e) check(cudaMemset(dp_.err, 0, sizeof(e)), "clear error word");
    return e;
}

uint32_t Engine::take_error(cudaStream_t st) {
    check(cudaStreamSynchronize(st), "stream synchronize");
    return take_error();
}

void Engine::decompose(const uint32_t* d_limbs, uint32_t* d_res, int operand, cudaStream_t st) {
    launch_dec(d_limbs, d_res, operand, 0, plan_.N, st);
    check(cudaGetLastError(), "decompose launch");
}

void Engine::transform(uint32_t* d_A, uint32_t* d_B, int mode, cudaStream_t st) {
    launch_ntt(dp_, d_A, d_B, mode, st);
    check(cudaGetLastError(), "transform launch");
}

// Both operands' decompose, as a product launches it (one paired launch on the
// tensor-core paths).
void Engine::decompose_pair_on(const DevPoint& d, const uint32_t* a, const uint32_t* b, uint32_t* A, uint32_t* B,
                               cudaStream_t st) {
    if (simt_) {
        launch_decompose(d, a, A, 0, 0, plan_.N, st);
        launch_decompose(d, b, B, 1, 0, plan_.N, st);
    } else if (dec_consts_) {
        launch_decompose_pipe(d, *dec_consts_, a, b, A, B, 0, 0, plan_.N, sms_, st);
    } else {
        launch_decompose_tc_pair(d, a, b, A, B, st);
    }
}

void Engine::decompose_pair(const uint32_t* d_limbs, uint32_t* d_res, cudaStream_t st) {
    const size_t nl = static_cast<size_t>(plan_.N) * plan_.L, kn = static_cast<size_t>(plan_.K) * plan_.N;
    decompose_pair_on(dp_, d_limbs, d_limbs + nl, d_res, d_res + kn, st);
    check(cudaGetLastError(), "decompose launch");
}

void Engine::crt(const uint32_t* d_y, uint32_t* d_c, cudaStream_t st) {
    launch_crt_any(dp_, d_y, d_c, 0, plan_.N, st);
    check(cudaGetLastError(), "crt launch");
}

void Engine::product(const DevPoint& d, const uint32_t* d_a, const uint32_t* d_b, uint32_t* A, uint32_t* B,
                     uint32_t* d_c, cudaStream_t st) {
    const uint32_t N = plan_.N;
    decompose_pair_on(d, d_a, d_b, A, B, st);
    launch_ntt(d, A, B, kRowProduct, st);
    launch_crt_any(d, A, d_c, 0, N, st);
    check(cudaGetLastError(), "product launch");
}

void Engine::run_device(const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t st) {
    product(dp_, d_a, d_b, A_, B_, d_c, st);
}

namespace {

bool is_pinned(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

}  // namespace

void Engine::ensure_host_path() {
    if (la_) return;
    const size_t n = words(), bytes = n * sizeof(uint32_t);
    la_ = dalloc<uint32_t>(n);
    lb_ = dalloc<uint32_t>(n);
    lc_ = dalloc<uint32_t>(n);
    check(cudaHostAlloc(reinterpret_cast<void**>(&ha_), bytes, cudaHostAllocDefault), "pinned");
    check(cudaHostAlloc(reinterpret_cast<void**>(&hb_), bytes, cudaHostAllocDefault), "pinned");
    check(cudaHostAlloc(reinterpret_cast<void**>(&hc_), bytes, cudaHostAllocDefault), "pinned");
    // I/O chunks: equal slices on 128-coefficient boundaries, so a chunk's
    // decompose and CRT blocks never straddle two.  Each chunk costs about
    // 13 us of launches and pipeline start-up, so the default aims at 16 MiB of
    // operand limbs per chunk, 1 to 4 chunks; tune_host_path() measures the
    // candidates on this point.  FPM_IO_CHUNKS overrides both.
    const size_t in_bytes = 2 * bytes;
    int want = static_cast<int>(std::min<size_t>(4, std::max<size_t>(1, (in_bytes + (size_t(8) << 20)) >> 24)));
    if (const char* v = std::getenv("FPM_IO_CHUNKS")) want = std::max(1, std::atoi(v));
    set_chunks(want);
    pool_.reset(new CopyPool(default_copy_threads()));
}

void Engine::set_chunks(int want) {
    const uint32_t N = plan_.N;
    const uint32_t unit = 128;
    const uint32_t units = (N + unit - 1) / unit;
    const uint32_t nch = std::min<uint32_t>(static_cast<uint32_t>(std::max(1, want)), units);
    chunk_at_.clear();
    for (uint32_t k = 0; k <= nch; ++k) chunk_at_.push_back(std::min(N, units * k / nch * unit));
    for (auto e : events_) cudaEventDestroy(e);
    events_.assign(4 * nch, nullptr);
    for (auto& e : events_) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
}

// The reference's fherma_init times its candidate copy modes on the point
// (solve.cu:805-862) and keeps the default unless another is at least 5%
// faster.  Here the mode follows from the caller's buffers (pinned: DMA from
// them directly; pageable: staged through pinned memory), and what the point
// decides is how many chunks the copies are cut into: 1 to 4 candidates, each
// run 1 + 3 times on the engine's own pinned buffers, median kept.
int Engine::tune_host_path() {
    ensure_host_path();
    if (std::getenv("FPM_IO_CHUNKS")) return static_cast<int>(chunk_at_.size() - 1);
    const int dflt = static_cast<int>(chunk_at_.size() - 1);
    const size_t bytes = words() * sizeof(uint32_t);
    std::memset(ha_, 0, bytes);
    std::memset(hb_, 0, bytes);
    auto time_it = [&](int n) {
        set_chunks(n);
        run_host(ha_, hb_, hc_);
        double t[3];
        for (double& x : t) {
            const auto t0 = std::chrono::steady_clock::now();
            run_host(ha_, hb_, hc_);
            x = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
        std::sort(t, t + 3);
        return t[1];
    };
    const double base = time_it(dflt);
    int best = dflt;
    double best_t = base;
    for (int n = 1; n <= 4; ++n) {
        if (n == dflt) continue;
        const double t = time_it(n);
        if (t < best_t) best_t = t, best = n;
    }
    if (best_t > 0.95 * base) best = dflt;
    set_chunks(best);
    return best;
}

void Engine::run_host(const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* (*out_fn)(void*),
                      void* out_arg) {
    if (!c && !out_fn) throw std::runtime_error("run_host: no destination");
    ensure_host_path();
    const int L = plan_.L;
    const size_t nch = chunk_at_.size() - 1;
    const bool pin_a = is_pinned(a), pin_b = is_pinned(b), pin_c = c && is_pinned(c);
    cudaEvent_t* in_ev = events_.data();              // 2 nch
    cudaEvent_t* crt_ev = events_.data() + 2 * nch;   // nch
    cudaEvent_t* out_ev = events_.data() + 3 * nch;   // nch

    // In: per chunk, (stage,) DMA, then that chunk's decompose.
    const uint32_t* src[2] = {a, b};
    const bool pinned[2] = {pin_a, pin_b};
    uint32_t* stage[2] = {ha_, hb_};
    uint32_t* dlimbs[2] = {la_, lb_};
    uint32_t* res[2] = {A_, B_};
    for (int op = 0; op < 2; ++op) {
        for (size_t k = 0; k < nch; ++k) {
            const uint32_t n0 = chunk_at_[k], n1 = chunk_at_[k + 1];
            const size_t off = static_cast<size_t>(n0) * L, bytes = static_cast<size_t>(n1 - n0) * L * 4;
            const uint32_t* from = src[op] + off;
            if (!pinned[op]) {
                pool_->copy(stage[op] + off, from, bytes);
                from = stage[op] + off;
            }
            check(cudaMemcpyAsync(dlimbs[op] + off, from, bytes, cudaMemcpyHostToDevice, copy_), "copy in");
            check(cudaEventRecord(in_ev[op * nch + k], copy_), "event");
            check(cudaStreamWaitEvent(stream_, in_ev[op * nch + k], 0), "wait");
            launch_dec(dlimbs[op], res[op], op, n0, n1, stream_);
        }
    }
    launch_ntt(dp_, A_, B_, kRowProduct, stream_);
    // Out: per chunk, the CRT, then its DMA (to c itself when c is pinned).
    uint32_t* dst = pin_c ? c : hc_;
    for (size_t k = 0; k < nch; ++k) {
        const uint32_t n0 = chunk_at_[k], n1 = chunk_at_[k + 1];
        const size_t off = static_cast<size_t>(n0) * L, bytes = static_cast<size_t>(n1 - n0) * L * 4;
        launch_crt_any(dp_, A_, lc_, n0, n1, stream_);
        check(cudaEventRecord(crt_ev[k], stream_), "event");
        check(cudaStreamWaitEvent(out_, crt_ev[k], 0), "wait");
        check(cudaMemcpyAsync(dst + off, lc_ + off, bytes, cudaMemcpyDeviceToHost, out_), "copy out");
        check(cudaEventRecord(out_ev[k], out_), "event");
    }
    check(cudaGetLastError(), "product launch");
    if (!c) c = out_fn(out_arg);
    if (!pin_c) {
        for (size_t k = 0; k < nch; ++k) {
            const uint32_t n0 = chunk_at_[k], n1 = chunk_at_[k + 1];
            const size_t off = static_cast<size_t>(n0) * L, bytes = static_cast<size_t>(n1 - n0) * L * 4;
            check(cudaEventSynchronize(out_ev[k]), "copy out");
            pool_->copy(c + off, hc_ + off, bytes);
        }
    } else {
        check(cudaEventSynchronize(out_ev[nch - 1]), "copy out");
    }
    if (const uint32_t e = take_error()) {
        throw PipelineTimeout("a kernel pipeline wait ran out of time (error word " + std::to_string(e) +
                              "); this product's result is not valid");
    }
}

}  // namespace fpm
