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
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <stdexcept>

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

template <class T>
T* Engine::dalloc(size_t count) {
    void* p = nullptr;
    check(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc");
    dmem_.push_back(p);
    return static_cast<T*>(p);
}

template <class T>
const T* Engine::upload(const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    T* d = dalloc<T>(v.size());
    check(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return d;
}

Engine::Engine(uint32_t N, uint32_t W, const uint32_t* q, int L, int pmax_log2)
    : plan_(make_plan(N, W, q, L, pmax_log2)) {
    try {
        check(cudaGetDevice(&device_), "cudaGetDevice");
        check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_), "SM count");
        ensure_kernel_attributes(device_);
        const HostPlan& pl = plan_;
        dp_.N = pl.N;
        dp_.logN = pl.g.logN;
        dp_.logR = pl.g.logR;
        dp_.logS = pl.g.logS;
        dp_.L = pl.L;
        dp_.K = pl.K;
        dp_.pc = upload(pl.pc);
        dp_.dec_a = upload(pl.dec_a);
        dp_.dec_b = upload(pl.dec_b);
        dp_.col_f = upload(pl.col_f);
        dp_.col_i = upload(pl.col_i);
        dp_.row_u_f = upload(pl.row_u_f);
        dp_.row_q_f = upload(pl.row_q_f);
        dp_.row_tw = nullptr;
        dp_.lazy = pl.lazy ? 1 : 0;
        dp_.full_f = upload(pl.full_f);
        dp_.full_i = upload(pl.full_i);
        dp_.q = upload(pl.q);
        dp_.q_top = pl.q_top;
        dp_.q_top_inv = 1.0 / pl.q_top;
        dp_.M = upload(pl.M);
        dp_.negvP = upload(pl.negvP);
        dp_.p_recip = upload(pl.p_recip);
        dp_.dec_kb = pl.dec_kb;
        dp_.dec_chunks = static_cast<int>(pl.dec_chunks);
        dp_.dec_img_a = upload(pl.dec_img_a);
        dp_.dec_img_b = upload(pl.dec_img_b);
        dp_.dec_fold = upload(pl.dec_fold);
        dp_.crt_u = pl.crt_u;
        dp_.crt_tmem_cols = pl.crt_tmem_cols;
        dp_.crt_img = upload(pl.crt_img);
        dp_.crt_img_v = upload(pl.crt_img_v);
        dp_.negp_top = pl.negp_top;
        dp_.wait_ns = kDefaultWaitNs;
        dp_.fault = 0;
        if (crt_uses_tc(pl)) crt_consts_.reset(new CrtConsts(make_crt_consts(pl)));
        if (decompose_pipe_supported(pl)) {
            const uint8_t* wa = upload(pl.dec_wimg_a);
            const uint8_t* wb = upload(pl.dec_wimg_b);
            dec_consts_.reset(new DecConsts(make_dec_consts(pl, wa, wb)));
        }
        if (!pl.g.small) {
            uint2* tw = dalloc<uint2>(static_cast<size_t>(pl.K) * pl.N);
            build_row_tables(dp_, tw, nullptr);
            check(cudaDeviceSynchronize(), "row tables");
            dp_.row_tw = tw;
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
    } else if (crt_consts_ && crt_pipe_supported(d, d_y, n0, n1)) {
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

void Engine::crt(const uint32_t* d_y, uint32_t* d_c, cudaStream_t st) {
    launch_crt_any(dp_, d_y, d_c, 0, plan_.N, st);
    check(cudaGetLastError(), "crt launch");
}

void Engine::product(const DevPoint& d, const uint32_t* d_a, const uint32_t* d_b, uint32_t* A, uint32_t* B,
                     uint32_t* d_c, cudaStream_t st) {
    const uint32_t N = plan_.N;
    if (simt_) {
        launch_decompose(d, d_a, A, 0, 0, N, st);
        launch_decompose(d, d_b, B, 1, 0, N, st);
    } else if (dec_consts_) {
        launch_decompose_pipe(d, *dec_consts_, d_a, d_b, A, B, 0, 0, N, sms_, st);
    } else {
        launch_decompose_tc_pair(d, d_a, d_b, A, B, st);
    }
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
    // operand limbs per chunk, 1 to 4 chunks (N = 65536 at 2048 bits: 2 chunks,
    // 1092 us a product against 1113 with 4 and 1166 with 8).  FPM_IO_CHUNKS
    // overrides it.
    const size_t in_bytes = 2 * bytes;
    int want = static_cast<int>(std::min<size_t>(4, std::max<size_t>(1, (in_bytes + (size_t(8) << 20)) >> 24)));
    if (const char* v = std::getenv("FPM_IO_CHUNKS")) want = std::max(1, std::atoi(v));
    const uint32_t N = plan_.N;
    const uint32_t unit = 128;
    const uint32_t units = (N + unit - 1) / unit;
    const uint32_t nch = std::min<uint32_t>(static_cast<uint32_t>(want), units);
    chunk_at_.clear();
    for (uint32_t k = 0; k <= nch; ++k) chunk_at_.push_back(std::min(N, units * k / nch * unit));
    events_.resize(4 * nch);
    for (auto& e : events_) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    pool_.reset(new CopyPool(default_copy_threads()));
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
