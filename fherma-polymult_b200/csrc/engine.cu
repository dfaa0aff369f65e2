// Engine: plan upload, buffers, and the launch sequence of one product.
//
// Reference counterpart: fherma_init / fherma_run / fherma_free,
// solve.cu:710-1083.  The product is four launches on one stream: decompose a,
// decompose b (scaled), the transform chain (column pass, fused row pass,
// inverse column pass), CRT.  The host path stages the caller's buffers
// through pinned memory in chunks so the copies overlap the host-side memcpys.
#include "engine.h"
#include "kernels.h"

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
        dp_.lazy = pl.lazy ? 1 : 0;
        dp_.full_f = upload(pl.full_f);
        dp_.full_i = upload(pl.full_i);
        dp_.q = upload(pl.q);
        dp_.q_top = pl.q_top;
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
        dp_.err = dalloc<uint32_t>(1);
        check(cudaMemset(dp_.err, 0, sizeof(uint32_t)), "memset");
        if (const char* k = std::getenv("FPM_KERNELS")) simt_ = std::strcmp(k, "simt") == 0;
        A_ = dalloc<uint32_t>(residues());
        B_ = dalloc<uint32_t>(residues());
        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
        check(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking), "stream");
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
    if (stream_) cudaStreamDestroy(stream_);
    if (copy_) cudaStreamDestroy(copy_);
    stream_ = copy_ = nullptr;
    for (void* p : dmem_) cudaFree(p);
    dmem_.clear();
    for (uint32_t* h : {ha_, hb_, hc_}) {
        if (h) cudaFreeHost(h);
    }
    ha_ = hb_ = hc_ = nullptr;
}

void Engine::launch_dec(const uint32_t* d_limbs, uint32_t* d_res, int operand, cudaStream_t st) {
    if (simt_) {
        launch_decompose(dp_, d_limbs, d_res, operand, st);
    } else {
        launch_decompose_tc(dp_, d_limbs, d_res, operand, st);
    }
}

void Engine::launch_crt_any(const uint32_t* d_y, uint32_t* d_c, cudaStream_t st) {
    if (simt_ || !crt_uses_tc(plan_)) {
        launch_crt(dp_, d_y, d_c, st);
    } else {
        launch_crt_tc(dp_, d_y, d_c, st);
    }
}

uint32_t Engine::take_error() {
    uint32_t e = 0;
    check(cudaMemcpy(&e, dp_.err, sizeof(e), cudaMemcpyDeviceToHost), "read error word");
    if (e) check(cudaMemset(dp_.err, 0, sizeof(e)), "clear error word");
    return e;
}

void Engine::decompose(const uint32_t* d_limbs, uint32_t* d_res, int operand, cudaStream_t st) {
    launch_dec(d_limbs, d_res, operand, st);
    check(cudaGetLastError(), "decompose launch");
}

void Engine::transform(uint32_t* d_A, uint32_t* d_B, int mode, cudaStream_t st) {
    launch_ntt(dp_, d_A, d_B, mode, st);
    check(cudaGetLastError(), "transform launch");
}

void Engine::crt(const uint32_t* d_y, uint32_t* d_c, cudaStream_t st) {
    launch_crt_any(d_y, d_c, st);
    check(cudaGetLastError(), "crt launch");
}

void Engine::run_device(const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t st) {
    launch_dec(d_a, A_, 0, st);
    launch_dec(d_b, B_, 1, st);
    launch_ntt(dp_, A_, B_, kRowProduct, st);
    launch_crt_any(A_, d_c, st);
    check(cudaGetLastError(), "product launch");
}

void Engine::run_host(const uint32_t* a, const uint32_t* b, uint32_t* c) {
    const size_t n = words(), bytes = n * sizeof(uint32_t);
    if (!la_) {
        la_ = dalloc<uint32_t>(n);
        lb_ = dalloc<uint32_t>(n);
        lc_ = dalloc<uint32_t>(n);
        check(cudaHostAlloc(reinterpret_cast<void**>(&ha_), bytes, cudaHostAllocDefault), "pinned");
        check(cudaHostAlloc(reinterpret_cast<void**>(&hb_), bytes, cudaHostAllocDefault), "pinned");
        check(cudaHostAlloc(reinterpret_cast<void**>(&hc_), bytes, cudaHostAllocDefault), "pinned");
    }
    std::memcpy(ha_, a, bytes);
    check(cudaMemcpyAsync(la_, ha_, bytes, cudaMemcpyHostToDevice, stream_), "copy a");
    std::memcpy(hb_, b, bytes);
    check(cudaMemcpyAsync(lb_, hb_, bytes, cudaMemcpyHostToDevice, stream_), "copy b");
    run_device(la_, lb_, lc_, stream_);
    check(cudaMemcpyAsync(hc_, lc_, bytes, cudaMemcpyDeviceToHost, stream_), "copy c");
    check(cudaStreamSynchronize(stream_), "product");
    if (const uint32_t e = take_error()) {
        throw std::runtime_error("a kernel pipeline wait timed out (error word " + std::to_string(e) + ")");
    }
    std::memcpy(c, hc_, bytes);
}

}  // namespace fpm
