// One point's resident state on one GPU: the plan tables in device memory,
// residue workspaces, pinned staging and the launch sequence of a product.
#pragma once

#include "copy_pool.h"
#include "device.cuh"
#include "plan.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

namespace fpm {

struct CrtConsts;
struct DecConsts;

class Engine {
public:
    // Builds the plan and uploads it (throws std::runtime_error).
    Engine(uint32_t N, uint32_t W, const uint32_t* q, int L, int pmax_log2 = kDefaultPrimeBits);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    const HostPlan& plan() const { return plan_; }
    const DevPoint& point() const { return dp_; }
    int device() const { return device_; }
    bool simt() const { return simt_; }
    int sms() const { return sms_; }
    // Kernel parameters of the pipelined decompose and CRT (null where a
    // point has no pipeline).
    const DecConsts* dec_consts() const { return dec_consts_.get(); }
    const CrtConsts* crt_consts() const { return crt_consts_.get(); }

    // c = a b on device buffers (N x L each), enqueued on st; the engine's
    // residue workspaces are used, so calls on one engine must not overlap.
    void run_device(const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t st);

    // As run_device, but the residue workspaces and the error word come from a
    // static device array of static_scratch_bytes() (static_scratch.cu), not
    // from this engine; allocates nothing.  Throws std::runtime_error when the
    // point's scratch does not fit or another device is current.
    void run_device_static(const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t st);
    size_t static_scratch_words_needed() const;

    // c = a b on host buffers (N x L each); returns when c is written.  Pinned
    // buffers are read and written by DMA directly; pageable ones are staged
    // through pinned memory by the copy pool.  Either way the operands move in
    // chunks, each chunk's decompose starting as soon as it has landed, and the
    // result moves out chunk by chunk behind the CRT.  With c == nullptr the
    // destination comes from out_fn(out_arg), called on this thread once the
    // whole product is enqueued and right before c is first written, so a
    // caller can allocate c while the GPU works.
    void run_host(const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* (*out_fn)(void*) = nullptr,
                  void* out_arg = nullptr);

    // Measures the host path's chunk counts on this point and keeps the
    // fastest (the default unless another is 5% faster); returns the count.
    // Synchronous, about a dozen products' time; fherma_init calls it.
    int tune_host_path();

    // Stages, for checks against the oracle.
    void decompose(const uint32_t* d_limbs, uint32_t* d_res, int operand, cudaStream_t st);
    // Both operands in one launch: d_limbs = a then b, d_res = A then B.
    void decompose_pair(const uint32_t* d_limbs, uint32_t* d_res, cudaStream_t st);
    void transform(uint32_t* d_A, uint32_t* d_B, int mode, cudaStream_t st);
    void crt(const uint32_t* d_y, uint32_t* d_c, cudaStream_t st);

    // Reads and clears the device error word (nonzero: a pipeline wait in a
    // tensor-core kernel timed out); synchronous.
    uint32_t take_error();
    // The same after waiting for the work enqueued on st.
    uint32_t take_error(cudaStream_t st);
    // Reads and clears the error word of the static scratch array on the
    // current device (fpm_run_device_noalloc's calls), after waiting for st.
    static uint32_t take_static_error(cudaStream_t st);

    // Limit of every pipeline wait in this engine's kernels, in nanoseconds
    // (DevPoint::wait_ns); applies to products enqueued afterwards.
    void set_wait_limit(uint64_t ns) { dp_.wait_ns = ns; }
    // Test hook (DevPoint::fault): the pipelines of products enqueued
    // afterwards leave one barrier phase without its arrival.
    void set_fault(uint32_t mask) { dp_.fault = mask; }

    // Device bytes this context uses: its own buffers plus its prime basis's
    // tables, which contexts with the same (N, L, bits of q, prime window) on
    // the device share.
    size_t device_bytes() const;
    // Copies the CRT tables built on the device, M (K x L) and negvP
    // ((K + 1) x L), to host memory; returns K.
    uint32_t crt_tables(uint32_t* M, uint32_t* negvP) const;

    size_t words() const { return static_cast<size_t>(plan_.N) * plan_.L; }
    size_t residues() const { return static_cast<size_t>(plan_.K) * plan_.N; }

private:
    size_t static_scratch_err_offset() const;
    // The product's launches on workspaces A, B with point d (whose err names
    // the error word to use).
    void product(const DevPoint& d, const uint32_t* d_a, const uint32_t* d_b, uint32_t* A, uint32_t* B, uint32_t* d_c,
                 cudaStream_t st);
    void release();
    void decompose_pair_on(const DevPoint& d, const uint32_t* a, const uint32_t* b, uint32_t* A, uint32_t* B,
                           cudaStream_t st);
    void launch_dec(const uint32_t* d_limbs, uint32_t* d_res, int operand, uint32_t n0, uint32_t n1,
                    cudaStream_t st);
    void launch_crt_any(const DevPoint& d, const uint32_t* d_y, uint32_t* d_c, uint32_t n0, uint32_t n1,
                        cudaStream_t st);
    void ensure_host_path();
    void set_chunks(int want);
    template <class T>
    T* dalloc(size_t count);
    template <class T>
    const T* upload(const std::vector<T>& v);

    struct Basis;
    std::shared_ptr<Basis> basis_;   // shared tables of the prime basis
    HostPlan plan_;                  // the basis's plan (big tables dropped) plus q
    DevPoint dp_{};
    size_t own_bytes_ = 0;
    int device_ = 0;
    int sms_ = 0;
    bool simt_ = false;        // FPM_KERNELS=simt: CUDA-core decompose and CRT
    std::vector<void*> dmem_;
    uint32_t* A_ = nullptr;   // K x N residues
    uint32_t* B_ = nullptr;
    uint32_t* la_ = nullptr;  // N x L device limbs for the host path
    uint32_t* lb_ = nullptr;
    uint32_t* lc_ = nullptr;
    uint32_t* ha_ = nullptr;  // pinned staging
    uint32_t* hb_ = nullptr;
    uint32_t* hc_ = nullptr;
    cudaStream_t stream_ = nullptr;   // kernels
    cudaStream_t copy_ = nullptr;     // host -> device
    cudaStream_t out_ = nullptr;      // device -> host
    std::vector<cudaEvent_t> events_;
    std::vector<uint32_t> chunk_at_;  // I/O chunk boundaries (coefficients)
    std::unique_ptr<CopyPool> pool_;
    std::shared_ptr<const CrtConsts> crt_consts_;   // pipelined CRT's kernel parameters
    std::shared_ptr<const DecConsts> dec_consts_;   // pipelined decompose's kernel parameters
};

// Shared-memory opt-ins, once per device per process.
void ensure_kernel_attributes(int device);

// Size of the static scratch array behind Engine::run_device_static.
size_t static_scratch_bytes();

}  // namespace fpm
