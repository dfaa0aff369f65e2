// The product with its scratch in a static device array (fpm_run_device_noalloc).
//
// Some callers cannot call cudaMalloc once they are running: a process under a
// fixed device-memory budget, or code that issues work where allocation is not
// allowed (for example while a stream is being captured).  fpm_run_device
// itself allocates nothing either, but it uses the residue workspaces that
// fpm_init allocated for its context.  This variant never touches those: the
// product's scratch -- the two residue workspaces (2 K N words) and the
// pipeline error word -- lives in one file-scope static device array of
// kStaticScratchBytes (80 MiB, enough for every point up to N = 65536 at
// W = 2048) that every GPU loading the library holds until
// the process exits.  The call allocates nothing, on the device or the host.
//
// The array's name is only a host-side stand-in for the device symbol; its
// device address is looked up once per device with cudaGetSymbolAddress (with
// that device current) and passed to the kernels.  The first call on each
// device does that lookup, which also loads this file's module; make that first
// call before any stream capture.
//
// Every call shares the array and it keeps the last call's contents: the
// residue workspaces are fully rewritten by the decompose kernels, and the
// error word is cleared at the start of each call.  Calls whose work overlaps
// on the GPU (different streams, or different host threads without ordering)
// race on the array; order them on one stream.
#include "engine.h"
#include "kernels.h"

#include <mutex>
#include <stdexcept>
#include <string>

namespace fpm {

namespace {

constexpr size_t kStaticScratchBytes = size_t(80) << 20;
constexpr size_t kStaticScratchWords = kStaticScratchBytes / sizeof(uint32_t);

static __device__ __align__(256) uint32_t g_fpm_static_scratch[kStaticScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_fpm_static_scratch on `device` (which must be current).
void* scratch_address(int device) {
    if (device < 0 || device >= kMaxDevices) throw std::runtime_error("static scratch: device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        check(cudaGetSymbolAddress(&p, g_fpm_static_scratch), "cudaGetSymbolAddress(static scratch)");
        g_scratch_addr[device] = p;
    }
    return g_scratch_addr[device];
}

}  // namespace

size_t static_scratch_bytes() { return kStaticScratchBytes; }

// Scratch layout in words: A and B (K N each), then the error word on its own
// 256-byte line.
size_t Engine::static_scratch_err_offset() const { return (2 * residues() + 63) / 64 * 64; }
size_t Engine::static_scratch_words_needed() const { return static_scratch_err_offset() + 64; }

void Engine::run_device_static(const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t st) {
    const size_t need = static_scratch_words_needed();
    if (need > kStaticScratchWords) {
        throw std::runtime_error("fpm_run_device_noalloc: this point needs " + std::to_string(need * 4) +
                                 " bytes of scratch (2 K N words for K = " + std::to_string(plan_.K) +
                                 ", N = " + std::to_string(plan_.N) + ") but the static scratch holds " +
                                 std::to_string(kStaticScratchBytes) + "; use fpm_run_device");
    }
    int cur = -1;
    check(cudaGetDevice(&cur), "cudaGetDevice");
    if (cur != device_) {
        throw std::runtime_error("fpm_run_device_noalloc: the context lives on device " + std::to_string(device_) +
                                 " but device " + std::to_string(cur) + " is current");
    }
    uint32_t* base = static_cast<uint32_t*>(scratch_address(cur));
    uint32_t* A = base;
    uint32_t* B = base + residues();
    uint32_t* err = base + static_scratch_err_offset();
    check(cudaMemsetAsync(err, 0, sizeof(uint32_t), st), "clear error word");
    DevPoint d = dp_;
    d.err = err;
    const uint32_t N = plan_.N;
    if (simt_) {
        launch_decompose(d, d_a, A, 0, 0, N, st);
        launch_decompose(d, d_b, B, 1, 0, N, st);
    } else {
        launch_decompose_tc(d, d_a, A, 0, 0, N, st);
        launch_decompose_tc(d, d_b, B, 1, 0, N, st);
    }
    launch_ntt(d, A, B, kRowProduct, st);
    if (simt_ || !crt_uses_tc(plan_)) {
        launch_crt(d, A, d_c, 0, N, st);
    } else {
        launch_crt_tc(d, A, d_c, 0, N, st);
    }
    check(cudaGetLastError(), "product launch");
}

}  // namespace fpm
