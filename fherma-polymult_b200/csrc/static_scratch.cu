// The product with its scratch in a static device array (fpm_run_device_noalloc).
//
// Some callers cannot call cudaMalloc once they are running: a process under a
// fixed device-memory budget that it may not grow, or a caller whose own rules
// forbid allocating on its hot path.  fpm_run_device
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
// The kernels are the ones fpm_run_device launches (the pipelined decompose
// and CRT where the point has them); their constants are the context's,
// uploaded by fpm_init, and the CRT's tensor map is encoded on the host.
//
// Every call shares the array and it keeps the last call's contents: the
// residue workspaces are fully rewritten by the decompose kernels.  The error
// word is not cleared by a call: a kernel whose pipeline wait runs out sets a
// bit in it, and the bit stays until fpm_noalloc_get_error reads and clears
// it, so a caller that checks after a run of calls learns whether any of them
// failed.  Calls whose work overlaps on the GPU (different streams, or
// different host threads without ordering) race on the array; order them on
// one stream.
//
// The address lookup is cached per device for the life of the process; after
// cudaDeviceReset on a device the cached address is stale, so the library must
// not be used on that device again in the same process.
#include "engine.h"
#include "kernels.h"

#include <mutex>
#include <stdexcept>
#include <string>

namespace fpm {

namespace {

constexpr size_t kStaticScratchBytes = size_t(80) << 20;
constexpr size_t kStaticScratchWords = kStaticScratchBytes / sizeof(uint32_t);
constexpr size_t kStaticErrWord = kStaticScratchWords - 64;

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

// Scratch layout in words: A and B (K N each) from the start, the error word in
// the array's last 256-byte line, the same for every point.
size_t Engine::static_scratch_err_offset() const { return kStaticErrWord; }
size_t Engine::static_scratch_words_needed() const { return (2 * residues() + 63) / 64 * 64 + 64; }

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
    DevPoint d = dp_;
    d.err = base + static_scratch_err_offset();
    product(d, d_a, d_b, base, base + residues(), d_c, st);
}

uint32_t Engine::take_static_error(cudaStream_t st) {
    int cur = -1;
    check(cudaGetDevice(&cur), "cudaGetDevice");
    // The error word sits at the same place for every point: right after the
    // largest workspaces the array can hold.
    uint32_t* err = static_cast<uint32_t*>(scratch_address(cur)) + kStaticErrWord;
    check(cudaStreamSynchronize(st), "stream synchronize");
    uint32_t e = 0;
    check(cudaMemcpy(&e, err, sizeof(e), cudaMemcpyDeviceToHost), "read error word");
    if (e) check(cudaMemset(err, 0, sizeof(e)), "clear error word");
    return e;
}

}  // namespace fpm
