// Decompose on the CUDA cores: limbs (N x L) -> residues (K x N).
//
// x mod p_j = sum_l x_l c_{j,l} mod p_j with c_{j,l} = 2^(32 l) mod p_j (times
// the pointwise scale for operand b); each term is a lazy Shoup product below
// 2p, the terms are summed in 64 bits and the sum reduced once at the end
// (reference: decompose_many, rns.cuh:110-128; k_decompose, solve.cu:98-126).
//
// A block takes 128 consecutive coefficients (a contiguous run of 128 L words,
// loaded coalesced into a shared tile with an odd row stride) and all K primes;
// thread t handles coefficient t % 128 for primes j = t / 128, t / 128 + 2, ...
// so each prime's 128 residues are stored by consecutive threads.
#include "device.cuh"
#include "kernels.h"

namespace fpm {

namespace {

constexpr int kDecThreads = 256;
constexpr uint32_t kDecCoeffs = 128;

__global__ void __launch_bounds__(kDecThreads)
    k_decompose_simt(DevPoint d, const uint32_t* __restrict__ limbs, uint32_t* __restrict__ res, int operand,
                     uint32_t n_begin, uint32_t n_end) {
    extern __shared__ uint32_t xs[];   // kDecCoeffs rows of L + 1 words
    const int L = d.L;
    const uint32_t stride = static_cast<uint32_t>(L) + 1;
    const uint32_t n0 = n_begin + blockIdx.x * kDecCoeffs;
    const uint32_t nk = min(kDecCoeffs, n_end - n0);
    const uint32_t* src = limbs + static_cast<size_t>(n0) * L;
    for (uint32_t i = threadIdx.x; i < nk * L; i += kDecThreads) {
        const uint32_t row = i / L, l = i - row * L;
        xs[row * stride + l] = src[i];
    }
    __syncthreads();
    const uint32_t n = threadIdx.x % kDecCoeffs;
    if (n >= nk) return;
    const uint2* cst = operand ? d.dec_b : d.dec_a;
    const uint32_t* x = xs + n * stride;
    for (int j = threadIdx.x / kDecCoeffs; j < d.K; j += kDecThreads / kDecCoeffs) {
        const PrimeConsts pc = d.pc[j];
        const uint2* c = cst + static_cast<size_t>(j) * L;
        uint64_t acc = 0;
        for (int l = 0; l < L; ++l) {
            const uint2 w = c[l];
            acc += shoup_lazy(x[l], w.x, w.y, pc.p);   // < 2p each: acc < 2^38
        }
        // acc = hi 2^32 + lo: lo mod p by a Shoup product with w = 1, hi 2^32
        // by one with w = 2^32 mod p.
        const uint32_t p = pc.p;
        const uint32_t r32 = static_cast<uint32_t>((1ull << 32) % p);
        const uint32_t one_s = static_cast<uint32_t>((1ull << 32) / p);
        const uint32_t lo = shoup(static_cast<uint32_t>(acc), 1u, one_s, p);
        const uint32_t hi = shoup(static_cast<uint32_t>(acc >> 32), r32, shoup_companion(r32, pc), p);
        res[static_cast<size_t>(j) * d.N + n0 + n] = add_mod(lo, hi, p);
    }
}

}  // namespace

void decompose_init_attributes() {
    check(cudaFuncSetAttribute(k_decompose_simt, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(kDecCoeffs * (kMaxL + 1) * sizeof(uint32_t))),
          "decompose smem");
}

void launch_decompose(const DevPoint& d, const uint32_t* limbs, uint32_t* res, int operand, uint32_t n_begin,
                      uint32_t n_end, cudaStream_t st) {
    if (n_end <= n_begin) return;
    const uint32_t blocks = (n_end - n_begin + kDecCoeffs - 1) / kDecCoeffs;
    const size_t smem = kDecCoeffs * (static_cast<size_t>(d.L) + 1) * sizeof(uint32_t);
    k_decompose_simt<<<blocks, kDecThreads, smem, st>>>(d, limbs, res, operand, n_begin, n_end);
}

}  // namespace fpm
