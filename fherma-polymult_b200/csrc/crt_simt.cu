// CRT on the CUDA cores: y_j (K x N) -> c (N x L) mod q.
//
// With y_j = c (P/p_j)^-1 mod p_j, the exact centred coefficient is
// sum_j y_j (P/p_j) - v P with v = round(sum_j y_j / p_j) (the 2^20 margin of
// the prime set keeps the rounding exact in double), so
//     c mod q = sum_j y_j M_j + negvP_v  (mod q),  M_j = P/p_j mod q
// (reference: CrtView rns.cuh:225-240, crt_columns / crt_combine
// rns_kernels.cuh:265-364).
//
// A block takes 32 coefficients (one per lane).  Warp w accumulates the limb
// columns [8w, 8w + 8] of sum_j y_j M_j for all 32 (y loads coalesce across
// lanes, M loads are warp-uniform); warp 0 also sums y_j / p_j.  Then warp 0
// adds the column partials and negvP_v with carries and reduces mod q, and the
// block stores the 32 coefficients' limbs contiguously.
#include "device.cuh"
#include "kernels.h"

namespace fpm {

namespace {

constexpr int kCrtThreads = 256;
constexpr int kCrtChunk = 8;      // limbs per warp
constexpr int kCrtCoeffs = 32;

size_t crt_smem_bytes(int L) {
    return sizeof(uint64_t) * 8 * kCrtCoeffs * (kCrtChunk + 1) + sizeof(double) * kCrtCoeffs +
           sizeof(uint32_t) * kCrtCoeffs * (L + 2);
}

__global__ void __launch_bounds__(kCrtThreads)
    k_crt_simt(DevPoint d, const uint32_t* __restrict__ Y, uint32_t* __restrict__ C, uint32_t n_begin, uint32_t n_end) {
    extern __shared__ __align__(16) uint64_t crt_smem[];
    uint64_t* part = crt_smem;                                          // [8][32][9]
    double* frac = reinterpret_cast<double*>(part + 8 * kCrtCoeffs * (kCrtChunk + 1));
    uint32_t* xw = reinterpret_cast<uint32_t*>(frac + kCrtCoeffs);      // [32][L + 2]
    const int L = d.L, K = d.K;
    const int chunks = (L + kCrtChunk - 1) / kCrtChunk;
    const uint32_t n0 = n_begin + blockIdx.x * kCrtCoeffs;
    const uint32_t nk = min(static_cast<uint32_t>(kCrtCoeffs), n_end - n0);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n = n0 + lane;

    if (w < chunks) {
        uint64_t acc[kCrtChunk + 1];
#pragma unroll
        for (int t = 0; t <= kCrtChunk; ++t) acc[t] = 0;
        double f = 0;
        const int l0 = w * kCrtChunk;
        for (int j = 0; j < K; ++j) {
            const uint32_t y = lane < static_cast<int>(nk) ? Y[static_cast<size_t>(j) * d.N + n] : 0u;
            if (w == 0) f += static_cast<double>(y) * d.p_recip[j];
            const uint32_t* m = d.M + static_cast<size_t>(j) * L + l0;
#pragma unroll
            for (int t = 0; t < kCrtChunk; ++t) {
                if (l0 + t < L) {
                    const uint64_t prod = static_cast<uint64_t>(y) * m[t];
                    acc[t] += static_cast<uint32_t>(prod);
                    acc[t + 1] += prod >> 32;
                }
            }
        }
        uint64_t* dst = part + (w * kCrtCoeffs + lane) * (kCrtChunk + 1);
#pragma unroll
        for (int t = 0; t <= kCrtChunk; ++t) dst[t] = acc[t];
        if (w == 0) frac[lane] = f;
    }
    __syncthreads();

    if (w == 0 && lane < static_cast<int>(nk)) {
        int v = static_cast<int>(floor(frac[lane] + 0.5));
        v = v < 0 ? 0 : (v > K ? K : v);
        const uint32_t* t = d.negvP + static_cast<size_t>(v) * L;
        uint32_t* x = xw + lane * (L + 2);
        uint64_t carry = 0;
        for (int l = 0; l < L + 2; ++l) {
            uint64_t s = carry + (l < L ? t[l] : 0u);
            const int c = l / kCrtChunk, r = l % kCrtChunk;
            if (c < chunks) s += part[(c * kCrtCoeffs + lane) * (kCrtChunk + 1) + r];
            if (r == 0 && c >= 1 && c - 1 < chunks) s += part[((c - 1) * kCrtCoeffs + lane) * (kCrtChunk + 1) + kCrtChunk];
            x[l] = static_cast<uint32_t>(s);
            carry = s >> 32;
        }
        reduce_mod_q(x, L + 2, d.q, L, d.q_top);
    }
    __syncthreads();

    uint32_t* out = C + static_cast<size_t>(n0) * L;
    for (uint32_t i = threadIdx.x; i < nk * static_cast<uint32_t>(L); i += kCrtThreads) {
        const uint32_t row = i / L, l = i - row * L;
        out[i] = xw[row * (L + 2) + l];
    }
}

}  // namespace

void crt_init_attributes() {
    check(cudaFuncSetAttribute(k_crt_simt, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(crt_smem_bytes(kMaxL))),
          "crt smem");
}

void launch_crt(const DevPoint& d, const uint32_t* Y, uint32_t* c, uint32_t n_begin, uint32_t n_end,
                cudaStream_t st) {
    if (n_end <= n_begin) return;
    const uint32_t blocks = (n_end - n_begin + kCrtCoeffs - 1) / kCrtCoeffs;
    k_crt_simt<<<blocks, kCrtThreads, crt_smem_bytes(d.L), st>>>(d, Y, c, n_begin, n_end);
}

}  // namespace fpm
