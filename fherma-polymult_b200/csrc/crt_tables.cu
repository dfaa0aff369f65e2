// The CRT constants of a modulus q, built on the device from the prime basis.
//
//   M_j     = prod_{i != j} p_i mod q                 (K x L limbs)
//   negvP_v = (q - v P mod q) mod q, v = 0 .. K        ((K + 1) x L)
//   the tensor-core CRT images (plan.h): crt_img holds M_j's low L - 1 limbs
//   byte-shifted into GEMM columns, crt_img_v the same with a row K for
//   negvP_1 = -P mod q (in the pipelined CRT's layout: every chunk but the
//   last 128-byte swizzled).
//
// Reference counterpart: rns_plan.h:224-247, where make_plan builds M_j and
// negvP on the host with an O(K^2 L) loop (one product of K - 1 primes mod q
// per j).  Here thread j of k_crt_products runs that product for its own j
// (thread K for P itself), so a new modulus costs one short launch instead of
// the host loop; the arithmetic (multiply by a word, then reduce_mod_q) is the
// host plan's own, so the tables are identical.
#include "device.cuh"
#include "kernels.h"

namespace fpm {

namespace {

// x (L limbs, x < q) = x * m mod q; t is scratch of L + 1 limbs.  LT > 0:
// L = LT at compile time, so every loop unrolls and x and t stay in
// registers (with a run-time L they live in local memory).
template <int LT>
__device__ __forceinline__ void mul_word_mod(uint32_t* x, uint32_t m, const uint32_t* q, int Lrt, double q_top,
                                             uint32_t* t) {
    const int L = LT > 0 ? LT : Lrt;
    uint64_t carry = 0;
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const uint64_t v = static_cast<uint64_t>(x[l]) * m + carry;
        t[l] = static_cast<uint32_t>(v);
        carry = v >> 32;
    }
    t[L] = static_cast<uint32_t>(carry);
    reduce_mod_q(t, L + 1, q, L, q_top);
#pragma unroll
    for (int l = 0; l < L; ++l) x[l] = t[l];
}

// Thread j < K: M_j.  Thread K: P mod q (into Pq).
template <int LT>
__global__ void k_crt_products(const PrimeConsts* pc, int K, const uint32_t* q, int Lrt, double q_top, uint32_t* M,
                               uint32_t* Pq) {
    const int L = LT > 0 ? LT : Lrt;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > K) return;
    constexpr int kL = LT > 0 ? LT : kMaxL;
    uint32_t x[kL], t[kL + 1];
#pragma unroll
    for (int l = 0; l < L; ++l) x[l] = l == 0 ? 1u : 0u;
    for (int i = 0; i < K; ++i) {
        if (i != j) mul_word_mod<LT>(x, pc[i].p, q, L, q_top, t);
    }
    uint32_t* out = j < K ? M + static_cast<size_t>(j) * L : Pq;
#pragma unroll
    for (int l = 0; l < L; ++l) out[l] = x[l];
}

// Thread v <= K: negvP_v.
__global__ void k_crt_negvp(const uint32_t* Pq, int K, const uint32_t* q, int L, double q_top, uint32_t* negvP) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v > K) return;
    uint32_t x[kMaxL], t[kMaxL + 1];
    for (int l = 0; l < L; ++l) x[l] = Pq[l];
    mul_word_mod<0>(x, static_cast<uint32_t>(v), q, L, q_top, t);
    bool zero = true;
    for (int l = 0; l < L; ++l) zero = zero && x[l] == 0;
    uint32_t* out = negvP + static_cast<size_t>(v) * L;
    uint32_t borrow = 0;
    for (int l = 0; l < L; ++l) {
        const uint64_t d = static_cast<uint64_t>(q[l]) - x[l] - borrow;
        out[l] = zero ? 0u : static_cast<uint32_t>(d);
        borrow = static_cast<uint32_t>(d >> 63);
    }
}

// Image row j (constant m, L limbs) into GEMM column 4 (j % 32) + s of chunk
// j / 32, byte position u: byte (u - s) of m's low L - 1 limbs.  One thread
// per (row, u); the image was zeroed.  Layout (crt_image_at): plain core
// matrices, or with swz every chunk but the last 128-byte swizzled.
__global__ void k_crt_image(const uint32_t* M, const uint32_t* negvP, int K, int L, uint32_t crt_u, int rows,
                            bool swz, uint8_t* img) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t j = idx / crt_u, u = idx - j * crt_u;
    if (j >= static_cast<uint32_t>(rows)) return;
    const uint32_t* m = j < static_cast<uint32_t>(K) ? M + static_cast<size_t>(j) * L : negvP + L;
    const uint32_t low_bytes = 4 * static_cast<uint32_t>(L - 1);
    for (uint32_t s = 0; s < 4 && s <= u; ++s) {
        const uint32_t byte = u - s;
        if (byte >= low_bytes) continue;
        img[crt_image_at(j, s, u, crt_u, rows, swz)] = static_cast<uint8_t>(m[byte / 4] >> (8 * (byte % 4)));
    }
}

}  // namespace

size_t crt_image_bytes(const HostPlan& pl, int rows) {
    return static_cast<size_t>(pl.crt_u) * 128 * static_cast<size_t>((rows + 31) / 32);
}

void build_crt_tables(const HostPlan& pl, const PrimeConsts* pc, const uint32_t* q, uint32_t* M, uint32_t* negvP,
                      uint32_t* Pq, uint8_t* img, uint8_t* img_v, cudaStream_t st) {
    const int K = pl.K, L = pl.L;
    // One thread per j runs K - 1 word products in sequence: small blocks
    // spread the K + 1 threads over SMs.
    const dim3 pg((K + 1 + 31) / 32), pb(32);
    switch (L) {
        case 64: k_crt_products<64><<<pg, pb, 0, st>>>(pc, K, q, L, pl.q_top, M, Pq); break;
        case 55: k_crt_products<55><<<pg, pb, 0, st>>>(pc, K, q, L, pl.q_top, M, Pq); break;
        case 28: k_crt_products<28><<<pg, pb, 0, st>>>(pc, K, q, L, pl.q_top, M, Pq); break;
        case 8: k_crt_products<8><<<pg, pb, 0, st>>>(pc, K, q, L, pl.q_top, M, Pq); break;
        default: k_crt_products<0><<<pg, pb, 0, st>>>(pc, K, q, L, pl.q_top, M, Pq); break;
    }
    check(cudaGetLastError(), "crt tables launch");
    k_crt_negvp<<<(K + 1 + 63) / 64, 64, 0, st>>>(Pq, K, q, L, pl.q_top, negvP);
    check(cudaGetLastError(), "crt tables launch");
    if (!crt_uses_tc(pl)) return;
    const int rows[2] = {K, K + 1};
    uint8_t* out[2] = {img, img_v};
    for (int i = 0; i < 2; ++i) {
        check(cudaMemsetAsync(out[i], 0, crt_image_bytes(pl, rows[i]), st), "crt image clear");
        const uint32_t threads = static_cast<uint32_t>(rows[i]) * pl.crt_u;
        k_crt_image<<<(threads + 255) / 256, 256, 0, st>>>(M, negvP, K, L, pl.crt_u, rows[i], i == 1, out[i]);
        check(cudaGetLastError(), "crt image launch");
    }
}

}  // namespace fpm
