// Word arithmetic modulo a prime p < 2^31, and multi-limb helpers modulo q.
// Shared by the host plan builder and the device kernels (all functions are
// __host__ __device__).
//
// Conventions:
//   * residues are u32 in [0, p) unless a function says otherwise;
//   * a constant w used many times carries its Shoup companion
//     ws = floor(w 2^32 / p) (Shoup's precomputed-quotient product), stored as a
//     uint2 {w, ws} so one 8-byte load fetches both;
//   * pneg = -p^-1 mod 2^32 (Montgomery), mu = floor(2^64 / p) split in two
//     words (used to derive Shoup companions of computed constants).
//
// Reference counterparts (Akram275/fherma-polymult): rns.cuh:46-93 (word ops),
// rns.cuh:143-155 (butterflies), rns.cuh:161-221 (multi-limb reduce).
#pragma once

#include <cstdint>
#include <cmath>

#if defined(__CUDACC__)
#define FPM_HD __host__ __device__ __forceinline__
#else
#define FPM_HD inline
#endif

#if !defined(__CUDACC__)
struct uint2 {
    uint32_t x, y;
};
struct uint4 {
    uint32_t x, y, z, w;
};
#else
#include <cuda_runtime.h>
#endif

namespace fpm {

constexpr int kMaxL = 64;       // limbs per coefficient (W <= 2048)
constexpr int kMaxK = 160;      // primes
constexpr int kMaxLogN = 22;
constexpr int kMarginBits = 20; // P > 2^20 2N q^2 makes the CRT rounding exact

// Per-prime constants, 16 bytes.
struct PrimeConsts {
    uint32_t p;
    uint32_t pneg;    // -p^-1 mod 2^32
    uint32_t mu_lo;   // floor(2^64 / p) = mu_hi 2^32 + mu_lo
    uint32_t mu_hi;
};

FPM_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) >> 32);
#endif
}

FPM_HD uint32_t umin32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return ::min(a, b);
#else
    return a < b ? a : b;
#endif
}

// x in [0, 2p) -> [0, p).  (x - p wraps to a large value when x < p.)
FPM_HD uint32_t reduce_once(uint32_t x, uint32_t p) { return umin32(x, x - p); }

FPM_HD uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) { return reduce_once(a + b, p); }

FPM_HD uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) {
    const uint32_t d = a - b;
    return umin32(d, d + p);
}

// a w mod p plus 0 or p (below 2p), for any a < 2^32: the quotient estimate
// mulhi(a, ws) is the true quotient or one less.
FPM_HD uint32_t shoup_lazy(uint32_t a, uint32_t w, uint32_t ws, uint32_t p) {
    return a * w - mulhi32(a, ws) * p;
}

FPM_HD uint32_t shoup(uint32_t a, uint32_t w, uint32_t ws, uint32_t p) {
    return reduce_once(shoup_lazy(a, w, ws, p), p);
}

FPM_HD uint32_t shoup(uint32_t a, uint2 w, uint32_t p) { return shoup(a, w.x, w.y, p); }

// Montgomery product a b 2^-32 mod p for a, b < p.
FPM_HD uint32_t mont_mul(uint32_t a, uint32_t b, uint32_t p, uint32_t pneg) {
    const uint64_t t = static_cast<uint64_t>(a) * b;
    const uint32_t m = static_cast<uint32_t>(t) * pneg;
    const uint32_t u = static_cast<uint32_t>((t + static_cast<uint64_t>(m) * p) >> 32);
    return reduce_once(u, p);
}

// The Shoup companion floor(w 2^32 / p) of a computed w < p, from mu:
// floor(w mu / 2^32) is the companion or one less (mu <= 2^64 / p), and the
// remainder w 2^32 - c p, exact modulo 2^32 because it is below 2p, tells which.
FPM_HD uint32_t shoup_companion(uint32_t w, const PrimeConsts& pc) {
    uint32_t c = mulhi32(w, pc.mu_lo) + w * pc.mu_hi;
    const uint32_t r = 0u - c * pc.p;
    return c + (r >= pc.p ? 1u : 0u);
}

FPM_HD uint2 make_twiddle(uint32_t w, const PrimeConsts& pc) {
    uint2 t;
    t.x = w;
    t.y = shoup_companion(w, pc);
    return t;
}

// Forward (Cooley-Tukey) butterfly: (x, y) -> (x + w y, x - w y).
FPM_HD void ct_butterfly(uint32_t& x, uint32_t& y, uint2 w, uint32_t p) {
    const uint32_t v = shoup(y, w.x, w.y, p);
    const uint32_t u = x;
    x = add_mod(u, v, p);
    y = sub_mod(u, v, p);
}

// Inverse (Gentleman-Sande) butterfly: (x, y) -> (x + y, (x - y) w).
FPM_HD void gs_butterfly(uint32_t& x, uint32_t& y, uint2 w, uint32_t p) {
    const uint32_t u = x, v = y;
    x = add_mod(u, v, p);
    y = shoup(sub_mod(u, v, p), w.x, w.y, p);
}

// Tensor-core operand images in the UMMA K-major 128-byte-swizzle layout: a
// row's K bytes split in 128-byte halves, each half a block of rows x 128
// bytes; row r of a half at r * 128, its 16-byte chunk c at (c ^ (r % 8)) * 16
// (the swizzle the tensor cores undo on the fly; blocks 1024-byte aligned).
FPM_HD size_t sw128_offset(uint32_t row, uint32_t k, uint32_t rows) {
    const uint32_t half = k >> 7, c = (k >> 4) & 7u;
    return static_cast<size_t>(half) * rows * 128 + static_cast<size_t>(row) * 128 + (((c ^ (row & 7u)) << 4) | (k & 15u));
}
FPM_HD size_t sw128_bytes(uint32_t rows, uint32_t kbytes) {
    return static_cast<size_t>(rows) * 128 * ((kbytes + 127) / 128);
}

FPM_HD uint32_t bitrev(uint32_t x, uint32_t bits) {
    if (bits == 0) return 0;
#if defined(__CUDA_ARCH__)
    return __brev(x) >> (32 - bits);
#else
    uint32_t r = 0;
    for (uint32_t i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
#endif
}

// ---------------------------------------------------------------------------
// Multi-limb numbers: n little-endian u32 limbs; q has L limbs and reads as 0
// above them.

FPM_HD bool limbs_geq(const uint32_t* x, int n, const uint32_t* q, int L) {
#pragma unroll
    for (int i = n - 1; i >= 0; --i) {
        const uint32_t qi = i < L ? q[i] : 0u;
        if (x[i] != qi) return x[i] > qi;
    }
    return true;
}

// x -= q (x >= q).
FPM_HD void limbs_sub(uint32_t* x, int n, const uint32_t* q, int L) {
    uint32_t borrow = 0;
#pragma unroll
    for (int i = 0; i < n; ++i) {
        const uint64_t d = static_cast<uint64_t>(x[i]) - (i < L ? q[i] : 0u) - borrow;
        x[i] = static_cast<uint32_t>(d);
        borrow = static_cast<uint32_t>(d >> 63);
    }
}

// x -= e * q * 2^(32 shift), for a result known to be non-negative.
FPM_HD void limbs_submul(uint32_t* x, int n, const uint32_t* q, int L, uint32_t e, int shift) {
    uint64_t carry = 0;
    uint32_t borrow = 0;
#pragma unroll
    for (int i = shift; i < n; ++i) {
        const int k = i - shift;
        const uint64_t prod = (k < L ? static_cast<uint64_t>(e) * q[k] : 0u) + carry;
        carry = prod >> 32;
        const uint64_t d = static_cast<uint64_t>(x[i]) - static_cast<uint32_t>(prod) - borrow;
        x[i] = static_cast<uint32_t>(d);
        borrow = static_cast<uint32_t>(d >> 63);
    }
}

// Limbs of q left out of its double-precision top (q_top): the quotient
// estimate below compares the top min(L, 3) limbs.
FPM_HD int top_drop(int L) { return L > 3 ? L - 3 : 0; }

// q's top min(L, 3) limbs as a double.
inline double modulus_top(const uint32_t* q, int L) {
    double t = 0;
    for (int i = L - 1; i >= top_drop(L); --i) t = t * 4294967296.0 + q[i];
    return t;
}

// x mod q in place, for x < 2^64 q (n limbs, n <= L + 2).  The quotient is
// estimated in double from the top limbs; both tops carry relative error near
// 2^-52, so one less than the floor of the estimate never exceeds the true
// quotient and leaves x below 3q, which at most two subtractions finish.
// (Same method as the reference's reduce_wide, rns.cuh:204-221.)
FPM_HD void reduce_mod_q(uint32_t* x, int n, const uint32_t* q, int L, double q_top) {
    double xd = 0;
#pragma unroll
    for (int i = n - 1; i >= top_drop(L); --i) xd = xd * 4294967296.0 + x[i];
    const double f = floor(xd / q_top);
    const uint64_t e = f >= 1 ? static_cast<uint64_t>(f) - 1 : 0;
    if (e >> 32) limbs_submul(x, n, q, L, static_cast<uint32_t>(e >> 32), 1);
    if (e) limbs_submul(x, n, q, L, static_cast<uint32_t>(e), 0);
    for (int guard = 0; guard < 4 && limbs_geq(x, n, q, L); ++guard) limbs_sub(x, n, q, L);
}

}  // namespace fpm
