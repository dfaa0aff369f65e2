// Register-blocked NTT rounds on a 2048-element shared-memory tile.
//
// A tile holds 2048 / 2^NSUB independent sub-transforms of 2^NSUB elements.  The
// tile index i carries the position x inside a sub-transform in bits
// [XS, XS + NSUB) and the sub-transform's id in the other bits (the row pass
// keeps rows contiguous, XS = 0; the column pass keeps a row's C = 2^XS
// columns contiguous, XS = 11 - NSUB).  256 threads each hold 8 elements in
// registers per "round" and apply up to three radix-2 stages to them between
// exchanges through shared memory.
//
// Round r covers the stage bits [lo, lo + cnt) of x, lo = NSUB - 3r - cnt
// (cnt = 3 but for a short last round); a thread's 8 elements differ in the x
// bits lo, lo + 1, lo + 2, i.e. element k sits at base | (k << (XS + lo)).
//
// Shared memory is swizzled by a GF(2)-linear map of the word index (SWZ::f).
// Within a round the 32 lanes of a warp take 5 "lane bits" chosen so that each
// bank bit depends on exactly one lane bit; every shared access of a round is
// then free of bank conflicts (for the sizes the engine is used at).
//
// Twiddles: the forward stage of distance 2^s pairs x and x + 2^s and uses
// entry 2^(NSUB-1-s) + (x >> (s+1)) of the sub-transform's table (the
// reference's psi^bitrev(m + i), rns_kernels.cuh:132-157, restricted to one
// sub-transform).  A round's (up to) 7 twiddles are entries y, 2y, 2y + 1 and
// 4y .. 4y + 3 for one y, so they arrive in three vector loads.
//
// Butterflies come in two forms (arith.cuh): LAZY (Harvey: values below 4p in
// the forward direction and below 2p in the inverse, needs p < 2^30) and full
// reduction (values canonical, any p < 2^31).
#pragma once

#include "arith.cuh"

namespace fpm {

constexpr int kNttThreads = 256;

// Row pass: bank bit c of word i is i_c ^ i_{c+5}.
struct SwzRow {
    static __device__ __forceinline__ uint32_t f(uint32_t i) { return i ^ ((i >> 5) & 31u); }
    static constexpr __host__ __device__ int partner(int c) { return c + 5; }
};
// Column pass: the 128-byte TMA swizzle (16-byte chunk index ^= 128-byte line
// index mod 8); bank bits 0, 1 are i_0, i_1 and bank bit c >= 2 is i_c ^ i_{c+3}.
struct SwzCol {
    static __device__ __forceinline__ uint32_t f(uint32_t i) { return i ^ (((i >> 5) & 7u) << 2); }
    static constexpr __host__ __device__ int partner(int c) { return c >= 2 ? c + 3 : -1; }
};

struct RoundMap {
    int lane[5];
    int warp[3];
};

template <int NSUB, int XS, class SWZ>
struct Rounds {
    static_assert(NSUB >= 6 && NSUB <= 11 && XS + NSUB <= 11, "2^6 .. 2^11-element sub-transforms");
    static constexpr int kCount = (NSUB + 2) / 3;
    static constexpr __host__ __device__ int cnt(int r) { return (r < kCount - 1 || NSUB % 3 == 0) ? 3 : NSUB % 3; }
    static constexpr __host__ __device__ int lo(int r) { return NSUB - 3 * r - cnt(r); }
    static constexpr __host__ __device__ bool is_reg(int r, int bit) {
        return bit >= XS + lo(r) && bit < XS + lo(r) + 3;
    }
    static constexpr __host__ __device__ RoundMap map(int r) {
        RoundMap m{};
        bool used[11] = {};
        for (int b = 0; b < 11; ++b) used[b] = is_reg(r, b);
        // lane bits: bank bit c itself, else its swizzle partner, else any free bit
        for (int c = 0; c < 5; ++c) {
            int pick = -1;
            if (!used[c]) {
                pick = c;
            } else {
                const int pc = SWZ::partner(c);
                if (pc >= 0 && pc < 11 && !used[pc]) pick = pc;
            }
            if (pick < 0) {
                for (int b = 0; b < 11 && pick < 0; ++b)
                    if (!used[b]) pick = b;
            }
            m.lane[c] = pick;
            used[pick] = true;
        }
        int w = 0;
        for (int b = 0; b < 11; ++b)
            if (!used[b]) m.warp[w++] = b;
        return m;
    }
};

// Bits of the lane (BITS = 5) or warp (BITS = 3) index that move by SH places.
template <int NSUB, int XS, class SWZ, int R, bool LANE>
__host__ __device__ constexpr uint32_t deposit_mask(int sh) {
    constexpr RoundMap m = Rounds<NSUB, XS, SWZ>::map(R);
    uint32_t mask = 0;
    for (int c = 0; c < (LANE ? 5 : 3); ++c)
        if ((LANE ? m.lane[c] : m.warp[c]) - c == sh) mask |= 1u << c;
    return mask;
}

template <int NSUB, int XS, class SWZ, int R, bool LANE>
__device__ __forceinline__ uint32_t deposit(uint32_t x) {
    uint32_t b = 0;
#pragma unroll
    for (int sh = 0; sh <= 10; ++sh) {
        const uint32_t mask = deposit_mask<NSUB, XS, SWZ, R, LANE>(sh);
        if (mask) b |= (x & mask) << sh;
    }
    return b;
}

// Logical index of element 0 of this thread in round R (lane bits and warp
// bits deposited group-wise: bits that move by the same distance move together).
template <int NSUB, int XS, class SWZ, int R>
__device__ __forceinline__ uint32_t round_base(uint32_t tid) {
    return deposit<NSUB, XS, SWZ, R, true>(tid & 31u) | deposit<NSUB, XS, SWZ, R, false>(tid >> 5);
}

template <int NSUB, int XS, class SWZ, int R>
__device__ __forceinline__ void load_round(const uint32_t* tile, uint32_t (&v)[8], uint32_t base) {
    constexpr int sh = XS + Rounds<NSUB, XS, SWZ>::lo(R);
    const uint32_t sb = SWZ::f(base);
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = tile[sb ^ SWZ::f(static_cast<uint32_t>(k) << sh)];
}

template <int NSUB, int XS, class SWZ, int R>
__device__ __forceinline__ void store_round(uint32_t* tile, const uint32_t (&v)[8], uint32_t base) {
    constexpr int sh = XS + Rounds<NSUB, XS, SWZ>::lo(R);
    const uint32_t sb = SWZ::f(base);
#pragma unroll
    for (int k = 0; k < 8; ++k) tile[sb ^ SWZ::f(static_cast<uint32_t>(k) << sh)] = v[k];
}

// ---- butterflies ------------------------------------------------------------------

template <bool LAZY>
__device__ __forceinline__ void bf_fwd(uint32_t& x, uint32_t& y, uint2 w, uint32_t p) {
    if constexpr (LAZY) {
        // x, y < 4p -> X, Y < 4p
        const uint32_t p2 = 2 * p;
        const uint32_t xr = umin32(x, x - p2);
        const uint32_t v = shoup_lazy(y, w.x, w.y, p);
        x = xr + v;
        y = xr - v + p2;
    } else {
        ct_butterfly(x, y, w, p);
    }
}

// Inverse butterfly; NEG: the twiddle is -w (the row pass reads inverse
// twiddles as negated forward ones), realised by swapping the difference.
template <bool LAZY, bool NEG>
__device__ __forceinline__ void bf_inv(uint32_t& x, uint32_t& y, uint2 w, uint32_t p) {
    if constexpr (LAZY) {
        // x, y < 2p -> X, Y < 2p
        const uint32_t p2 = 2 * p;
        const uint32_t s = x + y;
        const uint32_t d = NEG ? y - x + p2 : x - y + p2;
        x = umin32(s, s - p2);
        y = shoup_lazy(d, w.x, w.y, p);
    } else {
        const uint32_t u = x, v = y;
        x = add_mod(u, v, p);
        y = shoup(NEG ? sub_mod(v, u, p) : sub_mod(u, v, p), w.x, w.y, p);
    }
}

// ---- twiddle sources: entries y, {2y, 2y+1}, {4y .. 4y+3} of table g ---------------

struct Tw7 {
    uint2 w0, w1[2], w2[4];
};

struct SharedTable {    // one table for every sub-transform (16-byte aligned)
    const uint2* t;
    __device__ __forceinline__ Tw7 get(uint32_t, uint32_t y, int cnt) const {
        Tw7 r;
        if (cnt == 3) r.w0 = t[y];
        if (cnt >= 2) {
            const uint4 a = *reinterpret_cast<const uint4*>(t + 2 * y);
            r.w1[0] = make_uint2(a.x, a.y);
            r.w1[1] = make_uint2(a.z, a.w);
        }
        const uint4 b = *reinterpret_cast<const uint4*>(t + 4 * y);
        const uint4 c = *reinterpret_cast<const uint4*>(t + 4 * y + 2);
        r.w2[0] = make_uint2(b.x, b.y);
        r.w2[1] = make_uint2(b.z, b.w);
        r.w2[2] = make_uint2(c.x, c.y);
        r.w2[3] = make_uint2(c.z, c.w);
        return r;
    }
};

// Table of sub-transform g at t + g * STRIDE entries.  REFLECT: read the
// partner table (g ^ FLIP) at the index with its low bits complemented, which
// holds the negated inverse twiddles (see ntt.cu); the vector order reverses.
template <int NSUB, int STRIDE, bool REFLECT, uint32_t FLIP>
struct RowTable {
    const uint2* t;
    __device__ __forceinline__ Tw7 get(uint32_t g, uint32_t y, int cnt) const {
        const uint2* tb = t + (REFLECT ? (g ^ FLIP) : g) * STRIDE;
        Tw7 r;
        // y lies in [2^lev, 2^(lev+1)): its reflection is y ^ (2^lev - 1), and the
        // children 2y + t, 4y + t reflect to 2y* + 1 - t, 4y* + 3 - t.
        const uint32_t yy = REFLECT ? (y ^ ((1u << (31 - __clz(y))) - 1u)) : y;
        if (cnt == 3) r.w0 = tb[yy];
        if (cnt >= 2) {
            const uint4 a = *reinterpret_cast<const uint4*>(tb + 2 * yy);
            r.w1[REFLECT ? 1 : 0] = make_uint2(a.x, a.y);
            r.w1[REFLECT ? 0 : 1] = make_uint2(a.z, a.w);
        }
        const uint4 b = *reinterpret_cast<const uint4*>(tb + 4 * yy);
        const uint4 c = *reinterpret_cast<const uint4*>(tb + 4 * yy + 2);
        r.w2[REFLECT ? 3 : 0] = make_uint2(b.x, b.y);
        r.w2[REFLECT ? 2 : 1] = make_uint2(b.z, b.w);
        r.w2[REFLECT ? 1 : 2] = make_uint2(c.x, c.y);
        r.w2[REFLECT ? 0 : 3] = make_uint2(c.z, c.w);
        return r;
    }
};

// ---- rounds --------------------------------------------------------------------------

// Sub-transform id and the "virtual top" twiddle index y of the round.
template <int NSUB, int XS, class SWZ, int R>
__device__ __forceinline__ void round_tw_pos(uint32_t base, uint32_t& g, uint32_t& y) {
    constexpr int lo = Rounds<NSUB, XS, SWZ>::lo(R);
    const uint32_t x = (base >> XS) & ((1u << NSUB) - 1u);
    g = (base & ((1u << XS) - 1u)) | ((base >> (XS + NSUB)) << XS);
    y = (1u << (NSUB - 3 - lo)) | (x >> (lo + 3));
}

// Forward stages of round R on NV operands sharing the twiddles.
template <int NSUB, int XS, class SWZ, int R, bool LAZY, int NV, class TW>
__device__ __forceinline__ void fwd_round(uint32_t (&v)[NV][8], uint32_t base, const TW& tw, uint32_t p) {
    constexpr int cnt = Rounds<NSUB, XS, SWZ>::cnt(R);
    uint32_t g, y;
    round_tw_pos<NSUB, XS, SWZ, R>(base, g, y);
    const Tw7 w = tw.get(g, y, cnt);
    if constexpr (cnt == 3) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int o = 0; o < NV; ++o) bf_fwd<LAZY>(v[o][k], v[o][k + 4], w.w0, p);
    }
    if constexpr (cnt >= 2) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k & 2) continue;
#pragma unroll
            for (int o = 0; o < NV; ++o) bf_fwd<LAZY>(v[o][k], v[o][k + 2], w.w1[k >> 2], p);
        }
    }
#pragma unroll
    for (int k = 0; k < 8; k += 2)
#pragma unroll
        for (int o = 0; o < NV; ++o) bf_fwd<LAZY>(v[o][k], v[o][k + 1], w.w2[k >> 1], p);
}

// Inverse stages of round R (distances increasing).
template <int NSUB, int XS, class SWZ, int R, bool LAZY, bool NEG, class TW>
__device__ __forceinline__ void inv_round(uint32_t (&v)[8], uint32_t base, const TW& tw, uint32_t p) {
    constexpr int cnt = Rounds<NSUB, XS, SWZ>::cnt(R);
    uint32_t g, y;
    round_tw_pos<NSUB, XS, SWZ, R>(base, g, y);
    const Tw7 w = tw.get(g, y, cnt);
#pragma unroll
    for (int k = 0; k < 8; k += 2) bf_inv<LAZY, NEG>(v[k], v[k + 1], w.w2[k >> 1], p);
    if constexpr (cnt >= 2) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k & 2) continue;
            bf_inv<LAZY, NEG>(v[k], v[k + 2], w.w1[k >> 2], p);
        }
    }
    if constexpr (cnt == 3) {
#pragma unroll
        for (int k = 0; k < 4; ++k) bf_inv<LAZY, NEG>(v[k], v[k + 4], w.w0, p);
    }
}

}  // namespace fpm
