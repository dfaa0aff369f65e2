// Register-blocked NTT rounds on a 2048-element shared-memory tile.
//
// A tile holds 2048 / 2^NSUB independent sub-transforms of 2^NSUB elements
// (logical index i = g 2^NSUB + x: sub-transform g, position x).  256 threads
// each hold 8 elements in registers per "round" and apply up to three radix-2
// stages to them before the tile is exchanged through shared memory.
//
// Round r covers the stage bits [lo, lo + cnt) with lo = NSUB - 3r - cnt;
// cnt = 3 except for a short last round.  The thread's 8 elements differ in the
// three bits lo, lo+1, lo+2 (a short round carries the bits above its stages
// along), so element k of a thread sits at base | (k << lo).
//
// Shared memory is swizzled: word i lives at i ^ ((i >> 5) & 31).  Within a
// round the 32 lanes of a warp take the 5 "lane bits": bit c for c in 0..4,
// or bit c + 5 where c is one of the round's register bits.  Each bank bit c
// then depends on exactly one lane bit, so every shared-memory access of a
// round is bank-conflict free.  The remaining 3 thread bits index the warp.
//
// Twiddles: the forward stage of distance 2^s pairs x and x + 2^s, and its
// twiddle is entry y = 2^(NSUB-1-s) + (x >> (s+1)) of the sub-transform's
// table (psi^bitrev(m + i) in the reference's notation, rns_kernels.cuh:132-157,
// restricted to one sub-transform).  Entries are Shoup pairs {w, ws}.
#pragma once

#include "arith.cuh"

namespace fpm {

constexpr int kNttThreads = 256;

__device__ __forceinline__ uint32_t swz(uint32_t i) { return i ^ ((i >> 5) & 31u); }

template <int NSUB>
struct Rounds {
    static_assert(NSUB >= 6 && NSUB <= 11, "sub-transforms of 2^6 .. 2^11 elements");
    static constexpr int kCount = (NSUB + 2) / 3;
    static constexpr __host__ __device__ int cnt(int r) {
        return (r < kCount - 1 || NSUB % 3 == 0) ? 3 : NSUB % 3;
    }
    static constexpr __host__ __device__ int lo(int r) { return NSUB - 3 * r - cnt(r); }
    static constexpr __host__ __device__ bool is_reg(int r, int bit) { return bit >= lo(r) && bit < lo(r) + 3; }
    static constexpr __host__ __device__ int lane_pos(int r, int m) { return is_reg(r, m) ? m + 5 : m; }
    static constexpr __host__ __device__ bool is_lane(int r, int bit) {
        return lane_pos(r, 0) == bit || lane_pos(r, 1) == bit || lane_pos(r, 2) == bit || lane_pos(r, 3) == bit ||
               lane_pos(r, 4) == bit;
    }
    // m-th (ascending) bit of [0, 11) that is neither a register nor a lane bit.
    static constexpr __host__ __device__ int warp_pos(int r, int m) {
        int seen = 0;
        for (int b = 0; b < 11; ++b) {
            if (is_reg(r, b) || is_lane(r, b)) continue;
            if (seen == m) return b;
            ++seen;
        }
        return -1;
    }
};

// Logical index of element 0 of this thread in round R.
template <int NSUB, int R>
__device__ __forceinline__ uint32_t round_base(uint32_t tid) {
    using RP = Rounds<NSUB>;
    const uint32_t lane = tid & 31u, warp = tid >> 5;
    uint32_t b = 0;
#pragma unroll
    for (int m = 0; m < 5; ++m) b |= ((lane >> m) & 1u) << RP::lane_pos(R, m);
#pragma unroll
    for (int m = 0; m < 3; ++m) b |= ((warp >> m) & 1u) << RP::warp_pos(R, m);
    return b;
}

template <int NSUB, int R>
__device__ __forceinline__ void load_round(const uint32_t* tile, uint32_t (&v)[8], uint32_t base) {
    constexpr int lo = Rounds<NSUB>::lo(R);
    const uint32_t sb = swz(base);
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = tile[sb ^ swz(static_cast<uint32_t>(k) << lo)];
}

template <int NSUB, int R>
__device__ __forceinline__ void store_round(uint32_t* tile, const uint32_t (&v)[8], uint32_t base) {
    constexpr int lo = Rounds<NSUB>::lo(R);
    const uint32_t sb = swz(base);
#pragma unroll
    for (int k = 0; k < 8; ++k) tile[sb ^ swz(static_cast<uint32_t>(k) << lo)] = v[k];
}

// Twiddle table index for the stage of distance 2^s at the pair whose lower
// element is base | (k << lo).
template <int NSUB, int R>
__device__ __forceinline__ uint32_t tw_index(uint32_t base, int k, int s) {
    constexpr int lo = Rounds<NSUB>::lo(R);
    const uint32_t x = (base | (static_cast<uint32_t>(k) << lo)) & ((1u << NSUB) - 1u);
    return (1u << (NSUB - 1 - s)) | (x >> (s + 1));
}

// Forward (Cooley-Tukey) stages of round R on NV operands that share the same
// twiddles; tw(g, y) returns entry y of sub-transform g's table.
template <int NSUB, int R, int NV, class TW>
__device__ __forceinline__ void fwd_round(uint32_t (&v)[NV][8], uint32_t base, const TW& tw, uint32_t p) {
    using RP = Rounds<NSUB>;
    constexpr int lo = RP::lo(R), cnt = RP::cnt(R);
    const uint32_t g = base >> NSUB;
#pragma unroll
    for (int m = cnt - 1; m >= 0; --m) {
        const int s = lo + m;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k & (1 << m)) continue;
            const uint2 w = tw(g, tw_index<NSUB, R>(base, k, s));
#pragma unroll
            for (int o = 0; o < NV; ++o) ct_butterfly(v[o][k], v[o][k | (1 << m)], w, p);
        }
    }
}

// Inverse (Gentleman-Sande) stages of round R, distances increasing.
template <int NSUB, int R, class TW>
__device__ __forceinline__ void inv_round(uint32_t (&v)[8], uint32_t base, const TW& tw, uint32_t p) {
    using RP = Rounds<NSUB>;
    constexpr int lo = RP::lo(R), cnt = RP::cnt(R);
    const uint32_t g = base >> NSUB;
#pragma unroll
    for (int m = 0; m < cnt; ++m) {
        const int s = lo + m;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k & (1 << m)) continue;
            const uint2 w = tw(g, tw_index<NSUB, R>(base, k, s));
            gs_butterfly(v[k], v[k | (1 << m)], w, p);
        }
    }
}

// Twiddle sources.
struct SharedTable {     // one table for every sub-transform of the tile
    const uint2* t;
    __device__ __forceinline__ uint2 operator()(uint32_t, uint32_t y) const { return t[y]; }
};

template <int NSUB>
struct PerRowTable {     // table g at t + g 2^NSUB
    const uint2* t;
    __device__ __forceinline__ uint2 operator()(uint32_t g, uint32_t y) const { return t[(g << NSUB) + y]; }
};

}  // namespace fpm
