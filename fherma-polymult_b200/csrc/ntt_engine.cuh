// Register-blocked NTT rounds on a 2048-element shared-memory tile.
//
// A tile holds 2048 / 2^NSUB independent sub-transforms of 2^NSUB elements.  The
// tile index i carries the position x inside a sub-transform in bits
// [XS, XS + NSUB) and the sub-transform's id in the other bits (the row pass
// keeps rows contiguous, XS = 0; the column pass keeps a row's C = 2^XS
// columns contiguous, XS = 11 - NSUB).  2^(11 - RB) threads each hold E = 2^RB
// elements in registers per "round" and apply up to RB radix-2 stages to them
// between exchanges through shared memory (RB = 3: 256 threads x 8 elements;
// RB = 4: 128 threads x 16 elements, half the exchanges for NSUB = 7, 8, 10, 11).
//
// Round r covers the stage bits [lo, lo + cnt) of x, lo = NSUB - RB r - cnt
// (cnt = RB but for a short last round, which has lo = 0); a thread's E elements
// differ in the x bits lo .. lo + RB - 1, i.e. element k sits at
// base | (k << (XS + lo)).
//
// Shared memory is swizzled by a GF(2)-linear map of the word index (SWZ::f).
// Within a round the 32 lanes of a warp take 5 "lane bits" chosen so that each
// bank bit depends on exactly one lane bit; every shared access of a round is
// then free of bank conflicts.  Rounds<>::conflict_free() checks this at compile
// time for every round a kernel instantiates.
//
// Twiddles: the forward stage of distance 2^s pairs x and x + 2^s and uses
// entry 2^(NSUB-1-s) + (x >> (s+1)) of the sub-transform's table (the
// reference's psi^bitrev(m + i), rns_kernels.cuh:132-157, restricted to one
// sub-transform).  A round's twiddles are, for one y, the entries
// (y << t) .. (y << t) + 2^t - 1 of each level t < RB (level t is the stage of
// register bit RB - 1 - t): 1 + 2 + 4 (+ 8) entries in 16-byte vector loads.
// The row pass stores its tables round-major (row_table_pos), so that the lanes
// of a round, which may differ in y, read consecutive 16-byte pairs.
//
// Butterflies come in two forms (arith.cuh): LAZY (Harvey: values below 4p in
// the forward direction and below 2p in the inverse, needs p < 2^30) and full
// reduction (values canonical, any p < 2^31).
#pragma once

#include "arith.cuh"

namespace fpm {

// Threads of a transform block holding RB register bits per round.
template <int RB>
constexpr int ntt_threads() {
    return 1 << (11 - RB);
}
constexpr int kNttThreads = ntt_threads<3>();

// Row-pass layout: bank bit c of word i is i_c ^ i_{c+5}.  Any window of four
// contiguous register bits holds at most one of c, c + 5.
struct SwzRow {
    static constexpr __host__ __device__ uint32_t f(uint32_t i) { return i ^ ((i >> 5) & 31u); }
    static constexpr __host__ __device__ int partner(int c) { return c + 5; }
};
// Column layout for 8-element rounds: the 128-byte TMA swizzle (16-byte chunk
// index ^= 128-byte line index mod 8); bank bits 0, 1 are i_0, i_1 and bank bit
// c >= 2 is i_c ^ i_{c+3}.  (A 4-bit register window can hold c and c + 3, so
// 16-element rounds use SwzRow.)
struct SwzCol {
    static constexpr __host__ __device__ uint32_t f(uint32_t i) { return i ^ (((i >> 5) & 7u) << 2); }
    static constexpr __host__ __device__ int partner(int c) { return c >= 2 ? c + 3 : -1; }
};

struct RoundMap {
    int lane[5];
    int warp[3];
};

template <int NSUB, int XS, class SWZ, int RB = 3>
struct Rounds {
    static_assert(RB == 3 || RB == 4, "8 or 16 elements per thread");
    static_assert(NSUB >= 6 && NSUB <= 11 && XS + NSUB <= 11, "2^6 .. 2^11-element sub-transforms");
    static constexpr int kRegs = 1 << RB;
    static constexpr int kWarpBits = 6 - RB;
    static constexpr int kCount = (NSUB + RB - 1) / RB;
    static constexpr __host__ __device__ int cnt(int r) { return (r < kCount - 1 || NSUB % RB == 0) ? RB : NSUB % RB; }
    static constexpr __host__ __device__ int lo(int r) { return NSUB - RB * r - cnt(r); }
    static constexpr __host__ __device__ bool is_reg(int r, int bit) {
        return bit >= XS + lo(r) && bit < XS + lo(r) + RB;
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
        // Lanes in ascending bit order: any order keeps the exchanges free of
        // conflicts, and this one gives the 8 lanes of a quarter-warp consecutive
        // twiddle positions y where the round's lanes differ in y.
        for (int a = 0; a < 5; ++a)
            for (int c = 0; c + 1 < 5 - a; ++c)
                if (m.lane[c] > m.lane[c + 1]) {
                    const int s = m.lane[c];
                    m.lane[c] = m.lane[c + 1];
                    m.lane[c + 1] = s;
                }
        int w = 0;
        for (int b = 0; b < 11; ++b)
            if (!used[b]) m.warp[w++] = b;
        return m;
    }
    // The 32 lanes of a warp hit 32 distinct banks in every access of round r
    // (the map is linear, so the warp bits and the register index only add a
    // common offset).
    static constexpr bool conflict_free(int r) {
        const RoundMap m = map(r);
        bool seen[32] = {};
        for (uint32_t l = 0; l < 32; ++l) {
            uint32_t i = 0;
            for (int c = 0; c < 5; ++c) i |= ((l >> c) & 1u) << m.lane[c];
            const uint32_t bank = SWZ::f(i) & 31u;
            if (seen[bank]) return false;
            seen[bank] = true;
        }
        return true;
    }
    static constexpr bool all_conflict_free() {
        for (int r = 0; r < kCount; ++r)
            if (!conflict_free(r)) return false;
        return true;
    }
};

// Register bits per round: every pass holds 16 elements per thread where that
// saves a round (sub-transforms of 2^7, 2^8, 2^10, 2^11), else 8.  (The row pass
// gains only since its twiddle tables are prebuilt: generating them in the
// block cost twice as many entries per thread with 16-element rounds.)
constexpr __host__ __device__ int col_pass_rb(int log) { return (log + 3) / 4 < (log + 2) / 3 ? 4 : 3; }
constexpr __host__ __device__ int row_pass_rb(int log) { return col_pass_rb(log); }

// Twiddle-table layout of the row pass ("round-major").  Level l of a table
// (entries [2^l, 2^(l+1)), the stage of distance 2^(NSUB-1-l)) is read in round
// l / RB, whose twiddle position y lies in [2^LY, 2^(LY+1)), at local level
// t = l - LY: entries (y << t) + i, i < 2^t.  For t >= 2 the pair {i, i + 1}
// (i even) of y is stored at 2^l + 2 ((i / 2) 2^LY + y - 2^LY), so lanes that
// differ in y read consecutive 16-byte pairs; levels with t < 2 keep entry order.
constexpr __host__ __device__ int table_ly(int nsub, int rb, int l) {
    const int r = l / rb, count = (nsub + rb - 1) / rb;
    const int cnt = (r < count - 1 || nsub % rb == 0) ? rb : nsub % rb;
    return rb * r + cnt - rb;
}

constexpr __host__ __device__ uint32_t row_table_pos(int nsub, int rb, uint32_t e) {
    int l = 0;
    while ((2u << l) <= e) ++l;
    const int ly = table_ly(nsub, rb, l), t = l - ly;
    if (t < 2) return e;
    const uint32_t j = e - (1u << l), i = j & ((1u << t) - 1u), yo = j >> t;
    return (1u << l) + (i & 1u) + 2u * (((i >> 1) << ly) + yo);
}

// Bits of the lane (5) or warp (kWarpBits) index that move by SH places.
template <int NSUB, int XS, class SWZ, int RB, int R, bool LANE>
__host__ __device__ constexpr uint32_t deposit_mask(int sh) {
    using RP = Rounds<NSUB, XS, SWZ, RB>;
    constexpr RoundMap m = RP::map(R);
    uint32_t mask = 0;
    for (int c = 0; c < (LANE ? 5 : RP::kWarpBits); ++c)
        if ((LANE ? m.lane[c] : m.warp[c]) - c == sh) mask |= 1u << c;
    return mask;
}

template <int NSUB, int XS, class SWZ, int RB, int R, bool LANE>
__device__ __forceinline__ uint32_t deposit(uint32_t x) {
    uint32_t b = 0;
#pragma unroll
    for (int sh = 0; sh <= 10; ++sh) {
        const uint32_t mask = deposit_mask<NSUB, XS, SWZ, RB, R, LANE>(sh);
        if (mask) b |= (x & mask) << sh;
    }
    return b;
}

// Logical index of element 0 of this thread in round R (lane bits and warp
// bits deposited group-wise: bits that move by the same distance move together).
template <int NSUB, int XS, class SWZ, int RB, int R>
__device__ __forceinline__ uint32_t round_base(uint32_t tid) {
    return deposit<NSUB, XS, SWZ, RB, R, true>(tid & 31u) | deposit<NSUB, XS, SWZ, RB, R, false>(tid >> 5);
}

template <int NSUB, int XS, class SWZ, int RB, int R>
__device__ __forceinline__ void load_round(const uint32_t* tile, uint32_t (&v)[1 << RB], uint32_t base) {
    constexpr int sh = XS + Rounds<NSUB, XS, SWZ, RB>::lo(R);
    const uint32_t sb = SWZ::f(base);
#pragma unroll
    for (int k = 0; k < (1 << RB); ++k) v[k] = tile[sb ^ SWZ::f(static_cast<uint32_t>(k) << sh)];
}

template <int NSUB, int XS, class SWZ, int RB, int R>
__device__ __forceinline__ void store_round(uint32_t* tile, const uint32_t (&v)[1 << RB], uint32_t base) {
    constexpr int sh = XS + Rounds<NSUB, XS, SWZ, RB>::lo(R);
    const uint32_t sb = SWZ::f(base);
#pragma unroll
    for (int k = 0; k < (1 << RB); ++k) tile[sb ^ SWZ::f(static_cast<uint32_t>(k) << sh)] = v[k];
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

// ---- twiddle sources ---------------------------------------------------------------

// A round's twiddles: level t (t < RB) holds 2^t entries at w[2^t - 1 ..].
template <int RB>
struct Tw {
    uint2 w[(1 << RB) - 1];
};

// Entries (y << t) + i, i < 2^t, of table tb into r.w[2^t - 1 + i]; REV: into
// r.w[2^t - 1 + (2^t - 1 - i)] (the reflected partner table reads backwards).
// LY >= 0: the table is round-major (row_table_pos) and y lies in
// [2^LY, 2^(LY+1)); LY < 0: entry order.
template <int RB, int T, bool REV, int LY>
__device__ __forceinline__ void tw_level(Tw<RB>& r, const uint2* tb, uint32_t y) {
    constexpr int n = 1 << T, off = n - 1;
    if constexpr (T == 0) {
        r.w[0] = tb[y];
    } else {
#pragma unroll
        for (int m = 0; m < n; m += 2) {
            const uint32_t at = (LY >= 0 && T >= 2) ? ((1u << (LY + T)) + (static_cast<uint32_t>(m) << LY) +
                                                       2u * (y - (1u << LY)))
                                                    : (y << T) + m;
            const uint4 a = *reinterpret_cast<const uint4*>(tb + at);
            r.w[off + (REV ? n - 1 - m : m)] = make_uint2(a.x, a.y);
            r.w[off + (REV ? n - 2 - m : m + 1)] = make_uint2(a.z, a.w);
        }
    }
}

// Levels RB - cnt .. RB - 1 (a short round skips its top levels).
template <int RB, bool REV, int LY, int T = 0>
__device__ __forceinline__ void tw_levels(Tw<RB>& r, const uint2* tb, uint32_t y, int cnt) {
    if constexpr (T < RB) {
        if (T >= RB - cnt) tw_level<RB, T, REV, LY>(r, tb, y);
        tw_levels<RB, REV, LY, T + 1>(r, tb, y, cnt);
    }
}

struct SharedTable {    // one table for every sub-transform, entry order (16-byte aligned)
    const uint2* t;
    template <int RB, int LY>
    __device__ __forceinline__ Tw<RB> get(uint32_t, uint32_t y, int cnt) const {
        Tw<RB> r;
        tw_levels<RB, false, -1>(r, t, y, cnt);
        return r;
    }
};

// Round-major table of sub-transform g at t + g * STRIDE entries.  REFLECT:
// read the partner table (g ^ FLIP) at the position with its low bits
// complemented, which holds the negated inverse twiddles (see ntt.cu); the
// vector order reverses.
template <int NSUB, int STRIDE, bool REFLECT, uint32_t FLIP>
struct RowTable {
    const uint2* t;
    template <int RB, int LY>
    __device__ __forceinline__ Tw<RB> get(uint32_t g, uint32_t y, int cnt) const {
        const uint2* tb = t + (REFLECT ? (g ^ FLIP) : g) * STRIDE;
        // y lies in [2^LY, 2^(LY+1)): its reflection is y ^ (2^LY - 1), and the
        // children (y << t) + i reflect to (y* << t) + 2^t - 1 - i.
        const uint32_t yy = REFLECT ? (y ^ ((1u << LY) - 1u)) : y;
        Tw<RB> r;
        tw_levels<RB, REFLECT, LY>(r, tb, yy, cnt);
        return r;
    }
};

// ---- rounds --------------------------------------------------------------------------

// Sub-transform id and the "virtual top" twiddle index y of the round.
template <int NSUB, int XS, class SWZ, int RB, int R>
__device__ __forceinline__ void round_tw_pos(uint32_t base, uint32_t& g, uint32_t& y) {
    constexpr int lo = Rounds<NSUB, XS, SWZ, RB>::lo(R);
    const uint32_t x = (base >> XS) & ((1u << NSUB) - 1u);
    g = (base & ((1u << XS) - 1u)) | ((base >> (XS + NSUB)) << XS);
    y = (1u << (NSUB - RB - lo)) | (x >> (lo + RB));
}

// Forward stages of round R on NV operands sharing the twiddles (distances
// decreasing: level t works on register bit RB - 1 - t).
template <int NSUB, int XS, class SWZ, int RB, int R, bool LAZY, int NV, class TW>
__device__ __forceinline__ void fwd_round(uint32_t (&v)[NV][1 << RB], uint32_t base, const TW& tw, uint32_t p) {
    constexpr int cnt = Rounds<NSUB, XS, SWZ, RB>::cnt(R);
    uint32_t g, y;
    round_tw_pos<NSUB, XS, SWZ, RB, R>(base, g, y);
    const Tw<RB> w = tw.template get<RB, NSUB - RB - Rounds<NSUB, XS, SWZ, RB>::lo(R)>(g, y, cnt);
#pragma unroll
    for (int t = RB - cnt; t < RB; ++t) {
        const int db = RB - 1 - t;
#pragma unroll
        for (int k = 0; k < (1 << RB); ++k) {
            if (k & (1 << db)) continue;
#pragma unroll
            for (int o = 0; o < NV; ++o)
                bf_fwd<LAZY>(v[o][k], v[o][k | (1 << db)], w.w[(1 << t) - 1 + (k >> (db + 1))], p);
        }
    }
}

// Inverse stages of round R (distances increasing).
template <int NSUB, int XS, class SWZ, int RB, int R, bool LAZY, bool NEG, class TW>
__device__ __forceinline__ void inv_round(uint32_t (&v)[1 << RB], uint32_t base, const TW& tw, uint32_t p) {
    constexpr int cnt = Rounds<NSUB, XS, SWZ, RB>::cnt(R);
    uint32_t g, y;
    round_tw_pos<NSUB, XS, SWZ, RB, R>(base, g, y);
    const Tw<RB> w = tw.template get<RB, NSUB - RB - Rounds<NSUB, XS, SWZ, RB>::lo(R)>(g, y, cnt);
#pragma unroll
    for (int t = RB - 1; t >= RB - cnt; --t) {
        const int db = RB - 1 - t;
#pragma unroll
        for (int k = 0; k < (1 << RB); ++k) {
            if (k & (1 << db)) continue;
            bf_inv<LAZY, NEG>(v[k], v[k | (1 << db)], w.w[(1 << t) - 1 + (k >> (db + 1))], p);
        }
    }
}

}  // namespace fpm
