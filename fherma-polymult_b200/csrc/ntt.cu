// Negacyclic NTT kernels: the column pass, the fused row pass (forward rows of
// both operands, pointwise product, inverse rows) and the inverse column pass of
// the four-step transform, plus a one-block-per-prime kernel for N <= 1024.
//
// Reference counterparts (Akram275/fherma-polymult): k_ntt_cols solve.cu:130-166,
// k_ntt_rows_mul solve.cu:195-233, with the stage structure of
// rns_kernels.cuh:105-174.  Here (ntt_engine.cuh):
//   * every pass keeps 16 elements per thread in registers for up to four
//     stages at a time where that saves a round (8 and three otherwise); the
//     first and last rounds read and write global memory directly, shared
//     memory carries only the exchanges between rounds;
//   * A and B share each twiddle load, a round's 7 (15) twiddles come in 3 (8)
//     vector loads; the row pass's tables are stored round-major, so those
//     loads are free of bank conflicts;
//   * the row pass uses only the FORWARD twiddle tables of its rows (prebuilt
//     once per context from two small per-prime tables and brought into
//     shared memory by bulk asynchronous copies), and pairs row u with
//     row R - 1 - u: the inverse
//     twiddle of row u at entry y is minus the forward twiddle of row R - 1 - u
//     at y with its low bits complemented (psi^(N - e) = -psi^-e), so one
//     table set serves both directions;
//   * with primes below 2^30 the butterflies are Harvey's lazy ones (values
//     below 4p forward, 2p inverse).
#include "device.cuh"
#include "group.cuh"
#include "kernels.h"
#include "ntt_engine.cuh"
#include "pdl.cuh"
#include "tc.cuh"
#include "tmap.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>

namespace fpm {

namespace {

template <int NSUB, int XS, class SWZ, int RB>
using RP = Rounds<NSUB, XS, SWZ, RB>;

// Column-pass shared layout for RB register bits.
template <int RB>
using SwzC = std::conditional_t<RB == 3, SwzCol, SwzRow>;

// The threads that own one tile: the whole block, or one 128-thread half of a
// 256-thread block (the grouped row pass of mixed geometries runs two
// 128-thread tiles per block).
struct BlockTeam {
    static __device__ __forceinline__ uint32_t tid() { return threadIdx.x; }
    static __device__ __forceinline__ void sync() { __syncthreads(); }
};
struct HalfTeam {
    static __device__ __forceinline__ uint32_t tid() { return threadIdx.x & 127u; }
    static __device__ __forceinline__ void sync() {
        asm volatile("bar.sync %0, 128;" ::"r"(1u + (threadIdx.x >> 7)) : "memory");
    }
};

// Round R through shared memory on NV tiles.
template <int NSUB, int XS, class SWZ, int RB, int R, bool LAZY, int NV, class TEAM = BlockTeam, class TW>
__device__ __forceinline__ void fwd_step(uint32_t* const (&tiles)[NV], const TW& tw, uint32_t p) {
    const uint32_t base = round_base<NSUB, XS, SWZ, RB, R>(TEAM::tid());
    uint32_t v[NV][1 << RB];
#pragma unroll
    for (int o = 0; o < NV; ++o) load_round<NSUB, XS, SWZ, RB, R>(tiles[o], v[o], base);
    fwd_round<NSUB, XS, SWZ, RB, R, LAZY, NV>(v, base, tw, p);
#pragma unroll
    for (int o = 0; o < NV; ++o) store_round<NSUB, XS, SWZ, RB, R>(tiles[o], v[o], base);
    TEAM::sync();
}

template <int NSUB, int XS, class SWZ, int RB, int R, int REND, bool LAZY, int NV, class TEAM = BlockTeam,
          class TW>
__device__ __forceinline__ void fwd_range(uint32_t* const (&tiles)[NV], const TW& tw, uint32_t p) {
    if constexpr (R < REND) {
        fwd_step<NSUB, XS, SWZ, RB, R, LAZY, NV, TEAM>(tiles, tw, p);
        fwd_range<NSUB, XS, SWZ, RB, R + 1, REND, LAZY, NV, TEAM>(tiles, tw, p);
    }
}

// Inverse rounds R, R - 1, ..., RLO through shared memory.
template <int NSUB, int XS, class SWZ, int RB, int R, int RLO, bool LAZY, bool NEG, class TEAM = BlockTeam,
          class TW>
__device__ __forceinline__ void inv_range(uint32_t* tile, const TW& tw, uint32_t p) {
    if constexpr (R >= RLO) {
        const uint32_t base = round_base<NSUB, XS, SWZ, RB, R>(TEAM::tid());
        uint32_t v[1 << RB];
        load_round<NSUB, XS, SWZ, RB, R>(tile, v, base);
        inv_round<NSUB, XS, SWZ, RB, R, LAZY, NEG>(v, base, tw, p);
        store_round<NSUB, XS, SWZ, RB, R>(tile, v, base);
        TEAM::sync();
        inv_range<NSUB, XS, SWZ, RB, R - 1, RLO, LAZY, NEG, TEAM>(tile, tw, p);
    }
}

// Canonical residue from a lazy one (< 4p).
__device__ __forceinline__ uint32_t canon4(uint32_t x, uint32_t p) {
    x = umin32(x, x - 2 * p);
    return umin32(x, x - p);
}

// ---------------------------------------------------------------------------
// Column pass: a block owns C = 2^XS adjacent columns c0 .. c0 + C - 1 of one
// prime and all R = 2^LOGR rows; tile index i = u C + c (row u = position in the
// sub-transform, column c = sub-transform).  Element (u, c) is X[u S + c0 + c].
// S = 2^LOGS is a template parameter too, so a thread's strided global
// accesses are one base address plus immediates.

template <int LOGR, int LOGS>
__device__ __forceinline__ uint32_t col_offset(uint32_t i, uint32_t c0) {
    constexpr int XS = 11 - LOGR;
    return ((i >> XS) << LOGS) + c0 + (i & ((1u << XS) - 1u));
}

template <int LOGR, int LOGS, int RB, int R, int NV>
__device__ __forceinline__ void col_global_load(const uint32_t* const (&X)[NV], uint32_t (&v)[NV][1 << RB],
                                                uint32_t base, uint32_t c0) {
    constexpr int XS = 11 - LOGR, sh = RP<LOGR, XS, SwzC<RB>, RB>::lo(R);
    constexpr uint32_t step = (1u << LOGS) << sh;
    const uint32_t at = col_offset<LOGR, LOGS>(base, c0);
#pragma unroll
    for (int o = 0; o < NV; ++o) {
        const uint32_t* x = X[o] + at;
#pragma unroll
        for (int k = 0; k < (1 << RB); ++k) v[o][k] = x[k * step];
    }
}

template <int LOGR, int LOGS, int RB, int R, int NV>
__device__ __forceinline__ void col_global_store(uint32_t* const (&X)[NV], const uint32_t (&v)[NV][1 << RB],
                                                 uint32_t base, uint32_t c0) {
    constexpr int XS = 11 - LOGR, sh = RP<LOGR, XS, SwzC<RB>, RB>::lo(R);
    constexpr uint32_t step = (1u << LOGS) << sh;
    const uint32_t at = col_offset<LOGR, LOGS>(base, c0);
#pragma unroll
    for (int o = 0; o < NV; ++o) {
        uint32_t* x = X[o] + at;
#pragma unroll
        for (int k = 0; k < (1 << RB); ++k) x[k * step] = v[o][k];
    }
}

template <int LOGR, int LOGS, bool LAZY>
__device__ __forceinline__ void col_fwd_body(const DevPoint& d, uint32_t* A, uint32_t* B, int j, uint32_t bx) {
    extern __shared__ __align__(1024) uint32_t smem[];
    constexpr int RB = col_pass_rb(LOGR), E = 1 << RB, T = ntt_threads<RB>();
    constexpr int XS = 11 - LOGR;
    using SWZ = SwzC<RB>;
    static_assert(RP<LOGR, XS, SWZ, RB>::all_conflict_free(), "column rounds must be free of bank conflicts");
    constexpr uint32_t R = 1u << LOGR, C = 1u << XS;
    constexpr int last = RP<LOGR, XS, SWZ, RB>::kCount - 1;
    uint32_t* ta = smem;
    uint32_t* tb = smem + 2048;
    uint2* tw = reinterpret_cast<uint2*>(smem + 4096);
    constexpr size_t N = size_t(1) << (LOGR + LOGS);
    const uint32_t c0 = bx * C;
    const uint32_t p = d.pc[j].p;
    uint32_t* const X[2] = {A + j * N, B + j * N};
    for (uint32_t y = threadIdx.x; y < R; y += T) tw[y] = d.col_f[static_cast<size_t>(j) * R + y];
    const SharedTable table{tw};
    uint32_t* const tiles[2] = {ta, tb};
    {
        const uint32_t base = round_base<LOGR, XS, SWZ, RB, 0>(threadIdx.x);
        uint32_t v[2][E];
        const uint32_t* const Xc[2] = {X[0], X[1]};
        col_global_load<LOGR, LOGS, RB, 0, 2>(Xc, v, base, c0);
        __syncthreads();   // the twiddle table
        fwd_round<LOGR, XS, SWZ, RB, 0, LAZY, 2>(v, base, table, p);
#pragma unroll
        for (int o = 0; o < 2; ++o) store_round<LOGR, XS, SWZ, RB, 0>(tiles[o], v[o], base);
        __syncthreads();
    }
    fwd_range<LOGR, XS, SWZ, RB, 1, last, LAZY, 2>(tiles, table, p);
    {
        const uint32_t base = round_base<LOGR, XS, SWZ, RB, last>(threadIdx.x);
        uint32_t v[2][E];
#pragma unroll
        for (int o = 0; o < 2; ++o) load_round<LOGR, XS, SWZ, RB, last>(tiles[o], v[o], base);
        fwd_round<LOGR, XS, SWZ, RB, last, LAZY, 2>(v, base, table, p);
        col_global_store<LOGR, LOGS, RB, last, 2>(X, v, base, c0);
    }
}

template <int LOGR, int LOGS, bool LAZY>
__device__ __forceinline__ void col_inv_body(const DevPoint& d, uint32_t* A, int j, uint32_t bx) {
    extern __shared__ __align__(1024) uint32_t smem[];
    constexpr int RB = col_pass_rb(LOGR), E = 1 << RB, T = ntt_threads<RB>();
    constexpr int XS = 11 - LOGR;
    using SWZ = SwzC<RB>;
    static_assert(RP<LOGR, XS, SWZ, RB>::all_conflict_free(), "column rounds must be free of bank conflicts");
    constexpr uint32_t R = 1u << LOGR, C = 1u << XS;
    constexpr int last = RP<LOGR, XS, SWZ, RB>::kCount - 1;
    uint32_t* ta = smem;
    uint2* tw = reinterpret_cast<uint2*>(smem + 2048);
    constexpr size_t N = size_t(1) << (LOGR + LOGS);
    const uint32_t c0 = bx * C;
    const uint32_t p = d.pc[j].p;
    uint32_t* const X[1] = {A + j * N};
    for (uint32_t y = threadIdx.x; y < R; y += T) tw[y] = d.col_i[static_cast<size_t>(j) * R + y];
    const SharedTable table{tw};
    {
        const uint32_t base = round_base<LOGR, XS, SWZ, RB, last>(threadIdx.x);
        uint32_t v[1][E];
        const uint32_t* const Xc[1] = {X[0]};
        col_global_load<LOGR, LOGS, RB, last, 1>(Xc, v, base, c0);
        __syncthreads();
        inv_round<LOGR, XS, SWZ, RB, last, LAZY, false>(v[0], base, table, p);
        store_round<LOGR, XS, SWZ, RB, last>(ta, v[0], base);
        __syncthreads();
    }
    inv_range<LOGR, XS, SWZ, RB, last - 1, 1, LAZY, false>(ta, table, p);
    {
        const uint32_t base = round_base<LOGR, XS, SWZ, RB, 0>(threadIdx.x);
        uint32_t v[1][E];
        load_round<LOGR, XS, SWZ, RB, 0>(ta, v[0], base);
        inv_round<LOGR, XS, SWZ, RB, 0, LAZY, false>(v[0], base, table, p);
        if constexpr (LAZY) {
#pragma unroll
            for (int k = 0; k < E; ++k) v[0][k] = reduce_once(v[0][k], p);   // y_j canonical for the CRT
        }
        col_global_store<LOGR, LOGS, RB, 0, 1>(X, v, base, c0);
    }
}

// ---------------------------------------------------------------------------
// Column passes staged through TMA (R = 64 rows: N = 2^12 .. 2^17).  With
// 8-element rounds the column tile's shared layout (SwzCol) is exactly the
// 128-byte TMA swizzle of a box of 64 rows x 32 words, so a tile arrives by
// one cp.async.bulk.tensor load per operand and leaves by one tensor store;
// the first and last rounds read and write shared memory.  The kernels are
// persistent: a CTA walks tiles t = blockIdx.x + i gridDim.x (tile t = prime
// t / per, column block t % per) through two buffers, the next tile's boxes and
// its prime's 64 twiddles (a bulk copy) landing while the current tile is
// transformed.  Tensor maps cover this GPU's own residue arrays only.

constexpr uint32_t kColTmaBox = 2048 * sizeof(uint32_t);                 // one operand's tile
constexpr uint32_t kColTmaTw = 64 * sizeof(uint2);                       // R = 64 twiddles
constexpr uint32_t kColFwdStage = 17 * 1024;                             // A, B, twiddles (1024-aligned)
constexpr uint32_t kColInvStage = 9 * 1024;                              // A, twiddles
// ST = 2: persistent, two buffers (next tile in flight); ST = 1: one tile
// per CTA, one buffer, eight CTAs per SM (other CTAs' work covers a CTA's wait).
template <int ST>
constexpr size_t col_fwd_tma_smem() { return ST * size_t(kColFwdStage) + 16; }
template <int ST>
constexpr size_t col_inv_tma_smem() { return ST * size_t(kColInvStage) + 16; }

template <int LOGS, bool FWD>
__device__ __forceinline__ void col_tma_issue(const DevPoint& d, const CUtensorMap* tmA, const CUtensorMap* tmB,
                                              uint8_t* stage, uint64_t* bar, uint32_t t) {
    constexpr uint32_t per = (1u << LOGS) / 32;
    const uint32_t j = t / per, bx = t - (t / per) * per;
    tc::mbar_arrive_expect_tx(bar, (FWD ? 2 : 1) * kColTmaBox + kColTmaTw);
    tc::tma_load_2d(stage, tmA, static_cast<int>(bx * 32), static_cast<int>(j * 64), bar);
    if constexpr (FWD) tc::tma_load_2d(stage + kColTmaBox, tmB, static_cast<int>(bx * 32), static_cast<int>(j * 64), bar);
    const uint2* tw = (FWD ? d.col_f : d.col_i) + static_cast<size_t>(j) * 64;
    tc::bulk_g2s(stage + (FWD ? 2 : 1) * kColTmaBox, tw, kColTmaTw, bar);
}

template <int LOGS, bool LAZY, int ST>
__global__ void __launch_bounds__(256, ST == 1 ? 8 : 6)
    k_ntt_col_fwd_tma(DevPoint d, const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    constexpr int LOGR = 6, XS = 5, RB = 3, E = 8;
    using SWZ = SwzCol;
    static_assert(RP<LOGR, XS, SWZ, RB>::all_conflict_free(), "column rounds must be free of bank conflicts");
    constexpr int last = RP<LOGR, XS, SWZ, RB>::kCount - 1;
    constexpr uint32_t per = (1u << LOGS) / 32;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + ST * kColFwdStage);
    const uint32_t tiles = per * static_cast<uint32_t>(d.K);
    if (threadIdx.x == 0) {
        tc::mbar_init(&full[0], 1);
        tc::mbar_init(&full[1], 1);
        tc::fence_mbar_init();
        tc::prefetch_tmap(&tmA);
        tc::prefetch_tmap(&tmB);
    }
    __syncthreads();
    pdl_launch_dependents();
    pdl_wait();
    if (threadIdx.x == 0 && blockIdx.x < tiles) col_tma_issue<LOGS, true>(d, &tmA, &tmB, smem_raw, &full[0], blockIdx.x);
    uint32_t i = 0;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++i) {
        const int s = ST == 1 ? 0 : (i & 1);
        uint8_t* stage = smem_raw + s * kColFwdStage;
        uint32_t* const tiles2[2] = {reinterpret_cast<uint32_t*>(stage), reinterpret_cast<uint32_t*>(stage + kColTmaBox)};
        const SharedTable table{reinterpret_cast<const uint2*>(stage + 2 * kColTmaBox)};
        const uint32_t j = t / per;
        const uint32_t p = d.pc[j].p;
        if (!tc::wait_parity(&full[s], (ST == 1 ? i : i >> 1) & 1, d.wait_ns) && threadIdx.x == 0)
            atomicOr(d.err, 4u);
        {
            const uint32_t base = round_base<LOGR, XS, SWZ, RB, 0>(threadIdx.x);
            uint32_t v[2][E];
#pragma unroll
            for (int o = 0; o < 2; ++o) load_round<LOGR, XS, SWZ, RB, 0>(tiles2[o], v[o], base);
            fwd_round<LOGR, XS, SWZ, RB, 0, LAZY, 2>(v, base, table, p);
#pragma unroll
            for (int o = 0; o < 2; ++o) store_round<LOGR, XS, SWZ, RB, 0>(tiles2[o], v[o], base);
            __syncthreads();
        }
        // The next tile's loads, into the other buffer once the stores of the
        // tile that used it have read it.
        if (ST == 2 && threadIdx.x == 0 && t + gridDim.x < tiles) {
            tc::bulk_wait_read();
            col_tma_issue<LOGS, true>(d, &tmA, &tmB, smem_raw + (s ^ 1) * kColFwdStage, &full[s ^ 1], t + gridDim.x);
        }
        fwd_range<LOGR, XS, SWZ, RB, 1, last, LAZY, 2>(tiles2, table, p);
        {
            const uint32_t base = round_base<LOGR, XS, SWZ, RB, last>(threadIdx.x);
            uint32_t v[2][E];
#pragma unroll
            for (int o = 0; o < 2; ++o) load_round<LOGR, XS, SWZ, RB, last>(tiles2[o], v[o], base);
            fwd_round<LOGR, XS, SWZ, RB, last, LAZY, 2>(v, base, table, p);
#pragma unroll
            for (int o = 0; o < 2; ++o) store_round<LOGR, XS, SWZ, RB, last>(tiles2[o], v[o], base);
        }
        tc::fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t bx = t - j * per;
            tc::tma_store_2d(&tmA, tiles2[0], static_cast<int>(bx * 32), static_cast<int>(j * 64));
            tc::tma_store_2d(&tmB, tiles2[1], static_cast<int>(bx * 32), static_cast<int>(j * 64));
            tc::bulk_commit();
        }
    }
    // The stores must have read shared memory before the CTA exits; their
    // writes complete with the grid.
    if (threadIdx.x == 0) tc::bulk_wait_read();
}

template <int LOGS, bool LAZY, int ST>
__global__ void __launch_bounds__(256, 8) k_ntt_col_inv_tma(DevPoint d, const __grid_constant__ CUtensorMap tmA) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    constexpr int LOGR = 6, XS = 5, RB = 3, E = 8;
    using SWZ = SwzCol;
    static_assert(RP<LOGR, XS, SWZ, RB>::all_conflict_free(), "column rounds must be free of bank conflicts");
    constexpr int last = RP<LOGR, XS, SWZ, RB>::kCount - 1;
    constexpr uint32_t per = (1u << LOGS) / 32;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + ST * kColInvStage);
    const uint32_t tiles = per * static_cast<uint32_t>(d.K);
    if (threadIdx.x == 0) {
        tc::mbar_init(&full[0], 1);
        tc::mbar_init(&full[1], 1);
        tc::fence_mbar_init();
        tc::prefetch_tmap(&tmA);
    }
    __syncthreads();
    pdl_launch_dependents();
    pdl_wait();
    if (threadIdx.x == 0 && blockIdx.x < tiles) col_tma_issue<LOGS, false>(d, &tmA, &tmA, smem_raw, &full[0], blockIdx.x);
    uint32_t i = 0;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++i) {
        const int s = ST == 1 ? 0 : (i & 1);
        uint8_t* stage = smem_raw + s * kColInvStage;
        uint32_t* ta = reinterpret_cast<uint32_t*>(stage);
        const SharedTable table{reinterpret_cast<const uint2*>(stage + kColTmaBox)};
        const uint32_t j = t / per;
        const uint32_t p = d.pc[j].p;
        if (!tc::wait_parity(&full[s], (ST == 1 ? i : i >> 1) & 1, d.wait_ns) && threadIdx.x == 0)
            atomicOr(d.err, 4u);
        {
            const uint32_t base = round_base<LOGR, XS, SWZ, RB, last>(threadIdx.x);
            uint32_t v[E];
            load_round<LOGR, XS, SWZ, RB, last>(ta, v, base);
            inv_round<LOGR, XS, SWZ, RB, last, LAZY, false>(v, base, table, p);
            store_round<LOGR, XS, SWZ, RB, last>(ta, v, base);
            __syncthreads();
        }
        if (ST == 2 && threadIdx.x == 0 && t + gridDim.x < tiles) {
            tc::bulk_wait_read();
            col_tma_issue<LOGS, false>(d, &tmA, &tmA, smem_raw + (s ^ 1) * kColInvStage, &full[s ^ 1], t + gridDim.x);
        }
        inv_range<LOGR, XS, SWZ, RB, last - 1, 1, LAZY, false>(ta, table, p);
        {
            const uint32_t base = round_base<LOGR, XS, SWZ, RB, 0>(threadIdx.x);
            uint32_t v[E];
            load_round<LOGR, XS, SWZ, RB, 0>(ta, v, base);
            inv_round<LOGR, XS, SWZ, RB, 0, LAZY, false>(v, base, table, p);
            if constexpr (LAZY) {
#pragma unroll
                for (int k = 0; k < E; ++k) v[k] = reduce_once(v[k], p);   // y_j canonical for the CRT
            }
            store_round<LOGR, XS, SWZ, RB, 0>(ta, v, base);
        }
        tc::fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t bx = t - j * per;
            tc::tma_store_2d(&tmA, ta, static_cast<int>(bx * 32), static_cast<int>(j * 64));
            tc::bulk_commit();
        }
    }
    // The stores must have read shared memory before the CTA exits; their
    // writes complete with the grid.
    if (threadIdx.x == 0) tc::bulk_wait_read();
}

// ---------------------------------------------------------------------------
// Row pass.  A block owns G = 2048 / S rows of one prime: tile row g < G/2 is
// row u0 + g, tile row g >= G/2 is row R - 1 - u0 - (g - G/2), so rows g and
// g ^ G/2 are partners (u, R - 1 - u).  With G = 1 (S = 2048) the block owns one
// row and builds its partner's table beside its own.
//
// Forward table of row u, entry y in [2^lev, 2^(lev+1)), stage b = LOGS-1-lev:
// psi^(2^b (1 + 2 bitrev(u)) + 2^(b+1+logR) bitrev(y - 2^lev)) = U[u][b] Q[y].
// Tables are round-major: position row_table_pos(y) holds entry y, and the
// plan stores Q in the same order, so position p is U[u][b(p)] Q'[p] with the
// level of p equal to that of y.  k_row_tables builds every row's table once
// per context (K x R x S pairs); a row block copies its rows' tables into
// shared memory asynchronously.

template <int LOGS>
struct RowGeom {
    static constexpr uint32_t S = 1u << LOGS;
    static constexpr uint32_t G = 2048u >> LOGS;
    static constexpr uint32_t kSlots = G >= 2 ? G : 2;
    static constexpr uint32_t kStride = S + 4;                 // entries; pads rows across banks
    static constexpr uint32_t kFlip = G >= 2 ? G / 2 : 1;
    static constexpr uint32_t kPairsPerBlock = G >= 2 ? G / 2 : 1;
};

template <int LOGS>
__device__ __forceinline__ uint32_t row_of_slot(uint32_t slot, uint32_t u0, uint32_t R) {
    using RG = RowGeom<LOGS>;
    if constexpr (RG::G >= 2) {
        return slot < RG::G / 2 ? u0 + slot : R - 1 - u0 - (slot - RG::G / 2);
    } else {
        return slot == 0 ? u0 : R - 1 - u0;
    }
}

// Copies the block's row tables (slot s holds row row_of_slot(s)) from the
// prebuilt K x R x S array into shared memory with bulk asynchronous copies
// (one per row table, S Shoup pairs, issued by the lanes of warp 0), counted
// on the mbarrier `bar`, which the caller waits on (phase parity `phase`)
// before its first twiddle read.  Called by warp 0 only.
template <int LOGS>
__device__ __forceinline__ void row_tables_bulk(uint2* tf, const DevPoint& d, int j, uint32_t u0, uint64_t* bar) {
    using RG = RowGeom<LOGS>;
    const uint32_t R = 1u << d.logR;
    constexpr uint32_t kBytes = RG::S * sizeof(uint2);
    const int lane = threadIdx.x & 31;
    if (lane == 0) tc::mbar_arrive_expect_tx(bar, RG::kSlots * kBytes);
    __syncwarp();
    for (uint32_t slot = lane; slot < RG::kSlots; slot += 32) {
        const uint32_t u = row_of_slot<LOGS>(slot, u0, R);
        tc::bulk_g2s(tf + slot * RG::kStride, d.row_tw + (static_cast<size_t>(j) * R + u) * RG::S, kBytes, bar);
    }
}

// One row's forward table, position p (round-major): U[u][b(p)] Q'[p] with its
// Shoup companion, where the plan stores Q' in the same order and b(p) =
// LOGS - 1 - level(p).  Position 0 is unused.
__global__ void __launch_bounds__(256) k_row_tables(DevPoint d, uint2* out) {
    const int j = blockIdx.y;
    const uint32_t u = blockIdx.x, logS = d.logS, S = 1u << logS, R = 1u << d.logR;
    const PrimeConsts pc = d.pc[j];
    const uint2* qf = d.row_q_f + static_cast<size_t>(j) * S;
    const uint2* uf = d.row_u_f + (static_cast<size_t>(j) * R + u) * logS;
    uint2* o = out + (static_cast<size_t>(j) * R + u) * S;
    for (uint32_t p = threadIdx.x; p < S; p += blockDim.x) {
        if (p == 0) {
            o[0] = make_uint2(0, 0);
            continue;
        }
        const uint32_t b = logS - 1 - (31 - __clz(p));
        const uint2 f = uf[b], q1 = qf[p];
        o[p] = make_twiddle(shoup(f.x, q1.x, q1.y, pc.p), pc);
    }
}

template <int LOGS>
__device__ __forceinline__ size_t row_offset(uint32_t i, uint32_t u0, uint32_t R) {
    return static_cast<size_t>(row_of_slot<LOGS>(i >> LOGS, u0, R)) * (1u << LOGS) + (i & ((1u << LOGS) - 1u));
}

// The row pass's tables barrier sits after the tiles and the tables.
template <int LOGS>
constexpr size_t row_bar_offset() {
    return 2 * 2048 * sizeof(uint32_t) + RowGeom<LOGS>::kSlots * RowGeom<LOGS>::kStride * sizeof(uint2);
}

// phase: parity of this tile's use of the tables barrier (the block's tile
// count so far, mod 2); the barrier is initialised by the kernel.
// smem: this team's region (row_smem_t<LOGS>() bytes, 1024-byte aligned);
// tbar: its tables barrier (initialised, count 1).
template <int LOGS, bool LAZY, class TEAM = BlockTeam>
__device__ __forceinline__ void row_body(const DevPoint& d, uint32_t* A, uint32_t* B, int mode, int j, uint32_t bx,
                                         uint32_t phase, uint32_t* smem, uint64_t* tbar) {
    using RG = RowGeom<LOGS>;
    constexpr int RB = row_pass_rb(LOGS), E = 1 << RB, T = ntt_threads<RB>();
    using RPR = RP<LOGS, 0, SwzRow, RB>;
    static_assert(RPR::all_conflict_free(), "row rounds must be free of bank conflicts");
    constexpr int last = RPR::kCount - 1;
    uint32_t* ta = smem;
    uint32_t* tb = smem + 2048;
    uint2* tf = reinterpret_cast<uint2*>(smem + 4096);
    const uint32_t u0 = bx * RG::kPairsPerBlock;
    const uint32_t R = 1u << d.logR;
    const PrimeConsts pc = d.pc[j];
    const uint32_t p = pc.p;
    uint32_t* a = A + static_cast<size_t>(j) * d.N;
    uint32_t* b = B + static_cast<size_t>(j) * d.N;
    const RowTable<LOGS, RG::kStride, false, RG::kFlip> fw{tf};
    const RowTable<LOGS, RG::kStride, true, RG::kFlip> iw{tf};
    uint32_t* const tiles[2] = {ta, tb};

    // The tables stream into shared memory while round 0 loads its elements.
    if (TEAM::tid() < 32) row_tables_bulk<LOGS>(tf, d, j, u0, tbar);
    // Round 0 straight from global memory (the thread's E elements lie in one
    // row).
    {
        const uint32_t base = round_base<LOGS, 0, SwzRow, RB, 0>(TEAM::tid());
        constexpr int sh = RPR::lo(0);
        uint32_t v[2][E];
        const size_t at = row_offset<LOGS>(base, u0, R);
#pragma unroll
        for (int k = 0; k < E; ++k) {
            v[0][k] = a[at + (k << sh)];
            v[1][k] = b[at + (k << sh)];
        }
        // The bound only guards against a copy that never lands: past it the
        // error word gets bit 2 and the block goes on (with wrong twiddles).
        if (!tc::wait_parity(tbar, phase, d.wait_ns) && (TEAM::tid() & 31) == 0) atomicOr(d.err, 4u);
        fwd_round<LOGS, 0, SwzRow, RB, 0, LAZY, 2>(v, base, fw, p);
#pragma unroll
        for (int o = 0; o < 2; ++o) store_round<LOGS, 0, SwzRow, RB, 0>(tiles[o], v[o], base);
        TEAM::sync();
    }
    fwd_range<LOGS, 0, SwzRow, RB, 1, last, LAZY, 2, TEAM>(tiles, fw, p);
    // Last forward round, the pointwise product and the first inverse round in
    // registers.
    {
        const uint32_t base = round_base<LOGS, 0, SwzRow, RB, last>(TEAM::tid());
        uint32_t v[2][E];
        load_round<LOGS, 0, SwzRow, RB, last>(ta, v[0], base);
        load_round<LOGS, 0, SwzRow, RB, last>(tb, v[1], base);
        fwd_round<LOGS, 0, SwzRow, RB, last, LAZY, 2>(v, base, fw, p);
        if (mode == kRowForward) {
            if constexpr (LAZY) {
#pragma unroll
                for (int k = 0; k < E; ++k) {
                    v[0][k] = canon4(v[0][k], p);
                    v[1][k] = canon4(v[1][k], p);
                }
            }
            store_round<LOGS, 0, SwzRow, RB, last>(ta, v[0], base);
            store_round<LOGS, 0, SwzRow, RB, last>(tb, v[1], base);
            TEAM::sync();
            for (uint32_t i = TEAM::tid(); i < 2048; i += T) {
                const size_t at = row_offset<LOGS>(i, u0, R);
                a[at] = ta[SwzRow::f(i)];
                b[at] = tb[SwzRow::f(i)];
            }
            return;
        }
#pragma unroll
        for (int k = 0; k < E; ++k) {
            uint32_t x = v[0][k], y = v[1][k];
            if constexpr (LAZY) {
                // below 2p each, so the Montgomery product stays below 2p
                x = umin32(x, x - 2 * p);
                y = umin32(y, y - 2 * p);
            }
            v[0][k] = mont_mul(x, y, p, pc.pneg);
        }
        inv_round<LOGS, 0, SwzRow, RB, last, LAZY, true>(v[0], base, iw, p);
        store_round<LOGS, 0, SwzRow, RB, last>(ta, v[0], base);
        TEAM::sync();
    }
    inv_range<LOGS, 0, SwzRow, RB, last - 1, 1, LAZY, true, TEAM>(ta, iw, p);
    // Inverse round 0 straight to global memory.
    {
        const uint32_t base = round_base<LOGS, 0, SwzRow, RB, 0>(TEAM::tid());
        constexpr int sh = RPR::lo(0);
        uint32_t v[E];
        load_round<LOGS, 0, SwzRow, RB, 0>(ta, v, base);
        inv_round<LOGS, 0, SwzRow, RB, 0, LAZY, true>(v, base, iw, p);
        if (LAZY && d.logR == 0) {
            // No column pass follows: these are the y_j, canonical for the CRT.
#pragma unroll
            for (int k = 0; k < E; ++k) v[k] = reduce_once(v[k], p);
        }
        const size_t at = row_offset<LOGS>(base, u0, R);
#pragma unroll
        for (int k = 0; k < E; ++k) a[at + (k << sh)] = v[k];
    }
}

// Threads of each pass, and the resident blocks per SM that the column
// kernels' registers are sized for: 8-element rounds MIN8 blocks of 256
// threads, 16-element rounds 8 blocks of 128 (64 registers, measured fastest
// against 80 and 128).
template <int LOGR>
constexpr int col_threads() {
    return ntt_threads<col_pass_rb(LOGR)>();
}
template <int LOGS>
constexpr int row_threads() {
    return ntt_threads<row_pass_rb(LOGS)>();
}
template <int LOGR, int MIN8>
constexpr int col_min_blocks() {
    return col_pass_rb(LOGR) == 3 ? MIN8 : 8;
}
// Row kernels: five blocks of 256 threads (8-element rounds, 48 registers), or
// five of 128 (16-element rounds, up to 96 registers).  At N = 65536 (K = 139)
// the 16-element row pass measured 54.9 us with five blocks per SM against
// 56.4 with six (80 registers) and 54.5 with four; 64 registers spill.
template <int LOGS>
constexpr int row_min_blocks() {
    return 5;
}

// Blocks per prime of each pass.
template <int LOGR>
__host__ __device__ constexpr uint32_t col_blocks(uint32_t logS) {
    return (1u << logS) >> (11 - LOGR);
}

template <int LOGS>
__host__ __device__ __forceinline__ uint32_t row_blocks(uint32_t logR) {
    using RG = RowGeom<LOGS>;
    return RG::G >= 2 ? (1u << logR) / RG::G : (1u << logR);
}

// Plain launches: grid (blocks per prime, K).
template <int LOGR, int LOGS, bool LAZY>
__global__ void __launch_bounds__(col_threads<LOGR>(), (col_min_blocks<LOGR, 6>()))
    k_ntt_col_fwd(DevPoint d, uint32_t* A, uint32_t* B) {
    pdl_launch_dependents();
    pdl_wait();
    col_fwd_body<LOGR, LOGS, LAZY>(d, A, B, blockIdx.y, blockIdx.x);
}

template <int LOGR, int LOGS, bool LAZY>
__global__ void __launch_bounds__(col_threads<LOGR>(), (col_min_blocks<LOGR, 6>()))
    k_ntt_col_inv(DevPoint d, uint32_t* A) {
    pdl_launch_dependents();
    pdl_wait();
    col_inv_body<LOGR, LOGS, LAZY>(d, A, blockIdx.y, blockIdx.x);
}

template <int LOGS, bool LAZY>
__global__ void __launch_bounds__(row_threads<LOGS>(), (row_min_blocks<LOGS>())) k_ntt_row(DevPoint d, uint32_t* A, uint32_t* B, int mode) {
    extern __shared__ __align__(1024) uint32_t smem[];
    uint64_t* tbar = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(smem) + row_bar_offset<LOGS>());
    if (threadIdx.x == 0) {
        tc::mbar_init(tbar, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    pdl_launch_dependents();
    pdl_wait();
    row_body<LOGS, LAZY, BlockTeam>(d, A, B, mode, blockIdx.y, blockIdx.x, 0, smem, tbar);
}

// Grouped launches over products of one geometry class: a (possibly
// persistent) 1-D grid walks the table's blocks; block b of item i is prime
// j0 + local / per, tile local % per (an item is a group of one product's
// primes).
template <int LOGR, int LOGS, bool LAZY>
__global__ void __launch_bounds__(col_threads<LOGR>(), (col_min_blocks<LOGR, 6>()))
    k_ntt_col_fwd_group(const __grid_constant__ GroupTable t) {
    constexpr uint32_t per = col_blocks<LOGR>(LOGS);
    for (uint32_t b = blockIdx.x; b < t.total; b += gridDim.x) {
        if (b != blockIdx.x) __syncthreads();   // the previous tile's shared memory
        const uint32_t i = group_locate(t, b);
        const GroupItem& it = t.item[i];
        const uint32_t local = b - t.first[i];
        col_fwd_body<LOGR, LOGS, LAZY>(it.d, it.A, it.B, it.j0 + local / per, local % per);
    }
}

template <int LOGR, int LOGS, bool LAZY>
__global__ void __launch_bounds__(col_threads<LOGR>(), (col_min_blocks<LOGR, 6>()))
    k_ntt_col_inv_group(const __grid_constant__ GroupTable t) {
    constexpr uint32_t per = col_blocks<LOGR>(LOGS);
    for (uint32_t b = blockIdx.x; b < t.total; b += gridDim.x) {
        if (b != blockIdx.x) __syncthreads();
        const uint32_t i = group_locate(t, b);
        const GroupItem& it = t.item[i];
        const uint32_t local = b - t.first[i];
        col_inv_body<LOGR, LOGS, LAZY>(it.d, it.A, it.j0 + local / per, local % per);
    }
}

template <int LOGS, bool LAZY>
__global__ void __launch_bounds__(row_threads<LOGS>(), (row_min_blocks<LOGS>())) k_ntt_row_group(const __grid_constant__ GroupTable t) {
    extern __shared__ __align__(1024) uint32_t smem[];
    uint64_t* tbar = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(smem) + row_bar_offset<LOGS>());
    if (threadIdx.x == 0) {
        tc::mbar_init(tbar, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    uint32_t n = 0;
    for (uint32_t b = blockIdx.x; b < t.total; b += gridDim.x, ++n) {
        if (b != blockIdx.x) __syncthreads();
        const uint32_t i = group_locate(t, b);
        const GroupItem& it = t.item[i];
        const uint32_t local = b - t.first[i], per = row_blocks<LOGS>(it.d.logR);
        row_body<LOGS, LAZY>(it.d, it.A, it.B, kRowProduct, it.j0 + local / per, local % per, n & 1, smem, tbar);
    }
}

// ---------------------------------------------------------------------------
// Grouped passes over products of mixed row lengths (every item R = 64:
// N = 2^12 .. 2^17, one prime window): one launch per pass for a whole batch.
// The column passes switch on the item's row length; the row pass runs
// 256-thread blocks, one tile per block for 8-element rounds and two
// 128-thread tiles per block (HalfTeam, named barriers, a shared-memory region
// and tables barrier each) for 16-element rounds.

template <class F>
__device__ __forceinline__ void with_row_log(uint32_t logS, F&& f) {
    switch (logS) {
        case 6: f(std::integral_constant<int, 6>{}); break;
        case 7: f(std::integral_constant<int, 7>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 9: f(std::integral_constant<int, 9>{}); break;
        case 10: f(std::integral_constant<int, 10>{}); break;
        default: f(std::integral_constant<int, 11>{}); break;
    }
}

template <bool LAZY>
__global__ void __launch_bounds__(256, 6) k_ntt_col_fwd_mixed(const __grid_constant__ GroupTable t) {
    for (uint32_t b = blockIdx.x; b < t.total; b += gridDim.x) {
        if (b != blockIdx.x) __syncthreads();
        const uint32_t i = group_locate(t, b);
        const GroupItem& it = t.item[i];
        const uint32_t local = b - t.first[i], per = (1u << it.d.logS) >> 5;
        with_row_log(it.d.logS, [&](auto ls) {
            col_fwd_body<6, decltype(ls)::value, LAZY>(it.d, it.A, it.B, it.j0 + local / per, local % per);
        });
    }
}

template <bool LAZY>
__global__ void __launch_bounds__(256, 6) k_ntt_col_inv_mixed(const __grid_constant__ GroupTable t) {
    for (uint32_t b = blockIdx.x; b < t.total; b += gridDim.x) {
        if (b != blockIdx.x) __syncthreads();
        const uint32_t i = group_locate(t, b);
        const GroupItem& it = t.item[i];
        const uint32_t local = b - t.first[i], per = (1u << it.d.logS) >> 5;
        with_row_log(it.d.logS, [&](auto ls) {
            col_inv_body<6, decltype(ls)::value, LAZY>(it.d, it.A, it.j0 + local / per, local % per);
        });
    }
}

// Shared memory: two regions of `region` bytes, each ending in its tables
// barrier.  Block b of item i: tile local(b) (one per block) or tiles
// 2 local(b) + half (two per block), tile = (prime, row block).
template <bool LAZY>
__global__ void __launch_bounds__(256, 3) k_ntt_row_mixed(const __grid_constant__ GroupTable t, uint32_t region) {
    extern __shared__ __align__(1024) uint32_t smem[];
    uint8_t* base = reinterpret_cast<uint8_t*>(smem);
    uint64_t* tbar[2] = {reinterpret_cast<uint64_t*>(base + region - 16),
                         reinterpret_cast<uint64_t*>(base + 2 * region - 16)};
    if (threadIdx.x == 0) {
        tc::mbar_init(tbar[0], 1);
        tc::mbar_init(tbar[1], 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    uint32_t uses[2] = {0, 0};   // every thread counts both regions' uses
    const uint32_t half = threadIdx.x >> 7;
    for (uint32_t b = blockIdx.x; b < t.total; b += gridDim.x) {
        if (b != blockIdx.x) __syncthreads();
        const uint32_t i = group_locate(t, b);
        const GroupItem& it = t.item[i];
        const uint32_t local = b - t.first[i];
        with_row_log(it.d.logS, [&](auto ls) {
            constexpr int LS = decltype(ls)::value;
            const uint32_t per = row_blocks<LS>(6);
            if constexpr (row_threads<LS>() == 256) {
                row_body<LS, LAZY, BlockTeam>(it.d, it.A, it.B, kRowProduct, it.j0 + local / per, local % per,
                                              uses[0] & 1, smem, tbar[0]);
                ++uses[0];
            } else {
                const uint32_t tile = 2 * local + half;
                row_body<LS, LAZY, HalfTeam>(it.d, it.A, it.B, kRowProduct, it.j0 + tile / per, tile % per,
                                             uses[half] & 1, reinterpret_cast<uint32_t*>(base + half * region),
                                             tbar[half]);
                ++uses[0];
                ++uses[1];
            }
        });
    }
}

// ---------------------------------------------------------------------------
// N <= 1024: one block per prime holds both operands; one butterfly per
// thread per stage, full twiddle tables from global memory, full reduction.

__global__ void __launch_bounds__(kNttThreads) k_ntt_small(DevPoint d, uint32_t* A, uint32_t* B, int mode) {
    extern __shared__ __align__(1024) uint32_t smem[];
    const uint32_t N = d.N, logN = d.logN;
    uint32_t* ta = smem;
    uint32_t* tb = smem + N;
    const int j = blockIdx.x;
    const PrimeConsts pc = d.pc[j];
    const uint2* tf = d.full_f + static_cast<size_t>(j) * N;
    const uint2* ti = d.full_i + static_cast<size_t>(j) * N;
    uint32_t* a = A + static_cast<size_t>(j) * N;
    uint32_t* b = B + static_cast<size_t>(j) * N;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
        ta[i] = a[i];
        tb[i] = b[i];
    }
    __syncthreads();
    for (int s = static_cast<int>(logN) - 1; s >= 0; --s) {
        for (uint32_t bf = threadIdx.x; bf < N / 2; bf += blockDim.x) {
            const uint32_t i = bf >> s, lo = (i << (s + 1)) | (bf & ((1u << s) - 1)), hi = lo + (1u << s);
            const uint2 w = tf[(N >> (s + 1)) + i];
            ct_butterfly(ta[lo], ta[hi], w, pc.p);
            ct_butterfly(tb[lo], tb[hi], w, pc.p);
        }
        __syncthreads();
    }
    if (mode == kRowForward) {
        for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
            a[i] = ta[i];
            b[i] = tb[i];
        }
        return;
    }
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) ta[i] = mont_mul(ta[i], tb[i], pc.p, pc.pneg);
    __syncthreads();
    for (uint32_t s = 0; s < logN; ++s) {
        for (uint32_t bf = threadIdx.x; bf < N / 2; bf += blockDim.x) {
            const uint32_t i = bf >> s, lo = (i << (s + 1)) | (bf & ((1u << s) - 1)), hi = lo + (1u << s);
            gs_butterfly(ta[lo], ta[hi], ti[(N >> (s + 1)) + i], pc.p);
        }
        __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) a[i] = ta[i];
}

size_t col_fwd_smem_t(uint32_t logR) { return 2 * 2048 * sizeof(uint32_t) + (size_t(1) << logR) * sizeof(uint2); }
size_t col_inv_smem_t(uint32_t logR) { return 2048 * sizeof(uint32_t) + (size_t(1) << logR) * sizeof(uint2); }

template <int LOGS>
constexpr size_t row_smem_t() {
    return row_bar_offset<LOGS>() + 16;
}

template <int LOGR, int LOGS, bool LAZY>
void col_attrs() {
    const int fwd = static_cast<int>(col_fwd_smem_t(LOGR)), inv = static_cast<int>(col_inv_smem_t(LOGR));
    check(cudaFuncSetAttribute(k_ntt_col_fwd<LOGR, LOGS, LAZY>, cudaFuncAttributeMaxDynamicSharedMemorySize, fwd),
          "col smem");
    check(cudaFuncSetAttribute(k_ntt_col_inv<LOGR, LOGS, LAZY>, cudaFuncAttributeMaxDynamicSharedMemorySize, inv),
          "col smem");
    check(cudaFuncSetAttribute(k_ntt_col_fwd_group<LOGR, LOGS, LAZY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               fwd),
          "col smem");
    check(cudaFuncSetAttribute(k_ntt_col_inv_group<LOGR, LOGS, LAZY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               inv),
          "col smem");
}

template <int LOGS, bool LAZY>
void row_attrs() {
    const int bytes = static_cast<int>(row_smem_t<LOGS>());
    check(cudaFuncSetAttribute(k_ntt_row<LOGS, LAZY>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
          "row smem");
    check(cudaFuncSetAttribute(k_ntt_row_group<LOGS, LAZY>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
          "row smem");
}

// Calls f(std::integral_constant<int, V>) for V = v in [6, 11].
template <class F>
void with_log(uint32_t v, F&& f) {
    switch (v) {
        case 6: f(std::integral_constant<int, 6>{}); break;
        case 7: f(std::integral_constant<int, 7>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 9: f(std::integral_constant<int, 9>{}); break;
        case 10: f(std::integral_constant<int, 10>{}); break;
        case 11: f(std::integral_constant<int, 11>{}); break;
        default: throw std::runtime_error("unsupported transform geometry");
    }
}

// Calls f(integral_constant LOGR, integral_constant LOGS) for a four-step
// geometry (make_geometry): LOGR = 6 with LOGS in [6, 11], or LOGS = 11 with
// LOGR in [7, 11].
template <class F>
void with_cols(uint32_t logR, uint32_t logS, F&& f) {
    if (logR == 6) {
        with_log(logS, [&](auto s) { f(std::integral_constant<int, 6>{}, s); });
    } else if (logS == 11) {
        with_log(logR, [&](auto r) { f(r, std::integral_constant<int, 11>{}); });
    } else {
        throw std::runtime_error("unsupported transform geometry");
    }
}

// One grouped pass: the kernel, its shared memory, and (occupancy) its
// resident blocks per SM.
template <bool LAZY>
void group_pass(const GroupTable* t, int pass, uint32_t logR, uint32_t logS, uint32_t grid, cudaStream_t st,
                int* occupancy) {
    auto run = [&](auto kernel, int threads, size_t smem) {
        if (occupancy) {
            check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy, kernel, threads, smem), "occupancy");
        } else {
            kernel<<<grid, threads, smem, st>>>(*t);
        }
    };
    if (pass == kPassColFwd) {
        with_cols(logR, logS, [&](auto r, auto s) {
            constexpr int LR = decltype(r)::value, LS = decltype(s)::value;
            run(k_ntt_col_fwd_group<LR, LS, LAZY>, col_threads<LR>(), col_fwd_smem_t(LR));
        });
    } else if (pass == kPassColInv) {
        with_cols(logR, logS, [&](auto r, auto s) {
            constexpr int LR = decltype(r)::value, LS = decltype(s)::value;
            run(k_ntt_col_inv_group<LR, LS, LAZY>, col_threads<LR>(), col_inv_smem_t(LR));
        });
    } else if (pass == kPassRow) {
        with_log(logS, [&](auto c) {
            constexpr int L = decltype(c)::value;
            run(k_ntt_row_group<L, LAZY>, row_threads<L>(), row_smem_t<L>());
        });
    } else {
        throw std::runtime_error("grouped transform: unknown pass");
    }
}

template <int LOGS, bool LAZY>
void col_tma_attrs() {
    check(cudaFuncSetAttribute(k_ntt_col_fwd_tma<LOGS, LAZY, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(col_fwd_tma_smem<1>())),
          "col smem");
    check(cudaFuncSetAttribute(k_ntt_col_inv_tma<LOGS, LAZY, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(col_inv_tma_smem<1>())),
          "col smem");
    check(cudaFuncSetAttribute(k_ntt_col_fwd_tma<LOGS, LAZY, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(col_fwd_tma_smem<2>())),
          "col smem");
    check(cudaFuncSetAttribute(k_ntt_col_inv_tma<LOGS, LAZY, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(col_inv_tma_smem<2>())),
          "col smem");
}

template <bool LAZY>
void attrs_all() {
    col_tma_attrs<6, LAZY>();
    col_tma_attrs<7, LAZY>();
    col_tma_attrs<8, LAZY>();
    col_tma_attrs<9, LAZY>();
    col_tma_attrs<10, LAZY>();
    col_tma_attrs<11, LAZY>();
    for (uint32_t s = 6; s <= 11; ++s)
        with_cols(6, s, [&](auto lr, auto ls) { col_attrs<decltype(lr)::value, decltype(ls)::value, LAZY>(); });
    for (uint32_t r = 7; r <= 11; ++r)
        with_cols(r, 11, [&](auto lr, auto ls) { col_attrs<decltype(lr)::value, decltype(ls)::value, LAZY>(); });
    row_attrs<6, LAZY>();
    row_attrs<7, LAZY>();
    row_attrs<8, LAZY>();
    row_attrs<9, LAZY>();
    row_attrs<10, LAZY>();
    row_attrs<11, LAZY>();
}

// SMs of the current device (the persistent column grids take one slot per
// resident CTA).
int device_sms() {
    static int cached[64] = {};
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) check(cudaDeviceGetAttribute(&cached[dev], cudaDevAttrMultiProcessorCount, dev), "SM count");
    return cached[dev];
}

// The TMA column passes take R = 64 and 16-byte aligned residue arrays.
bool col_tma_ok(const DevPoint& d, const uint32_t* A, const uint32_t* B) {
    return d.logR == 6 && d.logS >= 6 && d.logS <= 11 && (reinterpret_cast<uintptr_t>(A) & 15) == 0 &&
           (reinterpret_cast<uintptr_t>(B) & 15) == 0;
}

// The residues K x N viewed as K R rows of S words.
CUtensorMap col_tmap(const DevPoint& d, const uint32_t* X) {
    return make_tmap_u32(X, static_cast<uint64_t>(d.K) << 6, d.N >> 6, d.N >> 6, 64, 32, TmaSwizzle::k128B);
}

// Column-pass variant: FPM_COL_PASS = plain (per-thread loads and stores;
// the default, measured fastest: at N = 65536, K = 139 the forward and
// inverse passes take 21.8 and 13.2 us against 23.5 and 14.0 for tma1 and
// 25.4 and 14.3 for tma2), tma1 (TMA, one tile per CTA) or tma2 (TMA,
// persistent, two buffers), read once.
int col_pass_variant() {
    static const int v = [] {
        const char* e = std::getenv("FPM_COL_PASS");
        if (!e) return 0;
        if (!std::strcmp(e, "tma1")) return 1;
        if (!std::strcmp(e, "tma2")) return 2;
        return 0;
    }();
    return v;
}

template <bool LAZY>
void launch_col_fwd_t(const DevPoint& d, uint32_t* A, uint32_t* B, cudaStream_t st) {
    const int var = col_pass_variant();
    if (var && col_tma_ok(d, A, B)) {
        with_log(d.logS, [&](auto s) {
            constexpr int LS = decltype(s)::value;
            const uint32_t tiles = ((1u << LS) / 32) * static_cast<uint32_t>(d.K);
            if (var == 2) {
                const uint32_t grid = std::min<uint32_t>(tiles, 6u * static_cast<uint32_t>(device_sms()));
                check(launch_pdl(k_ntt_col_fwd_tma<LS, LAZY, 2>, dim3(grid), dim3(256), col_fwd_tma_smem<2>(), st, d,
                                 col_tmap(d, A), col_tmap(d, B)),
                      "col_fwd launch");
            } else {
                check(launch_pdl(k_ntt_col_fwd_tma<LS, LAZY, 1>, dim3(tiles), dim3(256), col_fwd_tma_smem<1>(), st, d,
                                 col_tmap(d, A), col_tmap(d, B)),
                      "col_fwd launch");
            }
        });
        return;
    }
    with_cols(d.logR, d.logS, [&](auto r, auto s) {
        constexpr int LR = decltype(r)::value, LS = decltype(s)::value;
        const dim3 grid(col_blocks<LR>(LS), d.K);
        check(launch_pdl(k_ntt_col_fwd<LR, LS, LAZY>, grid, dim3(col_threads<LR>()), col_fwd_smem_t(LR), st, d, A,
                         B),
              "col_fwd launch");
    });
}

template <bool LAZY>
void launch_col_inv_t(const DevPoint& d, uint32_t* A, cudaStream_t st) {
    const int var = col_pass_variant();
    if (var && col_tma_ok(d, A, A)) {
        with_log(d.logS, [&](auto s) {
            constexpr int LS = decltype(s)::value;
            const uint32_t tiles = ((1u << LS) / 32) * static_cast<uint32_t>(d.K);
            if (var == 2) {
                const uint32_t grid = std::min<uint32_t>(tiles, 8u * static_cast<uint32_t>(device_sms()));
                check(launch_pdl(k_ntt_col_inv_tma<LS, LAZY, 2>, dim3(grid), dim3(256), col_inv_tma_smem<2>(), st, d,
                                 col_tmap(d, A)),
                      "col_inv launch");
            } else {
                check(launch_pdl(k_ntt_col_inv_tma<LS, LAZY, 1>, dim3(tiles), dim3(256), col_inv_tma_smem<1>(), st, d,
                                 col_tmap(d, A)),
                      "col_inv launch");
            }
        });
        return;
    }
    with_cols(d.logR, d.logS, [&](auto r, auto s) {
        constexpr int LR = decltype(r)::value, LS = decltype(s)::value;
        const dim3 grid(col_blocks<LR>(LS), d.K);
        check(launch_pdl(k_ntt_col_inv<LR, LS, LAZY>, grid, dim3(col_threads<LR>()), col_inv_smem_t(LR), st, d, A),
              "col_inv launch");
    });
}

template <int LOGS, bool LAZY>
void launch_row_t(const DevPoint& d, uint32_t* A, uint32_t* B, int mode, cudaStream_t st) {
    using RG = RowGeom<LOGS>;
    const uint32_t R = 1u << d.logR;
    const dim3 grid(RG::G >= 2 ? R / RG::G : R, d.K);
    check(launch_pdl(k_ntt_row<LOGS, LAZY>, grid, dim3(row_threads<LOGS>()), row_smem_t<LOGS>(), st, d, A, B, mode),
          "row launch");
}

template <bool LAZY>
void launch_ntt_t(const DevPoint& d, uint32_t* A, uint32_t* B, int mode, cudaStream_t st) {
    const bool col_fwd = mode == kRowProduct || mode == kRowForward || mode == kPassColFwd;
    const bool row = mode == kRowProduct || mode == kRowForward || mode == kPassRow;
    const bool col_inv = mode == kRowProduct || mode == kPassColInv;
    const int row_mode = mode == kRowForward ? kRowForward : kRowProduct;
    if (col_fwd && d.logR) launch_col_fwd_t<LAZY>(d, A, B, st);
    if (row) switch (d.logS) {
        case 6: launch_row_t<6, LAZY>(d, A, B, row_mode, st); break;
        case 7: launch_row_t<7, LAZY>(d, A, B, row_mode, st); break;
        case 8: launch_row_t<8, LAZY>(d, A, B, row_mode, st); break;
        case 9: launch_row_t<9, LAZY>(d, A, B, row_mode, st); break;
        case 10: launch_row_t<10, LAZY>(d, A, B, row_mode, st); break;
        case 11: launch_row_t<11, LAZY>(d, A, B, row_mode, st); break;
        default: throw std::runtime_error("unsupported row length");
    }
    if (col_inv && d.logR) launch_col_inv_t<LAZY>(d, A, st);
}

}  // namespace

bool ntt_mixed_ok(const DevPoint& d) { return d.logN > kSmallLogN && d.logR == 6 && d.logS >= 6 && d.logS <= 11; }

uint32_t ntt_mixed_blocks(int pass, uint32_t logS, uint32_t primes) {
    if (pass != kPassRow) return primes * ((1u << logS) >> 5);
    uint32_t per = 0, threads = 0;
    with_log(logS, [&](auto ls) {
        constexpr int LS = decltype(ls)::value;
        per = row_blocks<LS>(6);
        threads = row_threads<LS>();
    });
    return threads == 256 ? primes * per : primes * per / 2;
}

namespace {

uint32_t row_mixed_region(uint32_t max_log_s) {
    size_t r = 0;
    for (uint32_t ls = 6; ls <= max_log_s && ls <= 11; ++ls) {
        with_log(ls, [&](auto l) { r = std::max(r, row_smem_t<decltype(l)::value>()); });
    }
    return static_cast<uint32_t>((r + 1023) / 1024 * 1024);
}

template <bool LAZY>
void mixed_pass(const GroupTable* t, int pass, uint32_t max_log_s, uint32_t grid, cudaStream_t st, int* occupancy) {
    auto run = [&](auto kernel, size_t smem, auto... extra) {
        if (occupancy) {
            check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy, kernel, 256, smem), "occupancy");
        } else {
            kernel<<<grid, 256, smem, st>>>(*t, extra...);
        }
    };
    if (pass == kPassColFwd) {
        run(k_ntt_col_fwd_mixed<LAZY>, col_fwd_smem_t(6));
    } else if (pass == kPassColInv) {
        run(k_ntt_col_inv_mixed<LAZY>, col_inv_smem_t(6));
    } else if (pass == kPassRow) {
        const uint32_t region = row_mixed_region(max_log_s);
        run(k_ntt_row_mixed<LAZY>, 2 * size_t(region), region);
    } else {
        throw std::runtime_error("mixed transform: unknown pass");
    }
}

template <bool LAZY>
void mixed_attrs() {
    check(cudaFuncSetAttribute(k_ntt_col_fwd_mixed<LAZY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(col_fwd_smem_t(6))),
          "mixed smem");
    check(cudaFuncSetAttribute(k_ntt_col_inv_mixed<LAZY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(col_inv_smem_t(6))),
          "mixed smem");
    check(cudaFuncSetAttribute(k_ntt_row_mixed<LAZY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(2 * row_mixed_region(11))),
          "mixed smem");
}

}  // namespace

void launch_ntt_mixed(const GroupTable& t, int pass, bool lazy, uint32_t max_log_s, uint32_t grid, cudaStream_t st) {
    if (t.total == 0) return;
    if (grid == 0 || grid > t.total) grid = t.total;
    if (lazy) {
        mixed_pass<true>(&t, pass, max_log_s, grid, st, nullptr);
    } else {
        mixed_pass<false>(&t, pass, max_log_s, grid, st, nullptr);
    }
    check(cudaGetLastError(), "mixed transform launch");
}

int ntt_mixed_occupancy(int pass, bool lazy, uint32_t max_log_s) {
    int n = 0;
    if (lazy) {
        mixed_pass<true>(nullptr, pass, max_log_s, 0, nullptr, &n);
    } else {
        mixed_pass<false>(nullptr, pass, max_log_s, 0, nullptr, &n);
    }
    return n;
}

void build_row_tables(const DevPoint& d, uint2* out, cudaStream_t st) {
    k_row_tables<<<dim3(1u << d.logR, d.K), 256, 0, st>>>(d, out);
    check(cudaGetLastError(), "row tables launch");
}

void ntt_init_attributes() {
    attrs_all<true>();
    attrs_all<false>();
    mixed_attrs<true>();
    mixed_attrs<false>();
    check(cudaFuncSetAttribute(k_ntt_small, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 1024 * 4),
          "small smem");
}

// The product's transform chain on residues A, B (K x N each): y_j in A.
// mode kRowForward stops after the forward transforms (A, B bit-reversed,
// canonical).
void launch_ntt(const DevPoint& d, uint32_t* A, uint32_t* B, int mode, cudaStream_t st) {
    if (d.logN <= kSmallLogN) {
        if (mode == kRowProduct || mode == kRowForward || mode == kPassRow)
            k_ntt_small<<<d.K, kNttThreads, 2 * d.N * sizeof(uint32_t), st>>>(d, A, B,
                                                                                mode == kRowForward ? kRowForward
                                                                                                    : kRowProduct);
        return;
    }
    if (d.lazy) {
        launch_ntt_t<true>(d, A, B, mode, st);
    } else {
        launch_ntt_t<false>(d, A, B, mode, st);
    }
}

uint32_t ntt_blocks_per_prime(int pass, uint32_t logR, uint32_t logS) {
    if (pass == kPassRow) {
        const uint32_t G = 2048u >> logS;
        return G >= 2 ? (1u << logR) / G : (1u << logR);
    }
    return (1u << logS) >> (11 - logR);
}

void launch_ntt_group(const GroupTable& t, int pass, uint32_t logR, uint32_t logS, bool lazy, uint32_t grid,
                      cudaStream_t st) {
    if (t.total == 0) return;
    if (grid == 0 || grid > t.total) grid = t.total;
    if (lazy) {
        group_pass<true>(&t, pass, logR, logS, grid, st, nullptr);
    } else {
        group_pass<false>(&t, pass, logR, logS, grid, st, nullptr);
    }
}

int ntt_group_occupancy(int pass, uint32_t logR, uint32_t logS, bool lazy) {
    int n = 0;
    if (lazy) {
        group_pass<true>(nullptr, pass, logR, logS, 0, nullptr, &n);
    } else {
        group_pass<false>(nullptr, pass, logR, logS, 0, nullptr, &n);
    }
    return n;
}

}  // namespace fpm
