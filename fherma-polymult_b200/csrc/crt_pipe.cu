// CRT on the tensor cores as a persistent, warp-specialised pipeline.
//
// Arithmetic (reference CrtView rns.cuh:225-240, crt_columns / crt_combine
// rns_kernels.cuh:265-364): c = sum_j y_j M_j - v P mod q, v = round(sum_j
// y_j / p_j).  Here -v P rides in the GEMM as a (K+1)-th row: multiplier v,
// constant -P mod q, so
//
//     X = sum_{j<K} y_j M_j + v (-P mod q) = c (mod q),   X < 2^38 q.
//
// The low L - 1 limbs of every constant go through the 8-bit GEMM
// D[m][u] = sum_{j,s} byte_s(y_j(m)) byte_{u-s}(Mlow_j) (entries < 2^26); the
// top limb and the rounding sum run on the CUDA cores.  The prime basis covers
// 2^20 N q^2, so sum_j y_j / p_j lies within 2^-21 of an integer and a
// fixed-point sum with r_j = floor(2^50 / p_j) (error below 2^-11) rounds to v.
//
// Organisation on the B200: one CTA per SM walks tiles of 128 coefficients
// (one MMA M); tile i of a CTA accumulates into TMEM buffer i % 2 (256 columns
// each), so a tile's epilogue overlaps the next tile's staging and MMAs:
//   * the constant image (U x 128 bytes per chunk of 32 primes, the last chunk
//     cut to the K steps it uses) is loaded once per CTA by bulk copies and
//     stays resident in shared memory, so the MMAs never wait for constants;
//   * warp 2 (one thread) streams y through a ring of 16 KB stages (as many as
//     shared memory holds beside the constants, 2 to 4) with 2-D TMA copies:
//     per chunk a box of 32 primes x 128 coefficients of the prime-major
//     K x N array;
//   * warps 3-6, one thread per row, read their row's 32 values of a chunk from
//     the ring (conflict-free), write them in the MMA's K-major byte layout
//     (two-slot A ring), add up the rounding sum and the top limb, and put v in
//     the last chunk;
//   * warp 1 (one thread) issues a chunk's MMAs as soon as its A slot is full;
//   * warps 7-10 and 11-14 are two epilogue groups, one per TMEM buffer, one
//     thread per row: a quotient estimate e from the top TMEM columns (within
//     one of floor(X / q)), then one pass from the bottom limb up that
//     assembles X from D with carries, subtracts e q, stores the limbs of its
//     row and tracks the borrows that tell whether X - e q lies in [0, q); the
//     rare row that does not (about 2^-11 of them) adds or subtracts q in a
//     second pass over what it stored.
// Per-prime constants and q come from kernel parameters (constant bank).
// The kernel is compiled for the common limb counts (L = 64, 55, 28, 8) and
// once for any L.
//
// Every wait is bounded (DevPoint::wait_ns); a timeout raises an abort flag
// that every role checks, the copy and MMA issuers wait out what they have in
// flight, and the error word gets bit 1.
#include "device.cuh"
#include "kernels.h"
#include "pdl.cuh"
#include "tc.cuh"
#include "tmap.h"

namespace fpm {

namespace {

constexpr int kThreads = 480;             // 15 warps
constexpr int kMmaWarp = 1;
constexpr int kYWarp = 2;
constexpr int kStagerWarp0 = 3;           // warps 3-6
constexpr int kEpiWarp0 = 7;              // warps 7-10 (group 0), 11-14 (group 1)
constexpr uint32_t kCrtTile = 128;        // coefficients per tile
constexpr uint32_t kChunk = 32;           // K rows (primes) per chunk
constexpr int kMaxChunks = kMaxK / kChunk;   // K + 1 <= kMaxK rows
constexpr int kMaxYStages = 4;
constexpr uint32_t kASlot = 16384;        // [8 core columns][128 rows][16 bytes]
constexpr uint32_t kYSlot = kChunk * kCrtTile * 4;   // [32 primes][128 coefficients] u32
constexpr int kX = kMaxL + 2;
constexpr size_t kSmemLimit = 227 * 1024;

// Shared-memory plan, the same on host and device: the resident constants
// from 0, then the A ring, the y ring, the per-tile top-limb words and the
// barriers.
struct Layout {
    uint32_t b_bytes;      // resident constant image
    uint32_t ystages;      // y ring depth
    __host__ __device__ size_t a_off() const { return (size_t(b_bytes) + 1023) / 1024 * 1024; }
    __host__ __device__ size_t y_off() const { return a_off() + 2 * size_t(kASlot); }
    __host__ __device__ size_t meta_off() const { return y_off() + ystages * size_t(kYSlot); }
    __host__ __device__ size_t bar_off() const { return meta_off() + 2 * kCrtTile * sizeof(uint4); }
    __host__ __device__ size_t bytes() const { return bar_off() + 32 * 8 + 16; }
};

// Bytes of the constant image the MMAs read: full chunks of U x 128 bytes,
// the last one cut to the K steps (8 rows each) its K + 1 - 32 (nch - 1) rows
// need (a prefix of the chunk: 2 core columns of U x 16 bytes per step).
__host__ __device__ inline uint32_t resident_b_bytes(int K, uint32_t U) {
    const int nch = (K + 1 + static_cast<int>(kChunk) - 1) / static_cast<int>(kChunk);
    const int last_rows = K + 1 - static_cast<int>(kChunk) * (nch - 1);
    const uint32_t last_steps = static_cast<uint32_t>(last_rows + 7) / 8;
    return static_cast<uint32_t>(nch - 1) * U * 128 + last_steps * 2 * U * 16;
}

Layout make_layout(int K, uint32_t U) {
    Layout l{resident_b_bytes(K, U), kMaxYStages};
    while (l.ystages > 2 && l.bytes() > kSmemLimit) --l.ystages;
    return l;
}

struct Smem {
    uint8_t* b;          // resident constant image
    uint8_t* a;          // [2][kASlot]
    uint32_t* y;         // [ystages][32][128]
    uint4* meta;         // [2][128] {top-limb words 0, 1, 2, -}
    uint64_t* b_full;    // [1] the constant image landed
    uint64_t* a_full;    // [2] 128 rows staged
    uint64_t* a_empty;   // [2] its MMAs finished
    uint64_t* y_full;    // [kMaxYStages] TMA box landed
    uint64_t* y_empty;   // [kMaxYStages] 128 rows read it
    uint64_t* d_full;    // [2] a tile's MMAs finished (per TMEM buffer)
    uint64_t* d_empty;   // [2] its epilogue group has read TMEM
    uint64_t* m_full;    // [2] a tile's top-limb words staged
    uint64_t* m_empty;   // [2] and read
    uint32_t* tmem_base;
    volatile uint32_t* abort;
};

__device__ inline Smem carve(uint8_t* base, const Layout& lay) {
    Smem s;
    s.b = base;
    s.a = base + lay.a_off();
    s.y = reinterpret_cast<uint32_t*>(base + lay.y_off());
    s.meta = reinterpret_cast<uint4*>(base + lay.meta_off());
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + lay.bar_off());
    s.b_full = bars;
    s.a_full = bars + 1;
    s.a_empty = bars + 3;
    s.y_full = bars + 5;
    s.y_empty = bars + 5 + kMaxYStages;
    s.d_full = bars + 5 + 2 * kMaxYStages;
    s.d_empty = s.d_full + 2;
    s.m_full = s.d_full + 4;
    s.m_empty = s.d_full + 6;
    s.tmem_base = reinterpret_cast<uint32_t*>(bars + 32);
    s.abort = s.tmem_base + 1;
    return s;
}

// Waits for this thread's TMEM loads; naming the registers keeps every read of
// them below the wait.
__device__ __forceinline__ void tmem_wait(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}

// LT > 0: L = LT at compile time; LT = 0: any L (predicated).
template <int LT>
__global__ void __launch_bounds__(kThreads, 1)
    k_crt_pipe(DevPoint d, const __grid_constant__ CrtConsts cc, const __grid_constant__ CUtensorMap tmY,
               uint32_t* __restrict__ C, uint32_t n_begin, uint32_t n_end, Layout lay) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    pdl_launch_dependents();
    const Smem sm = carve(smem_raw, lay);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int L = LT > 0 ? LT : d.L;
    const int K = d.K;
    const uint32_t U = LT > 0 ? (4 * LT - 1 + 31) / 32 * 32 : d.crt_u;
    const int nch = (K + 1 + static_cast<int>(kChunk) - 1) / static_cast<int>(kChunk);   // K + 1 rows
    const uint32_t tiles = (n_end - n_begin + kCrtTile - 1) / kCrtTile;
    const uint32_t ys_n = lay.ystages;
    const uint64_t lim = d.wait_ns;

    if (threadIdx.x == 0) {
        tc::mbar_init(sm.b_full, 1);
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&sm.a_full[i], kCrtTile);
            tc::mbar_init(&sm.a_empty[i], 1);
            tc::mbar_init(&sm.d_full[i], 1);
            tc::mbar_init(&sm.d_empty[i], kCrtTile);
            tc::mbar_init(&sm.m_full[i], kCrtTile);
            tc::mbar_init(&sm.m_empty[i], kCrtTile);
        }
        for (uint32_t i = 0; i < ys_n; ++i) {
            tc::mbar_init(&sm.y_full[i], 1);
            tc::mbar_init(&sm.y_empty[i], kCrtTile);
        }
        *sm.abort = 0;
        tc::fence_mbar_init();
        // The constant image is read-only plan data: it loads under the
        // preceding kernel's tail.  (Test hook: with kFaultCrt it is never
        // requested, so the MMA issuer's wait for it runs out.)
        if (!(d.fault & kFaultCrt)) {
            tc::mbar_arrive_expect_tx(sm.b_full, lay.b_bytes);
            const uint32_t chunk_bytes = U * 128;
            for (uint32_t off = 0; off < lay.b_bytes; off += chunk_bytes) {
                const uint32_t n = lay.b_bytes - off < chunk_bytes ? lay.b_bytes - off : chunk_bytes;
                tc::bulk_g2s(sm.b + off, d.crt_img_v + off, n, sm.b_full);
            }
        }
    }
    if (warp == kYWarp && lane == 0) tc::prefetch_tmap(&tmY);
    if (warp == 0) tc::tmem_alloc(sm.tmem_base, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *sm.tmem_base;

    if (warp == 0) {
        // The constant image must land before the CTA may exit (after an abort too).
        if (lane == 0 && !(d.fault & kFaultCrt)) tc::wait_parity(sm.b_full, 0, lim);
        __syncwarp();
    } else if (warp == kYWarp) {
        // ---- y boxes through the TMA ring ----
        if (lane == 0) {
            pdl_wait();   // y is the preceding kernel's output
            uint32_t par[kMaxYStages] = {};
            bool armed[kMaxYStages] = {};
            uint32_t g = 0;
            bool ok = true;
            for (uint32_t t = blockIdx.x; ok && t < tiles; t += gridDim.x) {
                const int x = static_cast<int>(n_begin + t * kCrtTile);
                for (int c = 0; c < nch; ++c, ++g) {
                    const uint32_t s = g % ys_n, u = g / ys_n;
                    if (u >= 1 && !(ok = tc::wait_or_abort(&sm.y_empty[s], (u - 1) & 1, sm.abort, lim))) break;
                    tc::mbar_arrive_expect_tx(&sm.y_full[s], kYSlot);
                    tc::tma_load_2d(sm.y + s * (kYSlot / 4), &tmY, x, c * static_cast<int>(kChunk), &sm.y_full[s]);
                    par[s] = u & 1;
                    armed[s] = true;
                }
            }
            for (uint32_t s = 0; s < ys_n; ++s) {
                if (armed[s]) tc::wait_parity(&sm.y_full[s], par[s], lim);
            }
        }
        __syncwarp();
    } else if (warp == kMmaWarp) {
        // ---- MMA issuer ----
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_u8(U);
            uint32_t g = 0, i = 0;
            uint64_t* last_bar = nullptr;
            uint32_t last_par = 0;
            bool ok = tc::wait_or_abort(sm.b_full, 0, sm.abort, lim);
            for (uint32_t t = blockIdx.x; ok && t < tiles; t += gridDim.x, ++i) {
                const uint32_t buf = i & 1, use = i >> 1;
                if (use >= 1 && !(ok = tc::wait_or_abort(&sm.d_empty[buf], (use - 1) & 1, sm.abort, lim))) break;
                for (int c = 0; c < nch; ++c, ++g) {
                    const int s = g & 1;
                    const uint32_t ph = (g >> 1) & 1;
                    ok = tc::wait_or_abort(&sm.a_full[s], ph, sm.abort, lim);
                    if (!ok) break;
                    tc::tc_fence_after();
                    const uint32_t a0 = tc::smem_addr(sm.a + s * kASlot), b0 = tc::smem_addr(sm.b + c * U * 128);
                    // K steps of 8 rows; the last chunk stops after row K.
                    const int rows_c = min(static_cast<int>(kChunk), K + 1 - c * static_cast<int>(kChunk));
                    const uint32_t ksteps = static_cast<uint32_t>(rows_c + 7) / 8;
                    for (uint32_t kk = 0; kk < ksteps; ++kk) {
                        const uint64_t ad = tc::smem_desc(a0 + kk * 2 * 2048, 2048, 128);
                        const uint64_t bd = tc::smem_desc(b0 + kk * 2 * (U * 16), U * 16, 128);
                        tc::mma_u8(tmem + buf * 256, ad, bd, idesc, c > 0 || kk > 0);
                    }
                    tc::mma_commit(&sm.a_empty[s]);
                    last_bar = &sm.a_empty[s];
                    last_par = ph;
                }
                if (!ok) break;
                tc::mma_commit(&sm.d_full[buf]);
            }
            // MMAs still running must finish before the CTA may exit.
            if (last_bar) tc::wait_parity(last_bar, last_par, lim);
        }
        __syncwarp();
    } else if (warp < kEpiWarp0) {
        // ---- stagers: thread = one row of the tile ----
        pdl_wait();
        const uint32_t m = threadIdx.x - kStagerWarp0 * 32;
        uint32_t g = 0, i = 0;
        for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++i) {
            const uint32_t n0 = n_begin + t * kCrtTile;
            const bool live = m < min(kCrtTile, n_end - n0);
            uint64_t vacc = 0, tlo = 0, thi = 0;   // sum y r50; sum y (top & 0xFFFF); sum y (top >> 16)
            bool ok = true;
#pragma unroll
            for (int c = 0; c < kMaxChunks; ++c) {
                if (c >= nch) break;
                uint32_t yv[kChunk];
                const uint32_t ys = g % ys_n, yu = g / ys_n;
                ok = tc::wait_or_abort(&sm.y_full[ys], yu & 1, sm.abort, lim);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
                const uint32_t* yrow = sm.y + ys * (kYSlot / 4) + m;
#pragma unroll
                for (int jj = 0; jj < static_cast<int>(kChunk); ++jj) yv[jj] = yrow[jj * kCrtTile];
                tc::mbar_arrive(&sm.y_empty[ys]);
#pragma unroll
                for (int jj = 0; jj < static_cast<int>(kChunk); ++jj) {
                    const int j = c * static_cast<int>(kChunk) + jj;
                    if (j < K) {
                        vacc += static_cast<uint64_t>(yv[jj]) * cc.r50[j];
                        tlo += static_cast<uint64_t>(yv[jj]) * cc.mlo[j];
                        thi += static_cast<uint64_t>(yv[jj]) * cc.mhi[j];
                    }
                }
                if (c == nch - 1) {
                    // Row K: the multiplier v of -P mod q.
                    int v = static_cast<int>((vacc + (1ull << 49)) >> 50);
                    v = v > K ? K : v;
                    const uint32_t vu = live ? static_cast<uint32_t>(v) : 0u;
                    tlo += static_cast<uint64_t>(vu) * cc.mlo[K];
                    thi += static_cast<uint64_t>(vu) * cc.mhi[K];
#pragma unroll
                    for (int jj = 0; jj < static_cast<int>(kChunk); ++jj)
                        if (c * static_cast<int>(kChunk) + jj == K) yv[jj] = vu;
                }
                const int s = g & 1;
                if (g >= 2) {
                    ok = tc::wait_or_abort(&sm.a_empty[s], ((g - 2) >> 1) & 1, sm.abort, lim);
                    ok = __all_sync(0xffffffffu, ok);
                    if (!ok) break;
                }
                uint8_t* as = sm.a + s * kASlot + m * 16;
#pragma unroll
                for (int q4 = 0; q4 < 8; ++q4)
                    *reinterpret_cast<uint4*>(as + q4 * 2048) =
                        make_uint4(yv[4 * q4], yv[4 * q4 + 1], yv[4 * q4 + 2], yv[4 * q4 + 3]);
                tc::fence_proxy_async_smem();
                tc::mbar_arrive(&sm.a_full[s]);
                ++g;
            }
            if (!ok) break;
            const int p = i & 1;
            if (i >= 2) {
                ok = tc::wait_or_abort(&sm.m_empty[p], ((i - 2) >> 1) & 1, sm.abort, lim);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
            }
            // Top-limb sum = tlo + thi 2^16, as three words.
            const uint64_t t0 = tlo + ((thi & 0xFFFFu) << 16);
            const uint64_t t1 = (t0 >> 32) + (thi >> 16);
            sm.meta[p * kCrtTile + m] =
                make_uint4(static_cast<uint32_t>(t0), static_cast<uint32_t>(t1), static_cast<uint32_t>(t1 >> 32), 0u);
            tc::mbar_arrive(&sm.m_full[p]);
        }
    } else {
        // ---- epilogue group grp (TMEM buffer grp): thread = one row ----
        pdl_wait();
        const uint32_t grp = static_cast<uint32_t>(warp - kEpiWarp0) >> 2, qd = warp & 3;
        const uint32_t row = qd * 32 + lane;
        const uint32_t tq = tmem + ((qd * 32) << 16) + grp * 256;
        const uint32_t npieces = U / 16;
        const int n = L + 2, drop = top_drop(L);
        const uint32_t top_piece = static_cast<uint32_t>(4 * drop) / 16;
        const bool gvec = (L & 3) == 0 && (reinterpret_cast<uintptr_t>(C) & 15) == 0;   // 16-byte row stores
        constexpr int kXL = LT > 0 ? LT + 2 : kX;        // limbs handled
        constexpr int kPieces = (kXL + 3) / 4;
        uint32_t k = 0;   // this group's tiles so far
        for (uint32_t t = blockIdx.x + grp * gridDim.x; t < tiles; t += 2 * gridDim.x, ++k) {
            const uint32_t n0 = n_begin + t * kCrtTile;
            const uint32_t rows_t = min(kCrtTile, n_end - n0);
            const bool live = row < rows_t;
            uint32_t* crow = C + static_cast<size_t>(n0 + (live ? row : 0)) * L;
            bool ok = tc::wait_or_abort(&sm.m_full[grp], k & 1, sm.abort, lim);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            const uint4 meta = sm.meta[grp * kCrtTile + row];
            tc::mbar_arrive(&sm.m_empty[grp]);
            ok = tc::wait_or_abort(&sm.d_full[grp], k & 1, sm.abort, lim);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            tc::tc_fence_after();
            uint32_t ra[16], rb[16];
            // Quotient estimate from the columns at and above limb `drop` and the
            // top-limb words: |estimate - X / q| < 2^-11, so e is within one.
            double xd = 0;
            for (uint32_t pc = npieces; pc-- > top_piece;) {
                tc::tmem_ld16(tq + pc * 16, ra);
                tmem_wait(ra);
#pragma unroll
                for (int kk = 15; kk >= 0; --kk) xd = xd * 256.0 + ra[kk];
            }
            xd = ldexp(xd, static_cast<int>(8 * 16 * top_piece) - 32 * drop) +
                 ldexp(static_cast<double>(meta.x), 32 * (L - 1 - drop)) +
                 ldexp(static_cast<double>(meta.y), 32 * (L - drop)) +
                 ldexp(static_cast<double>(meta.z), 32 * (L + 1 - drop));
            const double f = floor(xd * d.q_top_inv);
            const uint64_t e = f > 0 ? static_cast<uint64_t>(f) : 0;
            const uint32_t e_lo = static_cast<uint32_t>(e), e_hi = static_cast<uint32_t>(e >> 32);
            // One pass from the bottom: X with carries, minus e q; the borrows
            // of X - e q (b0) and of (X - e q) - q (b1).  TMEM pieces are
            // double-buffered: piece pc + 1 loads while piece pc is used.
            uint64_t carry = 0, c0 = 0;
            uint32_t b0 = 0, b1 = 0;
            uint32_t o[4];
            tc::tmem_ld16(tq, ra);
            tmem_wait(ra);
#pragma unroll
            for (int pc = 0; pc < kPieces; ++pc) {
                uint32_t(&cur)[16] = (pc & 1) ? rb : ra;
                uint32_t(&nxt)[16] = (pc & 1) ? ra : rb;
                const bool have = static_cast<uint32_t>(pc) < npieces;
                const bool more = static_cast<uint32_t>(pc + 1) < npieces;
                if (more) tc::tmem_ld16(tq + (pc + 1) * 16, nxt);
#pragma unroll
                for (int ii = 0; ii < 4; ++ii) {
                    const int kl = 4 * pc + ii;
                    if (kl < kXL && kl < n) {
                        uint64_t w = carry;
                        if (have) {
                            w += cur[4 * ii];
                            w += static_cast<uint64_t>(cur[4 * ii + 1]) * 256u;
                            w += static_cast<uint64_t>(cur[4 * ii + 2]) * 65536u;
                            w += static_cast<uint64_t>(cur[4 * ii + 3]) * 16777216u;
                        }
                        if (kl == L - 1) w += meta.x;
                        if (kl == L) w += meta.y;
                        if (kl == L + 1) w += meta.z;
                        carry = w >> 32;
                        const uint32_t qk = cc.q[kl];
                        const uint64_t acc = static_cast<uint64_t>(e_lo) * qk + c0;
                        c0 = (acc >> 32) + static_cast<uint64_t>(e_hi) * qk;
                        const uint64_t dy =
                            static_cast<uint64_t>(static_cast<uint32_t>(w)) - static_cast<uint32_t>(acc) - b0;
                        const uint32_t yk = static_cast<uint32_t>(dy);
                        b0 = static_cast<uint32_t>(dy >> 63);
                        b1 = static_cast<uint32_t>((static_cast<uint64_t>(yk) - qk - b1) >> 63);
                        o[ii] = yk;
                        if (kl < L && live) {
                            if (gvec) {
                                if (ii == 3) *reinterpret_cast<uint4*>(crow + kl - 3) = make_uint4(o[0], o[1], o[2], o[3]);
                            } else {
                                crow[kl] = yk;
                            }
                        }
                    }
                }
                if (more) tmem_wait(nxt);
            }
            // TMEM is read: the MMAs of this buffer's next tile may start.
            tc::tc_fence_before();
            tc::mbar_arrive(&sm.d_empty[grp]);
            // X - e q is negative (add q) or at least q (subtract q): rare.
            if (live && (b0 || !b1)) {
                uint32_t cb = 0;
                for (int kk = 0; kk < L; ++kk) {
                    const uint32_t x = crow[kk], qk = cc.q[kk];
                    if (b0) {
                        const uint64_t sum = static_cast<uint64_t>(x) + qk + cb;
                        crow[kk] = static_cast<uint32_t>(sum);
                        cb = static_cast<uint32_t>(sum >> 32);
                    } else {
                        const uint64_t dd = static_cast<uint64_t>(x) - qk - cb;
                        crow[kk] = static_cast<uint32_t>(dd);
                        cb = static_cast<uint32_t>(dd >> 63);
                    }
                }
            }
        }
    }

    tc::tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *sm.abort) atomicOr(d.err, 2u);
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 512);
    }
}

template <int LT>
void set_attr() {
    check(cudaFuncSetAttribute(k_crt_pipe<LT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(kSmemLimit)),
          "crt_pipe smem");
}

}  // namespace

CrtConsts make_crt_consts(const HostPlan& pl, const uint32_t* top) {
    CrtConsts cc{};
    for (int j = 0; j <= pl.K; ++j) {
        if (j < pl.K) cc.r50[j] = static_cast<uint32_t>((1ull << 50) / pl.primes[j]);
        cc.mlo[j] = top[j] & 0xFFFFu;
        cc.mhi[j] = top[j] >> 16;
    }
    for (int k = 0; k < pl.L; ++k) cc.q[k] = pl.q[k];
    return cc;
}

bool crt_pipe_supported(const DevPoint& d, const uint32_t* Y, uint32_t n_begin, uint32_t n_end) {
    // TMA boxes of y: 16-byte aligned base, row pitch (N words) and column
    // coordinates (n_begin) a multiple of 4 words; the constants resident.
    return d.L >= 2 && d.crt_u <= 256 && d.K + 1 <= kMaxK && d.crt_img_v && (d.N & 3) == 0 && d.N >= kCrtTile &&
           (n_begin & 3) == 0 && n_end <= d.N && (reinterpret_cast<uintptr_t>(Y) & 15) == 0 &&
           make_layout(d.K, d.crt_u).bytes() <= kSmemLimit;
}

void crt_pipe_init_attributes() {
    set_attr<0>();
    set_attr<64>();
    set_attr<55>();
    set_attr<28>();
    set_attr<8>();
}

void launch_crt_pipe(const DevPoint& d, const CrtConsts& cc, const uint32_t* Y, uint32_t* c, uint32_t n_begin,
                     uint32_t n_end, int sms, cudaStream_t st) {
    if (n_end <= n_begin) return;
    const uint32_t tiles = (n_end - n_begin + kCrtTile - 1) / kCrtTile;
    const uint32_t grid = tiles < static_cast<uint32_t>(sms) ? tiles : static_cast<uint32_t>(sms);
    const Layout lay = make_layout(d.K, d.crt_u);
    // y: K rows of N words, boxes of 32 primes x 128 coefficients.
    const CUtensorMap tm = make_tmap_u32(Y, static_cast<uint64_t>(d.K), d.N, d.N, kChunk, kCrtTile, TmaSwizzle::kNone);
    const size_t smem = lay.bytes();
    cudaError_t e = cudaSuccess;
    switch (d.L) {
        case 64: e = launch_pdl(k_crt_pipe<64>, dim3(grid), dim3(kThreads), smem, st, d, cc, tm, c, n_begin, n_end, lay); break;
        case 55: e = launch_pdl(k_crt_pipe<55>, dim3(grid), dim3(kThreads), smem, st, d, cc, tm, c, n_begin, n_end, lay); break;
        case 28: e = launch_pdl(k_crt_pipe<28>, dim3(grid), dim3(kThreads), smem, st, d, cc, tm, c, n_begin, n_end, lay); break;
        case 8: e = launch_pdl(k_crt_pipe<8>, dim3(grid), dim3(kThreads), smem, st, d, cc, tm, c, n_begin, n_end, lay); break;
        default: e = launch_pdl(k_crt_pipe<0>, dim3(grid), dim3(kThreads), smem, st, d, cc, tm, c, n_begin, n_end, lay); break;
    }
    check(e, "crt launch");
}

}  // namespace fpm
