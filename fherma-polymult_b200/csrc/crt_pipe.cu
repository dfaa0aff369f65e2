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
// Organisation on the B200:
//   * one CTA per SM walks super-tiles of 256 coefficients; TMEM's 512 columns
//     hold the two 128-row halves of a super-tile (U <= 256 columns each);
//   * warp 0 (one thread) streams the constant image in, chunk by chunk,
//     through a two-slot ring;
//   * warps 2-9, one thread per row, load y straight from HBM (coalesced,
//     the next chunk's loads in flight under the current chunk's work), write
//     it into the MMA's K-major byte layout, add up the rounding sum and the
//     top limb, and put v in the last chunk;
//   * warp 1 (one thread) issues the MMAs, two halves per chunk;
//   * warps 10-17, one thread per row: a quotient estimate e from the top
//     TMEM columns (within one of floor(X / q)), then one pass from the bottom
//     limb up that assembles X from D with carries, subtracts e q, stores the
//     limbs and tracks the borrows that tell whether X - e q lies in [0, q);
//     the rare row that does not (about 2^-11 of them) adds or subtracts q in
//     a second pass over what it stored.
// Per-prime constants and q come from kernel parameters (constant bank), so
// shared memory carries only the MMA operands and the per-row top limbs.
// The kernel is compiled for the common limb counts (L = 64, 55, 28, 8) and
// once for any L.
//
// Every wait is bounded; a timeout raises an abort flag that every role
// checks, the producer and the MMA thread wait out what they have in flight,
// and the error word gets bit 1.
#include "device.cuh"
#include "kernels.h"
#include "pdl.cuh"
#include "tc.cuh"

namespace fpm {

namespace {

constexpr int kThreads = 576;             // 18 warps
constexpr int kStagerWarp0 = 2;           // warps 2-9
constexpr int kEpiWarp0 = 10;             // warps 10-17
constexpr uint32_t kSuper = 256;          // coefficients per super-tile
constexpr uint32_t kChunk = 32;           // K rows (primes) per chunk
constexpr int kMaxChunks = kMaxK / kChunk;   // K + 1 <= kMaxK rows
constexpr uint32_t kSlot = 32768;         // bytes: A slot (two halves), B slot (U <= 256)
constexpr int kX = kMaxL + 2;

struct Smem {
    uint8_t* a;          // [2][2 halves][16 KB]
    uint8_t* b;          // [2][U x 128]
    uint4* meta;         // [2][256] {top limb words 0, 1, 2, -}
    uint32_t* outs;      // [2 halves][128 rows][out_stride(L)] result limbs
    uint64_t* b_full;    // [2]
    uint64_t* a_full;    // [2]
    uint64_t* mma_done;  // [2]
    uint64_t* d_full;    // [1]
    uint64_t* d_empty;   // [2]
    uint64_t* m_full;    // [2]
    uint64_t* m_empty;   // [2]
    uint64_t* o_ready;   // [2] a half's result rows are in outs
    uint64_t* o_free;    // [2] a half's rows have been copied out
    uint32_t* tmem_base;
    volatile uint32_t* abort;
};

// Words per staged result row: a 16-byte-chunk stride that is odd (vector
// rows, L a multiple of 4) or an odd word stride (scalar rows), so the
// epilogue's row writes and the copy-out's reads are free of bank conflicts.
__host__ __device__ constexpr int out_stride(int L) { return (L & 3) == 0 ? 4 * ((L / 4) | 1) : (L | 1); }
constexpr int kMaxOutStride = out_stride(kMaxL);

constexpr size_t kMetaOff = 4 * size_t(kSlot);
constexpr size_t kOutOff = kMetaOff + 2 * kSuper * sizeof(uint4);
constexpr size_t kBarOff = kOutOff + size_t(kSuper) * kMaxOutStride * 4;
constexpr size_t kSmemBytes = kBarOff + 17 * 8 + 16;

__device__ inline Smem carve(uint8_t* base) {
    Smem s;
    s.a = base;
    s.b = base + 2 * kSlot;
    s.meta = reinterpret_cast<uint4*>(base + kMetaOff);
    s.outs = reinterpret_cast<uint32_t*>(base + kOutOff);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + kBarOff);
    s.b_full = bars;
    s.a_full = bars + 2;
    s.mma_done = bars + 4;
    s.d_full = bars + 6;
    s.d_empty = bars + 7;
    s.m_full = bars + 9;
    s.m_empty = bars + 11;
    s.o_ready = bars + 13;
    s.o_free = bars + 15;
    s.tmem_base = reinterpret_cast<uint32_t*>(bars + 17);
    s.abort = s.tmem_base + 1;
    return s;
}

// y_j of one coefficient, streamed past L1.
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// Bounded wait that also gives up once another role has raised the abort flag.
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity, volatile uint32_t* abort) {
    if (tc::mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = tc::globaltimer();
    while (!tc::mbar_try_wait_sleep(bar, parity)) {
        if (*abort) return false;
        if (tc::globaltimer() - t0 > tc::kWaitNs) {
            *abort = 1;
            return false;
        }
    }
    return true;
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
    k_crt_pipe(DevPoint d, const __grid_constant__ CrtConsts cc, const uint32_t* __restrict__ Y,
               uint32_t* __restrict__ C, uint32_t n_begin, uint32_t n_end) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    pdl_launch_dependents();
    const Smem sm = carve(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int L = LT > 0 ? LT : d.L;
    const int K = d.K;
    const uint32_t U = LT > 0 ? (4 * LT - 1 + 31) / 32 * 32 : d.crt_u;
    const uint32_t N = d.N;
    const int nch = (K + 1 + static_cast<int>(kChunk) - 1) / static_cast<int>(kChunk);   // K + 1 rows
    const uint32_t tiles = (n_end - n_begin + kSuper - 1) / kSuper;

    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&sm.b_full[i], 1);
            tc::mbar_init(&sm.a_full[i], 256);
            tc::mbar_init(&sm.mma_done[i], 1);
            tc::mbar_init(&sm.d_empty[i], 128);
            tc::mbar_init(&sm.m_full[i], 256);
            tc::mbar_init(&sm.m_empty[i], 256);
            tc::mbar_init(&sm.o_ready[i], 128);
            tc::mbar_init(&sm.o_free[i], 128);
        }
        tc::mbar_init(sm.d_full, 1);
        *sm.abort = 0;
        tc::fence_mbar_init();
    }
    if (warp == 0) tc::tmem_alloc(sm.tmem_base, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *sm.tmem_base;
    pdl_wait();   // y and c belong to the kernels around this one

    if (warp == 0) {
        // ---- producer: constant chunks, two-slot ring ----
        if (lane == 0) {
            const uint32_t bbytes = U * 128;
            uint32_t b_par[2] = {0, 0};   // parity of each slot's last arming
            bool armed_b[2] = {false, false};
            uint32_t g = 0;
            for (uint32_t t = blockIdx.x; t < tiles && !*sm.abort; t += gridDim.x) {
                for (int c = 0; c < nch; ++c, ++g) {
                    const int s = g & 1;
                    if (g >= 2 && !wait_or_abort(&sm.mma_done[s], ((g - 2) >> 1) & 1, sm.abort)) break;
                    tc::mbar_arrive_expect_tx(&sm.b_full[s], bbytes);
                    tc::bulk_g2s(sm.b + s * kSlot, d.crt_img_v + static_cast<size_t>(c) * bbytes, bbytes,
                                 &sm.b_full[s]);
                    b_par[s] = (g >> 1) & 1;
                    armed_b[s] = true;
                }
                if (*sm.abort) break;
            }
            // Copies still in flight must land before the CTA may exit.
            for (int s = 0; s < 2; ++s) {
                if (armed_b[s]) tc::wait_parity(&sm.b_full[s], b_par[s]);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_u8(U);
            uint32_t g = 0, it = 0;
            bool issued = false;
            uint32_t last_s = 0, last_par = 0;
            for (uint32_t t = blockIdx.x; t < tiles && !*sm.abort; t += gridDim.x, ++it) {
                bool ok = true;
                if (it >= 1) {
                    ok = wait_or_abort(&sm.d_empty[0], (it - 1) & 1, sm.abort) &&
                         wait_or_abort(&sm.d_empty[1], (it - 1) & 1, sm.abort);
                }
                for (int c = 0; c < nch && ok; ++c, ++g) {
                    const int s = g & 1;
                    ok = wait_or_abort(&sm.b_full[s], (g >> 1) & 1, sm.abort) &&
                         wait_or_abort(&sm.a_full[s], (g >> 1) & 1, sm.abort);
                    if (!ok) break;
                    tc::tc_fence_after();
                    const uint32_t a0 = tc::smem_addr(sm.a + s * kSlot), b0 = tc::smem_addr(sm.b + s * kSlot);
                    // K steps of 8 rows; the last chunk stops after row K.
                    const int rows_c = min(static_cast<int>(kChunk), K + 1 - c * static_cast<int>(kChunk));
                    const uint32_t ksteps = static_cast<uint32_t>(rows_c + 7) / 8;
                    for (uint32_t h = 0; h < 2; ++h) {
                        for (uint32_t kk = 0; kk < ksteps; ++kk) {
                            const uint64_t ad = tc::smem_desc(a0 + h * 16384 + kk * 2 * 2048, 2048, 128);
                            const uint64_t bd = tc::smem_desc(b0 + kk * 2 * (U * 16), U * 16, 128);
                            tc::mma_u8(tmem + h * 256, ad, bd, idesc, c > 0 || kk > 0);
                        }
                    }
                    tc::mma_commit(&sm.mma_done[s]);
                    issued = true;
                    last_s = s;
                    last_par = (g >> 1) & 1;
                }
                if (!ok) break;
                tc::mma_commit(sm.d_full);
            }
            // MMAs still running must finish before the CTA may exit.
            if (issued) tc::wait_parity(&sm.mma_done[last_s], last_par);
        }
        __syncwarp();
    } else if (warp < kEpiWarp0) {
        // ---- stagers: thread = one row of the super-tile ----
        const uint32_t row = threadIdx.x - kStagerWarp0 * 32;
        const uint32_t h = row >> 7, m = row & 127;
        uint32_t g = 0, it = 0;
        for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
            const uint32_t n0 = n_begin + t * kSuper;
            const bool live = row < min(kSuper, n_end - n0);
            const uint32_t* yrow = Y + n0 + row;
            uint64_t vacc = 0, tlo = 0, thi = 0;   // sum y r50; sum y (top & 0xFFFF); sum y (top >> 16)
            bool ok = true;
            uint32_t ya[kChunk], yb[kChunk];
#pragma unroll
            for (int jj = 0; jj < static_cast<int>(kChunk); ++jj)
                ya[jj] = (live && jj < K) ? ld_stream(yrow + static_cast<size_t>(jj) * N) : 0u;
#pragma unroll
            for (int c = 0; c < kMaxChunks; ++c) {
                if (c >= nch) break;
                uint32_t(&yv)[kChunk] = (c & 1) ? yb : ya;
                uint32_t(&yn)[kChunk] = (c & 1) ? ya : yb;
                if (c + 1 < kMaxChunks && c + 1 < nch) {
                    // The next chunk's loads go out before this chunk's work.
#pragma unroll
                    for (int jj = 0; jj < static_cast<int>(kChunk); ++jj) {
                        const int j = (c + 1) * static_cast<int>(kChunk) + jj;
                        yn[jj] = (live && j < K) ? ld_stream(yrow + static_cast<size_t>(j) * N) : 0u;
                    }
                }
                const int s = g & 1;
                if (g >= 2) ok = wait_or_abort(&sm.mma_done[s], ((g - 2) >> 1) & 1, sm.abort);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
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
                uint8_t* as = sm.a + s * kSlot + h * 16384 + m * 16;
#pragma unroll
                for (int q4 = 0; q4 < 8; ++q4)
                    *reinterpret_cast<uint4*>(as + q4 * 2048) =
                        make_uint4(yv[4 * q4], yv[4 * q4 + 1], yv[4 * q4 + 2], yv[4 * q4 + 3]);
                tc::fence_proxy_async_smem();
                tc::mbar_arrive(&sm.a_full[s]);
                ++g;
            }
            if (!ok) break;
            const int p = it & 1;
            if (it >= 2) {
                ok = wait_or_abort(&sm.m_empty[p], ((it - 2) >> 1) & 1, sm.abort);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
            }
            // Top-limb sum = tlo + thi 2^16, as three words.
            const uint64_t t0 = tlo + ((thi & 0xFFFFu) << 16);
            const uint64_t t1 = (t0 >> 32) + (thi >> 16);
            sm.meta[p * kSuper + row] =
                make_uint4(static_cast<uint32_t>(t0), static_cast<uint32_t>(t1), static_cast<uint32_t>(t1 >> 32), 0u);
            tc::mbar_arrive(&sm.m_full[p]);
        }
    } else {
        // ---- epilogue: thread = one row of one half ----
        const int ew = warp - kEpiWarp0;
        const uint32_t h = ew >> 2, qd = warp & 3;
        const uint32_t row = h * 128 + qd * 32 + lane;
        const uint32_t tq = tmem + ((qd * 32) << 16) + h * 256;
        const uint32_t npieces = U / 16;
        const int n = L + 2, drop = top_drop(L);
        const uint32_t top_piece = static_cast<uint32_t>(4 * drop) / 16;
        const bool svec = (L & 3) == 0;                                             // 16-byte rows in outs
        const bool gvec = svec && (reinterpret_cast<uintptr_t>(C) & 15) == 0;      // 16-byte global stores
        const int ostride = LT > 0 ? out_stride(LT) : out_stride(L);
        const uint32_t hrow = qd * 32 + lane;                                       // row within the half
        uint32_t* srow = sm.outs + (h * 128 + hrow) * ostride;
        constexpr int kXL = LT > 0 ? LT + 2 : kX;        // limbs handled
        constexpr int kPieces = (kXL + 3) / 4;
        uint32_t it = 0;
        for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
            const uint32_t n0 = n_begin + t * kSuper;
            const bool live = row < min(kSuper, n_end - n0);
            const int p = it & 1;
            bool ok = wait_or_abort(&sm.m_full[p], (it >> 1) & 1, sm.abort);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            const uint4 meta = sm.meta[p * kSuper + row];
            tc::mbar_arrive(&sm.m_empty[p]);
            ok = wait_or_abort(sm.d_full, it & 1, sm.abort);
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
                for (int k = 15; k >= 0; --k) xd = xd * 256.0 + ra[k];
            }
            xd = ldexp(xd, static_cast<int>(8 * 16 * top_piece) - 32 * drop) +
                 ldexp(static_cast<double>(meta.x), 32 * (L - 1 - drop)) +
                 ldexp(static_cast<double>(meta.y), 32 * (L - drop)) +
                 ldexp(static_cast<double>(meta.z), 32 * (L + 1 - drop));
            const double f = floor(xd * d.q_top_inv);
            const uint64_t e = f > 0 ? static_cast<uint64_t>(f) : 0;
            const uint32_t e_lo = static_cast<uint32_t>(e), e_hi = static_cast<uint32_t>(e >> 32);
            if (it >= 1) {
                // The previous super-tile's rows of this half have left outs.
                ok = wait_or_abort(&sm.o_free[h], (it - 1) & 1, sm.abort);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
            }
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
                for (int i = 0; i < 4; ++i) {
                    const int k = 4 * pc + i;
                    if (k < kXL && k < n) {
                        uint64_t w = carry;
                        if (have) {
                            w += cur[4 * i];
                            w += static_cast<uint64_t>(cur[4 * i + 1]) * 256u;
                            w += static_cast<uint64_t>(cur[4 * i + 2]) * 65536u;
                            w += static_cast<uint64_t>(cur[4 * i + 3]) * 16777216u;
                        }
                        if (k == L - 1) w += meta.x;
                        if (k == L) w += meta.y;
                        if (k == L + 1) w += meta.z;
                        carry = w >> 32;
                        const uint32_t qk = cc.q[k];
                        const uint64_t acc = static_cast<uint64_t>(e_lo) * qk + c0;
                        c0 = (acc >> 32) + static_cast<uint64_t>(e_hi) * qk;
                        const uint64_t dy =
                            static_cast<uint64_t>(static_cast<uint32_t>(w)) - static_cast<uint32_t>(acc) - b0;
                        const uint32_t yk = static_cast<uint32_t>(dy);
                        b0 = static_cast<uint32_t>(dy >> 63);
                        b1 = static_cast<uint32_t>((static_cast<uint64_t>(yk) - qk - b1) >> 63);
                        o[i] = yk;
                        if (k < L) {
                            if (svec) {
                                if (i == 3) *reinterpret_cast<uint4*>(srow + k - 3) = make_uint4(o[0], o[1], o[2], o[3]);
                            } else {
                                srow[k] = yk;
                            }
                        }
                    }
                }
                if (more) tmem_wait(nxt);
            }
            // TMEM is read: the next super-tile's MMAs may start on this half.
            tc::tc_fence_before();
            tc::mbar_arrive(&sm.d_empty[h]);
            // X - e q is negative (add q) or at least q (subtract q): rare.
            if (live && (b0 || !b1)) {
                uint32_t cb = 0;
                for (int k = 0; k < L; ++k) {
                    const uint32_t x = srow[k], qk = cc.q[k];
                    if (b0) {
                        const uint64_t sum = static_cast<uint64_t>(x) + qk + cb;
                        srow[k] = static_cast<uint32_t>(sum);
                        cb = static_cast<uint32_t>(sum >> 32);
                    } else {
                        const uint64_t dd = static_cast<uint64_t>(x) - qk - cb;
                        srow[k] = static_cast<uint32_t>(dd);
                        cb = static_cast<uint32_t>(dd >> 63);
                    }
                }
            }
            // The half's 128 rows are one contiguous run of c: copy it out
            // with coalesced stores once every row is in outs.
            tc::mbar_arrive(&sm.o_ready[h]);
            ok = wait_or_abort(&sm.o_ready[h], it & 1, sm.abort);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            {
                const int rows_h = max(0, min(128, static_cast<int>(min(kSuper, n_end - n0)) - static_cast<int>(128 * h)));
                uint32_t* gbase = C + static_cast<size_t>(n0 + 128 * h) * L;
                const uint32_t* sbase = sm.outs + h * 128 * ostride;
                if (gvec) {
                    const int q4 = L / 4, n4 = rows_h * q4;
                    for (int i4 = static_cast<int>(hrow); i4 < n4; i4 += 128) {
                        const int r = i4 / q4, c4 = i4 - r * q4;
                        *reinterpret_cast<uint4*>(gbase + 4 * i4) =
                            *reinterpret_cast<const uint4*>(sbase + r * ostride + 4 * c4);
                    }
                } else {
                    const int nw = rows_h * L;
                    for (int i = static_cast<int>(hrow); i < nw; i += 128) {
                        const int r = i / L;
                        gbase[i] = sbase[r * ostride + (i - r * L)];
                    }
                }
            }
            tc::mbar_arrive(&sm.o_free[h]);
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
                               static_cast<int>(kSmemBytes)),
          "crt_pipe smem");
}

}  // namespace

CrtConsts make_crt_consts(const HostPlan& pl) {
    CrtConsts cc{};
    for (int j = 0; j < pl.K; ++j) {
        cc.r50[j] = static_cast<uint32_t>((1ull << 50) / pl.primes[j]);
        const uint32_t top = pl.M[static_cast<size_t>(j) * pl.L + pl.L - 1];
        cc.mlo[j] = top & 0xFFFFu;
        cc.mhi[j] = top >> 16;
    }
    cc.mlo[pl.K] = pl.negp_top & 0xFFFFu;
    cc.mhi[pl.K] = pl.negp_top >> 16;
    for (int k = 0; k < pl.L; ++k) cc.q[k] = pl.q[k];
    return cc;
}

bool crt_pipe_supported(const DevPoint& d, const uint32_t* Y, uint32_t n_begin, uint32_t n_end) {
    // Bulk copies of y rows need 16-byte aligned starts and lengths.
    return d.L >= 2 && d.crt_u <= 256 && d.K + 1 <= kMaxK && d.crt_img_v && (d.N & 3) == 0 &&
           (n_begin & 3) == 0 && (n_end & 3) == 0 && (reinterpret_cast<uintptr_t>(Y) & 15) == 0;
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
    const uint32_t tiles = (n_end - n_begin + kSuper - 1) / kSuper;
    const uint32_t grid = tiles < static_cast<uint32_t>(sms) ? tiles : static_cast<uint32_t>(sms);
    cudaError_t e = cudaSuccess;
    switch (d.L) {
        case 64: e = launch_pdl(k_crt_pipe<64>, dim3(grid), dim3(kThreads), kSmemBytes, st, d, cc, Y, c, n_begin, n_end); break;
        case 55: e = launch_pdl(k_crt_pipe<55>, dim3(grid), dim3(kThreads), kSmemBytes, st, d, cc, Y, c, n_begin, n_end); break;
        case 28: e = launch_pdl(k_crt_pipe<28>, dim3(grid), dim3(kThreads), kSmemBytes, st, d, cc, Y, c, n_begin, n_end); break;
        case 8: e = launch_pdl(k_crt_pipe<8>, dim3(grid), dim3(kThreads), kSmemBytes, st, d, cc, Y, c, n_begin, n_end); break;
        default: e = launch_pdl(k_crt_pipe<0>, dim3(grid), dim3(kThreads), kSmemBytes, st, d, cc, Y, c, n_begin, n_end); break;
    }
    check(e, "crt launch");
}

}  // namespace fpm
