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
// 2^20 N q^2, so sum_j y_j / p_j lies within 2^-21 of an integer v and any
// estimate within 1/2 - 2^-21 rounds to it.  The stagers sum in single
// precision: x = y_j >> sh_j (sh_j = bits of p_j - 23, so x < 2^23) is formed
// exactly as the float 2^23 + x by setting the exponent bits, multiplied by
// cf_j = 2^sh_j / p_j and added with FFMA; the 2^23 cf_j parts (each at most
// 2) add up to the constant voff, removed at the end.  Error: the dropped low
// bits, below 2^sh_j / p_j <= 2^-22 per term, and the roundings, below 2^-24
// of partial sums under 3 (K + 1) each; the host bounds the total
// (CrtConsts::est_err, 2^-8 at K = 160) and the kernel is used only while it
// is under 1/4.
//
// Organisation on the B200: one CTA per SM walks tiles of 128 coefficients
// (one MMA M); tile i of a CTA accumulates into TMEM buffer i % 2 (256 columns
// each), so a tile's epilogue overlaps the next tile's staging and MMAs:
//   * the constant image (U x 128 bytes per chunk of 32 primes, the last chunk
//     cut to the K steps it uses) is loaded once per CTA by bulk copies and
//     stays resident in shared memory, so the MMAs never wait for constants;
//   * warp 2 (one thread) streams y through a ring of 16 KB slots (as many as
//     shared memory holds beside the constants, 2 to 6) with 2-D TMA copies:
//     per chunk a box of 32 primes x 128 coefficients of the prime-major
//     K x N array;
//   * warps 2-9, two threads per row (each half of a chunk's 32 primes), read
//     their 16 values from the slot (conflict-free), meet at a named barrier,
//     and write the same values back into that slot in the MMA's K-major,
//     128-byte-swizzled byte layout (a box and an A operand are both 16 KB,
//     so one ring serves both and every slot is a y box in flight while the
//     MMAs need none); they also add up the rounding sum and the top limb,
//     and in the last chunk the two halves pool their sums through shared
//     memory and the first puts v in the row;
//   * warp 0 (one thread) issues a chunk's MMAs as soon as its slot holds A,
//     and frees the slot for the next box when they finish;
//   * warps 10-13 and 14-17 are two epilogue groups, one per TMEM buffer, one
//     thread per row: a quotient estimate e from the top TMEM columns (within
//     one of floor(X / q)), then one pass from the bottom limb up that
//     assembles X from D with carries, subtracts e q, stores the limbs of its
//     row and tracks the borrows that tell whether X - e q lies in [0, q); the
//     rare row that does not (about 2^-11 of them) adds or subtracts q in a
//     second pass over what it stored.
// Per-prime constants and q come in as kernel parameters and are copied to
// shared memory at the start: read from the parameter bank inside the loops
// (a few KB swept by every chunk and every limb) they made the stagers and
// the epilogue several times slower.
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

#include <cmath>

namespace fpm {

namespace {

constexpr int kThreads = 576;             // 18 warps
constexpr int kMmaWarp = 0;               // also allocates TMEM
constexpr int kYWarp = 1;
constexpr int kStagerWarp0 = 2;           // warps 2-9: row m, half h of each chunk
constexpr int kStagers = 256;
constexpr int kEpiWarp0 = 10;             // warps 10-13 (group 0), 14-17 (group 1)
constexpr uint32_t kCrtTile = 128;        // coefficients per tile
constexpr uint32_t kChunk = 32;           // K rows (primes) per chunk
constexpr int kMaxSlots = 6;
// A slot holds a y box, [32 primes][128 coefficients] u32, and then the A
// operand made from it, 128 rows x 128 bytes, 128-byte swizzled.
constexpr uint32_t kSlot = kChunk * kCrtTile * 4;
constexpr uint32_t kStagerBar = 1;        // named barrier of the 256 stager threads
constexpr int kX = kMaxL + 2;
constexpr size_t kSmemLimit = 227 * 1024;
// Shared copies of the constants: {cf_j bits, top_j, sh_j, 0} per row
// j < 32 nch (zero beyond the K + 1 rows), then q.
constexpr size_t kConstBytes = (kMaxK + 1) * sizeof(uint4) + ((kMaxL + 2) * 4 + 15) / 16 * 16;

// Shared-memory plan, the same on host and device: the resident constants
// from 0, then the slot ring (1024-byte aligned), the per-tile top-limb words,
// the constants and the barriers.
struct Layout {
    uint32_t b_bytes;      // resident constant image
    uint32_t slots;        // ring depth
    __host__ __device__ size_t slot_off() const { return (size_t(b_bytes) + 1023) / 1024 * 1024; }
    __host__ __device__ size_t meta_off() const { return slot_off() + slots * size_t(kSlot); }
    __host__ __device__ size_t xch_off() const { return meta_off() + 2 * kCrtTile * sizeof(uint4); }
    __host__ __device__ size_t const_off() const { return xch_off() + kCrtTile * sizeof(uint4); }
    __host__ __device__ size_t bar_off() const { return const_off() + kConstBytes; }
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
    Layout l{resident_b_bytes(K, U), kMaxSlots};
    while (l.slots > 2 && l.bytes() > kSmemLimit) --l.slots;
    return l;
}

struct Smem {
    uint8_t* b;          // resident constant image
    uint8_t* slot;       // [slots][kSlot]
    uint4* meta;         // [2][128] {top-limb words 0, 1, 2, -}
    uint4* xch;          // [128] second halves' sums {rounding sum, top-limb words 0, 1, 2}
    uint4* kc;           // [kMaxK + 1] {cf_j bits, top_j, sh_j, 0}
    uint32_t* qs;        // [L + 2] q, zero above L
    uint64_t* b_full;    // [1] the constant image landed
    uint64_t* y_full;    // [kMaxSlots] the slot's TMA box landed
    uint64_t* a_full;    // [kMaxSlots] 128 rows of A staged in it
    uint64_t* s_empty;   // [kMaxSlots] its MMAs finished
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
    s.slot = base + lay.slot_off();
    s.meta = reinterpret_cast<uint4*>(base + lay.meta_off());
    s.xch = reinterpret_cast<uint4*>(base + lay.xch_off());
    s.kc = reinterpret_cast<uint4*>(base + lay.const_off());
    s.qs = reinterpret_cast<uint32_t*>(base + lay.const_off() + (kMaxK + 1) * sizeof(uint4));
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + lay.bar_off());
    s.b_full = bars;
    s.y_full = bars + 1;
    s.a_full = bars + 1 + kMaxSlots;
    s.s_empty = bars + 1 + 2 * kMaxSlots;
    s.d_full = bars + 1 + 3 * kMaxSlots;
    s.d_empty = s.d_full + 2;
    s.m_full = s.d_full + 4;
    s.m_empty = s.d_full + 6;
    s.tmem_base = reinterpret_cast<uint32_t*>(bars + 32);
    s.abort = s.tmem_base + 1;
    return s;
}

static_assert(1 + 3 * kMaxSlots + 8 <= 32, "barriers fit before tmem_base");

// bar.red.and over the 256 stager threads: true when every one passed true.
// All of them reach it whatever their outcome, so none can be left waiting.
__device__ __forceinline__ bool stagers_all(bool p) {
    uint32_t r;
    asm volatile(
        "{ .reg .pred pi, po; setp.ne.u32 pi, %1, 0; bar.red.and.pred po, %2, %3, pi; selp.u32 %0, 1, 0, po; }"
        : "=r"(r)
        : "r"(static_cast<uint32_t>(p)), "n"(kStagerBar), "n"(kStagers)
        : "memory");
    return r != 0;
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
    // The 128-byte swizzle is a function of the shared address: the
    // operand atoms need a 1024-byte aligned base (error bit 4 otherwise).
    if (tc::smem_addr(smem_raw) & 1023u) {
        if (threadIdx.x == 0) atomicOr(d.err, 4u);
        return;
    }
    const Smem sm = carve(smem_raw, lay);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int L = LT > 0 ? LT : d.L;
    const int K = d.K;
    const uint32_t U = LT > 0 ? (4 * LT - 1 + 31) / 32 * 32 : d.crt_u;
    const int nch = (K + 1 + static_cast<int>(kChunk) - 1) / static_cast<int>(kChunk);   // K + 1 rows
    const uint32_t tiles = (n_end - n_begin + kCrtTile - 1) / kCrtTile;
    const uint32_t ns = lay.slots;
    const uint64_t lim = d.wait_ns;

    if (threadIdx.x == 0) {
        tc::mbar_init(sm.b_full, 1);
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&sm.d_full[i], 1);
            tc::mbar_init(&sm.d_empty[i], kCrtTile);
            tc::mbar_init(&sm.m_full[i], kCrtTile);
            tc::mbar_init(&sm.m_empty[i], kCrtTile);
        }
        for (uint32_t i = 0; i < ns; ++i) {
            tc::mbar_init(&sm.y_full[i], 1);
            tc::mbar_init(&sm.a_full[i], kStagers);
            tc::mbar_init(&sm.s_empty[i], 1);
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
    for (int j = threadIdx.x; j <= kMaxK; j += kThreads)
        sm.kc[j] = make_uint4(j < K ? __float_as_uint(cc.cf[j]) : 0u, j <= K ? cc.top[j] : 0u, j < K ? cc.sh[j] : 0u, 0u);
    for (int k = threadIdx.x; k < kMaxL + 2; k += kThreads) sm.qs[k] = cc.q[k];
    if (warp == kYWarp && lane == 0) tc::prefetch_tmap(&tmY);
    if (warp == 0) tc::tmem_alloc(sm.tmem_base, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *sm.tmem_base;

    if (warp == kYWarp) {
        // ---- y boxes through the TMA ring ----
        if (lane == 0) {
            pdl_wait();   // y is the preceding kernel's output
            uint32_t par[kMaxSlots] = {};
            bool armed[kMaxSlots] = {};
            uint32_t g = 0;
            bool ok = true;
            for (uint32_t t = blockIdx.x; ok && t < tiles; t += gridDim.x) {
                const int x = static_cast<int>(n_begin + t * kCrtTile);
                for (int c = 0; c < nch; ++c, ++g) {
                    const uint32_t s = g % ns, u = g / ns;
                    if (u >= 1 && !(ok = tc::wait_or_abort(&sm.s_empty[s], (u - 1) & 1, sm.abort, lim))) break;
                    tc::mbar_arrive_expect_tx(&sm.y_full[s], kSlot);
                    tc::tma_load_2d(sm.slot + s * kSlot, &tmY, x, c * static_cast<int>(kChunk), &sm.y_full[s]);
                    par[s] = u & 1;
                    armed[s] = true;
                }
            }
            for (uint32_t s = 0; s < ns; ++s) {
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
                    const uint32_t s = g % ns;
                    const uint32_t ph = (g / ns) & 1;
                    ok = tc::wait_or_abort(&sm.a_full[s], ph, sm.abort, lim);
                    if (!ok) break;
                    tc::tc_fence_after();
                    const uint32_t a0 = tc::smem_addr(sm.slot + s * kSlot), b0 = tc::smem_addr(sm.b + c * U * 128);
                    // K steps of 8 rows; the last chunk stops after row K.
                    const int rows_c = min(static_cast<int>(kChunk), K + 1 - c * static_cast<int>(kChunk));
                    const uint32_t ksteps = static_cast<uint32_t>(rows_c + 7) / 8;
                    // A and the full constant chunks are 128-byte swizzled;
                    // the short last chunk keeps the plain core-matrix layout
                    // (only its first K steps are resident).
                    const bool swz_b = c + 1 < nch;
                    for (uint32_t kk = 0; kk < ksteps; ++kk) {
                        const uint64_t ad = tc::smem_desc_sw128(a0 + kk * 32);
                        const uint64_t bd = swz_b ? tc::smem_desc_sw128(b0 + kk * 32)
                                                  : tc::smem_desc(b0 + kk * 2 * (U * 16), U * 16, 128);
                        tc::mma_u8(tmem + buf * 256, ad, bd, idesc, c > 0 || kk > 0);
                    }
                    tc::mma_commit(&sm.s_empty[s]);
                    last_bar = &sm.s_empty[s];
                    last_par = ph;
                }
                if (!ok) break;
                tc::mma_commit(&sm.d_full[buf]);
            }
            // MMAs still running, and the constant image (after an abort
            // too), must finish before the CTA may exit.
            if (last_bar) tc::wait_parity(last_bar, last_par, lim);
            if (!(d.fault & kFaultCrt)) tc::wait_parity(sm.b_full, 0, lim);
        }
        __syncwarp();
    } else if (warp < kEpiWarp0) {
        // ---- stagers: thread = row m, primes 16 h .. 16 h + 15 of each chunk ----
        pdl_wait();
        const uint32_t st = threadIdx.x - kStagerWarp0 * 32;
        const uint32_t m = st & (kCrtTile - 1), h = st / kCrtTile;
        constexpr int kHalf = static_cast<int>(kChunk) / 2;
        uint32_t g = 0, i = 0;
        for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++i) {
            const uint32_t n0 = n_begin + t * kCrtTile;
            const bool live = m < min(kCrtTile, n_end - n0);
            // The rounding sum as kPart float partial sums; the top-limb sum
            // sum_j y_j top_j (< 2^71) as 96 bits (t01, t2), fed by 64-bit
            // pairs of products (each < 2^63 with 31-bit primes, so a pair
            // cannot wrap).
            constexpr int kPart = 4;
            float vf[kPart] = {};
            uint64_t t01 = 0;
            uint32_t t2 = 0;
            bool ok = true;
#pragma unroll 1
            for (int c = 0; c < nch; ++c) {
                uint32_t yv[kHalf];
                const uint32_t s = g % ns;
                ok = tc::wait_or_abort(&sm.y_full[s], (g / ns) & 1, sm.abort, lim);
                ok = __all_sync(0xffffffffu, ok);
                if (ok) {
                    const uint32_t* yrow = reinterpret_cast<const uint32_t*>(sm.slot + s * kSlot) + h * kHalf * kCrtTile + m;
#pragma unroll
                    for (int jj = 0; jj < kHalf; ++jj) yv[jj] = yrow[jj * kCrtTile];
                }
                // Every row has read the box before any writes A over it (and
                // the eight warps leave together on an abort).
                ok = stagers_all(ok);
                if (!ok) break;
                // Rows j >= K of the box read as zero and cf_j = 0 there, so
                // every row of the chunk takes part without a test.
                const uint4* kc = sm.kc + c * static_cast<int>(kChunk) + h * kHalf;
#pragma unroll
                for (int q2 = 0; q2 < kHalf / 2; ++q2) {
                    uint64_t grp = 0;
#pragma unroll
                    for (int jj = 2 * q2; jj < 2 * q2 + 2; ++jj) {
                        const uint4 kj = kc[jj];
                        const float yf = __uint_as_float((yv[jj] >> kj.z) + 0x4B000000u);
                        vf[jj % kPart] = fmaf(yf, __uint_as_float(kj.x), vf[jj % kPart]);
                        grp += static_cast<uint64_t>(yv[jj]) * kj.y;
                    }
                    t01 += grp;
                    t2 += t01 < grp ? 1u : 0u;
                }
                // Row m's 128 bytes in the 128-byte-swizzle layout
                // (sw128_offset); this half owns 16-byte pieces 4 h .. 4 h + 3.
                uint8_t* as = sm.slot + s * kSlot + m * 128;
                const bool last = c == nch - 1;
                if (last) {
                    // Row K: the multiplier v of -P mod q, from both halves'
                    // sums; the first half writes it (and its own pieces) once
                    // the second has written its pieces and sums.
                    const float vh = (vf[0] + vf[1]) + (vf[2] + vf[3]);
                    if (h == 1) {
#pragma unroll
                        for (int q4 = 0; q4 < 4; ++q4)
                            *reinterpret_cast<uint4*>(as + (((4 + q4) ^ (m & 7)) << 4)) =
                                make_uint4(yv[4 * q4], yv[4 * q4 + 1], yv[4 * q4 + 2], yv[4 * q4 + 3]);
                        sm.xch[m] = make_uint4(__float_as_uint(vh), static_cast<uint32_t>(t01),
                                               static_cast<uint32_t>(t01 >> 32), t2);
                    }
                    stagers_all(true);
                    if (h == 0) {
                        const uint4 x = sm.xch[m];
                        int v = __float2int_rn((vh + __uint_as_float(x.x)) - cc.voff);
                        v = v < 0 ? 0 : (v > K ? K : v);
                        const uint32_t vu = live ? static_cast<uint32_t>(v) : 0u;
                        const uint64_t other = (static_cast<uint64_t>(x.z) << 32) | x.y;
                        t01 += other;
                        t2 += x.w + (t01 < other ? 1u : 0u);
                        const uint64_t pv = static_cast<uint64_t>(vu) * sm.kc[K].y;
                        t01 += pv;
                        t2 += t01 < pv ? 1u : 0u;
                        const uint32_t kk = static_cast<uint32_t>(K) % kChunk;
#pragma unroll
                        for (int jj = 0; jj < kHalf; ++jj)
                            if (static_cast<uint32_t>(jj) == kk) yv[jj] = vu;
#pragma unroll
                        for (int q4 = 0; q4 < 4; ++q4)
                            *reinterpret_cast<uint4*>(as + ((q4 ^ (m & 7)) << 4)) =
                                make_uint4(yv[4 * q4], yv[4 * q4 + 1], yv[4 * q4 + 2], yv[4 * q4 + 3]);
                        if (kk >= static_cast<uint32_t>(kHalf))
                            *reinterpret_cast<uint32_t*>(as + (((kk >> 2) ^ (m & 7)) << 4) + 4 * (kk & 3)) = vu;
                    }
                } else {
#pragma unroll
                    for (int q4 = 0; q4 < 4; ++q4)
                        *reinterpret_cast<uint4*>(as + (((4 * h + q4) ^ (m & 7)) << 4)) =
                            make_uint4(yv[4 * q4], yv[4 * q4 + 1], yv[4 * q4 + 2], yv[4 * q4 + 3]);
                }
                tc::fence_proxy_async_smem();
                tc::mbar_arrive(&sm.a_full[s]);
                ++g;
            }
            if (!ok) break;
            const int p = i & 1;
            if (h == 0 && i >= 2) {
                ok = tc::wait_or_abort(&sm.m_empty[p], ((i - 2) >> 1) & 1, sm.abort, lim);
                ok = __all_sync(0xffffffffu, ok);
            }
            ok = stagers_all(ok);
            if (!ok) break;
            if (h == 0) {
                // Top-limb sum as three words.
                sm.meta[p * kCrtTile + m] =
                    make_uint4(static_cast<uint32_t>(t01), static_cast<uint32_t>(t01 >> 32), t2, 0u);
                tc::mbar_arrive(&sm.m_full[p]);
            }
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
            const double fq = xd * d.q_top_inv;
            const double f = floor(fq);
            const uint64_t e = f > 0 ? static_cast<uint64_t>(f) : 0;
            const uint32_t e_lo = static_cast<uint32_t>(e), e_hi = static_cast<uint32_t>(e >> 32);
            // With the fraction of the estimate at least 2^-8 from an integer,
            // e = floor(X / q) exactly and X - e q lies in [0, q); otherwise it
            // lies in [-q, 2q) and the row is checked after the pass.
            const double frac = fq - f;
            const bool near = !(frac >= 0x1p-8 && frac <= 1.0 - 0x1p-8);
            // One pass from the bottom.  X = Z0 + 2^8 Z1 + 2^16 Z2 + 2^24 Z3,
            // Z_s the number whose limb l is D[4 l + s] (< 2^26), so limb l of
            // 2^(8 s) Z_s is one funnel shift of Z_s[l - 1] and Z_s[l] and the
            // limb's share of X is z0 + s1 + s2 + s3 < 2^34 with no products.
            // e q enters as words: lo(e_lo q_l) + hi(e_lo q_(l-1)) +
            // lo(e_hi q_(l-1)) + hi(e_hi q_(l-2)).  Both are formed off the
            // carry chain; the chain itself is one signed 64-bit add a limb.
            // TMEM pieces are double-buffered: piece pc + 1 loads while piece
            // pc is used.
            uint64_t pp = 0, hp = 0, hp2 = 0;
            uint32_t z1p = 0, z2p = 0, z3p = 0;
            int64_t cy = 0;
            uint32_t o[4], over = 0;
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
                        const uint32_t z0 = have ? cur[4 * ii] : 0u, z1 = have ? cur[4 * ii + 1] : 0u;
                        const uint32_t z2 = have ? cur[4 * ii + 2] : 0u, z3 = have ? cur[4 * ii + 3] : 0u;
                        uint64_t sd = static_cast<uint64_t>(z0) + __funnelshift_l(z1p, z1, 8) +
                                      static_cast<uint64_t>(__funnelshift_l(z2p, z2, 16)) + __funnelshift_l(z3p, z3, 24);
                        z1p = z1;
                        z2p = z2;
                        z3p = z3;
                        if (kl == L - 1) sd += meta.x;
                        if (kl == L) sd += meta.y;
                        if (kl == L + 1) sd += meta.z;
                        const uint32_t qk = sm.qs[kl];
                        const uint64_t P = static_cast<uint64_t>(e_lo) * qk, H = static_cast<uint64_t>(e_hi) * qk;
                        const uint64_t t = (P & 0xFFFFFFFFu) + (pp >> 32) + (hp & 0xFFFFFFFFu) + (hp2 >> 32);
                        pp = P;
                        hp2 = hp;
                        hp = H;
                        const int64_t v = static_cast<int64_t>(sd) - static_cast<int64_t>(t) + cy;
                        cy = v >> 32;
                        const uint32_t yk = static_cast<uint32_t>(v);
                        o[ii] = yk;
                        if (kl < L) {
                            if (live) {
                                if (gvec) {
                                    if (ii == 3) *reinterpret_cast<uint4*>(crow + kl - 3) = make_uint4(o[0], o[1], o[2], o[3]);
                                } else {
                                    crow[kl] = yk;
                                }
                            }
                        } else {
                            over |= yk;   // limbs L and L + 1 of a non-negative result
                        }
                    }
                }
                if (more) tmem_wait(nxt);
            }
            // TMEM is read: the MMAs of this buffer's next tile may start.
            tc::tc_fence_before();
            tc::mbar_arrive(&sm.d_empty[grp]);
            // r = X - e q in [-q, 2q): negative (cy < 0) adds q; a row near an
            // integer quotient subtracts q when r >= q (r past limb L - 1, or
            // its low L limbs at least q).  Rare: a second pass over the row.
            if (live && (cy < 0 || near)) {
                bool sub = false;
                if (cy >= 0) {
                    sub = over != 0;
                    if (!sub) {
                        uint32_t cb = 0;
                        for (int kk = 0; kk < L; ++kk)
                            cb = static_cast<uint32_t>((static_cast<uint64_t>(crow[kk]) - sm.qs[kk] - cb) >> 63);
                        sub = cb == 0;
                    }
                }
                if (cy < 0 || sub) {
                    uint32_t cb = 0;
                    for (int kk = 0; kk < L; ++kk) {
                        const uint32_t x = crow[kk], qk = sm.qs[kk];
                        if (cy < 0) {
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
    // The rounding sum's constants and its error bound (see the head of
    // this file): truncation sum_j 2^sh_j / p_j, one rounding of a partial
    // sum per term, the final adds and voff's own rounding.
    double off = 0, trunc = 0, tmax = 0;
    for (int j = 0; j <= pl.K; ++j) {
        if (j < pl.K) {
            const uint32_t p = pl.primes[j];
            int bits = 0;
            while (bits < 32 && (p >> bits) != 0) ++bits;
            const uint32_t sh = bits > 23 ? static_cast<uint32_t>(bits - 23) : 0u;
            cc.sh[j] = sh;
            cc.cf[j] = static_cast<float>(std::ldexp(1.0, static_cast<int>(sh)) / p);
            off += 8388608.0 * static_cast<double>(cc.cf[j]);
            trunc += std::ldexp(1.0, static_cast<int>(sh)) / p;
            tmax += 2 * 8388608.0 * static_cast<double>(cc.cf[j]);
        }
        cc.top[j] = top[j];
    }
    cc.voff = static_cast<float>(off);
    const double ulp = std::ldexp(1.0, -24);
    cc.est_err = static_cast<float>(trunc + (pl.K + 4) * tmax * ulp + off * ulp);
    for (int k = 0; k < pl.L; ++k) cc.q[k] = pl.q[k];
    return cc;
}

bool crt_pipe_supported(const DevPoint& d, const CrtConsts& cc, const uint32_t* Y, uint32_t n_begin,
                        uint32_t n_end) {
    // TMA boxes of y: 16-byte aligned base, row pitch (N words) and column
    // coordinates (n_begin) a multiple of 4 words; the constants resident.
    return d.L >= 2 && d.crt_u <= 256 && d.K + 1 <= kMaxK && d.crt_img_v && (d.N & 3) == 0 && d.N >= kCrtTile &&
           (n_begin & 3) == 0 && n_end <= d.N && (reinterpret_cast<uintptr_t>(Y) & 15) == 0 &&
           make_layout(d.K, d.crt_u).bytes() <= kSmemLimit && cc.est_err < 0.25f;
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
