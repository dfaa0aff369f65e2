// Decompose on the tensor cores as a persistent, warp-specialised pipeline.
//
// Same arithmetic as decompose_tc.cu (reference decompose_many rns.cuh:110-128):
//
//     D[m][4j + s] = sum_k byte_k(x_m) * byte_s(2^(8k) sigma_j mod p_j)   (< 2^24)
//     x_m mod p_j  = (sum_s D[m][4j + s] 2^(8s)) mod p_j
//
// Organisation on the B200: one CTA per SM works on one operand (a pair launch
// splits the CTAs between a and b) and walks its 128-coefficient tiles:
//   * warp 0 loads the operand's whole constant image once (chunks of 64
//     primes x 4 bytes x 4L bytes, the last one packed: at most 160 KB,
//     resident in shared memory) and then, one thread, issues the MMAs at the
//     widest shape (N = 256 columns per chunk): D goes to one of two
//     256-column TMEM buffers;
//   * warps 1-4 copy each tile's limbs into a ring of two slots in the MMA's
//     128-byte-swizzled K-major layout (the layout the tensor cores read at
//     full rate) with asynchronous copies (cp.async) whose completion the
//     slot's mbarrier tracks (cp.async.mbarrier.arrive), so a slot is handed
//     to the MMAs the moment its copies land: a warp moves 8 rows x 4
//     sixteen-byte groups at a time, so the global loads are 64-byte runs and
//     the eight lanes of each shared-store phase hit eight different bank
//     groups;
//   * warps 5-20, four per TMEM lane quadrant, one coefficient per thread,
//     each take 16 of a chunk's 64 primes: read D, fold the 49-bit sums mod
//     p_j and store the residues (a warp writes 32 consecutive words per
//     prime).
// The fold constants come from kernel parameters.  Every wait is bounded
// (DevPoint::wait_ns); a timeout raises an abort flag that every role checks,
// and the error word gets bit 0.
#include "device.cuh"
#include "kernels.h"
#include "pdl.cuh"
#include "tc.cuh"

namespace fpm {

namespace {

constexpr int kThreads = 672;                      // 21 warps
constexpr int kLoadWarp0 = 1;                      // warps 1-4
constexpr int kLoaders = 128;
constexpr int kEpiWarp0 = 5;                       // warps 5-20
constexpr int kEpi = 512;
constexpr uint32_t kRows = 128;
constexpr uint32_t kCols = 256;                    // GEMM columns per full chunk (64 primes)

// Operand tiles and the constant image in the 128-byte-swizzle layout
// (sw128_offset): a tile is 128 rows, a constant chunk 256 columns (the last
// nlast), each with kb K bytes.
__host__ __device__ inline uint32_t a_bytes(uint32_t kb) { return static_cast<uint32_t>(sw128_bytes(kRows, kb)); }
__host__ __device__ inline size_t b_bytes(uint32_t kb, int nch, uint32_t nlast) {
    return (static_cast<size_t>(nch) - 1) * sw128_bytes(kCols, kb) + sw128_bytes(nlast, kb);
}
__host__ inline size_t smem_bytes(uint32_t kb, int nch, uint32_t nlast) {
    return b_bytes(kb, nch, nlast) + 2 * a_bytes(kb) + 128;
}

struct Smem {
    uint8_t* b;            // resident constant image
    uint8_t* a;            // [2] operand tiles
    uint64_t* b_full;      // [1]
    uint64_t* a_full;      // [2]
    uint64_t* a_empty;     // [2]
    uint64_t* d_full;      // [2]
    uint64_t* d_empty;     // [2]
    uint32_t* tmem_base;
    volatile uint32_t* abort;
};

__device__ inline Smem carve(uint8_t* base, uint32_t kb, int nch, uint32_t nlast) {
    Smem s;
    s.b = base;
    s.a = base + b_bytes(kb, nch, nlast);
    uint64_t* bars = reinterpret_cast<uint64_t*>(s.a + 2 * a_bytes(kb));
    s.b_full = bars;
    s.a_full = bars + 1;
    s.a_empty = bars + 3;
    s.d_full = bars + 5;
    s.d_empty = bars + 7;
    s.tmem_base = reinterpret_cast<uint32_t*>(bars + 9);
    s.abort = s.tmem_base + 1;
    return s;
}

// Asynchronous global -> shared copies of 16 or 4 bytes; with have == false
// nothing is read and the destination is zero-filled.
__device__ __forceinline__ void cp_async16_zfill(void* dst, const void* src, bool have) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(tc::smem_addr(dst)), "l"(src),
                 "r"(have ? 16u : 0u)
                 : "memory");
}
__device__ __forceinline__ void cp_async4_zfill(void* dst, const void* src, bool have) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(tc::smem_addr(dst)), "l"(src),
                 "r"(have ? 4u : 0u)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// One arrival on `bar` once every cp.async this thread issued so far has
// completed (the barrier's count includes it: .noinc).
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(tc::smem_addr(bar)) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Waits for this thread's two 32-column TMEM loads; naming the registers
// keeps every read of them below the wait.
#define FPM_R16(x, o) "+r"(x[o + 0]), "+r"(x[o + 1]), "+r"(x[o + 2]), "+r"(x[o + 3]), "+r"(x[o + 4]), \
    "+r"(x[o + 5]), "+r"(x[o + 6]), "+r"(x[o + 7]), "+r"(x[o + 8]), "+r"(x[o + 9]), "+r"(x[o + 10]), \
    "+r"(x[o + 11]), "+r"(x[o + 12]), "+r"(x[o + 13]), "+r"(x[o + 14]), "+r"(x[o + 15])
__device__ __forceinline__ void tmem_wait2(uint32_t (&r)[2][32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" : FPM_R16(r[0], 0)::"memory");
    asm volatile("" : FPM_R16(r[0], 16)::"memory");
    asm volatile("" : FPM_R16(r[1], 0)::"memory");
    asm volatile("" : FPM_R16(r[1], 16)::"memory");
}
#undef FPM_R16

// A GEMM sum D is below 4L 255^2 <= 256 * 65025 (L <= 64), so both halves of
// sum_s D_s 2^(8s), A = D_0 + 2^8 D_1 and B = D_2 + 2^8 D_3, are below
// 257 * 256 * 65025 < 2^32, and the residue is (A + B 2^16) mod p:
// f = {p, 2^16 mod p, its Shoup companion, floor(2^32 / p)}.  LAZY leaves a
// value below 4p, congruent to the same residue, for a transform whose first
// butterflies take lazy input.
static_assert(kMaxL <= 64, "D_0 + 2^8 D_1 must fit 32 bits");
template <bool LAZY>
__device__ __forceinline__ uint32_t fold_halves(uint32_t A, uint32_t B, uint4 f) {
    if constexpr (LAZY) {
        // (A - q1 p) + (B f.y - q2 p), each term in [0, 2p) (Shoup): one
        // product by p for both quotients, the same value below 4p.
        const uint32_t q = mulhi32(A, f.w) + mulhi32(B, f.z);
        return B * f.y + A - q * f.x;
    } else {
        return add_mod(shoup(A, 1u, f.w, f.x), shoup(B, f.y, f.z, f.x), f.x);
    }
}

// CTAs [0, split) take operand 0 (la -> ra), [split, gridDim.x) operand 1.
template <bool LAZY>
__global__ void __launch_bounds__(kThreads, 1)
    k_decompose_pipe(DevPoint d, const __grid_constant__ DecConsts fc, const uint32_t* __restrict__ la,
                     const uint32_t* __restrict__ lb, uint32_t* __restrict__ ra, uint32_t* __restrict__ rb,
                     int operand0, uint32_t n_begin, uint32_t n_end, uint32_t split) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    pdl_launch_dependents();
    // The 128-byte swizzle is a function of the shared address: the
    // operand atoms need a 1024-byte aligned base (error bit 4 otherwise).
    if (tc::smem_addr(smem_raw) & 1023u) {
        if (threadIdx.x == 0) atomicOr(d.err, 4u);
        return;
    }
    const uint32_t kb = d.dec_kb;
    const int nch = static_cast<int>(fc.chunks);
    const uint32_t nlast = fc.last_cols;
    const Smem sm = carve(smem_raw, kb, nch, nlast);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int L = d.L, K = d.K;
    const bool second = blockIdx.x >= split;
    const int operand = operand0 + (second ? 1 : 0);
    const uint32_t* limbs = second ? lb : la;
    uint32_t* res = second ? rb : ra;
    const uint8_t* img = fc.img[operand];
    const uint32_t g0 = second ? split : 0, gs = second ? gridDim.x - split : split;
    const uint32_t tiles = (n_end - n_begin + kRows - 1) / kRows;
    const uint32_t chunk_bytes = static_cast<uint32_t>(sw128_bytes(kCols, kb));
    const uint64_t lim = d.wait_ns;

    if (threadIdx.x == 0) {
        tc::mbar_init(sm.b_full, 1);
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&sm.a_full[i], kLoaders);
            tc::mbar_init(&sm.a_empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&sm.d_full[i], 1);
            tc::mbar_init(&sm.d_empty[i], kEpi);
        }
        *sm.abort = 0;
        tc::fence_mbar_init();
        // The constant image is read-only plan data: it loads under the
        // preceding kernel's tail.
        // (Test hook: with kFaultDecompose the image is never requested, so the
        // MMA issuer's wait for it runs out.)
        const uint32_t total = static_cast<uint32_t>(b_bytes(kb, nch, nlast));
        if (!(d.fault & kFaultDecompose)) {
            tc::mbar_arrive_expect_tx(sm.b_full, total);
            for (uint32_t off = 0; off < total; off += chunk_bytes) {
                const uint32_t n = total - off < chunk_bytes ? total - off : chunk_bytes;
                tc::bulk_g2s(sm.b + off, img + off, n, sm.b_full);
            }
        }
    }
    if (warp == 0) tc::tmem_alloc(sm.tmem_base, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *sm.tmem_base;
    pdl_wait();   // the limbs and the residues belong to the kernels around this one

    if (warp == 0) {
        // ---- MMA issuer ----
        if (lane == 0) {
            const uint32_t idesc_full = tc::idesc_u8(kCols), idesc_last = tc::idesc_u8(nlast);
            bool ok = tc::wait_or_abort(sm.b_full, 0, sm.abort, lim);
            uint64_t* last_bar = nullptr;   // the barrier of the latest commit
            uint32_t last_par = 0;
            uint32_t g = 0, i = 0;
            for (uint32_t t = blockIdx.x - g0; ok && t < tiles; t += gs, ++i) {
                const int s = i & 1;
                ok = tc::wait_or_abort(&sm.a_full[s], (i >> 1) & 1, sm.abort, lim);
                if (!ok) break;
                // The limbs came through the generic proxy (cp.async).
                tc::fence_proxy_async_smem();
                const uint32_t a0 = tc::smem_addr(sm.a + s * a_bytes(kb));
                for (int c = 0; c < nch; ++c, ++g) {
                    const int buf = g & 1;
                    if (g >= 2) {
                        ok = tc::wait_or_abort(&sm.d_empty[buf], ((g - 2) >> 1) & 1, sm.abort, lim);
                        if (!ok) break;
                    }
                    tc::tc_fence_after();
                    const bool lastc = c == nch - 1;
                    const uint32_t cols = lastc ? nlast : kCols;
                    const uint32_t b0 = tc::smem_addr(sm.b + c * chunk_bytes);
                    for (uint32_t kk = 0; kk < kb / 32; ++kk) {
                        const uint32_t half = kk >> 2, step = (kk & 3) * 32;
                        const uint64_t ad = tc::smem_desc_sw128(a0 + half * kRows * 128 + step);
                        const uint64_t bd = tc::smem_desc_sw128(b0 + half * cols * 128 + step);
                        tc::mma_u8(tmem + buf * kCols, ad, bd, lastc ? idesc_last : idesc_full, kk > 0);
                    }
                    tc::mma_commit(&sm.d_full[buf]);
                    last_bar = &sm.d_full[buf];
                    last_par = (g >> 1) & 1;
                }
                if (!ok) break;
                tc::mma_commit(&sm.a_empty[s]);
                last_bar = &sm.a_empty[s];
                last_par = (i >> 1) & 1;
            }
            // MMAs still running must finish before the CTA may exit.
            if (last_bar) tc::wait_parity(last_bar, last_par, lim);
            // So must the constant image, if an abort came before it landed.
            if (!(d.fault & kFaultDecompose)) tc::wait_parity(sm.b_full, 0, lim);
        }
        __syncwarp();
    } else if (warp < kEpiWarp0) {
        // ---- loaders: each tile's limbs, K-major with a padded K stride ----
        // The copies go from global to shared memory asynchronously (cp.async,
        // zero-filled where a position has no limb: rows past nk, limbs past
        // L), so one whole tile is in flight while the previous one completes.
        // A warp covers an 8-row x 4-group block per instruction: every lane
        // group of a shared-store phase hits distinct banks.
        const uint32_t lt = threadIdx.x - kLoadWarp0 * 32, lw = lt >> 5;
        const bool vec = (reinterpret_cast<uintptr_t>(limbs) & 15u) == 0 && (L & 3) == 0;
        const uint32_t G = kb / 16;                    // 16-byte K groups per row
        const uint32_t r = lane & 7, gi = lane >> 3;   // row in block, group (or limb) in block
        const uint32_t gbs = (G + 3) / 4;
        uint32_t i = 0;
        bool ok = true;
        for (uint32_t t = blockIdx.x - g0; t < tiles; t += gs, ++i) {
            const int s = i & 1;
            if (i >= 2) {
                ok = tc::wait_or_abort(&sm.a_empty[s], ((i - 2) >> 1) & 1, sm.abort, lim);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
            }
            uint8_t* at = sm.a + s * a_bytes(kb);
            const uint32_t n0 = n_begin + t * kRows;
            const uint32_t nk = min(kRows, n_end - n0);
            if (vec) {
                // Block (mb, gb): rows 8 mb .. + 7, 16-byte groups 4 gb .. + 3
                // (group gq of a row is limbs 4 gq .. 4 gq + 3).
                const uint32_t q4 = static_cast<uint32_t>(L) / 4;
                const uint4* src4 = reinterpret_cast<const uint4*>(limbs + static_cast<size_t>(n0) * L);
                for (uint32_t blk = lw; blk < 16 * gbs; blk += kLoaders / 32) {
                    const uint32_t mm = 8 * (blk & 15) + r, gq = 4 * (blk >> 4) + gi;
                    if (gq < G) {
                        const bool have = mm < nk && gq < q4;
                        cp_async16_zfill(at + sw128_offset(mm, 16 * gq, kRows), have ? src4 + mm * q4 + gq : src4,
                                         have);
                    }
                }
            } else {
                // Block (mb, gq): rows 8 mb .. + 7, limbs 4 gq .. 4 gq + 3.
                const uint32_t* src = limbs + static_cast<size_t>(n0) * L;
                for (uint32_t blk = lw; blk < 16 * G; blk += kLoaders / 32) {
                    const uint32_t mm = 8 * (blk & 15) + r, l = 4 * (blk >> 4) + gi;
                    const bool have = mm < nk && l < static_cast<uint32_t>(L);
                    cp_async4_zfill(at + sw128_offset(mm, 4 * l, kRows), have ? src + mm * L + l : src, have);
                }
            }
            // The slot's barrier completes when this thread's copies have
            // landed (the hardware arrives for it), so the loader goes on to
            // the next slot at once; the MMA issuer fences the async proxy.
            cp_async_commit();
            cp_async_arrive_noinc(&sm.a_full[s]);
        }
        // Whatever is still in flight lands before the CTA may exit.
        cp_async_wait<0>();
    } else {
        // ---- epilogue: thread = one coefficient, 16 primes of each chunk ----
        const int ew = warp - kEpiWarp0;
        const uint32_t qd = warp & 3, piece = ew >> 2;
        const uint32_t m = qd * 32 + lane;
        const uint32_t tq = tmem + ((qd * 32) << 16) + piece * 64;
        uint32_t g = 0;
        for (uint32_t t = blockIdx.x - g0; t < tiles; t += gs) {
            const uint32_t n0 = n_begin + t * kRows;
            const bool live = m < min(kRows, n_end - n0);
            bool ok = true;
            for (int c = 0; c < nch; ++c, ++g) {
                const int buf = g & 1;
                ok = tc::wait_or_abort(&sm.d_full[buf], (g >> 1) & 1, sm.abort, lim);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
                tc::tc_fence_after();
                const int j0 = c * 64 + static_cast<int>(piece) * 16;
                uint32_t r[2][32];
                tc::tmem_ld32(tq + buf * kCols, r[0]);
                tc::tmem_ld32(tq + buf * kCols + 32, r[1]);
                tmem_wait2(r);
                // The 32 half-sums are formed before the buffer is released:
                // half as many values stay live through the folds.
                uint32_t hs[16][2];
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    const uint32_t* rr = r[k >> 3] + 4 * (k & 7);
                    hs[k][0] = rr[0] + (rr[1] << 8);
                    hs[k][1] = rr[2] + (rr[3] << 8);
                }
                tc::tc_fence_before();
                tc::mbar_arrive(&sm.d_empty[buf]);
                if (j0 < K) {
                    // One running pointer down the primes' rows (no 64-bit
                    // product per store).
                    uint32_t* out = res + static_cast<size_t>(j0) * d.N + n0 + m;
                    const size_t stride = d.N;
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const int j = j0 + k;
                        if (live && j < K) *out = fold_halves<LAZY>(hs[k][0], hs[k][1], fc.fold[j]);
                        out += stride;
                    }
                }
            }
            if (!ok) break;
        }
    }

    tc::tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *sm.abort) atomicOr(d.err, 1u);
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 512);
    }
}

}  // namespace

DecConsts make_dec_consts(const HostPlan& pl, const uint8_t* img_a, const uint8_t* img_b) {
    DecConsts dc{};
    for (int j = 0; j < pl.K; ++j) dc.fold[j] = pl.dec_fold[j];
    dc.img[0] = img_a;
    dc.img[1] = img_b;
    dc.chunks = pl.dec_wchunks;
    dc.last_cols = pl.dec_wlast;
    // The four-step transforms start with lazy butterflies; the one-block
    // transform (N <= 1024) and the full-reduction window want canonical input.
    dc.lazy_out = pl.lazy && pl.g.logN > kSmallLogN ? 1u : 0u;
    return dc;
}

bool decompose_pipe_supported(const HostPlan& pl) {
    return pl.K <= kMaxK && pl.dec_wchunks >= 1 && pl.dec_wlast >= 16 && pl.dec_wlast <= 256 &&
           smem_bytes(pl.dec_kb, static_cast<int>(pl.dec_wchunks), pl.dec_wlast) <= 227 * 1024;
}

void decompose_pipe_init_attributes() {
    check(cudaFuncSetAttribute(k_decompose_pipe<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024),
          "decompose_pipe smem");
    check(cudaFuncSetAttribute(k_decompose_pipe<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024),
          "decompose_pipe smem");
}

void launch_decompose_pipe(const DevPoint& d, const DecConsts& dc, const uint32_t* a, const uint32_t* b,
                           uint32_t* A, uint32_t* B, int operand0, uint32_t n_begin, uint32_t n_end, int sms,
                           cudaStream_t st) {
    if (n_end <= n_begin) return;
    const uint32_t tiles = (n_end - n_begin + kRows - 1) / kRows;
    const int operands = b ? 2 : 1;
    // CTAs per operand: one per SM in all, no more than the operand's tiles.
    uint32_t per = static_cast<uint32_t>(sms) / operands;
    if (per < 1) per = 1;
    if (per > tiles) per = tiles;
    const uint32_t grid = per * operands;
    const uint32_t split = operands == 2 ? per : grid;
    check(launch_pdl(dc.lazy_out ? k_decompose_pipe<true> : k_decompose_pipe<false>, dim3(grid), dim3(kThreads),
                     smem_bytes(d.dec_kb, static_cast<int>(dc.chunks), dc.last_cols), st, d, dc, a,
                     b ? b : a, A, B ? B : A, operand0, n_begin, n_end, split),
          "decompose launch");
}

}  // namespace fpm
