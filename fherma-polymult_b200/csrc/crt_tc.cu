// CRT on the 5th-generation tensor cores (tcgen05, kind::i8).
//
// c mod q = sum_j y_j M_j + negvP_v (mod q), M_j = P/p_j mod q,
// v = round(sum_j y_j / p_j) (reference CrtView, rns.cuh:225-240; crt_columns /
// crt_combine, rns_kernels.cuh:265-364).
//
// The big sum X = sum_j y_j M_j (K 31-bit words times K L-limb constants per
// coefficient) is split as X = Xlow + Xtop 2^(32(L-1)), Xtop = sum_j y_j M_j[L-1].
// Xlow is an 8-bit GEMM:
//
//     D[m][u] = sum_{j,s} byte_s(y_j(m)) * byte_{u-s}(Mlow_j)     (u < 4L - 1)
//     Xlow(m) = sum_u D[m][u] 2^(8u)
//
// (A: the y bytes of 128 coefficients, K-major; B: a prebuilt image of the M
// bytes with each prime's four byte-shifts, so one GEMM column is one byte
// position; every D entry is below 4K 255^2 < 2^26.)  Keeping the top limb of M
// out of the GEMM holds D to at most 256 TMEM columns; the epilogue adds Xtop,
// which it accumulates on the CUDA cores while staging y, together with the
// double-precision rounding sum for v.
//
// Block = 128 coefficients (MMA M), 160 threads:
//   warp 0      : TMEM allocation, B chunk copies, MMA issue (one thread)
//   warps 1 - 4 : thread = coefficient row: stage y into the A slots chunk by
//                 chunk (32 primes), then the epilogue: carries over D, Xtop,
//                 negvP_v, reduction mod q, coalesced store of the limbs.
#include "device.cuh"
#include "kernels.h"
#include "tc.cuh"

namespace fpm {

namespace {

constexpr int kThreads = 160;
constexpr uint32_t kRows = 128;
constexpr uint32_t kChunk = 32;                     // primes per K-chunk (128 A bytes per row)
constexpr uint32_t kASlot = kRows * kChunk * 4;     // 16 KB: [8 core columns][128 rows][16 B]

struct Smem {
    uint8_t* a[2];
    uint8_t* b[2];
    uint32_t* x;           // epilogue limbs, [128][L + 2] (aliases the slots)
    uint64_t* a_full;      // [2] 128 arrivals
    uint64_t* b_full;      // [2] bulk copy landed
    uint64_t* mma_done;    // [2] chunk's MMAs finished (slots free)
    uint64_t* d_ready;     // all MMAs finished
    uint32_t* tmem_base;
};

__host__ __device__ inline uint32_t slots_bytes(uint32_t u) { return 2 * kASlot + 2 * u * 128; }

__device__ inline Smem carve(uint8_t* base, uint32_t u) {
    Smem s;
    s.a[0] = base;
    s.a[1] = base + kASlot;
    s.b[0] = base + 2 * kASlot;
    s.b[1] = s.b[0] + u * 128;
    s.x = reinterpret_cast<uint32_t*>(base);
    uint8_t* tail = base + ((slots_bytes(u) > kRows * (kMaxL + 2) * 4 ? slots_bytes(u) : kRows * (kMaxL + 2) * 4));
    s.a_full = reinterpret_cast<uint64_t*>(tail);
    s.b_full = s.a_full + 2;
    s.mma_done = s.a_full + 4;
    s.d_ready = s.a_full + 6;
    s.tmem_base = reinterpret_cast<uint32_t*>(s.a_full + 7);
    return s;
}

__global__ void __launch_bounds__(kThreads)
    k_crt_tc(DevPoint d, const uint32_t* __restrict__ Y, uint32_t* __restrict__ C) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t U = d.crt_u;            // GEMM columns (byte positions), multiple of 32, <= 256
    const int nch = (d.K + kChunk - 1) / kChunk;
    const Smem sm = carve(smem_raw, U);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n0 = blockIdx.x * kRows;
    const uint32_t nk = min(kRows, d.N - n0);
    const int L = d.L, K = d.K;
    const uint32_t tcols = d.crt_tmem_cols;

    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&sm.a_full[i], kRows);
            tc::mbar_init(&sm.b_full[i], 1);
            tc::mbar_init(&sm.mma_done[i], 1);
        }
        tc::mbar_init(sm.d_ready, 1);
        tc::fence_mbar_init();
    }
    if (warp == 0) tc::tmem_alloc(sm.tmem_base, tcols);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *sm.tmem_base;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            const uint32_t chunk_bytes = U * 128;
            const int pre = nch < 2 ? nch : 2;
            for (int c = 0; c < pre; ++c) {
                tc::mbar_arrive_expect_tx(&sm.b_full[c], chunk_bytes);
                tc::bulk_g2s(sm.b[c], d.crt_img + static_cast<size_t>(c) * chunk_bytes, chunk_bytes, &sm.b_full[c]);
            }
            const uint32_t idesc = tc::idesc_u8(U);
            for (int c = 0; c < nch && ok; ++c) {
                const int s = c & 1;
                ok = tc::wait_parity(&sm.b_full[s], (c >> 1) & 1) && tc::wait_parity(&sm.a_full[s], (c >> 1) & 1);
                if (!ok) break;
                tc::tc_fence_after();
                const uint32_t a0 = tc::smem_addr(sm.a[s]), b0 = tc::smem_addr(sm.b[s]);
                for (uint32_t kk = 0; kk < 4; ++kk) {
                    const uint64_t ad = tc::smem_desc(a0 + kk * 2 * (kRows * 16), kRows * 16, 128);
                    const uint64_t bd = tc::smem_desc(b0 + kk * 2 * (U * 16), U * 16, 128);
                    tc::mma_u8(tmem, ad, bd, idesc, c > 0 || kk > 0);
                }
                tc::mma_commit(&sm.mma_done[s]);
                if (c >= 1 && c + 1 < nch) {
                    const int s1 = (c - 1) & 1;
                    ok = tc::wait_parity(&sm.mma_done[s1], ((c - 1) >> 1) & 1);
                    if (!ok) break;
                    tc::mbar_arrive_expect_tx(&sm.b_full[s1], chunk_bytes);
                    tc::bulk_g2s(sm.b[s1], d.crt_img + static_cast<size_t>(c + 1) * chunk_bytes, chunk_bytes,
                                 &sm.b_full[s1]);
                }
            }
            if (ok) tc::mma_commit(sm.d_ready);
        }
        __syncwarp();
    } else {
        const uint32_t q = warp & 3;
        const uint32_t m = q * 32 + lane;
        const bool live = m < nk;
        double frac = 0;
        uint64_t top_lo = 0, top_hi = 0;   // Xtop = top_lo + top_hi 2^32
        for (int c = 0; c < nch; ++c) {
            const int s = c & 1;
            if (c >= 2) {
                ok = tc::wait_parity(&sm.mma_done[s], ((c - 2) >> 1) & 1);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
            }
            uint8_t* slot = sm.a[s];
#pragma unroll
            for (int g = 0; g < 8; ++g) {
                uint32_t w[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int j = c * kChunk + g * 4 + t;
                    uint32_t y = 0;
                    if (j < K && live) {
                        y = Y[static_cast<size_t>(j) * d.N + n0 + m];
                        frac += static_cast<double>(y) * d.p_recip[j];
                        const uint64_t prod = static_cast<uint64_t>(y) * d.M[static_cast<size_t>(j) * L + L - 1];
                        top_lo += static_cast<uint32_t>(prod);
                        top_hi += prod >> 32;
                    }
                    w[t] = y;
                }
                *reinterpret_cast<uint4*>(slot + g * (kRows * 16) + m * 16) = make_uint4(w[0], w[1], w[2], w[3]);
            }
            tc::fence_proxy_async_smem();
            tc::mbar_arrive(&sm.a_full[s]);
        }
        if (ok) {
            ok = tc::wait_parity(sm.d_ready, 0);
            ok = __all_sync(0xffffffffu, ok);
        }
        if (ok) {
            tc::tc_fence_after();
            int v = static_cast<int>(floor(frac + 0.5));
            v = v < 0 ? 0 : (v > K ? K : v);
            const uint32_t* nv = d.negvP + static_cast<size_t>(v) * L;
            const uint64_t t1 = (top_lo >> 32) + top_hi;   // Xtop = lo32(top_lo) + t1 2^32
            const uint32_t tq = tmem + ((q * 32) << 16);
            uint32_t* x = sm.x + m * (L + 2);
            uint64_t carry = 0;
            // Limbs from D, 8 per 32-column piece, then the limbs above D.
            for (uint32_t piece = 0; piece < U / 32; ++piece) {
                uint32_t r[32];
                tc::tmem_ld32(tq + piece * 32, r);
                tc::tmem_ld_wait();
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int l = piece * 8 + i;
                    if (l >= L + 2) break;
                    uint64_t w = carry + static_cast<uint64_t>(r[4 * i]) + (static_cast<uint64_t>(r[4 * i + 1]) << 8) +
                                 (static_cast<uint64_t>(r[4 * i + 2]) << 16) +
                                 (static_cast<uint64_t>(r[4 * i + 3]) << 24);
                    if (l < L) w += nv[l];
                    if (l == L - 1) w += static_cast<uint32_t>(top_lo);
                    if (l == L) w += static_cast<uint32_t>(t1);
                    if (l == L + 1) w += t1 >> 32;
                    x[l] = static_cast<uint32_t>(w);
                    carry = w >> 32;
                }
            }
            for (int l = static_cast<int>(U / 4); l < L + 2; ++l) {
                uint64_t w = carry;
                if (l < L) w += nv[l];
                if (l == L - 1) w += static_cast<uint32_t>(top_lo);
                if (l == L) w += static_cast<uint32_t>(t1);
                if (l == L + 1) w += t1 >> 32;
                x[l] = static_cast<uint32_t>(w);
                carry = w >> 32;
            }
            reduce_mod_q(x, L + 2, d.q, L, d.q_top);
        }
    }

    if (!ok) atomicOr(d.err, 2u);
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, tcols);
    }
    uint32_t* out = C + static_cast<size_t>(n0) * L;
    for (uint32_t i = threadIdx.x; i < nk * static_cast<uint32_t>(L); i += kThreads) {
        const uint32_t row = i / L, l = i - row * L;
        out[i] = sm.x[row * (L + 2) + l];
    }
}

// Large enough that the blocks sharing an SM never ask for more than its 512
// TMEM columns in total.
size_t smem_bytes(uint32_t u, uint32_t tmem_cols) {
    const size_t body = slots_bytes(u) > kRows * (kMaxL + 2) * 4 ? slots_bytes(u) : kRows * (kMaxL + 2) * 4;
    const size_t need = body + 8 * sizeof(uint64_t);
    const size_t per_sm = 228 * 1024;
    const size_t floor_bytes = per_sm / (512 / tmem_cols + 1) + 1024;
    return need > floor_bytes ? need : floor_bytes;
}

}  // namespace

void crt_tc_init_attributes() {
    check(cudaFuncSetAttribute(k_crt_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem_bytes(256, 256))),
          "crt_tc smem");
}

void launch_crt_tc(const DevPoint& d, const uint32_t* Y, uint32_t* c, cudaStream_t st) {
    const uint32_t blocks = (d.N + kRows - 1) / kRows;
    k_crt_tc<<<blocks, kThreads, smem_bytes(d.crt_u, d.crt_tmem_cols), st>>>(d, Y, c);
}

}  // namespace fpm
