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
#include "group.cuh"
#include "kernels.h"
#include "tc.cuh"

namespace fpm {

namespace {

constexpr int kThreads = 160;
constexpr uint32_t kRows = 128;
constexpr uint32_t kChunk = 32;                     // primes per K-chunk (128 A bytes per row)
constexpr uint32_t kASlot = kRows * kChunk * 4;     // 16 KB: [8 core columns][128 rows][16 B]

struct Smem {
    uint8_t* a0;           // A slot s at a0 + s * kASlot
    uint8_t* b0;           // B slot s at b0 + s * u * 128
    uint32_t* x;           // output limbs, [128][L + 2] (aliases the slots)
    uint64_t* a_full;      // [2] 128 arrivals
    uint64_t* b_full;      // [2] bulk copy landed
    uint64_t* mma_done;    // [2] chunk's MMAs finished (slots free)
    uint64_t* d_ready;     // all MMAs finished
    uint32_t* tmem_base;
    double* p_recip;       // [kMaxK] 1 / p_j
    uint32_t* m_top;       // [kMaxK] M_j[L - 1]
    uint32_t* q;           // [kMaxL]
};

__host__ __device__ inline uint32_t slots_bytes(uint32_t u) { return 2 * kASlot + 2 * u * 128; }
__host__ __device__ inline uint32_t body_bytes(uint32_t u) {
    return slots_bytes(u) > kRows * (kMaxL + 2) * 4 ? slots_bytes(u) : kRows * (kMaxL + 2) * 4;
}
constexpr uint32_t kTailBytes = 64 + kMaxK * 8 + kMaxK * 4 + kMaxL * 4;

__device__ inline Smem carve(uint8_t* base, uint32_t u) {
    Smem s;
    s.a0 = base;
    s.b0 = base + 2 * kASlot;
    s.x = reinterpret_cast<uint32_t*>(base);
    uint8_t* tail = base + body_bytes(u);
    s.a_full = reinterpret_cast<uint64_t*>(tail);
    s.b_full = s.a_full + 2;
    s.mma_done = s.a_full + 4;
    s.d_ready = s.a_full + 6;
    s.tmem_base = reinterpret_cast<uint32_t*>(s.a_full + 7);
    s.p_recip = reinterpret_cast<double*>(tail + 64);
    s.m_top = reinterpret_cast<uint32_t*>(s.p_recip + kMaxK);
    s.q = s.m_top + kMaxK;
    return s;
}

constexpr int kX = kMaxL + 2;   // register limbs of the epilogue (predicated to L + 2)

// Coefficients n0 .. n0 + nk - 1 (nk <= 128).
__device__ __forceinline__ void crt_body(const DevPoint& d, const uint32_t* __restrict__ Y, uint32_t* __restrict__ C,
                                         uint32_t n0, uint32_t nk) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t U = d.crt_u;            // GEMM columns (byte positions), multiple of 32, <= 256
    const int nch = (d.K + kChunk - 1) / kChunk;
    const Smem sm = carve(smem_raw, U);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
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
    for (int j = threadIdx.x; j < K; j += kThreads) {
        sm.p_recip[j] = d.p_recip[j];
        sm.m_top[j] = d.M[static_cast<size_t>(j) * L + L - 1];
    }
    for (int l = threadIdx.x; l < L; l += kThreads) sm.q[l] = d.q[l];
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
                tc::bulk_g2s(sm.b0 + c * chunk_bytes, d.crt_img + static_cast<size_t>(c) * chunk_bytes, chunk_bytes, &sm.b_full[c]);
            }
            const uint32_t idesc = tc::idesc_u8(U);
            for (int c = 0; c < nch && ok; ++c) {
                const int s = c & 1;
                ok = tc::wait_parity(&sm.b_full[s], (c >> 1) & 1, d.wait_ns) && tc::wait_parity(&sm.a_full[s], (c >> 1) & 1, d.wait_ns);
                if (!ok) break;
                tc::tc_fence_after();
                const uint32_t a0 = tc::smem_addr(sm.a0 + s * kASlot), b0 = tc::smem_addr(sm.b0 + s * chunk_bytes);
                for (uint32_t kk = 0; kk < 4; ++kk) {
                    const uint64_t ad = tc::smem_desc(a0 + kk * 2 * (kRows * 16), kRows * 16, 128);
                    const uint64_t bd = tc::smem_desc(b0 + kk * 2 * (U * 16), U * 16, 128);
                    tc::mma_u8(tmem, ad, bd, idesc, c > 0 || kk > 0);
                }
                tc::mma_commit(&sm.mma_done[s]);
                if (c >= 1 && c + 1 < nch) {
                    const int s1 = (c - 1) & 1;
                    ok = tc::wait_parity(&sm.mma_done[s1], ((c - 1) >> 1) & 1, d.wait_ns);
                    if (!ok) break;
                    tc::mbar_arrive_expect_tx(&sm.b_full[s1], chunk_bytes);
                    tc::bulk_g2s(sm.b0 + s1 * chunk_bytes, d.crt_img + static_cast<size_t>(c + 1) * chunk_bytes, chunk_bytes,
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
                ok = tc::wait_parity(&sm.mma_done[s], ((c - 2) >> 1) & 1, d.wait_ns);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
            }
            uint8_t* slot = sm.a0 + s * kASlot;
            // All of the chunk's loads first, then the arithmetic.
            uint32_t yv[kChunk];
#pragma unroll
            for (int t = 0; t < static_cast<int>(kChunk); ++t) {
                const int j = c * kChunk + t;
                yv[t] = (j < K && live) ? __ldg(Y + static_cast<size_t>(j) * d.N + n0 + m) : 0u;
            }
#pragma unroll
            for (int t = 0; t < static_cast<int>(kChunk); ++t) {
                const int j = c * kChunk + t;
                if (j < K) {
                    frac += static_cast<double>(yv[t]) * sm.p_recip[j];
                    const uint64_t prod = static_cast<uint64_t>(yv[t]) * sm.m_top[j];
                    top_lo += static_cast<uint32_t>(prod);
                    top_hi += prod >> 32;
                }
            }
#pragma unroll
            for (int g = 0; g < 8; ++g)
                *reinterpret_cast<uint4*>(slot + g * (kRows * 16) + m * 16) =
                    make_uint4(yv[4 * g], yv[4 * g + 1], yv[4 * g + 2], yv[4 * g + 3]);
            tc::fence_proxy_async_smem();
            tc::mbar_arrive(&sm.a_full[s]);
        }
        if (ok) {
            ok = tc::wait_parity(sm.d_ready, 0, d.wait_ns);
            ok = __all_sync(0xffffffffu, ok);
        }
        if (ok) {
            tc::tc_fence_after();
            int v = static_cast<int>(floor(frac + 0.5));
            v = v < 0 ? 0 : (v > K ? K : v);
            const uint32_t* nv = d.negvP + static_cast<size_t>(v) * L;
            const uint64_t t1 = (top_lo >> 32) + top_hi;   // Xtop = lo32(top_lo) + t1 2^32
            const uint32_t tq = tmem + ((q * 32) << 16);
            const uint32_t npieces = U / 32;
            // This row's negvP_v, fetched before the serial carry chain needs it.
            uint32_t nvr[kMaxL];
#pragma unroll
            for (int l = 0; l < kMaxL; ++l) nvr[l] = l < L ? __ldg(nv + l) : 0u;
            // x = D's byte columns with carries, + negvP_v, + Xtop 2^(32(L-1)):
            // kX register limbs, every loop fully unrolled and predicated on L.
            uint32_t x[kX];
            uint64_t carry = 0;
            uint32_t r[32];
#pragma unroll
            for (int l = 0; l < kX; ++l) {
                const int i = l & 7;
                if (i == 0) {
                    // D columns 4l .. 4l + 31 (limbs l .. l + 7), zero above U.
                    if (l / 8 < 8 && static_cast<uint32_t>(l / 8) < npieces) {
                        tc::tmem_ld32(tq + (l / 8) * 32, r);
                        tc::tmem_ld_wait();
                    } else {
#pragma unroll
                        for (int t = 0; t < 32; ++t) r[t] = 0;
                    }
                }
                uint64_t w = carry + static_cast<uint64_t>(r[4 * i]) + (static_cast<uint64_t>(r[4 * i + 1]) << 8) +
                             (static_cast<uint64_t>(r[4 * i + 2]) << 16) + (static_cast<uint64_t>(r[4 * i + 3]) << 24);
                if (l < kMaxL) w += nvr[l < kMaxL ? l : 0];
                if (l == L - 1) w += static_cast<uint32_t>(top_lo);
                if (l == L) w += static_cast<uint32_t>(t1);
                if (l == L + 1) w += t1 >> 32;
                x[l] = l < L + 2 ? static_cast<uint32_t>(w) : 0u;
                carry = w >> 32;
            }
            // x mod q: quotient estimate from the top limbs in double, minus one,
            // then at most two subtractions (arith.cuh reduce_mod_q, in registers).
            const int n = L + 2, drop = top_drop(L);
            double xd = 0;
#pragma unroll
            for (int i = kX - 1; i >= 0; --i)
                if (i < n && i >= drop) xd = xd * 4294967296.0 + x[i];
            const double f = floor(xd / d.q_top);
            const uint64_t e = f >= 1 ? static_cast<uint64_t>(f) - 1 : 0;
#pragma unroll
            for (int pass = 0; pass < 2; ++pass) {
                const int shift = pass == 0 ? 1 : 0;
                const uint32_t ee = pass == 0 ? static_cast<uint32_t>(e >> 32) : static_cast<uint32_t>(e);
                uint64_t cy = 0;
                uint32_t borrow = 0;
#pragma unroll
                for (int i = 0; i < kX; ++i) {
                    const int k = i - shift;
                    const uint64_t prod = (k >= 0 && k < L ? static_cast<uint64_t>(ee) * sm.q[k] : 0u) + cy;
                    cy = prod >> 32;
                    const uint64_t dd = static_cast<uint64_t>(x[i]) - static_cast<uint32_t>(prod) - borrow;
                    if (i < n) {
                        x[i] = static_cast<uint32_t>(dd);
                        borrow = static_cast<uint32_t>(dd >> 63);
                    }
                }
            }
#pragma unroll
            for (int pass = 0; pass < 2; ++pass) {
                int cmp = 0;   // sign of x - q, from the top limb down
#pragma unroll
                for (int i = kX - 1; i >= 0; --i) {
                    if (i < n && cmp == 0) {
                        const uint32_t qi = i < L ? sm.q[i] : 0u;
                        cmp = x[i] > qi ? 1 : (x[i] < qi ? -1 : 0);
                    }
                }
                if (cmp >= 0) {
                    uint32_t borrow = 0;
#pragma unroll
                    for (int i = 0; i < kX; ++i) {
                        if (i < n) {
                            const uint64_t dd = static_cast<uint64_t>(x[i]) - (i < L ? sm.q[i] : 0u) - borrow;
                            x[i] = static_cast<uint32_t>(dd);
                            borrow = static_cast<uint32_t>(dd >> 63);
                        }
                    }
                }
            }
            uint32_t* xs = sm.x + m * (L + 2);
#pragma unroll
            for (int i = 0; i < kMaxL; ++i)
                if (i < L) xs[i] = x[i];
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

__global__ void __launch_bounds__(kThreads, 1)
    k_crt_tc(DevPoint d, const uint32_t* __restrict__ Y, uint32_t* __restrict__ C, uint32_t n_begin, uint32_t n_end) {
    const uint32_t n0 = n_begin + blockIdx.x * kRows;
    crt_body(d, Y, C, n0, min(kRows, n_end - n0));
}

// Grouped: item i owns ceil(N / 128) blocks; y_j in its A, c out.
__global__ void __launch_bounds__(kThreads, 1) k_crt_tc_group(const __grid_constant__ GroupTable t) {
    const uint32_t i = group_locate(t, blockIdx.x);
    const GroupItem& it = t.item[i];
    const uint32_t n0 = (blockIdx.x - t.first[i]) * kRows;
    crt_body(it.d, it.A, it.c, n0, min(kRows, it.d.N - n0));
}

// Large enough that the blocks sharing an SM never ask for more than its 512
// TMEM columns in total.
size_t smem_bytes(uint32_t u, uint32_t tmem_cols) {
    const size_t need = body_bytes(u) + kTailBytes;
    const size_t per_sm = 228 * 1024;
    const size_t floor_bytes = per_sm / (512 / tmem_cols + 1) + 1024;
    return need > floor_bytes ? need : floor_bytes;
}

}  // namespace

void crt_tc_init_attributes() {
    const int bytes = static_cast<int>(smem_bytes(256, 256));
    check(cudaFuncSetAttribute(k_crt_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes), "crt_tc smem");
    check(cudaFuncSetAttribute(k_crt_tc_group, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes), "crt_tc smem");
}

uint32_t crt_tc_group_blocks(uint32_t N) { return (N + kRows - 1) / kRows; }

void launch_crt_tc_group(const GroupTable& t, cudaStream_t st) {
    if (t.total == 0) return;
    uint32_t u = 0, cols = 0;
    for (uint32_t i = 0; i < t.count; ++i) {
        u = t.item[i].d.crt_u > u ? t.item[i].d.crt_u : u;
        cols = t.item[i].d.crt_tmem_cols > cols ? t.item[i].d.crt_tmem_cols : cols;
    }
    k_crt_tc_group<<<t.total, kThreads, smem_bytes(u, cols), st>>>(t);
}

void launch_crt_tc(const DevPoint& d, const uint32_t* Y, uint32_t* c, uint32_t n_begin, uint32_t n_end,
                   cudaStream_t st) {
    if (n_end <= n_begin) return;
    const uint32_t blocks = (n_end - n_begin + kRows - 1) / kRows;
    k_crt_tc<<<blocks, kThreads, smem_bytes(d.crt_u, d.crt_tmem_cols), st>>>(d, Y, c, n_begin, n_end);
}

}  // namespace fpm
