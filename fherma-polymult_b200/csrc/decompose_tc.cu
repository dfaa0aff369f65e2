// Decompose on the 5th-generation tensor cores (tcgen05, kind::i8).
//
// x mod p_j = sum_k byte_k(x) (2^(8k) mod p_j) mod p_j over the 4L bytes of a
// coefficient.  Splitting each constant into its 4 bytes turns the sum into an
// integer GEMM over 8-bit operands:
//
//     D[m][4j + s] = sum_k byte_k(x_m) * byte_s(2^(8k) sigma_j mod p_j)
//     x_m mod p_j  = (sum_s D[m][4j + s] 2^(8s)) mod p_j
//
// with sigma_j = 1 for operand a and the pointwise scale for operand b.  Every
// D entry is below 4L 255^2 < 2^24, so the s32 accumulators are exact and the
// fold in the epilogue (a 49-bit value reduced mod p_j) is the only modular
// step.  (Reference: the same sum on CUDA cores, decompose_many rns.cuh:110-128.)
//
// Block = 128 coefficients (the MMA's M); the operand tile A (128 x 4L bytes,
// a contiguous run of the caller's limbs) is staged once in shared memory in
// the canonical K-major layout; the constant matrix B streams in chunks of 32
// primes (128 GEMM columns, a prebuilt image, one bulk copy each) through two
// shared-memory slots, and D alternates between two 128-column TMEM buffers,
// so the MMAs of chunk c + 1 overlap the epilogue of chunk c.
//   warp 0      : TMEM allocation, B copies, MMA issue (one thread)
//   warps 1 - 8 : epilogue, two warps per TMEM lane quadrant (each takes half of
//                 a chunk's 32 primes), one thread per lane (= coefficient):
//                 tcgen05.ld, fold, coalesced stores of each prime's residues.
#include "device.cuh"
#include "group.cuh"
#include "kernels.h"
#include "pdl.cuh"
#include "tc.cuh"

namespace fpm {

namespace {

constexpr int kThreads = 288;                      // warp 0 + 8 epilogue warps
constexpr uint32_t kEpi = 256;                     // epilogue threads
constexpr uint32_t kRows = 128;
constexpr uint32_t kCols = 128;                    // GEMM columns per chunk (32 primes)
constexpr uint32_t kALbo = kRows * 16 + 16;        // A: K-adjacent core matrices, padded
                                                   // so a warp's 32 word stores hit 32 banks

struct Smem {
    uint8_t* a;
    uint8_t* b0;           // B slot s at b0 + s * kCols * kb
    uint64_t* full;        // [2] B chunk landed
    uint64_t* mma_done;    // [2] MMAs of the chunk finished (D ready, B slot free)
    uint64_t* tmem_empty;  // [2] epilogue finished reading the D buffer
    uint32_t* tmem_base;
    uint4* fold;           // [kMaxK] fold constants, staged once per block
};

__host__ __device__ inline uint32_t a_bytes(uint32_t kb) { return (kb / 16) * kALbo; }

__device__ inline Smem carve(uint8_t* base, uint32_t kb) {
    Smem s;
    s.a = base;
    s.b0 = base + ((a_bytes(kb) + 127) & ~127u);
    s.full = reinterpret_cast<uint64_t*>(s.b0 + 2 * kCols * kb);
    s.mma_done = s.full + 2;
    s.tmem_empty = s.full + 4;
    s.tmem_base = reinterpret_cast<uint32_t*>(s.full + 6);
    s.fold = reinterpret_cast<uint4*>(s.full + 8);
    return s;
}

// A GEMM sum D is below 4L 255^2 <= 256 * 65025 (L <= 64), so both halves of
// sum_s D_s 2^(8s), A = D_0 + 2^8 D_1 and B = D_2 + 2^8 D_3, are below 2^32;
// the residue is (A + B 2^16) mod p with f = {p, 2^16 mod p, its Shoup
// companion, floor(2^32 / p)}.
static_assert(kMaxL <= 64, "D_0 + 2^8 D_1 must fit 32 bits");
__device__ __forceinline__ uint32_t fold_halves(uint32_t A, uint32_t B, uint4 f) {
    return add_mod(shoup(A, 1u, f.w, f.x), shoup(B, f.y, f.z, f.x), f.x);
}

// Coefficients n0 .. n0 + nk - 1 (nk <= 128) of one operand.
__device__ __forceinline__ void dec_body(const DevPoint& d, const uint32_t* __restrict__ limbs,
                                         uint32_t* __restrict__ res, int operand, uint32_t n0, uint32_t nk) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t kb = d.dec_kb;          // GEMM K in bytes (4L rounded up to 32)
    const int nch = d.dec_chunks;
    const Smem sm = carve(smem_raw, kb);
    const uint8_t* img = operand ? d.dec_img_b : d.dec_img_a;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int L = d.L;

    const uint32_t chunk_bytes = kCols * kb;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&sm.full[i], 1);
            tc::mbar_init(&sm.mma_done[i], 1);
            tc::mbar_init(&sm.tmem_empty[i], kEpi);
        }
        tc::fence_mbar_init();
        // The first two constant chunks load under the operand tile's load.
        for (int c = 0; c < (nch < 2 ? nch : 2); ++c) {
            tc::mbar_arrive_expect_tx(&sm.full[c], chunk_bytes);
            tc::bulk_g2s(sm.b0 + c * chunk_bytes, img + static_cast<size_t>(c) * chunk_bytes, chunk_bytes, &sm.full[c]);
        }
    }
    if (warp == 0) tc::tmem_alloc(sm.tmem_base, 2 * kCols);
    for (int j = threadIdx.x; j < d.K; j += kThreads) sm.fold[j] = d.dec_fold[j];

    // The operand tile and the residues are the only global data a preceding
    // kernel may still be using.
    pdl_wait();
    // Operand tile: word l of row m goes to core matrix l / 4 along K, row m.
    // The block's nk L words are contiguous and 16-byte aligned (n0 L 4 = 512 L
    // bytes), so they are read as 16-byte chunks, 8 in flight per thread.
    {
        const uint32_t kw = kb / 4;
        if (kw != static_cast<uint32_t>(L) || nk < kRows) {
            // Zero padding: rows past nk and words past L.
            for (uint32_t i = threadIdx.x; i < a_bytes(kb) / 16; i += kThreads)
                reinterpret_cast<uint4*>(sm.a)[i] = make_uint4(0, 0, 0, 0);
            __syncthreads();
        }
        const uint32_t total = nk * static_cast<uint32_t>(L);
        // 16-byte loads need the caller's limbs 16-byte aligned (the block's
        // start n0 L 4 is a multiple of 16 then); otherwise every word goes
        // through the word-wise tail path below.
        const bool vec = (reinterpret_cast<uintptr_t>(limbs) & 15u) == 0;
        const uint32_t n16 = vec ? total / 4 : 0;
        const uint4* src4 = reinterpret_cast<const uint4*>(limbs + static_cast<size_t>(n0) * L);
        // w / L = mulhi(w, ceil(2^32 / L)) exactly for w < 2^16 (L = 1 divides trivially).
        const uint32_t inv_l = L == 1 ? 0u : 0xFFFFFFFFu / static_cast<uint32_t>(L) + 1;
        auto row_of = [&](uint32_t w) { return L == 1 ? w : __umulhi(w, inv_l); };
        auto place = [&](uint32_t w, uint32_t v) {
            const uint32_t m = row_of(w), l = w - m * L;
            *reinterpret_cast<uint32_t*>(sm.a + (l >> 2) * kALbo + m * 16 + (l & 3) * 4) = v;
        };
        for (uint32_t i0 = threadIdx.x; i0 < n16; i0 += 8 * kThreads) {
            uint4 v[8];
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const uint32_t i = i0 + b * kThreads;
                v[b] = i < n16 ? __ldg(src4 + i) : make_uint4(0, 0, 0, 0);
            }
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const uint32_t i = i0 + b * kThreads;
                if (i >= n16) continue;
                if ((L & 3) == 0) {
                    const uint32_t w = 4 * i, m = row_of(w), l = w - m * L;
                    *reinterpret_cast<uint4*>(sm.a + (l >> 2) * kALbo + m * 16) = v[b];
                } else {
                    place(4 * i, v[b].x);
                    place(4 * i + 1, v[b].y);
                    place(4 * i + 2, v[b].z);
                    place(4 * i + 3, v[b].w);
                }
            }
        }
        const uint32_t* src = limbs + static_cast<size_t>(n0) * L;
        for (uint32_t w = 4 * n16 + threadIdx.x; w < total; w += kThreads) place(w, src[w]);
    }
    tc::fence_proxy_async_smem();
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *sm.tmem_base;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_u8(kCols);
            const uint32_t a0 = tc::smem_addr(sm.a);
            for (int c = 0; c < nch && ok; ++c) {
                const int s = c & 1;
                ok = tc::wait_parity(&sm.full[s], (c >> 1) & 1, d.wait_ns);
                if (ok && c >= 2) ok = tc::wait_parity(&sm.tmem_empty[s], ((c - 2) >> 1) & 1, d.wait_ns);
                if (!ok) break;
                tc::tc_fence_after();
                const uint32_t b0 = tc::smem_addr(sm.b0 + s * chunk_bytes);
                for (uint32_t kk = 0; kk < kb / 32; ++kk) {
                    const uint64_t ad = tc::smem_desc(a0 + kk * 2 * kALbo, kALbo, 128);
                    const uint64_t bd = tc::smem_desc(b0 + kk * 2 * (kCols * 16), kCols * 16, 128);
                    tc::mma_u8(tmem + s * kCols, ad, bd, idesc, kk > 0);
                }
                tc::mma_commit(&sm.mma_done[s]);
                if (c >= 1 && c + 1 < nch) {
                    const int s1 = (c - 1) & 1;
                    ok = tc::wait_parity(&sm.mma_done[s1], ((c - 1) >> 1) & 1, d.wait_ns);
                    if (!ok) break;
                    tc::mbar_arrive_expect_tx(&sm.full[s1], chunk_bytes);
                    tc::bulk_g2s(sm.b0 + s1 * chunk_bytes, img + static_cast<size_t>(c + 1) * chunk_bytes, chunk_bytes,
                                 &sm.full[s1]);
                }
            }
            if (ok) {
                // The last MMAs must finish before the block can release TMEM.
                const int c = nch - 1;
                ok = tc::wait_parity(&sm.mma_done[c & 1], (c >> 1) & 1, d.wait_ns);
            }
        }
        __syncwarp();
    } else {
        const uint32_t q = warp & 3;                   // TMEM lane quadrant of this warp
        const int half = (warp - 1) >> 2;              // which 16 primes of each chunk
        const uint32_t m = q * 32 + lane;
        const uint32_t tq = tmem + ((q * 32) << 16);
        for (int c = 0; c < nch; ++c) {
            const int s = c & 1;
            ok = tc::wait_parity(&sm.mma_done[s], (c >> 1) & 1, d.wait_ns);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            tc::tc_fence_after();
#pragma unroll 1
            for (int piece = 2 * half; piece < 2 * half + 2; ++piece) {
                const int j0 = c * 32 + piece * 8;
                uint4 f[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) f[i] = sm.fold[min(j0 + i, d.K - 1)];
                uint32_t r[32];
                tc::tmem_ld32(tq + s * kCols + piece * 32, r);
                tc::tmem_ld_wait();
                uint32_t out[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    out[i] = fold_halves(r[4 * i] + (r[4 * i + 1] << 8), r[4 * i + 2] + (r[4 * i + 3] << 8), f[i]);
                }
                if (m < nk) {
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        if (j0 + i < d.K) res[static_cast<size_t>(j0 + i) * d.N + n0 + m] = out[i];
                }
            }
            tc::tc_fence_before();
            tc::mbar_arrive(&sm.tmem_empty[s]);
        }
    }

    if (!ok) atomicOr(d.err, 1u);
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 2 * kCols);
    }
}

// Grid (tiles, operands): blockIdx.y = 1 takes the second operand (lb, rb).
__global__ void __launch_bounds__(kThreads)
    k_decompose_tc(DevPoint d, const uint32_t* __restrict__ la, const uint32_t* __restrict__ lb,
                   uint32_t* __restrict__ ra, uint32_t* __restrict__ rb, int operand0, uint32_t n_begin,
                   uint32_t n_end) {
    pdl_launch_dependents();
    const uint32_t n0 = n_begin + blockIdx.x * kRows;
    const bool second = blockIdx.y != 0;
    dec_body(d, second ? lb : la, second ? rb : ra, operand0 + static_cast<int>(blockIdx.y), n0,
             min(kRows, n_end - n0));
}

// Grouped: item i owns 2 ceil(N / 128) blocks, operand a's tiles then b's.
__global__ void __launch_bounds__(kThreads) k_decompose_tc_group(const __grid_constant__ GroupTable t) {
    const uint32_t i = group_locate(t, blockIdx.x);
    const GroupItem& it = t.item[i];
    const uint32_t local = blockIdx.x - t.first[i], tiles = (it.d.N + kRows - 1) / kRows;
    const int operand = local >= tiles;
    const uint32_t n0 = (local - (operand ? tiles : 0)) * kRows;
    dec_body(it.d, operand ? it.b : it.a, operand ? it.B : it.A, operand, n0, min(kRows, it.d.N - n0));
}

// At least 78 KB, so no more than two blocks (2 x 256 TMEM columns) share an SM.
size_t smem_bytes(uint32_t kb) {
    const size_t need = ((a_bytes(kb) + 127) & ~127u) + 2 * kCols * kb + 8 * sizeof(uint64_t) + kMaxK * sizeof(uint4);
    return need > 78 * 1024 ? need : 78 * 1024;
}

}  // namespace

void decompose_tc_init_attributes() {
    const int bytes = static_cast<int>(smem_bytes(4 * kMaxL));
    check(cudaFuncSetAttribute(k_decompose_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
          "decompose_tc smem");
    check(cudaFuncSetAttribute(k_decompose_tc_group, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
          "decompose_tc smem");
}

uint32_t decompose_tc_group_blocks(uint32_t N) { return 2 * ((N + kRows - 1) / kRows); }

void launch_decompose_tc_group(const GroupTable& t, cudaStream_t st) {
    if (t.total == 0) return;
    uint32_t kb = 0;
    for (uint32_t i = 0; i < t.count; ++i) kb = t.item[i].d.dec_kb > kb ? t.item[i].d.dec_kb : kb;
    k_decompose_tc_group<<<t.total, kThreads, smem_bytes(kb), st>>>(t);
}

void launch_decompose_tc(const DevPoint& d, const uint32_t* limbs, uint32_t* res, int operand, uint32_t n_begin,
                         uint32_t n_end, cudaStream_t st) {
    if (n_end <= n_begin) return;
    const uint32_t blocks = (n_end - n_begin + kRows - 1) / kRows;
    check(launch_pdl(k_decompose_tc, dim3(blocks), dim3(kThreads), smem_bytes(d.dec_kb), st, d, limbs, limbs, res,
                     res, operand, n_begin, n_end),
          "decompose launch");
}

void launch_decompose_tc_pair(const DevPoint& d, const uint32_t* a, const uint32_t* b, uint32_t* A, uint32_t* B,
                              cudaStream_t st) {
    const dim3 grid((d.N + kRows - 1) / kRows, 2);
    check(launch_pdl(k_decompose_tc, grid, dim3(kThreads), smem_bytes(d.dec_kb), st, d, a, b, A, B, 0, 0u, d.N),
          "decompose launch");
}

}  // namespace fpm
