// Host-side setup for one point (N, q): the prime set and every constant table
// the kernels read.  Built once per point, outside any timed call.
//
// Reference counterpart: rns_plan.h:118-280 (make_plan, add_full_twiddles,
// use_gen_twiddles).  The prime set, the choice of each prime's root psi_j and
// the CRT constants follow the reference exactly (same primes in the same
// order, so residues compare stage by stage with the oracle); the twiddle
// tables are laid out for this library's kernels instead.
#pragma once

#include "arith.cuh"

#include <cstdint>
#include <string>
#include <vector>

namespace fpm {

// How the length-N transform is cut for the kernels.
//   logN <= kSmallLogN : one block per prime holds the whole transform
//                        (k_ntt_small), full twiddle tables.
//   logN == 11         : one 2048-element tile per prime (row kernel, R = 1).
//   logN >= 12         : four-step, N = R x S with S = 2^min(11, logN - 6):
//                        column pass (stages of distance >= S, along the R
//                        rows of each column) and row pass (distance < S).
//                        The longest rows (so R = 64 up to N = 2^17) make the
//                        column tiles widest, C = 2048 / R adjacent words per
//                        row; measured fastest at every N from 2^13 to 2^18
//                        (N = 2^16, 2048-bit q: 180 us against 190 for 256 x 256,
//                        N = 2^18: 758 against 960 for 512 x 512).
constexpr uint32_t kSmallLogN = 10;
constexpr uint32_t kTileLog = 11;            // 2048-element tiles
constexpr uint32_t kTile = 1u << kTileLog;

struct Geometry {
    uint32_t logN = 0, logR = 0, logS = 0;
    bool small = false;
};

Geometry make_geometry(uint32_t logN);

struct HostPlan {
    uint32_t N = 0, W = 0;
    int L = 0, K = 0;
    Geometry g;
    int qbits = 0;                // bits of q: the prime basis depends on q only through them
    std::vector<uint32_t> q;      // L
    double q_top = 0;             // top limbs of q as a double
    int pmax_log2 = 30;           // primes below 2^pmax_log2
    bool lazy = true;             // pmax_log2 <= 30: lazy butterflies

    std::vector<uint32_t> primes;            // K
    std::vector<PrimeConsts> pc;             // K
    std::vector<uint32_t> psi, ipsi;         // K

    // Decompose: x mod p_j = sum_l x_l c_{j,l}.  a uses c = 2^(32 l) mod p_j;
    // b folds in the pointwise scale N^-1 (P/p_j)^-1 2^32 (the 2^32 undoes the
    // Montgomery product in the pointwise step), so the inverse transform ends
    // in y_j directly.  K x L Shoup pairs each.
    std::vector<uint2> dec_a, dec_b;

    // Column pass twiddles (logN >= 12): psi^(S bitrev_logR(y)) for y in [1, R),
    // K x R pairs (entry 0 unused); inverse with psi^-1.
    std::vector<uint2> col_f, col_i;
    // Row pass twiddle generators: the forward twiddle of stage b (distance 2^b)
    // for row u and group r' is psi^(2^b (1 + 2 bitrev_logR(u)) + 2^(b+1+logR) bitrev(r'))
    // = U[u][b] * Q[y] with y = 2^(logS-1-b) + r'.  (The inverse twiddles are
    // negated forward ones of the partner row R - 1 - u, see ntt.cu.)
    //   row_u_f: K x R x logS pairs, row_q_f: K x S pairs (entry 0 unused), each
    //   prime's S entries in the round-major order of row_table_pos.
    std::vector<uint2> row_u_f, row_q_f;
    // Small transforms (logN <= kSmallLogN): psi^bitrev_logN(y), K x N pairs.
    std::vector<uint2> full_f, full_i;

    // CRT: M_j = P / p_j mod q (K x L), negvP_v = -v P mod q ((K + 1) x L),
    // 1 / p_j (K).
    std::vector<uint32_t> M, negvP;
    std::vector<double> p_recip;

    // Tensor-core decompose (decompose_tc.cu): the GEMM's B operand, the bytes of
    // c_{j,k} = 2^(8k) sigma_j mod p_j (k < 4L) split per byte s into GEMM column
    // 4j + s, in chunks of 32 primes (128 columns), each chunk a ready-made
    // shared-memory image in the UMMA K-major no-swizzle layout
    // [dec_kb / 16 core columns][128 rows][16 bytes].  One image per operand.
    uint32_t dec_kb = 0;                     // GEMM K in bytes: 4L rounded up to 32
    uint32_t dec_chunks = 0;                 // ceil(K / 32)
    std::vector<uint8_t> dec_img_a, dec_img_b;
    // The same constants in chunks of 64 primes (256 columns) for the
    // pipelined decompose, in the UMMA K-major 128-byte-swizzle layout
    // (sw128_offset, one block per 128 K bytes); the last chunk has
    // dec_wlast columns.
    uint32_t dec_wchunks = 0, dec_wlast = 0;
    std::vector<uint8_t> dec_wimg_a, dec_wimg_b;
    std::vector<uint4> dec_fold;             // K: {p, 2^16 mod p, its Shoup companion, floor(2^32 / p)}

    // Tensor-core CRT (crt_tc.cu), L >= 2: B operand, row u (a byte position of
    // X_low = sum_j y_j M_j[0 .. L-2]) and column 4j + s hold byte (u - s) of
    // M_j's low L - 1 limbs; u < crt_u = 4L - 1 rounded up to 32.  Chunks of 32
    // primes (128 K bytes), image [8 core columns][crt_u rows][16 bytes].
    uint32_t crt_u = 0;
    uint32_t crt_tmem_cols = 0;              // power of two >= crt_u
    std::vector<uint8_t> crt_img;
    // The same image with a row K for -P mod q (= negvP_1), and that
    // constant's top limb: the pipelined CRT multiplies it by v in the GEMM.
    // Laid out for that kernel (crt_image_at with swz): every 32-prime chunk
    // but the last 128-byte swizzled, the last in core matrices.
    std::vector<uint8_t> crt_img_v;
    uint32_t negp_top = 0;
};

// Byte of a CRT image: row j (a constant; K-byte 4 (j % 32) + s of chunk
// j / 32) at GEMM column u, for images of `rows` rows and crt_u columns.
// Plain: the core-matrix layout [8 core columns][crt_u][16 bytes] per chunk;
// swz: every chunk but the last in the 128-byte-swizzle layout (sw128_offset),
// the last plain (the pipelined CRT keeps only its first K steps resident).
FPM_HD size_t crt_image_at(uint32_t j, uint32_t s, uint32_t u, uint32_t crt_u, int rows, bool swz) {
    const uint32_t kbyte = 4 * (j % 32) + s, chunk = j / 32;
    const size_t base = static_cast<size_t>(chunk) * crt_u * 128;
    const uint32_t last = static_cast<uint32_t>(rows - 1) / 32;
    if (swz && chunk < last) return base + sw128_offset(u, kbyte, crt_u);
    return base + (kbyte / 16) * (crt_u * 16) + u * 16 + (kbyte % 16);
}

// Which CRT kernel the point uses: the tensor-core one needs L >= 2.
inline bool crt_uses_tc(const HostPlan& pl) { return pl.L >= 2; }

// Device bytes an Engine for this plan holds (tables, residue workspaces and
// the limb buffers of the host path).
size_t device_footprint(const HostPlan& pl);

// Throws std::runtime_error on an out-of-range point (N not a power of two in
// [2, 2^22], L outside [1, 64], q's top limb zero, not enough primes).
// pmax_log2 = 30 (default) keeps every prime below 2^30, which the lazy
// butterflies need; 31 reproduces the reference's prime set exactly
// (rns_plan.h:141-153) and uses fully reduced butterflies.
constexpr int kDefaultPrimeBits = 30;
HostPlan make_plan(uint32_t N, uint32_t W, const uint32_t* q, int L, int pmax_log2 = kDefaultPrimeBits);

// The plan in two parts.  make_plan_basis builds everything that depends on q
// only through its bit length -- the prime set, twiddles, decompose constants
// and images -- so one basis serves every modulus of that width;
// set_modulus adds q and the tables built from it (M, negvP, the CRT images,
// negp_top), set_modulus_limbs only q and q_top (for callers that build the
// rest on the device).  make_plan is make_plan_basis + set_modulus.
// modulus_bits checks q (L in range, nonzero top limb) and returns its bits;
// check_length throws unless N is a power of two in [2, 2^kMaxLogN].
int modulus_bits(const uint32_t* q, int L);
void check_length(uint32_t N);
HostPlan make_plan_basis(uint32_t N, uint32_t W, int L, int qbits, int pmax_log2 = kDefaultPrimeBits);
void set_modulus_limbs(HostPlan& pl, const uint32_t* q);
void set_modulus(HostPlan& pl, const uint32_t* q);

}  // namespace fpm
