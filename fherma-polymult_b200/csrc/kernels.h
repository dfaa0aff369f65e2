// Host-side launch interface of the kernels.
#pragma once

#include "device.cuh"
#include "plan.h"

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace fpm {

// A failed CUDA call ("<what>: <CUDA message>").  Invalid points and other
// argument errors are plain std::runtime_error.
struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(const std::string& msg, cudaError_t c) : std::runtime_error(msg), code(c) {}
};

// A pipeline wait in a tensor-core kernel ran out of time (DevPoint::wait_ns):
// the kernel returned early and that product's result is wrong.
struct PipelineTimeout : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e), e);
}

// Default limit of a pipeline wait (DevPoint::wait_ns): 2 s.
constexpr uint64_t kDefaultWaitNs = 2000000000ull;

// Columns per column-pass tile of 2048 elements.
template <int LOGR>
constexpr uint32_t kTileCols = 2048u >> LOGR;

size_t col_fwd_smem(uint32_t logR);
size_t col_inv_smem(uint32_t logR);
size_t row_smem();

// One-time per process: shared-memory opt-ins for the kernels.
void ntt_init_attributes();
void decompose_init_attributes();
void crt_init_attributes();
void decompose_tc_init_attributes();
void crt_tc_init_attributes();

// limbs (N x L, coefficient-major) -> residues (K x N); operand 1 (b) is
// scaled for the pointwise step.
// Coefficients [n_begin, n_end) only (multiples of 128 but for the end).
void launch_decompose(const DevPoint& d, const uint32_t* limbs, uint32_t* res, int operand, uint32_t n_begin,
                      uint32_t n_end, cudaStream_t st);

// Residues A, B -> y_j in A (mode kRowProduct), or the forward transforms of
// both in place (mode kRowForward).
void launch_ntt(const DevPoint& d, uint32_t* A, uint32_t* B, int mode, cudaStream_t st);
// Every row's forward twiddle table (K x R x S, round-major) into out, from the
// point's generators row_u_f and row_q_f; once per context.
void build_row_tables(const DevPoint& d, uint2* out, cudaStream_t st);

// The same on the tensor cores.
void launch_decompose_tc(const DevPoint& d, const uint32_t* limbs, uint32_t* res, int operand, uint32_t n_begin,
                         uint32_t n_end, cudaStream_t st);

// Both operands of a product in one launch: a -> A (operand 0), b -> B (1).
void launch_decompose_tc_pair(const DevPoint& d, const uint32_t* a, const uint32_t* b, uint32_t* A, uint32_t* B,
                              cudaStream_t st);

// y_j (K x N) -> c (N x L) mod q: CUDA cores, and tensor cores (L >= 2).
void launch_crt(const DevPoint& d, const uint32_t* Y, uint32_t* c, uint32_t n_begin, uint32_t n_end,
                cudaStream_t st);
void launch_crt_tc(const DevPoint& d, const uint32_t* Y, uint32_t* c, uint32_t n_begin, uint32_t n_end,
                   cudaStream_t st);

// The persistent CRT pipeline (crt_pipe.cu): one CTA per SM, `sms` at most.
// Needs L >= 2 and N, n_begin, n_end multiples of 4.  Its per-prime constants
// travel as a kernel parameter.
struct CrtConsts {
    float cf[kMaxK];            // 2^sh_j / p_j in single precision, for the rounding sum
    uint32_t sh[kMaxK];         // sh_j: y_j >> sh_j < 2^23 and 2^(23 + sh_j) / p_j <= 2
    float voff;                 // sum_j 2^23 cf_j: the offset the rounding sum removes
    float est_err;              // a bound on the rounding sum's error (must stay below 1/4)
    uint32_t top[kMaxK + 1];    // top limb of constant j (j = K: -P mod q)
    uint32_t q[kMaxL + 2];      // q, zero above L
};
// top: the K constants' top limbs M_j[L - 1], then (-P mod q)'s top limb.
CrtConsts make_crt_consts(const HostPlan& pl, const uint32_t* top);

// The modulus tables of a context on the device (crt_tables.cu): M (K x L),
// negvP ((K + 1) x L), and for L >= 2 the tensor-core CRT images img (K rows)
// and img_v (K + 1 rows) of crt_image_bytes each; Pq is scratch of L words.
// pl needs its basis and q / q_top; pc and q are device copies.
size_t crt_image_bytes(const HostPlan& pl, int rows);
void build_crt_tables(const HostPlan& pl, const PrimeConsts* pc, const uint32_t* q, uint32_t* M, uint32_t* negvP,
                      uint32_t* Pq, uint8_t* img, uint8_t* img_v, cudaStream_t st);
bool crt_pipe_supported(const DevPoint& d, const CrtConsts& cc, const uint32_t* Y, uint32_t n_begin, uint32_t n_end);
void crt_pipe_init_attributes();
void launch_crt_pipe(const DevPoint& d, const CrtConsts& cc, const uint32_t* Y, uint32_t* c, uint32_t n_begin,
                     uint32_t n_end, int sms, cudaStream_t st);

// The persistent decompose pipeline (decompose_pipe.cu): one CTA per SM; with
// b != nullptr the CTAs split between a -> A (operand 0) and b -> B (1),
// otherwise all take a -> A as operand `operand0`.
struct DecConsts {
    uint4 fold[kMaxK];          // {p, 2^16 mod p, its Shoup companion, floor(2^32 / p)}
    const uint8_t* img[2];      // device copies of the plan's wide images, operands a and b
    uint32_t chunks;            // chunks of 64 primes
    uint32_t last_cols;         // GEMM columns of the last chunk
    uint32_t lazy_out;          // 1: residues below 4p (congruent), for lazy first butterflies
};
DecConsts make_dec_consts(const HostPlan& pl, const uint8_t* img_a, const uint8_t* img_b);
bool decompose_pipe_supported(const HostPlan& pl);
void decompose_pipe_init_attributes();
void launch_decompose_pipe(const DevPoint& d, const DecConsts& dc, const uint32_t* a, const uint32_t* b,
                           uint32_t* A, uint32_t* B, int operand0, uint32_t n_begin, uint32_t n_end, int sms,
                           cudaStream_t st);

// Grouped launches (group.cuh): one launch covers every item of the table,
// whose first[] the caller fills with these per-item block counts.
struct GroupTable;
uint32_t decompose_tc_group_blocks(uint32_t N);   // both operands
uint32_t crt_tc_group_blocks(uint32_t N);
uint32_t ntt_blocks_per_prime(int pass, uint32_t logR, uint32_t logS);
void launch_decompose_tc_group(const GroupTable& t, cudaStream_t st);
void launch_crt_tc_group(const GroupTable& t, cudaStream_t st);
// pass kPassColFwd / kPassRow (product) / kPassColInv over items of one
// (logR, logS); grid 0 = one block per tile, else a persistent grid.
void launch_ntt_group(const GroupTable& t, int pass, uint32_t logR, uint32_t logS, bool lazy, uint32_t grid,
                      cudaStream_t st);
int ntt_group_occupancy(int pass, uint32_t logR, uint32_t logS, bool lazy);
// The same over items of mixed row lengths (R = 64 each, logS <= max_log_s):
// one launch per pass whatever the geometries; blocks per item from
// ntt_mixed_blocks (the row pass runs two 128-thread tiles per block for
// 16-element rounds).
bool ntt_mixed_ok(const DevPoint& d);
uint32_t ntt_mixed_blocks(int pass, uint32_t logS, uint32_t primes);
void launch_ntt_mixed(const GroupTable& t, int pass, bool lazy, uint32_t max_log_s, uint32_t grid, cudaStream_t st);
int ntt_mixed_occupancy(int pass, bool lazy, uint32_t max_log_s);

}  // namespace fpm
