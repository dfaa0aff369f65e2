// Device-side description of one product's point: sizes, and pointers into
// the device copies of the HostPlan tables (plan.h).  Passed to kernels by
// value.  Residue buffers are K x N u32, prime-major: X[j * N + n].
#pragma once

#include "arith.cuh"

#include <cstdint>

namespace fpm {

struct DevPoint {
    uint32_t N, logN, logR, logS;
    int L, K;
    int lazy;                  // primes below 2^30: lazy (Harvey) butterflies
    const PrimeConsts* pc;     // K
    const uint2* dec_a;        // K x L
    const uint2* dec_b;        // K x L
    const uint2* col_f;        // K x R
    const uint2* col_i;
    const uint2* row_u_f;      // K x R x logS
    const uint2* row_q_f;      // K x S
    const uint2* row_tw;       // K x R x S: row u's forward table, round-major (built once)
    const uint2* full_f;       // K x N (small transforms)
    const uint2* full_i;
    const uint32_t* q;         // L
    double q_top;
    double q_top_inv;          // 1 / q_top, for the quotient estimate
    const uint32_t* M;         // K x L
    const uint32_t* negvP;     // (K + 1) x L
    const double* p_recip;     // K
    // tensor-core decompose
    uint32_t dec_kb;
    int dec_chunks;
    const uint8_t* dec_img_a;
    const uint8_t* dec_img_b;
    const uint4* dec_fold;     // K
    // tensor-core CRT
    uint32_t crt_u;
    uint32_t crt_tmem_cols;
    const uint8_t* crt_img;
    const uint8_t* crt_img_v;  // K + 1 rows: row K is -P mod q (pipelined CRT)
    uint32_t negp_top;         // (-P mod q)'s top limb
    // error word: bit 0 decompose, bit 1 CRT (a pipeline wait timed out)
    uint32_t* err;
    // How long any pipeline wait may last before the kernel gives up, sets the
    // error word and returns (nanoseconds; 2 s unless a caller shortens it).
    uint64_t wait_ns;
    // Test hook, 0 in every product: bit 0 makes the pipelined decompose, bit 1
    // the pipelined CRT, leave one barrier phase that a role waits on without
    // its arrival, so that wait runs out (kFault* below).
    uint32_t fault;
};

enum FaultBits : uint32_t {
    kFaultDecompose = 1u,
    kFaultCrt = 2u,
};

// What the row kernel does with its tile.
enum RowMode : int {
    kRowProduct = 0,   // forward rows of A and B, pointwise A B, inverse rows -> A
    kRowForward = 1,   // forward rows of A and B only (for stage checks)
    // single launches of the four-step chain, for timing one kernel at a time
    kPassColFwd = 2,
    kPassRow = 3,
    kPassColInv = 4,
};

}  // namespace fpm
