/*
 * CPU oracle for the exact negacyclic product c = a*b mod (X^N + 1, q).
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg use it, and only as the checker.
 *
 * It restates the reference implementation's algorithm (Akram275/fherma-polymult,
 * rns.cuh, rns_plan.h, rns_kernels.cuh) in plain C with straightforward loops, so
 * that every intermediate the GPU path produces (residues, transformed residues,
 * CRT inputs y_j, final limbs) has an independent value to be compared against.
 * Each function names the reference lines it follows.
 *
 * Parity of this restatement is pinned two ways (tests/test_oracle.py):
 *   - against golden vectors written by the reference's own CPU build
 *     (oracle/Makefile compiles main.cpp + solve_cpu.cpp from the reference tree;
 *     tests/golden/make_golden.py runs it), and
 *   - against an independent GMP Kronecker-substitution product (oracle/bigint.py).
 */
#ifndef FPM_RNS_ORACLE_H
#define FPM_RNS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_plan ora_plan;

/* Build the plan for (N, q[L]).  pmax_log2 selects the prime window: primes are
 * scanned downward from 2^pmax_log2 (31 reproduces the reference's prime set,
 * rns_plan.h:141-153).  Returns 0 and sets *out, or returns nonzero and writes a
 * message into err. */
int ora_plan_make(uint32_t N, const uint32_t* q, int L, int pmax_log2, ora_plan** out, char* err,
                  size_t errlen);
void ora_plan_free(ora_plan* pl);

int ora_plan_K(const ora_plan* pl);
int ora_plan_L(const ora_plan* pl);
uint32_t ora_plan_N(const ora_plan* pl);
/* K primes, in the plan's order. */
void ora_plan_primes(const ora_plan* pl, uint32_t* out);
/* psi_j, the primitive 2N-th root each prime's transform uses. */
void ora_plan_roots(const ora_plan* pl, uint32_t* out);
/* M_j = P / p_j mod q (K x L) and -vP mod q (v = 0..K, (K + 1) x L). */
void ora_plan_crt_tables(const ora_plan* pl, uint32_t* M, uint32_t* negvP);

/* Stages.  Residue arrays are K x N, prime-major (res[j * N + n]). */
void ora_decompose(const ora_plan* pl, const uint32_t* limbs /* N x L */, uint32_t* res);
void ora_ntt_forward(const ora_plan* pl, uint32_t* res);   /* natural in, bit-reversed out */
void ora_ntt_inverse(const ora_plan* pl, uint32_t* res);   /* bit-reversed in, natural out, no scaling */
/* A <- A * B * N^-1 * (P/p_j)^-1 mod p_j, so the inverse transform yields y_j. */
void ora_pointwise(const ora_plan* pl, uint32_t* A, const uint32_t* B);
void ora_crt(const ora_plan* pl, const uint32_t* y /* K x N */, uint32_t* c /* N x L */);

/* Whole product; y_out (K x N, may be NULL) receives the CRT inputs. */
int ora_polymul(const ora_plan* pl, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* y_out);

#ifdef __cplusplus
}
#endif

#endif
