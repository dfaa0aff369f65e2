/*
 * CPU oracle for the exact negacyclic product (TEST INFRASTRUCTURE ONLY; see
 * rns_oracle.h).  Plain C11, deliberately simple: u64 / unsigned __int128
 * arithmetic, one full twiddle table per prime, schoolbook multi-limb helpers.
 *
 * Reference lines restated here (paths inside Akram275/fherma-polymult):
 *   plan ............ rns_plan.h:118-249 (make_plan), 252-267 (full twiddles)
 *   decompose ....... rns.cuh:110-128 (decompose_many)
 *   forward NTT ..... rns_kernels.cuh:161-166 (fwd_butterfly), 132-157 (stage order)
 *   inverse NTT ..... rns_kernels.cuh:168-174 (inv_butterfly)
 *   pointwise ....... rns_kernels.cuh:178-181 (pointwise), rns_plan.h:211-219 (scale)
 *   CRT ............. rns_kernels.cuh:265-364 (crt_columns / crt_combine),
 *                     rns.cuh:161-221 (geq, sub_in_place, submul, reduce_wide)
 */
#include "rns_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORA_MAX_L 64
#define ORA_MAX_K 160
#define ORA_MAX_LOGN 22
#define ORA_MARGIN_BITS 20

struct ora_plan {
    uint32_t N, logN;
    int L, K;
    uint32_t* q;        /* L */
    double q_top;       /* q's top three limbs as a double (rns_plan.h:136) */
    uint32_t* p;        /* K */
    uint32_t* psi;      /* K: primitive 2N-th root */
    uint32_t* ipsi;     /* K: its inverse */
    uint32_t* pow2;     /* K x L: 2^(32 l) mod p_j */
    uint32_t* scale;    /* K: N^-1 (P/p_j)^-1 mod p_j */
    uint32_t* tw;       /* K x N: psi^bitrev(i) */
    uint32_t* itw;      /* K x N: psi^-bitrev(i) */
    double* p_recip;    /* K */
    uint32_t* M;        /* K x L */
    uint32_t* negvP;    /* (K + 1) x L */
};

static void set_err(char* err, size_t len, const char* fmt, ...) {
    if (!err || !len) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, len, fmt, ap);
    va_end(ap);
}

static uint32_t pow_mod(uint64_t b, uint64_t e, uint32_t p) {
    uint64_t r = 1;
    b %= p;
    for (; e; e >>= 1, b = b * b % p)
        if (e & 1) r = r * b % p;
    return (uint32_t)r;
}

/* Deterministic Miller-Rabin for n < 2^32 with bases 2, 3, 5, 7
 * (rns_plan.h:66-87 uses the same bases). */
static int is_prime_u32(uint32_t n) {
    static const uint32_t bases[4] = {2, 3, 5, 7};
    if (n < 2) return 0;
    for (int i = 0; i < 4; ++i)
        if (n % bases[i] == 0) return n == bases[i];
    uint32_t d = n - 1;
    int r = 0;
    while (!(d & 1)) d >>= 1, ++r;
    for (int i = 0; i < 4; ++i) {
        uint64_t x = pow_mod(bases[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int composite = 1;
        for (int k = 1; k < r && composite; ++k) {
            x = x * x % n;
            if (x == n - 1) composite = 0;
        }
        if (composite) return 0;
    }
    return 1;
}

static uint32_t bitrev(uint32_t x, uint32_t bits) {
    uint32_t r = 0;
    for (uint32_t i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

static int bit_length(const uint32_t* x, int n) {
    for (int i = n - 1; i >= 0; --i)
        if (x[i]) return 32 * i + 32 - __builtin_clz(x[i]);
    return 0;
}

/* ---- multi-limb helpers (rns.cuh:161-221) ------------------------------- */

static int geq(const uint32_t* x, int n, const uint32_t* q, int L) {
    for (int i = n - 1; i >= 0; --i) {
        uint32_t qi = i < L ? q[i] : 0;
        if (x[i] != qi) return x[i] > qi;
    }
    return 1;
}

/* x -= q; returns the borrow out. */
static uint32_t sub_in_place(uint32_t* x, int n, const uint32_t* q, int L) {
    uint32_t borrow = 0;
    for (int i = 0; i < n; ++i) {
        uint64_t d = (uint64_t)x[i] - (i < L ? q[i] : 0) - borrow;
        x[i] = (uint32_t)d;
        borrow = (uint32_t)(d >> 63);
    }
    return borrow;
}

/* x -= (e * q) << (32 * shift); returns the borrow out (nonzero means the
 * caller's non-negativity premise failed). */
static uint32_t submul(uint32_t* x, int n, const uint32_t* q, int L, uint32_t e, int shift) {
    uint64_t carry = 0;
    uint32_t borrow = 0;
    for (int i = shift; i < n; ++i) {
        int k = i - shift;
        uint64_t prod = (k < L ? (uint64_t)e * q[k] : 0) + carry;
        carry = prod >> 32;
        uint64_t d = (uint64_t)x[i] - (uint32_t)prod - borrow;
        x[i] = (uint32_t)d;
        borrow = (uint32_t)(d >> 63);
    }
    return borrow | (carry != 0);
}

static int dropped_limbs(int L) { return L > 3 ? L - 3 : 0; }

/* x mod q in place for x < 2^64 q: a quotient estimate from the top limbs in
 * double, one less than its floor, then at most a few subtractions
 * (rns.cuh:212-221).  Aborts if the estimate ever overshoots. */
static void reduce_wide(uint32_t* x, int n, const uint32_t* q, int L, double q_top) {
    double xd = 0;
    for (int i = n - 1; i >= dropped_limbs(L); --i) xd = xd * 4294967296.0 + x[i];
    double f = floor(xd / q_top);
    uint64_t e = f >= 1 ? (uint64_t)f - 1 : 0;
    uint32_t bad = 0;
    if (e >> 32) bad |= submul(x, n, q, L, (uint32_t)(e >> 32), 1);
    if (e) bad |= submul(x, n, q, L, (uint32_t)e, 0);
    if (bad) {
        fprintf(stderr, "rns_oracle: reduce_wide quotient estimate overshot\n");
        abort();
    }
    int guard = 0;
    while (geq(x, n, q, L)) {
        sub_in_place(x, n, q, L);
        if (++guard > 8) {
            fprintf(stderr, "rns_oracle: reduce_wide needed more than 8 subtractions\n");
            abort();
        }
    }
}

/* x = x * m mod q for x < q (rns_plan.h:102-114). */
static void mul_small_mod(uint32_t* x, uint32_t m, const ora_plan* pl) {
    uint32_t t[ORA_MAX_L + 1];
    uint64_t carry = 0;
    for (int l = 0; l < pl->L; ++l) {
        uint64_t v = (uint64_t)x[l] * m + carry;
        t[l] = (uint32_t)v;
        carry = v >> 32;
    }
    t[pl->L] = (uint32_t)carry;
    reduce_wide(t, pl->L + 1, pl->q, pl->L, pl->q_top);
    memcpy(x, t, sizeof(uint32_t) * pl->L);
}

/* ---- plan (rns_plan.h:118-249) ------------------------------------------ */

void ora_plan_free(ora_plan* pl) {
    if (!pl) return;
    free(pl->q);
    free(pl->p);
    free(pl->psi);
    free(pl->ipsi);
    free(pl->pow2);
    free(pl->scale);
    free(pl->tw);
    free(pl->itw);
    free(pl->p_recip);
    free(pl->M);
    free(pl->negvP);
    free(pl);
}

int ora_plan_make(uint32_t N, const uint32_t* q, int L, int pmax_log2, ora_plan** out, char* err,
                  size_t errlen) {
    *out = NULL;
    if (N < 2 || (N & (N - 1)) || N > (1u << ORA_MAX_LOGN)) {
        set_err(err, errlen, "N must be a power of two in [2, 2^%d]; got %u", ORA_MAX_LOGN, N);
        return 1;
    }
    if (L < 1 || L > ORA_MAX_L) {
        set_err(err, errlen, "L must be in [1, %d]; got %d", ORA_MAX_L, L);
        return 1;
    }
    if (pmax_log2 < 20 || pmax_log2 > 31) {
        set_err(err, errlen, "prime window 2^%d unsupported", pmax_log2);
        return 1;
    }
    if (bit_length(q, L) <= 32 * (L - 1)) {
        set_err(err, errlen, "q has fewer limbs than L");
        return 1;
    }
    ora_plan* pl = (ora_plan*)calloc(1, sizeof(ora_plan));
    pl->N = N;
    while ((1u << pl->logN) < N) ++pl->logN;
    pl->L = L;
    pl->q = (uint32_t*)malloc(sizeof(uint32_t) * L);
    memcpy(pl->q, q, sizeof(uint32_t) * L);
    for (int i = L - 1; i >= dropped_limbs(L); --i) pl->q_top = pl->q_top * 4294967296.0 + q[i];
    const int qbits = bit_length(q, L);

    /* Primes p = 1 (mod step), step = max(2N, 2^16), scanned downward from the
     * top of the window until their product exceeds 2^20 * 2N * q^2
     * (rns_plan.h:138-153). */
    const double need_bits = 2.0 * qbits + pl->logN + 1 + ORA_MARGIN_BITS;
    double have_bits = 0;
    const uint32_t step = 2 * N > (1u << 16) ? 2 * N : (1u << 16);
    const uint32_t top = (uint32_t)((1ull << pmax_log2) - 1);
    uint32_t primes[ORA_MAX_K + 1];
    int K = 0;
    for (uint32_t c = top / step * step + 1; have_bits <= need_bits; c -= step) {
        if (c < step) {
            set_err(err, errlen, "not enough primes p < 2^%d with p = 1 (mod %u) for N = %u, q of %d bits",
                    pmax_log2, step, N, qbits);
            ora_plan_free(pl);
            return 1;
        }
        if (!is_prime_u32(c)) continue;
        if (K == ORA_MAX_K) {
            set_err(err, errlen, "more than %d primes needed", ORA_MAX_K);
            ora_plan_free(pl);
            return 1;
        }
        primes[K++] = c;
        have_bits += log2((double)c);
    }
    pl->K = K;
    pl->p = (uint32_t*)malloc(sizeof(uint32_t) * K);
    memcpy(pl->p, primes, sizeof(uint32_t) * K);
    pl->psi = (uint32_t*)malloc(sizeof(uint32_t) * K);
    pl->ipsi = (uint32_t*)malloc(sizeof(uint32_t) * K);
    pl->pow2 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)K * L);
    pl->scale = (uint32_t*)malloc(sizeof(uint32_t) * K);
    pl->tw = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)K * N);
    pl->itw = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)K * N);
    pl->p_recip = (double*)malloc(sizeof(double) * K);

    for (int j = 0; j < K; ++j) {
        const uint32_t p = pl->p[j];
        for (int l = 0; l < L; ++l) pl->pow2[(size_t)j * L + l] = pow_mod(2, 32ull * l, p);
        /* psi: the first g^((p-1)/2N), g = 2, 3, ..., whose N-th power is -1
         * (rns_plan.h:191-195). */
        uint32_t psi = 0;
        for (uint32_t g = 2; !psi; ++g) {
            uint32_t cand = pow_mod(g, (p - 1) / (2ull * N), p);
            if (pow_mod(cand, N, p) == p - 1) psi = cand;
        }
        pl->psi[j] = psi;
        pl->ipsi[j] = pow_mod(psi, p - 2, p);
        for (uint32_t i = 0; i < N; ++i) {
            uint32_t e = bitrev(i, pl->logN);
            pl->tw[(size_t)j * N + i] = pow_mod(psi, e, p);
            pl->itw[(size_t)j * N + i] = pow_mod(pl->ipsi[j], e, p);
        }
        /* scale = N^-1 (P/p_j)^-1 mod p_j (rns_plan.h:211-219, without the 2^32
         * that the reference adds to undo its Montgomery product). */
        uint64_t Pj = 1;
        for (int i = 0; i < K; ++i)
            if (i != j) Pj = Pj * (pl->p[i] % p) % p;
        uint64_t n_inv = pow_mod(N, p - 2, p), Pj_inv = pow_mod(Pj, p - 2, p);
        pl->scale[j] = (uint32_t)(n_inv * Pj_inv % p);
        pl->p_recip[j] = 1.0 / p;
    }

    /* M_j = prod_{i != j} p_i mod q and P mod q (rns_plan.h:224-236). */
    pl->M = (uint32_t*)calloc((size_t)K * L, sizeof(uint32_t));
    uint32_t Pq[ORA_MAX_L] = {0};
    Pq[0] = 1;
    for (int j = 0; j < K; ++j) {
        uint32_t* m = pl->M + (size_t)j * L;
        m[0] = 1;
        for (int i = 0; i < K; ++i)
            if (i != j) mul_small_mod(m, pl->p[i], pl);
        mul_small_mod(Pq, pl->p[j], pl);
    }
    /* negvP_v = (q - v P mod q) mod q for v = 0..K (rns_plan.h:238-247). */
    pl->negvP = (uint32_t*)calloc((size_t)(K + 1) * L, sizeof(uint32_t));
    for (int v = 1; v <= K; ++v) {
        uint32_t t[ORA_MAX_L];
        memcpy(t, Pq, sizeof(uint32_t) * L);
        mul_small_mod(t, (uint32_t)v, pl);
        if (bit_length(t, L) == 0) continue;
        uint32_t* neg = pl->negvP + (size_t)v * L;
        memcpy(neg, pl->q, sizeof(uint32_t) * L);
        sub_in_place(neg, L, t, L);
    }
    *out = pl;
    return 0;
}

int ora_plan_K(const ora_plan* pl) { return pl->K; }
int ora_plan_L(const ora_plan* pl) { return pl->L; }
uint32_t ora_plan_N(const ora_plan* pl) { return pl->N; }
void ora_plan_primes(const ora_plan* pl, uint32_t* out) { memcpy(out, pl->p, sizeof(uint32_t) * pl->K); }
void ora_plan_roots(const ora_plan* pl, uint32_t* out) { memcpy(out, pl->psi, sizeof(uint32_t) * pl->K); }
void ora_plan_crt_tables(const ora_plan* pl, uint32_t* M, uint32_t* negvP) {
    if (M) memcpy(M, pl->M, sizeof(uint32_t) * (size_t)pl->K * pl->L);
    if (negvP) memcpy(negvP, pl->negvP, sizeof(uint32_t) * (size_t)(pl->K + 1) * pl->L);
}

/* ---- stages -------------------------------------------------------------- */

/* x mod p_j = sum_l limb_l * (2^(32 l) mod p_j) mod p_j (rns.cuh:110-128). */
void ora_decompose(const ora_plan* pl, const uint32_t* limbs, uint32_t* res) {
    const uint32_t N = pl->N;
    const int L = pl->L;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < pl->K; ++j) {
        const uint64_t p = pl->p[j];
        const uint32_t* pw = pl->pow2 + (size_t)j * L;
        for (uint32_t n = 0; n < N; ++n) {
            const uint32_t* x = limbs + (size_t)n * L;
            unsigned __int128 acc = 0;
            for (int l = 0; l < L; ++l) acc += (uint64_t)x[l] * pw[l];
            res[(size_t)j * N + n] = (uint32_t)(acc % p);
        }
    }
}

/* Cooley-Tukey, distance t = N/2 .. 1, twiddle psi^bitrev(m + i) for group i of
 * the m = N / (2t) groups: (x, y) -> (x + w y, x - w y)
 * (rns_kernels.cuh:161-166 with the pairs of col_pair / row_pair, :132-157). */
void ora_ntt_forward(const ora_plan* pl, uint32_t* res) {
    const uint32_t N = pl->N;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < pl->K; ++j) {
        const uint64_t p = pl->p[j];
        const uint32_t* tw = pl->tw + (size_t)j * N;
        uint32_t* x = res + (size_t)j * N;
        for (uint32_t t = N / 2; t >= 1; t /= 2) {
            const uint32_t m = N / (2 * t);
            for (uint32_t i = 0; i < m; ++i) {
                const uint64_t w = tw[m + i];
                for (uint32_t k = 2 * t * i; k < 2 * t * i + t; ++k) {
                    const uint64_t u = x[k], v = x[k + t] * w % p;
                    x[k] = (uint32_t)((u + v) % p);
                    x[k + t] = (uint32_t)((u + p - v) % p);
                }
            }
        }
    }
}

/* Gentleman-Sande, distance t = 1 .. N/2, twiddle psi^-bitrev(m + i):
 * (x, y) -> (x + y, (x - y) w) (rns_kernels.cuh:168-174). */
void ora_ntt_inverse(const ora_plan* pl, uint32_t* res) {
    const uint32_t N = pl->N;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < pl->K; ++j) {
        const uint64_t p = pl->p[j];
        const uint32_t* tw = pl->itw + (size_t)j * N;
        uint32_t* x = res + (size_t)j * N;
        for (uint32_t t = 1; t < N; t *= 2) {
            const uint32_t m = N / (2 * t);
            for (uint32_t i = 0; i < m; ++i) {
                const uint64_t w = tw[m + i];
                for (uint32_t k = 2 * t * i; k < 2 * t * i + t; ++k) {
                    const uint64_t u = x[k], v = x[k + t];
                    x[k] = (uint32_t)((u + v) % p);
                    x[k + t] = (uint32_t)((u + p - v) % p * w % p);
                }
            }
        }
    }
}

/* A <- A B N^-1 (P/p_j)^-1 (rns_kernels.cuh:178-181, rns_plan.h:211-219). */
void ora_pointwise(const ora_plan* pl, uint32_t* A, const uint32_t* B) {
    const uint32_t N = pl->N;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < pl->K; ++j) {
        const uint64_t p = pl->p[j], s = pl->scale[j];
        for (uint32_t n = 0; n < N; ++n) {
            const size_t at = (size_t)j * N + n;
            A[at] = (uint32_t)((uint64_t)A[at] * B[at] % p * s % p);
        }
    }
}

/* One output coefficient from its K residues y_j = c (P/p_j)^-1 mod p_j:
 * v = round(sum_j y_j / p_j) clamped to [0, K]; c = sum_j y_j M_j + negvP_v
 * mod q (rns_kernels.cuh:265-364, rns.cuh:212-221). */
void ora_crt(const ora_plan* pl, const uint32_t* y, uint32_t* c) {
    const uint32_t N = pl->N;
    const int L = pl->L, K = pl->K;
#pragma omp parallel for schedule(static)
    for (uint32_t n = 0; n < N; ++n) {
        uint64_t col[ORA_MAX_L + 2];
        double frac = 0;
        for (int l = 0; l < L + 2; ++l) col[l] = 0;
        for (int j = 0; j < K; ++j) {
            const uint64_t yj = y[(size_t)j * N + n];
            frac += (double)yj * pl->p_recip[j];
            const uint32_t* m = pl->M + (size_t)j * L;
            for (int l = 0; l < L; ++l) {
                const uint64_t prod = yj * m[l];
                col[l] += (uint32_t)prod;     /* each column stays below K 2^32 < 2^40 */
                col[l + 1] += prod >> 32;
            }
        }
        int v = (int)floor(frac + 0.5);
        v = v < 0 ? 0 : (v > K ? K : v);
        const uint32_t* t = pl->negvP + (size_t)v * L;
        for (int l = 0; l < L; ++l) col[l] += t[l];
        uint32_t x[ORA_MAX_L + 2];
        uint64_t carry = 0;
        for (int l = 0; l < L + 2; ++l) {
            const uint64_t s = col[l] + carry;
            x[l] = (uint32_t)s;
            carry = s >> 32;
        }
        reduce_wide(x, L + 2, pl->q, L, pl->q_top);
        memcpy(c + (size_t)n * L, x, sizeof(uint32_t) * L);
    }
}

int ora_polymul(const ora_plan* pl, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* y_out) {
    const size_t words = (size_t)pl->K * pl->N;
    uint32_t* A = (uint32_t*)malloc(sizeof(uint32_t) * words);
    uint32_t* B = (uint32_t*)malloc(sizeof(uint32_t) * words);
    if (!A || !B) {
        free(A);
        free(B);
        return 1;
    }
    ora_decompose(pl, a, A);
    ora_decompose(pl, b, B);
    ora_ntt_forward(pl, A);
    ora_ntt_forward(pl, B);
    ora_pointwise(pl, A, B);
    ora_ntt_inverse(pl, A);
    if (y_out) memcpy(y_out, A, sizeof(uint32_t) * words);
    ora_crt(pl, A, c);
    free(A);
    free(B);
    return 0;
}
