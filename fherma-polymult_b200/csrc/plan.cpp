// Host-side setup tables for one point; see plan.h.
#include "plan.h"

#include "ntt_engine.cuh"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace fpm {

namespace {

uint32_t pow_mod(uint64_t b, uint64_t e, uint32_t p) {
    uint64_t r = 1;
    b %= p;
    for (; e; e >>= 1, b = b * b % p) {
        if (e & 1) r = r * b % p;
    }
    return static_cast<uint32_t>(r);
}

// Deterministic Miller-Rabin for 32-bit n (bases 2, 3, 5, 7 suffice below 3.2e9).
bool is_prime(uint32_t n) {
    if (n < 2) return false;
    for (uint32_t d : {2u, 3u, 5u, 7u}) {
        if (n % d == 0) return n == d;
    }
    uint32_t d = n - 1;
    int r = 0;
    while (!(d & 1)) d >>= 1, ++r;
    for (uint32_t a : {2u, 3u, 5u, 7u}) {
        uint64_t x = pow_mod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool composite = true;
        for (int i = 1; i < r && composite; ++i) {
            x = x * x % n;
            if (x == n - 1) composite = false;
        }
        if (composite) return false;
    }
    return true;
}

uint32_t shoup_of(uint32_t w, uint32_t p) {
    return static_cast<uint32_t>((static_cast<uint64_t>(w) << 32) / p);
}

uint2 pair(uint32_t w, uint32_t p) {
    uint2 t;
    t.x = w;
    t.y = shoup_of(w, p);
    return t;
}

int bit_length(const uint32_t* x, int n) {
    for (int i = n - 1; i >= 0; --i) {
        if (x[i]) return 32 * i + 32 - __builtin_clz(x[i]);
    }
    return 0;
}

// x = x * m mod q for x < q.
void mul_small_mod(std::vector<uint32_t>& x, uint32_t m, const HostPlan& pl) {
    std::vector<uint32_t> t(pl.L + 1);
    uint64_t carry = 0;
    for (int l = 0; l < pl.L; ++l) {
        const uint64_t v = static_cast<uint64_t>(x[l]) * m + carry;
        t[l] = static_cast<uint32_t>(v);
        carry = v >> 32;
    }
    t[pl.L] = static_cast<uint32_t>(carry);
    reduce_mod_q(t.data(), pl.L + 1, pl.q.data(), pl.L, pl.q_top);
    std::copy(t.begin(), t.begin() + pl.L, x.begin());
}

}  // namespace

Geometry make_geometry(uint32_t logN) {
    Geometry g;
    g.logN = logN;
    if (logN <= kSmallLogN) {
        g.small = true;
        g.logS = logN;
        g.logR = 0;
    } else if (logN == kTileLog) {
        g.logS = logN;
        g.logR = 0;
    } else {
        g.logS = std::min<uint32_t>(kTileLog, logN - 6);
        g.logR = logN - g.logS;
    }
    return g;
}

size_t device_footprint(const HostPlan& pl) {
    auto bytes = [](const auto& v) { return v.size() * sizeof(v[0]); };
    size_t t = bytes(pl.pc) + bytes(pl.dec_a) + bytes(pl.dec_b) + bytes(pl.col_f) + bytes(pl.col_i) +
               bytes(pl.row_u_f) + bytes(pl.row_q_f) +
               bytes(pl.full_f) + bytes(pl.full_i) + bytes(pl.q) + bytes(pl.M) + bytes(pl.negvP) +
               bytes(pl.p_recip) + bytes(pl.dec_img_a) + bytes(pl.dec_img_b) + bytes(pl.dec_fold) +
               bytes(pl.dec_wimg_a) + bytes(pl.dec_wimg_b) +
               bytes(pl.crt_img) + bytes(pl.crt_img_v) + sizeof(uint32_t);
    if (!pl.g.small) t += static_cast<size_t>(pl.K) * pl.N * sizeof(uint2);   // row twiddle tables
    t += 2 * static_cast<size_t>(pl.K) * pl.N * sizeof(uint32_t);   // residue workspaces
    t += 3 * static_cast<size_t>(pl.N) * pl.L * sizeof(uint32_t);   // host-path limb buffers
    return t;
}

int modulus_bits(const uint32_t* q, int L) {
    if (L < 1 || L > kMaxL) {
        throw std::runtime_error("unsupported limb count L = " + std::to_string(L) + ": expected 1 to " +
                                 std::to_string(kMaxL) + " limbs (moduli of up to " + std::to_string(32 * kMaxL) +
                                 " bits)");
    }
    const int qbits = bit_length(q, L);
    if (qbits <= 32 * (L - 1)) {
        throw std::runtime_error("modulus q has a zero top limb: its " + std::to_string(qbits) +
                                 " bits fit in fewer than the " + std::to_string(L) + " limbs given");
    }
    return qbits;
}

void check_length(uint32_t N) {
    if (N < 2 || (N & (N - 1)) || N > (1u << kMaxLogN)) {
        throw std::runtime_error("unsupported transform length N = " + std::to_string(N) +
                                 ": expected a power of two from 2 to 2^" + std::to_string(kMaxLogN));
    }
}

HostPlan make_plan(uint32_t N, uint32_t W, const uint32_t* q, int L, int pmax_log2) {
    check_length(N);
    const int qbits = modulus_bits(q, L);
    HostPlan pl = make_plan_basis(N, W, L, qbits, pmax_log2);
    set_modulus(pl, q);
    return pl;
}

HostPlan make_plan_basis(uint32_t N, uint32_t W, int L, int qbits, int pmax_log2) {
    check_length(N);
    if (L < 1 || L > kMaxL || qbits <= 32 * (L - 1) || qbits > 32 * L) {
        throw std::runtime_error("unsupported modulus: " + std::to_string(qbits) + " bits in L = " +
                                 std::to_string(L) + " limbs (1 to " + std::to_string(kMaxL) +
                                 " limbs, nonzero top limb)");
    }
    if (pmax_log2 < 24 || pmax_log2 > 31) throw std::runtime_error("prime window must be 2^24 .. 2^31");
    HostPlan pl;
    pl.N = N;
    pl.W = W;
    pl.L = L;
    pl.pmax_log2 = pmax_log2;
    pl.lazy = pmax_log2 <= 30;
    uint32_t logN = 0;
    while ((1u << logN) < N) ++logN;
    pl.g = make_geometry(logN);
    pl.qbits = qbits;

    // Primes p = 1 (mod step), step = max(2N, 2^16), from the top of the window
    // downward until sum log2 p > 2 bits(q) + logN + 1 + 20: then |c| < N q^2 is
    // below P / 2^21 and the CRT's rounding is exact (reference rns_plan.h:138-153).
    const double need_bits = 2.0 * qbits + logN + 1 + kMarginBits;
    double have_bits = 0;
    const uint32_t step = std::max(2 * N, 1u << 16);
    const uint32_t top = static_cast<uint32_t>((1ull << pmax_log2) - 1);
    for (uint32_t c = top / step * step + 1; have_bits <= need_bits; c -= step) {
        if (c < step) {
            throw std::runtime_error("not enough primes p < 2^" + std::to_string(pmax_log2) + " with p = 1 (mod " +
                                     std::to_string(step) + ") for N = " + std::to_string(N) + ", q of " +
                                     std::to_string(qbits) + " bits");
        }
        if (!is_prime(c)) continue;
        pl.primes.push_back(c);
        have_bits += std::log2(static_cast<double>(c));
        if (static_cast<int>(pl.primes.size()) > kMaxK) {
            throw std::runtime_error("more than " + std::to_string(kMaxK) + " primes needed");
        }
    }
    pl.K = static_cast<int>(pl.primes.size());
    const int K = pl.K;
    const Geometry& g = pl.g;
    const uint32_t R = 1u << g.logR, S = 1u << g.logS;

    pl.pc.resize(K);
    pl.psi.resize(K);
    pl.ipsi.resize(K);
    pl.dec_a.resize(static_cast<size_t>(K) * L);
    pl.dec_b.resize(static_cast<size_t>(K) * L);
    pl.p_recip.resize(K);
    if (g.small) {
        pl.full_f.resize(static_cast<size_t>(K) * N);
        pl.full_i.resize(static_cast<size_t>(K) * N);
    } else {
        pl.row_u_f.resize(static_cast<size_t>(K) * R * g.logS);
        pl.row_q_f.resize(static_cast<size_t>(K) * S);
        if (g.logR) {
            pl.col_f.resize(static_cast<size_t>(K) * R);
            pl.col_i.resize(static_cast<size_t>(K) * R);
        }
    }

    for (int j = 0; j < K; ++j) {
        const uint32_t p = pl.primes[j];
        PrimeConsts& c = pl.pc[j];
        c.p = p;
        uint32_t inv = 1;   // p^-1 mod 2^32 by Newton's iteration
        for (int i = 0; i < 5; ++i) inv *= 2 - p * inv;
        c.pneg = 0u - inv;
        const unsigned __int128 mu = (static_cast<unsigned __int128>(1) << 64) / p;
        c.mu_lo = static_cast<uint32_t>(mu);
        c.mu_hi = static_cast<uint32_t>(mu >> 32);

        // psi_j: the first g^((p-1)/2N), g = 2, 3, ..., whose N-th power is -1
        // (the reference's choice, rns_plan.h:191-195).
        uint32_t psi = 0;
        for (uint32_t gen = 2; !psi; ++gen) {
            const uint32_t cand = pow_mod(gen, (p - 1) / (2ull * N), p);
            if (pow_mod(cand, N, p) == p - 1) psi = cand;
        }
        const uint32_t ipsi = pow_mod(psi, p - 2, p);
        pl.psi[j] = psi;
        pl.ipsi[j] = ipsi;

        // Pointwise scale N^-1 (P/p_j)^-1 2^32 (reference rns_plan.h:211-219).
        uint64_t Pj = 1;
        for (int i = 0; i < K; ++i) {
            if (i != j) Pj = Pj * (pl.primes[i] % p) % p;
        }
        const uint64_t scale = static_cast<uint64_t>(pow_mod(N, p - 2, p)) * pow_mod(Pj, p - 2, p) % p *
                               ((1ull << 32) % p) % p;
        for (int l = 0; l < L; ++l) {
            const uint32_t w = pow_mod(2, 32ull * l, p);
            pl.dec_a[static_cast<size_t>(j) * L + l] = pair(w, p);
            pl.dec_b[static_cast<size_t>(j) * L + l] = pair(static_cast<uint32_t>(w * scale % p), p);
        }
        pl.p_recip[j] = 1.0 / p;

        if (g.small) {
            for (uint32_t y = 0; y < N; ++y) {
                const uint32_t e = bitrev(y, logN);
                pl.full_f[static_cast<size_t>(j) * N + y] = pair(pow_mod(psi, e, p), p);
                pl.full_i[static_cast<size_t>(j) * N + y] = pair(pow_mod(ipsi, e, p), p);
            }
            continue;
        }
        for (uint32_t y = 1; y < R; ++y) {
            const uint64_t e = static_cast<uint64_t>(S) * bitrev(y, g.logR);
            pl.col_f[static_cast<size_t>(j) * R + y] = pair(pow_mod(psi, e, p), p);
            pl.col_i[static_cast<size_t>(j) * R + y] = pair(pow_mod(ipsi, e, p), p);
        }
        for (uint32_t u = 0; u < R; ++u) {
            for (uint32_t b = 0; b < g.logS; ++b) {
                const uint64_t e = (1ull << b) * (1 + 2ull * bitrev(u, g.logR));
                const size_t at = (static_cast<size_t>(j) * R + u) * g.logS + b;
                pl.row_u_f[at] = pair(pow_mod(psi, e, p), p);
            }
        }
        // Stored round-major (row_table_pos), the order the row pass reads.
        const int rb = row_pass_rb(static_cast<int>(g.logS));
        for (uint32_t y = 1; y < S; ++y) {
            uint32_t lev = 0;   // y in [2^lev, 2^(lev+1)): stage b = logS - 1 - lev
            while ((2u << lev) <= y) ++lev;
            const uint32_t b = g.logS - 1 - lev;
            const uint32_t r = y - (1u << lev);
            const uint64_t e = (1ull << (b + 1 + g.logR)) * bitrev(r, lev);
            const uint32_t at = row_table_pos(static_cast<int>(g.logS), rb, y);
            pl.row_q_f[static_cast<size_t>(j) * S + at] = pair(pow_mod(psi, e, p), p);
        }
    }

    // Tensor-core decompose images and fold constants.
    pl.dec_kb = (4 * static_cast<uint32_t>(L) + 31) / 32 * 32;
    pl.dec_chunks = static_cast<uint32_t>((K + 31) / 32);
    const size_t dchunk = static_cast<size_t>(128) * pl.dec_kb;
    pl.dec_img_a.assign(dchunk * pl.dec_chunks, 0);
    pl.dec_img_b.assign(dchunk * pl.dec_chunks, 0);
    pl.dec_fold.resize(K);
    // Wide images: chunks of 64 primes (256 GEMM columns, the MMA's widest N);
    // the last chunk packed to its own width, a multiple of 16 columns.
    pl.dec_wchunks = static_cast<uint32_t>((K + 63) / 64);
    pl.dec_wlast = (4 * static_cast<uint32_t>(K - 64 * (static_cast<int>(pl.dec_wchunks) - 1)) + 15) / 16 * 16;
    const size_t wchunk = sw128_bytes(256, pl.dec_kb);   // 128-byte-swizzle layout (sw128_offset)
    pl.dec_wimg_a.assign(wchunk * (pl.dec_wchunks - 1) + sw128_bytes(pl.dec_wlast, pl.dec_kb), 0);
    pl.dec_wimg_b.assign(pl.dec_wimg_a.size(), 0);
    for (int j = 0; j < K; ++j) {
        const uint32_t p = pl.primes[j];
        const uint32_t r16 = (1u << 16) % p;
        pl.dec_fold[j] = uint4{p, r16, shoup_of(r16, p), static_cast<uint32_t>((1ull << 32) / p)};
        const uint32_t scale_b = pl.dec_b[static_cast<size_t>(j) * L].x;   // 2^0 * scale
        const size_t chunk = static_cast<size_t>(j / 32) * dchunk;
        for (int s = 0; s < 4; ++s) {
            const uint32_t col = 4 * (j % 32) + s;
            for (uint32_t k = 0; k < 4 * static_cast<uint32_t>(L); ++k) {
                const uint32_t ca = pow_mod(2, 8ull * k, p);
                const uint32_t cb = static_cast<uint32_t>(static_cast<uint64_t>(ca) * scale_b % p);
                const size_t at = chunk + (k / 16) * (128 * 16) + col * 16 + (k % 16);
                pl.dec_img_a[at] = static_cast<uint8_t>(ca >> (8 * s));
                pl.dec_img_b[at] = static_cast<uint8_t>(cb >> (8 * s));
                const uint32_t wc = static_cast<uint32_t>(j / 64), wcol = 4 * (j % 64) + s;
                const uint32_t wcols = wc + 1 < pl.dec_wchunks ? 256 : pl.dec_wlast;
                const size_t wat = wc * wchunk + sw128_offset(wcol, k, wcols);
                pl.dec_wimg_a[wat] = static_cast<uint8_t>(ca >> (8 * s));
                pl.dec_wimg_b[wat] = static_cast<uint8_t>(cb >> (8 * s));
            }
        }
    }

    if (crt_uses_tc(pl)) {
        pl.crt_u = (4 * static_cast<uint32_t>(L) - 1 + 31) / 32 * 32;
        pl.crt_tmem_cols = 32;
        while (pl.crt_tmem_cols < pl.crt_u) pl.crt_tmem_cols *= 2;
    }
    return pl;
}

void set_modulus_limbs(HostPlan& pl, const uint32_t* q) {
    const int bits = modulus_bits(q, pl.L);
    if (bits != pl.qbits) {
        throw std::runtime_error("modulus of " + std::to_string(bits) + " bits given to a prime basis built for " +
                                 std::to_string(pl.qbits) + " bits");
    }
    pl.q.assign(q, q + pl.L);
    pl.q_top = modulus_top(q, pl.L);
}

void set_modulus(HostPlan& pl, const uint32_t* q) {
    set_modulus_limbs(pl, q);
    const int K = pl.K, L = pl.L;
    // M_j = prod_{i != j} p_i mod q, P mod q, and negvP_v = (q - v P mod q) mod q
    // for v = 0..K (reference rns_plan.h:224-247).
    pl.M.assign(static_cast<size_t>(K) * L, 0);
    std::vector<uint32_t> Pq(L, 0);
    Pq[0] = 1;
    for (int j = 0; j < K; ++j) {
        std::vector<uint32_t> m(L, 0);
        m[0] = 1;
        for (int i = 0; i < K; ++i) {
            if (i != j) mul_small_mod(m, pl.primes[i], pl);
        }
        std::copy(m.begin(), m.end(), pl.M.begin() + static_cast<size_t>(j) * L);
        mul_small_mod(Pq, pl.primes[j], pl);
    }
    pl.negvP.assign(static_cast<size_t>(K + 1) * L, 0);
    for (int v = 1; v <= K; ++v) {
        std::vector<uint32_t> t = Pq;
        mul_small_mod(t, static_cast<uint32_t>(v), pl);
        if (bit_length(t.data(), L) == 0) continue;
        std::vector<uint32_t> neg = pl.q;
        limbs_sub(neg.data(), L, t.data(), L);
        std::copy(neg.begin(), neg.end(), pl.negvP.begin() + static_cast<size_t>(v) * L);
    }

    // Tensor-core CRT image.
    if (crt_uses_tc(pl)) {
        const uint32_t chunks = static_cast<uint32_t>((K + 31) / 32);
        const size_t cchunk = static_cast<size_t>(pl.crt_u) * 128;
        const uint32_t low_bytes = 4 * static_cast<uint32_t>(L - 1);
        // Row j of an image holds the byte shifts of constant j's low L - 1 limbs.
        auto build = [&](std::vector<uint8_t>& img, int rows, bool swz, auto&& limbs_of) {
            img.assign(cchunk * static_cast<size_t>((rows + 31) / 32), 0);
            for (int j = 0; j < rows; ++j) {
                const uint32_t* m = limbs_of(j);
                for (int s = 0; s < 4; ++s) {
                    for (uint32_t u = s; u < pl.crt_u && u - s < low_bytes; ++u) {
                        const uint32_t byte = u - s;
                        img[crt_image_at(j, s, u, pl.crt_u, rows, swz)] =
                            static_cast<uint8_t>(m[byte / 4] >> (8 * (byte % 4)));
                    }
                }
            }
        };
        (void)chunks;
        build(pl.crt_img, K, false, [&](int j) { return &pl.M[static_cast<size_t>(j) * L]; });
        // The same with one more row, -P mod q: its multiplier is v, so the
        // GEMM itself adds -v P (the pipelined CRT needs no negvP table).
        build(pl.crt_img_v, K + 1, true, [&](int j) {
            return j < K ? &pl.M[static_cast<size_t>(j) * L] : &pl.negvP[static_cast<size_t>(L)];
        });
        pl.negp_top = pl.negvP[static_cast<size_t>(L) + L - 1];
    }
}

}  // namespace fpm
