// C entry points around the reference's own CPU implementation (solve_cpu.cpp
// from Akram275/fherma-polymult, compiled from the reference tree by
// oracle/Makefile into oracle/_ref/libref_cpu.so).
//
// TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle and by bench.py's
// reference arm / cpu_baseline to time the reference's CPU path.  The shipped
// library never loads it.
//
// The reference's entry points are C++ (fherma.h:46-48: fherma_init(const
// fherma::Point&), fherma_run(void*, const fherma::Inputs&), fherma_free(void*)),
// so this shim builds the std::vector-based structs from plain pointers.
#include "fherma.h"
#include "rns_plan.h"

#include <omp.h>

#include <chrono>
#include <cstring>
#include <exception>
#include <string>

namespace {
thread_local std::string g_error;
}

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

// Runs `reps` products c = a*b mod (X^N + 1, q) through the reference's
// fherma_init / fherma_run / fherma_free.  seconds[i] gets the wall time of the
// i-th fherma_run call (steady_clock around the call, as main.cpp:182-186 times
// it); c receives the last product.  Returns 0 on success, 1 if the reference
// threw (message in ref_last_error()).
int ref_polymul(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, const uint32_t* a,
                const uint32_t* b, uint32_t* c, int reps, double* seconds) {
    void* state = nullptr;
    try {
        fherma::Point p;
        p.N = N;
        p.W = W;
        p.L = L;
        p.q.shape = {static_cast<int64_t>(L)};
        p.q.data.assign(q, q + L);
        state = fherma_init(p);
        const size_t words = static_cast<size_t>(N) * L;
        fherma::Inputs in;
        in.a.shape = in.b.shape = {static_cast<int64_t>(N), static_cast<int64_t>(L)};
        in.a.data.assign(a, a + words);
        in.b.data.assign(b, b + words);
        for (int r = 0; r < reps; ++r) {
            const auto t0 = std::chrono::steady_clock::now();
            fherma::Outputs out = fherma_run(state, in);
            const std::chrono::duration<double> dt = std::chrono::steady_clock::now() - t0;
            if (seconds) seconds[r] = dt.count();
            if (r + 1 == reps) std::memcpy(c, out.c.data.data(), words * sizeof(uint32_t));
        }
        fherma_free(state);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        if (state) fherma_free(state);
        return 1;
    }
}

// OpenMP threads for the reference's parallel loops (n <= 0: all processors).
// Returns the count in effect.
int ref_set_threads(int n) {
    omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
    return n > 0 ? n : omp_get_num_procs();
}

// The reference's setup tables for (N, q[L]) (rns_plan.h:118-249), so the
// oracle's plan can be compared entry by entry.  Buffers must hold at least
// 160 primes / roots, 160 x L words of M and 161 x L words of negvP.
// Returns 0 with *K set, or 1 if make_plan threw.
int ref_plan(uint32_t N, uint32_t L, const uint32_t* q, int* K, uint32_t* primes, uint32_t* roots,
             uint32_t* M, uint32_t* negvP) {
    try {
        const rns::Plan pl = rns::make_plan(N, q, static_cast<int>(L));
        *K = pl.K;
        std::memcpy(primes, pl.p.data(), pl.p.size() * sizeof(uint32_t));
        std::memcpy(roots, pl.root.data(), pl.root.size() * sizeof(uint32_t));
        std::memcpy(M, pl.M.data(), pl.M.size() * sizeof(uint32_t));
        std::memcpy(negvP, pl.negvP.data(), pl.negvP.size() * sizeof(uint32_t));
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

}  // extern "C"
