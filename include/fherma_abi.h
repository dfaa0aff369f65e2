// fherma_abi.h - the reference's C++ entry points, as this library exports them.
//
// The reference's harness (main.cpp, generated by the FHERMA platform) binds
// three C++ functions by their mangled names (fherma.toml:7-10):
//
//     void*           fherma_init(const fherma::Point&);          fherma.h:46
//     fherma::Outputs fherma_run(void*, const fherma::Inputs&);   fherma.h:47
//     void            fherma_free(void*);                         fherma.h:48
//
// The structs below are written to be layout-identical to the reference's
// fherma.h:16-41 (same member types in the same order, libstdc++ vectors), so
// the mangled symbols and the objects passed through them match; this is the
// one interface that has to be alike, and it is restated here rather than
// included from the reference tree.
//
// Semantics (reference fherma.h, solve.cu):
//   * fherma_init throws std::runtime_error for an out-of-range point;
//   * fherma_run throws std::runtime_error if a or b is not N x L, and returns c
//     with shape {N, L}, every coefficient canonical in [0, q);
//   * fherma_free accepts nullptr.
#pragma once

#include <cstdint>
#include <vector>

namespace fherma {

template <class T>
struct Tensor {
    std::vector<int64_t> shape;
    std::vector<T> data;   // row-major

    int64_t count() const {
        int64_t n = 1;
        for (int64_t d : shape) n *= d;
        return n;
    }
};

struct Point {
    uint32_t N = 0;
    uint32_t W = 0;
    uint32_t L = 0;
    Tensor<uint32_t> q;   // L limbs
};

struct Inputs {
    Tensor<uint32_t> a;   // N x L
    Tensor<uint32_t> b;   // N x L
};

struct Outputs {
    Tensor<uint32_t> c;   // N x L
};

}  // namespace fherma

#if defined(__GNUC__)
#define FHERMA_API __attribute__((visibility("default")))
#else
#define FHERMA_API
#endif

FHERMA_API void* fherma_init(const fherma::Point& p);
FHERMA_API fherma::Outputs fherma_run(void* state, const fherma::Inputs& in);
FHERMA_API void fherma_free(void* state);
