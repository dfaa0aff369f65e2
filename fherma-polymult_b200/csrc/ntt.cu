// Negacyclic NTT kernels: the column pass, the fused row pass (forward rows of
// both operands, pointwise product, inverse rows) and the inverse column pass of
// the four-step transform, plus a one-block-per-prime kernel for N <= 1024.
//
// Reference counterparts (Akram275/fherma-polymult): k_ntt_cols solve.cu:130-166,
// k_ntt_rows_mul solve.cu:195-233, with the stage structure of
// rns_kernels.cuh:105-174.  Here every pass keeps 8 elements per thread in
// registers for up to three stages at a time (ntt_engine.cuh), the row pass
// builds its twiddles in shared memory from two small per-prime tables, and A
// and B share each twiddle load.
#include "device.cuh"
#include "kernels.h"
#include "ntt_engine.cuh"

namespace fpm {

namespace {

// ---------------------------------------------------------------------------
// Column pass: a block owns C = 2048 / R adjacent columns c0 .. c0 + C - 1 of one
// prime, all R rows: tile sub-transform g = column, position x = row u.
// Element (u, c) is X[u S + c0 + c].

template <int LOGR>
__device__ __forceinline__ void col_load(uint32_t* tile, const uint32_t* X, uint32_t S, uint32_t c0) {
    constexpr uint32_t C = kTileCols<LOGR>;
#pragma unroll 4
    for (uint32_t i = threadIdx.x; i < 2048; i += kNttThreads) {
        const uint32_t c = i & (C - 1), u = i >> (11 - LOGR);
        tile[swz((c << LOGR) | u)] = X[static_cast<size_t>(u) * S + c0 + c];
    }
}

template <int LOGR>
__device__ __forceinline__ void col_store(const uint32_t* tile, uint32_t* X, uint32_t S, uint32_t c0) {
    constexpr uint32_t C = kTileCols<LOGR>;
#pragma unroll 4
    for (uint32_t i = threadIdx.x; i < 2048; i += kNttThreads) {
        const uint32_t c = i & (C - 1), u = i >> (11 - LOGR);
        X[static_cast<size_t>(u) * S + c0 + c] = tile[swz((c << LOGR) | u)];
    }
}

template <int NSUB, int R, int NV, class TW>
__device__ __forceinline__ void fwd_step(uint32_t* const (&tiles)[NV], const TW& tw, uint32_t p) {
    const uint32_t base = round_base<NSUB, R>(threadIdx.x);
    uint32_t v[NV][8];
#pragma unroll
    for (int o = 0; o < NV; ++o) load_round<NSUB, R>(tiles[o], v[o], base);
    fwd_round<NSUB, R, NV>(v, base, tw, p);
#pragma unroll
    for (int o = 0; o < NV; ++o) store_round<NSUB, R>(tiles[o], v[o], base);
    __syncthreads();
}

template <int NSUB, int R, class TW>
__device__ __forceinline__ void inv_step(uint32_t* tile, const TW& tw, uint32_t p) {
    const uint32_t base = round_base<NSUB, R>(threadIdx.x);
    uint32_t v[8];
    load_round<NSUB, R>(tile, v, base);
    inv_round<NSUB, R>(v, base, tw, p);
    store_round<NSUB, R>(tile, v, base);
    __syncthreads();
}

// Forward rounds R .. REND - 1.
template <int NSUB, int NV, class TW, int R, int REND>
__device__ __forceinline__ void fwd_range(uint32_t* const (&tiles)[NV], const TW& tw, uint32_t p) {
    if constexpr (R < REND) {
        fwd_step<NSUB, R, NV>(tiles, tw, p);
        fwd_range<NSUB, NV, TW, R + 1, REND>(tiles, tw, p);
    }
}

// Inverse rounds R, R - 1, ..., 0.
template <int NSUB, class TW, int R>
__device__ __forceinline__ void inv_from(uint32_t* tile, const TW& tw, uint32_t p) {
    if constexpr (R >= 0) {
        inv_step<NSUB, R>(tile, tw, p);
        inv_from<NSUB, TW, R - 1>(tile, tw, p);
    }
}

template <int LOGR>
__global__ void __launch_bounds__(kNttThreads) k_ntt_col_fwd(DevPoint d, uint32_t* A, uint32_t* B) {
    extern __shared__ __align__(16) uint32_t smem[];
    constexpr uint32_t R = 1u << LOGR, C = kTileCols<LOGR>;
    uint32_t* ta = smem;
    uint32_t* tb = smem + 2048;
    uint2* tw = reinterpret_cast<uint2*>(smem + 4096);
    const int j = blockIdx.y;
    const uint32_t S = 1u << d.logS, c0 = blockIdx.x * C;
    const uint32_t p = d.pc[j].p;
    for (uint32_t y = threadIdx.x; y < R; y += kNttThreads) tw[y] = d.col_f[static_cast<size_t>(j) * R + y];
    col_load<LOGR>(ta, A + static_cast<size_t>(j) * d.N, S, c0);
    col_load<LOGR>(tb, B + static_cast<size_t>(j) * d.N, S, c0);
    __syncthreads();
    uint32_t* const tiles[2] = {ta, tb};
    fwd_range<LOGR, 2, SharedTable, 0, Rounds<LOGR>::kCount>(tiles, SharedTable{tw}, p);
    col_store<LOGR>(ta, A + static_cast<size_t>(j) * d.N, S, c0);
    col_store<LOGR>(tb, B + static_cast<size_t>(j) * d.N, S, c0);
}

template <int LOGR>
__global__ void __launch_bounds__(kNttThreads) k_ntt_col_inv(DevPoint d, uint32_t* A) {
    extern __shared__ __align__(16) uint32_t smem[];
    constexpr uint32_t R = 1u << LOGR, C = kTileCols<LOGR>;
    uint32_t* ta = smem;
    uint2* tw = reinterpret_cast<uint2*>(smem + 2048);
    const int j = blockIdx.y;
    const uint32_t S = 1u << d.logS, c0 = blockIdx.x * C;
    const uint32_t p = d.pc[j].p;
    for (uint32_t y = threadIdx.x; y < R; y += kNttThreads) tw[y] = d.col_i[static_cast<size_t>(j) * R + y];
    col_load<LOGR>(ta, A + static_cast<size_t>(j) * d.N, S, c0);
    __syncthreads();
    inv_from<LOGR, SharedTable, Rounds<LOGR>::kCount - 1>(ta, SharedTable{tw}, p);
    col_store<LOGR>(ta, A + static_cast<size_t>(j) * d.N, S, c0);
}

// ---------------------------------------------------------------------------
// Row pass: a block owns G = 2048 / S consecutive rows u0 .. u0 + G - 1 of one
// prime (2048 contiguous elements).  It first builds each row's forward and
// inverse twiddle tables in shared memory: entry y of row u for the stage of
// distance 2^b is U[u][b] * Q[y] (plan.h), with its Shoup companion derived
// from mu.

template <int LOGS>
__device__ __forceinline__ void row_twiddles(uint2* tf, uint2* ti, const DevPoint& d, int j, uint32_t u0) {
    constexpr uint32_t S = 1u << LOGS;
    const PrimeConsts pc = d.pc[j];
    const uint32_t R = 1u << d.logR;
    const uint2* uf = d.row_u_f + (static_cast<size_t>(j) * R + u0) * LOGS;
    const uint2* ui = d.row_u_i + (static_cast<size_t>(j) * R + u0) * LOGS;
    const uint2* qf = d.row_q_f + static_cast<size_t>(j) * S;
    const uint2* qi = d.row_q_i + static_cast<size_t>(j) * S;
    for (uint32_t i = threadIdx.x; i < 2048; i += kNttThreads) {
        const uint32_t g = i >> LOGS, y = i & (S - 1);
        if (y == 0) continue;
        const uint32_t b = LOGS - 1 - (31 - __clz(y));
        const uint2 f = uf[g * LOGS + b], fi = ui[g * LOGS + b];
        const uint2 q1 = qf[y], q2 = qi[y];
        tf[i] = make_twiddle(shoup(f.x, q1.x, q1.y, pc.p), pc);
        ti[i] = make_twiddle(shoup(fi.x, q2.x, q2.y, pc.p), pc);
    }
}

template <int LOGS>
__global__ void __launch_bounds__(kNttThreads) k_ntt_row(DevPoint d, uint32_t* A, uint32_t* B, int mode) {
    extern __shared__ __align__(16) uint32_t smem[];
    constexpr uint32_t S = 1u << LOGS, G = 2048u >> LOGS;
    uint32_t* ta = smem;
    uint32_t* tb = smem + 2048;
    uint2* tf = reinterpret_cast<uint2*>(smem + 4096);
    uint2* ti = tf + 2048;
    const int j = blockIdx.y;
    const uint32_t u0 = blockIdx.x * G;
    const PrimeConsts pc = d.pc[j];
    uint32_t* a = A + static_cast<size_t>(j) * d.N + static_cast<size_t>(u0) * S;
    uint32_t* b = B + static_cast<size_t>(j) * d.N + static_cast<size_t>(u0) * S;
    row_twiddles<LOGS>(tf, ti, d, j, u0);
#pragma unroll 4
    for (uint32_t i = threadIdx.x; i < 2048; i += kNttThreads) {
        ta[swz(i)] = a[i];
        tb[swz(i)] = b[i];
    }
    __syncthreads();
    using RP = Rounds<LOGS>;
    constexpr int last = RP::kCount - 1;
    const PerRowTable<LOGS> fw{tf}, iw{ti};
    uint32_t* const tiles[2] = {ta, tb};
    // Forward rounds but the last through shared memory.
    fwd_range<LOGS, 2, PerRowTable<LOGS>, 0, last>(tiles, fw, pc.p);
    // The last forward round stays in registers when the product follows.
    {
        const uint32_t base = round_base<LOGS, last>(threadIdx.x);
        uint32_t v[2][8];
        load_round<LOGS, last>(ta, v[0], base);
        load_round<LOGS, last>(tb, v[1], base);
        fwd_round<LOGS, last, 2>(v, base, fw, pc.p);
        if (mode == kRowForward) {
            store_round<LOGS, last>(ta, v[0], base);
            store_round<LOGS, last>(tb, v[1], base);
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) v[0][k] = mont_mul(v[0][k], v[1][k], pc.p, pc.pneg);
            inv_round<LOGS, last>(v[0], base, iw, pc.p);
            store_round<LOGS, last>(ta, v[0], base);
        }
        __syncthreads();
    }
    if (mode == kRowForward) {
#pragma unroll 4
        for (uint32_t i = threadIdx.x; i < 2048; i += kNttThreads) {
            a[i] = ta[swz(i)];
            b[i] = tb[swz(i)];
        }
        return;
    }
    if constexpr (last > 0) inv_from<LOGS, PerRowTable<LOGS>, last - 1>(ta, iw, pc.p);
#pragma unroll 4
    for (uint32_t i = threadIdx.x; i < 2048; i += kNttThreads) a[i] = ta[swz(i)];
}

// ---------------------------------------------------------------------------
// N <= 1024: one block per prime holds both operands; one butterfly per
// thread per stage, full twiddle tables from global memory.

__global__ void __launch_bounds__(kNttThreads) k_ntt_small(DevPoint d, uint32_t* A, uint32_t* B, int mode) {
    extern __shared__ __align__(16) uint32_t smem[];
    const uint32_t N = d.N, logN = d.logN;
    uint32_t* ta = smem;
    uint32_t* tb = smem + N;
    const int j = blockIdx.x;
    const PrimeConsts pc = d.pc[j];
    const uint2* tf = d.full_f + static_cast<size_t>(j) * N;
    const uint2* ti = d.full_i + static_cast<size_t>(j) * N;
    uint32_t* a = A + static_cast<size_t>(j) * N;
    uint32_t* b = B + static_cast<size_t>(j) * N;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
        ta[i] = a[i];
        tb[i] = b[i];
    }
    __syncthreads();
    for (int s = static_cast<int>(logN) - 1; s >= 0; --s) {
        for (uint32_t bf = threadIdx.x; bf < N / 2; bf += blockDim.x) {
            const uint32_t i = bf >> s, lo = (i << (s + 1)) | (bf & ((1u << s) - 1)), hi = lo + (1u << s);
            const uint2 w = tf[(N >> (s + 1)) + i];
            ct_butterfly(ta[lo], ta[hi], w, pc.p);
            ct_butterfly(tb[lo], tb[hi], w, pc.p);
        }
        __syncthreads();
    }
    if (mode == kRowForward) {
        for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
            a[i] = ta[i];
            b[i] = tb[i];
        }
        return;
    }
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) ta[i] = mont_mul(ta[i], tb[i], pc.p, pc.pneg);
    __syncthreads();
    for (uint32_t s = 0; s < logN; ++s) {
        for (uint32_t bf = threadIdx.x; bf < N / 2; bf += blockDim.x) {
            const uint32_t i = bf >> s, lo = (i << (s + 1)) | (bf & ((1u << s) - 1)), hi = lo + (1u << s);
            gs_butterfly(ta[lo], ta[hi], ti[(N >> (s + 1)) + i], pc.p);
        }
        __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) a[i] = ta[i];
}

template <int LOGR>
void set_col_attrs() {
    check(cudaFuncSetAttribute(k_ntt_col_fwd<LOGR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(col_fwd_smem(LOGR))),
          "col smem");
    check(cudaFuncSetAttribute(k_ntt_col_inv<LOGR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(col_inv_smem(LOGR))),
          "col smem");
}

template <int LOGS>
void set_row_attrs() {
    check(cudaFuncSetAttribute(k_ntt_row<LOGS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(row_smem())),
          "row smem");
}

template <int LOGR>
void launch_col_fwd_t(const DevPoint& d, uint32_t* A, uint32_t* B, cudaStream_t st) {
    const dim3 grid((1u << d.logS) / kTileCols<LOGR>, d.K);
    k_ntt_col_fwd<LOGR><<<grid, kNttThreads, col_fwd_smem(LOGR), st>>>(d, A, B);
}

template <int LOGR>
void launch_col_inv_t(const DevPoint& d, uint32_t* A, cudaStream_t st) {
    const dim3 grid((1u << d.logS) / kTileCols<LOGR>, d.K);
    k_ntt_col_inv<LOGR><<<grid, kNttThreads, col_inv_smem(LOGR), st>>>(d, A);
}

template <int LOGS>
void launch_row_t(const DevPoint& d, uint32_t* A, uint32_t* B, int mode, cudaStream_t st) {
    const dim3 grid((1u << d.logR) / (2048u >> LOGS), d.K);
    k_ntt_row<LOGS><<<grid, kNttThreads, row_smem(), st>>>(d, A, B, mode);
}

}  // namespace

size_t col_fwd_smem(uint32_t logR) { return 2 * 2048 * sizeof(uint32_t) + (size_t(1) << logR) * sizeof(uint2); }
size_t col_inv_smem(uint32_t logR) { return 2048 * sizeof(uint32_t) + (size_t(1) << logR) * sizeof(uint2); }
size_t row_smem() { return 2 * 2048 * sizeof(uint32_t) + 2 * 2048 * sizeof(uint2); }

void ntt_init_attributes() {
    set_col_attrs<6>();
    set_col_attrs<7>();
    set_col_attrs<8>();
    set_col_attrs<9>();
    set_col_attrs<10>();
    set_col_attrs<11>();
    set_row_attrs<6>();
    set_row_attrs<7>();
    set_row_attrs<8>();
    set_row_attrs<9>();
    set_row_attrs<10>();
    set_row_attrs<11>();
    check(cudaFuncSetAttribute(k_ntt_small, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 1024 * 4),
          "small smem");
}

// The product's transform chain on residues A, B (K x N each): y_j in A.
// mode kRowForward stops after the forward transforms (A, B bit-reversed).
void launch_ntt(const DevPoint& d, uint32_t* A, uint32_t* B, int mode, cudaStream_t st) {
    if (d.logN <= kSmallLogN) {
        k_ntt_small<<<d.K, kNttThreads, 2 * d.N * sizeof(uint32_t), st>>>(d, A, B, mode);
        return;
    }
    switch (d.logR) {
        case 0: break;
        case 6: launch_col_fwd_t<6>(d, A, B, st); break;
        case 7: launch_col_fwd_t<7>(d, A, B, st); break;
        case 8: launch_col_fwd_t<8>(d, A, B, st); break;
        case 9: launch_col_fwd_t<9>(d, A, B, st); break;
        case 10: launch_col_fwd_t<10>(d, A, B, st); break;
        case 11: launch_col_fwd_t<11>(d, A, B, st); break;
        default: throw std::runtime_error("unsupported column length");
    }
    switch (d.logS) {
        case 6: launch_row_t<6>(d, A, B, mode, st); break;
        case 7: launch_row_t<7>(d, A, B, mode, st); break;
        case 8: launch_row_t<8>(d, A, B, mode, st); break;
        case 9: launch_row_t<9>(d, A, B, mode, st); break;
        case 10: launch_row_t<10>(d, A, B, mode, st); break;
        case 11: launch_row_t<11>(d, A, B, mode, st); break;
        default: throw std::runtime_error("unsupported row length");
    }
    if (mode == kRowForward) return;
    switch (d.logR) {
        case 0: break;
        case 6: launch_col_inv_t<6>(d, A, st); break;
        case 7: launch_col_inv_t<7>(d, A, st); break;
        case 8: launch_col_inv_t<8>(d, A, st); break;
        case 9: launch_col_inv_t<9>(d, A, st); break;
        case 10: launch_col_inv_t<10>(d, A, st); break;
        case 11: launch_col_inv_t<11>(d, A, st); break;
        default: throw std::runtime_error("unsupported column length");
    }
}

}  // namespace fpm
