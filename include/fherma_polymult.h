/*
 * fherma_polymult.h - C ABI of the B200 exact negacyclic multiplier.
 *
 *     c = a * b  mod (X^N + 1, q)
 *
 * computed exactly for coefficients of up to 2048 bits, each stored as L
 * little-endian u32 limbs (L = ceil(W / 32)); operands and result are N x L
 * arrays, coefficient-major, with every coefficient in [0, q).
 *
 * Plain C: opaque handles, pointers and sizes; no C++ or torch types.  Every
 * function returns 0 on success or one of the FPM_E* codes; the message of the
 * last failure on the calling thread is in fpm_last_error().  There is no CPU
 * fallback: without a usable CUDA device, fpm_init fails with FPM_ECUDA.
 *
 * The reference (Akram275/fherma-polymult) exposes the same three steps as C++
 * functions taking std::vector-based structs (fherma.h:46-48).  Those exact C++
 * symbols are exported too (declared in fherma_abi.h), so the reference's
 * generated harness links against this library unchanged.
 */
#ifndef FHERMA_POLYMULT_H
#define FHERMA_POLYMULT_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FPM_API __attribute__((visibility("default")))
#else
#define FPM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define FPM_OK 0
#define FPM_EINVAL 1    /* bad argument or out-of-range point (N, L, q) */
#define FPM_ECUDA 2     /* CUDA runtime failure */
#define FPM_ENOMEM 3    /* device or host allocation failed */
#define FPM_EINTERNAL 4 /* anything else */
#define FPM_ETIMEOUT 5  /* a kernel pipeline wait ran out of time: the product's result is not valid */

typedef struct fpm_ctx fpm_ctx;

typedef struct fpm_info {
    uint32_t N, W, L;
    uint32_t K;           /* primes in the RNS basis */
    uint32_t logN, logR, logS; /* transform geometry: N = 2^logR x 2^logS */
    int32_t device;       /* CUDA device the context lives on (-1: host-only query) */
    uint64_t device_bytes; /* device memory the context holds: tables + workspaces */
    uint32_t prime_bits;  /* every prime is below 2^prime_bits */
} fpm_info;

/* Replaces fherma_init (reference fherma.h:46, solve.cu:710-869): builds the
 * prime basis and constant tables for (N, q) and keeps them resident on the
 * current CUDA device.  q has L limbs with a nonzero top limb; N is a power of
 * two in [2, 2^22]; 1 <= L <= 64.  W is recorded, as the reference does. */
FPM_API int fpm_init(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, fpm_ctx** out);

/* fpm_init with the RNS prime window chosen explicitly: prime_bits = 30 keeps
 * every prime below 2^30 (lazy butterflies, the default), 31 reproduces the
 * reference's prime set exactly (rns_plan.h:141-153); 0 means the default,
 * which the environment variable FPM_PRIME_BITS may override.  Results are
 * identical either way. */
FPM_API int fpm_init_ex(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int prime_bits, fpm_ctx** out);

/* Replaces fherma_run (reference fherma.h:47, solve.cu:871-1059): one product
 * on HOST buffers a, b, c (N x L u32 each, any host memory); returns when c is
 * written.  Calls on one context must not overlap. */
FPM_API int fpm_run(fpm_ctx* ctx, const uint32_t* a, const uint32_t* b, uint32_t* c);

/* Counterpart of the copy-mode measurement in the reference's fherma_init
 * (solve.cu:805-862): times the host path of fpm_run on this point with 1 to
 * 4 copy chunks (each candidate 1 + 3 products on the context's own pinned
 * buffers) and keeps the fastest, the default unless another is 5% faster;
 * the count is returned in *chunks (may be NULL).  Synchronous.  fherma_init
 * calls it; without it fpm_run uses the default. */
FPM_API int fpm_tune_host_path(fpm_ctx* ctx, int* chunks);

/* One product on DEVICE buffers (N x L u32 each), enqueued on `stream` (a
 * cudaStream_t, NULL for the legacy default stream); returns after enqueueing.
 * Calls on one context must be ordered on one stream (they share workspaces). */
FPM_API int fpm_run_device(fpm_ctx* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, void* stream);

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory once they are running -- a process held to a fixed device-memory
 * budget, or a caller issuing work where cudaMalloc is not allowed -- this is
 * fpm_run_device with the product's scratch (the two K x N residue workspaces
 * and the error word) in one static device array of 80 MiB that every GPU
 * loading the library holds until the process exits; the call itself
 * allocates nothing.  The caller passes a context from fpm_init (made on the
 * current device) and the device buffers a, b, c (N x L u32 each).  A point
 * needing more than 80 MiB of scratch (2 K N words: every point up to
 * N = 65536 at W = 2048 fits) returns FPM_EINVAL with a message naming both
 * sizes.  The first call on each device looks up the array's address and
 * loads its module: make it before any stream capture.  All calls, from every
 * context, share the one array: calls whose work overlaps on the GPU race, so
 * order them on one stream.  The kernels are those of fpm_run_device.  A
 * kernel whose pipeline wait runs out sets the array's error word, which
 * stays set until fpm_noalloc_get_error reads and clears it. */
FPM_API int fpm_run_device_noalloc(fpm_ctx* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c,
                                   void* stream);

/* Device-path errors (the reference reports CUDA failures by exception from
 * fherma_run, solve.cu:84-88; the device entry points here return after
 * enqueueing, so a failure inside their kernels is read afterwards).  Every
 * wait inside the tensor-core kernels is bounded (2 s by default); one that
 * runs out makes the kernel set a bit in an error word and return early, so
 * the GPU never hangs but that product's c is wrong.  fpm_run checks the word
 * itself and returns FPM_ETIMEOUT.
 *
 * fpm_get_error waits for the work enqueued on `stream`, then reads and
 * clears the context's error word: FPM_ETIMEOUT if any product of this
 * context since the last check (fpm_run_device, stage entry points) had a wait
 * run out, FPM_OK otherwise.  fpm_noalloc_get_error does the same for the
 * error word of the static scratch array on the current device, which every
 * fpm_run_device_noalloc call on that device shares; it allocates nothing. */
FPM_API int fpm_get_error(fpm_ctx* ctx, void* stream);
FPM_API int fpm_noalloc_get_error(void* stream);

/* The limit of every pipeline wait in the context's kernels, in nanoseconds
 * (default 2e9); applies to products enqueued afterwards on this context
 * (batches and servers copy it when they are created). */
FPM_API int fpm_set_wait_limit(fpm_ctx* ctx, uint64_t ns);

/* Test hook, for checking the error path without faulting the GPU: with mask
 * bit 0 (decompose) or bit 1 (CRT) set, the pipelined kernel of later
 * products on this context never requests one of its shared-memory copies, so
 * the wait for it runs out after the wait limit and the call reports
 * FPM_ETIMEOUT.  0 restores normal operation. */
FPM_API int fpm_debug_inject_stall(fpm_ctx* ctx, uint32_t mask);

/* Replaces fherma_free (reference fherma.h:48, solve.cu:1061-1083); accepts
 * NULL. */
FPM_API void fpm_free(fpm_ctx* ctx);

/* Message of the last failure on this thread ("" if none). */
FPM_API const char* fpm_last_error(void);

FPM_API int fpm_get_info(const fpm_ctx* ctx, fpm_info* out);
/* Host-only: the plan fpm_init would build for (N, q) (no CUDA call): fills
 * out (device = -1) and, if primes is not NULL, the K primes.  Used to check a
 * point and to size its device footprint before admitting it. */
FPM_API int fpm_plan_info(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, fpm_info* out, uint32_t* primes);
FPM_API int fpm_plan_info_ex(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int prime_bits, fpm_info* out,
                             uint32_t* primes);
/* The K primes of the RNS basis, in order (same set and order as the
 * reference's make_plan, rns_plan.h:138-153). */
FPM_API int fpm_get_primes(const fpm_ctx* ctx, uint32_t* out);
/* The context's CRT constants as built on the device by fpm_init: M_j =
 * P / p_j mod q (K x L limbs) and negvP_v = -v P mod q ((K + 1) x L), the
 * tables of the reference's make_plan (rns_plan.h:224-247).  fpm_init builds
 * them from the prime basis with one short kernel; the q-independent tables
 * (twiddles, decompose constants) are shared by every context on the device
 * with the same N, L, bit length of q and prime window, so a context for a new
 * modulus of a width in use builds and uploads only these. */
FPM_API int fpm_get_crt_tables(const fpm_ctx* ctx, uint32_t* M, uint32_t* negvP);

/* Stage entry points on device buffers, enqueued on `stream` (no reference
 * counterpart as functions; they expose the reference's kernels' results for
 * stage-by-stage checks):
 *   decompose: limbs (N x L) -> residues (K x N, prime-major); operand 0 gives
 *              a mod p_j, operand 1 gives b mod p_j times the pointwise scale
 *              N^-1 (P/p_j)^-1 2^32 (reference k_decompose, solve.cu:98-126).
 *              With 30-bit primes and N > 1024 the values are left below
 *              4 p_j (congruent; the transform's first butterflies are lazy),
 *              otherwise they are canonical; operand 2 does both in the one
 *              launch a product uses: d_limbs holds a then b (2 N L words),
 *              d_res receives A then B (2 K N words);
 *   transform: mode 0: A, B -> y_j = INTT(NTT(A) NTT(B)) in A (reference
 *              k_ntt_cols / k_ntt_rows_mul, solve.cu:130-233); mode 1: forward
 *              transforms of A and B in place, bit-reversed order;
 *   crt:       y (K x N) -> c (N x L) mod q (reference k_crt, solve.cu:264-277). */
FPM_API int fpm_stage_decompose(fpm_ctx* ctx, const uint32_t* d_limbs, uint32_t* d_res, int operand, void* stream);
FPM_API int fpm_stage_transform(fpm_ctx* ctx, uint32_t* d_A, uint32_t* d_B, int mode, void* stream);
/* Modes 2, 3, 4 of fpm_stage_transform launch one kernel of the chain alone
 * (forward column pass, fused row pass, inverse column pass), for timing. */
FPM_API int fpm_stage_crt(fpm_ctx* ctx, const uint32_t* d_y, uint32_t* d_c, void* stream);

/* ------------------------------------------------------------------------
 * Batches (no reference counterpart; the reference runs one product per
 * fherma_run call).  A batch runs many products of uneven N and q width in
 * one CUDA graph of grouped launches: each stage kernel covers the tiles of
 * every product at once, so small products fill the GPU beside large ones.
 * Each product's point is a context from fpm_init (its tables stay resident);
 * the batch owns device buffers for every product's a, b and c and its
 * residue workspaces.  A context may appear in several batches and more than
 * once in one; contexts must outlive the batch. */
typedef struct fpm_batch fpm_batch;

typedef struct fpm_batch_info {
    uint32_t count;        /* products */
    int32_t layout;        /* 0 one stream; 1 transform geometries as parallel graph
                              branches; 2 a whole branch per geometry; 3 one launch per
                              stage (every transform pass covers all products with
                              N = 2^12 .. 2^17 in one launch, whatever their lengths) */
    int32_t order;         /* 0 as given; 1 largest product first */
    int32_t prime_group;   /* primes per transform work item (0: all of a product's) */
    int32_t grid;          /* transform grids: 0 one block per tile, k > 0 persistent */
    int32_t pipe_min_log_n; /* products with logN >= this (0: none) take the one-product
                               pipelined decompose and CRT */
    int32_t launches;      /* kernel launches in one graph replay */
    uint64_t device_bytes; /* device memory the batch holds */
    double tuned_us;       /* graph time of the chosen schedule (0 until fpm_batch_tune) */
} fpm_batch_info;

/* Builds a batch over ctxs[0 .. count-1] (all on the current device) and
 * captures its graph with the default schedule. */
FPM_API int fpm_batch_create(fpm_ctx* const* ctxs, uint32_t count, fpm_batch** out);
/* Device buffers of product i (N_i x L_i u32 each): write a and b, read c. */
FPM_API int fpm_batch_buffers(fpm_batch* batch, uint32_t i, uint32_t** d_a, uint32_t** d_b, uint32_t** d_c);
/* Every product on the batch's device buffers: one graph launch on `stream`
 * (a cudaStream_t; returns after enqueueing).  Replays on one batch must be
 * ordered on one stream. */
FPM_API int fpm_batch_run_device(fpm_batch* batch, void* stream);
/* The same from host arrays: a[i], b[i] in, c[i] out (N_i x L_i u32 each);
 * returns when every c[i] is written. */
FPM_API int fpm_batch_run(fpm_batch* batch, const uint32_t* const* a, const uint32_t* const* b, uint32_t* const* c);
/* Autotuner: times every candidate schedule on this batch (one warm-up and
 * `reps` graph replays each, on the batch's current buffers) and keeps the
 * fastest; the result is reported in info (may be NULL). */
FPM_API int fpm_batch_tune(fpm_batch* batch, int reps, fpm_batch_info* info);
/* Sets a schedule explicitly (fields as in fpm_batch_info) and recaptures. */
FPM_API int fpm_batch_set_schedule(fpm_batch* batch, int layout, int order, int prime_group, int grid,
                                   int pipe_min_log_n);
FPM_API int fpm_batch_get_info(const fpm_batch* batch, fpm_batch_info* out);
FPM_API void fpm_batch_free(fpm_batch* batch);

/* ------------------------------------------------------------------------
 * Serving (no reference counterpart).  A server keeps a set of points
 * (contexts from fpm_init, tables resident) and a device arena of
 * budget_bytes.  Each request -- c = a b on one of the points, host buffers --
 * needs 3 N L + 2 K N words of the arena (fpm_server_footprint) and is
 * admitted in arrival order once that much is free and one of `lanes` CUDA
 * streams is idle; a lane takes up to max_batch arrived requests and runs
 * them as one micro-batch of grouped launches (copies in, decompose,
 * transforms, CRT, copies out).  Lanes run concurrently, so requests that
 * arrive while others are on the GPU start as soon as a lane and memory free
 * up (continuous batching).  Host buffers should be pinned (cudaHostAlloc)
 * for the copies to overlap.  Contexts must outlive the server. */
typedef struct fpm_server fpm_server;

typedef struct fpm_server_stats {
    uint64_t completed, failed;
    uint64_t batches;          /* micro-batches launched */
    uint32_t lanes, max_lanes_busy;
    uint64_t budget_bytes, peak_bytes; /* arena size and its high-water mark */
} fpm_server_stats;

FPM_API int fpm_server_create(fpm_ctx* const* points, uint32_t count, uint64_t budget_bytes, int lanes,
                              int max_batch, fpm_server** out);
/* Adds a point to a running server (thread-safe) and returns its index in
 * *index; requests on it may be submitted at once.  Since the prime-basis
 * tables are shared across contexts (fpm_get_crt_tables), a context for a new
 * modulus of a width the server already holds takes little set-up, so new
 * moduli can join mid-stream.  The context must outlive the server. */
FPM_API int fpm_server_add_point(fpm_server* srv, fpm_ctx* point, uint32_t* index);
/* Device bytes one request on `point` takes from the arena. */
FPM_API int fpm_server_footprint(const fpm_server* srv, uint32_t point, uint64_t* bytes);
/* Queues a request (thread-safe; returns at once).  FPM_EINVAL if it can
 * never fit the budget. */
FPM_API int fpm_server_submit(fpm_server* srv, uint32_t point, const uint32_t* a, const uint32_t* b, uint32_t* c,
                              uint64_t* ticket);
/* Blocks until the request's c is written; latency from submit, in us. */
FPM_API int fpm_server_wait(fpm_server* srv, uint64_t ticket, double* latency_us);
/* Replays a trace: request i on point[i] is submitted arrival_us[i]
 * microseconds after the call starts; returns when all are done, with each
 * request's latency in latency_us[i]. */
FPM_API int fpm_server_replay(fpm_server* srv, uint32_t n, const uint32_t* point, const double* arrival_us,
                              const uint32_t* const* a, const uint32_t* const* b, uint32_t* const* c,
                              double* latency_us);
FPM_API int fpm_server_get_stats(const fpm_server* srv, fpm_server_stats* out);
FPM_API void fpm_server_free(fpm_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* FHERMA_POLYMULT_H */
