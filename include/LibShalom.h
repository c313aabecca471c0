/*
 * LibShalom.h -- B200 (sm_100a) small and irregular-shaped GEMM library.
 *
 * Drop-in C ABI for the public interface of LibShalom
 * (NN_LIB/LibShalom.h:9-41 of the ARMv8 reference).  The five reference
 * entry points keep their names, argument order, types and void returns;
 * this header is plain C (the reference header needs C++ for <vector>), so
 * callers relink against this library after recompiling.
 *
 * Differences a caller must know:
 *   - A, B and C are meant to be DEVICE pointers (cudaMalloc'd or managed
 *     memory).  The drop-in calls also accept the reference's own use, HOST
 *     buffers (malloc'd or page-locked; classified with
 *     cudaPointerGetAttributes): such a call runs as the matching _host call
 *     below, copying its operands through the library's staging slots.
 *   - Calls are synchronous by default (C is final when the call returns),
 *     as in the reference; LibShalom_set_sync(0) makes them stream-ordered
 *     on the stream given to LibShalom_set_stream().
 *   - Errors: the reference silently ignores bad input (void, no checks).
 *     Here every call records a status readable with
 *     LibShalom_get_last_error() (per host thread); nothing is launched
 *     for invalid arguments.
 *   - transa: the reference ignores it (NN_LIB/NN_SMM.c:8,33 comment it
 *     out).  Here transa == Trans means A is stored K x M (BLAS meaning).
 *   - LibShalom_dgemm with transb == Trans: the reference does nothing
 *     (NN_SMM.c:30-37); here it computes C = A * B^T.
 *   - Every row and column of C is computed (the reference leaves some
 *     tail rows/columns unwritten in DGEMM_NN and the NGM mp drivers).
 */
#ifndef LIBSHALOM_B200_H
#define LIBSHALOM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LIBSHALOM_API __attribute__((visibility("default")))
#else
#define LIBSHALOM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* NN_LIB/LibShalom.h:9-12 */
#define NoTrans 0
#define Trans 1

/* NN_LIB/LibShalom.h:14-16: the reference's cache-blocking constants.  Here
 * GEMM_K is the K-block at which the plain sgemm_mp path folds its running
 * partial into C (the reference's k_tag accumulation), which keeps the
 * plain FP32 rounding order equal to the reference mp drivers'. */
#define GEMM_K 320
#define GEMM_N 4096
#define GEMM_M 256

/* ---------------------------------------------------------------------- */
/* Drop-in entry points                                                   */
/* ---------------------------------------------------------------------- */

/* C[M x N] = A[M x K] * op(B), row-major; op(B) = B (K x N) for NoTrans, B^T
 * with B stored N x K for Trans.  Replaces NN_LIB/LibShalom.h:22
 * (implementation NN_LIB/NN_SMM.c:5-27: SGEMM_NN / SGEMM_NN_L1 /
 * SGEMM_NT).  Plain FP32: k-sequential fused multiply-add per element. */
LIBSHALOM_API void LibShalom_sgemm(int transa, int transb, float *C, float *A, float *B,
                     long M, long N, long K);

/* Irregular-shaped SGEMM (tall-skinny / im2col shapes).  Replaces
 * NN_LIB/LibShalom.h:27 (implementation NN_LIB/SMM_thread.c:75-113 and the
 * drivers of SMM_NN_new.c / SMM_NT_new.c).  Uses the precision mode set by
 * LibShalom_set_precision() (default plain FP32). */
LIBSHALOM_API void LibShalom_sgemm_mp(int transa, int transb, float *C, float *A, float *B,
                        long M, long N, long K);

/* C = A * op(B) in FP64.  Replaces NN_LIB/LibShalom.h:38 (implementation
 * NN_LIB/NN_SMM.c:30-37 -> DGEMM_NN.c:5). */
LIBSHALOM_API void LibShalom_dgemm(int transa, int transb, double *C, double *A, double *B,
                     long M, long N, long K);

/* Replaces NN_LIB/LibShalom.h:40 (SMM_thread.c:116-130).  The reference sets
 * its OpenMP thread count; here num caps the number of CTAs resident at once
 * for every kernel of the library (num <= 0 removes the cap: all SMs). */
LIBSHALOM_API void LibShalom_set_thread_nums(int num);

/* Replaces NN_LIB/LibShalom.h:41 (SMM_thread.c:132-137).  Forces the
 * tm x tn partition of C for the NEXT LibShalom_sgemm_mp call only (the
 * reference resets Tm after each mp call, SMM_thread.c:112): the C tile grid
 * is split into tm x tn rectangular groups, one CTA per group. */
LIBSHALOM_API void LibShalom_set_thread_ways(int tm, int tn);

/* ---------------------------------------------------------------------- */
/* Status and execution control (no counterpart in the reference, which   */
/* has no error reporting)                                                 */
/* ---------------------------------------------------------------------- */

#define LIBSHALOM_SUCCESS 0
#define LIBSHALOM_ERR_INVALID_VALUE 1 /* bad size, pointer, trans or mode */
#define LIBSHALOM_ERR_UNSUPPORTED 2   /* valid request this build cannot run */
#define LIBSHALOM_ERR_CUDA 3          /* a CUDA runtime call failed */
#define LIBSHALOM_ERR_NO_DEVICE 4     /* no sm_100 device visible */
#define LIBSHALOM_ERR_ALLOC 5         /* workspace allocation failed */
#define LIBSHALOM_ERR_DEVICE_TIMEOUT 6 /* a bounded device-side wait expired */

/* Status of the last library call made by this host thread. */
LIBSHALOM_API int LibShalom_get_last_error(void);
/* Static description of a status code. */
LIBSHALOM_API const char *LibShalom_error_string(int status);

/* Stream for all later launches (a cudaStream_t; NULL = default stream).
 * Switching streams first waits for the library's work on the old stream,
 * whose calls may still read the library's device buffers. */
LIBSHALOM_API int LibShalom_set_stream(void *stream);
/* 1 (default): calls return after the result is written.  0: calls are
 * stream-ordered and return after the launch. */
LIBSHALOM_API int LibShalom_set_sync(int synchronous);
/* Wait for all work the library queued on its stream. */
LIBSHALOM_API int LibShalom_synchronize(void);

/* Arithmetic of LibShalom_sgemm_mp and LibShalom_sgemm_batched*. */
#define LIBSHALOM_PREC_FP32 0   /* plain FP32 FMA on the CUDA cores */
#define LIBSHALOM_PREC_BF16X3 1 /* hi/lo BF16 split, 3 tcgen05 products */
#define LIBSHALOM_PREC_BF16X6 2 /* hi/mid/lo BF16 split, 6 tcgen05 products */
LIBSHALOM_API int LibShalom_set_precision(int mode);
LIBSHALOM_API int LibShalom_get_precision(void);

/* Split-K factor for LibShalom_sgemm_mp: 0 = chosen by the tile scheduler
 * (default), 1 = never split, s > 1 = split K into s slices. */
LIBSHALOM_API int LibShalom_set_splitk(int splits);

/* Tuning hooks (no counterpart in the reference).  The single and mp entry
 * points take their tile configuration (plain kernels) and split-K factor
 * from a table of measured choices per shape class (half-octaves of M, N, K;
 * written by libshalom_b200/autotune.py on a B200 and compiled in), else from
 * a cost model.  set_tile_config forces a plain tile configuration
 * (0..6 FP32: 32x32, 64x64, 128x32, 32x128, 128x64, 64x128, 128x128;
 * 0..3 FP64: 32x32, 64x64, 128x32, 32x128; -1 = table/model); a value the
 * data type does not have makes the call fail with
 * LIBSHALOM_ERR_INVALID_VALUE; calls with transa == Trans always use
 * configuration 1 (64x64).  set_autotune(0) ignores the table.
 * get_plan reports the tile configuration (-1 on the tensor-core path) and
 * split-K factor of the last single / mp call and the table's entry count. */
LIBSHALOM_API int LibShalom_set_tile_config(int cfg);

/* Graph cache (no counterpart in the reference): with enable != 0 and a
 * non-default stream set, a LibShalom_sgemm / _sgemm_mp / _dgemm call whose
 * pointers, sizes and library settings repeat is captured into a CUDA graph
 * the second time and replayed by one graph launch from then on (up to 256
 * cached calls; a call that makes the library's workspace grow recaptures).
 * The data behind the pointers may change between calls.  Replays do not
 * report an expired device-side wait as LIBSHALOM_ERR_DEVICE_TIMEOUT.
 * enable == 0 (default) frees the cached graphs. */
LIBSHALOM_API int LibShalom_set_graph_cache(int enable);
LIBSHALOM_API int LibShalom_set_autotune(int enable);
LIBSHALOM_API int LibShalom_get_plan(int *tile_config, int *splits, int *table_entries);

/* Operand staging of the tensor-core kernels: 1 (default) = TMA
 * (cp.async.bulk.tensor) with warp-specialized producer / converter / MMA /
 * epilogue warps whenever the operands are 16-byte aligned with 16-byte row
 * strides; 0 = always the cp.async kernel (any alignment).  Results are the
 * same either way. */
LIBSHALOM_API int LibShalom_set_tma(int enable);

/* Self-check of failure detection (no counterpart in the reference).  Every
 * wait of the library's tensor-core kernels on an mbarrier is bounded: after
 * its limit the waiting role sets an abort flag and a device status word,
 * the other roles give up when they see the flag, the kernel frees what it
 * holds and returns, and a synchronous call reports
 * LIBSHALOM_ERR_DEVICE_TIMEOUT instead of hanging the GPU.  This call runs
 * that path on purpose: a one-CTA kernel waits on an mbarrier that nothing
 * arrives at (one warp for `iterations` polls, 0 = 4096, the other with the
 * kernels' own limit).  Synchronous.  Returns LIBSHALOM_ERR_DEVICE_TIMEOUT
 * when the waits expired, the kernel returned and the host read the status
 * (the expected outcome, after which the context stays usable);
 * LIBSHALOM_SUCCESS would mean the expiry went unreported. */
LIBSHALOM_API int LibShalom_selftest_wait_expiry(int iterations);

/* Release the library's device workspace and cached plans. */
LIBSHALOM_API void LibShalom_finalize(void);

/* ---------------------------------------------------------------------- */
/* Batched entry points (no counterpart in the reference)                 */
/* ---------------------------------------------------------------------- */

/* One GEMM of a grouped batch: C = alpha * A * op(B) + beta * C, row-major.
 * lda/ldb/ldc <= 0 select the packed defaults (K, N or K, N). */
typedef struct LibShalom_sgemm_entry {
  const float *A;
  const float *B;
  float *C;
  int32_t M, N, K;
  int32_t transb;
  int32_t lda, ldb, ldc;
  float alpha, beta;
  int32_t reserved;
} LibShalom_sgemm_entry; /* 64 bytes */

typedef struct LibShalom_dgemm_entry {
  const double *A;
  const double *B;
  double *C;
  int32_t M, N, K;
  int32_t transb;
  int32_t lda, ldb, ldc;
  int32_t reserved;
  double alpha, beta;
} LibShalom_dgemm_entry; /* 72 bytes */

/* Grouped SGEMM over `count` entries that live in DEVICE memory.  Entries
 * are independent unless they name the same C; entries that share a C must
 * be contiguous in the array, have the same M and N, and are applied in
 * array order by one CTA. */
LIBSHALOM_API int LibShalom_sgemm_batched(const LibShalom_sgemm_entry *entries, long count);

/* Uniform batch: count GEMMs of one shape, matrix g at A + g*strideA etc. */
LIBSHALOM_API int LibShalom_sgemm_batched_strided(int transb, long M, long N, long K,
                                    float alpha, const float *A, long strideA,
                                    const float *B, long strideB, float beta,
                                    float *C, long strideC, long count);

/* Host-memory calls.  The reference's calls take HOST pointers; these do
 * too (A, B and C in host memory; page-locked memory lets the copies run
 * asynchronously), with the math, dispatch and status of the device-pointer
 * calls of the same name.  The operands travel through a device staging
 * buffer of three slots held by the library until LibShalom_finalize: the
 * batched call is cut into chunks of whole GEMMs (about 64 MB of operands
 * each) whose host-to-device copies, kernels and device-to-host copies
 * overlap on three streams.  In asynchronous mode (LibShalom_set_sync(0))
 * the call returns once everything is queued and the library's stream is
 * ordered after the last copy back; the host buffers must stay valid until
 * then.  The batched call needs strideC >= M * N when count > 1; beta != 0
 * copies C in as well. */
LIBSHALOM_API void LibShalom_sgemm_host(int transa, int transb, float *C, const float *A,
                                        const float *B, long M, long N, long K);
LIBSHALOM_API void LibShalom_sgemm_mp_host(int transa, int transb, float *C, const float *A,
                                           const float *B, long M, long N, long K);
LIBSHALOM_API void LibShalom_dgemm_host(int transa, int transb, double *C, const double *A,
                                        const double *B, long M, long N, long K);
LIBSHALOM_API int LibShalom_sgemm_batched_strided_host(int transb, long M, long N, long K,
                                                       float alpha, const float *A,
                                                       long strideA, const float *B,
                                                       long strideB, float beta, float *C,
                                                       long strideC, long count);

/* Deferred drop-in calls (no counterpart in the reference): after
 * LibShalom_defer_begin, LibShalom_sgemm, LibShalom_sgemm_mp and
 * LibShalom_dgemm (device pointers, transa == NoTrans) are recorded as
 * entries in a page-locked host ring instead of launched, and return at once;
 * LibShalom_defer_flush copies the recorded entries to the device in one
 * transfer per precision, runs them as grouped batches (the
 * LibShalom_sgemm_batched / _dgemm_batched kernels under the precision and
 * DGEMM method of the recorded calls) and ends the deferral.  Many small calls then
 * cost a few launches instead of one each.  Plain FP32 and FP64 FMA results
 * are the same as the direct LibShalom_sgemm / LibShalom_dgemm calls';
 * LibShalom_sgemm_mp's GEMM_K blocking is not applied.  Order: a call that
 * reads a matrix a pending call writes, writes one a pending call reads, or
 * writes a pending call's C other than the directly preceding call's (same M
 * and N) first flushes the pending calls, and calls that cannot be recorded
 * (transa == Trans, or M N K above 128^3: the grouped kernels give each call
 * to one CTA, so larger calls run faster directly) flush and then run
 * directly; matrices
 * that overlap without sharing a base pointer are the caller's to keep
 * apart.  Every other call that launches work (the batched, _ex, _host,
 * stack, convolution and no-allocation calls) launches the pending calls
 * first, and so do LibShalom_set_stream, _set_precision, _set_dgemm_method,
 * _set_thread_nums and LibShalom_finalize: pending calls run under the
 * settings they were recorded with, on the device that was current then,
 * and are never dropped.  Results are ready once the flush has completed (synchronous mode)
 * or in stream order after it.  LibShalom_defer_pending returns the number
 * of recorded calls not yet launched. */
LIBSHALOM_API int LibShalom_defer_begin(void);
LIBSHALOM_API int LibShalom_defer_flush(void);
LIBSHALOM_API int LibShalom_defer_pending(void);

/* Split-K SGEMM that allocates nothing.  No counterpart in the reference.
 * For callers that cannot allocate device memory (their GPU memory is owned
 * by another allocator, or a cudaMalloc in the middle of a call is not
 * acceptable): same math and rounding order per K slice as
 * LibShalom_sgemm_mp with LibShalom_set_splitk(splits), precision always
 * plain FP32, but the partial sums live in a fixed array compiled into the
 * library (LIBSHALOM_NOALLOC_SCRATCH_FLOATS floats, held on every GPU that
 * loads the library until exit).  Returns LIBSHALOM_ERR_INVALID_VALUE, and
 * launches nothing, when splits * M * N exceeds that size.  The first call
 * on a device looks up the array's device address; make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race. */
#define LIBSHALOM_NOALLOC_SCRATCH_FLOATS (2L * 1024 * 1024) /* 8 MiB */
LIBSHALOM_API int LibShalom_sgemm_mp_noalloc(int transa, int transb, float *C, const float *A,
                                             const float *B, long M, long N, long K,
                                             int splits);

/* Plain calls with explicit leading dimensions and scaling (no counterpart in
 * the reference, whose API has implicit leading dimensions and no alpha /
 * beta): C = alpha op(A) op(B) + beta C, row-major, lda >= K (A NoTrans) or M
 * (A Trans), ldb >= N (B NoTrans) or K (B Trans), ldc >= N.  Scheduled like
 * LibShalom_sgemm_mp (tuning table, split-K; LibShalom_set_precision selects
 * the split-BF16 path of the FP32 call, which needs transa == NoTrans).
 * Return the status. */
LIBSHALOM_API int LibShalom_sgemm_ex(int transa, int transb, long M, long N, long K, float alpha,
                                     const float *A, long lda, const float *B, long ldb,
                                     float beta, float *C, long ldc);
LIBSHALOM_API int LibShalom_dgemm_ex(int transa, int transb, long M, long N, long K,
                                     double alpha, const double *A, long lda, const double *B,
                                     long ldb, double beta, double *C, long ldc);

/* Grouped DGEMM (same rules as LibShalom_sgemm_batched).  Arithmetic set by
 * LibShalom_set_dgemm_method. */
LIBSHALOM_API int LibShalom_dgemm_batched(const LibShalom_dgemm_entry *entries, long count);

/* Stack front end (no counterpart in the reference): a batch described the
 * way block-sparse chemistry codes keep their multiplication stacks -- data
 * pools plus per-product element offsets -- instead of per-GEMM pointers.
 * Product i: C_pool[c_off[i]..] = alpha A_pool[a_off[i]..] op(B_pool[b_off[i]..])
 * + beta C, dense row-major blocks (lda = K, ldb = N or K for Trans, ldc = N).
 * M / N / K are device arrays of count sizes, or NULL to give every product
 * m / n / k.  The offset arrays are device arrays.  Products that name the same
 * C offset consecutively accumulate in order (a run), exactly as in
 * LibShalom_dgemm_batched, whose arithmetic (LibShalom_set_dgemm_method) this
 * call uses.  The struct itself is read on the host. */
typedef struct LibShalom_dgemm_stack_desc {
  const double *A_pool;
  const double *B_pool;
  double *C_pool;
  const int32_t *M, *N, *K;
  int32_t m, n, k;
  int32_t transb;
  const int64_t *a_off, *b_off, *c_off;
  double alpha, beta;
} LibShalom_dgemm_stack_desc;
LIBSHALOM_API int LibShalom_dgemm_stack(const LibShalom_dgemm_stack_desc *stack, long count);

/* 2-D convolution front end (no counterpart in the reference; its CNN
 * benchmark feeds LibShalom_sgemm_mp with im2col shapes): FP32 NCHW
 * cross-correlation, x [n][c][h][w], weights [oc][c][kh][kw], y [n][oc][oh][ow]
 * with oh = (h + 2 ph - kh) / sh + 1, ow = (w + 2 pw - kw) / sw + 1, zero
 * padding; per image the GEMM (oc x c kh kw) (c kh kw x oh ow).  In FP32
 * precision it runs as an implicit GEMM on the CUDA cores (the tile loader
 * reads the im2col columns straight from x; no column buffer), with the mp
 * path's rounding order (GEMM_K blocks); in the split-BF16 modes each image
 * is expanded by im2col into a library buffer and multiplied on the mp path.
 * Device pointers; returns the status. */
LIBSHALOM_API int LibShalom_sconv2d_nchw(const float *x, long n, long c, long h, long w,
                                         const float *weights, long oc, long kh, long kw,
                                         long sh, long sw, long ph, long pw, float *y);

/* Arithmetic of LibShalom_dgemm_batched (no counterpart in the reference).
 * Runs whose C block is larger than 32 x 32 always take the FMA kernel. */
#define LIBSHALOM_DGEMM_FMA 0   /* FP64 FMA on the CUDA cores (default) */
#define LIBSHALOM_DGEMM_DMMA 1  /* FP64 tensor cores (mma.sync m8n8k4 f64) */
#define LIBSHALOM_DGEMM_OZAKI 2 /* Ozaki scheme: INT8 digit slices on the tensor
                                   cores, exact INT32 sums, FP64 recombination;
                                   finite inputs only */
/* slices: signed 7-bit digits per operand element for LIBSHALOM_DGEMM_OZAKI,
 * 4..9, 0 = 9.  Each product's error is about (S + 4) 2^(-7S) K max|A_i.|
 * max|op(B)_.j| per element: 9 digits keep it near 1e-16 of that scale, 8
 * near 2e-15, which can exceed 1e-14 of max|C| after cancellation.  Ignored
 * by the other methods. */
LIBSHALOM_API int LibShalom_set_dgemm_method(int method, int slices);
LIBSHALOM_API int LibShalom_get_dgemm_method(void);

#ifdef __cplusplus
}
#endif

#endif /* LIBSHALOM_B200_H */
