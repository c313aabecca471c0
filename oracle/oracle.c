/*
 * oracle.c -- CPU restatement of the LibShalom small/irregular GEMM path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this file.  It is used by tests/ (as the checker), by
 * __graft_entry__.smoke() (as the checker) and by bench.py's cpu_baseline
 * leg / `--impl reference` arm (as the timed CPU restatement of the
 * reference, because the reference's AArch64 NEON assembly cannot be built
 * or run on an x86 host).
 *
 * Parity status: the reference ships no golden vectors, known-answer tests
 * or fixtures for this path (its only checks are abs-tolerance comparisons
 * against OpenBLAS inside unbuilt benchmark mains:
 * NN_LIB/benchmark.c:154-173 (tol 1e-4) and evaluate/test.c:75-102
 * (tol 0.01, call commented out)).  The restatement below follows the
 * reference's arithmetic order as read from its assembly; where that order
 * is pinned by executing the reference's own instruction stream (see
 * oracle/neon_emu.py when present) the tests say so, otherwise parity is
 * "unpinned".
 *
 * Contents
 *   1. Input generators
 *        - drand48-compatible LCG, reproducing the reference benchmarks'
 *          random_matrix(): a[i] = 2.0*(float)drand48() - 1.0
 *          (benchmark/small_SGEMM/LibShalom_sgemm.c:26-34).
 *        - normal(0,1)*10^u generator for the batched-DGEMM workload.
 *   2. Exact-math oracles: C = alpha*A*op(B) + beta*C accumulated in
 *      double (FP32 inputs) or x87 long double (FP64 inputs).
 *   3. Reference-order restatements (FP32/FP64 rounding order of the
 *      reference kernels):
 *        - k-sequential FMA per output element (KERNEL5x16_* of
 *          NN_LIB/test_temp.c:622-1082, test_temp_L1.c, the KERNEL5x16 rows
 *          of test_SMM_NT.c:315-775 and DGEMM_NN.c's KERNEL7x6_*);
 *        - the lane-split dot product of SGEMM_NT's first 5-row block of
 *          every 16-column strip (PACK_KERNEL5x4_*, test_SMM_NT.c:9-270:
 *          four k (mod 4) partial sums combined as (s0+s1)+(s2+s3) by
 *          faddp);
 *        - the GEMM_K=320 K-blocking of the mp drivers
 *          (NN_LIB/SMM_NN_new.c:209-231 with k_tag: block 0 stores,
 *          later blocks add their fresh partial into C, M8N12_PACK_ADD_C).
 *   4. CPU baseline "port": the reference's algorithm restated in C for
 *      x86 (5x16 FP32 register tile with the B strip packed during the
 *      first row block, 7x6 FP64 tile, the Dete_grad_* Tm x Tn OpenMP
 *      thread grid, GEMM_K blocking), plus OpenMP loops over batches.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_GEMM_K 320 /* NN_LIB/LibShalom.h:14 */

/* ------------------------------------------------------------------ */
/* 1. generators                                                       */
/* ------------------------------------------------------------------ */

/* drand48: X_{n+1} = (a X_n + c) mod 2^48, a = 0x5DEECE66D, c = 0xB.
 * srand48(s) sets X_0 = (s << 16) | 0x330E (POSIX). drand48 returns
 * X_{n+1} / 2^48 (exactly representable in a double). */
static const uint64_t LCG_A = 0x5DEECE66DULL;
static const uint64_t LCG_C = 0xBULL;
static const uint64_t LCG_MASK = (1ULL << 48) - 1;

static uint64_t lcg_seed(uint64_t seed) {
  return (((seed & 0xffffffffULL) << 16) | 0x330EULL) & LCG_MASK;
}

/* advance the LCG state by n steps in O(log n) */
static uint64_t lcg_skip(uint64_t x, uint64_t n) {
  uint64_t acc_mult = 1, acc_plus = 0;
  uint64_t cur_mult = LCG_A, cur_plus = LCG_C;
  while (n) {
    if (n & 1) {
      acc_mult = (acc_mult * cur_mult) & LCG_MASK;
      acc_plus = (acc_plus * cur_mult + cur_plus) & LCG_MASK;
    }
    cur_plus = ((cur_mult + 1) * cur_plus) & LCG_MASK;
    cur_mult = (cur_mult * cur_mult) & LCG_MASK;
    n >>= 1;
  }
  return (acc_mult * x + acc_plus) & LCG_MASK;
}

static inline double lcg_next(uint64_t *x) {
  *x = (LCG_A * *x + LCG_C) & LCG_MASK;
  return (double)*x * (1.0 / 281474976710656.0);
}

/* raw drand48 stream: out[i] = the (skip+i+1)-th drand48() after srand48(seed) */
void orc_drand48(uint64_t seed, uint64_t skip, long n, double *out) {
  uint64_t x = lcg_skip(lcg_seed(seed), skip);
  for (long i = 0; i < n; ++i) out[i] = lcg_next(&x);
}

/* random_matrix() of the reference benchmarks, element by element:
 * a = 2.0 * (float)drand48() - 1.0, stored to float. */
void orc_fill_uniform_f32(uint64_t seed, uint64_t skip, long n, float *out) {
  uint64_t x = lcg_skip(lcg_seed(seed), skip);
  for (long i = 0; i < n; ++i) {
    float f = (float)lcg_next(&x);
    out[i] = (float)(2.0 * (double)f - 1.0);
  }
}

/* same generator widened to double (FP64 variant of random_matrix) */
void orc_fill_uniform_f64(uint64_t seed, uint64_t skip, long n, double *out) {
  uint64_t x = lcg_skip(lcg_seed(seed), skip);
  for (long i = 0; i < n; ++i) out[i] = 2.0 * lcg_next(&x) - 1.0;
}

/* normal(0,1) * 10^u, u ~ U[-3,3] drawn once per matrix: one matrix of n
 * entries consumes 1 + 2*ceil(n/2) draws (u first, then Box-Muller pairs). */
void orc_fill_normal_scaled_f64(uint64_t seed, uint64_t skip, long n,
                                double *out, double *scale_out) {
  uint64_t x = lcg_skip(lcg_seed(seed), skip);
  double u = -3.0 + 6.0 * lcg_next(&x);
  double s = pow(10.0, u);
  if (scale_out) *scale_out = s;
  for (long i = 0; i < n; i += 2) {
    double u1 = lcg_next(&x), u2 = lcg_next(&x);
    double r = sqrt(-2.0 * log(1.0 - u1));
    double t = 6.283185307179586476925286766559 * u2;
    out[i] = s * r * cos(t);
    if (i + 1 < n) out[i + 1] = s * r * sin(t);
  }
}

/* ------------------------------------------------------------------ */
/* 2. exact-math oracles                                               */
/* ------------------------------------------------------------------ */
/* Row-major: A is M x K (lda), op(B) = B (K x N, ldb) when transb == 0,
 * B^T with B stored N x K (ldb) when transb != 0.  C is M x N (ldc).
 * out = alpha * A op(B) + beta * Cin   (Cin may be NULL when beta == 0). */

void orc_sgemm_f64(int transb, long M, long N, long K, double alpha,
                   const float *A, long lda, const float *B, long ldb,
                   double beta, const float *Cin, long ldc, double *out) {
#pragma omp parallel for schedule(static) if (M * N * K > (1L << 22))
  for (long i = 0; i < M; ++i)
    for (long j = 0; j < N; ++j) {
      double acc = 0.0;
      if (transb)
        for (long k = 0; k < K; ++k)
          acc += (double)A[i * lda + k] * (double)B[j * ldb + k];
      else
        for (long k = 0; k < K; ++k)
          acc += (double)A[i * lda + k] * (double)B[k * ldb + j];
      double r = alpha * acc;
      if (beta != 0.0) r += beta * (double)Cin[i * ldc + j];
      out[i * N + j] = r;
    }
}

/* |A| |op(B)| in double, for componentwise error bounds */
void orc_sgemm_absprod(int transb, long M, long N, long K, const float *A,
                       long lda, const float *B, long ldb, double *out) {
#pragma omp parallel for schedule(static) if (M * N * K > (1L << 22))
  for (long i = 0; i < M; ++i)
    for (long j = 0; j < N; ++j) {
      double acc = 0.0;
      for (long k = 0; k < K; ++k) {
        double b = transb ? B[j * ldb + k] : B[k * ldb + j];
        acc += fabs((double)A[i * lda + k]) * fabs(b);
      }
      out[i * N + j] = acc;
    }
}

/* FP64 oracle in x87 extended precision (64-bit significand) */
void orc_dgemm_ld(int transb, long M, long N, long K, double alpha,
                  const double *A, long lda, const double *B, long ldb,
                  double beta, const double *Cin, long ldc, double *out) {
#pragma omp parallel for schedule(static) if (M * N * K > (1L << 22))
  for (long i = 0; i < M; ++i)
    for (long j = 0; j < N; ++j) {
      long double acc = 0.0L;
      if (transb)
        for (long k = 0; k < K; ++k)
          acc += (long double)A[i * lda + k] * (long double)B[j * ldb + k];
      else
        for (long k = 0; k < K; ++k)
          acc += (long double)A[i * lda + k] * (long double)B[k * ldb + j];
      long double r = (long double)alpha * acc;
      if (beta != 0.0) r += (long double)beta * (long double)Cin[i * ldc + j];
      out[i * N + j] = (double)r;
    }
}

/* ------------------------------------------------------------------ */
/* 3. reference-order restatements                                     */
/* ------------------------------------------------------------------ */

/* k-sequential FMA per element: acc = a0*b0 (fmul), acc = fma(ak,bk,acc).
 * This is the rounding order of KERNEL5x16_BEGIN_K/K0..K7 (fmul then fmla
 * by element; test_temp.c:622-1082, test_SMM_NT.c:315-775) and of
 * DGEMM_NN's KERNEL7x6_* + EDGE_K_KERNEL7x6 (DGEMM_NN.c:2333-2470).
 * kblock > 0 restates the mp drivers' GEMM_K blocking: each block's
 * partial starts fresh and is added into C (SMM_NN_new.c:209-231,
 * M8N12_PACK_ADD_C at Kernel/SMM_m8n12_new.h:77-91). */
void orc_sgemm_kseq(int transb, long M, long N, long K, const float *A,
                    long lda, const float *B, long ldb, float *C, long ldc,
                    long kblock) {
  if (kblock <= 0) kblock = K > 0 ? K : 1;
#pragma omp parallel for schedule(static) if (M * N * K > (1L << 22))
  for (long i = 0; i < M; ++i)
    for (long j = 0; j < N; ++j) {
      float c = 0.0f;
      for (long k0 = 0; k0 < K; k0 += kblock) {
        long k1 = k0 + kblock < K ? k0 + kblock : K;
        float acc = 0.0f;
        for (long k = k0; k < k1; ++k) {
          float b = transb ? B[j * ldb + k] : B[k * ldb + j];
          acc = (k == k0) ? A[i * lda + k] * b : fmaf(A[i * lda + k], b, acc);
        }
        c = (k0 == 0) ? acc : c + acc;
      }
      C[i * ldc + j] = c;
    }
}

void orc_dgemm_kseq(int transb, long M, long N, long K, const double *A,
                    long lda, const double *B, long ldb, double *C,
                    long ldc) {
#pragma omp parallel for schedule(static) if (M * N * K > (1L << 22))
  for (long i = 0; i < M; ++i)
    for (long j = 0; j < N; ++j) {
      double acc = 0.0;
      for (long k = 0; k < K; ++k) {
        double b = transb ? B[j * ldb + k] : B[k * ldb + j];
        acc = (k == 0) ? A[i * lda + k] * b : fma(A[i * lda + k], b, acc);
      }
      C[i * ldc + j] = acc;
    }
}

/* DGEMM_NN rounding order (DGEMM_NN.c:5, driver at :2333).  Columns in the
 * 6-wide strips and in the N4 tail block are k-sequential FMA chains
 * (KERNEL7x6_*, EDGE_K_KERNEL7x6, N4 kernels).  The single trailing column
 * of the N1 tail (N % 2 == 1, BEGIN_N1 at :3319) runs the KERNEL4x1/1x1
 * kernels (:2265-2332): lane 0 accumulates even k, lane 1 odd k (fmul, then
 * fmla over pairs of k), an odd last k is fmadd-ed into lane 0
 * (EDGE_K_KERNEL1x1) and SAVE adds the lanes with faddp: C = s_even + s_odd.
 * The N2 tail (N % 6 in {2,3}) is not restated: its output is wrong in the
 * reference for several row tails (see the golden fixtures), and rows with
 * M % 7 in {1,3,4} past 7*(M/7) are never written by the reference.  This
 * function computes every element with the order of the path that covers its
 * column. */
void orc_dgemm_reforder(long M, long N, long K, const double *A,
                        const double *B, double *C) {
  const long n1col = (N % 2 == 1) ? N - 1 : -1;
  for (long i = 0; i < M; ++i)
    for (long j = 0; j < N; ++j) {
      const double *a = A + i * K;
      if (j == n1col && K >= 2) {
        double s0 = a[0] * B[j], s1 = a[1] * B[N + j];
        long k = 2;
        for (; k + 1 < K; k += 2) {
          s0 = fma(a[k], B[k * N + j], s0);
          s1 = fma(a[k + 1], B[(k + 1) * N + j], s1);
        }
        if (k < K) s0 = fma(a[k], B[k * N + j], s0);
        C[i * N + j] = s0 + s1;
      } else {
        double acc = a[0] * B[j];
        for (long k = 1; k < K; ++k) acc = fma(a[k], B[k * N + j], acc);
        C[i * N + j] = acc;
      }
    }
}

/* SGEMM_NT rounding order (test_SMM_NT.c:6 driver at :2181).  For every
 * 16-column strip (and the trailing 8-column strip), rows 0..4 run the
 * pack-fused PACK_KERNEL5x4_* kernels: lane l of the accumulator holds
 * s_l = sum over k = l (mod 4), started by fmul and continued by fmla in k
 * order, and the faddp tree of PACK_KERNEL5x4_END_K (:207-269) returns
 * (s0 + s1) + (s2 + s3).  All other rows use KERNEL5x16/4x16/... on the
 * packed strip, which is k-sequential.  Requires K % 4 == 0 (the reference
 * additionally requires K % 8 == 0 and N % 8 == 0). */
void orc_sgemm_nt_reforder(long M, long N, long K, const float *A,
                           const float *B, float *C) {
  for (long j = 0; j < N; ++j)
    for (long i = 0; i < M; ++i) {
      const float *a = A + i * K, *b = B + j * K;
      if (i < 5) {
        float s[4];
        for (int l = 0; l < 4; ++l) {
          s[l] = a[l] * b[l];
          for (long k = l + 4; k < K; k += 4) s[l] = fmaf(a[k], b[k], s[l]);
        }
        C[i * N + j] = (s[0] + s[1]) + (s[2] + s[3]);
      } else {
        float acc = a[0] * b[0];
        for (long k = 1; k < K; ++k) acc = fmaf(a[k], b[k], acc);
        C[i * N + j] = acc;
      }
    }
}

/* ------------------------------------------------------------------ */
/* 4. CPU baseline port of the reference algorithm                    */
/* ------------------------------------------------------------------ */

/* 5x16 FP32 register tile over a 16-column B strip packed k-major
 * (the SB panel of test_temp.c / test_SMM_NT.c).  Tails use the same code
 * with masked extents (the reference uses 4/3/2/1x16 and N8/N4/N2/N1
 * kernels; the arithmetic order per element is the same k-sequential FMA). */
static void port_strip(long M, long K, long nb, const float *A, long lda,
                       const float *SB, float *C, long ldc, int add) {
  long i = 0;
  /* full 5-row blocks: constant trip counts so the compiler keeps the 5x16
   * accumulator tile in vector registers (the v12..v31 tile of KERNEL5x16) */
  for (; i + 5 <= M; i += 5) {
    float acc[5][16];
    for (int r = 0; r < 5; ++r)
      for (int c = 0; c < 16; ++c) acc[r][c] = 0.0f;
    const float *a0 = A + i * lda;
    for (long k = 0; k < K; ++k) {
      const float *b = SB + k * 16;
      for (int r = 0; r < 5; ++r) {
        float a = a0[r * lda + k];
        for (int c = 0; c < 16; ++c) acc[r][c] = fmaf(a, b[c], acc[r][c]);
      }
    }
    for (int r = 0; r < 5; ++r)
      for (long c = 0; c < nb; ++c) {
        float *dst = C + (i + r) * ldc + c;
        *dst = add ? *dst + acc[r][c] : acc[r][c];
      }
  }
  for (; i < M; i += 5) {
    long mb = M - i < 5 ? M - i : 5;
    float acc[5][16];
    for (long r = 0; r < 5; ++r)
      for (int c = 0; c < 16; ++c) acc[r][c] = 0.0f;
    for (long k = 0; k < K; ++k) {
      const float *b = SB + k * 16;
      for (long r = 0; r < mb; ++r) {
        float a = A[(i + r) * lda + k];
        for (int c = 0; c < 16; ++c) acc[r][c] = fmaf(a, b[c], acc[r][c]);
      }
    }
    for (long r = 0; r < mb; ++r)
      for (long c = 0; c < nb; ++c) {
        float *dst = C + (i + r) * ldc + c;
        *dst = add ? *dst + acc[r][c] : acc[r][c];
      }
  }
}

/* Pack a 16-column strip of op(B) into SB[k][16] (zero padded). */
static void port_pack(int transb, long K, long j0, long nb, const float *B,
                      long ldb, float *SB) {
  for (long k = 0; k < K; ++k)
    for (int c = 0; c < 16; ++c)
      SB[k * 16 + c] =
          c < nb ? (transb ? B[(j0 + c) * ldb + k] : B[k * ldb + j0 + c]) : 0.0f;
}

/* LibShalom_sgemm restated (NN_LIB/NN_SMM.c:5-27): single thread. */
void orc_port_sgemm(int transb, long M, long N, long K, const float *A,
                    long lda, const float *B, long ldb, float *C, long ldc) {
  float *SB = (float *)malloc(sizeof(float) * (K > 0 ? K : 1) * 16);
  for (long j = 0; j < N; j += 16) {
    long nb = N - j < 16 ? N - j : 16;
    port_pack(transb, K, j, nb, B, ldb, SB);
    port_strip(M, K, nb, A, lda, SB, C + j, ldc, 0);
  }
  free(SB);
}

/* LibShalom_dgemm restated: 7x6 FP64 tile (DGEMM_NN.c:2333-3420), NN only,
 * every row and column computed (the reference skips rows with
 * M % 7 in {1,3,4}). */
void orc_port_dgemm(long M, long N, long K, const double *A, long lda,
                    const double *B, long ldb, double *C, long ldc,
                    int accumulate) {
  for (long j = 0; j < N; j += 6) {
    long nb = N - j < 6 ? N - j : 6;
    for (long i = 0; i < M; i += 7) {
      long mb = M - i < 7 ? M - i : 7;
      double acc[7][6];
      memset(acc, 0, sizeof(acc));
      for (long k = 0; k < K; ++k)
        for (long r = 0; r < mb; ++r) {
          double a = A[(i + r) * lda + k];
          for (long c = 0; c < 6; ++c)
            acc[r][c] = fma(a, c < nb ? B[k * ldb + j + c] : 0.0, acc[r][c]);
        }
      for (long r = 0; r < mb; ++r)
        for (long c = 0; c < nb; ++c) {
          double *dst = C + (i + r) * ldc + j + c;
          *dst = accumulate ? *dst + acc[r][c] : acc[r][c];
        }
    }
  }
}

/* Dete_grad_N_threads_nums / Dete_grad_M_threads_nums
 * (NN_LIB/SMM_thread.c:14-72) with vec = all divisors of T. */
static void port_thread_grid(int T, long M, long N, int transb, int by_m,
                             int *Tm, int *Tn) {
  int divs[64], nd = 0;
  for (int i = 1; i <= T && nd < 64; ++i)
    if (T % i == 0) divs[nd++] = i;
  if (!by_m) {
    int tn = (int)ceil(sqrt((transb ? 1.0 : 4.0) * T * (float)N / (float)M));
    for (int i = 0; i < nd; ++i)
      if (tn <= divs[i]) {
        if (i > 0 && (tn - divs[i - 1] <= divs[i] - tn)) tn = divs[i - 1];
        else tn = divs[i];
        break;
      }
    if (tn >= T) tn = T;
    if (tn < 1) tn = 1;
    *Tn = tn;
    *Tm = T / tn;
  } else {
    int tm = (int)ceil(sqrt(T * (float)M / (float)N));
    for (int i = 0; i < nd; ++i)
      if (tm <= divs[i]) { tm = divs[i]; break; }
    if (tm >= T) tm = T;
    if (tm < 1) tm = 1;
    *Tm = tm;
    *Tn = T / tm;
  }
}

/* LibShalom_sgemm_mp restated (SMM_thread.c:75-113 dispatch, SMM_NN_new.c /
 * SMM_NT_new.c drivers): a Tm x Tn grid of OpenMP threads, each owning a
 * slab of C (remainders assigned, unlike the reference's NGM drivers), the
 * K dimension blocked by GEMM_K = 320 with block 0 storing and later blocks
 * accumulating.  The per-element order equals orc_sgemm_kseq(kblock=320). */
void orc_port_sgemm_mp(int transb, long M, long N, long K, const float *A,
                       const float *B, float *C, int threads) {
  int T = threads > 0 ? threads : 1, Tm, Tn;
  int by_m = transb ? !(M < N) : (N > 0 && M / N >= 5);
  port_thread_grid(T, M, N, transb, by_m, &Tm, &Tn);
  long ldb = transb ? K : N;
#pragma omp parallel num_threads(Tm * Tn)
  {
#ifdef _OPENMP
    int id = omp_get_thread_num();
#else
    int id = 0;
#endif
    int ti = id / Tn, tj = id % Tn;
    long mper = (M + Tm - 1) / Tm, nper = (N + Tn - 1) / Tn;
    nper = (nper + 15) / 16 * 16;
    long i0 = ti * mper, i1 = i0 + mper < M ? i0 + mper : M;
    long j0 = tj * nper, j1 = j0 + nper < N ? j0 + nper : N;
    float *SB = (float *)malloc(sizeof(float) * ORC_GEMM_K * 16);
    for (long j = j0; j < j1; j += 16) {
      long nb = j1 - j < 16 ? j1 - j : 16;
      for (long k0 = 0; k0 < K; k0 += ORC_GEMM_K) {
        long kb = K - k0 < ORC_GEMM_K ? K - k0 : ORC_GEMM_K;
        const float *Bk = transb ? B + k0 : B + k0 * ldb;
        port_pack(transb, kb, j, nb, Bk, ldb, SB);
        if (i1 > i0)
          port_strip(i1 - i0, kb, nb, A + i0 * K + k0, K, SB,
                     C + i0 * N + j, N, k0 != 0);
      }
    }
    free(SB);
  }
}

/* Batched restatements: OpenMP over independent GEMMs.  Each entry i has
 * A_i = A + offA[i], B_i = B + offB[i], C_i = C + offC[i] (row-major, packed
 * leading dimensions), out_i = alpha*A_i op(B_i) + beta_i*C_i. */
void orc_port_sgemm_batched(long count, const int *M, const int *N,
                            const int *K, const int *transb,
                            const float *beta, const float *A,
                            const long *offA, const float *B,
                            const long *offB, float *C, const long *offC,
                            int threads) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
  for (long g = 0; g < count; ++g) {
    long m = M[g], n = N[g], k = K[g];
    long ldb = transb[g] ? k : n;
    float *c = C + offC[g];
    if (beta[g] == 0.0f) {
      orc_port_sgemm(transb[g], m, n, k, A + offA[g], k, B + offB[g], ldb, c, n);
    } else {
      float *tmp = (float *)malloc(sizeof(float) * (m * n > 0 ? m * n : 1));
      orc_port_sgemm(transb[g], m, n, k, A + offA[g], k, B + offB[g], ldb, tmp, n);
      for (long e = 0; e < m * n; ++e) c[e] = tmp[e] + beta[g] * c[e];
      free(tmp);
    }
  }
}

/* uniform batch: count GEMMs of one shape, matrices packed back to back */
void orc_port_sgemm_strided(int transb, long M, long N, long K, long count,
                            const float *A, const float *B, float *C,
                            int threads) {
  long ldb = transb ? K : N;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
  for (long g = 0; g < count; ++g)
    orc_port_sgemm(transb, M, N, K, A + g * M * K, K, B + g * K * N, ldb,
                   C + g * M * N, N);
}

/* batched DGEMM, C += A*B, runs of `run` consecutive products share one C
 * block (owner computes per run: deterministic, no atomics). */
void orc_port_dgemm_batched(long count, const int *M, const int *N,
                            const int *K, const double *A, const long *offA,
                            const double *B, const long *offB, double *C,
                            const long *offC, int threads) {
  /* entries that share offC are contiguous; each thread owns whole runs */
  long nruns = 0;
  long *starts = (long *)malloc(sizeof(long) * (count + 1));
  for (long g = 0; g < count; ++g)
    if (g == 0 || offC[g] != offC[g - 1]) starts[nruns++] = g;
  starts[nruns] = count;
#pragma omp parallel for schedule(dynamic, 8) num_threads(threads > 0 ? threads : 1)
  for (long r = 0; r < nruns; ++r)
    for (long g = starts[r]; g < starts[r + 1]; ++g)
      orc_port_dgemm(M[g], N[g], K[g], A + offA[g], K[g], B + offB[g], N[g],
                     C + offC[g], N[g], 1);
  free(starts);
}

/* FP64 oracle for the batched DGEMM workload: every C element of a run is
 * accumulated in x87 long double over all products of the run, in run
 * order, and rounded to double once. */
void orc_dgemm_batched_ld(long count, const int *M, const int *N, const int *K,
                          const double *A, const long *offA, const double *B,
                          const long *offB, double *C, const long *offC) {
  long g = 0;
  while (g < count) {
    long e = g + 1;
    while (e < count && offC[e] == offC[g]) ++e;
    long m = M[g], n = N[g];
    double *c = C + offC[g];
    for (long i = 0; i < m; ++i)
      for (long j = 0; j < n; ++j) {
        long double acc = c[i * n + j];
        for (long p = g; p < e; ++p) {
          const double *a = A + offA[p], *b = B + offB[p];
          long k = K[p];
          for (long kk = 0; kk < k; ++kk)
            acc += (long double)a[i * k + kk] * (long double)b[kk * n + j];
        }
        c[i * n + j] = (double)acc;
      }
    g = e;
  }
}

/* correctly rounded fused multiply-add, element-wise (used by the AArch64
 * interpreter in neon_emu.py to execute fmla / fmadd exactly) */
void orc_fma_f32_vec(long n, const float *a, const float *b, const float *c, float *out) {
  for (long i = 0; i < n; ++i) out[i] = fmaf(a[i], b[i], c[i]);
}
void orc_fma_f64_vec(long n, const double *a, const double *b, const double *c, double *out) {
  for (long i = 0; i < n; ++i) out[i] = fma(a[i], b[i], c[i]);
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
