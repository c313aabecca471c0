// ls_simt.cuh -- plain FP32 / FP64 GEMM tiles on the CUDA cores.
//
// One CTA computes a BM x BN tile of C = alpha * op(A) op(B) + beta * C over
// a K range.  The reference's "packing inside the micro-kernel" (the first
// PACK_KERNEL pass writes the packed B panel while computing,
// NN_LIB/test_temp.c:9-536, test_SMM_NT.c:9-270) becomes the staging step of
// the tile itself: each K-slab of A and op(B) is copied by cp.async from
// row-major global memory straight into shared memory, in the operand's own
// row-major layout (no transpose pass, no packed copy in global memory), in a
// STAGES-deep ring so several slabs' loads are in flight while the current
// one is multiplied.  Rows whose k runs along the 128-byte smem row (A[m][k],
// and B[n][k] for Trans) are XOR-swizzled in 16-byte units so that the lanes
// of a quarter warp, which read rows RG apart, hit distinct banks; rows along
// m / n (A[k][m] for transa, B[k][n]) are read as consecutive vectors.  The
// copies are 16 bytes wide when the operand's rows are 16-byte aligned, else
// element-wise.  Tails in m, n and k are zero-filled by the copies and
// predicated in the stores, replacing the reference's 4/3/2/1x16,
// N8/N4/N2/N1 and EDGE_K kernel families.
//
// Rounding order: every output element is one fused multiply-add chain over
// k in increasing order starting from zero, the order of the reference's
// KERNEL5x16_* / KERNEL7x6_* register tiles.  With KBLOCK > 0 the chain is
// restarted every KBLOCK values of k and each block's partial is added into
// the running sum, the GEMM_K = 320 blocking of the reference mp drivers
// (NN_LIB/SMM_NN_new.c:209-231, k_tag != 0 -> ADD_C).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ls {

template <typename T>
struct GemmArgs {
  const T *A;
  const T *B;
  T *C;
  long M, N, K;
  long lda, ldb, ldc;
  int transa, transb;
  T alpha, beta;
};

template <typename T, int BM_, int BN_, int TM_, int TN_>
struct SimtCfg {
  static constexpr int BM = BM_, BN = BN_, TM = TM_, TN = TN_;
  // K per slab: one 128-byte shared-memory row of k (32 floats, 16 doubles)
  static constexpr int BK = 128 / (int)sizeof(T);
  static constexpr int EPU = 16 / (int)sizeof(T);  // elements per 16-byte unit
  static constexpr int STAGES = 3;
  static constexpr int TX = BN / TN, TY = BM / TM, NTH = TX * TY;
  // rows of a thread: NRGM groups of RGM consecutive rows, groups BM/NRGM apart
  static constexpr int RGM = TM >= 4 ? 4 : TM, NRGM = TM / RGM;
  static constexpr int RGN = TN >= 4 ? 4 : TN, NRGN = TN / RGN;
  static constexpr int A_ELEMS = BM * BK, B_ELEMS = BN * BK;  // per stage
  static constexpr int STAGE_ELEMS = A_ELEMS + B_ELEMS;
  static constexpr int SMEM_ELEMS = STAGES * STAGE_ELEMS;
  static_assert(BM % TM == 0 && BN % TN == 0, "tile");
  static_assert(TM % RGM == 0 && TN % RGN == 0, "groups");
  static_assert(TX >= 8, "a quarter warp shares one row group of A");
};

// vector read of R consecutive elements from shared memory
template <typename T, int R>
__device__ __forceinline__ void lds_vec(const T *p, T *out) {
#pragma unroll
  for (int i = 0; i < R; ++i) out[i] = p[i];
}
template <>
__device__ __forceinline__ void lds_vec<float, 4>(const float *p, float *out) {
  float4 v = *reinterpret_cast<const float4 *>(p);
  out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
}
template <>
__device__ __forceinline__ void lds_vec<float, 2>(const float *p, float *out) {
  float2 v = *reinterpret_cast<const float2 *>(p);
  out[0] = v.x; out[1] = v.y;
}
template <>
__device__ __forceinline__ void lds_vec<double, 2>(const double *p, double *out) {
  double2 v = *reinterpret_cast<const double2 *>(p);
  out[0] = v.x; out[1] = v.y;
}
template <>
__device__ __forceinline__ void lds_vec<double, 4>(const double *p, double *out) {
  double2 v0 = *reinterpret_cast<const double2 *>(p);
  double2 v1 = *reinterpret_cast<const double2 *>(p + 2);
  out[0] = v0.x; out[1] = v0.y; out[2] = v1.x; out[3] = v1.y;
}

__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }

// ---- cp.async (global -> shared), zero fill past src_bytes ----
__device__ __forceinline__ void simt_cp16(uint32_t saddr, const void *g, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(g),
               "r"(src_bytes)
               : "memory");
}
template <int BYTES>
__device__ __forceinline__ void simt_cp(uint32_t saddr, const void *g, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(saddr), "l"(g), "n"(BYTES),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void simt_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void simt_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Where the tile reads op(B)[k][n] from: the dense row-major B of the
// GemmArgs (the GEMM calls), or a gather such as the implicit im2col columns
// of a convolution (ls_frontend.cu).  A gather returns the element's address
// (nullptr for a zero); only called for k < K and n < N.
struct DenseB {
  static constexpr bool kDense = true;
  template <typename T>
  __device__ __forceinline__ const T *ptr(const GemmArgs<T> &g, long k, long n) const {
    return g.transb ? g.B + n * g.ldb + k : g.B + k * g.ldb + n;
  }
};

// Copies an R x Cc block of a row-major matrix (rows at src + r * ld; rows
// >= rv or columns >= cv zero-filled) into rows of Cc elements at `dst`
// (Cc * sizeof(T) bytes a row); with SWZ the 16-byte unit u of row r is
// stored at u ^ ((r / RG) & 7) (rows of 128 bytes).
template <typename T, int R, int Cc, int NTH, bool SWZ, int RG>
__device__ __forceinline__ void stage_rows(uint32_t dst, const T *src, long ld, long rv, long cv,
                                           bool vec, int tid) {
  constexpr int EPU = 16 / (int)sizeof(T), UPR = Cc / EPU, CHUNKS = R * UPR;
#pragma unroll
  for (int e0 = 0; e0 < CHUNKS; e0 += NTH) {
    const int e = e0 + tid;
    if (CHUNKS % NTH != 0 && e >= CHUNKS) break;
    const int r = e / UPR, u = e - r * UPR;
    const int pu = SWZ ? (u ^ ((r / RG) & 7)) : u;
    const uint32_t d = dst + (uint32_t)(r * Cc * (int)sizeof(T) + pu * 16);
    const long c = (long)u * EPU;
    const int n = r < rv ? (int)max(0L, min((long)EPU, cv - c)) : 0;
    const T *p = src + (long)r * ld + c;
    if (vec) {
      simt_cp16(d, n > 0 ? (const void *)p : (const void *)src, n * (int)sizeof(T));
    } else {
#pragma unroll
      for (int w = 0; w < EPU; ++w)
        simt_cp<(int)sizeof(T)>(d + w * (int)sizeof(T),
                                w < n ? (const void *)(p + w) : (const void *)src,
                                w < n ? (int)sizeof(T) : 0);
    }
  }
}

// The tile of simt_tile with the operand layouts fixed: TA (A stored K x M)
// and TB (B stored N x K).
template <typename T, class Cfg, int KBLOCK, class BSrc, bool TA, bool TB>
__device__ __forceinline__ void simt_tile_impl(const GemmArgs<T> &g, long m0, long n0, long kb,
                                               long ke, T *out, long ldo, T alpha, T beta,
                                               T *smem, const BSrc &bsrc) {
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, EPU = Cfg::EPU;
  constexpr int TM = Cfg::TM, TN = Cfg::TN, NTH = Cfg::NTH, STAGES = Cfg::STAGES;
  constexpr int RGM = Cfg::RGM, RGN = Cfg::RGN, NRGM = Cfg::NRGM, NRGN = Cfg::NRGN;
  const int tid = threadIdx.x;
  const int tx = tid % Cfg::TX, ty = tid / Cfg::TX;
  const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(smem);
  const long M = g.M, N = g.N;

  // 16-byte copies need every staged row to start on a 16-byte boundary
  const T *A = g.A;
  const bool vec_a = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (g.lda % EPU == 0);
  const bool vec_b = BSrc::kDense && ((reinterpret_cast<uintptr_t>(g.B) & 15) == 0) &&
                     (g.ldb % EPU == 0);

  auto issue = [&](int st, long k0) {
    const uint32_t sa = s_base + (uint32_t)(st * Cfg::STAGE_ELEMS * (int)sizeof(T));
    const uint32_t sb = sa + (uint32_t)(Cfg::A_ELEMS * (int)sizeof(T));
    if (!TA)  // A[m][k]: BM rows of BK
      stage_rows<T, BM, BK, NTH, true, RGM>(sa, A + m0 * g.lda + k0, g.lda, M - m0, ke - k0,
                                             vec_a, tid);
    else      // A stored K x M: BK rows of BM
      stage_rows<T, BK, BM, NTH, false, 1>(sa, A + k0 * g.lda + m0, g.lda, ke - k0, M - m0,
                                           vec_a, tid);
    if constexpr (BSrc::kDense) {
      if (TB)  // B[n][k]: BN rows of BK
        stage_rows<T, BN, BK, NTH, true, RGN>(sb, g.B + n0 * g.ldb + k0, g.ldb, N - n0, ke - k0,
                                               vec_b, tid);
      else     // B[k][n]: BK rows of BN
        stage_rows<T, BK, BN, NTH, false, 1>(sb, g.B + k0 * g.ldb + n0, g.ldb, ke - k0, N - n0,
                                             vec_b, tid);
    } else {
      // gathered B (NoTrans layout [k][n]): one element per copy
#pragma unroll
      for (int e0 = 0; e0 < BK * BN; e0 += NTH) {
        const int e = e0 + tid;
        if ((BK * BN) % NTH != 0 && e >= BK * BN) break;
        const int k = e / BN, n = e - k * BN;
        const T *p = (k0 + k < ke && n0 + n < N) ? bsrc.ptr(g, k0 + k, n0 + n) : nullptr;
        simt_cp<(int)sizeof(T)>(sb + (uint32_t)(e * (int)sizeof(T)),
                                p ? (const void *)p : (const void *)A, p ? (int)sizeof(T) : 0);
      }
    }
  };

  T acc[TM][TN];
  T blk[KBLOCK > 0 ? TM : 1][KBLOCK > 0 ? TN : 1];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
  if (KBLOCK > 0) {
#pragma unroll
    for (int i = 0; i < (KBLOCK > 0 ? TM : 1); ++i)
#pragma unroll
      for (int j = 0; j < (KBLOCK > 0 ? TN : 1); ++j) blk[i][j] = T(0);
  }

  // rows of A / columns of B this thread multiplies (tile coordinates)
  int rows[TM], cols[TN];
#pragma unroll
  for (int i = 0; i < TM; ++i) rows[i] = (i / RGM) * (BM / NRGM) + ty * RGM + (i % RGM);
#pragma unroll
  for (int j = 0; j < TN; ++j) cols[j] = (j / RGN) * (BN / NRGN) + tx * RGN + (j % RGN);

  const int nslab = (int)((ke - kb + BK - 1) / BK);
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nslab) issue(s, kb + (long)s * BK);
    simt_commit();  // empty groups keep the group count uniform
  }

  for (int s = 0; s < nslab; ++s) {
    simt_wait<STAGES - 2>();  // this thread's copies of slab s have landed
    __syncthreads();          // ... and everyone's; slab s - 1 is consumed
    {
      const int sn = s + STAGES - 1;
      if (sn < nslab) issue(sn % STAGES, kb + (long)sn * BK);
      simt_commit();
    }
    const T *as = smem + (s % STAGES) * Cfg::STAGE_ELEMS;
    const T *bs = as + Cfg::A_ELEMS;
#pragma unroll 2
    for (int kq = 0; kq < BK / EPU; ++kq) {
      // EPU consecutive k: a[i][t] = op(A)[row_i][k + t], b[t][j] = op(B)[k + t][col_j]
      T a[TM][EPU], b[EPU][TN];
      if (!TA) {
#pragma unroll
        for (int i = 0; i < TM; ++i)
          lds_vec<T, EPU>(as + rows[i] * BK + (kq ^ ((rows[i] / RGM) & 7)) * EPU, a[i]);
      } else {
#pragma unroll
        for (int t = 0; t < EPU; ++t)
#pragma unroll
          for (int gi = 0; gi < NRGM; ++gi) {
            T v[RGM];
            lds_vec<T, RGM>(as + (kq * EPU + t) * BM + gi * (BM / NRGM) + ty * RGM, v);
#pragma unroll
            for (int r = 0; r < RGM; ++r) a[gi * RGM + r][t] = v[r];
          }
      }
      if (TB) {
        T v[TN][EPU];
#pragma unroll
        for (int j = 0; j < TN; ++j)
          lds_vec<T, EPU>(bs + cols[j] * BK + (kq ^ ((cols[j] / RGN) & 7)) * EPU, v[j]);
#pragma unroll
        for (int t = 0; t < EPU; ++t)
#pragma unroll
          for (int j = 0; j < TN; ++j) b[t][j] = v[j][t];
      } else {
#pragma unroll
        for (int t = 0; t < EPU; ++t)
#pragma unroll
          for (int gj = 0; gj < NRGN; ++gj)
            lds_vec<T, RGN>(bs + (kq * EPU + t) * BN + gj * (BN / NRGN) + tx * RGN,
                            b[t] + gj * RGN);
      }
      // one FMA chain per element, k increasing
#pragma unroll
      for (int t = 0; t < EPU; ++t) {
        if constexpr (KBLOCK > 0) {
#pragma unroll
          for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) blk[i][j] = fma_t(a[i][t], b[t][j], blk[i][j]);
        } else {
#pragma unroll
          for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) acc[i][j] = fma_t(a[i][t], b[t][j], acc[i][j]);
        }
      }
    }
    if constexpr (KBLOCK > 0) {
      // fold at every KBLOCK boundary (measured from kb) and at the end
      const long kdone = (long)(s + 1) * BK;
      if (kdone % (KBLOCK > 0 ? KBLOCK : 1) == 0 || s + 1 == nslab) {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) {
            acc[i][j] = acc[i][j] + blk[i][j];
            blk[i][j] = T(0);
          }
      }
    }
  }
  simt_wait<0>();
  __syncthreads();  // the ring is free for the caller's next tile

  // epilogue
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const long gm = m0 + rows[i];
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const long gn = n0 + cols[j];
      if (gn >= N) continue;
      T *dst = out + gm * ldo + gn;
      T v = alpha * acc[i][j];
      if (beta != T(0)) v = fma_t(beta, *dst, v);
      *dst = v;
    }
  }
}

// Computes the tile at (m0, n0) over k in [kb, ke) and writes
//   out[r*ldo + c] = alpha * acc + beta * out[r*ldo + c]   (beta != 0)
//   out[r*ldo + c] = alpha * acc                           (beta == 0)
// for the in-range part.  TA / TB: A stored K x M / B stored N x K (they must
// match g.transa / g.transb; a gathered B is read NoTrans).  `smem` holds
// Cfg::SMEM_ELEMS elements (16-byte aligned).
template <typename T, class Cfg, int KBLOCK, bool TA, bool TB, class BSrc = DenseB>
__device__ __forceinline__ void simt_tile(const GemmArgs<T> &g, long m0, long n0, long kb,
                                          long ke, T *out, long ldo, T alpha, T beta, T *smem,
                                          const BSrc &bsrc = BSrc()) {
  static_assert(BSrc::kDense || !TB, "a gathered B is read in the NoTrans layout");
  simt_tile_impl<T, Cfg, KBLOCK, BSrc, TA, TB>(g, m0, n0, kb, ke, out, ldo, alpha, beta, smem,
                                               bsrc);
}

}  // namespace ls
