// ls_simt.cuh -- plain FP32 / FP64 GEMM tiles on the CUDA cores.
//
// One CTA computes a BM x BN tile of C = alpha * op(A) op(B) + beta * C over
// a K range.  The reference's "packing inside the micro-kernel" (the first
// PACK_KERNEL pass writes the packed B panel while computing,
// NN_LIB/test_temp.c:9-536, test_SMM_NT.c:9-270) becomes the staging step of
// the tile itself: each K-slab of A and op(B) is read from row-major global
// memory straight into shared memory in the k-major layout the inner loop
// consumes (A transposed to As[k][m], op(B) to Bs[k][n]), double buffered so
// the next slab's global loads overlap the current slab's FMAs.  There is no
// separate packing pass and no packed copy in global memory.  Tails in m, n
// and k are predicated in the loads (zero fill) and stores, replacing the
// reference's 4/3/2/1x16, N8/N4/N2/N1 and EDGE_K kernel families.
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

template <typename T, int BM_, int BN_, int BK_, int TM_, int TN_>
struct SimtCfg {
  static constexpr int BM = BM_, BN = BN_, BK = BK_, TM = TM_, TN = TN_;
  static constexpr int TX = BN / TN, TY = BM / TM, NTH = TX * TY;
  // rows of a thread: NRGM groups of RGM consecutive rows, groups BM/NRGM apart
  static constexpr int RGM = TM >= 4 ? 4 : TM, NRGM = TM / RGM;
  static constexpr int RGN = TN >= 4 ? 4 : TN, NRGN = TN / RGN;
  static constexpr int PA = BM + 4, PB = BN + 4;  // padded pitches (elements)
  static constexpr int A_PER = BM * BK / NTH, B_PER = BK * BN / NTH;
  static constexpr int SMEM_ELEMS = 2 * BK * (PA + PB);
  static_assert(BM % TM == 0 && BN % TN == 0, "tile");
  static_assert((BM * BK) % NTH == 0 && (BK * BN) % NTH == 0, "loader");
  static_assert(TM % RGM == 0 && TN % RGN == 0, "groups");
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

// Where the tile reads op(B)[k][n] from: the dense row-major B of the
// GemmArgs (the GEMM calls), or a gather such as the implicit im2col columns
// of a convolution (ls_frontend.cu).  Only called for k < K and n < N.
struct DenseB {
  template <typename T>
  __device__ __forceinline__ T operator()(const GemmArgs<T> &g, long k, long n) const {
    return g.transb ? g.B[n * g.ldb + k] : g.B[k * g.ldb + n];
  }
};

// Computes the tile at (m0, n0) over k in [kb, ke) and writes
//   out[r*ldo + c] = alpha * acc + beta * out[r*ldo + c]   (beta != 0)
//   out[r*ldo + c] = alpha * acc                           (beta == 0)
// for the in-range part.  `smem` holds Cfg::SMEM_ELEMS elements.
template <typename T, class Cfg, int KBLOCK, class BSrc = DenseB>
__device__ __forceinline__ void simt_tile(const GemmArgs<T> &g, long m0,
                                          long n0, long kb, long ke, T *out,
                                          long ldo, T alpha, T beta, T *smem,
                                          const BSrc &bsrc = BSrc()) {
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK;
  constexpr int TM = Cfg::TM, TN = Cfg::TN, NTH = Cfg::NTH;
  constexpr int PA = Cfg::PA, PB = Cfg::PB;
  const int tid = threadIdx.x;
  const int tx = tid % Cfg::TX, ty = tid / Cfg::TX;

  T *As = smem;                 // [2][BK][PA]
  T *Bs = smem + 2 * BK * PA;   // [2][BK][PB]

  T ra[Cfg::A_PER], rb[Cfg::B_PER];

  const T *A = g.A;
  const long M = g.M, N = g.N, lda = g.lda;
  const int ta = g.transa, tb = g.transb;

  auto load_slab = [&](long k0) {
#pragma unroll
    for (int i = 0; i < Cfg::A_PER; ++i) {
      int e = tid + i * NTH;
      int m, k;
      if (!ta) { k = e % BK; m = e / BK; } else { m = e % BM; k = e / BM; }
      long gm = m0 + m, gk = k0 + k;
      T v = T(0);
      if (gm < M && gk < ke) v = ta ? A[gk * lda + gm] : A[gm * lda + gk];
      ra[i] = v;
    }
#pragma unroll
    for (int i = 0; i < Cfg::B_PER; ++i) {
      int e = tid + i * NTH;
      int n, k;
      if (!tb) { n = e % BN; k = e / BN; } else { k = e % BK; n = e / BK; }
      long gn = n0 + n, gk = k0 + k;
      T v = T(0);
      if (gn < N && gk < ke) v = bsrc(g, gk, gn);
      rb[i] = v;
    }
  };
  auto store_slab = [&](int buf) {
    T *as = As + buf * BK * PA, *bs = Bs + buf * BK * PB;
#pragma unroll
    for (int i = 0; i < Cfg::A_PER; ++i) {
      int e = tid + i * NTH;
      int m, k;
      if (!ta) { k = e % BK; m = e / BK; } else { m = e % BM; k = e / BM; }
      as[k * PA + m] = ra[i];
    }
#pragma unroll
    for (int i = 0; i < Cfg::B_PER; ++i) {
      int e = tid + i * NTH;
      int n, k;
      if (!tb) { n = e % BN; k = e / BN; } else { k = e % BK; n = e / BK; }
      bs[k * PB + n] = rb[i];
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

  const int nslab = (int)((ke - kb + BK - 1) / BK);
  if (nslab > 0) {
    load_slab(kb);
    store_slab(0);
  }
  __syncthreads();

  for (int s = 0; s < nslab; ++s) {
    const int buf = s & 1;
    const bool more = s + 1 < nslab;
    if (more) load_slab(kb + (long)(s + 1) * BK);
    const T *as = As + buf * BK * PA, *bs = Bs + buf * BK * PB;
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T a[TM], b[TN];
#pragma unroll
      for (int gi = 0; gi < Cfg::NRGM; ++gi)
        lds_vec<T, Cfg::RGM>(as + kk * PA + gi * (BM / Cfg::NRGM) + ty * Cfg::RGM,
                             a + gi * Cfg::RGM);
#pragma unroll
      for (int gj = 0; gj < Cfg::NRGN; ++gj)
        lds_vec<T, Cfg::RGN>(bs + kk * PB + gj * (BN / Cfg::NRGN) + tx * Cfg::RGN,
                             b + gj * Cfg::RGN);
      if constexpr (KBLOCK > 0) {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) blk[i][j] = fma_t(a[i], b[j], blk[i][j]);
      } else {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) acc[i][j] = fma_t(a[i], b[j], acc[i][j]);
      }
    }
    if constexpr (KBLOCK > 0) {
      // fold at every KBLOCK boundary (measured from kb) and at the end
      const long kdone = (long)(s + 1) * BK;
      if (kdone % (KBLOCK > 0 ? KBLOCK : 1) == 0 || !more) {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) {
            acc[i][j] = acc[i][j] + blk[i][j];
            blk[i][j] = T(0);
          }
      }
    }
    if (more) store_slab(buf ^ 1);
    __syncthreads();
  }

  // epilogue
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int r = (i / Cfg::RGM) * (BM / Cfg::NRGM) + ty * Cfg::RGM + (i % Cfg::RGM);
    const long gm = m0 + r;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int c = (j / Cfg::RGN) * (BN / Cfg::NRGN) + tx * Cfg::RGN + (j % Cfg::RGN);
      const long gn = n0 + c;
      if (gn >= N) continue;
      T *dst = out + gm * ldo + gn;
      T v = alpha * acc[i][j];
      if (beta != T(0)) v = fma_t(beta, *dst, v);
      *dst = v;
    }
  }
}

}  // namespace ls
