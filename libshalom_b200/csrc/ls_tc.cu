// ls_tc.cu -- split-BF16 SGEMM on the sm_100a tensor cores (tcgen05 + TMEM).
//
// Each FP32 input x is split into BF16 parts, x = hi + mid + lo (three parts,
// 24 significant bits: LIBSHALOM_PREC_BF16X6) or x ~ hi + lo (two parts, 16
// bits: LIBSHALOM_PREC_BF16X3).  C = A B is then a sum of BF16 products on the
// tensor cores with FP32 accumulation in TMEM:
//   D_main = sum A_hi B_hi
//   D_corr = sum A_hi B_mid + A_mid B_hi + A_hi B_lo + A_lo B_hi + A_mid B_mid
//            (bf16x3: A_hi B_lo + A_lo B_hi)
// and C = alpha (D_main + D_corr) + beta C in the epilogue.  Keeping the
// correction terms in their own accumulator keeps their rounding 2^-8 below
// the main term's.
//
// The reference's "packing inside the micro-kernel" is the staging step here:
// every K-slab of A and op(B) goes from row-major global memory into a ring of
// FP32 shared-memory stages with cp.async (issued STAGES-1 slabs ahead, so
// HBM keeps a deep queue of requests while the CTA converts and multiplies),
// is split to BF16 by the CTA's threads and written in the K-major
// core-matrix layout tcgen05.mma reads.  There is no separate packing pass and
// no packed copy in global memory.  Two BF16 operand buffers alternate,
// released by tcgen05.commit on an mbarrier.
//
// Small GEMMs (M <= 64) are packed G to a tile: the A rows of G GEMMs fill
// the 128 rows of the MMA, their B columns sit side by side in its N, and
// only the diagonal blocks of the 128 x N product are written back.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include "ls_common.cuh"
#include "ls_tc_launch.h"
#include "ls_simt_launch.h"
#include "ls_tc_ptx.cuh"

namespace ls {

namespace {

constexpr int TC_THREADS = 512;
constexpr int TC_BM = 128;          // MMA M (TMEM lanes)
constexpr int TC_BK = 32;           // K per slab (two MMA K-steps of 16)
constexpr int TC_MAX_N = 128;       // MMA N per tile
constexpr int TC_TMEM_COLS = 256;   // D_main (0..127) + D_corr (128..255)
constexpr int STAGES = 3;           // FP32 staging ring depth

// BF16 operand buffers: [split][A | B][4 chunks of 8 k][128 rows][16 bytes]
constexpr int SPLIT_BYTES = 16384;
constexpr int BUF_BYTES = 3 * SPLIT_BYTES;
constexpr int CHUNK_BYTES = 128 * 16;

// FP32 staging stage: A as [128 rows][36 floats] (32 used, padded against
// bank conflicts); B as [128 rows][36] when B is N x K (Trans) or
// [32 k][132 floats] when B is K x N (NoTrans).
constexpr int SA_PITCH = 36;
constexpr int SBT_PITCH = 36;
constexpr int SBN_PITCH = 132;
constexpr int STAGE_A_BYTES = 128 * SA_PITCH * 4;  // 18432
constexpr int STAGE_B_BYTES = 128 * SBT_PITCH * 4; // 18432 (>= 32 * 132 * 4 = 16896)
constexpr int STAGE_BYTES = STAGE_A_BYTES + STAGE_B_BYTES;

constexpr int OFF_BUF = 0;
constexpr int OFF_STAGE = 2 * BUF_BYTES;                    // 98304
constexpr int OFF_BAR = OFF_STAGE + STAGES * STAGE_BYTES;   // 208896
constexpr int TC_SMEM = OFF_BAR + 64;                       // 208960

struct TcProblem {
  const float *A;
  const float *B;
  float *C;
  long sA, sB, sC;  // element strides between consecutive GEMMs of the batch
  int M, N, K;
  int lda, ldb, ldc;
  int transb;
  float alpha, beta;
  long count;      // GEMMs in the batch
  int G;           // GEMMs packed per tile (block diagonal); 1 = tiled GEMM
  int tile_n;      // MMA N of every tile (multiple of 16, <= 128)
  int tiles_m, tiles_n;  // tiles per GEMM when G == 1
  long num_tiles;
  int nk;          // K slabs
  int vec_a, vec_b;  // 16-byte cp.async allowed for A / B rows
  int vec_c;       // 16-byte stores allowed for C rows
  int kc_slabs;    // DRAIN kernels: slabs per TMEM accumulation chunk
  // split-K of one GEMM: "GEMM" g of the batch is K slice g of a single
  // product (A and B not offset; the slice's K range starts at g * kslice),
  // written to partial C_g = C + g * sC; 0 = no split
  int kslice;
  unsigned *err;   // device status word (bounded waits)
};

struct TileInfo {
  long g0;   // first GEMM of the tile
  int ng;    // GEMMs in the tile
  int m0, n0;
};

__device__ __forceinline__ TileInfo decode_tile(const TcProblem &p, long t) {
  TileInfo ti;
  if (p.G > 1) {
    ti.g0 = t * p.G;
    ti.ng = (int)min((long)p.G, p.count - ti.g0);
    ti.m0 = 0;
    ti.n0 = 0;
  } else {
    const long per = (long)p.tiles_m * p.tiles_n;
    ti.g0 = t / per;
    const int r = (int)(t % per);
    ti.ng = 1;
    ti.m0 = (r / p.tiles_n) * TC_BM;
    ti.n0 = (r % p.tiles_n) * p.tile_n;
  }
  return ti;
}

// split 8 floats into hi / mid / lo BF16 (packed pairs, element 0 in the low half)
template <int NSPLIT>
__device__ __forceinline__ void split8(const float *x, uint4 &h, uint4 &m, uint4 &l) {
  uint32_t hh[4], mm[4], ll[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float x0 = x[2 * i], x1 = x[2 * i + 1];
    __nv_bfloat162 b = __floats2bfloat162_rn(x0, x1);
    const float r0 = x0 - __low2float(b), r1 = x1 - __high2float(b);
    __nv_bfloat162 c = __floats2bfloat162_rn(r0, r1);
    hh[i] = *reinterpret_cast<uint32_t *>(&b);
    mm[i] = *reinterpret_cast<uint32_t *>(&c);
    if (NSPLIT == 3) {
      const float s0 = r0 - __low2float(c), s1 = r1 - __high2float(c);
      __nv_bfloat162 d = __floats2bfloat162_rn(s0, s1);
      ll[i] = *reinterpret_cast<uint32_t *>(&d);
    } else {
      ll[i] = 0;
    }
  }
  h = make_uint4(hh[0], hh[1], hh[2], hh[3]);
  m = make_uint4(mm[0], mm[1], mm[2], mm[3]);
  l = make_uint4(ll[0], ll[1], ll[2], ll[3]);
}

// ---- cp.async (global -> shared), zero fill past src_bytes ----
__device__ __forceinline__ void cp_async16(uint32_t saddr, const void *g, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(g),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t saddr, const void *g, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(saddr), "l"(g),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// DRAIN: every p.kc_slabs K slabs the TMEM accumulators are added (round to
// nearest) into FP32 registers and restarted.  The tensor core's FP32
// accumulation truncates, so its error grows with the number of K steps it
// accumulates; draining bounds that to kc_slabs * 2 steps (used for long-K
// GEMMs).
template <int NSPLIT, bool DRAIN>
__global__ void __launch_bounds__(TC_THREADS, 1) k_tc_sgemm(TcProblem p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + OFF_BAR);  // [2]
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + OFF_BAR + 16);
  volatile int *s_abort = reinterpret_cast<volatile int *>(smem + OFF_BAR + 20);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t smem_base = ptx::smem_u32(smem);

  if (tid == 0) {
    ptx::mbar_init(&bars[0], 1);
    ptx::mbar_init(&bars[1], 1);
    *s_abort = 0;
    ptx::fence_mbar_init();
  }
  if (warp == 0) {
    ptx::tmem_alloc(tmem_slot, TC_TMEM_COLS);
    ptx::tmem_relinquish();
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = ptx::idesc_bf16_f32(TC_BM, p.tile_n);
  const int tn = p.tile_n;

  // ---- per-thread assignments, constant over the kernel ----
  // cp.async chunks (16-byte path): A and B (Trans) rows r0 and r0 + 64,
  // 4-float chunk c4; B (NoTrans): k-row and column of chunks tid and tid + 512
  const int r0 = tid >> 3, c4 = (tid & 7) * 4;
  const int cpr = tn >> 2;  // 4-float chunks per k-row of a B (NoTrans) slab
  int bn_kr[2], bn_j[2];
  bool bn_on[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int e = tid + q * TC_THREADS;
    bn_on[q] = e < 32 * cpr;
    bn_kr[q] = bn_on[q] ? e / cpr : 0;
    bn_j[q] = bn_on[q] ? (e - bn_kr[q] * cpr) * 4 : 0;
  }
  // conversion items: A row cr, K chunk cc; B row/column bj, K chunk bc
  const int cr = tid & 127, cc = tid >> 7;
  const bool b_item = tid < 4 * tn;
  const int bj = b_item ? tid % tn : 0, bc = b_item ? tid / tn : 0;

  // producer state for its current tile: source rows of A and B
  const float *a_src[2] = {nullptr, nullptr};
  const float *b_src[2] = {nullptr, nullptr};
  int b_cnt[2] = {0, 0};  // valid floats in a B (NoTrans) chunk
  auto producer_tile = [&](long t) {
    const TileInfo ti = decode_tile(p, t);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int r = r0 + 64 * q;
      int gi, i;
      bool ok;
      if (p.G > 1) { gi = r / p.M; i = r - gi * p.M; ok = gi < ti.ng; }
      else { gi = 0; i = ti.m0 + r; ok = i < p.M; }
      a_src[q] = ok ? p.A + (ti.g0 + gi) * p.sA + (long)i * p.lda : nullptr;
      if (p.transb) {
        int gj, jj;
        if (p.G > 1) { gj = r / p.N; jj = r - gj * p.N; ok = r < tn && gj < ti.ng; }
        else { gj = 0; jj = ti.n0 + r; ok = r < tn && jj < p.N; }
        b_src[q] = ok ? p.B + (ti.g0 + gj) * p.sB + (long)jj * p.ldb : nullptr;
      } else {
        const int j = bn_j[q];
        int gj, jj;
        if (p.G > 1) { gj = j / p.N; jj = j - gj * p.N; ok = bn_on[q] && gj < ti.ng; }
        else { gj = 0; jj = ti.n0 + j; ok = bn_on[q] && jj < p.N; }
        b_src[q] = ok ? p.B + (ti.g0 + gj) * p.sB + jj : nullptr;
        b_cnt[q] = ok ? min(4, p.N - jj) : 0;
      }
    }
  };

  // ---- producer: cp.async of slab s of the producer's tile into stage st ----
  auto issue_slab = [&](long t, int s, int st) {
    // split-K: "GEMM" g0 of the batch is K slice g0 of one product
    const int k0 = s * TC_BK + (p.kslice ? (int)decode_tile(p, t).g0 * p.kslice : 0);
    const uint32_t sa = smem_base + OFF_STAGE + st * STAGE_BYTES;
    const uint32_t sb = sa + STAGE_A_BYTES;
    if (p.vec_a) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const bool ok = a_src[q] != nullptr && k0 + c4 < p.K;
        cp_async16(sa + ((r0 + 64 * q) * SA_PITCH + c4) * 4, ok ? a_src[q] + k0 + c4 : p.A,
                   ok ? 4 * min(4, p.K - k0 - c4) : 0);
      }
    } else {
      const TileInfo ti = decode_tile(p, t);
      for (int e = tid; e < 128 * 32; e += TC_THREADS) {
        const int r = e >> 5, k = e & 31;
        int gi, i;
        if (p.G > 1) { gi = r / p.M; i = r - gi * p.M; } else { gi = 0; i = ti.m0 + r; }
        const bool ok = ((p.G > 1) ? (gi < ti.ng) : (i < p.M)) && k0 + k < p.K;
        const float *src = ok ? p.A + (ti.g0 + gi) * p.sA + (long)i * p.lda + k0 + k : p.A;
        cp_async4(sa + (r * SA_PITCH + k) * 4, src, ok ? 4 : 0);
      }
    }
    if (p.vec_b) {
      if (p.transb) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          if (r0 + 64 * q < tn) {
            const bool ok = b_src[q] != nullptr && k0 + c4 < p.K;
            cp_async16(sb + ((r0 + 64 * q) * SBT_PITCH + c4) * 4,
                       ok ? b_src[q] + k0 + c4 : p.B, ok ? 4 * min(4, p.K - k0 - c4) : 0);
          }
        }
      } else {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          if (bn_on[q]) {
            const int kk = k0 + bn_kr[q];
            const bool ok = b_src[q] != nullptr && kk < p.K;
            cp_async16(sb + (bn_kr[q] * SBN_PITCH + bn_j[q]) * 4,
                       ok ? b_src[q] + (long)kk * p.ldb : p.B, ok ? 4 * b_cnt[q] : 0);
          }
        }
      }
    } else {
      const TileInfo ti = decode_tile(p, t);
      if (p.transb) {
        for (int e = tid; e < tn * 32; e += TC_THREADS) {
          const int j = e >> 5, k = e & 31;
          int gj, jj;
          if (p.G > 1) { gj = j / p.N; jj = j - gj * p.N; } else { gj = 0; jj = ti.n0 + j; }
          const bool ok = ((p.G > 1) ? (gj < ti.ng) : (jj < p.N)) && k0 + k < p.K;
          const float *src = ok ? p.B + (ti.g0 + gj) * p.sB + (long)jj * p.ldb + k0 + k : p.B;
          cp_async4(sb + (j * SBT_PITCH + k) * 4, src, ok ? 4 : 0);
        }
      } else {
        for (int e = tid; e < 32 * tn; e += TC_THREADS) {
          const int kr = e / tn, j = e - kr * tn;
          int gj, jj;
          if (p.G > 1) { gj = j / p.N; jj = j - gj * p.N; } else { gj = 0; jj = ti.n0 + j; }
          const bool ok = ((p.G > 1) ? (gj < ti.ng) : (jj < p.N)) && k0 + kr < p.K;
          const float *src = ok ? p.B + (ti.g0 + gj) * p.sB + (long)(k0 + kr) * p.ldb + jj : p.B;
          cp_async4(sb + (kr * SBN_PITCH + j) * 4, src, ok ? 4 : 0);
        }
      }
    }
  };

  // ---- converter: staging stage st -> split BF16 operands in buffer buf ----
  // consecutive threads take consecutive rows: the 16-byte shared stores of a
  // quarter warp cover 128 contiguous bytes (no bank conflicts)
  auto convert_slab = [&](int st, int buf) {
    const float *fa = reinterpret_cast<const float *>(smem + OFF_STAGE + st * STAGE_BYTES);
    const float *fb = fa + STAGE_A_BYTES / 4;
    unsigned char *base = smem + OFF_BUF + buf * BUF_BYTES;
    {
      float x[8];
      const float4 u = *reinterpret_cast<const float4 *>(fa + cr * SA_PITCH + 8 * cc);
      const float4 v = *reinterpret_cast<const float4 *>(fa + cr * SA_PITCH + 8 * cc + 4);
      x[0] = u.x; x[1] = u.y; x[2] = u.z; x[3] = u.w;
      x[4] = v.x; x[5] = v.y; x[6] = v.z; x[7] = v.w;
      uint4 h, m, l;
      split8<NSPLIT>(x, h, m, l);
      const int off = cc * CHUNK_BYTES + cr * 16;
      *reinterpret_cast<uint4 *>(base + off) = h;
      *reinterpret_cast<uint4 *>(base + SPLIT_BYTES + off) = m;
      if (NSPLIT == 3) *reinterpret_cast<uint4 *>(base + 2 * SPLIT_BYTES + off) = l;
    }
    if (b_item) {
      float x[8];
      if (p.transb) {
        const float4 u = *reinterpret_cast<const float4 *>(fb + bj * SBT_PITCH + 8 * bc);
        const float4 v = *reinterpret_cast<const float4 *>(fb + bj * SBT_PITCH + 8 * bc + 4);
        x[0] = u.x; x[1] = u.y; x[2] = u.z; x[3] = u.w;
        x[4] = v.x; x[5] = v.y; x[6] = v.z; x[7] = v.w;
      } else {
#pragma unroll
        for (int t = 0; t < 8; ++t) x[t] = fb[(8 * bc + t) * SBN_PITCH + bj];
      }
      uint4 h, m, l;
      split8<NSPLIT>(x, h, m, l);
      const int off = 8192 + bc * CHUNK_BYTES + bj * 16;
      *reinterpret_cast<uint4 *>(base + off) = h;
      *reinterpret_cast<uint4 *>(base + SPLIT_BYTES + off) = m;
      if (NSPLIT == 3) *reinterpret_cast<uint4 *>(base + 2 * SPLIT_BYTES + off) = l;
    }
  };

  // epilogue geometry: warp quarter wq owns TMEM lanes 32*wq..; the four
  // warpgroups wg own consecutive ranges of the 8-column chunks
  const int wq = warp & 3, wg = warp >> 2;
  const int nch = tn / 8;
  const int per = (nch + 3) / 4;
  const int c_begin = min(nch, wg * per), c_end = min(nch, c_begin + per);
  constexpr int RMAX = DRAIN ? 32 : 1;  // register sum (DRAIN): 4 chunks x 8 columns
  float R[RMAX];
#pragma unroll
  for (int u = 0; u < RMAX; ++u) R[u] = 0.0f;
  auto fold_chunks = [&]() {
    if constexpr (DRAIN) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int ch = c_begin + q;
        if (ch < c_end) {
          float dm[8], dc[8];
          const uint32_t ta = tmem + ((uint32_t)(wq * 32) << 16) + ch * 8;
          ptx::tmem_ld8(ta, dm);
          ptx::tmem_ld8(ta + 128, dc);
          ptx::tmem_wait_ld();
#pragma unroll
          for (int u = 0; u < 8; ++u) R[q * 8 + u] += dm[u] + dc[u];
        }
      }
    }
  };

  // producer cursor (tile tp, slab spp), STAGES-1 slabs ahead of the consumer
  long tp = blockIdx.x;
  int spp = 0;
  if (tp < p.num_tiles) producer_tile(tp);
  auto produce_next = [&](int st) {
    if (tp < p.num_tiles) issue_slab(tp, spp, st);
    cp_async_commit();  // empty groups keep the group count uniform
    if (++spp == p.nk) {
      spp = 0;
      tp += gridDim.x;
      if (tp < p.num_tiles) producer_tile(tp);
    }
  };
#pragma unroll
  for (int i = 0; i < STAGES - 1; ++i) produce_next(i);

  long sc = 0;  // slabs consumed by this CTA (selects stage, buffer and mbarrier phase)
  for (long t = blockIdx.x; t < p.num_tiles; t += gridDim.x) {
    const TileInfo ti = decode_tile(p, t);
    for (int s = 0; s < p.nk; ++s, ++sc) {
      const int buf = (int)(sc & 1);
      const int st = (int)(sc % STAGES);
      cp_async_wait<STAGES - 2>();  // this thread's copies of slab sc have landed
      __syncthreads();              // ... and everyone else's
      bool ok = true;
      if (sc >= 2) ok = ptx::mbar_wait_bounded(&bars[buf], (uint32_t)(((sc >> 1) - 1) & 1));
      if (!ok) {
        *s_abort = 1;
        atomicOr(p.err, 1u);
      } else {
        convert_slab(st, buf);
      }
      // refill the stage consumed one slab ago (every thread is past its conversion)
      produce_next((int)((sc + STAGES - 1) % STAGES));
      ptx::fence_proxy_async_smem();
      __syncthreads();
      if (*s_abort) goto done;
      if (tid == 0) {
        ptx::tc_fence_after();
        const uint32_t bb = smem_base + OFF_BUF + buf * BUF_BYTES;
        const int s_in = DRAIN ? s % p.kc_slabs : s;  // slab within the accumulation chunk
        const int ksteps = min(2, (p.K - s * TC_BK + 15) / 16);
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          if (ks >= ksteps) break;
          const uint32_t acc = (s_in > 0 || ks > 0) ? 1u : 0u;
          uint64_t a[3], b[3];
#pragma unroll
          for (int sp = 0; sp < NSPLIT; ++sp) {
            a[sp] = ptx::smem_desc(bb + sp * SPLIT_BYTES + ks * 2 * CHUNK_BYTES, CHUNK_BYTES, 128);
            b[sp] = ptx::smem_desc(bb + sp * SPLIT_BYTES + 8192 + ks * 2 * CHUNK_BYTES,
                                   CHUNK_BYTES, 128);
          }
          const uint32_t dm = tmem, dc = tmem + 128;
          ptx::mma_bf16(dm, a[0], b[0], idesc, acc);
          ptx::mma_bf16(dc, a[0], b[1], idesc, acc);
          ptx::mma_bf16(dc, a[1], b[0], idesc, 1u);
          if (NSPLIT == 3) {
            ptx::mma_bf16(dc, a[0], b[2], idesc, 1u);
            ptx::mma_bf16(dc, a[2], b[0], idesc, 1u);
            ptx::mma_bf16(dc, a[1], b[1], idesc, 1u);
          }
        }
        ptx::mma_commit(&bars[buf]);
      }
      if (DRAIN && (s + 1) % p.kc_slabs == 0 && s + 1 < p.nk) {
        // chunk boundary: fold the accumulators into the register sum
        const bool ok2 = ptx::mbar_wait_bounded(&bars[buf], (uint32_t)((sc >> 1) & 1));
        if (!ok2) {
          *s_abort = 1;
          atomicOr(p.err, 1u);
        }
        ptx::tc_fence_after();
        fold_chunks();
        ptx::tc_fence_before();
        __syncthreads();
        if (*s_abort) goto done;
      }
    }

    // ---- epilogue: TMEM -> registers -> C ----
    {
      const long last = sc - 1;
      const bool ok = ptx::mbar_wait_bounded(&bars[last & 1], (uint32_t)((last >> 1) & 1));
      if (!ok) {
        *s_abort = 1;
        atomicOr(p.err, 1u);
      }
      ptx::tc_fence_after();
      const int r = wq * 32 + lane;
      int gi, i, jlo, jhi;  // this row's GEMM, its row, and its valid tile columns
      bool rok;
      if (p.G > 1) {
        gi = r / p.M; i = r - gi * p.M; rok = gi < ti.ng;
        jlo = gi * p.N; jhi = jlo + p.N;
      } else {
        gi = 0; i = ti.m0 + r; rok = i < p.M;
        jlo = 0; jhi = min(tn, p.N - ti.n0);
      }
      rok = rok && ok;
      float *crow = p.C + (ti.g0 + gi) * p.sC + (long)i * p.ldc + (ti.n0 - jlo);
      // crow[j] is the C element of tile column j (j in [jlo, jhi))
      const bool vec = p.vec_c && ((p.G == 1) || (p.N % 4 == 0));
      auto store8 = [&](int ch, const float *v) {
        const int j0 = ch * 8;
        if (!rok || j0 + 8 <= jlo || j0 >= jhi) return;
        if (vec && j0 >= jlo && j0 + 8 <= jhi) {
          float4 o0, o1;
          if (p.beta != 0.0f) {
            const float4 c0 = *reinterpret_cast<const float4 *>(crow + j0);
            const float4 c1 = *reinterpret_cast<const float4 *>(crow + j0 + 4);
            o0 = make_float4(__fmaf_rn(p.beta, c0.x, p.alpha * v[0]),
                             __fmaf_rn(p.beta, c0.y, p.alpha * v[1]),
                             __fmaf_rn(p.beta, c0.z, p.alpha * v[2]),
                             __fmaf_rn(p.beta, c0.w, p.alpha * v[3]));
            o1 = make_float4(__fmaf_rn(p.beta, c1.x, p.alpha * v[4]),
                             __fmaf_rn(p.beta, c1.y, p.alpha * v[5]),
                             __fmaf_rn(p.beta, c1.z, p.alpha * v[6]),
                             __fmaf_rn(p.beta, c1.w, p.alpha * v[7]));
          } else {
            o0 = make_float4(p.alpha * v[0], p.alpha * v[1], p.alpha * v[2], p.alpha * v[3]);
            o1 = make_float4(p.alpha * v[4], p.alpha * v[5], p.alpha * v[6], p.alpha * v[7]);
          }
          *reinterpret_cast<float4 *>(crow + j0) = o0;
          *reinterpret_cast<float4 *>(crow + j0 + 4) = o1;
        } else {
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int j = j0 + u;
            if (j >= jlo && j < jhi) {
              float x = p.alpha * v[u];
              if (p.beta != 0.0f) x = __fmaf_rn(p.beta, crow[j], x);
              crow[j] = x;
            }
          }
        }
      };
      if constexpr (DRAIN) {
        fold_chunks();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int ch = c_begin + q;
          if (ch < c_end) store8(ch, R + q * 8);
        }
#pragma unroll
        for (int u = 0; u < RMAX; ++u) R[u] = 0.0f;
      } else {
        for (int ch = c_begin; ch < c_end; ++ch) {
          float dm[8], dc[8];
          const uint32_t ta = tmem + ((uint32_t)(wq * 32) << 16) + ch * 8;
          ptx::tmem_ld8(ta, dm);
          ptx::tmem_ld8(ta + 128, dc);
          ptx::tmem_wait_ld();
#pragma unroll
          for (int u = 0; u < 8; ++u) dm[u] += dc[u];
          store8(ch, dm);
        }
      }
      ptx::tc_fence_before();
      __syncthreads();
      if (*s_abort) goto done;
    }
  }

done:
  cp_async_wait<0>();  // no copy may still target shared memory when the CTA exits
  __syncthreads();
  if (*s_abort && sc > 0) {
    // give MMAs still in flight a bounded chance to finish before freeing TMEM
    ptx::mbar_wait_bounded(&bars[(sc - 1) & 1], (uint32_t)(((sc - 1) >> 1) & 1));
  }
  if (warp == 0) {
    ptx::tc_fence_after();
    ptx::tmem_dealloc(tmem, TC_TMEM_COLS);
  }
}

// ===========================================================================
// Warp-specialized TMA variant (operands that TMA can address: 16-byte
// aligned bases and row strides).  Roles, all connected by mbarriers:
//   warp 0      producer: one thread issues cp.async.bulk.tensor loads of the
//               A and op(B) slabs into a 3-deep FP32 ring (A and B (Trans)
//               boxes land 128-byte swizzled)
//   warp 1      MMA: one thread issues tcgen05.mma into one of two TMEM
//               accumulator sets (512 columns), so the epilogue of one tile or
//               accumulation chunk overlaps the MMAs of the next
//   converters  FP32 slab -> split BF16 core matrices (2 buffers): 8 or 16
//               warps (WsRoles below)
//   epilogue    TMEM -> registers -> C (and the register fold of the long-K
//               chunks): 8 or 4 warps.  With beta = 0 and a TMA-addressable C
//               (one GEMM per tile) each warp stages 32 rows x 32 columns of C
//               in a 4 KB shared buffer (128-byte swizzle) and writes them
//               with one cp.async.bulk.tensor store: full-line writes instead
//               of one 16-byte piece per row and thread, which would occupy
//               the L1 data path the MMAs and converters share.
// The shared-memory data path bounds the kernel: one MMA of 128 x 128 x 16
// reads 8 KB of operands in its 64 cycles, the SM's whole 128 B/clk.
// ===========================================================================
constexpr int WS_STAGES = 3;
constexpr int WS_STAGE_BYTES = 32768;                           // A 16 KB + B 16 KB
constexpr int WS_OFF_BUF = 0;                                   // 2 BF16 operand buffers
constexpr int WS_OFF_STAGE = 2 * BUF_BYTES;                     // 98304 (1024-aligned)
constexpr int WS_CST_WARP = 4096;                               // C staging per epilogue warp
constexpr int WS_OFF_CST = WS_OFF_STAGE + WS_STAGES * WS_STAGE_BYTES;  // 196608
constexpr int WS_OFF_BAR = WS_OFF_CST + 8 * WS_CST_WARP;        // 229376
constexpr int WS_SMEM = WS_OFF_BAR + 256;
static_assert(WS_SMEM <= 232448, "TMA kernel exceeds 227 KB of shared memory");
constexpr int W_CONV0 = 2, N_CONV = 8;

// Warp roles of k_tc_ws: warp 0 producer, warp 1 MMA, then NC converter and
// NE epilogue warps.  WIDE (short K, C written by TMA stores): 16 converters
// and 4 epilogue warps (one per TMEM lane quarter), since the split is the
// busiest role there.  Otherwise 8 + 8: long-K tiles hold the register fold of
// 64 columns per epilogue thread, and packed small GEMMs store C row by row.
template <bool WIDE>
struct WsRoles {
  static constexpr int NC = WIDE ? 16 : 8;
  static constexpr int NE = WIDE ? 4 : 8;
  static constexpr int W_EPI = 2 + NC;
  static constexpr int THREADS = (2 + NC + NE) * 32;
  static constexpr int BLOCKS = 16 / NE;  // 32-column blocks of C per epilogue warp
};
constexpr int WS_TMEM_COLS = 512;  // 2 x (D_main 128 + D_corr 128)

// mbarrier slots (8 bytes each) after WS_OFF_BAR
enum { B_FULL = 0, B_EMPTY = 4, B_BFULL = 8, B_BEMPTY = 10, B_AFULL = 12, B_AEMPTY = 14,
       B_FINAL = 16, B_COUNT = 17 };

struct WsArgs {
  TcProblem p;
  uint32_t tx_bytes;  // A box + B box bytes per slab
  int nn_w;           // B (NoTrans) box width in floats (row pitch of the staged slab)
  int c_tma;          // C written by TMA stores (boxes of 32 columns x 32 rows)
};

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(ptx::smem_u32(bar)) : "memory");
}
// Arrival that publishes no memory.  The default arrive has release
// semantics: it orders this thread's earlier memory operations, the
// epilogue's global C stores included, before the arrival.  Arrivals that
// only say "done reading" (TMEM read back and waited for, a queue slot
// copied into registers) have nothing to publish.
__device__ __forceinline__ void mbar_arrive_relaxed(uint64_t *bar) {
  asm volatile("mbarrier.arrive.relaxed.cta.shared::cta.b64 _, [%0];" ::"r"(ptx::smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes),
               "r"(ptx::smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint64_t *bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(ptx::smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// Slow path of ws_wait: the thread suspends in the barrier wait (up to about
// a microsecond per try, woken when the phase completes) instead of polling,
// so waiting roles take no issue slots or shared-memory bandwidth from the
// working ones.  Gives up after `limit` tries or two seconds, whichever
// comes first, or as soon as another role has aborted.  Inlined: a call
// would make the caller save its live registers to local memory around every
// wait.
__device__ __forceinline__ bool ws_wait_slow(uint64_t *bar, uint32_t parity,
                                             volatile int *abort_flag, unsigned *err,
                                             uint32_t limit) {
  const uint64_t t0 = ptx::globaltimer_ns();
  for (uint32_t it = 0; it < limit; ++it) {
    if (ptx::mbar_try_wait_suspend(bar, parity, 1000)) return true;
    if ((it & 15) == 15) {
      if (*abort_flag) return false;
      if (ptx::globaltimer_ns() - t0 > 2000000000ull) break;
    }
  }
  *abort_flag = 1;
  atomicOr(err, 1u);
  return false;
}

// Bounded wait: one test inline, the rest in ws_wait_slow.
__device__ __forceinline__ bool ws_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag,
                                        unsigned *err, uint32_t limit = 1u << 22) {
  if (ptx::mbar_try_wait(bar, parity)) return true;
  return ws_wait_slow(bar, parity, abort_flag, err, limit);
}

// BLX > 0: each epilogue warp holds at most BLX 32-column blocks of C (a
// DRAIN kernel for tiles of at most 32 * BLX * (epilogue warps / 4) columns
// keeps a smaller register fold)
template <int NSPLIT, bool DRAIN, bool WIDE, int BLX = 0>
__global__ void __launch_bounds__(WsRoles<WIDE>::THREADS, 1)
    k_tc_ws(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
            const __grid_constant__ CUtensorMap tmC, const WsArgs args) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const TcProblem &p = args.p;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + WS_OFF_BAR);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + WS_OFF_BAR + 8 * B_COUNT);
  volatile int *s_abort = reinterpret_cast<volatile int *>(smem + WS_OFF_BAR + 8 * B_COUNT + 4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t smem_base = ptx::smem_u32(smem);
  const int tn = p.tile_n;
  const int kc = DRAIN ? p.kc_slabs : (1 << 30);
  static_assert(!(DRAIN && WIDE), "the long-K fold needs 8 epilogue warps");
  using Roles = WsRoles<WIDE>;

  if (tid == 0) {
    for (int i = 0; i < WS_STAGES; ++i) {
      ptx::mbar_init(&bars[B_FULL + i], 1);
      ptx::mbar_init(&bars[B_EMPTY + i], Roles::NC);
    }
    for (int i = 0; i < 2; ++i) {
      ptx::mbar_init(&bars[B_BFULL + i], Roles::NC);
      ptx::mbar_init(&bars[B_BEMPTY + i], 1);
      ptx::mbar_init(&bars[B_AFULL + i], 1);
      ptx::mbar_init(&bars[B_AEMPTY + i], Roles::NE);
    }
    ptx::mbar_init(&bars[B_FINAL], 1);
    *s_abort = 0;
    ptx::fence_mbar_init();
  }
  if (warp == 1) {
    ptx::tmem_alloc(tmem_slot, WS_TMEM_COLS);
    ptx::tmem_relinquish();
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ------------------------------ producer ------------------------------
    if (lane == 0) {
      long j = 0;
      for (long t = blockIdx.x; t < p.num_tiles && !*s_abort; t += gridDim.x) {
        const TileInfo ti = decode_tile(p, t);
        for (int s = 0; s < p.nk; ++s, ++j) {
          const int st = (int)(j % WS_STAGES);
          if (j >= WS_STAGES &&
              !ws_wait(&bars[B_EMPTY + st], (uint32_t)(((j / WS_STAGES) - 1) & 1), s_abort, p.err))
            break;
          const uint32_t dst = smem_base + WS_OFF_STAGE + st * WS_STAGE_BYTES;
          mbar_arrive_tx(&bars[B_FULL + st], args.tx_bytes);
          const int k0 = s * TC_BK;
          // split-K: slice g reads K range [g*kslice, (g+1)*kslice) of one matrix
          const int g = p.kslice ? 0 : (int)ti.g0;
          const int kk = k0 + (p.kslice ? (int)ti.g0 * p.kslice : 0);
          tma_load_3d(dst, &tmA, &bars[B_FULL + st], kk, ti.m0, g);
          if (p.transb) tma_load_3d(dst + 16384, &tmB, &bars[B_FULL + st], kk, ti.n0, g);
          else tma_load_3d(dst + 16384, &tmB, &bars[B_FULL + st], ti.n0, kk, g);
        }
      }
    }
  } else if (warp == 1) {
    // -------------------------------- MMA ---------------------------------
    if (lane == 0) {
      const uint32_t idesc = ptx::idesc_bf16_f32(TC_BM, tn);
      long j = 0, u = 0;
      bool ok = true;
      for (long t = blockIdx.x; ok && t < p.num_tiles; t += gridDim.x) {
        for (int s = 0; ok && s < p.nk; ++s, ++j) {
          const int s_in = s % kc;
          if (s_in == 0) {
            // new accumulation chunk: wait until the epilogue has drained this set
            const int a = (int)(u & 1);
            if (u >= 2 && !ws_wait(&bars[B_AEMPTY + a], (uint32_t)(((u >> 1) - 1) & 1), s_abort,
                                   p.err)) {
              ok = false;
              break;
            }
          }
          const int b = (int)(j & 1);
          if (!ws_wait(&bars[B_BFULL + b], (uint32_t)((j >> 1) & 1), s_abort, p.err)) {
            ok = false;
            break;
          }
          ptx::tc_fence_after();
          const uint32_t acc_base = tmem + (uint32_t)((u & 1) * 256);
          const uint32_t bb = smem_base + WS_OFF_BUF + b * BUF_BYTES;
          const int ksteps = min(2, (p.K - s * TC_BK + 15) / 16);
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {
            if (ks >= ksteps) break;
            const uint32_t acc = (s_in > 0 || ks > 0) ? 1u : 0u;
            uint64_t da[3], db[3];
#pragma unroll
            for (int sp = 0; sp < NSPLIT; ++sp) {
              da[sp] = ptx::smem_desc(bb + sp * SPLIT_BYTES + ks * 2 * CHUNK_BYTES, CHUNK_BYTES, 128);
              db[sp] = ptx::smem_desc(bb + sp * SPLIT_BYTES + 8192 + ks * 2 * CHUNK_BYTES,
                                      CHUNK_BYTES, 128);
            }
            ptx::mma_bf16(acc_base, da[0], db[0], idesc, acc);
            ptx::mma_bf16(acc_base + 128, da[0], db[1], idesc, acc);
            ptx::mma_bf16(acc_base + 128, da[1], db[0], idesc, 1u);
            if (NSPLIT == 3) {
              ptx::mma_bf16(acc_base + 128, da[0], db[2], idesc, 1u);
              ptx::mma_bf16(acc_base + 128, da[2], db[0], idesc, 1u);
              ptx::mma_bf16(acc_base + 128, da[1], db[1], idesc, 1u);
            }
          }
          ptx::mma_commit(&bars[B_BEMPTY + b]);  // operand buffer b may be refilled
          if (s_in == kc - 1 || s == p.nk - 1) {
            ptx::mma_commit(&bars[B_AFULL + (u & 1)]);  // accumulation chunk complete
            ++u;
          }
        }
      }
      // every MMA this thread issued has completed before TMEM is freed
      ptx::mma_commit(&bars[B_FINAL]);
      ptx::mbar_wait_bounded(&bars[B_FINAL], 0);
    }
  } else if (warp < Roles::W_EPI) {
    // ----------------------------- converters -----------------------------
    // items of a slab: A (row cr, 8-k chunk c) and B (column jj, chunk c),
    // 512 of each, taken round-robin by the NCT threads (a fixed mapping:
    // consecutive lanes take consecutive rows).  Rows and columns past the
    // tile's GEMMs and the chunks past K of a last half slab are not
    // converted: the MMA reads stale shared memory there, which reaches only
    // output rows and columns that are never stored (and no MMA k-step at all).
    constexpr int NCT = Roles::NC * 32;
    constexpr int PER = 512 / NCT;
    const int ct = tid - W_CONV0 * 32;
    const bool nn = !p.transb;
    const int nn_w = args.nn_w;
    // quotients by tn and N through float reciprocals: exact for the ranges
    // here (e < 4 tn <= 512, jj < 128), whose fractions stay at least 1/256
    // away from the next integer
    const float inv_tn = 1.0f / (float)tn, inv_n = 1.0f / (float)max(1, p.N);
    long j = 0;
    bool ok = true;
    for (long t = blockIdx.x; ok && t < p.num_tiles; t += gridDim.x) {
      const TileInfo ti = decode_tile(p, t);
      const int a_rows = p.G > 1 ? ti.ng * p.M : min(TC_BM, p.M - ti.m0);
      const int b_cols = p.G > 1 ? ti.ng * p.N : min(tn, p.N - ti.n0);
      for (int s = 0; s < p.nk; ++s, ++j) {
        const int st = (int)(j % WS_STAGES), b = (int)(j & 1);
        if (!ws_wait(&bars[B_FULL + st], (uint32_t)((j / WS_STAGES) & 1), s_abort, p.err)) {
          ok = false;
          break;
        }
        if (j >= 2 && !ws_wait(&bars[B_BEMPTY + b], (uint32_t)(((j >> 1) - 1) & 1), s_abort,
                               p.err)) {
          ok = false;
          break;
        }
        const int nchunk = p.K - s * TC_BK <= 16 ? 2 : 4;  // the MMA's k-steps x 2
        const unsigned char *stg = smem + WS_OFF_STAGE + st * WS_STAGE_BYTES;
        unsigned char *base = smem + WS_OFF_BUF + b * BUF_BYTES;
#pragma unroll
        for (int q = 0; q < PER; ++q) {
          const int idx = ct + q * NCT;
          const int cr = idx & 127, c = idx >> 7;
          if (cr < a_rows && c < nchunk) {
            const unsigned char *row = stg + cr * 128;
            const float4 u0 =
                *reinterpret_cast<const float4 *>(row + (((2 * c) ^ (cr & 7)) << 4));
            const float4 u1 =
                *reinterpret_cast<const float4 *>(row + (((2 * c + 1) ^ (cr & 7)) << 4));
            float x[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
            uint4 h, m, l;
            split8<NSPLIT>(x, h, m, l);
            const int off = c * CHUNK_BYTES + cr * 16;
            *reinterpret_cast<uint4 *>(base + off) = h;
            *reinterpret_cast<uint4 *>(base + SPLIT_BYTES + off) = m;
            if (NSPLIT == 3) *reinterpret_cast<uint4 *>(base + 2 * SPLIT_BYTES + off) = l;
          }
        }
#pragma unroll
        for (int q = 0; q < PER; ++q) {
          const int e = ct + q * NCT;
          const int c = (int)(((float)e + 0.5f) * inv_tn), jj = e - c * tn;
          if (e < 4 * tn && jj < b_cols && c < nchunk) {
            float x[8];
            if (!nn) {
              const unsigned char *row = stg + 16384 + jj * 128;
              const float4 u0 =
                  *reinterpret_cast<const float4 *>(row + (((2 * c) ^ (jj & 7)) << 4));
              const float4 u1 =
                  *reinterpret_cast<const float4 *>(row + (((2 * c + 1) ^ (jj & 7)) << 4));
              x[0] = u0.x; x[1] = u0.y; x[2] = u0.z; x[3] = u0.w;
              x[4] = u1.x; x[5] = u1.y; x[6] = u1.z; x[7] = u1.w;
            } else {
              // [g][32 k][nn_w] (packed) or [32 k][tn]: column jj of GEMM g = jj / N
              const float *fb = reinterpret_cast<const float *>(stg + 16384);
              int col = jj, gofs = 0;
              if (p.G > 1) {
                const int g = (int)(((float)jj + 0.5f) * inv_n);
                col = jj - g * p.N;
                gofs = g * 32 * nn_w;
              }
#pragma unroll
              for (int tk = 0; tk < 8; ++tk) x[tk] = fb[gofs + (8 * c + tk) * nn_w + col];
            }
            uint4 h, m, l;
            split8<NSPLIT>(x, h, m, l);
            const int off = 8192 + c * CHUNK_BYTES + jj * 16;
            *reinterpret_cast<uint4 *>(base + off) = h;
            *reinterpret_cast<uint4 *>(base + SPLIT_BYTES + off) = m;
            if (NSPLIT == 3) *reinterpret_cast<uint4 *>(base + 2 * SPLIT_BYTES + off) = l;
          }
        }
        ptx::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&bars[B_EMPTY + st]);  // staging slab consumed
          mbar_arrive(&bars[B_BFULL + b]);   // operand buffer ready for the MMA
        }
      }
    }
  } else {
    // ------------------------------ epilogue ------------------------------
    // warp (TMEM lane quarter wq, column group grp) owns the 32-column blocks
    // grp, grp + NG, ... of its 32 rows: chunk q (8 columns) of the warp is
    // tile chunk chunk_of(q)
    constexpr int NG = Roles::NE / 4, BL = BLX > 0 ? BLX : Roles::BLOCKS;
    constexpr int NBUF = 8 / Roles::NE;  // 4 KB staging buffers per warp
    const int ew = warp - Roles::W_EPI;
    const int wq = warp & 3, grp = ew >> 2;
    const int r = wq * 32 + lane;
    const int nch = tn / 8;
    auto chunk_of = [&](int q) { return 4 * (grp + NG * (q >> 2)) + (q & 3); };
    int nb = 0;  // 32-column blocks of this warp inside the tile
    while (nb < BL && chunk_of(4 * nb) < nch) ++nb;
    const bool ctma = args.c_tma != 0;
    unsigned char *cst = smem + WS_OFF_CST + ew * NBUF * WS_CST_WARP;
    const uint32_t cst_u = smem_base + WS_OFF_CST + ew * NBUF * WS_CST_WARP;
    int sb = 0;  // (lane 0) bulk stores issued by this warp
    constexpr int RMAX = DRAIN ? 32 * BL : 1;
    float R[RMAX];
    long u = 0;
    bool ok = true;
    for (long t = blockIdx.x; ok && t < p.num_tiles; t += gridDim.x) {
      const TileInfo ti = decode_tile(p, t);
      int gi, i, jlo, jhi;
      bool rok;
      if (p.G > 1) {
        gi = r / p.M; i = r - gi * p.M; rok = gi < ti.ng;
        jlo = gi * p.N; jhi = jlo + p.N;
      } else {
        gi = 0; i = ti.m0 + r; rok = i < p.M;
        jlo = 0; jhi = min(tn, p.N - ti.n0);
      }
      float *crow = p.C + (ti.g0 + gi) * p.sC + (long)i * p.ldc + (ti.n0 - jlo);
      const bool vec = p.vec_c && ((p.G == 1) || (p.N % 4 == 0));
      auto store8 = [&](int ch, const float *v) {
        const int j0 = ch * 8;
        if (!rok || j0 + 8 <= jlo || j0 >= jhi) return;
        if (vec && j0 >= jlo && j0 + 8 <= jhi) {
          float4 o0, o1;
          if (p.beta != 0.0f) {
            const float4 c0 = *reinterpret_cast<const float4 *>(crow + j0);
            const float4 c1 = *reinterpret_cast<const float4 *>(crow + j0 + 4);
            o0 = make_float4(__fmaf_rn(p.beta, c0.x, p.alpha * v[0]),
                             __fmaf_rn(p.beta, c0.y, p.alpha * v[1]),
                             __fmaf_rn(p.beta, c0.z, p.alpha * v[2]),
                             __fmaf_rn(p.beta, c0.w, p.alpha * v[3]));
            o1 = make_float4(__fmaf_rn(p.beta, c1.x, p.alpha * v[4]),
                             __fmaf_rn(p.beta, c1.y, p.alpha * v[5]),
                             __fmaf_rn(p.beta, c1.z, p.alpha * v[6]),
                             __fmaf_rn(p.beta, c1.w, p.alpha * v[7]));
          } else {
            o0 = make_float4(p.alpha * v[0], p.alpha * v[1], p.alpha * v[2], p.alpha * v[3]);
            o1 = make_float4(p.alpha * v[4], p.alpha * v[5], p.alpha * v[6], p.alpha * v[7]);
          }
          *reinterpret_cast<float4 *>(crow + j0) = o0;
          *reinterpret_cast<float4 *>(crow + j0 + 4) = o1;
        } else {
#pragma unroll
          for (int w = 0; w < 8; ++w) {
            const int jc = j0 + w;
            if (jc >= jlo && jc < jhi) {
              float x = p.alpha * v[w];
              if (p.beta != 0.0f) x = __fmaf_rn(p.beta, crow[jc], x);
              crow[jc] = x;
            }
          }
        }
      };
      // block pb (chunks 4 pb .. 4 pb + 3 of the warp, values v[32]) of this
      // warp's rows -> a staging buffer -> one TMA store; columns past tn are
      // past N (the host requires tiles_n == 1 or tn % 32 == 0) and clipped
      auto store_block = [&](int pb, const float *v) {
        const int buf = NBUF > 1 ? (sb & 1) : 0;
        if (lane == 0 && sb >= NBUF) {
          if (NBUF > 1) ptx::bulk_wait_read<1>();  // the store that last used buf is done
          else ptx::bulk_wait_read<0>();
        }
        __syncwarp();
        unsigned char *row = cst + buf * WS_CST_WARP + lane * 128;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const float *x = v + 4 * c;
          *reinterpret_cast<float4 *>(row + ((c ^ (lane & 7)) << 4)) =
              make_float4(p.alpha * x[0], p.alpha * x[1], p.alpha * x[2], p.alpha * x[3]);
        }
        ptx::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          ptx::tma_store_3d(&tmC, cst_u + buf * WS_CST_WARP, ti.n0 + chunk_of(4 * pb) * 8,
                            ti.m0 + wq * 32, (int)ti.g0);
          ptx::bulk_commit();
        }
        ++sb;
      };
      auto release = [&](int a) {
        ptx::tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_relaxed(&bars[B_AEMPTY + a]);
      };
      const bool rows_in = ti.m0 + wq * 32 < p.M;  // G == 1 when ctma
      // chunks holding columns of the GEMMs whose rows this warp covers
      // (warp-uniform; every chunk for one GEMM per tile)
      int c_lo = 0, c_hi = nch;
      if (p.G > 1) {
        const int g_lo = (wq * 32) / p.M, g_hi = min(ti.ng - 1, (wq * 32 + 31) / p.M);
        c_lo = g_lo < ti.ng ? (g_lo * p.N) / 8 : nch;
        c_hi = g_lo < ti.ng ? min(nch, ((g_hi + 1) * p.N + 7) / 8) : nch;
      }
      const int nchunks = DRAIN ? (p.nk + kc - 1) / kc : 1;
#pragma unroll
      for (int w = 0; w < RMAX; ++w) R[w] = 0.0f;
      for (int cu = 0; cu < nchunks; ++cu, ++u) {
        const int a = (int)(u & 1);
        if (!ws_wait(&bars[B_AFULL + a], (uint32_t)((u >> 1) & 1), s_abort, p.err)) {
          ok = false;
          break;
        }
        ptx::tc_fence_after();
        const uint32_t acc_base = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)(a * 256);
        if constexpr (DRAIN) {
#pragma unroll
          for (int q = 0; q < 4 * BL; ++q) {
            const int ch = chunk_of(q);
            if (ch >= c_lo && ch < c_hi) {
              float dm[8], dc[8];
              ptx::tmem_ld8(acc_base + ch * 8, dm);
              ptx::tmem_ld8(acc_base + 128 + ch * 8, dc);
              ptx::tmem_wait_ld();
#pragma unroll
              for (int w = 0; w < 8; ++w) R[q * 8 + w] += dm[w] + dc[w];
            }
          }
          release(a);
        } else if (ctma) {
          // block by block: TMEM loads, then (after the last block's loads)
          // release the accumulator, then stage and store
          if (nb == 0) release(a);
#pragma unroll
          for (int pb = 0; pb < BL; ++pb) {
            if (pb < nb) {
              float v[32];
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                const int ch = chunk_of(4 * pb + q);
                float dc[8];
                if (ch < nch) {
                  ptx::tmem_ld8(acc_base + ch * 8, v + 8 * q);
                  ptx::tmem_ld8(acc_base + 128 + ch * 8, dc);
                } else {
#pragma unroll
                  for (int w = 0; w < 8; ++w) v[8 * q + w] = dc[w] = 0.0f;
                }
                ptx::tmem_wait_ld();
#pragma unroll
                for (int w = 0; w < 8; ++w) v[8 * q + w] += dc[w];
              }
              if (pb == nb - 1) release(a);
              if (rows_in) store_block(pb, v);
            }
          }
        } else {
          for (int q = 0; q < 4 * BL; ++q) {
            const int ch = chunk_of(q);
            if (ch < c_lo || ch >= c_hi) continue;
            float dm[8], dc[8];
            ptx::tmem_ld8(acc_base + ch * 8, dm);
            ptx::tmem_ld8(acc_base + 128 + ch * 8, dc);
            ptx::tmem_wait_ld();
#pragma unroll
            for (int w = 0; w < 8; ++w) dm[w] += dc[w];
            store8(ch, dm);
          }
          release(a);
        }
      }
      if constexpr (DRAIN) {
        if (ok) {
          if (ctma) {
            if (rows_in) {
#pragma unroll
              for (int pb = 0; pb < BL; ++pb)
                if (pb < nb) store_block(pb, R + 32 * pb);
            }
          } else {
#pragma unroll
            for (int q = 0; q < 4 * BL; ++q) {
              const int ch = chunk_of(q);
              if (ch < nch) store8(ch, R + q * 8);
            }
          }
        }
      }
    }
    // the kernel's C writes are complete before the CTA exits
    if (lane == 0 && sb > 0) ptx::bulk_wait_all();
  }

  __syncthreads();
  if (warp == 1) {
    ptx::tc_fence_after();
    ptx::tmem_dealloc(tmem, WS_TMEM_COLS);
  }
}

// ===========================================================================
// Grouped batches (LibShalom_sgemm_batched): arbitrary per-GEMM pointers,
// shapes, transposes, leading dimensions, alpha and beta, read from device
// entries.  Same converter / MMA / epilogue warps as the TMA kernel; the
// producer is two warps of cp.async (any alignment) whose completion arrives
// on the stage's mbarrier (cp.async.mbarrier.arrive.noinc).  The FP32 slab is
// staged in the same layout the TMA kernel uses (A and B (Trans) rows of 128
// bytes with the 128-byte swizzle, B (NoTrans) as [32 k][tile_n]).
//
// Work plan (built on the device, sized by the entry count alone, so a call
// needs no host round trip): runs of entries sharing C are sorted by their K
// work (counting sort over GRP_CLASSES classes, heaviest first) and the
// persistent CTAs take the sorted runs round-robin.  Inside a CTA a scheduler
// warp expands its runs into (tile, product) items for the other roles.  The
// products of a run are applied in array order by the one CTA that owns the
// run (C = alpha_p A_p op(B_p) + beta_p C, product by product).
// ===========================================================================
constexpr int GRP_CLASSES = 64;  // work classes (total K slabs of the run, capped)

// workspace layout of the plan (unsigned words)
struct GrpPlan {
  unsigned *class_runs;   // [GRP_CLASSES] runs per class
  unsigned *class_off;    // [GRP_CLASSES] first sorted slot of each class
  unsigned *class_fill;   // [GRP_CLASSES] slots taken so far
  unsigned *n_runs;       // [1]
  unsigned *run_first;    // [count] first entry of the run in sorted slot s
  unsigned *run_len;      // [count]
};

struct GrpArgs {
  const LibShalom_sgemm_entry *entries;
  long count;
  const unsigned *run_first, *run_len, *n_runs;
  unsigned *err;
  int kc_slabs;
};


__device__ __forceinline__ int grp_tile_n(int N) { return min(TC_MAX_N, (N + 15) / 16 * 16); }

__device__ __forceinline__ bool grp_run_start(const LibShalom_sgemm_entry *e, long i) {
  return i == 0 || e[i].C != e[i - 1].C;
}

// K work of the run starting at entry i (capped class index) and its length
__device__ __forceinline__ int grp_run_class(const LibShalom_sgemm_entry *e, long count, long i,
                                             long *len) {
  long slabs = 0, j = i;
  do {
    slabs += max(1, (e[j].K + TC_BK - 1) / TC_BK);
    ++j;
  } while (j < count && e[j].C == e[i].C);
  *len = j - i;
  return (int)min(slabs, (long)GRP_CLASSES - 1);
}

// pass 1: runs per work class
__global__ void k_grp_count(const LibShalom_sgemm_entry *e, long count, GrpPlan pl) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count;
       i += (long)gridDim.x * blockDim.x) {
    if (!grp_run_start(e, i)) continue;
    long len;
    atomicAdd(&pl.class_runs[grp_run_class(e, count, i, &len)], 1u);
  }
}

// pass 2: first sorted slot of every class, heaviest class first
__global__ void k_grp_offsets(GrpPlan pl) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    unsigned acc = 0;
    for (int c = GRP_CLASSES - 1; c >= 0; --c) {
      pl.class_off[c] = acc;
      acc += pl.class_runs[c];
    }
    *pl.n_runs = acc;
  }
}

// pass 3: every run takes a slot in its class's range
__global__ void k_grp_place(const LibShalom_sgemm_entry *e, long count, GrpPlan pl) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count;
       i += (long)gridDim.x * blockDim.x) {
    if (!grp_run_start(e, i)) continue;
    long len;
    const int cls = grp_run_class(e, count, i, &len);
    const unsigned slot = pl.class_off[cls] + atomicAdd(&pl.class_fill[cls], 1u);
    pl.run_first[slot] = (unsigned)i;
    pl.run_len[slot] = (unsigned)len;
  }
}


// Work queue of the grouped kernel.  One scheduler warp walks the CTA's runs
// 32 at a time (one lane per run: plan slot, run length and tile count in
// parallel), expands them into (tile, product) items and writes the items
// into a 32-slot ring in shared memory; the other roles read the items from
// there.  Every item is one product on one output tile; the epilogue releases
// its slot once the item's last accumulator has been read from TMEM, after
// which every other role has finished with it too.
struct __align__(16) GSlot {
  const float *A, *B;
  float *C;
  int M, N, K, lda;
  int ldbx;  // ldb, or ~ldb when B is transposed
  int ldc, m0, n0;
  float alpha, beta;
};
static_assert(sizeof(GSlot) == 64, "queue slot is four 16-byte words");

constexpr int GQ = 32;  // queue slots
// staging ring: the FP32 slab in the TMA kernel's layout (A and B (Trans)
// rows of 128 bytes, 128-byte swizzle; B (NoTrans) as [32 k][tile_n])
constexpr int G_STAGES = 4;
constexpr int G_STAGE_A = 16384;
constexpr int G_STAGE_BYTES = 2 * G_STAGE_A;
constexpr int G_OFF_STAGE = 2 * BUF_BYTES;            // after the two BF16 operand buffers
constexpr int G_OFF_BAR = G_OFF_STAGE + G_STAGES * G_STAGE_BYTES;
constexpr int G_OFF_QBAR = G_OFF_BAR + 256;          // GQ full + GQ empty mbarriers
constexpr int G_OFF_Q = G_OFF_QBAR + 2 * GQ * 8;    // GQ slots
constexpr int G_SMEM = G_OFF_Q + GQ * (int)sizeof(GSlot);
static_assert(G_SMEM <= 232448, "grouped kernel exceeds 227 KB of shared memory");

// warp 0 MMA, 1 scheduler, 2-9 converters (which also stage the operands),
// 10-25 epilogue.  The MMAs compute C^T (op(B)^T as the 128-row operand, A as
// the N operand): TMEM lanes are the tile's columns, so the 16 epilogue warps
// (4 TMEM lane quarters x 4 row quarters) hold one column and up to 32 rows a
// thread and read / write C one row of 32 consecutive floats per instruction.
constexpr int G_W_MMA = 0, G_W_SCHED = 1, G_W_CONV0 = 2, G_W_EPI0 = 10;
constexpr int G_N_EPI = 16;
constexpr int G_WARPS = 26;
constexpr int G_THREADS = G_WARPS * 32;

// one queue item as the consuming roles use it
struct GItem {
  const float *A, *B;
  float *C;
  int M, N, K, lda, ldb, ldc, m0, n0, transb, tn, nk;
  float alpha, beta;
};

__device__ __forceinline__ bool q_get(const unsigned char *smem, long j, GItem &it,
                                      volatile int *s_abort, unsigned *err) {
  uint64_t *qfull = reinterpret_cast<uint64_t *>(const_cast<unsigned char *>(smem) + G_OFF_QBAR);
  const int slot = (int)(j % GQ);
  if (!__all_sync(0xffffffffu, ws_wait(&qfull[slot], (uint32_t)((j / GQ) & 1), s_abort, err)))
    return false;
  const GSlot s = reinterpret_cast<const GSlot *>(smem + G_OFF_Q)[slot];
  it.A = s.A; it.B = s.B; it.C = s.C;
  it.M = s.M; it.N = s.N; it.K = s.K; it.lda = s.lda;
  it.transb = s.ldbx < 0;
  it.ldb = it.transb ? ~s.ldbx : s.ldbx;
  it.ldc = s.ldc; it.m0 = s.m0; it.n0 = s.n0;
  it.alpha = s.alpha; it.beta = s.beta;
  it.tn = grp_tile_n(max(1, it.N));
  it.nk = max(1, (it.K + TC_BK - 1) / TC_BK);
  return true;
}

// C[i] += v at L2 (red.global.add.f32: round to nearest even; subnormal
// inputs and sums flush to zero)
__device__ __forceinline__ void red_add_f32(float *p, float v) {
  asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(ptx::smem_u32(bar))
               : "memory");
}

// floats per cp.async for rows of a matrix: 4 (16-byte), 2 (8-byte) or 1
__device__ __forceinline__ int row_vec(const float *p, int ld) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  if ((a & 15) == 0 && (ld & 3) == 0) return 4;
  if ((a & 7) == 0 && (ld & 1) == 0) return 2;
  return 1;
}

__device__ __forceinline__ void cp_async8(uint32_t saddr, const void *g, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(saddr), "l"(g),
               "r"(src_bytes)
               : "memory");
}

// 16-byte staging chunk: n valid floats at src (0..4), the rest zero-filled;
// vw = floats per copy the row alignment allows
__device__ __forceinline__ void stage_chunk(uint32_t dst, const float *src, int n, int vw,
                                            const float *any) {
  if (vw == 4) {
    cp_async16(dst, n > 0 ? src : any, 4 * n);
  } else if (vw == 2) {
    cp_async8(dst, n > 0 ? src : any, 4 * min(2, n));
    cp_async8(dst + 8, n > 2 ? src + 2 : any, 4 * max(0, n - 2));
  } else {
#pragma unroll
    for (int w = 0; w < 4; ++w) cp_async4(dst + 4 * w, w < n ? src + w : any, w < n ? 4 : 0);
  }
}

// Rows of an item that only touch output rows / columns outside C are not
// staged or converted: the tensor core then reads whatever an earlier item
// left in those shared-memory rows, which reaches only output rows >= M or
// columns >= N, never stored.  Inside the valid rows every k >= K is zero in
// both operands, so the padded K adds exact zeros.
template <int NSPLIT>
__global__ void __launch_bounds__(G_THREADS, 1) k_tc_grouped(const GrpArgs g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + G_OFF_BAR);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + G_OFF_BAR + 8 * B_COUNT);
  volatile int *s_abort = reinterpret_cast<volatile int *>(smem + G_OFF_BAR + 8 * B_COUNT + 4);
  uint64_t *qfull = reinterpret_cast<uint64_t *>(smem + G_OFF_QBAR);
  uint64_t *qempty = qfull + GQ;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t smem_base = ptx::smem_u32(smem);
  const int kc = g.kc_slabs;

  if (tid == 0) {
    for (int i = 0; i < G_STAGES; ++i) {
      ptx::mbar_init(&bars[B_FULL + i], N_CONV * 32);
      ptx::mbar_init(&bars[B_EMPTY + i], N_CONV);
    }
    for (int i = 0; i < 2; ++i) {
      ptx::mbar_init(&bars[B_BFULL + i], N_CONV);
      ptx::mbar_init(&bars[B_BEMPTY + i], 1);
      ptx::mbar_init(&bars[B_AFULL + i], 1);
      ptx::mbar_init(&bars[B_AEMPTY + i], G_N_EPI);
    }
    ptx::mbar_init(&bars[B_FINAL], 1);
    for (int i = 0; i < GQ; ++i) {
      ptx::mbar_init(&qfull[i], 1);
      ptx::mbar_init(&qempty[i], G_N_EPI);
    }
    *s_abort = 0;
    ptx::fence_mbar_init();
  }
  if (warp == G_W_MMA) {
    ptx::tmem_alloc(tmem_slot, WS_TMEM_COLS);
    ptx::tmem_relinquish();
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == G_W_SCHED) {
    // ------------------------------ scheduler ------------------------------
    const long n_runs = (long)*g.n_runs;
    const long stride = gridDim.x;
    const unsigned FULL = 0xffffffffu;
    GSlot *qs = reinterpret_cast<GSlot *>(smem + G_OFF_Q);
    long q = 0;  // items written
    bool ok = true;
    for (long s0 = blockIdx.x; ok && s0 < n_runs; s0 += 32 * stride) {
      const long my_s = s0 + (long)lane * stride;
      int first = 0, len = 1, tn = 16, tiles_n = 1;
      long items = 0;
      if (my_s < n_runs) {
        first = (int)g.run_first[my_s];
        len = max(1, (int)g.run_len[my_s]);
        const int M = g.entries[first].M, N = g.entries[first].N;
        if (M > 0 && N > 0) {
          tn = grp_tile_n(N);
          tiles_n = (N + tn - 1) / tn;
          items = (long)((M + TC_BM - 1) / TC_BM) * tiles_n * len;
        }
      }
      long incl = items;  // inclusive prefix of items over the lanes
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
      }
      const long total = __shfl_sync(FULL, incl, 31);
      for (long base = 0; ok && base < total; base += 32) {
        const long i = base + lane;
        int r = 0;  // run of item i: runs whose inclusive prefix is <= i
        for (int k = 0; k < 32; ++k) r += __shfl_sync(FULL, incl, k) <= i ? 1 : 0;
        r = min(r, 31);
        const long r_start = __shfl_sync(FULL, incl, r) - __shfl_sync(FULL, items, r);
        const int r_first = __shfl_sync(FULL, first, r), r_len = __shfl_sync(FULL, len, r);
        const int r_tn = __shfl_sync(FULL, tn, r), r_tiles_n = __shfl_sync(FULL, tiles_n, r);
        bool lane_ok = true;
        if (i < total) {
          // items of a run: tile-major, products of a tile in array order
          const long loc = i - r_start;
          const int t = (int)(loc / r_len), p = (int)(loc - (long)t * r_len);
          const LibShalom_sgemm_entry e = g.entries[r_first + p];
          GSlot sl;
          const int K = max(0, e.K);
          sl.A = e.A; sl.B = e.B; sl.C = e.C;
          sl.M = e.M; sl.N = e.N; sl.K = K;
          sl.lda = e.lda > 0 ? e.lda : K;
          const int ldb = e.ldb > 0 ? e.ldb : (e.transb ? K : e.N);
          sl.ldbx = e.transb ? ~ldb : ldb;
          sl.ldc = e.ldc > 0 ? e.ldc : e.N;
          sl.m0 = (t / r_tiles_n) * TC_BM;
          sl.n0 = (t % r_tiles_n) * r_tn;
          sl.alpha = e.alpha; sl.beta = e.beta;
          const long qi = q + lane;
          const int slot = (int)(qi % GQ);
          if (qi >= GQ &&
              !ws_wait(&qempty[slot], (uint32_t)(((qi / GQ) - 1) & 1), s_abort, g.err)) {
            lane_ok = false;
          } else {
            qs[slot] = sl;
            mbar_arrive(&qfull[slot]);
          }
        }
        ok = __all_sync(FULL, lane_ok);
        q += min(32L, total - base);
      }
    }
    if (ok && lane == 0) {
      // end of the CTA's work: an item with M = -1
      const int slot = (int)(q % GQ);
      if (q < GQ || ws_wait(&qempty[slot], (uint32_t)(((q / GQ) - 1) & 1), s_abort, g.err)) {
        GSlot sl{};
        sl.M = -1;
        qs[slot] = sl;
        mbar_arrive(&qfull[slot]);
      }
    }
  } else if (warp == G_W_MMA) {
    // -------------------------------- MMA ---------------------------------
    // The whole warp walks the items and waits, so that none of its lanes
    // sits at the block barrier while the issuing lane works; lane 0 issues
    // the MMAs and the commits.
    const unsigned FULL = 0xffffffffu;
    long js = 0, u = 0;
    bool ok = true;
    for (long j = 0; ok; ++j) {
      GItem it;
      if (!q_get(smem, j, it, s_abort, g.err)) break;
      if (it.M < 0) break;
      // C^T = op(B)^T A^T: the 128 MMA rows (TMEM lanes) are the tile's
      // columns, the MMA N its rows (rounded to 16)
      const int mrows = min(TC_BM, it.M - it.m0);
      const uint32_t idesc = ptx::idesc_bf16_f32(TC_BM, (mrows + 15) / 16 * 16);
      for (int s = 0; s < it.nk; ++s, ++js) {
        const int s_in = s % kc;
        if (s_in == 0 && u >= 2) {
          const int a = (int)(u & 1);
          if (!__all_sync(FULL, ws_wait(&bars[B_AEMPTY + a], (uint32_t)(((u >> 1) - 1) & 1),
                                        s_abort, g.err))) {
            ok = false;
            break;
          }
        }
        const int b = (int)(js & 1);
        if (!__all_sync(FULL, ws_wait(&bars[B_BFULL + b], (uint32_t)((js >> 1) & 1), s_abort,
                                      g.err))) {
          ok = false;
          break;
        }
        ptx::tc_fence_after();
        const bool last = s_in == kc - 1 || s == it.nk - 1;
        if (lane == 0) {
          const uint32_t acc_base = tmem + (uint32_t)((u & 1) * 256);
          const uint32_t bb = smem_base + WS_OFF_BUF + b * BUF_BYTES;
          const int ksteps = max(1, min(2, (it.K - s * TC_BK + 15) / 16));
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {
            if (ks >= ksteps) break;
            const uint32_t acc = (s_in > 0 || ks > 0) ? 1u : 0u;
            uint64_t da[3], db[3];  // da: op(B) columns (MMA rows), db: A rows
#pragma unroll
            for (int sp = 0; sp < NSPLIT; ++sp) {
              da[sp] = ptx::smem_desc(bb + sp * SPLIT_BYTES + 8192 + ks * 2 * CHUNK_BYTES,
                                      CHUNK_BYTES, 128);
              db[sp] = ptx::smem_desc(bb + sp * SPLIT_BYTES + ks * 2 * CHUNK_BYTES, CHUNK_BYTES, 128);
            }
            ptx::mma_bf16(acc_base, da[0], db[0], idesc, acc);
            ptx::mma_bf16(acc_base + 128, da[0], db[1], idesc, acc);
            ptx::mma_bf16(acc_base + 128, da[1], db[0], idesc, 1u);
            if (NSPLIT == 3) {
              ptx::mma_bf16(acc_base + 128, da[0], db[2], idesc, 1u);
              ptx::mma_bf16(acc_base + 128, da[2], db[0], idesc, 1u);
              ptx::mma_bf16(acc_base + 128, da[1], db[1], idesc, 1u);
            }
          }
          ptx::mma_commit(&bars[B_BEMPTY + b]);
          if (last) ptx::mma_commit(&bars[B_AFULL + (u & 1)]);
        }
        __syncwarp();
        if (last) ++u;
      }
    }
    if (lane == 0) ptx::mma_commit(&bars[B_FINAL]);
    __syncwarp();
    ptx::mbar_wait_bounded(&bars[B_FINAL], 0);
  } else if (warp < G_W_EPI0) {
    // --------------------- converters (and operand loads) ---------------------
    // The 256 converter threads also stage the operands: before converting
    // slab js they issue the cp.async copies of slab js + G_STAGES - 1 (a
    // second cursor over the queue), all of them arriving on that stage's
    // mbarrier.  Only valid rows / columns are staged; k >= K inside them is
    // zero-filled.
    const int ct = tid - G_W_CONV0 * 32;
    constexpr int NP = N_CONV * 32;
    const int cr = ct & 127, cc0 = ct >> 7;
    bool ok = true;
    // load cursor
    long jl = 0, jsl = 0;
    int sl = 0;
    bool have_l = false, l_end = false;
    GItem il;
    auto issue_next = [&]() -> bool {
      if (l_end) return true;
      if (!have_l) {
        if (!q_get(smem, jl, il, s_abort, g.err)) return false;
        if (il.M < 0) {
          l_end = true;
          return true;
        }
        have_l = true;
        sl = 0;
      }
      const int st = (int)(jsl % G_STAGES);
      if (jsl >= G_STAGES &&
          !__all_sync(0xffffffffu, ws_wait(&bars[B_EMPTY + st],
                                           (uint32_t)(((jsl / G_STAGES) - 1) & 1), s_abort, g.err)))
        return false;
      const int mrows = min(TC_BM, il.M - il.m0), ncols = min(il.tn, il.N - il.n0);
      const int va = row_vec(il.A, il.lda), vb = row_vec(il.B, il.ldb);
      const uint32_t sa = smem_base + G_OFF_STAGE + st * G_STAGE_BYTES;
      const uint32_t sb = sa + G_STAGE_A;
      const int k0 = sl * TC_BK;
      const int kv = max(0, min(TC_BK, il.K - k0));  // valid k of the slab
      // A: valid rows x 8 chunks of 4 floats; swizzled 128-byte rows
      for (int e = ct; e < mrows * 8; e += NP) {
        const int r = e >> 3, q = e & 7;
        const uint32_t dst = sa + r * 128 + ((q ^ (r & 7)) << 4);
        const float *src = il.A + (long)(il.m0 + r) * il.lda + k0 + 4 * q;
        stage_chunk(dst, src, max(0, min(4, kv - 4 * q)), va, il.A);
      }
      if (il.transb) {
        for (int e = ct; e < ncols * 8; e += NP) {
          const int r = e >> 3, q = e & 7;
          const uint32_t dst = sb + r * 128 + ((q ^ (r & 7)) << 4);
          const float *src = il.B + (long)(il.n0 + r) * il.ldb + k0 + 4 * q;
          stage_chunk(dst, src, max(0, min(4, kv - 4 * q)), vb, il.B);
        }
      } else {
        // [32 k][tn] floats; the valid columns of every k row (zero past K)
        const int cpr = (ncols + 3) >> 2;
        const float inv_cpr = 1.0f / (float)cpr;  // exact quotients: e < 32 cpr <= 1024
        for (int e = ct; e < 32 * cpr; e += NP) {
          const int kr = (int)(((float)e + 0.5f) * inv_cpr), col = (e - kr * cpr) * 4;
          const uint32_t dst = sb + (kr * il.tn + col) * 4;
          const float *src = il.B + (long)(k0 + kr) * il.ldb + il.n0 + col;
          stage_chunk(dst, src, kr < kv ? min(4, ncols - col) : 0, vb, il.B);
        }
      }
      cp_async_mbar_arrive(&bars[B_FULL + st]);  // arrives when this thread's copies land
      ++jsl;
      if (++sl == il.nk) {
        have_l = false;
        ++jl;
      }
      return true;
    };
    for (int i = 0; ok && i < G_STAGES - 1; ++i) ok = issue_next();
    long js = 0;
    for (long j = 0; ok; ++j) {
      GItem it;
      if (!q_get(smem, j, it, s_abort, g.err)) break;
      if (it.M < 0) break;
      const int tn = it.tn;
      const int mrows = min(TC_BM, it.M - it.m0), ncols = min(tn, it.N - it.n0);
      // e / tn through an exact float reciprocal (e < 4 tn <= 512)
      const float inv_tn = 1.0f / (float)tn;
      for (int s = 0; s < it.nk; ++s, ++js) {
        if (!issue_next()) {
          ok = false;
          break;
        }
        const int st = (int)(js % G_STAGES), b = (int)(js & 1);
        if (!__all_sync(0xffffffffu, ws_wait(&bars[B_FULL + st], (uint32_t)((js / G_STAGES) & 1),
                                             s_abort, g.err))) {
          ok = false;
          break;
        }
        if (js >= 2 && !__all_sync(0xffffffffu, ws_wait(&bars[B_BEMPTY + b],
                                                        (uint32_t)(((js >> 1) - 1) & 1), s_abort,
                                                        g.err))) {
          ok = false;
          break;
        }
        const unsigned char *stg = smem + G_OFF_STAGE + st * G_STAGE_BYTES;
        unsigned char *base = smem + WS_OFF_BUF + b * BUF_BYTES;
        // a last slab of at most 16 valid k takes one MMA k-step: its upper
        // two 8-k chunks are never read, so they are not converted
        const int nchunk = it.K - s * TC_BK <= 16 ? 2 : 4;
        if (cr < mrows) {
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int c = cc0 + 2 * q;
            if (c >= nchunk) break;
            const unsigned char *row = stg + cr * 128;
            const float4 u0 = *reinterpret_cast<const float4 *>(row + (((2 * c) ^ (cr & 7)) << 4));
            const float4 u1 =
                *reinterpret_cast<const float4 *>(row + (((2 * c + 1) ^ (cr & 7)) << 4));
            float x[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
            uint4 h, m, l;
            split8<NSPLIT>(x, h, m, l);
            const int off = c * CHUNK_BYTES + cr * 16;
            *reinterpret_cast<uint4 *>(base + off) = h;
            *reinterpret_cast<uint4 *>(base + SPLIT_BYTES + off) = m;
            if (NSPLIT == 3) *reinterpret_cast<uint4 *>(base + 2 * SPLIT_BYTES + off) = l;
          }
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int e = ct + q * 256;
          const int c = (int)(((float)e + 0.5f) * inv_tn), jj = e - c * tn;
          if (e < 4 * tn && jj < ncols && c < nchunk) {
            float x[8];
            if (it.transb) {
              const unsigned char *row = stg + G_STAGE_A + jj * 128;
              const float4 u0 =
                  *reinterpret_cast<const float4 *>(row + (((2 * c) ^ (jj & 7)) << 4));
              const float4 u1 =
                  *reinterpret_cast<const float4 *>(row + (((2 * c + 1) ^ (jj & 7)) << 4));
              x[0] = u0.x; x[1] = u0.y; x[2] = u0.z; x[3] = u0.w;
              x[4] = u1.x; x[5] = u1.y; x[6] = u1.z; x[7] = u1.w;
            } else {
              const float *fb = reinterpret_cast<const float *>(stg + G_STAGE_A);
#pragma unroll
              for (int tk = 0; tk < 8; ++tk) x[tk] = fb[(8 * c + tk) * tn + jj];
            }
            uint4 h, m, l;
            split8<NSPLIT>(x, h, m, l);
            const int off = 8192 + c * CHUNK_BYTES + jj * 16;
            *reinterpret_cast<uint4 *>(base + off) = h;
            *reinterpret_cast<uint4 *>(base + SPLIT_BYTES + off) = m;
            if (NSPLIT == 3) *reinterpret_cast<uint4 *>(base + 2 * SPLIT_BYTES + off) = l;
          }
        }
        ptx::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&bars[B_EMPTY + st]);
          mbar_arrive(&bars[B_BFULL + b]);
        }
      }
    }
    cp_async_wait<0>();
  } else {
    // ------------------------------ epilogue ------------------------------
    // The accumulator holds C^T: TMEM lane = tile column, TMEM column = tile
    // row.  Thread (lane quarter wq, lane) owns column n0 + 32 wq + lane and
    // up to 32 rows (4 chunks of 8) of its warp's row quarter, so every beta
    // load and every store of one row is 32 consecutive floats across the
    // warp, whatever the alignment of C.  Each TMEM chunk is added into R as
    // alpha*D and released at once; at the end C = beta*C + R, eight rows at
    // a time (their loads issued together).
    const int wq = warp & 3, quarter = (warp - G_W_EPI0) >> 2;
    const int jc = wq * 32 + lane;  // tile column of this thread
    long u = 0;
    bool ok = true;
    for (long j = 0; ok; ++j) {
      GItem it;
      if (!q_get(smem, j, it, s_abort, g.err)) break;
      if (it.M < 0) break;
      const int mrows = min(TC_BM, it.M - it.m0);
      const int nchr = (mrows + 15) / 16 * 2, per = (nchr + 3) / 4;  // chunks of 8 rows
      const int c_begin = min(nchr, quarter * per), c_end = min(nchr, c_begin + per);
      const bool cok = jc < min(it.tn, it.N - it.n0);
      // this thread's rows: i0 .. i0 + n_rows - 1, at C[m0 + i][n0 + jc]
      const int i0 = c_begin * 8, n_rows = max(0, min(mrows, c_end * 8) - i0);
      const long ld = it.ldc;
      float *c0 = it.C + (long)(it.m0 + i0) * ld + it.n0 + jc;
      // beta == 1 (accumulation, and every run's later products): C += R by
      // fire-and-forget reductions, so no read of C waits in this warp's
      // item order; other nonzero betas read C first
      const bool acc1 = it.beta == 1.0f;
      const bool rd = cok && it.beta != 0.0f && !acc1;
      float R[32];
#pragma unroll
      for (int t = 0; t < 32; ++t) R[t] = 0.0f;
      const int nchunks = (it.nk + kc - 1) / kc;
      for (int cu = 0; cu < nchunks; ++cu, ++u) {
        const int a = (int)(u & 1);
        if (!__all_sync(0xffffffffu,
                        ws_wait(&bars[B_AFULL + a], (uint32_t)((u >> 1) & 1), s_abort, g.err))) {
          ok = false;
          break;
        }
        ptx::tc_fence_after();
        const uint32_t acc_base = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)(a * 256);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (c_begin + q < c_end) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              float dm[4], dc[4];
              ptx::tmem_ld4(acc_base + (c_begin + q) * 8 + 4 * h, dm);
              ptx::tmem_ld4(acc_base + 128 + (c_begin + q) * 8 + 4 * h, dc);
              ptx::tmem_wait_ld();
#pragma unroll
              for (int w = 0; w < 4; ++w) R[q * 8 + 4 * h + w] += it.alpha * (dm[w] + dc[w]);
            }
          }
        }
        ptx::tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_relaxed(&bars[B_AEMPTY + a]);
      }
      __syncwarp();
      if (ok && lane == 0) mbar_arrive_relaxed(&qempty[j % GQ]);
      // the whole warp stays together (lanes past N store nothing): a lane
      // that ran ahead into the next item would leave the warp diverged at
      // its collective TMEM loads
      if (!ok) continue;
      const int nr = cok ? n_rows : 0;
      if (acc1) {
#pragma unroll
        for (int t = 0; t < 32; ++t)
          if (t < nr) red_add_f32(c0 + (long)t * ld, R[t]);
      } else {
        float *pc = c0;
#pragma unroll
        for (int g8 = 0; g8 < 4; ++g8) {
          float cv[8];
#pragma unroll
          for (int w = 0; w < 8; ++w)
            cv[w] = rd && g8 * 8 + w < nr ? __ldcg(pc + (long)w * ld) : 0.0f;  // L2: sees earlier reductions
#pragma unroll
          for (int w = 0; w < 8; ++w) {
            const int t = g8 * 8 + w;
            if (t < nr) pc[(long)w * ld] = rd ? __fmaf_rn(it.beta, cv[w], R[t]) : R[t];
          }
          pc += 8 * ld;
        }
      }
    }
  }

  __syncthreads();
  if (warp == G_W_MMA) {
    ptx::tc_fence_after();
    ptx::tmem_dealloc(tmem, WS_TMEM_COLS);
  }
}

// device status word for the bounded waits
__device__ unsigned g_tc_err;

// Self-check of the bounded waits: an mbarrier nothing ever arrives at.  Warp
// 0 polls it `limit` times, gives up, raises the abort flag and sets the
// status word; warp 1 polls it with the kernels' full limit and gives up as
// soon as it sees the abort flag -- the path by which every role of a
// tensor-core kernel leaves after one role's wait has expired.
__global__ void k_wait_expiry(uint32_t limit, unsigned *err) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    ptx::mbar_init(&bar, 1);
    abort_flag = 0;
    ptx::fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x < 32) ws_wait(&bar, 0, &abort_flag, err, limit);
  else ws_wait(&bar, 0, &abort_flag, err);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link libcuda directly)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    else
      cudaGetLastError();
  }
  return fn;
}

bool aligned16(const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15) == 0; }

// 3-D FP32 tensor map: dims (d0 innermost, d1, d2), byte strides of d1 and d2.
bool encode_map(CUtensorMap *map, const float *base, uint64_t d0, uint64_t d1, uint64_t d2,
                uint64_t s1_bytes, uint64_t s2_bytes, uint32_t b0, uint32_t b1, uint32_t b2,
                bool swizzle128) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[3] = {d0, d1, d2};
  const cuuint64_t strides[2] = {s1_bytes, s2_bytes};
  const cuuint32_t box[3] = {b0, b1, b2};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims,
                         strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Tensor maps for the warp-specialized kernel, or false when TMA cannot
// address the operands (unaligned base or row stride, overlapping batches).
bool ws_maps(const TcProblem &p, CUtensorMap *ma, CUtensorMap *mb, CUtensorMap *mc, WsArgs *wa) {
  // split-K slices all read the one matrix pair: a single-batch tensor map
  const long count = p.kslice ? 1 : p.count;
  const long sA = count > 1 ? p.sA : (long)p.M * p.lda;
  const long rowsB = p.transb ? p.N : p.K;
  const long sB = count > 1 ? p.sB : rowsB * p.ldb;
  if (!aligned16(p.A) || !aligned16(p.B) || p.lda % 4 || p.ldb % 4 || sA % 4 || sB % 4)
    return false;
  if (count > 1 && (sA < (long)p.M * p.lda || sB < rowsB * p.ldb)) return false;
  const bool packed = p.G > 1;
  if (packed && !p.transb && p.N % 4) return false;  // B box rows must be 16-byte multiples
  const uint32_t a1 = packed ? p.M : TC_BM, a2 = packed ? p.G : 1;
  if (!encode_map(ma, p.A, p.K, p.M, count, (uint64_t)p.lda * 4, (uint64_t)sA * 4, TC_BK, a1,
                  a2, true))
    return false;
  uint32_t b0, b1, b2;
  if (p.transb) {
    b0 = TC_BK; b1 = packed ? p.N : p.tile_n; b2 = packed ? p.G : 1;
    if (!encode_map(mb, p.B, p.K, p.N, count, (uint64_t)p.ldb * 4, (uint64_t)sB * 4, b0, b1, b2,
                    true))
      return false;
  } else {
    b0 = packed ? p.N : p.tile_n; b1 = TC_BK; b2 = packed ? p.G : 1;
    if (!encode_map(mb, p.B, p.N, p.K, count, (uint64_t)p.ldb * 4, (uint64_t)sB * 4, b0, b1, b2,
                    false))
      return false;
  }
  wa->p = p;
  wa->tx_bytes = (uint32_t)(TC_BK * a1 * a2 + b0 * b1 * b2) * 4;
  wa->nn_w = p.transb ? 0 : (int)b0;
  // C by TMA stores: beta = 0 (nothing to read), one GEMM per tile, 16-byte
  // aligned rows, and every 32-column box either inside the tile or past N
  wa->c_tma = 0;
  const long sC = p.count > 1 ? p.sC : (long)p.M * p.ldc;
  if (p.beta == 0.0f && p.G == 1 && aligned16(p.C) && p.ldc % 4 == 0 && sC % 4 == 0 &&
      (p.count == 1 || sC >= (long)p.M * p.ldc) && (p.tiles_n == 1 || p.tile_n % 32 == 0) &&
      encode_map(mc, p.C, p.N, p.M, p.count, (uint64_t)p.ldc * 4, (uint64_t)sC * 4, 32, 32, 1,
                 true))
    wa->c_tma = 1;
  return true;
}

// The 16-byte paths of the kernels assume 16-byte aligned rows of every GEMM
// of the batch; a plan that claims one without it is refused on the host.
bool vec_flags_hold(const TcProblem &p) {
  const bool packed_cols = p.G > 1 && !p.transb && p.N % 4 != 0;
  if (p.vec_a && !(aligned16(p.A) && p.lda % 4 == 0 && p.sA % 4 == 0)) return false;
  if (p.vec_b && !(aligned16(p.B) && p.ldb % 4 == 0 && p.sB % 4 == 0 && !packed_cols))
    return false;
  if (p.vec_c && !(aligned16(p.C) && p.ldc % 4 == 0 && p.sC % 4 == 0)) return false;
  return true;
}

int tc_launch(TcProblem &p, int mode) {
  State &st = state();
  if (!vec_flags_hold(p)) return LIBSHALOM_ERR_UNSUPPORTED;
  void *errp = nullptr;
  LS_CUDA_TRY(cudaGetSymbolAddress(&errp, g_tc_err));
  p.err = reinterpret_cast<unsigned *>(errp);
  const bool drain = p.nk > p.kc_slabs;
  CUtensorMap ma, mb, mc;
  memset(&mc, 0, sizeof(mc));
  WsArgs wa;
  if (st.use_tma && ws_maps(p, &ma, &mb, &mc, &wa)) {
    const bool wide = !drain && wa.c_tma;
    // long K on tiles of at most 64 columns: one 32-column block per epilogue
    // warp, a fold of 32 registers instead of 64 (no spills)
    const bool narrow = drain && p.tile_n <= 32 * (WsRoles<false>::NE / 4);
    const void *kern =
        mode == LIBSHALOM_PREC_BF16X6
            ? (narrow ? (const void *)k_tc_ws<3, true, false, 1>
               : drain ? (const void *)k_tc_ws<3, true, false>
               : wide  ? (const void *)k_tc_ws<3, false, true>
                       : (const void *)k_tc_ws<3, false, false>)
            : (narrow ? (const void *)k_tc_ws<2, true, false, 1>
               : drain ? (const void *)k_tc_ws<2, true, false>
               : wide  ? (const void *)k_tc_ws<2, false, true>
                       : (const void *)k_tc_ws<2, false, false>);
    const int threads = wide ? WsRoles<true>::THREADS : WsRoles<false>::THREADS;
    (void)occupancy_of(kern, threads, WS_SMEM, 1);  // raises the shared-memory limit
    const int grid = grid_for(p.num_tiles, 1);
    void *args[] = {&ma, &mb, &mc, &wa};
    LS_CUDA_TRY(cudaLaunchKernel(kern, dim3(grid), dim3(threads), args, WS_SMEM, st.stream));
  } else {
    const void *kern = mode == LIBSHALOM_PREC_BF16X6
                           ? (drain ? (const void *)k_tc_sgemm<3, true> : (const void *)k_tc_sgemm<3, false>)
                           : (drain ? (const void *)k_tc_sgemm<2, true> : (const void *)k_tc_sgemm<2, false>);
    (void)occupancy_of(kern, TC_THREADS, TC_SMEM, 1);  // raises the shared-memory limit
    const int grid = grid_for(p.num_tiles, 1);
    void *args[] = {&p};
    LS_CUDA_TRY(cudaLaunchKernel(kern, dim3(grid), dim3(TC_THREADS), args, TC_SMEM, st.stream));
  }
  LS_CUDA_TRY(cudaGetLastError());
  if (st.sync) {
    // synchronous mode: report an expired device-side wait as a status
    unsigned err = 0;
    LS_CUDA_TRY(cudaStreamSynchronize(st.stream));
    LS_CUDA_TRY(cudaMemcpyFromSymbol(&err, g_tc_err, sizeof(err)));
    if (err) {
      const unsigned zero = 0;
      LS_CUDA_TRY(cudaMemcpyToSymbol(g_tc_err, &zero, sizeof(zero)));
      return LIBSHALOM_ERR_DEVICE_TIMEOUT;
    }
  }
  return LIBSHALOM_SUCCESS;
}

void plan_tiles(TcProblem &p) {
  if (p.M <= 64 && p.N <= 64) {
    // block-diagonal packing of whole GEMMs into one 128-row tile
    const int g_rows = TC_BM / p.M;
    const int g_cols = TC_MAX_N / p.N;
    p.G = std::max(1, std::min(g_rows, g_cols));
    p.tile_n = std::min(TC_MAX_N, (int)cdiv((long)p.G * p.N, 16) * 16);
    p.tiles_m = p.tiles_n = 1;
    p.num_tiles = cdiv(p.count, p.G);
  } else {
    p.G = 1;
    p.tile_n = std::min(TC_MAX_N, (int)cdiv(p.N, 16) * 16);
    p.tiles_m = (int)cdiv(p.M, TC_BM);
    p.tiles_n = (int)cdiv(p.N, p.tile_n);
    p.num_tiles = (long)p.tiles_m * p.tiles_n * p.count;
  }
  p.nk = (int)std::max(1L, cdiv(p.K, TC_BK));
  p.kc_slabs = 128 / TC_BK;  // TMEM accumulation chunk: 128 values of K
}

}  // namespace

static bool tc_mode_ok(int mode) {
  return mode == LIBSHALOM_PREC_BF16X3 || mode == LIBSHALOM_PREC_BF16X6;
}

int tc_sgemm_strided(const GemmArgs<float> &g, long sA, long sB, long sC, long count,
                     int mode) {
  if (!tc_mode_ok(mode)) return LIBSHALOM_ERR_INVALID_VALUE;
  if (g.transa) return LIBSHALOM_ERR_UNSUPPORTED;
  if (g.M > (1L << 30) || g.N > (1L << 30) || g.K > (1L << 30) || g.lda > INT32_MAX ||
      g.ldb > INT32_MAX || g.ldc > INT32_MAX)
    return LIBSHALOM_ERR_UNSUPPORTED;
  TcProblem p{};
  p.A = g.A; p.B = g.B; p.C = g.C;
  p.sA = sA; p.sB = sB; p.sC = sC;
  p.M = (int)g.M; p.N = (int)g.N; p.K = (int)g.K;
  p.lda = (int)g.lda; p.ldb = (int)g.ldb; p.ldc = (int)g.ldc;
  p.transb = g.transb;
  p.alpha = g.alpha; p.beta = g.beta;
  p.count = count;
  plan_tiles(p);
  p.vec_a = aligned16(g.A) && g.lda % 4 == 0 && sA % 4 == 0;
  p.vec_b = aligned16(g.B) && g.ldb % 4 == 0 && sB % 4 == 0 &&
            (g.transb || p.G == 1 || g.N % 4 == 0);
  p.vec_c = aligned16(g.C) && g.ldc % 4 == 0 && sC % 4 == 0;
  return tc_launch(p, mode);
}

// Split factor for one GEMM on the tensor cores: K is cut into s slices of
// equal length (s divides K / 32, slices of at least 64 k) when the output
// tiles alone cannot fill the machine.  forced > 1 asks for about that many.
static int tc_pick_splits(const GemmArgs<float> &g, int forced) {
  if (forced == 1 || g.K % TC_BK || g.K < 2 * TC_BK) return 1;
  const long q = g.K / TC_BK;
  const int tn = (int)std::min<long>(TC_MAX_N, cdiv(g.N, 16) * 16);
  const long tiles = cdiv(g.M, TC_BM) * cdiv(g.N, tn);
  const int sms = state().num_sms;
  long want = forced > 1 ? forced : (tiles >= sms ? 1 : (2L * sms) / tiles);
  want = std::min(want, q / 2);  // every slice keeps at least 2 slabs
  for (long d = want; d > 1; --d)
    if (q % d == 0) return (int)d;
  return 1;
}

int tc_sgemm_single(const GemmArgs<float> &g, int mode, int splits, int *used) {
  if (!tc_mode_ok(mode)) return LIBSHALOM_ERR_INVALID_VALUE;
  const int s = g.transa ? 1 : tc_pick_splits(g, splits);
  if (used) *used = s;
  if (s <= 1) return tc_sgemm_strided(g, 0, 0, 0, 1, mode);
  // K slices as a batch of s partial products into the workspace, then an
  // ordered reduction C = alpha * sum_z partial_z + beta * C
  void *ws = nullptr;
  int rc = workspace(sizeof(float) * (size_t)s * g.M * g.N, &ws);
  if (rc) return rc;
  float *partial = static_cast<float *>(ws);
  TcProblem p{};
  p.A = g.A; p.B = g.B; p.C = partial;
  p.sA = 0; p.sB = 0; p.sC = g.M * g.N;
  p.M = (int)g.M; p.N = (int)g.N; p.K = (int)g.K;
  p.lda = (int)g.lda; p.ldb = (int)g.ldb; p.ldc = (int)g.N;
  p.transb = g.transb;
  p.alpha = 1.0f; p.beta = 0.0f;
  p.count = s;
  p.G = 1;
  p.tile_n = std::min(TC_MAX_N, (int)cdiv(p.N, 16) * 16);
  p.tiles_m = (int)cdiv(p.M, TC_BM);
  p.tiles_n = (int)cdiv(p.N, p.tile_n);
  p.num_tiles = (long)p.tiles_m * p.tiles_n * s;
  p.kslice = p.K / s;
  p.nk = p.kslice / TC_BK;
  p.kc_slabs = 128 / TC_BK;
  // the TMA kernel when the operands allow it, else the cp.async kernel
  p.vec_a = aligned16(g.A) && g.lda % 4 == 0;
  p.vec_b = aligned16(g.B) && g.ldb % 4 == 0;
  p.vec_c = p.N % 4 == 0;  // partials: aligned workspace, rows of N floats
  rc = tc_launch(p, mode);
  if (rc) return rc;
  return run_splitk_reduce_f32(partial, s, g.M, g.N, g.C, g.ldc, g.alpha, g.beta);
}

int tc_wait_expiry_selftest(int iterations) {
  State &st = state();
  void *errp = nullptr;
  LS_CUDA_TRY(cudaGetSymbolAddress(&errp, g_tc_err));
  LS_CUDA_TRY(cudaStreamSynchronize(st.stream));  // no other kernel may own the word
  LS_CUDA_TRY(cudaMemsetAsync(errp, 0, sizeof(unsigned), st.stream));
  const uint32_t limit = iterations > 0 ? (uint32_t)std::min(iterations, 1 << 22) : 4096u;
  k_wait_expiry<<<1, 64, 0, st.stream>>>(limit, reinterpret_cast<unsigned *>(errp));
  LS_CUDA_TRY(cudaGetLastError());
  LS_CUDA_TRY(cudaStreamSynchronize(st.stream));
  unsigned err = 0;
  LS_CUDA_TRY(cudaMemcpyFromSymbol(&err, g_tc_err, sizeof(err)));
  const unsigned zero = 0;
  LS_CUDA_TRY(cudaMemcpyToSymbol(g_tc_err, &zero, sizeof(zero)));
  return err ? LIBSHALOM_ERR_DEVICE_TIMEOUT : LIBSHALOM_SUCCESS;
}

int tc_sgemm_grouped(const LibShalom_sgemm_entry *entries, long count, int mode) {
  if (!tc_mode_ok(mode)) return LIBSHALOM_ERR_INVALID_VALUE;
  if (count > (1L << 30)) return LIBSHALOM_ERR_UNSUPPORTED;
  State &st = state();
  // plan workspace: 256-word header (class tables, run count), then two
  // arrays sized by the entry count
  const size_t words = 256 + 2 * (size_t)count;
  void *ws = nullptr;
  int rc = workspace(words * sizeof(unsigned), &ws);
  if (rc) return rc;
  unsigned *w = static_cast<unsigned *>(ws);
  GrpPlan pl;
  pl.class_runs = w;
  pl.class_off = w + GRP_CLASSES;
  pl.class_fill = w + 2 * GRP_CLASSES;
  pl.n_runs = w + 3 * GRP_CLASSES;
  pl.run_first = w + 256;
  pl.run_len = pl.run_first + count;
  LS_CUDA_TRY(cudaMemsetAsync(w, 0, 256 * sizeof(unsigned), st.stream));
  const int pgrid = (int)std::max(1L, std::min(cdiv(count, 256), (long)st.num_sms * 8));
  k_grp_count<<<pgrid, 256, 0, st.stream>>>(entries, count, pl);
  k_grp_offsets<<<1, 32, 0, st.stream>>>(pl);
  k_grp_place<<<pgrid, 256, 0, st.stream>>>(entries, count, pl);
  LS_CUDA_TRY(cudaGetLastError());

  void *errp = nullptr;
  LS_CUDA_TRY(cudaGetSymbolAddress(&errp, g_tc_err));
  GrpArgs g;
  g.entries = entries;
  g.count = count;
  g.run_first = pl.run_first;
  g.run_len = pl.run_len;
  g.n_runs = pl.n_runs;
  g.err = reinterpret_cast<unsigned *>(errp);
  g.kc_slabs = 128 / TC_BK;
  const void *kern = mode == LIBSHALOM_PREC_BF16X6 ? (const void *)k_tc_grouped<3>
                                                   : (const void *)k_tc_grouped<2>;
  (void)occupancy_of(kern, G_THREADS, G_SMEM, 1);  // raises the shared-memory limit
  const int grid = grid_for((long)st.num_sms, 1);
  void *args[] = {&g};
  LS_CUDA_TRY(cudaLaunchKernel(kern, dim3(grid), dim3(G_THREADS), args, G_SMEM, st.stream));
  LS_CUDA_TRY(cudaGetLastError());
  if (st.sync) {
    unsigned err = 0;
    LS_CUDA_TRY(cudaStreamSynchronize(st.stream));
    LS_CUDA_TRY(cudaMemcpyFromSymbol(&err, g_tc_err, sizeof(err)));
    if (err) {
      const unsigned zero = 0;
      LS_CUDA_TRY(cudaMemcpyToSymbol(g_tc_err, &zero, sizeof(zero)));
      return LIBSHALOM_ERR_DEVICE_TIMEOUT;
    }
  }
  return LIBSHALOM_SUCCESS;
}

}  // namespace ls
