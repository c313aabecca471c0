// ls_dgemm_warp.cu -- grouped FP64 GEMM on the tensor cores
// (LibShalom_dgemm_batched with LIBSHALOM_DGEMM_DMMA or LIBSHALOM_DGEMM_OZAKI).
//
// Work unit: one run (maximal group of consecutive entries naming the same C)
// whose C block fits one warp tile (M, N <= 32).  One warp owns the run: the
// C block lives in the warp's registers as tensor-core accumulator fragments
// from the run's first product to its last, so shared C blocks need no atomics
// and the result does not depend on scheduling.  Runs with M or N > 32 go to
// the CUDA-core tile kernel.
//
// Operand staging: every product is cut into K pieces (at most 32, fewer when
// A and op(B) of 32 would not fit a slot), and the warp copies each piece into
// one of three 8.5 KB per-warp slots, two pieces ahead of the one it
// multiplies (any leading dimension, any 8-byte alignment): an operand whose
// piece is one contiguous range (leading dimension equal to the row length)
// is copied as the 16-byte aligned window around that range by one bulk copy
// (cp.async.bulk, its bytes counted on the slot's mbarrier); otherwise every
// row segment is copied as its own window with 16-byte cp.async, at a pitch of
// 16 (len/2 + 1) bytes.  Data starts 0 or 1 doubles into a window (the
// address mod 16).  Waits on the slot barriers are bounded.  The description of every piece goes into a
// per-warp ring next to the slots, so the entries, run table and pointer
// arithmetic stay on the load side.
//
// Arithmetic:
//   DMMA   mma.sync m8n8k4 FP64 (the FP64 tensor-core instruction; tcgen05 has
//          no FP64 kind): C = beta C + (alpha A) op(B), accumulated in FP64.
//   OZAKI  Ozaki-scheme emulation: per piece, A's rows and op(B)'s columns
//          are scaled by powers of two (|x| < 2^e) and their fixed-point
//          images floor(|x| 2^(7S-e)) are cut into S signed 7-bit digits
//          (exact).  The digit products a_s b_t with s + t <= S + 1 run as INT8
//          tensor-core MMAs (mma.sync m16n8k32, exact INT32 sums per diagonal
//          s + t = d); the diagonals are combined in FP64 from the smallest
//          weight up (Horner in 2^-7) and scaled back by 2^(e_i + f_j - 14).
//          Error per element about (S + 4) 2^(-7S) K max|A_i.| max|B_.j| plus
//          the FP64 roundings of the combination; inputs must be finite.
#include <cuda_runtime.h>

#include <algorithm>

#include "ls_common.cuh"
#include "ls_simt_launch.h"

namespace ls {

namespace {

constexpr int DW_WARPS = 8;                // warps per CTA (one run each)
constexpr int DW_SLOTS = 3;                // staging slots per warp
constexpr int DW_SLOT_BYTES = 8704;        // a 32 x 32 C block as row windows (32 x 272 B)
constexpr int DW_MAXK = 32;                // K per piece

enum : int { PF_FIRST_OF_PRODUCT = 1, PF_LOAD_C = 2, PF_LAST_OF_RUN = 4 };

// one piece as the compute side sees it (in the per-warp ring)
struct __align__(16) DPiece {
  const double *A, *B;  // A and op(B) at the piece's first k
  double *C;
  double alpha, beta;
  int M, N, kc, lda, ldb, ldc, transb, flags;
  // staged layout of A (or of C in the C piece) and of B: B's byte offset in
  // the slot, and per operand flat (one window) or row windows, the distance
  // in doubles between row starts, and the source address's double parity
  int b_off, a_flat, a_step, a_sh0, b_flat, b_step, b_sh0, pad_;
};
// per warp: slots, piece ring, one mbarrier per slot
constexpr int DW_RING_OFF = DW_SLOTS * DW_SLOT_BYTES;
constexpr int DW_BAR_OFF = DW_RING_OFF + DW_SLOTS * (int)sizeof(DPiece);
constexpr int DW_WARP_BYTES = (DW_BAR_OFF + DW_SLOTS * 8 + 127) & ~127;  // slots stay 16-byte aligned
static_assert(DW_SLOT_BYTES % 16 == 0 && DW_WARP_BYTES % 16 == 0, "bulk-copy destinations");
constexpr int DW_SMEM = DW_WARPS * DW_WARP_BYTES;
static_assert(DW_SMEM <= 232448, "per-CTA shared memory");

struct DwPlan {
  unsigned *n_small, *n_large;
  unsigned *small_first, *small_len;
  unsigned *large_first, *large_len;
};

// runs whose C block fits a warp tile go to the small list
__global__ void k_dw_plan(const LibShalom_dgemm_entry *e, long count, DwPlan pl) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count;
       i += (long)gridDim.x * blockDim.x) {
    if (i > 0 && e[i].C == e[i - 1].C) continue;
    long j = i + 1;
    while (j < count && e[j].C == e[i].C) ++j;
    if (e[i].M <= 32 && e[i].N <= 32) {
      const unsigned slot = atomicAdd(pl.n_small, 1u);
      pl.small_first[slot] = (unsigned)i;
      pl.small_len[slot] = (unsigned)(j - i);
    } else {
      const unsigned slot = atomicAdd(pl.n_large, 1u);
      pl.large_first[slot] = (unsigned)i;
      pl.large_len[slot] = (unsigned)(j - i);
    }
  }
}

__device__ __forceinline__ void cp16(uint32_t saddr, uintptr_t g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Staged matrix of `rows` row segments of `len` doubles (row r at p + r*ld).
// Bytes a layout takes in a slot:
//   flat (one window over the whole range, for ld == len or a single row)
//   rows (one window per row at a pitch of 16 (len/2 + 1) bytes)
__device__ __forceinline__ bool can_flat(int rows, int len, int ld) { return ld == len || rows == 1; }
__device__ __forceinline__ int flat_bytes(int rows, int len, int ld) {
  return 16 * ((8 * ((rows - 1) * ld + len) + 8 + 15) / 16);
}
__device__ __forceinline__ int win_pitch(int len) { return 16 * (len / 2 + 1); }
__device__ __forceinline__ int stage_bytes(int rows, int len, int ld) {
  if (rows <= 0 || len <= 0) return 0;
  return can_flat(rows, len, ld) ? flat_bytes(rows, len, ld) : rows * win_pitch(len);
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy(uint32_t dst, uintptr_t src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void cp_async_arrive(uint32_t bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}

// copy the staged matrix into dst (only 16-byte blocks that hold at least one
// element are read): a contiguous one as a single bulk copy issued by lane 0
// (its bytes are added to the slot barrier's transaction count), row windows
// with 16-byte cp.async by all lanes; returns the layout fields
__device__ __forceinline__ void stage_mat(uint32_t dst, const double *p, int rows, int len, int ld,
                                      int lane, int &flat, int &step, int &sh0, uint32_t bar) {
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(p);
  sh0 = (int)((a0 >> 3) & 1);
  if (rows <= 0 || len <= 0) {
    flat = 1; step = ld;
    return;
  }
  if (can_flat(rows, len, ld)) {
    flat = 1; step = ld;
    const uintptr_t w0 = a0 & ~uintptr_t(15);
    const uintptr_t end = a0 + 8 * ((uintptr_t)(rows - 1) * ld + len);
    const uint32_t bytes = (uint32_t)(((end - w0 + 15) >> 4) << 4);
    if (lane == 0) {
      mbar_expect_tx(bar, bytes);
      bulk_copy(dst, w0, bytes, bar);
    }
    return;
  }
  flat = 0;
  const int cpr = len / 2 + 1, pitch = 16 * cpr;
  step = pitch / 8;
  const int per = 32 / cpr, lr = lane / cpr, lq = lane - lr * cpr;
  if (lr >= per) return;
  for (int r = lr; r < rows; r += per) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p + (long)r * ld);
    const uintptr_t w = (a & ~uintptr_t(15)) + 16 * lq;
    if (w < a + 8 * (uintptr_t)len) cp16(dst + r * pitch + 16 * lq, w);
  }
}

// a staged matrix as the compute side reads it
struct SView {
  const double *base;
  int flat, step, sh0, ld;
  // double index of row r's first element
  __device__ __forceinline__ int start(int r) const {
    return flat ? sh0 + r * ld : r * step + ((sh0 + r * ld) & 1);
  }
  __device__ __forceinline__ double at(int r, int c) const { return base[start(r) + c]; }
};

// entry fields a lane holds for one product of the current run
struct DEnt {
  const double *A, *B;
  int K, lda, ldb, transb;
  double alpha, beta;
};

// The load side of one warp: walks its runs (round-robin over all warps),
// issues the copies of one piece at a time into the slot ring and writes the
// piece description.  Lane l holds the entry of product (batch base + l) of
// the current run.
struct DLoader {
  const LibShalom_dgemm_entry *entries;
  const unsigned *run_first, *run_len;
  long n_runs, r;  // current run slot
  long stride;
  int first, len, M, N, ldc;
  double *C;
  int p, kc0, stage;  // product, K offset, 0 = C piece pending
  int base;           // first product held by the lanes
  DEnt ent;           // this lane's entry (product base + lane)
  bool done;

  __device__ void load_batch(int lane) {
    const int pi = base + lane;
    if (pi < len) {
      const LibShalom_dgemm_entry &e = entries[first + pi];
      ent.A = e.A; ent.B = e.B;
      ent.K = max(0, e.K);
      ent.transb = e.transb;
      ent.lda = e.lda > 0 ? e.lda : ent.K;
      ent.ldb = e.ldb > 0 ? e.ldb : (e.transb ? ent.K : N);
      ent.alpha = e.alpha; ent.beta = e.beta;
    }
  }
  // move to the first run at or after slot r with a non-empty C block
  __device__ void open_run(int lane) {
    for (; r < n_runs; r += stride) {
      first = (int)run_first[r];
      len = (int)run_len[r];
      const LibShalom_dgemm_entry &e0 = entries[first];
      M = e0.M; N = e0.N;
      if (M <= 0 || N <= 0 || len <= 0) continue;
      C = e0.C;
      ldc = e0.ldc > 0 ? e0.ldc : N;
      p = 0; kc0 = 0; stage = 0; base = 0;
      load_batch(lane);
      return;
    }
    done = true;
  }
  __device__ void init(const LibShalom_dgemm_entry *e, const unsigned *f, const unsigned *l,
                       long nr, long gw, long nw, int lane) {
    entries = e; run_first = f; run_len = l; n_runs = nr; r = gw; stride = nw; done = false;
    open_run(lane);
  }
  // write the next piece into ring slot `slot` and issue its copies; false
  // when the warp has no more pieces (warp-uniform)
  __device__ bool issue(unsigned char *wsm, int slot, int lane) {
    if (done) return false;
    unsigned char *sbuf = wsm + slot * DW_SLOT_BYTES;
    DPiece *ring = reinterpret_cast<DPiece *>(wsm + DW_RING_OFF);
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(sbuf);
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(wsm + DW_BAR_OFF + 8 * slot);
    DPiece pc;
    pc.M = M; pc.N = N; pc.C = C; pc.ldc = ldc;
    if (stage == 0) {
      // the run's C block
      pc.flags = PF_LOAD_C;
      pc.A = nullptr; pc.B = nullptr; pc.kc = 0; pc.lda = pc.ldb = 0; pc.transb = 0;
      pc.alpha = 1.0; pc.beta = 1.0;
      pc.b_off = 0; pc.b_flat = 1; pc.b_step = 0; pc.b_sh0 = 0;
      stage_mat(sa, C, M, N, ldc, lane, pc.a_flat, pc.a_step, pc.a_sh0, bar);
      stage = 1;
    } else {
      const int src = p - base;
      const unsigned FULL = 0xffffffffu;
      DEnt e;
      e.A = reinterpret_cast<const double *>(
          __shfl_sync(FULL, reinterpret_cast<unsigned long long>(ent.A), src));
      e.B = reinterpret_cast<const double *>(
          __shfl_sync(FULL, reinterpret_cast<unsigned long long>(ent.B), src));
      e.K = __shfl_sync(FULL, ent.K, src);
      e.lda = __shfl_sync(FULL, ent.lda, src);
      e.ldb = __shfl_sync(FULL, ent.ldb, src);
      e.transb = __shfl_sync(FULL, ent.transb, src);
      e.alpha = __shfl_sync(FULL, ent.alpha, src);
      e.beta = __shfl_sync(FULL, ent.beta, src);
      // the longest piece (<= 32) whose A and op(B) fit a slot
      int kc = max(0, min(DW_MAXK, e.K - kc0));
      auto bytes_of = [&](int k) {
        const int ba = (stage_bytes(M, k, e.lda) + 15) & ~15;
        return ba + (e.transb ? stage_bytes(N, k, e.ldb) : stage_bytes(k, N, e.ldb));
      };
      while (kc > 1 && bytes_of(kc) > DW_SLOT_BYTES) kc = kc > 4 ? (kc - 1) & ~3 : kc - 1;
      pc.flags = kc0 == 0 ? PF_FIRST_OF_PRODUCT : 0;
      pc.A = e.A + kc0;
      pc.B = e.transb ? e.B + kc0 : e.B + (long)kc0 * e.ldb;
      pc.kc = kc;
      pc.lda = e.lda; pc.ldb = e.ldb; pc.transb = e.transb;
      pc.alpha = e.alpha; pc.beta = e.beta;
      pc.b_off = (stage_bytes(M, kc, e.lda) + 15) & ~15;
      stage_mat(sa, pc.A, M, kc, pc.lda, lane, pc.a_flat, pc.a_step, pc.a_sh0, bar);
      if (e.transb)
        stage_mat(sa + pc.b_off, pc.B, N, kc, pc.ldb, lane, pc.b_flat, pc.b_step, pc.b_sh0, bar);
      else
        stage_mat(sa + pc.b_off, pc.B, kc, N, pc.ldb, lane, pc.b_flat, pc.b_step, pc.b_sh0, bar);
      // advance (a product with K = 0 is one empty piece)
      kc0 += max(kc, 1);
      if (kc0 >= e.K) {
        kc0 = 0;
        if (++p >= len) {
          pc.flags |= PF_LAST_OF_RUN;
          r += stride;
          open_run(lane);
        } else if (p - base >= 32) {
          base += 32;
          load_batch(lane);
        }
      }
    }
    if (lane == 0) ring[slot] = pc;
    // the slot's phase completes when every lane's cp.async copies and the
    // bulk copies' bytes have landed
    cp_async_arrive(bar);
    return true;
  }
};

// ---------------------------------------------------------------------------
// Arithmetic policies.  Both keep the C block as 32 doubles a thread; pos()
// maps an accumulator index to its (row, column) in the 32 x 32 block.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

struct ArithDmma {
  // fragments of 8 x 8: index (mf * 4 + nf) * 2 + h
  __device__ static void pos(int i, int lane, int &row, int &col) {
    const int mf = i >> 3, nf = (i >> 1) & 3, h = i & 1;
    row = 8 * mf + (lane >> 2);
    col = 8 * nf + 2 * (lane & 3) + h;
  }
  __device__ static void piece(double (&acc)[32], const DPiece &pc, const SView &A,
                               const SView &B, int lane) {
    const int gr = lane >> 2, gc = lane & 3;
    int sa[4], sb[4];  // row starts this thread reads
#pragma unroll
    for (int mf = 0; mf < 4; ++mf) {
      const int rr = 8 * mf + gr;
      sa[mf] = rr < pc.M ? A.start(rr) : 0;
    }
#pragma unroll
    for (int nf = 0; nf < 4; ++nf) {
      const int nn = 8 * nf + gr;
      sb[nf] = pc.transb && nn < pc.N ? B.start(nn) : 0;
    }
    const bool scale = pc.alpha != 1.0;
    for (int k0 = 0; k0 < pc.kc; k0 += 4) {
      const int k = k0 + gc;
      const int skb = (!pc.transb && k < pc.kc) ? B.start(k) : 0;
      double a[4], b[4];
#pragma unroll
      for (int mf = 0; mf < 4; ++mf) {
        const int rr = 8 * mf + gr;
        a[mf] = (rr < pc.M && k < pc.kc) ? A.base[sa[mf] + k] : 0.0;
        if (scale) a[mf] *= pc.alpha;
      }
#pragma unroll
      for (int nf = 0; nf < 4; ++nf) {
        const int nn = 8 * nf + gr;
        double v = 0.0;
        if (nn < pc.N && k < pc.kc)
          v = pc.transb ? B.base[sb[nf] + k] : B.base[skb + nn];
        b[nf] = v;
      }
      // all 16 fragments, branch-free: fragments past M / N multiply zeros
#pragma unroll
      for (int mf = 0; mf < 4; ++mf)
#pragma unroll
        for (int nf = 0; nf < 4; ++nf)
          dmma(acc[(mf * 4 + nf) * 2], acc[(mf * 4 + nf) * 2 + 1], a[mf], b[nf]);
    }
  }
};

__device__ __forceinline__ void imma(int (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                     uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// smallest e with m < 2^e (m >= 0 finite; 0 for m == 0)
__device__ __forceinline__ int exp_above(double m) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(m);
  if (bits == 0) return 0;
  const int be = (int)(bits >> 52);
  if (be != 0) return be - 1022;
  return (63 - __clzll((long long)bits)) - 1073;
}

// floor(|x| * 2^(s7 - e)) for |x| < 2^e: an integer below 2^s7 (s7 <= 63)
__device__ __forceinline__ unsigned long long fixed_point(double x, int e, int s7) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(x) & 0x7fffffffffffffffull;
  const int be = (int)(bits >> 52);
  unsigned long long mant = bits & 0xfffffffffffffull;
  int ex2 = -1074;
  if (be != 0) {
    mant |= 1ull << 52;
    ex2 = be - 1075;
  }
  const int sa = ex2 + s7 - e;
  if (sa >= 64 || sa <= -64) return 0;
  return sa >= 0 ? mant << sa : mant >> (-sa);
}

// the S signed 7-bit digits of x (most significant first) into byte `byte`
// of d[0..S-1]
template <int S>
__device__ __forceinline__ void put_digits(uint32_t (&d)[S], double x, int e, int byte) {
  const unsigned long long v = fixed_point(x, e, 7 * S);
  const bool neg = x < 0.0;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    int g = (int)((v >> (7 * (S - 1 - s))) & 127u);
    if (neg) g = -g;
    d[s] |= ((uint32_t)g & 0xffu) << (8 * byte);
  }
}

template <int S>
struct ArithOzaki {
  // fragments of 16 x 8: index (mt * 4 + nt) * 4 + q
  __device__ static void pos(int i, int lane, int &row, int &col) {
    const int mt = i >> 4, nt = (i >> 2) & 3, q = i & 3;
    row = 16 * mt + (lane >> 2) + 8 * (q >> 1);
    col = 8 * nt + 2 * (lane & 3) + (q & 1);
  }
  __device__ static double opb(const DPiece &pc, const SView &B, int k, int n) {
    return pc.transb ? B.at(n, k) : B.at(k, n);
  }
  __device__ static void piece(double (&acc)[32], const DPiece &pc, const SView &A,
                               const SView &B, int lane) {
    const unsigned FULL = 0xffffffffu;
    const int gid = lane >> 2, tig = lane & 3;
    // exponents: lane r for row r of A, lane j for column j of op(B)
    int ea = 0, eb = 0;
    if (lane < pc.M) {
      const int st = A.start(lane);
      double m = 0.0;
      for (int k = 0; k < pc.kc; ++k) m = fmax(m, fabs(A.base[st + k]));
      ea = exp_above(m);
    }
    if (lane < pc.N) {
      double m = 0.0;
      for (int k = 0; k < pc.kc; ++k) m = fmax(m, fabs(opb(pc, B, k, lane)));
      eb = exp_above(m);
    }
    int erow[2][2];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int h = 0; h < 2; ++h) erow[mt][h] = __shfl_sync(FULL, ea, 16 * mt + gid + 8 * h);
    const int MT = (pc.M + 15) >> 4, NT = (pc.N + 7) >> 3;
    // A digits: [mt][register][slice]
    uint32_t ad[2][4][S];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int rg = 0; rg < 4; ++rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) ad[mt][rg][s] = 0u;
        const int row = 16 * mt + gid + 8 * (rg & 1);
        const int kb = 4 * tig + 16 * (rg >> 1);
        if (mt < MT && row < pc.M) {
          const int st = A.start(row);
#pragma unroll 1
          for (int w = 0; w < 4; ++w) {
            const int k = kb + w;
            if (k < pc.kc) {
              put_digits<S>(ad[mt][rg], A.base[st + k], erow[mt][rg & 1], w);
            }
          }
        }
      }
    // Column tiles in a rolled loop: the body (45 digit MMAs per row tile at
    // 9 slices) is kept once in the instruction stream, which a 4-way unrolled
    // copy overflowed; the accumulator is written through a static select.
#pragma unroll 1
    for (int nt = 0; nt < NT; ++nt) {
      const int fb_nt = __shfl_sync(FULL, eb, 8 * nt + gid);
      int fcol_nt[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) fcol_nt[h] = __shfl_sync(FULL, eb, 8 * nt + 2 * tig + h);
      // B digits of this column tile: [register][slice]
      uint32_t bd[2][S];
      const int col = 8 * nt + gid;
#pragma unroll
      for (int rg = 0; rg < 2; ++rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) bd[rg][s] = 0u;
        if (col < pc.N) {
#pragma unroll 1
          for (int w = 0; w < 4; ++w) {
            const int k = 4 * tig + 16 * rg + w;
            if (k < pc.kc) {
              put_digits<S>(bd[rg], opb(pc, B, k, col), fb_nt, w);
            }
          }
        }
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        if (mt >= MT) continue;
        // sum over the diagonals s + t = d (slices numbered from 1), from the
        // smallest weight 2^-7(S+1) up: F = D_d + 2^-7 F
        double F[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int d = S + 1; d >= 2; --d) {
          int D[4] = {0, 0, 0, 0};
#pragma unroll
          for (int s = 1; s <= S; ++s) {
            const int t = d - s;
            if (t < 1 || t > S) continue;
            const uint32_t a4[4] = {ad[mt][0][s - 1], ad[mt][1][s - 1], ad[mt][2][s - 1],
                                    ad[mt][3][s - 1]};
            imma(D, a4, bd[0][t - 1], bd[1][t - 1]);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) F[q] = fma(F[q], 0.0078125, (double)D[q]);
        }
        // sum = 2^-14 F; element scale 2^(e_i + f_j)
        double pv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) pv[q] = ldexp(F[q], erow[mt][q >> 1] + fcol_nt[q & 1] - 14);
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
          if (n2 != nt) continue;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            double &c = acc[(mt * 4 + n2) * 4 + q];
            c = pc.alpha == 1.0 ? c + pv[q] : fma(pc.alpha, pv[q], c);
          }
        }
      }
    }
  }
};

// device status word: a slot barrier that never completed
__device__ unsigned g_dw_err;

// bounded wait for a phase of a slot barrier (about a second with back-off)
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  for (uint32_t it = 0; it < (1u << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(it < 4096 ? 32 : 256);
  }
  return false;
}

// ---------------------------------------------------------------------------
// The warp kernel: load side two pieces ahead, compute side per piece.
// ---------------------------------------------------------------------------
template <class Arith>
__global__ void __launch_bounds__(DW_WARPS * 32, 1)
    k_dgemm_tc(const LibShalom_dgemm_entry *entries, const unsigned *n_runs_p,
               const unsigned *run_first, const unsigned *run_len) {
  extern __shared__ __align__(16) unsigned char dsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *wsm = dsm + warp * DW_WARP_BYTES;
  const DPiece *ring = reinterpret_cast<const DPiece *>(wsm + DW_RING_OFF);
  uint64_t *bars = reinterpret_cast<uint64_t *>(wsm + DW_BAR_OFF);
  if (lane == 0) {
    for (int i = 0; i < DW_SLOTS; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 32;" ::"r"(
                       (uint32_t)__cvta_generic_to_shared(&bars[i]))
                   : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  const long n_runs = (long)*n_runs_p;
  DLoader ld;
  ld.init(entries, run_first, run_len, n_runs, (long)blockIdx.x * DW_WARPS + warp,
          (long)gridDim.x * DW_WARPS, lane);

  // prologue: two pieces in flight; piece i completes phase i / DW_SLOTS of
  // the barrier of slot i % DW_SLOTS
  long n_issued = 0;
  for (int s = 0; s < 2; ++s)
    if (ld.issue(wsm, s, lane)) ++n_issued;
  bool ok = true;
  double acc[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) acc[i] = 0.0;
  for (long i = 0; i < n_issued; ++i) {
    const int slot = (int)(i % DW_SLOTS);
    __syncwarp();  // every lane is done with the slot refilled next
    if (ld.issue(wsm, (int)((i + 2) % DW_SLOTS), lane)) ++n_issued;
    if (!bar_wait(&bars[slot], (uint32_t)((i / DW_SLOTS) & 1))) {
      ok = false;  // a copy never landed: stop, report, leave C alone
      if (lane == 0) atomicOr(&g_dw_err, 1u);
      break;
    }
    __syncwarp();
    const DPiece pc = ring[slot];
    const unsigned char *sbase = wsm + slot * DW_SLOT_BYTES;
    const SView A{reinterpret_cast<const double *>(sbase), pc.a_flat, pc.a_step, pc.a_sh0,
                  (pc.flags & PF_LOAD_C) ? pc.ldc : pc.lda};
    const SView B{reinterpret_cast<const double *>(sbase + pc.b_off), pc.b_flat, pc.b_step,
                  pc.b_sh0, pc.ldb};
    if (pc.flags & PF_LOAD_C) {
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        int row, col;
        Arith::pos(q, lane, row, col);
        acc[q] = (row < pc.M && col < pc.N) ? A.at(row, col) : 0.0;
      }
      continue;
    }
    if (pc.flags & PF_FIRST_OF_PRODUCT) {
      if (pc.beta == 0.0) {
#pragma unroll
        for (int q = 0; q < 32; ++q) acc[q] = 0.0;
      } else if (pc.beta != 1.0) {
#pragma unroll
        for (int q = 0; q < 32; ++q) acc[q] *= pc.beta;
      }
    }
    Arith::piece(acc, pc, A, B, lane);
    if (pc.flags & PF_LAST_OF_RUN) {
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        int row, col;
        Arith::pos(q, lane, row, col);
        if (row < pc.M && col < pc.N) pc.C[(long)row * pc.ldc + col] = acc[q];
      }
    }
  }
  if (!ok) {
    // copies still in flight land before the CTA's shared memory goes away
    for (long x = n_issued > DW_SLOTS ? n_issued - DW_SLOTS : 0; x < n_issued; ++x)
      bar_wait(&bars[x % DW_SLOTS], (uint32_t)((x / DW_SLOTS) & 1));
  }
  cp_wait<0>();
}

template <class Arith>
int launch_tc(const LibShalom_dgemm_entry *entries, long count, const DwPlan &pl) {
  State &st = state();
  const void *kern = (const void *)k_dgemm_tc<Arith>;
  (void)occupancy_of(kern, DW_WARPS * 32, DW_SMEM, 1);  // raises the shared-memory limit
  const int grid = grid_for(cdiv(count, DW_WARPS), 1);
  k_dgemm_tc<Arith><<<grid, DW_WARPS * 32, DW_SMEM, st.stream>>>(entries, pl.n_small,
                                                                 pl.small_first, pl.small_len);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

}  // namespace

// Grouped FP64 batch on the tensor cores: runs with M, N <= 32 through the
// warp kernel, the others through the CUDA-core tile kernel.  Workspace: two
// run counts + four arrays sized by the entry count.
int run_dgemm_warp(const LibShalom_dgemm_entry *entries, long count, int method, int slices) {
  if (method == LIBSHALOM_DGEMM_DMMA) return run_dgemm_dmma(entries, count);
  State &st = state();
  if (count > (1L << 30)) return LIBSHALOM_ERR_UNSUPPORTED;
  void *ws = nullptr;
  int rc = workspace((64 + 4 * (size_t)count) * sizeof(unsigned), &ws);
  if (rc) return rc;
  unsigned *w = static_cast<unsigned *>(ws);
  DwPlan pl{w, w + 1, w + 64, w + 64 + count, w + 64 + 2 * count, w + 64 + 3 * count};
  LS_CUDA_TRY(cudaMemsetAsync(w, 0, 2 * sizeof(unsigned), st.stream));
  const int pgrid = (int)std::max(1L, std::min(cdiv(count, 256), (long)st.num_sms * 8));
  k_dw_plan<<<pgrid, 256, 0, st.stream>>>(entries, count, pl);
  LS_CUDA_TRY(cudaGetLastError());
  if (method == LIBSHALOM_DGEMM_DMMA) {
    rc = launch_tc<ArithDmma>(entries, count, pl);
  } else {
    switch (slices) {
      case 4: rc = launch_tc<ArithOzaki<4>>(entries, count, pl); break;
      case 5: rc = launch_tc<ArithOzaki<5>>(entries, count, pl); break;
      case 6: rc = launch_tc<ArithOzaki<6>>(entries, count, pl); break;
      case 7: rc = launch_tc<ArithOzaki<7>>(entries, count, pl); break;
      case 8: rc = launch_tc<ArithOzaki<8>>(entries, count, pl); break;
      case 9: rc = launch_tc<ArithOzaki<9>>(entries, count, pl); break;
      default: return LIBSHALOM_ERR_INVALID_VALUE;
    }
  }
  if (rc) return rc;
  rc = run_dgemm_runs_list(entries, count, pl.n_large, pl.large_first, pl.large_len);
  if (rc || !st.sync) return rc;
  // synchronous mode: report an expired wait on a staging barrier
  unsigned err = 0;
  LS_CUDA_TRY(cudaStreamSynchronize(st.stream));
  LS_CUDA_TRY(cudaMemcpyFromSymbol(&err, g_dw_err, sizeof(err)));
  if (err) {
    const unsigned zero = 0;
    LS_CUDA_TRY(cudaMemcpyToSymbol(g_dw_err, &zero, sizeof(zero)));
    return LIBSHALOM_ERR_DEVICE_TIMEOUT;
  }
  return LIBSHALOM_SUCCESS;
}

}  // namespace ls
