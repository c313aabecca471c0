// ls_dgemm_dmma.cu -- grouped FP64 GEMM on the FP64 tensor cores
// (LibShalom_dgemm_batched / _dgemm_stack with LIBSHALOM_DGEMM_DMMA).
//
// Work unit: one run (maximal group of consecutive entries naming the same C)
// whose C block fits a 32 x 32 warp tile.  One warp owns a run from its first
// product to its last: the C block lives in the warp's registers as DMMA
// accumulator fragments, so runs need no atomics and the result does not
// depend on scheduling.  Runs are ordered heaviest first (counting sort on
// their operand volume) and dealt round-robin to the warps of the grid.
//
// Staging: each warp owns a byte ring in shared memory fed by bulk copies
// (cp.async.bulk, completion counted on one of DM_NB mbarriers).  A product
// is cut into pieces of at most 32 k; a piece's operands -- and, in the first
// piece of a run, the C block -- are each copied as the 16-byte aligned
// window around a contiguous range (one copy) or, for padded leading
// dimensions, as one window per row (one copy per row, issued by the lanes
// in parallel).  The warp keeps up to DM_NB pieces in flight and issues more
// whenever the ring has room, so HBM sees several products per warp ahead of
// the one being multiplied.  Only 16-byte blocks that hold at least one
// element are read.
//
// Arithmetic: mma.sync.m8n8k4 FP64 (tcgen05 has no FP64 kind), only over the
// ceil(M/8) x ceil(N/8) fragments a run's C block covers; k is padded to a
// multiple of 4 with zeros.  Product i of a run computes
// C = beta_i C + (alpha_i A_i) op(B_i) with FP64 accumulation.
#include <cuda_runtime.h>

#include <algorithm>

#include "ls_common.cuh"
#include "ls_simt_launch.h"

namespace ls {

namespace {

constexpr int DM_WARPS = 8;         // warps per CTA (one run each at a time)
constexpr int DM_RING = 26624;      // staging ring bytes per warp (>= the largest piece)
constexpr int DM_NB = 6;            // pieces in flight per warp (one mbarrier each)
constexpr int DM_MAXK = 32;         // k per piece
constexpr int DM_CLASSES = 64;      // run cost classes of the heaviest-first order

enum : int {
  DF_FIRST_OF_PRODUCT = 1,  // apply the product's beta before its k loop
  DF_LOAD_C = 2,            // first piece of a run: the C block is staged too
  DF_LAST_OF_RUN = 4,       // store C after this piece
  DF_TRANSB = 8,            // B stored N x K
  DF_ALPHA = 16,            // alpha != 1: scale A as it is read
};

// A staged matrix: element (r, c) at double index off + r*step + ((sh + r*par) & 1) + c
// of the ring (flat window: step = source ld, par = 0; row windows: step =
// pitch in doubles, par = source ld & 1)
struct SMat {
  int off, step, sh, par;
  __device__ __forceinline__ int idx(int r) const { return off + r * step + ((sh + r * par) & 1); }
};

struct __align__(16) DmPiece {
  double alpha, beta;
  double *C;
  int M, N, kc, flags;
  SMat a, b, c;
  int ldc;
  unsigned end;  // ring position (monotonic byte count) after this piece
};
static_assert(sizeof(DmPiece) % 16 == 0, "piece records stay 16-byte aligned");

constexpr int DM_DESC_OFF = DM_RING;
constexpr int DM_BAR_OFF = DM_DESC_OFF + DM_NB * (int)sizeof(DmPiece);
constexpr int DM_WARP_BYTES = (DM_BAR_OFF + DM_NB * 8 + 127) & ~127;
constexpr int DM_SMEM = DM_WARPS * DM_WARP_BYTES;
static_assert(DM_SMEM <= 232448, "per-CTA shared memory");
// the largest piece: A, B and C of 32 x 32 as row windows of 272 bytes
static_assert(DM_RING >= 3 * 32 * 272, "one piece always fits the ring");

struct DmPlan {
  unsigned *n_small, *n_large;
  unsigned *class_runs, *class_off, *class_fill;  // [DM_CLASSES] each
  unsigned *small_first, *small_len;
  unsigned *large_first, *large_len;
};

__device__ __forceinline__ bool dm_run_start(const LibShalom_dgemm_entry *e, long i) {
  return i == 0 || e[i].C != e[i - 1].C;
}

// run starting at entry i: length, whether its C block fits a warp tile, and
// its cost class (operand doubles / 256, capped)
__device__ __forceinline__ void dm_run_info(const LibShalom_dgemm_entry *e, long count, long i,
                                            long *len, bool *small, int *cls) {
  const int M = e[i].M, N = e[i].N;
  long cost = (long)M * N, j = i;
  do {
    const long K = max(0, e[j].K);
    cost += K * (M + N);
    ++j;
  } while (j < count && e[j].C == e[i].C);
  *len = j - i;
  *small = M <= 32 && N <= 32;
  *cls = (int)min(cost / 256, (long)DM_CLASSES - 1);
}

__global__ void k_dm_count(const LibShalom_dgemm_entry *e, long count, DmPlan pl) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count;
       i += (long)gridDim.x * blockDim.x) {
    if (!dm_run_start(e, i)) continue;
    long len;
    bool small;
    int cls;
    dm_run_info(e, count, i, &len, &small, &cls);
    if (small) {
      atomicAdd(&pl.class_runs[cls], 1u);
    } else {
      const unsigned slot = atomicAdd(pl.n_large, 1u);
      pl.large_first[slot] = (unsigned)i;
      pl.large_len[slot] = (unsigned)len;
    }
  }
}

__global__ void k_dm_offsets(DmPlan pl) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    unsigned acc = 0;
    for (int c = DM_CLASSES - 1; c >= 0; --c) {
      pl.class_off[c] = acc;
      acc += pl.class_runs[c];
    }
    *pl.n_small = acc;
  }
}

__global__ void k_dm_place(const LibShalom_dgemm_entry *e, long count, DmPlan pl) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count;
       i += (long)gridDim.x * blockDim.x) {
    if (!dm_run_start(e, i)) continue;
    long len;
    bool small;
    int cls;
    dm_run_info(e, count, i, &len, &small, &cls);
    if (!small) continue;
    const unsigned slot = pl.class_off[cls] + atomicAdd(&pl.class_fill[cls], 1u);
    pl.small_first[slot] = (unsigned)i;
    pl.small_len[slot] = (unsigned)len;
  }
}

// ---- PTX helpers ----
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void *src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
// bounded wait for a phase (about a second with back-off)
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(it < 4096 ? 32 : 256);
  }
  return false;
}
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Ring bytes of a staged matrix of `rows` segments of `cols` doubles (row r at
// p + r*ld), its layout, and the bytes its copies move (*tx; smaller than the
// ring bytes for row windows whose start is 16-byte aligned).  Flat (one
// window) when the segments form one range.
__device__ __forceinline__ int stage_plan(const double *p, int rows, int cols, int ld, SMat &m,
                                          bool &flat, int *tx) {
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(p);
  m.sh = (int)((a0 >> 3) & 1);
  if (rows <= 0 || cols <= 0) {
    flat = true;
    m.step = 0; m.par = 0;
    *tx = 0;
    return 0;
  }
  flat = ld == cols || rows == 1;
  if (flat) {
    m.step = ld;
    m.par = 0;
    const uintptr_t w0 = a0 & ~uintptr_t(15);
    const uintptr_t end = a0 + 8 * ((uintptr_t)(rows - 1) * ld + cols);
    *tx = (int)(((end - w0 + 15) >> 4) << 4);
    return *tx;
  }
  // row r starts (sh + r ld) & 1 doubles into its window of 16 ceil((8 cols +
  // 8 sh_r) / 16) bytes
  const int pitch = 16 * ((8 * cols + 8 + 15) / 16);
  m.step = pitch / 8;
  m.par = ld & 1;
  const int odd = m.par ? (m.sh ? (rows + 1) / 2 : rows / 2) : (m.sh ? rows : 0);
  const int w_even = 16 * ((8 * cols + 15) / 16), w_odd = 16 * ((8 * cols + 8 + 15) / 16);
  *tx = (rows - odd) * w_even + odd * w_odd;
  return rows * pitch;
}

// Issues the copies of a staged matrix into ring byte offset `dst_off`
// (16-byte aligned): a flat window by lane 0, row windows by all lanes.
__device__ __forceinline__ void stage_issue(uint32_t ring, int dst_off, const double *p, int rows,
                                            int cols, int ld, bool flat, int step, uint32_t bar,
                                            int lane) {
  if (rows <= 0 || cols <= 0) return;
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(p);
  if (flat) {
    if (lane != 0) return;
    const uintptr_t w0 = a0 & ~uintptr_t(15);
    const uintptr_t end = a0 + 8 * ((uintptr_t)(rows - 1) * ld + cols);
    bulk_copy(ring + dst_off, reinterpret_cast<const void *>(w0),
              (uint32_t)(((end - w0 + 15) >> 4) << 4), bar);
    return;
  }
  for (int r = lane; r < rows; r += 32) {
    const uintptr_t a = a0 + 8 * (uintptr_t)r * ld;
    const uintptr_t w = a & ~uintptr_t(15);
    const uint32_t bytes = (uint32_t)(((a + 8 * (uintptr_t)cols - w + 15) >> 4) << 4);
    bulk_copy(ring + dst_off + r * step * 8, reinterpret_cast<const void *>(w), bytes, bar);
  }
}

// entry fields of one product (held by lane j for product base + j)
struct DmEnt {
  const double *A, *B;
  int K, lda, ldb, transb;
  double alpha, beta;
};

__device__ __forceinline__ DmEnt load_ent(const LibShalom_dgemm_entry *e, int N) {
  DmEnt d;
  d.A = e->A; d.B = e->B;
  d.K = max(0, e->K);
  d.transb = e->transb;
  d.lda = e->lda > 0 ? e->lda : d.K;
  d.ldb = e->ldb > 0 ? e->ldb : (e->transb ? d.K : N);
  d.alpha = e->alpha; d.beta = e->beta;
  return d;
}

__device__ __forceinline__ DmEnt shfl_ent(const DmEnt &x, int src) {
  const unsigned F = 0xffffffffu;
  DmEnt d;
  d.A = reinterpret_cast<const double *>(
      __shfl_sync(F, reinterpret_cast<unsigned long long>(x.A), src));
  d.B = reinterpret_cast<const double *>(
      __shfl_sync(F, reinterpret_cast<unsigned long long>(x.B), src));
  d.K = __shfl_sync(F, x.K, src);
  d.lda = __shfl_sync(F, x.lda, src);
  d.ldb = __shfl_sync(F, x.ldb, src);
  d.transb = __shfl_sync(F, x.transb, src);
  d.alpha = __shfl_sync(F, x.alpha, src);
  d.beta = __shfl_sync(F, x.beta, src);
  return d;
}

// A run as the load side holds it: warp-uniform header, and in every lane the
// entry of one product of the current batch of 32.
struct DmRun {
  long slot;  // index in the sorted run list
  int first, len, M, N, ldc, base;  // len <= 0: no run
  double *C;
  DmEnt ent;
};

// Header of the run in list slot `slot` (len 0 past the list's end).
__device__ __forceinline__ void run_header(DmRun &r, long slot, long n_runs,
                                           const unsigned *run_first, const unsigned *run_len) {
  r.slot = slot;
  r.first = 0;
  r.len = 0;
  if (slot < n_runs) {
    r.first = (int)run_first[slot];
    r.len = (int)run_len[slot];
  }
}

// Loads the rest of a run whose header is known: its C block and, in lane j,
// the entry of product j.
__device__ __forceinline__ void run_body(DmRun &r, const LibShalom_dgemm_entry *entries,
                                         int lane) {
  if (r.len <= 0) return;
  const LibShalom_dgemm_entry *e0 = entries + r.first;
  r.M = e0->M;
  r.N = e0->N;
  r.C = e0->C;
  r.ldc = e0->ldc > 0 ? e0->ldc : r.N;
  r.base = 0;
  if (lane < r.len) r.ent = load_ent(entries + r.first + lane, r.N);
}

// The compute side of one piece: acc[mf][nf] holds C fragment (mf, nf).
template <bool TRANSB>
__device__ __forceinline__ void piece_dmma(double (&acc)[4][4][2], const double *ring,
                                           const DmPiece &pc, int lane) {
  const int g = lane >> 2, q = lane & 3;
  const int MF = (pc.M + 7) >> 3, NF = (pc.N + 7) >> 3;
  const bool scale = (pc.flags & DF_ALPHA) != 0;
  int ao[4], bo[4];
  bool ar[4], bc[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const int r = 8 * f + g;
    ar[f] = r < pc.M;
    ao[f] = ar[f] ? pc.a.idx(r) : 0;
    bc[f] = r < pc.N;
    bo[f] = (TRANSB && bc[f]) ? pc.b.idx(r) : 0;
  }
  for (int k0 = 0; k0 < pc.kc; k0 += 4) {
    const int k = k0 + q;
    const bool kin = k < pc.kc;
    const int bk = (!TRANSB && kin) ? pc.b.idx(k) : 0;
    double a[4], b[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      if (f < MF) {
        a[f] = (ar[f] && kin) ? ring[ao[f] + k] : 0.0;
        if (scale) a[f] *= pc.alpha;
      }
      if (f < NF) b[f] = (bc[f] && kin) ? ring[TRANSB ? bo[f] + k : bk + 8 * f + g] : 0.0;
    }
#pragma unroll
    for (int mf = 0; mf < 4; ++mf) {
      if (mf >= MF) break;
#pragma unroll
      for (int nf = 0; nf < 4; ++nf) {
        if (nf >= NF) break;
        dmma(acc[mf][nf][0], acc[mf][nf][1], a[mf], b[nf]);
      }
    }
  }
}

// device status word: a ring barrier that never completed
__device__ unsigned g_dm_err;

__global__ void __launch_bounds__(DM_WARPS * 32, 1)
    k_dgemm_dmma(const LibShalom_dgemm_entry *entries, const unsigned *n_runs_p,
                 const unsigned *run_first, const unsigned *run_len) {
  extern __shared__ __align__(128) unsigned char dsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *wsm = dsm + warp * DM_WARP_BYTES;
  const double *ringd = reinterpret_cast<const double *>(wsm);
  const uint32_t ring = smem_addr(wsm);
  DmPiece *desc = reinterpret_cast<DmPiece *>(wsm + DM_DESC_OFF);
  const uint32_t bars = smem_addr(wsm + DM_BAR_OFF);
  if (lane == 0) {
    for (int i = 0; i < DM_NB; ++i) bar_init(bars + 8 * i, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  const long n_runs = (long)*n_runs_p;
  const long stride = (long)gridDim.x * DM_WARPS;

  // Load side: the current run (entries in the lanes), the next one (loaded
  // a run ahead) and the header of the one after (loaded two runs ahead), so
  // that opening a run never waits for global memory.
  DmRun cur, nxt, hdr;
  run_header(cur, (long)blockIdx.x * DM_WARPS + warp, n_runs, run_first, run_len);
  run_header(nxt, cur.slot + stride, n_runs, run_first, run_len);
  run_header(hdr, nxt.slot + stride, n_runs, run_first, run_len);
  run_body(cur, entries, lane);
  run_body(nxt, entries, lane);
  int lp = 0, lk = 0;           // product of cur and k offset of the next piece
  unsigned head = 0, tail = 0;  // ring bytes allocated / released (monotonic)
  long issued = 0, done = 0;

  // Issues the next piece when a barrier and ring room are free; false when
  // there is nothing left to issue or no room yet (warp-uniform).
  auto issue = [&]() -> bool {
    if (cur.len <= 0) return false;
    const DmEnt e = shfl_ent(cur.ent, lp - cur.base);
    const int M = cur.M, N = cur.N;
    const int kc = max(0, min(DM_MAXK, e.K - lk));
    DmPiece pc;
    pc.M = M; pc.N = N; pc.kc = kc; pc.C = cur.C; pc.ldc = cur.ldc;
    pc.alpha = e.alpha; pc.beta = e.beta;
    const bool first = lp == 0 && lk == 0;
    const bool load_c = first && e.beta != 0.0;
    const double *pa = e.A + lk;
    const double *pb = e.transb ? e.B + lk : e.B + (long)lk * e.ldb;
    bool fa, fb, fc = true;
    int ta, tb, tc = 0;
    const int ba = stage_plan(pa, M, kc, e.lda, pc.a, fa, &ta);
    const int bb = e.transb ? stage_plan(pb, N, kc, e.ldb, pc.b, fb, &tb)
                            : stage_plan(pb, kc, N, e.ldb, pc.b, fb, &tb);
    const int bcb = load_c ? stage_plan(cur.C, M, N, cur.ldc, pc.c, fc, &tc) : 0;
    const int need = ba + bb + bcb;
    // contiguous room in the ring: an empty ring (nothing in flight)
    // restarts at offset 0; a piece that would straddle the ring's end
    // starts at its beginning
    if (issued == done) head = tail = 0;
    unsigned pos = head;
    const unsigned off0 = head % DM_RING;
    if (off0 + need > (unsigned)DM_RING) pos += DM_RING - off0;
    if (pos + need - tail > (unsigned)DM_RING) return false;
    const int base_off = (int)(pos % DM_RING);
    pc.a.off = base_off / 8;
    pc.b.off = (base_off + ba) / 8;
    pc.c.off = (base_off + ba + bb) / 8;
    pc.end = pos + need;
    // advance the load cursor (a product with K = 0 is one empty piece)
    int nlk = lk + max(kc, 1), nlp = lp;
    bool last_of_run = false;
    if (nlk >= e.K) {
      nlk = 0;
      last_of_run = ++nlp >= cur.len;
    }
    pc.flags = (lk == 0 ? DF_FIRST_OF_PRODUCT : 0) | (first ? DF_LOAD_C : 0) |
               (last_of_run ? DF_LAST_OF_RUN : 0) | (e.transb ? DF_TRANSB : 0) |
               (e.alpha != 1.0 ? DF_ALPHA : 0);
    const int slot = (int)(issued % DM_NB);
    const uint32_t bar = bars + 8 * slot;
    if (lane == 0) {
      desc[slot] = pc;
      bar_arrive_tx(bar, (uint32_t)(ta + tb + tc));  // announced before any copy lands
    }
    __syncwarp();
    // the ring bytes being refilled were last read through the generic proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    stage_issue(ring, base_off, pa, M, kc, e.lda, fa, pc.a.step, bar, lane);
    if (e.transb) stage_issue(ring, base_off + ba, pb, N, kc, e.ldb, fb, pc.b.step, bar, lane);
    else stage_issue(ring, base_off + ba, pb, kc, N, e.ldb, fb, pc.b.step, bar, lane);
    if (load_c)
      stage_issue(ring, base_off + ba + bb, cur.C, M, N, cur.ldc, fc, pc.c.step, bar, lane);
    head = pos + need;
    ++issued;
    lk = nlk;
    lp = nlp;
    if (last_of_run) {
      cur = nxt;
      nxt = hdr;
      run_body(nxt, entries, lane);
      run_header(hdr, nxt.slot + stride, n_runs, run_first, run_len);
      lp = 0;
    } else if (lk == 0 && lp - cur.base >= 32) {
      cur.base += 32;  // runs of more than 32 products: the next batch of entries
      if (lane < cur.len - cur.base) cur.ent = load_ent(entries + cur.first + cur.base + lane, cur.N);
    }
    return true;
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int g = lane >> 2, q = lane & 3;
  bool ok = true;
  for (;;) {
    while (issued - done < DM_NB && issue()) {
    }
    if (done == issued) {
      // an empty ring always takes the next piece, so work left here is a defect
      if (cur.len > 0) {
        ok = false;
        if (lane == 0) atomicOr(&g_dm_err, 2u);
      }
      break;
    }
    const int slot = (int)(done % DM_NB);
    if (!bar_wait(bars + 8 * slot, (uint32_t)((done / DM_NB) & 1))) {
      ok = false;
      if (lane == 0) atomicOr(&g_dm_err, 1u);
      break;
    }
    __syncwarp();
    const DmPiece pc = desc[slot];
    if (pc.flags & DF_LOAD_C) {
      // the run's C block (staged only when the first product reads it)
      const bool have_c = pc.beta != 0.0;
#pragma unroll
      for (int mf = 0; mf < 4; ++mf)
#pragma unroll
        for (int nf = 0; nf < 4; ++nf)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = 8 * mf + g, c = 8 * nf + 2 * q + h;
            acc[mf][nf][h] = (have_c && r < pc.M && c < pc.N) ? ringd[pc.c.idx(r) + c] : 0.0;
          }
    }
    if (pc.flags & DF_FIRST_OF_PRODUCT) {
      if (pc.beta == 0.0) {
#pragma unroll
        for (int mf = 0; mf < 4; ++mf)
#pragma unroll
          for (int nf = 0; nf < 4; ++nf) acc[mf][nf][0] = acc[mf][nf][1] = 0.0;
      } else if (pc.beta != 1.0) {
#pragma unroll
        for (int mf = 0; mf < 4; ++mf)
#pragma unroll
          for (int nf = 0; nf < 4; ++nf) {
            acc[mf][nf][0] *= pc.beta;
            acc[mf][nf][1] *= pc.beta;
          }
      }
    }
    if (pc.flags & DF_TRANSB) piece_dmma<true>(acc, ringd, pc, lane);
    else piece_dmma<false>(acc, ringd, pc, lane);
    if (pc.flags & DF_LAST_OF_RUN) {
#pragma unroll
      for (int mf = 0; mf < 4; ++mf)
#pragma unroll
        for (int nf = 0; nf < 4; ++nf)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = 8 * mf + g, c = 8 * nf + 2 * q + h;
            if (r < pc.M && c < pc.N) pc.C[(long)r * pc.ldc + c] = acc[mf][nf][h];
          }
    }
    // every lane's reads of this piece's ring bytes have been consumed
    __syncwarp();
    tail = pc.end;
    ++done;
  }
  if (!ok) {
    // copies still in flight land before the CTA's shared memory goes away
    for (long x = done; x < issued; ++x)
      bar_wait(bars + 8 * (int)(x % DM_NB), (uint32_t)((x / DM_NB) & 1));
  }
}

}  // namespace

int run_dgemm_dmma(const LibShalom_dgemm_entry *entries, long count) {
  State &st = state();
  if (count > (1L << 30)) return LIBSHALOM_ERR_UNSUPPORTED;
  void *ws = nullptr;
  const size_t words = 64 + 3 * DM_CLASSES + 4 * (size_t)count;
  int rc = workspace(words * sizeof(unsigned), &ws);
  if (rc) return rc;
  unsigned *w = static_cast<unsigned *>(ws);
  DmPlan pl;
  pl.n_small = w;
  pl.n_large = w + 1;
  pl.class_runs = w + 64;
  pl.class_off = pl.class_runs + DM_CLASSES;
  pl.class_fill = pl.class_off + DM_CLASSES;
  pl.small_first = pl.class_fill + DM_CLASSES;
  pl.small_len = pl.small_first + count;
  pl.large_first = pl.small_len + count;
  pl.large_len = pl.large_first + count;
  LS_CUDA_TRY(cudaMemsetAsync(w, 0, (64 + 3 * DM_CLASSES) * sizeof(unsigned), st.stream));
  const int pgrid = (int)std::max(1L, std::min(cdiv(count, 256), (long)st.num_sms * 8));
  k_dm_count<<<pgrid, 256, 0, st.stream>>>(entries, count, pl);
  k_dm_offsets<<<1, 32, 0, st.stream>>>(pl);
  k_dm_place<<<pgrid, 256, 0, st.stream>>>(entries, count, pl);
  LS_CUDA_TRY(cudaGetLastError());
  const void *kern = (const void *)k_dgemm_dmma;
  (void)occupancy_of(kern, DM_WARPS * 32, DM_SMEM, 1);  // raises the shared-memory limit
  const int grid = grid_for(cdiv(count, DM_WARPS), 1);
  k_dgemm_dmma<<<grid, DM_WARPS * 32, DM_SMEM, st.stream>>>(entries, pl.n_small, pl.small_first,
                                                           pl.small_len);
  LS_CUDA_TRY(cudaGetLastError());
  rc = run_dgemm_runs_list(entries, count, pl.n_large, pl.large_first, pl.large_len);
  if (rc || !st.sync) return rc;
  // synchronous mode: report an expired wait on a ring barrier
  unsigned err = 0;
  LS_CUDA_TRY(cudaStreamSynchronize(st.stream));
  LS_CUDA_TRY(cudaMemcpyFromSymbol(&err, g_dm_err, sizeof(err)));
  if (err) {
    const unsigned zero = 0;
    LS_CUDA_TRY(cudaMemcpyToSymbol(g_dm_err, &zero, sizeof(zero)));
    return LIBSHALOM_ERR_DEVICE_TIMEOUT;
  }
  return LIBSHALOM_SUCCESS;
}

}  // namespace ls
