// ls_simt.cu -- plain FP32 / FP64 kernels and their launchers: single GEMM
// (LibShalom_sgemm / _sgemm_mp / _dgemm), split-K reduction, uniform and
// grouped batches.
#include <algorithm>
#include <cmath>

#include "ls_common.cuh"
#include "ls_simt.cuh"
#include "ls_simt_launch.h"

namespace ls {

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// Single GEMM, persistent over work items (tile_m, tile_n, k-slice).
// splits == 1: the tile is written to C with alpha/beta.
// splits > 1: slice z writes its partial to partial[z][M][N].
template <typename T, class Cfg, int KBLOCK, bool TA, bool TB>
__global__ void __launch_bounds__(Cfg::NTH)
k_gemm_single(GemmArgs<T> g, int tiles_m, int tiles_n, int ways_m, int ways_n,
              int splits, long kchunk, T *partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *smem = reinterpret_cast<T *>(smem_raw);
  // Work item -> (k slice z, tile row tm, tile column tn).  Without a ways
  // partition a work item is one tile.  With LibShalom_set_thread_ways the
  // tile grid is cut into ways_m x ways_n rectangular groups and a work item
  // is one group: the CTA that takes it walks all of the group's tiles.
  const bool grouped = ways_m > 0;
  const int gm = grouped ? (tiles_m + ways_m - 1) / ways_m : 1;
  const int gn = grouped ? (tiles_n + ways_n - 1) / ways_n : 1;
  const long units = grouped ? (long)ways_m * ways_n : (long)tiles_m * tiles_n;
  const int per_unit = gm * gn;
  for (long w = blockIdx.x; w < units * splits; w += gridDim.x) {
    const int z = (int)(w / units);
    const long u = w % units;
    for (int q = 0; q < per_unit; ++q) {
      int tm, tn;
      if (grouped) {
        tm = (int)(u / ways_n) * gm + q / gn;
        tn = (int)(u % ways_n) * gn + q % gn;
        if (tm >= tiles_m || tn >= tiles_n) continue;
      } else {
        tm = (int)(u / tiles_n);
        tn = (int)(u % tiles_n);
      }
      const long kb = (long)z * kchunk;
      const long ke = min(g.K, kb + kchunk);
      T *out = splits == 1 ? g.C : partial + (long)z * g.M * g.N;
      const long ldo = splits == 1 ? g.ldc : g.N;
      const T alpha = splits == 1 ? g.alpha : T(1);
      const T beta = splits == 1 ? g.beta : T(0);
      simt_tile<T, Cfg, KBLOCK, TA, TB>(g, (long)tm * Cfg::BM, (long)tn * Cfg::BN, kb, ke, out,
                                        ldo, alpha, beta, smem);
    }
  }
}

// C = alpha * sum_z partial[z] + beta * C, slices summed in order z = 0, 1, ...
template <typename T>
__global__ void k_splitk_reduce(const T *partial, int splits, long M, long N,
                                T *C, long ldc, T alpha, T beta) {
  const long total = M * N;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    T s = partial[e];
    for (int z = 1; z < splits; ++z) s = s + partial[(long)z * total + e];
    const long i = e / N, j = e % N;
    T *dst = C + i * ldc + j;
    T v = alpha * s;
    if (beta != T(0)) v = fma_t(beta, *dst, v);
    *dst = v;
  }
}

// Uniform batch: work item = (gemm, tile).
template <typename T, class Cfg, bool TB>
__global__ void __launch_bounds__(Cfg::NTH)
k_gemm_strided(GemmArgs<T> g, long sA, long sB, long sC, long count,
               int tiles_m, int tiles_n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *smem = reinterpret_cast<T *>(smem_raw);
  const long tiles = (long)tiles_m * tiles_n;
  const long items = tiles * count;
  for (long w = blockIdx.x; w < items; w += gridDim.x) {
    const long b = w / tiles, t = w % tiles;
    GemmArgs<T> h = g;
    h.A = g.A + b * sA;
    h.B = g.B + b * sB;
    h.C = g.C + b * sC;
    simt_tile<T, Cfg, 0, false, TB>(h, (t / tiles_n) * Cfg::BM, (t % tiles_n) * Cfg::BN, 0, h.K,
                                    h.C, h.ldc, h.alpha, h.beta, smem);
  }
}

template <typename T> struct EntryOf;
template <> struct EntryOf<float> { using type = LibShalom_sgemm_entry; };
template <> struct EntryOf<double> { using type = LibShalom_dgemm_entry; };

// Grouped batch.  Work unit = a run of consecutive entries naming the same C
// (a single entry is a run of one).  CTAs take entry indices from an atomic
// counter; an index that continues a run is skipped (its run's owner
// processes it), so every C block is owned by exactly one CTA and the
// products of a run are applied in array order.
template <typename T, class Cfg>
__global__ void __launch_bounds__(Cfg::NTH)
k_gemm_grouped(const typename EntryOf<T>::type *entries, long count,
               unsigned long long *counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *smem = reinterpret_cast<T *>(smem_raw);
  __shared__ long s_idx;
  for (;;) {
    if (threadIdx.x == 0) {
      long i = (long)atomicAdd(counter, 1ULL);
      // skip indices that continue a run
      while (i < count && i > 0 && entries[i].C == entries[i - 1].C)
        i = (long)atomicAdd(counter, 1ULL);
      s_idx = i;
    }
    __syncthreads();
    const long first = s_idx;
    __syncthreads();
    if (first >= count) break;
    long last = first + 1;
    while (last < count && entries[last].C == entries[first].C) ++last;

    const auto &e0 = entries[first];
    const int tiles_m = (e0.M + Cfg::BM - 1) / Cfg::BM;
    const int tiles_n = (e0.N + Cfg::BN - 1) / Cfg::BN;
    for (int t = 0; t < tiles_m * tiles_n; ++t) {
      for (long p = first; p < last; ++p) {
        const auto &e = entries[p];
        GemmArgs<T> h;
        h.A = e.A; h.B = e.B; h.C = e.C;
        h.M = e.M; h.N = e.N; h.K = e.K;
        h.transa = 0; h.transb = e.transb;
        h.lda = e.lda > 0 ? e.lda : e.K;
        h.ldb = e.ldb > 0 ? e.ldb : (e.transb ? e.K : e.N);
        h.ldc = e.ldc > 0 ? e.ldc : e.N;
        h.alpha = (T)e.alpha; h.beta = (T)e.beta;
        if (h.transb)
          simt_tile<T, Cfg, 0, false, true>(h, (long)(t / tiles_n) * Cfg::BM,
                                            (long)(t % tiles_n) * Cfg::BN, 0, h.K, h.C, h.ldc,
                                            h.alpha, h.beta, smem);
        else
          simt_tile<T, Cfg, 0, false, false>(h, (long)(t / tiles_n) * Cfg::BM,
                                             (long)(t % tiles_n) * Cfg::BN, 0, h.K, h.C, h.ldc,
                                             h.alpha, h.beta, smem);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// tile configurations
// ---------------------------------------------------------------------------
using S32 = SimtCfg<float, 32, 32, 2, 2>;
using S64 = SimtCfg<float, 64, 64, 4, 4>;
using S128x32 = SimtCfg<float, 128, 32, 4, 4>;
using S32x128 = SimtCfg<float, 32, 128, 4, 4>;
using S128x64 = SimtCfg<float, 128, 64, 8, 4>;
using S64x128 = SimtCfg<float, 64, 128, 4, 8>;
using S128 = SimtCfg<float, 128, 128, 8, 8>;

using D32 = SimtCfg<double, 32, 32, 2, 2>;
using D64 = SimtCfg<double, 64, 64, 4, 4>;
using D128x32 = SimtCfg<double, 128, 32, 4, 4>;
using D32x128 = SimtCfg<double, 32, 128, 4, 4>;

struct CfgInfo {
  int bm, bn, eff_pct, per_sm;
};
// configuration of calls with transa == Trans (S64 / D64)
constexpr int TRANSA_CFG = 1;

template <typename T, class Cfg>
static size_t smem_of() {
  return (size_t)Cfg::SMEM_ELEMS * sizeof(T);
}

template <typename T, class Cfg, int KBLOCK, bool TA, bool TB>
static int launch_single_l(const GemmArgs<T> &g, int splits, long kchunk,
                           T *partial, int ways_m, int ways_n, int per_sm) {
  const int tiles_m = (int)cdiv(g.M, Cfg::BM), tiles_n = (int)cdiv(g.N, Cfg::BN);
  const long items = (long)tiles_m * tiles_n * splits;
  const size_t smem = smem_of<T, Cfg>();
  auto kern = k_gemm_single<T, Cfg, KBLOCK, TA, TB>;
  per_sm = occupancy_of((const void *)kern, Cfg::NTH, smem, per_sm);
  int grid = ways_m > 0 ? grid_for((long)ways_m * ways_n * splits, per_sm)
                       : grid_for(items, per_sm);
  kern<<<grid, Cfg::NTH, smem, state().stream>>>(g, tiles_m, tiles_n, ways_m, ways_n,
                                                 splits, kchunk, partial);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

// NN and NT layouts for every configuration; A stored K x M (transa) only for
// TRANSA_CFG, which run_gemm picks for those calls
template <typename T, class Cfg, int KBLOCK, bool WITH_TA>
static int launch_single(const GemmArgs<T> &g, int splits, long kchunk,
                         T *partial, int ways_m, int ways_n, int per_sm) {
  if constexpr (WITH_TA) {
    if (g.transa)
      return g.transb ? launch_single_l<T, Cfg, KBLOCK, true, true>(g, splits, kchunk, partial,
                                                                     ways_m, ways_n, per_sm)
                      : launch_single_l<T, Cfg, KBLOCK, true, false>(g, splits, kchunk, partial,
                                                                      ways_m, ways_n, per_sm);
  }
  if (g.transa) return LIBSHALOM_ERR_INVALID_VALUE;
  return g.transb ? launch_single_l<T, Cfg, KBLOCK, false, true>(g, splits, kchunk, partial,
                                                                  ways_m, ways_n, per_sm)
                  : launch_single_l<T, Cfg, KBLOCK, false, false>(g, splits, kchunk, partial,
                                                                   ways_m, ways_n, per_sm);
}

// ---------------------------------------------------------------------------
// scheduler: pick a tile configuration and a split-K factor
// ---------------------------------------------------------------------------
// Cost model: a tile of BM x BN over K costs BM*BN*K / eff, tiles run in
// waves of (SMs * CTAs per SM).  eff grows with the register tile (more FMAs
// per shared-memory load).  Split-K is used when the tile grid fills less
// than half the machine and K is long.
static const CfgInfo kSCfgs[] = {
    {32, 32, 30, 6},    // 0 S32
    {64, 64, 55, 4},    // 1 S64
    {128, 32, 55, 4},   // 2 S128x32
    {32, 128, 55, 4},   // 3 S32x128
    {128, 64, 70, 2},   // 4 S128x64
    {64, 128, 70, 2},   // 5 S64x128
    {128, 128, 85, 1},  // 6 S128
};
static const CfgInfo kDCfgs[] = {
    {32, 32, 40, 4},    // 0 D32
    {64, 64, 70, 2},    // 1 D64
    {128, 32, 70, 2},   // 2 D128x32
    {32, 128, 70, 2},   // 3 D32x128
};

static int pick_cfg(const CfgInfo *cfgs, int ncfg, long M, long N, long K,
                    int sms, int cap) {
  double best = 1e300;
  int bi = 0;
  for (int i = 0; i < ncfg; ++i) {
    const long tiles = cdiv(M, cfgs[i].bm) * cdiv(N, cfgs[i].bn);
    long slots = (long)sms * cfgs[i].per_sm;
    if (cap > 0) slots = std::min<long>(slots, cap);
    const long waves = cdiv(tiles, slots);
    // a partially filled last wave still takes a whole wave per SM, but
    // spreading fewer tiles over idle SMs is free: waves count per-SM load
    const double per_tile = (double)cfgs[i].bm * cfgs[i].bn * (double)std::max(K, 1L) /
                            (cfgs[i].eff_pct / 100.0);
    // CTAs that share an SM split its throughput
    const double share = std::min<double>(cfgs[i].per_sm,
                                          std::max<double>(1.0, (double)tiles / sms));
    const double cost = waves * per_tile * share / cfgs[i].per_sm;
    if (cost < best * 0.999) { best = cost; bi = i; }
  }
  return bi;
}

static int pick_splits(long tiles, long K, int sms, int cap, int forced) {
  if (forced > 0) return (int)std::max(1L, std::min<long>(forced, cdiv(K, 1)));
  long machine = cap > 0 ? std::min(cap, sms) : sms;
  if (tiles * 2 > machine || K < 1024) return 1;
  long s = machine / tiles;
  s = std::min<long>(s, K / 320);
  s = std::min<long>(s, 32);
  return (int)std::max(1L, s);
}

template <typename T>
struct Dispatch;

#define LS_SINGLE_CASE(IDX, CFG, TA)                                                   \
  case IDX:                                                                            \
    return kblock ? launch_single<T, CFG, 320, TA>(g, splits, kchunk, partial, wm, wn, per_sm) \
                  : launch_single<T, CFG, 0, TA>(g, splits, kchunk, partial, wm, wn, per_sm);

template <>
struct Dispatch<float> {
  static int single(int cfg, const GemmArgs<float> &g, int splits, long kchunk,
                    float *partial, int wm, int wn, bool kblock) {
    using T = float;
    const int per_sm = kSCfgs[cfg].per_sm;
    switch (cfg) {
      LS_SINGLE_CASE(0, S32, false)
      LS_SINGLE_CASE(1, S64, true)
      LS_SINGLE_CASE(2, S128x32, false)
      LS_SINGLE_CASE(3, S32x128, false)
      LS_SINGLE_CASE(4, S128x64, false)
      LS_SINGLE_CASE(5, S64x128, false)
      LS_SINGLE_CASE(6, S128, false)
    }
    return LIBSHALOM_ERR_INVALID_VALUE;
  }
  static const CfgInfo *cfgs(int *n) { *n = 7; return kSCfgs; }
};

template <>
struct Dispatch<double> {
  static int single(int cfg, const GemmArgs<double> &g, int splits, long kchunk,
                    double *partial, int wm, int wn, bool kblock) {
    using T = double;
    const int per_sm = kDCfgs[cfg].per_sm;
    (void)kblock;
    switch (cfg) {
      case 0: return launch_single<T, D32, 0, false>(g, splits, kchunk, partial, wm, wn, per_sm);
      case 1: return launch_single<T, D64, 0, true>(g, splits, kchunk, partial, wm, wn, per_sm);
      case 2: return launch_single<T, D128x32, 0, false>(g, splits, kchunk, partial, wm, wn, per_sm);
      case 3: return launch_single<T, D32x128, 0, false>(g, splits, kchunk, partial, wm, wn, per_sm);
    }
    return LIBSHALOM_ERR_INVALID_VALUE;
  }
  static const CfgInfo *cfgs(int *n) { *n = 4; return kDCfgs; }
};

template <typename T>
int run_gemm(const GemmArgs<T> &g, const SimtOptions &opt, SimtPlan *plan_out) {
  State &st = state();
  int ncfg;
  const CfgInfo *cfgs = Dispatch<T>::cfgs(&ncfg);
  if (opt.force_cfg >= ncfg) return LIBSHALOM_ERR_INVALID_VALUE;
  int cfg = opt.force_cfg >= 0 ? opt.force_cfg
                               : pick_cfg(cfgs, ncfg, g.M, g.N, g.K, st.num_sms, st.thread_cap);
  if (g.transa) cfg = TRANSA_CFG;  // the one configuration built for A stored K x M
  const long tiles = cdiv(g.M, cfgs[cfg].bm) * cdiv(g.N, cfgs[cfg].bn);
  int splits = opt.allow_split ? pick_splits(tiles, g.K, st.num_sms, st.thread_cap, opt.splits)
                               : 1;
  long kchunk = g.K > 0 ? g.K : 1;
  if (splits > 1) {
    kchunk = cdiv(g.K, splits);
    if (opt.kblock) kchunk = cdiv(kchunk, 320) * 320;  // keep GEMM_K blocks aligned
    else kchunk = cdiv(kchunk, 16) * 16;
    splits = (int)cdiv(g.K, kchunk);
  }
  if (plan_out) {
    plan_out->cfg = cfg;
    plan_out->bm = cfgs[cfg].bm;
    plan_out->bn = cfgs[cfg].bn;
    plan_out->splits = splits;
    plan_out->kchunk = kchunk;
  }
  T *partial = nullptr;
  if (splits > 1) {
    void *ws = nullptr;
    int rc = workspace(sizeof(T) * (size_t)splits * g.M * g.N, &ws);
    if (rc) return rc;
    partial = reinterpret_cast<T *>(ws);
  }
  int rc = Dispatch<T>::single(cfg, g, splits, kchunk, partial, opt.ways_m, opt.ways_n,
                               opt.kblock);
  if (rc) return rc;
  if (splits > 1) {
    const long total = g.M * g.N;
    int grid = (int)std::min<long>(cdiv(total, 256), (long)st.num_sms * 8);
    k_splitk_reduce<T><<<std::max(grid, 1), 256, 0, st.stream>>>(partial, splits, g.M, g.N,
                                                                g.C, g.ldc, g.alpha, g.beta);
    LS_CUDA_TRY(cudaGetLastError());
  }
  return LIBSHALOM_SUCCESS;
}

// Split-K GEMM whose partial sums live in a caller-provided device buffer of
// at least splits * M * N floats; allocates nothing.
int run_gemm_splitk_external(const GemmArgs<float> &g, int splits, float *partial) {
  State &st = state();
  int ncfg;
  const CfgInfo *cfgs = Dispatch<float>::cfgs(&ncfg);
  const int cfg = g.transa ? TRANSA_CFG
                          : pick_cfg(cfgs, ncfg, g.M, g.N, g.K, st.num_sms, st.thread_cap);
  // K slices stay whole GEMM_K blocks; K = 0 is one empty slice (C = beta C)
  const long kchunk = g.K > 0 ? cdiv(cdiv(g.K, splits), 320) * 320 : 1;
  const int used = g.K > 0 ? (int)cdiv(g.K, kchunk) : 1;
  int rc = Dispatch<float>::single(cfg, g, used, kchunk, partial, 0, 0, true);
  if (rc || used == 1) return rc;  // one slice: the tile kernel wrote C itself
  const long total = g.M * g.N;
  const int grid = (int)std::min<long>(cdiv(total, 256), (long)st.num_sms * 8);
  k_splitk_reduce<float><<<std::max(grid, 1), 256, 0, st.stream>>>(partial, used, g.M, g.N,
                                                                  g.C, g.ldc, g.alpha, g.beta);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

int run_splitk_reduce_f32(const float *partial, int splits, long M, long N, float *C, long ldc,
                          float alpha, float beta) {
  State &st = state();
  const long total = M * N;
  const int grid = (int)std::min<long>(cdiv(total, 256), (long)st.num_sms * 8);
  k_splitk_reduce<float><<<std::max(grid, 1), 256, 0, st.stream>>>(partial, splits, M, N, C, ldc,
                                                                  alpha, beta);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

template int run_gemm<float>(const GemmArgs<float> &, const SimtOptions &, SimtPlan *);
template int run_gemm<double>(const GemmArgs<double> &, const SimtOptions &, SimtPlan *);

// uniform batches: one configuration per shape class
template <typename T, class Cfg>
static int launch_strided(const GemmArgs<T> &g, long sA, long sB, long sC, long count,
                          int per_sm) {
  const int tiles_m = (int)cdiv(g.M, Cfg::BM), tiles_n = (int)cdiv(g.N, Cfg::BN);
  const long items = (long)tiles_m * tiles_n * count;
  const size_t smem = smem_of<T, Cfg>();
  auto kern = g.transb ? k_gemm_strided<T, Cfg, true> : k_gemm_strided<T, Cfg, false>;
  per_sm = occupancy_of((const void *)kern, Cfg::NTH, smem, per_sm);
  const int grid = grid_for(items, per_sm);
  kern<<<grid, Cfg::NTH, smem, state().stream>>>(g, sA, sB, sC, count, tiles_m, tiles_n);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

template <>
int run_strided<float>(const GemmArgs<float> &g, long sA, long sB, long sC, long count) {
  if (g.M <= 32 && g.N <= 32) return launch_strided<float, S32>(g, sA, sB, sC, count, 6);
  if (g.M <= 64 && g.N <= 64) return launch_strided<float, S64>(g, sA, sB, sC, count, 4);
  return launch_strided<float, S128>(g, sA, sB, sC, count, 1);
}
template <>
int run_strided<double>(const GemmArgs<double> &g, long sA, long sB, long sC, long count) {
  if (g.M <= 32 && g.N <= 32) return launch_strided<double, D32>(g, sA, sB, sC, count, 4);
  return launch_strided<double, D64>(g, sA, sB, sC, count, 2);
}

template <typename T, class Cfg>
static int launch_grouped(const typename EntryOf<T>::type *entries, long count, int per_sm) {
  void *ws = nullptr;
  int rc = workspace(64, &ws);
  if (rc) return rc;
  unsigned long long *counter = reinterpret_cast<unsigned long long *>(ws);
  LS_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), state().stream));
  const size_t smem = smem_of<T, Cfg>();
  auto kern = k_gemm_grouped<T, Cfg>;
  per_sm = occupancy_of((const void *)kern, Cfg::NTH, smem, per_sm);
  const int grid = grid_for(count, per_sm);
  kern<<<grid, Cfg::NTH, smem, state().stream>>>(entries, count, counter);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

int run_grouped_s(const LibShalom_sgemm_entry *entries, long count) {
  return launch_grouped<float, S64>(entries, count, 4);
}
// Grouped FP64 batches go to the run kernel of ls_dgemm.cu (C tile held in
// registers across a run, cp.async double buffer); the generic tile kernel
// above stays available for comparison.
int run_grouped_d(const LibShalom_dgemm_entry *entries, long count) {
  return run_dgemm_runs(entries, count);
}

int run_grouped_d_generic(const LibShalom_dgemm_entry *entries, long count) {
  return launch_grouped<double, D32>(entries, count, 4);
}

}  // namespace ls
