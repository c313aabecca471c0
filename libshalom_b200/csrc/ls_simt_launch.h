// ls_simt_launch.h -- host-side entry points of the plain CUDA-core kernels.
#pragma once

#include "../../include/LibShalom.h"
#include "ls_simt.cuh"

namespace ls {

struct SimtOptions {
  bool allow_split = true;  // let the scheduler split K across CTAs
  int splits = 0;           // >0 forces the split factor
  bool kblock = false;      // GEMM_K = 320 fold (reference mp rounding order)
  int ways_m = 0, ways_n = 0;  // LibShalom_set_thread_ways partition
  int force_cfg = -1;       // tile configuration override (autotuner/tests)
};

struct SimtPlan {
  int cfg = -1, bm = 0, bn = 0, splits = 1;
  long kchunk = 0;
};

template <typename T>
int run_gemm(const GemmArgs<T> &g, const SimtOptions &opt, SimtPlan *plan_out);

template <typename T>
int run_strided(const GemmArgs<T> &g, long sA, long sB, long sC, long count);

int run_grouped_s(const LibShalom_sgemm_entry *entries, long count);
int run_grouped_d(const LibShalom_dgemm_entry *entries, long count);
int run_grouped_d_generic(const LibShalom_dgemm_entry *entries, long count);
// C = alpha * sum_z partial[z] + beta * C, partial slices summed in order
int run_splitk_reduce_f32(const float *partial, int splits, long M, long N, float *C, long ldc,
                          float alpha, float beta);
// ls_dgemm.cu: runs of products sharing C, C tile held in registers
int run_dgemm_runs(const LibShalom_dgemm_entry *entries, long count);
int run_dgemm_runs_list(const LibShalom_dgemm_entry *entries, long count, const unsigned *n_runs,
                        const unsigned *run_first, const unsigned *run_len);
// ls_dgemm_warp.cu: runs with M, N <= 32 on the FP64 (DMMA) or INT8 (Ozaki)
// tensor cores, the rest through run_dgemm_runs_list
int run_dgemm_warp(const LibShalom_dgemm_entry *entries, long count, int method, int slices);
// ls_dgemm_dmma.cu: runs with M, N <= 32 on the FP64 tensor cores (warp per
// run, bulk-copy ring), the rest through run_dgemm_runs_list
int run_dgemm_dmma(const LibShalom_dgemm_entry *entries, long count);

// Plain FP32 split-K GEMM (GEMM_K-aligned slices, rounding order of the mp
// path per slice) with the partial sums in `partial` (>= splits * M * N
// floats, device memory owned by the caller).  Allocates nothing.
int run_gemm_splitk_external(const GemmArgs<float> &g, int splits, float *partial);

// ls_tune.cu: measured choices per shape class (kind, half-octaves of M, N, K)
enum TuneKind {
  TUNE_S_SINGLE = 0,   // plain FP32, LibShalom_sgemm (tile configuration)
  TUNE_S_MP = 1,       // plain FP32, LibShalom_sgemm_mp (tile configuration + split-K)
  TUNE_D_SINGLE = 2,   // plain FP64, LibShalom_dgemm
  TUNE_TC_BF16X3 = 3,  // split-BF16 x3, LibShalom_sgemm_mp (split-K)
  TUNE_TC_BF16X6 = 4,  // split-BF16 x6, LibShalom_sgemm_mp (split-K)
};
int half_octave(long x);
bool tune_lookup(int kind, long M, long N, long K, int *cfg, int *splits);
int tune_table_size();

}  // namespace ls
