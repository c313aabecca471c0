// ls_tc_launch.h -- host-side entry points of the split-BF16 tcgen05 kernels.
#pragma once

#include "../../include/LibShalom.h"
#include "ls_simt.cuh"

namespace ls {

// Single (irregular) SGEMM on the tensor cores; `mode` is a
// LIBSHALOM_PREC_BF16X* value, `splits` as LibShalom_set_splitk.
// splits: 0 = chosen here, s > 0 = about s slices; *used (if given) gets the
// factor launched
int tc_sgemm_single(const GemmArgs<float> &g, int mode, int splits, int *used = nullptr);

// Uniform batch on the tensor cores.
int tc_sgemm_strided(const GemmArgs<float> &g, long sA, long sB, long sC, long count, int mode);

// Grouped batch (entries in device memory) on the tensor cores.
int tc_sgemm_grouped(const LibShalom_sgemm_entry *entries, long count, int mode);

// Runs the bounded-wait self-check kernel (an mbarrier nothing arrives at);
// returns LIBSHALOM_ERR_DEVICE_TIMEOUT when its waits expired and reported.
int tc_wait_expiry_selftest(int iterations);

}  // namespace ls
