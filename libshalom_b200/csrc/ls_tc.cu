// ls_tc.cu -- split-BF16 GEMM on the sm_100a tensor cores (tcgen05 + TMEM).
#include "ls_common.cuh"
#include "ls_tc_launch.h"

namespace ls {

int tc_sgemm_single(const GemmArgs<float> &, int, int) { return LIBSHALOM_ERR_UNSUPPORTED; }
int tc_sgemm_strided(const GemmArgs<float> &, long, long, long, long, int) {
  return LIBSHALOM_ERR_UNSUPPORTED;
}
int tc_sgemm_grouped(const LibShalom_sgemm_entry *, long, int) {
  return LIBSHALOM_ERR_UNSUPPORTED;
}

}  // namespace ls
