// ls_frontend.h -- kernels of the stack and convolution front ends.
#pragma once

#include "../../include/LibShalom.h"

namespace ls {

struct StackArgs {
  const double *A, *B;
  double *C;
  const int32_t *M, *N, *K;
  int32_t m, n, k, transb;
  const int64_t *a_off, *b_off, *c_off;
  double alpha, beta;
};

// entries of a stack (device array of count LibShalom_dgemm_entry)
int stack_to_entries(const StackArgs &s, long count, LibShalom_dgemm_entry *out);

// col: [c*kh*kw][oh*ow] expansion of one NCHW image x [c][h][w]
int im2col(const float *x, long c, long h, long w, long kh, long kw, long sh, long sw, long ph,
           long pw, long oh, long ow, float *col);

// y[i] [oc][oh*ow] = wt [oc][c*kh*kw] x col(x[i]) for the n images, FP32 on the
// CUDA cores, with the im2col columns gathered inside the GEMM tile's loader
// (no column buffer).  Sizes must fit int32 (checked by the caller).
int conv_implicit(const float *x, long n, long c, long h, long w, const float *wt, long oc,
                  long kh, long kw, long sh, long sw, long ph, long pw, long oh, long ow,
                  float *y);

}  // namespace ls
