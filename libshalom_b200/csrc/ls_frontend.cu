// ls_frontend.cu -- front ends that feed the GEMM paths: the DBCSR-style
// stack of (M, N, K, offsets into pools) -> grouped DGEMM entries, and the
// im2col expansion of a 2-D convolution (NCHW).
#include <cuda_runtime.h>

#include <algorithm>

#include "ls_common.cuh"
#include "ls_frontend.h"

namespace ls {

namespace {

__global__ void k_stack_entries(StackArgs s, long count, LibShalom_dgemm_entry *out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count;
       i += (long)gridDim.x * blockDim.x) {
    LibShalom_dgemm_entry e;
    e.M = s.M ? s.M[i] : s.m;
    e.N = s.N ? s.N[i] : s.n;
    e.K = s.K ? s.K[i] : s.k;
    e.transb = s.transb;
    e.lda = e.K;
    e.ldb = s.transb ? e.K : e.N;
    e.ldc = e.N;
    e.reserved = 0;
    e.A = s.A + s.a_off[i];
    e.B = s.B + s.b_off[i];
    e.C = s.C + s.c_off[i];
    e.alpha = s.alpha;
    e.beta = s.beta;
    out[i] = e;
  }
}

// col[(ci * kh + r) * kw + q][oy * ow + ox] = x[ci][oy*sh - ph + r][ox*sw - pw + q] (0 outside)
__global__ void k_im2col(const float *x, long c, long h, long w, long kh, long kw, long sh,
                         long sw, long ph, long pw, long oh, long ow, float *col) {
  const long ncol = oh * ow, rows = c * kh * kw;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < rows * ncol;
       idx += (long)gridDim.x * blockDim.x) {
    const long row = idx / ncol, p = idx - row * ncol;
    const long ci = row / (kh * kw), rq = row - ci * kh * kw, r = rq / kw, q = rq - r * kw;
    const long oy = p / ow, ox = p - oy * ow;
    const long iy = oy * sh - ph + r, ix = ox * sw - pw + q;
    col[idx] = (iy >= 0 && iy < h && ix >= 0 && ix < w) ? x[(ci * h + iy) * w + ix] : 0.0f;
  }
}

}  // namespace

int stack_to_entries(const StackArgs &s, long count, LibShalom_dgemm_entry *out) {
  State &st = state();
  const int grid = (int)std::max(1L, std::min(cdiv(count, 256), (long)st.num_sms * 8));
  k_stack_entries<<<grid, 256, 0, st.stream>>>(s, count, out);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

int im2col(const float *x, long c, long h, long w, long kh, long kw, long sh, long sw, long ph,
           long pw, long oh, long ow, float *col) {
  State &st = state();
  const long total = c * kh * kw * oh * ow;
  const int grid = (int)std::max(1L, std::min(cdiv(total, 256), (long)st.num_sms * 16));
  k_im2col<<<grid, 256, 0, st.stream>>>(x, c, h, w, kh, kw, sh, sw, ph, pw, oh, ow, col);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

}  // namespace ls
