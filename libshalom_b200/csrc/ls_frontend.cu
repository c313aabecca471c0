// ls_frontend.cu -- front ends that feed the GEMM paths: the DBCSR-style
// stack of (M, N, K, offsets into pools) -> grouped DGEMM entries, the
// im2col expansion of a 2-D convolution (NCHW), and the implicit-GEMM
// convolution whose tile loader gathers the im2col columns itself.
#include <cuda_runtime.h>

#include <algorithm>

#include "ls_common.cuh"
#include "ls_frontend.h"
#include "ls_simt.cuh"

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

// op(B)[k][p] of the convolution GEMM y[oc][p] = wt[oc][k] col[k][p]: the
// im2col element for k = (ci, r, q), p = (oy, ox), read from the image
struct ConvB {
  static constexpr bool kDense = false;
  const float *x;  // this image, [c][h][w]
  int h, w, kw, khw, sh, sw, ph, pw, ow;
  // address of the element, nullptr in the zero padding
  __device__ __forceinline__ const float *ptr(const GemmArgs<float> &, long k, long p) const {
    const int kk = (int)k, pp = (int)p;
    const int ci = kk / khw, rq = kk - ci * khw, r = rq / kw, q = rq - r * kw;
    const int oy = pp / ow, ox = pp - oy * ow;
    const int iy = oy * sh - ph + r, ix = ox * sw - pw + q;
    return (iy >= 0 && iy < h && ix >= 0 && ix < w) ? x + ((long)ci * h + iy) * w + ix : nullptr;
  }
};

// persistent over (image, tile_m, tile_n); per output element the mp path's
// rounding order: FMA chains over k restarted every GEMM_K = 320 values of k,
// the block sums added in increasing k
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NTH)
    k_conv_implicit(GemmArgs<float> g, ConvB b, long n_img, long img_stride, int tiles_m,
                    int tiles_n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float *smem = reinterpret_cast<float *>(smem_raw);
  const long per_img = (long)tiles_m * tiles_n;
  for (long wi = blockIdx.x; wi < per_img * n_img; wi += gridDim.x) {
    const long img = wi / per_img;
    const int t = (int)(wi - img * per_img);
    ConvB bi = b;
    bi.x = b.x + img * img_stride;
    simt_tile<float, Cfg, GEMM_K, false, false, ConvB>(g, (long)(t / tiles_n) * Cfg::BM,
                                    (long)(t % tiles_n) * Cfg::BN, 0, g.K,
                                    g.C + img * g.M * g.N, g.N, 1.0f, 0.0f, smem, bi);
  }
}

using ConvCfg = SimtCfg<float, 64, 64, 4, 4>;

}  // namespace

int conv_implicit(const float *x, long n, long c, long h, long w, const float *wt, long oc,
                  long kh, long kw, long sh, long sw, long ph, long pw, long oh, long ow,
                  float *y) {
  State &st = state();
  GemmArgs<float> g;
  g.A = wt; g.B = nullptr; g.C = y;
  g.M = oc; g.N = oh * ow; g.K = c * kh * kw;
  g.lda = g.K; g.ldb = g.N; g.ldc = g.N;
  g.transa = 0; g.transb = 0;
  g.alpha = 1.0f; g.beta = 0.0f;
  ConvB b;
  b.x = x;
  b.h = (int)h; b.w = (int)w; b.kw = (int)kw; b.khw = (int)(kh * kw);
  b.sh = (int)sh; b.sw = (int)sw; b.ph = (int)ph; b.pw = (int)pw; b.ow = (int)ow;
  const int tiles_m = (int)cdiv(g.M, ConvCfg::BM), tiles_n = (int)cdiv(g.N, ConvCfg::BN);
  const size_t smem = sizeof(float) * ConvCfg::SMEM_ELEMS;
  const int per_sm = occupancy_of((const void *)k_conv_implicit<ConvCfg>, ConvCfg::NTH, smem, 1);
  const int grid = grid_for((long)tiles_m * tiles_n * n, per_sm);
  k_conv_implicit<ConvCfg><<<grid, ConvCfg::NTH, smem, st.stream>>>(g, b, n, c * h * w, tiles_m,
                                                                    tiles_n);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

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
