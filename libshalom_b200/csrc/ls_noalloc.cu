// ls_noalloc.cu -- LibShalom_sgemm_mp_noalloc: the split-K SGEMM of
// LibShalom_sgemm_mp for callers that cannot allocate device memory.
//
// LibShalom_sgemm_mp keeps its split-K partial sums in a workspace that the
// library grows with cudaMalloc on first use.  Some callers cannot allow that:
// code whose device memory is entirely owned by another allocator (a caching
// allocator that reserved the GPU's memory up front), or code that must not
// see a cudaMalloc/cudaFree in the middle of a call, since those can fail
// under memory pressure and synchronise the device.  This entry point keeps
// the partial sums in a fixed array compiled into the library instead, so a
// call performs no allocation of any kind.
//
// The array lives in device global memory as a file-scope __device__
// variable: every GPU that loads the library holds its
// LIBSHALOM_NOALLOC_SCRATCH_FLOATS floats (8 MiB) until the process exits.
// In host code its name is only a host-side stand-in, so the device address
// is looked up with cudaGetSymbolAddress, once per device, on the first call
// made while that device is current.  Make that first call before any stream
// capture.
//
// All calls share the one array and it keeps whatever the last call left in
// it.  Every slice writes its whole partial block before the reduction reads
// it, so nothing needs clearing; but calls that overlap on the GPU (launched
// on different streams, or from several host threads with asynchronous mode)
// race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include "ls_common.cuh"
#include "ls_simt_launch.h"

namespace ls {

static __device__ __align__(256) float g_noalloc_partials[LIBSHALOM_NOALLOC_SCRATCH_FLOATS];

// device address of g_noalloc_partials, per device ordinal (set up lazily)
static float *g_noalloc_ptr[64];

static int noalloc_scratch(float **out) {
  const int dev = state().device;
  if (dev < 0 || dev >= 64) return LIBSHALOM_ERR_NO_DEVICE;
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) {
      note_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_partials)", __FILE__, __LINE__);
      return LIBSHALOM_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = static_cast<float *>(p);
  }
  *out = g_noalloc_ptr[dev];
  return LIBSHALOM_SUCCESS;
}

static int sgemm_mp_noalloc(int transa, int transb, float *C, const float *A, const float *B,
                            long M, long N, long K, int splits) {
  if ((transa != NoTrans && transa != Trans) || (transb != NoTrans && transb != Trans))
    return LIBSHALOM_ERR_INVALID_VALUE;
  if (M < 0 || N < 0 || K < 0 || splits < 1) return LIBSHALOM_ERR_INVALID_VALUE;
  if (M == 0 || N == 0) return LIBSHALOM_SUCCESS;
  if (!C || (K > 0 && (!A || !B))) return LIBSHALOM_ERR_INVALID_VALUE;
  // the partial sums of every slice must fit the static array
  if (M > (1L << 30) || N > (1L << 30) ||
      (double)splits * (double)M * (double)N > (double)LIBSHALOM_NOALLOC_SCRATCH_FLOATS)
    return LIBSHALOM_ERR_INVALID_VALUE;
  int rc = flush_deferred();  // ordered after pending deferred calls
  if (rc) return rc;
  rc = ensure_device();
  if (rc) return rc;
  float *scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  GemmArgs<float> g;
  g.A = A; g.B = B; g.C = C;
  g.M = M; g.N = N; g.K = K;
  g.transa = transa; g.transb = transb;
  g.lda = transa ? M : K;
  g.ldb = transb ? K : N;
  g.ldc = N;
  g.alpha = 1.0f; g.beta = 0.0f;
  rc = run_gemm_splitk_external(g, splits, scratch);
  if (rc) return rc;
  return finish_launch("sgemm_mp_noalloc");
}

}  // namespace ls

extern "C" int LibShalom_sgemm_mp_noalloc(int transa, int transb, float *C, const float *A,
                                          const float *B, long M, long N, long K, int splits) {
  std::lock_guard<std::mutex> lk(ls::state().mu);
  const int rc = ls::sgemm_mp_noalloc(transa, transb, C, A, B, M, N, K, splits);
  ls::set_error(rc);
  return rc;
}
