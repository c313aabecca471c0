// ls_api.cu -- the C ABI of include/LibShalom.h: argument checking, library
// state, workspace and dispatch to the kernels.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <unordered_map>
#include <unordered_set>

#include "ls_common.cuh"
#include "ls_frontend.h"
#include "ls_simt_launch.h"
#include "ls_tc_launch.h"

namespace ls {

static thread_local int t_last_error = LIBSHALOM_SUCCESS;

void set_error(int status) { t_last_error = status; }
int last_error() { return t_last_error; }

void note_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
  if (getenv("LIBSHALOM_DEBUG"))
    fprintf(stderr, "libshalom: %s failed: %s (%s:%d)\n", what, cudaGetErrorString(e), file,
            line);
}

State &state() {
  static State s;
  return s;
}

int ensure_device() {
  State &st = state();
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    note_cuda_error(e, "cudaGetDevice", __FILE__, __LINE__);
    return LIBSHALOM_ERR_NO_DEVICE;
  }
  if (dev == st.device) return LIBSHALOM_SUCCESS;
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) {
    note_cuda_error(e, "cudaGetDeviceProperties", __FILE__, __LINE__);
    return LIBSHALOM_ERR_NO_DEVICE;
  }
  if (prop.major != 10) return LIBSHALOM_ERR_NO_DEVICE;  // built for sm_100a only
  st.device = dev;
  st.num_sms = prop.multiProcessorCount;
  st.cc_major = prop.major;
  st.cc_minor = prop.minor;
  st.smem_optin = prop.sharedMemPerBlockOptin;
  return LIBSHALOM_SUCCESS;
}

int workspace(size_t bytes, void **out) {
  State &st = state();
  if (bytes < 256) bytes = 256;
  if (st.ws && st.ws_bytes >= bytes && st.ws_device == st.device) {
    *out = st.ws;
    return LIBSHALOM_SUCCESS;
  }
  if (st.ws) {
    // kernels queued earlier may still read the old buffer
    LS_CUDA_TRY(cudaStreamSynchronize(st.stream));
    cudaFree(st.ws);
    st.ws = nullptr;
    st.ws_bytes = 0;
  }
  size_t want = std::max(bytes, (size_t)1 << 20);
  if (cudaMalloc(&st.ws, want) != cudaSuccess) {
    cudaGetLastError();
    st.ws = nullptr;
    return LIBSHALOM_ERR_ALLOC;
  }
  st.ws_bytes = want;
  st.ws_device = st.device;
  ++st.ws_generation;  // graphs captured with the old buffer are stale
  *out = st.ws;
  return LIBSHALOM_SUCCESS;
}

int grid_for(long work_items, int per_sm) {
  State &st = state();
  long slots = (long)st.num_sms * std::max(per_sm, 1);
  if (st.thread_cap > 0) slots = std::min<long>(slots, st.thread_cap);
  long g = std::min(work_items, slots);
  return (int)std::max(g, 1L);
}

int occupancy_of(const void *kern, int threads, size_t smem, int fallback) {
  static std::mutex m;
  static std::unordered_map<const void *, int> cache;
  std::lock_guard<std::mutex> lk(m);
  auto it = cache.find(kern);
  if (it != cache.end()) return it->second;
  if (smem >= 48 * 1024 &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess) {
    cudaGetLastError();
    return fallback;
  }
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem) != cudaSuccess ||
      n <= 0) {
    cudaGetLastError();
    return fallback;
  }
  cache[kern] = n;
  return n;
}

int finish_launch(const char *what) {
  State &st = state();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    note_cuda_error(e, what, __FILE__, __LINE__);
    return LIBSHALOM_ERR_CUDA;
  }
  if (st.sync) {
    e = cudaStreamSynchronize(st.stream);
    if (e != cudaSuccess) {
      note_cuda_error(e, what, __FILE__, __LINE__);
      return LIBSHALOM_ERR_CUDA;
    }
  }
  return LIBSHALOM_SUCCESS;
}

// Buffer of the front ends (grown on demand like the workspace).
static int frontend_buffer(size_t bytes, void **out) {
  State &st = state();
  if (bytes < 256) bytes = 256;
  if (st.fe && st.fe_bytes >= bytes && st.fe_device == st.device) {
    *out = st.fe;
    return LIBSHALOM_SUCCESS;
  }
  if (st.fe) {
    LS_CUDA_TRY(cudaStreamSynchronize(st.stream));
    cudaFree(st.fe);
    st.fe = nullptr;
    st.fe_bytes = 0;
  }
  const size_t want = std::max(bytes, (size_t)1 << 20);
  if (cudaMalloc(&st.fe, want) != cudaSuccess) {
    cudaGetLastError();
    st.fe = nullptr;
    return LIBSHALOM_ERR_ALLOC;
  }
  st.fe_bytes = want;
  st.fe_device = st.device;
  *out = st.fe;
  return LIBSHALOM_SUCCESS;
}

// lda / ldb / ldc = 0: the row-major defaults of the drop-in calls
template <typename T>
static int gemm_common(int transa, int transb, T *C, const T *A, const T *B, long M, long N,
                       long K, bool mp, T alpha = T(1), T beta = T(0), long lda = 0,
                       long ldb = 0, long ldc = 0) {
  if ((transa != NoTrans && transa != Trans) || (transb != NoTrans && transb != Trans))
    return LIBSHALOM_ERR_INVALID_VALUE;
  if (M < 0 || N < 0 || K < 0) return LIBSHALOM_ERR_INVALID_VALUE;
  if (lda < 0 || ldb < 0 || ldc < 0) return LIBSHALOM_ERR_INVALID_VALUE;
  if ((lda && lda < (transa ? M : K)) || (ldb && ldb < (transb ? K : N)) || (ldc && ldc < N))
    return LIBSHALOM_ERR_INVALID_VALUE;
  if (M == 0 || N == 0) return LIBSHALOM_SUCCESS;
  if (!C || (K > 0 && (!A || !B))) return LIBSHALOM_ERR_INVALID_VALUE;
  if (lda > INT32_MAX || ldb > INT32_MAX || ldc > INT32_MAX) return LIBSHALOM_ERR_INVALID_VALUE;
  // int32 tile indices inside the kernels
  if (M > (1L << 30) || N > (1L << 30) || K > (1L << 40)) return LIBSHALOM_ERR_INVALID_VALUE;
  int rc = ensure_device();
  if (rc) return rc;
  State &st = state();
  GemmArgs<T> g;
  g.A = A; g.B = B; g.C = C;
  g.M = M; g.N = N; g.K = K;
  g.transa = transa; g.transb = transb;
  g.lda = lda ? lda : (transa ? M : K);
  g.ldb = ldb ? ldb : (transb ? K : N);
  g.ldc = ldc ? ldc : N;
  g.alpha = alpha; g.beta = beta;
  SimtOptions opt;
  if (mp) {
    opt.kblock = true;
    opt.splits = st.splitk;
    opt.allow_split = st.splitk != 1;
    opt.ways_m = st.ways_m;
    opt.ways_n = st.ways_n;
    st.ways_m = st.ways_n = 0;  // one-shot, like the reference's Tm = 0 reset
  } else {
    opt.allow_split = false;
  }
  const bool tc = mp && sizeof(T) == 4 && st.precision != LIBSHALOM_PREC_FP32;
  // measured shape-class choices, unless forced by the caller
  const int kind = tc ? (st.precision == LIBSHALOM_PREC_BF16X3 ? TUNE_TC_BF16X3 : TUNE_TC_BF16X6)
                      : sizeof(T) == 8 ? TUNE_D_SINGLE
                                       : (mp ? TUNE_S_MP : TUNE_S_SINGLE);
  int t_cfg = -1, t_splits = 0;
  const bool hit = st.autotune && !transa && (sizeof(T) == 4 || !mp) &&
                   tune_lookup(kind, M, N, K, &t_cfg, &t_splits);
  opt.force_cfg = st.tile_cfg >= 0 ? st.tile_cfg : (hit ? t_cfg : -1);
  if (hit && mp && st.splitk == 0 && t_splits > 0) opt.splits = t_splits;
  if (tc) {
    int used = 0;
    rc = tc_sgemm_single((const GemmArgs<float> &)g, st.precision, opt.splits, &used);
    st.last_cfg = -1;
    st.last_splits = used;
  } else {
    SimtPlan plan;
    rc = run_gemm<T>(g, opt, &plan);
    st.last_cfg = plan.cfg;
    st.last_splits = plan.splits;
  }
  if (rc) return rc;
  return finish_launch("gemm");
}

// ---------------------------------------------------------------------------
// Graph cache of the drop-in single / mp calls.  A call whose arguments and
// library settings repeat exactly is captured into a CUDA graph the second
// time it is seen (the first run has already sized the workspace) and
// replayed from then on with one cudaGraphLaunch.  Entries remember the
// workspace generation they were captured with; a workspace that moved
// invalidates them.  Needs a non-default stream (LibShalom_set_stream).
// ---------------------------------------------------------------------------
struct GraphKey {
  int kind, transa, transb, precision, tile_cfg, autotune, splitk, ways_m, ways_n, device;
  const void *A, *B, *C;
  long M, N, K;
  cudaStream_t stream;
  bool operator==(const GraphKey &o) const { return memcmp(this, &o, sizeof(*this)) == 0; }
};
struct GraphKeyHash {
  size_t operator()(const GraphKey &k) const {
    const unsigned char *p = reinterpret_cast<const unsigned char *>(&k);
    size_t h = 1469598103934665603ull;
    for (size_t i = 0; i < sizeof(k); ++i) h = (h ^ p[i]) * 1099511628211ull;
    return h;
  }
};
struct GraphEntry {
  int uses = 0;
  unsigned generation = 0;
  cudaGraphExec_t exec = nullptr;
};
static std::unordered_map<GraphKey, GraphEntry, GraphKeyHash> &graph_cache() {
  static std::unordered_map<GraphKey, GraphEntry, GraphKeyHash> m;
  return m;
}
static void graph_cache_clear() {
  for (auto &kv : graph_cache())
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  graph_cache().clear();
}
constexpr size_t kGraphCacheMax = 256;

template <typename T>
static int gemm_cached(int kind, int transa, int transb, T *C, const T *A, const T *B, long M,
                       long N, long K, bool mp) {
  State &st = state();
  if (!st.graph_cache || st.stream == nullptr || M <= 0 || N <= 0)
    return gemm_common<T>(transa, transb, C, A, B, M, N, K, mp);
  int rc = ensure_device();
  if (rc) return rc;
  GraphKey key;
  memset(&key, 0, sizeof(key));  // padding bytes take part in the hash
  key.kind = kind; key.transa = transa; key.transb = transb; key.precision = st.precision;
  key.tile_cfg = st.tile_cfg; key.autotune = st.autotune; key.splitk = st.splitk;
  key.ways_m = st.ways_m; key.ways_n = st.ways_n; key.device = st.device;
  key.A = A; key.B = B; key.C = C; key.M = M; key.N = N; key.K = K; key.stream = st.stream;
  auto &cache = graph_cache();
  auto it = cache.find(key);
  if (it != cache.end() && it->second.exec && it->second.generation == st.ws_generation) {
    st.ways_m = st.ways_n = 0;  // one-shot, as on the direct path
    LS_CUDA_TRY(cudaGraphLaunch(it->second.exec, st.stream));
    return finish_launch("gemm (graph)");
  }
  if (it == cache.end()) {
    if (cache.size() >= kGraphCacheMax) graph_cache_clear();
    cache[key].uses = 1;
    return gemm_common<T>(transa, transb, C, A, B, M, N, K, mp);  // first sight: run it
  }
  // second sight (or stale graph): capture this run, then launch the graph
  GraphEntry &ge = it->second;
  if (ge.exec) {
    cudaGraphExecDestroy(ge.exec);
    ge.exec = nullptr;
  }
  const int sync = st.sync;
  st.sync = 0;  // no host synchronisation inside the capture
  LS_CUDA_TRY(cudaStreamBeginCapture(st.stream, cudaStreamCaptureModeThreadLocal));
  rc = gemm_common<T>(transa, transb, C, A, B, M, N, K, mp);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(st.stream, &graph);
  st.sync = sync;
  if (rc || ce != cudaSuccess || !graph) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    cache.erase(key);
    return rc ? rc : LIBSHALOM_ERR_CUDA;
  }
  const cudaError_t ie = cudaGraphInstantiate(&ge.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) {
    cudaGetLastError();
    cache.erase(key);
    return LIBSHALOM_ERR_CUDA;
  }
  ge.generation = st.ws_generation;
  ++ge.uses;
  LS_CUDA_TRY(cudaGraphLaunch(ge.exec, st.stream));
  return finish_launch("gemm (graph)");
}

}  // namespace ls

// ---------------------------------------------------------------------------
// Host-memory calls.  The reference's API takes host pointers; these entry
// points do too.  Operands go through a device staging buffer of three slots:
// a call is cut into chunks of whole GEMMs that rotate over the slots, with
// the host->device copies on one stream, the kernels on the library's stream
// and the device->host copies on a third, ordered by per-slot events.  Both
// copy directions and the kernels of neighbouring chunks (and of consecutive
// calls) overlap; page-locked host memory makes the copies asynchronous.
// ---------------------------------------------------------------------------
namespace ls {

static constexpr size_t HS_CHUNK_BYTES = 64u << 20;  // target operand bytes per chunk

static void host_staging_release() {
  State &st = state();
  if (st.hs_in) cudaStreamSynchronize(st.hs_in);
  if (st.hs_out) cudaStreamSynchronize(st.hs_out);
  if (st.hs) cudaFree(st.hs);
  for (int i = 0; i < 3; ++i) {
    if (st.hs_ev_in[i]) cudaEventDestroy(st.hs_ev_in[i]);
    if (st.hs_ev_done[i]) cudaEventDestroy(st.hs_ev_done[i]);
    if (st.hs_ev_out[i]) cudaEventDestroy(st.hs_ev_out[i]);
    st.hs_ev_in[i] = st.hs_ev_done[i] = st.hs_ev_out[i] = nullptr;
  }
  if (st.hs_in) cudaStreamDestroy(st.hs_in);
  if (st.hs_out) cudaStreamDestroy(st.hs_out);
  st.hs_in = st.hs_out = nullptr;
  st.hs = nullptr;
  st.hs_slot_bytes = 0;
  st.hs_device = -1;
}

// Staging slots of at least slot_bytes each, the copy streams and events of
// the current device.
static int host_staging(size_t slot_bytes) {
  State &st = state();
  if (st.hs_device != st.device) {
    if (st.hs_device >= 0) {
      // the staging of another device: finish its work and drop it
      int cur = st.device;
      cudaSetDevice(st.hs_device);
      host_staging_release();
      cudaSetDevice(cur);
    }
    LS_CUDA_TRY(cudaStreamCreateWithFlags(&st.hs_in, cudaStreamNonBlocking));
    LS_CUDA_TRY(cudaStreamCreateWithFlags(&st.hs_out, cudaStreamNonBlocking));
    for (int i = 0; i < 3; ++i) {
      LS_CUDA_TRY(cudaEventCreateWithFlags(&st.hs_ev_in[i], cudaEventDisableTiming));
      LS_CUDA_TRY(cudaEventCreateWithFlags(&st.hs_ev_done[i], cudaEventDisableTiming));
      LS_CUDA_TRY(cudaEventCreateWithFlags(&st.hs_ev_out[i], cudaEventDisableTiming));
    }
    st.hs_device = st.device;
  }
  if (st.hs && st.hs_slot_bytes >= slot_bytes) return LIBSHALOM_SUCCESS;
  if (st.hs) {
    // copies and kernels queued earlier may still use the old slots
    LS_CUDA_TRY(cudaStreamSynchronize(st.hs_in));
    LS_CUDA_TRY(cudaStreamSynchronize(st.stream));
    LS_CUDA_TRY(cudaStreamSynchronize(st.hs_out));
    cudaFree(st.hs);
    st.hs = nullptr;
    st.hs_slot_bytes = 0;
  }
  const size_t want = (std::max(slot_bytes, (size_t)1 << 20) + 255) / 256 * 256;
  if (cudaMalloc(&st.hs, 3 * want) != cudaSuccess) {
    cudaGetLastError();
    st.hs = nullptr;
    return LIBSHALOM_ERR_ALLOC;
  }
  st.hs_slot_bytes = want;
  return LIBSHALOM_SUCCESS;
}

// elements a chunk of n matrices of `elems` elements at host stride `stride`
// occupies in a slot: the host span itself when matrices overlap or touch
// (stride <= elems, device stride = stride), else packed (device stride = elems)
static long staged_elems(long n, long elems, long stride) {
  if (elems == 0 || n == 0) return 0;
  return stride <= elems ? (n - 1) * stride + elems : n * elems;
}
static long staged_stride(long elems, long stride) { return stride <= elems ? stride : elems; }

template <typename T>
static int copy_in(T *dst, const T *src, long n, long elems, long stride, cudaStream_t s) {
  if (elems == 0 || n == 0) return LIBSHALOM_SUCCESS;
  if (stride <= elems) {
    LS_CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(T) * staged_elems(n, elems, stride),
                                cudaMemcpyHostToDevice, s));
  } else {
    LS_CUDA_TRY(cudaMemcpy2DAsync(dst, sizeof(T) * elems, src, sizeof(T) * stride,
                                  sizeof(T) * elems, n, cudaMemcpyHostToDevice, s));
  }
  return LIBSHALOM_SUCCESS;
}

static size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// count GEMMs (matrix g of A at A + g * sA, ...) through the staging slots;
// compute(dA, dB, dC, dsA, dsB, dsC, g0, n) launches the kernels of GEMMs
// g0 .. g0 + n - 1 on the library's stream.  C (elems_c per GEMM) must not
// overlap between GEMMs; it is copied in only when c_in.
template <typename T, typename Compute>
static int host_pipeline(long count, long elems_a, long sA, const T *A, long elems_b, long sB,
                         const T *B, long elems_c, long sC, T *C, bool c_in, Compute compute) {
  State &st = state();
  const size_t per = sizeof(T) * (size_t)(elems_a + elems_b + elems_c);
  const long cc = std::max(1L, std::min(count, (long)(HS_CHUNK_BYTES / std::max(per, (size_t)1))));
  const size_t off_b = align256(sizeof(T) * staged_elems(cc, elems_a, sA));
  const size_t off_c = off_b + align256(sizeof(T) * staged_elems(cc, elems_b, sB));
  const size_t slot = off_c + align256(sizeof(T) * (size_t)cc * elems_c);
  int rc = host_staging(slot);
  if (rc) return rc;
  const long dsA = staged_stride(elems_a, sA), dsB = staged_stride(elems_b, sB);
  int last = -1;
  for (long g0 = 0; g0 < count; g0 += cc) {
    const long n = std::min(cc, count - g0);
    const int s = (int)(st.hs_next++ % 3);
    unsigned char *base = static_cast<unsigned char *>(st.hs) + (size_t)s * st.hs_slot_bytes;
    T *dA = reinterpret_cast<T *>(base), *dB = reinterpret_cast<T *>(base + off_b);
    T *dC = reinterpret_cast<T *>(base + off_c);
    // the slot's previous chunk has been computed and copied out
    LS_CUDA_TRY(cudaStreamWaitEvent(st.hs_in, st.hs_ev_out[s], 0));
    if ((rc = copy_in(dA, A + g0 * sA, n, elems_a, sA, st.hs_in))) return rc;
    if ((rc = copy_in(dB, B + g0 * sB, n, elems_b, sB, st.hs_in))) return rc;
    if (c_in && (rc = copy_in(dC, C + g0 * sC, n, elems_c, sC, st.hs_in))) return rc;
    LS_CUDA_TRY(cudaEventRecord(st.hs_ev_in[s], st.hs_in));
    LS_CUDA_TRY(cudaStreamWaitEvent(st.stream, st.hs_ev_in[s], 0));
    if ((rc = compute(dA, dB, dC, dsA, dsB, elems_c, g0, n))) return rc;
    LS_CUDA_TRY(cudaEventRecord(st.hs_ev_done[s], st.stream));
    LS_CUDA_TRY(cudaStreamWaitEvent(st.hs_out, st.hs_ev_done[s], 0));
    if (sC == elems_c || n == 1)
      LS_CUDA_TRY(cudaMemcpyAsync(C + g0 * sC, dC, sizeof(T) * (size_t)n * elems_c,
                                  cudaMemcpyDeviceToHost, st.hs_out));
    else
      LS_CUDA_TRY(cudaMemcpy2DAsync(C + g0 * sC, sizeof(T) * sC, dC, sizeof(T) * elems_c,
                                    sizeof(T) * elems_c, n, cudaMemcpyDeviceToHost,
                                    st.hs_out));
    LS_CUDA_TRY(cudaEventRecord(st.hs_ev_out[s], st.hs_out));
    last = s;
  }
  // the caller's stream is ordered after the last copy out
  if (last >= 0) LS_CUDA_TRY(cudaStreamWaitEvent(st.stream, st.hs_ev_out[last], 0));
  return finish_launch("host pipeline");
}

template <typename T>
static int gemm_host(int transa, int transb, T *C, const T *A, const T *B, long M, long N,
                     long K, bool mp) {
  if ((transa != NoTrans && transa != Trans) || (transb != NoTrans && transb != Trans) ||
      M < 0 || N < 0 || K < 0)
    return LIBSHALOM_ERR_INVALID_VALUE;
  if (M == 0 || N == 0) return LIBSHALOM_SUCCESS;
  if (!C || (K > 0 && (!A || !B))) return LIBSHALOM_ERR_INVALID_VALUE;
  int rc = ensure_device();
  if (rc) return rc;
  auto compute = [&](T *dA, T *dB, T *dC, long, long, long, long, long) {
    return gemm_common<T>(transa, transb, dC, dA, dB, M, N, K, mp);
  };
  return host_pipeline<T>(1, M * K, M * K, A, K * N, K * N, B, M * N, M * N, C, false, compute);
}

}  // namespace ls

// ---------------------------------------------------------------------------
// Deferred drop-in calls: a host-pinned descriptor ring.  Between
// LibShalom_defer_begin and LibShalom_defer_flush the drop-in calls record an
// entry (pointers, sizes) in page-locked host memory instead of launching; the
// flush copies the FP32 and the FP64 entries to the device in one transfer
// each and runs them as grouped batches, so N small calls cost two or three
// launches instead of N.  Recorded calls keep their sequential meaning for
// exact-pointer aliasing: a call that reads a matrix an earlier pending call
// writes, writes a matrix an earlier pending call reads, or writes a C an
// earlier pending call wrote (other than the directly preceding call with
// the same M and N, which the grouped kernels apply in order) first flushes
// the pending calls.  Calls whose matrices overlap without sharing a base
// pointer are the caller's to keep apart.
// ---------------------------------------------------------------------------
namespace ls {

struct DeferSets {
  std::unordered_set<const void *> reads, writes;
  const void *last_c = nullptr;
  long last_m = -1, last_n = -1;
  void clear() {
    reads.clear();
    writes.clear();
    last_c = nullptr;
    last_m = last_n = -1;
  }
};
static DeferSets &defer_sets() {
  static DeferSets d;
  return d;
}

// no flush's copy still reads the rings
static int ring_idle() {
  State &st = state();
  if (st.ring_busy) {
    LS_CUDA_TRY(cudaEventSynchronize(st.ring_ev));
    st.ring_busy = false;
  }
  return LIBSHALOM_SUCCESS;
}

template <typename E>
static int ring_grow(E **ring, long *cap, long need) {
  if (need <= *cap) return LIBSHALOM_SUCCESS;
  long ncap = std::max(need, std::max(256L, 2 * *cap));
  E *n = nullptr;
  if (cudaHostAlloc(reinterpret_cast<void **>(&n), sizeof(E) * (size_t)ncap,
                    cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return LIBSHALOM_ERR_ALLOC;
  }
  if (*ring) {
    memcpy(n, *ring, sizeof(E) * (size_t)*cap);
    cudaFreeHost(*ring);
  }
  *ring = n;
  *cap = ncap;
  return LIBSHALOM_SUCCESS;
}

// launches the pending entries (stream-ordered) and empties the rings
static int defer_launch() {
  State &st = state();
  DeferSets &ds = defer_sets();
  const long ns = st.ring_s_n, nd = st.ring_d_n;
  ds.clear();
  if (ns == 0 && nd == 0) return LIBSHALOM_SUCCESS;
  st.ring_s_n = st.ring_d_n = 0;
  int rc = ensure_device();
  if (rc) return rc;
  if (!st.ring_ev) LS_CUDA_TRY(cudaEventCreateWithFlags(&st.ring_ev, cudaEventDisableTiming));
  const size_t bs = sizeof(LibShalom_sgemm_entry) * (size_t)ns;
  const size_t bd = sizeof(LibShalom_dgemm_entry) * (size_t)nd;
  void *buf = nullptr;
  if ((rc = frontend_buffer((bs + 255) / 256 * 256 + bd, &buf))) return rc;
  auto *dev_s = static_cast<LibShalom_sgemm_entry *>(buf);
  auto *dev_d = reinterpret_cast<LibShalom_dgemm_entry *>(static_cast<unsigned char *>(buf) +
                                                          (bs + 255) / 256 * 256);
  if (ns) LS_CUDA_TRY(cudaMemcpyAsync(dev_s, st.ring_s, bs, cudaMemcpyHostToDevice, st.stream));
  if (nd) LS_CUDA_TRY(cudaMemcpyAsync(dev_d, st.ring_d, bd, cudaMemcpyHostToDevice, st.stream));
  LS_CUDA_TRY(cudaEventRecord(st.ring_ev, st.stream));
  st.ring_busy = true;
  if (ns)
    rc = st.precision == LIBSHALOM_PREC_FP32 ? run_grouped_s(dev_s, ns)
                                             : tc_sgemm_grouped(dev_s, ns, st.precision);
  if (!rc && nd)
    rc = st.dgemm_method == LIBSHALOM_DGEMM_FMA
             ? run_grouped_d(dev_d, nd)
             : run_dgemm_warp(dev_d, nd, st.dgemm_method, st.ozaki_slices);
  if (rc) return rc;
  return finish_launch("defer_flush");
}

int flush_deferred() {
  State &st = state();
  if (st.ring_s_n == 0 && st.ring_d_n == 0) {
    defer_sets().clear();
    return LIBSHALOM_SUCCESS;
  }
  int cur = -1;
  LS_CUDA_TRY(cudaGetDevice(&cur));
  if (st.ring_device < 0 || cur == st.ring_device) return defer_launch();
  // the pending calls name memory of the device they were recorded on
  LS_CUDA_TRY(cudaSetDevice(st.ring_device));
  const int rc = defer_launch();
  LS_CUDA_TRY(cudaSetDevice(cur));
  return rc;
}

// Largest call worth recording (M N K): the grouped kernels give each call to
// one CTA, so a larger call runs faster directly, over many CTAs.
constexpr double DEFER_MAX_MNK = 2097152.0;  // 128^3

// Records a drop-in call while deferring.  Returns 1 when the call was
// recorded (or is an empty problem, or failed), 0 when it must run directly
// (transa, or M N K above DEFER_MAX_MNK) after the pending calls.
template <typename T>
static int defer_record(int transa, int transb, T *C, const T *A, const T *B, long M, long N,
                        long K, int *status) {
  State &st = state();
  *status = LIBSHALOM_SUCCESS;
  if ((transa != NoTrans && transa != Trans) || (transb != NoTrans && transb != Trans) ||
      M < 0 || N < 0 || K < 0) {
    *status = LIBSHALOM_ERR_INVALID_VALUE;
    return 1;
  }
  if (M == 0 || N == 0) return 1;
  if (!C || (K > 0 && (!A || !B))) {
    *status = LIBSHALOM_ERR_INVALID_VALUE;
    return 1;
  }
  int rc = ensure_device();
  if (!rc && st.ring_s_n + st.ring_d_n > 0 && st.device != st.ring_device)
    rc = flush_deferred();  // calls recorded on another device run there first
  if (rc) {
    *status = rc;
    return 1;
  }
  DeferSets &ds = defer_sets();
  const bool fits = transa == NoTrans && (double)M * (double)N * (double)K <= DEFER_MAX_MNK;
  const bool waw_ok = C == ds.last_c && M == ds.last_m && N == ds.last_n;
  const bool hazard = ds.writes.count(A) || ds.writes.count(B) || ds.reads.count(C) ||
                      (ds.writes.count(C) && !waw_ok);
  if (!fits || hazard) {
    // run (or start a new batch) after everything recorded so far
    rc = defer_launch();
    if (rc) {
      *status = rc;
      return 1;
    }
    if (!fits) return 0;
  }
  rc = ring_idle();
  if (!rc) {
    if (sizeof(T) == 4) rc = ring_grow(&st.ring_s, &st.ring_s_cap, st.ring_s_n + 1);
    else rc = ring_grow(&st.ring_d, &st.ring_d_cap, st.ring_d_n + 1);
  }
  if (rc) {
    *status = rc;
    return 1;
  }
  const int32_t ldb = (int32_t)(transb ? K : N);
  if (st.ring_s_n + st.ring_d_n == 0) st.ring_device = st.device;
  if (sizeof(T) == 4) {
    LibShalom_sgemm_entry &e = st.ring_s[st.ring_s_n++];
    e.A = reinterpret_cast<const float *>(A);
    e.B = reinterpret_cast<const float *>(B);
    e.C = reinterpret_cast<float *>(C);
    e.M = (int32_t)M; e.N = (int32_t)N; e.K = (int32_t)K; e.transb = transb;
    e.lda = (int32_t)K; e.ldb = ldb; e.ldc = (int32_t)N;
    e.alpha = 1.0f; e.beta = 0.0f; e.reserved = 0;
  } else {
    LibShalom_dgemm_entry &e = st.ring_d[st.ring_d_n++];
    e.A = reinterpret_cast<const double *>(A);
    e.B = reinterpret_cast<const double *>(B);
    e.C = reinterpret_cast<double *>(C);
    e.M = (int32_t)M; e.N = (int32_t)N; e.K = (int32_t)K; e.transb = transb;
    e.lda = (int32_t)K; e.ldb = ldb; e.ldc = (int32_t)N;
    e.alpha = 1.0; e.beta = 0.0; e.reserved = 0;
  }
  ds.reads.insert(A);
  ds.reads.insert(B);
  ds.writes.insert(C);
  ds.last_c = C;
  ds.last_m = M;
  ds.last_n = N;
  return 1;
}

// Operand classification of the drop-in calls.  The reference's callers pass
// malloc'd HOST buffers to LibShalom_sgemm / _sgemm_mp / _dgemm (its
// Hello.c:13-37 does exactly that); this library's drop-ins take device
// memory.  A call whose operands include host memory (pageable or page-locked)
// therefore runs through the host-memory pipeline of the _host calls instead
// of handing host addresses to a kernel.  Device and managed memory run on
// the device path.  Under unified addressing an address that was device
// memory once stays a device address, so device pointers are remembered.
static bool is_host_memory(const void *p) {
  static const void *seen[32] = {};
  static unsigned next = 0;
  if (!p) return false;
  for (const void *q : seen)
    if (q == p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;  // not classifiable: left to the device path's own checks
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) {
    seen[next++ % 32] = p;
    return false;
  }
  return true;  // cudaMemoryTypeHost (page-locked) or cudaMemoryTypeUnregistered
}

// the drop-in calls: host operands through the host pipeline; recorded while
// deferring; else run now
template <typename T>
static int dropin(int kind, int transa, int transb, T *C, const T *A, const T *B, long M,
                  long N, long K, bool mp) {
  const bool args_ok = (transa == NoTrans || transa == Trans) &&
                       (transb == NoTrans || transb == Trans) && M > 0 && N > 0 && K >= 0 &&
                       C && (K == 0 || (A && B));
  if (args_ok && ensure_device() == LIBSHALOM_SUCCESS &&
      (is_host_memory(C) || (K > 0 && (is_host_memory(A) || is_host_memory(B))))) {
    const int rc = flush_deferred();
    return rc ? rc : gemm_host<T>(transa, transb, C, A, B, M, N, K, mp);
  }
  if (state().deferring) {
    int status = LIBSHALOM_SUCCESS;
    if (defer_record<T>(transa, transb, C, A, B, M, N, K, &status) != 0) return status;
  }
  return gemm_cached<T>(kind, transa, transb, C, A, B, M, N, K, mp);
}

}  // namespace ls

using namespace ls;

extern "C" {

void LibShalom_sgemm(int transa, int transb, float *C, float *A, float *B, long M, long N,
                     long K) {
  std::lock_guard<std::mutex> lk(state().mu);
  set_error(dropin<float>(0, transa, transb, C, A, B, M, N, K, false));
}

void LibShalom_sgemm_mp(int transa, int transb, float *C, float *A, float *B, long M, long N,
                        long K) {
  std::lock_guard<std::mutex> lk(state().mu);
  set_error(dropin<float>(1, transa, transb, C, A, B, M, N, K, true));
}

void LibShalom_dgemm(int transa, int transb, double *C, double *A, double *B, long M, long N,
                     long K) {
  std::lock_guard<std::mutex> lk(state().mu);
  set_error(dropin<double>(2, transa, transb, C, A, B, M, N, K, false));
}

int LibShalom_defer_begin(void) {
  std::lock_guard<std::mutex> lk(state().mu);
  state().deferring = 1;
  set_error(LIBSHALOM_SUCCESS);
  return LIBSHALOM_SUCCESS;
}

int LibShalom_defer_flush(void) {
  std::lock_guard<std::mutex> lk(state().mu);
  const int rc = defer_launch();
  state().deferring = 0;
  set_error(rc);
  return rc;
}

int LibShalom_defer_pending(void) {
  std::lock_guard<std::mutex> lk(state().mu);
  const long n = state().ring_s_n + state().ring_d_n;
  return (int)std::min(n, (long)INT32_MAX);
}

// The setters below change how later calls launch; calls still pending in a
// deferred section are launched first, under the settings they were made with.

void LibShalom_set_thread_nums(int num) {
  std::lock_guard<std::mutex> lk(state().mu);
  const int rc = flush_deferred();
  if (!rc) state().thread_cap = num > 0 ? num : 0;
  set_error(rc);
}

void LibShalom_set_thread_ways(int tm, int tn) {
  std::lock_guard<std::mutex> lk(state().mu);
  if (tm <= 0 || tn <= 0) {
    set_error(LIBSHALOM_ERR_INVALID_VALUE);
    return;
  }
  state().ways_m = tm;
  state().ways_n = tn;
  set_error(LIBSHALOM_SUCCESS);
}

int LibShalom_get_last_error(void) { return last_error(); }

const char *LibShalom_error_string(int status) {
  switch (status) {
    case LIBSHALOM_SUCCESS: return "success";
    case LIBSHALOM_ERR_INVALID_VALUE: return "invalid argument";
    case LIBSHALOM_ERR_UNSUPPORTED: return "unsupported request";
    case LIBSHALOM_ERR_CUDA: return "CUDA runtime error";
    case LIBSHALOM_ERR_NO_DEVICE: return "no sm_100 device";
    case LIBSHALOM_ERR_ALLOC: return "device workspace allocation failed";
    case LIBSHALOM_ERR_DEVICE_TIMEOUT: return "bounded device wait expired";
  }
  return "unknown status";
}

int LibShalom_set_stream(void *stream) {
  std::lock_guard<std::mutex> lk(state().mu);
  State &st = state();
  const int rc = flush_deferred();
  cudaStream_t next = reinterpret_cast<cudaStream_t>(stream);
  if (!rc && next != st.stream) {
    // The library's device buffers (workspace, front-end buffer, the copy of
    // the deferred entries) are handed from call to call in stream order.
    // Work queued on the old stream may still read them, so it is finished
    // before calls on the new stream can overwrite them.  (A stream the
    // caller has already destroyed reports an error here, which is ignored:
    // its queued work completes anyway.)
    if (st.ws || st.fe) {
      if (cudaStreamSynchronize(st.stream) != cudaSuccess) cudaGetLastError();
    }
    st.stream = next;
  }
  set_error(rc);
  return rc;
}

int LibShalom_set_sync(int synchronous) {
  std::lock_guard<std::mutex> lk(state().mu);
  state().sync = synchronous ? 1 : 0;
  set_error(LIBSHALOM_SUCCESS);
  return LIBSHALOM_SUCCESS;
}

int LibShalom_synchronize(void) {
  std::lock_guard<std::mutex> lk(state().mu);
  cudaError_t e = cudaStreamSynchronize(state().stream);
  int rc = e == cudaSuccess ? LIBSHALOM_SUCCESS : LIBSHALOM_ERR_CUDA;
  if (rc) note_cuda_error(e, "cudaStreamSynchronize", __FILE__, __LINE__);
  set_error(rc);
  return rc;
}

int LibShalom_set_precision(int mode) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = LIBSHALOM_SUCCESS;
  if (mode != LIBSHALOM_PREC_FP32 && mode != LIBSHALOM_PREC_BF16X3 &&
      mode != LIBSHALOM_PREC_BF16X6)
    rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (!(rc = flush_deferred()))
    state().precision = mode;
  set_error(rc);
  return rc;
}

int LibShalom_get_precision(void) { return state().precision; }

int LibShalom_set_dgemm_method(int method, int slices) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = LIBSHALOM_SUCCESS;
  if (method != LIBSHALOM_DGEMM_FMA && method != LIBSHALOM_DGEMM_DMMA &&
      method != LIBSHALOM_DGEMM_OZAKI)
    rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (slices != 0 && (slices < 4 || slices > 9))
    rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (!(rc = flush_deferred())) {
    state().dgemm_method = method;
    state().ozaki_slices = slices == 0 ? 9 : slices;
  }
  set_error(rc);
  return rc;
}

int LibShalom_get_dgemm_method(void) { return state().dgemm_method; }

int LibShalom_set_graph_cache(int enable) {
  std::lock_guard<std::mutex> lk(state().mu);
  state().graph_cache = enable != 0;
  if (!enable) graph_cache_clear();
  set_error(LIBSHALOM_SUCCESS);
  return LIBSHALOM_SUCCESS;
}

int LibShalom_set_tile_config(int cfg) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = LIBSHALOM_SUCCESS;
  if (cfg < -1 || cfg > 6) rc = LIBSHALOM_ERR_INVALID_VALUE;
  else state().tile_cfg = cfg;
  set_error(rc);
  return rc;
}

int LibShalom_set_autotune(int enable) {
  std::lock_guard<std::mutex> lk(state().mu);
  state().autotune = enable != 0;
  set_error(LIBSHALOM_SUCCESS);
  return LIBSHALOM_SUCCESS;
}

int LibShalom_get_plan(int *tile_config, int *splits, int *table_entries) {
  std::lock_guard<std::mutex> lk(state().mu);
  if (tile_config) *tile_config = state().last_cfg;
  if (splits) *splits = state().last_splits;
  if (table_entries) *table_entries = tune_table_size();
  set_error(LIBSHALOM_SUCCESS);
  return LIBSHALOM_SUCCESS;
}

int LibShalom_set_splitk(int splits) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = LIBSHALOM_SUCCESS;
  if (splits < 0) rc = LIBSHALOM_ERR_INVALID_VALUE;
  else state().splitk = splits;
  set_error(rc);
  return rc;
}

int LibShalom_set_tma(int enable) {
  std::lock_guard<std::mutex> lk(state().mu);
  state().use_tma = enable != 0;
  set_error(LIBSHALOM_SUCCESS);
  return LIBSHALOM_SUCCESS;
}

void LibShalom_finalize(void) {
  std::lock_guard<std::mutex> lk(state().mu);
  State &st = state();
  // calls still pending in a deferred section run before anything is freed
  const int flushed = flush_deferred();
  if (st.ws || st.fe) cudaStreamSynchronize(st.stream);
  graph_cache_clear();
  if (st.ring_busy && st.ring_ev) cudaEventSynchronize(st.ring_ev);
  if (st.ring_ev) cudaEventDestroy(st.ring_ev);
  if (st.ring_s) cudaFreeHost(st.ring_s);
  if (st.ring_d) cudaFreeHost(st.ring_d);
  st.ring_ev = nullptr;
  st.ring_s = nullptr;
  st.ring_d = nullptr;
  st.ring_s_n = st.ring_s_cap = st.ring_d_n = st.ring_d_cap = 0;
  st.ring_busy = false;
  st.deferring = 0;
  defer_sets().clear();
  if (st.hs_device >= 0) {
    int cur = -1;
    cudaGetDevice(&cur);
    cudaSetDevice(st.hs_device);
    host_staging_release();
    if (cur >= 0) cudaSetDevice(cur);
  }
  if (st.ws) cudaFree(st.ws);
  if (st.fe) cudaFree(st.fe);
  st.ws = nullptr;
  st.ws_bytes = 0;
  st.ws_device = -1;
  st.fe = nullptr;
  st.fe_bytes = 0;
  st.fe_device = -1;
  st.ring_device = -1;
  set_error(flushed);
}

int LibShalom_selftest_wait_expiry(int iterations) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = iterations < 0 ? LIBSHALOM_ERR_INVALID_VALUE : flush_deferred();
  if (!rc) rc = ensure_device();
  if (!rc) rc = tc_wait_expiry_selftest(iterations);
  set_error(rc);
  return rc;
}

static bool entries_ok(const void *entries, long count) {
  return count >= 0 && (count == 0 || entries != nullptr);
}

int LibShalom_sgemm_batched(const LibShalom_sgemm_entry *entries, long count) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = LIBSHALOM_SUCCESS;
  if (!entries_ok(entries, count)) rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (count > 0 && !(rc = flush_deferred()) && !(rc = ensure_device())) {
    if (state().precision == LIBSHALOM_PREC_FP32) rc = run_grouped_s(entries, count);
    else rc = tc_sgemm_grouped(entries, count, state().precision);
    if (!rc) rc = finish_launch("sgemm_batched");
  }
  set_error(rc);
  return rc;
}

int LibShalom_sgemm_batched_strided(int transb, long M, long N, long K, float alpha,
                                    const float *A, long strideA, const float *B, long strideB,
                                    float beta, float *C, long strideC, long count) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = LIBSHALOM_SUCCESS;
  if ((transb != NoTrans && transb != Trans) || M < 0 || N < 0 || K < 0 || count < 0 ||
      strideA < 0 || strideB < 0 || strideC < 0)
    rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (count > 0 && M > 0 && N > 0 && (!C || (K > 0 && (!A || !B))))
    rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (count > 0 && M > 0 && N > 0 && !(rc = flush_deferred()) && !(rc = ensure_device())) {
    GemmArgs<float> g;
    g.A = A; g.B = B; g.C = C;
    g.M = M; g.N = N; g.K = K;
    g.transa = 0; g.transb = transb;
    g.lda = K; g.ldb = transb ? K : N; g.ldc = N;
    g.alpha = alpha; g.beta = beta;
    if (state().precision == LIBSHALOM_PREC_FP32)
      rc = run_strided<float>(g, strideA, strideB, strideC, count);
    else
      rc = tc_sgemm_strided(g, strideA, strideB, strideC, count, state().precision);
    if (!rc) rc = finish_launch("sgemm_batched_strided");
  }
  set_error(rc);
  return rc;
}

int LibShalom_sgemm_batched_strided_host(int transb, long M, long N, long K, float alpha,
                                         const float *A, long strideA, const float *B,
                                         long strideB, float beta, float *C, long strideC,
                                         long count) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = LIBSHALOM_SUCCESS;
  if ((transb != NoTrans && transb != Trans) || M < 0 || N < 0 || K < 0 || count < 0 ||
      strideA < 0 || strideB < 0 || strideC < 0)
    rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (count > 1 && strideC < M * N)
    rc = LIBSHALOM_ERR_INVALID_VALUE;  // the copies out would overlap
  else if (count > 0 && M > 0 && N > 0 && (!C || (K > 0 && (!A || !B))))
    rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (count > 0 && M > 0 && N > 0 && !(rc = flush_deferred()) && !(rc = ensure_device())) {
    const int prec = state().precision;
    auto compute = [&](float *dA, float *dB, float *dC, long dsA, long dsB, long dsC, long,
                       long n) {
      GemmArgs<float> g;
      g.A = dA; g.B = dB; g.C = dC;
      g.M = M; g.N = N; g.K = K;
      g.transa = 0; g.transb = transb;
      g.lda = K; g.ldb = transb ? K : N; g.ldc = N;
      g.alpha = alpha; g.beta = beta;
      const int r = prec == LIBSHALOM_PREC_FP32
                        ? run_strided<float>(g, dsA, dsB, dsC, n)
                        : tc_sgemm_strided(g, dsA, dsB, dsC, n, prec);
      if (r) return r;
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) {
        note_cuda_error(e, "sgemm_batched_strided_host", __FILE__, __LINE__);
        return (int)LIBSHALOM_ERR_CUDA;
      }
      return (int)LIBSHALOM_SUCCESS;
    };
    rc = host_pipeline<float>(count, M * K, strideA, A, K * N, strideB, B, M * N,
                              count > 1 ? strideC : M * N, C, beta != 0.0f, compute);
  }
  set_error(rc);
  return rc;
}

void LibShalom_sgemm_host(int transa, int transb, float *C, const float *A, const float *B,
                          long M, long N, long K) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = flush_deferred();
  if (!rc) rc = gemm_host<float>(transa, transb, C, A, B, M, N, K, false);
  set_error(rc);
}

void LibShalom_sgemm_mp_host(int transa, int transb, float *C, const float *A, const float *B,
                             long M, long N, long K) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = flush_deferred();
  if (!rc) rc = gemm_host<float>(transa, transb, C, A, B, M, N, K, true);
  set_error(rc);
}

void LibShalom_dgemm_host(int transa, int transb, double *C, const double *A, const double *B,
                          long M, long N, long K) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = flush_deferred();
  if (!rc) rc = gemm_host<double>(transa, transb, C, A, B, M, N, K, false);
  set_error(rc);
}

int LibShalom_dgemm_batched(const LibShalom_dgemm_entry *entries, long count) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = LIBSHALOM_SUCCESS;
  if (!entries_ok(entries, count)) rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (count > 0 && !(rc = flush_deferred()) && !(rc = ensure_device())) {
    const State &st = state();
    rc = st.dgemm_method == LIBSHALOM_DGEMM_FMA
             ? run_grouped_d(entries, count)
             : run_dgemm_warp(entries, count, st.dgemm_method, st.ozaki_slices);
    if (!rc) rc = finish_launch("dgemm_batched");
  }
  set_error(rc);
  return rc;
}

int LibShalom_sgemm_ex(int transa, int transb, long M, long N, long K, float alpha,
                       const float *A, long lda, const float *B, long ldb, float beta, float *C,
                       long ldc) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = flush_deferred();
  if (!rc)
    rc = gemm_common<float>(transa, transb, C, A, B, M, N, K, true, alpha, beta,
                                    std::max(lda, 1L), std::max(ldb, 1L), std::max(ldc, 1L));
  set_error(rc);
  return rc;
}

int LibShalom_dgemm_ex(int transa, int transb, long M, long N, long K, double alpha,
                       const double *A, long lda, const double *B, long ldb, double beta,
                       double *C, long ldc) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = flush_deferred();
  if (!rc)
    rc = gemm_common<double>(transa, transb, C, A, B, M, N, K, true, alpha, beta,
                                     std::max(lda, 1L), std::max(ldb, 1L), std::max(ldc, 1L));
  set_error(rc);
  return rc;
}

int LibShalom_dgemm_stack(const LibShalom_dgemm_stack_desc *stack, long count) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = LIBSHALOM_SUCCESS;
  if (!stack || count < 0 || count > (1L << 30)) rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (count > 0 && (!stack->a_off || !stack->b_off || !stack->c_off || !stack->C_pool ||
                         ((!stack->M && stack->m < 0) || (!stack->N && stack->n < 0) ||
                          (!stack->K && stack->k < 0)) ||
                         (stack->transb != NoTrans && stack->transb != Trans)))
    rc = LIBSHALOM_ERR_INVALID_VALUE;
  else if (count > 0 && !(rc = flush_deferred()) && !(rc = ensure_device())) {
    void *buf = nullptr;
    rc = frontend_buffer(sizeof(LibShalom_dgemm_entry) * (size_t)count, &buf);
    if (!rc) {
      StackArgs a;
      a.A = stack->A_pool; a.B = stack->B_pool; a.C = stack->C_pool;
      a.M = stack->M; a.N = stack->N; a.K = stack->K;
      a.m = stack->m; a.n = stack->n; a.k = stack->k; a.transb = stack->transb;
      a.a_off = stack->a_off; a.b_off = stack->b_off; a.c_off = stack->c_off;
      a.alpha = stack->alpha; a.beta = stack->beta;
      auto *ent = static_cast<LibShalom_dgemm_entry *>(buf);
      rc = stack_to_entries(a, count, ent);
      if (!rc) {
        const State &st = state();
        rc = st.dgemm_method == LIBSHALOM_DGEMM_FMA
                 ? run_grouped_d(ent, count)
                 : run_dgemm_warp(ent, count, st.dgemm_method, st.ozaki_slices);
      }
      if (!rc) rc = finish_launch("dgemm_stack");
    }
  }
  set_error(rc);
  return rc;
}

int LibShalom_sconv2d_nchw(const float *x, long n, long c, long h, long w, const float *wt,
                           long oc, long kh, long kw, long sh, long sw, long ph, long pw,
                           float *y) {
  std::lock_guard<std::mutex> lk(state().mu);
  int rc = LIBSHALOM_SUCCESS;
  if (n < 0 || c <= 0 || h <= 0 || w <= 0 || oc <= 0 || kh <= 0 || kw <= 0 || sh <= 0 ||
      sw <= 0 || ph < 0 || pw < 0 || !x || !wt || !y)
    rc = LIBSHALOM_ERR_INVALID_VALUE;
  const long oh = (h + 2 * ph - kh) / sh + 1, ow = (w + 2 * pw - kw) / sw + 1;
  if (!rc && (h + 2 * ph < kh || w + 2 * pw < kw)) rc = LIBSHALOM_ERR_INVALID_VALUE;
  // the implicit GEMM indexes k = (ci, r, q) and p = (oy, ox) in int32
  const bool small_idx = c * kh * kw < INT32_MAX && oh * ow < INT32_MAX && c * h * w < INT32_MAX;
  if (!rc && n > 0 && state().precision == LIBSHALOM_PREC_FP32 && small_idx &&
      !(rc = flush_deferred()) && !(rc = ensure_device())) {
    // FP32: implicit GEMM, the tile loader gathers the im2col columns (no buffer)
    rc = conv_implicit(x, n, c, h, w, wt, oc, kh, kw, sh, sw, ph, pw, oh, ow, y);
    if (!rc) rc = finish_launch("sconv2d_nchw");
  } else if (!rc && n > 0 && !(rc = flush_deferred()) && !(rc = ensure_device())) {
    const long K = c * kh * kw, P = oh * ow;
    void *buf = nullptr;
    rc = frontend_buffer(sizeof(float) * (size_t)K * P, &buf);
    float *col = static_cast<float *>(buf);
    for (long i = 0; !rc && i < n; ++i) {
      rc = im2col(x + i * c * h * w, c, h, w, kh, kw, sh, sw, ph, pw, oh, ow, col);
      // y_i [oc][P] = wt [oc][K] col [K][P]
      if (!rc) rc = gemm_common<float>(NoTrans, NoTrans, y + i * oc * P, wt, col, oc, P, K, true);
    }
  }
  set_error(rc);
  return rc;
}

}  // extern "C"
