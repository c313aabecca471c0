// ls_common.cuh -- shared state, status codes and launch helpers of the
// B200 LibShalom library.  Host code only sees plain pointers and sizes;
// nothing here depends on torch.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/LibShalom.h"

namespace ls {

// ---------------------------------------------------------------------------
// status
// ---------------------------------------------------------------------------
void set_error(int status);  // records the status for this host thread
int last_error();

#define LS_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) {                                \
      ::ls::note_cuda_error(_e, #expr, __FILE__, __LINE__); \
      return LIBSHALOM_ERR_CUDA;                            \
    }                                                       \
  } while (0)

void note_cuda_error(cudaError_t e, const char *what, const char *file,
                     int line);

// ---------------------------------------------------------------------------
// library state (one instance per process; guarded by mu)
// ---------------------------------------------------------------------------
struct State {
  std::mutex mu;
  int device = -1;
  int num_sms = 0;
  int cc_major = 0, cc_minor = 0;
  size_t smem_optin = 0;
  cudaStream_t stream = nullptr;
  int sync = 1;
  int thread_cap = 0;        // LibShalom_set_thread_nums; <=0 = no cap
  int ways_m = 0, ways_n = 0;  // LibShalom_set_thread_ways (one-shot)
  int precision = LIBSHALOM_PREC_FP32;
  int dgemm_method = LIBSHALOM_DGEMM_FMA;
  int ozaki_slices = 9;
  int splitk = 0;
  int tile_cfg = -1;  // forced plain tile configuration (-1: table, then model)
  int autotune = 1;   // consult the measured shape-class table
  int last_cfg = -1, last_splits = 0;  // plan of the last single / mp call
  // tensor-core kernels: the TMA warp-specialized variant where the operands
  // allow it (LIBSHALOM_NO_TMA=1 in the environment selects the cp.async one)
  bool use_tma = true;
  // device workspace (split-K partials, work counters, work lists)
  void *ws = nullptr;
  size_t ws_bytes = 0;
  int ws_device = -1;
  // front-end buffer (stack entries, im2col columns): separate from the
  // workspace, which the GEMM paths the front ends call use themselves
  void *fe = nullptr;
  size_t fe_bytes = 0;
  int fe_device = -1;
  unsigned ws_generation = 0;  // bumped whenever the workspace moves
  int graph_cache = 0;         // replay repeated identical single / mp calls
  // host-memory calls: device staging of three slots, the two copy streams
  // and, per slot, the events "inputs copied", "computed", "output copied"
  void *hs = nullptr;
  size_t hs_slot_bytes = 0;
  int hs_device = -1;
  cudaStream_t hs_in = nullptr, hs_out = nullptr;
  cudaEvent_t hs_ev_in[3] = {}, hs_ev_done[3] = {}, hs_ev_out[3] = {};
  unsigned hs_next = 0;
  // deferred drop-in calls (LibShalom_defer_begin .. LibShalom_defer_flush):
  // entries in page-locked host rings, copied to the device in one transfer
  // per precision at the flush; ring_ev marks that transfer's completion
  int deferring = 0;
  LibShalom_sgemm_entry *ring_s = nullptr;
  LibShalom_dgemm_entry *ring_d = nullptr;
  long ring_s_n = 0, ring_s_cap = 0, ring_d_n = 0, ring_d_cap = 0;
  cudaEvent_t ring_ev = nullptr;
  bool ring_busy = false;  // a flush's copies may still read the rings
  int ring_device = -1;    // device current when the pending calls were recorded
};

State &state();

// Makes sure a device is current and its properties are cached.  Returns a
// LIBSHALOM_* status.
int ensure_device();

// Device workspace of at least `bytes` bytes (grown on demand, stream
// ordered: the caller's stream is synchronised before a regrow;
// LibShalom_set_stream finishes the old stream's work before a switch).
int workspace(size_t bytes, void **out);

// Launches the drop-in calls recorded since LibShalom_defer_begin (on the
// device that was current when they were recorded), so that whatever the
// caller does next is ordered after them.  No-op when nothing is pending.
int flush_deferred();

// Number of CTAs to launch for `work_items` independent items of a kernel
// with `per_sm` resident CTAs per SM, honouring LibShalom_set_thread_nums.
int grid_for(long work_items, int per_sm);

// Resident CTAs per SM of `kern` at `threads` threads and `smem` dynamic
// shared bytes (raises the kernel's dynamic shared-memory limit when needed;
// cached per kernel).  Returns `fallback` if the query fails.
int occupancy_of(const void *kern, int threads, size_t smem, int fallback);

// After a launch: check the launch, and synchronise when the library runs in
// synchronous mode.  Returns a LIBSHALOM_* status.
int finish_launch(const char *what);

inline long cdiv(long a, long b) { return (a + b - 1) / b; }

}  // namespace ls
