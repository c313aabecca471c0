// ls_dgemm.cu -- grouped FP64 GEMM (LibShalom_dgemm_batched) for the
// small-block workloads of atomic-orbital chemistry codes: tens of thousands
// of products with M, N, K of a few to a few dozen, where consecutive products
// accumulate into the same C block (C += A_p B_p).
//
// Work unit: one run (maximal group of consecutive entries naming the same C)
// and one 32 x 32 tile of its C block.  The CTA (256 threads, 4 outputs each)
// loads the C tile once, applies the run's products in array order with the C
// tile held in registers (C = alpha_p A_p op(B_p) + beta_p C), and writes it
// once -- the owner-computes rule that keeps shared C blocks race-free and the
// result deterministic without atomics.  Each product is a fused multiply-add
// chain over k in increasing order (the reference's KERNEL7x6 order) followed
// by C = fma(beta, C, alpha * acc).
//
// Runs are found on the device (k_drun_plan: one slot per run start), so the
// call needs no host round trip.
#include <cuda_runtime.h>

#include <algorithm>

#include "ls_common.cuh"
#include "ls_simt_launch.h"

namespace ls {

namespace {

constexpr int DR_T = 32;  // C tile edge

struct DrunPlan {
  unsigned *n_runs;
  unsigned *run_first;
  unsigned *run_len;
};

__global__ void k_drun_plan(const LibShalom_dgemm_entry *e, long count, DrunPlan pl) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count;
       i += (long)gridDim.x * blockDim.x) {
    if (i > 0 && e[i].C == e[i - 1].C) continue;
    long j = i + 1;
    while (j < count && e[j].C == e[i].C) ++j;
    const unsigned slot = atomicAdd(pl.n_runs, 1u);
    pl.run_first[slot] = (unsigned)i;
    pl.run_len[slot] = (unsigned)(j - i);
  }
}

__device__ __forceinline__ void cp_async8(uint32_t saddr, const void *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr), "l"(g) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// Ring-staged variant.  The CTA walks its sequence of items -- (run, 32 x 32
// C tile, product, K slice of up to 64) -- with a producer cursor running up
// to RG_Q items ahead of the consumer: every item's A and op(B) pieces are
// copied (8-byte cp.async, exact sizes, compact layouts) into the next free
// bytes of a 96 KB shared-memory ring, and each thread's copies arrive on the
// item's mbarrier when they land (cp.async.mbarrier.arrive.noinc).  So many
// small products are in flight at once instead of one fixed-size slab.  The
// producer and consumer cursors compute the same placements (same rule), so
// no queue is shared between them.
// ---------------------------------------------------------------------------
constexpr int RG_THREADS = 256;
constexpr int RG_KS = 64;                  // K slice of an item
constexpr int RG_RING = 96 * 1024;         // bytes
constexpr int RG_Q = 16;                   // items in flight (mbarrier slots)
constexpr int RG_SMEM = RG_RING + RG_Q * 8;

struct RgCursor {
  long r;       // run slot (round-robin over CTAs)
  int t, p, k;  // C tile, product, K slice
  bool valid;
};

struct RgItem {
  const double *A, *B;
  int transb, lda, ldb;
  int m0, n0, k0, mcnt, ncnt, kcnt;
  int bytes;  // staged bytes (A then B), 16-byte rounded
};

__device__ __forceinline__ bool rg_mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"((uint32_t)__cvta_generic_to_shared(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__global__ void __launch_bounds__(RG_THREADS, 2)
    k_dgemm_ring(const LibShalom_dgemm_entry *entries, const unsigned *n_runs_p,
                 const unsigned *run_first, const unsigned *run_len, unsigned *err) {
  extern __shared__ __align__(16) unsigned char rsm[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(rsm + RG_RING);
  const int tid = threadIdx.x;
  const long n_runs = (long)*n_runs_p;
  __shared__ int s_abort;
  if (tid == 0) {
    for (int i = 0; i < RG_Q; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(
                       (uint32_t)__cvta_generic_to_shared(&bars[i])),
                   "r"(RG_THREADS));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  __syncthreads();

  auto tiles_of = [&](const LibShalom_dgemm_entry &e) {
    return (e.M > 0 && e.N > 0) ? ((e.M + DR_T - 1) / DR_T) * ((e.N + DR_T - 1) / DR_T) : 0;
  };
  auto kslices_of = [&](const LibShalom_dgemm_entry &e) {
    return max(1, (max(0, e.K) + RG_KS - 1) / RG_KS);
  };
  auto first = [&](RgCursor &c) {
    c.t = c.p = c.k = 0;
    for (c.r = blockIdx.x; c.r < n_runs; c.r += gridDim.x)
      if (tiles_of(entries[run_first[c.r]]) > 0) { c.valid = true; return; }
    c.valid = false;
  };
  auto advance = [&](RgCursor &c) {
    if (!c.valid) return;
    const unsigned f = run_first[c.r], len = run_len[c.r];
    if (++c.k < kslices_of(entries[f + c.p])) return;
    c.k = 0;
    if (++c.p < (int)len) return;
    c.p = 0;
    if (++c.t < tiles_of(entries[f])) return;
    c.t = 0;
    for (c.r += gridDim.x; c.r < n_runs; c.r += gridDim.x)
      if (tiles_of(entries[run_first[c.r]]) > 0) return;
    c.valid = false;
  };
  auto item_of = [&](const RgCursor &c) {
    const unsigned f = run_first[c.r];
    const LibShalom_dgemm_entry &e0 = entries[f];
    const LibShalom_dgemm_entry &e = entries[f + c.p];
    RgItem it;
    const int K = max(0, e.K);
    it.A = e.A; it.B = e.B;
    it.transb = e.transb;
    it.lda = e.lda > 0 ? e.lda : K;
    it.ldb = e.ldb > 0 ? e.ldb : (e.transb ? K : e0.N);
    const int tiles_n = (e0.N + DR_T - 1) / DR_T;
    it.m0 = (c.t / tiles_n) * DR_T;
    it.n0 = (c.t % tiles_n) * DR_T;
    it.k0 = c.k * RG_KS;
    it.mcnt = min(DR_T, e0.M - it.m0);
    it.ncnt = min(DR_T, e0.N - it.n0);
    it.kcnt = max(0, min(RG_KS, K - it.k0));
    it.bytes = ((it.mcnt + it.ncnt) * it.kcnt * 8 + 15) & ~15;
    return it;
  };
  // placement rule shared by producer and consumer: an item never wraps
  auto place = [&](long &head, int bytes) -> int {
    long off = head % RG_RING;
    if (off + bytes > RG_RING) {
      head += RG_RING - off;
      off = 0;
    }
    head += bytes;
    return (int)off;
  };

  RgCursor pc, cc;
  first(pc);
  cc = pc;
  long ip = 0, ic = 0, head_p = 0, head_c = 0, tail = 0;
  double c[4], acc[4];
  const int tx = tid & 31, ty = tid >> 5;  // outputs (4*ty + i, tx)

  while (cc.valid) {
    // ---- produce: stage items ahead while slots and ring space allow ----
    while (pc.valid && ip < ic + RG_Q) {
      const RgItem it = item_of(pc);
      long h = head_p;
      const int off = place(h, it.bytes);
      if (h - tail > RG_RING) break;  // no room until the consumer releases
      head_p = h;
      const uint32_t base = (uint32_t)__cvta_generic_to_shared(rsm + off);
      const int na = it.mcnt * it.kcnt, nb = it.kcnt * it.ncnt;
      for (int e = tid; e < na; e += RG_THREADS) {  // A piece as [m][k]
        const int m = e / it.kcnt, k = e - m * it.kcnt;
        cp_async8(base + e * 8, it.A + (long)(it.m0 + m) * it.lda + it.k0 + k);
      }
      for (int e = tid; e < nb; e += RG_THREADS) {  // op(B) piece as [k][n]
        int k, n;
        const double *src;
        if (!it.transb) {
          k = e / it.ncnt; n = e - k * it.ncnt;
          src = it.B + (long)(it.k0 + k) * it.ldb + it.n0 + n;
        } else {
          n = e / it.kcnt; k = e - n * it.kcnt;
          src = it.B + (long)(it.n0 + n) * it.ldb + it.k0 + k;
        }
        cp_async8(base + (na + k * it.ncnt + n) * 8, src);
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(
                       (uint32_t)__cvta_generic_to_shared(&bars[ip % RG_Q]))
                   : "memory");
      ++ip;
      advance(pc);
    }

    // ---- consume item ic ----
    const RgItem it = item_of(cc);
    const int off = place(head_c, it.bytes);
    {
      bool ok = false;
      for (uint32_t n = 0; n < (1u << 22); ++n) {
        if (rg_mbar_try(&bars[ic % RG_Q], (uint32_t)((ic / RG_Q) & 1))) { ok = true; break; }
        if (n > 64) __nanosleep(64);
      }
      if (!ok) {
        atomicOr(err, 1u);
        s_abort = 1;
      }
    }
    __syncthreads();
    if (s_abort) break;
    const unsigned f = run_first[cc.r];
    const LibShalom_dgemm_entry &e0 = entries[f];
    const LibShalom_dgemm_entry &ep = entries[f + cc.p];
    const int ldc = e0.ldc > 0 ? e0.ldc : e0.N;
    double *Ct = e0.C + (long)it.m0 * ldc + it.n0;
    if (cc.p == 0 && cc.k == 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int m = 4 * ty + i;
        c[i] = (m < it.mcnt && tx < it.ncnt) ? Ct[(long)m * ldc + tx] : 0.0;
      }
    }
    if (cc.k == 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] = 0.0;
    }
    const double *As = reinterpret_cast<const double *>(rsm + off);
    const double *Bs = As + it.mcnt * it.kcnt;
    if (tx < it.ncnt) {
      for (int k = 0; k < it.kcnt; ++k) {
        const double b = Bs[k * it.ncnt + tx];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int m = min(4 * ty + i, it.mcnt - 1);  // rows past mcnt: computed, not stored
          acc[i] = __fma_rn(As[m * it.kcnt + k], b, acc[i]);
        }
      }
    }
    const bool product_done = cc.k + 1 >= kslices_of(ep);
    if (product_done) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double v = ep.alpha * acc[i];
        c[i] = ep.beta != 0.0 ? __fma_rn(ep.beta, c[i], v) : v;
      }
      if (cc.p + 1 == (int)run_len[cc.r]) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int m = 4 * ty + i;
          if (m < it.mcnt && tx < it.ncnt) Ct[(long)m * ldc + tx] = c[i];
        }
      }
    }
    __syncthreads();  // every thread is done reading the item: release it
    tail = head_c;
    ++ic;
    advance(cc);
  }
  cp_wait<0>();
  __syncthreads();
}

// device status word of the bounded waits
__device__ unsigned g_dr_err;

}  // namespace

// Grouped FP64 batch through the run kernel.  Workspace: run count + two
// arrays sized by the entry count.
int run_dgemm_runs(const LibShalom_dgemm_entry *entries, long count) {
  State &st = state();
  if (count > (1L << 30)) return LIBSHALOM_ERR_UNSUPPORTED;
  void *ws = nullptr;
  int rc = workspace((64 + 2 * (size_t)count) * sizeof(unsigned), &ws);
  if (rc) return rc;
  unsigned *w = static_cast<unsigned *>(ws);
  DrunPlan pl{w, w + 64, w + 64 + count};
  LS_CUDA_TRY(cudaMemsetAsync(w, 0, sizeof(unsigned), st.stream));
  const int pgrid = (int)std::max(1L, std::min(cdiv(count, 256), (long)st.num_sms * 8));
  k_drun_plan<<<pgrid, 256, 0, st.stream>>>(entries, count, pl);
  LS_CUDA_TRY(cudaGetLastError());
  void *errp = nullptr;
  LS_CUDA_TRY(cudaGetSymbolAddress(&errp, g_dr_err));
  const int per_sm = std::min(2, occupancy_of((const void *)k_dgemm_ring, RG_THREADS, RG_SMEM, 1));
  const int grid = grid_for(count, per_sm);
  k_dgemm_ring<<<grid, RG_THREADS, RG_SMEM, st.stream>>>(entries, pl.n_runs, pl.run_first,
                                                         pl.run_len,
                                                         static_cast<unsigned *>(errp));
  LS_CUDA_TRY(cudaGetLastError());
  if (st.sync) {
    unsigned err = 0;
    LS_CUDA_TRY(cudaStreamSynchronize(st.stream));
    LS_CUDA_TRY(cudaMemcpyFromSymbol(&err, g_dr_err, sizeof(err)));
    if (err) {
      const unsigned zero = 0;
      LS_CUDA_TRY(cudaMemcpyToSymbol(g_dr_err, &zero, sizeof(zero)));
      return LIBSHALOM_ERR_DEVICE_TIMEOUT;
    }
  }
  return LIBSHALOM_SUCCESS;
}

}  // namespace ls
