// ls_dgemm.cu -- grouped FP64 GEMM (LibShalom_dgemm_batched) for the
// small-block workloads of atomic-orbital chemistry codes: tens of thousands
// of products with M, N, K of a few to a few dozen, where consecutive products
// accumulate into the same C block (C += A_p B_p).
//
// Work unit: one run (maximal group of consecutive entries naming the same C)
// and one 32 x 32 tile of its C block.  The CTA (64 threads, 4 x 4 outputs
// each, six CTAs per SM) loads the C tile once, applies the run's products in array order with
// the C tile held in registers (C = alpha_p A_p op(B_p) + beta_p C), and writes
// it once -- the owner-computes rule that keeps shared C blocks race-free and
// the result deterministic without atomics.  A and op(B) arrive in 32 x 32
// slabs through an 8-byte cp.async double buffer that prefetches the next slab
// (of the same product, the next product or the next run) while the current
// one is multiplied, staged transposed (A as [k][m]) so the inner loop reads
// contiguous vectors.  Each product is a fused multiply-add chain over k in
// increasing order (the reference's KERNEL7x6 order) followed by
// C = fma(beta, C, alpha * acc).
//
// Runs are found on the device (k_drun_plan: one slot per run start), so the
// call needs no host round trip.
#include <cuda_runtime.h>

#include <algorithm>

#include "ls_common.cuh"
#include "ls_simt_launch.h"

namespace ls {

namespace {

constexpr int DR_THREADS = 64;
constexpr int DR_T = 32;       // C tile edge and K slab
constexpr int DR_P = 34;       // padded pitch (doubles) of the staged slabs
constexpr int DR_STAGE = 2 * DR_T * DR_P;  // doubles per stage: A^T and B

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

struct DJob {
  const double *A, *B;
  int M, N, K, lda, ldb, transb;
  double alpha, beta;
};

__device__ __forceinline__ DJob djob(const LibShalom_dgemm_entry &e) {
  DJob j;
  j.A = e.A; j.B = e.B;
  j.M = e.M; j.N = e.N; j.K = max(0, e.K);
  j.transb = e.transb;
  j.lda = e.lda > 0 ? e.lda : j.K;
  j.ldb = e.ldb > 0 ? e.ldb : (e.transb ? j.K : j.N);
  j.alpha = e.alpha; j.beta = e.beta;
  return j;
}

__device__ __forceinline__ void cp_async8(uint32_t saddr, const void *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Position in this CTA's sequence of slabs: run slot r (round-robin over the
// CTAs), C tile t of the run, product p of the run, K slab k of the product.
struct DCursor {
  long r;
  int t, p, k;
};

__global__ void __launch_bounds__(DR_THREADS, 6)
    k_dgemm_runs(const LibShalom_dgemm_entry *entries, const unsigned *n_runs_p,
                 const unsigned *run_first, const unsigned *run_len) {
  __shared__ __align__(16) double stage[2][DR_STAGE];
  const int tid = threadIdx.x;
  const int tx = tid & 7, ty = tid >> 3;  // outputs: rows 4ty..4ty+3; cols 4tx..4tx+3
  const long n_runs = (long)*n_runs_p;

  auto tiles_of = [&](const LibShalom_dgemm_entry &e) {
    return ((e.M + DR_T - 1) / DR_T) * ((e.N + DR_T - 1) / DR_T);
  };
  auto slabs_of = [&](const LibShalom_dgemm_entry &e) { return max(1, (max(0, e.K) + DR_T - 1) / DR_T); };

  // advance a cursor to the next slab; returns false past the CTA's last run
  auto advance = [&](DCursor &c) -> bool {
    if (c.r >= n_runs) return false;
    const unsigned f = run_first[c.r], len = run_len[c.r];
    if (++c.k < slabs_of(entries[f + c.p])) return true;
    c.k = 0;
    if (++c.p < (int)len) return true;
    c.p = 0;
    if (++c.t < tiles_of(entries[f])) return true;
    c.t = 0;
    for (c.r += gridDim.x; c.r < n_runs; c.r += gridDim.x)
      if (tiles_of(entries[run_first[c.r]]) > 0) return true;
    return false;
  };
  auto first = [&](DCursor &c) -> bool {
    c.t = c.p = c.k = 0;
    for (c.r = blockIdx.x; c.r < n_runs; c.r += gridDim.x)
      if (tiles_of(entries[run_first[c.r]]) > 0) return true;
    return false;
  };

  // issue the cp.async copies of the slab at cursor c into stage buffer b
  auto load = [&](const DCursor &c, int b) {
    const unsigned f = run_first[c.r];
    const LibShalom_dgemm_entry &e0 = entries[f];
    const DJob jb = djob(entries[f + c.p]);
    const int tiles_n = (e0.N + DR_T - 1) / DR_T;
    const int m0 = (c.t / tiles_n) * DR_T, n0 = (c.t % tiles_n) * DR_T, k0 = c.k * DR_T;
    double *As = stage[b];
    double *Bs = stage[b] + DR_T * DR_P;
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(As);
    const uint32_t sb = (uint32_t)__cvta_generic_to_shared(Bs);
#pragma unroll
    for (int q = 0; q < (DR_T * DR_T) / DR_THREADS; ++q) {
      const int e = tid + q * DR_THREADS;
      // A element (m, k): consecutive threads take consecutive k (contiguous in memory)
      const int m = e >> 5, k = e & 31;
      if (m0 + m < jb.M && k0 + k < jb.K)
        cp_async8(sa + (k * DR_P + m) * 8, jb.A + (long)(m0 + m) * jb.lda + k0 + k);
      // B element (k, n) of op(B)
      if (!jb.transb) {
        const int kk = e >> 5, n = e & 31;
        if (k0 + kk < jb.K && n0 + n < jb.N)
          cp_async8(sb + (kk * DR_P + n) * 8, jb.B + (long)(k0 + kk) * jb.ldb + n0 + n);
      } else {
        const int n = e >> 5, kk = e & 31;
        if (k0 + kk < jb.K && n0 + n < jb.N)
          cp_async8(sb + (kk * DR_P + n) * 8, jb.B + (long)(n0 + n) * jb.ldb + k0 + kk);
      }
    }
  };

  DCursor cur, nxt;
  if (!first(cur)) return;
  nxt = cur;
  bool have_next = advance(nxt);
  load(cur, 0);
  cp_commit();

  double c[4][4], acc[4][4];
  int buf = 0;
  for (;;) {
    const unsigned f = run_first[cur.r];
    const LibShalom_dgemm_entry &e0 = entries[f];
    const DJob jb = djob(entries[f + cur.p]);
    const int tiles_n = (e0.N + DR_T - 1) / DR_T;
    const int m0 = (cur.t / tiles_n) * DR_T, n0 = (cur.t % tiles_n) * DR_T;
    double *Crow0 = entries[f].C + (long)(m0 + 4 * ty) * (e0.ldc > 0 ? e0.ldc : e0.N) + n0 + 4 * tx;
    const int ldc = e0.ldc > 0 ? e0.ldc : e0.N;
    if (cur.p == 0 && cur.k == 0) {
      // new C tile: load it (the run's first beta decides whether it is read)
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const bool ok = m0 + 4 * ty + i < e0.M && n0 + 4 * tx + j < e0.N;
          c[i][j] = ok ? Crow0[(long)i * ldc + j] : 0.0;
        }
    }
    if (cur.k == 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    }
    // prefetch the next slab into the other buffer, then wait for this one
    if (have_next) load(nxt, buf ^ 1);
    cp_commit();
    cp_wait<1>();
    __syncthreads();
    const double *As = stage[buf];
    const double *Bs = stage[buf] + DR_T * DR_P;
    const int kcnt = min(DR_T, jb.K - cur.k * DR_T);
    for (int k = 0; k < kcnt; ++k) {
      const double2 a0 = *reinterpret_cast<const double2 *>(As + k * DR_P + 4 * ty);
      const double2 a1 = *reinterpret_cast<const double2 *>(As + k * DR_P + 4 * ty + 2);
      const double2 b0 = *reinterpret_cast<const double2 *>(Bs + k * DR_P + 4 * tx);
      const double2 b1 = *reinterpret_cast<const double2 *>(Bs + k * DR_P + 4 * tx + 2);
      const double av[4] = {a0.x, a0.y, a1.x, a1.y};
      const double bv[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = __fma_rn(av[i], bv[j], acc[i][j]);
    }
    const bool product_done = cur.k + 1 >= max(1, (jb.K + DR_T - 1) / DR_T);
    if (product_done) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double v = jb.alpha * acc[i][j];
          c[i][j] = jb.beta != 0.0 ? __fma_rn(jb.beta, c[i][j], v) : v;
        }
      if (cur.p + 1 == (int)run_len[cur.r]) {
        // run complete for this tile: write it
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (m0 + 4 * ty + i < e0.M && n0 + 4 * tx + j < e0.N) Crow0[(long)i * ldc + j] = c[i][j];
      }
    }
    __syncthreads();  // everyone is done with this buffer before it is refilled
    if (!have_next) break;
    cur = nxt;
    have_next = advance(nxt);
    buf ^= 1;
  }
  cp_wait<0>();
}

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
  const int per_sm = occupancy_of((const void *)k_dgemm_runs, DR_THREADS, 0, 6);
  const int grid = grid_for(cdiv(count, 1), per_sm);
  k_dgemm_runs<<<grid, DR_THREADS, 0, st.stream>>>(entries, pl.n_runs, pl.run_first, pl.run_len);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

// The run kernel over a run list built by another plan (device counts).
int run_dgemm_runs_list(const LibShalom_dgemm_entry *entries, long count, const unsigned *n_runs,
                        const unsigned *run_first, const unsigned *run_len) {
  State &st = state();
  const int per_sm = occupancy_of((const void *)k_dgemm_runs, DR_THREADS, 0, 6);
  const int grid = grid_for(cdiv(count, 1), per_sm);
  k_dgemm_runs<<<grid, DR_THREADS, 0, st.stream>>>(entries, n_runs, run_first, run_len);
  LS_CUDA_TRY(cudaGetLastError());
  return LIBSHALOM_SUCCESS;
}

}  // namespace ls
