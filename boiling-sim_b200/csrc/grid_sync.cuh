// grid_sync.cuh -- bounded grid-wide barrier and deterministic FP64 reductions for
// persistent (cooperatively launched) kernels.
//
// The barrier is a sense-free generation counter: after a CTA barrier, each
// block's thread 0 makes the block's writes visible (fence.acq_rel.gpu, which
// is cumulative over what the CTA barrier ordered before it) and arrives with
// a fetch_add; the last arrival resets the count and publishes the next
// generation with a release store; the others poll the generation with
// acquire loads, back to back (no sleep: a sleep's wake-up granularity is
// longer than the barrier itself).  Every poll loop is bounded by wall time:
// after BAR_TIMEOUT_NS on the global timer (or BAR_SPIN_LIMIT polls) the block
// records BSP_ERR_TIMEOUT in ctl->err and returns false, and every block
// leaves the kernel at its next barrier once err is set.  Cooperative launch
// guarantees co-residency, so the limit is only a guard.
#pragma once
#include <cuda/atomic>
#include "bsp_common.cuh"

namespace bsp {

struct GridCtl {
  unsigned int bar_count;
  unsigned int bar_gen;
  int err;
  int iters;
  int status;
  int pad[3];
};

constexpr unsigned long long BAR_TIMEOUT_NS = 2000000000ull;  // 2 s
constexpr unsigned int BAR_SPIN_LIMIT = 1u << 26;              // polls, a second guard

__device__ __forceinline__ unsigned long long gs_global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool grid_barrier(GridCtl *ctl) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(ctl->bar_count);
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(ctl->bar_gen);
    cuda::atomic_ref<int, cuda::thread_scope_device> err(ctl->err);
    // the generation cannot move before this block arrives, so this is the
    // generation of the barrier being entered
    const unsigned int g = gen.load(cuda::memory_order_relaxed);
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    const unsigned int a = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
    if (a == gridDim.x - 1) {
      cnt.store(0u, cuda::memory_order_relaxed);
      gen.store(g + 1u, cuda::memory_order_release);
    } else {
      unsigned int spins = 0;
      unsigned long long t0 = 0;
      while (gen.load(cuda::memory_order_acquire) == g) {
        if ((++spins & 255u) == 0) {
          const unsigned long long now = gs_global_ns();
          if (t0 == 0) t0 = now;
          if (err.load(cuda::memory_order_relaxed) != 0) {  // another block gave up
            ok = 0;
            break;
          }
          if (now - t0 > BAR_TIMEOUT_NS || spins > BAR_SPIN_LIMIT) {
            err.store(BSP_ERR_TIMEOUT, cuda::memory_order_relaxed);
            ok = 0;
            break;
          }
        }
      }
    }
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    if (err.load(cuda::memory_order_relaxed) != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Sum K doubles over the block (fixed order) and store them at
// partials[k * stride + blockIdx.x].  sh must hold 32*K doubles.
template <int K>
__device__ __forceinline__ void block_partials(double (&v)[K], double *partials, int stride,
                                               double *sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < K; ++q)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < K; ++q) sh[q * 32 + warp] = v[q];
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[threadIdx.x * 32 + w];
    partials[threadIdx.x * stride + blockIdx.x] = s;
  }
}

// Every block reads the gridDim.x partials of slot q in the same order, so all
// blocks obtain bit-identical totals.  Result broadcast to the whole block.
template <int K>
__device__ __forceinline__ void grid_totals(const double *partials, int stride, double (&out)[K],
                                            double *sh) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 32) {
#pragma unroll
    for (int q = 0; q < K; ++q) {
      double s = 0.0;
      for (int b = lane; b < (int)gridDim.x; b += 32)
        s += *((volatile const double *)(partials + q * stride + b));
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) sh[q] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < K; ++q) out[q] = sh[q];
  __syncthreads();
}

}  // namespace bsp
