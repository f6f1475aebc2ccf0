// selftest.cu -- self-checks of the bounded device waits.
//
// Every spin in this library is bounded: the grid barrier of the persistent
// kernels (grid_sync.cuh) gives up after BAR_TIMEOUT_NS on the global timer
// and records BSP_ERR_TIMEOUT; the mbarrier wait of the TMA pipelines (tma.cuh) gives up
// after 2^20 polls.  These kernels make each wait run out on purpose -- a
// barrier one block never reaches, an mbarrier nothing arrives at -- so a test
// can check that the wait returns with the error status instead of hanging,
// and that the context stays usable afterwards.  Nothing faults or traps.
#include "grid_sync.cuh"
#include "tma.cuh"

namespace bsp {

// Two blocks; block 0 leaves without arriving, so block 1's barrier can only
// end by giving up.
__global__ void selftest_barrier_kernel(GridCtl *ctl, int *code) {
  if (blockIdx.x == 0) return;
  const bool ok = grid_barrier(ctl);
  if (threadIdx.x == 0) code[0] = ok ? BSP_OK : ctl->err;
}

// One mbarrier expecting one arrival that never comes.
__global__ void selftest_mbar_kernel(int *code) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) code[1] = mbar_wait(&bar, 0) ? BSP_OK : BSP_ERR_TIMEOUT;
}

}  // namespace bsp

extern "C" int bsp_selftest_waits(int *codes_dev, void *scratch_dev, cudaStream_t s) {
  using namespace bsp;
  if (!codes_dev || !scratch_dev) return BSP_ERR_NULL;
  if ((uintptr_t)scratch_dev & 7u) return BSP_ERR_ALIGN;
  cudaError_t e = cudaMemsetAsync(scratch_dev, 0, sizeof(GridCtl), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(codes_dev, 0xff, 2 * sizeof(int), s);
  if (e != cudaSuccess) return (int)e;
  selftest_barrier_kernel<<<2, 32, 0, s>>>(reinterpret_cast<GridCtl *>(scratch_dev), codes_dev);
  selftest_mbar_kernel<<<1, 32, 0, s>>>(codes_dev);
  return (int)cudaGetLastError();
}
