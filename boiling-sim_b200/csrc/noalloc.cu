// noalloc.cu -- an FP64 dot product for callers that cannot allocate device memory.
//
// dot_launch (krylov.cu) needs a caller-provided workspace for its per-block
// partial sums.  Some callers have none to give: a host that drives the solver
// through this C ABI from another language and only holds the pointers of the
// arrays it already owns, or a simulation loop that runs under a device-memory
// budget fixed at start-up and must not call cudaMalloc (or any allocating
// library routine) while stepping.  bsp_dot_noalloc serves them: its partial
// sums live in a file-scope __device__ array, so the call allocates nothing.
//
// Limits and sharing:
//   * the array holds NOALLOC_MAX_PARTIALS doubles (8 KiB per GPU that loads the
//     library, kept until process exit); each partial covers NOALLOC_CHUNK
//     elements, so n may be at most NOALLOC_MAX_PARTIALS * NOALLOC_CHUNK
//     (67,108,864); larger n is rejected with BSP_ERR_SHAPE;
//   * every call shares the one array and leaves its partials in it; each call
//     overwrites the partials it reads before reading them, so nothing needs
//     clearing, but calls that overlap on the GPU (different streams, or
//     different host threads) race on the array and must be serialised;
//   * host code cannot pass the array's name to a kernel (on the host it is only
//     a stand-in symbol): the device address is looked up with
//     cudaGetSymbolAddress, with the device current, by every call made
//     outside a stream capture, and kept per device for calls made inside one.
//     The first call on a device should therefore come before any stream
//     capture; after a cudaDeviceReset, the first call should again come
//     outside a capture (the module is loaded anew and the kept address is
//     stale until a call outside a capture refreshes it).
#include <mutex>

#include "bsp_common.cuh"

namespace bsp {

constexpr int NOALLOC_MAX_PARTIALS = 1024;
constexpr int64_t NOALLOC_CHUNK = 65536;
constexpr int NOALLOC_THREADS = 256;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_PARTIALS];

namespace {
std::mutex g_addr_mu;
double *g_addr[MAX_DEVICES] = {nullptr};
}  // namespace

__device__ __forceinline__ double noalloc_block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = l < (int)(blockDim.x >> 5) ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;  // valid in thread 0
}

// Block b sums x[c] * y[c] over [b * chunk, (b + 1) * chunk) in FP64.
__global__ void __launch_bounds__(NOALLOC_THREADS) noalloc_partial_kernel(
    const float *__restrict__ x, const float *__restrict__ y, int64_t n, int64_t chunk,
    double *__restrict__ partials) {
  __shared__ double sh[32];
  const int64_t b0 = (int64_t)blockIdx.x * chunk;
  const int64_t b1 = min(n, b0 + chunk);
  double s = 0.0;
  for (int64_t c = b0 + threadIdx.x; c < b1; c += NOALLOC_THREADS)
    s = fma((double)__ldg(x + c), (double)__ldg(y + c), s);
  s = noalloc_block_sum(s, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// Fixed-order sum of the first np partials into *result.
__global__ void __launch_bounds__(NOALLOC_THREADS) noalloc_final_kernel(
    const double *__restrict__ partials, int np, double *__restrict__ result) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int b = threadIdx.x; b < np; b += NOALLOC_THREADS) s += partials[b];
  s = noalloc_block_sum(s, sh);
  if (threadIdx.x == 0) *result = s;
}

// Device address of g_noalloc_partials on the current device: looked up on
// every call outside a stream capture (so a module reloaded after
// cudaDeviceReset is found again), taken from the per-device record inside one.
static int noalloc_scratch(double **out, cudaStream_t stream) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= MAX_DEVICES) return BSP_ERR_ARG;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &cap);
  if (e != cudaSuccess) return (int)e;
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    double *ptr = nullptr;
    e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_partials);
    if (e != cudaSuccess) return (int)e;
    g_addr[dev] = ptr;
  } else if (!g_addr[dev]) {
    return BSP_ERR_ARG;  // first call on this device made inside a capture
  }
  *out = g_addr[dev];
  return BSP_OK;
}

}  // namespace bsp

extern "C" int bsp_dot_noalloc(const float *x, const float *y, int64_t n, double *result,
                               cudaStream_t stream) {
  using namespace bsp;
  if (!result) return BSP_ERR_NULL;
  if (n < 0) return BSP_ERR_ARG;
  if (n > (int64_t)NOALLOC_MAX_PARTIALS * NOALLOC_CHUNK) return BSP_ERR_SHAPE;
  if (n > 0 && (!x || !y)) return BSP_ERR_NULL;
  double *partials = nullptr;
  int st = noalloc_scratch(&partials, stream);
  if (st != BSP_OK) return st;
  if (n == 0) return (int)cudaMemsetAsync(result, 0, sizeof(double), stream);
  const int np = (int)((n + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK);
  noalloc_partial_kernel<<<np, NOALLOC_THREADS, 0, stream>>>(x, y, n, NOALLOC_CHUNK, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  noalloc_final_kernel<<<1, NOALLOC_THREADS, 0, stream>>>(partials, np, result);
  return (int)cudaGetLastError();
}
