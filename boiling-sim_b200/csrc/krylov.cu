// krylov.cu -- vector primitives of the reference's PCG path, reference-compatible.
//
//   dot_launch                 crates/cuda-kernels/src/dot_reduce.cu:92-115
//   axpy_device_launch         crates/cuda-kernels/src/axpy_device.cu:33-45
//   scaled_axpy_launch         axpy_device.cu:65-77
//   divide_scalars_launch      axpy_device.cu:93-99
//   compute_b_launch           axpy_device.cu:125-137
//   zero_buffer_launch         axpy_device.cu:142-145
//   scale_inplace_launch       crates/cuda-kernels/src/scale.cu:11-34
//
// Differences from the reference, by design: the dot product accumulates in
// FP64 (per-thread partials, fixed-order block tree, then a fixed-order 256-way
// final tree in one block), so it is deterministic and independent of the
// launch shape; the reference sums FP32 partials serially on one thread.
#include "bsp_common.cuh"

namespace bsp {

int num_sms();

constexpr int DOT_THREADS = 256;
constexpr int DOT_PARTIALS = 256;  // doubles: 2 KiB of the >= 4 KiB workspace

__device__ __forceinline__ double block_sum_f64(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = l < (int)(blockDim.x >> 5) ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;  // valid in thread 0
}

// Partial sums over a fixed partition: block b owns elements [b*chunk, (b+1)*chunk).
__global__ void __launch_bounds__(DOT_THREADS) dot_partial_f64_kernel(
    const float *__restrict__ x, const float *__restrict__ y, int64_t n, int64_t chunk,
    double *__restrict__ partials) {
  __shared__ double sh[32];
  const int64_t b0 = (int64_t)blockIdx.x * chunk;
  const int64_t b1 = min(n, b0 + chunk);
  double s = 0.0;
  for (int64_t c = b0 + threadIdx.x; c < b1; c += DOT_THREADS)
    s = fma((double)__ldg(x + c), (double)__ldg(y + c), s);
  s = block_sum_f64(s, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(DOT_PARTIALS) dot_final_f64_kernel(
    const double *__restrict__ partials, int np, float *__restrict__ result_f32,
    double *__restrict__ result_f64) {
  __shared__ double sh[32];
  double v = threadIdx.x < np ? partials[threadIdx.x] : 0.0;
  v = block_sum_f64(v, sh);
  if (threadIdx.x == 0) {
    if (result_f32) *result_f32 = (float)v;
    if (result_f64) *result_f64 = v;
  }
}

cudaError_t dot_f64_impl(const float *x, const float *y, int64_t n, double *partials,
                         float *result_f32, double *result_f64, cudaStream_t s) {
  const int64_t chunk0 = (n + DOT_PARTIALS - 1) / DOT_PARTIALS;
  const int64_t chunk = ((chunk0 + 1023) / 1024) * 1024;
  const int np = (int)((n + chunk - 1) / chunk);
  dot_partial_f64_kernel<<<np, DOT_THREADS, 0, s>>>(x, y, n, chunk, partials);
  dot_final_f64_kernel<<<1, DOT_PARTIALS, 0, s>>>(partials, np, result_f32, result_f64);
  return cudaGetLastError();
}

__global__ void axpy_kernel(float *__restrict__ y, const float *__restrict__ x,
                            const float *__restrict__ alpha_ptr, int64_t n, int negate) {
  const float a = negate ? -(*alpha_ptr) : *alpha_ptr;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    y[c] = __fmaf_rn(a, x[c], y[c]);
}

__global__ void scaled_axpy_kernel(float *__restrict__ out, const float *__restrict__ z,
                                   const float *__restrict__ p_old,
                                   const float *__restrict__ beta_ptr, int64_t n) {
  const float b = *beta_ptr;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    out[c] = __fmaf_rn(b, p_old[c], z[c]);
}

__global__ void divide_kernel(const float *num, const float *den, float *res) {
  const float d = *den;
  *res = d == 0.0f ? 0.0f : __fdiv_rn(*num, d);
}

__global__ void compute_b_kernel(float *__restrict__ b, const float *__restrict__ div,
                                 const int *__restrict__ mat, int64_t n, float scale, int mf) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    b[c] = mat[c] != mf ? 0.0f : __fmul_rn(scale, div[c]);
}

__global__ void scale_kernel(float *__restrict__ x, int64_t n, float s) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    x[c] = __fmul_rn(x[c], s);
}

static inline int blocks_for(int64_t n) {
  int64_t b = (n + 255) / 256, cap = (int64_t)num_sms() * 16;
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

}  // namespace bsp

using namespace bsp;

extern "C" cudaError_t dot_launch(const float *x, const float *y, int n, float *workspace,
                                  float *result) {
  if (n <= 0) return cudaMemsetAsync(result, 0, sizeof(float), 0);
  if (((uintptr_t)workspace & 7u) != 0) return cudaErrorInvalidValue;
  return dot_f64_impl(x, y, n, reinterpret_cast<double *>(workspace), result, nullptr, 0);
}

extern "C" cudaError_t axpy_device_launch(float *y, const float *x, const float *alpha_ptr,
                                          int n, int negate_alpha) {
  if (n <= 0) return cudaSuccess;
  axpy_kernel<<<blocks_for(n), 256>>>(y, x, alpha_ptr, n, negate_alpha);
  return cudaGetLastError();
}

extern "C" cudaError_t scaled_axpy_launch(float *p_out, const float *z, const float *p_old,
                                          const float *beta_ptr, int n) {
  if (n <= 0) return cudaSuccess;
  scaled_axpy_kernel<<<blocks_for(n), 256>>>(p_out, z, p_old, beta_ptr, n);
  return cudaGetLastError();
}

extern "C" cudaError_t divide_scalars_launch(const float *num_ptr, const float *den_ptr,
                                             float *result_ptr) {
  divide_kernel<<<1, 1>>>(num_ptr, den_ptr, result_ptr);
  return cudaGetLastError();
}

extern "C" cudaError_t compute_b_launch(float *b, const float *div_u, const int *mat, int nx,
                                        int ny, int nz, float scale, int mat_fluid) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return cudaSuccess;
  const int64_t n = (int64_t)nx * ny * nz;
  compute_b_kernel<<<blocks_for(n), 256>>>(b, div_u, mat, n, scale, mat_fluid);
  return cudaGetLastError();
}

extern "C" cudaError_t zero_buffer_launch(float *buf, int n) {
  if (n <= 0) return cudaSuccess;
  return cudaMemsetAsync(buf, 0, sizeof(float) * (size_t)n, 0);
}

extern "C" cudaError_t scale_inplace_launch(float *x, int n, float s) {
  if (n <= 0) return cudaSuccess;
  scale_kernel<<<blocks_for(n), 256>>>(x, n, s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cudaDeviceSynchronize();
}

extern "C" const char *bsp_version(void) {
  return "bsproj 0.1 sm_100a";
}

extern "C" const char *bsp_error_string(int code) {
  switch (code) {
    case BSP_OK: return "success";
    case BSP_ERR_SHAPE: return "BSP_ERR_SHAPE: sizes or strides unusable";
    case BSP_ERR_NULL: return "BSP_ERR_NULL: required pointer is NULL";
    case BSP_ERR_ALIAS: return "BSP_ERR_ALIAS: output overlaps an input";
    case BSP_ERR_WORKSPACE: return "BSP_ERR_WORKSPACE: workspace too small or misaligned";
    case BSP_NOT_CONVERGED: return "BSP_NOT_CONVERGED: tolerance not reached within max_iter";
    case BSP_ERR_NONFINITE: return "BSP_ERR_NONFINITE: NaN or inf in the right-hand side";
    case BSP_ERR_TIMEOUT: return "BSP_ERR_TIMEOUT: device-side wait gave up";
    case BSP_ERR_ALIGN: return "BSP_ERR_ALIGN: pointer alignment unusable";
    case BSP_ERR_ARG: return "BSP_ERR_ARG: invalid argument";
    case BSP_ERR_CAPACITY: return "BSP_ERR_CAPACITY: more distinct cell classes than the table holds";
    default: return cudaGetErrorString((cudaError_t)code);
  }
}
