// projection.cu -- divergence, gradient subtract, no-slip and the Jacobi projection.
//
// Reference semantics:
//   compute_divergence                 python/boilingsim/fluid.py:201-218
//   subtract_pressure_gradient_{x,y,z} python/boilingsim/fluid.py:279-330
//   enforce_no_slip_{ux,uy,uz}         python/boilingsim/fluid.py:111-165
//   pressure_projection (sequence)     python/boilingsim/fluid.py:612-734
//
// The reference ends every projection with a full-field device->host copy of
// the diagnostic divergence to take max|div| on the host (fluid.py:733-734);
// here the diagnostic kernel reduces max|div| on the device and only 4 bytes
// are left for the caller to read.
#include "bsp_common.cuh"
#include "profile.cuh"

namespace bsp {

int num_sms();
template <int OP, class MaskT>
cudaError_t launch_stencil(float *out, const float *p, const float *div, const MaskT *mask,
                           int nx, int ny, int nz, float dx, float dt, float rho, int mf,
                           int ma, cudaStream_t s);
int jacobi_solve_impl(float *p, float *p_tmp, const float *div_u, float *rhs_ws,
                      const uint8_t *mask, int nx, int ny, int nz, float dx, float dt, float rho,
                      int n_iter, int tblock, cudaStream_t stream, bool p_zero_nonfluid);

// Block = (128 k, 2 j); grid = (k tiles, j tiles, i).  One cell per thread.
__global__ void __launch_bounds__(256) divergence_kernel(
    float *__restrict__ div, const float *__restrict__ ux, const float *__restrict__ uy,
    const float *__restrict__ uz, const uint8_t *__restrict__ mask, int nx, int ny, int nz,
    float dx, unsigned int *__restrict__ max_bits) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  float a = 0.0f;
  if (k < nz && j < ny) {
    const int64_t c = idx3(i, j, k, ny, nz);
    float v = 0.0f;
    if (mcls(__ldg(mask + c)) == BSP_FLUID) {
      const float u1 = __ldg(ux + ((int64_t)(i + 1) * ny + j) * nz + k);
      const float u0 = __ldg(ux + ((int64_t)i * ny + j) * nz + k);
      const float v1 = __ldg(uy + ((int64_t)i * (ny + 1) + j + 1) * nz + k);
      const float v0 = __ldg(uy + ((int64_t)i * (ny + 1) + j) * nz + k);
      const float w1 = __ldg(uz + ((int64_t)i * ny + j) * (nz + 1) + k + 1);
      const float w0 = __ldg(uz + ((int64_t)i * ny + j) * (nz + 1) + k);
      const float dudx = __fdiv_rn(__fsub_rn(u1, u0), dx);
      const float dvdy = __fdiv_rn(__fsub_rn(v1, v0), dx);
      const float dwdz = __fdiv_rn(__fsub_rn(w1, w0), dx);
      v = __fadd_rn(__fadd_rn(dudx, dvdy), dwdz);
    }
    div[c] = v;
    a = fabsf(v);
  }
  if (max_bits) {
    // |div| >= 0, so its bit pattern orders like the value.
    unsigned int bits = __float_as_uint(a);
    for (int o = 16; o > 0; o >>= 1) bits = max(bits, __shfl_xor_sync(0xffffffffu, bits, o));
    __shared__ unsigned int wmax[8];
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    if ((t & 31) == 0) wmax[t >> 5] = bits;
    __syncthreads();
    if (t == 0) {
      unsigned int m = 0;
      for (int w = 0; w < (int)(blockDim.x * blockDim.y) / 32; ++w) m = max(m, wmax[w]);
      atomicMax(max_bits, m);
    }
  }
}

// enforce_no_slip (fluid.py:111-165) followed by compute_divergence
// (fluid.py:201-218) in one pass.  One thread per lattice point (i, j, k) in
// [0,nx] x [0,ny] x [0,nz]: it zeroes the x-, y- and z-face with its index
// when that face touches a non-fluid cell or the domain boundary, and, on a
// fluid cell, computes the divergence from its six faces with the same rule
// applied to each face (a face is kept only between two fluid cells).  The
// result equals no-slip then divergence bit for bit: kept faces are read
// unchanged, zeroed faces contribute exactly 0.
__global__ void __launch_bounds__(256) noslip_divergence_kernel(
    float *__restrict__ div, float *__restrict__ ux, float *__restrict__ uy,
    float *__restrict__ uz, const uint8_t *__restrict__ mask, int nx, int ny, int nz, float dx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k > nz || j > ny) return;
  auto fluid = [&](int a, int b, int c) {
    return a >= 0 && a < nx && b >= 0 && b < ny && c >= 0 && c < nz &&
           mcls(__ldg(mask + idx3(a, b, c, ny, nz))) == BSP_FLUID;
  };
  // faces owned by this lattice point
  if (j < ny && k < nz && !(fluid(i - 1, j, k) && fluid(i, j, k)))
    ux[((int64_t)i * ny + j) * nz + k] = 0.0f;
  if (i < nx && k < nz && !(fluid(i, j - 1, k) && fluid(i, j, k)))
    uy[((int64_t)i * (ny + 1) + j) * nz + k] = 0.0f;
  if (i < nx && j < ny && !(fluid(i, j, k - 1) && fluid(i, j, k)))
    uz[((int64_t)i * ny + j) * (nz + 1) + k] = 0.0f;
  if (i >= nx || j >= ny || k >= nz) return;
  const int64_t c = idx3(i, j, k, ny, nz);
  float v = 0.0f;
  if (fluid(i, j, k)) {
    // a face of a fluid cell is kept iff the neighbour across it is fluid
    const float u1 = fluid(i + 1, j, k) ? ux[((int64_t)(i + 1) * ny + j) * nz + k] : 0.0f;
    const float u0 = fluid(i - 1, j, k) ? ux[((int64_t)i * ny + j) * nz + k] : 0.0f;
    const float v1 = fluid(i, j + 1, k) ? uy[((int64_t)i * (ny + 1) + j + 1) * nz + k] : 0.0f;
    const float v0 = fluid(i, j - 1, k) ? uy[((int64_t)i * (ny + 1) + j) * nz + k] : 0.0f;
    const float w1 = fluid(i, j, k + 1) ? uz[((int64_t)i * ny + j) * (nz + 1) + k + 1] : 0.0f;
    const float w0 = fluid(i, j, k - 1) ? uz[((int64_t)i * ny + j) * (nz + 1) + k] : 0.0f;
    v = __fadd_rn(__fadd_rn(__fdiv_rn(__fsub_rn(u1, u0), dx), __fdiv_rn(__fsub_rn(v1, v0), dx)),
                  __fdiv_rn(__fsub_rn(w1, w0), dx));
  }
  div[c] = v;
}

// One thread per cell c = (i, j, k): updates the x-face (i, j, k) if i >= 1,
// the y-face if j >= 1 and the z-face if k >= 1, each only when both cells
// adjacent to the face are fluid.  u -= ((dt/rho) * dp) / dx.
__global__ void __launch_bounds__(256) gradient_kernel(
    float *__restrict__ ux, float *__restrict__ uy, float *__restrict__ uz,
    const float *__restrict__ p, const uint8_t *__restrict__ mask, int nx, int ny, int nz,
    float dx, float dtr) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= nz || j >= ny) return;
  const int64_t c = idx3(i, j, k, ny, nz);
  if (mcls(__ldg(mask + c)) != BSP_FLUID) return;
  const float pc = __ldg(p + c);
  const int64_t plane = (int64_t)ny * nz;
  if (i >= 1 && mcls(__ldg(mask + c - plane)) == BSP_FLUID) {
    float *f = ux + ((int64_t)i * ny + j) * nz + k;
    *f = __fsub_rn(*f, __fdiv_rn(__fmul_rn(dtr, __fsub_rn(pc, __ldg(p + c - plane))), dx));
  }
  if (j >= 1 && mcls(__ldg(mask + c - nz)) == BSP_FLUID) {
    float *f = uy + ((int64_t)i * (ny + 1) + j) * nz + k;
    *f = __fsub_rn(*f, __fdiv_rn(__fmul_rn(dtr, __fsub_rn(pc, __ldg(p + c - nz))), dx));
  }
  if (k >= 1 && mcls(__ldg(mask + c - 1)) == BSP_FLUID) {
    float *f = uz + ((int64_t)i * ny + j) * (nz + 1) + k;
    *f = __fsub_rn(*f, __fdiv_rn(__fmul_rn(dtr, __fsub_rn(pc, __ldg(p + c - 1))), dx));
  }
}

// One thread per lattice point (i, j, k) in [0,nx] x [0,ny] x [0,nz]; each point
// owns the x-, y- and z-face with its index where that face exists.
__global__ void __launch_bounds__(256) no_slip_kernel(float *__restrict__ ux,
                                                      float *__restrict__ uy,
                                                      float *__restrict__ uz,
                                                      const uint8_t *__restrict__ mask, int nx,
                                                      int ny, int nz) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k > nz || j > ny) return;
  auto fluid = [&](int a, int b, int c) {
    return mcls(__ldg(mask + idx3(a, b, c, ny, nz))) == BSP_FLUID;
  };
  if (j < ny && k < nz) {
    if (i == 0 || i == nx || !fluid(i - 1, j, k) || !fluid(i, j, k))
      ux[((int64_t)i * ny + j) * nz + k] = 0.0f;
  }
  if (i < nx && k < nz) {
    if (j == 0 || j == ny || !fluid(i, j - 1, k) || !fluid(i, j, k))
      uy[((int64_t)i * (ny + 1) + j) * nz + k] = 0.0f;
  }
  if (i < nx && j < ny) {
    if (k == 0 || k == nz || !fluid(i, j, k - 1) || !fluid(i, j, k))
      uz[((int64_t)i * ny + j) * (nz + 1) + k] = 0.0f;
  }
}

// Four consecutive k cells per thread (nz % 4 == 0, 16-byte aligned fields):
// the same per-cell operations as divergence_kernel / gradient_kernel, so the
// same bits, with 16-byte loads of the mask word, ux, uy and div (the rows of
// uz are nz + 1 long and are read as scalars).  Block = (32 k-quads, 8 j).
__device__ __forceinline__ float q4v(const float4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}

__global__ void __launch_bounds__(256) divergence4_kernel(
    float *__restrict__ div, const float *__restrict__ ux, const float *__restrict__ uy,
    const float *__restrict__ uz, const uint8_t *__restrict__ mask, int nx, int ny, int nz,
    float dx, unsigned int *__restrict__ max_bits) {
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  unsigned int bits = 0u;  // max |div| of the thread's cells as a bit pattern
  if (k < nz && j < ny) {
    const int64_t c = idx3(i, j, k, ny, nz);
    const uint32_t mw = __ldg(reinterpret_cast<const uint32_t *>(mask + c));
    float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (mw & 0x80808080u) {
      const int64_t plane = (int64_t)ny * nz;
      const float4 u1 = __ldg(reinterpret_cast<const float4 *>(ux + c + plane));
      const float4 u0 = __ldg(reinterpret_cast<const float4 *>(ux + c));
      const int64_t cy = ((int64_t)i * (ny + 1) + j) * nz + k;
      const float4 v1 = __ldg(reinterpret_cast<const float4 *>(uy + cy + nz));
      const float4 v0 = __ldg(reinterpret_cast<const float4 *>(uy + cy));
      const float *wz = uz + ((int64_t)i * ny + j) * (nz + 1) + k;
      float w[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) w[q] = __ldg(wz + q);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if ((mw >> (8 * q)) & BSP_MFLUID) {
          const float dudx = __fdiv_rn(__fsub_rn(q4v(u1, q), q4v(u0, q)), dx);
          const float dvdy = __fdiv_rn(__fsub_rn(q4v(v1, q), q4v(v0, q)), dx);
          const float dwdz = __fdiv_rn(__fsub_rn(w[q + 1], w[q]), dx);
          v[q] = __fadd_rn(__fadd_rn(dudx, dvdy), dwdz);
        }
      }
    }
    *reinterpret_cast<float4 *>(div + c) = make_float4(v[0], v[1], v[2], v[3]);
    // |div| >= 0, so its bit pattern orders like the value (a NaN orders
    // above every number, as in the one-cell kernel)
#pragma unroll
    for (int q = 0; q < 4; ++q) bits = max(bits, __float_as_uint(fabsf(v[q])));
  }
  if (max_bits) {
    for (int o = 16; o > 0; o >>= 1) bits = max(bits, __shfl_xor_sync(0xffffffffu, bits, o));
    __shared__ unsigned int wmax[8];
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    if ((t & 31) == 0) wmax[t >> 5] = bits;
    __syncthreads();
    if (t == 0) {
      unsigned int m = 0;
      for (int w = 0; w < (int)(blockDim.x * blockDim.y) / 32; ++w) m = max(m, wmax[w]);
      atomicMax(max_bits, m);
    }
  }
}

__global__ void __launch_bounds__(256) gradient4_kernel(
    float *__restrict__ ux, float *__restrict__ uy, float *__restrict__ uz,
    const float *__restrict__ p, const uint8_t *__restrict__ mask, int nx, int ny, int nz,
    float dx, float dtr) {
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= nz || j >= ny) return;
  const int64_t c = idx3(i, j, k, ny, nz);
  const uint32_t mw = __ldg(reinterpret_cast<const uint32_t *>(mask + c));
  if (!(mw & 0x80808080u)) return;
  const int64_t plane = (int64_t)ny * nz;
  const float4 pc = __ldg(reinterpret_cast<const float4 *>(p + c));
  auto grad = [&](float f, float pa, float pb) {
    return __fsub_rn(f, __fdiv_rn(__fmul_rn(dtr, __fsub_rn(pa, pb)), dx));
  };
  // a face is updated when both cells beside it are fluid (bit 7 of both bytes)
  if (i >= 1) {
    const uint32_t both = mw & __ldg(reinterpret_cast<const uint32_t *>(mask + c - plane));
    if (both & 0x80808080u) {
      const float4 pi = __ldg(reinterpret_cast<const float4 *>(p + c - plane));
      float4 *fp = reinterpret_cast<float4 *>(ux + c);
      const float4 f = *fp;
      float r[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if ((both >> (8 * q)) & BSP_MFLUID) r[q] = grad(r[q], q4v(pc, q), q4v(pi, q));
      *fp = make_float4(r[0], r[1], r[2], r[3]);
    }
  }
  if (j >= 1) {
    const uint32_t both = mw & __ldg(reinterpret_cast<const uint32_t *>(mask + c - nz));
    if (both & 0x80808080u) {
      const float4 pj = __ldg(reinterpret_cast<const float4 *>(p + c - nz));
      float4 *fp = reinterpret_cast<float4 *>(uy + ((int64_t)i * (ny + 1) + j) * nz + k);
      const float4 f = *fp;
      float r[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if ((both >> (8 * q)) & BSP_MFLUID) r[q] = grad(r[q], q4v(pc, q), q4v(pj, q));
      *fp = make_float4(r[0], r[1], r[2], r[3]);
    }
  }
  // k faces: byte q of mk is the cell below cell q (for q = 0 the byte before
  // the word; no face below k = 0)
  const uint32_t below0 = k >= 1 ? (uint32_t)__ldg(mask + c - 1) : 0u;
  const uint32_t both = mw & ((mw << 8) | below0);
  if (both & 0x80808080u) {
    const float pkm = k >= 1 ? __ldg(p + c - 1) : 0.0f;
    const float pb[4] = {pkm, pc.x, pc.y, pc.z};
    float *fz = uz + ((int64_t)i * ny + j) * (nz + 1) + k;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if ((both >> (8 * q)) & BSP_MFLUID) fz[q] = grad(fz[q], q4v(pc, q), pb[q]);
  }
}

static inline bool aligned16_all(const void *a, const void *b, const void *c) {
  return (((uintptr_t)a | (uintptr_t)b | (uintptr_t)c) & 15u) == 0;
}

cudaError_t divergence_impl(float *div, const float *ux, const float *uy, const float *uz,
                            const uint8_t *mask, int nx, int ny, int nz, float dx,
                            float *max_abs_div, cudaStream_t s) {
  if (max_abs_div) {
    cudaError_t e = cudaMemsetAsync(max_abs_div, 0, sizeof(float), s);
    if (e != cudaSuccess) return e;
  }
  ProfScope ps(PROF_PROJ, s);
  if (nz % 4 == 0 && aligned16_all(div, ux, uy) && ((uintptr_t)mask & 3u) == 0) {
    dim3 block(32, 8);
    dim3 grid((nz / 4 + 31) / 32, (ny + 7) / 8, nx);
    divergence4_kernel<<<grid, block, 0, s>>>(div, ux, uy, uz, mask, nx, ny, nz, dx,
                                              reinterpret_cast<unsigned int *>(max_abs_div));
    return cudaGetLastError();
  }
  dim3 block(128, 2);
  dim3 grid((nz + 127) / 128, (ny + 1) / 2, nx);
  divergence_kernel<<<grid, block, 0, s>>>(div, ux, uy, uz, mask, nx, ny, nz, dx,
                                           reinterpret_cast<unsigned int *>(max_abs_div));
  return cudaGetLastError();
}

cudaError_t gradient_impl(float *ux, float *uy, float *uz, const float *p, const uint8_t *mask,
                          int nx, int ny, int nz, float dx, float dt, float rho, cudaStream_t s) {
  const float dtr = dt / rho;
  ProfScope ps(PROF_PROJ, s);
  if (nz % 4 == 0 && aligned16_all(p, ux, uy) && ((uintptr_t)mask & 3u) == 0) {
    dim3 block(32, 8);
    dim3 grid((nz / 4 + 31) / 32, (ny + 7) / 8, nx);
    gradient4_kernel<<<grid, block, 0, s>>>(ux, uy, uz, p, mask, nx, ny, nz, dx, dtr);
    return cudaGetLastError();
  }
  dim3 block(128, 2);
  dim3 grid((nz + 127) / 128, (ny + 1) / 2, nx);
  gradient_kernel<<<grid, block, 0, s>>>(ux, uy, uz, p, mask, nx, ny, nz, dx, dtr);
  return cudaGetLastError();
}

static inline bool dims_ok(int nx, int ny, int nz) {
  return nx > 0 && ny > 0 && nz > 0 && nx < 65535 && (int64_t)nx * ny * nz <= ((int64_t)1 << 40);
}

}  // namespace bsp

using namespace bsp;

extern "C" int bsp_divergence(float *div_u, const float *ux, const float *uy, const float *uz,
                              const uint8_t *mask, int nx, int ny, int nz, float dx,
                              float *max_abs_div, cudaStream_t stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!div_u || !ux || !uy || !uz || !mask) return BSP_ERR_NULL;
  if (!dims_ok(nx, ny, nz)) return BSP_ERR_SHAPE;
  return (int)divergence_impl(div_u, ux, uy, uz, mask, nx, ny, nz, dx, max_abs_div, stream);
}

extern "C" int bsp_subtract_gradient(float *ux, float *uy, float *uz, const float *p,
                                     const uint8_t *mask, int nx, int ny, int nz, float dx,
                                     float dt, float rho, cudaStream_t stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!ux || !uy || !uz || !p || !mask) return BSP_ERR_NULL;
  if (!dims_ok(nx, ny, nz)) return BSP_ERR_SHAPE;
  return (int)gradient_impl(ux, uy, uz, p, mask, nx, ny, nz, dx, dt, rho, stream);
}

extern "C" int bsp_enforce_no_slip(float *ux, float *uy, float *uz, const uint8_t *mask, int nx,
                                   int ny, int nz, cudaStream_t stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!ux || !uy || !uz || !mask) return BSP_ERR_NULL;
  if (!dims_ok(nx + 1, ny, nz)) return BSP_ERR_SHAPE;
  dim3 block(128, 2);
  dim3 grid((nz + 1 + 127) / 128, (ny + 2) / 2, nx + 1);
  ProfScope ps(PROF_PROJ, stream);
  no_slip_kernel<<<grid, block, 0, stream>>>(ux, uy, uz, mask, nx, ny, nz);
  return (int)cudaGetLastError();
}

namespace bsp {

cudaError_t noslip_divergence_impl(float *div, float *ux, float *uy, float *uz,
                                   const uint8_t *mask, int nx, int ny, int nz, float dx,
                                   cudaStream_t s) {
  dim3 block(128, 2);
  dim3 grid((nz + 1 + 127) / 128, (ny + 2) / 2, nx + 1);
  ProfScope ps(PROF_PROJ, s);
  noslip_divergence_kernel<<<grid, block, 0, s>>>(div, ux, uy, uz, mask, nx, ny, nz, dx);
  return cudaGetLastError();
}

// The Jacobi projection of fluid.py:612-734; with no_slip it is the
// no-slip / projection / no-slip sequence of pipeline.py:605-619, where the
// first no-slip is fused into the divergence and the second is dropped: the
// gradient subtract only writes faces between two fluid cells, and those are
// exactly the faces no-slip keeps, so the second no-slip would change nothing.
static int projection_jacobi(float *p, float *p_tmp, float *div_u, float *ux, float *uy,
                             float *uz, const uint8_t *mask, int nx, int ny, int nz, float dx,
                             float dt, float rho, int n_iter, int tblock, float *max_div_dev,
                             cudaStream_t stream, bool no_slip) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!p || !p_tmp || !div_u || !ux || !uy || !uz || !mask) return BSP_ERR_NULL;
  if (!dims_ok(nx + 1, ny, nz)) return BSP_ERR_SHAPE;
  if (p == p_tmp) return BSP_ERR_ALIAS;
  const size_t bytes = sizeof(float) * (size_t)nx * ny * nz;
  cudaError_t e = cudaMemsetAsync(p, 0, bytes, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(p_tmp, 0, bytes, stream);
  if (e != cudaSuccess) return (int)e;
  e = no_slip ? noslip_divergence_impl(div_u, ux, uy, uz, mask, nx, ny, nz, dx, stream)
              : divergence_impl(div_u, ux, uy, uz, mask, nx, ny, nz, dx, nullptr, stream);
  if (e != cudaSuccess) return (int)e;
  // div_u belongs to the projection until the diagnostic divergence below
  // overwrites it, so it holds rho dx^2 div / dt (in place) during the sweeps.
  int st = jacobi_solve_impl(p, p_tmp, div_u, div_u, mask, nx, ny, nz, dx, dt, rho, n_iter,
                             tblock, stream, /*p zeroed above*/ true);
  if (st != BSP_OK) return st;
  e = gradient_impl(ux, uy, uz, p, mask, nx, ny, nz, dx, dt, rho, stream);
  if (e != cudaSuccess) return (int)e;
  return (int)divergence_impl(div_u, ux, uy, uz, mask, nx, ny, nz, dx, max_div_dev, stream);
}

}  // namespace bsp

extern "C" int bsp_projection_jacobi(float *p, float *p_tmp, float *div_u, float *ux, float *uy,
                                     float *uz, const uint8_t *mask, int nx, int ny, int nz,
                                     float dx, float dt, float rho, int n_iter, int tblock,
                                     float *max_div_dev, cudaStream_t stream) {
  return projection_jacobi(p, p_tmp, div_u, ux, uy, uz, mask, nx, ny, nz, dx, dt, rho, n_iter,
                           tblock, max_div_dev, stream, false);
}

extern "C" int bsp_step_projection_jacobi(float *p, float *p_tmp, float *div_u, float *ux,
                                          float *uy, float *uz, const uint8_t *mask, int nx,
                                          int ny, int nz, float dx, float dt, float rho,
                                          int n_iter, int tblock, float *max_div_dev,
                                          cudaStream_t stream) {
  return projection_jacobi(p, p_tmp, div_u, ux, uy, uz, mask, nx, ny, nz, dx, dt, rho, n_iter,
                           tblock, max_div_dev, stream, true);
}

extern "C" int bsp_noslip_divergence(float *div_u, float *ux, float *uy, float *uz,
                                     const uint8_t *mask, int nx, int ny, int nz, float dx,
                                     cudaStream_t stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!div_u || !ux || !uy || !uz || !mask) return BSP_ERR_NULL;
  if (!dims_ok(nx + 1, ny, nz)) return BSP_ERR_SHAPE;
  return (int)noslip_divergence_impl(div_u, ux, uy, uz, mask, nx, ny, nz, dx, stream);
}
