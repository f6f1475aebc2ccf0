// advect.cu -- semi-Lagrangian advection of the MAC face velocities and the
// cell-centred temperature.
//
// Reference semantics:
//   _tri_sample, _sample_velocity_at     python/boilingsim/fluid.py:39-104
//   extend_temperature_into_solids       python/boilingsim/fluid.py:338-382
//   advect_temperature                   python/boilingsim/fluid.py:385-411
//   advect_ux / advect_uy / advect_uz    python/boilingsim/fluid.py:414-498
//   advect_all                           python/boilingsim/fluid.py:737-776
//
// Every operation is the reference expression as written, one IEEE single
// rounding each (__fadd_rn / __fmul_rn / __fdiv_rn, no contraction):
//   p      = origin + (idx + offset) * dx           per axis
//   p_back = p - u * dt                             u from three trilinear samples at p
//   f      = (p - origin) / dx - offset, clamped to [0, n - 1 - 1e-6] (float)
//   value  = ((c000 (1-tx) + c100 tx) (1-ty) + (c010 (1-tx) + c110 tx) ty) (1-tz) + ...
// (p - origin) / dx depends on the lattice index only and is computed once per
// CTA for its plane, rows and columns.  The clamp's upper bound rounds to
// n - 1 exactly for n above ~17; the +1 corner is then clamped to n - 1 (the
// reference would read one element past the array there).
//
// One thread per output point and plane, CTAs of 64 k x 4 j marching over 8
// consecutive i planes: the eight corners of each sample are read through the
// read-only cache, and a plane's samples reuse most of the lines fetched for
// the plane before.
#include <cuda_runtime.h>

#include "../../include/bsproj.h"
#include "bsp_common.cuh"

namespace bsp {
namespace sl {

struct Geo {
  int nx, ny, nz;
  float ox, oy, oz, dx, dt;
};

constexpr int BK = 64, BJ = 4, PL = 8;  // CTA: 64 k x 4 j, marching 8 planes

// Trilinear sample of field f (shape fxn x fyn x fzn, lattice offset (sx, sy,
// sz)) at the point whose scaled coordinates (p - origin) / dx are (gx, gy, gz).
// Offsets are 32-bit (fields hold fewer than 2^31 elements).
__device__ __forceinline__ float tri(const float *__restrict__ f, int fxn, int fyn, int fzn,
                                     float gx, float gy, float gz, float sx, float sy, float sz) {
  float fx = __fsub_rn(gx, sx), fy = __fsub_rn(gy, sy), fz = __fsub_rn(gz, sz);
  fx = fminf(fmaxf(fx, 0.0f), __fsub_rn((float)(fxn - 1), 1.0e-6f));
  fy = fminf(fmaxf(fy, 0.0f), __fsub_rn((float)(fyn - 1), 1.0e-6f));
  fz = fminf(fmaxf(fz, 0.0f), __fsub_rn((float)(fzn - 1), 1.0e-6f));
  const int i0 = __float2int_rz(fx), j0 = __float2int_rz(fy), k0 = __float2int_rz(fz);
  const float tx = __fsub_rn(fx, (float)i0), ty = __fsub_rn(fy, (float)j0),
              tz = __fsub_rn(fz, (float)k0);
  const int pl = fyn * fzn;
  const int di = i0 + 1 < fxn ? pl : 0, dj = j0 + 1 < fyn ? fzn : 0, dk = k0 + 1 < fzn ? 1 : 0;
  const float *q = f + (i0 * pl + j0 * fzn + k0);
  const float c000 = __ldg(q), c001 = __ldg(q + dk);
  const float c010 = __ldg(q + dj), c011 = __ldg(q + dj + dk);
  const float c100 = __ldg(q + di), c101 = __ldg(q + di + dk);
  const float c110 = __ldg(q + di + dj), c111 = __ldg(q + di + dj + dk);
  const float ux = __fsub_rn(1.0f, tx), uy = __fsub_rn(1.0f, ty), uz = __fsub_rn(1.0f, tz);
  const float c00 = __fadd_rn(__fmul_rn(c000, ux), __fmul_rn(c100, tx));
  const float c10 = __fadd_rn(__fmul_rn(c010, ux), __fmul_rn(c110, tx));
  const float c01 = __fadd_rn(__fmul_rn(c001, ux), __fmul_rn(c101, tx));
  const float c11 = __fadd_rn(__fmul_rn(c011, ux), __fmul_rn(c111, tx));
  const float c0 = __fadd_rn(__fmul_rn(c00, uy), __fmul_rn(c10, ty));
  const float c1 = __fadd_rn(__fmul_rn(c01, uy), __fmul_rn(c11, ty));
  return __fadd_rn(__fmul_rn(c0, uz), __fmul_rn(c1, tz));
}

// World and scaled coordinates of a CTA's lattice points, computed once per
// CTA: p = origin + (idx + s) dx and g = (p - origin) / dx per axis for its
// plane i, its BJ rows and its BK columns (they depend on the index only).
struct Coords {
  float px[PL], gx[PL], py[BJ], gy[BJ], pz[BK], gz[BK];
};

__device__ __forceinline__ void coords(Coords &c, float sx, float sy, float sz, const Geo &g) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  if (ty == 0) {
    const int k = blockIdx.x * BK + tx;
    const float p = __fadd_rn(g.oz, __fmul_rn(__fadd_rn((float)k, sz), g.dx));
    c.pz[tx] = p;
    c.gz[tx] = __fdiv_rn(__fsub_rn(p, g.oz), g.dx);
  } else if (ty == 1 && tx < BJ) {
    const int j = blockIdx.y * BJ + tx;
    const float p = __fadd_rn(g.oy, __fmul_rn(__fadd_rn((float)j, sy), g.dx));
    c.py[tx] = p;
    c.gy[tx] = __fdiv_rn(__fsub_rn(p, g.oy), g.dx);
  } else if (ty == 2 && tx < PL) {
    const int i = blockIdx.z * PL + tx;
    const float p = __fadd_rn(g.ox, __fmul_rn(__fadd_rn((float)i, sx), g.dx));
    c.px[tx] = p;
    c.gx[tx] = __fdiv_rn(__fsub_rn(p, g.ox), g.dx);
  }
  __syncthreads();
}

// The velocity at the point (three samples at its scaled coordinates) and the
// backtraced point's scaled coordinates.
__device__ __forceinline__ void backtrace(float &bx, float &by, float &bz, const Coords &c,
                                          int ii, const float *__restrict__ ux,
                                          const float *__restrict__ uy,
                                          const float *__restrict__ uz, const Geo &g) {
  const float px = c.px[ii], gx = c.gx[ii];
  const float py = c.py[threadIdx.y], gy = c.gy[threadIdx.y];
  const float pz = c.pz[threadIdx.x], gz = c.gz[threadIdx.x];
  const float u = tri(ux, g.nx + 1, g.ny, g.nz, gx, gy, gz, 0.0f, 0.5f, 0.5f);
  const float v = tri(uy, g.nx, g.ny + 1, g.nz, gx, gy, gz, 0.5f, 0.0f, 0.5f);
  const float w = tri(uz, g.nx, g.ny, g.nz + 1, gx, gy, gz, 0.5f, 0.5f, 0.0f);
  const float qx = __fsub_rn(px, __fmul_rn(u, g.dt));
  const float qy = __fsub_rn(py, __fmul_rn(v, g.dt));
  const float qz = __fsub_rn(pz, __fmul_rn(w, g.dt));
  bx = __fdiv_rn(__fsub_rn(qx, g.ox), g.dx);
  by = __fdiv_rn(__fsub_rn(qy, g.oy), g.dx);
  bz = __fdiv_rn(__fsub_rn(qz, g.oz), g.dx);
}

__device__ __forceinline__ bool fluid(const uint8_t *__restrict__ m, int64_t c) {
  return (__ldg(m + c) & BSP_MFLUID) != 0;
}

__global__ void __launch_bounds__(BK *BJ) extend_kernel(float *__restrict__ T_ext,
                                                        const float *__restrict__ T,
                                                        const uint8_t *__restrict__ m, int nx,
                                                        int ny, int nz) {
  const int k = blockIdx.x * BK + threadIdx.x, j = blockIdx.y * BJ + threadIdx.y;
  if (k >= nz || j >= ny) return;
  const int64_t pl = (int64_t)ny * nz;
  for (int ii = 0; ii < PL; ++ii) {
    const int i = blockIdx.z * PL + ii;
    if (i >= nx) break;
    const int64_t c = i * pl + (int64_t)j * nz + k;
    int64_t s = c;
    if (!fluid(m, c)) {
      // the six neighbour flags are loaded together, then the first fluid one
      // in the order -x, +x, -y, +y, -z, +z is taken
      const bool f0 = i > 0 && fluid(m, c - pl), f1 = i < nx - 1 && fluid(m, c + pl);
      const bool f2 = j > 0 && fluid(m, c - nz), f3 = j < ny - 1 && fluid(m, c + nz);
      const bool f4 = k > 0 && fluid(m, c - 1), f5 = k < nz - 1 && fluid(m, c + 1);
      s = f0 ? c - pl : f1 ? c + pl : f2 ? c - nz : f3 ? c + nz : f4 ? c - 1 : f5 ? c + 1 : c;
    }
    T_ext[c] = __ldg(T + s);
  }
}

__global__ void __launch_bounds__(BK *BJ) advect_T_kernel(
    float *__restrict__ T_new, const float *__restrict__ T_true, const float *__restrict__ T_ext,
    const float *__restrict__ ux, const float *__restrict__ uy, const float *__restrict__ uz,
    const uint8_t *__restrict__ m, Geo g) {
  __shared__ Coords cs;
  const int k = blockIdx.x * BK + threadIdx.x, j = blockIdx.y * BJ + threadIdx.y;
  coords(cs, 0.5f, 0.5f, 0.5f, g);
  if (k >= g.nz || j >= g.ny) return;
  for (int ii = 0; ii < PL; ++ii) {
    const int i = blockIdx.z * PL + ii;
    if (i >= g.nx) break;
    const int64_t c = ((int64_t)i * g.ny + j) * g.nz + k;
    if (!fluid(m, c)) {
      T_new[c] = __ldg(T_true + c);
      continue;
    }
    float bx, by, bz;
    backtrace(bx, by, bz, cs, ii, ux, uy, uz, g);
    T_new[c] = tri(T_ext, g.nx, g.ny, g.nz, bx, by, bz, 0.5f, 0.5f, 0.5f);
  }
}

template <int AX>
__global__ void __launch_bounds__(BK *BJ) advect_u_kernel(float *__restrict__ u_new,
                                                          const float *__restrict__ ux,
                                                          const float *__restrict__ uy,
                                                          const float *__restrict__ uz,
                                                          const uint8_t *__restrict__ m, Geo g) {
  __shared__ Coords cs;
  const int fxn = g.nx + (AX == 0), fyn = g.ny + (AX == 1), fzn = g.nz + (AX == 2);
  const int k = blockIdx.x * BK + threadIdx.x, j = blockIdx.y * BJ + threadIdx.y;
  const float sx = AX == 0 ? 0.0f : 0.5f, sy = AX == 1 ? 0.0f : 0.5f, sz = AX == 2 ? 0.0f : 0.5f;
  coords(cs, sx, sy, sz, g);
  if (k >= fzn || j >= fyn) return;
  const float *__restrict__ u = AX == 0 ? ux : (AX == 1 ? uy : uz);
  const int64_t pl = (int64_t)g.ny * g.nz;
  for (int ii = 0; ii < PL; ++ii) {
    const int i = blockIdx.z * PL + ii;
    if (i >= fxn) break;
    const int64_t f = ((int64_t)i * fyn + j) * fzn + k;
    const int a = AX == 0 ? i : (AX == 1 ? j : k);
    const int na = AX == 0 ? fxn : (AX == 1 ? fyn : fzn);
    if (a == 0 || a == na - 1) {
      u_new[f] = 0.0f;
      continue;
    }
    const int64_t c1 = i * pl + (int64_t)j * g.nz + k;
    const int64_t c0 = AX == 0 ? c1 - pl : (AX == 1 ? c1 - g.nz : c1 - 1);
    if (!fluid(m, c0) && !fluid(m, c1)) {
      u_new[f] = __ldg(u + f);
      continue;
    }
    float bx, by, bz;
    backtrace(bx, by, bz, cs, ii, ux, uy, uz, g);
    u_new[f] = tri(u, fxn, fyn, fzn, bx, by, bz, sx, sy, sz);
  }
}

// CTAs of the kernels: 64 k x 4 j, PL planes each
inline dim3 grid_pl(int nx, int ny, int nz) {
  return dim3((unsigned)((nz + BK - 1) / BK), (unsigned)((ny + BJ - 1) / BJ),
              (unsigned)((nx + PL - 1) / PL));
}

cudaError_t launch_velocity(int axis, float *u_new, const float *ux, const float *uy,
                            const float *uz, const uint8_t *m, const Geo &g, cudaStream_t s) {
  const dim3 blk(BK, BJ);
  if (axis == 0)
    advect_u_kernel<0><<<grid_pl(g.nx + 1, g.ny, g.nz), blk, 0, s>>>(u_new, ux, uy, uz, m, g);
  else if (axis == 1)
    advect_u_kernel<1><<<grid_pl(g.nx, g.ny + 1, g.nz), blk, 0, s>>>(u_new, ux, uy, uz, m, g);
  else
    advect_u_kernel<2><<<grid_pl(g.nx, g.ny, g.nz + 1), blk, 0, s>>>(u_new, ux, uy, uz, m, g);
  return cudaGetLastError();
}

bool dims_ok(int nx, int ny, int nz) {
  // grid.z = nx + 1 planes and grid.y = ceil((ny + 1) / BJ) rows must fit the launch limits;
  // the samplers use 32-bit element offsets
  return nx + 1 <= 65535 && (ny + 1 + BJ - 1) / BJ <= 65535 &&
         (int64_t)(nx + 1) * (ny + 1) * (nz + 1) < (1LL << 31);
}

}  // namespace sl
}  // namespace bsp

using namespace bsp::sl;

extern "C" int bsp_extend_temperature(float *T_ext, const float *T, const uint8_t *mask, int nx,
                                      int ny, int nz, cudaStream_t s) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!T_ext || !T || !mask) return BSP_ERR_NULL;
  if (T_ext == T) return BSP_ERR_ALIAS;
  if (!dims_ok(nx, ny, nz)) return BSP_ERR_SHAPE;
  extend_kernel<<<grid_pl(nx, ny, nz), dim3(BK, BJ), 0, s>>>(T_ext, T, mask, nx, ny, nz);
  return (int)cudaGetLastError();
}

extern "C" int bsp_advect_temperature(float *T_new, const float *T_true, const float *T_ext,
                                      const float *ux, const float *uy, const float *uz,
                                      const uint8_t *mask, int nx, int ny, int nz, float ox,
                                      float oy, float oz, float dx, float dt, cudaStream_t s) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!T_new || !T_true || !T_ext || !ux || !uy || !uz || !mask) return BSP_ERR_NULL;
  if (T_new == T_true || T_new == T_ext) return BSP_ERR_ALIAS;
  if (!dims_ok(nx, ny, nz) || !(dx > 0.0f)) return BSP_ERR_SHAPE;
  const Geo g{nx, ny, nz, ox, oy, oz, dx, dt};
  advect_T_kernel<<<grid_pl(nx, ny, nz), dim3(BK, BJ), 0, s>>>(T_new, T_true, T_ext, ux, uy,
                                                                 uz, mask, g);
  return (int)cudaGetLastError();
}

extern "C" int bsp_advect_velocity(int axis, float *u_new, const float *ux, const float *uy,
                                   const float *uz, const uint8_t *mask, int nx, int ny, int nz,
                                   float ox, float oy, float oz, float dx, float dt,
                                   cudaStream_t s) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!u_new || !ux || !uy || !uz || !mask) return BSP_ERR_NULL;
  if (axis < 0 || axis > 2) return BSP_ERR_ARG;
  if (u_new == ux || u_new == uy || u_new == uz) return BSP_ERR_ALIAS;
  if (!dims_ok(nx, ny, nz) || !(dx > 0.0f)) return BSP_ERR_SHAPE;
  const Geo g{nx, ny, nz, ox, oy, oz, dx, dt};
  return (int)launch_velocity(axis, u_new, ux, uy, uz, mask, g, s);
}

extern "C" int bsp_advect_all(float *ux, float *uy, float *uz, float *T, float *ux_tmp,
                              float *uy_tmp, float *uz_tmp, float *T_tmp, float *T_ext,
                              const uint8_t *mask, int nx, int ny, int nz, float ox, float oy,
                              float oz, float dx, float dt, int copy_back, cudaStream_t s) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!ux || !uy || !uz || !T || !ux_tmp || !uy_tmp || !uz_tmp || !T_tmp || !T_ext || !mask)
    return BSP_ERR_NULL;
  const float *outs[] = {ux_tmp, uy_tmp, uz_tmp, T_tmp, T_ext};
  const float *ins[] = {ux, uy, uz, T};
  for (const float *o : outs)
    for (const float *in : ins)
      if (o == in) return BSP_ERR_ALIAS;
  // the five outputs are written by different kernels while T_ext is still
  // being sampled: no two may share a base, and none may be the mask
  for (int a = 0; a < 5; ++a) {
    if ((const void *)outs[a] == (const void *)mask) return BSP_ERR_ALIAS;
    for (int b = a + 1; b < 5; ++b)
      if (outs[a] == outs[b]) return BSP_ERR_ALIAS;
  }
  if (!dims_ok(nx, ny, nz) || !(dx > 0.0f)) return BSP_ERR_SHAPE;
  const Geo g{nx, ny, nz, ox, oy, oz, dx, dt};
  cudaError_t e = cudaSuccess;
  for (int ax = 0; ax < 3 && e == cudaSuccess; ++ax)
    e = launch_velocity(ax, ax == 0 ? ux_tmp : (ax == 1 ? uy_tmp : uz_tmp), ux, uy, uz, mask, g,
                        s);
  if (e != cudaSuccess) return (int)e;
  extend_kernel<<<grid_pl(nx, ny, nz), dim3(BK, BJ), 0, s>>>(T_ext, T, mask, nx, ny, nz);
  advect_T_kernel<<<grid_pl(nx, ny, nz), dim3(BK, BJ), 0, s>>>(T_tmp, T, T_ext, ux, uy, uz,
                                                                 mask, g);
  e = cudaGetLastError();
  if (e != cudaSuccess || !copy_back) return (int)e;
  const size_t c = sizeof(float) * (size_t)nx * ny * nz;
  const size_t fx = sizeof(float) * (size_t)(nx + 1) * ny * nz;
  const size_t fy = sizeof(float) * (size_t)nx * (ny + 1) * nz;
  const size_t fz = sizeof(float) * (size_t)nx * ny * (nz + 1);
  e = cudaMemcpyAsync(ux, ux_tmp, fx, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(uy, uy_tmp, fy, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(uz, uz_tmp, fz, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(T, T_tmp, c, cudaMemcpyDeviceToDevice, s);
  return (int)e;
}
