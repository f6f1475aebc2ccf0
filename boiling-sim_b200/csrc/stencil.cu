// stencil.cu -- masked 7-point stencils on the MAC grid: Jacobi sweep, A*p, D^-1 r.
//
// Reference semantics:
//   jacobi_pressure_step   python/boilingsim/fluid.py:243-276
//   _pressure_neighbour    python/boilingsim/fluid.py:222-240
//   out-of-range = air     crates/cuda-kernels/src/jacobi_pressure.cu:121-124
//   laplacian_spmv_kernel  crates/cuda-kernels/src/laplacian_spmv.cu:62-143
//   diag_inverse_apply     crates/cuda-kernels/src/diag_inverse_apply.cu:44-89
//
// Two kernel shapes:
//   * column kernel (nz % 4 == 0, 16-byte aligned fields): a CTA is 8 warps; each
//     warp owns one j row and 128 consecutive k cells (one float4 per lane) and
//     marches along i with the i-1 / i / i+1 planes held in registers.  Per cell
//     HBM sees p(i+1), div, mask(i+1) and the store: 13 B/cell/sweep on the uint8
//     mask (16 with int32 mat).  j neighbours come from L1 (the next warp's
//     centre row), k neighbours from warp shuffles.
//   * generic kernel: one thread per cell, any shape or alignment.
// Both produce bit-identical results (same per-cell operation order).
#include "bsp_common.cuh"

namespace bsp {

// ---- class loads -----------------------------------------------------------
__device__ __forceinline__ uint32_t cls1(const uint8_t *m, int64_t c, int, int) {
  return mcls(__ldg(m + c));
}
__device__ __forceinline__ uint32_t cls1(const int32_t *m, int64_t c, int mf, int ma) {
  return classify(__ldg(m + c), mf, ma);
}
__device__ __forceinline__ uint32_t cls4(const uint8_t *m, int64_t c, int, int) {
  return __ldg(reinterpret_cast<const uint32_t *>(m + c)) & 0x03030303u;
}
__device__ __forceinline__ uint32_t cls4(const int32_t *m, int64_t c, int mf, int ma) {
  int4 v = __ldg(reinterpret_cast<const int4 *>(m + c));
  return classify(v.x, mf, ma) | (classify(v.y, mf, ma) << 8) |
         (classify(v.z, mf, ma) << 16) | (classify(v.w, mf, ma) << 24);
}

constexpr uint32_t AIR4 = 0x01010101u;

enum Op { OP_JACOBI = 0, OP_SPMV = 1 };

__device__ __forceinline__ float f4(const float4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}

// ---- column kernel ----------------------------------------------------------
template <int OP, class MaskT>
__global__ void __launch_bounds__(256) stencil_col_kernel(
    float *__restrict__ out, const float *__restrict__ p, const float *__restrict__ div,
    const MaskT *__restrict__ mask, int nx, int ny, int nz, int bi, float rdd, float dt,
    int mf, int ma) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nz4 = nz >> 2;
  const int k4 = blockIdx.x * 32 + lane;
  const int j = blockIdx.y * 8 + warp;
  if (j >= ny) return;  // warp-uniform
  const int i0 = blockIdx.z * bi;
  const int i1 = min(i0 + bi, nx);
  const bool act = k4 < nz4;
  const int k = k4 * 4;
  const int64_t plane = (int64_t)ny * nz;
  const int64_t col = (int64_t)j * nz + k;
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);

  float4 pm = zero4, pc = zero4;
  uint32_t cmm = AIR4, cmc = AIR4;
  if (act && i0 - 1 >= 0) {
    pm = __ldg(reinterpret_cast<const float4 *>(p + (i0 - 1) * plane + col));
    cmm = cls4(mask, (i0 - 1) * plane + col, mf, ma);
  }
  if (act) {
    pc = __ldg(reinterpret_cast<const float4 *>(p + i0 * plane + col));
    cmc = cls4(mask, i0 * plane + col, mf, ma);
  }
  for (int i = i0; i < i1; ++i) {
    const int64_t base = i * plane + col;
    float4 pn = zero4, pjm = zero4, pjp = zero4, dv = zero4;
    uint32_t cmn = AIR4, cjm = AIR4, cjp = AIR4;
    if (act) {
      if (i + 1 < nx) {
        pn = __ldg(reinterpret_cast<const float4 *>(p + base + plane));
        cmn = cls4(mask, base + plane, mf, ma);
      }
      if (j > 0) {
        pjm = __ldg(reinterpret_cast<const float4 *>(p + base - nz));
        cjm = cls4(mask, base - nz, mf, ma);
      }
      if (j + 1 < ny) {
        pjp = __ldg(reinterpret_cast<const float4 *>(p + base + nz));
        cjp = cls4(mask, base + nz, mf, ma);
      }
      if (OP == OP_JACOBI) dv = __ldg(reinterpret_cast<const float4 *>(div + base));
    }
    // k neighbours across lanes
    float pkm = __shfl_up_sync(0xffffffffu, pc.w, 1);
    uint32_t ckm = __shfl_up_sync(0xffffffffu, cmc, 1) >> 24;
    float pkp = __shfl_down_sync(0xffffffffu, pc.x, 1);
    uint32_t ckp = __shfl_down_sync(0xffffffffu, cmc, 1) & 0xffu;
    if (lane == 0) {
      pkm = 0.f;
      ckm = BSP_AIR;
      if (act && k > 0) {
        pkm = __ldg(p + base - 1);
        ckm = cls1(mask, base - 1, mf, ma);
      }
    }
    if (lane == 31) {
      pkp = 0.f;
      ckp = BSP_AIR;
      if (act && k + 4 < nz) {
        pkp = __ldg(p + base + 4);
        ckp = cls1(mask, base + 4, mf, ma);
      }
    }
    if (act) {
      float o[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint32_t cs = byte_of(cmc, q);
        const float ps = f4(pc, q);
        const float l = nbr(byte_of(cmm, q), f4(pm, q), ps);
        const float r = nbr(byte_of(cmn, q), f4(pn, q), ps);
        const float d = nbr(byte_of(cjm, q), f4(pjm, q), ps);
        const float u = nbr(byte_of(cjp, q), f4(pjp, q), ps);
        const float b = q == 0 ? nbr(ckm, pkm, ps) : nbr(byte_of(cmc, q - 1), f4(pc, q - 1), ps);
        const float f = q == 3 ? nbr(ckp, pkp, ps) : nbr(byte_of(cmc, q + 1), f4(pc, q + 1), ps);
        float v;
        if (OP == OP_JACOBI)
          v = jacobi_update(l, r, d, u, b, f, f4(dv, q), rdd, dt);
        else
          v = spmv_update(l, r, d, u, b, f, ps);
        o[q] = cs == BSP_FLUID ? v : 0.0f;
      }
      *reinterpret_cast<float4 *>(out + base) = make_float4(o[0], o[1], o[2], o[3]);
    }
    pm = pc;
    cmm = cmc;
    pc = pn;
    cmc = cmn;
  }
}

// ---- generic kernel -----------------------------------------------------------
template <int OP, class MaskT>
__global__ void __launch_bounds__(256) stencil_generic_kernel(
    float *__restrict__ out, const float *__restrict__ p, const float *__restrict__ div,
    const MaskT *__restrict__ mask, int nx, int ny, int nz, float rdd, float dt, int mf,
    int ma) {
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(c % nz);
    const int64_t t = c / nz;
    const int j = (int)(t % ny);
    const int i = (int)(t / ny);
    if (cls1(mask, c, mf, ma) != BSP_FLUID) {
      out[c] = 0.0f;
      continue;
    }
    const float ps = __ldg(p + c);
    const int64_t plane = (int64_t)ny * nz;
#define NBR(cond, off) \
  ((cond) ? nbr(cls1(mask, c + (off), mf, ma), __ldg(p + c + (off)), ps) : 0.0f)
    const float l = NBR(i > 0, -plane), r = NBR(i + 1 < nx, plane);
    const float d = NBR(j > 0, -(int64_t)nz), u = NBR(j + 1 < ny, (int64_t)nz);
    const float b = NBR(k > 0, -1), f = NBR(k + 1 < nz, 1);
#undef NBR
    out[c] = OP == OP_JACOBI ? jacobi_update(l, r, d, u, b, f, __ldg(div + c), rdd, dt)
                             : spmv_update(l, r, d, u, b, f, ps);
  }
}

// ---- diagonal preconditioner ------------------------------------------------------
template <class MaskT>
__global__ void __launch_bounds__(256) diag_inverse_kernel(float *__restrict__ z,
                                                           const float *__restrict__ r,
                                                           const MaskT *__restrict__ mask,
                                                           int nx, int ny, int nz, int mf,
                                                           int ma) {
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (cls1(mask, c, mf, ma) != BSP_FLUID) {
      z[c] = 0.0f;
      continue;
    }
    const int k = (int)(c % nz);
    const int64_t t = c / nz;
    const int j = (int)(t % ny);
    const int i = (int)(t / ny);
    const int64_t plane = (int64_t)ny * nz;
    int ns = 0;
#define SOL(cond, off) ns += ((cond) && cls1(mask, c + (off), mf, ma) == BSP_SOLID) ? 1 : 0
    SOL(i > 0, -plane);
    SOL(i + 1 < nx, plane);
    SOL(j > 0, -(int64_t)nz);
    SOL(j + 1 < ny, (int64_t)nz);
    SOL(k > 0, -1);
    SOL(k + 1 < nz, 1);
#undef SOL
    const float diag = 6.0f - (float)ns;
    z[c] = diag <= 0.0f ? r[c] : __fdiv_rn(r[c], diag);
  }
}

// mask byte = class | n_solid << 2 (n_solid counts face neighbours that are
// neither fluid nor air; out-of-range neighbours are air).
__global__ void mask_from_mat_kernel(uint8_t *__restrict__ mask, const int32_t *__restrict__ mat,
                                     int nx, int ny, int nz, int mf, int ma) {
  const int64_t n = (int64_t)nx * ny * nz;
  const int64_t plane = (int64_t)ny * nz;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(c % nz);
    const int64_t t = c / nz;
    const int j = (int)(t % ny);
    const int i = (int)(t / ny);
    const uint32_t cls = classify(__ldg(mat + c), mf, ma);
    uint32_t ns = 0;
#define SOL(cond, off) ns += ((cond) && classify(__ldg(mat + c + (off)), mf, ma) == BSP_SOLID) ? 1u : 0u
    SOL(i > 0, -plane);
    SOL(i + 1 < nx, plane);
    SOL(j > 0, -(int64_t)nz);
    SOL(j + 1 < ny, (int64_t)nz);
    SOL(k > 0, -1);
    SOL(k + 1 < nz, 1);
#undef SOL
    mask[c] = (uint8_t)(cls | (ns << 2));
  }
}

__global__ void selftest_div6_kernel(unsigned long long *bad) {
  unsigned long long local = 0;
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u <= 0xffffffffull;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const float x = __uint_as_float((uint32_t)u);
    const float a = __fdiv_rn(x, 6.0f), b = div6(x);
    const bool both_nan = (a != a) && (b != b);
    if (!both_nan && __float_as_uint(a) != __float_as_uint(b)) ++local;
  }
  if (local) atomicAdd(bad, local);
}

// ---- launch helpers --------------------------------------------------------------
static int g_num_sms = 0;
int num_sms() {
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

static inline bool aligned16(const void *ptr) { return ((uintptr_t)ptr & 15u) == 0; }

static inline int generic_blocks(int64_t n) {
  int64_t b = (n + 255) / 256;
  int64_t cap = (int64_t)num_sms() * 16;
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

// i-extent per CTA of the column kernel: enough CTAs for ~8 waves of 148 SMs
// while keeping the i-halo re-read (2/bi) small.
static inline int pick_bi(int nx, int ny, int nz) {
  const int64_t cols = (int64_t)((nz / 4 + 31) / 32) * ((ny + 7) / 8);
  const int64_t target = (int64_t)num_sms() * 8;
  int bi = 64;
  while (bi > 4 && cols * ((nx + bi - 1) / bi) < target) bi >>= 1;
  return bi;
}

template <int OP, class MaskT>
cudaError_t launch_stencil(float *out, const float *p, const float *div, const MaskT *mask,
                           int nx, int ny, int nz, float dx, float dt, float rho, int mf,
                           int ma, cudaStream_t s) {
  const float rdd = rho * dx * dx;  // (rho*dx)*dx in float, as the reference evaluates it
  const bool col_ok = (nz % 4 == 0) && aligned16(out) && aligned16(p) &&
                      (OP != OP_JACOBI || aligned16(div)) &&
                      (sizeof(MaskT) == 4 ? aligned16(mask) : (((uintptr_t)mask & 3u) == 0));
  if (col_ok) {
    const int bi = pick_bi(nx, ny, nz);
    dim3 grid((nz / 4 + 31) / 32, (ny + 7) / 8, (nx + bi - 1) / bi);
    stencil_col_kernel<OP, MaskT><<<grid, 256, 0, s>>>(out, p, div, mask, nx, ny, nz, bi, rdd,
                                                       dt, mf, ma);
  } else {
    const int64_t n = (int64_t)nx * ny * nz;
    stencil_generic_kernel<OP, MaskT><<<generic_blocks(n), 256, 0, s>>>(out, p, div, mask, nx,
                                                                        ny, nz, rdd, dt, mf, ma);
  }
  return cudaGetLastError();
}

template cudaError_t launch_stencil<OP_JACOBI, uint8_t>(float *, const float *, const float *,
                                                        const uint8_t *, int, int, int, float,
                                                        float, float, int, int, cudaStream_t);
template cudaError_t launch_stencil<OP_SPMV, uint8_t>(float *, const float *, const float *,
                                                      const uint8_t *, int, int, int, float,
                                                      float, float, int, int, cudaStream_t);

static inline bool shape_ok(int nx, int ny, int nz) {
  return (int64_t)nx * ny * nz <= (int64_t)1 << 40;
}

}  // namespace bsp

using namespace bsp;

// ===================================================================================
// reference-compatible launchers
// ===================================================================================

extern "C" cudaError_t jacobi_pressure_launch(float *p_new, const float *p_old,
                                              const float *div_u, const int *mat, int nx,
                                              int ny, int nz, float dx, float dt, float rho,
                                              int mat_fluid, int mat_air) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return cudaSuccess;
  return launch_stencil<OP_JACOBI, int32_t>(p_new, p_old, div_u, mat, nx, ny, nz, dx, dt, rho,
                                            mat_fluid, mat_air, 0);
}

extern "C" cudaError_t pressure_solve_launch(float *p, float *p_tmp, const float *div_u,
                                             const int *mat, int nx, int ny, int nz, float dx,
                                             float dt, float rho, int n_iter, int mat_fluid,
                                             int mat_air) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || n_iter <= 0) return cudaSuccess;
  for (int it = 0; it < n_iter; ++it) {
    float *dst = (it & 1) == 0 ? p_tmp : p;
    const float *src = (it & 1) == 0 ? p : p_tmp;
    cudaError_t e = launch_stencil<OP_JACOBI, int32_t>(dst, src, div_u, mat, nx, ny, nz, dx,
                                                       dt, rho, mat_fluid, mat_air, 0);
    if (e != cudaSuccess) return e;
  }
  if (n_iter & 1) {
    cudaError_t e = cudaMemcpyAsync(p, p_tmp, sizeof(float) * (size_t)nx * ny * nz,
                                    cudaMemcpyDeviceToDevice, 0);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

extern "C" cudaError_t laplacian_spmv_launch(float *Ap, const float *p, const int *mat, int nx,
                                             int ny, int nz, int mat_fluid, int mat_air) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return cudaSuccess;
  return launch_stencil<OP_SPMV, int32_t>(Ap, p, nullptr, mat, nx, ny, nz, 0.f, 1.f, 0.f,
                                          mat_fluid, mat_air, 0);
}

extern "C" cudaError_t diag_inverse_apply_launch(float *z, const float *r, const int *mat,
                                                 int nx, int ny, int nz, int mat_fluid,
                                                 int mat_air) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return cudaSuccess;
  const int64_t n = (int64_t)nx * ny * nz;
  diag_inverse_kernel<int32_t><<<generic_blocks(n), 256>>>(z, r, mat, nx, ny, nz, mat_fluid,
                                                           mat_air);
  return cudaGetLastError();
}

// ===================================================================================
// bsp_* entry points
// ===================================================================================

extern "C" int bsp_mask_from_mat(uint8_t *mask, const int32_t *mat, int nx, int ny, int nz,
                                 int mat_fluid, int mat_air, cudaStream_t stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!mask || !mat) return BSP_ERR_NULL;
  if (!shape_ok(nx, ny, nz)) return BSP_ERR_SHAPE;
  const int64_t n = (int64_t)nx * ny * nz;
  mask_from_mat_kernel<<<generic_blocks(n), 256, 0, stream>>>(mask, mat, nx, ny, nz, mat_fluid,
                                                              mat_air);
  return (int)cudaGetLastError();
}

extern "C" int bsp_jacobi_sweep(float *p_new, const float *p_old, const float *div_u,
                                const uint8_t *mask, int nx, int ny, int nz, float dx, float dt,
                                float rho, cudaStream_t stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!p_new || !p_old || !div_u || !mask) return BSP_ERR_NULL;
  if (!shape_ok(nx, ny, nz)) return BSP_ERR_SHAPE;
  if (p_new == p_old) return BSP_ERR_ALIAS;
  return (int)launch_stencil<OP_JACOBI, uint8_t>(p_new, p_old, div_u, mask, nx, ny, nz, dx, dt,
                                                 rho, BSP_FLUID, BSP_AIR, stream);
}

extern "C" int bsp_spmv(float *Ap, const float *p, const uint8_t *mask, int nx, int ny, int nz,
                        cudaStream_t stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!Ap || !p || !mask) return BSP_ERR_NULL;
  if (Ap == p) return BSP_ERR_ALIAS;
  return (int)launch_stencil<OP_SPMV, uint8_t>(Ap, p, nullptr, mask, nx, ny, nz, 0.f, 1.f, 0.f,
                                               BSP_FLUID, BSP_AIR, stream);
}

extern "C" int bsp_selftest_div6(unsigned long long *mismatches_dev, cudaStream_t stream) {
  if (!mismatches_dev) return BSP_ERR_NULL;
  cudaError_t e = cudaMemsetAsync(mismatches_dev, 0, sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return (int)e;
  selftest_div6_kernel<<<num_sms() * 8, 256, 0, stream>>>(mismatches_dev);
  return (int)cudaGetLastError();
}
