// mgfine.cu -- fine-level (level 0) kernels of the to-tolerance solver on the
// column layout of the sweep kernel.
//
// One generic driver, fine_col_kernel<Op>: a CTA is 8 warps; warp w owns fine
// row j = 8*blockIdx.y + w and 128 consecutive k cells (4 per lane) and marches
// i over an even-length chunk.  The Op supplies the stencil operand of a cell
// (ps for A*ps; OMEGA r / D for the smoothers, plus the coarse correction for
// the prolongation) and consumes, per cell, the centre operand and the
// neighbour sum s = l + r + d + u + b + f under the boundary rule (fluid ->
// operand, air -> 0, solid -> centre operand).  Operand planes i-1, i, i+1 and
// their mask words stay in registers; rows j +- 1 are formed from L1-resident
// loads; k +- 1 arrive by warp shuffles; neighbour selection is branch-free
// (sel_nbr).
//
// Requirements (checked by the caller; otherwise the row kernels of solver.cu
// run): nz % 4 == 0 and 16-byte aligned level-0 fields.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "bsp_common.cuh"
#include "solver.cuh"

namespace bsp {

constexpr float FOMEGA = 6.0f / 7.0f;

// ---- 4-wide storage access -----------------------------------------------------------
__device__ __forceinline__ float4 ld4s(const float *p, int64_t o) {
  return *reinterpret_cast<const float4 *>(p + o);
}
__device__ __forceinline__ float4 ld4s(const __half *p, int64_t o) {
  const uint2 u = *reinterpret_cast<const uint2 *>(p + o);
  const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 ld4s(const __nv_bfloat16 *p, int64_t o) {
  const uint2 u = *reinterpret_cast<const uint2 *>(p + o);
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void st4s(float *p, int64_t o, float4 v) {
  *reinterpret_cast<float4 *>(p + o) = v;
}
__device__ __forceinline__ void st4s(__half *p, int64_t o, float4 v) {
  __half2 a = __floats2half2_rn(v.x, v.y), b = __floats2half2_rn(v.z, v.w);
  uint2 u;
  u.x = *reinterpret_cast<uint32_t *>(&a);
  u.y = *reinterpret_cast<uint32_t *>(&b);
  *reinterpret_cast<uint2 *>(p + o) = u;
}
__device__ __forceinline__ void st4s(__nv_bfloat16 *p, int64_t o, float4 v) {
  __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
  uint2 u;
  u.x = *reinterpret_cast<uint32_t *>(&a);
  u.y = *reinterpret_cast<uint32_t *>(&b);
  *reinterpret_cast<uint2 *>(p + o) = u;
}
__device__ __forceinline__ float2 ld2s(const float *p, int64_t o) {
  return *reinterpret_cast<const float2 *>(p + o);
}
__device__ __forceinline__ float2 ld2s(const __half *p, int64_t o) {
  return __half22float2(*reinterpret_cast<const __half2 *>(p + o));
}
__device__ __forceinline__ float2 ld2s(const __nv_bfloat16 *p, int64_t o) {
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(p + o));
}
__device__ __forceinline__ void st2s(float *p, int64_t o, float2 v) {
  *reinterpret_cast<float2 *>(p + o) = v;
}
__device__ __forceinline__ void st2s(__half *p, int64_t o, float2 v) {
  *reinterpret_cast<__half2 *>(p + o) = __floats2half2_rn(v.x, v.y);
}
__device__ __forceinline__ void st2s(__nv_bfloat16 *p, int64_t o, float2 v) {
  *reinterpret_cast<__nv_bfloat162 *>(p + o) = __floats2bfloat162_rn(v.x, v.y);
}
__device__ __forceinline__ float ld1s(const float *p, int64_t o) { return p[o]; }
__device__ __forceinline__ float ld1s(const __half *p, int64_t o) { return __half2float(p[o]); }
__device__ __forceinline__ float ld1s(const __nv_bfloat16 *p, int64_t o) {
  return __bfloat162float(p[o]);
}
// value as it reads back after a store through T
__device__ __forceinline__ float rt(float v, const float *) { return v; }
__device__ __forceinline__ float rt(float v, const __half *) {
  return __half2float(__float2half_rn(v));
}
__device__ __forceinline__ float rt(float v, const __nv_bfloat16 *) {
  return __bfloat162float(__float2bfloat16_rn(v));
}

__device__ __forceinline__ float q4(const float4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}
// OMEGA / (6 - n_solid) for byte q of a mask word: the damped-Jacobi weight of
// the smoother.  The preconditioner needs no bit-exactness, so the quotient is
// the two-instruction approximate division; a cell with no non-solid
// neighbour (diagonal 0) gets weight 0.  Values on non-fluid cells are masked
// off by the callers.
__device__ __forceinline__ float wcalc(uint32_t ns) {
  const float d = 6.0f - (float)ns;
  return d > 0.0f ? __fdividef(FOMEGA, d) : 0.0f;
}
// The 8 possible weights, filled once per CTA by fine_col_kernel: a lookup is
// one bit-field extract and one shared load.
__shared__ float s_wtab[8];
__device__ __forceinline__ float wdinv_ns(uint32_t ns) { return s_wtab[ns & 7u]; }
__device__ __forceinline__ float wdq(uint32_t mw, int q) { return s_wtab[(mw >> (8 * q)) & 7u]; }
__device__ __forceinline__ uint32_t mload4(const uint8_t *m, int64_t o) {
  return __ldg(reinterpret_cast<const uint32_t *>(m + o));
}

__device__ __forceinline__ void block_partial(double v, double *partials, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += sh[w];
    partials[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = t;
  }
}

// ---- operations -------------------------------------------------------------------------
// Interface: init(st), val4(i,j,k,o,mw), val1(i,j,k,o,mbyte), emit(...), finish(sh).

// ps = z + beta ps_prev (ps = z on the first iteration); Ap = 6 ps - s; partial ps.Ap
template <class T>
struct PsApOp {
  static constexpr bool SYNC = false;
  const uint8_t *mask;
  const T *z, *prev;
  T *cur, *Ap;
  double *partials;
  float beta;
  bool first;
  double acc;

  __device__ void init(const SolverState *st) {
    first = st->inner_it == 0;
    beta = (float)st->beta;
    acc = 0.0;
  }
  __device__ float4 val4(int, int, int, int64_t o, uint32_t) const {
    const float4 zz = ld4s(z, o);
    if (first) return zz;
    const float4 pp = ld4s(prev, o);
    return make_float4(rt(fmaf(beta, pp.x, zz.x), cur), rt(fmaf(beta, pp.y, zz.y), cur),
                       rt(fmaf(beta, pp.z, zz.z), cur), rt(fmaf(beta, pp.w, zz.w), cur));
  }
  __device__ float val1(int, int, int, int64_t o, uint32_t) const {
    const float zz = ld1s(z, o);
    return first ? zz : rt(fmaf(beta, ld1s(prev, o), zz), cur);
  }
  __device__ void emit(int, int, int, int64_t o, bool act, uint32_t mc, const float4 &v,
                       const float (&s)[4], float2 *) {
    if (!act) return;
    float ap[4], vv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t fm = fluid_word(mc, q);
      vv[q] = __uint_as_float(__float_as_uint(q4(v, q)) & fm);
      ap[q] = rt(__uint_as_float(__float_as_uint(fmaf(6.0f, q4(v, q), -s[q])) & fm), cur);
      acc += (double)vv[q] * (double)ap[q];
    }
    st4s(cur, o, make_float4(vv[0], vv[1], vv[2], vv[3]));
    st4s(Ap, o, make_float4(ap[0], ap[1], ap[2], ap[3]));
  }
  __device__ void finish(double *sh) { block_partial(acc, partials, sh); }
};

// e^ = OMEGA r / D + e1[parent];  z = e^ + OMEGA (r - (6 e^ - s)) / D;  partial r.z
template <class T>
struct UpOp {
  static constexpr bool SYNC = false;
  const uint8_t *mask;
  const T *r, *e1;
  T *z;
  double *partials;
  int ny1, nz1;
  double acc;

  __device__ void init(const SolverState *) { acc = 0.0; }
  __device__ float4 val4(int i, int j, int k, int64_t o, uint32_t mw) const {
    const float4 rr = ld4s(r, o);
    const int64_t P = ((int64_t)(i >> 1) * ny1 + (j >> 1)) * nz1 + (k >> 1);
    const float2 ec = ld2s(e1, P);
    // the coarse correction is not zero on non-fluid fine cells: mask it
    auto fl = [&](float v, int q) {
      return __uint_as_float(__float_as_uint(v) & fluid_word(mw, q));
    };
    return make_float4(fl(fmaf(rr.x, wdq(mw, 0), ec.x), 0), fl(fmaf(rr.y, wdq(mw, 1), ec.x), 1),
                       fl(fmaf(rr.z, wdq(mw, 2), ec.y), 2), fl(fmaf(rr.w, wdq(mw, 3), ec.y), 3));
  }
  __device__ float val1(int i, int j, int k, int64_t o, uint32_t mb) const {
    const int64_t P = ((int64_t)(i >> 1) * ny1 + (j >> 1)) * nz1 + (k >> 1);
    return (mb & BSP_MFLUID) ? fmaf(ld1s(r, o), wdinv_ns(mb & 7u), ld1s(e1, P)) : 0.0f;
  }
  __device__ void emit(int, int, int, int64_t o, bool act, uint32_t mc, const float4 &v,
                       const float (&s)[4], float2 *) {
    if (!act) return;
    const float4 rr = ld4s(r, o);
    float zz[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float e = q4(v, q);
      const float zq = fmaf(q4(rr, q) - (6.0f * e - s[q]), wdq(mc, q), e);
      zz[q] = rt(__uint_as_float(__float_as_uint(zq) & fluid_word(mc, q)), z);
      acc += (double)q4(rr, q) * (double)zz[q];
    }
    st4s(z, o, make_float4(zz[0], zz[1], zz[2], zz[3]));
  }
  __device__ void finish(double *sh) { block_partial(acc, partials, sh); }
};

// e = OMEGA r / D (pre-smoothing from zero); the residual r - (6 e - s) of the
// 2x2x2 children of each coarse cell is summed, halved, into r1 (0 on coarse
// cells that are not fluid).  Rows j (even) and j+1 meet in shared memory.
template <class T>
struct DownOp {
  static constexpr bool SYNC = true;
  const uint8_t *mask, *mask1;
  const T *r;
  T *r1;
  int nx, ny, ny1, nz1;
  float2 acc;

  __device__ void init(const SolverState *) { acc = make_float2(0.f, 0.f); }
  __device__ float4 val4(int, int, int, int64_t o, uint32_t mw) const {
    const float4 rr = ld4s(r, o);
    return make_float4(rr.x * wdq(mw, 0), rr.y * wdq(mw, 1), rr.z * wdq(mw, 2),
                       rr.w * wdq(mw, 3));
  }
  __device__ float val1(int, int, int, int64_t o, uint32_t mb) const {
    return ld1s(r, o) * wdinv_ns(mb & 7u);
  }
  // Every warp of the CTA calls this for every plane (it may __syncthreads).
  __device__ void emit(int i, int j, int k, int64_t o, bool act, uint32_t mc, const float4 &v,
                       const float (&s)[4], float2 *xch) {
    if (act) {
      const float4 rr = ld4s(r, o);
      float res[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float rq = q4(rr, q) - (6.0f * q4(v, q) - s[q]);
        res[q] = __uint_as_float(__float_as_uint(rq) & fluid_word(mc, q));
      }
      acc.x += res[0] + res[1];
      acc.y += res[2] + res[3];
    }
    if (!((i & 1) || i + 1 == nx)) return;  // uniform over the CTA
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp & 1) xch[(warp >> 1) * 32 + lane] = acc;
    __syncthreads();
    if (!(warp & 1) && act) {
      float2 t = acc;
      if (j + 1 < ny) {
        const float2 o2 = xch[(warp >> 1) * 32 + lane];
        t.x += o2.x;
        t.y += o2.y;
      }
      const int64_t C = ((int64_t)(i >> 1) * ny1 + (j >> 1)) * nz1 + (k >> 1);
      const uint32_t m2 = __ldg(reinterpret_cast<const uint16_t *>(mask1 + C));
      st2s(r1, C, make_float2((m2 & BSP_MFLUID) ? 0.5f * t.x : 0.0f,
                              ((m2 >> 8) & BSP_MFLUID) ? 0.5f * t.y : 0.0f));
    }
    __syncthreads();
    acc = make_float2(0.f, 0.f);
  }
  __device__ void finish(double *) {}
};

// ---- generic driver -------------------------------------------------------------------
template <class Op>
__global__ void __launch_bounds__(256) fine_col_kernel(Op op, int nx, int ny, int nz, int bi,
                                                       const SolverState *st) {
  if (st->inner_done) return;  // uniform: the whole grid returns
  __shared__ double sh[8];
  __shared__ float2 xch[4 * 32];
  if (threadIdx.x < 8) s_wtab[threadIdx.x] = wcalc(threadIdx.x);
  __syncthreads();
  op.init(st);
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
  const int k = (blockIdx.x * 32 + lane) * 4;
  const bool act = j < ny && k < nz;
  const int i0 = blockIdx.z * bi;
  const int i1 = min(i0 + bi, nx);
  const int64_t plane = (int64_t)ny * nz;
  const bool has_jm = j > 0, has_jp = j + 1 < ny;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const uint8_t *mask = op.mask;
  int64_t o = act ? (int64_t)i0 * plane + (int64_t)j * nz + k : 0;
  float4 vm = z4, vc = z4;
  uint32_t mm = 0u, mc = 0u;
  if (act && i0 > 0) {
    mm = mload4(mask, o - plane);
    vm = op.val4(i0 - 1, j, k, o - plane, mm);
  }
  if (act) {
    mc = mload4(mask, o);
    vc = op.val4(i0, j, k, o, mc);
  }
  for (int i = i0; i < i1; ++i) {
    float4 vn = z4, vjm = z4, vjp = z4;
    uint32_t mn = 0u, mjm = 0u, mjp = 0u;
    if (act) {
      if (i + 1 < nx) {
        mn = mload4(mask, o + plane);
        vn = op.val4(i + 1, j, k, o + plane, mn);
      }
      if (has_jm) {
        mjm = mload4(mask, o - nz);
        vjm = op.val4(i, j - 1, k, o - nz, mjm);
      }
      if (has_jp) {
        mjp = mload4(mask, o + nz);
        vjp = op.val4(i, j + 1, k, o + nz, mjp);
      }
    }
    float vkm = __shfl_up_sync(0xffffffffu, vc.w, 1);
    uint32_t mkm = __shfl_up_sync(0xffffffffu, mc, 1);
    float vkp = __shfl_down_sync(0xffffffffu, vc.x, 1);
    uint32_t mkp = __shfl_down_sync(0xffffffffu, mc, 1);
    if (lane == 0) {
      vkm = 0.0f;
      mkm = 0u;
      if (act && k > 0) {
        const uint32_t mbyte = __ldg(mask + o - 1);
        mkm = mbyte << 24;
        vkm = op.val1(i, j, k - 1, o - 1, mbyte);
      }
    }
    if (lane == 31) {
      vkp = 0.0f;
      mkp = 0u;
      if (act && k + 4 < nz) {
        const uint32_t mbyte = __ldg(mask + o + 4);
        mkp = mbyte;
        vkp = op.val1(i, j, k + 4, o + 4, mbyte);
      }
    }
    // Every operand is exactly 0 on non-fluid cells and outside the grid, so the
    // boundary rule (fluid -> operand, air -> 0, solid -> centre operand) is
    // the plain sum of the six neighbours plus n_solid(centre) x centre.
    (void)mkm;
    (void)mkp;
    const float4 vb = make_float4(vkm, vc.x, vc.y, vc.z);
    const float4 vf = make_float4(vc.y, vc.z, vc.w, vkp);
    float s[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float ns = (float)((mc >> (8 * q)) & 7u);
      s[q] = fmaf(ns, q4(vc, q),
                  ((q4(vm, q) + q4(vn, q)) + (q4(vjm, q) + q4(vjp, q))) + (q4(vb, q) + q4(vf, q)));
    }
    op.emit(i, j, k, o, act, mc, vc, s, xch);
    vm = vc;
    mm = mc;
    vc = vn;
    mc = mn;
    if (act) o += plane;
  }
  op.finish(sh);
}

// ---- FP64 residual on the column layout --------------------------------------------------
// r = bscale div - (6 x - s) on fluid cells (0 elsewhere) with the FP64 iterate
// x, which is exactly 0 on non-fluid cells, so s = sum of the six neighbours +
// n_solid x_centre.  Partials: ||r||^2 (slot 0) and max|r| (slot 1).  WRITE:
// rhat = scale r (storage T) and e = 0 on every cell.
struct D4 {
  double a, b, c, d;
};
__device__ __forceinline__ D4 ld4d(const double *p, int64_t o) {
  const double2 u = *reinterpret_cast<const double2 *>(p + o);
  const double2 v = *reinterpret_cast<const double2 *>(p + o + 2);
  return D4{u.x, u.y, v.x, v.y};
}
__device__ __forceinline__ double dq(const D4 &v, int q) {
  return q == 0 ? v.a : (q == 1 ? v.b : (q == 2 ? v.c : v.d));
}

template <class T, bool WRITE>
__global__ void __launch_bounds__(256) resid64_col_kernel(int nx, int ny, int nz, int bi,
                                                          const uint8_t *mask, const float *div,
                                                          const double *x, double bscale, T *rhat,
                                                          float *e, double *partials,
                                                          const SolverState *st) {
  if (st->done) return;
  const double scale = st->scale;
  __shared__ double shs[8], shm[8];
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
  const int k = (blockIdx.x * 32 + lane) * 4;
  const bool act = j < ny && k < nz;
  const int i0 = blockIdx.z * bi;
  const int i1 = min(i0 + bi, nx);
  const int64_t plane = (int64_t)ny * nz;
  const D4 z4{0, 0, 0, 0};
  int64_t o = act ? (int64_t)i0 * plane + (int64_t)j * nz + k : 0;
  D4 xm = z4, xc = z4;
  if (act && i0 > 0) xm = ld4d(x, o - plane);
  if (act) xc = ld4d(x, o);
  double rr = 0.0, rmax = 0.0;
  for (int i = i0; i < i1; ++i) {
    D4 xn = z4, xjm = z4, xjp = z4;
    if (act) {
      if (i + 1 < nx) xn = ld4d(x, o + plane);
      if (j > 0) xjm = ld4d(x, o - nz);
      if (j + 1 < ny) xjp = ld4d(x, o + nz);
    }
    double xkm = __shfl_up_sync(0xffffffffu, xc.d, 1);
    double xkp = __shfl_down_sync(0xffffffffu, xc.a, 1);
    if (lane == 0) xkm = (act && k > 0) ? x[o - 1] : 0.0;
    if (lane == 31) xkp = (act && k + 4 < nz) ? x[o + 4] : 0.0;
    if (act) {
      const uint32_t mc = __ldg(reinterpret_cast<const uint32_t *>(mask + o));
      const float4 dv = *reinterpret_cast<const float4 *>(div + o);
      const D4 xb{xkm, xc.a, xc.b, xc.c}, xf{xc.b, xc.c, xc.d, xkp};
      float rq[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint32_t mb = (mc >> (8 * q)) & 0xffu;
        double r = 0.0;
        if (mb & BSP_MFLUID) {
          const double c = dq(xc, q);
          const double s = ((dq(xm, q) + dq(xn, q)) + (dq(xjm, q) + dq(xjp, q))) +
                           (dq(xb, q) + dq(xf, q)) + (double)(mb & 7u) * c;
          r = bscale * (double)q4(dv, q) - (6.0 * c - s);
        }
        rr += r * r;
        rmax = fmax(rmax, fabs(r));
        rq[q] = (float)(r * scale);
      }
      if (WRITE) {
        st4s(rhat, o, make_float4(rq[0], rq[1], rq[2], rq[3]));
        *reinterpret_cast<float4 *>(e + o) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    xm = xc;
    xc = xn;
    if (act) o += plane;
  }
  for (int off = 16; off > 0; off >>= 1) {
    rr += __shfl_xor_sync(0xffffffffu, rr, off);
    rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, off));
  }
  if (lane == 0) {
    shs[threadIdx.x >> 5] = rr;
    shm[threadIdx.x >> 5] = rmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, m = 0.0;
    for (int w = 0; w < 8; ++w) {
      a += shs[w];
      m = fmax(m, shm[w]);
    }
    const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    partials[b] = a;
    partials[PARTIAL_STRIDE + b] = m;
  }
}

// ---- launchers --------------------------------------------------------------------------
int num_sms();

// Planes per CTA: the largest even value <= 16 that still gives about two
// CTAs per SM (coarse levels are short; long plane chunks there leave the
// GPU idle).  Even, because the restriction pairs planes inside one CTA.
int fine_bi(int nx, int ny, int nz) {
  const int64_t cols = (int64_t)((nz / 4 + 31) / 32) * ((ny + 7) / 8);
  const int64_t target = 2LL * num_sms();
  int bi = 16;
  while (bi > 2 && cols * ((nx + bi - 1) / bi) < target) bi -= 2;
  return bi;
}

dim3 fine_grid(int nx, int ny, int nz) {
  const int bi = fine_bi(nx, ny, nz);
  return dim3((nz / 4 + 31) / 32, (ny + 7) / 8, (nx + bi - 1) / bi);
}
int fine_grid_blocks(int nx, int ny, int nz) {
  const dim3 g = fine_grid(nx, ny, nz);
  return (int)(g.x * g.y * g.z);
}

template <class T>
void launch_fine_psap(int nx, int ny, int nz, const uint8_t *mask, const T *z, const T *prev,
                      T *cur, T *Ap, double *partials, const SolverState *st, cudaStream_t s) {
  PsApOp<T> op{};
  op.mask = mask;
  op.z = z;
  op.prev = prev;
  op.cur = cur;
  op.Ap = Ap;
  op.partials = partials;
  fine_col_kernel<PsApOp<T>><<<fine_grid(nx, ny, nz), 256, 0, s>>>(op, nx, ny, nz,
                                                                   fine_bi(nx, ny, nz), st);
}

template <class T>
void launch_fine_up(const Level<T> &f, const Level<T> &c, T *z, double *partials,
                    const SolverState *st, cudaStream_t s) {
  UpOp<T> op{};
  op.mask = f.mask;
  op.r = f.r;
  op.e1 = c.e;
  op.z = z;
  op.partials = partials;
  op.ny1 = c.ny;
  op.nz1 = c.nz;
  fine_col_kernel<UpOp<T>><<<fine_grid(f.nx, f.ny, f.nz), 256, 0, s>>>(
      op, f.nx, f.ny, f.nz, fine_bi(f.nx, f.ny, f.nz), st);
}

template <class T>
void launch_fine_down(const Level<T> &f, const Level<T> &c, const SolverState *st,
                      cudaStream_t s) {
  DownOp<T> op{};
  op.mask = f.mask;
  op.mask1 = c.mask;
  op.r = f.r;
  op.r1 = c.r;
  op.nx = f.nx;
  op.ny = f.ny;
  op.ny1 = c.ny;
  op.nz1 = c.nz;
  fine_col_kernel<DownOp<T>><<<fine_grid(f.nx, f.ny, f.nz), 256, 0, s>>>(
      op, f.nx, f.ny, f.nz, fine_bi(f.nx, f.ny, f.nz), st);
}

template <class T>
int launch_resid64_col(int nx, int ny, int nz, const uint8_t *mask, const float *div,
                       const double *x, double bscale, T *rhat, float *e, double *partials,
                       const SolverState *st, bool write, cudaStream_t s) {
  const dim3 g = fine_grid(nx, ny, nz);
  const int bi = fine_bi(nx, ny, nz);
  if (write)
    resid64_col_kernel<T, true><<<g, 256, 0, s>>>(nx, ny, nz, bi, mask, div, x, bscale, rhat, e,
                                                  partials, st);
  else
    resid64_col_kernel<T, false><<<g, 256, 0, s>>>(nx, ny, nz, bi, mask, div, x, bscale, rhat,
                                                   e, partials, st);
  return (int)(g.x * g.y * g.z);
}

#define INST(T)                                                                              \
  template int launch_resid64_col<T>(int, int, int, const uint8_t *, const float *,          \
                                     const double *, double, T *, float *, double *,         \
                                     const SolverState *, bool, cudaStream_t);               \
  template void launch_fine_psap<T>(int, int, int, const uint8_t *, const T *, const T *, T *, \
                                    T *, double *, const SolverState *, cudaStream_t);         \
  template void launch_fine_up<T>(const Level<T> &, const Level<T> &, T *, double *,          \
                                  const SolverState *, cudaStream_t);                         \
  template void launch_fine_down<T>(const Level<T> &, const Level<T> &, const SolverState *,  \
                                    cudaStream_t);
INST(float)
INST(__half)
INST(__nv_bfloat16)
#undef INST

}  // namespace bsp
