// mgfine.cu -- fine-level (level 0) kernels of the to-tolerance solver on the
// column layout of the sweep kernel.
//
// One generic driver, fine_tile_kernel<Op>: a CTA is 8 output warps plus two
// halo warps; output warp w owns fine row j = 8*blockIdx.y + w and 128
// consecutive k cells (4 per lane) and marches i over an even-length chunk.
// The Op supplies the stencil operand of a cell (ps for A*ps; OMEGA r / D for
// the smoothers, plus the coarse correction for the prolongation) and
// consumes, per cell, the centre operand and the neighbour sum
// s = l + r + d + u + b + f under the boundary rule (fluid -> operand, air ->
// 0, solid -> centre operand).  Each operand is computed once per plane by the
// warp owning its row (the halo warps own rows j0-1 and j0+8) and shared
// through a double-buffered plane in shared memory for the j +- 1 neighbours;
// planes i-1, i, i+1 stay in registers; k +- 1 arrive by warp shuffles.
//
// Requirements (checked by the caller; otherwise the row kernels of solver.cu
// run): nz % 4 == 0 and 16-byte aligned level-0 fields.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <mutex>
#include <type_traits>
#include <utility>

#include "bsp_common.cuh"
#include "solver.cuh"
#include "tma.cuh"

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
__device__ __forceinline__ void st1s(float *p, int64_t o, float v) { p[o] = v; }
__device__ __forceinline__ void st1s(__half *p, int64_t o, float v) { p[o] = __float2half_rn(v); }
__device__ __forceinline__ void st1s(__nv_bfloat16 *p, int64_t o, float v) {
  p[o] = __float2bfloat16_rn(v);
}
// value as it reads back after a store through T
__device__ __forceinline__ float rt(float v, const float *) { return v; }
__device__ __forceinline__ float rt(float v, const __half *) {
  return __half2float(__float2half_rn(v));
}
__device__ __forceinline__ float rt(float v, const __nv_bfloat16 *) {
  return __bfloat162float(__float2bfloat16_rn(v));
}

// Round four values to storage T once: the packed words to store (s4p) and
// the values as they read back (rt of each).  One pack per pair and the
// unpack, instead of a round trip per value and a second pack at the store.
template <class T>
struct Pk4;
template <>
struct Pk4<float> {
  float4 w;
};
template <>
struct Pk4<__half> {
  uint2 w;
};
template <>
struct Pk4<__nv_bfloat16> {
  uint2 w;
};
__device__ __forceinline__ Pk4<float> pk4(float4 v, float4 &back, const float *) {
  back = v;
  return Pk4<float>{v};
}
__device__ __forceinline__ Pk4<__half> pk4(float4 v, float4 &back, const __half *) {
  const __half2 a = __floats2half2_rn(v.x, v.y), b = __floats2half2_rn(v.z, v.w);
  const float2 fa = __half22float2(a), fb = __half22float2(b);
  back = make_float4(fa.x, fa.y, fb.x, fb.y);
  return Pk4<__half>{make_uint2(*reinterpret_cast<const uint32_t *>(&a),
                                *reinterpret_cast<const uint32_t *>(&b))};
}
__device__ __forceinline__ Pk4<__nv_bfloat16> pk4(float4 v, float4 &back,
                                                  const __nv_bfloat16 *) {
  const __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
  const float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
  back = make_float4(fa.x, fa.y, fb.x, fb.y);
  return Pk4<__nv_bfloat16>{make_uint2(*reinterpret_cast<const uint32_t *>(&a),
                                       *reinterpret_cast<const uint32_t *>(&b))};
}
__device__ __forceinline__ void s4p(float *p, int64_t o, const Pk4<float> &v) {
  *reinterpret_cast<float4 *>(p + o) = v.w;
}
template <class H>
__device__ __forceinline__ void s4p(H *p, int64_t o, const Pk4<H> &v) {
  *reinterpret_cast<uint2 *>(p + o) = v.w;
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
// The 8 possible weights, filled once per CTA by fine_tile_kernel: a lookup is
// one bit-field extract and one shared load.
__shared__ float s_wtab[8];
__device__ __forceinline__ float wdinv_ns(uint32_t ns) { return s_wtab[ns & 7u]; }
__device__ __forceinline__ float wdq(uint32_t mw, int q) { return s_wtab[(mw >> (8 * q)) & 7u]; }
// The same weight indexed by mask bits 7 and 0-2 (the byte & 0x87): 0 on
// non-fluid cells.  Filled by fine_tma_kernel.
__shared__ float s_wtabf[0x88];
__device__ __forceinline__ float wdqf(uint32_t mw, int q) {
  return s_wtabf[(mw >> (8 * q)) & 0x87u];
}
// Ops with SUM6 = true take s as the plain sum of the six neighbour values
// (their smoothing step is written without the n_solid x centre term);
// the others s = that sum + n_solid x centre.
template <class Op, class = void>
struct op_sum6 : std::false_type {};
template <class Op>
struct op_sum6<Op, std::void_t<decltype(Op::SUM6)>> : std::integral_constant<bool, Op::SUM6> {};
constexpr float FOMEGA_C = 1.0f - 6.0f / 7.0f;  // 1 - OMEGA
__device__ __forceinline__ uint32_t mload4(const uint8_t *m, int64_t o) {
  return __ldg(reinterpret_cast<const uint32_t *>(m + o));
}

__device__ __forceinline__ int block_linear() {
  return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
}

template <int NW>
__device__ __forceinline__ void block_partial(double v, double *partials, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < NW; ++w) t += sh[w];
    partials[block_linear()] = t;
  }
}

// ---- operations -------------------------------------------------------------------------
// Interface: init(st); val4(i,j,k,o,mw) / val1(i,j,k,o,mbyte): the stencil
// operand of 4 cells / 1 cell (exactly 0 on non-fluid cells); emit(...) per
// output cell group; after_step(...) after the CTA barrier that ends plane i;
// finish<NW>(sh) once at the end (all threads of the CTA).

// Partial dot products: the four products of a thread's cells summed in FP32
// (one fixed FMA chain), widened once and added to the FP64 partial -- one
// conversion per four cells instead of two per cell.  The FP32 rounding of a
// four-term sum (a few 2^-24 of the sum of magnitudes) is far below the
// storage rounding of the vectors being dotted; the sums over threads, blocks
// and the grid stay FP64.
__device__ __forceinline__ double dot4w(const float (&a)[4], const float (&b)[4]) {
  return (double)fmaf(a[3], b[3], fmaf(a[2], b[2], fmaf(a[1], b[1], a[0] * b[0])));
}
__device__ __forceinline__ double dot4w(const float4 &a, const float (&b)[4]) {
  const float t[4] = {a.x, a.y, a.z, a.w};
  return dot4w(t, b);
}
__device__ __forceinline__ double sq4w(const float4 &a) {
  return (double)fmaf(a.w, a.w, fmaf(a.z, a.z, fmaf(a.y, a.y, a.x * a.x)));
}

// ps = z + beta ps_prev (ps = z on the first iteration); Ap = 6 ps - s; partial ps.Ap
template <class T>
struct PsApOp {
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
  __device__ void emit(int, int, int, int64_t o, uint32_t mc, const float4 &v,
                       const float (&s)[4], float2 *) {
    float ap[4], vv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t fm = fluid_word(mc, q);
      vv[q] = __uint_as_float(__float_as_uint(q4(v, q)) & fm);
      ap[q] = rt(__uint_as_float(__float_as_uint(fmaf(6.0f, q4(v, q), -s[q])) & fm), cur);
    }
    acc += dot4w(vv, ap);
    st4s(cur, o, make_float4(vv[0], vv[1], vv[2], vv[3]));
    st4s(Ap, o, make_float4(ap[0], ap[1], ap[2], ap[3]));
  }
  __device__ void after_step(int, int, int, bool, float2 *) {}
  template <int NW>
  __device__ void finish(double *sh) { block_partial<NW>(acc, partials, sh); }
  __device__ void skip() const { partials[block_linear()] = 0.0; }
};

// e^ = OMEGA r / D + alpha e1[parent];  z = e^ + OMEGA (r - (6 e^ - s)) / D;
// partial r.z
template <class T>
struct UpOp {
  static constexpr bool SUM6 = true;
  const uint8_t *mask;
  const T *r, *e1;
  T *z;
  double *partials;
  int ny1, nz1;
  float alpha;
  double acc;

  __device__ void init(const SolverState *) { acc = 0.0; }
  __device__ float4 val4(int i, int j, int k, int64_t o, uint32_t mw) const {
    const float4 rr = ld4s(r, o);
    const int64_t P = ((int64_t)(i >> 1) * ny1 + (j >> 1)) * nz1 + (k >> 1);
    float2 ec = ld2s(e1, P);
    ec.x *= alpha;
    ec.y *= alpha;
    // the coarse correction is not zero on non-fluid fine cells: mask it
    auto fl = [&](float v, int q) {
      return __uint_as_float(__float_as_uint(v) & fluid_word(mw, q));
    };
    return make_float4(fl(fmaf(rr.x, wdq(mw, 0), ec.x), 0), fl(fmaf(rr.y, wdq(mw, 1), ec.x), 1),
                       fl(fmaf(rr.z, wdq(mw, 2), ec.y), 2), fl(fmaf(rr.w, wdq(mw, 3), ec.y), 3));
  }
  __device__ float val1(int i, int j, int k, int64_t o, uint32_t mb) const {
    const int64_t P = ((int64_t)(i >> 1) * ny1 + (j >> 1)) * nz1 + (k >> 1);
    return (mb & BSP_MFLUID) ? fmaf(ld1s(r, o), wdinv_ns(mb & 7u), alpha * ld1s(e1, P)) : 0.0f;
  }
  __device__ void emit(int, int, int, int64_t o, uint32_t mc, const float4 &v,
                       const float (&s)[4], float2 *) {
    const float4 rr = ld4s(r, o);
    float zz[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      // z = e + w (r - A e) = (1 - OMEGA) e + w (r + sum6), w = OMEGA / D
      const float e = q4(v, q);
      const float w = wdq(mc, q);
      const float zq = w > 0.0f ? fmaf(w, q4(rr, q) + s[q], FOMEGA_C * e) : e;
      zz[q] = rt(__uint_as_float(__float_as_uint(zq) & fluid_word(mc, q)), z);
    }
    acc += dot4w(rr, zz);
    st4s(z, o, make_float4(zz[0], zz[1], zz[2], zz[3]));
  }
  __device__ void after_step(int, int, int, bool, float2 *) {}
  template <int NW>
  __device__ void finish(double *sh) { block_partial<NW>(acc, partials, sh); }
  __device__ void skip() const { partials[block_linear()] = 0.0; }
};

// e = OMEGA r / D (pre-smoothing from zero); the residual r - (6 e - s) of the
// 2x2x2 children of each coarse cell is summed, halved, into r1 (0 on coarse
// cells that are not fluid).  A pair of planes is summed in registers; rows j
// (even warp) and j+1 (odd warp) meet in shared memory across the barrier that
// ends the second plane of the pair.
template <class T>
struct DownOp {
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
  __device__ bool pair_end(int i) const { return (i & 1) || i + 1 == nx; }
  __device__ void emit(int i, int, int, int64_t o, uint32_t mc, const float4 &v,
                       const float (&s)[4], float2 *xch) {
    const float4 rr = ld4s(r, o);
    float res[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float rq = q4(rr, q) - (6.0f * q4(v, q) - s[q]);
      res[q] = __uint_as_float(__float_as_uint(rq) & fluid_word(mc, q));
    }
    acc.x += res[0] + res[1];
    acc.y += res[2] + res[3];
    const int warp = threadIdx.x >> 5;
    if (pair_end(i) && (warp & 1)) {
      xch[(warp >> 1) * 32 + (threadIdx.x & 31)] = acc;
      acc = make_float2(0.f, 0.f);
    }
  }
  // Called by the output warps (active or not) after the barrier ending plane i.
  __device__ void after_step(int i, int j, int k, bool act, float2 *xch) {
    const int warp = threadIdx.x >> 5;
    if (!pair_end(i) || (warp & 1)) return;
    if (act) {
      float2 t = acc;
      if (j + 1 < ny) {
        const float2 o2 = xch[(warp >> 1) * 32 + (threadIdx.x & 31)];
        t.x += o2.x;
        t.y += o2.y;
      }
      const int64_t C = ((int64_t)(i >> 1) * ny1 + (j >> 1)) * nz1 + (k >> 1);
      const uint32_t m2 = __ldg(reinterpret_cast<const uint16_t *>(mask1 + C));
      st2s(r1, C, make_float2((m2 & BSP_MFLUID) ? 0.5f * t.x : 0.0f,
                              ((m2 >> 8) & BSP_MFLUID) ? 0.5f * t.y : 0.0f));
    }
    acc = make_float2(0.f, 0.f);
  }
  template <int NW>
  __device__ void finish(double *) {}
  __device__ void skip() const {}
};

// ---- tile driver ------------------------------------------------------------------------
// A CTA owns ROWS consecutive j rows (output warps 0..ROWS-1, one row each, 128
// k cells: float4 per lane) plus two halo warps for rows j0-1 and j0+ROWS, and
// marches i over an even chunk [i0, i1).  Every operand value is computed once
// per plane by the warp that owns its row and published in a double-buffered
// shared-memory plane; rows j +- 1 are read back from there, planes i +- 1 stay
// in registers, k +- 1 arrive by shuffles (lanes 0 and 31 fetch the row's k
// halo together, in one branch).  One CTA barrier per plane.
constexpr int TILE_ROWS = 8;
constexpr int TILE_WARPS = TILE_ROWS + 2;
constexpr int TILE_THREADS = TILE_WARPS * 32;

template <class Op>
__global__ void __launch_bounds__(TILE_THREADS, 4) fine_tile_kernel(Op op, int nx, int ny, int nz,
                                                                 int bi, const uint8_t *tiles,
                                                                 const SolverState *st) {
  if (st->inner_done) return;  // uniform: the whole grid returns
  if (tiles && !tiles[block_linear()]) {
    if (threadIdx.x == 0) op.skip();
    return;
  }
  __shared__ double sh[TILE_WARPS];
  __shared__ float2 xch[(TILE_ROWS / 2) * 32];
  __shared__ float4 plane_buf[2][TILE_ROWS + 2][32];
  if (threadIdx.x < 8) s_wtab[threadIdx.x] = wcalc(threadIdx.x);
  __syncthreads();
  op.init(st);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int j0 = blockIdx.y * TILE_ROWS;
  // row slot in plane_buf: 0 = j0-1, 1..ROWS = output rows, ROWS+1 = j0+ROWS
  const int slot = warp < TILE_ROWS ? warp + 1 : (warp == TILE_ROWS ? 0 : TILE_ROWS + 1);
  const int j = j0 + slot - 1;
  const int k = (blockIdx.x * 32 + lane) * 4;
  const bool act = j >= 0 && j < ny && k < nz;
  const bool out = warp < TILE_ROWS;
  const int i0 = blockIdx.z * bi;
  const int i1 = min(i0 + bi, nx);
  const int64_t plane = (int64_t)ny * nz;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const uint8_t *mask = op.mask;
  int64_t o = act ? (int64_t)i0 * plane + (int64_t)j * nz + k : 0;
  float4 vm = z4, vc = z4;
  uint32_t mc = 0u;
  if (act) {
    mc = mload4(mask, o);
    vc = op.val4(i0, j, k, o, mc);
    if (out && i0 > 0) vm = op.val4(i0 - 1, j, k, o - plane, mload4(mask, o - plane));
  }
  plane_buf[i0 & 1][slot][lane] = vc;
  __syncthreads();
  for (int i = i0; i < i1; ++i) {
    float4 vn = z4;
    uint32_t mn = 0u;
    if (act && i + 1 < nx) {
      mn = mload4(mask, o + plane);
      vn = op.val4(i + 1, j, k, o + plane, mn);
    }
    plane_buf[(i + 1) & 1][slot][lane] = vn;
    if (out) {
      const float4 vjm = plane_buf[i & 1][slot - 1][lane];
      const float4 vjp = plane_buf[i & 1][slot + 1][lane];
      float vkm = __shfl_up_sync(0xffffffffu, vc.w, 1);
      float vkp = __shfl_down_sync(0xffffffffu, vc.x, 1);
      // k halo of the row: k0 - 1 for lane 0, k0 + 128 for lane 31
      const int kh = lane == 0 ? k - 1 : k + 4;
      float vh = 0.0f;
      if (act && (lane == 0 || lane == 31) && kh >= 0 && kh < nz) {
        const int64_t oh = o + (kh - k);
        vh = op.val1(i, j, kh, oh, __ldg(mask + oh));
      }
      if (lane == 0) vkm = vh;
      if (lane == 31) vkp = vh;
      // Every operand is exactly 0 on non-fluid cells and outside the grid, so
      // the boundary rule (fluid -> operand, air -> 0, solid -> centre operand)
      // is the plain sum of the six neighbours plus n_solid(centre) x centre.
      const float4 vb = make_float4(vkm, vc.x, vc.y, vc.z);
      const float4 vf = make_float4(vc.y, vc.z, vc.w, vkp);
      float s[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float sum6 = ((q4(vm, q) + q4(vn, q)) + (q4(vjm, q) + q4(vjp, q))) +
                           (q4(vb, q) + q4(vf, q));
        if constexpr (op_sum6<Op>::value) {
          s[q] = sum6;
        } else {
          const float ns = (float)((mc >> (8 * q)) & 7u);
          s[q] = fmaf(ns, q4(vc, q), sum6);
        }
      }
      if (act) op.emit(i, j, k, o, mc, vc, s, xch);
    }
    __syncthreads();
    if (out) op.after_step(i, j, k, act, xch);
    vm = vc;
    vc = vn;
    mc = mn;
    if (act) o += plane;
  }
  op.template finish<TILE_WARPS>(sh);
}

// ---- TMA-fed tile driver ----------------------------------------------------------------
// Same CTA shape and arithmetic as fine_tile_kernel, but the raw inputs of a
// plane (fine operand sources, the mask, the coarse correction) arrive as TMA
// tiles in a ring of STAGES shared-memory stages, issued STAGES-1 planes ahead
// by one thread: the bytes in flight no longer depend on how many warps wait.
// A tile covers rows j0-1 .. j0+8 and k0-PAD .. k0+127+PAD, so the j and k
// halos (and every cell outside the grid, zero-filled by the TMA unit) come
// with it; no global load is left on the plane loop but the stores.
//
// Stage layout (bytes): fine tensors A[, B] of T: 10 rows x (128 + 2 PAD)
// elements, PAD = 16 / sizeof(T); mask: 10 rows x 160 bytes (PAD 16); coarse
// tensor C of T: 6 rows x (64 + 2 PAD) elements.  All row strides are
// multiples of 16 bytes.
int fine_bi(int nx, int ny, int nz);
dim3 fine_grid(int nx, int ny, int nz);

constexpr int TMA_ROWS = TILE_ROWS + 2;
constexpr int MASK_W = 160;
constexpr int MASK_PAD = 16;

template <class T>
struct TmaGeom {
  static constexpr int PAD = 16 / (int)sizeof(T);
  static constexpr int FW = 128 + 2 * PAD;        // fine row width (elements)
  static constexpr int CW = 64 + 2 * PAD;         // coarse row width (elements)
  static constexpr int CROWS = TILE_ROWS / 2 + 2;  // coarse rows j0/2-1 .. j0/2+4
  static constexpr int FBYTES = TMA_ROWS * FW * (int)sizeof(T);
  static constexpr int MBYTES = TMA_ROWS * MASK_W;
  static constexpr int CBYTES = CROWS * CW * (int)sizeof(T);
};

// Tensor maps of one launch.  a, b: fine tensors of T; m: mask; c: coarse T.
struct TmaMaps {
  CUtensorMap a, b, m, c, e, p, q;  // q: fine uint8 parent-pattern tiles (trilinear transfers)
};

// Operand sources read from a stage.  rr: tile row 0..9 (j = j0 - 1 + rr);
// kl: k - k0 (-1 .. 128).
template <class T>
struct StageView {
  const T *a, *b, *c;
  const T *c2;        // the second coarse plane (trilinear prolongation)
  const uint8_t *q;   // fine parent-pattern tile (trilinear transfers)
  int plane;          // fine plane of this stage
  const uint8_t *m;
  const float *e;  // EP tiles: 8 output rows x 128 (no halo)
  const T *ps;
  __device__ uint32_t mask4(int rr, int lane) const {
    return *reinterpret_cast<const uint32_t *>(m + rr * MASK_W + MASK_PAD + lane * 4);
  }
  __device__ uint32_t mask1(int rr, int kl) const { return m[rr * MASK_W + MASK_PAD + kl]; }
  __device__ int fo(int rr, int kl) const { return rr * TmaGeom<T>::FW + TmaGeom<T>::PAD + kl; }
  // coarse parent of fine (row rr, kl): coarse row (j >> 1) - (j0/2 - 1) = (rr + 1) >> 1
  __device__ int co(int rr, int kl) const {
    return ((rr + 1) >> 1) * TmaGeom<T>::CW + TmaGeom<T>::PAD + (kl >> 1);
  }
};

template <class T>
struct TPsAp {
  static constexpr bool HAS_B = true, HAS_C = false, HAS_EP = false;
  static constexpr int STAGES = 4, MIN_BLOCKS = 3;
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
  __device__ float4 val4(const StageView<T> &v, int rr, int lane, uint32_t) const {
    const float4 zz = ld4s(v.a, v.fo(rr, lane * 4));
    if (first) return zz;
    const float4 pp = ld4s(v.b, v.fo(rr, lane * 4));
    return make_float4(rt(fmaf(beta, pp.x, zz.x), cur), rt(fmaf(beta, pp.y, zz.y), cur),
                       rt(fmaf(beta, pp.z, zz.z), cur), rt(fmaf(beta, pp.w, zz.w), cur));
  }
  __device__ float val1(const StageView<T> &v, int rr, int kl) const {
    const float zz = ld1s(v.a, v.fo(rr, kl));
    return first ? zz : rt(fmaf(beta, ld1s(v.b, v.fo(rr, kl)), zz), cur);
  }
  __device__ void emit(const StageView<T> &, int, int, int, int, int64_t o, uint32_t mc,
                       const float4 &v, const float (&s)[4], float2 *) {
    float ap[4], vv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t fm = fluid_word(mc, q);
      vv[q] = __uint_as_float(__float_as_uint(q4(v, q)) & fm);
      ap[q] = rt(__uint_as_float(__float_as_uint(fmaf(6.0f, q4(v, q), -s[q])) & fm), cur);
    }
    acc += dot4w(vv, ap);
    st4s(cur, o, make_float4(vv[0], vv[1], vv[2], vv[3]));
    st4s(Ap, o, make_float4(ap[0], ap[1], ap[2], ap[3]));
  }
  __device__ void after_step(int, int, int, bool, float2 *) {}
  template <int NW>
  __device__ void finish(double *sh) { block_partial<NW>(acc, partials, sh); }
  __device__ void skip() const { partials[block_linear()] = 0.0; }
};

template <class T>
struct TUp {
  static constexpr bool HAS_B = false, HAS_C = true, HAS_EP = false, SUM6 = true;
  static constexpr int STAGES = 4, MIN_BLOCKS = 4;
  T *z;
  double *partials;
  float alpha;
  double acc;
  // smoothing weights (0 on non-fluid cells) of the plane val4 saw last and
  // of the one before it, which emit of that plane uses
  float wn[4], wc[4];
  __device__ void init(const SolverState *) { acc = 0.0; }
  __device__ void shift_w(uint32_t mw) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      wc[q] = wn[q];
      wn[q] = wdqf(mw, q);
    }
  }
  __device__ float4 val4(const StageView<T> &v, int rr, int lane, uint32_t mw) {
    shift_w(mw);
    const float4 r4 = ld4s(v.a, v.fo(rr, lane * 4));
    float2 ec = ld2s(v.c, v.co(rr, lane * 4));
    ec.x *= alpha;
    ec.y *= alpha;
    auto fl = [&](float x, int q) {
      return __uint_as_float(__float_as_uint(x) & fluid_word(mw, q));
    };
    return make_float4(fl(fmaf(r4.x, wn[0], ec.x), 0), fl(fmaf(r4.y, wn[1], ec.x), 1),
                       fl(fmaf(r4.z, wn[2], ec.y), 2), fl(fmaf(r4.w, wn[3], ec.y), 3));
  }
  __device__ float val1(const StageView<T> &v, int rr, int kl) const {
    const uint32_t mb = v.mask1(rr, kl);
    return (mb & BSP_MFLUID)
               ? fmaf(ld1s(v.a, v.fo(rr, kl)), wdinv_ns(mb & 7u), alpha * ld1s(v.c, v.co(rr, kl)))
               : 0.0f;
  }
  __device__ void emit(const StageView<T> &v, int rr, int lane, int, int, int64_t o,
                       uint32_t, const float4 &e4, const float (&s)[4], float2 *) {
    const float4 r4 = ld4s(v.a, v.fo(rr, lane * 4));
    float zz[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      // z = e + w (r - A e) = (1 - OMEGA) e + w (r + sum6), w = OMEGA / D;
      // w = 0 on non-fluid cells, where e is 0
      const float e = q4(e4, q);
      const float w = wc[q];
      zz[q] = w > 0.0f ? fmaf(w, q4(r4, q) + s[q], FOMEGA_C * e) : e;
    }
    float4 zb;
    const Pk4<T> zp = pk4(make_float4(zz[0], zz[1], zz[2], zz[3]), zb, z);
    const float zr[4] = {zb.x, zb.y, zb.z, zb.w};
    acc += dot4w(r4, zr);
    s4p(z, o, zp);
  }
  __device__ void after_step(int, int, int, bool, float2 *) {}
  template <int NW>
  __device__ void finish(double *sh) { block_partial<NW>(acc, partials, sh); }
  __device__ void skip() const { partials[block_linear()] = 0.0; }
};

template <class T>
struct TDown {
  static constexpr bool HAS_B = false, HAS_C = false, HAS_EP = false;
  static constexpr int STAGES = 4, MIN_BLOCKS = 4;
  const uint8_t *mask1;
  T *r1;
  int nx, ny, ny1, nz1;
  float2 acc;
  __device__ void init(const SolverState *) { acc = make_float2(0.f, 0.f); }
  __device__ float4 val4(const StageView<T> &v, int rr, int lane, uint32_t mw) const {
    const float4 r4 = ld4s(v.a, v.fo(rr, lane * 4));
    return make_float4(r4.x * wdq(mw, 0), r4.y * wdq(mw, 1), r4.z * wdq(mw, 2),
                       r4.w * wdq(mw, 3));
  }
  __device__ float val1(const StageView<T> &v, int rr, int kl) const {
    return ld1s(v.a, v.fo(rr, kl)) * wdinv_ns(v.mask1(rr, kl) & 7u);
  }
  __device__ bool pair_end(int i) const { return (i & 1) || i + 1 == nx; }
  __device__ void emit(const StageView<T> &v, int rr, int lane, int i, int, int64_t,
                       uint32_t mc, const float4 &e4, const float (&s)[4], float2 *xch) {
    const float4 r4 = ld4s(v.a, v.fo(rr, lane * 4));
    float res[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float rq = q4(r4, q) - (6.0f * q4(e4, q) - s[q]);
      res[q] = __uint_as_float(__float_as_uint(rq) & fluid_word(mc, q));
    }
    acc.x += res[0] + res[1];
    acc.y += res[2] + res[3];
    const int warp = threadIdx.x >> 5;
    if (pair_end(i) && (warp & 1)) {
      xch[(warp >> 1) * 32 + lane] = acc;
      acc = make_float2(0.f, 0.f);
    }
  }
  __device__ void after_step(int i, int j, int k, bool act, float2 *xch) {
    const int warp = threadIdx.x >> 5;
    if (!pair_end(i) || (warp & 1)) return;
    if (act) {
      float2 t = acc;
      if (j + 1 < ny) {
        const float2 o2 = xch[(warp >> 1) * 32 + (threadIdx.x & 31)];
        t.x += o2.x;
        t.y += o2.y;
      }
      const int64_t C = ((int64_t)(i >> 1) * ny1 + (j >> 1)) * nz1 + (k >> 1);
      const uint32_t m2 = __ldg(reinterpret_cast<const uint16_t *>(mask1 + C));
      st2s(r1, C, make_float2((m2 & BSP_MFLUID) ? 0.5f * t.x : 0.0f,
                              ((m2 >> 8) & BSP_MFLUID) ? 0.5f * t.y : 0.0f));
    }
    acc = make_float2(0.f, 0.f);
  }
  template <int NW>
  __device__ void finish(double *) {}
  __device__ void skip() const {}
};

// The four values of a quad with the non-fluid ones set to 0.
__device__ __forceinline__ float4 fluid4(const float4 &v, uint32_t mw) {
  return make_float4(__uint_as_float(__float_as_uint(v.x) & fluid_word(mw, 0)),
                     __uint_as_float(__float_as_uint(v.y) & fluid_word(mw, 1)),
                     __uint_as_float(__float_as_uint(v.z) & fluid_word(mw, 2)),
                     __uint_as_float(__float_as_uint(v.w) & fluid_word(mw, 3)));
}

// ---- two smoothing sweeps per side on a coarse level (TMA path) ----------------------
// On a level l >= 1 the V-cycle can smooth twice before the restriction and
// twice after the prolongation (symmetric, so the preconditioner stays SPD):
//   TSmooth<T, false>  e_b = e_a + w (r - A e_a),  e_a = w r  formed on the fly
//   TDownE             res = r - A e_b  (e_b stored), restricted as TDown
//   TUpE               e_c = e_b + alpha P e_coarse (on the fly);
//                      e_d = e_c + w (r - A e_c)
//   TSmooth<T, true>   e = e_d + w (r - A e_d)  (e_d stored)
// with w = OMEGA / D; every value masked to fluid cells.  These are the
// operations of TDown / TUp with the stored correction as the smoothed
// quantity.

// One damped-Jacobi sweep: out = v + w (r - (6 v - s(v))); v = w r (FROM_B
// false) or the stored correction in b (true).
template <class T, bool FROM_B>
struct TSmooth {
  static constexpr bool HAS_B = FROM_B, HAS_C = false, HAS_EP = false;
  static constexpr int STAGES = 4, MIN_BLOCKS = 4;
  T *out;
  __device__ void init(const SolverState *) {}
  // the stored correction is read through the fluid mask: tiles without
  // fluid are skipped and never written, so a scratch buffer may hold stale
  // values there
  __device__ float4 val4(const StageView<T> &v, int rr, int lane, uint32_t mw) const {
    if (FROM_B) return fluid4(ld4s(v.b, v.fo(rr, lane * 4)), mw);
    const float4 r4 = ld4s(v.a, v.fo(rr, lane * 4));
    return make_float4(r4.x * wdq(mw, 0), r4.y * wdq(mw, 1), r4.z * wdq(mw, 2),
                       r4.w * wdq(mw, 3));
  }
  __device__ float val1(const StageView<T> &v, int rr, int kl) const {
    if (FROM_B) return (v.mask1(rr, kl) & BSP_MFLUID) ? ld1s(v.b, v.fo(rr, kl)) : 0.0f;
    return ld1s(v.a, v.fo(rr, kl)) * wdinv_ns(v.mask1(rr, kl) & 7u);
  }
  __device__ void emit(const StageView<T> &v, int rr, int lane, int, int, int64_t o,
                       uint32_t mc, const float4 &e4, const float (&s)[4], float2 *) {
    const float4 r4 = ld4s(v.a, v.fo(rr, lane * 4));
    float zz[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float e = q4(e4, q);
      const float zq = fmaf(q4(r4, q) - (6.0f * e - s[q]), wdq(mc, q), e);
      zz[q] = __uint_as_float(__float_as_uint(zq) & fluid_word(mc, q));
    }
    st4s(out, o, make_float4(zz[0], zz[1], zz[2], zz[3]));
  }
  __device__ void after_step(int, int, int, bool, float2 *) {}
  template <int NW>
  __device__ void finish(double *) {}
  __device__ void skip() const {}
};

// TDown with the pre-smoothed correction read from b (stored by TSmooth),
// through the fluid mask.
template <class T>
struct TDownE : TDown<T> {
  static constexpr bool HAS_B = true, HAS_C = false, HAS_EP = false;
  __device__ float4 val4(const StageView<T> &v, int rr, int lane, uint32_t mw) const {
    return fluid4(ld4s(v.b, v.fo(rr, lane * 4)), mw);
  }
  __device__ float val1(const StageView<T> &v, int rr, int kl) const {
    return (v.mask1(rr, kl) & BSP_MFLUID) ? ld1s(v.b, v.fo(rr, kl)) : 0.0f;
  }
};

// TUp with the pre-smoothed correction read from b instead of w r.
template <class T>
struct TUpE : TUp<T> {
  static constexpr bool HAS_B = true, HAS_C = true, HAS_EP = false;
  __device__ float4 val4(const StageView<T> &v, int rr, int lane, uint32_t mw) {
    this->shift_w(mw);
    const float4 b4 = ld4s(v.b, v.fo(rr, lane * 4));
    float2 ec = ld2s(v.c, v.co(rr, lane * 4));
    ec.x *= this->alpha;
    ec.y *= this->alpha;
    auto fl = [&](float x, int q) {
      return __uint_as_float(__float_as_uint(x) & fluid_word(mw, q));
    };
    return make_float4(fl(b4.x + ec.x, 0), fl(b4.y + ec.x, 1), fl(b4.z + ec.y, 2),
                       fl(b4.w + ec.y, 3));
  }
  __device__ float val1(const StageView<T> &v, int rr, int kl) const {
    const uint32_t mb = v.mask1(rr, kl);
    return (mb & BSP_MFLUID) ? ld1s(v.b, v.fo(rr, kl)) + this->alpha * ld1s(v.c, v.co(rr, kl))
                             : 0.0f;
  }
};

// ---- trilinear transfers between levels 0 and 1 --------------------------------------
// Cell-centred trilinear interpolation with the weights renormalised over the
// fluid coarse parents: fine cell f takes
//   P e_c (f) = sum_parents w(f, c) e_c / tot(f),  tot(f) = sum over fluid parents of w(f, c),
// w the product of the 1-D weights 3/4 (nearer parent) and 1/4, the parents of
// fine index x being (x - 1) >> 1 and the one after it (outside the grid: no
// parent).  tot(f) depends on the parities of (i, j, k) and on which of the
// eight parents are fluid: the fine "parent pattern" byte (bit 4a + 2b + c for
// parent offsets a, b, c) and a 2048-entry table of 1 / tot indexed by
// parity bits and pattern.  The restriction is R = 1/2 P^T: the residual
// times 1 / tot(f), gathered by tri_restrict with the same weights.  (A CPU
// model of the preconditioned CG: 22 -> 16 inner iterations on the 64x64x48
// pot, 25 -> 19 at 96x96x64, both with two sweeps a side on level 1.)
__device__ float g_tri_invtot[2048];

// Prolongation of the coarse correction onto the 4 fine cells of (row rr,
// lane) of a stage, times 1 / tot; the coarse tiles c (parent plane
// (plane - 1) >> 1) and c2 (the next), rows rr >> 1 and + 1.
template <class T>
__device__ __forceinline__ float4 tri_prolong4(const StageView<T> &v, const float *tab, int rr,
                                               int lane) {
  constexpr int CW = TmaGeom<T>::CW, PAD = TmaGeom<T>::PAD;
  const int pi = v.plane & 1, pj = (rr + 1) & 1;
  const float wi0 = pi ? 0.75f : 0.25f, wi1 = pi ? 0.25f : 0.75f;
  const float wj0 = pj ? 0.75f : 0.25f, wj1 = pj ? 0.25f : 0.75f;
  const int r0 = (rr >> 1) * CW, r1 = r0 + CW;
  const int col = PAD + 2 * lane - 1;
  float X[4];
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    const float a = fmaf(wj0, ld1s(v.c, r0 + col + kk), wj1 * ld1s(v.c, r1 + col + kk));
    const float b = fmaf(wj0, ld1s(v.c2, r0 + col + kk), wj1 * ld1s(v.c2, r1 + col + kk));
    X[kk] = fmaf(wi0, a, wi1 * b);
  }
  const uint32_t pat = *reinterpret_cast<const uint32_t *>(v.q + rr * MASK_W + MASK_PAD + lane * 4);
  const int par = (pi << 10) | (pj << 9);
  const float e0 = fmaf(0.25f, X[0], 0.75f * X[1]), e1 = fmaf(0.75f, X[1], 0.25f * X[2]);
  const float e2 = fmaf(0.25f, X[1], 0.75f * X[2]), e3 = fmaf(0.75f, X[2], 0.25f * X[3]);
  return make_float4(e0 * __ldg(tab + (par | (pat & 0xffu))),
                     e1 * __ldg(tab + (par | 256 | ((pat >> 8) & 0xffu))),
                     e2 * __ldg(tab + (par | ((pat >> 16) & 0xffu))),
                     e3 * __ldg(tab + (par | 256 | (pat >> 24))));
}
// The same for one fine cell at kl (-1 or 128: the tile's k halo).
template <class T>
__device__ __forceinline__ float tri_prolong1(const StageView<T> &v, const float *tab, int rr,
                                              int kl) {
  constexpr int CW = TmaGeom<T>::CW, PAD = TmaGeom<T>::PAD;
  const int pi = v.plane & 1, pj = (rr + 1) & 1, pk = kl & 1;
  const float wi0 = pi ? 0.75f : 0.25f, wi1 = pi ? 0.25f : 0.75f;
  const float wj0 = pj ? 0.75f : 0.25f, wj1 = pj ? 0.25f : 0.75f;
  const float wk0 = pk ? 0.75f : 0.25f, wk1 = pk ? 0.25f : 0.75f;
  const int r0 = (rr >> 1) * CW, r1 = r0 + CW;
  const int col = PAD + ((kl - 1) >> 1);
  float X[2];
#pragma unroll
  for (int kk = 0; kk < 2; ++kk) {
    const float a = fmaf(wj0, ld1s(v.c, r0 + col + kk), wj1 * ld1s(v.c, r1 + col + kk));
    const float b = fmaf(wj0, ld1s(v.c2, r0 + col + kk), wj1 * ld1s(v.c2, r1 + col + kk));
    X[kk] = fmaf(wi0, a, wi1 * b);
  }
  const uint32_t pat = v.q[rr * MASK_W + MASK_PAD + kl];
  return fmaf(wk0, X[0], wk1 * X[1]) * __ldg(tab + ((pi << 10) | (pj << 9) | (pk << 8) | pat));
}

// TUp with the trilinear prolongation from level 1.
template <class T>
struct TUp3 : TUp<T> {
  static constexpr bool HAS_B = false, HAS_C = true, HAS_EP = false, HAS_C2 = true, HAS_Q = true;
  const float *tab;
  __device__ float4 val4(const StageView<T> &v, int rr, int lane, uint32_t mw) {
    this->shift_w(mw);
    const float4 r4 = ld4s(v.a, v.fo(rr, lane * 4));
    const float4 ef = tri_prolong4(v, tab, rr, lane);
    const float al = this->alpha;
    const float *w = this->wn;
    auto fl = [&](float x, int q) {
      return __uint_as_float(__float_as_uint(x) & fluid_word(mw, q));
    };
    return make_float4(fl(fmaf(r4.x, w[0], al * ef.x), 0), fl(fmaf(r4.y, w[1], al * ef.y), 1),
                       fl(fmaf(r4.z, w[2], al * ef.z), 2), fl(fmaf(r4.w, w[3], al * ef.w), 3));
  }
  __device__ float val1(const StageView<T> &v, int rr, int kl) const {
    const uint32_t mb = v.mask1(rr, kl);
    return (mb & BSP_MFLUID) ? fmaf(ld1s(v.a, v.fo(rr, kl)), wdinv_ns(mb & 7u),
                                    this->alpha * tri_prolong1(v, tab, rr, kl))
                             : 0.0f;
  }
};

// The CG update of the previous iteration fused into the restriction:
// r_out = r_in - alpha Ap (stored through T and read back, as the separate
// update kernel), e += alpha ps on the CTA's output cells, partial ||r_out||^2,
// and the restriction of r_out as TDown.  r_in and r_out are different
// buffers: the tiles of neighbouring CTAs overlap, so an in-place update
// could be applied twice.  Without a pending update (first inner iteration of
// a refinement pass) r_out = r_in.
template <class T, bool TRI = false>
struct TDownU {
  // e and ps of the 8 output rows come as TMA tiles too (EP); 3 stages keep
  // three CTAs per SM.  TRI: the trilinear restriction instead of the 2x2x2
  // sums -- the residual divided by its parents' weight sum (the parent-pattern
  // tile q and the table tab) goes to rs, and tri_restrict gathers it.
  static constexpr bool HAS_B = true, HAS_C = false, HAS_EP = true, HAS_Q = TRI;
  static constexpr int STAGES = 3, MIN_BLOCKS = 3;
  const uint8_t *mask1;
  T *r1, *r_out;
  float *e;
  const T *ps;
  double *partials;
  T *rs;             // TRI: scaled residual (level-0 sized)
  const float *tab;  // TRI: 1 / parents' weight sum by parity and pattern
  int nx, ny, ny1, nz1;
  float alpha;
  bool upd;
  float2 acc;
  double rr;
  __device__ void init(const SolverState *st) {
    upd = st->pending != 0;
    alpha = upd ? (float)st->alpha : 0.0f;
    acc = make_float2(0.f, 0.f);
    rr = 0.0;
  }
  // the updated residual of the plane val4 saw last and of the one before it
  // (which emit of that plane stores)
  float4 rn4, rc4;
  __device__ float4 rnew4(const StageView<T> &v, int row, int lane) const {
    const float4 r4 = ld4s(v.a, v.fo(row, lane * 4));
    if (!upd) return r4;
    const float4 a4 = ld4s(v.b, v.fo(row, lane * 4));
    float4 back;
    pk4(make_float4(fmaf(-alpha, a4.x, r4.x), fmaf(-alpha, a4.y, r4.y),
                    fmaf(-alpha, a4.z, r4.z), fmaf(-alpha, a4.w, r4.w)),
        back, r_out);
    return back;
  }
  __device__ float4 val4(const StageView<T> &v, int row, int lane, uint32_t mw) {
    rc4 = rn4;
    rn4 = rnew4(v, row, lane);
    return make_float4(rn4.x * wdq(mw, 0), rn4.y * wdq(mw, 1), rn4.z * wdq(mw, 2),
                       rn4.w * wdq(mw, 3));
  }
  __device__ float val1(const StageView<T> &v, int row, int kl) const {
    float rv = ld1s(v.a, v.fo(row, kl));
    if (upd) rv = rt(fmaf(-alpha, ld1s(v.b, v.fo(row, kl)), rv), r_out);
    return rv * wdinv_ns(v.mask1(row, kl) & 7u);
  }
  __device__ bool pair_end(int i) const { return (i & 1) || i + 1 == nx; }
  __device__ void emit(const StageView<T> &v, int row, int lane, int i, int, int64_t o_,
                       uint32_t mc, const float4 &e4, const float (&s)[4], float2 *xch) {
    const int64_t o = o_;
    const float4 r4 = rc4;  // rnew4 of this plane, from its val4
    st4s(r_out, o, r4);
    if (upd) {
      float4 ee = *reinterpret_cast<const float4 *>(v.e + (row - 1) * 128 + lane * 4);
      const float4 pp = ld4s(v.ps, (row - 1) * 128 + lane * 4);
      ee = make_float4(fmaf(alpha, pp.x, ee.x), fmaf(alpha, pp.y, ee.y), fmaf(alpha, pp.z, ee.z),
                       fmaf(alpha, pp.w, ee.w));
      *reinterpret_cast<float4 *>(e + o) = ee;
    }
    rr += sq4w(r4);
    float res[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float rq = q4(r4, q) - (6.0f * q4(e4, q) - s[q]);
      res[q] = __uint_as_float(__float_as_uint(rq) & fluid_word(mc, q));
    }
    if (TRI) {
      const uint32_t pat = *reinterpret_cast<const uint32_t *>(v.q + row * MASK_W + MASK_PAD +
                                                               lane * 4);
      const int par = ((i & 1) << 10) | (((row + 1) & 1) << 9);
      float o[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        o[q] = res[q] * __ldg(tab + (par | ((q & 1) << 8) | ((pat >> (8 * q)) & 0xffu)));
      st4s(rs, o_, make_float4(o[0], o[1], o[2], o[3]));
      return;
    }
    acc.x += res[0] + res[1];
    acc.y += res[2] + res[3];
    const int warp = threadIdx.x >> 5;
    if (pair_end(i) && (warp & 1)) {
      xch[(warp >> 1) * 32 + lane] = acc;
      acc = make_float2(0.f, 0.f);
    }
  }
  __device__ void after_step(int i, int j, int k, bool act, float2 *xch) {
    if (TRI) return;
    const int warp = threadIdx.x >> 5;
    if (!pair_end(i) || (warp & 1)) return;
    if (act) {
      float2 t = acc;
      if (j + 1 < ny) {
        const float2 o2 = xch[(warp >> 1) * 32 + (threadIdx.x & 31)];
        t.x += o2.x;
        t.y += o2.y;
      }
      const int64_t C = ((int64_t)(i >> 1) * ny1 + (j >> 1)) * nz1 + (k >> 1);
      const uint32_t m2 = __ldg(reinterpret_cast<const uint16_t *>(mask1 + C));
      st2s(r1, C, make_float2((m2 & BSP_MFLUID) ? 0.5f * t.x : 0.0f,
                              ((m2 >> 8) & BSP_MFLUID) ? 0.5f * t.y : 0.0f));
    }
    acc = make_float2(0.f, 0.f);
  }
  template <int NW>
  __device__ void finish(double *sh) { block_partial<NW>(rr, partials, sh); }
  __device__ void skip() const { partials[block_linear()] = 0.0; }
};

// TDownU compiled for four CTAs per SM (registers capped at 48 a thread).
template <class T>
struct TDownU4 : TDownU<T> {
  static constexpr int MIN_BLOCKS = 4;
};

// BSP_TUNE_DOWNU_BLOCKS: CTAs per SM the fused update + restriction kernel is
// compiled for, 3 (default) or 4.  Measured at 384x384x256: 11.53 ms per
// solve with 3, 11.60 with 4 (48 registers and a small spill).
int g_downu_blocks = 3;

constexpr int align128(int b) { return (b + 127) / 128 * 128; }

// Every TMA destination starts on a 128-byte boundary.
// Optional operand flags of an op (false when the op does not declare them).
template <class Op, class = void>
struct op_c2 : std::false_type {};
template <class Op>
struct op_c2<Op, std::void_t<decltype(Op::HAS_C2)>> : std::integral_constant<bool, Op::HAS_C2> {};
template <class Op, class = void>
struct op_q : std::false_type {};
template <class Op>
struct op_q<Op, std::void_t<decltype(Op::HAS_Q)>> : std::integral_constant<bool, Op::HAS_Q> {};

template <class T, class Op>
struct TmaSmem {
  static constexpr int FB = TmaGeom<T>::FBYTES, MB = TmaGeom<T>::MBYTES,
                       CB = TmaGeom<T>::CBYTES;
  static constexpr int EB = TILE_ROWS * 128 * 4, PB = TILE_ROWS * 128 * (int)sizeof(T);
  static constexpr bool C2 = op_c2<Op>::value, Q = op_q<Op>::value;
  static constexpr int NST = Op::STAGES;
  static constexpr int OFF_B = align128(FB);
  static constexpr int OFF_M = OFF_B + (Op::HAS_B ? align128(FB) : 0);
  static constexpr int OFF_C = OFF_M + align128(MB);
  static constexpr int OFF_C2 = OFF_C + (Op::HAS_C ? align128(CB) : 0);
  static constexpr int OFF_Q = OFF_C2 + (C2 ? align128(CB) : 0);
  static constexpr int OFF_E = OFF_Q + (Q ? align128(MB) : 0);
  static constexpr int OFF_P = OFF_E + (Op::HAS_EP ? EB : 0);
  static constexpr int STAGE = OFF_P + (Op::HAS_EP ? align128(PB) : 0);
  static constexpr uint32_t TX = (uint32_t)(FB + (Op::HAS_B ? FB : 0) + MB + (Op::HAS_C ? CB : 0) +
                                            (C2 ? CB : 0) + (Q ? MB : 0) +
                                            (Op::HAS_EP ? EB + PB : 0));
  static constexpr int RING = STAGE * NST;
  // ring | plane_buf (2 x 10 x 32 float4) | mbarriers
  static constexpr int OFF_PLANE = RING;
  static constexpr int OFF_BAR = RING + 2 * TMA_ROWS * 32 * 16;
  static constexpr int TOTAL = OFF_BAR + NST * 8;
};

// The scalar update after a reducing level-0 kernel, run by its last CTA
// (kind != TAIL_NONE): every CTA, once its partial is written, takes a ticket;
// the CTA with the last one sums the partials in a fixed order (thread t the
// blocks t, t + TILE_THREADS, ..., then a fixed shuffle tree and the warps in
// order) and applies the update, then resets the ticket counter.
__device__ __forceinline__ void fine_tail(SolverState *st, int kind, const double *partials) {
  if (kind == TAIL_NONE || !partials) return;
  __shared__ int s_last;
  __shared__ double s_w[TILE_WARPS];
  const int nb = (int)(gridDim.x * gridDim.y * gridDim.z);
  __syncthreads();  // this CTA's partial is written
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&st->tail_count, 1) == nb - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double v = 0.0;
  for (int b = threadIdx.x; b < nb; b += TILE_THREADS)
    v += *reinterpret_cast<const volatile double *>(partials + b);
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < TILE_WARPS; ++w) t += s_w[w];
    apply_tail(st, kind, t);
    st->tail_count = 0;
  }
}

// An op's FP64 partials (slot 0, one per CTA), or NULL for ops that reduce nothing.
template <class Op, class = void>
struct has_partials : std::false_type {};
template <class Op>
struct has_partials<Op, std::void_t<decltype(std::declval<Op>().partials)>> : std::true_type {};
template <class Op>
__device__ __forceinline__ const double *op_partials(const Op &op) {
  if constexpr (has_partials<Op>::value)
    return op.partials;
  else
    return nullptr;
}

// The host side: one pending request, consumed by the next TMA launch.
struct TailReq {
  SolverState *st = nullptr;
  int kind = TAIL_NONE;
  bool taken = false;
};
static thread_local TailReq t_tail;
void fine_tail_request(SolverState *st, int kind) { t_tail = TailReq{st, kind, false}; }
bool fine_tail_taken() {
  const bool t = t_tail.taken;
  t_tail = TailReq{};
  return t;
}

template <class T, class Op>
__global__ void __launch_bounds__(TILE_THREADS, Op::MIN_BLOCKS) fine_tma_kernel(
    Op op, const __grid_constant__ TmaMaps maps, int nx, int ny, int nz, int bi,
    const uint8_t *tiles, const SolverState *st, SolverState *tail_st, int tail_kind) {
  // the tile flags are written at setup only; everything the previous kernel
  // of the stream writes is read (and the partials written) after pdl_wait
  if (tiles && !tiles[block_linear()]) {
    pdl_wait();
    if (st->inner_done) return;
    if (threadIdx.x == 0) op.skip();
    fine_tail(tail_st, tail_kind, op_partials(op));
    return;
  }
  using L = TmaSmem<T, Op>;
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ double sh[TILE_WARPS];
  __shared__ float2 xch[(TILE_ROWS / 2) * 32];
  // k-halo operands (k0 - 1, k0 + 128) of the output rows, per plane parity,
  // computed by the second halo warp one plane ahead
  __shared__ float hbuf[2][TILE_ROWS + 2][2];
  float4(*plane_buf)[TMA_ROWS][32] = reinterpret_cast<float4(*)[TMA_ROWS][32]>(dsm + L::OFF_PLANE);
  uint64_t *bars = reinterpret_cast<uint64_t *>(dsm + L::OFF_BAR);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const bool producer = threadIdx.x == TILE_ROWS * 32;  // lane 0 of the first halo warp
  const int j0 = blockIdx.y * TILE_ROWS;
  const int k0 = blockIdx.x * 128;
  const int i0 = blockIdx.z * bi;
  const int i1 = min(i0 + bi, nx);
  const int pbase = i0 - 1;  // first plane of the ring
  constexpr int PAD = TmaGeom<T>::PAD;
  if (threadIdx.x < 8) s_wtab[threadIdx.x] = wcalc(threadIdx.x);
  if (threadIdx.x < 0x88) s_wtabf[threadIdx.x] = threadIdx.x >= 0x80 ? wcalc(threadIdx.x & 7u) : 0.0f;
  if (producer) {
    for (int q = 0; q < L::NST; ++q) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  pdl_wait();
  if (st->inner_done) return;  // uniform: the whole grid returns
  auto issue = [&](int p) {  // producer only: plane p into its stage
    const int q = (p - pbase) % L::NST;
    unsigned char *base = dsm + q * L::STAGE;
    mbar_expect_tx(&bars[q], L::TX);
    tma_load3(base, &maps.a, k0 - PAD, j0 - 1, p, &bars[q]);
    if (Op::HAS_B) tma_load3(base + L::OFF_B, &maps.b, k0 - PAD, j0 - 1, p, &bars[q]);
    tma_load3(base + L::OFF_M, &maps.m, k0 - MASK_PAD, j0 - 1, p, &bars[q]);
    if (Op::HAS_C) {
      // trilinear: the two parent planes (p - 1) >> 1 and the one after it
      // (plane -1 arrives as zeros); else the parent plane p >> 1
      const int pc = L::C2 ? ((p - 1) >> 1) : (p >> 1);
      tma_load3(base + L::OFF_C, &maps.c, k0 / 2 - PAD, j0 / 2 - 1, pc, &bars[q]);
      if (L::C2) tma_load3(base + L::OFF_C2, &maps.c, k0 / 2 - PAD, j0 / 2 - 1, pc + 1, &bars[q]);
    }
    if (L::Q) tma_load3(base + L::OFF_Q, &maps.q, k0 - MASK_PAD, j0 - 1, p, &bars[q]);
    if (Op::HAS_EP) {
      tma_load3(base + L::OFF_E, &maps.e, k0, j0, p, &bars[q]);
      tma_load3(base + L::OFF_P, &maps.p, k0, j0, p, &bars[q]);
    }
  };
  auto view_s = [&](int stage, int p) {
    const unsigned char *base = dsm + stage * L::STAGE;
    StageView<T> v;
    v.a = reinterpret_cast<const T *>(base);
    v.b = reinterpret_cast<const T *>(base + L::OFF_B);
    v.m = base + L::OFF_M;
    v.c = reinterpret_cast<const T *>(base + L::OFF_C);
    v.c2 = reinterpret_cast<const T *>(base + L::OFF_C2);
    v.q = base + L::OFF_Q;
    v.plane = p;
    v.e = reinterpret_cast<const float *>(base + L::OFF_E);
    v.ps = reinterpret_cast<const T *>(base + L::OFF_P);
    return v;
  };
  bool ok = true;
  auto view = [&](int p) { return view_s((p - pbase) % L::NST, p); };
  auto wait = [&](int p) {
    const int n = p - pbase;
    if (!mbar_wait(&bars[n % L::NST], (uint32_t)((n / L::NST) & 1))) ok = false;
  };
  auto wait_s = [&](int stage, uint32_t phase) {
    if (!mbar_wait(&bars[stage], phase)) ok = false;
  };
  if (producer)
    for (int p = pbase; p <= min(pbase + L::NST - 1, i1); ++p) issue(p);
  op.init(st);
  // tile row of this warp: 0 = j0-1, 1..8 = output rows, 9 = j0+8
  const int rr = warp < TILE_ROWS ? warp + 1 : (warp == TILE_ROWS ? 0 : TILE_ROWS + 1);
  const int j = j0 + rr - 1;
  const int k = k0 + lane * 4;
  const bool act = j >= 0 && j < ny && k < nz;
  const bool out = warp < TILE_ROWS;
  const int64_t plane = (int64_t)ny * nz;
  float4 vm = make_float4(0.f, 0.f, 0.f, 0.f), vc;
  uint32_t mc;
  wait(pbase);
  if (out) {
    const StageView<T> v = view(pbase);
    vm = op.val4(v, rr, lane, v.mask4(rr, lane));
  }
  // the second halo warp's lanes 0..15: the k-halo operand of output row
  // 1 + lane / 2, side lane % 2 (k0 - 1, k0 + 128), of plane p
  const bool hw = warp == TILE_ROWS + 1 && lane < 2 * TILE_ROWS;
  auto halo = [&](const StageView<T> &v, int p) {
    if (hw) hbuf[p & 1][1 + (lane >> 1)][lane & 1] = op.val1(v, 1 + (lane >> 1), (lane & 1) ? 128 : -1);
  };
  wait(i0);
  {
    const StageView<T> v = view(i0);
    mc = v.mask4(rr, lane);
    vc = op.val4(v, rr, lane, mc);
    halo(v, i0);
  }
  plane_buf[i0 & 1][rr][lane] = vc;
  __syncthreads();
  if (producer && pbase + L::NST <= i1) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    issue(pbase + L::NST);
  }
  int64_t o = (int64_t)i0 * plane + (int64_t)j * nz + k;
  // the ring walked with running counters: plane p sits in stage
  // (p - pbase) % NST, filled for the ((p - pbase) / NST)-th time
  int st_cur = 1 % L::NST;                   // plane i0
  int st_nx = 2 % L::NST;                    // plane i0 + 1
  uint32_t ph_nx = (uint32_t)(2 / L::NST) & 1u;
  for (int i = i0; i < i1; ++i) {
    wait_s(st_nx, ph_nx);
    const StageView<T> vnx = view_s(st_nx, i + 1);
    const uint32_t mn = vnx.mask4(rr, lane);
    const float4 vn = op.val4(vnx, rr, lane, mn);
    plane_buf[(i + 1) & 1][rr][lane] = vn;
    if (i + 1 < i1) halo(vnx, i + 1);
    if (out) {
      const StageView<T> v = view_s(st_cur, i);
      const float4 vjm = plane_buf[i & 1][rr - 1][lane];
      const float4 vjp = plane_buf[i & 1][rr + 1][lane];
      float vkm = __shfl_up_sync(0xffffffffu, vc.w, 1);
      float vkp = __shfl_down_sync(0xffffffffu, vc.x, 1);
      // k halo of the row from the tile's padding (zero outside the grid),
      // computed one plane ahead by the halo warp
      if (lane == 0) vkm = hbuf[i & 1][rr][0];
      if (lane == 31) vkp = hbuf[i & 1][rr][1];
      const float4 vb = make_float4(vkm, vc.x, vc.y, vc.z);
      const float4 vf = make_float4(vc.y, vc.z, vc.w, vkp);
      float s[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float sum6 = ((q4(vm, q) + q4(vn, q)) + (q4(vjm, q) + q4(vjp, q))) +
                           (q4(vb, q) + q4(vf, q));
        if constexpr (op_sum6<Op>::value) {
          s[q] = sum6;
        } else {
          const float ns = (float)((mc >> (8 * q)) & 7u);
          s[q] = fmaf(ns, q4(vc, q), sum6);
        }
      }
      if (act) op.emit(v, rr, lane, i, j, o, mc, vc, s, xch);
    }
    __syncthreads();
    if (producer && i + L::NST <= i1) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(i + L::NST);
    }
    if (out) op.after_step(i, j, k, act, xch);
    vm = vc;
    vc = vn;
    mc = mn;
    o += plane;
    st_cur = st_nx;
    if (++st_nx == L::NST) {
      st_nx = 0;
      ph_nx ^= 1u;
    }
  }
  if (producer) {
    // every issued plane has been waited for above; confirm (bounded) that no
    // copy is still in flight before the CTA's shared memory goes away
    for (int p = max(pbase, i1 - L::NST + 1); p <= i1; ++p) wait(p);
  }
  if (!ok) atomicExch(const_cast<int *>(&st->dev_error), 1);
  pdl_trigger();
  op.template finish<TILE_WARPS>(sh);
  fine_tail(tail_st, tail_kind, op_partials(op));
}

// ---- TMA launch helpers (host) ----------------------------------------------------------
bool g_fine_tma_enabled = true;  // BSP_TUNE_FINE_TMA
// BSP_TUNE_PDL: the tile kernels and the scalar kernels of an inner iteration
// launched with programmatic dependent launch (each waits for its
// predecessor in griddepcontrol.wait, so only launch latency overlaps;
// measured 12.31 -> 12.21 ms per solve at 384x384x256)
bool g_pdl = true;

// The TMA path needs nz % 16 == 0 (16-byte mask rows) and 16-byte aligned bases.
static bool tma_eligible(int nz) { return g_fine_tma_enabled && nz % 16 == 0 && encode_tiled(); }
bool fine_tma_available(int nz) { return tma_eligible(nz); }

template <class T, class Op>
static bool launch_tma(const Op &op, const TmaMaps &maps, int nx, int ny, int nz,
                       const uint8_t *tiles, const SolverState *st, cudaStream_t s) {
  using L = TmaSmem<T, Op>;
  if (!smem_opt_in((const void *)fine_tma_kernel<T, Op>, L::TOTAL)) return false;
  // a pending scalar-update request goes with this launch (ops that write a
  // partial per CTA to slot 0 of their partials)
  SolverState *tst = t_tail.st;
  int tkind = tst ? t_tail.kind : TAIL_NONE;
  t_tail.st = nullptr;
  t_tail.kind = TAIL_NONE;
  const bool ok =
      launch_maybe_pdl(g_pdl, fine_grid(nx, ny, nz), dim3(TILE_THREADS), L::TOTAL, s,
                       fine_tma_kernel<T, Op>, op, maps, nx, ny, nz, fine_bi(nx, ny, nz), tiles,
                       st, tst, tkind) == cudaSuccess &&
      cudaGetLastError() == cudaSuccess;
  if (ok && tkind != TAIL_NONE) t_tail.taken = true;
  return ok;
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
                                                          const uint8_t *mask,
                                                          const uint8_t *tiles, const float *div,
                                                          const double *x, double bscale, T *rhat,
                                                          float *e, double *partials,
                                                          const SolverState *st) {
  if (st->done) return;
  if (!WRITE && st->norm_cached) return;  // x = 0: the ||b|| pass's partials stand
  if (tiles && !tiles[block_linear()]) {
    // no fluid: residual 0, and rhat and e are already 0 on these cells
    if (threadIdx.x == 0) {
      partials[block_linear()] = 0.0;
      partials[PARTIAL_STRIDE + block_linear()] = 0.0;
    }
    return;
  }
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
  // while the iterate is known to be zero its loads are skipped: the
  // operands keep their +0.0 defaults, the values the zeroed x holds
  const bool lx = act && !st->x_zero;
  if (lx && i0 > 0) xm = ld4d(x, o - plane);
  if (lx) xc = ld4d(x, o);
  double rr = 0.0, rmax = 0.0;
  for (int i = i0; i < i1; ++i) {
    D4 xn = z4, xjm = z4, xjp = z4;
    if (lx) {
      if (i + 1 < nx) xn = ld4d(x, o + plane);
      if (j > 0) xjm = ld4d(x, o - nz);
      if (j + 1 < ny) xjp = ld4d(x, o + nz);
    }
    double xkm = __shfl_up_sync(0xffffffffu, xc.d, 1);
    double xkp = __shfl_down_sync(0xffffffffu, xc.a, 1);
    if (lane == 0) xkm = (lx && k > 0) ? x[o - 1] : 0.0;
    if (lane == 31) xkp = (lx && k + 4 < nz) ? x[o + 4] : 0.0;
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
int g_fine_bi = 0;  // BSP_TUNE_FINE_BI: plane chunk of the level-0 tiles (0 = rule)

// BSP_TUNE_FINE_CTAS: CTAs per SM the plane chunking aims for (the chunk is
// the largest even plane count that still gives that many CTAs).  4: level 0
// of the 384x384x256 pot keeps 16-plane chunks, levels 1-2 get shorter chunks
// and more CTAs (measured 13.03 -> 12.38 ms per solve against 2; 8: 12.79).
int g_fine_ctas = 4;

int fine_bi(int nx, int ny, int nz) {
  if (g_fine_bi > 0) return g_fine_bi < 2 ? 2 : (g_fine_bi & ~1);
  const int64_t cols = (int64_t)((nz / 4 + 31) / 32) * ((ny + TILE_ROWS - 1) / TILE_ROWS);
  const int64_t target = (int64_t)g_fine_ctas * num_sms();
  int bi = 16;
  while (bi > 2 && cols * ((nx + bi - 1) / bi) < target) bi -= 2;
  return bi;
}

dim3 fine_grid(int nx, int ny, int nz) {
  const int bi = fine_bi(nx, ny, nz);
  return dim3((nz / 4 + 31) / 32, (ny + TILE_ROWS - 1) / TILE_ROWS, (nx + bi - 1) / bi);
}
int fine_grid_blocks(int nx, int ny, int nz) {
  const dim3 g = fine_grid(nx, ny, nz);
  return (int)(g.x * g.y * g.z);
}

template <class T>
void launch_fine_psap(int nx, int ny, int nz, const uint8_t *mask, const uint8_t *tiles,
                      const T *z, const T *prev, T *cur, T *Ap, double *partials,
                      const SolverState *st, cudaStream_t s) {
  if (tma_eligible(nz)) {
    constexpr int FW = TmaGeom<T>::FW;
    TmaMaps maps{};
    if (make_map(&maps.a, tma_dtype<T>(), sizeof(T), z, nx, ny, nz, FW, TMA_ROWS) &&
        make_map(&maps.b, tma_dtype<T>(), sizeof(T), prev, nx, ny, nz, FW, TMA_ROWS) &&
        make_map(&maps.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, mask, nx, ny, nz, MASK_W, TMA_ROWS)) {
      TPsAp<T> op{};
      op.cur = cur;
      op.Ap = Ap;
      op.partials = partials;
      if (launch_tma<T>(op, maps, nx, ny, nz, tiles, st, s)) return;
    }
  }
  PsApOp<T> op{};
  op.mask = mask;
  op.z = z;
  op.prev = prev;
  op.cur = cur;
  op.Ap = Ap;
  op.partials = partials;
  fine_tile_kernel<PsApOp<T>><<<fine_grid(nx, ny, nz), TILE_THREADS, 0, s>>>(
      op, nx, ny, nz, fine_bi(nx, ny, nz), tiles, st);
}

template <class T>
void launch_fine_up(const Level<T> &f, const Level<T> &c, T *z, double *partials, float alpha,
                    const SolverState *st, cudaStream_t s) {
  if (tma_eligible(f.nz) && c.nz * 2 == f.nz && c.ny * 2 >= f.ny && c.nx * 2 >= f.nx) {
    TmaMaps maps{};
    if (make_map(&maps.a, tma_dtype<T>(), sizeof(T), f.r, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                 TMA_ROWS) &&
        make_map(&maps.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, f.mask, f.nx, f.ny, f.nz, MASK_W,
                 TMA_ROWS) &&
        make_map(&maps.c, tma_dtype<T>(), sizeof(T), c.e, c.nx, c.ny, c.nz, TmaGeom<T>::CW,
                 TmaGeom<T>::CROWS)) {
      TUp<T> op{};
      op.z = z;
      op.partials = partials;
      op.alpha = alpha;
      if (launch_tma<T>(op, maps, f.nx, f.ny, f.nz, f.tiles, st, s)) return;
    }
  }
  UpOp<T> op{};
  op.alpha = alpha;
  op.mask = f.mask;
  op.r = f.r;
  op.e1 = c.e;
  op.z = z;
  op.partials = partials;
  op.ny1 = c.ny;
  op.nz1 = c.nz;
  fine_tile_kernel<UpOp<T>><<<fine_grid(f.nx, f.ny, f.nz), TILE_THREADS, 0, s>>>(
      op, f.nx, f.ny, f.nz, fine_bi(f.nx, f.ny, f.nz), f.tiles, st);
}

template <class T>
void launch_fine_down(const Level<T> &f, const Level<T> &c, const SolverState *st,
                      cudaStream_t s) {
  if (tma_eligible(f.nz)) {
    TmaMaps maps{};
    if (make_map(&maps.a, tma_dtype<T>(), sizeof(T), f.r, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                 TMA_ROWS) &&
        make_map(&maps.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, f.mask, f.nx, f.ny, f.nz, MASK_W,
                 TMA_ROWS)) {
      TDown<T> op{};
      op.mask1 = c.mask;
      op.r1 = c.r;
      op.nx = f.nx;
      op.ny = f.ny;
      op.ny1 = c.ny;
      op.nz1 = c.nz;
      if (launch_tma<T>(op, maps, f.nx, f.ny, f.nz, f.tiles, st, s)) return;
    }
  }
  DownOp<T> op{};
  op.mask = f.mask;
  op.mask1 = c.mask;
  op.r = f.r;
  op.r1 = c.r;
  op.nx = f.nx;
  op.ny = f.ny;
  op.ny1 = c.ny;
  op.nz1 = c.nz;
  fine_tile_kernel<DownOp<T>><<<fine_grid(f.nx, f.ny, f.nz), TILE_THREADS, 0, s>>>(
      op, f.nx, f.ny, f.nz, fine_bi(f.nx, f.ny, f.nz), f.tiles, st);
}

// Two-sweep smoothing launchers (TMA path only; false when it cannot run).
// launch_fine_smooth: out = one sweep from e_in (or from w r when e_in is
// NULL); launch_fine_down_e: residual of the stored e and its restriction to
// c.r; launch_fine_up_e: out = e_in + alpha P c.e, then one sweep.
template <class T>
bool launch_fine_smooth(const Level<T> &f, const T *e_in, T *out, const SolverState *st,
                        cudaStream_t s) {
  if (!tma_eligible(f.nz)) return false;
  TmaMaps maps{};
  if (!(make_map(&maps.a, tma_dtype<T>(), sizeof(T), f.r, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                 TMA_ROWS) &&
        make_map(&maps.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, f.mask, f.nx, f.ny, f.nz, MASK_W,
                 TMA_ROWS)))
    return false;
  if (e_in) {
    if (!make_map(&maps.b, tma_dtype<T>(), sizeof(T), e_in, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                  TMA_ROWS))
      return false;
    TSmooth<T, true> op{};
    op.out = out;
    return launch_tma<T>(op, maps, f.nx, f.ny, f.nz, f.tiles, st, s);
  }
  TSmooth<T, false> op{};
  op.out = out;
  return launch_tma<T>(op, maps, f.nx, f.ny, f.nz, f.tiles, st, s);
}

template <class T>
bool launch_fine_down_e(const Level<T> &f, const Level<T> &c, const T *e_in,
                        const SolverState *st, cudaStream_t s) {
  if (!tma_eligible(f.nz)) return false;
  TmaMaps maps{};
  if (!(make_map(&maps.a, tma_dtype<T>(), sizeof(T), f.r, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                 TMA_ROWS) &&
        make_map(&maps.b, tma_dtype<T>(), sizeof(T), e_in, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                 TMA_ROWS) &&
        make_map(&maps.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, f.mask, f.nx, f.ny, f.nz, MASK_W,
                 TMA_ROWS)))
    return false;
  TDownE<T> op{};
  op.mask1 = c.mask;
  op.r1 = c.r;
  op.nx = f.nx;
  op.ny = f.ny;
  op.ny1 = c.ny;
  op.nz1 = c.nz;
  return launch_tma<T>(op, maps, f.nx, f.ny, f.nz, f.tiles, st, s);
}

template <class T>
bool launch_fine_up_e(const Level<T> &f, const Level<T> &c, const T *e_in, T *out,
                      double *partials, float alpha, const SolverState *st, cudaStream_t s) {
  if (!(tma_eligible(f.nz) && c.nz * 2 == f.nz && c.ny * 2 >= f.ny && c.nx * 2 >= f.nx))
    return false;
  TmaMaps maps{};
  if (!(make_map(&maps.a, tma_dtype<T>(), sizeof(T), f.r, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                 TMA_ROWS) &&
        make_map(&maps.b, tma_dtype<T>(), sizeof(T), e_in, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                 TMA_ROWS) &&
        make_map(&maps.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, f.mask, f.nx, f.ny, f.nz, MASK_W,
                 TMA_ROWS) &&
        make_map(&maps.c, tma_dtype<T>(), sizeof(T), c.e, c.nx, c.ny, c.nz, TmaGeom<T>::CW,
                 TmaGeom<T>::CROWS)))
    return false;
  TUpE<T> op{};
  op.z = out;
  op.partials = partials;
  op.alpha = alpha;
  return launch_tma<T>(op, maps, f.nx, f.ny, f.nz, f.tiles, st, s);
}

// ---- trilinear transfers: setup, restriction, launchers ----------------------------
// Parent pattern of every fine fluid cell (0 elsewhere) from the coarse classes.
__global__ void tri_pattern_kernel(uint8_t *__restrict__ pat, const uint8_t *__restrict__ mask,
                                   const uint8_t *__restrict__ mask1, int nx, int ny, int nz,
                                   int cx, int cy, int cz) {
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    uint32_t bits = 0;
    if (mask[v] & BSP_MFLUID) {
      const int k = (int)(v % nz);
      const int64_t r = v / nz;
      const int j = (int)(r % ny), i = (int)(r / ny);
      const int i0 = (i - 1) >> 1, j0 = (j - 1) >> 1, k0 = (k - 1) >> 1;
      for (int b = 0; b < 8; ++b) {
        const int ci = i0 + (b >> 2), cj = j0 + ((b >> 1) & 1), ck = k0 + (b & 1);
        if (ci < 0 || cj < 0 || ck < 0 || ci >= cx || cj >= cy || ck >= cz) continue;
        if (mask1[((int64_t)ci * cy + cj) * cz + ck] & BSP_MFLUID) bits |= 1u << b;
      }
    }
    pat[v] = (uint8_t)bits;
  }
}

// r1 = 1/2 P^T applied to the scaled residual rs (already divided by tot):
// coarse cell c takes the fine cells 2c-1 .. 2c+2 of each axis with weights
// 1/4, 3/4, 3/4, 1/4; fluid coarse cells only.  A thread owns one coarse
// (j, k) column and marches a chunk of coarse planes, each fine plane's
// 4 x 4 sum computed once and shared by the two coarse planes it feeds.
template <class T>
__global__ void __launch_bounds__(128) tri_restrict_kernel(T *__restrict__ r1,
                                                           const T *__restrict__ rs,
                                                           const uint8_t *__restrict__ mask1,
                                                           int nx, int ny, int nz, int cx, int cy,
                                                           int cz, int cpc,
                                                           const SolverState *st) {
  if (st->inner_done) return;
  const int kc = blockIdx.x * blockDim.x + threadIdx.x;
  const int jc = blockIdx.y;
  const int c0 = blockIdx.z * cpc, c1 = min(c0 + cpc, cx);
  if (kc >= cz || jc >= cy) return;
  const float w[4] = {0.25f, 0.75f, 0.75f, 0.25f};
  auto plane_sum = [&](int f) {
    float sum = 0.0f;
    if (f < 0 || f >= nx) return sum;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int fj = 2 * jc - 1 + b;
      if (fj < 0 || fj >= ny) continue;
      const T *row = rs + ((int64_t)f * ny + fj) * nz;
      float t = 0.0f;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int fk = 2 * kc - 1 + a;
        if (fk >= 0 && fk < nz) t = fmaf(w[a], ld1s(row, fk), t);
      }
      sum = fmaf(w[b], t, sum);
    }
    return sum;
  };
  float pm = plane_sum(2 * c0 - 1), p0 = plane_sum(2 * c0);
  for (int c = c0; c < c1; ++c) {
    const float p1 = plane_sum(2 * c + 1), p2 = plane_sum(2 * c + 2);
    const float acc = fmaf(0.25f, p2, fmaf(0.75f, p1, fmaf(0.75f, p0, 0.25f * pm)));
    const int64_t C = ((int64_t)c * cy + jc) * cz + kc;
    st1s(r1, C, (mask1[C] & BSP_MFLUID) ? 0.5f * acc : 0.0f);
    pm = p1;
    p0 = p2;
  }
}

// 1 / tot for parity bits (pi << 10 | pj << 9 | pk << 8) and parent pattern,
// copied to the device once per device (a synchronous copy: call it outside
// any stream capture, as the solve entry points do); NULL if that failed.
const float *tri_table() {
  static std::once_flag once[64];
  static bool ok[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::call_once(once[dev & 63], [dev] {
    float h[2048];
    auto w = [](int par, int a) { return par ? (a ? 0.25f : 0.75f) : (a ? 0.75f : 0.25f); };
    for (int idx = 0; idx < 2048; ++idx) {
      const int pi = (idx >> 10) & 1, pj = (idx >> 9) & 1, pk = (idx >> 8) & 1, pat = idx & 255;
      float tot = 0.0f;
      for (int n = 0; n < 8; ++n)
        if (pat & (1 << n)) tot += w(pi, n >> 2) * w(pj, (n >> 1) & 1) * w(pk, n & 1);
      h[idx] = tot > 0.0f ? 1.0f / tot : 0.0f;
    }
    ok[dev & 63] = cudaMemcpyToSymbol(g_tri_invtot, h, sizeof(h)) == cudaSuccess;
  });
  if (!ok[dev & 63]) return nullptr;
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_tri_invtot) != cudaSuccess) return nullptr;
  return static_cast<const float *>(p);
}

template <class T>
void launch_tri_setup(uint8_t *pat, const Level<T> &f, const Level<T> &c, cudaStream_t s) {
  const int64_t n = (int64_t)f.nx * f.ny * f.nz;
  int64_t b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  tri_pattern_kernel<<<(int)(b > 0 ? b : 1), 256, 0, s>>>(pat, f.mask, c.mask, f.nx, f.ny, f.nz,
                                                          c.nx, c.ny, c.nz);
}

// Coarse planes per thread of tri_restrict (BSP_TUNE_TRI_CPC, default 8: a fine
// plane's 4 x 4 sum serves two coarse planes; 1 and 2 measured slower).
int g_tri_cpc = 8;

template <class T>
void launch_tri_restrict(const Level<T> &f, const Level<T> &c, const T *rs, const SolverState *st,
                         cudaStream_t s) {
  const int cpc = g_tri_cpc;
  dim3 grid((c.nz + 127) / 128, c.ny, (c.nx + cpc - 1) / cpc);
  tri_restrict_kernel<T><<<grid, 128, 0, s>>>(c.r, rs, c.mask, f.nx, f.ny, f.nz, c.nx, c.ny,
                                               c.nz, cpc, st);
}

// The trilinear prolongation + post-smoothing onto level 0 (TMA path only;
// false when it cannot run).
template <class T>
bool launch_fine_up_tri(const Level<T> &f, const Level<T> &c, T *z, double *partials,
                        float alpha, const uint8_t *pat, const float *tab, const SolverState *st,
                        cudaStream_t s) {
  if (!(tma_eligible(f.nz) && c.nz * 2 == f.nz && c.ny * 2 >= f.ny && c.nx * 2 >= f.nx && tab))
    return false;
  TmaMaps maps{};
  if (!(make_map(&maps.a, tma_dtype<T>(), sizeof(T), f.r, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                 TMA_ROWS) &&
        make_map(&maps.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, f.mask, f.nx, f.ny, f.nz, MASK_W,
                 TMA_ROWS) &&
        make_map(&maps.q, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, pat, f.nx, f.ny, f.nz, MASK_W,
                 TMA_ROWS) &&
        make_map(&maps.c, tma_dtype<T>(), sizeof(T), c.e, c.nx, c.ny, c.nz, TmaGeom<T>::CW,
                 TmaGeom<T>::CROWS)))
    return false;
  TUp3<T> op{};
  op.z = z;
  op.partials = partials;
  op.alpha = alpha;
  op.tab = tab;
  return launch_tma<T>(op, maps, f.nx, f.ny, f.nz, f.tiles, st, s);
}

// Level-0 restriction with the previous iteration's CG update fused in (TMA
// path only; false when it cannot run).  f.r is r_in.
template <class T>
bool launch_fine_down_update(const Level<T> &f, const Level<T> &c, T *r_out, float *e,
                             const T *ps, const T *Ap, double *partials, const SolverState *st,
                             cudaStream_t s, T *rs, const uint8_t *pat, const float *tab) {
  if (!tma_eligible(f.nz)) return false;
  TmaMaps maps{};
  if (!(make_map(&maps.a, tma_dtype<T>(), sizeof(T), f.r, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                 TMA_ROWS) &&
        make_map(&maps.b, tma_dtype<T>(), sizeof(T), Ap, f.nx, f.ny, f.nz, TmaGeom<T>::FW,
                 TMA_ROWS) &&
        make_map(&maps.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, f.mask, f.nx, f.ny, f.nz, MASK_W,
                 TMA_ROWS) &&
        make_map(&maps.e, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, e, f.nx, f.ny, f.nz, 128,
                 TILE_ROWS) &&
        make_map(&maps.p, tma_dtype<T>(), sizeof(T), ps, f.nx, f.ny, f.nz, 128, TILE_ROWS)))
    return false;
  if (rs) {
    // trilinear: the scaled residual to rs (tri_restrict gathers it)
    if (!pat || !tab ||
        !make_map(&maps.q, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, pat, f.nx, f.ny, f.nz, MASK_W,
                  TMA_ROWS))
      return false;
    TDownU<T, true> op{};
    op.mask1 = c.mask;
    op.r1 = c.r;
    op.r_out = r_out;
    op.e = e;
    op.ps = ps;
    op.partials = partials;
    op.rs = rs;
    op.tab = tab;
    op.nx = f.nx;
    op.ny = f.ny;
    op.ny1 = c.ny;
    op.nz1 = c.nz;
    return launch_tma<T>(op, maps, f.nx, f.ny, f.nz, f.tiles, st, s);
  }
  auto run = [&](auto op) {
    op.mask1 = c.mask;
    op.r1 = c.r;
    op.r_out = r_out;
    op.e = e;
    op.ps = ps;
    op.partials = partials;
    op.nx = f.nx;
    op.ny = f.ny;
    op.ny1 = c.ny;
    op.nz1 = c.nz;
    return launch_tma<T>(op, maps, f.nx, f.ny, f.nz, f.tiles, st, s);
  };
  if (g_downu_blocks == 4) return run(TDownU4<T>{});
  return run(TDownU<T>{});
}

// The FP64 residual keeps the 8-warp column layout (no operand to share: x
// is read directly) on the same tiles as fine_grid (8 rows per CTA).
static_assert(TILE_ROWS == 8, "the residual and update kernels share fine_grid's tiles");
template <class T>
int launch_resid64_col(int nx, int ny, int nz, const uint8_t *mask, const uint8_t *tiles,
                       const float *div, const double *x, double bscale, T *rhat, float *e,
                       double *partials, const SolverState *st, bool write, cudaStream_t s) {
  const dim3 g = fine_grid(nx, ny, nz);
  const int bi = fine_bi(nx, ny, nz);
  if (write)
    resid64_col_kernel<T, true><<<g, 256, 0, s>>>(nx, ny, nz, bi, mask, tiles, div, x, bscale,
                                                  rhat, e, partials, st);
  else
    resid64_col_kernel<T, false><<<g, 256, 0, s>>>(nx, ny, nz, bi, mask, tiles, div, x, bscale,
                                                   rhat, e, partials, st);
  return (int)(g.x * g.y * g.z);
}

// e += alpha ps; r -= alpha Ap (r stored as T, read back rounded); partial
// r.r.  One warp per row of a fine_grid tile, float4 per lane, marching i.
// No mask: ps and Ap are zero on non-fluid cells, so e and r stay unchanged
// there; tiles without fluid are skipped.
template <class T>
__global__ void __launch_bounds__(256) cg_update_col_kernel(int nx, int ny, int nz, int bi,
                                                            const uint8_t *tiles, float *e, T *r,
                                                            const T *ps, const T *Ap,
                                                            double *partials,
                                                            const SolverState *st) {
  if (st->inner_done) return;
  if (tiles && !tiles[block_linear()]) {
    if (threadIdx.x == 0) partials[block_linear()] = 0.0;
    return;
  }
  __shared__ double sh[8];
  const float alpha = (float)st->alpha;
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
  const int k = (blockIdx.x * 32 + lane) * 4;
  double acc = 0.0;
  if (j < ny && k < nz) {
    const int i0 = blockIdx.z * bi, i1 = min(i0 + bi, nx);
    const int64_t plane = (int64_t)ny * nz;
    int64_t o = ((int64_t)i0 * ny + j) * nz + k;
#pragma unroll 4
    for (int i = i0; i < i1; ++i, o += plane) {
      float4 ee = *reinterpret_cast<const float4 *>(e + o);
      const float4 pp = ld4s(ps, o), aa = ld4s(Ap, o);
      float4 rr = ld4s(r, o);
      ee = make_float4(fmaf(alpha, pp.x, ee.x), fmaf(alpha, pp.y, ee.y), fmaf(alpha, pp.z, ee.z),
                       fmaf(alpha, pp.w, ee.w));
      rr = make_float4(rt(fmaf(-alpha, aa.x, rr.x), r), rt(fmaf(-alpha, aa.y, rr.y), r),
                       rt(fmaf(-alpha, aa.z, rr.z), r), rt(fmaf(-alpha, aa.w, rr.w), r));
      *reinterpret_cast<float4 *>(e + o) = ee;
      st4s(r, o, rr);
      acc += sq4w(rr);
    }
  }
  block_partial<8>(acc, partials, sh);
}

template <class T>
int launch_cg_update_col(int nx, int ny, int nz, const uint8_t *tiles, float *e, T *r,
                         const T *ps, const T *Ap, double *partials, const SolverState *st,
                         cudaStream_t s) {
  const dim3 g = fine_grid(nx, ny, nz);
  cg_update_col_kernel<T><<<g, 256, 0, s>>>(nx, ny, nz, fine_bi(nx, ny, nz), tiles, e, r, ps,
                                            Ap, partials, st);
  return (int)(g.x * g.y * g.z);
}

// flags[b] = 1 if tile b of fine_grid(nx, ny, nz) holds a fluid cell.
__global__ void __launch_bounds__(256) tile_flags_kernel(int nx, int ny, int nz, int bi,
                                                         const uint8_t *mask, uint8_t *flags) {
  const int i0 = blockIdx.z * bi, i1 = min(i0 + bi, nx);
  const int j0 = blockIdx.y * TILE_ROWS;
  const int k0 = blockIdx.x * 128;
  int any = 0;
  for (int t = threadIdx.x; t < (i1 - i0) * TILE_ROWS * 128; t += blockDim.x) {
    const int kk = k0 + t % 128, jj = j0 + (t / 128) % TILE_ROWS, ii = i0 + t / (128 * TILE_ROWS);
    if (jj < ny && kk < nz && (mask[((int64_t)ii * ny + jj) * nz + kk] & BSP_MFLUID)) any = 1;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) flags[block_linear()] = any ? 1 : 0;
}

void launch_tile_flags(int nx, int ny, int nz, const uint8_t *mask, uint8_t *flags,
                       cudaStream_t s) {
  tile_flags_kernel<<<fine_grid(nx, ny, nz), 256, 0, s>>>(nx, ny, nz, fine_bi(nx, ny, nz), mask,
                                                          flags);
}

#define INST(T)                                                                              \
  template int launch_resid64_col<T>(int, int, int, const uint8_t *, const uint8_t *,        \
                                     const float *, const double *, double, T *, float *,    \
                                     double *, const SolverState *, bool, cudaStream_t);     \
  template int launch_cg_update_col<T>(int, int, int, const uint8_t *, float *, T *,         \
                                       const T *, const T *, double *, const SolverState *,  \
                                       cudaStream_t);                                        \
  template void launch_fine_psap<T>(int, int, int, const uint8_t *, const uint8_t *,         \
                                    const T *, const T *, T *, T *, double *,                 \
                                    const SolverState *, cudaStream_t);                       \
  template void launch_fine_up<T>(const Level<T> &, const Level<T> &, T *, double *, float,   \
                                  const SolverState *, cudaStream_t);                         \
  template void launch_fine_down<T>(const Level<T> &, const Level<T> &, const SolverState *,  \
                                    cudaStream_t);                                              \
  template bool launch_fine_down_update<T>(const Level<T> &, const Level<T> &, T *, float *,   \
                                           const T *, const T *, double *, const SolverState *, \
                                           cudaStream_t, T *, const uint8_t *, const float *);  \
  template void launch_tri_setup<T>(uint8_t *, const Level<T> &, const Level<T> &,              \
                                    cudaStream_t);                                              \
  template void launch_tri_restrict<T>(const Level<T> &, const Level<T> &, const T *,           \
                                       const SolverState *, cudaStream_t);                      \
  template bool launch_fine_up_tri<T>(const Level<T> &, const Level<T> &, T *, double *, float, \
                                      const uint8_t *, const float *, const SolverState *,      \
                                      cudaStream_t);                                            \
  template bool launch_fine_smooth<T>(const Level<T> &, const T *, T *, const SolverState *,    \
                                      cudaStream_t);                                            \
  template bool launch_fine_down_e<T>(const Level<T> &, const Level<T> &, const T *,            \
                                      const SolverState *, cudaStream_t);                       \
  template bool launch_fine_up_e<T>(const Level<T> &, const Level<T> &, const T *, T *,         \
                                    double *, float, const SolverState *, cudaStream_t);
INST(float)
INST(__half)
INST(__nv_bfloat16)
#undef INST

}  // namespace bsp
