// mgcoarse.cu -- every coarse level of one V-cycle in one cooperative kernel.
//
// Below level 0 the grids are small (level 1 of the 384x384x256 pot is
// 4.7 M cells and L2-resident; level 3 is 74 K cells) and one kernel launch
// per level and direction costs more in launch and drain latency than the
// work itself.  mg_cycle_kernel runs the whole coarse part of the V-cycle --
// restriction from level 1 down to the coarsest level, the coarsest solve,
// prolongation back up to level 1 -- in one launch with one CTA per SM:
//
//   down:  D1   t = OMEGA r / D on level 1                   (fluid; 0 elsewhere)
//          per level l = 1 .. L-2:
//          D2a  res = r - (6 t - s(t))                        (fluid)
//          D2b  r[l+1] = 1/2 sum of the 2x2x2 children's res  (fluid coarse cells),
//               and t[l+1] = OMEGA r[l+1] / D in the same pass
//   coarsest level L-1:  e = M r, M the dense inverse (or 64 Jacobi sweeps)
//   up, level l = L-2 .. 1:
//          U1   t = OMEGA r / D + alpha e[l+1][parent]        (fluid)
//          U2   e = t + OMEGA (r - (6 t - s(t))) / D          (fluid; 0 elsewhere)
//
// with s(t) = sum of the six neighbours' t + n_solid x centre t (t is 0 on
// every non-fluid cell and outside the grid, which gives the reference's
// boundary rule: fluid -> value, air -> 0, solid -> centre value).  These are
// the operations of the level-0 kernels (mgfine.cu) and of the per-level row
// kernels (solver.cu).  Phases on levels with more than TAIL_CELLS cells are
// spread over the whole grid and separated by the bounded grid barrier; the
// small levels below run in CTA 0 alone with __syncthreads between phases,
// while the other CTAs wait at the next grid barrier.  Every phase works on
// quads of 4 consecutive k cells (vector loads, nz % 4 == 0 on every level);
// t and res live in an FP32 scratch vector.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "bsp_common.cuh"
#include "grid_sync.cuh"
#include "solver.cuh"
#include "tma.cuh"

namespace bsp {

constexpr int CC_THREADS = 1024;
constexpr int TAIL_CELLS = 16384;
constexpr float CC_OMEGA = 6.0f / 7.0f;
constexpr int CC_COARSE_SWEEPS = 64;
constexpr int CC_TRACE_MAX = 48;
// Phase-boundary stamps of the last traced coarse cycle (BSP_TUNE_COARSE_TRACE).
__device__ unsigned long long g_cc_trace[CC_TRACE_MAX];

__device__ __forceinline__ float cl(const float *p, int64_t c) { return p[c]; }
__device__ __forceinline__ float cl(const __half *p, int64_t c) { return __half2float(p[c]); }
__device__ __forceinline__ float cl(const __nv_bfloat16 *p, int64_t c) {
  return __bfloat162float(p[c]);
}
__device__ __forceinline__ void cs(float *p, int64_t c, float v) { p[c] = v; }
__device__ __forceinline__ void cs(__half *p, int64_t c, float v) { p[c] = __float2half_rn(v); }
__device__ __forceinline__ void cs(__nv_bfloat16 *p, int64_t c, float v) {
  p[c] = __float2bfloat16_rn(v);
}
// value as it reads back after a store through T
__device__ __forceinline__ float cl_round(float v, const float *) { return v; }
__device__ __forceinline__ float cl_round(float v, const __half *) {
  return __half2float(__float2half_rn(v));
}
__device__ __forceinline__ float cl_round(float v, const __nv_bfloat16 *) {
  return __bfloat162float(__float2bfloat16_rn(v));
}

template <class T>
struct CoarseCycle {
  Level<T> lv[MAX_LEVELS];
  int L;
  float *scratch;     // FP32 t, >= max(cells of level 1, 3 x cells of the coarsest level)
  float *res;         // FP32 residuals of the restriction, >= cells of level 1
  const float *cinv;  // coarsest dense inverse, symmetric, n x n
  const int *cflag;   // 1: cinv valid
  GridCtl *ctl;
  float alpha;
  int fused_phases;   // 1: t formed where it is read (fewer phases and grid barriers)
  unsigned long long *trace;  // optional: CTA 0's %globaltimer at each phase boundary
  int cinv_bytes;     // > 0: CTA 0 copies the dense inverse into shared memory at launch
  int tail_smem;      // 1: the levels CTA 0 runs alone live in its shared memory
  int tail_off;       // byte offset of that region in the dynamic shared memory
  int tail_cells;     // cluster kernel: levels of at most this many cells run in CTA 0
};

// Dynamic shared memory of the coarse-cycle kernel: [dense inverse (CTA 0)]
// [coarsest right-hand side, FP32] [mbarrier of the inverse's bulk copy].
__device__ __forceinline__ float *cc_smem() {
  extern __shared__ __align__(16) float cc_dyn[];
  return cc_dyn;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

struct Span {  // the warps that share a phase: warp w0 of nw
  int w0, nw;
};

// OMEGA / (6 - n_solid) of a mask byte (0 when no neighbour is non-solid).
__device__ __forceinline__ float cc_w(const float *wtab, uint32_t m) { return wtab[m & 7u]; }
__device__ __forceinline__ float f4(const float4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}
__device__ __forceinline__ float4 ld4f(const float *p, int64_t c) {
  return *reinterpret_cast<const float4 *>(p + c);
}
__device__ __forceinline__ void st4f(float *p, int64_t c, float4 v) {
  *reinterpret_cast<float4 *>(p + c) = v;
}
__device__ __forceinline__ float4 ld4t(const float *p, int64_t c) { return ld4f(p, c); }
__device__ __forceinline__ float4 ld4t(const __half *p, int64_t c) {
  const uint2 u = *reinterpret_cast<const uint2 *>(p + c);
  const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 ld4t(const __nv_bfloat16 *p, int64_t c) {
  const uint2 u = *reinterpret_cast<const uint2 *>(p + c);
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
// Stores 4 values through T and returns them as they read back.
template <class T>
__device__ __forceinline__ float4 st4t(T *p, int64_t c, float4 v) {
  cs(p, c, v.x);
  cs(p, c + 1, v.y);
  cs(p, c + 2, v.z);
  cs(p, c + 3, v.w);
  return make_float4(cl_round(v.x, p), cl_round(v.y, p), cl_round(v.z, p), cl_round(v.w, p));
}
// Mask loads are plain (generic) loads: the small levels may live in shared
// memory (the tail staged by CTA 0), where the read-only global path cannot go.
__device__ __forceinline__ uint32_t ldm4(const uint8_t *m, int64_t c) {
  return *reinterpret_cast<const uint32_t *>(m + c);
}
__device__ __forceinline__ float fl_mask(float v, uint32_t mw, int q) {
  return ((mw >> (8 * q)) & BSP_MFLUID) ? v : 0.0f;
}

// Calls fn(i, j, k, c) for every quad (4 consecutive k cells, k % 4 == 0) of an
// (nx, ny, nz) grid with nz % 4 == 0, spread over the span's warps: a warp
// covers 32 / (nz/4) rows at a time when a row has fewer than 32 quads.
template <class Fn>
__device__ __forceinline__ void for_quads(int nx, int ny, int nz, Span sp, Fn fn) {
  const int lane = threadIdx.x & 31;
  const int nzq = nz >> 2;
  const int rows = nx * ny;
  if (nzq >= 32) {
    for (int row = sp.w0; row < rows; row += sp.nw) {
      const int i = row / ny, j = row - i * ny;
      for (int kq = lane; kq < nzq; kq += 32) fn(i, j, 4 * kq, (int64_t)row * nz + 4 * kq);
    }
    return;
  }
  const int rpw = 32 / nzq, sub = lane / nzq, kq = lane - sub * nzq;
  if (sub >= rpw) return;
#pragma unroll 2
  for (int row0 = sp.w0 * rpw; row0 < rows; row0 += sp.nw * rpw) {
    const int row = row0 + sub;
    if (row < rows) {
      const int i = row / ny, j = row - i * ny;
      fn(i, j, 4 * kq, (int64_t)row * nz + 4 * kq);
    }
  }
}

// Centre t and neighbour sum (without the n_solid term) of the 4 cells of a quad.
template <class T>
__device__ __forceinline__ void quad_nbr(const float *__restrict__ t, const Level<T> &f, int i,
                                         int j, int k, int64_t c, float4 &tc, float (&s)[4]) {
  const int64_t plane = (int64_t)f.ny * f.nz;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  tc = ld4f(t, c);
  const float4 a = i > 0 ? ld4f(t, c - plane) : z4;
  const float4 b = i + 1 < f.nx ? ld4f(t, c + plane) : z4;
  const float4 d = j > 0 ? ld4f(t, c - f.nz) : z4;
  const float4 u = j + 1 < f.ny ? ld4f(t, c + f.nz) : z4;
  const float km = k > 0 ? t[c - 1] : 0.0f;
  const float kp = k + 4 < f.nz ? t[c + 4] : 0.0f;
  const float4 lo = make_float4(km, tc.x, tc.y, tc.z), hi = make_float4(tc.y, tc.z, tc.w, kp);
#pragma unroll
  for (int q = 0; q < 4; ++q)
    s[q] = ((f4(a, q) + f4(b, q)) + (f4(d, q) + f4(u, q))) + (f4(lo, q) + f4(hi, q));
}

// D1: t = OMEGA r / D on fluid cells.
template <class T>
__device__ void phase_d1(const Level<T> &f, float *__restrict__ t, const float *wtab, Span sp) {
  for_quads(f.nx, f.ny, f.nz, sp, [&](int, int, int, int64_t c) {
    const uint32_t m = ldm4(f.mask, c);
    const float4 r = ld4t(f.r, c);
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = fl_mask(f4(r, q) * cc_w(wtab, m >> (8 * q)), m, q);
    st4f(t, c, make_float4(v[0], v[1], v[2], v[3]));
  });
}

// D2a: res = r - (6 t - s(t)) on fluid cells.
template <class T>
__device__ void phase_d2a(const Level<T> &f, const float *__restrict__ t, float *__restrict__ res,
                          Span sp) {
  for_quads(f.nx, f.ny, f.nz, sp, [&](int i, int j, int k, int64_t c) {
    const uint32_t m = ldm4(f.mask, c);
    const float4 r = ld4t(f.r, c);
    float4 tc;
    float s[4];
    quad_nbr(t, f, i, j, k, c, tc, s);
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float sq = fmaf((float)((m >> (8 * q)) & 7u), f4(tc, q), s[q]);
      v[q] = fl_mask(f4(r, q) - (6.0f * f4(tc, q) - sq), m, q);
    }
    st4f(res, c, make_float4(v[0], v[1], v[2], v[3]));
  });
}

// D2b: r[l+1] = 1/2 sum of the 2x2x2 children's res (fluid coarse cells), and
// the next level's D1, t[l+1] = OMEGA r[l+1] / D, in the same pass.
template <class T>
__device__ void phase_d2b(const Level<T> &f, const Level<T> &co, const float *__restrict__ res,
                          float *__restrict__ t, const float *wtab, Span sp) {
  for_quads(co.nx, co.ny, co.nz, sp, [&](int I, int J, int K, int64_t C) {
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int i = 2 * I + a, j = 2 * J + b;
        if (i < f.nx && j < f.ny) {
          const int64_t c = ((int64_t)i * f.ny + j) * f.nz + 2 * K;
          const float4 p = ld4f(res, c), q = ld4f(res, c + 4);
          acc[0] += p.x + p.y;
          acc[1] += p.z + p.w;
          acc[2] += q.x + q.y;
          acc[3] += q.z + q.w;
        }
      }
    const uint32_t m = ldm4(co.mask, C);
    float rv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) rv[q] = fl_mask(0.5f * acc[q], m, q);
    const float4 stored = st4t(co.r, C, make_float4(rv[0], rv[1], rv[2], rv[3]));
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = f4(stored, q) * cc_w(wtab, m >> (8 * q));
    st4f(t, C, make_float4(v[0], v[1], v[2], v[3]));
  });
}

// U1: t = OMEGA r / D + alpha e[l+1][parent] on fluid cells.
template <class T>
__device__ void phase_u1(const Level<T> &f, const Level<T> &co, float *__restrict__ t,
                         const float *wtab, float alpha, Span sp) {
  for_quads(f.nx, f.ny, f.nz, sp, [&](int i, int j, int k, int64_t c) {
    const uint32_t m = ldm4(f.mask, c);
    const float4 r = ld4t(f.r, c);
    const int64_t P = ((int64_t)(i >> 1) * co.ny + (j >> 1)) * co.nz + (k >> 1);
    const float e0 = alpha * cl(co.e, P), e1 = alpha * cl(co.e, P + 1);
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      v[q] = fl_mask(fmaf(f4(r, q), cc_w(wtab, m >> (8 * q)), q < 2 ? e0 : e1), m, q);
    st4f(t, c, make_float4(v[0], v[1], v[2], v[3]));
  });
}

// U2: e = t + OMEGA (r - (6 t - s(t))) / D on fluid cells, 0 elsewhere.
template <class T>
__device__ void phase_u2(const Level<T> &f, const float *__restrict__ t, const float *wtab,
                         Span sp) {
  for_quads(f.nx, f.ny, f.nz, sp, [&](int i, int j, int k, int64_t c) {
    const uint32_t m = ldm4(f.mask, c);
    const float4 r = ld4t(f.r, c);
    float4 tc;
    float s[4];
    quad_nbr(t, f, i, j, k, c, tc, s);
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float sq = fmaf((float)((m >> (8 * q)) & 7u), f4(tc, q), s[q]);
      v[q] = fl_mask(fmaf(f4(r, q) - (6.0f * f4(tc, q) - sq), cc_w(wtab, m >> (8 * q)),
                          f4(tc, q)),
                     m, q);
    }
    st4t(f.e, c, make_float4(v[0], v[1], v[2], v[3]));
  });
}

// ---- fused phases: t is recomputed where it is read instead of stored --------------
// D1 and U1 are pointwise, so the phase after each (D2a, U2) can form t at the
// centre and at every neighbour itself; this removes a grid-wide phase, its
// barrier and the t round trip through memory per level and direction, with
// the same floating-point operations (bit-identical results).

// t = OMEGA r / D (D1) of the 4 cells of quad c; 0 off fluid.
template <class T>
__device__ __forceinline__ float4 t_down4(const Level<T> &f, int64_t c, const float *wtab) {
  const uint32_t m = ldm4(f.mask, c);
  const float4 r = ld4t(f.r, c);
  float v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) v[q] = fl_mask(f4(r, q) * cc_w(wtab, m >> (8 * q)), m, q);
  return make_float4(v[0], v[1], v[2], v[3]);
}
template <class T>
__device__ __forceinline__ float t_down1(const Level<T> &f, int64_t c, const float *wtab) {
  const uint32_t m = f.mask[c];
  return (m & BSP_MFLUID) ? cl(f.r, c) * cc_w(wtab, m) : 0.0f;
}
// t = OMEGA r / D + alpha e[l+1][parent] (U1) of the quad at (i, j, k); 0 off fluid.
template <class T>
__device__ __forceinline__ float4 t_up4(const Level<T> &f, const Level<T> &co, int i, int j,
                                        int k, int64_t c, const float *wtab, float alpha) {
  const uint32_t m = ldm4(f.mask, c);
  const float4 r = ld4t(f.r, c);
  const int64_t P = ((int64_t)(i >> 1) * co.ny + (j >> 1)) * co.nz + (k >> 1);
  const float e0 = alpha * cl(co.e, P), e1 = alpha * cl(co.e, P + 1);
  float v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q)
    v[q] = fl_mask(fmaf(f4(r, q), cc_w(wtab, m >> (8 * q)), q < 2 ? e0 : e1), m, q);
  return make_float4(v[0], v[1], v[2], v[3]);
}
template <class T>
__device__ __forceinline__ float t_up1(const Level<T> &f, const Level<T> &co, int i, int j, int k,
                                       int64_t c, const float *wtab, float alpha) {
  const uint32_t m = f.mask[c];
  if (!(m & BSP_MFLUID)) return 0.0f;
  const int64_t P = ((int64_t)(i >> 1) * co.ny + (j >> 1)) * co.nz + (k >> 1);
  return fmaf(cl(f.r, c), cc_w(wtab, m), alpha * cl(co.e, P));
}

// D1 + D2a: res = r - (6 t - s(t)) with t = OMEGA r / D formed on the fly.
template <class T>
__device__ __forceinline__ void phase_down_fused(const Level<T> &f, float *__restrict__ res, const float *wtab,
                                 Span sp) {
  for_quads(f.nx, f.ny, f.nz, sp, [&](int i, int j, int k, int64_t c) {
    const int64_t plane = (int64_t)f.ny * f.nz;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    // neighbour pairs summed as soon as both are known (the same sums as
    // ((a + b) + (d + u)) + (lo + hi), fewer live registers)
    float4 ab, du;
    {
      const float4 a = i > 0 ? t_down4(f, c - plane, wtab) : z4;
      const float4 b = i + 1 < f.nx ? t_down4(f, c + plane, wtab) : z4;
      ab = make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
    }
    {
      const float4 d = j > 0 ? t_down4(f, c - f.nz, wtab) : z4;
      const float4 u = j + 1 < f.ny ? t_down4(f, c + f.nz, wtab) : z4;
      du = make_float4(d.x + u.x, d.y + u.y, d.z + u.z, d.w + u.w);
    }
    const float km = k > 0 ? t_down1(f, c - 1, wtab) : 0.0f;
    const float kp = k + 4 < f.nz ? t_down1(f, c + 4, wtab) : 0.0f;
    const uint32_t m = ldm4(f.mask, c);
    const float4 r = ld4t(f.r, c);
    const float4 tc = t_down4(f, c, wtab);
    const float4 lo = make_float4(km, tc.x, tc.y, tc.z), hi = make_float4(tc.y, tc.z, tc.w, kp);
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float s = (f4(ab, q) + f4(du, q)) + (f4(lo, q) + f4(hi, q));
      const float sq = fmaf((float)((m >> (8 * q)) & 7u), f4(tc, q), s);
      v[q] = fl_mask(f4(r, q) - (6.0f * f4(tc, q) - sq), m, q);
    }
    st4f(res, c, make_float4(v[0], v[1], v[2], v[3]));
  });
}

// D2b without the next level's t (the next down phase forms it itself).
template <class T>
__device__ __forceinline__ void phase_restrict(const Level<T> &f, const Level<T> &co, const float *__restrict__ res,
                               Span sp) {
  for_quads(co.nx, co.ny, co.nz, sp, [&](int I, int J, int K, int64_t C) {
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int i = 2 * I + a, j = 2 * J + b;
        if (i < f.nx && j < f.ny) {
          const int64_t c = ((int64_t)i * f.ny + j) * f.nz + 2 * K;
          const float4 p = ld4f(res, c), q = ld4f(res, c + 4);
          acc[0] += p.x + p.y;
          acc[1] += p.z + p.w;
          acc[2] += q.x + q.y;
          acc[3] += q.z + q.w;
        }
      }
    const uint32_t m = ldm4(co.mask, C);
    float rv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) rv[q] = fl_mask(0.5f * acc[q], m, q);
    st4t(co.r, C, make_float4(rv[0], rv[1], rv[2], rv[3]));
  });
}

// U1 + U2: e = t + OMEGA (r - (6 t - s(t))) / D with t = OMEGA r / D +
// alpha e[l+1][parent] formed on the fly.
template <class T>
__device__ __forceinline__ void phase_up_fused(const Level<T> &f, const Level<T> &co, const float *wtab,
                               float alpha, Span sp) {
  for_quads(f.nx, f.ny, f.nz, sp, [&](int i, int j, int k, int64_t c) {
    const int64_t plane = (int64_t)f.ny * f.nz;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 ab, du;
    {
      const float4 a = i > 0 ? t_up4(f, co, i - 1, j, k, c - plane, wtab, alpha) : z4;
      const float4 b = i + 1 < f.nx ? t_up4(f, co, i + 1, j, k, c + plane, wtab, alpha) : z4;
      ab = make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
    }
    {
      const float4 d = j > 0 ? t_up4(f, co, i, j - 1, k, c - f.nz, wtab, alpha) : z4;
      const float4 u = j + 1 < f.ny ? t_up4(f, co, i, j + 1, k, c + f.nz, wtab, alpha) : z4;
      du = make_float4(d.x + u.x, d.y + u.y, d.z + u.z, d.w + u.w);
    }
    const float km = k > 0 ? t_up1(f, co, i, j, k - 1, c - 1, wtab, alpha) : 0.0f;
    const float kp = k + 4 < f.nz ? t_up1(f, co, i, j, k + 4, c + 4, wtab, alpha) : 0.0f;
    const uint32_t m = ldm4(f.mask, c);
    const float4 r = ld4t(f.r, c);
    const float4 tc = t_up4(f, co, i, j, k, c, wtab, alpha);
    const float4 lo = make_float4(km, tc.x, tc.y, tc.z), hi = make_float4(tc.y, tc.z, tc.w, kp);
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float s = (f4(ab, q) + f4(du, q)) + (f4(lo, q) + f4(hi, q));
      const float sq = fmaf((float)((m >> (8 * q)) & 7u), f4(tc, q), s);
      v[q] = fl_mask(fmaf(f4(r, q) - (6.0f * f4(tc, q) - sq), cc_w(wtab, m >> (8 * q)),
                          f4(tc, q)),
                     m, q);
    }
    st4t(f.e, c, make_float4(v[0], v[1], v[2], v[3]));
  });
}

// Scalar neighbour sum for the coarsest-level sweeps.
template <class T>
__device__ __forceinline__ float nbr_sum1(const float *t, const Level<T> &f, int i, int j, int k,
                                          int c) {
  const int plane = f.ny * f.nz;
  const float a = i > 0 ? t[c - plane] : 0.0f;
  const float b = i + 1 < f.nx ? t[c + plane] : 0.0f;
  const float d = j > 0 ? t[c - f.nz] : 0.0f;
  const float u = j + 1 < f.ny ? t[c + f.nz] : 0.0f;
  const float bk = k > 0 ? t[c - 1] : 0.0f;
  const float fk = k + 1 < f.nz ? t[c + 1] : 0.0f;
  return ((a + b) + (d + u)) + (bk + fk);
}

// Coarsest level, by CTA 0: e = M r with the symmetric dense inverse (warp per
// output, lanes over the sum, fixed shuffle order), or, without one, damped
// Jacobi sweeps from zero in the scratch vector.
template <class T>
__device__ void coarsest_solve(const CoarseCycle<T> &a, const Level<T> &c, const float *wtab,
                               const float *minv) {
  const int n = c.nx * c.ny * c.nz;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (*a.cflag) {
    // e = M r; r staged in shared memory, M read from shared memory when it
    // was copied there at launch (minv), else from global memory
    float *rs = cc_smem() + (a.cinv_bytes >> 2);
    for (int q = threadIdx.x; q < n; q += blockDim.x) rs[q] = cl(c.r, q);
    __syncthreads();
    for (int o = warp; o < n; o += nw) {
      float acc = 0.0f;
      const float *row = minv + (int64_t)o * n;
#pragma unroll 4
      for (int q = lane; q < n; q += 32) acc = fmaf(row[q], rs[q], acc);
      for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
      if (lane == 0) cs(c.e, o, (c.mask[o] & BSP_MFLUID) ? acc : 0.0f);
    }
    return;
  }
  float *e0 = a.scratch, *e1 = a.scratch + n;
  for (int q = threadIdx.x; q < n; q += blockDim.x) e0[q] = 0.0f;
  __syncthreads();
  for (int sw = 0; sw < CC_COARSE_SWEEPS; ++sw) {
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
      const uint32_t m = c.mask[q];
      float v = 0.0f;
      if (m & BSP_MFLUID) {
        const int k = q % c.nz, j = (q / c.nz) % c.ny, i = q / (c.nz * c.ny);
        const float ec = e0[q];
        const float s = fmaf((float)(m & 7u), ec, nbr_sum1(e0, c, i, j, k, q));
        v = fmaf(cl(c.r, q) - (6.0f * ec - s), cc_w(wtab, m), ec);
      }
      e1[q] = v;
    }
    __syncthreads();
    float *tmp = e0;
    e0 = e1;
    e1 = tmp;
  }
  for (int q = threadIdx.x; q < n; q += blockDim.x) cs(c.e, q, e0[q]);
}

template <class T>
__global__ void __launch_bounds__(CC_THREADS, 1) mg_cycle_kernel(CoarseCycle<T> a,
                                                                 SolverState *st) {
  if (st->inner_done) return;  // uniform over the grid
  __shared__ float wtab[8];
  if (threadIdx.x < 8) {
    const float d = 6.0f - (float)threadIdx.x;
    wtab[threadIdx.x] = d > 0.0f ? __fdividef(CC_OMEGA, d) : 0.0f;
  }
  __syncthreads();
  const int wpb = blockDim.x >> 5;
  const Span all{(int)(blockIdx.x * wpb + (threadIdx.x >> 5)), (int)(gridDim.x * wpb)};
  const Span one{(int)(threadIdx.x >> 5), wpb};
  const int L = a.L;
  auto cells = [&](int l) { return (int64_t)a.lv[l].nx * a.lv[l].ny * a.lv[l].nz; };
  // levels >= tail run in CTA 0 alone
  int tail = 1;
  while (tail < L && cells(tail) > TAIL_CELLS) ++tail;
  // CTA 0 fetches the coarsest level's dense inverse into shared memory while
  // the grid works on the big levels (one bulk copy, bounded wait before use)
  uint64_t *cbar = reinterpret_cast<uint64_t *>(cc_smem() + (a.cinv_bytes >> 2) +
                                                ((a.cinv_bytes > 0) ? COARSEST_CELLS : 0));
  const bool cinv_copy = a.cinv_bytes > 0 && blockIdx.x == 0;
  bool cinv_waited = false;
  if (cinv_copy && threadIdx.x == 0) {
    mbar_init(cbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_expect_tx(cbar, (uint32_t)a.cinv_bytes);
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(smem_u32(cc_smem())),
        "l"(a.cinv), "r"((uint32_t)a.cinv_bytes), "r"(smem_u32(cbar))
        : "memory");
  }
  bool ok = true;
  int nmark = 0;
  auto mark = [&]() {  // tracing: CTA 0 stamps each phase boundary
    if (a.trace && blockIdx.x == 0 && threadIdx.x == 0 && nmark < CC_TRACE_MAX)
      a.trace[nmark++] = global_ns();
  };
  auto sync_all = [&]() {
    if (ok && !grid_barrier(a.ctl)) ok = false;
    mark();
  };
  mark();
  if (a.fused_phases) {
    // ---- down: per level the residual (t formed on the fly) and the restriction
    for (int l = 1; l + 1 < L && ok; ++l) {
      if (l < tail) {
        phase_down_fused(a.lv[l], a.res, wtab, all);
        sync_all();
        phase_restrict(a.lv[l], a.lv[l + 1], a.res, all);
        sync_all();
      } else if (blockIdx.x == 0) {
        phase_down_fused(a.lv[l], a.res, wtab, one);
        __syncthreads();
        phase_restrict(a.lv[l], a.lv[l + 1], a.res, one);
        __syncthreads();
        mark();
      }
    }
    if (blockIdx.x == 0 && ok) {
      const float *minv = a.cinv;
      if (cinv_copy) {
        __shared__ int s_cok;
        if (threadIdx.x == 0) s_cok = mbar_wait(cbar, 0) ? 1 : 0;
        __syncthreads();
        cinv_waited = true;
        if (s_cok) minv = cc_smem();
        else ok = false;
      }
      if (ok) coarsest_solve(a, a.lv[L - 1], wtab, minv);
      __syncthreads();
      mark();
      for (int l = L - 2; l >= tail && l >= 1 && ok; --l) {
        phase_up_fused(a.lv[l], a.lv[l + 1], wtab, a.alpha, one);
        __syncthreads();
        mark();
      }
    }
    const int top = min(tail, L - 1) - 1;
    if (top >= 1) sync_all();
    for (int l = top; l >= 1 && ok; --l) {
      phase_up_fused(a.lv[l], a.lv[l + 1], wtab, a.alpha, all);
      if (l > 1) sync_all();
    }
    mark();
  } else {
  // ---- down: t of level 1, then per level the residual pass and the
  // restriction (which also forms t of the next level)
  if (L > 2) {
    if (1 < tail) {
      phase_d1(a.lv[1], a.scratch, wtab, all);
      sync_all();
    } else if (blockIdx.x == 0) {
      phase_d1(a.lv[1], a.scratch, wtab, one);
      __syncthreads();
    }
  }
  for (int l = 1; l + 1 < L && ok; ++l) {
    if (l < tail) {
      phase_d2a(a.lv[l], a.scratch, a.res, all);
      sync_all();
      phase_d2b(a.lv[l], a.lv[l + 1], a.res, a.scratch, wtab, all);
      sync_all();
    } else if (blockIdx.x == 0 && !a.tail_smem) {
      phase_d2a(a.lv[l], a.scratch, a.res, one);
      __syncthreads();
      phase_d2b(a.lv[l], a.lv[l + 1], a.res, a.scratch, wtab, one);
      __syncthreads();
    }
  }
  if (blockIdx.x == 0 && ok) {
    const float *minv = a.cinv;
    if (cinv_copy) {
      __shared__ int s_cok2;
      if (threadIdx.x == 0) s_cok2 = mbar_wait(cbar, 0) ? 1 : 0;
      __syncthreads();
      cinv_waited = true;
      if (s_cok2) minv = cc_smem();
      else ok = false;
    }
    if (ok && a.tail_smem) {
      // The small levels in shared memory: masks and the tail level's
      // right-hand side copied in, every phase of the tail on-chip, the tail
      // level's correction copied back out for the big levels' up phases.
      Level<T> sv[MAX_LEVELS];
      unsigned char *sp = reinterpret_cast<unsigned char *>(cc_smem()) + a.tail_off;
      auto take = [&](int64_t b) {
        unsigned char *q = sp;
        sp += (b + 15) / 16 * 16;
        return q;
      };
      for (int l = tail; l < L; ++l) {
        const int64_t nl = cells(l);
        sv[l] = a.lv[l];
        sv[l].mask = take(nl);
        sv[l].r = reinterpret_cast<T *>(take(nl * (int64_t)sizeof(T)));
        sv[l].e = reinterpret_cast<T *>(take(nl * (int64_t)sizeof(T)));
        const uint32_t *gm = reinterpret_cast<const uint32_t *>(a.lv[l].mask);
        uint32_t *smk = reinterpret_cast<uint32_t *>(const_cast<uint8_t *>(sv[l].mask));
        for (int64_t q = threadIdx.x; q < nl / 4; q += blockDim.x) smk[q] = gm[q];
      }
      float *ts = reinterpret_cast<float *>(take(cells(tail) * 4));
      float *rs = reinterpret_cast<float *>(take(cells(tail) * 4));
      {
        const int64_t nb = cells(tail) * (int64_t)sizeof(T) / 8;  // 8-byte words
        const uint2 *g = reinterpret_cast<const uint2 *>(a.lv[tail].r);
        uint2 *d = reinterpret_cast<uint2 *>(sv[tail].r);
        for (int64_t q = threadIdx.x; q < nb; q += blockDim.x) d[q] = g[q];
      }
      __syncthreads();
      mark();
      if (tail + 1 < L) {
        phase_d1(sv[tail], ts, wtab, one);
        __syncthreads();
      }
      for (int l = tail; l + 1 < L; ++l) {
        phase_d2a(sv[l], ts, rs, one);
        __syncthreads();
        phase_d2b(sv[l], sv[l + 1], rs, ts, wtab, one);
        __syncthreads();
      }
      mark();
      coarsest_solve(a, sv[L - 1], wtab, minv);
      __syncthreads();
      mark();
      for (int l = L - 2; l >= tail; --l) {
        phase_u1(sv[l], sv[l + 1], ts, wtab, a.alpha, one);
        __syncthreads();
        phase_u2(sv[l], ts, wtab, one);
        __syncthreads();
      }
      {
        const int64_t nb = cells(tail) * (int64_t)sizeof(T) / 8;
        const uint2 *g = reinterpret_cast<const uint2 *>(sv[tail].e);
        uint2 *d = reinterpret_cast<uint2 *>(a.lv[tail].e);
        for (int64_t q = threadIdx.x; q < nb; q += blockDim.x) d[q] = g[q];
      }
      __threadfence();
      __syncthreads();
      mark();
    } else {
      if (ok) coarsest_solve(a, a.lv[L - 1], wtab, minv);
      __syncthreads();
      for (int l = L - 2; l >= tail && l >= 1; --l) {
        phase_u1(a.lv[l], a.lv[l + 1], a.scratch, wtab, a.alpha, one);
        __syncthreads();
        phase_u2(a.lv[l], a.scratch, wtab, one);
        __syncthreads();
      }
    }
  }
  // ---- up through the big levels
  const int top = min(tail, L - 1) - 1;  // highest-index big level still to prolongate
  if (top >= 1) sync_all();
  for (int l = top; l >= 1 && ok; --l) {
    phase_u1(a.lv[l], a.lv[l + 1], a.scratch, wtab, a.alpha, all);
    sync_all();
    phase_u2(a.lv[l], a.scratch, wtab, all);
    if (l > 1) sync_all();
  }
  }
  // the bulk copy must have landed before CTA 0's shared memory goes away
  if (cinv_copy && !cinv_waited && threadIdx.x == 0) mbar_wait(cbar, 0);
  if (!ok && threadIdx.x == 0) atomicExch(&st->dev_error, 1);
}

// ---- the coarse cycle in one thread-block cluster ----------------------------------
// The stored-t phases of mg_cycle_kernel spread over the CTAs of ONE cluster
// (BSP_TUNE_COARSE_CLUSTER CTAs, one per SM) and separated by the hardware
// cluster barrier -- arrive with release, wait with acquire semantics at
// cluster scope, so one phase's global stores are visible to every CTA of the
// cluster in the next -- instead of the software barrier over all SMs.  The
// levels below the cycle's top level are L2-resident and their phases bound
// by load latency, not by the number of SMs; a cluster barrier costs a
// fraction of a grid-wide one.  Levels of at most CL_TAIL_CELLS cells run in
// the cluster's CTA 0 alone with __syncthreads; the coarsest solve uses the
// dense inverse copied into CTA 0's shared memory at launch.  A cluster's CTAs
// are co-scheduled by the hardware: no spin wait.
// default of BSP_TUNE_CLUSTER_TAIL_CELLS.  With levels 1-3 on the tile kernels
// the cycle's levels hold 9,216 cells and fewer at 384x384x256, and CTA 0 alone
// runs them faster than the cluster with its barriers: 11.61 ms per solve at
// 2048, 11.52 at 16384 (0, every level cluster-wide: 11.66).
constexpr int CL_TAIL_CELLS = 16384;
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_ctas() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}

template <class T>
__global__ void __launch_bounds__(CC_THREADS, 1) mg_cluster_cycle_kernel(CoarseCycle<T> a,
                                                                         SolverState *st) {
  if (st->inner_done) return;  // uniform over the cluster
  __shared__ float wtab[8];
  if (threadIdx.x < 8) {
    const float d = 6.0f - (float)threadIdx.x;
    wtab[threadIdx.x] = d > 0.0f ? __fdividef(CC_OMEGA, d) : 0.0f;
  }
  __syncthreads();
  const int rank = (int)cluster_rank(), nct = (int)cluster_ctas();
  const int wpb = blockDim.x >> 5;
  const Span all{rank * wpb + (int)(threadIdx.x >> 5), nct * wpb};
  const Span one{(int)(threadIdx.x >> 5), wpb};
  const bool lead = rank == 0;
  const int L = a.L;
  auto cells = [&](int l) { return (int64_t)a.lv[l].nx * a.lv[l].ny * a.lv[l].nz; };
  int tail = 1;  // levels >= tail run in CTA 0 of the cluster alone
  while (tail < L && cells(tail) > a.tail_cells) ++tail;
  uint64_t *cbar = reinterpret_cast<uint64_t *>(cc_smem() + (a.cinv_bytes >> 2) +
                                                ((a.cinv_bytes > 0) ? COARSEST_CELLS : 0));
  const bool cinv_copy = a.cinv_bytes > 0 && lead;
  bool cinv_waited = false;
  if (cinv_copy && threadIdx.x == 0) {
    mbar_init(cbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_expect_tx(cbar, (uint32_t)a.cinv_bytes);
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(smem_u32(cc_smem())),
        "l"(a.cinv), "r"((uint32_t)a.cinv_bytes), "r"(smem_u32(cbar))
        : "memory");
  }
  bool ok = true;
  int nmark = 0;
  auto mark = [&]() {
    if (a.trace && lead && threadIdx.x == 0 && nmark < CC_TRACE_MAX)
      a.trace[nmark++] = global_ns();
  };
  auto csync = [&]() {
    cluster_sync_all();
    mark();
  };
  mark();
  // ---- down: t of the cycle's first level, then per level the residual pass
  // and the restriction (which also forms t of the next level)
  if (L > 2) {
    if (1 < tail) {
      phase_d1(a.lv[1], a.scratch, wtab, all);
      csync();
    } else if (lead) {
      phase_d1(a.lv[1], a.scratch, wtab, one);
      __syncthreads();
    }
  }
  for (int l = 1; l + 1 < L && l < tail; ++l) {
    phase_d2a(a.lv[l], a.scratch, a.res, all);
    csync();
    phase_d2b(a.lv[l], a.lv[l + 1], a.res, a.scratch, wtab, all);
    csync();
  }
  if (lead) {
    const float *minv = a.cinv;
    if (cinv_copy) {
      __shared__ int s_cok;
      if (threadIdx.x == 0) s_cok = mbar_wait(cbar, 0) ? 1 : 0;
      __syncthreads();
      cinv_waited = true;
      if (s_cok) minv = cc_smem();
      else ok = false;
    }
    if (a.tail_smem && tail < L) {
      // The tail levels in shared memory: masks and the first tail level's
      // right-hand side and t copied in (its down phases ran above: the
      // restriction into it left r and t in global memory), the rest of the
      // tail on-chip, the first tail level's correction copied back out.
      Level<T> sv[MAX_LEVELS];
      unsigned char *sp = reinterpret_cast<unsigned char *>(cc_smem()) + a.tail_off;
      auto take = [&](int64_t b) {
        unsigned char *q = sp;
        sp += (b + 15) / 16 * 16;
        return q;
      };
      for (int l = tail; l < L; ++l) {
        const int64_t nl = cells(l);
        sv[l] = a.lv[l];
        sv[l].mask = take(nl);
        sv[l].r = reinterpret_cast<T *>(take(nl * (int64_t)sizeof(T)));
        sv[l].e = reinterpret_cast<T *>(take(nl * (int64_t)sizeof(T)));
        const uint32_t *gm = reinterpret_cast<const uint32_t *>(a.lv[l].mask);
        uint32_t *smk = reinterpret_cast<uint32_t *>(const_cast<uint8_t *>(sv[l].mask));
        for (int64_t q = threadIdx.x; q < nl / 4; q += blockDim.x) smk[q] = gm[q];
      }
      const int64_t nt = cells(tail);
      float *ts = reinterpret_cast<float *>(take(nt * 4));
      float *rs = reinterpret_cast<float *>(take(nt * 4));
      {
        const int64_t nb = nt * (int64_t)sizeof(T) / 8;  // 8-byte words
        const uint2 *g = reinterpret_cast<const uint2 *>(a.lv[tail].r);
        uint2 *d = reinterpret_cast<uint2 *>(sv[tail].r);
        for (int64_t q = threadIdx.x; q < nb; q += blockDim.x) d[q] = g[q];
        const float4 *gt = reinterpret_cast<const float4 *>(a.scratch);
        float4 *dt = reinterpret_cast<float4 *>(ts);
        for (int64_t q = threadIdx.x; q < nt / 4; q += blockDim.x) dt[q] = gt[q];
      }
      __syncthreads();
      for (int l = tail; l + 1 < L; ++l) {
        phase_d2a(sv[l], ts, rs, one);
        __syncthreads();
        phase_d2b(sv[l], sv[l + 1], rs, ts, wtab, one);
        __syncthreads();
      }
      if (ok) coarsest_solve(a, sv[L - 1], wtab, minv);
      __syncthreads();
      for (int l = L - 2; l >= tail; --l) {
        phase_u1(sv[l], sv[l + 1], ts, wtab, a.alpha, one);
        __syncthreads();
        phase_u2(sv[l], ts, wtab, one);
        __syncthreads();
      }
      {
        const int64_t nb = nt * (int64_t)sizeof(T) / 8;
        const uint2 *g = reinterpret_cast<const uint2 *>(sv[tail].e);
        uint2 *d = reinterpret_cast<uint2 *>(a.lv[tail].e);
        for (int64_t q = threadIdx.x; q < nb; q += blockDim.x) d[q] = g[q];
      }
      __syncthreads();
    } else {
      for (int l = tail; l + 1 < L; ++l) {
        phase_d2a(a.lv[l], a.scratch, a.res, one);
        __syncthreads();
        phase_d2b(a.lv[l], a.lv[l + 1], a.res, a.scratch, wtab, one);
        __syncthreads();
      }
      if (ok) coarsest_solve(a, a.lv[L - 1], wtab, minv);
      __syncthreads();
      for (int l = L - 2; l >= tail && l >= 1; --l) {
        phase_u1(a.lv[l], a.lv[l + 1], a.scratch, wtab, a.alpha, one);
        __syncthreads();
        phase_u2(a.lv[l], a.scratch, wtab, one);
        __syncthreads();
      }
    }
    mark();
  }
  // ---- up through the levels the whole cluster runs
  const int top = min(tail, L - 1) - 1;
  if (top >= 1) csync();
  for (int l = top; l >= 1; --l) {
    phase_u1(a.lv[l], a.lv[l + 1], a.scratch, wtab, a.alpha, all);
    csync();
    phase_u2(a.lv[l], a.scratch, wtab, all);
    if (l > 1) csync();
  }
  mark();
  if (cinv_copy && !cinv_waited && threadIdx.x == 0) mbar_wait(cbar, 0);
  if (!ok && threadIdx.x == 0) atomicExch(&st->dev_error, 1);
}

// BSP_TUNE_CLUSTER_TAIL: the cluster kernel's tail levels staged in CTA 0's
// shared memory.  Measured slower at 384x384x256 (the tail 10.5 -> 17.4 us:
// staging in and out costs more than the on-chip phases save), so off.
bool g_coarse_cluster_tail_smem = false;

// BSP_TUNE_CLUSTER_TAIL_CELLS: levels of at most this many cells run in the
// cluster's CTA 0 alone (with __syncthreads instead of cluster barriers).
int g_cluster_tail_cells = CL_TAIL_CELLS;

// BSP_TUNE_COARSE_CLUSTER: CTAs of the one cluster that runs the coarse cycle
// (2..16), or 0 for the cooperative kernel over every SM.  Measured at
// 384x384x256 (levels 3-6 of the cycle): 12.18 ms per solve cooperative,
// 11.86 with 8 CTAs, 11.80 with 16 (coarse cycle 46 -> 38 us).
int g_coarse_cluster = 16;

bool g_coarse_fused_enabled = true;  // BSP_TUNE_COARSE_FUSED
// BSP_TUNE_COARSE_PHASES: 1 forms t where it is read -- D1 folded into the
// residual pass, U1 into the post-smoothing pass (4 fewer grid barriers per
// cycle, 7 recomputations of t per cell); 0 (default) runs them as phases of
// their own with t stored.  The results are the same bits.  Measured at
// 384x384x256: 14.44 ms per solve fused against 14.16 ms stored -- the level-1
// phases are bound by their load latency, which recomputation lengthens.
bool g_coarse_phases_fused = false;
// BSP_TUNE_COARSE_TRACE: 1 makes every coarse-cycle launch record CTA 0's
// %globaltimer at each phase boundary (bsp_coarse_trace_read); tracing only.
bool g_coarse_trace = false;
// BSP_TUNE_COARSE_TAIL: 1 runs the levels CTA 0 handles alone out of its
// shared memory (masks, right-hand sides, corrections and scratch copied in,
// the top one's correction copied out); 0 (default) keeps them in global
// memory, where they stay in L2 between cycles: measured at 384x384x256 the
// copies cost more than the on-chip phases save (4.76 against 4.38 ms of
// coarse cycles per solve).  The results are the same bits.
bool g_coarse_tail_smem = false;

// FP32 scratch of the coarse-cycle kernel: t (max(cells of level 1, 3 x cells
// of the coarsest level), rounded up to 64 floats) followed by res (cells of
// level 1).
size_t coarse_cycle_scratch_floats(const int *dims, int L) {
  if (L < 2) return 0;
  const size_t n1 = (size_t)dims[3] * dims[4] * dims[5];
  const size_t nc = (size_t)dims[3 * (L - 1)] * dims[3 * (L - 1) + 1] * dims[3 * (L - 1) + 2];
  const size_t t = ((n1 > 3 * nc ? n1 : 3 * nc) + 63) / 64 * 64;
  return t + n1;
}

// Launch the coarse part of a V-cycle (levels 1 .. L-1) as one cooperative
// kernel.  Returns false (nothing launched) when the fused path is off, a
// level below level 0 has nz % 4 != 0 (the phases work on 4-cell quads) or the
// grid cannot be co-resident; the caller then runs the per-level kernels.
template <class T>
bool launch_coarse_cycle(const Level<T> *lv, int L, float *scratch, const float *cinv,
                         const int *cflag, void *ctl, float alpha, SolverState *st,
                         cudaStream_t s) {
  if (!g_coarse_fused_enabled || L < 2) return false;
  for (int l = 1; l < L; ++l) {
    if ((int64_t)lv[l].nx * lv[l].ny * lv[l].nz >= ((int64_t)1 << 31)) return false;
    if (lv[l].nz % 4) return false;
  }
  static int blocks = -1;
  if (blocks < 0) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, mg_cycle_kernel<T>, CC_THREADS, 0) !=
            cudaSuccess ||
        per < 1)
      blocks = 0;
    else
      blocks = sms;
  }
  if (blocks <= 0) return false;
  CoarseCycle<T> a{};
  int dims[3 * MAX_LEVELS];
  for (int l = 0; l < L; ++l) {
    a.lv[l] = lv[l];
    dims[3 * l] = lv[l].nx;
    dims[3 * l + 1] = lv[l].ny;
    dims[3 * l + 2] = lv[l].nz;
  }
  a.L = L;
  const size_t n1 = (size_t)lv[1].nx * lv[1].ny * lv[1].nz;
  a.scratch = scratch;
  a.res = scratch + (coarse_cycle_scratch_floats(dims, L) - n1);
  a.cinv = cinv;
  a.cflag = cflag;
  a.ctl = reinterpret_cast<GridCtl *>(ctl);
  a.alpha = alpha;
  a.fused_phases = g_coarse_phases_fused ? 1 : 0;
  // CTA 0's dynamic shared memory: [dense inverse of the coarsest level, when
  // small (<= 96 KB)] [coarsest right-hand side: COARSEST_CELLS floats]
  // [mbarrier, 16 B] [the tail levels CTA 0 runs alone: masks, r, e of each,
  // then two FP32 vectors of the first tail level].  The inverse's copy size
  // is rounded up to 16 bytes (its workspace slot is 256-byte aligned and at
  // least that long).  The tail goes on-chip when it fits; the inverse when
  // what is left allows.
  const int64_t nc = (int64_t)lv[L - 1].nx * lv[L - 1].ny * lv[L - 1].nz;
  auto r16 = [](int64_t b) { return (b + 15) / 16 * 16; };
  int tail = 1;
  while (tail < L && (int64_t)lv[tail].nx * lv[tail].ny * lv[tail].nz > TAIL_CELLS) ++tail;
  int64_t tail_bytes = 0;
  if (tail < L) {
    for (int l = tail; l < L; ++l) {
      const int64_t nl = (int64_t)lv[l].nx * lv[l].ny * lv[l].nz;
      tail_bytes += r16(nl) + 2 * r16(nl * (int64_t)sizeof(T));
    }
    const int64_t nt = (int64_t)lv[tail].nx * lv[tail].ny * lv[tail].nz;
    tail_bytes += 2 * r16(nt * 4);
  }
  const int64_t base = COARSEST_CELLS * (int64_t)sizeof(float) + 16;
  const int64_t cinv_b = (nc <= COARSEST_CELLS && nc * nc * 4 <= 96 * 1024 &&
                          ((uintptr_t)cinv & 15u) == 0)
                             ? r16(nc * nc * 4)
                             : 0;
  constexpr int64_t DYN_MAX = 200 * 1024;
  bool use_tail = g_coarse_tail_smem && tail < L && tail_bytes + base <= DYN_MAX;
  a.cinv_bytes = (int)((use_tail ? tail_bytes : 0) + base + cinv_b <= DYN_MAX ? cinv_b : 0);
  size_t dyn = (size_t)(a.cinv_bytes + base + (use_tail ? tail_bytes : 0));
  // one opt-in per device at the largest size this launcher ever asks for
  if (dyn > 48 * 1024 && !smem_opt_in((const void *)mg_cycle_kernel<T>, (int)DYN_MAX)) {
    a.cinv_bytes = 0;
    use_tail = false;
    dyn = (size_t)base;
  }
  a.tail_smem = use_tail ? 1 : 0;
  a.tail_off = (int)(a.cinv_bytes + base);
  a.trace = nullptr;
  if (g_coarse_trace && cudaGetSymbolAddress((void **)&a.trace, g_cc_trace) != cudaSuccess)
    a.trace = nullptr;
  if (g_coarse_cluster >= 2 && g_coarse_cluster <= 16 && !a.fused_phases) {
    // one cluster: the inverse (and the coarsest right-hand side) and the
    // levels of at most CL_TAIL_CELLS cells in CTA 0's shared memory
    CoarseCycle<T> c = a;
    int ctail = 1;
    c.tail_cells = g_cluster_tail_cells;
    while (ctail < L && (int64_t)lv[ctail].nx * lv[ctail].ny * lv[ctail].nz > c.tail_cells)
      ++ctail;
    int64_t ctail_bytes = 0;
    if (ctail < L) {
      for (int l = ctail; l < L; ++l) {
        const int64_t nl = (int64_t)lv[l].nx * lv[l].ny * lv[l].nz;
        ctail_bytes += r16(nl) + 2 * r16(nl * (int64_t)sizeof(T));
      }
      ctail_bytes += 2 * r16((int64_t)lv[ctail].nx * lv[ctail].ny * lv[ctail].nz * 4);
    }
    c.cinv_bytes = cinv_b;  // the cooperative kernel's budget does not apply here
    c.tail_smem = (g_coarse_cluster_tail_smem && ctail < L &&
                   c.cinv_bytes + base + ctail_bytes <= DYN_MAX) ? 1 : 0;
    if (c.cinv_bytes + base > DYN_MAX) c.cinv_bytes = 0;
    c.tail_off = (int)(c.cinv_bytes + base);
    const int64_t cdyn = c.cinv_bytes + base + (c.tail_smem ? ctail_bytes : 0);
    static bool attr_ok[16] = {false};
    static bool attr_done[16] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    const int di = dev & 15;
    if (!attr_done[di]) {
      attr_done[di] = true;
      attr_ok[di] =
          cudaFuncSetAttribute(mg_cluster_cycle_kernel<T>,
                               cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess &&
          smem_opt_in((const void *)mg_cluster_cycle_kernel<T>, (int)DYN_MAX);
    }
    if (attr_ok[di]) {
      // every level of the cycle in CTA 0: one CTA is the whole launch (its
      // cluster barriers are then those of a one-CTA cluster)
      const int nct = ctail <= 1 ? 1 : g_coarse_cluster;
      cudaLaunchConfig_t cc{};
      cc.gridDim = dim3(nct);
      cc.blockDim = dim3(CC_THREADS);
      cc.dynamicSmemBytes = (size_t)cdyn;
      cc.stream = s;
      cudaLaunchAttribute ca[1];
      ca[0].id = cudaLaunchAttributeClusterDimension;
      ca[0].val.clusterDim.x = nct;
      ca[0].val.clusterDim.y = 1;
      ca[0].val.clusterDim.z = 1;
      cc.attrs = ca;
      cc.numAttrs = 1;
      int nclusters = 0;
      if (cudaOccupancyMaxActiveClusters(&nclusters, mg_cluster_cycle_kernel<T>, &cc) ==
              cudaSuccess &&
          nclusters >= 1)
        return cudaLaunchKernelEx(&cc, mg_cluster_cycle_kernel<T>, c, st) == cudaSuccess;
      cudaGetLastError();  // clear a refused query; the cooperative kernel follows
    }
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(CC_THREADS);
  cfg.dynamicSmemBytes = dyn;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, mg_cycle_kernel<T>, a, st) == cudaSuccess;
}

#define INST(T)                                                                             \
  template bool launch_coarse_cycle<T>(const Level<T> *, int, float *, const float *,       \
                                       const int *, void *, float, SolverState *, cudaStream_t);
INST(float)
INST(__half)
INST(__nv_bfloat16)
#undef INST

}  // namespace bsp

// Copies the phase-boundary stamps of the last traced coarse cycle (ns,
// %globaltimer of CTA 0; unused slots hold 0) and clears them; synchronous.
extern "C" int bsp_coarse_trace_read(unsigned long long *host, int n) {
  if (!host || n <= 0) return BSP_ERR_ARG;
  if (n > bsp::CC_TRACE_MAX) n = bsp::CC_TRACE_MAX;
  cudaError_t e = cudaMemcpyFromSymbol(host, bsp::g_cc_trace, sizeof(unsigned long long) * n);
  if (e != cudaSuccess) return (int)e;
  static const unsigned long long zero[bsp::CC_TRACE_MAX] = {0};
  return (int)cudaMemcpyToSymbol(bsp::g_cc_trace, zero, sizeof(zero));
}
