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
#include "profile.cuh"

namespace bsp {

// ---- class loads -----------------------------------------------------------
__device__ __forceinline__ uint32_t cls1(const uint8_t *m, int64_t c, int, int) {
  return mcls(__ldg(m + c));
}
__device__ __forceinline__ uint32_t cls1(const int32_t *m, int64_t c, int mf, int ma) {
  return classify(__ldg(m + c), mf, ma);
}
// Four packed mask bytes (bit 7 fluid, bit 6 solid) of cells c..c+3.
__device__ __forceinline__ uint32_t mw4(const uint8_t *m, int64_t c, int, int) {
  return __ldg(reinterpret_cast<const uint32_t *>(m + c));
}
__device__ __forceinline__ uint32_t mw4(const int32_t *m, int64_t c, int mf, int ma) {
  int4 v = __ldg(reinterpret_cast<const int4 *>(m + c));
  return enc_cls(classify(v.x, mf, ma)) | (enc_cls(classify(v.y, mf, ma)) << 8) |
         (enc_cls(classify(v.z, mf, ma)) << 16) | (enc_cls(classify(v.w, mf, ma)) << 24);
}
__device__ __forceinline__ uint32_t mw1(const uint8_t *m, int64_t c, int, int) {
  return __ldg(m + c);
}
__device__ __forceinline__ uint32_t mw1(const int32_t *m, int64_t c, int mf, int ma) {
  return enc_cls(classify(__ldg(m + c), mf, ma));
}

// Stencil flavours of the column kernel.
enum Op {
  OP_JACOBI = 0,      // p_new = (s - rho dx^2 div / dt) / 6, division per cell
  OP_SPMV = 1,        // A p = 6 p - s
  OP_JACOBI_RHS = 2,  // p_new = (s - rhs) / 6 with rhs = rho dx^2 div / dt precomputed
};

__device__ __forceinline__ float f4(const float4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}
__device__ __forceinline__ float4 ld4(const float *p) {
  return __ldg(reinterpret_cast<const float4 *>(p));
}

// ---- column kernel ----------------------------------------------------------
// CTA = 8 warps; warp w owns row j = blockIdx.y*8 + w and the 128 cells
// k = blockIdx.x*128 + 4*lane .. +3, and marches i over [blockIdx.z*bi, +bi).
// The i-1 / i / i+1 planes of p and of the mask stay in registers; j +- 1 come
// from L1 (neighbouring warps' rows); k +- 1 from warp shuffles.  Neighbour
// values are chosen with sel_nbr (two prmt + one lop3, no branches); the sum
// order is the reference's l, r, d, u, b, f.
//
// ZNF (sweep_znf_kernel below): the source field holds +0 on every non-fluid
// cell (true after one sweep, and for a projection, which zeroes p first).
// Then the neighbour rule fluid -> p_n, air -> 0, solid -> p_self is exactly
// p_n | (p_self & solid) on bit patterns (p_n is +0 on air and solid cells):
// one prmt + one lop3.
__device__ __forceinline__ float znf_nbr(uint32_t sw, int q, float pn, float ps) {
  const uint32_t sm = sign_bytes(sw, (uint32_t)(8 | q) * 0x1111u);
  return __uint_as_float(__float_as_uint(pn) | (__float_as_uint(ps) & sm));
}

template <int OP, class MaskT, bool FULL>
__global__ void __launch_bounds__(256) stencil_col_kernel(
    float *__restrict__ out, const float *__restrict__ p, const float *__restrict__ src,
    const MaskT *__restrict__ mask, int nx, int ny, int nz, int bi, float rdd, float dt,
    int mf, int ma) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (j >= ny) return;  // warp-uniform
  const int k = (blockIdx.x * 32 + lane) * 4;
  const bool act = FULL || k < nz;
  const int i0 = blockIdx.z * bi;
  const int i1 = min(i0 + bi, nx);
  const int64_t plane = (int64_t)ny * nz;
  const bool has_jm = j > 0, has_jp = j + 1 < ny;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  int64_t o = (int64_t)i0 * plane + (int64_t)j * nz + k;

  float4 pm = z4, pc = z4;
  uint32_t mm = 0u, mc = 0u;  // 0 = air
  if (act && i0 > 0) {
    pm = ld4(p + o - plane);
    mm = mw4(mask, o - plane, mf, ma);
  }
  if (act) {
    pc = ld4(p + o);
    mc = mw4(mask, o, mf, ma);
  }
  for (int i = i0; i < i1; ++i, o += plane) {
    float4 pn = z4, pjm = z4, pjp = z4, sv = z4;
    uint32_t mn = 0u, mjm = 0u, mjp = 0u;
    if (act) {
      if (i + 1 < nx) {
        pn = ld4(p + o + plane);
        mn = mw4(mask, o + plane, mf, ma);
      }
      if (has_jm) {
        pjm = ld4(p + o - nz);
        mjm = mw4(mask, o - nz, mf, ma);
      }
      if (has_jp) {
        pjp = ld4(p + o + nz);
        mjp = mw4(mask, o + nz, mf, ma);
      }
      if (OP != OP_SPMV) sv = ld4(src + o);
    }
    float pkm = __shfl_up_sync(0xffffffffu, pc.w, 1);
    uint32_t mkm = __shfl_up_sync(0xffffffffu, mc, 1);
    float pkp = __shfl_down_sync(0xffffffffu, pc.x, 1);
    uint32_t mkp = __shfl_down_sync(0xffffffffu, mc, 1);
    if (lane == 0) {
      const bool in = act && k > 0;
      pkm = in ? __ldg(p + o - 1) : 0.0f;
      mkm = in ? mw1(mask, o - 1, mf, ma) << 24 : 0u;
    }
    if (lane == 31) {
      const bool in = act && k + 4 < nz;
      pkp = in ? __ldg(p + o + 4) : 0.0f;
      mkp = in ? mw1(mask, o + 4, mf, ma) : 0u;
    }
    // mask words of the back (k-1) and front (k+1) neighbours of the 4 cells
    const uint32_t mb = (mc << 8) | (mkm >> 24);
    const uint32_t mfw = (mc >> 8) | (mkp << 24);
    const float4 pb = make_float4(pkm, pc.x, pc.y, pc.z);
    const float4 pf = make_float4(pc.y, pc.z, pc.w, pkp);
    if (act) {
      float o4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float ps = f4(pc, q);
        const float l = sel_nbr(mm, mm << 1, q, f4(pm, q), ps);
        const float r = sel_nbr(mn, mn << 1, q, f4(pn, q), ps);
        const float d = sel_nbr(mjm, mjm << 1, q, f4(pjm, q), ps);
        const float u = sel_nbr(mjp, mjp << 1, q, f4(pjp, q), ps);
        const float b = sel_nbr(mb, mb << 1, q, f4(pb, q), ps);
        const float f = sel_nbr(mfw, mfw << 1, q, f4(pf, q), ps);
        float v;
        if (OP == OP_SPMV) {
          v = spmv_update(l, r, d, u, b, f, ps);
        } else {
          const float s = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(l, r), d), u), b), f);
          const float rhs = OP == OP_JACOBI ? __fdiv_rn(__fmul_rn(rdd, f4(sv, q)), dt) : f4(sv, q);
          v = div6(__fsub_rn(s, rhs));
        }
        o4[q] = __uint_as_float(__float_as_uint(v) & fluid_word(mc, q));
      }
      *reinterpret_cast<float4 *>(out + o) = make_float4(o4[0], o4[1], o4[2], o4[3]);
    }
    pm = pc;
    mm = mc;
    pc = pn;
    mc = mn;
  }
}

// ---- ZNF sweep kernel -----------------------------------------------------------
// The column kernel's layout and arithmetic for p_new = (s - rhs) / 6 on a
// source that is +0 off fluid, with two warp-uniform shortcuts, both exact:
//  * a 128-cell row segment without a fluid cell stores +0 (a non-fluid
//    cell's result is +0 whatever its operands) and reads neither its j
//    neighbours nor rhs: 9 instead of 13 B/cell;
//  * a segment whose fluid cells have no solid face neighbour (mask bits 0-2,
//    the solid-neighbour count, zero on every fluid byte) sums the raw
//    neighbour values: fluid neighbours give p_n, air ones p_n = +0, which is
//    what the boundary rule selects, in the same order l, r, d, u, b, f.
// Other segments take the per-neighbour select of stencil_col_kernel.
template <bool RAW>
__device__ __forceinline__ float4 znf_segment(const float *__restrict__ p,
                                              const float *__restrict__ rhs,
                                              const uint8_t *__restrict__ mask, int64_t o,
                                              int lane, int k, int nz, bool act, bool has_jm,
                                              bool has_jp, const float4 &pm, const float4 &pc,
                                              const float4 &pn, uint32_t mm, uint32_t mc,
                                              uint32_t mn) {
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 pjm = z4, pjp = z4, sv = z4;
  uint32_t mjm = 0u, mjp = 0u;
  if (act) {
    if (has_jm) {
      pjm = ld4(p + o - nz);
      if (!RAW) mjm = mw4(mask, o - nz, 0, 0);
    }
    if (has_jp) {
      pjp = ld4(p + o + nz);
      if (!RAW) mjp = mw4(mask, o + nz, 0, 0);
    }
    sv = ld4(rhs + o);
  }
  float pkm = __shfl_up_sync(0xffffffffu, pc.w, 1);
  float pkp = __shfl_down_sync(0xffffffffu, pc.x, 1);
  uint32_t mkm = 0u, mkp = 0u;
  if (!RAW) {
    mkm = __shfl_up_sync(0xffffffffu, mc, 1);
    mkp = __shfl_down_sync(0xffffffffu, mc, 1);
  }
  if (lane == 0) {
    const bool in = act && k > 0;
    pkm = in ? __ldg(p + o - 1) : 0.0f;
    if (!RAW) mkm = in ? (uint32_t)__ldg(mask + o - 1) << 24 : 0u;
  }
  if (lane == 31) {
    const bool in = act && k + 4 < nz;
    pkp = in ? __ldg(p + o + 4) : 0.0f;
    if (!RAW) mkp = in ? (uint32_t)__ldg(mask + o + 4) : 0u;
  }
  const uint32_t mb = (mc << 8) | (mkm >> 24);
  const uint32_t mfw = (mc >> 8) | (mkp << 24);
  const float4 pb = make_float4(pkm, pc.x, pc.y, pc.z);
  const float4 pf = make_float4(pc.y, pc.z, pc.w, pkp);
  float o4[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float ps = f4(pc, q);
    float l, r, d, u, b, f;
    if (RAW) {
      l = f4(pm, q);
      r = f4(pn, q);
      d = f4(pjm, q);
      u = f4(pjp, q);
      b = f4(pb, q);
      f = f4(pf, q);
    } else {
      l = znf_nbr(mm << 1, q, f4(pm, q), ps);
      r = znf_nbr(mn << 1, q, f4(pn, q), ps);
      d = znf_nbr(mjm << 1, q, f4(pjm, q), ps);
      u = znf_nbr(mjp << 1, q, f4(pjp, q), ps);
      b = znf_nbr(mb << 1, q, f4(pb, q), ps);
      f = znf_nbr(mfw << 1, q, f4(pf, q), ps);
    }
    const float sum = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(l, r), d), u), b), f);
    const float v = div6(__fsub_rn(sum, f4(sv, q)));
    o4[q] = __uint_as_float(__float_as_uint(v) & fluid_word(mc, q));
  }
  return make_float4(o4[0], o4[1], o4[2], o4[3]);
}

// L2 prefetch of one 128-byte line (no register result, does not block).
__device__ __forceinline__ void prefetch_l2(const void *ptr) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

// PF > 0: each plane step also prefetches into L2 the p and mask rows of
// plane i + PF and, when plane i + 1 holds fluid in this segment, its rhs
// row, so that the next steps' loads wait on L2 instead of DRAM (one lane per
// 128-byte line).  Measured at 384x384x256: 93.5 us per sweep without, 81.4
// with PF = 2.
template <bool FULL, int PF>
__global__ void __launch_bounds__(256) sweep_znf_kernel(float *__restrict__ out,
                                                        const float *__restrict__ p,
                                                        const float *__restrict__ rhs,
                                                        const uint8_t *__restrict__ mask, int nx,
                                                        int ny, int nz, int bi) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (j >= ny) return;  // warp-uniform
  const int k = (blockIdx.x * 32 + lane) * 4;
  const bool act = FULL || k < nz;
  const int i0 = blockIdx.z * bi;
  const int i1 = min(i0 + bi, nx);
  const int64_t plane = (int64_t)ny * nz;
  const bool has_jm = j > 0, has_jp = j + 1 < ny;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  int64_t o = (int64_t)i0 * plane + (int64_t)j * nz + k;
  float4 pm = z4, pc = z4;
  uint32_t mm = 0u, mc = 0u;  // 0 = air
  if (act && i0 > 0) {
    pm = ld4(p + o - plane);
    mm = mw4(mask, o - plane, 0, 0);
  }
  if (act) {
    pc = ld4(p + o);
    mc = mw4(mask, o, 0, 0);
  }
  for (int i = i0; i < i1; ++i, o += plane) {
    float4 pn = z4;
    uint32_t mn = 0u;
    if (act && i + 1 < nx) {
      pn = ld4(p + o + plane);
      mn = mw4(mask, o + plane, 0, 0);
    }
    if (PF > 0 && act && i + PF < nx && (lane & 7) == 0) {
      prefetch_l2(p + o + PF * plane);
      if (lane == 0) prefetch_l2(mask + o + PF * plane);
    }
    float4 v = z4;
    if (__any_sync(0xffffffffu, (mc & 0x80808080u) != 0u)) {
      // fluid bytes' solid-neighbour counts: bit 0 of each fluid byte times 7
      const uint32_t fl7 = ((mc >> 7) & 0x01010101u) * 7u;
      if (__all_sync(0xffffffffu, (mc & fl7) == 0u))
        v = znf_segment<true>(p, rhs, mask, o, lane, k, nz, act, has_jm, has_jp, pm, pc, pn, mm,
                              mc, mn);
      else
        v = znf_segment<false>(p, rhs, mask, o, lane, k, nz, act, has_jm, has_jp, pm, pc, pn, mm,
                               mc, mn);
    }
    if (act) *reinterpret_cast<float4 *>(out + o) = v;
    if (PF > 0 && __any_sync(0xffffffffu, (mn & 0x80808080u) != 0u) && act && (lane & 7) == 0)
      prefetch_l2(rhs + o + plane);
    pm = pc;
    mm = mc;
    pc = pn;
    mc = mn;
  }
}

// BSP_TUNE_SWEEP_PREFETCH: the ZNF sweep's L2 prefetch distance in planes
// (0 off, 2 default, 3).
int g_sweep_prefetch = 2;

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
    if (OP == OP_SPMV) {
      out[c] = spmv_update(l, r, d, u, b, f, ps);
    } else {
      const float s = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(l, r), d), u), b), f);
      const float rhs =
          OP == OP_JACOBI ? __fdiv_rn(__fmul_rn(rdd, __ldg(div + c)), dt) : __ldg(div + c);
      out[c] = div6(__fsub_rn(s, rhs));
    }
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
    mask[c] = (uint8_t)(enc_cls(cls) | ns);
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
// Autotuner override of the column kernel's i-extent (0 = heuristic below).
int g_sweep_bi = 0;

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
                      (OP == OP_SPMV || aligned16(div)) &&
                      (sizeof(MaskT) == 4 ? aligned16(mask) : (((uintptr_t)mask & 3u) == 0));
  if (col_ok) {
    const int bi = g_sweep_bi > 0 ? g_sweep_bi : pick_bi(nx, ny, nz);
    dim3 grid((nz / 4 + 31) / 32, (ny + 7) / 8, (nx + bi - 1) / bi);
    if (nz % 128 == 0)
      stencil_col_kernel<OP, MaskT, true><<<grid, 256, 0, s>>>(out, p, div, mask, nx, ny, nz, bi,
                                                               rdd, dt, mf, ma);
    else
      stencil_col_kernel<OP, MaskT, false><<<grid, 256, 0, s>>>(out, p, div, mask, nx, ny, nz, bi,
                                                                rdd, dt, mf, ma);
  } else {
    const int64_t n = (int64_t)nx * ny * nz;
    stencil_generic_kernel<OP, MaskT><<<generic_blocks(n), 256, 0, s>>>(out, p, div, mask, nx,
                                                                        ny, nz, rdd, dt, mf, ma);
  }
  return cudaGetLastError();
}

// Jacobi sweep with precomputed rhs on a source whose non-fluid cells are +0
// (the ZNF column kernel), or the general kernels when the layout does not
// allow the column kernel.  Bit-identical to launch_stencil<OP_JACOBI_RHS>.
cudaError_t launch_sweep_znf(float *out, const float *p, const float *rhs, const uint8_t *mask,
                             int nx, int ny, int nz, cudaStream_t s) {
  const bool col_ok = (nz % 4 == 0) && aligned16(out) && aligned16(p) && aligned16(rhs) &&
                      (((uintptr_t)mask & 3u) == 0);
  if (!col_ok)
    return launch_stencil<OP_JACOBI_RHS, uint8_t>(out, p, rhs, mask, nx, ny, nz, 0.f, 1.f, 0.f,
                                                  BSP_FLUID, BSP_AIR, s);
  const int bi = g_sweep_bi > 0 ? g_sweep_bi : pick_bi(nx, ny, nz);
  dim3 grid((nz / 4 + 31) / 32, (ny + 7) / 8, (nx + bi - 1) / bi);
  if (nz % 128 == 0)
    (g_sweep_prefetch == 3   ? sweep_znf_kernel<true, 3>
     : g_sweep_prefetch == 2 ? sweep_znf_kernel<true, 2>
                             : sweep_znf_kernel<true, 0>)<<<grid, 256, 0, s>>>(
        out, p, rhs, mask, nx, ny, nz, bi);
  else
    (g_sweep_prefetch == 3   ? sweep_znf_kernel<false, 3>
     : g_sweep_prefetch == 2 ? sweep_znf_kernel<false, 2>
                             : sweep_znf_kernel<false, 0>)<<<grid, 256, 0, s>>>(
        out, p, rhs, mask, nx, ny, nz, bi);
  return cudaGetLastError();
}

template cudaError_t launch_stencil<OP_JACOBI, uint8_t>(float *, const float *, const float *,
                                                        const uint8_t *, int, int, int, float,
                                                        float, float, int, int, cudaStream_t);
template cudaError_t launch_stencil<OP_SPMV, uint8_t>(float *, const float *, const float *,
                                                      const uint8_t *, int, int, int, float,
                                                      float, float, int, int, cudaStream_t);
template cudaError_t launch_stencil<OP_JACOBI_RHS, uint8_t>(float *, const float *,
                                                            const float *, const uint8_t *, int,
                                                            int, int, float, float, float, int,
                                                            int, cudaStream_t);

// rhs[c] = (rho dx dx) div[c] / dt on fluid cells (0 elsewhere): the per-cell
// constant of the Jacobi update, bit-identical to the value each sweep of the
// reference computes (fluid.py:275).
// rhs may alias div (in-place conversion): no __restrict__ on those two.
__global__ void rhs_kernel(float *rhs, const float *div, const uint8_t *__restrict__ mask,
                           int64_t n, float rdd, float dt) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    rhs[c] = (__ldg(mask + c) & BSP_MFLUID) ? __fdiv_rn(__fmul_rn(rdd, div[c]), dt) : 0.0f;
}

cudaError_t launch_rhs(float *rhs, const float *div, const uint8_t *mask, int64_t n, float dx,
                       float dt, float rho, cudaStream_t s) {
  const float rdd = rho * dx * dx;
  ProfScope ps(PROF_PROJ, s);
  rhs_kernel<<<generic_blocks(n), 256, 0, s>>>(rhs, div, mask, n, rdd, dt);
  return cudaGetLastError();
}

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

namespace bsp {
extern bool g_fine_col_enabled;
extern float g_mg_alpha;
extern bool g_fine_tma_enabled;
extern bool g_coarse_fused_enabled;
extern bool g_fuse_update_enabled;
extern int g_fine_bi;
extern int g_sweep_tblock;
extern bool g_test_barrier_error;
extern bool g_coarse_phases_fused;
extern bool g_coarse_trace;
extern bool g_coarse_tail_smem;
extern int g_coarse_split;
extern int g_l1_sweeps;
extern bool g_pcg_quad;
extern bool g_l0_trilinear;
extern int g_tri_cpc;
extern bool g_fuse_scalars;
extern int g_fine_ctas;
extern bool g_pdl;
extern int g_coarse_cluster;
extern int g_cluster_tail_cells;
extern int g_downu_blocks;
extern bool g_coarse_cluster_tail_smem;
namespace utc {
extern int g_utc_nepi;
}  // namespace utc
namespace cond {
extern int g_cond_bi;
extern bool g_cond_tma;
}  // namespace cond
}

extern "C" int bsp_set_tuning(int key, int value) {
  switch (key) {
    case BSP_TUNE_SWEEP_BI:
      if (value < 0 || value > 4096) return BSP_ERR_ARG;
      bsp::g_sweep_bi = value;
      return BSP_OK;
    case BSP_TUNE_FINE_COLUMN:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_fine_col_enabled = value != 0;
      return BSP_OK;
    case BSP_TUNE_MG_ALPHA:
      if (value < 100 || value > 3000) return BSP_ERR_ARG;
      bsp::g_mg_alpha = (float)value / 1000.0f;
      return BSP_OK;
    case BSP_TUNE_FINE_TMA:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_fine_tma_enabled = value != 0;
      return BSP_OK;
    case BSP_TUNE_COARSE_FUSED:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_coarse_fused_enabled = value != 0;
      return BSP_OK;
    case BSP_TUNE_FUSE_UPDATE:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_fuse_update_enabled = value != 0;
      return BSP_OK;
    case BSP_TUNE_FINE_BI:
      if (value < 0 || value > 64) return BSP_ERR_ARG;
      bsp::g_fine_bi = value;
      return BSP_OK;
    case BSP_TUNE_SWEEP_TBLOCK:
      if (value < 1 || value > 2) return BSP_ERR_ARG;
      bsp::g_sweep_tblock = value;
      return BSP_OK;
    case BSP_TUNE_COND_BI:
      if (value < 0 || value > 4096) return BSP_ERR_ARG;
      bsp::cond::g_cond_bi = value;
      return BSP_OK;
    case BSP_TUNE_COND_TMA:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::cond::g_cond_tma = value != 0;
      return BSP_OK;
    case BSP_TUNE_CONV_EPILOGUE:
      if (value < 0 || value > 4) return BSP_ERR_ARG;
      bsp::utc::g_utc_nepi = value;
      return BSP_OK;
    case BSP_TUNE_DOWNU_BLOCKS:
      if (value != 3 && value != 4) return BSP_ERR_ARG;
      bsp::g_downu_blocks = value;
      return BSP_OK;
    case BSP_TUNE_CLUSTER_TAIL_CELLS:
      if (value < 0 || value > (1 << 20)) return BSP_ERR_ARG;
      bsp::g_cluster_tail_cells = value;
      return BSP_OK;
    case BSP_TUNE_SWEEP_PREFETCH:
      if (value != 0 && value != 2 && value != 3) return BSP_ERR_ARG;
      bsp::g_sweep_prefetch = value;
      return BSP_OK;
    case BSP_TUNE_CLUSTER_TAIL:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_coarse_cluster_tail_smem = value != 0;
      return BSP_OK;
    case BSP_TUNE_COARSE_CLUSTER:
      if (value != 0 && (value < 2 || value > 16)) return BSP_ERR_ARG;
      bsp::g_coarse_cluster = value;
      return BSP_OK;
    case BSP_TUNE_PDL:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_pdl = value != 0;
      return BSP_OK;
    case BSP_TUNE_FINE_CTAS:
      if (value < 1 || value > 16) return BSP_ERR_ARG;
      bsp::g_fine_ctas = value;
      return BSP_OK;
    case BSP_TUNE_FUSE_SCALARS:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_fuse_scalars = value != 0;
      return BSP_OK;
    case BSP_TUNE_TRI_CPC:
      if (value < 1 || value > 64) return BSP_ERR_ARG;
      bsp::g_tri_cpc = value;
      return BSP_OK;
    case BSP_TUNE_L0_TRILINEAR:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_l0_trilinear = value != 0;
      return BSP_OK;
    case BSP_TUNE_PCG_QUAD:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_pcg_quad = value != 0;
      return BSP_OK;
    case BSP_TUNE_L1_SWEEPS:
      if (value < 1 || value > 2) return BSP_ERR_ARG;
      bsp::g_l1_sweeps = value;
      return BSP_OK;
    case BSP_TUNE_COARSE_SPLIT:
      if (value < 0 || value > 3) return BSP_ERR_ARG;
      bsp::g_coarse_split = value;
      return BSP_OK;
    case BSP_TUNE_COARSE_PHASES:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_coarse_phases_fused = value != 0;
      return BSP_OK;
    case BSP_TUNE_COARSE_TAIL:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_coarse_tail_smem = value != 0;
      return BSP_OK;
    case BSP_TUNE_COARSE_TRACE:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_coarse_trace = value != 0;
      return BSP_OK;
    case BSP_TUNE_TEST_BARRIER_ERROR:
      if (value < 0 || value > 1) return BSP_ERR_ARG;
      bsp::g_test_barrier_error = value != 0;
      return BSP_OK;
    default:
      return BSP_ERR_ARG;
  }
}
