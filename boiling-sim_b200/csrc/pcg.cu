// pcg.cu -- Jacobi-preconditioned conjugate gradient as ONE persistent kernel.
//
// Algorithm: crates/cuda-kernels/src/pressure_solve_pcg.cu:89-243 --
//   b = -(rho dx^2/dt) div on fluid cells; p = 0; r = b; z = D^-1 r; ps = z;
//   loop: Ap = A ps; alpha = rz/pAp; p += alpha ps; r -= alpha Ap;
//         [it >= 8, it % 5 == 0: stop if r.r < tol^2 b.b]
//         z = D^-1 r; beta = rz_new/rz; ps = z + beta ps.
// with A = 6I - S (laplacian_spmv.cu:62-143) and D = 6 - n_solid
// (diag_inverse_apply.cu:44-89).
//
// B200 design: the reference issues ~10 launches and a blocking device->host
// copy per check; here one cooperative launch runs the whole loop.  Each
// iteration is two grid-wide phases separated by bounded grid barriers:
//   A: ps = z + beta ps_prev is formed on the fly (centre and neighbours), the
//      stencil A ps is applied and stored with ps; partial ps.Ap.
//   B: p, r, z updated elementwise; partial r.z and r.r.
// All inner products are FP64 with a fixed reduction order (deterministic for a
// given grid size).  Vector arithmetic stays FP32 with the reference's
// expressions (y = fma(a, x, y)).
// Work unit: one (i, j) row of nz cells per warp, lanes striding over k.
#include <type_traits>

#include "grid_sync.cuh"

namespace bsp {

int num_sms();

// One 1024-thread CTA per SM (the grid a whole number of CTAs per SM: a grid of
// 168 = 148 + 20 CTAs, the most the reference's 4 KB dot workspace has room
// for, left 20 SMs with twice the work, and each barrier waits for them).
constexpr int PCG_THREADS = 1024;

template <class MaskT>
struct PcgArgs {
  float *p;
  const float *div;
  const MaskT *mask;
  float *r, *z, *ps0, *ps1, *Ap;
  double *partials;  // 3 * stride doubles
  GridCtl *ctl;
  float *outs[7];  // optional device floats: alpha beta rzold rznew bsq rsq pAp
  int nx, ny, nz, mf, ma, max_iter, stride;
  int quad;      // 1: the four-cell form of the two phases (int32 ids, nz % 4 == 0)
  float scale;   // -(rho dx dx)/dt as float
  double tol2;   // tol^2
};

__device__ __forceinline__ uint32_t pcg_cls(const uint8_t *m, int64_t c, int, int) {
  return mcls(__ldg(m + c));
}
__device__ __forceinline__ uint32_t pcg_cls(const int32_t *m, int64_t c, int mf, int ma) {
  return classify(__ldg(m + c), mf, ma);
}
__device__ __forceinline__ int pcg_nsolid(const uint8_t *m, int64_t c, int, int, int, int, int,
                                          int, int, int) {
  return (int)mnsolid(__ldg(m + c));
}
__device__ __forceinline__ int pcg_nsolid(const int32_t *m, int64_t c, int i, int j, int k,
                                          int nx, int ny, int nz, int mf, int ma) {
  const int64_t plane = (int64_t)ny * nz;
  int ns = 0;
#define SOL(cond, off) ns += ((cond) && classify(__ldg(m + c + (off)), mf, ma) == BSP_SOLID) ? 1 : 0
  SOL(i > 0, -plane);
  SOL(i + 1 < nx, plane);
  SOL(j > 0, -(int64_t)nz);
  SOL(j + 1 < ny, (int64_t)nz);
  SOL(k > 0, -1);
  SOL(k + 1 < nz, 1);
#undef SOL
  return ns;
}

__device__ __forceinline__ float dinv_apply(float r, int ns) {
  const float d = 6.0f - (float)ns;
  return d <= 0.0f ? r : __fdiv_rn(r, d);
}

// ---- quad form (nz % 4 == 0, int32 material ids) ------------------------------------
// A warp takes a unit of 128 consecutive k cells of one (i, j) row, a lane
// four of them: vector loads and stores, the k +- 1 neighbours of a quad from
// the neighbouring lanes by shuffles (scalar loads at the unit's ends).  The
// same per-cell operations as the scalar form; only the FP64 partial sums run
// in another order.
__device__ __forceinline__ float q4v(const float4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}
__device__ __forceinline__ int q4i(const int4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}
__device__ __forceinline__ void cls4(const int4 &m, int mf, int ma, uint32_t (&c)[4]) {
  c[0] = classify(m.x, mf, ma);
  c[1] = classify(m.y, mf, ma);
  c[2] = classify(m.z, mf, ma);
  c[3] = classify(m.w, mf, ma);
}

// Phase A on one unit: ps = z + beta ps_prev (z on the first iteration) on
// fluid cells, Ap = 6 ps - s(ps); both 0 elsewhere; returns sum ps.Ap.
__device__ __forceinline__ double pcg_quad_a(const PcgArgs<int32_t> &a, float *cur,
                                             const float *prev, float bf, bool first, int i,
                                             int j, int k, int64_t c, bool valid) {
  const int nx = a.nx, ny = a.ny, nz = a.nz, mf = a.mf, ma = a.ma;
  const int lane = threadIdx.x & 31;
  const int64_t plane = (int64_t)ny * nz;
  // z and ps are written inside this kernel: plain (coherent) loads
  auto ps4 = [&](int64_t x) {
    const float4 z = *reinterpret_cast<const float4 *>(a.z + x);
    if (first) return z;
    const float4 pv = *reinterpret_cast<const float4 *>(prev + x);
    return make_float4(__fmaf_rn(bf, pv.x, z.x), __fmaf_rn(bf, pv.y, z.y),
                       __fmaf_rn(bf, pv.z, z.z), __fmaf_rn(bf, pv.w, z.w));
  };
  auto ps1 = [&](int64_t x) { return first ? a.z[x] : __fmaf_rn(bf, prev[x], a.z[x]); };
  uint32_t cc[4] = {BSP_AIR, BSP_AIR, BSP_AIR, BSP_AIR};
  float4 pc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (valid) {
    cls4(__ldg(reinterpret_cast<const int4 *>(a.mask + c)), mf, ma, cc);
    pc = ps4(c);
  }
  // k -1 of the quad's first cell and k + 1 of its last: the neighbouring
  // lanes' cells (every lane takes part in the shuffles)
  const float lw = __shfl_up_sync(0xffffffffu, pc.w, 1);
  const uint32_t lc = __shfl_up_sync(0xffffffffu, cc[3], 1);
  const float rx = __shfl_down_sync(0xffffffffu, pc.x, 1);
  const uint32_t rc = __shfl_down_sync(0xffffffffu, cc[0], 1);
  if (!valid) return 0.0;
  const bool any_fluid = cc[0] == BSP_FLUID || cc[1] == BSP_FLUID || cc[2] == BSP_FLUID ||
                         cc[3] == BSP_FLUID;
  if (!any_fluid) {
    *reinterpret_cast<float4 *>(cur + c) = make_float4(0.f, 0.f, 0.f, 0.f);
    *reinterpret_cast<float4 *>(a.Ap + c) = make_float4(0.f, 0.f, 0.f, 0.f);
    return 0.0;
  }
  // k - 1 and k + 4: from the lanes beside, or loaded at the unit's ends
  bool has_km = k > 0, has_kp = k + 4 < nz;
  float pkm = 0.0f, pkp = 0.0f;
  uint32_t ckm = BSP_AIR, ckp = BSP_AIR;
  if (has_km) {
    if (lane > 0) {
      pkm = lw;
      ckm = lc;
    } else {
      ckm = classify(__ldg(a.mask + c - 1), mf, ma);
      if (ckm == BSP_FLUID) pkm = ps1(c - 1);
    }
  }
  if (has_kp) {
    if (lane < 31) {
      pkp = rx;
      ckp = rc;
    } else {
      ckp = classify(__ldg(a.mask + c + 4), mf, ma);
      if (ckp == BSP_FLUID) pkp = ps1(c + 4);
    }
  }
  // the neighbour sum in the reference's order l, r, d, u, b, f, folded one
  // direction at a time (the same additions as spmv_update)
  const float vc[4] = {pc.x, pc.y, pc.z, pc.w};
  auto nb = [&](bool cond, uint32_t cls, float v, float psc) {
    return cond ? (cls == BSP_FLUID ? v : (cls == BSP_AIR ? 0.0f : psc)) : 0.0f;
  };
  float acc[4];
  const int64_t off[4] = {-plane, plane, -(int64_t)nz, (int64_t)nz};
  const bool in[4] = {i > 0, i + 1 < nx, j > 0, j + 1 < ny};
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    uint32_t cn[4] = {BSP_AIR, BSP_AIR, BSP_AIR, BSP_AIR};
    float4 pn = make_float4(0.f, 0.f, 0.f, 0.f);
    if (in[d]) {
      cls4(__ldg(reinterpret_cast<const int4 *>(a.mask + c + off[d])), mf, ma, cn);
      pn = ps4(c + off[d]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float t = nb(in[d], cn[q], q4v(pn, q), vc[q]);
      acc[q] = d == 0 ? t : __fadd_rn(acc[q], t);
    }
  }
  float ps_out[4], ap_out[4];
  double dot = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float psc = vc[q];
    const float bk = q == 0 ? nb(has_km, ckm, pkm, psc) : nb(true, cc[q - 1], vc[q - 1], psc);
    const float f = q == 3 ? nb(has_kp, ckp, pkp, psc) : nb(true, cc[q + 1], vc[q + 1], psc);
    const float sum = __fadd_rn(__fadd_rn(acc[q], bk), f);
    const float ap = __fmaf_rn(6.0f, psc, -sum);  // spmv_update
    const bool fl = cc[q] == BSP_FLUID;
    ps_out[q] = fl ? psc : 0.0f;
    ap_out[q] = fl ? ap : 0.0f;
    if (fl) dot += (double)psc * (double)ap;
  }
  *reinterpret_cast<float4 *>(cur + c) = make_float4(ps_out[0], ps_out[1], ps_out[2], ps_out[3]);
  *reinterpret_cast<float4 *>(a.Ap + c) =
      make_float4(ap_out[0], ap_out[1], ap_out[2], ap_out[3]);
  return dot;
}

// Phase B on one unit: p += alpha ps; r -= alpha Ap; z = D^-1 r on fluid
// cells (the others keep their 0); returns (sum r.z, sum r.r).
__device__ __forceinline__ void pcg_quad_b(const PcgArgs<int32_t> &a, const float *cur, float af,
                                           int i, int j, int k, int64_t c, bool valid,
                                           double &rz, double &rr2) {
  const int nx = a.nx, ny = a.ny, nz = a.nz, mf = a.mf, ma = a.ma;
  const int lane = threadIdx.x & 31;
  const int64_t plane = (int64_t)ny * nz;
  uint32_t cc[4] = {BSP_AIR, BSP_AIR, BSP_AIR, BSP_AIR};
  if (valid) cls4(__ldg(reinterpret_cast<const int4 *>(a.mask + c)), mf, ma, cc);
  const uint32_t lc = __shfl_up_sync(0xffffffffu, cc[3], 1);
  const uint32_t rc = __shfl_down_sync(0xffffffffu, cc[0], 1);
  if (!valid) return;
  if (!(cc[0] == BSP_FLUID || cc[1] == BSP_FLUID || cc[2] == BSP_FLUID || cc[3] == BSP_FLUID))
    return;
  // solid neighbours of each cell (in-grid only), in any order: a count
  uint32_t ckm = BSP_AIR, ckp = BSP_AIR;
  if (k > 0) ckm = lane > 0 ? lc : classify(__ldg(a.mask + c - 1), mf, ma);
  if (k + 4 < nz) ckp = lane < 31 ? rc : classify(__ldg(a.mask + c + 4), mf, ma);
  int ns[4] = {0, 0, 0, 0};
  const int64_t off[4] = {-plane, plane, -(int64_t)nz, (int64_t)nz};
  const bool in[4] = {i > 0, i + 1 < nx, j > 0, j + 1 < ny};
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    if (!in[d]) continue;
    uint32_t cn[4];
    cls4(__ldg(reinterpret_cast<const int4 *>(a.mask + c + off[d])), mf, ma, cn);
#pragma unroll
    for (int q = 0; q < 4; ++q) ns[q] += cn[q] == BSP_SOLID ? 1 : 0;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t kl = q == 0 ? ckm : cc[q - 1];
    const uint32_t kr = q == 3 ? ckp : cc[q + 1];
    ns[q] += (kl == BSP_SOLID ? 1 : 0) + (kr == BSP_SOLID ? 1 : 0);
  }
  const float4 cu = *reinterpret_cast<const float4 *>(cur + c);
  const float4 ap = *reinterpret_cast<const float4 *>(a.Ap + c);
  const float4 p0 = *reinterpret_cast<const float4 *>(a.p + c);
  const float4 r0 = *reinterpret_cast<const float4 *>(a.r + c);
  float po[4], ro[4], zo[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (cc[q] != BSP_FLUID) {
      po[q] = q4v(p0, q);
      ro[q] = q4v(r0, q);
      zo[q] = 0.0f;
      continue;
    }
    po[q] = __fmaf_rn(af, q4v(cu, q), q4v(p0, q));
    ro[q] = __fmaf_rn(-af, q4v(ap, q), q4v(r0, q));
    zo[q] = dinv_apply(ro[q], ns[q]);
    rz += (double)ro[q] * (double)zo[q];
    rr2 += (double)ro[q] * (double)ro[q];
  }
  *reinterpret_cast<float4 *>(a.p + c) = make_float4(po[0], po[1], po[2], po[3]);
  *reinterpret_cast<float4 *>(a.r + c) = make_float4(ro[0], ro[1], ro[2], ro[3]);
  *reinterpret_cast<float4 *>(a.z + c) = make_float4(zo[0], zo[1], zo[2], zo[3]);
}

template <class MaskT>
__global__ void __launch_bounds__(PCG_THREADS) pcg_persistent_kernel(PcgArgs<MaskT> a) {
  __shared__ double sh[32 * 3];
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * (PCG_THREADS / 32) + (threadIdx.x >> 5);
  const int tw = gridDim.x * (PCG_THREADS / 32);
  const int nx = a.nx, ny = a.ny, nz = a.nz, mf = a.mf, ma = a.ma;
  const int64_t rows = (int64_t)nx * ny;
  const int64_t plane = (int64_t)ny * nz;

  // ---- init: b, r = b, z = D^-1 r, p = 0; partial b.b and r.z ------------------
  {
    double v[2] = {0.0, 0.0};
    for (int64_t u = gw; u < rows; u += tw) {
      const int i = (int)(u / ny), j = (int)(u - (int64_t)(u / ny) * ny);
      const int64_t base = u * nz;
      for (int k = lane; k < nz; k += 32) {
        const int64_t c = base + k;
        float b = 0.0f, z = 0.0f;
        if (pcg_cls(a.mask, c, mf, ma) == BSP_FLUID) {
          b = __fmul_rn(a.scale, __ldg(a.div + c));
          z = dinv_apply(b, pcg_nsolid(a.mask, c, i, j, k, nx, ny, nz, mf, ma));
        }
        a.r[c] = b;
        a.z[c] = z;
        a.p[c] = 0.0f;
        v[0] += (double)b * (double)b;
        v[1] += (double)b * (double)z;
      }
    }
    block_partials<2>(v, a.partials, a.stride, sh);
  }
  if (!grid_barrier(a.ctl)) return;
  double tot[3];
  {
    double t2[2];
    grid_totals<2>(a.partials, a.stride, t2, sh);
    tot[0] = t2[0];
    tot[1] = t2[1];
  }
  const double bsq = tot[0];
  double rz = tot[1];
  double alpha = 0.0, beta = 0.0, rz_new = 0.0, rsq = bsq, pAp = 0.0;
  int iters = 0;
  int status = BSP_OK;
  if (!(bsq == bsq) || bsq > 1.0e300) status = BSP_ERR_NONFINITE;
  if (status == BSP_OK && bsq != 0.0) {
    const double tol_sq_bsq = a.tol2 * bsq;
    int it = 0;
    for (it = 0; it < a.max_iter; ++it) {
      float *cur = (it & 1) ? a.ps1 : a.ps0;
      const float *prev = (it & 1) ? a.ps0 : a.ps1;
      const float bf = (float)beta;
      const bool first = (it == 0);
      // ---- phase A: ps = z + beta ps_prev; Ap = A ps; partial ps.Ap -------------
      {
        double v[1] = {0.0};
        if constexpr (std::is_same<MaskT, int32_t>::value) {
          if (a.quad) {
            const int nchunk = (nz + 127) / 128;
            const int64_t units = rows * nchunk;
            for (int64_t un = gw; un < units; un += tw) {
              const int64_t u = un / nchunk;
              const int kc = (int)(un - u * nchunk);
              const int i = (int)(u / ny), j = (int)(u - (int64_t)i * ny);
              const int k = kc * 128 + lane * 4;
              v[0] += pcg_quad_a(a, cur, prev, bf, first, i, j, k, u * nz + k, k < nz);
            }
          }
        }
        for (int64_t u = a.quad ? rows : gw; u < rows; u += tw) {
          const int i = (int)(u / ny), j = (int)(u - (int64_t)(u / ny) * ny);
          const int64_t base = u * nz;
          for (int k = lane; k < nz; k += 32) {
            const int64_t c = base + k;
            if (pcg_cls(a.mask, c, mf, ma) != BSP_FLUID) {
              cur[c] = 0.0f;
              a.Ap[c] = 0.0f;
              continue;
            }
            // z and ps are written inside this kernel: plain (coherent) loads,
            // never the read-only __ldg path.
#define PS(x) (first ? a.z[(x)] : __fmaf_rn(bf, prev[(x)], a.z[(x)]))
            const float psc = PS(c);
#define NB(cond, off)                                                         \
  ((cond) ? ([&]() {                                                          \
    const uint32_t cn = pcg_cls(a.mask, c + (off), mf, ma);                   \
    return cn == BSP_FLUID ? PS(c + (off)) : (cn == BSP_AIR ? 0.0f : psc);    \
  })()                                                                        \
          : 0.0f)
            const float l = NB(i > 0, -plane), rr = NB(i + 1 < nx, plane);
            const float d = NB(j > 0, -(int64_t)nz), up = NB(j + 1 < ny, (int64_t)nz);
            const float bk = NB(k > 0, -1), f = NB(k + 1 < nz, 1);
#undef NB
#undef PS
            const float ap = spmv_update(l, rr, d, up, bk, f, psc);
            cur[c] = psc;
            a.Ap[c] = ap;
            v[0] += (double)psc * (double)ap;
          }
        }
        block_partials<1>(v, a.partials, a.stride, sh);
      }
      if (!grid_barrier(a.ctl)) return;
      {
        double t1[1];
        grid_totals<1>(a.partials, a.stride, t1, sh);
        pAp = t1[0];
      }
      alpha = (pAp == 0.0) ? 0.0 : rz / pAp;
      const float af = (float)alpha;
      // ---- phase B: p += alpha ps; r -= alpha Ap; z = D^-1 r; partial r.z, r.r --
      {
        double v[2] = {0.0, 0.0};
        if constexpr (std::is_same<MaskT, int32_t>::value) {
          if (a.quad) {
            const int nchunk = (nz + 127) / 128;
            const int64_t units = rows * nchunk;
            for (int64_t un = gw; un < units; un += tw) {
              const int64_t u = un / nchunk;
              const int kc = (int)(un - u * nchunk);
              const int i = (int)(u / ny), j = (int)(u - (int64_t)i * ny);
              const int k = kc * 128 + lane * 4;
              pcg_quad_b(a, cur, af, i, j, k, u * nz + k, k < nz, v[0], v[1]);
            }
          }
        }
        for (int64_t u = a.quad ? rows : gw; u < rows; u += tw) {
          const int i = (int)(u / ny), j = (int)(u - (int64_t)(u / ny) * ny);
          const int64_t base = u * nz;
          for (int k = lane; k < nz; k += 32) {
            const int64_t c = base + k;
            if (pcg_cls(a.mask, c, mf, ma) != BSP_FLUID) continue;
            const float pc = __fmaf_rn(af, cur[c], a.p[c]);
            const float rc = __fmaf_rn(-af, a.Ap[c], a.r[c]);
            const float zc = dinv_apply(rc, pcg_nsolid(a.mask, c, i, j, k, nx, ny, nz, mf, ma));
            a.p[c] = pc;
            a.r[c] = rc;
            a.z[c] = zc;
            v[0] += (double)rc * (double)zc;
            v[1] += (double)rc * (double)rc;
          }
        }
        block_partials<2>(v, a.partials + a.stride, a.stride, sh);
      }
      if (!grid_barrier(a.ctl)) return;
      {
        double t2[2];
        grid_totals<2>(a.partials + a.stride, a.stride, t2, sh);
        rz_new = t2[0];
        rsq = t2[1];
      }
      if (it >= 8 && (it % 5) == 0 && rsq < tol_sq_bsq) {
        ++it;
        break;
      }
      beta = (rz == 0.0) ? 0.0 : rz_new / rz;
      rz = rz_new;
    }
    iters = it;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.ctl->iters = iters;
    a.ctl->status = status;
    const double vals[7] = {alpha, beta, rz, rz_new, bsq, rsq, pAp};
#pragma unroll
    for (int q = 0; q < 7; ++q)
      if (a.outs[q]) *a.outs[q] = (float)vals[q];
  }
}

template <class MaskT>
static cudaError_t launch_pcg(PcgArgs<MaskT> &a, int max_blocks, cudaStream_t s) {
  int occ = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &occ, pcg_persistent_kernel<MaskT>, PCG_THREADS, 0);
  if (e != cudaSuccess) return e;
  if (occ <= 0) return cudaErrorCooperativeLaunchTooLarge;
  const int sms = num_sms();
  int per = max_blocks / sms;
  if (per > occ) per = occ;
  int nb = per >= 1 ? per * sms : max_blocks;
  const int64_t rows = (int64_t)a.nx * a.ny;
  const int64_t need = (rows + (PCG_THREADS / 32) - 1) / (PCG_THREADS / 32);
  if (need < nb) nb = (int)(need > 0 ? need : 1);
  a.stride = nb;
  void *args[] = {&a};
  return cudaLaunchCooperativeKernel((const void *)pcg_persistent_kernel<MaskT>, dim3(nb),
                                     dim3(PCG_THREADS), args, 0, s);
}

// BSP_TUNE_PCG_QUAD: 1 (default) runs the four-cell form of the PCG phases
// where it applies, 0 the one-cell form (the same per-cell operations)
bool g_pcg_quad = true;

// dot_workspace layout (>= 4096 bytes): [0,64) GridCtl, [64, 64 + 8*3*nb) partials
constexpr int COMPAT_MAX_BLOCKS = (4096 - 64) / 24;

}  // namespace bsp

using namespace bsp;

extern "C" cudaError_t pressure_solve_pcg_launch(
    float *p_out, const float *div_u, const int *mat, int nx, int ny, int nz, float dx, float dt,
    float rho, int mat_fluid, int mat_air, float pressure_tol, int max_iter, float *ws_b,
    float *ws_r, float *ws_z, float *ws_p_search, float *ws_Ap, float *dot_workspace,
    float *dev_alpha, float *dev_beta, float *dev_rzold, float *dev_rznew, float *dev_bsq,
    float *dev_rsq, float *dev_pAp, int *iter_count_host) {
  if (nx <= 0 || ny <= 0 || nz <= 0) {
    if (iter_count_host) *iter_count_host = 0;
    return cudaSuccess;
  }
  if (((uintptr_t)dot_workspace & 7u) != 0) return cudaErrorInvalidValue;
  GridCtl *ctl = reinterpret_cast<GridCtl *>(dot_workspace);
  cudaError_t e = cudaMemsetAsync(ctl, 0, sizeof(GridCtl), 0);
  if (e != cudaSuccess) return e;
  PcgArgs<int32_t> a{};
  a.p = p_out;
  a.div = div_u;
  a.mask = mat;
  a.r = ws_r;
  a.z = ws_z;
  a.ps0 = ws_p_search;
  a.ps1 = ws_b;  // b is not needed after the first pass: it holds the second search buffer
  a.Ap = ws_Ap;
  a.partials = reinterpret_cast<double *>(reinterpret_cast<char *>(dot_workspace) + 64);
  a.ctl = ctl;
  float *dst[7] = {dev_alpha, dev_beta, dev_rzold, dev_rznew, dev_bsq, dev_rsq, dev_pAp};
  for (int q = 0; q < 7; ++q) a.outs[q] = dst[q];
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.mf = mat_fluid;
  a.ma = mat_air;
  a.max_iter = max_iter < 0 ? 0 : max_iter;
  a.scale = -rho * dx * dx / dt;  // pressure_solve_pcg.cu:137 evaluation order
  a.tol2 = (double)pressure_tol * (double)pressure_tol;
  // vector loads of the four-cell form need 16-byte aligned rows
  a.quad = (nz % 4 == 0 && g_pcg_quad &&
            !(((uintptr_t)p_out | (uintptr_t)mat | (uintptr_t)ws_r | (uintptr_t)ws_z |
               (uintptr_t)ws_p_search | (uintptr_t)ws_b | (uintptr_t)ws_Ap) & 15u))
               ? 1
               : 0;
  e = launch_pcg<int32_t>(a, COMPAT_MAX_BLOCKS, 0);
  if (e != cudaSuccess) return e;
  GridCtl h{};
  e = cudaMemcpy(&h, ctl, sizeof(GridCtl), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  if (h.err != 0) return (cudaError_t)h.err;
  if (h.status != 0) return (cudaError_t)h.status;
  if (iter_count_host) *iter_count_host = h.iters;
  return cudaGetLastError();
}
