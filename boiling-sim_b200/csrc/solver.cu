// solver.cu -- to-tolerance pressure solve: FP64 iterative refinement around a
// multigrid-preconditioned conjugate gradient with reduced-precision storage.
//
// The linear system is the reference's (pressure_solve_pcg.cu:129-139,
// laplacian_spmv.cu:62-143):  A p = b,  (A p)_c = 6 p_c - sum g(n),
// g = p_n (fluid) | 0 (air, Dirichlet) | p_c (solid, Neumann),
// b_c = -rho dx^2 div_c / dt, on fluid cells.  Stopping rule
// ||b - A p||_2 <= tol ||b||_2 (python/boilingsim/config.py:166-176), with the
// residual evaluated in FP64 from an FP64 iterate.
//
// Structure (all on the device; the host only reads a done flag between
// chunks of iterations):
//   outer (FP64):  r = b - A x;  stop if ||r|| <= tol ||b||;
//                  rhat = s r (stored as T);  solve A e ~= rhat;  x += e / s
//   inner (FP32 arithmetic, T storage): CG preconditioned by one V-cycle,
//                  stopped when ||r_inner|| <= eta ||rhat|| or after max_inner.
//   V-cycle (Jacobi smoothing, weight OMEGA, one pre and one post sweep):
//     down l -> l+1: e_l = OMEGA D^-1 r_l (from zero, not stored);
//                    r_{l+1}[C] = 1/2 sum_{fluid children c} (r_l - A_l e_l)[c]
//     coarsest:      COARSE_SWEEPS Jacobi sweeps from zero in one CTA
//     up l+1 -> l:   e^ = OMEGA D^-1 r_l + e_{l+1}[parent];
//                    e_l = e^ + OMEGA D^-1 (r_l - A_l e^)
//   Coarse cells: AIR if any child is air adjacent to fluid, else FLUID if any
//   child is fluid, else SOLID (air away from fluid is treated as solid so
//   thin pot walls never turn into free surfaces at coarse levels).
// All inner products are FP64 with a fixed reduction order.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstring>
#include <mutex>
#include <vector>

#include <cstddef>

#include "bsp_common.cuh"
#include "grid_sync.cuh"
#include "profile.cuh"
#include "solver.cuh"

namespace bsp {

int num_sms();

constexpr float OMEGA = 6.0f / 7.0f;
// BSP_TUNE_FINE_COLUMN: level-0 kernels on the column layout (1) or per row (0)
bool g_fine_col_enabled = true;
// BSP_TUNE_MG_ALPHA: scale of the coarse-grid correction added by every
// prolongation (1 = plain correction; above 1 = over-correction).  Any value
// > 0 keeps the V-cycle a symmetric positive definite preconditioner: the
// coarse part alpha P A_c^-1 R is positive semi-definite and the damped
// Jacobi smoother is convergent.
float g_mg_alpha = 1.0f;
extern bool g_fine_tma_enabled;      // BSP_TUNE_FINE_TMA (mgfine.cu)
extern bool g_coarse_fused_enabled;  // BSP_TUNE_COARSE_FUSED (mgcoarse.cu)
extern bool g_coarse_phases_fused;   // BSP_TUNE_COARSE_PHASES (mgcoarse.cu)
extern bool g_coarse_tail_smem;      // BSP_TUNE_COARSE_TAIL (mgcoarse.cu)
// BSP_TUNE_COARSE_SPLIT: S = 1, 2 (default) or 3 runs levels 1 .. S of the
// V-cycle with the column tile kernels of level 0 (restriction, prolongation
// and smoothing) and the one-launch coarse cycle below them, as far as those
// levels take the column layout and the cooperative launch is available; 0
// runs every coarse level in the one launch.  Measured at 384x384x256 with two
// sweeps on level 1: 12.79 ms (S = 1), 12.60 ms (S = 2) per solve; with the
// one-cluster cycle below: 11.77 ms (S = 2), 11.56 ms (S = 3).
int g_coarse_split = 3;
// BSP_TUNE_L1_SWEEPS (split mode): smoothing sweeps on level 1 before the
// restriction and after the prolongation, 1 or 2 (default; symmetric, so the
// V-cycle stays an SPD preconditioner).  Measured at 384x384x256 (FP16
// storage): 36 -> 31 inner iterations, 13.8 -> 12.8 ms per solve.
int g_l1_sweeps = 2;
// BSP_TUNE_L0_TRILINEAR: 1 uses trilinear transfers between levels 0 and 1
// (fused TMA path, level 1 exactly half of level 0 in k), 0 piecewise-constant
bool g_l0_trilinear = false;
// BSP_TUNE_FUSE_SCALARS: 1 runs the inner check, beta and alpha in the last CTA
// of the level-0 TMA kernel before each (no one-block launches); 0 (default)
// launches them.  Measured at 384x384x256: 13.53 ms per solve fused against
// 13.21 ms with the launches -- every CTA's fence and ticket before it exits
// costs each level-0 kernel about 7 us, more than the launches it saves.
bool g_fuse_scalars = false;
extern int g_fine_ctas;  // BSP_TUNE_FINE_CTAS (mgfine.cu)
extern bool g_pdl;       // BSP_TUNE_PDL (mgfine.cu)
extern int g_coarse_cluster;  // BSP_TUNE_COARSE_CLUSTER (mgcoarse.cu)
extern int g_cluster_tail_cells;  // BSP_TUNE_CLUSTER_TAIL_CELLS (mgcoarse.cu)
extern int g_downu_blocks;        // BSP_TUNE_DOWNU_BLOCKS (mgfine.cu)
extern bool g_coarse_cluster_tail_smem;  // BSP_TUNE_CLUSTER_TAIL (mgcoarse.cu)
extern int g_tri_cpc;  // BSP_TUNE_TRI_CPC (mgfine.cu)
// BSP_TUNE_FUSE_UPDATE: CG update fused into the next level-0 restriction
bool g_fuse_update_enabled = true;
// BSP_TUNE_TEST_BARRIER_ERROR (tests only): the next host-driven solve starts
// with the coarse-cycle barrier's error word set
bool g_test_barrier_error = false;
constexpr int COARSE_SWEEPS = 64;
constexpr int RED_THREADS = 256;

// ---- storage conversions --------------------------------------------------------
__device__ __forceinline__ float ld(const float *p, int64_t c) { return p[c]; }
__device__ __forceinline__ float ld(const __half *p, int64_t c) { return __half2float(p[c]); }
__device__ __forceinline__ float ld(const __nv_bfloat16 *p, int64_t c) {
  return __bfloat162float(p[c]);
}
__device__ __forceinline__ void stv(float *p, int64_t c, float v) { p[c] = v; }
__device__ __forceinline__ void stv(__half *p, int64_t c, float v) { p[c] = __float2half_rn(v); }
__device__ __forceinline__ void stv(__nv_bfloat16 *p, int64_t c, float v) {
  p[c] = __float2bfloat16_rn(v);
}

// value as it reads back after a store through T
__device__ __forceinline__ float rnd(float v, const float *) { return v; }
__device__ __forceinline__ float rnd(float v, const __half *) {
  return __half2float(__float2half_rn(v));
}
__device__ __forceinline__ float rnd(float v, const __nv_bfloat16 *) {
  return __bfloat162float(__float2bfloat16_rn(v));
}

__device__ __forceinline__ uint32_t mk(const uint8_t *m, int64_t c) { return __ldg(m + c); }

// Row-unit iteration: one warp per (i, j) row, lanes striding over k.
struct RowIter {
  int64_t u, rows, step;
  __device__ RowIter(int nx, int ny)
      : u((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)),
        rows((int64_t)nx * ny),
        step((int64_t)gridDim.x * (blockDim.x >> 5)) {}
};

// ---- deterministic block partials ------------------------------------------------
template <int K>
__device__ __forceinline__ void store_partials(double (&v)[K], double *partials) {
  __shared__ double sh[K][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < K; ++q)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < K; ++q) sh[q][warp] = v[q];
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[threadIdx.x][w];
    partials[threadIdx.x * PARTIAL_STRIDE + blockIdx.x] = s;
  }
}

template <int K>
__device__ __forceinline__ void store_partials_max(double (&v)[K], double m, double *partials) {
  // slot K holds a max instead of a sum
  __shared__ double shm[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) shm[warp] = m;
  store_partials<K>(v, partials);
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s = fmax(s, shm[w]);
    partials[K * PARTIAL_STRIDE + blockIdx.x] = s;
  }
}

// Sum of slot q over nblocks partials, fixed order; valid in thread 0 of a
// RED_THREADS-thread block.
__device__ double reduce_slot(const double *partials, int q, int nblocks, bool is_max) {
  __shared__ double sh[RED_THREADS];
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += RED_THREADS) {
    const double v = partials[q * PARTIAL_STRIDE + b];
    s = is_max ? fmax(s, v) : s + v;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = is_max ? fmax(sh[threadIdx.x], sh[threadIdx.x + w])
                                                  : sh[threadIdx.x] + sh[threadIdx.x + w];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// ---- level setup ------------------------------------------------------------------
// Effective class: fluid, air adjacent to fluid (Dirichlet), otherwise solid.
__global__ void eff_class_kernel(uint8_t *__restrict__ out, const uint8_t *__restrict__ cls_in,
                                 int nx, int ny, int nz) {
  RowIter it(nx, ny);
  const int lane = threadIdx.x & 31;
  const int64_t plane = (int64_t)ny * nz;
  for (; it.u < it.rows; it.u += it.step) {
    const int i = (int)(it.u / ny), j = (int)(it.u % ny);
    for (int k = lane; k < nz; k += 32) {
      const int64_t c = it.u * nz + k;
      uint32_t cl = mcls(cls_in[c]);
      if (cl == BSP_AIR) {
        bool adj = false;
#define FL(cond, off) adj |= (cond) && mcls(cls_in[c + (off)]) == BSP_FLUID
        FL(i > 0, -plane);
        FL(i + 1 < nx, plane);
        FL(j > 0, -(int64_t)nz);
        FL(j + 1 < ny, (int64_t)nz);
        FL(k > 0, -1);
        FL(k + 1 < nz, 1);
#undef FL
        if (!adj) cl = BSP_SOLID;
      }
      out[c] = (uint8_t)enc_cls(cl);
    }
  }
}

// Coarse class from 2x2x2 children of effective classes.
__global__ void coarsen_kernel(uint8_t *__restrict__ coarse, const uint8_t *__restrict__ fine,
                               int fx, int fy, int fz, int cx, int cy, int cz) {
  RowIter it(cx, cy);
  const int lane = threadIdx.x & 31;
  for (; it.u < it.rows; it.u += it.step) {
    const int I = (int)(it.u / cy), J = (int)(it.u % cy);
    for (int K = lane; K < cz; K += 32) {
      bool air = false, fl = false;
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          for (int d = 0; d < 2; ++d) {
            const int i = 2 * I + a, j = 2 * J + b, k = 2 * K + d;
            if (i < fx && j < fy && k < fz) {
              const uint32_t cl = mcls(fine[((int64_t)i * fy + j) * fz + k]);
              air |= cl == BSP_AIR;
              fl |= cl == BSP_FLUID;
            }
          }
      coarse[it.u * cz + K] = (uint8_t)enc_cls(air ? BSP_AIR : (fl ? BSP_FLUID : BSP_SOLID));
    }
  }
}

// Add the solid-neighbour count (bits 2-4); out-of-range neighbours are air.
__global__ void nsolid_kernel(uint8_t *__restrict__ m, int nx, int ny, int nz) {
  RowIter it(nx, ny);
  const int lane = threadIdx.x & 31;
  const int64_t plane = (int64_t)ny * nz;
  for (; it.u < it.rows; it.u += it.step) {
    const int i = (int)(it.u / ny), j = (int)(it.u % ny);
    for (int k = lane; k < nz; k += 32) {
      const int64_t c = it.u * nz + k;
      uint32_t ns = 0;
#define SO(cond, off) ns += ((cond) && mcls(m[c + (off)]) == BSP_SOLID) ? 1u : 0u
      SO(i > 0, -plane);
      SO(i + 1 < nx, plane);
      SO(j > 0, -(int64_t)nz);
      SO(j + 1 < ny, (int64_t)nz);
      SO(k > 0, -1);
      SO(k + 1 < nz, 1);
#undef SO
      m[c] = (uint8_t)((m[c] & (BSP_MFLUID | BSP_MSOLID)) | ns);
    }
  }
}

// ---- stencil helpers ----------------------------------------------------------------
__device__ __forceinline__ float dg(uint32_t mb) { return 6.0f - (float)mnsolid(mb); }
// OMEGA / (6 - n_solid) by the approximate division (same as the level-0
// column kernels); 0 where the diagonal vanishes.
__device__ __forceinline__ float wdinv(uint32_t mb) {
  const float d = dg(mb);
  return d > 0.0f ? __fdividef(OMEGA, d) : 0.0f;
}

// e = OMEGA r / D on a fluid cell.
template <class T>
__device__ __forceinline__ float pre_e(const T *r, int64_t c, uint32_t mb) {
  return ld(r, c) * wdinv(mb);
}

// ---- V-cycle kernels ----------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) mg_down_kernel(Level<T> f, Level<T> co,
                                                      const SolverState *st) {
  if (st->inner_done) return;
  RowIter it(co.nx, co.ny);
  const int lane = threadIdx.x & 31;
  const int64_t plane = (int64_t)f.ny * f.nz;
  for (; it.u < it.rows; it.u += it.step) {
    const int I = (int)(it.u / co.ny), J = (int)(it.u % co.ny);
    for (int K = lane; K < co.nz; K += 32) {
      const int64_t C = it.u * co.nz + K;
      float acc = 0.0f;
      if (mcls(mk(co.mask, C)) == BSP_FLUID) {
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b)
            for (int d = 0; d < 2; ++d) {
              const int i = 2 * I + a, j = 2 * J + b, k = 2 * K + d;
              if (i >= f.nx || j >= f.ny || k >= f.nz) continue;
              const int64_t c = ((int64_t)i * f.ny + j) * f.nz + k;
              const uint32_t mc = mk(f.mask, c);
              if (mcls(mc) != BSP_FLUID) continue;
              const float ec = pre_e(f.r, c, mc);
#define NB(cond, off)                                                          \
  ((cond) ? ([&]() {                                                           \
    const uint32_t mn = mk(f.mask, c + (off));                                 \
    const uint32_t cn = mcls(mn);                                              \
    return cn == BSP_FLUID ? pre_e(f.r, c + (off), mn) : (cn == BSP_AIR ? 0.0f : ec); \
  })()                                                                         \
          : 0.0f)
              const float s = NB(i > 0, -plane) + NB(i + 1 < f.nx, plane) +
                              NB(j > 0, -(int64_t)f.nz) + NB(j + 1 < f.ny, (int64_t)f.nz) +
                              NB(k > 0, -1) + NB(k + 1 < f.nz, 1);
#undef NB
              acc += ld(f.r, c) - (6.0f * ec - s);
            }
        acc *= 0.5f;
      }
      stv(co.r, C, acc);
    }
  }
}

// Dense inverse of the coarsest operator, once per geometry: A (FP64, n x n,
// diagonal 6 - n_solid, -1 to fluid neighbours, identity rows on non-fluid
// cells) is inverted in place by Gauss-Jordan elimination without pivoting
// (the fluid block is symmetric positive definite when every fluid component
// touches a Dirichlet cell).  *flag = 1 on success; 0 if a pivot is not
// positive (a closed Neumann island), and the coarse solve then falls back to
// Jacobi sweeps.  One CTA; A lives in the workspace.
template <class T>
__global__ void __launch_bounds__(1024) coarse_invert_kernel(Level<T> L, double *A, float *minv,
                                                             int *flag) {
  const int n = L.nx * L.ny * L.nz;
  const int plane = L.ny * L.nz;
  __shared__ double fcol[COARSEST_CELLS];
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) A[q] = 0.0;
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    const uint32_t mc = mk(L.mask, c);
    if (mcls(mc) != BSP_FLUID) {
      A[(int64_t)c * n + c] = 1.0;
      continue;
    }
    A[(int64_t)c * n + c] = 6.0 - (double)mnsolid(mc);
    const int k = c % L.nz, j = (c / L.nz) % L.ny, i = c / plane;
#define OFF(cond, off) \
  if ((cond) && mcls(mk(L.mask, c + (off))) == BSP_FLUID) A[(int64_t)c * n + c + (off)] = -1.0
    OFF(i > 0, -plane);
    OFF(i + 1 < L.nx, plane);
    OFF(j > 0, -L.nz);
    OFF(j + 1 < L.ny, L.nz);
    OFF(k > 0, -1);
    OFF(k + 1 < L.nz, 1);
#undef OFF
  }
  __syncthreads();
  for (int kp = 0; kp < n; ++kp) {
    const double piv = A[(int64_t)kp * n + kp];
    if (!(piv > 1e-12)) {  // uniform: every thread read the same value
      if (threadIdx.x == 0) *flag = 0;
      return;
    }
    __syncthreads();
    for (int jj = threadIdx.x; jj < n; jj += blockDim.x) {
      const double v = jj == kp ? 1.0 : A[(int64_t)kp * n + jj];
      A[(int64_t)kp * n + jj] = v / piv;
    }
    for (int ii = threadIdx.x; ii < n; ii += blockDim.x) fcol[ii] = A[(int64_t)ii * n + kp];
    __syncthreads();
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
      const int ii = q / n, jj = q - ii * n;
      if (ii == kp) continue;
      const double a = jj == kp ? 0.0 : A[q];
      A[q] = a - fcol[ii] * A[(int64_t)kp * n + jj];
    }
    __syncthreads();
  }
  // stored symmetric (A^-1 is; Gauss-Jordan rounding is not), so the coarsest
  // solve keeps the V-cycle a symmetric preconditioner
  for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
    const int r = q / n, c = q - r * n;
    minv[q] = (float)(0.5 * (A[q] + A[(int64_t)c * n + r]));
  }
  if (threadIdx.x == 0) *flag = 1;
}

// Coarsest level: one CTA.  With the dense inverse, e = M r (M symmetric, so
// thread t reads column t with coalesced loads); otherwise COARSE_SWEEPS
// Jacobi sweeps from zero with the level in shared memory.
template <class T>
__global__ void __launch_bounds__(512) mg_coarse_kernel(Level<T> L, const float *minv,
                                                        const int *direct,
                                                        const SolverState *stt) {
  if (stt->inner_done) return;
  extern __shared__ float sm[];
  const int n = L.nx * L.ny * L.nz;
  float *e0 = sm, *e1 = sm + n, *rr = sm + 2 * n;
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    e0[c] = 0.0f;
    rr[c] = ld(L.r, c);
  }
  __syncthreads();
  if (*direct) {
    // n <= COARSEST_CELLS <= blockDim: split the j sum of each output over
    // blockDim / n threads, then combine in a fixed order
    __shared__ float part[512];
    const int parts = blockDim.x / n;
    const int t = threadIdx.x % n, pi = threadIdx.x / n;
    if (pi < parts) {
      const int j0 = (n * pi) / parts, j1 = (n * (pi + 1)) / parts;
      float acc = 0.0f;
      for (int jj = j0; jj < j1; ++jj) acc = fmaf(minv[(int64_t)jj * n + t], rr[jj], acc);
      part[pi * n + t] = acc;
    }
    __syncthreads();
    if (threadIdx.x < n) {
      float acc = 0.0f;
      for (int q = 0; q < parts; ++q) acc += part[q * n + threadIdx.x];
      stv(L.e, threadIdx.x, mcls(mk(L.mask, threadIdx.x)) == BSP_FLUID ? acc : 0.0f);
    }
    return;
  }
  const int plane = L.ny * L.nz;
  for (int s = 0; s < COARSE_SWEEPS; ++s) {
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      const uint32_t mc = mk(L.mask, c);
      if (mcls(mc) != BSP_FLUID) {
        e1[c] = 0.0f;
        continue;
      }
      const int k = c % L.nz, j = (c / L.nz) % L.ny, i = c / plane;
      const float ec = e0[c];
#define NB(cond, off)                                                                    \
  ((cond) ? (mcls(mk(L.mask, c + (off))) == BSP_FLUID                                    \
                 ? e0[c + (off)]                                                         \
                 : (mcls(mk(L.mask, c + (off))) == BSP_AIR ? 0.0f : ec))                 \
          : 0.0f)
      const float sum = NB(i > 0, -plane) + NB(i + 1 < L.nx, plane) + NB(j > 0, -L.nz) +
                        NB(j + 1 < L.ny, L.nz) + NB(k > 0, -1) + NB(k + 1 < L.nz, 1);
#undef NB
      e1[c] = ec + (rr[c] - (6.0f * ec - sum)) / dg(mc);
    }
    __syncthreads();
    float *t = e0;
    e0 = e1;
    e1 = t;
  }
  for (int c = threadIdx.x; c < n; c += blockDim.x) stv(L.e, c, e0[c]);
}

// Up: e^ = OMEGA D^-1 r + e_coarse[parent]; e = e^ + OMEGA D^-1 (r - A e^).
// Writes e to `out` (the level's e, or z at level 0) and, at level 0, the
// partial r.z.
template <class T, bool FINE>
__global__ void __launch_bounds__(256) mg_up_kernel(Level<T> f, Level<T> co, T *out,
                                                    double *partials, const SolverState *st,
                                                    float alpha) {
  if (st->inner_done) return;
  RowIter it(f.nx, f.ny);
  const int lane = threadIdx.x & 31;
  const int64_t plane = (int64_t)f.ny * f.nz;
  double rz = 0.0;
  for (; it.u < it.rows; it.u += it.step) {
    const int i = (int)(it.u / f.ny), j = (int)(it.u % f.ny);
    for (int k = lane; k < f.nz; k += 32) {
      const int64_t c = it.u * f.nz + k;
      const uint32_t mc = mk(f.mask, c);
      if (mcls(mc) != BSP_FLUID) {
        stv(out, c, 0.0f);
        continue;
      }
      auto ehat = [&](int ii, int jj, int kk, int64_t cc, uint32_t mb) {
        const int64_t P = ((int64_t)(ii >> 1) * co.ny + (jj >> 1)) * co.nz + (kk >> 1);
        return fmaf(alpha, ld(co.e, P), pre_e(f.r, cc, mb));
      };
      const float ec = ehat(i, j, k, c, mc);
#define NB(cond, di, dj, dk, off)                                                     \
  ((cond) ? ([&]() {                                                                  \
    const uint32_t mn = mk(f.mask, c + (off));                                        \
    const uint32_t cn = mcls(mn);                                                     \
    return cn == BSP_FLUID ? ehat(i + di, j + dj, k + dk, c + (off), mn)              \
                           : (cn == BSP_AIR ? 0.0f : ec);                             \
  })()                                                                                \
          : 0.0f)
      const float s = NB(i > 0, -1, 0, 0, -plane) + NB(i + 1 < f.nx, 1, 0, 0, plane) +
                      NB(j > 0, 0, -1, 0, -(int64_t)f.nz) +
                      NB(j + 1 < f.ny, 0, 1, 0, (int64_t)f.nz) + NB(k > 0, 0, 0, -1, -1) +
                      NB(k + 1 < f.nz, 0, 0, 1, 1);
#undef NB
      const float rc = ld(f.r, c);
      const float e = fmaf(rc - (6.0f * ec - s), wdinv(mc), ec);
      stv(out, c, e);
      if (FINE) rz += (double)rc * (double)ld(out, c);
    }
  }
  if (FINE) {
    double v[1] = {rz};
    store_partials<1>(v, partials);
  }
}

// ---- CG kernels ---------------------------------------------------------------------
// ps = z + beta ps_prev (first iteration: ps = z), formed at the centre and the
// neighbours; Ap = A ps; partial ps.Ap.
template <class T>
__global__ void __launch_bounds__(256) cg_ps_ap_kernel(int nx, int ny, int nz,
                                                       const uint8_t *mask, const T *z,
                                                       const T *prev, T *cur, T *Ap,
                                                       double *partials, const SolverState *st) {
  if (st->inner_done) return;
  const bool first = st->inner_it == 0;
  const float beta = (float)st->beta;
  RowIter it(nx, ny);
  const int lane = threadIdx.x & 31;
  const int64_t plane = (int64_t)ny * nz;
  double pap = 0.0;
  for (; it.u < it.rows; it.u += it.step) {
    const int i = (int)(it.u / ny), j = (int)(it.u % ny);
    for (int k = lane; k < nz; k += 32) {
      const int64_t c = it.u * nz + k;
      if (mcls(mk(mask, c)) != BSP_FLUID) {
        stv(cur, c, 0.0f);
        stv(Ap, c, 0.0f);
        continue;
      }
#define PS(x) (first ? ld(z, (x)) : rnd(fmaf(beta, ld(prev, (x)), ld(z, (x))), cur))
      const float psc = PS(c);
#define NB(cond, off)                                                        \
  ((cond) ? ([&]() {                                                         \
    const uint32_t cn = mcls(mk(mask, c + (off)));                           \
    return cn == BSP_FLUID ? PS(c + (off)) : (cn == BSP_AIR ? 0.0f : psc);   \
  })()                                                                       \
          : 0.0f)
      const float s = NB(i > 0, -plane) + NB(i + 1 < nx, plane) + NB(j > 0, -(int64_t)nz) +
                      NB(j + 1 < ny, (int64_t)nz) + NB(k > 0, -1) + NB(k + 1 < nz, 1);
#undef NB
#undef PS
      stv(cur, c, psc);
      const float psq = ld(cur, c);  // the stored (possibly rounded) direction
      const float ap = 6.0f * psq - s;
      stv(Ap, c, ap);
      pap += (double)psq * (double)ld(Ap, c);
    }
  }
  double v[1] = {pap};
  store_partials<1>(v, partials);
}

// e += alpha ps; r -= alpha Ap; partial r.r
template <class T>
__global__ void __launch_bounds__(256) cg_update_kernel(int64_t n, const uint8_t *mask,
                                                        float *e, T *r, const T *ps,
                                                        const T *Ap, double *partials,
                                                        const SolverState *st) {
  if (st->inner_done) return;
  const float alpha = (float)st->alpha;
  double rr = 0.0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (mcls(mk(mask, c)) != BSP_FLUID) continue;
    e[c] = fmaf(alpha, ld(ps, c), e[c]);
    stv(r, c, fmaf(-alpha, ld(Ap, c), ld(r, c)));
    const float rv = ld(r, c);
    rr += (double)rv * (double)rv;
  }
  double v[1] = {rr};
  store_partials<1>(v, partials);
}

// ---- outer (FP64) kernels --------------------------------------------------------------
// r = b - A x in FP64 on fluid cells; partial ||r||^2 and max|r|; if WRITE,
// rhat = scale r (stored as T), inner r = rhat, e = 0.
template <class T, bool WRITE>
__global__ void __launch_bounds__(256) residual64_kernel(int nx, int ny, int nz,
                                                         const uint8_t *mask, const float *div,
                                                         const double *x, double bscale,
                                                         T *rhat, float *e, double *partials,
                                                         const SolverState *st) {
  if (st->done) return;
  if (!WRITE && st->norm_cached) return;  // x = 0: the ||b|| pass's partials stand
  const double scale = st->scale;
  RowIter it(nx, ny);
  const int lane = threadIdx.x & 31;
  const int64_t plane = (int64_t)ny * nz;
  double rr = 0.0, rmax = 0.0;
  for (; it.u < it.rows; it.u += it.step) {
    const int i = (int)(it.u / ny), j = (int)(it.u % ny);
    for (int k = lane; k < nz; k += 32) {
      const int64_t c = it.u * nz + k;
      const uint32_t mc = mk(mask, c);
      double r = 0.0;
      if (mcls(mc) == BSP_FLUID) {
        const double xc = x[c];
#define NB(cond, off)                                                        \
  ((cond) ? ([&]() {                                                         \
    const uint32_t cn = mcls(mk(mask, c + (off)));                           \
    return cn == BSP_FLUID ? x[c + (off)] : (cn == BSP_AIR ? 0.0 : xc);      \
  })()                                                                       \
          : 0.0)
        const double s = NB(i > 0, -plane) + NB(i + 1 < nx, plane) + NB(j > 0, -(int64_t)nz) +
                         NB(j + 1 < ny, (int64_t)nz) + NB(k > 0, -1) + NB(k + 1 < nz, 1);
#undef NB
        r = bscale * (double)__ldg(div + c) - (6.0 * xc - s);
      }
      rr += r * r;
      rmax = fmax(rmax, fabs(r));
      if (WRITE) {
        stv(rhat, c, (float)(r * scale));
        e[c] = 0.0f;
      }
    }
  }
  double v[1] = {rr};
  store_partials_max<1>(v, rmax, partials);
}

// x += e / scale (FP64); at the end the float output is refreshed too.
__global__ void xupdate_kernel(int64_t n, double *x, const float *e, float *p_out,
                               SolverState *st) {
  if (st->done && !st->finalize) return;
  const double inv = 1.0 / st->scale;
  const bool add = !st->done;
  if (add && blockIdx.x == 0 && threadIdx.x == 0) st->x_zero = 0;  // read by later passes only
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    double v = x[c];
    if (add) {
      v += (double)e[c] * inv;
      x[c] = v;
    }
    if (p_out) p_out[c] = (float)v;
  }
}

// ---- scalar (control) kernels, one block --------------------------------------------
// Outer check after a residual pass.  Sets done / status, scale for rhat.
__global__ void __launch_bounds__(RED_THREADS) outer_check_kernel(SolverState *st,
                                                                  const double *partials,
                                                                  int nblocks, int fp32_store) {
  if (st->done) return;
  const double rr = reduce_slot(partials, 0, nblocks, false);
  const double rmax = reduce_slot(partials, 1, nblocks, true);
  if (threadIdx.x != 0) return;
  st->norm_cached = 0;  // later outer passes see a nonzero iterate
  if (st->dev_error) {
    st->status = BSP_ERR_TIMEOUT;
    st->done = 1;
    return;
  }
  st->r64_norm2 = rr;
  st->rel = st->b_norm2 > 0.0 ? sqrt(rr / st->b_norm2) : 0.0;
  if (!(rr == rr) || rr > 1e300) {
    st->status = BSP_ERR_NONFINITE;
    st->done = 1;
    return;
  }
  if (st->b_norm2 == 0.0 || st->rel <= st->tol) {
    st->done = 1;
    st->status = BSP_OK;
    return;
  }
  if (st->outer_it >= st->max_outer) {
    st->done = 1;
    st->status = BSP_NOT_CONVERGED;
    return;
  }
  // FP32 storage: scale 1/||r||_inf keeps rhat O(1); half precision: the same
  // keeps |rhat| <= 1 so FP16 never overflows on the right-hand side.
  st->scale = rmax > 0.0 ? 1.0 / rmax : 1.0;
  (void)fp32_store;
  st->inner_it = 0;
  st->inner_done = 0;
  st->pending = 0;
  st->rhat_norm2 = rr * st->scale * st->scale;
  // Do not over-solve the last pass: an inner reduction by
  // 0.5 tol ||b|| / ||r|| already meets the outer target.
  st->eta_eff = fmax(st->eta, 0.5 * st->tol * sqrt(st->b_norm2 / rr));
  st->outer_it += 1;
}

__global__ void __launch_bounds__(RED_THREADS) beta_kernel(SolverState *st,
                                                           const double *partials, int nblocks) {
  pdl_wait();
  pdl_trigger();
  if (st->inner_done) return;
  const double rz = reduce_slot(partials, 0, nblocks, false);
  if (threadIdx.x != 0) return;
  apply_beta(st, rz);
}

__global__ void __launch_bounds__(RED_THREADS) alpha_kernel(SolverState *st,
                                                            const double *partials, int nblocks) {
  pdl_wait();
  pdl_trigger();
  if (st->inner_done) return;
  const double pap = reduce_slot(partials, 0, nblocks, false);
  if (threadIdx.x != 0) return;
  apply_alpha(st, pap);  // applied by the next iteration's fused restriction, if any
}

// Inner check after the restriction that applied the pending CG update (the
// update of iteration q is fused into the restriction of iteration q + 1):
// the same test as inner_check_kernel on ||r||^2 of the updated residual.  No
// pending update (first iteration of a refinement pass): nothing to test.
__global__ void __launch_bounds__(RED_THREADS) inner_check_fused_kernel(SolverState *st,
                                                                        const double *partials,
                                                                        int nblocks) {
  pdl_wait();
  pdl_trigger();
  if (st->inner_done) return;
  const double rr = reduce_slot(partials, 0, nblocks, false);
  if (threadIdx.x != 0) return;
  apply_inner_check(st, rr);
}

__global__ void __launch_bounds__(RED_THREADS) inner_check_kernel(SolverState *st,
                                                                  const double *partials,
                                                                  int nblocks) {
  if (st->inner_done) return;
  const double rr = reduce_slot(partials, 0, nblocks, false);
  if (threadIdx.x != 0) return;
  st->inner_it += 1;
  st->total_inner += 1;
  st->rr_inner = rr;
  if (st->dev_error) {
    st->status = BSP_ERR_TIMEOUT;
    st->inner_done = 1;
    st->done = 1;
    return;
  }
  if (!(rr == rr) || rr <= st->eta_eff * st->eta_eff * st->rhat_norm2 ||
      st->inner_it >= st->max_inner || st->alpha == 0.0)
    st->inner_done = 1;
}

// ---- host side ----------------------------------------------------------------------
static inline int row_blocks(int64_t rows) {
  int64_t b = (rows + 7) / 8;
  int64_t cap = (int64_t)num_sms() * 8;
  if (cap > PARTIAL_STRIDE) cap = PARTIAL_STRIDE;
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}
static inline int flat_blocks(int64_t n) {
  int64_t b = (n + 255) / 256;
  int64_t cap = (int64_t)num_sms() * 8;
  if (cap > PARTIAL_STRIDE) cap = PARTIAL_STRIDE;
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

static inline size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

int build_hierarchy(int nx, int ny, int nz, int *dims /* 3*MAX_LEVELS */) {
  int L = 0;
  int x = nx, y = ny, z = nz;
  for (;;) {
    dims[3 * L] = x;
    dims[3 * L + 1] = y;
    dims[3 * L + 2] = z;
    ++L;
    if (L == MAX_LEVELS) break;
    // at least two levels: the level-0 up-pass produces z and its r.z partial
    if (L >= 2 && (int64_t)x * y * z <= COARSEST_CELLS) break;
    x = (x + 1) / 2;
    y = (y + 1) / 2;
    z = (z + 1) / 2;
  }
  return L;
}

size_t storage_bytes(int storage) { return storage == BSP_STORE_FP32 ? 4 : 2; }

// Workspace layout (all 256-byte aligned):
//   SolverState | partials (3 * PARTIAL_STRIDE doubles) | x (n doubles) | e (n floats)
//   | z, ps0, ps1, Ap, r, r2 (n T each) | per level l >= 1: mask, r, e (T)
//   | per level l >= 1 ... ; level-0 effective-class scratch reuses the level-1 slot order.
//   | level-0 parent patterns of the trilinear transfers (n bytes)
//   | coarsest-level dense inverse (float), its FP64 build scratch, direct flag
//   | per-level column-tile fluid flags (PARTIAL_STRIDE bytes per level)
//   | FP32 scratch and grid-barrier word of the coarse-cycle kernel
struct Layout {
  size_t state, partials, x, e, z, ps0, ps1, Ap, r, r2, lvl_mask[MAX_LEVELS], lvl_r[MAX_LEVELS],
      lvl_e[MAX_LEVELS], eff0, ppat, cinv, cA, cflag, tflags, cscratch, cctl, total;
  int L, dims[3 * MAX_LEVELS];
};

Layout make_layout(int nx, int ny, int nz, int storage) {
  Layout lo{};
  const size_t n = (size_t)nx * ny * nz, ts = storage_bytes(storage);
  size_t off = 0;
  auto take = [&](size_t b) {
    size_t o = off;
    off += al256(b);
    return o;
  };
  lo.state = take(sizeof(SolverState));
  lo.partials = take(sizeof(double) * 3 * PARTIAL_STRIDE);
  lo.x = take(8 * n);
  lo.e = take(4 * n);
  lo.z = take(ts * n);
  lo.ps0 = take(ts * n);
  lo.ps1 = take(ts * n);
  lo.Ap = take(ts * n);
  lo.r = take(ts * n);
  lo.r2 = take(ts * n);  // second level-0 residual buffer (fused CG update)
  lo.eff0 = take(n);
  lo.ppat = take(n);  // level-0 parent patterns of the trilinear transfers
  lo.L = build_hierarchy(nx, ny, nz, lo.dims);
  for (int l = 1; l < lo.L; ++l) {
    const size_t nl = (size_t)lo.dims[3 * l] * lo.dims[3 * l + 1] * lo.dims[3 * l + 2];
    lo.lvl_mask[l] = take(nl);
    lo.lvl_r[l] = take(ts * nl);
    lo.lvl_e[l] = take(ts * nl);
  }
  {
    const int l = lo.L - 1;
    size_t nc = (size_t)lo.dims[3 * l] * lo.dims[3 * l + 1] * lo.dims[3 * l + 2];
    if (nc > (size_t)COARSEST_CELLS) nc = 0;  // no direct solve: Jacobi sweeps
    lo.cinv = take(sizeof(float) * nc * nc + 4);
    lo.cA = take(sizeof(double) * nc * nc + 8);
    lo.cflag = take(sizeof(int));
  }
  lo.tflags = take((size_t)MAX_LEVELS * PARTIAL_STRIDE);  // column-tile fluid flags per level
  lo.cscratch = take(sizeof(float) * coarse_cycle_scratch_floats(lo.dims, lo.L));
  lo.cctl = take(64);  // grid barrier of the coarse-cycle kernel
  lo.total = off;
  return lo;
}

template <class T>
struct Ctx {
  Layout lo;
  char *base;
  SolverState *st;
  double *partials;
  Level<T> lv[MAX_LEVELS];
  int nx, ny, nz;
  int64_t n;
  const uint8_t *mask0;
  bool col;  // level-0 kernels on the column layout (nz % 4 == 0, aligned mask)
  // the coarse levels may run as one cooperative kernel, which needs the
  // whole GPU: not while other instances' kernels run beside it (batched
  // graphs with parallel branches)
  bool coop = true;
  // the CG update of iteration q runs inside the level-0 restriction of
  // iteration q + 1 (TMA path); the residual then alternates between r and r2
  bool fuse = false;
  // trilinear transfers between levels 0 and 1 (BSP_TUNE_L0_TRILINEAR, on the
  // fused TMA path): the scaled residual goes through z (free between the
  // restriction and the prolongation), patterns in lo.ppat
  bool tri = false;
  const float *tab = nullptr;
  T *r_write() const { return fuse ? (T *)(base + lo.r2) : lv[0].r; }  // rhat target
};

template <class T>
Ctx<T> make_ctx(void *ws, const uint8_t *mask, int nx, int ny, int nz, int storage) {
  Ctx<T> cx{};
  cx.lo = make_layout(nx, ny, nz, storage);
  cx.base = (char *)ws;
  cx.st = (SolverState *)(cx.base + cx.lo.state);
  cx.partials = (double *)(cx.base + cx.lo.partials);
  cx.nx = nx;
  cx.ny = ny;
  cx.nz = nz;
  cx.n = (int64_t)nx * ny * nz;
  cx.mask0 = mask;
  cx.col = (nz % 4 == 0) && (((uintptr_t)mask & 15u) == 0) && g_fine_col_enabled &&
           fine_grid_blocks(nx, ny, nz) <= PARTIAL_STRIDE;
  cx.fuse = cx.col && g_fuse_update_enabled && fine_tma_available(nz);
  for (int l = 0; l < cx.lo.L; ++l) {
    Level<T> &L = cx.lv[l];
    L.nx = cx.lo.dims[3 * l];
    L.ny = cx.lo.dims[3 * l + 1];
    L.nz = cx.lo.dims[3 * l + 2];
    if (l == 0) {
      L.mask = mask;
      L.r = (T *)(cx.base + cx.lo.r);
      L.e = (T *)(cx.base + cx.lo.z);
    } else {
      L.mask = (uint8_t *)(cx.base + cx.lo.lvl_mask[l]);
      L.r = (T *)(cx.base + cx.lo.lvl_r[l]);
      L.e = (T *)(cx.base + cx.lo.lvl_e[l]);
    }
    L.tiles = (L.nz % 4 == 0 && fine_grid_blocks(L.nx, L.ny, L.nz) <= PARTIAL_STRIDE)
                  ? (const uint8_t *)(cx.base + cx.lo.tflags + (size_t)l * PARTIAL_STRIDE)
                  : nullptr;
  }
  if (g_l0_trilinear && cx.fuse && cx.lo.L >= 2) {
    const Level<T> &c = cx.lv[1];
    if (c.nz * 2 == nz && c.ny * 2 >= ny && c.nx * 2 >= nx) {
      cx.tab = tri_table();  // built by the solve entry points, outside any capture
      cx.tri = cx.tab != nullptr;
    }
  }
  return cx;
}

template <class T>
cudaError_t setup_levels(Ctx<T> &cx, cudaStream_t s) {
  // effective classes of level 0 (scratch), then coarsen level by level
  uint8_t *eff0 = (uint8_t *)(cx.base + cx.lo.eff0);
  {
    ProfScope ps(PROF_CONTROL, s);
    eff_class_kernel<<<row_blocks((int64_t)cx.nx * cx.ny), 256, 0, s>>>(eff0, cx.mask0, cx.nx,
                                                                         cx.ny, cx.nz);
  }
  const uint8_t *prev = eff0;
  for (int l = 1; l < cx.lo.L; ++l) {
    Level<T> &f = cx.lv[l - 1], &c = cx.lv[l];
    {
      ProfScope ps(PROF_CONTROL, s);
      coarsen_kernel<<<row_blocks((int64_t)c.nx * c.ny), 256, 0, s>>>(
          (uint8_t *)c.mask, prev, f.nx, f.ny, f.nz, c.nx, c.ny, c.nz);
    }
    // effective reclassification in place is unsafe (neighbour reads): use the
    // e-slot of this level as scratch for the raw coarse classes
    uint8_t *tmp = (uint8_t *)c.e;
    cudaMemcpyAsync(tmp, c.mask, (size_t)c.nx * c.ny * c.nz, cudaMemcpyDeviceToDevice, s);
    {
      ProfScope ps(PROF_CONTROL, s);
      eff_class_kernel<<<row_blocks((int64_t)c.nx * c.ny), 256, 0, s>>>((uint8_t *)c.mask, tmp,
                                                                         c.nx, c.ny, c.nz);
    }
    {
      ProfScope ps(PROF_CONTROL, s);
      nsolid_kernel<<<row_blocks((int64_t)c.nx * c.ny), 256, 0, s>>>((uint8_t *)c.mask, c.nx,
                                                                      c.ny, c.nz);
    }
    prev = c.mask;
  }
  if (cx.tri) {
    ProfScope ps(PROF_CONTROL, s);
    launch_tri_setup<T>((uint8_t *)(cx.base + cx.lo.ppat), cx.lv[0], cx.lv[1], s);
  }
  // Every solver vector is zero on non-fluid cells and stays so (the kernels
  // write masked values; column tiles without fluid are never written).
  {
    const size_t ts = sizeof(T);
    cudaMemsetAsync(cx.base + cx.lo.z, 0, cx.lo.r2 + ts * cx.n - cx.lo.z, s);  // z ps0 ps1 Ap r r2
    cudaMemsetAsync(cx.base + cx.lo.e, 0, sizeof(float) * cx.n, s);
    cudaMemsetAsync(cx.base + cx.lo.cctl, 0, 64, s);
    for (int l = 1; l < cx.lo.L; ++l) {
      const Level<T> &c = cx.lv[l];
      const size_t nl = (size_t)c.nx * c.ny * c.nz;
      cudaMemsetAsync(c.r, 0, ts * nl, s);
      cudaMemsetAsync(c.e, 0, ts * nl, s);
    }
    for (int l = 0; l < cx.lo.L; ++l) {
      const Level<T> &v = cx.lv[l];
      if (v.tiles) {
        ProfScope ps(PROF_CONTROL, s);
        launch_tile_flags(v.nx, v.ny, v.nz, v.mask, const_cast<uint8_t *>(v.tiles), s);
      }
    }
  }
  {
    Level<T> &c = cx.lv[cx.lo.L - 1];
    int *flag = (int *)(cx.base + cx.lo.cflag);
    const int64_t nc = (int64_t)c.nx * c.ny * c.nz;
    cudaMemsetAsync(flag, 0, sizeof(int), s);
    if (nc <= COARSEST_CELLS) {
      ProfScope ps(PROF_CONTROL, s);
      coarse_invert_kernel<T><<<1, 1024, 0, s>>>(c, (double *)(cx.base + cx.lo.cA),
                                                 (float *)(cx.base + cx.lo.cinv), flag);
    }
  }
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_inner_iteration(Ctx<T> &cx, int it_parity, cudaStream_t s) {
  const int L = cx.lo.L;
  SolverState *st = cx.st;
  // levels on the column layout when their rows allow float4 access
  const bool col = cx.col;
  auto level_col = [&](int l) {
    const Level<T> &v = cx.lv[l];
    if (l == 0) return col;
    // coarse levels: only while a row keeps at least 16 lanes busy (8 on
    // level 3 with BSP_TUNE_COARSE_SPLIT = 3, which takes it onto the tile
    // kernels)
    const bool deep = g_coarse_split >= 3 && l >= 3;
    return g_fine_col_enabled && v.nz % 4 == 0 && v.nz >= (deep ? 32 : 64) &&
           (int64_t)v.nx * v.ny * v.nz >= (deep ? 32768 : 131072) &&
           fine_grid_blocks(v.nx, v.ny, v.nz) <= PARTIAL_STRIDE;
  };
  // V-cycle on r -> z: level-0 restriction, the coarse levels (one
  // cooperative kernel, or one kernel per level and direction), level-0
  // prolongation
  auto down = [&](int l, int cls) {
    Level<T> &f = cx.lv[l], &c = cx.lv[l + 1];
    ProfScope ps(cls, s);
    if (level_col(l))
      launch_fine_down<T>(f, c, st, s);
    else
      mg_down_kernel<T><<<row_blocks((int64_t)c.nx * c.ny), 256, 0, s>>>(f, c, st);
  };
  T *cur = (T *)(cx.base + (it_parity ? cx.lo.ps1 : cx.lo.ps0));
  T *prev = (T *)(cx.base + (it_parity ? cx.lo.ps0 : cx.lo.ps1));
  T *Ap = (T *)(cx.base + cx.lo.Ap);
  // level 0 of this iteration; with the fused update its residual is the
  // buffer of this parity (written by the restriction from the other one)
  Level<T> l0 = cx.lv[0];
  if (cx.fuse) {
    T *b0 = cx.lv[0].r, *b1 = (T *)(cx.base + cx.lo.r2);
    Level<T> in = cx.lv[0];
    in.r = it_parity ? b0 : b1;
    l0.r = it_parity ? b1 : b0;
    bool tail = false;
    {
      ProfScope ps(PROF_MG_DOWN0, s);
      // the inner check runs in the restriction's last CTA (BSP_TUNE_FUSE_SCALARS)
      if (g_fuse_scalars) fine_tail_request(st, TAIL_INNER_CHECK);
      const bool ok = launch_fine_down_update<T>(
          in, cx.lv[1], l0.r, (float *)(cx.base + cx.lo.e), prev, Ap, cx.partials, st, s,
          cx.tri ? (T *)(cx.base + cx.lo.z) : nullptr, (const uint8_t *)(cx.base + cx.lo.ppat),
          cx.tab);
      tail = fine_tail_taken();
      if (!ok) return cudaErrorNotSupported;
    }
    if (!tail) {
      ProfScope ps(PROF_CONTROL, s);
      launch_maybe_pdl(g_pdl, dim3(1), dim3(RED_THREADS), 0, s, inner_check_fused_kernel, st,
                       (const double *)cx.partials, fine_grid_blocks(cx.nx, cx.ny, cx.nz));
    }
    if (cx.tri) {
      // the trilinear restriction of the scaled residual (in z) to level 1
      ProfScope ps(PROF_MG_DOWN0, s);
      launch_tri_restrict<T>(cx.lv[0], cx.lv[1], (const T *)(cx.base + cx.lo.z), st, s);
    }
  } else {
    down(0, PROF_MG_DOWN0);
  }
  bool fused = false;
  // split: levels 1 .. S on the column tile kernels around a one-launch cycle
  // of levels S+1 .. L-1 (the cycle kernel takes the level above its first
  // one as lv[0])
  int S = 0;
  if (cx.coop)
    while (S < g_coarse_split && L - (S + 1) > 2 && level_col(S + 1)) ++S;
  // two sweeps a side on level 1: the pre-smoothed correction in lv[1].e, the
  // post-smoothing's intermediate in the coarse cycle's scratch (free once
  // that kernel has run; >= level-1 cells x 4 bytes; read through the mask)
  const bool two = S >= 1 && g_l1_sweeps == 2 && fine_tma_available(cx.lv[1].nz) &&
                   cx.lv[2].nz * 2 == cx.lv[1].nz && cx.lv[2].ny * 2 >= cx.lv[1].ny &&
                   cx.lv[2].nx * 2 >= cx.lv[1].nx;
  if (S > 0) {
    for (int l = 1; l <= S; ++l) {
      if (l == 1 && two) {
        ProfScope ps(PROF_MG_MID, s);
        if (!launch_fine_smooth<T>(cx.lv[1], nullptr, cx.lv[1].e, st, s) ||
            !launch_fine_down_e<T>(cx.lv[1], cx.lv[2], cx.lv[1].e, st, s))
          return cudaErrorNotSupported;
      } else {
        down(l, PROF_MG_MID);
      }
    }
    {
      ProfScope ps(PROF_MG_COARSE, s);
      fused = launch_coarse_cycle<T>(cx.lv + S, L - S, (float *)(cx.base + cx.lo.cscratch),
                                     (const float *)(cx.base + cx.lo.cinv),
                                     (const int *)(cx.base + cx.lo.cflag), cx.base + cx.lo.cctl,
                                     g_mg_alpha, st, s);
    }
    if (!fused) {
      for (int l = S + 1; l + 1 < L; ++l) down(l, PROF_MG_COARSE);
      Level<T> &c = cx.lv[L - 1];
      const int n = c.nx * c.ny * c.nz;
      {
        ProfScope ps(PROF_MG_COARSE, s);
        mg_coarse_kernel<T><<<1, 512, 3 * n * sizeof(float), s>>>(
            c, (const float *)(cx.base + cx.lo.cinv), (const int *)(cx.base + cx.lo.cflag), st);
      }
      for (int l = L - 2; l > S; --l) {
        Level<T> &f = cx.lv[l], &c2 = cx.lv[l + 1];
        ProfScope ps(PROF_MG_COARSE, s);
        if (level_col(l))
          launch_fine_up<T>(f, c2, f.e, cx.partials, g_mg_alpha, st, s);
        else
          mg_up_kernel<T, false><<<row_blocks((int64_t)f.nx * f.ny), 256, 0, s>>>(
              f, c2, f.e, cx.partials, st, g_mg_alpha);
      }
    }
    for (int l = S; l >= 1; --l) {
      ProfScope ps(PROF_MG_MID, s);
      if (l == 1 && two) {
        T *mid = (T *)(cx.base + cx.lo.cscratch);
        if (!launch_fine_up_e<T>(cx.lv[1], cx.lv[2], cx.lv[1].e, mid, cx.partials, g_mg_alpha,
                                 st, s) ||
            !launch_fine_smooth<T>(cx.lv[1], mid, cx.lv[1].e, st, s))
          return cudaErrorNotSupported;
      } else {
        launch_fine_up<T>(cx.lv[l], cx.lv[l + 1], cx.lv[l].e, cx.partials, g_mg_alpha, st, s);
      }
    }
  } else {
    ProfScope ps(PROF_MG_COARSE, s);
    fused = cx.coop && launch_coarse_cycle<T>(cx.lv, L, (float *)(cx.base + cx.lo.cscratch),
                                   (const float *)(cx.base + cx.lo.cinv),
                                   (const int *)(cx.base + cx.lo.cflag), cx.base + cx.lo.cctl,
                                   g_mg_alpha, st, s);
  }
  if (S == 0 && !fused) {
    for (int l = 1; l + 1 < L; ++l) down(l, PROF_MG_COARSE);
    {
      Level<T> &c = cx.lv[L - 1];
      const int n = c.nx * c.ny * c.nz;
      ProfScope ps(PROF_MG_COARSE, s);
      mg_coarse_kernel<T><<<1, 512, 3 * n * sizeof(float), s>>>(
          c, (const float *)(cx.base + cx.lo.cinv), (const int *)(cx.base + cx.lo.cflag), st);
    }
    for (int l = L - 2; l >= 1; --l) {
      Level<T> &f = cx.lv[l], &c = cx.lv[l + 1];
      ProfScope ps(PROF_MG_COARSE, s);
      if (level_col(l))  // its r.e partial is written but unused
        launch_fine_up<T>(f, c, f.e, cx.partials, g_mg_alpha, st, s);
      else
        mg_up_kernel<T, false><<<row_blocks((int64_t)f.nx * f.ny), 256, 0, s>>>(
            f, c, f.e, cx.partials, st, g_mg_alpha);
    }
  }
  T *z = (T *)(cx.base + cx.lo.z);
  const int nb0 = col ? fine_grid_blocks(cx.nx, cx.ny, cx.nz) : row_blocks((int64_t)cx.nx * cx.ny);
  bool tail = false;
  {
    ProfScope ps(PROF_MG_UP0, s);
    if (g_fuse_scalars && col) fine_tail_request(st, TAIL_BETA);
    if (cx.tri) {
      const bool ok = launch_fine_up_tri<T>(l0, cx.lv[1], z, cx.partials, g_mg_alpha,
                                            (const uint8_t *)(cx.base + cx.lo.ppat), cx.tab, st,
                                            s);
      tail = fine_tail_taken();
      if (!ok) return cudaErrorNotSupported;
    } else if (col) {
      launch_fine_up<T>(l0, cx.lv[1], z, cx.partials, g_mg_alpha, st, s);
      tail = fine_tail_taken();
    } else {
      mg_up_kernel<T, true><<<nb0, 256, 0, s>>>(l0, cx.lv[1], z, cx.partials, st, g_mg_alpha);
    }
  }
  if (!tail) {
    ProfScope ps(PROF_CONTROL, s);
    launch_maybe_pdl(g_pdl, dim3(1), dim3(RED_THREADS), 0, s, beta_kernel, st,
                     (const double *)cx.partials, nb0);
  }
  tail = false;
  {
    ProfScope ps(PROF_CG_PSAP, s);
    if (col) {
      if (g_fuse_scalars) fine_tail_request(st, TAIL_ALPHA);
      launch_fine_psap<T>(cx.nx, cx.ny, cx.nz, cx.mask0, cx.lv[0].tiles, z, prev, cur, Ap,
                          cx.partials, st, s);
      tail = fine_tail_taken();
    } else {
      cg_ps_ap_kernel<T><<<nb0, 256, 0, s>>>(cx.nx, cx.ny, cx.nz, cx.mask0, z, prev, cur, Ap,
                                             cx.partials, st);
    }
  }
  if (!tail) {
    ProfScope ps(PROF_CONTROL, s);
    launch_maybe_pdl(g_pdl, dim3(1), dim3(RED_THREADS), 0, s, alpha_kernel, st,
                     (const double *)cx.partials, nb0);
  }
  if (cx.fuse) return cudaGetLastError();  // the update runs in the next restriction
  int nbf = flat_blocks(cx.n);
  {
    ProfScope ps(PROF_CG_UPDATE, s);
    if (col)
      nbf = launch_cg_update_col<T>(cx.nx, cx.ny, cx.nz, cx.lv[0].tiles,
                                    (float *)(cx.base + cx.lo.e), cx.lv[0].r, cur, Ap,
                                    cx.partials, st, s);
    else
      cg_update_kernel<T><<<nbf, 256, 0, s>>>(cx.n, cx.mask0, (float *)(cx.base + cx.lo.e),
                                              cx.lv[0].r, cur, Ap, cx.partials, st);
  }
  {
    ProfScope ps(PROF_CONTROL, s);
    inner_check_kernel<<<1, RED_THREADS, 0, s>>>(st, cx.partials, nbf);
  }
  return cudaGetLastError();
}

// FP64 residual pass (norm pass, or WRITE: rhat and e = 0): the column kernel
// when level 0 runs on the column layout and div is 16-byte aligned, else the
// per-row kernel.  Returns the number of partial blocks written.
template <class T>
int launch_resid(Ctx<T> &cx, const float *div, const double *x, double bscale, T *rhat, float *e,
                 bool write, cudaStream_t s) {
  if (cx.col && ((uintptr_t)div & 15u) == 0)
    return launch_resid64_col<T>(cx.nx, cx.ny, cx.nz, cx.mask0, cx.lv[0].tiles, div, x, bscale,
                                 rhat, e, cx.partials, cx.st, write, s);
  const int nbr = row_blocks((int64_t)cx.nx * cx.ny);
  if (write)
    residual64_kernel<T, true><<<nbr, 256, 0, s>>>(cx.nx, cx.ny, cx.nz, cx.mask0, div, x, bscale,
                                                  rhat, e, cx.partials, cx.st);
  else
    residual64_kernel<T, false><<<nbr, 256, 0, s>>>(cx.nx, cx.ny, cx.nz, cx.mask0, div, x,
                                                   bscale, rhat, e, cx.partials, cx.st);
  return nbr;
}

// x is zeroed before the ||b|| pass unless that pass runs on the column kernel
// (which skips the loads of an iterate known to be zero) and a warm start then
// writes every cell of x.
template <class T>
bool x_needs_zeroing(const Ctx<T> &cx, const float *div, bool warm) {
  return !(warm && cx.col && ((uintptr_t)div & 15u) == 0);
}

// FP32 <-> FP64 copies of the iterate on fluid cells (0 elsewhere).  Four
// cells per step (16-byte float, 2 x 16-byte double and one mask word) when
// the pointers allow it, one otherwise; the same values either way.
__device__ __forceinline__ bool conv_vec(const void *f, const void *d, const uint8_t *m,
                                         int64_t n) {
  return (n & 3) == 0 && ((((uintptr_t)f | (uintptr_t)d) & 15u) == 0) &&
         (((uintptr_t)m & 3u) == 0);
}
// With st, a fluid value other than 0 clears st->norm_cached (the first outer
// residual is then not the ||b|| pass's) and st->x_zero.
__global__ void f32_to_f64_kernel(int64_t n, const float *a, double *b, const uint8_t *mask,
                                  SolverState *st) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int nonzero = 0;
  if (conv_vec(a, b, mask, n)) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n / 4; q += stride) {
      const uint32_t mw = *reinterpret_cast<const uint32_t *>(mask + 4 * q);
      const float4 v = *reinterpret_cast<const float4 *>(a + 4 * q);
      const double d0 = (mw & BSP_MFLUID) ? (double)v.x : 0.0;
      const double d1 = ((mw >> 8) & BSP_MFLUID) ? (double)v.y : 0.0;
      const double d2 = ((mw >> 16) & BSP_MFLUID) ? (double)v.z : 0.0;
      const double d3 = ((mw >> 24) & BSP_MFLUID) ? (double)v.w : 0.0;
      double2 *o = reinterpret_cast<double2 *>(b + 4 * q);
      o[0] = make_double2(d0, d1);
      o[1] = make_double2(d2, d3);
      nonzero |= (d0 != 0.0) | (d1 != 0.0) | (d2 != 0.0) | (d3 != 0.0);
    }
  } else {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
      const double d = mcls(mask[c]) == BSP_FLUID ? (double)a[c] : 0.0;
      b[c] = d;
      nonzero |= d != 0.0;
    }
  }
  // a NaN compares unequal to 0, so it also clears the flag
  if (__syncthreads_or(nonzero) && threadIdx.x == 0 && st) {
    st->norm_cached = 0;
    st->x_zero = 0;
  }
}
__global__ void f64_to_f32_kernel(int64_t n, const double *a, float *b, const uint8_t *mask) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  if (conv_vec(b, a, mask, n)) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n / 4; q += stride) {
      const uint32_t mw = *reinterpret_cast<const uint32_t *>(mask + 4 * q);
      const double2 v0 = reinterpret_cast<const double2 *>(a + 4 * q)[0];
      const double2 v1 = reinterpret_cast<const double2 *>(a + 4 * q)[1];
      *reinterpret_cast<float4 *>(b + 4 * q) =
          make_float4((mw & BSP_MFLUID) ? (float)v0.x : 0.0f,
                      ((mw >> 8) & BSP_MFLUID) ? (float)v0.y : 0.0f,
                      ((mw >> 16) & BSP_MFLUID) ? (float)v1.x : 0.0f,
                      ((mw >> 24) & BSP_MFLUID) ? (float)v1.y : 0.0f);
    }
    return;
  }
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride)
    b[c] = mcls(mask[c]) == BSP_FLUID ? (float)a[c] : 0.0f;
}
__global__ void __launch_bounds__(RED_THREADS) bnorm_kernel(SolverState *st,
                                                            const double *partials, int nblocks) {
  const double bb = reduce_slot(partials, 0, nblocks, false);
  if (threadIdx.x == 0) {
    st->b_norm2 = bb;
    st->norm_cached = 1;  // x is zero here; a nonzero warm start clears it
  }
}

// Host-side record of workspaces whose multigrid setup (coarse masks, coarsest
// inverse) is current, for callers that pass reuse_setup = 1 (their mask does
// not change between solves).
// A setup depends on the tile geometry too (the per-tile fluid flags): the
// level-0 plane chunk in force when it was built is part of its key.
extern int g_fine_bi;
struct SetupKey {
  const void *ws, *mask;
  int nx, ny, nz, storage, fine_bi, tri;  // tri: the parent patterns were built too
  int fine_ctas;                           // tile flags follow the plane chunking
};
static std::mutex g_setup_mu;
static SetupKey g_setups[16];
static int g_setup_next = 0;

static bool setup_cached(const void *ws, const void *mask, int nx, int ny, int nz, int storage) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  for (const SetupKey &k : g_setups)
    if (k.ws == ws && k.mask == mask && k.nx == nx && k.ny == ny && k.nz == nz &&
        k.storage == storage && k.fine_bi == g_fine_bi && k.tri == (int)g_l0_trilinear &&
        k.fine_ctas == g_fine_ctas)
      return true;
  return false;
}
static void remember_setup(const void *ws, const void *mask, int nx, int ny, int nz,
                           int storage) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  for (SetupKey &k : g_setups)
    if (k.ws == ws) k.ws = nullptr;  // a workspace holds one setup
  g_setups[g_setup_next] = SetupKey{ws, mask, nx, ny, nz, storage, g_fine_bi,
                                     (int)g_l0_trilinear, g_fine_ctas};
  g_setup_next = (g_setup_next + 1) % 16;
}

template <class T>
int solve_impl(void *ws, const uint8_t *mask, const float *div, float *p_out, int nx, int ny,
               int nz, float dx, float dt, float rho, const BspSolveParams *prm,
               BspSolveInfo *info, cudaStream_t s) {
  Ctx<T> cx = make_ctx<T>(ws, mask, nx, ny, nz, prm->storage);
  {
    const Level<T> &c = cx.lv[cx.lo.L - 1];
    if ((int64_t)c.nx * c.ny * c.nz > COARSEST_MAX) return BSP_ERR_SHAPE;
  }
  SolverState h{};
  h.tol = prm->tol;
  h.eta = prm->inner_tol;
  h.max_outer = prm->max_outer;
  h.max_inner = prm->max_inner;
  h.scale = 1.0;
  h.x_zero = 1;  // x is zeroed before the first residual pass
  cudaError_t e = cudaMemcpyAsync(cx.st, &h, sizeof(h), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return (int)e;
  // the coarse-cycle grid barrier starts every solve clean: a barrier that
  // gave up in an earlier solve leaves its error word and a partial count
  e = cudaMemsetAsync(cx.base + cx.lo.cctl, 0, 64, s);
  if (e != cudaSuccess) return (int)e;
  if (g_test_barrier_error) {
    // test hook (BSP_TUNE_TEST_BARRIER_ERROR): start this solve with the
    // barrier's error word set, as a barrier that gave up leaves it; the
    // coarse cycle then returns at its first barrier and the solve reports
    // BSP_ERR_TIMEOUT.  One-shot.
    g_test_barrier_error = false;
    const int v = BSP_ERR_TIMEOUT;
    e = cudaMemcpyAsync(cx.base + cx.lo.cctl + offsetof(GridCtl, err), &v, sizeof(int),
                        cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // v lives on this stack frame
    if (e != cudaSuccess) return (int)e;
  }
  if (!(prm->reuse_setup && setup_cached(ws, mask, nx, ny, nz, prm->storage))) {
    e = setup_levels<T>(cx, s);
    if (e != cudaSuccess) return (int)e;
    remember_setup(ws, mask, nx, ny, nz, prm->storage);
  }
  double *x = (double *)(cx.base + cx.lo.x);
  float *eb = (float *)(cx.base + cx.lo.e);
  const int nbr = row_blocks((int64_t)nx * ny);
  const int nbf = flat_blocks(cx.n);
  const double bscale = -((double)rho * (double)dx * (double)dx) / (double)dt;
  // ||b||^2: a residual pass with x = 0
  if (x_needs_zeroing<T>(cx, div, prm->warm_start && p_out)) {
    e = cudaMemsetAsync(x, 0, sizeof(double) * cx.n, s);
    if (e != cudaSuccess) return (int)e;
  }
  (void)nbr;
  int nres;
  {
    ProfScope ps(PROF_RESID64, s);
    nres = launch_resid<T>(cx, div, x, bscale, nullptr, nullptr, false, s);
  }
  {
    ProfScope ps(PROF_CONTROL, s);
    bnorm_kernel<<<1, RED_THREADS, 0, s>>>(cx.st, cx.partials, nres);
  }
  if (prm->warm_start && p_out) {
    ProfScope ps(PROF_CONTROL, s);
    f32_to_f64_kernel<<<nbf, 256, 0, s>>>(cx.n, p_out, x, mask, cx.st);
  }
  int flag = 0;
  for (int outer = 0; outer <= prm->max_outer; ++outer) {
    {
      ProfScope ps(PROF_RESID64, s);
      nres = launch_resid<T>(cx, div, x, bscale, nullptr, nullptr, false, s);
    }
    {
      ProfScope ps(PROF_CONTROL, s);
      outer_check_kernel<<<1, RED_THREADS, 0, s>>>(cx.st, cx.partials, nres,
                                                   prm->storage == BSP_STORE_FP32);
    }
    {
      ProfScope ps(PROF_RESID64, s);
      launch_resid<T>(cx, div, x, bscale, cx.r_write(), eb, true, s);
    }
    // 4-byte flag read (pageable: the copy completes before the sync returns)
    e = cudaMemcpyAsync(&flag, &cx.st->done, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess || flag) break;
    for (int chunk = 0;; ++chunk) {
      for (int q = 0; q < prm->check_every; ++q)
        launch_inner_iteration<T>(cx, (chunk * prm->check_every + q) & 1, s);
      e = cudaMemcpyAsync(&flag, &cx.st->inner_done, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess || flag) break;
    }
    if (e != cudaSuccess) break;
    ProfScope ps(PROF_XUPDATE, s);
    xupdate_kernel<<<nbf, 256, 0, s>>>(cx.n, x, eb, nullptr, cx.st);
  }
  if (e != cudaSuccess) return (int)e;
  SolverState fin{};
  if (p_out) {
    ProfScope ps(PROF_CONTROL, s);
    f64_to_f32_kernel<<<nbf, 256, 0, s>>>(cx.n, x, p_out, mask);
  }
  e = cudaMemcpyAsync(&fin, cx.st, sizeof(SolverState), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  if (info) {
    info->outer_iterations = fin.outer_it;
    info->inner_iterations = fin.total_inner;
    info->rel_residual = fin.rel;
    info->levels = cx.lo.L;
  }
  return fin.status;
}

// ======================================================================================
// Device-driven solve: the whole refinement loop as one CUDA graph.
//
//   prologue: state init, ||b||, (warm start x = p)
//   WHILE outer (default 1):  FP64 residual, outer check, residual -> rhat,
//                             arm inner condition,
//                             WHILE inner: two CG iterations, inner condition
//                             x += e / scale, outer condition
//   epilogue: p = (float) x
//
// The condition kernels count their own executions and clear the condition
// after max_inner + 2 (inner) / max_outer + 2 (outer) bodies, so both loops end
// whatever the rest of the state holds.  No host synchronisation inside.
// ======================================================================================
__global__ void init_state_kernel(SolverState *st, double tol, double eta, int max_outer,
                                  int max_inner) {
  SolverState s{};
  s.tol = tol;
  s.eta = eta;
  s.eta_eff = eta;
  s.max_outer = max_outer;
  s.max_inner = max_inner;
  s.scale = 1.0;
  s.x_zero = 1;  // x is zeroed before the first residual pass
  *st = s;
}
__global__ void arm_inner_kernel(cudaGraphConditionalHandle hi, SolverState *st) {
  st->guard_inner = 0;
  cudaGraphSetConditional(hi, st->done ? 0u : 1u);
}
__global__ void inner_cond_kernel(cudaGraphConditionalHandle hi, SolverState *st) {
  const int g = ++st->guard_inner;
  cudaGraphSetConditional(hi, (!st->inner_done && g <= st->max_inner + 2) ? 1u : 0u);
}
__global__ void outer_cond_kernel(cudaGraphConditionalHandle ho, SolverState *st) {
  const int g = ++st->guard_outer;
  cudaGraphSetConditional(ho, (!st->done && g <= st->max_outer + 2) ? 1u : 0u);
}

static cudaStream_t capture_stream() {
  static std::mutex mu;
  static cudaStream_t streams[64] = {nullptr};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64) return nullptr;
  if (!streams[dev]) cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
  return streams[dev];
}

static cudaError_t seg_begin(cudaStream_t cs, cudaGraph_t g,
                             const std::vector<cudaGraphNode_t> &deps) {
  return cudaStreamBeginCaptureToGraph(cs, g, deps.empty() ? nullptr : deps.data(), nullptr,
                                       deps.size(), cudaStreamCaptureModeThreadLocal);
}
static cudaError_t seg_end(cudaStream_t cs, std::vector<cudaGraphNode_t> &leaves) {
  cudaStreamCaptureStatus stt;
  const cudaGraphNode_t *d = nullptr;
  size_t nd = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(cs, &stt, nullptr, nullptr, &d, &nd);
  if (e == cudaSuccess) leaves.assign(d, d + nd);
  cudaGraph_t out = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(cs, &out);
  return e != cudaSuccess ? e : e2;
}
static cudaError_t add_while(cudaGraph_t g, const std::vector<cudaGraphNode_t> &deps,
                             cudaGraphConditionalHandle h, cudaGraphNode_t *node,
                             cudaGraph_t *body) {
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaError_t e = cudaGraphAddNode(node, g, deps.empty() ? nullptr : deps.data(), deps.size(), &cp);
  if (e == cudaSuccess) *body = cp.conditional.phGraph_out[0];
  return e;
}

// Appends one instance's solve to graph g after `deps`; `deps` returns its leaves.
template <class T>
cudaError_t append_solve(Ctx<T> &cx, const float *div, float *p_out, float dx, float dt, float rho,
                         const BspSolveParams *prm, cudaGraph_t g,
                         std::vector<cudaGraphNode_t> &deps) {
  cudaStream_t cs = capture_stream();
  if (!cs) return cudaErrorInvalidDevice;
  const int nx = cx.nx, ny = cx.ny, nz = cx.nz;
  const uint8_t *mask = cx.mask0;
  SolverState *st = cx.st;
  double *x = (double *)(cx.base + cx.lo.x);
  float *eb = (float *)(cx.base + cx.lo.e);
  const int nbr = row_blocks((int64_t)nx * ny);
  const int nbf = flat_blocks(cx.n);
  const double bscale = -((double)rho * (double)dx * (double)dx) / (double)dt;
  cudaError_t e;
  std::vector<cudaGraphNode_t> leaves;
  // prologue
  if ((e = seg_begin(cs, g, deps)) != cudaSuccess) return e;
  init_state_kernel<<<1, 1, 0, cs>>>(st, prm->tol, prm->inner_tol, prm->max_outer,
                                     prm->max_inner);
  // every replay starts with a clean coarse-cycle grid barrier (error word,
  // count and generation), whatever an earlier replay left there
  cudaMemsetAsync(cx.base + cx.lo.cctl, 0, 64, cs);
  if (x_needs_zeroing<T>(cx, div, prm->warm_start && p_out))
    cudaMemsetAsync(x, 0, sizeof(double) * cx.n, cs);
  (void)nbr;
  const int nres = launch_resid<T>(cx, div, x, bscale, nullptr, nullptr, false, cs);
  bnorm_kernel<<<1, RED_THREADS, 0, cs>>>(st, cx.partials, nres);
  if (prm->warm_start && p_out) f32_to_f64_kernel<<<nbf, 256, 0, cs>>>(cx.n, p_out, x, mask, st);
  if ((e = seg_end(cs, leaves)) != cudaSuccess) return e;
  cudaGraphConditionalHandle ho, hi;
  if ((e = cudaGraphConditionalHandleCreate(&ho, g, 1, cudaGraphCondAssignDefault)) != cudaSuccess)
    return e;
  if ((e = cudaGraphConditionalHandleCreate(&hi, g, 0, 0)) != cudaSuccess) return e;
  cudaGraphNode_t node_o, node_i;
  cudaGraph_t body_o, body_i;
  if ((e = add_while(g, leaves, ho, &node_o, &body_o)) != cudaSuccess) return e;
  // outer body, part 1
  if ((e = seg_begin(cs, body_o, {})) != cudaSuccess) return e;
  launch_resid<T>(cx, div, x, bscale, nullptr, nullptr, false, cs);
  outer_check_kernel<<<1, RED_THREADS, 0, cs>>>(st, cx.partials, nres,
                                                prm->storage == BSP_STORE_FP32);
  launch_resid<T>(cx, div, x, bscale, cx.r_write(), eb, true, cs);
  arm_inner_kernel<<<1, 1, 0, cs>>>(hi, st);
  if ((e = seg_end(cs, leaves)) != cudaSuccess) return e;
  if ((e = add_while(body_o, leaves, hi, &node_i, &body_i)) != cudaSuccess) return e;
  // inner body: two iterations (the search-direction buffers alternate)
  if ((e = seg_begin(cs, body_i, {})) != cudaSuccess) return e;
  launch_inner_iteration<T>(cx, 0, cs);
  launch_inner_iteration<T>(cx, 1, cs);
  inner_cond_kernel<<<1, 1, 0, cs>>>(hi, st);
  if ((e = seg_end(cs, leaves)) != cudaSuccess) return e;
  // outer body, part 2
  if ((e = seg_begin(cs, body_o, {node_i})) != cudaSuccess) return e;
  xupdate_kernel<<<nbf, 256, 0, cs>>>(cx.n, x, eb, nullptr, st);
  outer_cond_kernel<<<1, 1, 0, cs>>>(ho, st);
  if ((e = seg_end(cs, leaves)) != cudaSuccess) return e;
  // epilogue
  if ((e = seg_begin(cs, g, {node_o})) != cudaSuccess) return e;
  if (p_out) f64_to_f32_kernel<<<nbf, 256, 0, cs>>>(cx.n, x, p_out, mask);
  return seg_end(cs, deps);  // without p_out the segment is empty: leaves = {node_o}
}

// Executable graphs of recent solves, keyed by everything baked into them.
struct GraphKey {
  std::vector<uintptr_t> v;
  bool operator==(const GraphKey &o) const { return v == o.v; }
};
struct GraphEntry {
  GraphKey key;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};
static std::mutex g_graph_mu;
static std::vector<GraphEntry> g_graphs;

static cudaGraphExec_t graph_lookup(const GraphKey &k) {
  for (auto &e : g_graphs)
    if (e.key == k) return e.exec;
  return nullptr;
}
static void graph_store(const GraphKey &k, cudaGraph_t g, cudaGraphExec_t x) {
  if (g_graphs.size() >= 8) {
    cudaGraphExecDestroy(g_graphs.front().exec);
    cudaGraphDestroy(g_graphs.front().graph);
    g_graphs.erase(g_graphs.begin());
  }
  g_graphs.push_back(GraphEntry{k, g, x});
}

static void key_floats(GraphKey &k, float a, float b, float c) {
  uint32_t u[3];
  memcpy(&u[0], &a, 4);
  memcpy(&u[1], &b, 4);
  memcpy(&u[2], &c, 4);
  for (uint32_t x : u) k.v.push_back(x);
}
static void key_params(GraphKey &k, const BspSolveParams *p);

template <class T>
static int finish_info(const Ctx<T> &cx, BspSolveInfo *info, cudaStream_t s) {
  SolverState fin{};
  cudaError_t e = cudaMemcpyAsync(&fin, cx.st, sizeof(SolverState), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  if (info) {
    info->outer_iterations = fin.outer_it;
    info->inner_iterations = fin.total_inner;
    info->rel_residual = fin.rel;
    info->levels = cx.lo.L;
  }
  return fin.status;
}

// One batch of solves (count >= 1) as one graph launch: independent branches,
// one per instance.  Level setup runs (or is reused) before the launch.
template <class T>
int solve_graph_batch(int count, const BspBatchItem *items, const BspSolveParams *prm,
                      BspSolveInfo *infos, cudaStream_t s) {
  std::vector<Ctx<T>> cxs;
  GraphKey key;
  key.v.push_back((uintptr_t)count);
  key_params(key, prm);
  for (int q = 0; q < count; ++q) {
    const BspBatchItem &it = items[q];
    Ctx<T> cx = make_ctx<T>(it.workspace, it.mask, it.nx, it.ny, it.nz, prm->storage);
    cx.coop = count == 1;
    const Level<T> &c = cx.lv[cx.lo.L - 1];
    if ((int64_t)c.nx * c.ny * c.nz > COARSEST_MAX) return BSP_ERR_SHAPE;
    if (!(prm->reuse_setup &&
          setup_cached(it.workspace, it.mask, it.nx, it.ny, it.nz, prm->storage))) {
      cudaError_t e = setup_levels<T>(cx, s);
      if (e != cudaSuccess) return (int)e;
      remember_setup(it.workspace, it.mask, it.nx, it.ny, it.nz, prm->storage);
    }
    for (uintptr_t x : {(uintptr_t)it.workspace, (uintptr_t)it.mask, (uintptr_t)it.div,
                        (uintptr_t)it.p, (uintptr_t)it.nx, (uintptr_t)it.ny, (uintptr_t)it.nz})
      key.v.push_back(x);
    key_floats(key, it.dx, it.dt, it.rho);
    cxs.push_back(cx);
  }
  std::lock_guard<std::mutex> lk(g_graph_mu);
  cudaGraphExec_t exec = graph_lookup(key);
  if (!exec) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    prof_suspend(true);
    for (int q = 0; q < count && e == cudaSuccess; ++q) {
      std::vector<cudaGraphNode_t> deps;
      e = append_solve<T>(cxs[q], items[q].div, items[q].p, items[q].dx, items[q].dt,
                          items[q].rho, prm, g, deps);
    }
    prof_suspend(false);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
    if (e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return (int)e;
    }
    graph_store(key, g, exec);
  }
  cudaError_t e = cudaGraphLaunch(exec, s);
  if (e != cudaSuccess) return (int)e;
  if (!infos) return BSP_OK;  // asynchronous: results land in p when the stream reaches them
  int status = BSP_OK;
  for (int q = 0; q < count; ++q) {
    const int st = finish_info<T>(cxs[q], &infos[q], s);
    if (st != BSP_OK && status == BSP_OK) status = st;
  }
  return status;
}

static void key_params(GraphKey &k, const BspSolveParams *p) {
  uint64_t t, it;
  memcpy(&t, &p->tol, 8);
  memcpy(&it, &p->inner_tol, 8);
  for (uintptr_t x : {(uintptr_t)t, (uintptr_t)it, (uintptr_t)p->max_outer,
                      (uintptr_t)p->max_inner, (uintptr_t)p->storage,
                      (uintptr_t)p->warm_start})
    k.v.push_back(x);
  // launch-time tuning captured into the graph
  uint32_t a;
  memcpy(&a, &g_mg_alpha, 4);
  k.v.push_back((uintptr_t)a);
  k.v.push_back((uintptr_t)g_fine_col_enabled);
  k.v.push_back((uintptr_t)g_fine_tma_enabled);
  k.v.push_back((uintptr_t)g_coarse_fused_enabled);
  k.v.push_back((uintptr_t)g_coarse_phases_fused);
  k.v.push_back((uintptr_t)g_coarse_tail_smem);
  k.v.push_back((uintptr_t)g_coarse_split);
  k.v.push_back((uintptr_t)g_l1_sweeps);
  k.v.push_back((uintptr_t)g_l0_trilinear);
  k.v.push_back((uintptr_t)g_tri_cpc);
  k.v.push_back((uintptr_t)g_fuse_scalars);
  k.v.push_back((uintptr_t)g_fine_ctas);
  k.v.push_back((uintptr_t)g_pdl);
  k.v.push_back((uintptr_t)g_coarse_cluster);
  k.v.push_back((uintptr_t)g_cluster_tail_cells);
  k.v.push_back((uintptr_t)g_downu_blocks);
  k.v.push_back((uintptr_t)g_coarse_cluster_tail_smem);
  k.v.push_back((uintptr_t)g_fuse_update_enabled);
  k.v.push_back((uintptr_t)g_fine_bi);
}

}  // namespace bsp

using namespace bsp;

extern "C" size_t bsp_solver_workspace_bytes(int nx, int ny, int nz, int storage) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return 0;
  return make_layout(nx, ny, nz, storage).total;
}

extern "C" void bsp_solve_params_default(BspSolveParams *p) {
  if (!p) return;
  p->tol = 1e-6;
  p->inner_tol = 1e-3;
  p->max_outer = 8;
  p->max_inner = 200;
  p->storage = BSP_STORE_FP32;
  p->warm_start = 0;
  p->check_every = 8;
  p->reuse_setup = 0;
  p->use_graph = 0;
}

extern "C" int bsp_solve_tol(float *p, const float *div_u, const uint8_t *mask, int nx, int ny,
                             int nz, float dx, float dt, float rho, const BspSolveParams *params,
                             void *workspace, size_t workspace_bytes, double *x64_out,
                             BspSolveInfo *info, cudaStream_t stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!div_u || !mask || !params || !workspace) return BSP_ERR_NULL;
  if (((uintptr_t)workspace & 255u) != 0) return BSP_ERR_ALIGN;
  if (workspace_bytes < bsp_solver_workspace_bytes(nx, ny, nz, params->storage))
    return BSP_ERR_WORKSPACE;
  if (params->storage < 0 || params->storage > 2 || params->check_every <= 0 ||
      params->max_inner <= 0 || params->max_outer < 0 || !(params->tol >= 0.0))
    return BSP_ERR_ARG;
  if (g_l0_trilinear) tri_table();  // one synchronous copy per device, before any capture
  int st;
  if (params->use_graph) {
    const BspBatchItem item{p, div_u, mask, nx, ny, nz, dx, dt, rho, workspace, workspace_bytes};
    switch (params->storage) {
      case BSP_STORE_FP16:
        st = solve_graph_batch<__half>(1, &item, params, info, stream);
        break;
      case BSP_STORE_BF16:
        st = solve_graph_batch<__nv_bfloat16>(1, &item, params, info, stream);
        break;
      default:
        st = solve_graph_batch<float>(1, &item, params, info, stream);
    }
  } else {
    switch (params->storage) {
      case BSP_STORE_FP16:
        st = solve_impl<__half>(workspace, mask, div_u, p, nx, ny, nz, dx, dt, rho, params,
                                info, stream);
        break;
      case BSP_STORE_BF16:
        st = solve_impl<__nv_bfloat16>(workspace, mask, div_u, p, nx, ny, nz, dx, dt, rho,
                                       params, info, stream);
        break;
      default:
        st = solve_impl<float>(workspace, mask, div_u, p, nx, ny, nz, dx, dt, rho, params, info,
                               stream);
    }
  }
  if (x64_out && (st == BSP_OK || st == BSP_NOT_CONVERGED)) {
    const Layout lo = make_layout(nx, ny, nz, params->storage);
    cudaMemcpyAsync(x64_out, (char *)workspace + lo.x, sizeof(double) * (size_t)nx * ny * nz,
                    cudaMemcpyDeviceToDevice, stream);
  }
  return st;
}

extern "C" int bsp_solve_batch(int count, const BspBatchItem *items,
                               const BspSolveParams *params, BspSolveInfo *infos,
                               cudaStream_t stream) {
  if (count <= 0) return BSP_OK;
  if (!items || !params) return BSP_ERR_NULL;
  if (params->storage < 0 || params->storage > 2 || params->max_inner <= 0 ||
      params->max_outer < 0 || !(params->tol >= 0.0))
    return BSP_ERR_ARG;
  for (int q = 0; q < count; ++q) {
    const BspBatchItem &it = items[q];
    if (it.nx <= 0 || it.ny <= 0 || it.nz <= 0) return BSP_ERR_SHAPE;
    if (!it.p || !it.div || !it.mask || !it.workspace) return BSP_ERR_NULL;
    if (((uintptr_t)it.workspace & 255u) != 0) return BSP_ERR_ALIGN;
    if (it.workspace_bytes < bsp_solver_workspace_bytes(it.nx, it.ny, it.nz, params->storage))
      return BSP_ERR_WORKSPACE;
  }
  if (g_l0_trilinear) tri_table();  // one synchronous copy per device, before any capture
  switch (params->storage) {
    case BSP_STORE_FP16:
      return solve_graph_batch<__half>(count, items, params, infos, stream);
    case BSP_STORE_BF16:
      return solve_graph_batch<__nv_bfloat16>(count, items, params, infos, stream);
    default:
      return solve_graph_batch<float>(count, items, params, infos, stream);
  }
}
