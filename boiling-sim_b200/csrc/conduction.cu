// conduction.cu -- backward-Euler conduction: the Jacobi sweep of
//   (1 + sum gamma) T_new = T_old + sum gamma T_nbr
// and the conduction step around it.
//
// Reference semantics:
//   apply_implicit_conduction_update   python/boilingsim/thermal.py:259-388
//   conduct_one_step, implicit branch  python/boilingsim/thermal.py:647-658
//   MaterialProps arrays [fluid, pot_wall, air, carrot]  thermal.py:45-122
//
// Per non-air cell c of material ms the reference visits the faces -x, +x, -y,
// +y, -z, +z; a face on the domain edge is skipped.  For a neighbour of
// material mn the face coefficient is
//   mn == air:  gamma = ((dt h_conv) inv) / dx,  neighbour value T_amb
//   otherwise:  gamma = ((dt k_face) inv) / (dx dx),  k_face = ((2 ks) kn) / ((ks + kn) + 1e-12)
// with inv = 1 / (rho[ms] cp[ms]); rhs += gamma * T_nbr and diag += gamma in
// face order, and T_dst = (T_old + rhs) / (1 + diag).  Air cells are not
// written.  Every operation here is the same IEEE single operation in the
// same order (no contraction, correctly rounded division), so results are
// bit-identical to the reference arithmetic.
//
// gamma depends only on the two materials (and dt, dx, h_conv), so each CTA
// builds the table gamma[ms][mn] once in shared memory; a face costs one
// shared load.
//
// Column kernel (nz % 4 == 0, 16-byte aligned fields): the layout of the
// pressure sweep's column kernel -- a warp owns one j row and 128 consecutive
// k cells (one float4 per lane) and marches along i with the i-1 / i / i+1
// planes in registers, j neighbours from L1, k neighbours by warp shuffles.
// HBM traffic is one material byte per cell plus, on cells that are not air,
// T_iter, T_old and the store (12 B): the material words of plane i+1 (rows
// j-1, j, j+1) are loaded one plane ahead, so each T load is issued only when
// its four cells are not all air, without waiting on a dependent load.
//
// The first sweep of a step can also write the T_old snapshot (SNAP): it reads
// T on every cell once and stores it to T_old, replacing the separate copy.
#include <cuda_runtime.h>

#include "../../include/bsproj.h"
#include "bsp_common.cuh"

namespace bsp {
int num_sms();

namespace cond {

constexpr int MAXM = 8;  // material ids 0..7

__device__ __forceinline__ float gamma_entry(int ms, int mn, const float *__restrict__ kk,
                                             const float *__restrict__ rho,
                                             const float *__restrict__ cp, int n_mat, float dx,
                                             float dt, float h, int mair) {
  if (ms >= n_mat || mn >= n_mat) return 0.0f;
  const float inv = __fdiv_rn(1.0f, __fmul_rn(rho[ms], cp[ms]));
  if (mn == mair) return __fdiv_rn(__fmul_rn(__fmul_rn(dt, h), inv), dx);
  const float ks = kk[ms], kn = kk[mn];
  const float kf =
      __fdiv_rn(__fmul_rn(__fmul_rn(2.0f, ks), kn), __fadd_rn(__fadd_rn(ks, kn), 1.0e-12f));
  return __fdiv_rn(__fmul_rn(__fmul_rn(dt, kf), inv), __fmul_rn(dx, dx));
}

struct Params {
  const float *k, *rho, *cp;
  int n_mat;
  float dx, dt, h, tamb;
  int mair;
};

__device__ __forceinline__ void build_table(float *tab, const Params &P) {
  if (threadIdx.x < MAXM * MAXM)
    tab[threadIdx.x] = gamma_entry(threadIdx.x / MAXM, threadIdx.x % MAXM, P.k, P.rho, P.cp,
                                   P.n_mat, P.dx, P.dt, P.h, P.mair);
  __syncthreads();
}

// One face of one cell, in the reference's order of accumulation.
__device__ __forceinline__ void face(float &rhs, float &diag, const float *row, bool inb,
                                     uint32_t mn, float tn, uint32_t mair, float tamb) {
  if (inb) {
    const float g = row[mn & (MAXM - 1)];
    rhs = __fadd_rn(rhs, __fmul_rn(g, mn == mair ? tamb : tn));
    diag = __fadd_rn(diag, g);
  }
}

// ---- material words ----------------------------------------------------------------
__device__ __forceinline__ uint32_t mword(const uint8_t *m, int64_t c) {
  return __ldg(reinterpret_cast<const uint32_t *>(m + c));
}
__device__ __forceinline__ uint32_t mword(const int32_t *m, int64_t c) {
  const int4 v = __ldg(reinterpret_cast<const int4 *>(m + c));
  return ((uint32_t)v.x & 0xffu) | (((uint32_t)v.y & 0xffu) << 8) |
         (((uint32_t)v.z & 0xffu) << 16) | ((uint32_t)v.w << 24);
}
__device__ __forceinline__ uint32_t mbyte(const uint8_t *m, int64_t c) { return __ldg(m + c); }
__device__ __forceinline__ uint32_t mbyte(const int32_t *m, int64_t c) {
  return (uint32_t)__ldg(m + c) & 0xffu;
}
__device__ __forceinline__ float f4(const float4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}
__device__ __forceinline__ float4 ld4(const float *p) {
  return __ldg(reinterpret_cast<const float4 *>(p));
}

// ---- column kernel ----------------------------------------------------------------
// Branch-free per cell: a face on the domain edge gets the neighbour code OOB,
// whose table entries are 0, and a neighbour value of 0, so it adds +0 to
// rhs and diag -- the same bits as skipping the face (rhs and diag start at
// +0 and a sum that starts at +0 never becomes -0).  Air neighbours are
// replaced by T_amb once per loaded float4 instead of once per face.
constexpr uint32_t OOB = 0x0Fu;
constexpr uint32_t OOBW = 0x0F0F0F0Fu;
constexpr int TCOLS = 16;  // table row stride: material ids 0..7 and OOB

__device__ __forceinline__ float amb1(float v, uint32_t w, int q, uint32_t mair, float tamb) {
  return byte_of(w, q) == mair ? tamb : v;
}
__device__ __forceinline__ float4 amb4(float4 v, uint32_t w, uint32_t mair, float tamb) {
  return make_float4(amb1(v.x, w, 0, mair, tamb), amb1(v.y, w, 1, mair, tamb),
                     amb1(v.z, w, 2, mair, tamb), amb1(v.w, w, 3, mair, tamb));
}
__device__ __forceinline__ void face_t(float &rhs, float &diag, const float *row, uint32_t w,
                                       int q, float t) {
  const float g = row[(w >> (8 * q)) & (TCOLS - 1)];
  rhs = __fadd_rn(rhs, __fmul_rn(g, t));
  diag = __fadd_rn(diag, g);
}
// Some byte of w equals the air id (airw = air id in every byte).
__device__ __forceinline__ bool has_air(uint32_t w, uint32_t airw) {
  const uint32_t x = w ^ airw;
  return ((x - 0x01010101u) & ~x & 0x80808080u) != 0u;
}
__device__ __forceinline__ void st4(float *p, float4 v) {
  *reinterpret_cast<float4 *>(p) = v;
}

__device__ __forceinline__ void build_table16(float *tab, const Params &P) {
  if (threadIdx.x < MAXM * TCOLS)
    tab[threadIdx.x] = gamma_entry(threadIdx.x / TCOLS, threadIdx.x % TCOLS, P.k, P.rho, P.cp,
                                   P.n_mat, P.dx, P.dt, P.h, P.mair);
  __syncthreads();
}

template <class MatT, bool FULL, bool SNAP>
__global__ void __launch_bounds__(256) be_col_kernel(float *__restrict__ dst,
                                                     const float *__restrict__ src,
                                                     const float *__restrict__ told,
                                                     float *__restrict__ snap,
                                                     const MatT *__restrict__ mat, int nx, int ny,
                                                     int nz, int bi, Params P) {
  __shared__ float tab[MAXM * TCOLS];
  build_table16(tab, P);
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (j >= ny) return;  // warp-uniform, after the only barrier
  const int k = (blockIdx.x * 32 + lane) * 4;
  const bool act = FULL || k < nz;
  const int i0 = blockIdx.z * bi;
  const int i1 = min(i0 + bi, nx);
  const int64_t plane = (int64_t)ny * nz;
  const bool has_jm = j > 0, has_jp = j + 1 < ny;
  const uint32_t mair = (uint32_t)P.mair;
  const uint32_t airw = mair * 0x01010101u;
  const float tamb = P.tamb;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  int64_t o = (int64_t)i0 * plane + (int64_t)j * nz + k;

  // plane i0 - 1 and i0 of row j (air -> T_amb); material words of plane i0
  // for rows j -+ 1 and of plane i0 + 1 for row j.  Outside the domain: OOB.
  uint32_t mm = OOBW, mc = OOBW, mjm = OOBW, mjp = OOBW, mn = OOBW;
  float4 pm = z4, pc = z4;
  if (act) {
    if (i0 > 0) {
      mm = mword(mat, o - plane);
      if (mm != airw) pm = ld4(src + o - plane);
      pm = amb4(pm, mm, mair, tamb);
    }
    mc = mword(mat, o);
    if (SNAP || mc != airw) pc = ld4(src + o);
    if (SNAP) st4(snap + o, pc);
    pc = amb4(pc, mc, mair, tamb);
    if (has_jm) mjm = mword(mat, o - nz);
    if (has_jp) mjp = mword(mat, o + nz);
    if (i0 + 1 < nx) mn = mword(mat, o + plane);
  }
  for (int i = i0; i < i1; ++i, o += plane) {
    const bool has_in = i + 1 < nx;
    float4 pn = z4, pjm = z4, pjp = z4, tov = z4;
    uint32_t mn2 = OOBW, mjm2 = OOBW, mjp2 = OOBW;
    if (act) {
      if (has_in && (SNAP || mn != airw)) pn = ld4(src + o + plane);
      if (has_jm && mjm != airw) pjm = ld4(src + o - nz);
      if (has_jp && mjp != airw) pjp = ld4(src + o + nz);
      if (!SNAP && mc != airw) tov = ld4(told + o);
      if (has_in) {
        if (has_jm) mjm2 = mword(mat, o + plane - nz);
        if (has_jp) mjp2 = mword(mat, o + plane + nz);
        if (i + 2 < nx) mn2 = mword(mat, o + 2 * plane);
      }
      if (SNAP && i + 1 < i1) st4(snap + o + plane, pn);  // this CTA's planes only
    }
    pn = amb4(pn, mn, mair, tamb);
    pjm = amb4(pjm, mjm, mair, tamb);
    pjp = amb4(pjp, mjp, mair, tamb);
    if (SNAP) tov = pc;  // air cells changed, but only non-air cells are stored
    float pkm = __shfl_up_sync(0xffffffffu, pc.w, 1);
    uint32_t mkm = __shfl_up_sync(0xffffffffu, mc, 1);
    float pkp = __shfl_down_sync(0xffffffffu, pc.x, 1);
    uint32_t mkp = __shfl_down_sync(0xffffffffu, mc, 1);
    if (lane == 0) {
      if (act && k > 0) {
        const uint32_t b = mbyte(mat, o - 1);
        pkm = b == mair ? tamb : __ldg(src + o - 1);
        mkm = b << 24;
      } else {
        pkm = 0.0f;
        mkm = OOB << 24;
      }
    }
    if (lane == 31) {
      if (act && k + 4 < nz) {
        const uint32_t b = mbyte(mat, o + 4);
        pkp = b == mair ? tamb : __ldg(src + o + 4);
        mkp = b;
      } else {
        pkp = 0.0f;
        mkp = OOB;
      }
    }
    if (__any_sync(0xffffffffu, act && mc != airw)) {
      const uint32_t mb = (mc << 8) | (mkm >> 24);
      const uint32_t mf = (mc >> 8) | (mkp << 24);
      const float4 pb = make_float4(pkm, pc.x, pc.y, pc.z);
      const float4 pf = make_float4(pc.y, pc.z, pc.w, pkp);
      float o4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float *row = tab + (byte_of(mc, q) & (MAXM - 1)) * TCOLS;
        float rhs = 0.0f, diag = 0.0f;
        face_t(rhs, diag, row, mm, q, f4(pm, q));
        face_t(rhs, diag, row, mn, q, f4(pn, q));
        face_t(rhs, diag, row, mjm, q, f4(pjm, q));
        face_t(rhs, diag, row, mjp, q, f4(pjp, q));
        face_t(rhs, diag, row, mb, q, f4(pb, q));
        face_t(rhs, diag, row, mf, q, f4(pf, q));
        o4[q] = __fdiv_rn(__fadd_rn(f4(tov, q), rhs), __fadd_rn(1.0f, diag));
      }
      if (act && mc != airw) {
        if (!has_air(mc, airw)) {
          st4(dst + o, make_float4(o4[0], o4[1], o4[2], o4[3]));
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (byte_of(mc, q) != mair) dst[o + q] = o4[q];
        }
      }
    }
    pm = pc;
    mm = mc;
    pc = pn;
    mc = mn;
    mn = mn2;
    mjm = mjm2;
    mjp = mjp2;
  }
}

// ---- generic kernel: one thread per cell, any shape or alignment ---------------------
template <class MatT, bool SNAP>
__global__ void __launch_bounds__(256) be_generic_kernel(float *__restrict__ dst,
                                                         const float *__restrict__ src,
                                                         const float *__restrict__ told,
                                                         float *__restrict__ snap,
                                                         const MatT *__restrict__ mat, int nx,
                                                         int ny, int nz, Params P) {
  __shared__ float tab[MAXM * MAXM];
  build_table(tab, P);
  const int64_t n = (int64_t)nx * ny * nz;
  const int64_t plane = (int64_t)ny * nz;
  const uint32_t mair = (uint32_t)P.mair;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (SNAP) snap[c] = __ldg(src + c);
    const uint32_t ms = mbyte(mat, c);
    if (ms == mair) continue;
    const int k = (int)(c % nz);
    const int64_t t = c / nz;
    const int j = (int)(t % ny);
    const int i = (int)(t / ny);
    const float *row = tab + (ms & (MAXM - 1)) * MAXM;
    float rhs = 0.0f, diag = 0.0f;
#define FACE(cond, off)                                                                  \
  if (cond) face(rhs, diag, row, true, mbyte(mat, c + (off)), __ldg(src + c + (off)), mair, \
                 P.tamb)
    FACE(i > 0, -plane);
    FACE(i + 1 < nx, plane);
    FACE(j > 0, -(int64_t)nz);
    FACE(j + 1 < ny, (int64_t)nz);
    FACE(k > 0, -1);
    FACE(k + 1 < nz, 1);
#undef FACE
    const float to = SNAP ? __ldg(src + c) : __ldg(told + c);
    dst[c] = __fdiv_rn(__fadd_rn(to, rhs), __fadd_rn(1.0f, diag));
  }
}

// material id narrowing (int32 -> uint8), counting ids outside [0, n_mat)
__global__ void narrow_kernel(uint8_t *__restrict__ out, const int32_t *__restrict__ mat,
                              int64_t n, int n_mat, int *__restrict__ bad) {
  int local = 0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int m = __ldg(mat + c);
    local += (m < 0 || m >= n_mat) ? 1 : 0;
    out[c] = (uint8_t)(m & 0xff);
  }
  if (bad && local) atomicAdd(bad, local);
}

int g_cond_bi = 0;  // plane chunk of the column kernel (0 = rule below)

inline bool al16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

int pick_bi(int nx, int ny, int nz) {
  const int64_t cols = (int64_t)((nz / 4 + 31) / 32) * ((ny + 7) / 8);
  const int64_t target = (int64_t)num_sms() * 8;
  int bi = 64;
  while (bi > 4 && cols * ((nx + bi - 1) / bi) < target) bi >>= 1;
  return bi;
}

template <class MatT, bool SNAP>
cudaError_t launch_sweep(float *dst, const float *src, const float *told, float *snap,
                         const MatT *mat, int nx, int ny, int nz, const Params &P,
                         cudaStream_t s) {
  const bool col_ok = nz % 4 == 0 && al16(dst) && al16(src) && (SNAP ? al16(snap) : al16(told)) &&
                      (sizeof(MatT) == 4 ? al16(mat) : (((uintptr_t)mat & 3u) == 0));
  if (col_ok) {
    const int bi = g_cond_bi > 0 ? g_cond_bi : pick_bi(nx, ny, nz);
    dim3 grid((nz / 4 + 31) / 32, (ny + 7) / 8, (nx + bi - 1) / bi);
    if (nz % 128 == 0)
      be_col_kernel<MatT, true, SNAP>
          <<<grid, 256, 0, s>>>(dst, src, told, snap, mat, nx, ny, nz, bi, P);
    else
      be_col_kernel<MatT, false, SNAP>
          <<<grid, 256, 0, s>>>(dst, src, told, snap, mat, nx, ny, nz, bi, P);
  } else {
    const int64_t n = (int64_t)nx * ny * nz;
    int64_t b = (n + 255) / 256, cap = (int64_t)num_sms() * 16;
    be_generic_kernel<MatT, SNAP><<<(int)(b < cap ? b : cap), 256, 0, s>>>(
        dst, src, told, snap, mat, nx, ny, nz, P);
  }
  return cudaGetLastError();
}

int check_args(const void *a, const void *b, const void *m, const float *k, const float *rho,
               const float *cp, int n_mat, int mat_air, float dx) {
  if (!a || !b || !m || !k || !rho || !cp) return BSP_ERR_NULL;
  if (n_mat < 1 || n_mat > MAXM || mat_air < 0 || mat_air >= MAXM || !(dx > 0.0f))
    return BSP_ERR_ARG;
  return BSP_OK;
}

template <class MatT>
int sweep(float *T_dst, const float *T_iter, const float *T_old, const MatT *mat, int nx,
          int ny, int nz, const float *k, const float *rho, const float *cp, int n_mat,
          float dx, float dt, float h, float tamb, int mair, cudaStream_t s) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  int st = check_args(T_dst, T_iter, mat, k, rho, cp, n_mat, mair, dx);
  if (st != BSP_OK) return st;
  if (!T_old) return BSP_ERR_NULL;
  if (T_dst == T_iter) return BSP_ERR_ARG;
  const Params P{k, rho, cp, n_mat, dx, dt, h, tamb, mair};
  return (int)launch_sweep<MatT, false>(T_dst, T_iter, T_old, nullptr, mat, nx, ny, nz, P, s);
}

// The conduction step: T_old <- T (fused into the first sweep), n_iter sweeps
// T -> T_alt -> T ..., and T <- T_alt when n_iter is odd.  With n_iter == 0 the
// step is the snapshot alone.
template <class MatT>
int be_step(float *T, float *T_alt, float *T_old, const MatT *mat, int nx, int ny, int nz,
            const float *k, const float *rho, const float *cp, int n_mat, float dx, float dt,
            float h, float tamb, int mair, int n_iter, cudaStream_t s) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  int st = check_args(T, T_alt, mat, k, rho, cp, n_mat, mair, dx);
  if (st != BSP_OK) return st;
  if (!T_old) return BSP_ERR_NULL;
  if (n_iter < 0 || T == T_alt || T == T_old || T_alt == T_old) return BSP_ERR_ARG;
  const size_t bytes = sizeof(float) * (size_t)nx * ny * nz;
  const Params P{k, rho, cp, n_mat, dx, dt, h, tamb, mair};
  if (n_iter == 0)
    return (int)cudaMemcpyAsync(T_old, T, bytes, cudaMemcpyDeviceToDevice, s);
  cudaError_t e = launch_sweep<MatT, true>(T_alt, T, nullptr, T_old, mat, nx, ny, nz, P, s);
  for (int it = 1; it < n_iter && e == cudaSuccess; ++it) {
    const float *src = (it % 2 == 0) ? T : T_alt;
    float *dst = (it % 2 == 0) ? T_alt : T;
    e = launch_sweep<MatT, false>(dst, src, T_old, nullptr, mat, nx, ny, nz, P, s);
  }
  if (e == cudaSuccess && n_iter % 2 == 1)
    e = cudaMemcpyAsync(T, T_alt, bytes, cudaMemcpyDeviceToDevice, s);
  return (int)e;
}

}  // namespace cond
}  // namespace bsp

using namespace bsp::cond;

extern "C" int bsp_conduction_sweep(float *T_dst, const float *T_iter, const float *T_old,
                                    const int32_t *mat, int nx, int ny, int nz, const float *k,
                                    const float *rho, const float *cp, int n_mat, float dx,
                                    float dt, float h_conv_air, float T_amb, int mat_air,
                                    cudaStream_t s) {
  return sweep<int32_t>(T_dst, T_iter, T_old, mat, nx, ny, nz, k, rho, cp, n_mat, dx, dt,
                        h_conv_air, T_amb, mat_air, s);
}

extern "C" int bsp_conduction_sweep_u8(float *T_dst, const float *T_iter, const float *T_old,
                                       const uint8_t *mat_id, int nx, int ny, int nz,
                                       const float *k, const float *rho, const float *cp,
                                       int n_mat, float dx, float dt, float h_conv_air,
                                       float T_amb, int mat_air, cudaStream_t s) {
  return sweep<uint8_t>(T_dst, T_iter, T_old, mat_id, nx, ny, nz, k, rho, cp, n_mat, dx, dt,
                        h_conv_air, T_amb, mat_air, s);
}

extern "C" int bsp_conduction_be(float *T, float *T_alt, float *T_old, const int32_t *mat,
                                 int nx, int ny, int nz, const float *k, const float *rho,
                                 const float *cp, int n_mat, float dx, float dt,
                                 float h_conv_air, float T_amb, int mat_air, int n_iter,
                                 cudaStream_t s) {
  return be_step<int32_t>(T, T_alt, T_old, mat, nx, ny, nz, k, rho, cp, n_mat, dx, dt,
                          h_conv_air, T_amb, mat_air, n_iter, s);
}

extern "C" int bsp_conduction_be_u8(float *T, float *T_alt, float *T_old, const uint8_t *mat_id,
                                    int nx, int ny, int nz, const float *k, const float *rho,
                                    const float *cp, int n_mat, float dx, float dt,
                                    float h_conv_air, float T_amb, int mat_air, int n_iter,
                                    cudaStream_t s) {
  return be_step<uint8_t>(T, T_alt, T_old, mat_id, nx, ny, nz, k, rho, cp, n_mat, dx, dt,
                          h_conv_air, T_amb, mat_air, n_iter, s);
}

extern "C" int bsp_material_ids(uint8_t *mat_id, const int32_t *mat, int64_t n, int n_mat,
                                int *bad_count_dev, cudaStream_t s) {
  if (n <= 0) return BSP_OK;
  if (!mat_id || !mat) return BSP_ERR_NULL;
  if (n_mat < 1 || n_mat > MAXM) return BSP_ERR_ARG;
  int64_t b = (n + 255) / 256, cap = (int64_t)bsp::num_sms() * 16;
  narrow_kernel<<<(int)(b < cap ? b : cap), 256, 0, s>>>(mat_id, mat, n, n_mat, bad_count_dev);
  return (int)cudaGetLastError();
}
