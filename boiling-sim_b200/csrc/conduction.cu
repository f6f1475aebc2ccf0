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
#include "tma.cuh"

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

// ---- cell classes --------------------------------------------------------------------
// A non-air cell's update is fixed by its own material and the codes of its
// six neighbours (material id, or EDGE for a face on the domain edge): the
// key own | code(-x) << 3 | code(+x) << 6 | ... | code(+z) << 18.  The
// prepare pass numbers the distinct keys of a geometry 1..n (n <= 127); an air
// cell gets CLS_AIR (sign bit set), and 0 is what a TMA tile reads outside
// the grid.  Each CTA turns the keys into a table of (1 + sum gamma,
// gamma_-x .. gamma_+z) -- gamma 0 on EDGE faces, the denominator summed in
// face order as the reference does -- so a cell costs one class byte and two
// shared loads instead of six table lookups and the diagonal sum.  A value
// outside the grid (0) always meets gamma 0; an air value is replaced by
// T_amb, selected by the class byte's sign bit.
constexpr int NCLS = 256;  // table entries (ids >= n_classes, air included, are zero)
constexpr uint32_t CLS_AIR = 0x80u;
constexpr int CLS_MAX = 127;
constexpr int KEYBITS = 21;
constexpr uint32_t NKEYWORDS = 1u << (KEYBITS - 5);
constexpr uint32_t EDGE = 7u;
constexpr int SCAN_THREADS = 1024;

template <class MatT>
__device__ __forceinline__ uint32_t cell_key(const MatT *mat, int64_t c, int i, int j, int k,
                                             int nx, int ny, int nz, int64_t plane) {
  const uint32_t own = mbyte(mat, c) & 7u;
  const uint32_t cxm = i > 0 ? mbyte(mat, c - plane) & 7u : EDGE;
  const uint32_t cxp = i + 1 < nx ? mbyte(mat, c + plane) & 7u : EDGE;
  const uint32_t cym = j > 0 ? mbyte(mat, c - nz) & 7u : EDGE;
  const uint32_t cyp = j + 1 < ny ? mbyte(mat, c + nz) & 7u : EDGE;
  const uint32_t czm = k > 0 ? mbyte(mat, c - 1) & 7u : EDGE;
  const uint32_t czp = k + 1 < nz ? mbyte(mat, c + 1) & 7u : EDGE;
  return own | cxm << 3 | cxp << 6 | cym << 9 | cyp << 12 | czm << 15 | czp << 18;
}

__device__ __forceinline__ int mraw(const uint8_t *m, int64_t c) { return __ldg(m + c); }
__device__ __forceinline__ int mraw(const int32_t *m, int64_t c) { return __ldg(m + c); }

// Marks the keys present; ids outside [0, n_mat) are counted into *bad and
// marked nothing (the keys hold 3-bit codes).
template <class MatT>
__global__ void cls_mark_kernel(uint32_t *__restrict__ bitmap, const MatT *__restrict__ mat,
                                int nx, int ny, int nz, uint32_t mair, int n_mat,
                                int *__restrict__ bad) {
  const int64_t n = (int64_t)nx * ny * nz, plane = (int64_t)ny * nz;
  int local = 0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int raw = mraw(mat, c);
    if (raw < 0 || raw >= n_mat) {
      ++local;
      continue;
    }
    if ((uint32_t)raw == mair) continue;
    const int k = (int)(c % nz);
    const int64_t t = c / nz;
    const uint32_t key = cell_key(mat, c, (int)(t / ny), (int)(t % ny), k, nx, ny, nz, plane);
    const uint32_t bit = 1u << (key & 31u);
    if (!(__ldg(bitmap + (key >> 5)) & bit)) atomicOr(bitmap + (key >> 5), bit);
  }
  if (local) atomicAdd(bad, local);
}

// Exclusive prefix of the bitmap words' population counts; *count = total.
__global__ void __launch_bounds__(SCAN_THREADS) cls_scan_kernel(uint32_t *__restrict__ base,
                                                                const uint32_t *__restrict__ bitmap,
                                                                int *__restrict__ count) {
  constexpr int PER = NKEYWORDS / SCAN_THREADS;
  __shared__ uint32_t part[SCAN_THREADS];
  const int t = threadIdx.x;
  uint32_t sum = 0;
  for (int w = 0; w < PER; ++w) sum += __popc(bitmap[t * PER + w]);
  part[t] = sum;
  __syncthreads();
  for (int off = 1; off < SCAN_THREADS; off <<= 1) {  // Hillis-Steele inclusive scan
    const uint32_t v = t >= off ? part[t - off] : 0u;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  uint32_t run = part[t] - sum;
  for (int w = 0; w < PER; ++w) {
    base[t * PER + w] = run;
    run += __popc(bitmap[t * PER + w]);
  }
  if (t == SCAN_THREADS - 1) *count = (int)part[t];
}

template <class MatT>
__global__ void cls_assign_kernel(uint8_t *__restrict__ cls, uint32_t *__restrict__ patterns,
                                  const uint32_t *__restrict__ bitmap,
                                  const uint32_t *__restrict__ base, const MatT *__restrict__ mat,
                                  int nx, int ny, int nz, uint32_t mair) {
  const int64_t n = (int64_t)nx * ny * nz, plane = (int64_t)ny * nz;
  if (blockIdx.x == 0 && threadIdx.x == 0) patterns[0] = 0xffffffffu;  // air
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (mbyte(mat, c) == mair) {
      cls[c] = (uint8_t)CLS_AIR;
      continue;
    }
    const int k = (int)(c % nz);
    const int64_t t = c / nz;
    const uint32_t key = cell_key(mat, c, (int)(t / ny), (int)(t % ny), k, nx, ny, nz, plane);
    const uint32_t w = key >> 5, b = key & 31u;
    const uint32_t id = 1u + __ldg(base + w) + __popc(__ldg(bitmap + w) & ((1u << b) - 1u));
    cls[c] = (uint8_t)id;  // the host checked id <= CLS_MAX
    patterns[id] = key;    // every cell of a class writes the same key
  }
}

// Per-CTA class table: tab[2c] = (1 + sum gamma, g-x, g+x, g-y), tab[2c+1] =
// (g+y, g-z, g+z, 0).  gamma of a material pair as in gamma_entry; EDGE and
// ids >= n_mat give 0.  Class 0 (air) gets den 1 and zero gammas.
__device__ __forceinline__ void build_class_table(float4 *tab, float *gt,
                                                  const uint32_t *__restrict__ patterns, int ncls,
                                                  const Params &P) {
  if (threadIdx.x < MAXM * MAXM)
    gt[threadIdx.x] = gamma_entry(threadIdx.x / MAXM, threadIdx.x % MAXM, P.k, P.rho, P.cp,
                                  P.n_mat, P.dx, P.dt, P.h, P.mair);
  __syncthreads();
  for (int c = threadIdx.x; c < NCLS; c += blockDim.x) {
    float g[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float diag = 0.0f;
    if (c > 0 && c < ncls) {
      const uint32_t key = __ldg(patterns + c);
      const float *row = gt + (key & 7u) * MAXM;
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        g[f] = row[(key >> (3 + 3 * f)) & 7u];
        diag = __fadd_rn(diag, g[f]);
      }
    }
    tab[2 * c] = make_float4(__fadd_rn(1.0f, diag), g[0], g[1], g[2]);
    tab[2 * c + 1] = make_float4(g[3], g[4], g[5], 0.0f);
  }
  __syncthreads();
}

// Air values -> T_amb by the sign bit of each class byte (one prmt + one lop3).
__device__ __forceinline__ float ambq(float v, uint32_t w, int q, uint32_t tb) {
  const uint32_t m = sign_bytes(w, (uint32_t)(8 | q) * 0x1111u);
  return __uint_as_float((__float_as_uint(v) & ~m) | (tb & m));
}
__device__ __forceinline__ float4 amb04(float4 v, uint32_t w, float tamb) {
  const uint32_t tb = __float_as_uint(tamb);
  return make_float4(ambq(v.x, w, 0, tb), ambq(v.y, w, 1, tb), ambq(v.z, w, 2, tb),
                     ambq(v.w, w, 3, tb));
}
__device__ __forceinline__ float amb1(float v, uint32_t b, float tamb) {
  return (b & CLS_AIR) ? tamb : v;
}
// A word of four in-grid class bytes: some / every cell is not air.
__device__ __forceinline__ bool cls_some(uint32_t w) {
  return (w & 0x80808080u) != 0x80808080u;
}
__device__ __forceinline__ bool cls_every(uint32_t w) { return (w & 0x80808080u) == 0u; }

// One cell of class c: rhs over the faces -x, +x, -y, +y, -z, +z in order.
__device__ __forceinline__ float be_cell(const float4 *tab, uint32_t c, float tm, float tp,
                                         float tjm, float tjp, float tkm, float tkp, float to) {
  const float4 A = tab[2 * c], B = tab[2 * c + 1];
  float rhs = __fadd_rn(0.0f, __fmul_rn(A.y, tm));
  rhs = __fadd_rn(rhs, __fmul_rn(A.z, tp));
  rhs = __fadd_rn(rhs, __fmul_rn(A.w, tjm));
  rhs = __fadd_rn(rhs, __fmul_rn(B.x, tjp));
  rhs = __fadd_rn(rhs, __fmul_rn(B.y, tkm));
  rhs = __fadd_rn(rhs, __fmul_rn(B.z, tkp));
  return __fdiv_rn(__fadd_rn(to, rhs), A.x);
}
// Store the non-air cells of a word.
__device__ __forceinline__ void store_word(float *p, uint32_t w, const float (&v)[4]) {
  if (cls_every(w)) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (!(byte_of(w, q) & CLS_AIR)) p[q] = v[q];
  }
}

// Column kernel on class bytes (nz % 4 == 0): the layout of be_col_kernel.
// Words outside the grid are 0 (never loaded; their values are 0).
template <bool FULL, bool SNAP>
__global__ void __launch_bounds__(256) be_cls_col_kernel(
    float *__restrict__ dst, const float *__restrict__ src, const float *__restrict__ told,
    float *__restrict__ snap, const uint8_t *__restrict__ cls,
    const uint32_t *__restrict__ patterns, int ncls, int nx, int ny, int nz, int bi, Params P) {
  __shared__ float4 tab[2 * NCLS];
  __shared__ float gt[MAXM * MAXM];
  build_class_table(tab, gt, patterns, ncls, P);
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (j >= ny) return;  // warp-uniform, after the last barrier
  const int k = (blockIdx.x * 32 + lane) * 4;
  const bool act = FULL || k < nz;
  const int i0 = blockIdx.z * bi;
  const int i1 = min(i0 + bi, nx);
  const int64_t plane = (int64_t)ny * nz;
  const bool has_jm = j > 0, has_jp = j + 1 < ny;
  const float tamb = P.tamb;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  int64_t o = (int64_t)i0 * plane + (int64_t)j * nz + k;
  auto live = [](uint32_t w) { return w != 0u && cls_some(w); };  // in grid, not all air

  uint32_t wm = 0u, wc = 0u, wjm = 0u, wjp = 0u, wn = 0u;
  float4 pm = z4, pc = z4;
  if (act) {
    if (i0 > 0) {
      wm = mword(cls, o - plane);
      if (live(wm)) pm = ld4(src + o - plane);
    }
    wc = mword(cls, o);
    if (SNAP || live(wc)) pc = ld4(src + o);
    if (SNAP) st4(snap + o, pc);
    if (has_jm) wjm = mword(cls, o - nz);
    if (has_jp) wjp = mword(cls, o + nz);
    if (i0 + 1 < nx) wn = mword(cls, o + plane);
  }
  pm = amb04(pm, wm, tamb);
  pc = amb04(pc, wc, tamb);
  for (int i = i0; i < i1; ++i, o += plane) {
    const bool has_in = i + 1 < nx;
    float4 pn = z4, pjm = z4, pjp = z4, tov = z4;
    uint32_t wn2 = 0u, wjm2 = 0u, wjp2 = 0u;
    if (act) {
      if (has_in && (SNAP || live(wn))) pn = ld4(src + o + plane);
      if (live(wjm)) pjm = ld4(src + o - nz);
      if (live(wjp)) pjp = ld4(src + o + nz);
      if (!SNAP && live(wc)) tov = ld4(told + o);
      if (has_in) {
        if (has_jm) wjm2 = mword(cls, o + plane - nz);
        if (has_jp) wjp2 = mword(cls, o + plane + nz);
        if (i + 2 < nx) wn2 = mword(cls, o + 2 * plane);
      }
      if (SNAP && i + 1 < i1) st4(snap + o + plane, pn);  // this CTA's planes only
    }
    pn = amb04(pn, wn, tamb);
    pjm = amb04(pjm, wjm, tamb);
    pjp = amb04(pjp, wjp, tamb);
    if (SNAP) tov = pc;
    float pkm = __shfl_up_sync(0xffffffffu, pc.w, 1);
    float pkp = __shfl_down_sync(0xffffffffu, pc.x, 1);
    if (lane == 0) pkm = act && k > 0 ? amb1(__ldg(src + o - 1), __ldg(cls + o - 1), tamb) : 0.0f;
    if (lane == 31)
      pkp = act && k + 4 < nz ? amb1(__ldg(src + o + 4), __ldg(cls + o + 4), tamb) : 0.0f;
    if (__any_sync(0xffffffffu, act && live(wc))) {
      float o4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        o4[q] = be_cell(tab, byte_of(wc, q), f4(pm, q), f4(pn, q), f4(pjm, q), f4(pjp, q),
                        q == 0 ? pkm : f4(pc, q - 1), q == 3 ? pkp : f4(pc, q + 1), f4(tov, q));
      if (act && live(wc)) store_word(dst + o, wc, o4);
    }
    pm = pc;
    pc = pn;
    wc = wn;
    wn = wn2;
    wjm = wjm2;
    wjp = wjp2;
  }
}

// ---- TMA-fed class kernel ---------------------------------------------------------
// The production sweep for nz % 16 == 0.  A CTA of 8 compute warps owns 8 rows
// x 128 k of bi planes, one row per warp; a producer warp streams each plane's
// tiles -- T
// (rows j0-1 .. j0+8, k0-4 .. k0+131), class bytes (same rows, k0-16 ..
// k0+143) and T_old (the 8 output rows) -- into a ring of NST shared-memory
// stages, NST-1 planes ahead of the plane being computed, so the bytes in
// flight do not depend on how many warps are waiting.  Everything outside the
// grid arrives as TMA zero fill: class 0 and value 0, which meet gamma 0 in
// every class bordering the domain edge.  No global load is left in the plane
// loop.  Waits are bounded: a wait that gives up sets the error flag and the
// launch's results are not valid.
namespace tmac {
constexpr int ROWS = 8, TR = ROWS + 2;
constexpr int TP = 4, TW = 128 + 2 * TP;   // T tile row: 136 floats
constexpr int CP = 16, CW = 128 + 2 * CP;  // class tile row: 160 bytes
constexpr int NST = 4;
constexpr int al128(int b) { return (b + 127) / 128 * 128; }
constexpr int TB = TR * TW * 4, CB = TR * CW, OB = ROWS * 128 * 4;
constexpr int OFF_C = al128(TB), OFF_O = OFF_C + al128(CB), STAGE = OFF_O + OB;
constexpr int OFF_TAB = STAGE * NST, OFF_GT = OFF_TAB + 2 * NCLS * 16;
constexpr int OFF_BAR = OFF_GT + MAXM * MAXM * 4, TOTAL = OFF_BAR + NST * 8;
constexpr int THREADS = ROWS * 32;
constexpr int MAX_BI = 64;  // plane chunk cap of the TMA sweep
}  // namespace tmac

struct CondMaps {
  CUtensorMap t, c, o;
};

__device__ int g_cond_err;

__device__ __forceinline__ float4 lds4(const float *p) {
  return *reinterpret_cast<const float4 *>(p);
}
__device__ __forceinline__ uint32_t lds32(const uint8_t *p) {
  return *reinterpret_cast<const uint32_t *>(p);
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Warps 0..7 compute one row each; warp 8 is the producer.  Stage q has a
// "full" barrier (the TMA bytes of its plane have landed) and an "empty"
// barrier (all 8 compute warps are done with its plane); the producer refills
// a stage once it is empty, so a compute warp runs up to NST-2 planes ahead of
// the slowest one instead of meeting it at a CTA barrier every plane.
template <bool SNAP>
__global__ void __launch_bounds__(tmac::THREADS + 32, 4) be_cls_tma_kernel(
    float *__restrict__ dst, float *__restrict__ snap, const __grid_constant__ CondMaps maps,
    const uint32_t *__restrict__ patterns, int ncls, const uint8_t *__restrict__ tiles, int nx,
    int ny, int nz, int bi, Params P) {
  using namespace tmac;
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ uint8_t s_own[MAX_BI + 4];  // tile occupancy of planes pbase-1 .. i1+1
  __shared__ uint64_t s_empty[NST];
  float4 *tab = reinterpret_cast<float4 *>(dsm + OFF_TAB);
  float *gt = reinterpret_cast<float *>(dsm + OFF_GT);
  uint64_t *full = reinterpret_cast<uint64_t *>(dsm + OFF_BAR);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j0 = blockIdx.y * ROWS, k0 = blockIdx.x * 128;
  const int i0 = blockIdx.z * bi, i1 = min(i0 + bi, nx);
  const int pbase = i0 - 1;
  if (threadIdx.x == THREADS) {
    for (int q = 0; q < NST; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&s_empty[q], ROWS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int t = threadIdx.x; t < i1 - pbase + 3; t += blockDim.x) {
    const int p = pbase - 1 + t;
    s_own[t] = p < 0 || p >= nx
                   ? 0
                   : (tiles ? tiles[((int64_t)p * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x]
                            : 1);
  }
  build_class_table(tab, gt, patterns, ncls, P);  // ends with a barrier (all 9 warps)
  bool ok = true;

  if (warp == ROWS) {  // ---- producer warp ----
    if (lane == 0) {
      // Plane p's tiles into its stage.  Without a snapshot to take, T is
      // loaded only when plane p-1, p or p+1 of the tile holds a non-air cell
      // (nothing else reads it) and T_old only for computed planes that hold one.
      for (int p = pbase; p <= i1; ++p) {
        const uint32_t n = (uint32_t)(p - pbase), q = n & (NST - 1);
        if (n >= NST && !mbar_wait(&s_empty[q], ((n - NST) / NST) & 1u)) {
          ok = false;
          break;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        unsigned char *base = dsm + q * STAGE;
        const int f = p - pbase + 1;
        const bool need_t = SNAP || s_own[f - 1] || s_own[f] || s_own[f + 1];
        const bool need_o = !SNAP && p >= i0 && p < i1 && s_own[f];
        mbar_expect_tx(&full[q], (uint32_t)(CB + (need_t ? TB : 0) + (need_o ? OB : 0)));
        if (need_t) tma_load3(base, &maps.t, k0 - TP, j0 - 1, p, &full[q]);
        tma_load3(base + OFF_C, &maps.c, k0 - CP, j0 - 1, p, &full[q]);
        if (need_o) tma_load3(base + OFF_O, &maps.o, k0, j0, p, &full[q]);
      }
      // no copy may still be in flight when the CTA's shared memory goes away
      for (int p = max(pbase, i1 - NST + 1); p <= i1; ++p) {
        const uint32_t n = (uint32_t)(p - pbase);
        if (!mbar_wait(&full[n & (NST - 1)], (n / NST) & 1u)) ok = false;
      }
      if (!ok) atomicExch(&g_cond_err, 1);
    }
    return;
  }

  // ---- compute warps ----
  auto wait = [&](int p) {
    const uint32_t n = (uint32_t)(p - pbase);
    if (!mbar_wait(&full[n & (NST - 1)], (n / NST) & 1u)) ok = false;
  };
  auto release = [&](uint32_t q) {  // this warp is done with stage q
    __syncwarp();
    if (lane == 0) mbar_arrive(&s_empty[q]);
  };
  const int j = j0 + warp;
  const int k = k0 + lane * 4;
  const bool act = j < ny && k < nz;
  const float tamb = P.tamb;
  const int64_t plane = (int64_t)ny * nz;
  // offsets of this lane's four cells in a stage (tile row warp + 1)
  const int tro = (warp + 1) * TW + TP + lane * 4, cro = OFF_C + (warp + 1) * CW + CP + lane * 4;
  const int oro = OFF_O + (warp * 128 + lane * 4) * 4;
  wait(pbase);
  float4 pm = amb04(lds4(reinterpret_cast<const float *>(dsm) + tro), lds32(dsm + cro), tamb);
  release(0);
  wait(i0);
  const unsigned char *b1 = dsm + STAGE;  // plane i0 is in stage 1
  uint32_t wc = lds32(b1 + cro);
  float4 pcr = lds4(reinterpret_cast<const float *>(b1) + tro);
  float4 pc = amb04(pcr, wc, tamb);
  uint32_t sc = 1;  // stage of plane i
  int64_t o = (int64_t)i0 * plane + (int64_t)j * nz + k;
  for (int i = i0; i < i1; ++i, o += plane) {
    const uint32_t sn = (sc + 1) & (NST - 1);
    wait(i + 1);
    const unsigned char *bn = dsm + sn * STAGE;
    const uint32_t wn = lds32(bn + cro);
    const float4 pnr = lds4(reinterpret_cast<const float *>(bn) + tro);
    const float4 pn = amb04(pnr, wn, tamb);
    if (SNAP && act) st4(snap + o, pcr);
    const bool live = act && cls_some(wc);
    if (__any_sync(0xffffffffu, live)) {
      const unsigned char *bc = dsm + sc * STAGE;
      const float *tc = reinterpret_cast<const float *>(bc);
      const float4 pjm = amb04(lds4(tc + tro - TW), lds32(bc + cro - CW), tamb);
      const float4 pjp = amb04(lds4(tc + tro + TW), lds32(bc + cro + CW), tamb);
      float pkm = __shfl_up_sync(0xffffffffu, pc.w, 1);
      float pkp = __shfl_down_sync(0xffffffffu, pc.x, 1);
      if (lane == 0) pkm = amb1(tc[tro - 1], bc[cro - 1], tamb);
      if (lane == 31) pkp = amb1(tc[tro + 4], bc[cro + 4], tamb);
      const float4 tov = SNAP ? pcr : *reinterpret_cast<const float4 *>(bc + oro);
      float o4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        o4[q] = be_cell(tab, byte_of(wc, q), f4(pm, q), f4(pn, q), f4(pjm, q), f4(pjp, q),
                        q == 0 ? pkm : f4(pc, q - 1), q == 3 ? pkp : f4(pc, q + 1), f4(tov, q));
      if (live) store_word(dst + o, wc, o4);
    }
    release(sc);  // plane i's stage
    pm = pc;
    pc = pn;
    pcr = pnr;
    wc = wn;
    sc = sn;
  }
  // plane i1 (the last one read) is in stage sc: nothing refills it, no release needed
  if (!ok) atomicExch(&g_cond_err, 1);
}

// Tile occupancy for the TMA sweep: tiles[(i * TY + j / ROWS) * TX + k / 128]
// = 1 when that plane's ROWS x 128 tile holds a non-air cell (TY, TX: tiles
// per plane along j and k).
__global__ void tile_flags_kernel(uint8_t *__restrict__ tiles, const uint8_t *__restrict__ cls,
                                  int nx, int ny, int nz) {
  const int ty = (ny + tmac::ROWS - 1) / tmac::ROWS, tx = (nz + 127) / 128;
  const int64_t nw = (int64_t)nx * ny * (nz / 4);
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw;
       w += (int64_t)gridDim.x * blockDim.x) {
    if (!cls_some(__ldg(reinterpret_cast<const uint32_t *>(cls) + w))) continue;
    const int k = (int)(w % (nz / 4)) * 4;
    const int64_t t = w / (nz / 4);
    const int j = (int)(t % ny), i = (int)(t / ny);
    tiles[((int64_t)i * ty + j / tmac::ROWS) * tx + k / 128] = 1;
  }
}

// Class kernel for any shape or alignment: one thread per cell.
template <bool SNAP>
__global__ void __launch_bounds__(256) be_cls_generic_kernel(
    float *__restrict__ dst, const float *__restrict__ src, const float *__restrict__ told,
    float *__restrict__ snap, const uint8_t *__restrict__ cls,
    const uint32_t *__restrict__ patterns, int ncls, int nx, int ny, int nz, Params P) {
  __shared__ float4 tab[2 * NCLS];
  __shared__ float gt[MAXM * MAXM];
  build_class_table(tab, gt, patterns, ncls, P);
  const int64_t n = (int64_t)nx * ny * nz, plane = (int64_t)ny * nz;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (SNAP) snap[c] = __ldg(src + c);
    const uint32_t cl = __ldg(cls + c);
    if (cl & CLS_AIR) continue;
    const int k = (int)(c % nz);
    const int64_t t = c / nz;
    const int j = (int)(t % ny), i = (int)(t / ny);
#define NB(cond, off) ((cond) ? amb1(__ldg(src + c + (off)), __ldg(cls + c + (off)), P.tamb) : 0.0f)
    const float tv[6] = {NB(i > 0, -plane), NB(i + 1 < nx, plane), NB(j > 0, -(int64_t)nz),
                         NB(j + 1 < ny, (int64_t)nz), NB(k > 0, -1), NB(k + 1 < nz, 1)};
#undef NB
    const float4 A = tab[2 * cl], B = tab[2 * cl + 1];
    const float g[6] = {A.y, A.z, A.w, B.x, B.y, B.z};
    float rhs = 0.0f;
#pragma unroll
    for (int f = 0; f < 6; ++f) rhs = __fadd_rn(rhs, __fmul_rn(g[f], tv[f]));
    const float to = SNAP ? __ldg(src + c) : __ldg(told + c);
    dst[c] = __fdiv_rn(__fadd_rn(to, rhs), A.x);
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

bool g_cond_tma = true;  // TMA-fed class kernel when the layout allows it

int tma_bi(int nx, int ny, int nz) {
  if (g_cond_bi > 0) return min(g_cond_bi, tmac::MAX_BI);
  const int64_t cols = (int64_t)((nz + 127) / 128) * ((ny + tmac::ROWS - 1) / tmac::ROWS);
  int bi = 32;
  while (bi > 8 && cols * ((nx + bi - 1) / bi) < 8LL * num_sms()) bi >>= 1;  // 4 CTAs / SM
  return bi;
}

template <bool SNAP>
bool launch_cls_tma(float *dst, const float *src, const float *told, float *snap,
                    const uint8_t *cls, const uint32_t *patterns, int ncls, const uint8_t *tiles,
                    int nx, int ny, int nz, const Params &P, cudaStream_t s) {
  using namespace tmac;
  if (!g_cond_tma || nz % 16 || !al16(dst) || (SNAP && !al16(snap))) return false;
  CondMaps maps;
  if (!make_map(&maps.t, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, src, nx, ny, nz, TW, TR) ||
      !make_map(&maps.c, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, cls, nx, ny, nz, CW, TR))
    return false;
  if (!SNAP && !make_map(&maps.o, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, told, nx, ny, nz, 128, ROWS))
    return false;
  if (SNAP) maps.o = maps.t;
  // the shared-memory opt-in is per device
  if (!smem_opt_in((const void *)be_cls_tma_kernel<SNAP>, TOTAL)) return false;
  const int bi = tma_bi(nx, ny, nz);
  dim3 grid((nz + 127) / 128, (ny + ROWS - 1) / ROWS, (nx + bi - 1) / bi);
  be_cls_tma_kernel<SNAP><<<grid, THREADS + 32, TOTAL, s>>>(dst, snap, maps, patterns, ncls,
                                                            tiles, nx, ny, nz, bi, P);
  return cudaGetLastError() == cudaSuccess;
}

template <bool SNAP>
cudaError_t launch_cls_sweep(float *dst, const float *src, const float *told, float *snap,
                             const uint8_t *cls, const uint32_t *patterns, int ncls,
                             const uint8_t *tiles, int nx, int ny, int nz, const Params &P,
                             cudaStream_t s) {
  if (launch_cls_tma<SNAP>(dst, src, told, snap, cls, patterns, ncls, tiles, nx, ny, nz, P, s))
    return cudaGetLastError();
  const bool col_ok = nz % 4 == 0 && al16(dst) && al16(src) &&
                      (SNAP ? al16(snap) : al16(told)) && (((uintptr_t)cls & 3u) == 0);
  if (col_ok) {
    const int bi = g_cond_bi > 0 ? g_cond_bi : pick_bi(nx, ny, nz);
    dim3 grid((nz / 4 + 31) / 32, (ny + 7) / 8, (nx + bi - 1) / bi);
    if (nz % 128 == 0)
      be_cls_col_kernel<true, SNAP><<<grid, 256, 0, s>>>(dst, src, told, snap, cls, patterns,
                                                         ncls, nx, ny, nz, bi, P);
    else
      be_cls_col_kernel<false, SNAP><<<grid, 256, 0, s>>>(dst, src, told, snap, cls, patterns,
                                                          ncls, nx, ny, nz, bi, P);
  } else {
    const int64_t n = (int64_t)nx * ny * nz;
    int64_t b = (n + 255) / 256, cap = (int64_t)num_sms() * 16;
    be_cls_generic_kernel<SNAP><<<(int)(b < cap ? b : cap), 256, 0, s>>>(
        dst, src, told, snap, cls, patterns, ncls, nx, ny, nz, P);
  }
  return cudaGetLastError();
}

size_t prepare_workspace_bytes() { return 2 * sizeof(uint32_t) * NKEYWORDS + 256; }

template <class MatT>
int prepare(uint8_t *cls, uint32_t *patterns, int *n_classes_host, const MatT *mat, int nx,
            int ny, int nz, int n_mat, int mat_air, void *ws, size_t ws_bytes, cudaStream_t s) {
  if (!cls || !patterns || !n_classes_host || !mat || !ws) return BSP_ERR_NULL;
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_ERR_SHAPE;
  if (n_mat < 1 || n_mat > MAXM - 1 || mat_air < 0 || mat_air >= n_mat) return BSP_ERR_ARG;
  if (ws_bytes < prepare_workspace_bytes() || ((uintptr_t)ws & 15u)) return BSP_ERR_WORKSPACE;
  uint32_t *bitmap = static_cast<uint32_t *>(ws);
  uint32_t *base = bitmap + NKEYWORDS;
  int *count = reinterpret_cast<int *>(base + NKEYWORDS);  // [0] classes, [1] bad ids
  const int64_t n = (int64_t)nx * ny * nz;
  int64_t b = (n + 255) / 256, cap = (int64_t)num_sms() * 16;
  const int blocks = (int)(b < cap ? b : cap);
  cudaError_t e = cudaMemsetAsync(bitmap, 0, sizeof(uint32_t) * NKEYWORDS, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(count, 0, 2 * sizeof(int), s);
  if (e != cudaSuccess) return (int)e;
  cls_mark_kernel<MatT><<<blocks, 256, 0, s>>>(bitmap, mat, nx, ny, nz, (uint32_t)mat_air,
                                               n_mat, count + 1);
  cls_scan_kernel<<<1, SCAN_THREADS, 0, s>>>(base, bitmap, count);
  int host[2] = {0, 0};
  e = cudaMemcpyAsync(host, count, sizeof(host), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return (int)e;
  const int host_count = host[0];
  *n_classes_host = host_count + 1;
  if (host[1] > 0) {  // material ids outside [0, n_mat)
    *n_classes_host = 0;
    return BSP_ERR_ARG;
  }
  if (host_count > CLS_MAX) return BSP_ERR_CAPACITY;
  cls_assign_kernel<MatT><<<blocks, 256, 0, s>>>(cls, patterns, bitmap, base, mat, nx, ny, nz,
                                                 (uint32_t)mat_air);
  return (int)cudaGetLastError();
}

int cls_args(const void *a, const void *b, const uint8_t *cls, const uint32_t *patterns,
             int ncls, const float *k, const float *rho, const float *cp, int n_mat, int mat_air,
             float dx) {
  if (!a || !b || !cls || !patterns || !k || !rho || !cp) return BSP_ERR_NULL;
  if (ncls < 1 || ncls > CLS_MAX + 1 || n_mat < 1 || n_mat > MAXM - 1 || mat_air < 0 ||
      mat_air >= n_mat || !(dx > 0.0f))
    return BSP_ERR_ARG;
  return BSP_OK;
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

extern "C" size_t bsp_conduction_prepare_workspace_bytes(void) {
  return prepare_workspace_bytes();
}

extern "C" int bsp_conduction_prepare(uint8_t *cls, uint32_t *patterns, int *n_classes_host,
                                      const int32_t *mat, int nx, int ny, int nz, int n_mat,
                                      int mat_air, void *workspace, size_t workspace_bytes,
                                      cudaStream_t s) {
  return prepare<int32_t>(cls, patterns, n_classes_host, mat, nx, ny, nz, n_mat, mat_air,
                          workspace, workspace_bytes, s);
}

extern "C" int bsp_conduction_sweep_cls(float *T_dst, const float *T_iter, const float *T_old,
                                        const uint8_t *cls, const uint32_t *patterns,
                                        int n_classes, const uint8_t *tiles, int nx, int ny,
                                        int nz, const float *k,
                                        const float *rho, const float *cp, int n_mat, float dx,
                                        float dt, float h_conv_air, float T_amb, int mat_air,
                                        cudaStream_t s) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  int st = cls_args(T_dst, T_iter, cls, patterns, n_classes, k, rho, cp, n_mat, mat_air, dx);
  if (st != BSP_OK) return st;
  if (!T_old) return BSP_ERR_NULL;
  if (T_dst == T_iter) return BSP_ERR_ARG;
  const Params P{k, rho, cp, n_mat, dx, dt, h_conv_air, T_amb, mat_air};
  return (int)launch_cls_sweep<false>(T_dst, T_iter, T_old, nullptr, cls, patterns, n_classes,
                                      tiles, nx, ny, nz, P, s);
}

extern "C" int bsp_conduction_be_cls(float *T, float *T_alt, float *T_old, const uint8_t *cls,
                                     const uint32_t *patterns, int n_classes,
                                     const uint8_t *tiles, int nx, int ny, int nz,
                                     const float *k, const float *rho, const float *cp,
                                     int n_mat, float dx, float dt, float h_conv_air,
                                     float T_amb, int mat_air, int n_iter, cudaStream_t s) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  int st = cls_args(T, T_alt, cls, patterns, n_classes, k, rho, cp, n_mat, mat_air, dx);
  if (st != BSP_OK) return st;
  if (!T_old) return BSP_ERR_NULL;
  if (n_iter < 0 || T == T_alt || T == T_old || T_alt == T_old) return BSP_ERR_ARG;
  const size_t bytes = sizeof(float) * (size_t)nx * ny * nz;
  const Params P{k, rho, cp, n_mat, dx, dt, h_conv_air, T_amb, mat_air};
  if (n_iter == 0) return (int)cudaMemcpyAsync(T_old, T, bytes, cudaMemcpyDeviceToDevice, s);
  cudaError_t e = launch_cls_sweep<true>(T_alt, T, nullptr, T_old, cls, patterns, n_classes,
                                         tiles, nx, ny, nz, P, s);
  for (int it = 1; it < n_iter && e == cudaSuccess; ++it) {
    const float *src = (it % 2 == 0) ? T : T_alt;
    float *dst = (it % 2 == 0) ? T_alt : T;
    e = launch_cls_sweep<false>(dst, src, T_old, nullptr, cls, patterns, n_classes, tiles, nx,
                                ny, nz, P, s);
  }
  if (e == cudaSuccess && n_iter % 2 == 1)
    e = cudaMemcpyAsync(T, T_alt, bytes, cudaMemcpyDeviceToDevice, s);
  return (int)e;
}

extern "C" int bsp_conduction_error(int *flag_host) {
  if (!flag_host) return BSP_ERR_NULL;
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, bsp::cond::g_cond_err, sizeof(int));
  if (e == cudaSuccess) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(bsp::cond::g_cond_err, &zero, sizeof(int));
  }
  *flag_host = v;
  return (int)e;
}

extern "C" size_t bsp_conduction_tile_flags_bytes(int nx, int ny, int nz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return 0;
  return (size_t)nx * ((ny + tmac::ROWS - 1) / tmac::ROWS) * ((nz + 127) / 128);
}

extern "C" int bsp_conduction_tile_flags(uint8_t *tiles, const uint8_t *cls, int nx, int ny,
                                         int nz, cudaStream_t s) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return BSP_OK;
  if (!tiles || !cls) return BSP_ERR_NULL;
  if (nz % 4 || ((uintptr_t)cls & 3u)) return BSP_ERR_SHAPE;
  cudaError_t e = cudaMemsetAsync(tiles, 0, bsp_conduction_tile_flags_bytes(nx, ny, nz), s);
  if (e != cudaSuccess) return (int)e;
  const int64_t nw = (int64_t)nx * ny * (nz / 4);
  int64_t b = (nw + 255) / 256, cap = (int64_t)bsp::num_sms() * 16;
  tile_flags_kernel<<<(int)(b < cap ? b : cap), 256, 0, s>>>(tiles, cls, nx, ny, nz);
  return (int)cudaGetLastError();
}
