// sweep2.cu -- two Jacobi sweeps per HBM round trip (temporal blocking).
//
// p2 = J(J(p0)) with J the reference's sweep (fluid.py:243-276) in its hoisted
// right-hand-side form, bit-identical to two single sweeps: the same
// operations in the same order, the intermediate p1 kept in shared memory.
// It needs the source zero on non-fluid cells (the ZNF select of stencil.cu:
// fluid -> p_n, air -> 0, solid -> p_self is then p_n | (p_self & solid)),
// which holds from the second sweep of any solve and from the first when p
// starts at zero.
//
// A CTA owns 8 rows (j) x 128 cells (k) of the output and marches the plane
// index i.  Per source plane, TMA brings 12 rows of p0 and of the mask (j0-2
// .. j0+9, k0-PAD .. k0+127+PAD) and 10 rows of the right-hand side into a
// ring of NST mbarrier-completed shared-memory stages; cells outside the grid
// arrive as zeros (p = 0, class air), which is the reference's boundary rule.
// Step s computes p1 on plane s for 10 rows and the k halo (k0-1, k0+128)
// into a 3-plane ring, then p2 on plane s-1 for the 8 output rows, which
// needs p1 on planes s-2 .. s.  Two CTA barriers per step.
#include <cuda_runtime.h>
#include <stdint.h>

#include "bsp_common.cuh"
#include "profile.cuh"
#include "tma.cuh"

namespace bsp {

namespace sw2 {
constexpr int ROWS = 8;              // output rows per CTA
constexpr int R1 = ROWS + 2;         // rows of p1
constexpr int R0 = ROWS + 4;         // rows of p0 and of the mask
constexpr int PAD = 4;               // k halo of the float tiles (16 bytes)
constexpr int FW = 128 + 2 * PAD;    // float tile row (elements)
constexpr int MW = 160;              // mask tile row (bytes), k0-16 .. k0+143
constexpr int MPAD = 16;
constexpr int NST = 6;               // source-plane stages: 4 in use + 2 in flight
constexpr int WARPS = R1;            // warp w computes p1 row w; warps 0..7 also p2 row w
constexpr int THREADS = WARPS * 32;
constexpr int PB = R0 * FW * 4;                        // 6528
constexpr int MB = R0 * MW;                            // 1920
constexpr int RB = R1 * FW * 4;                        // 5440
constexpr int OFF_M = PB;                              // PB is a multiple of 128
constexpr int OFF_R = OFF_M + MB;                      // MB is a multiple of 128
constexpr int STAGE = OFF_R + (RB + 127) / 128 * 128;  // 13952
constexpr int RING = STAGE * NST;
constexpr int L1B = R1 * FW * 4;                       // one p1 plane
constexpr int OFF_L1 = RING;
constexpr int OFF_BAR = OFF_L1 + 3 * L1B;
constexpr int TOTAL = OFF_BAR + NST * 8;
constexpr uint32_t TX = (uint32_t)(PB + MB + RB);
}  // namespace sw2

struct Sweep2Maps {
  CUtensorMap p, m, r;
};

__device__ __forceinline__ float f4q(const float4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}
// fluid -> p_n, air -> 0, solid -> p_self on a source that is +0 off fluid;
// sw holds the neighbour's mask bytes shifted left by one (solid bit at bit 7).
__device__ __forceinline__ float znf_sel(uint32_t sw, int q, float pn, float ps) {
  const uint32_t sm = sign_bytes(sw, (uint32_t)(8 | q) * 0x1111u);
  return __uint_as_float(__float_as_uint(pn) | (__float_as_uint(ps) & sm));
}
// One sweep of up to 4 cells: (l, r, d, u, b, f) neighbours with their mask
// words, centre mask mc, right-hand side rhs; the reference's operation order.
__device__ __forceinline__ float sweep_cell(int q, uint32_t mm, uint32_t mn, uint32_t mjm,
                                            uint32_t mjp, uint32_t mb, uint32_t mf,
                                            uint32_t mc, float pl, float pr, float pd,
                                            float pu, float pbk, float pfr, float ps, float rhs) {
  const float l = znf_sel(mm << 1, q, pl, ps);
  const float r = znf_sel(mn << 1, q, pr, ps);
  const float d = znf_sel(mjm << 1, q, pd, ps);
  const float u = znf_sel(mjp << 1, q, pu, ps);
  const float b = znf_sel(mb << 1, q, pbk, ps);
  const float f = znf_sel(mf << 1, q, pfr, ps);
  const float s = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(l, r), d), u), b), f);
  const float v = div6(__fsub_rn(s, rhs));
  return __uint_as_float(__float_as_uint(v) & fluid_word(mc, q));
}

__global__ void __launch_bounds__(sw2::THREADS, 2) sweep2_kernel(
    float *__restrict__ out, const __grid_constant__ Sweep2Maps maps, int nx, int ny, int nz,
    int bi, int *__restrict__ err) {
  using namespace sw2;
  extern __shared__ __align__(128) unsigned char dsm[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(dsm + OFF_BAR);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool producer = threadIdx.x == 0;
  const int k0 = blockIdx.x * 128, j0 = blockIdx.y * ROWS;
  const int i0 = blockIdx.z * bi, i1 = min(i0 + bi, nx);
  const int pbase = i0 - 2;  // first source plane of the ring
  const int plast = i1 + 1;  // last source plane
  const int kl = lane * 4;
  if (producer) {
    for (int q = 0; q < NST; ++q) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int p) {
    const int q = (int)((unsigned)(p - pbase) % NST);
    unsigned char *base = dsm + q * STAGE;
    mbar_expect_tx(&bars[q], TX);
    tma_load3(base, &maps.p, k0 - PAD, j0 - 2, p, &bars[q]);
    tma_load3(base + OFF_M, &maps.m, k0 - MPAD, j0 - 2, p, &bars[q]);
    tma_load3(base + OFF_R, &maps.r, k0 - PAD, j0 - 1, p, &bars[q]);
  };
  bool ok = true;
  auto wait = [&](int p) {
    const unsigned n = (unsigned)(p - pbase);
    if (!mbar_wait(&bars[n % NST], (n / NST) & 1u)) ok = false;
  };
  auto P = [&](int p) {
    return reinterpret_cast<const float *>(dsm + ((unsigned)(p - pbase) % NST) * STAGE);
  };
  auto M = [&](int p) { return dsm + ((unsigned)(p - pbase) % NST) * STAGE + OFF_M; };
  auto R = [&](int p) {
    return reinterpret_cast<const float *>(dsm + ((unsigned)(p - pbase) % NST) * STAGE + OFF_R);
  };
  auto L1 = [&](int p) {  // p1 plane p (p >= i0 - 1)
    return reinterpret_cast<float *>(dsm + OFF_L1 + ((unsigned)(p - (i0 - 1)) % 3) * L1B);
  };
  auto m4 = [](const unsigned char *mrow, int x) {
    return *reinterpret_cast<const uint32_t *>(mrow + MPAD + x);
  };
  if (producer)
    for (int p = pbase; p <= min(pbase + NST - 1, plast); ++p) issue(p);
  wait(pbase);
  wait(pbase + 1);
  for (int s = i0 - 1; s <= i1; ++s) {
    wait(s + 1);
    // ---- p1 on plane s, row r = warp (j = j0 - 1 + r)
    {
      const int r = warp;
      const float *pc_ = P(s) + (r + 1) * FW + PAD, *pm_ = P(s - 1) + (r + 1) * FW + PAD,
                  *pn_ = P(s + 1) + (r + 1) * FW + PAD, *pd_ = P(s) + r * FW + PAD,
                  *pu_ = P(s) + (r + 2) * FW + PAD;
      const unsigned char *mc_ = M(s) + (r + 1) * MW, *mm_ = M(s - 1) + (r + 1) * MW,
                          *mn_ = M(s + 1) + (r + 1) * MW, *md_ = M(s) + r * MW,
                          *mu_ = M(s) + (r + 2) * MW;
      const float *rr_ = R(s) + r * FW + PAD;
      float *o1 = L1(s) + r * FW + PAD;
      const float4 pc = *reinterpret_cast<const float4 *>(pc_ + kl);
      const float4 pm = *reinterpret_cast<const float4 *>(pm_ + kl);
      const float4 pn = *reinterpret_cast<const float4 *>(pn_ + kl);
      const float4 pd = *reinterpret_cast<const float4 *>(pd_ + kl);
      const float4 pu = *reinterpret_cast<const float4 *>(pu_ + kl);
      const float4 rh = *reinterpret_cast<const float4 *>(rr_ + kl);
      const float pkm = pc_[kl - 1], pkp = pc_[kl + 4];
      const uint32_t mc = m4(mc_, kl), mm = m4(mm_, kl), mn = m4(mn_, kl), md = m4(md_, kl),
                     mu = m4(mu_, kl);
      const uint32_t mb = (mc << 8) | mc_[MPAD + kl - 1];
      const uint32_t mf = (mc >> 8) | ((uint32_t)mc_[MPAD + kl + 4] << 24);
      const float4 pb = make_float4(pkm, pc.x, pc.y, pc.z);
      const float4 pf = make_float4(pc.y, pc.z, pc.w, pkp);
      float v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        v[q] = sweep_cell(q, mm, mn, md, mu, mb, mf, mc, f4q(pm, q), f4q(pn, q), f4q(pd, q),
                          f4q(pu, q), f4q(pb, q), f4q(pf, q), f4q(pc, q), f4q(rh, q));
      *reinterpret_cast<float4 *>(o1 + kl) = make_float4(v[0], v[1], v[2], v[3]);
      // k halo of p1: k0 - 1 (lane 0) and k0 + 128 (lane 31), one cell each
      if (lane == 0 || lane == 31) {
        const int x = lane == 0 ? -1 : 128;
        const uint32_t c = mc_[MPAD + x];
        const float h = sweep_cell(0, mm_[MPAD + x], mn_[MPAD + x], md_[MPAD + x], mu_[MPAD + x],
                                   mc_[MPAD + x - 1], mc_[MPAD + x + 1], c, pm_[x], pn_[x],
                                   pd_[x], pu_[x], pc_[x - 1], pc_[x + 1], pc_[x], rr_[x]);
        o1[x] = h;
      }
    }
    __syncthreads();
    // ---- p2 on plane t = s - 1, row w (j = j0 + w)
    const int t = s - 1;
    if (t >= i0 && t < i1 && warp < ROWS) {
      const int w = warp;
      const int j = j0 + w, k = k0 + kl;
      const float *qc_ = L1(t) + (w + 1) * FW + PAD, *qm_ = L1(t - 1) + (w + 1) * FW + PAD,
                  *qn_ = L1(t + 1) + (w + 1) * FW + PAD, *qd_ = L1(t) + w * FW + PAD,
                  *qu_ = L1(t) + (w + 2) * FW + PAD;
      const unsigned char *mc_ = M(t) + (w + 2) * MW, *mm_ = M(t - 1) + (w + 2) * MW,
                          *mn_ = M(t + 1) + (w + 2) * MW, *md_ = M(t) + (w + 1) * MW,
                          *mu_ = M(t) + (w + 3) * MW;
      const float *rr_ = R(t) + (w + 1) * FW + PAD;
      const float4 pc = *reinterpret_cast<const float4 *>(qc_ + kl);
      const float4 pm = *reinterpret_cast<const float4 *>(qm_ + kl);
      const float4 pn = *reinterpret_cast<const float4 *>(qn_ + kl);
      const float4 pd = *reinterpret_cast<const float4 *>(qd_ + kl);
      const float4 pu = *reinterpret_cast<const float4 *>(qu_ + kl);
      const float4 rh = *reinterpret_cast<const float4 *>(rr_ + kl);
      const float pkm = qc_[kl - 1], pkp = qc_[kl + 4];
      const uint32_t mc = m4(mc_, kl), mm = m4(mm_, kl), mn = m4(mn_, kl), md = m4(md_, kl),
                     mu = m4(mu_, kl);
      const uint32_t mb = (mc << 8) | mc_[MPAD + kl - 1];
      const uint32_t mf = (mc >> 8) | ((uint32_t)mc_[MPAD + kl + 4] << 24);
      const float4 pb = make_float4(pkm, pc.x, pc.y, pc.z);
      const float4 pf = make_float4(pc.y, pc.z, pc.w, pkp);
      float v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        v[q] = sweep_cell(q, mm, mn, md, mu, mb, mf, mc, f4q(pm, q), f4q(pn, q), f4q(pd, q),
                          f4q(pu, q), f4q(pb, q), f4q(pf, q), f4q(pc, q), f4q(rh, q));
      if (j < ny && k < nz)
        *reinterpret_cast<float4 *>(out + ((int64_t)t * ny + j) * nz + k) =
            make_float4(v[0], v[1], v[2], v[3]);
    }
    __syncthreads();
    // source plane s - 2 is no longer read: refill its stage
    if (producer && s - 2 + NST <= plast && s - 2 >= pbase) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(s - 2 + NST);
    }
  }
  if (producer)  // confirm (bounded) that nothing is still in flight
    for (int p = max(pbase, plast - NST + 1); p <= plast; ++p) wait(p);
  if (!ok && threadIdx.x == 0) atomicExch(err, 1);
}

// Set by a sweep2 CTA whose bounded TMA wait gave up (the outputs of that
// launch are then not valid); read back by bsp_sweep2_error.
__device__ int g_sweep2_err;
int num_sms();
extern int g_sweep_bi;  // BSP_TUNE_SWEEP_BI (stencil.cu)

// Two sweeps p0 -> out (rhs already hoisted, p0 zero off fluid).  False when
// the TMA path cannot run (nz % 16 != 0, alignment, no driver entry point).
bool launch_sweep2(float *out, const float *p, const float *rhs, const uint8_t *mask, int nx,
                   int ny, int nz, cudaStream_t s) {
  using namespace sw2;
  if (nz % 16 || ((uintptr_t)out & 15u) || !encode_tiled()) return false;
  Sweep2Maps maps{};
  if (!(make_map(&maps.p, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, p, nx, ny, nz, FW, R0) &&
        make_map(&maps.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, mask, nx, ny, nz, MW, R0) &&
        make_map(&maps.r, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, rhs, nx, ny, nz, FW, R1)))
    return false;
  if (!smem_opt_in((const void *)sweep2_kernel, TOTAL)) return false;
  int *err = nullptr;
  if (cudaGetSymbolAddress((void **)&err, g_sweep2_err) != cudaSuccess) return false;
  const int64_t cols = (int64_t)((nz + 127) / 128) * ((ny + ROWS - 1) / ROWS);
  int bi = 16;
  while (bi > 2 && cols * ((nx + bi - 1) / bi) < 2LL * num_sms()) bi -= 2;
  if (g_sweep_bi > 0) bi = g_sweep_bi;
  dim3 grid((nz + 127) / 128, (ny + ROWS - 1) / ROWS, (nx + bi - 1) / bi);
  sweep2_kernel<<<grid, THREADS, TOTAL, s>>>(out, maps, nx, ny, nz, bi, err);
  return cudaGetLastError() == cudaSuccess;
}

}  // namespace bsp

// Device flag of a sweep2 launch whose TMA wait timed out: 1 if any did since
// the last call (the flag is cleared); synchronises the device.
extern "C" int bsp_sweep2_error(int *flag_host) {
  if (!flag_host) return BSP_ERR_NULL;
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, bsp::g_sweep2_err, sizeof(int));
  if (e == cudaSuccess) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(bsp::g_sweep2_err, &zero, sizeof(int));
  }
  *flag_host = v;
  return (int)e;
}
