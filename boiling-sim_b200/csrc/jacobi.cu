// jacobi.cu -- fixed-count Jacobi solve (crates/cuda-kernels/src/jacobi_pressure.cu:228-270
// on the uint8 class mask): n_iter ping-pong sweeps p -> p_tmp -> p ..., result in p.
//
// When the caller provides an rhs buffer (or the projection, which owns div_u
// for the duration of the solve), rho dx^2 div / dt is evaluated once per cell
// and every sweep reads it: the same float each sweep of the reference
// computes, so the result is bit-identical and the per-cell IEEE division
// leaves the sweep loop.
#include "bsp_common.cuh"
#include "profile.cuh"

namespace bsp {

template <int OP, class MaskT>
cudaError_t launch_stencil(float *out, const float *p, const float *div, const MaskT *mask,
                           int nx, int ny, int nz, float dx, float dt, float rho, int mf,
                           int ma, cudaStream_t s);
cudaError_t launch_rhs(float *rhs, const float *div, const uint8_t *mask, int64_t n, float dx,
                       float dt, float rho, cudaStream_t s);
cudaError_t launch_sweep_znf(float *out, const float *p, const float *rhs, const uint8_t *mask,
                             int nx, int ny, int nz, cudaStream_t s);

// p_zero_nonfluid: the caller guarantees p holds +0 on non-fluid cells (the
// projection zeroes p); every later source was written by a sweep, which
// writes +0 there, so from the second sweep on the ZNF kernel applies.
bool launch_sweep2(float *out, const float *p, const float *rhs, const uint8_t *mask, int nx,
                   int ny, int nz, cudaStream_t s);
int g_sweep_tblock = 1;  // BSP_TUNE_SWEEP_TBLOCK: sweeps per pass when a call passes 0

// n_iter sweeps p <-> p_tmp, result in p.  With tblock >= 2 (tblock 0: the
// BSP_TUNE_SWEEP_TBLOCK setting, 1 unless the autotuner chose 2), the right-hand
// side hoisted (rhs_ws) and the source zero off fluid, pairs of sweeps run as
// one temporally blocked pass (sweep2.cu); every sweep is bit-identical to
// the single-sweep kernel either way.  One sweep per pass is the default:
// the single sweep is already issue-limited (about 60 instructions per cell
// for the bit-exact select and division), so fusing two doubles the
// instruction work per byte moved and measured slower on the B200.
int jacobi_solve_impl(float *p, float *p_tmp, const float *div_u, float *rhs_ws,
                      const uint8_t *mask, int nx, int ny, int nz, float dx, float dt, float rho,
                      int n_iter, int tblock, cudaStream_t stream, bool p_zero_nonfluid) {
  if (n_iter <= 0) return BSP_OK;
  const int64_t n = (int64_t)nx * ny * nz;
  if (rhs_ws) {
    cudaError_t e = launch_rhs(rhs_ws, div_u, mask, n, dx, dt, rho, stream);
    if (e != cudaSuccess) return (int)e;
  }
  const int depth = tblock > 0 ? tblock : g_sweep_tblock;
  float *cur = p, *oth = p_tmp;
  for (int it = 0; it < n_iter;) {
    const bool znf = it > 0 || p_zero_nonfluid;
    if (rhs_ws && znf && depth >= 2 && n_iter - it >= 2) {
      bool done;
      {
        ProfScope ps(PROF_SWEEP, stream);
        done = launch_sweep2(oth, cur, rhs_ws, mask, nx, ny, nz, stream);
      }
      if (done) {
        float *t = cur;
        cur = oth;
        oth = t;
        it += 2;
        continue;
      }
    }
    ProfScope ps(PROF_SWEEP, stream);
    cudaError_t e =
        rhs_ws ? (znf ? launch_sweep_znf(oth, cur, rhs_ws, mask, nx, ny, nz, stream)
                      : launch_stencil<2, uint8_t>(oth, cur, rhs_ws, mask, nx, ny, nz, dx, dt,
                                                   rho, BSP_FLUID, BSP_AIR, stream))
               : launch_stencil<0, uint8_t>(oth, cur, div_u, mask, nx, ny, nz, dx, dt, rho,
                                            BSP_FLUID, BSP_AIR, stream);
    if (e != cudaSuccess) return (int)e;
    float *t = cur;
    cur = oth;
    oth = t;
    ++it;
  }
  if (cur != p) {
    cudaError_t e = cudaMemcpyAsync(p, cur, sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice,
                                    stream);
    if (e != cudaSuccess) return (int)e;
  }
  return BSP_OK;
}

}  // namespace bsp

extern "C" int bsp_jacobi_solve(float *p, float *p_tmp, const float *div_u, float *rhs_ws,
                                const uint8_t *mask, int nx, int ny, int nz, float dx, float dt,
                                float rho, int n_iter, int tblock, cudaStream_t stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || n_iter <= 0) return BSP_OK;
  if (!p || !p_tmp || !div_u || !mask) return BSP_ERR_NULL;
  if (p == p_tmp || rhs_ws == p || rhs_ws == p_tmp) return BSP_ERR_ALIAS;
  return bsp::jacobi_solve_impl(p, p_tmp, div_u, rhs_ws, mask, nx, ny, nz, dx, dt, rho, n_iter,
                                tblock, stream, false);
}
