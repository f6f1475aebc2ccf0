// jacobi.cu -- fixed-count Jacobi solve (crates/cuda-kernels/src/jacobi_pressure.cu:228-270
// on the uint8 class mask): n_iter ping-pong sweeps p -> p_tmp -> p ..., result in p.
#include "bsp_common.cuh"

namespace bsp {

template <int OP, class MaskT>
cudaError_t launch_stencil(float *out, const float *p, const float *div, const MaskT *mask,
                           int nx, int ny, int nz, float dx, float dt, float rho, int mf,
                           int ma, cudaStream_t s);

int jacobi_solve_impl(float *p, float *p_tmp, const float *div_u, const uint8_t *mask, int nx,
                      int ny, int nz, float dx, float dt, float rho, int n_iter, int tblock,
                      cudaStream_t stream) {
  (void)tblock;
  if (n_iter <= 0) return BSP_OK;
  for (int it = 0; it < n_iter; ++it) {
    float *dst = (it & 1) == 0 ? p_tmp : p;
    const float *src = (it & 1) == 0 ? p : p_tmp;
    cudaError_t e = launch_stencil<0, uint8_t>(dst, src, div_u, mask, nx, ny, nz, dx, dt, rho,
                                               BSP_FLUID, BSP_AIR, stream);
    if (e != cudaSuccess) return (int)e;
  }
  if (n_iter & 1) {
    cudaError_t e = cudaMemcpyAsync(p, p_tmp, sizeof(float) * (size_t)nx * ny * nz,
                                    cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) return (int)e;
  }
  return BSP_OK;
}

}  // namespace bsp

extern "C" int bsp_jacobi_solve(float *p, float *p_tmp, const float *div_u,
                                const uint8_t *mask, int nx, int ny, int nz, float dx, float dt,
                                float rho, int n_iter, int tblock, cudaStream_t stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || n_iter <= 0) return BSP_OK;
  if (!p || !p_tmp || !div_u || !mask) return BSP_ERR_NULL;
  if (p == p_tmp) return BSP_ERR_ALIAS;
  return bsp::jacobi_solve_impl(p, p_tmp, div_u, mask, nx, ny, nz, dx, dt, rho, n_iter, tblock,
                                stream);
}
