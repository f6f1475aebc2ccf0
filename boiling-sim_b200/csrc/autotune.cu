// autotune.cu -- the library's autotuner: times the candidate tile shapes and
// pass depths of a kernel family on the caller's own problem and keeps the
// fastest (bsp_set_tuning), so later calls of the same family use it.
//
//   bsp_autotune_jacobi: sweep plane chunk (BSP_TUNE_SWEEP_BI) x sweeps per
//     HBM pass (BSP_TUNE_SWEEP_TBLOCK: one, or two temporally blocked);
//   bsp_autotune_solve: plane chunk of the solver's level-0 tiles
//     (BSP_TUNE_FINE_BI) x the one-launch coarse cycle (BSP_TUNE_COARSE_FUSED).
//
// Every candidate runs the real kernels on the caller's buffers, timed with
// CUDA events on the caller's stream after one untimed run.  Results are
// bit-identical across candidates for the sweeps (the choices change only the
// decomposition); the solve's candidates all meet the caller's tolerance.
#include <cuda_runtime.h>

#include <vector>

#include "../../include/bsproj.h"

namespace bsp {
extern int g_sweep_bi, g_sweep_tblock, g_fine_bi;
extern bool g_coarse_fused_enabled;
int jacobi_solve_impl(float *p, float *p_tmp, const float *div_u, float *rhs_ws,
                      const uint8_t *mask, int nx, int ny, int nz, float dx, float dt, float rho,
                      int n_iter, int tblock, cudaStream_t stream, bool p_zero_nonfluid);
}  // namespace bsp

namespace {

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

void put(BspTuneChoice *out, int max_out, int *n, int key, int value, float ms, int status) {
  if (out && *n < max_out) out[*n] = BspTuneChoice{key, value, ms, status};
  ++*n;
}

}  // namespace

extern "C" int bsp_autotune_jacobi(float *p, float *p_tmp, const float *div_u, float *rhs_ws,
                                   const uint8_t *mask, int nx, int ny, int nz, float dx,
                                   float dt, float rho, int sweeps, BspTuneChoice *out,
                                   int max_out, int *n_out, cudaStream_t s) {
  using namespace bsp;
  if (!p || !p_tmp || !div_u || !rhs_ws || !mask || !n_out) return BSP_ERR_NULL;
  if (nx <= 0 || ny <= 0 || nz <= 0 || sweeps < 2) return BSP_ERR_ARG;
  const int bis[] = {0, 2, 4, 8, 16, 32};
  const int depths[] = {1, 2};
  const int save_bi = g_sweep_bi, save_tb = g_sweep_tblock;
  Timer t;
  float best = 1e30f;
  int best_bi = save_bi, best_tb = save_tb;
  *n_out = 0;
  const size_t bytes = sizeof(float) * (size_t)nx * ny * nz;
  for (int tb : depths)
    for (int bi : bis) {
      g_sweep_bi = bi;
      g_sweep_tblock = tb;
      int st = BSP_OK;
      float ms = 0.0f;
      for (int rep = 0; rep < 2 && st == BSP_OK; ++rep) {  // untimed, then timed
        cudaMemsetAsync(p, 0, bytes, s);
        cudaEventRecord(t.a, s);
        st = jacobi_solve_impl(p, p_tmp, div_u, rhs_ws, mask, nx, ny, nz, dx, dt, rho, sweeps,
                               0, s, true);
        cudaEventRecord(t.b, s);
      }
      if (st == BSP_OK) st = (int)cudaEventSynchronize(t.b);
      if (st == BSP_OK) cudaEventElapsedTime(&ms, t.a, t.b);
      const float per = ms / sweeps;
      put(out, max_out, n_out, BSP_TUNE_SWEEP_BI, bi | (tb << 16), per, st);
      if (st == BSP_OK && per < best) {
        best = per;
        best_bi = bi;
        best_tb = tb;
      }
    }
  g_sweep_bi = best_bi;
  g_sweep_tblock = best_tb;
  return (int)cudaGetLastError();
}

extern "C" int bsp_autotune_solve(float *p, const float *div_u, const uint8_t *mask, int nx,
                                  int ny, int nz, float dx, float dt, float rho,
                                  const BspSolveParams *params, void *workspace,
                                  size_t workspace_bytes, BspTuneChoice *out, int max_out,
                                  int *n_out, cudaStream_t s) {
  using namespace bsp;
  if (!p || !div_u || !mask || !params || !workspace || !n_out) return BSP_ERR_NULL;
  const int bis[] = {0, 4, 8, 12, 16, 24, 32};
  const bool fused[] = {true, false};
  const int save_bi = g_fine_bi;
  const bool save_fused = g_coarse_fused_enabled;
  Timer t;
  float best = 1e30f;
  int best_bi = save_bi;
  bool best_fused = save_fused;
  *n_out = 0;
  BspSolveParams prm = *params;
  prm.warm_start = 0;
  for (bool fz : fused)
    for (int bi : bis) {
      g_fine_bi = bi;
      g_coarse_fused_enabled = fz;
      BspSolveInfo info{};
      prm.reuse_setup = 0;  // the tile geometry changes with bi: build the setup
      int st = bsp_solve_tol(p, div_u, mask, nx, ny, nz, dx, dt, rho, &prm, workspace,
                             workspace_bytes, nullptr, &info, s);
      float ms = 0.0f;
      if (st == BSP_OK) {
        prm.reuse_setup = 1;
        cudaEventRecord(t.a, s);
        st = bsp_solve_tol(p, div_u, mask, nx, ny, nz, dx, dt, rho, &prm, workspace,
                           workspace_bytes, nullptr, &info, s);
        cudaEventRecord(t.b, s);
        if (st == BSP_OK) st = (int)cudaEventSynchronize(t.b);
        if (st == BSP_OK) cudaEventElapsedTime(&ms, t.a, t.b);
      }
      put(out, max_out, n_out, BSP_TUNE_FINE_BI, bi | ((fz ? 1 : 0) << 16), ms, st);
      if (st == BSP_OK && ms < best) {
        best = ms;
        best_bi = bi;
        best_fused = fz;
      }
    }
  g_fine_bi = best_bi;
  g_coarse_fused_enabled = best_fused;
  return (int)cudaGetLastError();
}
