/*
 * bsproj.h -- C ABI of the B200 pressure-projection library (libbsproj.so).
 *
 * Two groups of entry points:
 *
 *  1. Drop-in replacements for the reference's native launchers
 *     (crates/cuda-kernels/src/*.cu, bound from Rust in
 *     crates/cuda-kernels/src/lib.rs:16-186 and exposed to Python by
 *     crates/sim-core/src/cuda.rs).  Same symbol names, same argument lists,
 *     same meaning: int32 material ids, legacy default stream, cudaError_t
 *     return (0 = success), sizes <= 0 are a successful no-op.
 *
 *  2. bsp_* entry points: the B200-native path.  One byte of cell class per
 *     cell (BSP_CLASS_*), an explicit cudaStream_t, caller-owned workspace
 *     (bsp_*_workspace_bytes), 64-bit sizes.  They return cudaError_t values
 *     or one of the BSP_ERR_* codes below.
 *
 * All pointers are device pointers unless the name ends in _host.  Arrays are
 * C-contiguous (i, j, k) -> (i*ny + j)*nz + k; MAC faces ux (nx+1,ny,nz),
 * uy (nx,ny+1,nz), uz (nx,ny,nz+1).  No entry point allocates device memory
 * or frees it; none synchronises the device unless its comment says so.
 */
#ifndef BSPROJ_H
#define BSPROJ_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* project status codes (disjoint from cudaError_t values) */
#define BSP_OK 0
#define BSP_ERR_SHAPE 10001        /* sizes or strides unusable */
#define BSP_ERR_NULL 10002         /* required pointer is NULL */
#define BSP_ERR_ALIAS 10003        /* p and p_tmp overlap */
#define BSP_ERR_WORKSPACE 10004    /* workspace too small or misaligned */
#define BSP_NOT_CONVERGED 10005    /* tolerance not reached within max_iter */
#define BSP_ERR_NONFINITE 10006    /* NaN/inf met in the right-hand side */
#define BSP_ERR_TIMEOUT 10007      /* device-side wait gave up */
#define BSP_ERR_ALIGN 10008        /* pointer alignment unusable */
#define BSP_ERR_ARG 10009          /* other invalid argument */

/* cell classes of the uint8 mask */
#define BSP_CLASS_FLUID 0
#define BSP_CLASS_AIR 1
#define BSP_CLASS_SOLID 2

/* ------------------------------------------------------------------ */
/* 1. reference-compatible launchers                                   */
/* ------------------------------------------------------------------ */

/* One masked Jacobi sweep p_new <- J(p_old).
 * Replaces jacobi_pressure_launch, crates/cuda-kernels/src/jacobi_pressure.cu:184-208
 * (Warp kernel python/boilingsim/fluid.py:243-276). */
cudaError_t jacobi_pressure_launch(float *p_new, const float *p_old, const float *div_u,
                                   const int *mat, int nx, int ny, int nz, float dx,
                                   float dt, float rho, int mat_fluid, int mat_air);

/* n_iter ping-pong sweeps p <-> p_tmp; result always in p; p is the initial
 * guess.  Replaces pressure_solve_launch, jacobi_pressure.cu:228-270. */
cudaError_t pressure_solve_launch(float *p, float *p_tmp, const float *div_u, const int *mat,
                                  int nx, int ny, int nz, float dx, float dt, float rho,
                                  int n_iter, int mat_fluid, int mat_air);

/* Ap = (6I - S) p.  Replaces laplacian_spmv_launch, laplacian_spmv.cu:145-163. */
cudaError_t laplacian_spmv_launch(float *Ap, const float *p, const int *mat, int nx, int ny,
                                  int nz, int mat_fluid, int mat_air);

/* z = r / (6 - n_solid).  Replaces diag_inverse_apply_launch,
 * diag_inverse_apply.cu:91-111. */
cudaError_t diag_inverse_apply_launch(float *z, const float *r, const int *mat, int nx,
                                      int ny, int nz, int mat_fluid, int mat_air);

/* result[0] = x . y, accumulated in FP64 and rounded to float; workspace
 * >= 1024 floats (4 KiB).  Replaces dot_launch, dot_reduce.cu:92-115. */
cudaError_t dot_launch(const float *x, const float *y, int n, float *workspace,
                       float *result);

/* y += (+/-alpha[0]) x.  Replaces axpy_device_launch, axpy_device.cu:33-45. */
cudaError_t axpy_device_launch(float *y, const float *x, const float *alpha_ptr, int n,
                               int negate_alpha);

/* p_out = z + beta[0] p_old.  Replaces scaled_axpy_launch, axpy_device.cu:65-77. */
cudaError_t scaled_axpy_launch(float *p_out, const float *z, const float *p_old,
                               const float *beta_ptr, int n);

/* result = num / den (0 if den == 0).  Replaces divide_scalars_launch,
 * axpy_device.cu:93-99. */
cudaError_t divide_scalars_launch(const float *num_ptr, const float *den_ptr,
                                  float *result_ptr);

/* b = scale * div on fluid cells, 0 elsewhere.  Replaces compute_b_launch,
 * axpy_device.cu:125-137. */
cudaError_t compute_b_launch(float *b, const float *div_u, const int *mat, int nx, int ny,
                             int nz, float scale, int mat_fluid);

/* buf[0:n] = 0.  Replaces zero_buffer_launch, axpy_device.cu:142-145. */
cudaError_t zero_buffer_launch(float *buf, int n);

/* In-place x *= s, synchronous.  Replaces the FFI contract probe
 * scale_inplace_launch, crates/cuda-kernels/src/scale.cu:11-34. */
cudaError_t scale_inplace_launch(float *x, int n, float s);

/* Jacobi-preconditioned CG to ||r||_2 < tol ||b||_2, cold start, result in
 * p_out, iteration count to *iter_count_host.  Same contract as
 * pressure_solve_pcg_launch, pressure_solve_pcg.cu:89-243: caller-owned
 * workspaces (5 n-float vectors, >= 1024-float dot workspace, 7 device
 * scalars); the check cadence is every 5 iterations from iteration 8.  Inner
 * products are FP64 on the device; blocks the host at the end only. */
cudaError_t pressure_solve_pcg_launch(float *p_out, const float *div_u, const int *mat,
                                      int nx, int ny, int nz, float dx, float dt, float rho,
                                      int mat_fluid, int mat_air, float pressure_tol,
                                      int max_iter, float *ws_b, float *ws_r, float *ws_z,
                                      float *ws_p_search, float *ws_Ap, float *dot_workspace,
                                      float *dev_alpha, float *dev_beta, float *dev_rzold,
                                      float *dev_rznew, float *dev_bsq, float *dev_rsq,
                                      float *dev_pAp, int *iter_count_host);

/* ------------------------------------------------------------------ */
/* 2. B200-native entry points                                         */
/* ------------------------------------------------------------------ */

/* Library build/version string (static storage). */
const char *bsp_version(void);

/* Message for a status code returned by any entry point (static storage). */
const char *bsp_error_string(int code);

/* mask[c] = class of mat[c] (BSP_CLASS_*, bits 0-1) | n_solid << 2, where
 * n_solid counts the face neighbours that are neither fluid nor air (the
 * Jacobi preconditioner diagonal is 6 - n_solid, diag_inverse_apply.cu:62-78).
 * Derived once per geometry: the reference's mat is static after
 * build_pot_geometry (python/boilingsim/geometry.py:341-541). */
int bsp_mask_from_mat(uint8_t *mask, const int32_t *mat, int nx, int ny, int nz,
                      int mat_fluid, int mat_air, cudaStream_t stream);

/* One Jacobi sweep on the uint8 mask (fluid.py:243-276).  Bit-identical to
 * the reference arithmetic. */
int bsp_jacobi_sweep(float *p_new, const float *p_old, const float *div_u,
                     const uint8_t *mask, int nx, int ny, int nz, float dx, float dt,
                     float rho, cudaStream_t stream);

/* n_iter sweeps, ping-pong p <-> p_tmp, result in p (jacobi_pressure.cu:228-270
 * on the uint8 mask).  tblock = sweeps fused per HBM pass (0 = autotuned,
 * 1 = one sweep per launch); results are bit-identical for every tblock. */
int bsp_jacobi_solve(float *p, float *p_tmp, const float *div_u, const uint8_t *mask,
                     int nx, int ny, int nz, float dx, float dt, float rho, int n_iter,
                     int tblock, cudaStream_t stream);

/* div = divergence of the MAC velocity on fluid cells, 0 elsewhere
 * (fluid.py:201-218).  If max_abs_div is non-NULL it receives max|div| as a
 * device float (it is overwritten, not accumulated). */
int bsp_divergence(float *div_u, const float *ux, const float *uy, const float *uz,
                   const uint8_t *mask, int nx, int ny, int nz, float dx,
                   float *max_abs_div, cudaStream_t stream);

/* u -= dt/rho grad p on interior faces between two fluid cells, all three
 * components in one pass (fluid.py:279-330). */
int bsp_subtract_gradient(float *ux, float *uy, float *uz, const float *p,
                          const uint8_t *mask, int nx, int ny, int nz, float dx, float dt,
                          float rho, cudaStream_t stream);

/* Zero every MAC face touching a non-fluid cell or the domain boundary
 * (fluid.py:111-165). */
int bsp_enforce_no_slip(float *ux, float *uy, float *uz, const uint8_t *mask, int nx,
                        int ny, int nz, cudaStream_t stream);

/* Whole Jacobi projection (fluid.py:612-734): zero p and p_tmp, divergence,
 * n_iter sweeps, gradient subtract, diagnostic divergence.  max|div| after
 * the projection is written to *max_div_dev (device float).  No host sync. */
int bsp_projection_jacobi(float *p, float *p_tmp, float *div_u, float *ux, float *uy,
                          float *uz, const uint8_t *mask, int nx, int ny, int nz, float dx,
                          float dt, float rho, int n_iter, int tblock, float *max_div_dev,
                          cudaStream_t stream);

/* Ap = (6I - S) p on the uint8 mask (laplacian_spmv.cu:62-143). */
int bsp_spmv(float *Ap, const float *p, const uint8_t *mask, int nx, int ny, int nz,
             cudaStream_t stream);

/* Exhaustive self-check of the device division-by-6 against IEEE division
 * over all 2^32 float bit patterns; the mismatch count is written to the
 * device counter *mismatches_dev (zeroed first). */
int bsp_selftest_div6(unsigned long long *mismatches_dev, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* BSPROJ_H */
