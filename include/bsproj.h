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
#define BSP_ERR_CAPACITY 10010     /* more distinct cell classes than a table holds */

/* uint8 cell mask: bit 7 fluid, bit 6 solid (air: neither -- a zero byte is
 * air, like a cell outside the grid), bits 0-2 number of solid face neighbours */
#define BSP_CLASS_FLUID 0x80
#define BSP_CLASS_SOLID 0x40
#define BSP_CLASS_AIR 0x00
#define BSP_MASK_NSOLID 0x07

/* autotuner keys of bsp_set_tuning */
#define BSP_TUNE_SWEEP_BI 1     /* i-planes per CTA of the sweep kernels (0 = heuristic) */
#define BSP_TUNE_FINE_COLUMN 2  /* solver level-0 kernels: 1 column layout, 0 row layout */
#define BSP_TUNE_MG_ALPHA 3     /* coarse-correction scale of the V-cycle, in 1/1000 (100..3000) */
#define BSP_TUNE_FINE_TMA 4     /* column-layout solver kernels fed by TMA tiles: 1 on, 0 off */
#define BSP_TUNE_COARSE_FUSED 5 /* coarse V-cycle levels in one cooperative kernel: 1 on, 0 off */
#define BSP_TUNE_FUSE_UPDATE 6  /* CG update fused into the next restriction (TMA path): 1 on, 0 off */
#define BSP_TUNE_FINE_BI 7      /* i-planes per CTA tile of the solver's level-0 kernels (0 = rule) */
#define BSP_TUNE_SWEEP_TBLOCK 8 /* sweeps per HBM pass when a call passes tblock = 0 (1 or 2) */
#define BSP_TUNE_COND_BI 9      /* i-planes per CTA of the conduction sweeps (0 = rule) */
#define BSP_TUNE_COND_TMA 10    /* conduction class sweep fed by TMA tiles: 1 on, 0 off */
/* Tests only: 1 makes the next host-driven bsp_solve_tol start with the
 * coarse-cycle grid barrier's error word set, as a barrier that gave up
 * leaves it (that solve returns BSP_ERR_TIMEOUT; the key clears itself). */
#define BSP_TUNE_TEST_BARRIER_ERROR 11
#define BSP_TUNE_COARSE_PHASES 12 /* coarse cycle forms t where it is read: 1 on, 0 off (default) */
#define BSP_TUNE_COARSE_TRACE 13  /* tracing: coarse-cycle launches stamp their phase boundaries */
#define BSP_TUNE_COARSE_TAIL 14   /* coarse levels of CTA 0 in shared memory: 1 on, 0 off (default) */
#define BSP_TUNE_COARSE_SPLIT 15  /* levels 1..S (S = 0..3, 3 default) on the column tile kernels,
                                     the one-launch cycle below them */
#define BSP_TUNE_CONV_EPILOGUE 16 /* tensor-core convolution: epilogue warpgroups 2..4, 1 = two CTAs
                                     per SM with one each, 0 = per layer (default) */
#define BSP_TUNE_L1_SWEEPS 17     /* with COARSE_SPLIT: smoothing sweeps a side on level 1, 1 or 2
                                     (default) */
#define BSP_TUNE_PCG_QUAD 18      /* reference-compatible PCG: four-cell form 1 (default), one-cell 0 */
#define BSP_TUNE_L0_TRILINEAR 19  /* trilinear transfers between levels 0 and 1: 1 on, 0 off */
#define BSP_TUNE_TRI_CPC 20       /* coarse planes per thread of the trilinear restriction (1..64) */
#define BSP_TUNE_FUSE_SCALARS 21  /* CG scalars in the last CTA of the level-0 kernels: 1, 0 (default) */
#define BSP_TUNE_FINE_CTAS 22     /* CTAs per SM the tile kernels' plane chunking aims for (default 4) */
#define BSP_TUNE_PDL 23           /* tile and scalar kernels of an inner iteration by programmatic
                                     dependent launch: 1 on (default), 0 off */
#define BSP_TUNE_COARSE_CLUSTER 24 /* coarse cycle in one thread-block cluster of 2..16 CTAs with
                                      hardware cluster barriers (default 16); 0: cooperative
                                      kernel over all SMs */
#define BSP_TUNE_CLUSTER_TAIL 25  /* with COARSE_CLUSTER: levels of <= 2048 cells in CTA 0's shared
                                     memory, 1 on, 0 off (default) */
#define BSP_TUNE_SWEEP_PREFETCH 26 /* plain Jacobi sweep's L2 prefetch distance in planes:
                                      0 off, 2 (default) or 3 */
#define BSP_TUNE_CLUSTER_TAIL_CELLS 27 /* cluster coarse cycle: levels of at most this many cells
                                          run in its CTA 0 alone (default 16384) */
#define BSP_TUNE_DOWNU_BLOCKS 28  /* CTAs per SM of the fused CG update + restriction: 3 (default)
                                     or 4 (48 registers a thread) */

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

/* mask[c] = class of mat[c] (BSP_CLASS_*) | n_solid, where
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
 * on the uint8 mask).  If rhs_ws (n floats, 16-byte aligned) is given, the
 * per-cell constant rho dx^2 div / dt is evaluated into it once and the
 * sweeps read it (bit-identical results, no division per sweep); rhs_ws may
 * equal div_u, which then holds that constant afterwards.  tblock: sweeps
 * per HBM pass -- 0 or 1 (default) one, 2 fuses pairs of sweeps into one
 * temporally blocked pass (needs rhs_ws, nz % 16 == 0 and the source zero
 * off fluid, i.e. from the second sweep, or the first when p starts at
 * zero); the result is bit-identical either way. */
int bsp_jacobi_solve(float *p, float *p_tmp, const float *div_u, float *rhs_ws,
                     const uint8_t *mask, int nx, int ny, int nz, float dx, float dt, float rho,
                     int n_iter, int tblock, cudaStream_t stream);

/* 1 in *flag_host if a temporally blocked sweep pass gave up a bounded
 * device-side wait since the last call (its output is then invalid); clears
 * the flag.  Synchronises the device.  No reference counterpart. */
int bsp_sweep2_error(int *flag_host);

/* Set an autotuner parameter (BSP_TUNE_*) for subsequent launches in this
 * process.  Not thread-safe against concurrent launches. */
int bsp_set_tuning(int key, int value);

/* Per-kernel-class event timing (tracing).  While enabled, every launch of an
 * instrumented kernel is bracketed by CUDA events on its stream.  Classes:
 * 0 sweep, 1 restriction from the fine level, 2 prolongation onto the fine
 * level, 3 search direction + A ps, 4 CG vector update, 5 FP64 residual,
 * 6 FP64 iterate update, 7 coarse multigrid levels, 8 control / setup
 * kernels, 9 divergence / gradient / no-slip / rhs, 10 learned warm start
 * (network layers on the tensor cores, input packing, head).
 * bsp_profile_read waits for the recorded launches, writes the summed
 * milliseconds and launch counts of classes 0..nclass-1 and clears the
 * record. */
#define BSP_PROF_NCLASS 12
/* Tracing of the one-launch coarse V-cycle (with BSP_TUNE_COARSE_TRACE = 1):
 * host[0 .. n) receives CTA 0's %globaltimer (ns) at each phase boundary of
 * the last cycle launched (0 in unused slots, at most 48), and the record is
 * cleared.  Synchronous. */
int bsp_coarse_trace_read(unsigned long long *host, int n);
int bsp_profile_enable(int on);
int bsp_profile_read(double *ms, long long *launches, int nclass);

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

/* enforce_no_slip then compute_divergence (fluid.py:111-165, 201-218) in one
 * pass: zeroes every face that touches a non-fluid cell or the domain
 * boundary and writes the divergence of the result.  Bit-identical to the
 * two calls in sequence. */
int bsp_noslip_divergence(float *div_u, float *ux, float *uy, float *uz, const uint8_t *mask,
                          int nx, int ny, int nz, float dx, cudaStream_t stream);

/* The projection part of a time step, pipeline.py:605-619: no-slip,
 * bsp_projection_jacobi, no-slip.  The first no-slip is fused into the
 * divergence; the second is a no-op (the gradient subtract writes only faces
 * between two fluid cells) and is not launched.  Same arguments and results
 * as the three reference calls in sequence. */
int bsp_step_projection_jacobi(float *p, float *p_tmp, float *div_u, float *ux, float *uy,
                               float *uz, const uint8_t *mask, int nx, int ny, int nz,
                               float dx, float dt, float rho, int n_iter, int tblock,
                               float *max_div_dev, cudaStream_t stream);

/* Ap = (6I - S) p on the uint8 mask (laplacian_spmv.cu:62-143). */
int bsp_spmv(float *Ap, const float *p, const uint8_t *mask, int nx, int ny, int nz,
             cudaStream_t stream);

/* ---- to-tolerance solve ------------------------------------------------
 * Solves A p = b (the system of pressure_solve_pcg.cu:129-139) to
 * ||b - A p||_2 <= tol ||b||_2 with the residual evaluated in FP64 from an
 * FP64 iterate: FP64 iterative refinement around a conjugate gradient
 * preconditioned by a geometric multigrid V-cycle (Jacobi smoothing), inner
 * vectors stored in FP32, FP16 or BF16, inner products in FP64.  Replaces the
 * to-tolerance role of pressure_solve_pcg_launch (pressure_solve_pcg.cu:89-243,
 * tolerance semantics python/boilingsim/config.py:166-176). */
#define BSP_STORE_FP32 0
#define BSP_STORE_FP16 1
#define BSP_STORE_BF16 2

typedef struct BspSolveParams {
  double tol;       /* relative residual target (FP64 residual) */
  double inner_tol; /* inner CG stops at ||r_inner|| <= inner_tol ||rhat|| */
  int max_outer;    /* refinement passes */
  int max_inner;    /* CG iterations per pass */
  int storage;      /* BSP_STORE_* for the inner vectors and multigrid levels */
  int warm_start;   /* 1: p holds the initial guess on entry; 0: cold start */
  int check_every;  /* inner iterations enqueued between host reads of the done flag */
  int reuse_setup;  /* 1: the mask is unchanged since the last solve on this workspace,
                       reuse its multigrid setup (coarse masks, coarsest inverse) */
  int use_graph;    /* 1: run the whole solve as one CUDA graph (conditional WHILE
                       nodes, no host synchronisation; built once per pointer set) */
} BspSolveParams;

/* One instance of a batched solve. */
typedef struct BspBatchItem {
  float *p;              /* out: pressure (in, when warm_start) */
  const float *div;      /* divergence */
  const uint8_t *mask;   /* uint8 cell mask of this instance */
  int nx, ny, nz;
  float dx, dt, rho;
  void *workspace;       /* bsp_solver_workspace_bytes(nx, ny, nz, storage) bytes */
  size_t workspace_bytes;
} BspBatchItem;

typedef struct BspSolveInfo {
  int outer_iterations;
  int inner_iterations;
  int levels;
  int pad;
  double rel_residual; /* FP64 ||b - A x|| / ||b|| of the FP64 iterate */
} BspSolveInfo;

void bsp_solve_params_default(BspSolveParams *params);

/* Bytes of caller-owned workspace the solve needs (256-byte aligned). */
size_t bsp_solver_workspace_bytes(int nx, int ny, int nz, int storage);

/* p (float, out; in when warm_start) receives the FP64 iterate rounded to
 * float (0 on non-fluid cells); x64_out (optional, device doubles) receives
 * the FP64 iterate itself.  Returns BSP_OK, BSP_NOT_CONVERGED, or an error.
 * Synchronises the stream once per refinement pass and once per
 * check_every inner iterations (4-byte flag reads). */
int bsp_solve_tol(float *p, const float *div_u, const uint8_t *mask, int nx, int ny, int nz,
                  float dx, float dt, float rho, const BspSolveParams *params, void *workspace,
                  size_t workspace_bytes, double *x64_out, BspSolveInfo *info,
                  cudaStream_t stream);

/* *result_dev = x . y accumulated in FP64 (fixed reduction order), for
 * callers that cannot allocate device memory.  No counterpart in the
 * reference: it is dot_launch without the workspace argument, for hosts that
 * reach this library through its C ABI holding only their own arrays, or
 * that step under a device-memory budget fixed at start-up and may not call
 * cudaMalloc.  Its partial sums live in a file-scope __device__ array of 1024
 * doubles (8 KiB per GPU, kept until exit); n may be at most 67,108,864
 * (1024 partials x 65,536 elements), larger n returns BSP_ERR_SHAPE.  All
 * calls share that array: calls that overlap on the GPU race and must be
 * serialised.  Every call made outside a stream capture looks up the
 * array's device address (cudaGetSymbolAddress) and keeps it per device for
 * calls made inside one; the first call on a device, and the first after a
 * cudaDeviceReset (which reloads the module), should therefore come outside
 * any stream capture (a first call inside one returns BSP_ERR_ARG).
 * Allocates nothing; never calls cudaMalloc or cudaFree. */
#define BSP_DOT_NOALLOC_MAX_N 67108864LL
int bsp_dot_noalloc(const float *x, const float *y, int64_t n, double *result_dev,
                    cudaStream_t stream);

/* Solves `count` independent systems (uneven sizes allowed, one workspace
 * each) with one CUDA graph launch: every instance is an independent branch
 * of the graph running its own refinement and CG loops as conditional WHILE
 * nodes, so small instances overlap on the GPU.  The graph is built on the
 * first call for a given item set and replayed afterwards.  If infos is
 * non-NULL the call waits for the batch and fills one BspSolveInfo per item
 * (returning the first non-OK status); otherwise it returns after the
 * launch.  Batched pot scenes of the benchmark configuration (64 instances). */
int bsp_solve_batch(int count, const BspBatchItem *items, const BspSolveParams *params,
                    BspSolveInfo *infos, cudaStream_t stream);

/* ---- autotuner ------------------------------------------------------------
 * Time the candidate decompositions of a kernel family on the caller's own
 * problem (CUDA events on `stream`, one untimed run first) and keep the
 * fastest through bsp_set_tuning.  out[0 .. min(*n_out, max_out)) receives
 * one row per candidate: key, value (low 16 bits: the plane chunk, 0 = rule;
 * bit 16: the second switch), milliseconds (per sweep / per solve) and the
 * candidate's status.  The buffers are overwritten.  No reference
 * counterpart (the reference has no tuning step). */
typedef struct BspTuneChoice {
  int key, value;
  float ms;
  int status;
} BspTuneChoice;

/* Sweep plane chunk x sweeps per HBM pass (one, or two temporally blocked);
 * `sweeps` sweeps per candidate on p / p_tmp / rhs_ws (p is zeroed first). */
int bsp_autotune_jacobi(float *p, float *p_tmp, const float *div_u, float *rhs_ws,
                        const uint8_t *mask, int nx, int ny, int nz, float dx, float dt,
                        float rho, int sweeps, BspTuneChoice *out, int max_out, int *n_out,
                        cudaStream_t stream);

/* Plane chunk of the to-tolerance solver's level-0 tiles x the one-launch
 * coarse cycle, each candidate a full bsp_solve_tol with `params`. */
int bsp_autotune_solve(float *p, const float *div_u, const uint8_t *mask, int nx, int ny,
                       int nz, float dx, float dt, float rho, const struct BspSolveParams *params,
                       void *workspace, size_t workspace_bytes, BspTuneChoice *out, int max_out,
                       int *n_out, cudaStream_t stream);

/* ---- semi-Lagrangian advection --------------------------------------------------
 * python/boilingsim/fluid.py:39-104, 338-498, 737-776 on the uint8 cell mask
 * (bsp_mask_from_mat).  Bit-identical to the reference expressions evaluated
 * one rounding per operation.  (ox, oy, oz) is the grid origin (world
 * position of cell (0,0,0)'s corner), dx the cell size. */

/* extend_temperature_into_solids: T_ext = T on fluid cells; elsewhere the T
 * of the first fluid face neighbour in the order -x, +x, -y, +y, -z, +z, else
 * the cell's own T. */
int bsp_extend_temperature(float *T_ext, const float *T, const uint8_t *mask, int nx, int ny,
                           int nz, cudaStream_t stream);
/* advect_temperature: fluid cells sample T_ext (trilinear) at the point
 * backtraced by the velocity at the cell centre; other cells copy T_true. */
int bsp_advect_temperature(float *T_new, const float *T_true, const float *T_ext,
                           const float *ux, const float *uy, const float *uz, const uint8_t *mask,
                           int nx, int ny, int nz, float ox, float oy, float oz, float dx,
                           float dt, cudaStream_t stream);
/* advect_ux / advect_uy / advect_uz (axis 0 / 1 / 2) into u_new: boundary
 * faces 0, faces between two non-fluid cells keep their value, others sample
 * their component at the backtraced face centre. */
int bsp_advect_velocity(int axis, float *u_new, const float *ux, const float *uy,
                        const float *uz, const uint8_t *mask, int nx, int ny, int nz, float ox,
                        float oy, float oz, float dx, float dt, cudaStream_t stream);
/* advect_all: the three velocity components and T from the old fields into
 * the tmp arrays (T via T_ext); copy_back != 0 then copies them into ux, uy,
 * uz, T as the reference does (0 leaves the results in the tmp arrays). */
int bsp_advect_all(float *ux, float *uy, float *uz, float *T, float *ux_tmp, float *uy_tmp,
                   float *uz_tmp, float *T_tmp, float *T_ext, const uint8_t *mask, int nx,
                   int ny, int nz, float ox, float oy, float oz, float dx, float dt,
                   int copy_back, cudaStream_t stream);

/* ---- backward-Euler conduction -------------------------------------------------
 * The implicit conduction step of python/boilingsim/thermal.py.  mat holds
 * material ids in [0, n_mat) (n_mat <= 8), indexing the device arrays k, rho,
 * cp (W/(m K), kg/m^3, J/(kg K)); mat_air is the air id.  T in kelvin.
 *
 * One Jacobi sweep, apply_implicit_conduction_update (thermal.py:259-388):
 *   T_dst = (T_old + sum gamma T_nbr) / (1 + sum gamma)
 * on every non-air cell (faces -x, +x, -y, +y, -z, +z; domain-edge faces
 * skipped; an air neighbour contributes gamma * T_amb with Newton cooling
 * gamma = dt h_conv_air / (rho cp dx); otherwise the harmonic-mean face
 * conductivity).  Air cells of T_dst are not written.  Bit-identical to the
 * reference arithmetic.  T_dst must not alias T_iter. */
int bsp_conduction_sweep(float *T_dst, const float *T_iter, const float *T_old,
                         const int32_t *mat, int nx, int ny, int nz, const float *k,
                         const float *rho, const float *cp, int n_mat, float dx, float dt,
                         float h_conv_air, float T_amb, int mat_air, cudaStream_t stream);
/* The same on uint8 material ids (bsp_material_ids): 13 B/cell per sweep. */
int bsp_conduction_sweep_u8(float *T_dst, const float *T_iter, const float *T_old,
                            const uint8_t *mat_id, int nx, int ny, int nz, const float *k,
                            const float *rho, const float *cp, int n_mat, float dx, float dt,
                            float h_conv_air, float T_amb, int mat_air, cudaStream_t stream);
/* The backward-Euler branch of conduct_one_step (thermal.py:647-658):
 * T_old <- T; n_iter sweeps ping-ponging T -> T_alt -> T ...; when n_iter is
 * odd, T <- T_alt (every cell).  The snapshot is written by the first sweep. */
int bsp_conduction_be(float *T, float *T_alt, float *T_old, const int32_t *mat, int nx, int ny,
                      int nz, const float *k, const float *rho, const float *cp, int n_mat,
                      float dx, float dt, float h_conv_air, float T_amb, int mat_air,
                      int n_iter, cudaStream_t stream);
int bsp_conduction_be_u8(float *T, float *T_alt, float *T_old, const uint8_t *mat_id, int nx,
                         int ny, int nz, const float *k, const float *rho, const float *cp,
                         int n_mat, float dx, float dt, float h_conv_air, float T_amb,
                         int mat_air, int n_iter, cudaStream_t stream);
/* uint8 material ids from the int32 material grid (geometry.py:359); ids
 * outside [0, n_mat) are counted into *bad_count_dev (may be NULL). */
int bsp_material_ids(uint8_t *mat_id, const int32_t *mat, int64_t n, int n_mat,
                     int *bad_count_dev, cudaStream_t stream);

/* Cell classes for the conduction sweep.  A non-air cell's update depends
 * only on its material and its six neighbours' (domain edge included), so the
 * distinct neighbourhoods of a geometry are numbered once: cls[c] = class of
 * cell c (1 .. n_classes-1; 0x80 = air), patterns[1 .. n_classes) = each
 * class's neighbourhood key (own id | code(-x) << 3 | code(+x) << 6 | ... |
 * code(+z) << 18, code 7 = domain edge).  Requires n_mat <= 7.  Synchronises
 * the stream once (reads the class count into *n_classes_host); returns
 * BSP_ERR_CAPACITY when the geometry has more than 127 classes (use the
 * material-id entry points then) and BSP_ERR_ARG when mat holds an id
 * outside [0, n_mat).  patterns holds 256 entries. */
size_t bsp_conduction_prepare_workspace_bytes(void);
int bsp_conduction_prepare(uint8_t *cls, uint32_t *patterns, int *n_classes_host,
                           const int32_t *mat, int nx, int ny, int nz, int n_mat, int mat_air,
                           void *workspace, size_t workspace_bytes, cudaStream_t stream);
/* Tile occupancy of a class grid for the TMA-fed sweep: one byte per plane
 * and 8-row x 128-cell tile (nx x ceil(ny/8) x ceil(nz/128)), 1 when the
 * tile holds a non-air cell; the sweep then skips loads no update reads.
 * Needs nz % 4 == 0. */
size_t bsp_conduction_tile_flags_bytes(int nx, int ny, int nz);
int bsp_conduction_tile_flags(uint8_t *tiles, const uint8_t *cls, int nx, int ny, int nz,
                              cudaStream_t stream);
/* The sweep and the step of bsp_conduction_sweep / bsp_conduction_be on cell
 * classes: the same results bit for bit, one class byte per cell.  tiles
 * (from bsp_conduction_tile_flags, or NULL) lets the TMA-fed sweep skip the
 * temperature tiles of all-air regions. */
int bsp_conduction_sweep_cls(float *T_dst, const float *T_iter, const float *T_old,
                             const uint8_t *cls, const uint32_t *patterns, int n_classes,
                             const uint8_t *tiles, int nx, int ny, int nz, const float *k,
                             const float *rho, const float *cp, int n_mat, float dx, float dt,
                             float h_conv_air, float T_amb, int mat_air, cudaStream_t stream);
/* Read and clear the device flag that a TMA-fed conduction sweep sets when a
 * bounded wait gave up (its results are then not valid); synchronous. */
int bsp_conduction_error(int *flag_host);
int bsp_conduction_be_cls(float *T, float *T_alt, float *T_old, const uint8_t *cls,
                          const uint32_t *patterns, int n_classes, const uint8_t *tiles, int nx,
                          int ny, int nz, const float *k, const float *rho, const float *cp,
                          int n_mat, float dx, float dt, float h_conv_air, float T_amb,
                          int mat_air, int n_iter, cudaStream_t stream);

/* ---- learned warm start: U-Net layers --------------------------------------
 * Building blocks of the pressure warm-start network (a 3-level 3-D U-Net
 * over channels-last BF16 activations [nx][ny][nz][c]).  bsp_bf16_t is the
 * bfloat16 bit pattern.  No reference counterpart: the reference's warm
 * start is the previous step's pressure (python/boilingsim/fluid.py). */
typedef uint16_t bsp_bf16_t;

/* 3x3x3 same-padded convolution, implicit GEMM on the BF16 tensor cores with
 * FP32 accumulation: out[v][co] = relu?(bias[co] + sum w[tap][ci][co] *
 * in[v+tap][ci]).  cin, cout multiples of 16; in, w 16-byte aligned. */
int bsp_unet_conv3_fwd(bsp_bf16_t *out, const bsp_bf16_t *in, const bsp_bf16_t *w,
                       const float *bias, int nx, int ny, int nz, int cin, int cout, int relu,
                       cudaStream_t stream);
/* Workspace for bsp_unet_conv3_wgrad (per-chunk partial weight gradients). */
size_t bsp_unet_wgrad_workspace_bytes(int nx, int ny, int nz, int cin, int cout);
/* Weight (FP32 [27][cin][cout]) and optional bias gradient of conv3 from the
 * output gradient g and the layer input; deterministic chunk order. */
int bsp_unet_conv3_wgrad(float *dw, float *db, const bsp_bf16_t *g, const bsp_bf16_t *in,
                         int nx, int ny, int nz, int cin, int cout, float *workspace,
                         size_t workspace_bytes, cudaStream_t stream);
/* wt[26-tap][co][ci] = w[tap][ci][co]: the input-gradient convolution's weights. */
int bsp_unet_flip_weights(bsp_bf16_t *wt, const bsp_bf16_t *w, int cin, int cout,
                          cudaStream_t stream);
/* g *= (act > 0) elementwise. */
int bsp_unet_relu_bwd(bsp_bf16_t *g, const bsp_bf16_t *act, int64_t n, cudaStream_t stream);
/* 2x2x2 average pool of the fine grid (nx, ny, nz even), or its adjoint
 * (backward != 0; accumulate adds into out). */
int bsp_unet_pool(bsp_bf16_t *out, const bsp_bf16_t *in, int nx, int ny, int nz, int c,
                  int backward, int accumulate, cudaStream_t stream);
/* Nearest 2x upsampling onto the fine grid (nx, ny, nz even), or its adjoint. */
int bsp_unet_up(bsp_bf16_t *out, const bsp_bf16_t *in, int nx, int ny, int nz, int c,
                int backward, cudaStream_t stream);
/* a += b elementwise (skip connections). */
int bsp_unet_add(bsp_bf16_t *a, const bsp_bf16_t *b, int64_t n, cudaStream_t stream);
/* Network input channels from the scaled divergence and the cell mask. */
int bsp_unet_pack_input(bsp_bf16_t *x, const float *div, const uint8_t *mask, int64_t nvox,
                        float inv_scale, cudaStream_t stream);
/* 1x1 output head: p = scale * (hb + hw . x) on fluid cells, 0 elsewhere. */
int bsp_unet_head_fwd(float *p, const bsp_bf16_t *x, const float *hw, const float *hb,
                      const uint8_t *mask, int64_t nvox, float scale, cudaStream_t stream);
/* Scaled L2 loss of pred against target with its head-input gradient gx and
 * per-block partial sums (loss, head weights, bias) in partials. */
int bsp_unet_head_loss(bsp_bf16_t *gx, float *partials, int nblocks, const float *pred,
                       const float *target, const bsp_bf16_t *x, const float *hw,
                       const uint8_t *mask, int64_t nvox, float inv_scale, float inv_nfl,
                       cudaStream_t stream);
/* Head backward from a given output gradient gy (energy / residual losses). */
int bsp_unet_head_bwd(bsp_bf16_t *gx, float *partials, int nblocks, const float *gy,
                      const bsp_bf16_t *x, const float *hw, const uint8_t *mask, int64_t nvox,
                      cudaStream_t stream);
/* out[slot] = sum over blocks of partials[slot][block], in block order. */
int bsp_unet_sum_partials(float *out, const float *partials, int nblocks, int nslots,
                          cudaStream_t stream);
/* One Adam step on FP32 master weights w with BF16 copy wb. */
int bsp_unet_adam(float *w, bsp_bf16_t *wb, float *m, float *v, const float *g, int64_t n,
                  float lr, float b1, float b2, float eps, int step, cudaStream_t stream);

/* Self-check of the bounded device waits: one grid barrier that a block never
 * reaches (grid_sync.cuh) and one mbarrier wait that nothing completes
 * (tma.cuh), each given up after its poll bound (about a second).
 * codes_dev[0] and codes_dev[1] (device ints) receive BSP_ERR_TIMEOUT when
 * the wait gave up as designed; scratch_dev is >= 64 bytes of device memory
 * for the barrier's control words (zeroed here).  The context stays usable.
 * No reference counterpart (the reference has no bounded waits). */
int bsp_selftest_waits(int *codes_dev, void *scratch_dev, cudaStream_t stream);

/* ---- learned warm start: inference on the fifth-generation tensor cores -----
 * The same network run by tcgen05.mma kernels (accumulators in tensor memory,
 * operands staged by TMA) on a padded layout: a level of interior size
 * (nx, ny, nz) is stored as bsp_unet_tc_rows(nx, ny, nz) rows x c channels
 * (BF16), row ((i+1)(ny+2) + (j+1))(nz+2) + (k+1) for cell (i, j, k), with a
 * one-cell halo of zeros that supplies the convolutions' zero padding.
 * Buffers must start zero-filled (the first and last halo planes are never
 * written) and 16-byte aligned.  No reference counterpart. */
int64_t bsp_unet_tc_rows(int nx, int ny, int nz);
/* Weight image of one layer for bsp_unet_tc_conv3 from w[27][cout][cin]
 * (the layout of bsp_unet_conv3_fwd); 27 cin cout BF16, rebuilt whenever the
 * weights change. */
int bsp_unet_tc_weights(bsp_bf16_t *wimg, const bsp_bf16_t *w, int cin, int cout,
                        cudaStream_t stream);
/* 3x3x3 convolution on padded rows: out = relu?(conv(in) + bias), then + skip
 * (rounded to BF16 before the add, as bsp_unet_add after the layer) when
 * skip != NULL; halo rows of out get zeros.  cin, cout multiples of 16
 * (cout > 64 in tiles of 64); bias 16-byte aligned; at most 2^30 padded
 * rows.  Persistent kernel, one CTA per SM. */
int bsp_unet_tc_conv3(bsp_bf16_t *out, const bsp_bf16_t *in, const bsp_bf16_t *wimg,
                      const float *bias, const bsp_bf16_t *skip, int nx, int ny, int nz,
                      int cin, int cout, int relu, cudaStream_t stream);
/* Reads and clears the flag a tensor-core convolution sets when a bounded
 * wait gave up (its output is then not valid); synchronous. */
int bsp_unet_tc_error(int *flag_host);
/* Cycle accounting of bsp_unet_tc_conv3, summed over CTAs since the last
 * call: [0] producer waiting for a free stage, [1] MMA issuer waiting for a
 * full stage, [2] MMA issuer waiting for a free accumulator, [3] epilogue
 * waiting for a complete accumulator, [4] epilogue busy, [5] CTA lifetime,
 * [6] work items, [7] MMA issuer busy.  Copies the counters into
 * counters_host[8] (when not NULL), clears them and switches the accounting
 * on (enable != 0) or off for later launches; synchronous. */
int bsp_unet_tc_trace(unsigned long long *counters_host, int enable);
/* The network's input scale on the device: *s_dev = RMS of div over the fluid
 * cells (1 if there are none or it is 0), FP64 sums in a fixed order, in a
 * caller workspace of bsp_unet_scale_workspace_bytes(). */
size_t bsp_unet_scale_workspace_bytes(void);
int bsp_unet_input_scale(float *s_dev, const float *div, const uint8_t *mask, int nx, int ny,
                         int nz, void *workspace, size_t workspace_bytes, cudaStream_t stream);
/* bsp_unet_pack_input, bsp_unet_pool (forward), bsp_unet_up (forward) and
 * bsp_unet_head_fwd on the padded layout (every output row written, halo rows
 * as zeros; the head writes the unpadded FP32 pressure).  The input is
 * div / s_dev[0]; the head's output scale is factor * s_dev[0]. */
int bsp_unet_tc_pack(bsp_bf16_t *x, const float *div, const uint8_t *mask, int nx, int ny,
                     int nz, const float *s_dev, cudaStream_t stream);
int bsp_unet_tc_pool(bsp_bf16_t *out, const bsp_bf16_t *in, int nx, int ny, int nz, int c,
                     cudaStream_t stream);
int bsp_unet_tc_up(bsp_bf16_t *out, const bsp_bf16_t *in, int nx, int ny, int nz, int c,
                   cudaStream_t stream);
int bsp_unet_tc_head(float *p, const bsp_bf16_t *x, const float *hw, const float *hb,
                     const uint8_t *mask, int nx, int ny, int nz, const float *s_dev,
                     float factor, cudaStream_t stream);

/* The network run on the grid coarsened 2x: divc (nx/2, ny/2, nz/2) = mean
 * divergence over the fluid children of each coarse fluid cell (maskc: the
 * coarse cell classes), 0 elsewhere; and the coarse pressure pc brought back
 * onto the fine fluid cells by trilinear interpolation (cell centres, edge
 * values held), 0 elsewhere.  nx, ny, nz even. */
int bsp_unet_restrict_div(float *divc, const uint8_t *maskc, const float *div,
                          const uint8_t *mask, int nx, int ny, int nz, cudaStream_t stream);
int bsp_unet_prolong(float *p, const float *pc, const uint8_t *mask, int nx, int ny, int nz,
                     cudaStream_t stream);

/* Energy-optimal scale of a starting pressure p (in place): with b = factor
 * div on fluid cells (factor = -rho dx^2 / dt) and Ap = A p (bsp_spmv),
 * p *= gamma = (b . p) / (p . A p), which minimises the A-norm error of
 * gamma p, so the scaled guess is never worse than starting from zero (gamma
 * = 0 when p . A p <= 0).  FP64 sums in a fixed order in a workspace of
 * bsp_unet_scale_workspace_bytes(); gamma_dev (optional) receives gamma. */
int bsp_unet_energy_scale(float *p, const float *Ap, const float *div, const uint8_t *mask,
                          int nx, int ny, int nz, float factor, void *workspace,
                          size_t workspace_bytes, float *gamma_dev, cudaStream_t stream);
/* bsp_unet_energy_scale with a keep rule: the scaled guess is kept only when
 * its relative residual ||b - gamma A p|| / ||b|| (from the same FP64 sums)
 * is below keep_below, else p is zeroed (gamma = 0) and the solve starts from
 * zero; keep_below <= 0 always keeps it.  relres_dev (optional) receives that
 * residual.  Device-side, no host synchronisation. */
int bsp_unet_energy_scale_keep(float *p, const float *Ap, const float *div, const uint8_t *mask,
                               int nx, int ny, int nz, float factor, float keep_below,
                               void *workspace, size_t workspace_bytes, float *gamma_dev,
                               float *relres_dev, cudaStream_t stream);

/* Exhaustive self-check of the device division-by-6 against IEEE division
 * over all 2^32 float bit patterns; the mismatch count is written to the
 * device counter *mismatches_dev (zeroed first). */
int bsp_selftest_div6(unsigned long long *mismatches_dev, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* BSPROJ_H */
