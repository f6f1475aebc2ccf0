/*
 * proj_oracle.c -- CPU ORACLE for the pressure-projection path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA library is
 * compared against (tests/, the smoke check, and the cpu_baseline leg of the
 * benchmark).  It is never linked into, called by, or used as a fallback for
 * the product library.
 *
 * It restates, in plain C, the arithmetic of the reference boiling-sim
 * projection path:
 *
 *   compute_divergence          python/boilingsim/fluid.py:201-218
 *   _pressure_neighbour         python/boilingsim/fluid.py:222-240
 *   jacobi_pressure_step        python/boilingsim/fluid.py:243-276
 *                               (+ out-of-range neighbour = air,
 *                                crates/cuda-kernels/src/jacobi_pressure.cu:121-124)
 *   pressure_solve_launch       crates/cuda-kernels/src/jacobi_pressure.cu:228-270
 *   subtract_pressure_gradient_{x,y,z}  python/boilingsim/fluid.py:279-330
 *   pressure_projection         python/boilingsim/fluid.py:612-734
 *   enforce_no_slip_{ux,uy,uz}  python/boilingsim/fluid.py:111-165
 *   laplacian_spmv_kernel       crates/cuda-kernels/src/laplacian_spmv.cu:62-143
 *   diag_inverse_apply_kernel   crates/cuda-kernels/src/diag_inverse_apply.cu:44-89
 *   compute_b_kernel            crates/cuda-kernels/src/axpy_device.cu:105-123
 *   pressure_solve_pcg_launch   crates/cuda-kernels/src/pressure_solve_pcg.cu:89-243
 *   apply_implicit_conduction_update  python/boilingsim/thermal.py:259-388
 *   conduct_one_step (backward-Euler branch)  python/boilingsim/thermal.py:647-658
 *   _tri_sample, _sample_velocity_at  python/boilingsim/fluid.py:39-104
 *   extend_temperature_into_solids, advect_temperature, advect_u{x,y,z}
 *                               python/boilingsim/fluid.py:338-498
 *   advect_all                  python/boilingsim/fluid.py:737-776
 *
 * Bit-faithfulness rules (FP32 part): every value is a C float, dx/dt/rho are
 * float before any arithmetic (Warp `float` is f32), operations are evaluated
 * left to right exactly as written in the reference, and the file is compiled
 * with -ffp-contract=off so no multiply-add is fused unless written as fmaf().
 *
 * The FP64 part (apply_A_f64 / rhs_f64 / cg_f64 / rel_residual_f64) states the
 * same linear system A p = b in double precision:
 *   (A p)_c = 6 p_c - sum_n g(n),  g = p_n (fluid) | 0 (air) | p_c (solid)
 *   b_c     = -rho dx^2 div_c / dt            (pressure_solve_pcg.cu:129-139)
 * and solves it with diagonal-preconditioned CG to give the "FP64 oracle" p*.
 *
 * The backward-Euler conduction part (or_conduction_*) is parity unpinned
 * against reference outputs: the reference kernel exists only as Warp code,
 * which cannot run here, and its tests hold no vectors for it.  It restates
 * the kernel operation by operation and is checked against closed-form
 * answers of the discrete system (tests/test_conduction_oracle.py).
 * The advection part (or_*advect*, or_extend_temperature_f32) is likewise
 * parity unpinned against reference outputs (Warp code; the reference's
 * advection test checks a drift bound, restated in tests/test_advect_oracle.py).
 * Both follow the expressions as written, one rounding per operation, as
 * Warp's CPU build evaluates them; a GPU build that contracts multiply-adds
 * (rhs + g*T, the trilinear blends) can differ in the last bit.
 *
 * OpenMP parallelises the element-wise loops; reductions use a fixed
 * per-block partial-sum layout so results do not depend on the thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define IDX(i, j, k) (((int64_t)(i) * ny + (j)) * nz + (k))

/* ------------------------------------------------------------------ */
/* utilities                                                           */
/* ------------------------------------------------------------------ */

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

static inline int mat_at(const int32_t *mat, int i, int j, int k, int nx, int ny,
                         int nz, int mat_air) {
    if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz) return mat_air;
    return mat[IDX(i, j, k)];
}

static inline float p_at(const float *p, int i, int j, int k, int nx, int ny, int nz) {
    if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz) return 0.0f;
    return p[IDX(i, j, k)];
}

/* fluid.py:222-240 */
static inline float nbr_f32(int m_nbr, float p_nbr, float p_self, int mat_fluid,
                            int mat_air) {
    if (m_nbr == mat_fluid) return p_nbr;
    if (m_nbr == mat_air) return 0.0f;
    return p_self;
}

/* ------------------------------------------------------------------ */
/* FP32 restatement                                                     */
/* ------------------------------------------------------------------ */

/* fluid.py:201-218.  Each term is divided by dx before summing. */
void or_divergence_f32(float *div, const float *ux, const float *uy, const float *uz,
                       const int32_t *mat, int nx, int ny, int nz, float dx,
                       int mat_fluid) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IDX(i, j, k);
                if (mat[c] != mat_fluid) {
                    div[c] = 0.0f;
                    continue;
                }
                /* ux: (nx+1, ny, nz); uy: (nx, ny+1, nz); uz: (nx, ny, nz+1) */
                float u1 = ux[((int64_t)(i + 1) * ny + j) * nz + k];
                float u0 = ux[((int64_t)i * ny + j) * nz + k];
                float v1 = uy[((int64_t)i * (ny + 1) + (j + 1)) * nz + k];
                float v0 = uy[((int64_t)i * (ny + 1) + j) * nz + k];
                float w1 = uz[((int64_t)i * ny + j) * (nz + 1) + (k + 1)];
                float w0 = uz[((int64_t)i * ny + j) * (nz + 1) + k];
                float dudx = (u1 - u0) / dx;
                float dvdy = (v1 - v0) / dx;
                float dwdz = (w1 - w0) / dx;
                div[c] = (dudx + dvdy) + dwdz;
            }
}

/* fluid.py:243-276 with out-of-range = air (jacobi_pressure.cu:121-124). */
void or_jacobi_step_f32(float *p_new, const float *p_old, const float *div,
                        const int32_t *mat, int nx, int ny, int nz, float dx, float dt,
                        float rho, int mat_fluid, int mat_air) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IDX(i, j, k);
                if (mat[c] != mat_fluid) {
                    p_new[c] = 0.0f;
                    continue;
                }
                float ps = p_old[c];
#define NB(di, dj, dk)                                                            \
    nbr_f32(mat_at(mat, i + (di), j + (dj), k + (dk), nx, ny, nz, mat_air),       \
            p_at(p_old, i + (di), j + (dj), k + (dk), nx, ny, nz), ps, mat_fluid, \
            mat_air)
                float pl = NB(-1, 0, 0), pr = NB(1, 0, 0);
                float pd = NB(0, -1, 0), pu = NB(0, 1, 0);
                float pb = NB(0, 0, -1), pf = NB(0, 0, 1);
#undef NB
                float s = ((((pl + pr) + pd) + pu) + pb) + pf;
                float rhs = (((rho * dx) * dx) * div[c]) / dt;
                p_new[c] = (s - rhs) / 6.0f;
            }
}

/* jacobi_pressure.cu:228-270: ping-pong p -> p_tmp -> p ..., result in p. */
void or_pressure_solve_f32(float *p, float *p_tmp, const float *div, const int32_t *mat,
                           int nx, int ny, int nz, float dx, float dt, float rho,
                           int n_iter, int mat_fluid, int mat_air) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || n_iter <= 0) return;
    for (int it = 0; it < n_iter; ++it) {
        float *dst = (it & 1) == 0 ? p_tmp : p;
        const float *src = (it & 1) == 0 ? p : p_tmp;
        or_jacobi_step_f32(dst, src, div, mat, nx, ny, nz, dx, dt, rho, mat_fluid,
                           mat_air);
    }
    if (n_iter & 1) memcpy(p, p_tmp, sizeof(float) * (size_t)nx * ny * nz);
}

/* fluid.py:279-330.  u -= ((dt/rho) * dp) / dx on interior faces whose two
 * cells are both fluid; boundary faces untouched. */
void or_subtract_gradient_f32(float *ux, float *uy, float *uz, const float *p,
                              const int32_t *mat, int nx, int ny, int nz, float dx,
                              float dt, float rho, int mat_fluid) {
    const float dtr = dt / rho;
#pragma omp parallel for schedule(static)
    for (int i = 1; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                if (mat[IDX(i - 1, j, k)] != mat_fluid || mat[IDX(i, j, k)] != mat_fluid)
                    continue;
                int64_t f = ((int64_t)i * ny + j) * nz + k;
                ux[f] = ux[f] - (dtr * (p[IDX(i, j, k)] - p[IDX(i - 1, j, k)])) / dx;
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 1; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                if (mat[IDX(i, j - 1, k)] != mat_fluid || mat[IDX(i, j, k)] != mat_fluid)
                    continue;
                int64_t f = ((int64_t)i * (ny + 1) + j) * nz + k;
                uy[f] = uy[f] - (dtr * (p[IDX(i, j, k)] - p[IDX(i, j - 1, k)])) / dx;
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 1; k < nz; ++k) {
                if (mat[IDX(i, j, k - 1)] != mat_fluid || mat[IDX(i, j, k)] != mat_fluid)
                    continue;
                int64_t f = ((int64_t)i * ny + j) * (nz + 1) + k;
                uz[f] = uz[f] - (dtr * (p[IDX(i, j, k)] - p[IDX(i, j, k - 1)])) / dx;
            }
}

/* fluid.py:111-165: zero every face that touches a non-fluid cell and the
 * domain-boundary faces. */
void or_enforce_no_slip_f32(float *ux, float *uy, float *uz, const int32_t *mat, int nx,
                            int ny, int nz, int mat_fluid) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i <= nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t f = ((int64_t)i * ny + j) * nz + k;
                if (i == 0 || i == nx || mat[IDX(i - 1, j, k)] != mat_fluid ||
                    mat[IDX(i, j, k)] != mat_fluid)
                    ux[f] = 0.0f;
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j <= ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t f = ((int64_t)i * (ny + 1) + j) * nz + k;
                if (j == 0 || j == ny || mat[IDX(i, j - 1, k)] != mat_fluid ||
                    mat[IDX(i, j, k)] != mat_fluid)
                    uy[f] = 0.0f;
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k <= nz; ++k) {
                int64_t f = ((int64_t)i * ny + j) * (nz + 1) + k;
                if (k == 0 || k == nz || mat[IDX(i, j, k - 1)] != mat_fluid ||
                    mat[IDX(i, j, k)] != mat_fluid)
                    uz[f] = 0.0f;
            }
}

/* max |div| over all cells (fluid.py:733-734 reads the full array). */
float or_max_abs_f32(const float *a, int64_t n) {
    float m = 0.0f;
#pragma omp parallel for reduction(max : m) schedule(static)
    for (int64_t c = 0; c < n; ++c) {
        float v = fabsf(a[c]);
        if (v > m) m = v;
    }
    return m;
}

/* fluid.py:612-734 for the Jacobi back-end: zero p and p_tmp, divergence,
 * n_iter sweeps (result canonicalised into p), gradient subtract, diagnostic
 * divergence; returns max|div|. */
float or_projection_jacobi_f32(float *p, float *p_tmp, float *div, float *ux, float *uy,
                               float *uz, const int32_t *mat, int nx, int ny, int nz,
                               float dx, float dt, float rho, int n_iter, int mat_fluid,
                               int mat_air) {
    int64_t n = (int64_t)nx * ny * nz;
    memset(p, 0, sizeof(float) * n);
    memset(p_tmp, 0, sizeof(float) * n);
    or_divergence_f32(div, ux, uy, uz, mat, nx, ny, nz, dx, mat_fluid);
    or_pressure_solve_f32(p, p_tmp, div, mat, nx, ny, nz, dx, dt, rho, n_iter, mat_fluid,
                          mat_air);
    or_subtract_gradient_f32(ux, uy, uz, p, mat, nx, ny, nz, dx, dt, rho, mat_fluid);
    or_divergence_f32(div, ux, uy, uz, mat, nx, ny, nz, dx, mat_fluid);
    return or_max_abs_f32(div, n);
}

/* laplacian_spmv.cu:62-143: Ap = 6 p_self - s, non-fluid -> 0.  `fused`
 * selects the contraction the reference's default nvcc build emits
 * (fma(6, p_self, -s)); fused = 0 is the --fmad=false build. */
void or_spmv_f32(float *Ap, const float *p, const int32_t *mat, int nx, int ny, int nz,
                 int mat_fluid, int mat_air, int fused) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IDX(i, j, k);
                if (mat[c] != mat_fluid) {
                    Ap[c] = 0.0f;
                    continue;
                }
                float ps = p[c];
#define NB(di, dj, dk)                                                          \
    nbr_f32(mat_at(mat, i + (di), j + (dj), k + (dk), nx, ny, nz, mat_air),     \
            p_at(p, i + (di), j + (dj), k + (dk), nx, ny, nz), ps, mat_fluid,   \
            mat_air)
                float pl = NB(-1, 0, 0), pr = NB(1, 0, 0);
                float pd = NB(0, -1, 0), pu = NB(0, 1, 0);
                float pb = NB(0, 0, -1), pf = NB(0, 0, 1);
#undef NB
                float s = ((((pl + pr) + pd) + pu) + pb) + pf;
                Ap[c] = fused ? fmaf(6.0f, ps, -s) : (6.0f * ps) - s;
            }
}

/* diag_inverse_apply.cu:44-89: z = r / (6 - n_solid); air neighbours do not
 * reduce the diagonal; diag <= 0 -> z = r. */
void or_diag_inverse_f32(float *z, const float *r, const int32_t *mat, int nx, int ny,
                         int nz, int mat_fluid, int mat_air) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IDX(i, j, k);
                if (mat[c] != mat_fluid) {
                    z[c] = 0.0f;
                    continue;
                }
                int ns = 0;
                static const int D[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0},
                                            {0, 1, 0},  {0, 0, -1}, {0, 0, 1}};
                for (int q = 0; q < 6; ++q) {
                    int m = mat_at(mat, i + D[q][0], j + D[q][1], k + D[q][2], nx, ny, nz,
                                   mat_air);
                    if (m != mat_fluid && m != mat_air) ++ns;
                }
                float diag = 6.0f - (float)ns;
                z[c] = (diag <= 0.0f) ? r[c] : r[c] / diag;
            }
}

/* axpy_device.cu:105-123: b = scale * div on fluid cells, scale computed in
 * float as ((-rho) * dx * dx) / dt (pressure_solve_pcg.cu:137). */
void or_compute_b_f32(float *b, const float *div, const int32_t *mat, int nx, int ny,
                      int nz, float dx, float dt, float rho, int mat_fluid) {
    const float scale = (((-rho) * dx) * dx) / dt;
    int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) b[c] = (mat[c] != mat_fluid) ? 0.0f : scale * div[c];
}

/* CG vector updates of axpy_device.cu, as the reference's default (FMA on)
 * build evaluates them: y = alpha x + y contracted to fmaf (axpy_device.cu:
 * 20-31; negate_alpha flips the sign of alpha first), p_out = z + beta p_old
 * contracted to fmaf(beta, p_old, z) (:51-63), num / den with den == 0 -> 0
 * (:84-91).  scale.cu:11-17 is a plain product. */
void or_axpy_f32(float *y, const float *x, float alpha, int64_t n, int negate) {
    const float a = negate ? -alpha : alpha;
    for (int64_t c = 0; c < n; ++c) y[c] = fmaf(a, x[c], y[c]);
}
void or_scaled_axpy_f32(float *out, const float *z, const float *p_old, float beta,
                        int64_t n) {
    for (int64_t c = 0; c < n; ++c) out[c] = fmaf(beta, p_old[c], z[c]);
}
float or_divide_f32(float num, float den) { return den == 0.0f ? 0.0f : num / den; }
void or_scale_f32(float *x, int64_t n, float s) {
    for (int64_t c = 0; c < n; ++c) x[c] = x[c] * s;
}

/* Deterministic FP64 dot of two float vectors: fixed 4096-element blocks,
 * block partials summed in order. */
double or_dot_f32_f64(const float *x, const float *y, int64_t n) {
    const int64_t B = 4096;
    int64_t nb = (n + B - 1) / B;
    double *part = (double *)calloc((size_t)(nb > 0 ? nb : 1), sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < nb; ++b) {
        double s = 0.0;
        int64_t e = (b + 1) * B < n ? (b + 1) * B : n;
        for (int64_t c = b * B; c < e; ++c) s += (double)x[c] * (double)y[c];
        part[b] = s;
    }
    double s = 0.0;
    for (int64_t b = 0; b < nb; ++b) s += part[b];
    free(part);
    return s;
}

/* pressure_solve_pcg.cu:89-243 restated with FP64 inner products (the product
 * library's choice; the reference reduces in FP32).  Vector arithmetic is
 * FP32 with the reference's expressions:
 *   p += alpha * ps; r -= alpha * Ap; ps = z + beta * ps  (fmaf, as nvcc's
 *   default contraction emits for y = a*x + y).
 * Convergence: rsq < tol^2 * bsq checked at iter >= 8, iter % 5 == 0.
 * Returns the iteration count.  Work vectors are allocated internally. */
int or_pcg_f32(float *p, const float *div, const int32_t *mat, int nx, int ny, int nz,
               float dx, float dt, float rho, int mat_fluid, int mat_air, float tol,
               int max_iter) {
    int64_t n = (int64_t)nx * ny * nz;
    if (n <= 0) return 0;
    float *b = (float *)malloc(sizeof(float) * n);
    float *r = (float *)malloc(sizeof(float) * n);
    float *z = (float *)malloc(sizeof(float) * n);
    float *ps = (float *)malloc(sizeof(float) * n);
    float *Ap = (float *)malloc(sizeof(float) * n);
    or_compute_b_f32(b, div, mat, nx, ny, nz, dx, dt, rho, mat_fluid);
    double bsq = or_dot_f32_f64(b, b, n);
    int iter = 0;
    memset(p, 0, sizeof(float) * n);
    if (bsq == 0.0) goto done;
    {
        double tol_sq_bsq = (double)tol * (double)tol * bsq;
        memcpy(r, b, sizeof(float) * n);
        or_diag_inverse_f32(z, r, mat, nx, ny, nz, mat_fluid, mat_air);
        memcpy(ps, z, sizeof(float) * n);
        double rz = or_dot_f32_f64(r, z, n);
        for (iter = 0; iter < max_iter; ++iter) {
            or_spmv_f32(Ap, ps, mat, nx, ny, nz, mat_fluid, mat_air, 1);
            double pAp = or_dot_f32_f64(ps, Ap, n);
            float alpha = (pAp == 0.0) ? 0.0f : (float)(rz / pAp);
#pragma omp parallel for schedule(static)
            for (int64_t c = 0; c < n; ++c) {
                p[c] = fmaf(alpha, ps[c], p[c]);
                r[c] = fmaf(-alpha, Ap[c], r[c]);
            }
            if (iter >= 8 && (iter % 5) == 0) {
                double rsq = or_dot_f32_f64(r, r, n);
                if (rsq < tol_sq_bsq) {
                    ++iter;
                    break;
                }
            }
            or_diag_inverse_f32(z, r, mat, nx, ny, nz, mat_fluid, mat_air);
            double rz_new = or_dot_f32_f64(r, z, n);
            float beta = (rz == 0.0) ? 0.0f : (float)(rz_new / rz);
#pragma omp parallel for schedule(static)
            for (int64_t c = 0; c < n; ++c) ps[c] = fmaf(beta, ps[c], z[c]);
            rz = rz_new;
        }
    }
done:
    free(b);
    free(r);
    free(z);
    free(ps);
    free(Ap);
    return iter;
}

/* ------------------------------------------------------------------ */
/* FP64 statement of the linear system                                  */
/* ------------------------------------------------------------------ */

/* (A p)_c for fluid c; 0 elsewhere.  p is double. */
void or_apply_A_f64(double *Ap, const double *p, const int32_t *mat, int nx, int ny,
                    int nz, int mat_fluid, int mat_air) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IDX(i, j, k);
                if (mat[c] != mat_fluid) {
                    Ap[c] = 0.0;
                    continue;
                }
                double ps = p[c], s = 0.0;
                static const int D[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0},
                                            {0, 1, 0},  {0, 0, -1}, {0, 0, 1}};
                for (int q = 0; q < 6; ++q) {
                    int ii = i + D[q][0], jj = j + D[q][1], kk = k + D[q][2];
                    int m = mat_at(mat, ii, jj, kk, nx, ny, nz, mat_air);
                    if (m == mat_fluid)
                        s += p[IDX(ii, jj, kk)];
                    else if (m != mat_air)
                        s += ps;
                }
                Ap[c] = 6.0 * ps - s;
            }
}

/* b_c = -rho dx^2 div_c / dt on fluid cells (double arithmetic). */
void or_rhs_f64(double *b, const float *div, const int32_t *mat, int64_t n, double dx,
                double dt, double rho, int mat_fluid) {
    double scale = -rho * dx * dx / dt;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) b[c] = (mat[c] != mat_fluid) ? 0.0 : scale * div[c];
}

static double dot_f64(const double *x, const double *y, int64_t n) {
    const int64_t B = 4096;
    int64_t nb = (n + B - 1) / B;
    double *part = (double *)calloc((size_t)(nb > 0 ? nb : 1), sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < nb; ++b) {
        double s = 0.0;
        int64_t e = (b + 1) * B < n ? (b + 1) * B : n;
        for (int64_t c = b * B; c < e; ++c) s += x[c] * y[c];
        part[b] = s;
    }
    double s = 0.0;
    for (int64_t b = 0; b < nb; ++b) s += part[b];
    free(part);
    return s;
}

/* FP64 diagonal-preconditioned CG on A p = b (b double).  Cold start.  Stops
 * at ||r||_2 <= tol ||b||_2 (true residual recomputed every 50 iterations) or
 * max_iter.  Writes the relative residual reached to *rel_out.  Returns the
 * iteration count. */
int or_cg_f64(double *p, const double *b, const int32_t *mat, int nx, int ny, int nz,
              int mat_fluid, int mat_air, double tol, int max_iter, double *rel_out) {
    int64_t n = (int64_t)nx * ny * nz;
    double *r = (double *)malloc(sizeof(double) * n);
    double *z = (double *)malloc(sizeof(double) * n);
    double *ps = (double *)malloc(sizeof(double) * n);
    double *Ap = (double *)malloc(sizeof(double) * n);
    double *dinv = (double *)malloc(sizeof(double) * n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IDX(i, j, k);
                if (mat[c] != mat_fluid) {
                    dinv[c] = 0.0;
                    continue;
                }
                int ns = 0;
                static const int D[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0},
                                            {0, 1, 0},  {0, 0, -1}, {0, 0, 1}};
                for (int q = 0; q < 6; ++q) {
                    int m = mat_at(mat, i + D[q][0], j + D[q][1], k + D[q][2], nx, ny, nz,
                                   mat_air);
                    if (m != mat_fluid && m != mat_air) ++ns;
                }
                double d = 6.0 - ns;
                dinv[c] = d > 0.0 ? 1.0 / d : 1.0;
            }
    double bnorm = sqrt(dot_f64(b, b, n));
    int it = 0;
    memset(p, 0, sizeof(double) * n);
    double rel = 0.0;
    if (bnorm == 0.0) goto out;
    memcpy(r, b, sizeof(double) * n);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) z[c] = dinv[c] * r[c];
    memcpy(ps, z, sizeof(double) * n);
    double rz = dot_f64(r, z, n);
    rel = 1.0;
    for (it = 0; it < max_iter; ++it) {
        or_apply_A_f64(Ap, ps, mat, nx, ny, nz, mat_fluid, mat_air);
        double pAp = dot_f64(ps, Ap, n);
        if (pAp <= 0.0) break;
        double alpha = rz / pAp;
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < n; ++c) {
            p[c] += alpha * ps[c];
            r[c] -= alpha * Ap[c];
        }
        if ((it + 1) % 50 == 0) {
            /* replace the recursive residual by the true one */
            or_apply_A_f64(Ap, p, mat, nx, ny, nz, mat_fluid, mat_air);
#pragma omp parallel for schedule(static)
            for (int64_t c = 0; c < n; ++c) r[c] = b[c] - Ap[c];
        }
        rel = sqrt(dot_f64(r, r, n)) / bnorm;
        if (rel <= tol) {
            ++it;
            break;
        }
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < n; ++c) z[c] = dinv[c] * r[c];
        double rz_new = dot_f64(r, z, n);
        double beta = rz_new / rz;
        rz = rz_new;
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < n; ++c) ps[c] = z[c] + beta * ps[c];
    }
    /* final true residual */
    or_apply_A_f64(Ap, p, mat, nx, ny, nz, mat_fluid, mat_air);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) r[c] = b[c] - Ap[c];
    rel = sqrt(dot_f64(r, r, n)) / bnorm;
out:
    if (rel_out) *rel_out = rel;
    free(r);
    free(z);
    free(ps);
    free(Ap);
    free(dinv);
    return it;
}

/* ||b - A p||_2 / ||b||_2 in FP64 for a float pressure p, with b built from
 * div in double (the residual definition of config.py:166-176). */
double or_rel_residual_f64(const float *p, const float *div, const int32_t *mat, int nx,
                           int ny, int nz, double dx, double dt, double rho,
                           int mat_fluid, int mat_air) {
    int64_t n = (int64_t)nx * ny * nz;
    double *pd = (double *)malloc(sizeof(double) * n);
    double *b = (double *)malloc(sizeof(double) * n);
    double *Ap = (double *)malloc(sizeof(double) * n);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) pd[c] = (mat[c] == mat_fluid) ? (double)p[c] : 0.0;
    or_rhs_f64(b, div, mat, n, dx, dt, rho, mat_fluid);
    or_apply_A_f64(Ap, pd, mat, nx, ny, nz, mat_fluid, mat_air);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) Ap[c] = b[c] - Ap[c];
    double rr = dot_f64(Ap, Ap, n), bb = dot_f64(b, b, n);
    free(pd);
    free(b);
    free(Ap);
    return bb > 0.0 ? sqrt(rr / bb) : 0.0;
}

/* ------------------------------------------------------------------ */
/* Backward-Euler conduction (FP32 restatement)                        */
/* ------------------------------------------------------------------ */

/* Face coefficient gamma of thermal.py:300-388 for a non-air cell of
 * material ms facing material mn: Newton cooling (h_conv, neighbour held at
 * T_amb) when mn is air, else the harmonic-mean conductivity
 *   k_face = ((2 ks) kn) / ((ks + kn) + 1e-12),  gamma = ((dt k_face) inv) / (dx dx)
 * with inv = 1 / (rho cp) of the cell's own material (thermal.py:290-293). */
static inline float be_gamma(int ms, int mn, const float *k, const float *rho,
                             const float *cp, float dx, float dt, float h_conv_air,
                             int mat_air) {
    const float inv = 1.0f / (rho[ms] * cp[ms]);
    if (mn == mat_air) return ((dt * h_conv_air) * inv) / dx;
    const float ks = k[ms], kn = k[mn];
    const float kf = ((2.0f * ks) * kn) / ((ks + kn) + 1.0e-12f);
    return ((dt * kf) * inv) / (dx * dx);
}

/* One Jacobi sweep of the backward-Euler conduction system,
 * apply_implicit_conduction_update (thermal.py:259-388):
 *   T_dst = (T_old + sum gamma T_nbr) / (1 + sum gamma)
 * faces visited -x, +x, -y, +y, -z, +z; a face on the domain edge is
 * skipped; an air neighbour contributes gamma * T_amb.  Air cells are not
 * written (T_dst keeps its previous contents there). */
void or_conduction_sweep_f32(float *T_dst, const float *T_iter, const float *T_old,
                             const int32_t *mat, int nx, int ny, int nz, const float *k,
                             const float *rho, const float *cp, float dx, float dt,
                             float h_conv_air, float T_amb, int mat_air) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int kk = 0; kk < nz; ++kk) {
                const int64_t c = IDX(i, j, kk);
                const int ms = mat[c];
                if (ms == mat_air) continue;
                float rhs_sum = 0.0f, diag_extra = 0.0f;
                const int di[6] = {-1, 1, 0, 0, 0, 0};
                const int dj[6] = {0, 0, -1, 1, 0, 0};
                const int dk[6] = {0, 0, 0, 0, -1, 1};
                for (int f = 0; f < 6; ++f) {
                    const int a = i + di[f], b = j + dj[f], e = kk + dk[f];
                    if (a < 0 || a >= nx || b < 0 || b >= ny || e < 0 || e >= nz) continue;
                    const int64_t n = IDX(a, b, e);
                    const int mn = mat[n];
                    const float g = be_gamma(ms, mn, k, rho, cp, dx, dt, h_conv_air, mat_air);
                    rhs_sum = rhs_sum + g * (mn == mat_air ? T_amb : T_iter[n]);
                    diag_extra = diag_extra + g;
                }
                T_dst[c] = (T_old[c] + rhs_sum) / (1.0f + diag_extra);
            }
}

/* The backward-Euler branch of conduct_one_step (thermal.py:647-658):
 * T_old <- T; n_iter sweeps ping-ponging T -> T_alt -> T ...; an odd count
 * ends with T <- T_alt (the whole array, air cells included). */
void or_conduction_be_f32(float *T, float *T_alt, float *T_old, const int32_t *mat, int nx,
                          int ny, int nz, const float *k, const float *rho, const float *cp,
                          float dx, float dt, float h_conv_air, float T_amb, int mat_air,
                          int n_iter) {
    if (nx <= 0 || ny <= 0 || nz <= 0) return;
    const size_t bytes = sizeof(float) * (size_t)nx * ny * nz;
    memcpy(T_old, T, bytes);
    for (int it = 0; it < n_iter; ++it) {
        const float *src = (it % 2 == 0) ? T : T_alt;
        float *dst = (it % 2 == 0) ? T_alt : T;
        or_conduction_sweep_f32(dst, src, T_old, mat, nx, ny, nz, k, rho, cp, dx, dt,
                                h_conv_air, T_amb, mat_air);
    }
    if (n_iter % 2 == 1) memcpy(T, T_alt, bytes);
}

/* ------------------------------------------------------------------ */
/* Semi-Lagrangian advection (FP32 restatement)                        */
/* ------------------------------------------------------------------ */

/* _tri_sample (fluid.py:39-88): trilinear sample of a field of shape
 * (fx_n, fy_n, fz_n) living on the lattice offset (ox, oy, oz) at world point
 * (px, py, pz).  Coordinates clamp to [0, n - 1 - 1e-6] in float (for n above
 * ~17 the upper bound rounds to n - 1 exactly; the +1 corner index is then
 * clamped to n - 1 here, where the reference would read past the array). */
static float tri_sample(const float *f, int fx_n, int fy_n, int fz_n, float px, float py,
                        float pz, const float *org, float dx, float ox, float oy, float oz) {
    float fx = (px - org[0]) / dx - ox;
    float fy = (py - org[1]) / dx - oy;
    float fz = (pz - org[2]) / dx - oz;
    const float hx = (float)(fx_n - 1) - 1.0e-6f, hy = (float)(fy_n - 1) - 1.0e-6f,
                hz = (float)(fz_n - 1) - 1.0e-6f;
    fx = fminf(fmaxf(fx, 0.0f), hx);
    fy = fminf(fmaxf(fy, 0.0f), hy);
    fz = fminf(fmaxf(fz, 0.0f), hz);
    const int i0 = (int)fx, j0 = (int)fy, k0 = (int)fz;
    const float tx = fx - (float)i0, ty = fy - (float)j0, tz = fz - (float)k0;
    const int i1 = i0 + 1 < fx_n ? i0 + 1 : fx_n - 1;
    const int j1 = j0 + 1 < fy_n ? j0 + 1 : fy_n - 1;
    const int k1 = k0 + 1 < fz_n ? k0 + 1 : fz_n - 1;
#define F(a, b, c) f[((int64_t)(a) * fy_n + (b)) * fz_n + (c)]
    const float c000 = F(i0, j0, k0), c100 = F(i1, j0, k0), c010 = F(i0, j1, k0),
                c110 = F(i1, j1, k0), c001 = F(i0, j0, k1), c101 = F(i1, j0, k1),
                c011 = F(i0, j1, k1), c111 = F(i1, j1, k1);
#undef F
    const float c00 = c000 * (1.0f - tx) + c100 * tx;
    const float c10 = c010 * (1.0f - tx) + c110 * tx;
    const float c01 = c001 * (1.0f - tx) + c101 * tx;
    const float c11 = c011 * (1.0f - tx) + c111 * tx;
    const float c0 = c00 * (1.0f - ty) + c10 * ty;
    const float c1 = c01 * (1.0f - ty) + c11 * ty;
    return c0 * (1.0f - tz) + c1 * tz;
}

/* _sample_velocity_at (fluid.py:91-104) then the backtrace p - u dt. */
static void backtrace(float *bx, float *by, float *bz, float px, float py, float pz,
                      const float *ux, const float *uy, const float *uz, int nx, int ny, int nz,
                      const float *org, float dx, float dt) {
    const float u = tri_sample(ux, nx + 1, ny, nz, px, py, pz, org, dx, 0.0f, 0.5f, 0.5f);
    const float v = tri_sample(uy, nx, ny + 1, nz, px, py, pz, org, dx, 0.5f, 0.0f, 0.5f);
    const float w = tri_sample(uz, nx, ny, nz + 1, px, py, pz, org, dx, 0.5f, 0.5f, 0.0f);
    *bx = px - u * dt;
    *by = py - v * dt;
    *bz = pz - w * dt;
}

/* extend_temperature_into_solids (fluid.py:338-382). */
void or_extend_temperature_f32(float *T_ext, const float *T, const int32_t *mat, int nx, int ny,
                               int nz, int mat_fluid) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                const int64_t c = IDX(i, j, k);
                float v = T[c];
                if (mat[c] != mat_fluid) {
                    if (i > 0 && mat[IDX(i - 1, j, k)] == mat_fluid) v = T[IDX(i - 1, j, k)];
                    else if (i < nx - 1 && mat[IDX(i + 1, j, k)] == mat_fluid) v = T[IDX(i + 1, j, k)];
                    else if (j > 0 && mat[IDX(i, j - 1, k)] == mat_fluid) v = T[IDX(i, j - 1, k)];
                    else if (j < ny - 1 && mat[IDX(i, j + 1, k)] == mat_fluid) v = T[IDX(i, j + 1, k)];
                    else if (k > 0 && mat[IDX(i, j, k - 1)] == mat_fluid) v = T[IDX(i, j, k - 1)];
                    else if (k < nz - 1 && mat[IDX(i, j, k + 1)] == mat_fluid) v = T[IDX(i, j, k + 1)];
                }
                T_ext[c] = v;
            }
}

/* advect_temperature (fluid.py:385-411): p = origin + (idx + 0.5) dx per axis. */
void or_advect_temperature_f32(float *T_new, const float *T_true, const float *T_ext,
                               const float *ux, const float *uy, const float *uz,
                               const int32_t *mat, int nx, int ny, int nz, const float *org,
                               float dx, float dt, int mat_fluid) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                const int64_t c = IDX(i, j, k);
                if (mat[c] != mat_fluid) {
                    T_new[c] = T_true[c];
                    continue;
                }
                const float px = org[0] + ((float)i + 0.5f) * dx;
                const float py = org[1] + ((float)j + 0.5f) * dx;
                const float pz = org[2] + ((float)k + 0.5f) * dx;
                float bx, by, bz;
                backtrace(&bx, &by, &bz, px, py, pz, ux, uy, uz, nx, ny, nz, org, dx, dt);
                T_new[c] = tri_sample(T_ext, nx, ny, nz, bx, by, bz, org, dx, 0.5f, 0.5f, 0.5f);
            }
}

/* advect_ux / advect_uy / advect_uz (fluid.py:414-498), axis 0 / 1 / 2:
 * boundary faces -> 0; faces whose two cells are both non-fluid keep their
 * value; others sample their own component at the backtraced point. */
void or_advect_velocity_f32(int axis, float *u_new, const float *ux, const float *uy,
                            const float *uz, const int32_t *mat, int nx, int ny, int nz,
                            const float *org, float dx, float dt, int mat_fluid) {
    const int fx_n = nx + (axis == 0), fy_n = ny + (axis == 1), fz_n = nz + (axis == 2);
    const float *u = axis == 0 ? ux : (axis == 1 ? uy : uz);
    const float ox = axis == 0 ? 0.0f : 0.5f, oy = axis == 1 ? 0.0f : 0.5f,
                oz = axis == 2 ? 0.0f : 0.5f;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < fx_n; ++i)
        for (int j = 0; j < fy_n; ++j)
            for (int k = 0; k < fz_n; ++k) {
                const int64_t f = ((int64_t)i * fy_n + j) * fz_n + k;
                const int a = axis == 0 ? i : (axis == 1 ? j : k);
                const int na = axis == 0 ? fx_n : (axis == 1 ? fy_n : fz_n);
                if (a == 0 || a == na - 1) {
                    u_new[f] = 0.0f;
                    continue;
                }
                const int64_t c1 = IDX(i, j, k);
                const int64_t c0 = axis == 0 ? IDX(i - 1, j, k)
                                             : (axis == 1 ? IDX(i, j - 1, k) : IDX(i, j, k - 1));
                if (mat[c0] != mat_fluid && mat[c1] != mat_fluid) {
                    u_new[f] = u[f];
                    continue;
                }
                const float px = org[0] + ((float)i + ox) * dx;
                const float py = org[1] + ((float)j + oy) * dx;
                const float pz = org[2] + ((float)k + oz) * dx;
                float bx, by, bz;
                backtrace(&bx, &by, &bz, px, py, pz, ux, uy, uz, nx, ny, nz, org, dx, dt);
                u_new[f] = tri_sample(u, fx_n, fy_n, fz_n, bx, by, bz, org, dx, ox, oy, oz);
            }
}

/* advect_all (fluid.py:737-776): velocities and T from the old fields into
 * the tmp arrays, then copied back. */
void or_advect_all_f32(float *ux, float *uy, float *uz, float *T, float *ux_tmp, float *uy_tmp,
                       float *uz_tmp, float *T_tmp, float *T_ext, const int32_t *mat, int nx,
                       int ny, int nz, const float *org, float dx, float dt, int mat_fluid) {
    or_advect_velocity_f32(0, ux_tmp, ux, uy, uz, mat, nx, ny, nz, org, dx, dt, mat_fluid);
    or_advect_velocity_f32(1, uy_tmp, ux, uy, uz, mat, nx, ny, nz, org, dx, dt, mat_fluid);
    or_advect_velocity_f32(2, uz_tmp, ux, uy, uz, mat, nx, ny, nz, org, dx, dt, mat_fluid);
    or_extend_temperature_f32(T_ext, T, mat, nx, ny, nz, mat_fluid);
    or_advect_temperature_f32(T_tmp, T, T_ext, ux, uy, uz, mat, nx, ny, nz, org, dx, dt,
                              mat_fluid);
    memcpy(ux, ux_tmp, sizeof(float) * (size_t)(nx + 1) * ny * nz);
    memcpy(uy, uy_tmp, sizeof(float) * (size_t)nx * (ny + 1) * nz);
    memcpy(uz, uz_tmp, sizeof(float) * (size_t)nx * ny * (nz + 1));
    memcpy(T, T_tmp, sizeof(float) * (size_t)nx * ny * nz);
}
