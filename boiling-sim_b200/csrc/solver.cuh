// solver.cuh -- types shared by the to-tolerance solver kernels.
#pragma once
#include <cstdint>

#include "bsp_common.cuh"

namespace bsp {

constexpr int MAX_LEVELS = 12;
constexpr int COARSEST_CELLS = 256;   // the hierarchy stops at or below this size
constexpr int COARSEST_MAX = 4096;    // one CTA holds the coarsest level in shared memory
constexpr int PARTIAL_STRIDE = 16384;  // max blocks of any reducing kernel

template <class T>
struct Level {
  int nx, ny, nz;
  const uint8_t *mask;  // class | n_solid << 2 (effective classes for l >= 1)
  T *r;                 // right-hand side of this level
  T *e;                 // correction of this level (level 0: z)
  // One byte per CTA tile of the column-layout grid (fine_grid): nonzero when
  // the tile holds a fluid cell.  Tiles without fluid are skipped: every
  // vector of the solver is zero on non-fluid cells and stays so.  Null: no
  // skipping.
  const uint8_t *tiles;
};

// Device-resident control block of one solve.  Written only by the one-block
// control kernels; read by every other kernel at entry.
struct SolverState {
  double tol, eta, eta_eff;
  double b_norm2, r64_norm2, rel, scale, rhat_norm2;
  double rz, beta, alpha, rr_inner;
  int max_outer, max_inner;
  int outer_it, inner_it, total_inner;
  int done, inner_done, status, finalize;
  int dev_error;  // set by a kernel whose bounded wait gave up
  int pending;    // a CG update (alpha, ps, Ap) waits to be applied by the next restriction
  // loop guards of the graph-driven solve: counted by the condition kernels
  // themselves so every WHILE node ends even if other state went wrong
  int guard_inner, guard_outer;
  int tail_count;  // CTAs of the current level-0 kernel done (its last CTA runs the scalar update)
  // 1 from the ||b|| pass until the first outer check while the iterate is
  // still zero: the partials of that pass are the first outer residual's, so
  // the norm pass before the first outer check returns at entry
  int norm_cached;
  // 1 while the FP64 iterate x is known to be all zero (x is zeroed before
  // the first residual pass; cleared by a nonzero warm start and by the
  // first x update): the residual kernels then skip its loads
  int x_zero;
};

// The scalar updates that follow a level-0 kernel's FP64 partial sums: by a
// one-block kernel (solver.cu) or by the last CTA of the producing kernel
// (fine_tma_kernel), the same code either way.
enum TailKind { TAIL_NONE = 0, TAIL_INNER_CHECK = 1, TAIL_BETA = 2, TAIL_ALPHA = 3 };
// after the fused update + restriction: count the iteration, test ||r||
__device__ __forceinline__ void apply_inner_check(SolverState *st, double rr) {
  if (!st->pending) return;
  st->pending = 0;
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
// after the prolongation (z and r.z): beta = rz_new / rz
__device__ __forceinline__ void apply_beta(SolverState *st, double rz) {
  st->beta = (st->inner_it == 0 || st->rz == 0.0) ? 0.0 : rz / st->rz;
  st->rz = rz;
}
// after A ps (ps.Ap): alpha = rz / ps.Ap; the update is applied by the next restriction
__device__ __forceinline__ void apply_alpha(SolverState *st, double pap) {
  st->alpha = pap > 0.0 ? st->rz / pap : 0.0;
  st->pending = 1;
}
__device__ __forceinline__ void apply_tail(SolverState *st, int kind, double v) {
  if (kind == TAIL_INNER_CHECK) apply_inner_check(st, v);
  else if (kind == TAIL_BETA) apply_beta(st, v);
  else if (kind == TAIL_ALPHA) apply_alpha(st, v);
}
// Host: the next level-0 TMA launch runs `kind` in its last CTA;
// fine_tail_taken() says whether it did (clearing the request either way).
void fine_tail_request(SolverState *st, int kind);
bool fine_tail_taken();

// Level-0 kernels on the column layout (mgfine.cu); nz % 4 == 0 required.
int fine_grid_blocks(int nx, int ny, int nz);
template <class T>
void launch_fine_psap(int nx, int ny, int nz, const uint8_t *mask, const uint8_t *tiles,
                      const T *z, const T *prev, T *cur, T *Ap, double *partials,
                      const SolverState *st, cudaStream_t s);
template <class T>
void launch_fine_up(const Level<T> &f, const Level<T> &c, T *z, double *partials, float alpha,
                    const SolverState *st, cudaStream_t s);
template <class T>
void launch_fine_down(const Level<T> &f, const Level<T> &c, const SolverState *st,
                      cudaStream_t s);
// Two smoothing sweeps per side on a coarse level (TMA tile kernels; false
// when they cannot run): one sweep from e_in (w r when NULL) into out; the
// residual of the stored e restricted to c.r; out = e_in + alpha P c.e and
// one sweep.
template <class T>
bool launch_fine_smooth(const Level<T> &f, const T *e_in, T *out, const SolverState *st,
                        cudaStream_t s);
template <class T>
bool launch_fine_down_e(const Level<T> &f, const Level<T> &c, const T *e_in,
                        const SolverState *st, cudaStream_t s);
template <class T>
bool launch_fine_up_e(const Level<T> &f, const Level<T> &c, const T *e_in, T *out,
                      double *partials, float alpha, const SolverState *st, cudaStream_t s);
// FP64 residual on the column layout; returns the number of partial blocks.
template <class T>
int launch_resid64_col(int nx, int ny, int nz, const uint8_t *mask, const uint8_t *tiles,
                       const float *div, const double *x, double bscale, T *rhat, float *e,
                       double *partials, const SolverState *st, bool write, cudaStream_t s);
// e += alpha ps; r -= alpha Ap; partial r.r -- streaming over the column
// tiles (no mask: ps and Ap are zero off fluid); returns the partial count.
template <class T>
int launch_cg_update_col(int nx, int ny, int nz, const uint8_t *tiles, float *e, T *r,
                         const T *ps, const T *Ap, double *partials, const SolverState *st,
                         cudaStream_t s);
// Level-0 restriction with the previous iteration's CG update fused in
// (mgfine.cu, TMA path); false when it cannot run.  f.r is r_in.
template <class T>
bool launch_fine_down_update(const Level<T> &f, const Level<T> &c, T *r_out, float *e,
                             const T *ps, const T *Ap, double *partials, const SolverState *st,
                             cudaStream_t s, T *rs = nullptr, const uint8_t *pat = nullptr,
                             const float *tab = nullptr);
// Trilinear transfers between levels 0 and 1 (mgfine.cu): the 1 / tot table
// (device address, built once per device), the fine parent patterns (once per
// geometry), the gather of the scaled residual into c.r, and the prolongation
// + post-smoothing onto level 0 (TMA path; false when it cannot run).
const float *tri_table();
template <class T>
void launch_tri_setup(uint8_t *pat, const Level<T> &f, const Level<T> &c, cudaStream_t s);
template <class T>
void launch_tri_restrict(const Level<T> &f, const Level<T> &c, const T *rs, const SolverState *st,
                         cudaStream_t s);
template <class T>
bool launch_fine_up_tri(const Level<T> &f, const Level<T> &c, T *z, double *partials,
                        float alpha, const uint8_t *pat, const float *tab, const SolverState *st,
                        cudaStream_t s);
bool fine_tma_available(int nz);
// The coarse part of a V-cycle (levels 1 .. L-1) as one cooperative kernel
// (mgcoarse.cu); false when not launched (the per-level kernels then run).
template <class T>
bool launch_coarse_cycle(const Level<T> *lv, int L, float *scratch, const float *cinv,
                         const int *cflag, void *ctl, float alpha, SolverState *st,
                         cudaStream_t s);
size_t coarse_cycle_scratch_floats(const int *dims, int L);
// One flag byte per column tile: any fluid cell in the tile.
void launch_tile_flags(int nx, int ny, int nz, const uint8_t *mask, uint8_t *flags,
                       cudaStream_t s);

}  // namespace bsp
