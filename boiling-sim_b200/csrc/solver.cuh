// solver.cuh -- types shared by the to-tolerance solver kernels.
#pragma once
#include <cstdint>

namespace bsp {

constexpr int MAX_LEVELS = 12;
constexpr int COARSEST_CELLS = 512;   // the hierarchy stops at or below this size
constexpr int COARSEST_MAX = 4096;    // one CTA holds the coarsest level in shared memory
constexpr int PARTIAL_STRIDE = 2048;  // max blocks of any reducing kernel

template <class T>
struct Level {
  int nx, ny, nz;
  const uint8_t *mask;  // class | n_solid << 2 (effective classes for l >= 1)
  T *r;                 // right-hand side of this level
  T *e;                 // correction of this level (level 0: z)
};

// Device-resident control block of one solve.  Written only by the one-block
// control kernels; read by every other kernel at entry.
struct SolverState {
  double tol, eta;
  double b_norm2, r64_norm2, rel, scale, rhat_norm2;
  double rz, beta, alpha, rr_inner;
  int max_outer, max_inner;
  int outer_it, inner_it, total_inner;
  int done, inner_done, status, finalize, pad;
};

}  // namespace bsp
