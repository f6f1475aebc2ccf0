// profile.cuh -- optional per-kernel-class CUDA-event timing inside the library.
//
// When enabled (bsp_profile_enable), each launch of an instrumented kernel is
// bracketed by two events on its own stream; bsp_profile_read sums the elapsed
// times per class.  Disabled, a ProfScope costs one branch.
#pragma once
#include <cuda_runtime.h>

namespace bsp {

enum ProfClass {
  PROF_SWEEP = 0,      // Jacobi sweep (column or generic kernel)
  PROF_MG_DOWN0 = 1,   // restriction from the fine level
  PROF_MG_UP0 = 2,     // prolongation + post-smoothing onto the fine level (z)
  PROF_CG_PSAP = 3,    // search direction + A ps
  PROF_CG_UPDATE = 4,  // e += alpha ps, r -= alpha Ap
  PROF_RESID64 = 5,    // FP64 residual passes
  PROF_XUPDATE = 6,    // FP64 iterate update
  PROF_MG_COARSE = 7,  // coarse-level multigrid: the one-launch cycle (or per-level kernels)
  PROF_CONTROL = 8,    // one-block scalar kernels, level setup, conversions
  PROF_PROJ = 9,       // divergence, gradient subtract, no-slip, rhs
  PROF_UNET = 10,      // learned warm start: network layers, input packing, head
  PROF_MG_MID = 11,    // levels 1-2 of the V-cycle on the column tile kernels (split mode)
  PROF_NCLASS = 12
};

bool prof_enabled();
// While a graph is being captured, event timing is suspended (events recorded
// into a graph would be re-recorded on every replay).
void prof_suspend(bool on);
void prof_record(int cls, cudaEvent_t a, cudaEvent_t b);
cudaEvent_t prof_event();

struct ProfScope {
  int cls;
  cudaStream_t s;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(int c, cudaStream_t st) : cls(c), s(st) {
    if (prof_enabled()) {
      a = prof_event();
      b = prof_event();
      cudaEventRecord(a, s);
    }
  }
  ~ProfScope() {
    if (a) {
      cudaEventRecord(b, s);
      prof_record(cls, a, b);
    }
  }
};

}  // namespace bsp
