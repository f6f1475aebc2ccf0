// profile.cu -- storage for the library's optional per-kernel event timing.
#include <mutex>
#include <vector>

#include "bsp_common.cuh"
#include "profile.cuh"

namespace bsp {

namespace {
struct Rec {
  int cls;
  cudaEvent_t a, b;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_pool;
}  // namespace

thread_local bool g_suspended = false;

bool prof_enabled() { return g_on && !g_suspended; }
void prof_suspend(bool on) { g_suspended = on; }

cudaEvent_t prof_event() {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void prof_record(int cls, cudaEvent_t a, cudaEvent_t b) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_recs.push_back({cls, a, b});
}

}  // namespace bsp

extern "C" int bsp_profile_enable(int on) {
  std::lock_guard<std::mutex> lk(bsp::g_mu);
  bsp::g_on = on != 0;
  return BSP_OK;
}

// Sums the recorded launches per class (waits for their stop events), then
// clears the record.  ms[c] and launches[c] for c < nclass.
extern "C" int bsp_profile_read(double *ms, long long *launches, int nclass) {
  std::vector<bsp::Rec> recs;
  {
    std::lock_guard<std::mutex> lk(bsp::g_mu);
    recs.swap(bsp::g_recs);
  }
  for (int c = 0; c < nclass; ++c) {
    if (ms) ms[c] = 0.0;
    if (launches) launches[c] = 0;
  }
  cudaError_t err = cudaSuccess;
  for (const auto &r : recs) {
    float t = 0.0f;
    cudaError_t e = cudaEventSynchronize(r.b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.a, r.b);
    if (e != cudaSuccess) err = e;
    if (r.cls >= 0 && r.cls < nclass) {
      if (ms) ms[r.cls] += t;
      if (launches) launches[r.cls] += 1;
    }
  }
  std::lock_guard<std::mutex> lk(bsp::g_mu);
  for (const auto &r : recs) {
    bsp::g_pool.push_back(r.a);
    bsp::g_pool.push_back(r.b);
  }
  return (int)err;
}
