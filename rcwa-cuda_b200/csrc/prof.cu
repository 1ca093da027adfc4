// Optional per-kernel timing with CUDA events on the launching stream.
// When enabled (rcwa_profile_enable), the hot kernels are bracketed by event
// pairs; rcwa_profile_query() synchronises on those events and returns the
// summed device time and launch count of one kernel family.  Disabled by
// default: the solve path then records nothing.
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace rcwa {

namespace {
struct Rec {
  cudaEvent_t a, b;
};
std::mutex g_mu;
bool g_on = false;
std::map<std::string, std::vector<Rec>> g_recs;
std::map<std::string, double> g_flops;
std::vector<cudaEvent_t> g_pool;

cudaEvent_t get_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

static thread_local int t_suspend = 0;

bool prof_on() { return g_on && t_suspend == 0; }

// Calls that must not create any CUDA object suspend event recording on their
// thread for their duration.
void prof_suspend(bool on) { t_suspend += on ? 1 : -1; }

void* prof_begin(cudaStream_t s) {
  if (!g_on || t_suspend) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  cudaEvent_t e = get_event();
  cudaEventRecord(e, s);
  return (void*)e;
}

void prof_end(cudaStream_t s, void* tok, const char* name) {
  if (!g_on || !tok) return;
  std::lock_guard<std::mutex> lk(g_mu);
  cudaEvent_t e = get_event();
  cudaEventRecord(e, s);
  g_recs[name].push_back(Rec{(cudaEvent_t)tok, e});
}

void prof_add_flops(const char* name, double flops) {
  if (!g_on) return;
  std::lock_guard<std::mutex> lk(g_mu);
  g_flops[name] += flops;
}

}  // namespace rcwa

extern "C" {

int rcwa_profile_enable(int on) {
  std::lock_guard<std::mutex> lk(rcwa::g_mu);
  rcwa::g_on = on != 0;
  return RCWA_OK;
}

int rcwa_profile_reset(void) {
  std::lock_guard<std::mutex> lk(rcwa::g_mu);
  for (auto& kv : rcwa::g_recs)
    for (auto& r : kv.second) {
      cudaEventSynchronize(r.b);
      rcwa::g_pool.push_back(r.a);
      rcwa::g_pool.push_back(r.b);
    }
  rcwa::g_recs.clear();
  rcwa::g_flops.clear();
  return RCWA_OK;
}

int rcwa_profile_query(const char* name, double* total_ms, uint64_t* launches, double* flops) {
  if (!name || !total_ms || !launches || !flops) {
    rcwa::set_last_error("NULL argument");
    return RCWA_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(rcwa::g_mu);
  *total_ms = 0.0;
  *launches = 0;
  auto fi = rcwa::g_flops.find(name);
  *flops = fi == rcwa::g_flops.end() ? 0.0 : fi->second;
  auto it = rcwa::g_recs.find(name);
  if (it == rcwa::g_recs.end()) return RCWA_OK;
  for (auto& r : it->second) {
    RCWA_CUDA_TRY(cudaEventSynchronize(r.b));
    float ms = 0.f;
    RCWA_CUDA_TRY(cudaEventElapsedTime(&ms, r.a, r.b));
    *total_ms += ms;
    *launches += 1;
  }
  return RCWA_OK;
}

}  // extern "C"
