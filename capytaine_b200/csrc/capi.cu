// Error reporting and small utilities of the C ABI.
#include <cstdio>
#include <cstring>
#include <string>
#include <atomic>
#include <mutex>
#include <vector>
#include "common.cuh"

namespace bem {
namespace {
thread_local std::string g_last_error;
}
std::atomic<long long> g_launches{0};
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {
struct TimerState {
  std::mutex mu;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pairs[kKClassCount];
};
TimerState& timers() {
  static TimerState t;
  return t;
}
std::atomic<int> g_timing{0};
const char* const kClassNames[kKClassCount] = {
    "assemble_kernel",   "zgemm_dmma_kernel",  "cgemm_tf32_update_kernel", "clu_gj_kernel",
    "clu_panel_kernel",  "ctrsm_persistent_kernel", "zlu_diag_kernel",  "zlu_panel_kernel",
    "ztrsm_persistent_kernel", "zgemm_ts_partial_kernel+reduce"};
void clear_timers_locked(TimerState& t) {
  for (auto& v : t.pairs) {
    for (auto& pr : v) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
    v.clear();
  }
}
}  // namespace

TimedLaunch::TimedLaunch(int kernel_class, cudaStream_t stream) : cls(kernel_class), s(stream), e0(nullptr) {
  if (!g_timing.load(std::memory_order_relaxed)) return;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventRecord(e0, s) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    e0 = nullptr;
  }
}

TimedLaunch::~TimedLaunch() {
  if (!e0) return;
  cudaEvent_t e1 = nullptr;
  if (cudaEventCreate(&e1) != cudaSuccess || cudaEventRecord(e1, s) != cudaSuccess) {
    if (e1) cudaEventDestroy(e1);
    cudaEventDestroy(e0);
    return;
  }
  TimerState& t = timers();
  std::lock_guard<std::mutex> lock(t.mu);
  t.pairs[cls].emplace_back(e0, e1);
}

int set_error(int code, const char* msg) {
  g_last_error = msg ? msg : "";
  return code;
}

int set_cuda_error(cudaError_t e, const char* where) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%s: %s (%s)", where, cudaGetErrorString(e), cudaGetErrorName(e));
  g_last_error = buf;
  if (e == cudaErrorMemoryAllocation) return BEM_ERR_OUT_OF_MEMORY;
  return BEM_ERR_CUDA;
}

}  // namespace bem

extern "C" const char* bem_last_error(void) { return bem::g_last_error.c_str(); }

extern "C" int bem_version(void) { return 100; }

extern "C" long long bem_launch_count(void) { return bem::g_launches.load(std::memory_order_relaxed); }

extern "C" int bem_kernel_timer_enable(int on) {
  bem::TimerState& t = bem::timers();
  std::lock_guard<std::mutex> lock(t.mu);
  bem::clear_timers_locked(t);
  bem::g_timing.store(on ? 1 : 0);
  return BEM_OK;
}

extern "C" const char* bem_kernel_class_name(int kernel_class) {
  if (kernel_class < 0 || kernel_class >= bem::kKClassCount) return "";
  return bem::kClassNames[kernel_class];
}

extern "C" int bem_kernel_timer_read(int kernel_class, double* total_ms, long long* launches) {
  if (kernel_class < 0 || kernel_class >= bem::kKClassCount || !total_ms || !launches)
    return bem::set_error(BEM_ERR_INVALID_ARGUMENT, "bem_kernel_timer_read: bad arguments");
  bem::TimerState& t = bem::timers();
  std::lock_guard<std::mutex> lock(t.mu);
  double sum = 0.0;
  for (auto& pr : t.pairs[kernel_class]) {
    BEM_CUDA_CHECK(cudaEventSynchronize(pr.second));
    float ms = 0.0f;
    BEM_CUDA_CHECK(cudaEventElapsedTime(&ms, pr.first, pr.second));
    sum += ms;
  }
  *total_ms = sum;
  *launches = (long long)t.pairs[kernel_class].size();
  return BEM_OK;
}
