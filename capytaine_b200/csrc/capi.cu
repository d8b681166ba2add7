// Error reporting and small utilities of the C ABI.
#include <cstdio>
#include <cstring>
#include <string>
#include <atomic>
#include "common.cuh"

namespace bem {
namespace {
thread_local std::string g_last_error;
}
std::atomic<long long> g_launches{0};
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

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
