// Allocation-free variant of bem_zgemm_ts (Y = alpha A X + beta Y for a tall
// complex128 A and a few columns X).
//
// Who needs it: callers that may only hand this library buffers they already
// own and cannot allocate device memory themselves — for example a host
// application that reserves one fixed device pool up front and forbids any
// later device allocation, or a latency-critical loop in which a cudaMalloc
// (which can synchronise the device and fragment memory) is not acceptable.
// bem_zgemm_ts needs a caller-provided workspace for its split-K partial sums;
// this variant keeps those partial sums in a file-scope device array instead.
//
// Limits and sharing rules:
//  * the scratch array holds kStaticScratch = 524288 complex128 entries (8 MiB),
//    reserved on every GPU that loads this library, for the life of the process;
//    a call needs M * nrhs * batch <= kStaticScratch entries (the number of
//    K-splits shrinks to fit, down to one) and is rejected with
//    BEM_ERR_INVALID_ARGUMENT otherwise;
//  * every call on a device uses the same array and leaves its partial sums in
//    it; each call overwrites every entry it later reads, so nothing needs to be
//    cleared, but calls whose work overlaps on the GPU (different streams, or
//    several host threads without ordering) race on the array and must be
//    serialised by the caller;
//  * the first call on each device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it with the
//    device's current context; make that first call before any stream capture
//    on that device.  A call made in a different context of that device (the
//    primary context was reset by cudaDeviceReset and re-created) looks the
//    address up again, so that no stale address reaches a kernel;
//  * batch <= 65535 (one grid z-slice per matrix).
// No cudaMalloc, cudaFree or allocating library routine is called here.
#include <cuda.h>
#include <algorithm>
#include <mutex>
#include "common.cuh"

namespace bem {
namespace {

constexpr int kStaticScratch = 1 << 19;  // complex128 entries (8 MiB)
constexpr int kSRows = 128;
constexpr int kSMaxRhs = 16;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double2 g_static_scratch[kStaticScratch];

std::mutex g_scratch_mutex;
double2* g_scratch_ptr[kMaxDevices] = {nullptr};
CUcontext g_scratch_ctx[kMaxDevices] = {nullptr};

// cuCtxGetCurrent through the runtime's driver entry points (no link-time
// dependency on libcuda, as for the tensor maps).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current_fn() {
  static CtxGetCurrentFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(p);
  }
  return fn;
}

// Device address of g_static_scratch for the current device, looked up on the
// first call in each context of the device.
int static_scratch_address(double2** out) {
  int dev = 0;
  BEM_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return set_error(BEM_ERR_UNSUPPORTED, "device index out of range");
  CtxGetCurrentFn get_ctx = ctx_get_current_fn();
  if (!get_ctx) return set_error(BEM_ERR_CUDA, "cuCtxGetCurrent is not available from the driver");
  // null until the runtime has made a context current in this host thread
  CUcontext ctx = nullptr;
  if (get_ctx(&ctx) != CUDA_SUCCESS) ctx = nullptr;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_ptr[dev] == nullptr || ctx == nullptr || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    // also makes the device's primary context current in this thread
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || p == nullptr) {
      g_scratch_ptr[dev] = nullptr;
      return set_error(BEM_ERR_CUDA, "cudaGetSymbolAddress of the static scratch array failed");
    }
    if (get_ctx(&ctx) != CUDA_SUCCESS || ctx == nullptr) {
      g_scratch_ptr[dev] = nullptr;
      return set_error(BEM_ERR_CUDA, "no current CUDA context for the static scratch array");
    }
    g_scratch_ptr[dev] = static_cast<double2*>(p);
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return BEM_OK;
}

constexpr int kXStage = 256;  // K values of X staged in shared memory at a time

__global__ void __launch_bounds__(kSRows) zgemm_ts_partial_static_kernel(int M, int K, int nrhs, int kchunk,
                                                                        const double2* __restrict__ A, int64_t lda,
                                                                        int64_t strideA,
                                                                        const double2* __restrict__ X, int64_t ldx,
                                                                        int64_t strideX, double2* __restrict__ part) {
  extern __shared__ double2 xs[];  // kXStage x nrhs
  const int b = blockIdx.z, split = blockIdx.y;
  const int k0 = split * kchunk;
  const int k1 = min(K, k0 + kchunk);
  A += (size_t)b * strideA;
  X += (size_t)b * strideX;
  const int row = blockIdx.x * kSRows + threadIdx.x;
  double2 acc[kSMaxRhs];
#pragma unroll
  for (int c = 0; c < kSMaxRhs; ++c) acc[c] = make_double2(0.0, 0.0);
  for (int ks = k0; ks < k1; ks += kXStage) {
    const int kn = min(kXStage, k1 - ks);
    __syncthreads();
    for (int idx = threadIdx.x; idx < kn * nrhs; idx += blockDim.x) {
      const int kk = idx % kn, c = idx / kn;
      xs[c * kXStage + kk] = X[(size_t)(ks + kk) + (size_t)c * ldx];
    }
    __syncthreads();
    if (row < M) {
      const double2* a = A + row + (size_t)ks * lda;
      for (int kk = 0; kk < kn; ++kk) {
        const double2 v = __ldcs(a + (size_t)kk * lda);
#pragma unroll
        for (int c = 0; c < kSMaxRhs; ++c) {
          if (c < nrhs) {
            const double2 x = xs[c * kXStage + kk];
            acc[c].x += v.x * x.x - v.y * x.y;
            acc[c].y += v.x * x.y + v.y * x.x;
          }
        }
      }
    }
  }
  if (row >= M) return;
  double2* p = part + ((size_t)b * gridDim.y + split) * (size_t)M * nrhs;
#pragma unroll
  for (int c = 0; c < kSMaxRhs; ++c)
    if (c < nrhs) p[(size_t)c * M + row] = acc[c];
}

__global__ void zgemm_ts_reduce_static_kernel(int M, int nrhs, int nsplit, double2 alpha, double2 beta,
                                              const double2* __restrict__ part, double2* __restrict__ Y, int64_t ldy,
                                              int64_t strideY) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y, b = blockIdx.z;
  if (row >= M) return;
  double2 s = make_double2(0.0, 0.0);
  for (int sp = 0; sp < nsplit; ++sp) {
    const double2 v = part[(((size_t)b * nsplit + sp) * nrhs + c) * (size_t)M + row];
    s.x += v.x;
    s.y += v.y;
  }
  double2* y = Y + (size_t)b * strideY + (size_t)c * ldy + row;
  double2 out = make_double2(alpha.x * s.x - alpha.y * s.y, alpha.x * s.y + alpha.y * s.x);
  if (beta.x != 0.0 || beta.y != 0.0) {
    const double2 o = *y;
    out.x += beta.x * o.x - beta.y * o.y;
    out.y += beta.x * o.y + beta.y * o.x;
  }
  *y = out;
}

}  // namespace
}  // namespace bem

using namespace bem;

extern "C" int64_t bem_zgemm_ts_static_capacity(void) { return kStaticScratch; }

extern "C" int bem_zgemm_ts_static(int M, int K, int nrhs, double alpha_re, double alpha_im, const void* A_dev,
                                   int64_t lda, int64_t strideA, const void* X_dev, int64_t ldx, int64_t strideX,
                                   double beta_re, double beta_im, void* Y_dev, int64_t ldy, int64_t strideY,
                                   int batch, void* stream) {
  if (M <= 0 || K <= 0 || nrhs <= 0 || nrhs > kSMaxRhs || batch <= 0 || !A_dev || !X_dev || !Y_dev || lda < M ||
      ldx < K || ldy < M)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zgemm_ts_static: bad arguments (nrhs must be <= 16)");
  if (batch > 65535)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zgemm_ts_static: batch must be <= 65535 (one grid slice each)");
  const long long per_split = (long long)M * nrhs * batch;
  if (per_split > kStaticScratch) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "bem_zgemm_ts_static: M*nrhs*batch = %lld exceeds the static scratch capacity of %d complex "
                  "entries; use bem_zgemm_ts with a caller workspace",
                  per_split, kStaticScratch);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  double2* scratch = nullptr;
  int st = static_scratch_address(&scratch);
  if (st) return st;
  // As many K-splits as bem_zgemm_ts would use, reduced to fit the array.
  int nsplit = std::max(1, std::min(64, K / 96));
  nsplit = (int)std::min<long long>(nsplit, kStaticScratch / per_split);
  nsplit = std::max(nsplit, 1);
  const int kchunk = ceil_div(K, nsplit);
  const size_t smem = (size_t)kXStage * nrhs * sizeof(double2);  // <= 64 KiB
  if (smem > 48 * 1024)
    BEM_CUDA_CHECK(cudaFuncSetAttribute(zgemm_ts_partial_static_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
  cudaStream_t s = (cudaStream_t)stream;
  zgemm_ts_partial_static_kernel<<<dim3(ceil_div(M, kSRows), nsplit, batch), kSRows, smem, s>>>(
      M, K, nrhs, kchunk, (const double2*)A_dev, lda, strideA, (const double2*)X_dev, ldx, strideX, scratch);
  zgemm_ts_reduce_static_kernel<<<dim3(ceil_div(M, 256), nrhs, batch), 256, 0, s>>>(
      M, nrhs, nsplit, make_double2(alpha_re, alpha_im), make_double2(beta_re, beta_im), scratch, (double2*)Y_dev,
      ldy, strideY);
  count_launches(2);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}
