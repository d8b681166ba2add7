// Shared device definitions for the capytaine_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/capytaine_b200.h"

namespace bem {

// Constants of libDelhommeau constants.f90:22-32.  The Fortran literals carry no
// kind suffix, so they are single precision values promoted to double.
constexpr double kPI = (double)(float)3.141592653588979;
constexpr double kMinusOneOverFourPi = -1.0 / (4.0 * kPI);
constexpr double kEulerGamma = (double)(float)0.5772156649;
constexpr double kLog2 = 0.69314718055994530942;
constexpr double kEpsilon = 2.220446049250313e-16;  // EPSILON(1d0)
// Default-real thresholds of Green_Rankine.f90 / Green_wave.f90 / matrices.f90.
constexpr double kLit1em3 = (double)1e-3f;
constexpr double kLit1em4 = (double)1e-4f;
constexpr double kLit1em5 = (double)1e-5f;
constexpr double kLit1em6 = (double)1e-6f;
constexpr double kLit1em7 = (double)1e-7f;
constexpr double kLit1em8 = (double)1e-8f;
constexpr double kLit1em10 = (double)1e-10f;
constexpr double kLit1em2 = (double)1e-2f;

constexpr int kNbTab = 5;
constexpr int kLegacyGrid = 0;
constexpr int kScaledNemoh3Grid = 1;
constexpr int kHighFreq = 0;
constexpr int kLowFreq = 1;
constexpr int kLowFreqWithRankinePart = 2;

struct c64d {
  double re, im;
};

__host__ __device__ inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

#ifdef __CUDACC__
// x rounded to the nearest TF32 value (10 mantissa bits, ties away from zero,
// the low 13 bits cleared).  The tensor cores read a float32 operand as TF32
// by dropping those bits, which errs by up to 2^-10 and always towards zero;
// operands stored rounded err by at most 2^-11 and without that bias, which
// accumulates over the depth of a product otherwise.
__device__ __forceinline__ float tf32_rn(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
#endif

// Error recording shared by all entry points.
int set_cuda_error(cudaError_t e, const char* where);
int set_error(int code, const char* msg);
// Running count of kernels this library has launched (bem_launch_count).
void count_launches(int n);

// Optional per-kernel device timing (bem_kernel_timer_*): while enabled, a
// TimedLaunch scope records a CUDA event pair on the launch stream around the
// launches it encloses, attributed to one of these kernel classes.
enum KernelClass {
  kKAssemble = 0,
  kKZgemmDmma,
  kKCgemmTf32,
  kKCluGj,
  kKCluPanel,
  kKCtrsm,
  kKZluDiag,
  kKZluPanel,
  kKZtrsm,
  kKZgemmTs,
  kKClassCount
};
struct TimedLaunch {
  TimedLaunch(int kernel_class, cudaStream_t stream);
  ~TimedLaunch();
  int cls;
  cudaStream_t s;
  cudaEvent_t e0;
};

// Default iteration limit of the flag waits in the persistent block
// substitutions (polls of ~64 ns sleeps: a wait gives up after about a
// quarter of a second and reports BEM_ERR_TIMEOUT).
constexpr long long kDefaultSpinLimit = 4000000;

// Stream-ordered pieces shared between the solver files.
int zgemm_ts_enqueue(int M, int K, int nrhs, double alpha_re, double alpha_im, const void* A_dev, int64_t lda,
                     int64_t strideA, const void* X_dev, int64_t ldx, int64_t strideX, double beta_re,
                     double beta_im, void* Y_dev, int64_t ldy, int64_t strideY, int batch, void* work_dev,
                     void* stream, const int* skip, const int* mskip = nullptr);
// skip: one flag (the whole call returns at once while it is set); mskip:
// per-matrix flags (the work of matrix b is skipped while mskip[b] is set).
int clu_solve_enqueue(void* work_dev, int npad, int batch, void* B_dev, int64_t ldb, int64_t strideB, int nrhs,
                      int* err_dev, cudaStream_t s, const int* skip, long long spin_limit = kDefaultSpinLimit,
                      int withheld = -1, const int* mskip = nullptr);
int zlu_solve_enqueue(const void* A_dev, int n, int64_t lda, int64_t stride, int batch, const int* piv_dev,
                      const void* work_dev, void* B_dev, int64_t ldb, int64_t strideB, int nrhs, int* err_dev,
                      cudaStream_t s, const int* skip, long long spin_limit, const int* mskip = nullptr);
int* zlu_done_flag(void* work_dev, int n, int batch);

// Float32 planes of the mixed LU's workspace (lu_mixed.cu): matrix b's real
// plane at *re + b * stride, its imaginary plane im floats further, column-
// major with leading dimension ld (= npad).
int clu_planes(void* work_dev, int npad, float** re, int64_t* ld, int64_t* stride, int64_t* im);

// Packed copy of a complex update's result (tc_gemm.cu), written by its
// epilogue in the A operand layout of the next block step of the mixed LU:
//   kPackRows: row i -> [Re C(i, 0..127) | Im C(i, 0..127)]  (n = 128)
enum PackMode { kPackNone = 0, kPackRows = 1 };

// C (m x n complex in two float32 planes) -= A' B' (store = 0) or = A' B'
// (store = 1) on the tensor cores from packed operands; an optional second
// operand pair adds K' depth in the same pass over C; limit_host: per-matrix
// active sizes (grouped launches); pack: a packed copy of the result; lshape:
// only the first tile row and column of the square block, corner excluded;
// reserve_sms: SMs that a kernel beside this one holds (left out of the
// launch's width).
int cgemm_tf32_update(const float* Aop, int64_t a_rows, int a_row0, const float* Bop, int64_t b_rows, int b_row0,
                      int kp, float* Cr, float* Ci, int64_t ldc, int64_t c_stride, int c_row0, int c_col0, int m,
                      int n, int batch, int* err, cudaStream_t stream, int store = 0, const float* Aop1 = nullptr,
                      const float* Bop1 = nullptr, int run = 0, long long wait_limit = 0,
                      const int* limit_host = nullptr, float* pack = nullptr, int pack_mode = kPackNone,
                      int64_t pack_stride = 0, bool lshape = false, int reserve_sms = 0);

}  // namespace bem

#define BEM_CUDA_CHECK(call)                                  \
  do {                                                        \
    cudaError_t _e = (call);                                  \
    if (_e != cudaSuccess) return bem::set_cuda_error(_e, #call); \
  } while (0)
