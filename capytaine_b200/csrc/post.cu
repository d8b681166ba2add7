// Right-hand sides, potentials and forces of the indirect BEM solve.
//
// * bem_build_rhs: radiation boundary conditions -i*omega*(dof . n) and
//   diffraction boundary conditions -(u_Airy . n) on the hull, zero on lid
//   panels (capytaine bem/problems_and_results.py:373-381, 440-449;
//   bem/airy_waves.py:56-95, infinite or finite depth).
// * bem_zgemm_ts: Y = alpha A X + beta Y for a tall matrix A (n x K, complex128,
//   column-major) and a few columns X (K x nrhs): the potential S @ sigma
//   (bem/solver.py:197-198) and the residuals b - K x.  Memory-bound on A: split
//   over K into partial sums reduced in a fixed order (deterministic).
// * bem_integrate_pressure / bem_froude_krylov: force integrals
//   F_d = sum_i p_i (-dof_d . n_i) area_i (bodies/bodies.py:238-250) of the
//   radiated/diffracted pressure i*omega*rho*phi and of the incident-wave
//   pressure (airy_waves.py:19-53, 98-102).
#include <cmath>

#include "common.cuh"

namespace bem {
namespace {


// Depth profiles of the Airy wave at height z (airy_waves.py:41-47, 80-85):
// cosh(k (z + h)) / cosh(k h) and sinh(k (z + h)) / cosh(k h) when 0 <= k h < 20,
// else both e^{k z} (the infinite-depth profile).
template <bool FINITE_DEPTH>
__device__ __forceinline__ void airy_profiles(double k, double z, double depth, double& cih, double& sih) {
  if constexpr (FINITE_DEPTH) {
    const double kh = k * depth;
    if (kh >= 0.0 && kh < 20.0) {
      const double ch = cosh(kh);
      cih = cosh(k * (z + depth)) / ch;
      sih = sinh(k * (z + depth)) / ch;
      return;
    }
  }
  cih = exp(k * z);
  sih = cih;
}

template <bool FINITE_DEPTH>
__global__ void build_rhs_kernel(int n, int64_t ldb, int64_t strideB, int batch, const double* __restrict__ omega,
                                 const double* __restrict__ wavenumber, double g, double depth, int ndof,
                                 const double* __restrict__ dofn, int nhead, const double* __restrict__ headings,
                                 const double* __restrict__ centers, const double* __restrict__ normals,
                                 const int* __restrict__ hull, double2* __restrict__ B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (i >= n) return;
  double2* Bb = B + (size_t)b * strideB;
  const double w = omega[b], k = wavenumber[b];
  const bool on_hull = hull == nullptr || hull[i] != 0;
  for (int d = 0; d < ndof; ++d) {
    const double v = on_hull ? dofn[(size_t)d * n + i] : 0.0;
    Bb[(size_t)i + (size_t)d * ldb] = make_double2(0.0, -w * v);  // -1j * omega * (dof . n)
  }
  const double x = centers[3 * i], y = centers[3 * i + 1], z = centers[3 * i + 2];
  const double nx = normals[3 * i], ny = normals[3 * i + 1], nz = normals[3 * i + 2];
  for (int h = 0; h < nhead; ++h) {
    double2 bc = make_double2(0.0, 0.0);
    if (on_hull) {
      const double beta = headings[h];
      double sb, cb;
      sincos(beta, &sb, &cb);
      const double wbar = x * cb + y * sb;
      double s, c;
      sincos(k * wbar, &s, &c);
      double cih, sih;
      airy_profiles<FINITE_DEPTH>(k, z, depth, cih, sih);
      const double amp_c = g * k / w * cih, amp_s = g * k / w * sih;
      // v = (g k / w) e^{i k wbar} (cos b cih, sin b cih, -i sih); v . n
      const double2 ec = make_double2(amp_c * c, amp_c * s);
      const double2 es = make_double2(amp_s * c, amp_s * s);
      const double horiz = cb * nx + sb * ny;
      // ec * horiz + es * (-i) * nz
      const double2 vn = make_double2(ec.x * horiz + es.y * nz, ec.y * horiz - es.x * nz);
      bc = make_double2(-vn.x, -vn.y);
    }
    Bb[(size_t)i + (size_t)(ndof + h) * ldb] = bc;
  }
}

constexpr int kTsRows = 256;
constexpr int kTsMaxRhs = 16;
constexpr int kTsUnroll = 8;

// Partial products of the split-K tall GEMM: one thread per row of A, the
// CTA's column chunk of X in shared memory (row kk holds NC right-hand sides,
// zero beyond nrhs), kTsUnroll streamed 16-byte loads of A in flight per
// thread before their FMAs.
template <int NC>
__global__ void __launch_bounds__(kTsRows) zgemm_ts_partial_kernel(int M, int K, int nrhs, int kchunk,
                                                                  const double2* __restrict__ A, int64_t lda,
                                                                  int64_t strideA, const double2* __restrict__ X,
                                                                  int64_t ldx, int64_t strideX,
                                                                  double2* __restrict__ part, const int* skip,
                                                                  const int* mskip) {
  if (skip && *skip) return;
  extern __shared__ double2 xs[];  // xs[kk * NC + c]
  const int b = blockIdx.z;
  if (mskip && mskip[b]) return;  // matrix b is not needed (converged)
  const int split = blockIdx.y;
  const int k0 = split * kchunk;
  const int kc = min(K, k0 + kchunk) - k0;
  A += (size_t)b * strideA;
  X += (size_t)b * strideX;
  for (int c = 0; c < NC; ++c)
    for (int kk = threadIdx.x; kk < kc; kk += blockDim.x)
      xs[kk * NC + c] = (c < nrhs) ? X[(size_t)(k0 + kk) + (size_t)c * ldx] : make_double2(0.0, 0.0);
  __syncthreads();
  const int row = blockIdx.x * kTsRows + threadIdx.x;
  if (row >= M) return;
  double2 acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = make_double2(0.0, 0.0);
  const double2* a = A + row + (size_t)k0 * lda;
  for (int kk = 0; kk < kc; kk += kTsUnroll) {
    double2 v[kTsUnroll];
#pragma unroll
    for (int u = 0; u < kTsUnroll; ++u)
      v[u] = (kk + u < kc) ? __ldcs(a + (size_t)(kk + u) * lda) : make_double2(0.0, 0.0);
#pragma unroll
    for (int u = 0; u < kTsUnroll; ++u) {
      if (kk + u < kc) {
        const double2* xr = xs + (kk + u) * NC;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const double2 x = xr[c];
          acc[c].x = fma(v[u].x, x.x, fma(-v[u].y, x.y, acc[c].x));
          acc[c].y = fma(v[u].x, x.y, fma(v[u].y, x.x, acc[c].y));
        }
      }
    }
  }
  double2* p = part + ((size_t)b * gridDim.y + split) * (size_t)M * nrhs;
#pragma unroll
  for (int c = 0; c < NC; ++c)
    if (c < nrhs) p[(size_t)c * M + row] = acc[c];
}

__global__ void zgemm_ts_reduce_kernel(int M, int nrhs, int nsplit, double2 alpha, double2 beta,
                                       const double2* __restrict__ part, double2* __restrict__ Y, int64_t ldy,
                                       int64_t strideY, const int* skip, const int* mskip) {
  if (skip && *skip) return;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y, b = blockIdx.z;
  if (mskip && mskip[b]) return;
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

// F[b][c][d] = coef_b * sum_i phi[b][i][c] * w[d][i], coef_b = i omega_b rho
__global__ void integrate_pressure_kernel(int n, int nrhs, int ndof, const double2* __restrict__ phi, int64_t ldp,
                                          int64_t strideP, const double* __restrict__ omega, double rho,
                                          const double* __restrict__ wdof, double2* __restrict__ F) {
  const int d = blockIdx.x, c = blockIdx.y, b = blockIdx.z;
  const double2* p = phi + (size_t)b * strideP + (size_t)c * ldp;
  const double* w = wdof + (size_t)d * n;
  double sx = 0.0, sy = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double2 v = p[i];
    sx += v.x * w[i];
    sy += v.y * w[i];
  }
  __shared__ double rx[256], ry[256];
  rx[threadIdx.x] = sx;
  ry[threadIdx.x] = sy;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off) {
      rx[threadIdx.x] += rx[threadIdx.x + off];
      ry[threadIdx.x] += ry[threadIdx.x + off];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double cw = omega[b] * rho;  // coef = (0, cw)
    F[((size_t)b * nrhs + c) * ndof + d] = make_double2(-cw * ry[0], cw * rx[0]);
  }
}

// Froude-Krylov: p0 = rho g cih(z) e^{i k (x cos b + y sin b)}, F[b][h][d] = sum_i p0_i w[d][i]
template <bool FINITE_DEPTH>
__global__ void froude_krylov_kernel(int n, int ndof, int nhead, const double* __restrict__ wavenumber, double rho,
                                     double g, double depth, const double* __restrict__ headings,
                                     const double* __restrict__ centers, const double* __restrict__ wdof,
                                     double2* __restrict__ F) {
  const int d = blockIdx.x, h = blockIdx.y, b = blockIdx.z;
  const double k = wavenumber[b];
  double sb, cb;
  sincos(headings[h], &sb, &cb);
  const double* w = wdof + (size_t)d * n;
  double sx = 0.0, sy = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = centers[3 * i], y = centers[3 * i + 1], z = centers[3 * i + 2];
    double s, c;
    sincos(k * (x * cb + y * sb), &s, &c);
    double cih, sih;
    airy_profiles<FINITE_DEPTH>(k, z, depth, cih, sih);
    const double amp = rho * g * cih * w[i];
    sx += amp * c;
    sy += amp * s;
  }
  __shared__ double rx[256], ry[256];
  rx[threadIdx.x] = sx;
  ry[threadIdx.x] = sy;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off) {
      rx[threadIdx.x] += rx[threadIdx.x + off];
      ry[threadIdx.x] += ry[threadIdx.x + off];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) F[((size_t)b * nhead + h) * ndof + d] = make_double2(rx[0], ry[0]);
}

}  // namespace
}  // namespace bem

using namespace bem;

extern "C" int bem_build_rhs(int n, int batch, const double* omega_dev, const double* wavenumber_dev, double g,
                             double water_depth, int ndof, const double* dofn_dev, int nhead,
                             const double* headings_dev, const double* centers_dev, const double* normals_dev,
                             const int32_t* hull_dev, void* B_dev, int64_t ldb, int64_t strideB, void* stream) {
  if (n <= 0 || batch <= 0 || ndof < 0 || nhead < 0 || ldb < n || !B_dev || !omega_dev || !wavenumber_dev ||
      (ndof > 0 && !dofn_dev) || (nhead > 0 && (!headings_dev || !centers_dev || !normals_dev)) ||
      !(water_depth > 0.0))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_build_rhs: bad arguments");
  dim3 grid(ceil_div(n, 128), batch);
  if (std::isinf(water_depth))
    build_rhs_kernel<false><<<grid, 128, 0, (cudaStream_t)stream>>>(n, ldb, strideB, batch, omega_dev, wavenumber_dev,
                                                                    g, water_depth, ndof, dofn_dev, nhead,
                                                                    headings_dev, centers_dev, normals_dev, hull_dev,
                                                                    (double2*)B_dev);
  else
    build_rhs_kernel<true><<<grid, 128, 0, (cudaStream_t)stream>>>(n, ldb, strideB, batch, omega_dev, wavenumber_dev,
                                                                   g, water_depth, ndof, dofn_dev, nhead,
                                                                   headings_dev, centers_dev, normals_dev, hull_dev,
                                                                   (double2*)B_dev);
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}

// Splits of the K dimension: up to 24 for parallelism, more when a chunk of
// X would not fit in shared memory (768 rows x 16 columns x 16 bytes = 192 KiB).
static int ts_nsplit(int K) { return std::max(std::max(1, std::min(24, K / 256)), ceil_div(K, 768)); }

extern "C" int64_t bem_zgemm_ts_workspace_bytes(int M, int K, int nrhs, int batch) {
  return (int64_t)batch * ts_nsplit(K) * (int64_t)M * nrhs * (int64_t)sizeof(double2);
}

namespace bem {
int zgemm_ts_enqueue(int M, int K, int nrhs, double alpha_re, double alpha_im, const void* A_dev, int64_t lda,
                     int64_t strideA, const void* X_dev, int64_t ldx, int64_t strideX, double beta_re,
                     double beta_im, void* Y_dev, int64_t ldy, int64_t strideY, int batch, void* work_dev,
                     void* stream, const int* skip, const int* mskip) {
  if (M <= 0 || K <= 0 || nrhs <= 0 || nrhs > kTsMaxRhs || batch <= 0 || !A_dev || !X_dev || !Y_dev || !work_dev ||
      lda < M || ldx < K || ldy < M)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zgemm_ts: bad arguments (nrhs must be <= 16)");
  const int nsplit = ts_nsplit(K);
  const int kchunk = ceil_div(K, nsplit);
  const int nc = nrhs <= 8 ? 8 : 16;
  const size_t smem = (size_t)kchunk * nc * sizeof(double2);
  if (smem > 200 * 1024) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zgemm_ts: chunk too large");
  cudaStream_t s = (cudaStream_t)stream;
  static bool configured = false;
  if (!configured) {
    BEM_CUDA_CHECK(cudaFuncSetAttribute(zgemm_ts_partial_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024));
    BEM_CUDA_CHECK(cudaFuncSetAttribute(zgemm_ts_partial_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024));
    configured = true;
  }
  TimedLaunch tl(kKZgemmTs, s);
  const dim3 grid(ceil_div(M, kTsRows), nsplit, batch);
  if (nc == 8)
    zgemm_ts_partial_kernel<8><<<grid, kTsRows, smem, s>>>(M, K, nrhs, kchunk, (const double2*)A_dev, lda, strideA,
                                                           (const double2*)X_dev, ldx, strideX, (double2*)work_dev, skip,
                                                           mskip);
  else
    zgemm_ts_partial_kernel<16><<<grid, kTsRows, smem, s>>>(M, K, nrhs, kchunk, (const double2*)A_dev, lda, strideA,
                                                            (const double2*)X_dev, ldx, strideX, (double2*)work_dev, skip,
                                                           mskip);
  zgemm_ts_reduce_kernel<<<dim3(ceil_div(M, 256), nrhs, batch), 256, 0, s>>>(
      M, nrhs, nsplit, make_double2(alpha_re, alpha_im), make_double2(beta_re, beta_im), (const double2*)work_dev,
      (double2*)Y_dev, ldy, strideY, skip, mskip);
  count_launches(2);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}
}  // namespace bem

extern "C" int bem_zgemm_ts(int M, int K, int nrhs, double alpha_re, double alpha_im, const void* A_dev, int64_t lda,
                            int64_t strideA, const void* X_dev, int64_t ldx, int64_t strideX, double beta_re,
                            double beta_im, void* Y_dev, int64_t ldy, int64_t strideY, int batch, void* work_dev,
                            void* stream) {
  return bem::zgemm_ts_enqueue(M, K, nrhs, alpha_re, alpha_im, A_dev, lda, strideA, X_dev, ldx, strideX, beta_re,
                               beta_im, Y_dev, ldy, strideY, batch, work_dev, stream, nullptr, nullptr);
}

extern "C" int bem_integrate_pressure(int n, int batch, int nrhs, int ndof, const void* phi_dev, int64_t ldp,
                                      int64_t strideP, const double* omega_dev, double rho, const double* wdof_dev,
                                      void* F_dev, void* stream) {
  if (n <= 0 || batch <= 0 || nrhs <= 0 || ndof <= 0 || !phi_dev || !omega_dev || !wdof_dev || !F_dev || ldp < n)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_integrate_pressure: bad arguments");
  integrate_pressure_kernel<<<dim3(ndof, nrhs, batch), 256, 0, (cudaStream_t)stream>>>(
      n, nrhs, ndof, (const double2*)phi_dev, ldp, strideP, omega_dev, rho, wdof_dev, (double2*)F_dev);
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}

extern "C" int bem_froude_krylov(int n, int batch, int ndof, int nhead, const double* wavenumber_dev, double rho,
                                 double g, double water_depth, const double* headings_dev, const double* centers_dev,
                                 const double* wdof_dev, void* F_dev, void* stream) {
  if (n <= 0 || batch <= 0 || ndof <= 0 || nhead <= 0 || !wavenumber_dev || !headings_dev || !centers_dev ||
      !wdof_dev || !F_dev || !(water_depth > 0.0))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_froude_krylov: bad arguments");
  const dim3 grid(ndof, nhead, batch);
  if (std::isinf(water_depth))
    froude_krylov_kernel<false><<<grid, 256, 0, (cudaStream_t)stream>>>(
        n, ndof, nhead, wavenumber_dev, rho, g, water_depth, headings_dev, centers_dev, wdof_dev, (double2*)F_dev);
  else
    froude_krylov_kernel<true><<<grid, 256, 0, (cudaStream_t)stream>>>(
        n, ndof, nhead, wavenumber_dev, rho, g, water_depth, headings_dev, centers_dev, wdof_dev, (double2*)F_dev);
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}
