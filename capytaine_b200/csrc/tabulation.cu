// Tabulation of the Delhommeau integrals on the GPU.
//
// Replaces delhommeau_integrals::numerical_integration / construct_tabulation /
// default_r_spacing / default_z_spacing (libs/libDelhommeau/src/
// Delhommeau_integrals.f90:43-153, 190-270).  One thread per (r, z) cell runs
// the Simpson sum over theta in the reference's order, accumulating in float64;
// exp(z)E1(z) is evaluated in float32 complex arithmetic as in the reference.
// This file is compiled with -fmad=false so that every float32 operation of the
// rational approximations rounds on its own, as the reference's does.
#include <cmath>
#include "integrals.cuh"

namespace bem {
namespace {
__global__ void __launch_bounds__(128) tabulation_kernel(const double* __restrict__ r_range, int nr,
                                                         const double* __restrict__ z_range, int nz, int npts,
                                                         double* __restrict__ table) {
  const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= (long long)nr * nz) return;
  // z fastest across the warp: neighbouring z share the same r, the cost per cell is similar.
  const int i = (int)(cell / nz);
  const int j = (int)(cell % nz);
  double out[kNbTab];
  numerical_integration_device(r_range[i], z_range[j], npts, out);
#pragma unroll
  for (int k = 0; k < kNbTab; ++k) table[cell * kNbTab + k] = out[k];
}
}  // namespace

}  // namespace bem

extern "C" int bem_default_r_spacing(int nr, double rmax, int grid_shape, double* out) {
  if (nr < 0 || (nr > 0 && out == nullptr)) return bem::set_error(BEM_ERR_INVALID_ARGUMENT, "bad r spacing arguments");
  if (nr == 0) return BEM_OK;
  const int nr_ref = 676, index_of_1_ref = 81;
  out[0] = 0.0;
  if (grid_shape == bem::kLegacyGrid) {
    for (int i = 2; i <= nr; ++i) {
      const float a = std::pow(10.0f, ((float)i - 1.0f) / 5.0f - 6.0f);
      const float b = (float)std::abs(i - 32) / 3.0f + 4.0f / 3.0f;
      out[i - 1] = (double)std::fmin(a, b);
    }
  } else {
    const int index_of_1 = (int)std::lround((float)((float)nr * 1.0f / (float)nr_ref * (float)index_of_1_ref));
    for (int i = 1; i <= nr; ++i) {
      if (i < index_of_1) {
        const float e = -10.0f * (1.0f - (float)(i - 1) / (float)(index_of_1 - 1));
        out[i - 1] = (double)std::pow(10.0f, e);
      } else {
        out[i - 1] = (rmax - 1.0) / (double)(nr - index_of_1) * (double)(i - index_of_1) + 1.0;
      }
    }
  }
  return BEM_OK;
}

extern "C" int bem_default_z_spacing(int nz, double zmin, int grid_shape, double* out) {
  if (nz < 0 || (nz > 0 && out == nullptr)) return bem::set_error(BEM_ERR_INVALID_ARGUMENT, "bad z spacing arguments");
  if (nz == 0) return BEM_OK;
  if (grid_shape == bem::kLegacyGrid) {
    for (int j = 1; j <= nz; ++j) {
      const float a = std::pow(10.0f, (float)j / 5.0f - 6.0f);
      const float b = std::pow(10.0f, (float)j / 8.0f - 4.5f);
      out[j - 1] = -(double)std::fmin(a, b);
    }
    if (nz == 46) out[45] = -16.0;
  } else {
    const double dz = (std::log10(std::fabs(zmin)) + 10.0) / (double)nz;
    for (int j = 1; j <= nz; ++j) out[j - 1] = -std::fmin(std::pow(10.0, dz * (double)j - 10.0), std::fabs(zmin));
  }
  return BEM_OK;
}

extern "C" int bem_construct_tabulation(const double* r_range_dev, int nr, const double* z_range_dev, int nz,
                                        int npts, double* table_dev, void* stream) {
  if (nr <= 0 || nz <= 0) return BEM_OK;
  if (!r_range_dev || !z_range_dev || !table_dev || npts <= 0)
    return bem::set_error(BEM_ERR_INVALID_ARGUMENT, "bem_construct_tabulation: null pointer or npts <= 0");
  const long long cells = (long long)nr * nz;
  const int threads = 128;
  bem::tabulation_kernel<<<bem::ceil_div(cells, threads), threads, 0, (cudaStream_t)stream>>>(
      r_range_dev, nr, z_range_dev, nz, npts, table_dev);
  bem::count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}

extern "C" int bem_tabulation_inverse_denominators(const double* range_host, int n, double* out_host) {
  if (!range_host || !out_host || n < 3)
    return bem::set_error(BEM_ERR_INVALID_ARGUMENT, "bem_tabulation_inverse_denominators: bad arguments");
  for (int i = 0; i < 3 * n; ++i) out_host[i] = 0.0;
  for (int c = 1; c + 1 < n; ++c) {
    const double u1 = range_host[c - 1], u2 = range_host[c], u3 = range_host[c + 1];
    out_host[3 * c] = 1.0 / ((u1 - u2) * (u1 - u3));
    out_host[3 * c + 1] = 1.0 / ((u2 - u3) * (u2 - u1));
    out_host[3 * c + 2] = 1.0 / ((u3 - u1) * (u3 - u2));
  }
  return BEM_OK;
}
