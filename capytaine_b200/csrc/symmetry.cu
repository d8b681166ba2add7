// Block transforms of the symmetric-mesh engines.
//
// A mesh made of m images g_0 h, ..., g_{m-1} h of one sub-mesh h under a
// group of symmetries of the free-surface Green function (reflections in
// vertical planes, rotations about Oz) has influence matrices whose block
// (I, J) depends only on g_I^-1 g_J: they are fixed by the first column of
// blocks C_j = G(g_j h, h) (capytaine bem/engines.py:178-247).  A linear
// combination over the group (a discrete Fourier transform for rotations,
// sums and differences for reflections; tools/block_circulant_matrices.py:
// 138-162, 276-301, 410-419) turns the dense system into independent systems
// of size N / m (N / (m / 2) for dihedral symmetry, whose macro-blocks are 2 x 2
// sub-blocks), and maps right-hand sides and solutions between the whole mesh
// and those systems.  All three are one operation on complex128 data:
//
//   out[f][o][c][r] = sum_i W[o][i] in[f][src[i]][c][r]
//
// with separate strides for the frequency f, the block index, the column c
// and the row r (unit stride), so that the same kernel reads row blocks of the
// first block column, writes column-major systems with their own leading
// dimension, and gathers or scatters the segments of a vector.
#include "common.cuh"

namespace bem {
namespace {

constexpr int kCombRows = 128;  // threads per CTA, one row each
constexpr int kCombOut = 8;     // outputs (o) per thread

__global__ void __launch_bounds__(kCombRows) block_combine_kernel(
    const double2* __restrict__ in, int64_t ifs, int64_t ibs, int64_t ics, double2* __restrict__ out, int64_t ofs,
    int64_t obs, int64_t ocs, const double2* __restrict__ W, const int* __restrict__ src, int mi, int mo, int rows,
    int ochunks) {
  const int r = blockIdx.x * kCombRows + threadIdx.x;
  const int c = blockIdx.y;
  const int f = blockIdx.z / ochunks;
  const int o0 = (blockIdx.z % ochunks) * kCombOut;
  if (r >= rows) return;
  const int no = min(kCombOut, mo - o0);
  double2 acc[kCombOut];
#pragma unroll
  for (int u = 0; u < kCombOut; ++u) acc[u] = make_double2(0.0, 0.0);
  const double2* base = in + (size_t)f * ifs + (size_t)c * ics + r;
  for (int i = 0; i < mi; ++i) {
    const int b = src ? __ldg(src + i) : i;
    const double2 v = base[(int64_t)b * ibs];
#pragma unroll
    for (int u = 0; u < kCombOut; ++u) {
      if (u < no) {
        const double2 w = __ldg(W + (size_t)(o0 + u) * mi + i);
        acc[u].x = fma(w.x, v.x, fma(-w.y, v.y, acc[u].x));
        acc[u].y = fma(w.x, v.y, fma(w.y, v.x, acc[u].y));
      }
    }
  }
  double2* ob = out + (size_t)f * ofs + (size_t)c * ocs + r;
#pragma unroll
  for (int u = 0; u < kCombOut; ++u)
    if (u < no) ob[(int64_t)(o0 + u) * obs] = acc[u];
}

}  // namespace
}  // namespace bem

extern "C" int bem_block_combine(const void* in_dev, int64_t in_fstride, int64_t in_bstride, int64_t in_cstride,
                                 void* out_dev, int64_t out_fstride, int64_t out_bstride, int64_t out_cstride,
                                 const void* weights_dev, const int32_t* source_dev, int mi, int mo, int rows, int cols,
                                 int nf, void* stream) {
  using namespace bem;
  if (rows < 0 || cols < 0 || nf < 0) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_block_combine: negative size");
  if (rows == 0 || cols == 0 || nf == 0) return BEM_OK;
  if (!in_dev || !out_dev || !weights_dev)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_block_combine: null pointer");
  if (mi < 1 || mo < 1) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_block_combine: no block");
  const int ochunks = ceil_div(mo, kCombOut);
  if (cols > 65535 || (int64_t)nf * ochunks > 65535)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_block_combine: more than 65535 columns or frequency chunks");
  if (in_cstride < rows || out_cstride < rows)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_block_combine: column stride smaller than the rows");
  dim3 grid(ceil_div(rows, kCombRows), cols, nf * ochunks);
  cudaStream_t s = (cudaStream_t)stream;
  block_combine_kernel<<<grid, kCombRows, 0, s>>>((const double2*)in_dev, in_fstride, in_bstride, in_cstride,
                                                  (double2*)out_dev, out_fstride, out_bstride, out_cstride,
                                                  (const double2*)weights_dev, (const int*)source_dev, mi, mo, rows,
                                                  ochunks);
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}
