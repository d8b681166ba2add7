// Mixed-precision complex LU with float64-residual iterative refinement.
//
// Replaces the complex128 zgetrf/zgetrs solve of capytaine
// (tools/block_circulant_matrices.py:361-385, bem/engines.py:300-346) by:
//   * a float32 copy of K in two planes (real, imaginary), column-major, padded
//     to a multiple of 128 with the identity;
//   * a blocked right-looking block LU with 128-wide blocks, A = L U with L
//     unit block lower (L_ik = A_ik A_kk^{-1}) and U block upper (the updated
//     block rows): each diagonal block is inverted by Gauss-Jordan elimination
//     with partial pivoting among its rows, held in registers; the panel is the
//     product A21 A_kk^{-1}; the trailing update C -= L21 U12 runs on the
//     tcgen05 tensor cores (TF32 inputs, FP32 accumulation; tc_gemm.cu) from
//     packed operands (A12 and A21 by a pack kernel, L21 by the epilogue of
//     the panel product).  No row permutation leaves the diagonal blocks, so
//     the solves need none;
//   * block substitutions with these factors (persistent kernel); the block
//     rows of U are stored pre-multiplied by the diagonal inverses (U' =
//     A_kk^{-1} A12, computed beside the panel), so that the backward sweep
//     applies A_ii^{-1} to its own right-hand side before its dependencies;
//   * iterative refinement: x += LU^{-1} (b - K x) with the residual computed
//     in float64 against the float64 matrix until the relative residual of
//     every right-hand side is below the requested tolerance.
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <vector>
#include "common.cuh"

namespace bem {

namespace {

constexpr int kB = 128;        // LU block
constexpr int kPT = 64;        // panel tile width
constexpr int kSplitK = 6 * kB;  // K' of the split-TF32 panel product: (hi, lo, hi) x (re, im) x 128
constexpr int kRhs = 16;       // right-hand sides per solve launch
constexpr int kOpBuffers = 3;  // packed operands of the current, previous and next block steps

__device__ __forceinline__ float2 fmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float fabs1(float2 a) { return fabsf(a.x) + fabsf(a.y); }
// a b + c on a pair of floats in one instruction (fma.rn.f32x2: per element the
// correctly rounded fused multiply-add of fmaf)
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n.reg .b64 ra, rb, rc, rd;\n"
      "mov.b64 ra, {%2, %3};\nmov.b64 rb, {%4, %5};\nmov.b64 rc, {%6, %7};\n"
      "fma.rn.f32x2 rd, ra, rb, rc;\nmov.b64 {%0, %1}, rd;\n}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}

struct Planes {
  float* re;
  float* im;
  int64_t ld;      // = npad
  int64_t stride;  // floats between matrices (re and im planes of one matrix are plane apart)
};
// The part of x that TF32 keeps (the low 13 mantissa bits cleared); x - hi is
// exact in float32 and is the "lo" part of the split product.
__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xffffe000u); }

__device__ __forceinline__ float2 ldp(const Planes& W, int b, int r, int c) {
  const size_t o = (size_t)b * W.stride + (size_t)r + (size_t)c * W.ld;
  return make_float2(W.re[o], W.im[o]);
}
__device__ __forceinline__ void stp(const Planes& W, int b, int r, int c, float2 v) {
  const size_t o = (size_t)b * W.stride + (size_t)r + (size_t)c * W.ld;
  W.re[o] = v.x;
  W.im[o] = v.y;
}

// K (complex128, n x n, leading dimension ldk) -> planes (npad x npad) with the
// identity on the padding.
__global__ void convert_pad_kernel(const double2* __restrict__ K, int64_t ldk, int64_t strideK, int n, int npad,
                                   Planes W) {
  const int b = blockIdx.z;
  const int c = blockIdx.y;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < npad; r += gridDim.x * blockDim.x) {
    float2 v;
    if (r < n && c < n) {
      const double2 z = K[(size_t)b * strideK + (size_t)r + (size_t)c * ldk];
      v = make_float2((float)z.x, (float)z.y);
    } else {
      v = make_float2(r == c ? 1.0f : 0.0f, 0.0f);
    }
    stp(W, b, r, c, v);
  }
}

// Gauss-Jordan inverse of a diagonal block: 8 warps, thread (warp w, lane l)
// owns rows l + 32 a (a < 4) and columns w + 8 m (m < 16) of the 128 x 128
// block in registers; column j = 8 m + w is slot m of warp w.
// Pivoting is implicit: rows never move.  Step j picks the pivot of column j
// among the rows not yet used as pivot rows (row p_j) and eliminates column j
// from every other row with the unnormalised row p_j:
//   a_r -= (a_rj / a_pj) a_p   (r != p_j),
// the in-place inverse's column j ending as -a_rj / a_pj, with 1 in row p_j.
// Row p_j thus stays scaled by its pivot; at the end
//   A^{-1}(j', p_c) = a(p_j', c) / pivot_j'
// (row p_j' holds the j'-th pivot row, the slot of column c the inverse's
// column p_c).
#ifndef BEM_GJ_WARPS
#define BEM_GJ_WARPS 8
#endif
#ifndef BEM_GJ_DEPTH
#define BEM_GJ_DEPTH 4
#endif
constexpr int kGjWarps = BEM_GJ_WARPS;
constexpr int kGjSlots = kB / kGjWarps;  // columns per warp
constexpr int kGjDepth = BEM_GJ_DEPTH;   // pivot columns published ahead of the slowest warp
static_assert(kGjSlots <= 16 && kGjWarps * kGjSlots == kB, "a warp holds at most 16 columns of the block");
constexpr int kGjLd = kB + 1;            // column stride of the staged inverse (fewer bank conflicts)
constexpr int kGjOutBytes = kB * kGjLd * (int)sizeof(float2);  // dynamic shared memory of the inverse
constexpr long long kGjWaitLimit = 1ll << 22;  // polls of a bounded wait (about a second)

// acc - a b in two fused multiply-adds per component, in this order:
//   acc.x = fmaf(a.y, b.y, fmaf(-a.x, b.x, acc.x)),
//   acc.y = fmaf(-a.y, b.x, fmaf(-a.x, b.y, acc.y)),
// as two pair instructions: an = (-a.x, -a.x), ay = (a.y, -a.y) (once per
// multiplier), b and bs = (b.y, b.x) (once per pivot-row entry).
__device__ __forceinline__ float2 cfms2(float2 acc, float2 an, float2 ay, float2 b, float2 bs) {
  return fma2(ay, bs, fma2(an, b, acc));
}

__device__ __forceinline__ uint32_t gj_smem(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void gj_bar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(gj_smem(bar)), "r"(count));
}
__device__ __forceinline__ void gj_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(gj_smem(bar)) : "memory");
}
__device__ __forceinline__ bool gj_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(gj_smem(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

struct GjShared {
  // full[s]: the column of buffer s is published (32 arrivals, the owner's
  // lanes); empty[s]: every warp has read it (8 arrivals, one per warp).
  uint64_t full[kGjDepth];
  uint64_t empty[kGjDepth];
  float2 colbuf[kGjDepth][kB];      // pivot column of step j in buffer j % kGjDepth, by row
  alignas(16) float2 xbuf[kGjWarps][kGjSlots];  // per warp: its entries of the pivot row
  float2 rowscale[kB];              // 1 / pivot of the step whose pivot row is this row
  int piv_row[kB];                  // pivot row of each step
  int jinv[kB];                     // step of each pivot row
  unsigned used[kB / 32];           // rows already used as pivot rows
  int s_piv[kGjDepth];              // pivot row of the column in each buffer
  int abort;                        // a wait ran out: every warp leaves
};

// Bounded wait of a whole warp for phase `parity` of bar (every lane polls,
// so that every lane acquires the published data); false for the whole warp
// when a lane reached the limit or another warp gave up (the warp then leaves
// its loop, with no lane left behind in a warp-synchronous call).
__device__ __forceinline__ bool gj_wait(uint64_t* bar, uint32_t parity, GjShared& sh, int* __restrict__ err) {
  bool ok = false, gave_up = false;
  for (long long it = 0; it < kGjWaitLimit; ++it) {
    if (gj_try_wait(bar, parity)) {
      ok = true;
      break;
    }
    if (*(volatile int*)&sh.abort) {
      gave_up = true;
      break;
    }
  }
  if (!ok && !gave_up) {
    *(volatile int*)&sh.abort = 1;
    atomicExch(err, 1);
  }
  return __all_sync(0xffffffffu, ok);
}

// Column j (register slot M of this warp) after the update of step j - 1
// (multipliers f, pivot-row entry um; f = 0 for column 0): pivot among the
// unused rows, the column published to buffer j % kGjDepth with its pivot
// row; flags an exactly zero pivot in info.  Returns the pivot row (the slot
// becomes the unit vector of that row once the warp's own update of step
// j - 1 is done).
template <int M>
__device__ __forceinline__ int gj_publish(const float2 (&a)[4][kGjSlots], const float2 (&f)[4], float2 um, int j,
                                          int kk, int b, int lane, GjShared& sh, int* __restrict__ info) {
  constexpr int S = M < kGjSlots ? M : 0;  // M >= kGjSlots: a case the switch never takes
  float2 t[4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
    t[i] = cfms2(a[i][S], make_float2(-f[i].x, -f[i].x), make_float2(f[i].y, -f[i].y), um, make_float2(um.y, um.x));
  // this lane's candidate: the largest |t| among its unused rows (the first of
  // equal ones, the smallest row), as an ordered key (the bits of the
  // non-negative float plus one; 0: none, the used rows and NaN); then the
  // largest key of the warp and, among equal keys, the smallest row
  unsigned key = 0u;
  int li = kB;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float av = fabs1(t[i]);
    const unsigned kv = (((sh.used[i] >> lane) & 1u) || isnan(av)) ? 0u : __float_as_uint(av) + 1u;
    if (kv > key) {
      key = kv;
      li = lane + 32 * i;
    }
  }
  const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
  int bi = (int)__reduce_min_sync(0xffffffffu, key == kmax ? (unsigned)li : (unsigned)kB);
  const float best = kmax ? __uint_as_float(kmax - 1u) : -1.0f;
  if (bi >= kB) {  // no comparable candidate (NaN): the first unused row
#pragma unroll
    for (int i = 3; i >= 0; --i)
      if (~sh.used[i]) bi = 32 * i + __ffs(~sh.used[i]) - 1;
  }
  const int s = j % kGjDepth;
#pragma unroll
  for (int i = 0; i < 4; ++i) sh.colbuf[s][lane + 32 * i] = t[i];
  if (lane == 0) {
    sh.s_piv[s] = bi;
    sh.piv_row[j] = bi;
    sh.used[bi >> 5] |= 1u << (bi & 31);
    if (!(best > 0.0f) && info[b] == 0) info[b] = kk + j + 1;
  }
  gj_arrive(&sh.full[s]);  // release: this lane's writes above
  return bi;
}

template <int M>
__device__ __forceinline__ void gj_unit(float2 (&a)[4][kGjSlots], int bi, int lane) {
  constexpr int S = M < kGjSlots ? M : 0;  // M >= kGjSlots: a case the switch never takes
#pragma unroll
  for (int i = 0; i < 4; ++i) a[i][S] = make_float2(lane + 32 * i == bi ? 1.0f : 0.0f, 0.0f);
}

// Inverse of the diagonal block A_kk by Gauss-Jordan elimination with partial
// pivoting among its rows (implicit, see above), the block in registers.  The
// warps do not step together: the owner of column j + 1 updates that column
// first, picks its pivot and publishes it (shared-memory buffers guarded by
// mbarriers, kGjDepth columns deep) before its update of the other columns,
// so that the pivot search of the next column overlaps the rank-one updates
// of the other warps; every warp takes the pivot row's entries of its own
// columns from its own lanes.  The step body is one loop over the columns
// (register slots addressed through a switch only for the owner's column).
// Output: inv (128 x 128, column-major) = A_kk^{-1}, and its packed copies for
// the panel product (binv) and the block row of U' (ainv); info flags an
// exactly zero pivot; err is set when a bounded wait runs out.
__global__ void __launch_bounds__(32 * kGjWarps, 1) clu_gj_kernel(Planes W, int kk, int* __restrict__ info,
                                                                 float2* __restrict__ inv, int nblk,
                                                                 float* __restrict__ binv,
                                                                 float* __restrict__ ainv, int* __restrict__ err) {
  __shared__ GjShared sh;
  const int b = blockIdx.x, tid = threadIdx.x;
  const int lane = tid & 31, w = tid >> 5;
  float2 a[4][kGjSlots];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int m = 0; m < kGjSlots; ++m) a[i][m] = ldp(W, b, kk + lane + 32 * i, kk + w + kGjWarps * m);
  if (tid < kB / 32) sh.used[tid] = 0u;
  if (tid < kGjDepth) {
    gj_bar_init(&sh.full[tid], 32);
    gj_bar_init(&sh.empty[tid], kGjWarps);
  }
  if (tid == 0) sh.abort = 0;
  __syncthreads();
  float2 f[4];
  if (w == 0) {  // column 0: slot 0 of warp 0, nothing to update yet
#pragma unroll
    for (int i = 0; i < 4; ++i) f[i] = make_float2(0.0f, 0.0f);
    const int bi = gj_publish<0>(a, f, make_float2(0.0f, 0.0f), 0, kk, b, lane, sh, info);
    gj_unit<0>(a, bi, lane);
  }
  float2* xw = sh.xbuf[w];
#pragma unroll 1
  for (int j = 0; j < kB; ++j) {
    const int s = j % kGjDepth;
    if (!gj_wait(&sh.full[s], (j / kGjDepth) & 1, sh, err)) break;
    const int p = sh.s_piv[s];
    const int lp = p & 31, sp = p >> 5;
    if (lane == lp) {
      switch (sp) {  // one lane: a branch per register slot instead of selects
#define BEM_GJ_ROWOUT(S) \
  case S:                \
    _Pragma("unroll") for (int m = 0; m < kGjSlots; m += 2) \
      reinterpret_cast<float4*>(xw)[m / 2] = make_float4(a[S][m].x, a[S][m].y, a[S][m + 1].x, a[S][m + 1].y); \
    break;
        BEM_GJ_ROWOUT(0) BEM_GJ_ROWOUT(1) BEM_GJ_ROWOUT(2) BEM_GJ_ROWOUT(3)
#undef BEM_GJ_ROWOUT
      }
    }
    const float2 piv = sh.colbuf[s][p];
    const float d = piv.x * piv.x + piv.y * piv.y;
    const float rd = d > 0.0f ? __frcp_rn(d) : 0.0f;  // = 1.0f / d, correctly rounded
    const float2 dinv = make_float2(piv.x * rd, -piv.y * rd);
    if (tid == 0) sh.rowscale[p] = dinv;
    // multipliers a_rj / pivot; 0 on the pivot row, which stays as it is
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float2 c = sh.colbuf[s][lane + 32 * i];
      f[i] = (lane + 32 * i == p) ? make_float2(0.0f, 0.0f) : fmul(c, dinv);
    }
    __syncwarp();  // the pivot row is in the warp's buffer; the warp's reads of column j are done
    if (lane == 0) gj_arrive(&sh.empty[s]);
    const int nj = j + 1;
    const bool owner = nj < kB && w == (nj & (kGjWarps - 1));
    int bi = 0;
    if (owner) {
      // buffer nj % kGjDepth is free once every warp has read column nj - kGjDepth
      if (nj >= kGjDepth && !gj_wait(&sh.empty[nj % kGjDepth], ((nj / kGjDepth) - 1) & 1, sh, err)) break;
      switch (nj / kGjWarps) {
#define BEM_GJ_PUB(M) \
  case M:             \
    bi = gj_publish<M>(a, f, xw[M < kGjSlots ? M : 0], nj, kk, b, lane, sh, info); \
    break;
        BEM_GJ_PUB(0) BEM_GJ_PUB(1) BEM_GJ_PUB(2) BEM_GJ_PUB(3) BEM_GJ_PUB(4) BEM_GJ_PUB(5) BEM_GJ_PUB(6)
        BEM_GJ_PUB(7) BEM_GJ_PUB(8) BEM_GJ_PUB(9) BEM_GJ_PUB(10) BEM_GJ_PUB(11) BEM_GJ_PUB(12) BEM_GJ_PUB(13)
        BEM_GJ_PUB(14) BEM_GJ_PUB(15)
#undef BEM_GJ_PUB
      }
    }
    // rank-one update of every column of the warp: a - f u (u the pivot row,
    // read from the warp's buffer two entries per load)
    float4 u4[kGjSlots / 2];
#pragma unroll
    for (int m = 0; m < kGjSlots / 2; ++m) u4[m] = reinterpret_cast<const float4*>(xw)[m];
    float2 fn[4], fy[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      fn[i] = make_float2(-f[i].x, -f[i].x);
      fy[i] = make_float2(f[i].y, -f[i].y);
    }
#pragma unroll
    for (int m = 0; m < kGjSlots; ++m) {
      const float2 um = (m & 1) ? make_float2(u4[m / 2].z, u4[m / 2].w) : make_float2(u4[m / 2].x, u4[m / 2].y);
      const float2 us = make_float2(um.y, um.x);
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i][m] = cfms2(a[i][m], fn[i], fy[i], um, us);
    }
    if (owner) {
      switch (nj / kGjWarps) {
#define BEM_GJ_UNIT(M) \
  case M:              \
    gj_unit<M>(a, bi, lane); \
    break;
        BEM_GJ_UNIT(0) BEM_GJ_UNIT(1) BEM_GJ_UNIT(2) BEM_GJ_UNIT(3) BEM_GJ_UNIT(4) BEM_GJ_UNIT(5) BEM_GJ_UNIT(6)
        BEM_GJ_UNIT(7) BEM_GJ_UNIT(8) BEM_GJ_UNIT(9) BEM_GJ_UNIT(10) BEM_GJ_UNIT(11) BEM_GJ_UNIT(12)
        BEM_GJ_UNIT(13) BEM_GJ_UNIT(14) BEM_GJ_UNIT(15)
#undef BEM_GJ_UNIT
      }
    }
    __syncwarp();  // the warp's reads of its buffer are done before the next step rewrites it
  }
  __syncthreads();
  if (sh.abort) return;
  if (tid < kB) sh.jinv[sh.piv_row[tid]] = tid;
  __syncthreads();
  // A_kk^{-1}(jinv[r], piv_row[c]) = a(r, c) / pivot: staged in shared memory
  // at its place (column-major, column stride kGjLd), so that the three
  // outputs below are written with coalesced stores (the permuted rows would
  // scatter every store otherwise).
  extern __shared__ float2 gj_out[];  // kB columns of kGjLd
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = lane + 32 * i;
    const int row = sh.jinv[r];
    const float2 sc = sh.rowscale[r];
#pragma unroll
    for (int m = 0; m < kGjSlots; ++m)
      gj_out[(size_t)sh.piv_row[w + kGjWarps * m] * kGjLd + row] = fmul(a[i][m], sc);
  }
  __syncthreads();
  // inv: column-major 128 x 128
  float2* out = inv + ((size_t)b * nblk + kk / kB) * kB * kB;
  for (int idx = tid; idx < kB * kB; idx += blockDim.x) {
    const int row = idx & (kB - 1), col = idx >> 7;
    out[idx] = gj_out[col * kGjLd + row];
  }
  // the A operand of U' = A_kk^{-1} A12: row r = [Re A_kk^{-1}(r, :) | Im A_kk^{-1}(r, :)]
  float* ao = ainv + (size_t)b * kB * 2 * kB;
  for (int idx = tid; idx < kB * kB; idx += blockDim.x) {
    const int col = idx & (kB - 1), row = idx >> 7;
    const float2 v = gj_out[col * kGjLd + row];
    ao[(size_t)row * 2 * kB + col] = tf32_rn(v.x);
    ao[(size_t)row * 2 * kB + kB + col] = tf32_rn(v.y);
  }
  // the B operand of the split-TF32 product L21 = A21 A_kk^{-1} (three
  // K-blocks of 256: hi, hi, lo; see clu_pack_kernel for the A side):
  // row t: [Re X(:, t) | -Im X(:, t)] per block, row 128 + t: [Im X(:, t) | Re X(:, t)]
  float* bo = binv + (size_t)b * (2 * kB) * kSplitK;
  for (int idx = tid; idx < kB * kB; idx += blockDim.x) {
    const int row = idx & (kB - 1), col = idx >> 7;
    const float2 v = gj_out[col * kGjLd + row];
    const float2 hi = make_float2(tf32_hi(v.x), tf32_hi(v.y));
    const float2 lo = make_float2(v.x - hi.x, v.y - hi.y);
    float* rr = bo + (size_t)col * kSplitK + row;
    float* ri = bo + (size_t)(kB + col) * kSplitK + row;
    rr[0] = hi.x;
    rr[kB] = -hi.y;
    rr[2 * kB] = hi.x;
    rr[3 * kB] = -hi.y;
    rr[4 * kB] = lo.x;
    rr[5 * kB] = -lo.y;
    ri[0] = hi.y;
    ri[kB] = hi.x;
    ri[2 * kB] = hi.y;
    ri[3 * kB] = hi.x;
    ri[4 * kB] = lo.y;
    ri[5 * kB] = lo.x;
  }
}

// Operand packing of block step kk of the block LU (A_kk^{-1} comes packed
// from the Gauss-Jordan kernel, L21 from the epilogue of the panel product).
// Blocks [0, nrest): the block row to the right of the diagonal, 64 columns
// each, packed as the B operand (U12 = A12).  Blocks [nrest, nrest +
// nrows/32): 32 rows of the block column [col0, col0 + 128) from row row0 on,
// packed K-major into A3 as the split-TF32 operand of the panel product (A21).
// Both through shared memory, so that reads and writes are coalesced.
// Bop: [batch][2*npad][2*kB]; A3: [batch][npad][kSplitK].
__global__ void __launch_bounds__(256) clu_pack_kernel(Planes W, int npad, int kk, int nrest, int row0, int col0,
                                                       float* __restrict__ Bop, float* __restrict__ A3, int t0) {
  __shared__ float tre[kB][33], tim[kB][33];  // [column][row] of a 32 x 128 tile
  const int b = blockIdx.y, tid = threadIdx.x;
  const size_t kp = 2 * kB;
  const int t = blockIdx.x + t0;  // a launch may cover a range of the blocks only
  if (t < nrest) {
    // 128 x 64 of A12: B operand rows of the complex columns c0 .. c0+63;
    // thread (q, cc): rows 4 q .. 4 q + 3 of column cc (16-byte loads and stores)
    const int c0 = kk + kB + t * kPT;
    const int j0 = c0 & ~(kB - 1);
    float* Bb = Bop + (size_t)b * 2 * npad * kp;
    const float* re = W.re + (size_t)b * W.stride;
    const float* im = W.im + (size_t)b * W.stride;
    const int q = tid & 31;
    for (int c = tid >> 5; c < kPT; c += 8) {
      const size_t g = (size_t)(c0 + c) * W.ld + kk + 4 * q;
      float4 ur = *reinterpret_cast<const float4*>(re + g);
      float4 ui = *reinterpret_cast<const float4*>(im + g);
      ur = make_float4(tf32_rn(ur.x), tf32_rn(ur.y), tf32_rn(ur.z), tf32_rn(ur.w));  // TF32 operands
      ui = make_float4(tf32_rn(ui.x), tf32_rn(ui.y), tf32_rn(ui.z), tf32_rn(ui.w));
      const int jj = c0 - j0 + c;
      float4* rowR = reinterpret_cast<float4*>(Bb + (size_t)(2 * j0 + jj) * kp);
      float4* rowI = reinterpret_cast<float4*>(Bb + (size_t)(2 * j0 + kB + jj) * kp);
      rowR[q] = ur;
      rowR[kB / 4 + q] = make_float4(-ui.x, -ui.y, -ui.z, -ui.w);
      rowI[q] = ui;
      rowI[kB / 4 + q] = ur;
    }
    return;
  }
  const int r0 = row0 + (t - nrest) * 32;
  const float* re = W.re + (size_t)b * W.stride;
  const float* im = W.im + (size_t)b * W.stride;
  {
    // thread (q, c): rows 4 q .. 4 q + 3 of column c, 16-byte loads
    const int q = tid & 7;
    for (int c = tid >> 3; c < kB; c += 32) {
      const size_t g = (size_t)(col0 + c) * W.ld + r0 + 4 * q;
      const float4 vr = *reinterpret_cast<const float4*>(re + g);
      const float4 vi = *reinterpret_cast<const float4*>(im + g);
      tre[c][4 * q] = vr.x;
      tre[c][4 * q + 1] = vr.y;
      tre[c][4 * q + 2] = vr.z;
      tre[c][4 * q + 3] = vr.w;
      tim[c][4 * q] = vi.x;
      tim[c][4 * q + 1] = vi.y;
      tim[c][4 * q + 2] = vi.z;
      tim[c][4 * q + 3] = vi.w;
    }
  }
  __syncthreads();
  // split rows [hi | lo | hi], each [Re(128) | Im(128)], for the panel
  // product; thread (q, i0): entries 4 q .. 4 q + 3 of rows i0, i0 + 4, ...
  float* dst = A3 + (size_t)b * npad * kSplitK + (size_t)r0 * kSplitK;
  const int q = tid & 63;
  const float(*src)[33] = q < 32 ? tre : tim;
  const int cb = 4 * (q & 31);
  for (int i = tid >> 6; i < 32; i += 4) {
    float h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float x = src[cb + e][i];
      h[e] = tf32_hi(x);
      l[e] = x - h[e];
    }
    float4* row = reinterpret_cast<float4*>(dst + (size_t)i * kSplitK);
    row[q] = make_float4(h[0], h[1], h[2], h[3]);
    row[2 * kB / 4 + q] = make_float4(l[0], l[1], l[2], l[3]);
    row[4 * kB / 4 + q] = make_float4(h[0], h[1], h[2], h[3]);
  }
}

// 16-byte asynchronous global -> shared copy and its completion wait.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst))),
               "l"(gsrc)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ int ld_acquire_i(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_i(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// Persistent block substitution with the block LU factors; B complex128 in
// place.  Forward: y_i = b_i - sum_{j<i} L_ij y_j (unit block lower).  Backward:
// x_i = A_ii^{-1} y_i - sum_{j>i} U'_ij x_j with U'_ij = A_ii^{-1} U_ij stored in
// the factorisation, so each step of the dependency chain is one block product
// in both sweeps.  Each CTA owns one 128-row block.  The off-diagonal blocks
// of its dependencies stream through a ring of kRing shared-memory slots, a
// quarter block (32 columns, real and imaginary planes) per slot, copied
// asynchronously (16-byte pieces) kRing - 1 quarters ahead of the product, so
// the next blocks load while the current one is multiplied; only the
// right-hand side of a dependency waits for its flag.  Thread (r, h)
// accumulates row r over the half h of each quarter's columns for all NC
// columns (NC/2 16-byte broadcast reads of the right-hand sides); the halves
// meet in P at the end of each block.
// Ring sizes: 5 slots (188 KB with 8 right-hand sides, one CTA per SM) when
// every block row of the launch is resident at once; 2 slots (88 KB, two
// CTAs per SM) when the block rows fill more than one wave of SMs, where
// twice the resident CTAs hide more latency than a deeper ring.
constexpr int kRingDeep = 5, kRingShallow = 2;
constexpr int kQCols = 32;                   // columns of a quarter block
constexpr int kQFloats = 2 * kQCols * kB;    // one slot: [plane][column][row]

// acc += Re(A) y and acci += Im(A) y over the quarter's half h of columns for
// row r (two pair instructions per entry and right-hand side, y = (Re, Im));
// fold_rhs turns the two into the complex product A y.
template <int NC>
__device__ __forceinline__ void quarter_times_rhs(const float* __restrict__ Tre, const float* __restrict__ Tim,
                                                  const float2* __restrict__ Y, int r, int h,
                                                  float2 (&acc)[NC], float2 (&acci)[NC]) {
#pragma unroll 4
  for (int mm = 16 * h; mm < 16 * h + 16; ++mm) {
    const float ar = Tre[mm * kB + r], ai = Tim[mm * kB + r];
    const float2 ar2 = make_float2(ar, ar), ai2 = make_float2(ai, ai);
    const float4* y4 = reinterpret_cast<const float4*>(Y + mm * NC);
#pragma unroll
    for (int c2 = 0; c2 < NC / 2; ++c2) {
      const float4 y = y4[c2];
      const float2 y0 = make_float2(y.x, y.y), y1 = make_float2(y.z, y.w);
      acc[2 * c2] = fma2(ar2, y0, acc[2 * c2]);
      acci[2 * c2] = fma2(ai2, y0, acci[2 * c2]);
      acc[2 * c2 + 1] = fma2(ar2, y1, acc[2 * c2 + 1]);
      acci[2 * c2 + 1] = fma2(ai2, y1, acci[2 * c2 + 1]);
    }
  }
}
template <int NC>
__device__ __forceinline__ void fold_rhs(float2 (&acc)[NC], float2 (&acci)[NC]) {
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    acc[c] = make_float2(acc[c].x - acci[c].y, acc[c].y + acci[c].x);
    acci[c] = make_float2(0.0f, 0.0f);
  }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int NC, int kRing>
__global__ void __launch_bounds__(256, kRing == kRingShallow ? 2 : 1) ctrsm_persistent_kernel(Planes W, int nblk, int batch,
                                                               const float2* __restrict__ inv, double2* B,
                                                               int64_t ldb, int64_t strideB, int nrhs, int forward,
                                                               int* flags, int* ticket, int* err, const int* skip,
                                                               long long spin_limit, int withheld,
                                                               const int* mskip) {
  static_assert(kRing >= 2, "the ring keeps one quarter in flight beside the one multiplied");
  // quarters of the diagonal inverse staged at a time: all four, or two per
  // pass when the ring has fewer than four slots (a divisor of 4, never more
  // slots than the ring has)
  constexpr int kDiagPass = kRing >= 4 ? 4 : 2;
  static_assert(4 % kDiagPass == 0 && kDiagPass <= kRing, "diagonal staging must fit the ring");
  if (skip && *skip) return;  // refinement already converged
  extern __shared__ __align__(16) float fsmf[];
  float* ring = fsmf;                                                  // kRing slots of kQFloats
  float2* X = reinterpret_cast<float2*>(ring + kRing * kQFloats);      // X[r*NC + c]
  float2* Y = X + kB * NC;                                             // Y[m*NC + c]
  float2* P = Y + kB * NC;                                             // P[r*NC + c]
  __shared__ int s_t;
  const int tid = threadIdx.x;
  const int r = tid & (kB - 1), h = tid >> 7;
  if (tid == 0) s_t = atomicAdd(ticket, 1);
  __syncthreads();
  const int t = s_t;
  const int b = t % batch, step = t / batch;
  if (mskip && mskip[b]) return;  // converged matrix: every CTA of it returns, no wait targets it
  const int i = forward ? step : (nblk - 1 - step);
  double2* Bb = B + (size_t)b * strideB;
  const int r0 = i * kB;
  for (int idx = tid; idx < kB * NC; idx += blockDim.x) {
    const int rr = idx & (kB - 1), c = idx >> 7;
    float2 v = make_float2(0.0f, 0.0f);
    if (c < nrhs) {
      const double2 d = __ldcg(Bb + (size_t)(r0 + rr) + (size_t)c * ldb);
      v = make_float2((float)d.x, (float)d.y);
    }
    X[rr * NC + c] = v;
  }
  const int ndep = forward ? i : (nblk - 1 - i);
  const float* Wre = W.re + (size_t)b * W.stride;
  const float* Wim = W.im + (size_t)b * W.stride;
  float2 acc[NC], acci[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = acci[c] = make_float2(0.0f, 0.0f);
  if (!forward) {
    // x_i = A_ii^{-1} b_i - sum_j U'_ij x_j with U' = A_ii^{-1} U: the product
    // with the diagonal inverse comes first, off the chain of dependencies,
    // its four quarters staged kDiagPass at a time in the first slots
    const float2* Inv = inv + ((size_t)b * nblk + i) * kB * kB;
#pragma unroll 1
    for (int q0 = 0; q0 < 4; q0 += kDiagPass) {
      // columns [32 q0, 32 (q0 + kDiagPass)) of the inverse into slots 0 .. kDiagPass - 1
      for (int idx = tid; idx < kDiagPass * kQCols * kB; idx += blockDim.x) {
        const int col = q0 * kQCols + (idx >> 7), row = idx & (kB - 1);
        const float2 v = __ldg(Inv + (size_t)col * kB + row);  // element (row, col)
        float* slot = ring + (col / kQCols - q0) * kQFloats;
        slot[(col % kQCols) * kB + row] = v.x;
        slot[kQCols * kB + (col % kQCols) * kB + row] = v.y;
      }
      __syncthreads();
#pragma unroll 1
      for (int qq = q0; qq < q0 + kDiagPass; ++qq) {
        const float* slot = ring + (qq - q0) * kQFloats;
        quarter_times_rhs<NC>(slot, slot + kQCols * kB, X + qq * kQCols * NC, r, h, acc, acci);
      }
      __syncthreads();  // the slots are restaged by the next pass
    }
    fold_rhs<NC>(acc, acci);
    if (h == 1) {
#pragma unroll
      for (int c = 0; c < NC; ++c) P[r * NC + c] = acc[c];
    }
    __syncthreads();
    if (h == 0) {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float2 o = P[r * NC + c];
        X[r * NC + c] = make_float2(acc[c].x + o.x, acc[c].y + o.y);
      }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = make_float2(0.0f, 0.0f);
    __syncthreads();  // the slots are reused for the off-diagonal blocks
  }
  // quarter q of the dependencies (block q / 4, columns 32 (q % 4) ..) into
  // its ring slot: 32 columns x 128 rows per plane, 8 sixteen-byte pieces per
  // thread
  const int nq = 4 * ndep;
  auto issue = [&](int q) {
    const int jd = q >> 2, qq = q & 3;
    const int j = forward ? jd : (nblk - 1 - jd);
    float* slot = ring + (q % kRing) * kQFloats;
    for (int idx = tid; idx < kQCols * 32; idx += blockDim.x) {
      const int mm = idx >> 5, piece = idx & 31;
      const size_t g = (size_t)(r0 + piece * 4) + (size_t)(j * kB + qq * kQCols + mm) * W.ld;
      cp_async16(slot + mm * kB + piece * 4, Wre + g);
      cp_async16(slot + kQCols * kB + mm * kB + piece * 4, Wim + g);
    }
  };
#pragma unroll 1
  for (int q = 0; q < kRing - 1; ++q) {
    if (q < nq) issue(q);
    cp_async_commit();
  }
#pragma unroll 1
  for (int q = 0; q < nq; ++q) {
    const int jd = q >> 2, qq = q & 3;
    __syncthreads();  // every thread is done with the slot refilled below (and with Y, at a new block)
    if (qq == 0) {
      const int j = forward ? jd : (nblk - 1 - jd);
      if (tid == 0) {
        long long it = 0;
        while (ld_acquire_i(flags + (size_t)b * nblk + j) == 0) {
          if (++it > spin_limit) {
            atomicExch(err, 1);
            break;
          }
          __nanosleep(64);
        }
      }
      __syncthreads();
      for (int idx = tid; idx < kB * NC; idx += blockDim.x) {
        const int m = idx & (kB - 1), c = idx >> 7;
        float2 v = make_float2(0.0f, 0.0f);
        if (c < nrhs) {
          const double2 d = __ldcg(Bb + (size_t)(j * kB + m) + (size_t)c * ldb);
          v = make_float2((float)d.x, (float)d.y);
        }
        Y[m * NC + c] = v;
      }
    }
    if (q + kRing - 1 < nq) issue(q + kRing - 1);
    cp_async_commit();
    cp_async_wait_group<kRing - 1>();  // this thread's copies of quarter q have landed
    __syncthreads();                   // everyone's copies, and Y
    const float* slot = ring + (q % kRing) * kQFloats;
    quarter_times_rhs<NC>(slot, slot + kQCols * kB, Y + qq * kQCols * NC, r, h, acc, acci);
    if (qq == 3) {
      fold_rhs<NC>(acc, acci);
      if (h == 1) {
#pragma unroll
        for (int c = 0; c < NC; ++c) P[r * NC + c] = acc[c];
      }
      __syncthreads();
      if (h == 0) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const float2 o = P[r * NC + c];
          float2 x = X[r * NC + c];
          x.x -= acc[c].x + o.x;
          x.y -= acc[c].y + o.y;
          X[r * NC + c] = x;
        }
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[c] = make_float2(0.0f, 0.0f);
    }
  }
  cp_async_wait_all();
  // forward (unit block lower factor): y_i = X; backward: x_i = X
  __syncthreads();
  for (int idx = tid; idx < kB * NC; idx += blockDim.x) {
    const int rr = idx & (kB - 1), c = idx >> 7;
    if (c < nrhs) {
      const float2 v = X[rr * NC + c];
      Bb[(size_t)(r0 + rr) + (size_t)c * ldb] = make_double2((double)v.x, (double)v.y);
    }
  }
  __threadfence();
  __syncthreads();
  // withheld >= 0 only from the bounded-wait test entry point: that block row
  // never publishes its flag, so the waits on it run out
  if (tid == 0 && i != withheld) st_release_i(flags + (size_t)b * nblk + i, 1);
}

constexpr int trsm_smem_bytes(int nc, int ring) { return ring * kQFloats * (int)sizeof(float) + 3 * kB * nc * (int)sizeof(float2); }

// x += r (the correction solved in place in r), then r = b for the residual.
__global__ void ir_update_kernel(double2* __restrict__ X, double2* __restrict__ R, const double2* __restrict__ Bv,
                                 int n, int nrhs, int64_t ld, int64_t stride, const int* skip, const int* mskip) {
  if (skip && *skip) return;
  const int b = blockIdx.z, c = blockIdx.y;
  if (mskip && mskip[b]) return;  // this matrix has converged
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const size_t o = (size_t)b * stride + (size_t)c * ld + r;
    const double2 x = X[o], d = R[o];
    X[o] = make_double2(x.x + d.x, x.y + d.y);
    R[o] = Bv[o];
  }
}

// Squared norms of columns: out[(b*nrhs + c)] = sum |V(:, c)|^2 over n rows.
__global__ void colnorm2_kernel(const double2* __restrict__ V, int n, int64_t ld, int64_t stride,
                                double* __restrict__ out, const int* skip, const int* mskip) {
  if (skip && *skip) return;
  const int c = blockIdx.x, b = blockIdx.y, nrhs = gridDim.x;
  if (mskip && mskip[b]) return;
  const double2* v = V + (size_t)b * stride + (size_t)c * ld;
  double s = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) s += v[r].x * v[r].x + v[r].y * v[r].y;
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[(size_t)b * nrhs + c] = red[0];
}

// Convergence test of one refinement iteration on the device: relative
// residual sqrt(|r_v|^2 / |b_v|^2) (absolute where b_v = 0) of every column,
// per matrix the worst of its nrhs columns: a matrix whose worst is <= tol is
// marked converged in mdone (the next iterations skip its work); *done when
// every matrix has converged (the iterations enqueued after return at once).
// state: [worst over all matrices, iterations].
__global__ void refine_check_kernel(const double* __restrict__ bn, const double* __restrict__ rn, int nrhs,
                                    int batch, double tol, int* done, double* state, int* mdone) {
  if (*done) return;
  __shared__ double red[32];
  __shared__ int all_done;
  if (threadIdx.x == 0) all_done = 1;
  __syncthreads();
  double worst = 0.0;
  for (int b = threadIdx.x; b < batch; b += blockDim.x) {
    double wb = 0.0;
    for (int c = 0; c < nrhs; ++c) {
      const int v = b * nrhs + c;
      wb = fmax(wb, bn[v] > 0.0 ? sqrt(rn[v] / bn[v]) : sqrt(rn[v]));
    }
    if (wb <= tol) mdone[b] = 1;
    else all_done = 0;  // benign race: every writer writes 0
    worst = fmax(worst, wb);
  }
  for (int off = 16; off > 0; off >>= 1) worst = fmax(worst, __shfl_xor_sync(0xffffffffu, worst, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = worst;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) worst = fmax(worst, red[w]);
    state[0] = worst;
    state[1] += 1.0;
    if (all_done) *done = 1;
  }
}

bool g_mixed_configured = false;
int configure_mixed() {
  if (g_mixed_configured) return BEM_OK;
  BEM_CUDA_CHECK(cudaFuncSetAttribute(clu_gj_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGjOutBytes));
  BEM_CUDA_CHECK(cudaFuncSetAttribute(ctrsm_persistent_kernel<8, kRingDeep>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, trsm_smem_bytes(8, kRingDeep)));
  BEM_CUDA_CHECK(cudaFuncSetAttribute(ctrsm_persistent_kernel<16, kRingDeep>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, trsm_smem_bytes(16, kRingDeep)));
  BEM_CUDA_CHECK(cudaFuncSetAttribute(ctrsm_persistent_kernel<8, kRingShallow>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, trsm_smem_bytes(8, kRingShallow)));
  BEM_CUDA_CHECK(cudaFuncSetAttribute(ctrsm_persistent_kernel<16, kRingShallow>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      trsm_smem_bytes(16, kRingShallow)));
  g_mixed_configured = true;
  return BEM_OK;
}

// Streaming multiprocessors of the current device (cached per device).
int sm_count(int* out) {
  static int counts[64] = {0};
  int dev = 0;
  BEM_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(BEM_ERR_UNSUPPORTED, "device index out of range");
  if (!counts[dev]) BEM_CUDA_CHECK(cudaDeviceGetAttribute(&counts[dev], cudaDevAttrMultiProcessorCount, dev));
  *out = counts[dev];
  return BEM_OK;
}

// Workspace layout (bytes): [planes 2*npad^2 floats][Aop npad*2kB floats][Bop 2*npad*2kB floats]
// [diagonal inverses nblk*kB*kB float2][flags batch*nblk + 1 ints], each per matrix except flags.
struct MixedWork {
  float* W;
  float* Aop;
  float* Bop;
  float2* inv;
  float* binv;  // batch x 256 x kSplitK: packed A_kk^{-1} of the current block
  float* a3;    // batch x npad x kSplitK: split A21 of the current block
  float* ainv;  // 2 x batch x 128 x 256: A_kk^{-1} of the last two blocks as the A operand [Re | Im]
  int* flags;
};
MixedWork carve(void* work, int npad, int batch) {
  char* p = (char*)work;
  const int nblk = npad / kB;
  MixedWork w;
  w.W = (float*)p;
  p += (size_t)batch * 2 * npad * npad * sizeof(float);
  w.Aop = (float*)p;  // three buffers of batch x npad x 256
  p += kOpBuffers * (size_t)batch * npad * 2 * kB * sizeof(float);
  w.Bop = (float*)p;  // three buffers of batch x 2 npad x 256
  p += kOpBuffers * (size_t)batch * 2 * npad * 2 * kB * sizeof(float);
  w.inv = (float2*)p;
  p += (size_t)batch * nblk * kB * kB * sizeof(float2);
  w.binv = (float*)p;
  p += (size_t)batch * (2 * kB) * kSplitK * sizeof(float);
  w.a3 = (float*)p;
  p += (size_t)batch * npad * kSplitK * sizeof(float);
  w.ainv = (float*)p;
  p += 2 * (size_t)batch * kB * 2 * kB * sizeof(float);
  w.flags = (int*)p;
  return w;
}
Planes planes_of(const MixedWork& w, int npad) {
  return Planes{w.W, w.W + (size_t)npad * npad, npad, 2 * (int64_t)npad * npad};
}

// Streams and events of the lookahead in the block LU, one set per (device,
// caller stream): factorisations enqueued on different streams (concurrent
// requests of a server) overlap on the device without sharing a side stream.
// `side` (highest priority) runs the chain of the next block (inverse,
// panel), `upper` (lowest priority) the block rows of U' that only the solves
// need.  The mutex is held
// while a factorisation is enqueued, so the events are never re-recorded by
// another caller in between.
struct Lookahead {
  std::mutex mu;
  cudaStream_t side = nullptr;
  cudaStream_t upper = nullptr;
  cudaEvent_t diag = nullptr;
  cudaEvent_t strips = nullptr;
  cudaEvent_t colpack = nullptr;
  cudaEvent_t panel = nullptr;
  cudaEvent_t upper_done[2] = {nullptr, nullptr};
};
std::mutex g_lookahead_mu;
std::map<std::pair<int, cudaStream_t>, std::unique_ptr<Lookahead>> g_lookahead;
int lookahead_for(cudaStream_t caller, Lookahead** out) {
  int dev = 0;
  BEM_CUDA_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_lookahead_mu);
  std::unique_ptr<Lookahead>& la = g_lookahead[std::make_pair(dev, caller)];
  if (!la) {
    auto fresh = std::make_unique<Lookahead>();
    int least = 0, greatest = 0;
    BEM_CUDA_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    BEM_CUDA_CHECK(cudaStreamCreateWithPriority(&fresh->side, cudaStreamNonBlocking, greatest));
    BEM_CUDA_CHECK(cudaStreamCreateWithPriority(&fresh->upper, cudaStreamNonBlocking, least));
    BEM_CUDA_CHECK(cudaEventCreateWithFlags(&fresh->diag, cudaEventDisableTiming));
    BEM_CUDA_CHECK(cudaEventCreateWithFlags(&fresh->strips, cudaEventDisableTiming));
    BEM_CUDA_CHECK(cudaEventCreateWithFlags(&fresh->colpack, cudaEventDisableTiming));
    BEM_CUDA_CHECK(cudaEventCreateWithFlags(&fresh->panel, cudaEventDisableTiming));
    for (auto& e : fresh->upper_done) BEM_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    la = std::move(fresh);
  }
  *out = la.get();
  return BEM_OK;
}

}  // namespace
}  // namespace bem

using namespace bem;

extern "C" int64_t bem_clu_workspace_bytes(int npad, int batch) {
  if (npad <= 0 || npad % kB || batch <= 0) return -1;
  const int64_t nblk = npad / kB;
  return (int64_t)batch * 2 * npad * (int64_t)npad * 4 + kOpBuffers * (int64_t)batch * npad * 2 * kB * 4 +
         kOpBuffers * (int64_t)batch * 2 * npad * 2 * kB * 4 + (int64_t)batch * nblk * kB * kB * 8 +
         (int64_t)batch * (2 * kB) * kSplitK * 4 + (int64_t)batch * npad * kSplitK * 4 +
         2 * (int64_t)batch * kB * 2 * kB * 4 +
         ((int64_t)batch * nblk + 2 + batch) * 4 + 1024;
}

namespace bem {
namespace {
int clu_factor_impl(const void* K_dev, int64_t ldk, int64_t strideK, int n, int npad, int batch, const int* act,
                    int* piv_dev, int* info_dev, void* work_dev, int* err_dev, void* stream,
                    bool planes_ready = false);

// Identity on the padding of planes that already hold K (rows or columns n ..
// npad - 1), the counterpart of convert_pad_kernel when the assembly wrote
// the float32 planes itself.
// One warp per column (blockDim 32 x 8): columns below n only have their
// rows n .. npad - 1 written, the columns from n on all of theirs.
__global__ void pad_planes_kernel(int n, int npad, Planes W) {
  const int b = blockIdx.y, c = blockIdx.x * blockDim.y + threadIdx.y;
  if (c >= npad) return;
  for (int r = (c < n ? n : 0) + threadIdx.x; r < npad; r += blockDim.x)
    stp(W, b, r, c, make_float2(r == c ? 1.0f : 0.0f, 0.0f));
}
}  // namespace

int clu_planes(void* work_dev, int npad, float** re, int64_t* ld, int64_t* stride, int64_t* im) {
  if (!work_dev || npad <= 0 || npad % kB || (reinterpret_cast<uintptr_t>(work_dev) & 1023))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "mixed LU workspace: npad a multiple of 128, 1024-byte alignment");
  // the planes come first in the workspace (carve)
  *re = reinterpret_cast<float*>(work_dev);
  *ld = npad;
  *stride = 2 * (int64_t)npad * npad;
  *im = (int64_t)npad * npad;
  return BEM_OK;
}
}  // namespace bem

extern "C" int bem_clu_factor_planes(int n, int npad, int batch, int* piv_dev, int* info_dev, void* work_dev,
                                     int* err_dev, void* stream) {
  return clu_factor_impl(nullptr, n, (int64_t)n * n, n, npad, batch, nullptr, piv_dev, info_dev, work_dev, err_dev,
                         stream, true);
}

extern "C" int bem_clu_factor(const void* K_dev, int64_t ldk, int64_t strideK, int n, int npad, int batch,
                              int* piv_dev, int* info_dev, void* work_dev, int* err_dev, void* stream) {
  return clu_factor_impl(K_dev, ldk, strideK, n, npad, batch, nullptr, piv_dev, info_dev, work_dev, err_dev, stream);
}

extern "C" int bem_clu_factor_grouped(const void* K_dev, int64_t ldk, int64_t strideK, int n, int npad, int batch,
                                      const int* active_host, int* piv_dev, int* info_dev, void* work_dev,
                                      int* err_dev, void* stream) {
  if (!active_host) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_clu_factor_grouped: null active sizes");
  for (int b = 0; b < batch; ++b)
    if (active_host[b] <= 0 || active_host[b] % kB || active_host[b] > npad)
      return set_error(BEM_ERR_INVALID_ARGUMENT,
                       "bem_clu_factor_grouped: active sizes must be multiples of 128 in (0, npad]");
  return clu_factor_impl(K_dev, ldk, strideK, n, npad, batch, active_host, piv_dev, info_dev, work_dev, err_dev,
                         stream);
}

namespace bem {
namespace {
int clu_factor_impl(const void* K_dev, int64_t ldk, int64_t strideK, int n, int npad, int batch, const int* act,
                    int* piv_dev, int* info_dev, void* work_dev, int* err_dev, void* stream, bool planes_ready) {
  if ((!K_dev && !planes_ready) || !piv_dev || !info_dev || !work_dev || !err_dev || n <= 0 || npad < n ||
      npad % kB || batch <= 0 || ldk < n)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_clu_factor: bad arguments (npad multiple of 128, >= n)");
  if (reinterpret_cast<uintptr_t>(work_dev) & 1023)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_clu_factor: workspace must be 1024-byte aligned");
  int st = configure_mixed();
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  MixedWork w = carve(work_dev, npad, batch);
  Planes W = planes_of(w, npad);
  const int nblk = npad / kB;
  int launches = 0;
  BEM_CUDA_CHECK(cudaMemsetAsync(info_dev, 0, sizeof(int) * batch, s));
  if (planes_ready) {  // K is in the planes already: the identity padding only
    if (npad > n)
      pad_planes_kernel<<<dim3(ceil_div(npad, 8), batch), dim3(32, 8), 0, s>>>(n, npad, W);
  } else {
    convert_pad_kernel<<<dim3(ceil_div(npad, 256), npad, batch), 256, 0, s>>>((const double2*)K_dev, ldk, strideK,
                                                                             n, npad, W);
  }
  ++launches;
  const size_t abuf = (size_t)batch * npad * 2 * kB, bbuf = (size_t)batch * 2 * npad * 2 * kB;
  // The updates and the panel product give each CTA an even share of up to
  // 32 tiles (the accumulator double buffer pays over a run; the runs end at
  // staggered times, so an SM frees up every few microseconds); U' (low
  // priority, off the chain) one tile per CTA, so that it never holds SMs
  // the chain needs for long.
  constexpr int kBigRun = 0, kSideRun = 1;
  float* Aop[kOpBuffers] = {w.Aop, w.Aop + abuf, w.Aop + 2 * abuf};
  float* Bop[kOpBuffers] = {w.Bop, w.Bop + bbuf, w.Bop + 2 * bbuf};
  const size_t ainv_buf = (size_t)batch * kB * 2 * kB;
  const int64_t a_stride = (int64_t)npad * 2 * kB;
  // Inverse of diagonal block kk (its A operand copy in ainv buffer of the
  // block's parity).
  auto inverse = [&](int kk, cudaStream_t on) {
    TimedLaunch tl(kKCluGj, on);
    clu_gj_kernel<<<batch, 32 * kGjWarps, kGjOutBytes, on>>>(W, kk, info_dev, w.inv, nblk, w.binv,
                                         w.ainv + ((kk / kB) & 1) * ainv_buf, err_dev);
    ++launches;
  };
  // L21 = A21 A_kk^{-1} (split TF32: A_hi B_hi + A_lo B_hi + A_hi B_lo,
  // float32-level multipliers) into the working matrix and, packed, into the
  // A operand buffer of the block.
  auto panel = [&](int kk, int buf, cudaStream_t on) -> int {
    const int m = npad - kk - kB;
    if (m <= 0) return BEM_OK;
    TimedLaunch tl(kKCluPanel, on);
    return cgemm_tf32_update(w.a3, npad, kk + kB, w.binv, 2 * kB, 0, kSplitK, W.re, W.im, npad, W.stride, kk + kB,
                             kk, m, kB, batch, err_dev, on, 1, nullptr, nullptr, kBigRun, 0, act, Aop[buf],
                             kPackRows, a_stride);
  };
  // Block row of U scaled by the diagonal inverse, U' = A_kk^{-1} A12 (TF32),
  // for the backward substitution only (A12 itself is packed in Bop).
  auto upper = [&](int kk, int buf, cudaStream_t on) -> int {
    const int m = npad - kk - kB;
    if (m <= 0) return BEM_OK;
    TimedLaunch tl(kKCluPanel, on);
    return cgemm_tf32_update(w.ainv + ((kk / kB) & 1) * ainv_buf, kB, 0, Bop[buf], 2 * (int64_t)npad,
                             2 * (kk + kB), 2 * kB, W.re, W.im, npad, W.stride, kk, kk + kB, kB, m, batch, err_dev,
                             on, 1, nullptr, nullptr, kSideRun, 0, act);
  };
  // C rows r0.. (m), complex columns c0.. (nc) -= L21 U12 of the block step whose
  // packed operands are in buffer buf, and of a second step (buffer buf2 >= 0)
  // in the same pass over C (depth 256); optionally a packed copy of the result.
  auto update = [&](int buf, int r0, int c0, int m, int nc, int buf2, int run, bool lshape = false,
                    int reserve = 0) -> int {
    if (m <= 0 || nc <= 0) return BEM_OK;
    return cgemm_tf32_update(Aop[buf], npad, r0, Bop[buf], 2 * (int64_t)npad, 2 * c0, 2 * kB, W.re, W.im, npad,
                             W.stride, r0, c0, m, nc, batch, err_dev, s, 0, buf2 >= 0 ? Aop[buf2] : nullptr,
                             buf2 >= 0 ? Bop[buf2] : nullptr, run, 0, act, nullptr, kPackNone, 0, lshape, reserve);
  };
  Lookahead* la = nullptr;
  if ((st = lookahead_for(s, &la))) return st;
  std::lock_guard<std::mutex> lock(la->mu);
  // Right-looking block LU with a lookahead of one block, the trailing updates
  // of two consecutive block steps applied in one pass over C (depth 256: the
  // update is bound by reading and writing C).  Step k, on the caller's
  // stream: the diagonal block k+1 gets every update still pending on it and
  // its inverse starts on the side stream; then block row and block column
  // k+1 get theirs (one L-shaped launch) and are packed as the operands of
  // step k+1 (A12 as the B operand, A21 split for the panel product) while
  // the inverse runs; the panel L21 follows on the side stream (its epilogue
  // packs the A operand), U' on the third stream.  Meanwhile, at every
  // second step, the rest of the trailing matrix gets the updates of steps
  // k-1 and k together.
  // Operands of steps k-1, k, k+1 live in three buffers; A_kk^{-1} for U' in
  // two.
  // Block 0: the operands come straight from the converted matrix.
  inverse(0, s);
  if (npad > kB) {
    const int m = npad - kB;
    TimedLaunch tl(kKCluPanel, s);
    clu_pack_kernel<<<dim3(m / kPT + m / 32, batch), 256, 0, s>>>(W, npad, 0, m / kPT, kB, 0, Bop[0], w.a3, 0);
    ++launches;
  }
  if ((st = panel(0, 0, s))) return st;
  BEM_CUDA_CHECK(cudaEventRecord(la->panel, s));
  BEM_CUDA_CHECK(cudaStreamWaitEvent(la->upper, la->panel, 0));
  if ((st = upper(0, 0, la->upper))) return st;
  BEM_CUDA_CHECK(cudaEventRecord(la->upper_done[0], la->upper));
  for (int kk = 0, step = 0; kk + kB < npad; kk += kB, ++step) {
    const int cur = step % kOpBuffers, prev = (step + kOpBuffers - 1) % kOpBuffers;
    const int nxt = (step + 1) % kOpBuffers;
    const int kn = kk + kB, rest = npad - kn - kB;
    const int pend = (step & 1) ? prev : -1;  // step k-1 still pending beyond block k
    // U' of block k-1 (third stream) has read the A_kk^{-1} copy that the
    // inverse of block k+1 overwrites (and, before it, U' of block k-2 the
    // operand buffer that the strips below overwrite)
    BEM_CUDA_CHECK(cudaStreamWaitEvent(s, la->upper_done[(step + 1) & 1], 0));
    if ((st = update(cur, kn, kn, kB, kB, pend, kSideRun))) return st;  // diagonal block kn
    BEM_CUDA_CHECK(cudaEventRecord(la->diag, s));
    BEM_CUDA_CHECK(cudaStreamWaitEvent(la->side, la->diag, 0));
    inverse(kn, la->side);
    // block row kn and block column kn below the diagonal (one L-shaped
    // launch), then their packed copies (A12 as the B operand, A21 split for
    // the panel product), beside the inverse.  (Packing behind the inverse on
    // the side stream at the steps with a big update, so that the big update
    // starts right after the strips, measured slower: the pack then shares
    // the SMs and HBM with the big update.)
    const bool big_step = (step & 1) && rest > 0;
    if (rest > 0) {
      // the inverse of block kn holds one SM per matrix meanwhile
      if ((st = update(cur, kn, kn, rest + kB, rest + kB, pend, 0, true, batch))) return st;
      // the block column's split copy first: the panel product starts on it
      // while the block row is packed as the next step's B operand
      TimedLaunch tl(kKCluPanel, s);
      clu_pack_kernel<<<dim3(rest / 32, batch), 256, 0, s>>>(W, npad, kn, rest / kPT, kn + kB, kn, Bop[nxt], w.a3,
                                                            rest / kPT);
      BEM_CUDA_CHECK(cudaEventRecord(la->colpack, s));
      clu_pack_kernel<<<dim3(rest / kPT, batch), 256, 0, s>>>(W, npad, kn, rest / kPT, kn + kB, kn, Bop[nxt], w.a3,
                                                             0);
      launches += 2;
    } else {
      BEM_CUDA_CHECK(cudaEventRecord(la->colpack, s));
    }
    BEM_CUDA_CHECK(cudaEventRecord(la->strips, s));
    BEM_CUDA_CHECK(cudaStreamWaitEvent(la->side, la->colpack, 0));
    if ((st = panel(kn, nxt, la->side))) return st;
    BEM_CUDA_CHECK(cudaEventRecord(la->panel, la->side));
    // U' reads the block row's B operand and the inverse
    BEM_CUDA_CHECK(cudaStreamWaitEvent(la->upper, la->strips, 0));
    BEM_CUDA_CHECK(cudaStreamWaitEvent(la->upper, la->panel, 0));
    if ((st = upper(kn, nxt, la->upper))) return st;
    BEM_CUDA_CHECK(cudaEventRecord(la->upper_done[(step + 1) & 1], la->upper));
    if (big_step) {
      if ((st = update(cur, kn + kB, kn + kB, rest, rest, prev, kBigRun))) return st;
    }
    BEM_CUDA_CHECK(cudaStreamWaitEvent(s, la->panel, 0));
  }
  // the last block rows of U' are part of the factors
  BEM_CUDA_CHECK(cudaEventRecord(la->upper_done[0], la->upper));
  BEM_CUDA_CHECK(cudaStreamWaitEvent(s, la->upper_done[0], 0));
  count_launches(launches);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}
}  // namespace
}  // namespace bem

namespace bem {
// Forward and backward block substitution with the float32 factors, in place on
// B (npad x nrhs complex128 per matrix); returns at once while *skip != 0.  Also
// the preconditioner of the GMRES solver.
int clu_solve_enqueue(void* work_dev, int npad, int batch, void* B_dev, int64_t ldb, int64_t strideB, int nrhs,
                      int* err_dev, cudaStream_t s, const int* skip, long long spin_limit, int withheld,
                      const int* mskip) {
  int st = configure_mixed();
  if (st) return st;
  MixedWork w = carve(work_dev, npad, batch);
  Planes W = planes_of(w, npad);
  const int nblk = npad / kB;
  int* ticket = w.flags + (size_t)batch * nblk;
  int launches = 0;
  int sms = 0;
  if ((st = sm_count(&sms))) return st;
  // more block rows than SMs: two CTAs per SM with the shallow ring
  const bool shallow = (long long)nblk * batch > sms;
  for (int c0 = 0; c0 < nrhs; c0 += kRhs) {
    const int nc = std::min(kRhs, nrhs - c0);
    double2* Bc = (double2*)B_dev + (size_t)c0 * ldb;
    for (int forward = 1; forward >= 0; --forward) {
      BEM_CUDA_CHECK(cudaMemsetAsync(w.flags, 0, sizeof(int) * ((size_t)batch * nblk + 1), s));
      TimedLaunch tl(kKCtrsm, s);
#define BEM_CTRSM(NC, R)                                                                                \
  ctrsm_persistent_kernel<NC, R><<<nblk * batch, 256, trsm_smem_bytes(NC, R), s>>>(                     \
      W, nblk, batch, w.inv, Bc, ldb, strideB, nc, forward, w.flags, ticket, err_dev, skip, spin_limit, \
      withheld, mskip)
      if (nc <= 8) {
        if (shallow) BEM_CTRSM(8, kRingShallow); else BEM_CTRSM(8, kRingDeep);
      } else {
        if (shallow) BEM_CTRSM(16, kRingShallow); else BEM_CTRSM(16, kRingDeep);
      }
#undef BEM_CTRSM
      ++launches;
    }
  }
  count_launches(launches);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}
}  // namespace bem

extern "C" int bem_clu_solve(void* work_dev, int npad, int batch, const int* piv_dev, void* B_dev, int64_t ldb,
                             int64_t strideB, int nrhs, int* err_dev, void* stream) {
  if (!work_dev || !piv_dev || !B_dev || !err_dev || npad <= 0 || npad % kB || batch <= 0 || nrhs <= 0 ||
      ldb < npad)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_clu_solve: bad arguments");
  return clu_solve_enqueue(work_dev, npad, batch, B_dev, ldb, strideB, nrhs, err_dev, (cudaStream_t)stream,
                           nullptr);
}

extern "C" int bem_clu_solve_bounded(void* work_dev, int npad, int batch, const int* piv_dev, void* B_dev,
                                     int64_t ldb, int64_t strideB, int nrhs, long long spin_limit, int withheld_block,
                                     int* err_dev, void* stream) {
  if (!work_dev || !piv_dev || !B_dev || !err_dev || npad <= 0 || npad % kB || batch <= 0 || nrhs <= 0 ||
      ldb < npad || spin_limit <= 0 || withheld_block < -1 || withheld_block >= npad / kB)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_clu_solve_bounded: bad arguments");
  return clu_solve_enqueue(work_dev, npad, batch, B_dev, ldb, strideB, nrhs, err_dev, (cudaStream_t)stream,
                           nullptr, spin_limit, withheld_block);
}

extern "C" int bem_zgemm_ts(int M, int K, int nrhs, double alpha_re, double alpha_im, const void* A_dev, int64_t lda,
                            int64_t strideA, const void* X_dev, int64_t ldx, int64_t strideX, double beta_re,
                            double beta_im, void* Y_dev, int64_t ldy, int64_t strideY, int batch, void* work_dev,
                            void* stream);

namespace bem {
// Iterative refinement x += F^{-1} (b - K x) with the residual in float64
// against the float64 K, where F^{-1} is `solve_in_place` (the float32 block
// LU of the mixed engine, or the float64 block LU itself, whose pivoting stays
// inside the diagonal blocks: the residual test then checks, and the
// iteration repairs, what that pivoting loses).  x = 0, r = b to start; per
// iteration: r <- F^{-1} r, x += r, r = b - K x, worst relative residual per
// column, convergence flag on the device.  `done` is an int of the solver's
// workspace; norms_dev holds 2 batch nrhs + 2 doubles.
template <class Solve>
int refine_loop(Solve solve_in_place, int* done, int* mdone, const void* K_dev, int64_t ldk, int64_t strideK, int n,
                int npad,
                int batch, const void* B_dev, void* X_dev, void* R_dev, int64_t ldb, int64_t strideB, int nrhs,
                double tol, int max_iter, void* ts_work_dev, double* norms_dev, int* iters_out, double* resid_out,
                cudaStream_t s) {
  const int nvec = batch * nrhs;
  double* bn = norms_dev;
  double* rn = norms_dev + nvec;
  double* state = norms_dev + 2 * nvec;  // [worst, iterations]
  int launches = 1;
  // |b|^2 per column; x = 0, r = b, not converged
  colnorm2_kernel<<<dim3(nrhs, batch), 256, 0, s>>>((const double2*)B_dev, n, ldb, strideB, bn, nullptr,
                                                    nullptr);
  // Only the nrhs columns of each matrix: the caller may interleave other
  // columns (a wider right-hand-side block solved in chunks) between them.
  for (int b = 0; b < batch; ++b) {
    const size_t o = (size_t)b * strideB;
    BEM_CUDA_CHECK(cudaMemset2DAsync((double2*)X_dev + o, ldb * sizeof(double2), 0, npad * sizeof(double2), nrhs, s));
    BEM_CUDA_CHECK(cudaMemcpy2DAsync((double2*)R_dev + o, ldb * sizeof(double2), (const double2*)B_dev + o,
                                     ldb * sizeof(double2), npad * sizeof(double2), nrhs, cudaMemcpyDeviceToDevice,
                                     s));
  }
  BEM_CUDA_CHECK(cudaMemsetAsync(done, 0, sizeof(int), s));
  BEM_CUDA_CHECK(cudaMemsetAsync(mdone, 0, sizeof(int) * batch, s));
  BEM_CUDA_CHECK(cudaMemsetAsync(state, 0, 2 * sizeof(double), s));
  // Iterations are enqueued in groups without host synchronisation; once the
  // device-side test has converged the rest of the group returns at once.
  constexpr int kGroup = 4;
  double host_state[2] = {0.0, 0.0};
  int enqueued = 0;
  while (enqueued < max_iter) {
    const int group = std::min(kGroup, max_iter - enqueued);
    for (int g = 0; g < group; ++g) {
      // r <- F^{-1} r in place (the padded rows of r stay zero)
      int st = solve_in_place(R_dev, (const int*)done, (const int*)mdone);
      if (st) return st;
      // x += r ; r = b ; r -= K x (float64); matrices already converged skip all of it
      ir_update_kernel<<<dim3(ceil_div(n, 256), nrhs, batch), 256, 0, s>>>(
          (double2*)X_dev, (double2*)R_dev, (const double2*)B_dev, n, nrhs, ldb, strideB, done, mdone);
      st = zgemm_ts_enqueue(n, n, nrhs, -1.0, 0.0, K_dev, ldk, strideK, X_dev, ldb, strideB, 1.0, 0.0, R_dev, ldb,
                            strideB, batch, ts_work_dev, s, done, mdone);
      if (st) return st;
      colnorm2_kernel<<<dim3(nrhs, batch), 256, 0, s>>>((const double2*)R_dev, n, ldb, strideB, rn, done, mdone);
      refine_check_kernel<<<1, 256, 0, s>>>(bn, rn, nrhs, batch, tol, done, state, mdone);
      launches += 3;
    }
    enqueued += group;
    const double before = host_state[0];
    BEM_CUDA_CHECK(cudaMemcpyAsync(host_state, state, sizeof(host_state), cudaMemcpyDeviceToHost, s));
    BEM_CUDA_CHECK(cudaStreamSynchronize(s));
    if (host_state[0] <= tol && host_state[1] > 0.0) break;
    // A contracting iteration gains far more than a factor 2 per group; one
    // that does not (the factors too far from K, e.g. near an irregular
    // frequency) stops here and reports non-convergence.
    if (enqueued > group && !(host_state[0] < 0.5 * before)) break;
  }
  count_launches(launches);
  *iters_out = (int)host_state[1];
  *resid_out = host_state[0];
  BEM_CUDA_CHECK(cudaGetLastError());
  if (!(host_state[0] <= tol)) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "iterative refinement stopped at relative residual %.3e after %d iterations",
                  host_state[0], (int)host_state[1]);
    return set_error(BEM_ERR_NOT_CONVERGED, msg);
  }
  return BEM_OK;
}
}  // namespace bem

extern "C" int bem_refine_solve(const void* K_dev, int64_t ldk, int64_t strideK, int n, int npad, int batch,
                                void* work_dev, const int* piv_dev, const void* B_dev, void* X_dev, void* R_dev,
                                int64_t ldb, int64_t strideB, int nrhs, double tol, int max_iter, void* ts_work_dev,
                                double* norms_dev, int* err_dev, int* iters_out, double* resid_out, void* stream) {
  if (!K_dev || !work_dev || !piv_dev || !B_dev || !X_dev || !R_dev || !ts_work_dev || !norms_dev || !err_dev ||
      !iters_out || !resid_out || nrhs <= 0 || nrhs > 16 || max_iter <= 0 || ldb < npad || npad % kB || n > npad ||
      batch <= 0)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_refine_solve: bad arguments (nrhs <= 16)");
  cudaStream_t s = (cudaStream_t)stream;
  MixedWork w = carve(work_dev, npad, batch);
  int* done = w.flags + (size_t)batch * (npad / kB) + 1;
  int* mdone = done + 1;  // batch ints (bem_clu_workspace_bytes counts them)
  auto solve = [&](void* R, const int* skip, const int* mskip) {
    return clu_solve_enqueue(work_dev, npad, batch, R, ldb, strideB, nrhs, err_dev, s, skip, kDefaultSpinLimit, -1,
                             mskip);
  };
  return refine_loop(solve, done, mdone, K_dev, ldk, strideK, n, npad, batch, B_dev, X_dev, R_dev, ldb, strideB, nrhs, tol,
                     max_iter, ts_work_dev, norms_dev, iters_out, resid_out, s);
}

extern "C" int bem_zlu_refine_solve(const void* K_dev, int64_t ldk, int64_t strideK, int n, const void* LU_dev,
                                    int npad, int64_t ldlu, int64_t strideLU, int batch, const int* piv_dev,
                                    void* lu_work_dev, const void* B_dev, void* X_dev, void* R_dev, int64_t ldb,
                                    int64_t strideB, int nrhs, double tol, int max_iter, void* ts_work_dev,
                                    double* norms_dev, int* err_dev, int* iters_out, double* resid_out,
                                    void* stream) {
  if (!K_dev || !LU_dev || !lu_work_dev || !piv_dev || !B_dev || !X_dev || !R_dev || !ts_work_dev || !norms_dev ||
      !err_dev || !iters_out || !resid_out || nrhs <= 0 || nrhs > 16 || max_iter <= 0 || npad <= 0 || npad % 64 ||
      n > npad || n <= 0 || ldk < n || ldlu < npad || ldb < npad || batch <= 0)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zlu_refine_solve: bad arguments (nrhs <= 16, npad % 64 == 0)");
  cudaStream_t s = (cudaStream_t)stream;
  int* done = zlu_done_flag(lu_work_dev, npad, batch);
  int* mdone = done + 1;  // batch ints (bem_zlu_workspace_bytes counts them)
  auto solve = [&](void* R, const int* skip, const int* mskip) {
    return zlu_solve_enqueue(LU_dev, npad, ldlu, strideLU, batch, piv_dev, lu_work_dev, R, ldb, strideB, nrhs,
                             err_dev, s, skip, kDefaultSpinLimit, mskip);
  };
  return refine_loop(solve, done, mdone, K_dev, ldk, strideK, n, npad, batch, B_dev, X_dev, R_dev, ldb, strideB, nrhs, tol,
                     max_iter, ts_work_dev, norms_dev, iters_out, resid_out, s);
}
