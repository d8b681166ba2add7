// Batched blocked complex128 LU factorisation and triangular solves (sm_100a).
//
// Replaces the LAPACK zgetrf / zgetrs calls behind scipy.linalg.lu_factor /
// lu_solve in capytaine (tools/block_circulant_matrices.py:361-385, used by
// bem/engines.py:300-346).  Matrices are column-major complex128, one matrix per
// frequency, `batch` of them `stride` elements apart, each padded to a multiple
// of kNB = 64 with the identity on the padded diagonal.
//
// Factorisation (right-looking, one step per 64-column block):
//   1. diagonal block: LU in shared memory with partial pivoting among the rows
//      of the block (the permutation P is block diagonal, so P A = L U holds
//      exactly);
//   2. panels: the block row is permuted (left part included, as LAPACK's
//      zlaswp does) and solved with L11; the block column below is solved with
//      U11;
//   3. trailing update A22 -= A21 A12 with double-precision tensor-core MMAs
//      (mma.sync m8n8k4 f64), four real products per complex tile.
// Solves: diagonal blocks are inverted once; forward and backward block
// substitutions run as one persistent kernel each, block rows handed out in
// dependency order through an atomic ticket so that every wait targets a block
// row whose CTA is already running; waits are bounded and report a timeout.
#include <algorithm>
#include "common.cuh"

namespace bem {
namespace {

constexpr int kNB = 64;
constexpr int kLd = kNB + 1;  // shared-memory leading dimension of a 64x64 tile

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cfms(double2 acc, double2 a, double2 b) {  // acc - a*b
  return make_double2(acc.x - (a.x * b.x - a.y * b.y), acc.y - (a.x * b.y + a.y * b.x));
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }

// ---------------------------------------------------------------------------
// 1. Diagonal block factorisation.
__global__ void __launch_bounds__(256) zlu_diag_kernel(double2* __restrict__ A, int64_t lda, int64_t stride, int kk,
                                                       int* __restrict__ piv, int64_t piv_stride,
                                                       int* __restrict__ info) {
  extern __shared__ double2 sm[];
  double2* T = sm;  // T[c*kLd + r]
  __shared__ int perm[kNB];
  __shared__ int s_piv;
  const int b = blockIdx.x;
  double2* Ab = A + (size_t)b * stride;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) {
    const int r = idx % kNB, c = idx / kNB;
    T[c * kLd + r] = Ab[(size_t)(kk + r) + (size_t)(kk + c) * lda];
  }
  if (tid < kNB) perm[tid] = tid;
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5;
  for (int j = 0; j < kNB; ++j) {
    // pivot search among rows j..63 of column j (first maximum of |re|+|im|, as izamax)
    if (warp == 0) {
      double best = -1.0;
      int bi = j;
      for (int r = j + lane; r < kNB; r += 32) {
        const double v = cabs1(T[j * kLd + r]);
        if (v > best) {
          best = v;
          bi = r;
        }
      }
      for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (lane == 0) {
        s_piv = bi;
        if (!(best > 0.0) && info[b] == 0) info[b] = kk + j + 1;
      }
    }
    __syncthreads();
    const int p = s_piv;
    if (p != j) {
      if (tid < kNB) {
        const double2 t = T[tid * kLd + j];
        T[tid * kLd + j] = T[tid * kLd + p];
        T[tid * kLd + p] = t;
      }
      if (tid == 0) {
        const int t = perm[j];
        perm[j] = perm[p];
        perm[p] = t;
      }
    }
    __syncthreads();
    const double2 pivot = T[j * kLd + j];
    const bool ok = cabs1(pivot) > 0.0;
    if (ok) {
      for (int r = j + 1 + tid; r < kNB; r += blockDim.x) T[j * kLd + r] = cdiv(T[j * kLd + r], pivot);
    }
    __syncthreads();
    // rank-1 update: warp w takes columns j+1+w, j+1+w+8, ...
    for (int c = j + 1 + warp; c < kNB; c += 8) {
      const double2 tcj = T[c * kLd + j];
      for (int r = j + 1 + lane; r < kNB; r += 32) T[c * kLd + r] = cfms(T[c * kLd + r], T[j * kLd + r], tcj);
    }
    __syncthreads();
  }
  for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) {
    const int r = idx % kNB, c = idx / kNB;
    Ab[(size_t)(kk + r) + (size_t)(kk + c) * lda] = T[c * kLd + r];
  }
  if (tid < kNB) piv[(size_t)b * piv_stride + kk + tid] = perm[tid];
}

// ---------------------------------------------------------------------------
// 2. Panels.  blockIdx.x enumerates: [0, nleft) left tiles of the block row
// (permute only), [nleft, nleft+nright) right tiles (permute + L11 solve), then
// tiles below the diagonal block (U11 solve).
__global__ void __launch_bounds__(256) zlu_panel_kernel(double2* __restrict__ A, int64_t lda, int64_t stride, int n,
                                                        int kk, const int* __restrict__ piv, int64_t piv_stride) {
  extern __shared__ double2 sm[];
  double2* D = sm;              // factored diagonal block D[c*kLd + r]
  double2* X = sm + kNB * kLd;  // working tile X[c*kLd + r]
  __shared__ int perm[kNB];
  const int b = blockIdx.y;
  double2* Ab = A + (size_t)b * stride;
  const int tid = threadIdx.x;
  const int nleft = kk / kNB;
  const int nright = (n - kk - kNB) / kNB;
  const int t = blockIdx.x;
  int kind, c0 = 0, r0 = 0;
  if (t < nleft) {
    kind = 0;
    c0 = t * kNB;
  } else if (t < nleft + nright) {
    kind = 1;
    c0 = kk + kNB + (t - nleft) * kNB;
  } else {
    kind = 2;
    r0 = kk + kNB + (t - nleft - nright) * kNB;
  }
  if (tid < kNB) perm[tid] = piv[(size_t)b * piv_stride + kk + tid];
  if (kind != 0) {
    for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) {
      const int r = idx % kNB, c = idx / kNB;
      D[c * kLd + r] = Ab[(size_t)(kk + r) + (size_t)(kk + c) * lda];
    }
  }
  __syncthreads();
  if (kind <= 1) {
    // rows kk..kk+63, columns c0..c0+63, permuted
    for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) {
      const int r = idx % kNB, c = idx / kNB;
      X[c * kLd + r] = Ab[(size_t)(kk + perm[r]) + (size_t)(c0 + c) * lda];
    }
    __syncthreads();
    if (kind == 1) {
      // X <- L11^{-1} X, column sweep over the unit lower factor
      const int warp = tid >> 5, lane = tid & 31;
      for (int i = 0; i < kNB - 1; ++i) {
        for (int c = warp; c < kNB; c += 8) {
          const double2 xi = X[c * kLd + i];
          for (int r = i + 1 + lane; r < kNB; r += 32) X[c * kLd + r] = cfms(X[c * kLd + r], D[i * kLd + r], xi);
        }
        __syncthreads();
      }
    }
    for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) {
      const int r = idx % kNB, c = idx / kNB;
      Ab[(size_t)(kk + r) + (size_t)(c0 + c) * lda] = X[c * kLd + r];
    }
  } else {
    // rows r0..r0+63, columns kk..kk+63: X <- X U11^{-1}
    for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) {
      const int r = idx % kNB, c = idx / kNB;
      X[c * kLd + r] = Ab[(size_t)(r0 + r) + (size_t)(kk + c) * lda];
    }
    __syncthreads();
    const int rr = tid & (kNB - 1), cs = tid >> 6;  // 64 rows x 4 column phases
    for (int j = 0; j < kNB; ++j) {
      const double2 ujj = D[j * kLd + j];
      if (tid < kNB && cabs1(ujj) > 0.0) X[j * kLd + tid] = cdiv(X[j * kLd + tid], ujj);
      __syncthreads();
      const double2 xj = X[j * kLd + rr];
      for (int c = j + 1 + cs; c < kNB; c += 4) X[c * kLd + rr] = cfms(X[c * kLd + rr], xj, D[c * kLd + j]);
      __syncthreads();
    }
    for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) {
      const int r = idx % kNB, c = idx / kNB;
      Ab[(size_t)(r0 + r) + (size_t)(kk + c) * lda] = X[c * kLd + r];
    }
  }
}

// ---------------------------------------------------------------------------
// 3. Complex GEMM with double-precision tensor-core MMAs:
//    C[M x N] = beta*C + alpha * A[M x K] B[K x N]   (alpha, beta real)
// A, B, C column-major complex128.  Tile 64x64 per CTA (4 warps of 32x32),
// K in steps of 16.  M, N, K multiples of 64 / 16 are not required: edges are
// guarded.
constexpr int kBM = 64, kBN = 64, kBK = 16, kPadMN = 4;

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(128) zgemm_dmma_kernel(int M, int N, int K, double alpha, const double2* __restrict__ A,
                                                         int64_t lda, int64_t strideA, const double2* __restrict__ B,
                                                         int64_t ldb, int64_t strideB, double beta,
                                                         double2* __restrict__ C, int64_t ldc, int64_t strideC) {
  __shared__ double As[2][kBK][kBM + kPadMN];  // [re/im][k][m]
  __shared__ double Bs[2][kBK][kBN + kPadMN];  // [re/im][k][n]
  const int bz = blockIdx.z;
  A += (size_t)bz * strideA;
  B += (size_t)bz * strideB;
  C += (size_t)bz * strideC;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  double acc_re[4][4][2], acc_im[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      acc_re[i][j][0] = acc_re[i][j][1] = 0.0;
      acc_im[i][j][0] = acc_im[i][j][1] = 0.0;
    }
  const int qr = lane >> 2, qc = lane & 3;
  for (int k0 = 0; k0 < K; k0 += kBK) {
    // A tile: 64 (m) x 16 (k); thread loads m = tid % 64, k = tid / 64 + 2 i
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int m = tid & 63, k = (tid >> 6) + 2 * i;
      double2 v = make_double2(0.0, 0.0);
      if (m0 + m < M && k0 + k < K) v = A[(size_t)(m0 + m) + (size_t)(k0 + k) * lda];
      As[0][k][m] = v.x;
      As[1][k][m] = v.y;
    }
    // B tile: 16 (k) x 64 (n); thread loads k = tid % 16, n = tid / 16 + 8 i
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = tid & 15, nn = (tid >> 4) + 8 * i;
      double2 v = make_double2(0.0, 0.0);
      if (n0 + nn < N && k0 + k < K) v = B[(size_t)(k0 + k) + (size_t)(n0 + nn) * ldb];
      Bs[0][k][nn] = v.x;
      Bs[1][k][nn] = v.y;
    }
    __syncthreads();
#pragma unroll
    for (int kq = 0; kq < kBK; kq += 4) {
      double ar[4], ai[4], nai[4], br[4], bi[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        ar[i] = As[0][kq + qc][wm + 8 * i + qr];
        ai[i] = As[1][kq + qc][wm + 8 * i + qr];
        nai[i] = -ai[i];
        br[i] = Bs[0][kq + qc][wn + 8 * i + qr];
        bi[i] = Bs[1][kq + qc][wn + 8 * i + qr];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(acc_re[i][j][0], acc_re[i][j][1], ar[i], br[j]);
          dmma(acc_re[i][j][0], acc_re[i][j][1], nai[i], bi[j]);
          dmma(acc_im[i][j][0], acc_im[i][j][1], ar[i], bi[j]);
          dmma(acc_im[i][j][0], acc_im[i][j][1], ai[i], br[j]);
        }
    }
    __syncthreads();
  }
  // epilogue: fragment (row qr, columns 2 qc, 2 qc + 1) of each 8x8 sub-tile
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = m0 + wm + 8 * i + qr;
        const int nn = n0 + wn + 8 * j + 2 * qc + h;
        if (m < M && nn < N) {
          double2* p = C + (size_t)m + (size_t)nn * ldc;
          double2 c = (beta == 0.0) ? make_double2(0.0, 0.0) : *p;
          c.x = beta * c.x + alpha * acc_re[i][j][h];
          c.y = beta * c.y + alpha * acc_im[i][j][h];
          *p = c;
        }
      }
}

// ---------------------------------------------------------------------------
// Inverses of the diagonal blocks: L_ii^{-1} (unit lower) and U_ii^{-1}.
// Output layout: inv[(b * nblk + i) * 2 + {0: L, 1: U}] is a 64x64 column-major tile.
__global__ void __launch_bounds__(128) ztri_inv_kernel(const double2* __restrict__ A, int64_t lda, int64_t stride,
                                                       int nblk, double2* __restrict__ inv) {
  extern __shared__ double2 sm[];
  double2* D = sm;              // factored block
  double2* W = sm + kNB * kLd;  // inverse being built, W[c*kLd + r]
  const int i = blockIdx.x, b = blockIdx.y;
  const double2* Ab = A + (size_t)b * stride;
  const int kk = i * kNB;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) {
    const int r = idx % kNB, c = idx / kNB;
    D[c * kLd + r] = Ab[(size_t)(kk + r) + (size_t)(kk + c) * lda];
  }
  __syncthreads();
  double2* out = inv + ((size_t)b * nblk + i) * 2 * kNB * kNB;
  // L^{-1}: thread c solves L x = e_c (forward substitution), column c of the inverse.
  if (tid < kNB) {
    const int c = tid;
    for (int r = 0; r < kNB; ++r) {
      double2 v = make_double2(r == c ? 1.0 : 0.0, 0.0);
      for (int m = c; m < r; ++m) v = cfms(v, D[m * kLd + r], W[c * kLd + m]);
      W[c * kLd + r] = (r < c) ? make_double2(0.0, 0.0) : v;
    }
  }
  __syncthreads();
  for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) out[idx] = W[(idx / kNB) * kLd + idx % kNB];
  __syncthreads();
  // U^{-1}: thread c solves U x = e_c (backward substitution).
  if (tid < kNB) {
    const int c = tid;
    for (int r = kNB - 1; r >= 0; --r) {
      double2 v = make_double2(r == c ? 1.0 : 0.0, 0.0);
      if (r > c) {
        W[c * kLd + r] = make_double2(0.0, 0.0);
        continue;
      }
      for (int m = r + 1; m <= c; ++m) v = cfms(v, D[m * kLd + r], W[c * kLd + m]);
      const double2 d = D[r * kLd + r];
      W[c * kLd + r] = (cabs1(d) > 0.0) ? cdiv(v, d) : make_double2(0.0, 0.0);
    }
  }
  __syncthreads();
  for (int idx = tid; idx < kNB * kNB; idx += blockDim.x)
    out[kNB * kNB + idx] = W[(idx / kNB) * kLd + idx % kNB];
}

// ---------------------------------------------------------------------------
// Persistent block substitution.  forward: y = L^{-1} P b; backward: x = U^{-1} y.
// B: (n, nrhs) column-major per matrix, in place.  flags: batch*nblk ints, zero
// on entry; ticket: one int, zero on entry; err: set to 1 when a wait times out.
constexpr long long kSpinLimit = 4000000;  // x ~64 ns sleeps ~ a quarter second

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

constexpr int kTrsmRhs = 16;             // right-hand sides per launch
constexpr int kLdR = kTrsmRhs + 1;

__global__ void __launch_bounds__(256) ztrsm_persistent_kernel(const double2* __restrict__ A, int64_t lda,
                                                               int64_t stride, int nblk, int batch,
                                                               const int* __restrict__ piv, int64_t piv_stride,
                                                               const double2* __restrict__ inv, double2* B,
                                                               int64_t ldb, int64_t strideB, int nrhs, int forward,
                                                               int* flags, int* ticket, int* err, const int* skip,
                                                               long long spin_limit, const int* mskip) {
  if (skip && *skip) return;  // refinement already converged
  extern __shared__ double2 sm[];
  double2* Inv = sm;                 // inverse of the diagonal block, Inv[m*kLd + r]
  double2* L = Inv + kNB * kLd;      // off-diagonal block A[i-block, j-block], L[m*kLd + r]
  double2* X = L + kNB * kLd;        // own block, X[r*kLdR + c]
  double2* Y = X + kNB * kLdR;       // dependency block, Y[m*kLdR + c]
  __shared__ int s_t;
  const int tid = threadIdx.x;
  if (tid == 0) s_t = atomicAdd(ticket, 1);
  __syncthreads();
  const int t = s_t;
  const int b = t % batch;
  if (mskip && mskip[b]) return;  // converged matrix: every CTA of it returns, no wait targets it
  const int step = t / batch;
  const int i = forward ? step : (nblk - 1 - step);
  const double2* Ab = A + (size_t)b * stride;
  double2* Bb = B + (size_t)b * strideB;
  const int r0 = i * kNB;
  const double2* invg = inv + ((size_t)b * nblk + i) * 2 * kNB * kNB + (forward ? 0 : kNB * kNB);
  // Prefetch the inverse of the diagonal block and the own right-hand sides
  // (permuted rows for the forward sweep); neither depends on other block rows.
  for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) Inv[(idx / kNB) * kLd + idx % kNB] = invg[idx];
  for (int idx = tid; idx < kNB * nrhs; idx += blockDim.x) {
    const int r = idx % kNB, c = idx / kNB;
    const int src = forward ? piv[(size_t)b * piv_stride + r0 + r] : r;
    X[r * kLdR + c] = __ldcg(Bb + (size_t)(r0 + src) + (size_t)c * ldb);
  }
  // Dependencies in the order they complete: 0..i-1 forward, nblk-1..i+1 backward.
  const int ndep = forward ? i : (nblk - 1 - i);
  for (int q = 0; q < ndep; ++q) {
    const int j = forward ? q : (nblk - 1 - q);
    // the off-diagonal block does not depend on the flag: load it first
    const double2* src = Ab + (size_t)r0 + (size_t)(j * kNB) * lda;
    for (int idx = tid; idx < kNB * kNB; idx += blockDim.x) {
      const int r = idx % kNB, m = idx / kNB;
      L[m * kLd + r] = src[(size_t)r + (size_t)m * lda];
    }
    if (tid == 0) {
      long long it = 0;
      while (ld_acquire(flags + (size_t)b * nblk + j) == 0) {
        if (++it > spin_limit) {
          atomicExch(err, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __syncthreads();
    for (int idx = tid; idx < kNB * nrhs; idx += blockDim.x) {
      const int m = idx % kNB, c = idx / kNB;
      Y[m * kLdR + c] = __ldcg(Bb + (size_t)(j * kNB + m) + (size_t)c * ldb);
    }
    __syncthreads();
    for (int idx = tid; idx < kNB * nrhs; idx += blockDim.x) {
      const int r = idx % kNB, c = idx / kNB;
      double2 acc = X[r * kLdR + c];
#pragma unroll 16
      for (int m = 0; m < kNB; ++m) acc = cfms(acc, L[m * kLd + r], Y[m * kLdR + c]);
      X[r * kLdR + c] = acc;
    }
    __syncthreads();
  }
  __syncthreads();
  double2 res[4];  // kNB * kTrsmRhs / blockDim.x
  int cnt = 0;
  for (int idx = tid; idx < kNB * nrhs; idx += blockDim.x) {
    const int r = idx % kNB, c = idx / kNB;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll 16
    for (int m = 0; m < kNB; ++m) {
      const double2 a = Inv[m * kLd + r];
      const double2 x = X[m * kLdR + c];
      acc.x += a.x * x.x - a.y * x.y;
      acc.y += a.x * x.y + a.y * x.x;
    }
    res[cnt++] = acc;
  }
  cnt = 0;
  for (int idx = tid; idx < kNB * nrhs; idx += blockDim.x) {
    const int r = idx % kNB, c = idx / kNB;
    Bb[(size_t)(r0 + r) + (size_t)c * ldb] = res[cnt++];
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) st_release(flags + (size_t)b * nblk + i, 1);
}

__global__ void pad_identity_kernel(double2* A, int64_t lda, int64_t stride, int n, int npad) {
  // zero the padded rows/columns and put ones on the padded diagonal
  const int b = blockIdx.y;
  double2* Ab = A + (size_t)b * stride;
  const long long total = (long long)npad * (npad - n) * 2;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long half = (long long)npad * (npad - n);
    long long e = idx < half ? idx : idx - half;
    int r, c;
    if (idx < half) {  // padded columns
      r = (int)(e % npad);
      c = n + (int)(e / npad);
    } else {  // padded rows of the first n columns... and all columns
      r = n + (int)(e % (npad - n));
      c = (int)(e / (npad - n));
    }
    Ab[(size_t)r + (size_t)c * lda] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
}

}  // namespace
}  // namespace bem

using namespace bem;

namespace {
int check_lu_args(const void* A, int n, int64_t lda, int batch) {
  if (!A) return set_error(BEM_ERR_INVALID_ARGUMENT, "null matrix pointer");
  if (n <= 0 || n % kNB != 0) return set_error(BEM_ERR_INVALID_ARGUMENT, "n must be a positive multiple of 64");
  if (lda < n) return set_error(BEM_ERR_INVALID_ARGUMENT, "lda < n");
  if (batch <= 0) return set_error(BEM_ERR_INVALID_ARGUMENT, "batch <= 0");
  return BEM_OK;
}
bool g_smem_configured = false;
int configure_smem() {
  if (g_smem_configured) return BEM_OK;
  const int big = 2 * kNB * kLd * (int)sizeof(double2);
  BEM_CUDA_CHECK(cudaFuncSetAttribute(zlu_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  BEM_CUDA_CHECK(cudaFuncSetAttribute(zlu_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  BEM_CUDA_CHECK(cudaFuncSetAttribute(ztri_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  const int trsm = (2 * kNB * kLd + 2 * kNB * kLdR) * (int)sizeof(double2);
  BEM_CUDA_CHECK(cudaFuncSetAttribute(ztrsm_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, trsm));
  g_smem_configured = true;
  return BEM_OK;
}
}  // namespace

extern "C" int bem_zpad_identity(void* A_dev, int64_t lda, int64_t stride, int batch, int n, int npad, void* stream) {
  if (!A_dev || n < 0 || npad < n || lda < npad || batch <= 0)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zpad_identity: bad arguments");
  if (npad == n) return BEM_OK;
  dim3 grid(256, batch);
  pad_identity_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>((double2*)A_dev, lda, stride, n, npad);
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}

extern "C" int bem_zgemm(int M, int N, int K, double alpha, const void* A_dev, int64_t lda, int64_t strideA,
                         const void* B_dev, int64_t ldb, int64_t strideB, double beta, void* C_dev, int64_t ldc,
                         int64_t strideC, int batch, void* stream) {
  if (M < 0 || N < 0 || K < 0 || batch <= 0) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zgemm: bad sizes");
  if (M == 0 || N == 0) return BEM_OK;
  if (!A_dev || !B_dev || !C_dev) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zgemm: null pointer");
  dim3 grid(ceil_div(M, kBM), ceil_div(N, kBN), batch);
  zgemm_dmma_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(M, N, K, alpha, (const double2*)A_dev, lda, strideA,
                                                            (const double2*)B_dev, ldb, strideB, beta,
                                                            (double2*)C_dev, ldc, strideC);
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}

extern "C" int64_t bem_zlu_workspace_bytes(int n, int batch) {
  const int nblk = n / kNB;
  // inverses, block-row flags, then ticket, refinement flag and per-matrix convergence flags
  return (int64_t)batch * nblk * 2 * kNB * kNB * (int64_t)sizeof(double2) + (int64_t)batch * nblk * 4 +
         (int64_t)batch * 4 + 256;
}

extern "C" int bem_zlu_factor(void* A_dev, int n, int64_t lda, int64_t stride, int batch, int* piv_dev,
                              int* info_dev, void* work_dev, void* stream) {
  int st = check_lu_args(A_dev, n, lda, batch);
  if (st) return st;
  if (!piv_dev || !info_dev || !work_dev) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zlu_factor: null pointer");
  if ((st = configure_smem())) return st;
  cudaStream_t s = (cudaStream_t)stream;
  double2* A = (double2*)A_dev;
  const int smem = 2 * kNB * kLd * (int)sizeof(double2);
  BEM_CUDA_CHECK(cudaMemsetAsync(info_dev, 0, sizeof(int) * batch, s));
  for (int kk = 0; kk < n; kk += kNB) {
    {
      TimedLaunch tl(kKZluDiag, s);
      zlu_diag_kernel<<<batch, 256, kNB * kLd * sizeof(double2), s>>>(A, lda, stride, kk, piv_dev, n, info_dev);
    }
    count_launches(1);
    const int nleft = kk / kNB, nrest = (n - kk - kNB) / kNB;
    const int ntiles = nleft + 2 * nrest;
    if (ntiles > 0) {
      TimedLaunch tl(kKZluPanel, s);
      zlu_panel_kernel<<<dim3(ntiles, batch), 256, smem, s>>>(A, lda, stride, n, kk, piv_dev, n);
      count_launches(1);
    }
    if (nrest > 0) {
      const int m = n - kk - kNB;
      dim3 grid(ceil_div(m, kBM), ceil_div(m, kBN), batch);
      TimedLaunch tl(kKZgemmDmma, s);
      zgemm_dmma_kernel<<<grid, 128, 0, s>>>(m, m, kNB, -1.0, A + (size_t)(kk + kNB) + (size_t)kk * lda, lda, stride,
                                             A + (size_t)kk + (size_t)(kk + kNB) * lda, lda, stride, 1.0,
                                             A + (size_t)(kk + kNB) + (size_t)(kk + kNB) * lda, lda, stride);
      count_launches(1);
    }
  }
  // diagonal block inverses for the solves
  const int nblk = n / kNB;
  ztri_inv_kernel<<<dim3(nblk, batch), 128, smem, s>>>(A, lda, stride, nblk, (double2*)work_dev);
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}

namespace bem {
// Address of the "converged" flag of a refinement with these factors: an int
// in the workspace tail after the block-row flags and the ticket.
int* zlu_done_flag(void* work_dev, int n, int batch) {
  const int nblk = n / kNB;
  int* flags = (int*)((char*)work_dev + (size_t)batch * nblk * 2 * kNB * kNB * sizeof(double2));
  return flags + (size_t)batch * nblk + 1;
}

// Forward and backward block substitutions with the float64 factors, in place
// on B; every launch returns at once while *skip != 0.
int zlu_solve_enqueue(const void* A_dev, int n, int64_t lda, int64_t stride, int batch, const int* piv_dev,
                      const void* work_dev, void* B_dev, int64_t ldb, int64_t strideB, int nrhs, int* err_dev,
                      cudaStream_t s, const int* skip, long long spin_limit, const int* mskip) {
  int st = configure_smem();
  if (st) return st;
  const int nblk = n / kNB;
  const double2* inv = (const double2*)work_dev;
  int* flags = (int*)((char*)work_dev + (size_t)batch * nblk * 2 * kNB * kNB * sizeof(double2));
  int* ticket = flags + (size_t)batch * nblk;
  const int smem = (2 * kNB * kLd + 2 * kNB * kLdR) * (int)sizeof(double2);
  for (int c0 = 0; c0 < nrhs; c0 += kTrsmRhs) {
    const int nc = std::min(kTrsmRhs, nrhs - c0);
    double2* Bc = (double2*)B_dev + (size_t)c0 * ldb;
    for (int forward = 1; forward >= 0; --forward) {
      BEM_CUDA_CHECK(cudaMemsetAsync(flags, 0, sizeof(int) * ((size_t)batch * nblk + 1), s));
      TimedLaunch tl(kKZtrsm, s);
      ztrsm_persistent_kernel<<<nblk * batch, 256, smem, s>>>((const double2*)A_dev, lda, stride, nblk, batch,
                                                             piv_dev, n, inv, Bc, ldb, strideB, nc, forward, flags,
                                                             ticket, err_dev, skip, spin_limit, mskip);
      count_launches(1);
    }
  }
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}
}  // namespace bem

extern "C" int bem_zlu_solve(const void* A_dev, int n, int64_t lda, int64_t stride, int batch, const int* piv_dev,
                             const void* work_dev, void* B_dev, int64_t ldb, int64_t strideB, int nrhs,
                             int* err_dev, void* stream) {
  int st = check_lu_args(A_dev, n, lda, batch);
  if (st) return st;
  if (!piv_dev || !work_dev || !B_dev || !err_dev) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zlu_solve: null");
  if (nrhs <= 0 || nrhs > kNB) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zlu_solve: nrhs must be in [1, 64]");
  if (ldb < n) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_zlu_solve: ldb < n");
  return zlu_solve_enqueue(A_dev, n, lda, stride, batch, piv_dev, work_dev, B_dev, ldb, strideB, nrhs, err_dev,
                           (cudaStream_t)stream, nullptr, kSpinLimit);
}

