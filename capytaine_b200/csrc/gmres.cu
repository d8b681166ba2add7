// Restarted GMRES for the dense complex128 BEM systems, batched over matrices and
// right-hand sides, optionally right-preconditioned by the float32 block LU.
//
// Without a preconditioner this is the iteration of scipy.sparse.linalg.gmres
// (SciPy 1.18 `_isolve/iterative.py`) as capytaine calls it in solve_gmres
// (capytaine bem/engines.py:74-89: x0 = 0, restart 20, tolerance
// max(atol, rtol |b|)): modified Gram-Schmidt Arnoldi, complex Givens
// rotations, back substitution of the Hessenberg system at the end of each
// restart cycle, the true residual b - A x checked after each cycle and the
// inner tolerance adapted as SciPy does (gh-8400 rule).  With the float32 LU
// factors of bem_clu_factor as M^-1 it is flexible GMRES (Saad, "A flexible
// inner-outer preconditioned GMRES algorithm", SIAM J. Sci. Comput. 14, 1993):
// each preconditioned vector z_k = M^-1 v_k is kept and the cycle ends with
// x += Z y, so that A Z = V H holds for the vectors actually formed.  The
// float32 substitutions make M^-1 slightly nonlinear (their rounding depends on
// the vector), which matters when K is close to singular near an irregular
// frequency: |M^-1| then reaches 1e5-1e6 and a second application M^-1 (V y)
// at the end of a cycle no longer matches the products the Arnoldi process
// saw.  With Z kept, the Arnoldi residual is the true residual (float64
// products), so a preconditioner that is poor in a few directions costs a few
// iterations, not the convergence test.  This is GMRES-based iterative
// refinement of the mixed-precision LU (capytaine calls SciPy's GMRES without
// a preconditioner).
//
// Every column of every matrix is an independent system ("system" below).  All
// systems advance in lockstep: one matrix-vector product serves the current
// Krylov vectors of all columns of a matrix (one read of A per iteration), one
// CTA per system runs the Arnoldi step, the rotations and the tests.  Systems
// that have left the inner loop or converged are skipped; kernels of
// iterations with no active system return at once (device flags), so the host
// enqueues iterations in groups and synchronises once per group.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include "common.cuh"

namespace bem {


namespace {

constexpr int kThreads = 512;
constexpr int kMaxRestart = 64;
constexpr int kGroup = 4;  // inner iterations enqueued between host checks

struct GmresSystem {
  double bnrm2;            // |b|
  double atol;             // max(atol, rtol |b|)
  double ptol;             // inner (preconditioned-residual) tolerance
  double ptol_max_factor;  // SciPy's adaptive factor
  double presid;           // |S[col+1]| after the last rotation
  double rnorm;            // true residual norm after the last cycle
  int col_end;             // last Arnoldi column of the current cycle (-1: none)
  int active;              // in the inner loop of the current cycle
  int ran;                 // took part in the current cycle
  int done;                // left for good (converged, or failed)
  int failed;              // breakdown without convergence
  int breakdown;           // exact-solution indicator of the current cycle
  int iters;               // inner iterations so far
  int pad;
};

struct Flags {
  int skip_inner;  // no system in the inner loop: iteration kernels return at once
  int skip_all;    // every system done
  int ticket;      // last-CTA election
  int active_count;
};

struct HostState {
  double worst_rel;  // max over systems of |r| / |b|
  double max_iters;
  double nfailed;
  double all_done;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconjmul(double2 a, double2 b) {  // conj(a) b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  // Smith's algorithm
  if (fabs(b.x) >= fabs(b.y)) {
    const double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  const double r = b.x / b.y, d = b.x * r + b.y;
  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__device__ __forceinline__ double cabs2(double2 a) { return hypot(a.x, a.y); }

// Sum over the CTA of (re, im) pairs; every thread gets the total.
__device__ double2 block_sum2(double2 v, double2* red) {
  for (int off = 16; off > 0; off >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();  // red reused across calls
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double2 t = make_double2(0.0, 0.0);
  for (int w = 0; w < nw; ++w) {
    t.x += red[w].x;
    t.y += red[w].y;
  }
  return t;
}

// Elects the last CTA of the grid to finish; it publishes the grid-wide result.
__device__ bool last_cta(Flags* f) {
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = (atomicAdd(&f->ticket, 1) == (int)gridDim.x - 1);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

struct Layout {
  int n, npad, nrhs, m;
  int64_t ldb, strideB;
  __device__ int64_t vec_off(int sys) const {  // offset of system sys in a [batch][nrhs][npad] buffer
    const int b = sys / nrhs, c = sys % nrhs;
    return ((int64_t)b * nrhs + c) * npad;
  }
  __device__ int64_t v_off(int sys, int k) const {  // Krylov vector k: [batch][k][nrhs][npad]
    const int b = sys / nrhs, c = sys % nrhs;
    return (((int64_t)b * (m + 1) + k) * nrhs + c) * npad;
  }
  __device__ int64_t x_off(int sys) const {  // X and B: [batch] stride strideB, column ldb
    const int b = sys / nrhs, c = sys % nrhs;
    return (int64_t)b * strideB + (int64_t)c * ldb;
  }
};

// |b| and the tolerances; R = b (rows < n).  scipy: atol = max(atol, rtol |b|);
// |b| = 0 returns x = 0; an initial residual below atol returns at once.
__global__ void __launch_bounds__(kThreads) gmres_setup_kernel(Layout L, const double2* __restrict__ Bv,
                                                               double2* __restrict__ R, GmresSystem* sys,
                                                               double atol, double rtol, Flags* flags,
                                                               HostState* hs) {
  __shared__ double2 red[32];
  const int s = blockIdx.x;
  const double2* b = Bv + L.x_off(s);
  double2* r = R + L.vec_off(s);
  double acc = 0.0;
  for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
    const double2 v = b[i];
    r[i] = v;
    acc += v.x * v.x + v.y * v.y;
  }
  const double bn = sqrt(block_sum2(make_double2(acc, 0.0), red).x);
  if (threadIdx.x == 0) {
    GmresSystem g{};
    g.bnrm2 = bn;
    g.atol = fmax(atol, rtol * bn);
    g.ptol_max_factor = 1.0;
    g.col_end = -1;
    g.rnorm = bn;
    g.done = (bn == 0.0 || bn < g.atol) ? 1 : 0;
    sys[s] = g;
  }
  if (last_cta(flags) && threadIdx.x == 0) {
    int all = 1;
    for (int t = 0; t < (int)gridDim.x; ++t) all &= sys[t].done;
    flags->skip_all = all;
    flags->skip_inner = all;
    flags->ticket = 0;
    hs->all_done = all;
    hs->worst_rel = 0.0;
    hs->max_iters = 0.0;
    hs->nfailed = 0.0;
  }
}

// W = R for the systems still running (start of a cycle).
__global__ void gmres_copy_kernel(Layout L, const double2* __restrict__ R, double2* __restrict__ W,
                                  const GmresSystem* sys, const Flags* flags) {
  if (flags->skip_all) return;
  const int s = blockIdx.y;
  if (sys[s].done) return;
  const int64_t o = L.vec_off(s);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.n; i += gridDim.x * blockDim.x) W[o + i] = R[o + i];
}

// Start of a cycle: v0 = r / |r| (r in W), S = (|r|, 0, ...).  On the first
// cycle also ptol = |b| min(1, atol / |b|) (SciPy's rule without a left
// preconditioner).
__global__ void __launch_bounds__(kThreads) gmres_start_kernel(Layout L, const double2* __restrict__ W,
                                                               double2* __restrict__ V, double2* __restrict__ Svec,
                                                               GmresSystem* sys, int first, Flags* flags) {
  __shared__ double2 red[32];
  if (flags->skip_all) return;
  const int s = blockIdx.x;
  GmresSystem g = sys[s];
  int act = 0;
  if (!g.done) {
    const double2* z = W + L.vec_off(s);
    double acc = 0.0;
    for (int i = threadIdx.x; i < L.n; i += blockDim.x) acc += z[i].x * z[i].x + z[i].y * z[i].y;
    const double tmp = sqrt(block_sum2(make_double2(acc, 0.0), red).x);
    double2* v0 = V + L.v_off(s, 0);
    const double inv = tmp > 0.0 ? 1.0 / tmp : 0.0;
    for (int i = threadIdx.x; i < L.npad; i += blockDim.x) {
      const double2 zi = i < L.n ? z[i] : make_double2(0.0, 0.0);
      v0[i] = make_double2(zi.x * inv, zi.y * inv);
    }
    if (threadIdx.x == 0) {
      double2* S = Svec + (int64_t)s * (L.m + 1);
      S[0] = make_double2(tmp, 0.0);
      for (int k = 1; k <= L.m; ++k) S[k] = make_double2(0.0, 0.0);
      if (first) g.ptol = tmp * fmin(g.ptol_max_factor, g.atol / g.bnrm2);
      g.col_end = -1;
      g.breakdown = 0;
      if (tmp > 0.0) {
        g.active = 1;
        g.ran = 1;
      } else {  // r = 0: x is exact
        g.active = 0;
        g.ran = 0;
        g.done = 1;
      }
      sys[s] = g;
    }
    act = tmp > 0.0;
  } else if (threadIdx.x == 0) {
    sys[s].active = 0;
    sys[s].ran = 0;
  }
  if (threadIdx.x == 0 && act) atomicAdd(&flags->active_count, 1);
  if (last_cta(flags) && threadIdx.x == 0) {
    flags->skip_inner = (atomicAdd(&flags->active_count, 0) == 0);
    flags->active_count = 0;
    flags->ticket = 0;
  }
}

// One Arnoldi step for column `col` of every active system: w (in W) is
// orthogonalised against v_0..v_col by modified Gram-Schmidt (one pass over w
// per vector, the subtraction of v_{k-1} fused with the product with v_k),
// h_{col+1} = |w|, v_{col+1} = w / h_{col+1}; then the previous rotations, the
// new rotation (LAPACK zlartg convention: c real, r = f / |f| sqrt(|f|^2 +
// |g|^2)), the Hessenberg right-hand side S and the inner residual |S[col+1]|.
__global__ void __launch_bounds__(kThreads) gmres_arnoldi_kernel(Layout L, int col, double2* __restrict__ W,
                                                                 double2* __restrict__ V, double2* __restrict__ H,
                                                                 double2* __restrict__ Gs, double* __restrict__ Gc,
                                                                 double2* __restrict__ Svec, GmresSystem* sys,
                                                                 Flags* flags) {
  __shared__ double2 red[32];
  if (flags->skip_inner) return;
  const int s = blockIdx.x;
  int still = 0;
  if (sys[s].active) {
    double2* w = W + L.vec_off(s);
    double2* h = H + ((int64_t)s * L.m + col) * (L.m + 1);  // h[col][0..m]
    double2 hprev = make_double2(0.0, 0.0);
    double h0 = 0.0, h1 = 0.0;
    for (int k = 0; k <= col + 1; ++k) {
      const double2* vk = V + L.v_off(s, k <= col ? k : col);
      const double2* vp = V + L.v_off(s, k > 0 ? k - 1 : 0);
      double2 acc = make_double2(0.0, 0.0);
      double nrm = 0.0;
      for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
        double2 wi = w[i];
        if (k > 0) {
          const double2 p = cmul(hprev, vp[i]);
          wi.x -= p.x;
          wi.y -= p.y;
          w[i] = wi;
        }
        if (k == 0 || k == col + 1) nrm += wi.x * wi.x + wi.y * wi.y;
        if (k <= col) {
          const double2 t = cconjmul(vk[i], wi);
          acc.x += t.x;
          acc.y += t.y;
        }
      }
      if (k <= col) {
        const double2 t = block_sum2(make_double2(acc.x, acc.y), red);
        const double2 tn = k == 0 ? block_sum2(make_double2(nrm, 0.0), red) : make_double2(0.0, 0.0);
        if (k == 0) h0 = sqrt(tn.x);
        hprev = t;
        if (threadIdx.x == 0) h[k] = t;
      } else {
        h1 = sqrt(block_sum2(make_double2(nrm, 0.0), red).x);
      }
    }
    const bool brk = !(h1 > kEpsilon * h0);
    double2* vn = V + L.v_off(s, col + 1);
    const double inv = brk ? 1.0 : 1.0 / h1;
    for (int i = threadIdx.x; i < L.npad; i += blockDim.x) {
      const double2 wi = i < L.n ? w[i] : make_double2(0.0, 0.0);
      vn[i] = make_double2(wi.x * inv, wi.y * inv);
    }
    if (threadIdx.x == 0) {
      GmresSystem g = sys[s];
      h[col + 1] = make_double2(brk ? 0.0 : h1, 0.0);
      double* gc = Gc + (int64_t)s * L.m;
      double2* gs = Gs + (int64_t)s * L.m;
      for (int k = 0; k < col; ++k) {
        const double c = gc[k];
        const double2 sn = gs[k], n0 = h[k], n1 = h[k + 1];
        const double2 a = cmul(sn, n1), b = cmul(make_double2(sn.x, -sn.y), n0);
        h[k] = make_double2(c * n0.x + a.x, c * n0.y + a.y);
        h[k + 1] = make_double2(c * n1.x - b.x, c * n1.y - b.y);
      }
      const double2 f = h[col], gg = h[col + 1];
      double c;
      double2 sn, r;
      const double af = cabs2(f), ag = cabs2(gg);
      if (ag == 0.0) {
        c = 1.0;
        sn = make_double2(0.0, 0.0);
        r = f;
      } else if (af == 0.0) {
        c = 0.0;
        sn = make_double2(gg.x / ag, -gg.y / ag);
        r = make_double2(ag, 0.0);
      } else {
        const double d = hypot(af, ag);
        const double2 ph = make_double2(f.x / af, f.y / af);  // f / |f|
        c = af / d;
        sn = cmul(ph, make_double2(gg.x / d, -gg.y / d));       // (f/|f|) conj(g) / d
        r = make_double2(ph.x * d, ph.y * d);
      }
      gc[col] = c;
      gs[col] = sn;
      h[col] = r;
      h[col + 1] = make_double2(0.0, 0.0);
      double2* S = Svec + (int64_t)s * (L.m + 1);
      const double2 sc = S[col];
      const double2 t = cmul(make_double2(-sn.x, sn.y), sc);  // -conj(s) S[col]
      S[col] = make_double2(c * sc.x, c * sc.y);
      S[col + 1] = t;
      g.presid = cabs2(t);
      g.iters += 1;
      g.breakdown = brk ? 1 : 0;
      g.col_end = col;
      if (g.presid <= g.ptol || brk || col == L.m - 1) g.active = 0;
      sys[s] = g;
      still = g.active;
    }
  }
  if (threadIdx.x == 0 && still) atomicAdd(&flags->active_count, 1);
  if (last_cta(flags) && threadIdx.x == 0) {
    flags->skip_inner = (atomicAdd(&flags->active_count, 0) == 0);
    flags->active_count = 0;
    flags->ticket = 0;
  }
}

// End of a cycle: y = H^-1 S by back substitution (SciPy's pseudo-solve of
// singular cases), x += P y with P the basis the products were taken of (V
// without a preconditioner, the kept Z = M^-1 V with one); R = b for the
// residual.
__global__ void __launch_bounds__(kThreads) gmres_update_kernel(Layout L, const double2* __restrict__ P,
                                                                const double2* __restrict__ H,
                                                                double2* __restrict__ Svec, const double2* __restrict__ Bv,
                                                                double2* __restrict__ X, double2* __restrict__ R,
                                                                const GmresSystem* sys, const Flags* flags) {
  __shared__ double2 y[kMaxRestart];
  if (flags->skip_all) return;
  const int s = blockIdx.x;
  const GmresSystem g = sys[s];
  if (!g.ran || g.col_end < 0) return;
  const int col = g.col_end;
  if (threadIdx.x == 0) {
    const double2* h = H + (int64_t)s * L.m * (L.m + 1);  // h[c][r] at c*(m+1) + r
    double2* S = Svec + (int64_t)s * (L.m + 1);
    const double2 hcc = h[col * (L.m + 1) + col];
    if (hcc.x == 0.0 && hcc.y == 0.0) S[col] = make_double2(0.0, 0.0);
    for (int k = 0; k <= col; ++k) y[k] = S[k];
    for (int k = col; k > 0; --k) {
      if (y[k].x != 0.0 || y[k].y != 0.0) {
        y[k] = cdiv(y[k], h[k * (L.m + 1) + k]);
        const double2 t = y[k];
        for (int j = 0; j < k; ++j) {
          const double2 p = cmul(t, h[k * (L.m + 1) + j]);
          y[j].x -= p.x;
          y[j].y -= p.y;
        }
      }
    }
    if (y[0].x != 0.0 || y[0].y != 0.0) y[0] = cdiv(y[0], h[0]);
  }
  __syncthreads();
  double2* x = X + L.x_off(s);
  const double2* b = Bv + L.x_off(s);
  double2* r = R + L.vec_off(s);
  for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
    double2 xi = x[i];
    for (int k = 0; k <= col; ++k) {
      const double2 p = cmul(y[k], P[L.v_off(s, k) + i]);
      xi.x += p.x;
      xi.y += p.y;
    }
    x[i] = xi;
    r[i] = b[i];
  }
}

// z_col = v_col of the systems in the inner loop, into Z's slot col (same
// layout as V), where M^-1 then solves in place (flexible GMRES keeps it).
__global__ void gmres_gather_kernel(Layout L, const double2* __restrict__ V, int col, double2* __restrict__ Z,
                                    const GmresSystem* sys, const Flags* flags) {
  if (flags->skip_inner) return;
  const int s = blockIdx.y;
  if (!sys[s].active) return;
  const double2* v = V + L.v_off(s, col);
  double2* z = Z + L.v_off(s, col);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.npad; i += gridDim.x * blockDim.x) z[i] = v[i];
}

// After r = b - A x: convergence (|r| <= atol), breakdown failure, SciPy's
// adaptation of the inner tolerance; the last CTA publishes the state for the host.
__global__ void __launch_bounds__(kThreads) gmres_check_kernel(Layout L, const double2* __restrict__ R,
                                                               GmresSystem* sys, Flags* flags, HostState* hs) {
  __shared__ double2 red[32];
  if (flags->skip_all) return;
  const int s = blockIdx.x;
  GmresSystem g = sys[s];
  if (g.ran && g.col_end >= 0) {
    const double2* r = R + L.vec_off(s);
    double acc = 0.0;
    for (int i = threadIdx.x; i < L.n; i += blockDim.x) acc += r[i].x * r[i].x + r[i].y * r[i].y;
    const double rn = sqrt(block_sum2(make_double2(acc, 0.0), red).x);
    if (threadIdx.x == 0) {
      g.rnorm = rn;
      if (rn <= g.atol) {
        g.done = 1;
      } else if (g.breakdown) {
        g.done = 1;
        g.failed = 1;
      } else {
        if (g.presid <= g.ptol)
          g.ptol_max_factor = fmax(kEpsilon, 0.25 * g.ptol_max_factor);
        else
          g.ptol_max_factor = fmin(1.0, 1.5 * g.ptol_max_factor);
        g.ptol = g.presid * fmin(g.ptol_max_factor, g.atol / rn);
      }
      g.ran = 0;
      sys[s] = g;
    }
  }
  if (last_cta(flags) && threadIdx.x == 0) {
    int all = 1, nf = 0, it = 0;
    double worst = 0.0;
    for (int t = 0; t < (int)gridDim.x; ++t) {
      const GmresSystem q = sys[t];
      all &= q.done;
      nf += q.failed;
      it = max(it, q.iters);
      // systems whose |b| was below atol were solved by x = 0 at the start
      if (q.bnrm2 > 0.0 && q.bnrm2 >= q.atol) worst = fmax(worst, q.rnorm / q.bnrm2);
    }
    flags->skip_all = all;
    flags->skip_inner = all;
    flags->ticket = 0;
    hs->all_done = all;
    hs->nfailed = nf;
    hs->max_iters = it;
    hs->worst_rel = worst;
  }
}

struct GmresWork {
  double2* V;
  double2* W;
  double2* Z;
  double2* R;
  double2* H;
  double2* Gs;
  double* Gc;
  double2* S;
  GmresSystem* sys;
  Flags* flags;
  HostState* hs;
  void* ts;
};

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

size_t carve_gmres(void* base, int n, int npad, int nrhs, int batch, int m, GmresWork* w) {
  const size_t nsys = (size_t)batch * nrhs;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += align256(bytes);
    return o;
  };
  const size_t oV = take(sizeof(double2) * nsys * (m + 1) * npad);
  const size_t oW = take(sizeof(double2) * nsys * npad);
  const size_t oZ = take(sizeof(double2) * nsys * (m + 1) * npad);  // kept M^-1 v_k (flexible GMRES)
  const size_t oR = take(sizeof(double2) * nsys * npad);
  const size_t oH = take(sizeof(double2) * nsys * m * (m + 1));
  const size_t oGs = take(sizeof(double2) * nsys * m);
  const size_t oGc = take(sizeof(double) * nsys * m);
  const size_t oS = take(sizeof(double2) * nsys * (m + 1));
  const size_t oSys = take(sizeof(GmresSystem) * nsys);
  const size_t oF = take(sizeof(Flags));
  const size_t oHs = take(sizeof(HostState));
  const size_t oTs = take((size_t)bem_zgemm_ts_workspace_bytes(n, n, nrhs, batch));
  if (w && base) {
    char* p = (char*)base;
    w->V = (double2*)(p + oV);
    w->W = (double2*)(p + oW);
    w->Z = (double2*)(p + oZ);
    w->R = (double2*)(p + oR);
    w->H = (double2*)(p + oH);
    w->Gs = (double2*)(p + oGs);
    w->Gc = (double*)(p + oGc);
    w->S = (double2*)(p + oS);
    w->sys = (GmresSystem*)(p + oSys);
    w->flags = (Flags*)(p + oF);
    w->hs = (HostState*)(p + oHs);
    w->ts = (void*)(p + oTs);
  }
  return off;
}

}  // namespace
}  // namespace bem

using namespace bem;

extern "C" int64_t bem_gmres_workspace_bytes(int n, int npad, int nrhs, int batch, int restart) {
  if (n <= 0 || npad < n || nrhs <= 0 || nrhs > 16 || batch <= 0 || restart <= 0 || restart > kMaxRestart)
    return -1;
  return (int64_t)carve_gmres(nullptr, n, npad, nrhs, batch, restart, nullptr);
}

extern "C" int bem_gmres_solve(const void* A_dev, int64_t lda, int64_t strideA, int n, int npad, int batch,
                               const void* B_dev, void* X_dev, int64_t ldb, int64_t strideB, int nrhs, double atol,
                               double rtol, int restart, int max_cycles, void* precond_work_dev, void* work_dev,
                               int* err_dev, int* iters_out, double* resid_out, void* stream) {
  if (!A_dev || !B_dev || !X_dev || !work_dev || !iters_out || !resid_out || n <= 0 || npad < n || lda < n ||
      ldb < n || batch <= 0 || nrhs <= 0 || nrhs > 16 || restart <= 0 || restart > kMaxRestart || max_cycles <= 0 ||
      !(atol >= 0.0) || !(rtol >= 0.0) || (precond_work_dev && (!err_dev || npad % 128)))
    return set_error(BEM_ERR_INVALID_ARGUMENT,
                     "bem_gmres_solve: bad arguments (nrhs <= 16, restart <= 64, npad multiple of 128 with a "
                     "preconditioner)");
  if (reinterpret_cast<uintptr_t>(work_dev) & 255)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_gmres_solve: workspace must be 256-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  const int m = std::min(restart, n);
  GmresWork w;
  carve_gmres(work_dev, n, npad, nrhs, batch, m, &w);
  const int nsys = batch * nrhs;
  Layout L{n, npad, nrhs, m, ldb, strideB};
  const int64_t ldv = npad, strideV = (int64_t)(m + 1) * nrhs * npad, strideW = (int64_t)nrhs * npad;
  int launches = 0;
  // Padded rows of W and R stay zero; V is cleared so that the lockstep
  // products never read uninitialised vectors of idle systems.
  BEM_CUDA_CHECK(cudaMemsetAsync(w.V, 0, sizeof(double2) * (size_t)nsys * (m + 1) * npad, s));
  BEM_CUDA_CHECK(cudaMemsetAsync(w.W, 0, sizeof(double2) * (size_t)nsys * npad, s));
  BEM_CUDA_CHECK(cudaMemsetAsync(w.R, 0, sizeof(double2) * (size_t)nsys * npad, s));
  if (precond_work_dev)
    BEM_CUDA_CHECK(cudaMemsetAsync(w.Z, 0, sizeof(double2) * (size_t)nsys * (m + 1) * npad, s));
  BEM_CUDA_CHECK(cudaMemsetAsync(w.flags, 0, sizeof(Flags), s));
  for (int b = 0; b < batch; ++b)
    BEM_CUDA_CHECK(cudaMemset2DAsync((double2*)X_dev + (size_t)b * strideB, ldb * sizeof(double2), 0,
                                     n * sizeof(double2), nrhs, s));
  gmres_setup_kernel<<<nsys, kThreads, 0, s>>>(L, (const double2*)B_dev, w.R, w.sys, atol, rtol, w.flags, w.hs);
  ++launches;
  HostState host{};
  bool converged = false;
  int cycle = 0;
  for (; cycle < max_cycles; ++cycle) {
    // v0 = r / |r|
    gmres_copy_kernel<<<dim3(ceil_div(n, 256), nsys), 256, 0, s>>>(L, w.R, w.W, w.sys, w.flags);
    ++launches;
    gmres_start_kernel<<<nsys, kThreads, 0, s>>>(L, w.W, w.V, w.S, w.sys, cycle == 0, w.flags);
    ++launches;
    for (int col = 0; col < m;) {
      const int group = std::min(kGroup, m - col);
      for (int g = 0; g < group; ++g, ++col) {
        // w = A v_col, or w = A M^-1 v_col, for all systems (one read of each A)
        int st;
        if (precond_work_dev) {
          gmres_gather_kernel<<<dim3(ceil_div(npad, 256), nsys), 256, 0, s>>>(L, w.V, col, w.Z, w.sys, w.flags);
          ++launches;
          double2* zc = w.Z + (size_t)col * nrhs * npad;
          st = clu_solve_enqueue(precond_work_dev, npad, batch, zc, npad, strideV, nrhs, err_dev, s,
                                 &w.flags->skip_inner);
          if (st) return st;
          st = zgemm_ts_enqueue(n, n, nrhs, 1.0, 0.0, A_dev, lda, strideA, zc, ldv, strideV, 0.0, 0.0, w.W, npad,
                                strideW, batch, w.ts, stream, &w.flags->skip_inner);
        } else {
          st = zgemm_ts_enqueue(n, n, nrhs, 1.0, 0.0, A_dev, lda, strideA, w.V + (size_t)col * nrhs * npad, ldv,
                                strideV, 0.0, 0.0, w.W, npad, strideW, batch, w.ts, stream, &w.flags->skip_inner);
        }
        if (st) return st;
        gmres_arnoldi_kernel<<<nsys, kThreads, 0, s>>>(L, col, w.W, w.V, w.H, w.Gs, w.Gc, w.S, w.sys, w.flags);
        ++launches;
      }
      if (col < m) {
        int skip_inner = 0;
        BEM_CUDA_CHECK(cudaMemcpyAsync(&skip_inner, &w.flags->skip_inner, sizeof(int), cudaMemcpyDeviceToHost, s));
        BEM_CUDA_CHECK(cudaStreamSynchronize(s));
        if (skip_inner) break;
      }
    }
    gmres_update_kernel<<<nsys, kThreads, 0, s>>>(L, precond_work_dev ? w.Z : w.V, w.H, w.S,
                                                  (const double2*)B_dev, (double2*)X_dev, w.R, w.sys, w.flags);
    ++launches;
    // r = b - A x
    int st = zgemm_ts_enqueue(n, n, nrhs, -1.0, 0.0, A_dev, lda, strideA, X_dev, ldb, strideB, 1.0, 0.0, w.R, npad,
                              strideW, batch, w.ts, stream, &w.flags->skip_all);
    if (st) return st;
    gmres_check_kernel<<<nsys, kThreads, 0, s>>>(L, w.R, w.sys, w.flags, w.hs);
    ++launches;
    BEM_CUDA_CHECK(cudaMemcpyAsync(&host, w.hs, sizeof(HostState), cudaMemcpyDeviceToHost, s));
    BEM_CUDA_CHECK(cudaStreamSynchronize(s));
    if (host.all_done != 0.0) {
      converged = host.nfailed == 0.0;
      ++cycle;
      break;
    }
  }
  count_launches(launches);
  BEM_CUDA_CHECK(cudaGetLastError());
  *iters_out = (int)host.max_iters;
  *resid_out = host.worst_rel;
  if (!converged) {
    char msg[200];
    std::snprintf(msg, sizeof(msg),
                  "No convergence of the GMRES after %d restart cycles (%d iterations, %d systems broke down); "
                  "worst relative residual %.3e",
                  cycle, (int)host.max_iters, (int)host.nfailed, host.worst_rel);
    return set_error(BEM_ERR_NOT_CONVERGED, msg);
  }
  return BEM_OK;
}
