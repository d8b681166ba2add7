// Assembly of the Delhommeau influence matrices S and K (or D, or the full
// gradient) for one wavenumber in infinite depth.
//
// Replaces matrices::build_matrices, add_diagonal_term and add_rankine_term_only
// (libs/libDelhommeau/src/matrices.f90:28-432) with the callees
// Green_Rankine.f90:28-338 (exact and one-point Rankine integrals, reflected
// through the free surface), Green_wave.f90:50-271 (wave term, free-surface
// self-panel term) and Delhommeau_integrals.f90:157-402 (tabulation lookup,
// asymptotic branch).
//
// Work decomposition: a CTA owns 128 consecutive collocation points (rows I) and
// a tile of kTileJ source panels (columns J) staged in shared memory.  Each
// thread walks its row across the tile, so each column store of a warp is 32
// consecutive complex entries of the column-major output.
//
// Precision: BEM_PREC_FP64 evaluates every term in float64.  BEM_PREC_MIXED
// evaluates the tabulated wave term (table values, Lagrange interpolation,
// gradient assembly) in float32 and keeps the Rankine terms in float64: the
// exact near-field integrals are singular (log/atan), and the one-point far
// field dominates the real part of K, whose float32 rounding would perturb the
// O(k)-small imaginary part of the source strengths (radiation damping at low
// frequency) beyond 1e-5 relative.
#include <cmath>
#include "integrals.cuh"

namespace bem {
namespace {

constexpr int kRows = 128;   // threads per CTA = rows per CTA
constexpr int kTileJ = 32;   // panels per CTA

struct FaceRec {
  double v[12];  // 4 vertices
  double c[3];
  double n[3];
  double area;
  double radius;
  double q0[3];  // first quadrature point
  double w0;     // its weight
};

// Plain Euclidean norm, used inside the exact integrals (last-ulp differences only).
__device__ __forceinline__ double dnorm3(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }

// Fortran NORM2 with gfortran's scaled accumulation, every operation rounded
// on its own.  The near/far switch `r0 > 7*radius` (Green_Rankine.f90:50,227)
// meets exact ties on regular meshes (panel pairs exactly 7 radii apart); this
// norm makes the tie resolve the same way as in the CPU restatement.
__device__ __forceinline__ double norm2_scaled(const double* x, int n) {
  double scale = 0.0, result = 1.0;
  for (int i = 0; i < n; ++i) {
    if (x[i] != 0.0) {
      const double ax = fabs(x[i]);
      if (scale < ax) {
        const double v = __ddiv_rn(scale, ax);
        result = __dadd_rn(1.0, __dmul_rn(__dmul_rn(result, v), v));
        scale = ax;
      } else {
        const double v = __ddiv_rn(ax, scale);
        result = __dadd_rn(result, __dmul_rn(v, v));
      }
    }
  }
  return __dmul_rn(scale, __dsqrt_rn(result));
}
__device__ __forceinline__ double norm2_3(double a, double b, double c) {
  const double v[3] = {a, b, c};
  return norm2_scaled(v, 3);
}
__device__ __forceinline__ double norm2_2(double a, double b) {
  const double v[2] = {a, b};
  return norm2_scaled(v, 2);
}

// Green_Rankine.f90:68-157
__device__ void exact_rankine(const double M[3], const FaceRec& f, bool deriv_first, double& G, double dG[3]) {
  const double* c = f.c;
  const double* n = f.n;
  const double GZ = (M[0] - c[0]) * n[0] + (M[1] - c[1]) * n[1] + (M[2] - c[2]) * n[2];
  double RR[4], DRX[4][3];
#pragma unroll
  for (int L = 0; L < 4; ++L) {
    const double d0 = M[0] - f.v[3 * L], d1 = M[1] - f.v[3 * L + 1], d2 = M[2] - f.v[3 * L + 2];
    RR[L] = dnorm3(d0, d1, d2);
    const double inv = 1.0 / RR[L];
    DRX[L][0] = d0 * inv;
    DRX[L][1] = d1 * inv;
    DRX[L][2] = d2 * inv;
  }
  G = 0.0;
  dG[0] = dG[1] = dG[2] = 0.0;
  const double sgn = copysign(1.0, GZ);
  const double aGZ = fabs(GZ);
  const bool use_atan = aGZ >= kLit1em4 * f.radius;
#pragma unroll
  for (int L = 0; L < 4; ++L) {
    const int Ln = (L + 1) & 3;
    const double e0 = f.v[3 * Ln] - f.v[3 * L], e1 = f.v[3 * Ln + 1] - f.v[3 * L + 1],
                 e2 = f.v[3 * Ln + 2] - f.v[3 * L + 2];
    const double DK = dnorm3(e0, e1, e2);
    if (DK >= kLit1em3 * f.radius) {
      const double PJ0 = e0 / DK, PJ1 = e1 / DK, PJ2 = e2 / DK;
      const double GYX0 = n[1] * PJ2 - n[2] * PJ1;
      const double GYX1 = n[2] * PJ0 - n[0] * PJ2;
      const double GYX2 = n[0] * PJ1 - n[1] * PJ0;
      const double GY = (M[0] - f.v[3 * L]) * GYX0 + (M[1] - f.v[3 * L + 1]) * GYX1 + (M[2] - f.v[3 * L + 2]) * GYX2;
      const double S = RR[Ln] + RR[L];
      const double ANT = 2 * GY * DK;
      const double DNT = S * S - DK * DK + 2 * aGZ * S;
      const double ANL = S + DK;
      const double DNL = S - DK;
      const double ALDEN = log(ANL / DNL);
      const double AT = use_atan ? atan(ANT / DNT) : 0.0;
      const double ANLX0 = DRX[Ln][0] + DRX[L][0], ANLX1 = DRX[Ln][1] + DRX[L][1], ANLX2 = DRX[Ln][2] + DRX[L][2];
      const double two_dk = 2 * DK;
      const double a1 = 2 * (S + aGZ), a2 = 2 * sgn * S;
      const double DNTX0 = a1 * ANLX0 + a2 * n[0];
      const double DNTX1 = a1 * ANLX1 + a2 * n[1];
      const double DNTX2 = a1 * ANLX2 + a2 * n[2];
      if (fabs(GY) < kLit1em5) {
        G = G - 2 * AT * aGZ;
      } else {
        G = G + GY * ALDEN - 2 * AT * aGZ;
      }
      const double c1 = GY * (DNL - ANL) / (ANL * DNL);
      const double cA = 2 * sgn * AT;
      const double cB = 2 * aGZ / (ANT * ANT + DNT * DNT);
      dG[0] = dG[0] + ALDEN * GYX0 - cA * n[0] + c1 * ANLX0 - cB * (two_dk * GYX0 * DNT - DNTX0 * ANT);
      dG[1] = dG[1] + ALDEN * GYX1 - cA * n[1] + c1 * ANLX1 - cB * (two_dk * GYX1 * DNT - DNTX1 * ANT);
      dG[2] = dG[2] + ALDEN * GYX2 - cA * n[2] + c1 * ANLX2 - cB * (two_dk * GYX2 * DNT - DNTX2 * ANT);
    }
  }
  if (!deriv_first) {
    dG[0] = -dG[0];
    dG[1] = -dG[1];
    dG[2] = -dG[2];
  }
}

// Green_Rankine.f90:161-198 (derivative with respect to the first variable)
// v = face centre - point, computed in float64 by the caller.
template <class R>
__device__ __forceinline__ void one_point_rankine(R v0, R v1, R v2, R area, R& G, R dG[3]) {
  const R ro2 = v0 * v0 + v1 * v1 + v2 * v2;
  const R ro = sqrt(ro2);
  if (ro > (R)kLit1em7) {
    G = area / ro;
    const R s = G / ro2;
    dG[0] = v0 * s;
    dG[1] = v1 * s;
    dG[2] = v2 * s;
  } else {
    G = 0;
    dG[0] = dG[1] = dG[2] = 0;
  }
}

__device__ __forceinline__ int f_nint(double x) {
  if (!(fabs(x) < 2.0e9)) return (x > 0) ? 2000000000 : -2000000000;  // also NaN
  return (int)round(x);
}
__device__ __forceinline__ int f_int(double x) {
  if (!(fabs(x) < 2.0e9)) return (x > 0) ? 2000000000 : -2000000000;
  return (int)trunc(x);
}

// Delhommeau_integrals.f90:301-363 (1-based indices)
__device__ __forceinline__ int nearest_r_index(double r, int nr, double rmax, int grid) {
  if (grid == kLegacyGrid) {
    if (r < kLit1em6) return 1;
    if (r < 1.0) return f_int(5 * (log10(r) + 6) + 1);
    return f_int(3 * r + 28);
  }
  const int index_of_1 = (int)lroundf((float)(nr * 81) / 676.0f);
  if (r < kLit1em10) return 1;
  if (r < 1.0) return f_nint((log10(r) / 10.0 + 1.0) * (double)(index_of_1 - 1) + 1);
  return f_nint((r - 1) * (double)(nr - index_of_1) / (rmax - 1) + (double)index_of_1);
}
// dz: (log10|z_last| + 10) / nz of the scaled grid, computed once per thread
// (the same arithmetic as per call).
__device__ __forceinline__ int nearest_z_index(double z, int nz, double zlast, int grid, double dz) {
  const double absz = fabs(z);
  if (grid == kLegacyGrid) {
    if (absz > kLit1em2) return f_int(8 * (log10(absz) + 4.5));
    return f_int(5 * (log10(absz) + 6));
  }
  return f_nint((log10(absz) + 10) / dz);
}
__device__ __forceinline__ double scaled_dz(double zlast, int nz) { return (log10(fabs(zlast)) + 10.0) / (double)nz; }

__device__ __forceinline__ double pl2(double u1, double u2, double u3, double x) {
  return ((x - u1) * (x - u2)) / ((u3 - u1) * (u3 - u2));
}

// Delhommeau_integrals.f90:157-186
template <class R>
__device__ void asymptotic(R r, R z, R out[5]) {
  const R one_over_r = (R)1 / fmax(r, (R)kLit1em10);
  const R one_over_r1 = (R)1 / hypot(r, z);
  const R expz_sqr = exp(z) * sqrt((R)(2 * kPI) * one_over_r);
  R s, c;
  sincos(r - (R)(kPI / 4), &s, &c);
  const R r13 = one_over_r1 * one_over_r1 * one_over_r1;
  out[0] = 2 * (-expz_sqr * s + z * r13 - one_over_r1);
  out[1] = 2 * (-expz_sqr * s + z * r13);
  out[2] = 2 * (expz_sqr * c);
  out[3] = 2 * (-expz_sqr * (c - s * one_over_r / 2) + r * r13);
  out[4] = 2 * (-expz_sqr * (s + c * one_over_r / 2));
}

struct TabView {
  int npts, grid, nr, nz;
  const double* r_range;
  const double* z_range;
  const double* tab;
  const float* tab32;
  double rmax, zlast;
  // optional: reciprocals of the Lagrange denominators of each stencil
  // (3 per centre node, bem_tabulation_inverse_denominators); NULL: divisions
  const double* rinv;
  const double* zinv;
  double dz;
  // set by tab_prologue on the device: the scaled grid's node index of r = 1,
  // the slope of its linear part and 1 / dz (the float32 index estimates)
  int index_of_1;
  double r_slope, inv_dz;
};
__device__ __forceinline__ void tab_prologue(TabView& T) {
  if (T.nr > 1 && T.nz > 1) {
    T.rmax = __ldg(T.r_range + T.nr - 1);
    T.zlast = __ldg(T.z_range + T.nz - 1);
    T.dz = scaled_dz(T.zlast, T.nz);
    T.index_of_1 = (int)lroundf((float)(T.nr * 81) / 676.0f);
    T.r_slope = (double)(T.nr - T.index_of_1) / (T.rmax - 1);
    T.inv_dz = 1 / T.dz;
  }
}

// f_nint(q) when q is more than `margin` away from every rounding boundary
// (q an estimate of the float64 argument of the rounding, within margin of
// it): then both round to the same node.  false: decide with the float64
// expression.
__device__ __forceinline__ bool nint_clear(double q, double margin, int& out) {
  if (!(fabs(q) < 1.0e9)) return false;
  const double fl = floor(q);
  const double fr = q - fl;
  if (fabs(fr - 0.5) <= margin) return false;
  out = (int)fl + (fr > 0.5 ? 1 : 0);
  return true;
}
// Delhommeau_integrals.f90:301-363 on the scaled grid from float32 logarithms
// and precomputed slopes, falling back to the float64 expressions of
// nearest_r_index / nearest_z_index within a margin of a rounding boundary
// (log10f is within 2 ulp, i.e. 2e-6 absolute for |log10| <= 16; the margins
// allow 1e-4): the same nodes as those, at a fraction of the float64 cost.
__device__ __forceinline__ int nearest_r_index_fast(double r, const TabView& T) {
  if (T.grid != kLegacyGrid && r >= kLit1em10) {
    int i;
    if (r < 1.0) {
      const double q = ((double)log10f((float)r) / 10.0 + 1.0) * (double)(T.index_of_1 - 1) + 1;
      if (nint_clear(q, 1e-5 * (double)(T.index_of_1 - 1), i)) return i;
    } else {
      if (nint_clear((r - 1) * T.r_slope + (double)T.index_of_1, 1e-9, i)) return i;
    }
  }
  return nearest_r_index(r, T.nr, T.rmax, T.grid);
}
__device__ __forceinline__ int nearest_z_index_fast(double z, const TabView& T) {
  if (T.grid != kLegacyGrid) {
    int j;
    const double q = ((double)log10f((float)fabs(z)) + 10) * T.inv_dz;
    if (nint_clear(q, 1e-4 * T.inv_dz, j)) return j;
  }
  return nearest_z_index(z, T.nz, T.zlast, T.grid, T.dz);
}
// Lagrange weights of the three stencil nodes u[0..2] at x (node i's weight
// prod_{k != i} (x - u_k) / (u_i - u_k)), the reciprocal denominators from inv
// when given.
__device__ __forceinline__ void lagrange3(double x, double u1, double u2, double u3, const double* inv, double w[3]) {
  if (inv) {
    w[0] = ((x - u2) * (x - u3)) * __ldg(inv);
    w[1] = ((x - u3) * (x - u1)) * __ldg(inv + 1);
    w[2] = ((x - u1) * (x - u2)) * __ldg(inv + 2);
  } else {
    w[0] = pl2(u2, u3, u1, x);
    w[1] = pl2(u3, u1, u2, x);
    w[2] = pl2(u1, u2, u3, x);
  }
}

// The five integrals at (r, z): table (3x3 Lagrange), asymptotic form or
// direct integration (Green_wave.f90:226-240).
template <class R>
__device__ void integrals_at(double r, double z, const TabView& T, R out[5]) {
  if (T.nz <= 1 || T.nr <= 1) {
    double o[5];
    numerical_integration_device(r, z, T.npts, o);
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = (R)o[k];
    return;
  }
  if (fabs(z) < fabs(T.zlast) && r < T.rmax) {
    int i = nearest_r_index_fast(r, T);
    i = max(2, min(T.nr - 1, i));
    int j = nearest_z_index_fast(z, T);
    j = max(2, min(T.nz - 1, j));
    const int ic = i - 1, jc = j - 1;
    const double r1 = __ldg(T.r_range + ic - 1), r2 = __ldg(T.r_range + ic), r3 = __ldg(T.r_range + ic + 1);
    const double z1 = __ldg(T.z_range + jc - 1), z2 = __ldg(T.z_range + jc), z3 = __ldg(T.z_range + jc + 1);
    double wr[3], wz[3];
    lagrange3(r, r1, r2, r3, T.rinv ? T.rinv + 3 * ic : nullptr, wr);
    lagrange3(z, z1, z2, z3, T.zinv ? T.zinv + 3 * jc : nullptr, wz);
    const R xl0 = (R)wr[0], xl1 = (R)wr[1], xl2 = (R)wr[2];
    const R zl0 = (R)wz[0], zl1 = (R)wz[1], zl2 = (R)wz[2];
    R acc[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) acc[k] = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const size_t base = ((size_t)(ic - 1 + a) * T.nz + (jc - 1)) * kNbTab;
      const R xa = (a == 0) ? xl0 : (a == 1) ? xl1 : xl2;
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        R t0, t1, t2;
        if constexpr (sizeof(R) == 8) {
          t0 = __ldg(T.tab + base + k);
          t1 = __ldg(T.tab + base + kNbTab + k);
          t2 = __ldg(T.tab + base + 2 * kNbTab + k);
        } else {
          t0 = __ldg(T.tab32 + base + k);
          t1 = __ldg(T.tab32 + base + kNbTab + k);
          t2 = __ldg(T.tab32 + base + 2 * kNbTab + k);
        }
        acc[k] += xa * (t0 * zl0 + t1 * zl1 + t2 * zl2);
      }
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = acc[k];
    return;
  }
  asymptotic<R>((R)r, (R)z, out);
}

// Green_wave.f90:162-271 at one quadrature point, multiplied by weight w.
template <class R>
__device__ void wave_part(const double x[3], const double xj[3], double k, const TabView& T, int sing, R w,
                          R& Gre, R& Gim, R dGre[3], R dGim[3]) {
  const double dx = x[0] - xj[0], dy = x[1] - xj[1];
  const double r = k * norm2_2(dx, dy);
  const double z = k * (x[2] + xj[2]);
  const R r1 = (R)hypot(r, z);
  R drdx1 = 0, drdx2 = 0;
  if (fabs(r) > 16 * kEpsilon) {
    drdx1 = (R)(k * k * dx / r);
    drdx2 = (R)(k * k * dy / r);
  }
  const R dzdx3 = (R)k;
  R I[5];
  integrals_at<R>(r, z, T, I);
  R gre, gim = I[2];
  R d0r, d1r, d2r;
  const R d0i = drdx1 * I[4], d1i = drdx2 * I[4], d2i = dzdx3 * I[2];
  if (sing == kHighFreq) {
    gre = I[1];
    const R r13 = r1 * r1 * r1;
    d0r = drdx1 * I[3] - 2 * drdx1 * (R)r / r13;
    d1r = drdx2 * I[3] - 2 * drdx2 * (R)r / r13;
    d2r = dzdx3 * gre - 2 * dzdx3 * (R)z / r13;
  } else {
    gre = I[0];
    d0r = drdx1 * I[3];
    d1r = drdx2 * I[3];
    d2r = (sing == kLowFreq) ? dzdx3 * (gre + 2 / r1) : dzdx3 * gre;
  }
  const R kw = (R)k * w;
  Gre += kw * gre;
  Gim += kw * gim;
  dGre[0] += kw * d0r;
  dGre[1] += kw * d1r;
  dGre[2] += kw * d2r;
  dGim[0] += kw * d0i;
  dGim[1] += kw * d1i;
  dGim[2] += kw * d2i;
}

template <class Out>
struct OutT;
template <>
struct OutT<double2> {
  __device__ static double2 make(double re, double im) { return make_double2(re, im); }
};
template <>
struct OutT<float2> {
  __device__ static float2 make(double re, double im) { return make_float2((float)re, (float)im); }
};

// RANKINE_PART: write only the wavenumber-independent Rankine part of each
// entry, unscaled, to rank_out(I, J) = (sum of the direct and reflected Rankine
// G, dot normal . their gradient) with the same arithmetic as the full entry.
template <class Out, bool MIXED, bool RANKINE_PART = false>
// Four CTAs per SM (128 registers, a small spill): measured 12% faster than the
// three that 168 registers allow on this FP64-latency-bound kernel.
__global__ void __launch_bounds__(kRows, 4) assemble_kernel(const bem_assembly_args a, TabView T, double k_wave,
                                                         int gf_sing, bool finite_k, double sign_refl,
                                                         double2* __restrict__ rank_out = nullptr,
                                                         int64_t rank_ld = 0) {
  __shared__ FaceRec faces[kTileJ];
  if (T.nr > 1 && T.nz > 1) {
    // Grid bounds of the tabulation (last r and z values).
    tab_prologue(T);
  }
  const int J0 = blockIdx.y * kTileJ;
  const int nJ = min(kTileJ, a.nb_faces - J0);
  // Stage the tile's panels: thread t fills face t (<= kTileJ faces).
  if ((int)threadIdx.x < nJ) {
    const int J = J0 + threadIdx.x;
    FaceRec& f = faces[threadIdx.x];
#pragma unroll
    for (int L = 0; L < 4; ++L) {
      const int v = a.faces_dev[4 * J + L];
      f.v[3 * L] = a.vertices_dev[3 * v];
      f.v[3 * L + 1] = a.vertices_dev[3 * v + 1];
      f.v[3 * L + 2] = a.vertices_dev[3 * v + 2];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      f.c[d] = a.centers_dev[3 * J + d];
      f.n[d] = a.normals_dev[3 * J + d];
      f.q0[d] = a.quad_points_dev[(size_t)3 * a.nb_quad_points * J + d];
    }
    f.area = a.areas_dev[J];
    f.radius = a.radii_dev[J];
    f.w0 = a.quad_weights_dev[(size_t)a.nb_quad_points * J];
  }
  __syncthreads();
  const int I = blockIdx.x * kRows + threadIdx.x;
  if (I >= a.n) return;
  const double M[3] = {a.points_dev[3 * I], a.points_dev[3 * I + 1], a.points_dev[3 * I + 2]};
  const bool adjoint = a.adjoint_double_layer != 0;
  double nI[3] = {0, 0, 0};
  if (adjoint) {
    nI[0] = a.dot_normals_dev[3 * I];
    nI[1] = a.dot_normals_dev[3 * I + 1];
    nI[2] = a.dot_normals_dev[3 * I + 2];
  }
  const bool rankine_only = isinf(a.free_surface);
  const int diag_limit = min(a.n, a.nb_faces);
  double diag_coef = 0.5;
  if (a.diagonal_term && I < diag_limit) {
    // matrices.f90:348 uses the centre of face i of mesh2
    diag_coef = (fabs(a.centers_dev[3 * I + 2] - a.free_surface) < kLit1em8) ? 1.0 : 0.5;
  }
  Out* S = reinterpret_cast<Out*>(a.S_dev);
  Out* K = reinterpret_cast<Out*>(a.K_dev);
  bool nan_seen = false;
  using R = typename std::conditional<MIXED, float, double>::type;

  for (int jj = 0; jj < nJ; ++jj) {
    const FaceRec& f = faces[jj];
    const int J = J0 + jj;
    // ---- Rankine term (exact near field, one point far field) ------------
    double Gr = 0, dGr[3] = {0, 0, 0};
    {
      const double d0 = M[0] - f.c[0], d1 = M[1] - f.c[1], d2 = M[2] - f.c[2];
      const double r0 = norm2_3(d0, d1, d2);
      if (r0 > 7 * f.radius) {
        double g, dg[3];
        one_point_rankine<double>(-d0, -d1, -d2, f.area, g, dg);
        Gr = g;
        dGr[0] = dg[0];
        dGr[1] = dg[1];
        dGr[2] = dg[2];
      } else {
        exact_rankine(M, f, true, Gr, dGr);
      }
    }
    double Gre = Gr;
    double dGre[3] = {dGr[0], dGr[1], dGr[2]};
    double Gim = 0, dGim[3] = {0, 0, 0};
    if (!rankine_only) {
      // ---- reflected Rankine term, mirror z -> -z ---------------------------
      double Gf, dGf[3];
      {
        const double dh = norm2_2(M[0] - f.c[0], M[1] - f.c[1]);
        const double r1 = hypot(dh, -M[2] - f.c[2]);
        const double Mr[3] = {M[0], M[1], -M[2]};
        if (r1 > 7 * f.radius) {
          double g, dg[3];
          one_point_rankine<double>(f.c[0] - Mr[0], f.c[1] - Mr[1], f.c[2] - Mr[2], f.area, g, dg);
          Gf = g;
          dGf[0] = dg[0];
          dGf[1] = dg[1];
          dGf[2] = dg[2];
        } else {
          exact_rankine(Mr, f, true, Gf, dGf);
        }
        dGf[2] = -dGf[2];  // reflection coefficient c0 = -1
      }
      Gre += sign_refl * Gf;
      dGre[0] += sign_refl * dGf[0];
      dGre[1] += sign_refl * dGf[1];
      dGre[2] += sign_refl * dGf[2];
      if (gf_sing == kLowFreqWithRankinePart) dGre[2] += 2 * k_wave * Gf;
      // ---- wave term --------------------------------------------------------
      if (finite_k && !RANKINE_PART) {
        const double dxh = M[0] - f.c[0], dyh = M[1] - f.c[1];
        const double rr = k_wave * norm2_2(dxh, dyh);
        const double zz = k_wave * (M[2] + f.c[2]);
        if (fabs(rr) < kLit1em10 && fabs(zz) < kLit1em10) {
          // Green_wave.f90:128-158, panel on the free surface with itself
          const double re = (1 - log(k_wave * k_wave * f.area / kPI)) + 2 * (kEulerGamma - kLog2);
          const double ka = k_wave * f.area;
          const double gre = ka * re, gim = ka * (-2 * kPI);
          Gre += gre;
          Gim += gim;
          dGre[2] += k_wave * (gre + 4 * sqrt(kPI * f.area));
          dGim[2] += k_wave * gim;
        } else {
          R wr = 0, wi = 0, wdr[3] = {0, 0, 0}, wdi[3] = {0, 0, 0};
          wave_part<R>(M, f.q0, k_wave, T, gf_sing, (R)f.w0, wr, wi, wdr, wdi);
          for (int q = 1; q < a.nb_quad_points; ++q) {
            const double* qp = a.quad_points_dev + ((size_t)a.nb_quad_points * J + q) * 3;
            const double xq[3] = {qp[0], qp[1], qp[2]};
            wave_part<R>(M, xq, k_wave, T, gf_sing, (R)a.quad_weights_dev[(size_t)a.nb_quad_points * J + q], wr, wi,
                         wdr, wdi);
          }
          Gre += wr;
          Gim += wi;
          dGre[0] += wdr[0];
          dGre[1] += wdr[1];
          dGre[2] += wdr[2];
          dGim[0] += wdi[0];
          dGim[1] += wdi[1];
          dGim[2] += wdi[2];
        }
      }
    }
    if (!adjoint) {
      // Derivative with respect to the source point: Rankine gradient flips,
      // the reflected and wave gradients flip horizontally only
      // (Green_Rankine.f90:154-156, 289-294; Green_wave.f90:120-122).
      // Recombine from the parts: the direct Rankine part flips fully.
      dGre[0] = -dGre[0];
      dGre[1] = -dGre[1];
      dGim[0] = -dGim[0];
      dGim[1] = -dGim[1];
      dGre[2] = dGre[2] - 2 * dGr[2];
    }
    if constexpr (RANKINE_PART) {
      const double* dn = adjoint ? nI : (a.dot_normals_dev + 3 * J);
      const double kdot = dn[0] * dGre[0] + dn[1] * dGre[1] + dn[2] * dGre[2];
      rank_out[(size_t)I + (size_t)rank_ld * J] = make_double2(Gre, kdot);
      nan_seen |= isnan(Gre) || isnan(kdot);
      continue;
    }
    const double sre = kMinusOneOverFourPi * Gre, sim = kMinusOneOverFourPi * Gim;
    const size_t sidx = (size_t)I + (size_t)a.lds * J;
    S[sidx] = OutT<Out>::make(sre, sim);
    nan_seen |= isnan(sre) || isnan(sim);
    const bool on_diag = a.diagonal_term && I == J && I < diag_limit;
    const size_t kidx = (size_t)I + (size_t)a.ldk * J;
    if (a.early_dot_product) {
      const double* dn = adjoint ? nI : (a.dot_normals_dev + 3 * J);
      double kre = kMinusOneOverFourPi * (dn[0] * dGre[0] + dn[1] * dGre[1] + dn[2] * dGre[2]);
      const double kim = kMinusOneOverFourPi * (dn[0] * dGim[0] + dn[1] * dGim[1] + dn[2] * dGim[2]);
      if (on_diag) kre += diag_coef;
      K[kidx] = OutT<Out>::make(kre, kim);
      nan_seen |= isnan(kre) || isnan(kim);
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double kre = kMinusOneOverFourPi * dGre[c];
        const double kim = kMinusOneOverFourPi * dGim[c];
        if (on_diag) kre += diag_coef * a.dot_normals_dev[3 * I + c];
        K[kidx + (size_t)c * a.k_plane_stride] = OutT<Out>::make(kre, kim);
        nan_seen |= isnan(kre) || isnan(kim);
      }
    }
  }
  if (nan_seen && a.nan_flag_dev) atomicOr(a.nan_flag_dev, 1);
}

// Wave term of Green_wave.f90:162-271 at one point pair for a unit weight:
// (g, gradient) before the final multiplication by k w, from the horizontal
// offset (dx, dy) of the two points, r = k |(dx, dy)| and z = k (x3 + xj3).
// Swapping the two points leaves g and the vertical derivative unchanged and
// negates the horizontal derivatives exactly (they are linear in (dx, dy)),
// which the symmetric assembly below relies on.  The distances are plain
// square roots and the gradient factors reciprocals (last-ulp differences from
// the scaled norm and the divisions of wave_part; the stencil of the table is
// chosen from r and z as there).  r = z = 0 (a free-surface panel with
// itself) never reaches it.
__device__ __forceinline__ void wave_core(double dx, double dy, double r, double z, double k, const TabView& T,
                                          int sing, double& gre, double& gim, double dr[3], double di[3]) {
  const double ir1 = rsqrt(r * r + z * z);  // 1 / |(r, z)|
  double drdx1 = 0, drdx2 = 0;
  if (fabs(r) > 16 * kEpsilon) {
    const double q = k * k / r;
    drdx1 = q * dx;
    drdx2 = q * dy;
  }
  const double dzdx3 = k;
  double I[5];
  integrals_at<double>(r, z, T, I);
  gim = I[2];
  di[0] = drdx1 * I[4];
  di[1] = drdx2 * I[4];
  di[2] = dzdx3 * I[2];
  if (sing == kHighFreq) {
    gre = I[1];
    const double ir13 = ir1 * ir1 * ir1;
    dr[0] = drdx1 * I[3] - 2 * drdx1 * r * ir13;
    dr[1] = drdx2 * I[3] - 2 * drdx2 * r * ir13;
    dr[2] = dzdx3 * gre - 2 * dzdx3 * z * ir13;
  } else {
    gre = I[0];
    dr[0] = drdx1 * I[3];
    dr[1] = drdx2 * I[3];
    dr[2] = (sing == kLowFreq) ? dzdx3 * (gre + 2 * ir1) : dzdx3 * gre;
  }
}

// The same wave term with the table interpolation, the asymptotic form and the
// gradient assembly in float32 (the mixed-precision assembly of a mesh with
// itself).  r and z, the stencil indices and the distances to the stencil
// nodes stay float64, so that the stencil is the float64 one and the Lagrange
// weights lose nothing to cancellation.
__device__ __forceinline__ float pl2_f(double x, double u1, double u2, double u3) {
  return ((float)(x - u1) * (float)(x - u2)) / ((float)(u3 - u1) * (float)(u3 - u2));
}
__device__ __forceinline__ void integrals_at_f32(double r, double z, const TabView& T, float out[5]) {
  if (fabs(z) < fabs(T.zlast) && r < T.rmax) {
    int i = nearest_r_index(r, T.nr, T.rmax, T.grid);
    i = max(2, min(T.nr - 1, i));
    int j = nearest_z_index(z, T.nz, T.zlast, T.grid, T.dz);
    j = max(2, min(T.nz - 1, j));
    const int ic = i - 1, jc = j - 1;
    const double r1 = __ldg(T.r_range + ic - 1), r2 = __ldg(T.r_range + ic), r3 = __ldg(T.r_range + ic + 1);
    const double z1 = __ldg(T.z_range + jc - 1), z2 = __ldg(T.z_range + jc), z3 = __ldg(T.z_range + jc + 1);
    const float xl[3] = {pl2_f(r, r2, r3, r1), pl2_f(r, r3, r1, r2), pl2_f(r, r1, r2, r3)};
    const float zl0 = pl2_f(z, z2, z3, z1), zl1 = pl2_f(z, z3, z1, z2), zl2 = pl2_f(z, z1, z2, z3);
    float acc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float* t = T.tab32 + ((size_t)(ic - 1 + a) * T.nz + (jc - 1)) * kNbTab;
#pragma unroll
      for (int k = 0; k < 5; ++k)
        acc[k] += xl[a] * (__ldg(t + k) * zl0 + __ldg(t + kNbTab + k) * zl1 + __ldg(t + 2 * kNbTab + k) * zl2);
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = acc[k];
    return;
  }
  asymptotic<float>((float)r, (float)z, out);
}
__device__ __forceinline__ void wave_core_f32(double dx, double dy, double r, double z, double k, const TabView& T,
                                              int sing, double& gre, double& gim, double dr[3], double di[3]) {
  const float rf = (float)r, zf = (float)z;
  const float r1 = sqrtf(rf * rf + zf * zf);
  float drdx1 = 0.f, drdx2 = 0.f;
  if (fabs(r) > 16 * kEpsilon) {
    const float kk = (float)(k * k) / rf;
    drdx1 = kk * (float)dx;
    drdx2 = kk * (float)dy;
  }
  const float dzdx3 = (float)k;
  float I[5];
  integrals_at_f32(r, z, T, I);
  float g_re, d0, d1, d2;
  if (sing == kHighFreq) {
    g_re = I[1];
    const float r13 = r1 * r1 * r1;
    d0 = drdx1 * I[3] - 2.f * drdx1 * rf / r13;
    d1 = drdx2 * I[3] - 2.f * drdx2 * rf / r13;
    d2 = dzdx3 * g_re - 2.f * dzdx3 * zf / r13;
  } else {
    g_re = I[0];
    d0 = drdx1 * I[3];
    d1 = drdx2 * I[3];
    d2 = (sing == kLowFreq) ? dzdx3 * (g_re + 2.f / r1) : dzdx3 * g_re;
  }
  gre = g_re;
  gim = I[2];
  dr[0] = d0;
  dr[1] = d1;
  dr[2] = d2;
  di[0] = drdx1 * I[4];
  di[1] = drdx2 * I[4];
  di[2] = dzdx3 * I[2];
}

constexpr int kSymT = 128;    // square tile: 128 rows x 128 columns, one thread per row
constexpr int kSymChunk = 8;  // columns per mirrored write-back

struct SymFace {
  double x[3];   // collocation point = quadrature point = centre
  double dn[3];  // dot normal of the face
  double area, w, zc;
};

// S and K of a mesh with itself from a cached Rankine part: the CTA of tile
// (bi, bj), bi <= bj, evaluates the wave term once per pair (I, J) and writes
// both (I, J) and, off the diagonal tiles, (J, I) (through shared memory, so
// that the mirrored stores stay coalesced).  FP64, complex128 outputs, K with
// the dot product taken.
// Up to kSymBatch wavenumbers per launch (blockIdx.z), passed by value.
constexpr int kSymBatch = 64;
struct SymBatch {
  double k[kSymBatch];
  int64_t s_stride, k_stride;  // elements between the outputs of consecutive wavenumbers
  // optional float32 copy of K in the planes of the mixed LU's workspace
  // (real plane at w, imaginary plane w_im floats further; leading dimension
  // w_ld, w_stride floats between wavenumbers): the LU then needs no
  // conversion pass over K
  float* w;
  int64_t w_ld, w_stride, w_im;
};

// GENERAL: any collocation points (rows, a.n) against the panels of mesh2
// (columns, a.nb_faces): every tile is evaluated, nothing is mirrored.
// Five CTAs per SM (the shared-memory limit; 96 registers): 3% faster than four.
// INPLACE: the Rankine part is K itself (rank == K, rank_ld == ldk); every
// entry is read, then written, by one thread, and no entry is read after
// another thread wrote it (tile (bi, bj), bi < bj, and its mirror (bj, bi)
// belong to one CTA), so the read-only cache path is not used for it.
// F32: the wave term by wave_core_f32 (float32 interpolation; the cached
// Rankine part and the accumulation stay float64).
template <bool GENERAL, bool INPLACE = false, bool F32 = false>
__global__ void __launch_bounds__(kSymT, 5) wave_symmetric_kernel(bem_assembly_args a, TabView T, SymBatch kb,
                                                               int gf_sing, const double2* rank, int64_t rank_ld) {
  const int bi = blockIdx.x, bj = blockIdx.y;
  if (!GENERAL && bi > bj) return;
  const double k = kb.k[blockIdx.z];
  a.S_dev = reinterpret_cast<double2*>(a.S_dev) + blockIdx.z * kb.s_stride;
  a.K_dev = reinterpret_cast<double2*>(a.K_dev) + blockIdx.z * kb.k_stride;
  float* Wre = kb.w ? kb.w + blockIdx.z * kb.w_stride : nullptr;
  __shared__ SymFace faces[kSymT];
  __shared__ double4 mir[kSymChunk][kSymT];  // (S_w re, S_w im, K_w re, K_w im) of entries (J, I)
  if (T.nr > 1 && T.nz > 1) {
    tab_prologue(T);
  }
  const int tid = threadIdx.x;
  const int N = a.n;
  const int NJ = GENERAL ? a.nb_faces : a.n;
  const int I0 = bi * kSymT, J0 = bj * kSymT;
  const bool adjoint = a.adjoint_double_layer != 0;
  {
    const int J = J0 + tid;
    if (J < NJ) {
      SymFace& f = faces[tid];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        f.x[d] = a.quad_points_dev[3 * J + d];
        // general: the dot normals are mesh2's only without the adjoint
        f.dn[d] = (!GENERAL || !adjoint) ? a.dot_normals_dev[3 * J + d] : 0.0;
      }
      f.area = a.areas_dev[J];
      f.w = a.quad_weights_dev[J];
      f.zc = a.centers_dev[3 * J + 2];
    }
  }
  __syncthreads();
  const int I = I0 + tid;
  const bool row_ok = I < N;
  const bool diag_tile = GENERAL || bi == bj;  // no mirrored entries
  double M[3] = {0, 0, 0}, nI[3] = {0, 0, 0}, wI = 0;
  if (row_ok) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      M[d] = a.points_dev[3 * I + d];
      // general: the dot normals are the rows' only with the adjoint
      nI[d] = (!GENERAL || adjoint) ? a.dot_normals_dev[3 * I + d] : 0.0;
    }
    if (!GENERAL) wI = a.quad_weights_dev[I];
  }
  const double kwI = k * wI;
  double2* S = reinterpret_cast<double2*>(a.S_dev);
  double2* K = reinterpret_cast<double2*>(a.K_dev);
  bool nan_seen = false;
  const int nJ = min(kSymT, NJ - J0);
  for (int jc = 0; jc < nJ; jc += kSymChunk) {
#pragma unroll 1
    for (int u = 0; u < kSymChunk; ++u) {
      const int jj = jc + u;
      if (!row_ok || jj >= nJ) continue;
      const SymFace& f = faces[jj];
      const int J = J0 + jj;
      double gre, gim, dr[3], di[3];
      const double dx = M[0] - f.x[0], dy = M[1] - f.x[1];
      const double rr = k * sqrt(dx * dx + dy * dy);
      const double zz = k * (M[2] + f.x[2]);
      const bool self_fs = fabs(rr) < kLit1em10 && fabs(zz) < kLit1em10;
      const size_t ridx = (size_t)I + (size_t)rank_ld * J;
      const double2 rk = INPLACE ? rank[ridx] : __ldg(rank + ridx);
      double sre, sim, kre, kim;
      if (self_fs) {
        // Green_wave.f90:128-158, panel on the free surface with itself (I == J)
        const double re = (1 - log(k * k * f.area / kPI)) + 2 * (kEulerGamma - kLog2);
        const double ka = k * f.area;
        const double g_re = ka * re, g_im = ka * (-2 * kPI);
        const double dz_re = k * (g_re + 4 * sqrt(kPI * f.area)), dz_im = k * g_im;
        const double* dn = adjoint ? nI : f.dn;
        sre = kMinusOneOverFourPi * (rk.x + g_re);
        sim = kMinusOneOverFourPi * g_im;
        kre = kMinusOneOverFourPi * (rk.y + dn[2] * dz_re);
        kim = kMinusOneOverFourPi * (dn[2] * dz_im);
      } else {
        if constexpr (F32) wave_core_f32(dx, dy, rr, zz, k, T, gf_sing, gre, gim, dr, di);
        else wave_core(dx, dy, rr, zz, k, T, gf_sing, gre, gim, dr, di);
        const double kwJ = k * f.w;
        double vr[3] = {kwJ * dr[0], kwJ * dr[1], kwJ * dr[2]};
        double vi[3] = {kwJ * di[0], kwJ * di[1], kwJ * di[2]};
        if (!adjoint) {
          vr[0] = -vr[0];
          vr[1] = -vr[1];
          vi[0] = -vi[0];
          vi[1] = -vi[1];
        }
        const double* dn = adjoint ? nI : f.dn;
        sre = kMinusOneOverFourPi * (rk.x + kwJ * gre);
        sim = kMinusOneOverFourPi * (kwJ * gim);
        kre = kMinusOneOverFourPi * (rk.y + (dn[0] * vr[0] + dn[1] * vr[1] + dn[2] * vr[2]));
        kim = kMinusOneOverFourPi * (dn[0] * vi[0] + dn[1] * vi[1] + dn[2] * vi[2]);
        if (!diag_tile) {
          // entry (J, I): horizontal derivatives change sign
          double wr[3] = {-kwI * dr[0], -kwI * dr[1], kwI * dr[2]};
          double wi[3] = {-kwI * di[0], -kwI * di[1], kwI * di[2]};
          if (!adjoint) {
            wr[0] = -wr[0];
            wr[1] = -wr[1];
            wi[0] = -wi[0];
            wi[1] = -wi[1];
          }
          const double* dm = adjoint ? f.dn : nI;
          mir[u][tid] = make_double4(kwI * gre, kwI * gim, dm[0] * wr[0] + dm[1] * wr[1] + dm[2] * wr[2],
                                     dm[0] * wi[0] + dm[1] * wi[1] + dm[2] * wi[2]);
        }
      }
      // matrices.f90:348: the centre of face I (= J) of mesh2
      if (a.diagonal_term && I == J) kre += (fabs(f.zc - a.free_surface) < kLit1em8) ? 1.0 : 0.5;
      S[(size_t)I + (size_t)a.lds * J] = make_double2(sre, sim);
      K[(size_t)I + (size_t)a.ldk * J] = make_double2(kre, kim);
      if (Wre) {
        const size_t w = (size_t)I + (size_t)kb.w_ld * J;
        Wre[w] = (float)kre;
        Wre[kb.w_im + w] = (float)kim;
      }
      nan_seen |= isnan(sre) || isnan(sim) || isnan(kre) || isnan(kim);
    }
    if (!diag_tile) {
      __syncthreads();
      // mirrored entries: rows J0 + jc + u, columns I0 + c; 8 threads per column
      const int u = tid & (kSymChunk - 1);
      const int J = J0 + jc + u;
#pragma unroll 1
      for (int c = tid >> 3; c < kSymT; c += kSymT / kSymChunk) {
        const int Ic = I0 + c;
        if (jc + u < nJ && Ic < N) {
          const double4 m = mir[u][c];
          const size_t ridx = (size_t)J + (size_t)rank_ld * Ic;
          const double2 rk = INPLACE ? rank[ridx] : __ldg(rank + ridx);
          const double sre = kMinusOneOverFourPi * (rk.x + m.x), sim = kMinusOneOverFourPi * m.y;
          const double kre = kMinusOneOverFourPi * (rk.y + m.z), kim = kMinusOneOverFourPi * m.w;
          S[(size_t)J + (size_t)a.lds * Ic] = make_double2(sre, sim);
          K[(size_t)J + (size_t)a.ldk * Ic] = make_double2(kre, kim);
          if (Wre) {
            const size_t w = (size_t)J + (size_t)kb.w_ld * Ic;
            Wre[w] = (float)kre;
            Wre[kb.w_im + w] = (float)kim;
          }
          nan_seen |= isnan(sre) || isnan(sim) || isnan(kre) || isnan(kim);
        }
      }
      __syncthreads();
    }
  }
  if (nan_seen && a.nan_flag_dev) atomicOr(a.nan_flag_dev, 1);
}

// ---- finite depth (Delhommeau's method) -------------------------------------
// Green_Rankine.f90:202-338: Rankine term at the image (x, y, c0 z + c1) of M,
// exact or one point by the distance to the face (one point when forced).
__device__ __forceinline__ void reflected_rankine(const double M[3], const FaceRec& f, bool deriv_first, double c0,
                                                  double c1, bool one_point, double& G, double dG[3]) {
  const double Mr[3] = {M[0], M[1], c0 * M[2] + c1};
  const double r1 = hypot(norm2_2(M[0] - f.c[0], M[1] - f.c[1]), Mr[2] - f.c[2]);
  if (one_point || r1 > 7 * f.radius) {
    one_point_rankine<double>(f.c[0] - Mr[0], f.c[1] - Mr[1], f.c[2] - Mr[2], f.area, G, dG);
  } else {
    exact_rankine(Mr, f, true, G, dG);
  }
  dG[2] = c0 * dG[2];
  if (!deriv_first) {
    dG[0] = -dG[0];
    dG[1] = -dG[1];
    if (c0 > 0) dG[2] = -dG[2];
  }
}

// Green_wave.f90:50-124 for the point x and the face of centre c (quadrature
// points of face J, each mirrored through the sea bottom when mirror_face).
__device__ void wave_term(const double x[3], const double c[3], const bem_assembly_args& a, const FaceRec& f, int J,
                          bool mirror_face, double depth, double k, const TabView& T, int sing, bool deriv_first,
                          double& gre, double& gim, double dr[3], double di[3]) {
  gre = gim = 0;
  dr[0] = dr[1] = dr[2] = di[0] = di[1] = di[2] = 0;
  const double rr = k * norm2_2(x[0] - c[0], x[1] - c[1]);
  const double zz = k * (x[2] + c[2]);
  if (fabs(rr) < kLit1em10 && fabs(zz) < kLit1em10) {
    // Green_wave.f90:128-158, panel on the free surface with itself
    const double re = (1 - log(k * k * f.area / kPI)) + 2 * (kEulerGamma - kLog2);
    gre = k * f.area * re;
    gim = k * f.area * (-2 * kPI);
    dr[2] = k * (gre + 4 * sqrt(kPI * f.area));
    di[2] = k * gim;
  } else {
    for (int q = 0; q < a.nb_quad_points; ++q) {
      const double* qp = a.quad_points_dev + ((size_t)a.nb_quad_points * J + q) * 3;
      const double xq[3] = {qp[0], qp[1], mirror_face ? -qp[2] - 2 * depth : qp[2]};
      wave_part<double>(x, xq, k, T, sing, a.quad_weights_dev[(size_t)a.nb_quad_points * J + q], gre, gim, dr, di);
    }
  }
  if (!deriv_first) {
    dr[0] = -dr[0];
    dr[1] = -dr[1];
    di[0] = -di[0];
    di[1] = -di[1];
  }
}

// matrices.f90:28-325 in finite depth, Delhommeau's method: the
// infinite-depth Rankine terms, the Rankine images through the sea bottom
// (matrices.f90:212-268), the four wave terms of Green_wave.f90:311-425 and the
// Prony terms of Green_wave.f90:427-508.  One thread per collocation point,
// the panels of a tile in shared memory; every term in float64, outputs Out
// (complex128 or complex64), K with the dot product taken or the three
// gradient planes, as the general kernel.  prony: rates then amplitudes
// (2 x nexp).
template <class Out>
__global__ void __launch_bounds__(kRows) assemble_finite_depth_kernel(const bem_assembly_args a, TabView T,
                                                                      double depth, int legacy,
                                                                      const double* __restrict__ prony, int nexp,
                                                                      int gf_sing) {
  __shared__ FaceRec faces[kTileJ];
  if (T.nr > 1 && T.nz > 1) {
    tab_prologue(T);
  }
  const int J0 = blockIdx.y * kTileJ;
  const int nJ = min(kTileJ, a.nb_faces - J0);
  if ((int)threadIdx.x < nJ) {
    const int J = J0 + threadIdx.x;
    FaceRec& f = faces[threadIdx.x];
#pragma unroll
    for (int L = 0; L < 4; ++L) {
      const int v = a.faces_dev[4 * J + L];
      f.v[3 * L] = a.vertices_dev[3 * v];
      f.v[3 * L + 1] = a.vertices_dev[3 * v + 1];
      f.v[3 * L + 2] = a.vertices_dev[3 * v + 2];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      f.c[d] = a.centers_dev[3 * J + d];
      f.n[d] = a.normals_dev[3 * J + d];
      f.q0[d] = a.quad_points_dev[(size_t)3 * a.nb_quad_points * J + d];
    }
    f.area = a.areas_dev[J];
    f.radius = a.radii_dev[J];
    f.w0 = a.quad_weights_dev[(size_t)a.nb_quad_points * J];
  }
  __syncthreads();
  const int I = blockIdx.x * kRows + threadIdx.x;
  if (I >= a.n) return;
  const double M[3] = {a.points_dev[3 * I], a.points_dev[3 * I + 1], a.points_dev[3 * I + 2]};
  const double Msym[3] = {M[0], M[1], -M[2] - 2 * depth};
  const bool adjoint = a.adjoint_double_layer != 0;
  double nI[3] = {0, 0, 0};
  if (adjoint) {
    nI[0] = a.dot_normals_dev[3 * I];
    nI[1] = a.dot_normals_dev[3 * I + 1];
    nI[2] = a.dot_normals_dev[3 * I + 2];
  }
  const double k = a.wavenumber;
  const bool finite_k = k > 0.0 && isfinite(k);
  const double sign_refl = (gf_sing == kHighFreq) ? -1.0 : 1.0;
  const int diag_limit = min(a.n, a.nb_faces);
  double diag_coef = 0.5;
  if (a.diagonal_term && I < diag_limit)
    diag_coef = (fabs(a.centers_dev[3 * I + 2] - a.free_surface) < kLit1em8) ? 1.0 : 0.5;
  double A = 0.0;
  if (finite_k) {
    const double amh = k * depth;
    const double akh = amh * tanh(amh);
    A = (amh + akh) * (amh + akh) / (4 * amh * (amh * amh - akh * akh + akh));
  }
  Out* S = reinterpret_cast<Out*>(a.S_dev);
  Out* K = reinterpret_cast<Out*>(a.K_dev);
  bool nan_seen = false;
  for (int jj = 0; jj < nJ; ++jj) {
    const FaceRec& f = faces[jj];
    const int J = J0 + jj;
    double Gre = 0, Gim = 0, dGre[3] = {0, 0, 0}, dGim[3] = {0, 0, 0};
    double g, dg[3];
    // direct Rankine term
    {
      const double d0 = M[0] - f.c[0], d1 = M[1] - f.c[1], d2 = M[2] - f.c[2];
      if (norm2_3(d0, d1, d2) > 7 * f.radius) {
        one_point_rankine<double>(-d0, -d1, -d2, f.area, g, dg);
      } else {
        exact_rankine(M, f, true, g, dg);
      }
      if (!adjoint) {
        dg[0] = -dg[0];
        dg[1] = -dg[1];
        dg[2] = -dg[2];
      }
      Gre += g;
      dGre[0] += dg[0];
      dGre[1] += dg[1];
      dGre[2] += dg[2];
    }
    // free-surface image (one point in the legacy method), with the variant's sign
    reflected_rankine(M, f, adjoint, -1.0, 0.0, legacy != 0, g, dg);
    Gre += sign_refl * g;
    dGre[0] += sign_refl * dg[0];
    dGre[1] += sign_refl * dg[1];
    dGre[2] += sign_refl * dg[2];
    if (gf_sing == kLowFreqWithRankinePart) dGre[2] += 2 * k * g;
    // sea-bottom image, then the images through both boundaries
    reflected_rankine(M, f, adjoint, -1.0, -2 * depth, false, g, dg);
    Gre += g;
    dGre[0] += dg[0];
    dGre[1] += dg[1];
    dGre[2] += dg[2];
    const double c_one_point[3][2] = {{1.0, -2 * depth}, {1.0, 2 * depth}, {-1.0, -4 * depth}};
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      reflected_rankine(M, f, adjoint, c_one_point[t][0], c_one_point[t][1], true, g, dg);
      Gre += sign_refl * g;
      dGre[0] += sign_refl * dg[0];
      dGre[1] += sign_refl * dg[1];
      dGre[2] += sign_refl * dg[2];
    }
    // four infinite-depth wave terms (point, face, each possibly mirrored through the bottom)
    if (finite_k) {
      const double csym[3] = {f.c[0], f.c[1], -f.c[2] - 2 * depth};
      double wre = 0, wim = 0, wdr[3] = {0, 0, 0}, wdi[3] = {0, 0, 0};
#pragma unroll 1
      for (int t = 0; t < 4; ++t) {
        const bool mx = (t & 1) != 0, mf = (t & 2) != 0;
        // z of the gradient mirrored: (x_sym, face) when deriv_first, (x, face_sym)
        // otherwise, (x_sym, face_sym) always (Green_wave.f90:375-411)
        const bool flip_z = (mx && mf) || (mx && adjoint) || (mf && !adjoint);
        double gr, gi, dr[3], di[3];
        wave_term(mx ? Msym : M, mf ? csym : f.c, a, f, J, mf, depth, k, T, gf_sing, adjoint, gr, gi, dr, di);
        if (flip_z) {
          dr[2] = -dr[2];
          di[2] = -di[2];
        }
        wre += gr;
        wim += gi;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          wdr[d] += dr[d];
          wdi[d] += di[d];
        }
      }
      Gre += A * wre;
      Gim += A * wim;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        dGre[d] += A * wdr[d];
        dGim[d] += A * wdi[d];
      }
    }
    // Prony exponentials: four Rankine images each, weighted a / 2
    for (int e = 0; e < nexp; ++e) {
      const double lam = __ldg(prony + e), amp = __ldg(prony + nexp + e);
      const double cp[4][2] = {{1.0, depth * lam - 2 * depth},
                               {-1.0, -depth * lam},
                               {-1.0, depth * lam - 4 * depth},
                               {1.0, -depth * lam + 2 * depth}};
#pragma unroll 1
      for (int t = 0; t < 4; ++t) {
        reflected_rankine(M, f, adjoint, cp[t][0], cp[t][1], false, g, dg);
        Gre += amp / 2 * g;
        dGre[0] += amp / 2 * dg[0];
        dGre[1] += amp / 2 * dg[1];
        dGre[2] += amp / 2 * dg[2];
      }
    }
    const double sre = kMinusOneOverFourPi * Gre, sim = kMinusOneOverFourPi * Gim;
    S[(size_t)I + (size_t)a.lds * J] = OutT<Out>::make(sre, sim);
    nan_seen |= isnan(sre) || isnan(sim);
    const bool on_diag = a.diagonal_term && I == J && I < diag_limit;
    const size_t kidx = (size_t)I + (size_t)a.ldk * J;
    if (a.early_dot_product) {
      const double* dn = adjoint ? nI : (a.dot_normals_dev + 3 * J);
      double kre = kMinusOneOverFourPi * (dn[0] * dGre[0] + dn[1] * dGre[1] + dn[2] * dGre[2]);
      const double kim = kMinusOneOverFourPi * (dn[0] * dGim[0] + dn[1] * dGim[1] + dn[2] * dGim[2]);
      if (on_diag) kre += diag_coef;
      K[kidx] = OutT<Out>::make(kre, kim);
      nan_seen |= isnan(kre) || isnan(kim);
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double kre = kMinusOneOverFourPi * dGre[c];
        const double kim = kMinusOneOverFourPi * dGim[c];
        if (on_diag) kre += diag_coef * a.dot_normals_dev[3 * I + c];
        K[kidx + (size_t)c * a.k_plane_stride] = OutT<Out>::make(kre, kim);
        nan_seen |= isnan(kre) || isnan(kim);
      }
    }
  }
  if (nan_seen && a.nan_flag_dev) atomicOr(a.nan_flag_dev, 1);
}

}  // namespace
}  // namespace bem

extern "C" int bem_assemble(const bem_assembly_args* args, void* stream) {
  using namespace bem;
  if (!args) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: null args");
  const bem_assembly_args& a = *args;
  if (a.n < 0 || a.nb_faces < 0) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: negative size");
  if (a.n == 0 || a.nb_faces == 0) return BEM_OK;
  if (!a.points_dev || !a.vertices_dev || !a.faces_dev || !a.centers_dev || !a.normals_dev || !a.areas_dev ||
      !a.radii_dev || !a.quad_points_dev || !a.quad_weights_dev || !a.S_dev || !a.K_dev)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: null pointer");
  if (a.nb_quad_points < 1) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: nb_quad_points < 1");
  if (a.lds < a.n || a.ldk < a.n) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: leading dimension < n");
  if (!a.early_dot_product && a.k_plane_stride < a.ldk * (int64_t)a.nb_faces)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: gradient planes overlap");
  if ((a.early_dot_product || a.diagonal_term) && !a.dot_normals_dev)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: dot_normals required");
  const bool rankine_only = std::isinf(a.free_surface);
  const bool finite_k = (a.wavenumber > 0.0) && std::isfinite(a.wavenumber);
  const bool tabulated = a.nr > 1 && a.nz > 1;
  if (!rankine_only && finite_k) {
    if (tabulated && (!a.r_range_dev || !a.z_range_dev || !a.table_dev))
      return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: tabulation pointers missing");
    if (!tabulated && a.tabulation_nb_integration_points <= 0)
      return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: nb_integration_points <= 0");
    if (a.precision == BEM_PREC_MIXED && tabulated && !a.table32_dev)
      return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: mixed precision needs the float32 table");
  }
  const TabView T{a.tabulation_nb_integration_points, a.tabulation_grid_shape, a.nr, a.nz, a.r_range_dev,
                  a.z_range_dev, a.table_dev, a.table32_dev, 0.0, 0.0, a.r_inv_den_dev, a.z_inv_den_dev, 0.0};
  int gf_sing = a.gf_singularities;
  // Singularity variant overrides of delhommeau.py:472-487.
  if (a.wavenumber == 0.0) gf_sing = kLowFreq;
  else if (std::isinf(a.wavenumber)) gf_sing = kHighFreq;
  const double sign_refl = (gf_sing == kHighFreq) ? -1.0 : 1.0;
  dim3 grid(ceil_div(a.n, kRows), ceil_div(a.nb_faces, kTileJ));
  cudaStream_t s = (cudaStream_t)stream;
  const bool mixed = a.precision == BEM_PREC_MIXED;
  if (a.out_dtype == BEM_DTYPE_C128) {
    TimedLaunch tl(kKAssemble, s);
    if (mixed) assemble_kernel<double2, true><<<grid, kRows, 0, s>>>(a, T, a.wavenumber, gf_sing, finite_k, sign_refl);
    else assemble_kernel<double2, false><<<grid, kRows, 0, s>>>(a, T, a.wavenumber, gf_sing, finite_k, sign_refl);
  } else if (a.out_dtype == BEM_DTYPE_C64) {
    TimedLaunch tl(kKAssemble, s);
    if (mixed) assemble_kernel<float2, true><<<grid, kRows, 0, s>>>(a, T, a.wavenumber, gf_sing, finite_k, sign_refl);
    else assemble_kernel<float2, false><<<grid, kRows, 0, s>>>(a, T, a.wavenumber, gf_sing, finite_k, sign_refl);
  } else {
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble: unknown out_dtype");
  }
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}

namespace {
int check_common(const bem_assembly_args& a, const char* who) {
  using namespace bem;
  char msg[200];
  if (a.n <= 0 || a.nb_faces <= 0) {
    std::snprintf(msg, sizeof(msg), "%s: empty mesh", who);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  if (!a.points_dev || !a.vertices_dev || !a.faces_dev || !a.centers_dev || !a.normals_dev || !a.areas_dev ||
      !a.radii_dev || !a.quad_points_dev || !a.quad_weights_dev || !a.dot_normals_dev) {
    std::snprintf(msg, sizeof(msg), "%s: null pointer", who);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  if (std::isinf(a.free_surface) || a.gf_singularities == BEM_GF_LOW_FREQ_WITH_RANKINE_PART || !a.early_dot_product) {
    std::snprintf(msg, sizeof(msg),
                  "%s: needs a free surface, early dot product and gf_singularities high_freq or low_freq", who);
    return set_error(BEM_ERR_UNSUPPORTED, msg);
  }
  return BEM_OK;
}
}  // namespace

extern "C" int bem_assemble_rankine_part(const bem_assembly_args* args, void* out_dev, int64_t ld, void* stream) {
  using namespace bem;
  if (!args || !out_dev) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_rankine_part: null pointer");
  const bem_assembly_args& a = *args;
  int st = check_common(a, "bem_assemble_rankine_part");
  if (st) return st;
  if (ld < a.n) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_rankine_part: ld < n");
  // the reflected-term sign of the variant used at this wavenumber (delhommeau.py:472-487)
  int gf_sing = a.gf_singularities;
  if (a.wavenumber == 0.0) gf_sing = kLowFreq;
  else if (std::isinf(a.wavenumber)) gf_sing = kHighFreq;
  const double sign_refl = (gf_sing == kHighFreq) ? -1.0 : 1.0;
  const TabView T{0, 0, 0, 0, nullptr, nullptr, nullptr, nullptr, 0.0, 0.0, nullptr, nullptr, 0.0};
  dim3 grid(ceil_div(a.n, kRows), ceil_div(a.nb_faces, kTileJ));
  cudaStream_t s = (cudaStream_t)stream;
  {
    TimedLaunch tl(kKAssemble, s);
    assemble_kernel<double2, false, true><<<grid, kRows, 0, s>>>(a, T, a.wavenumber, gf_sing, false, sign_refl,
                                                                 (double2*)out_dev, ld);
  }
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}

namespace bem {
namespace {
// Shared by the single- and multi-wavenumber entry points: checks, then one
// launch per group of up to kSymBatch wavenumbers (grid z = wavenumber).
// planes (optional): float32 copy of K into planes[0 .. nk) (real plane, the
// imaginary plane planes_im floats further, leading dimension planes_ld,
// planes_stride floats between wavenumbers).
int wave_symmetric_launch(const bem_assembly_args* args, const void* rankine_dev, int64_t ld, const double* ks,
                          int nk, int64_t s_stride, int64_t k_stride, void* stream, const char* who,
                          bool general = false, bool inplace = false, float* planes = nullptr,
                          int64_t planes_ld = 0, int64_t planes_stride = 0, int64_t planes_im = 0) {
  char msg[200];
  if (!args || !rankine_dev || !ks || nk <= 0) {
    std::snprintf(msg, sizeof(msg), "%s: null pointer or no wavenumber", who);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  const bem_assembly_args& a = *args;
  int st = check_common(a, who);
  if (st) return st;
  if (!a.S_dev || !a.K_dev) {
    std::snprintf(msg, sizeof(msg), "%s: null output", who);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  if (general) {
    if (a.nb_quad_points != 1 || a.centers_dev != a.quad_points_dev) {
      std::snprintf(msg, sizeof(msg), "%s: needs one quadrature point per face and the same array for the "
                    "centres and the quadrature points", who);
      return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
    }
  } else if (a.n != a.nb_faces || a.nb_quad_points != 1 || a.points_dev != a.quad_points_dev ||
             a.centers_dev != a.quad_points_dev) {
    std::snprintf(msg, sizeof(msg), "%s: needs one mesh, one quadrature point per face, and the same array for "
                  "points, centres and quadrature points", who);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  for (int i = 0; i < nk; ++i)
    if (!(ks[i] > 0.0) || !std::isfinite(ks[i])) {
      std::snprintf(msg, sizeof(msg), "%s: wavenumber must be finite and > 0", who);
      return set_error(BEM_ERR_UNSUPPORTED, msg);
    }
  if (a.out_dtype != BEM_DTYPE_C128 || (a.precision != BEM_PREC_FP64 && a.precision != BEM_PREC_MIXED)) {
    std::snprintf(msg, sizeof(msg), "%s: complex128 outputs only", who);
    return set_error(BEM_ERR_UNSUPPORTED, msg);
  }
  if (a.lds < a.n || a.ldk < a.n || ld < a.n) {
    std::snprintf(msg, sizeof(msg), "%s: leading dimension < n", who);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  if (nk > 1 && (s_stride < a.lds * (int64_t)a.nb_faces || k_stride < a.ldk * (int64_t)a.nb_faces)) {
    std::snprintf(msg, sizeof(msg), "%s: output strides smaller than one matrix", who);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  const bool tabulated = a.nr > 1 && a.nz > 1;
  if (tabulated && (!a.r_range_dev || !a.z_range_dev || !a.table_dev)) {
    std::snprintf(msg, sizeof(msg), "%s: tabulation pointers missing", who);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  if (!tabulated && a.tabulation_nb_integration_points <= 0) {
    std::snprintf(msg, sizeof(msg), "%s: nb_integration_points <= 0", who);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  // float32 wave term: needs the float32 copy of the table (direct integration stays float64)
  const bool f32 = a.precision == BEM_PREC_MIXED && tabulated;
  if (f32 && !a.table32_dev) {
    std::snprintf(msg, sizeof(msg), "%s: mixed precision needs table32_dev", who);
    return set_error(BEM_ERR_INVALID_ARGUMENT, msg);
  }
  const TabView T{a.tabulation_nb_integration_points, a.tabulation_grid_shape, a.nr, a.nz, a.r_range_dev,
                  a.z_range_dev, a.table_dev, a.table32_dev, 0.0, 0.0, a.r_inv_den_dev, a.z_inv_den_dev, 0.0};
  const int nbi = ceil_div(a.n, kSymT), nbj = ceil_div(general ? a.nb_faces : a.n, kSymT);
  cudaStream_t s = (cudaStream_t)stream;
  int launches = 0;
  for (int k0 = 0; k0 < nk; k0 += kSymBatch) {
    const int cnt = std::min(kSymBatch, nk - k0);
    SymBatch kb{};
    for (int i = 0; i < cnt; ++i) kb.k[i] = ks[k0 + i];
    kb.s_stride = s_stride;
    kb.k_stride = k_stride;
    kb.w = planes ? planes + (size_t)k0 * planes_stride : nullptr;
    kb.w_ld = planes_ld;
    kb.w_stride = planes_stride;
    kb.w_im = planes_im;
    bem_assembly_args ak = a;
    ak.S_dev = reinterpret_cast<double2*>(a.S_dev) + (size_t)k0 * s_stride;
    ak.K_dev = reinterpret_cast<double2*>(a.K_dev) + (size_t)k0 * k_stride;
    {
      TimedLaunch tl(kKAssemble, s);
      if (f32 && !general && !inplace)
        wave_symmetric_kernel<false, false, true><<<dim3(nbi, nbj, cnt), kSymT, 0, s>>>(
            ak, T, kb, a.gf_singularities, (const double2*)rankine_dev, ld);
      else if (f32 && !general)
        wave_symmetric_kernel<false, true, true><<<dim3(nbi, nbj, cnt), kSymT, 0, s>>>(
            ak, T, kb, a.gf_singularities, (const double2*)rankine_dev, ld);
      else if (f32)
        wave_symmetric_kernel<true, false, true><<<dim3(nbi, nbj, cnt), kSymT, 0, s>>>(
            ak, T, kb, a.gf_singularities, (const double2*)rankine_dev, ld);
      else if (general)
        wave_symmetric_kernel<true><<<dim3(nbi, nbj, cnt), kSymT, 0, s>>>(ak, T, kb, a.gf_singularities,
                                                                         (const double2*)rankine_dev, ld);
      else if (inplace)
        wave_symmetric_kernel<false, true><<<dim3(nbi, nbj, cnt), kSymT, 0, s>>>(ak, T, kb, a.gf_singularities,
                                                                                (const double2*)rankine_dev, ld);
      else
        wave_symmetric_kernel<false><<<dim3(nbi, nbj, cnt), kSymT, 0, s>>>(ak, T, kb, a.gf_singularities,
                                                                          (const double2*)rankine_dev, ld);
    }
    ++launches;
  }
  count_launches(launches);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}
}  // namespace
}  // namespace bem

extern "C" int bem_assemble_wave_symmetric(const bem_assembly_args* args, const void* rankine_dev, int64_t ld,
                                           void* stream) {
  using namespace bem;
  const double k = args ? args->wavenumber : 0.0;
  return wave_symmetric_launch(args, rankine_dev, ld, &k, 1, 0, 0, stream, "bem_assemble_wave_symmetric");
}

extern "C" int bem_assemble_wave_symmetric_batched(const bem_assembly_args* args, const void* rankine_dev,
                                                   int64_t ld, const double* wavenumbers_host, int nk,
                                                   int64_t s_stride, int64_t k_stride, void* stream) {
  using namespace bem;
  return wave_symmetric_launch(args, rankine_dev, ld, wavenumbers_host, nk, s_stride, k_stride, stream,
                               "bem_assemble_wave_symmetric_batched");
}

extern "C" int bem_assemble_wave_symmetric_batched_lu(const bem_assembly_args* args, const void* rankine_dev,
                                                      int64_t ld, const double* wavenumbers_host, int nk,
                                                      int64_t s_stride, int64_t k_stride, void* lu_work_dev,
                                                      int npad, int first, void* stream) {
  using namespace bem;
  if (!args || !lu_work_dev || npad < args->n || npad % 128 || first < 0)
    return set_error(BEM_ERR_INVALID_ARGUMENT,
                     "bem_assemble_wave_symmetric_batched_lu: bad workspace arguments (npad a multiple of 128, "
                     ">= n)");
  float* re = nullptr;
  int64_t pld = 0, pstride = 0, pim = 0;
  int st = clu_planes(lu_work_dev, npad, &re, &pld, &pstride, &pim);
  if (st) return st;
  return wave_symmetric_launch(args, rankine_dev, ld, wavenumbers_host, nk, s_stride, k_stride, stream,
                               "bem_assemble_wave_symmetric_batched_lu", false, false,
                               re + (size_t)first * pstride, pld, pstride, pim);
}

extern "C" int bem_assemble_wave_cached(const bem_assembly_args* args, const void* rankine_dev, int64_t ld,
                                        const double* wavenumbers_host, int nk, int64_t s_stride, int64_t k_stride,
                                        void* stream) {
  using namespace bem;
  return wave_symmetric_launch(args, rankine_dev, ld, wavenumbers_host, nk, s_stride, k_stride, stream,
                               "bem_assemble_wave_cached", true);
}

extern "C" int bem_assemble_symmetric(const bem_assembly_args* args, void* stream) {
  using namespace bem;
  if (!args || !args->K_dev) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_symmetric: null pointer");
  const bem_assembly_args& a = *args;
  if (a.n != a.nb_faces || a.nb_quad_points != 1 || a.points_dev != a.quad_points_dev ||
      a.centers_dev != a.quad_points_dev)
    return set_error(BEM_ERR_INVALID_ARGUMENT,
                     "bem_assemble_symmetric: needs one mesh, one quadrature point per face, and the same array for "
                     "points, centres and quadrature points");
  if (a.out_dtype != BEM_DTYPE_C128 || a.precision != BEM_PREC_FP64)
    return set_error(BEM_ERR_UNSUPPORTED, "bem_assemble_symmetric: complex128 outputs, float64 only");
  if (!(a.wavenumber > 0.0) || !std::isfinite(a.wavenumber))
    return set_error(BEM_ERR_UNSUPPORTED, "bem_assemble_symmetric: wavenumber must be finite and > 0");
  // the Rankine part into K (same leading dimension), then the wave term in place
  int st = bem_assemble_rankine_part(args, a.K_dev, a.ldk, stream);
  if (st) return st;
  const double k = a.wavenumber;
  return wave_symmetric_launch(args, a.K_dev, a.ldk, &k, 1, 0, 0, stream, "bem_assemble_symmetric", false, true);
}

extern "C" int bem_assemble_finite_depth(const bem_assembly_args* args, double depth, int method,
                                         const double* prony_dev, int nexp, void* stream) {
  using namespace bem;
  if (!args) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: null args");
  const bem_assembly_args& a = *args;
  if (a.n < 0 || a.nb_faces < 0) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: negative size");
  if (a.n == 0 || a.nb_faces == 0) return BEM_OK;
  if (!a.points_dev || !a.vertices_dev || !a.faces_dev || !a.centers_dev || !a.normals_dev || !a.areas_dev ||
      !a.radii_dev || !a.quad_points_dev || !a.quad_weights_dev || !a.S_dev || !a.K_dev || !a.dot_normals_dev)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: null pointer");
  if (!(depth > 0.0) || !std::isfinite(depth))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: depth must be finite and > 0");
  if (std::isinf(a.free_surface))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: a finite depth needs a free surface");
  if (nexp < 0 || nexp > 64 || (nexp > 0 && !prony_dev))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: 0 to 64 Prony terms");
  if (method != 0 && method != 1)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: method 0 (legacy) or 1 (newer)");
  if (a.precision != BEM_PREC_FP64)
    return set_error(BEM_ERR_UNSUPPORTED, "bem_assemble_finite_depth: float64 arithmetic only");
  if (a.out_dtype != BEM_DTYPE_C128 && a.out_dtype != BEM_DTYPE_C64)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: unknown out_dtype");
  if (a.nb_quad_points < 1 || a.lds < a.n || a.ldk < a.n)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: quadrature or leading dimension");
  if (!a.early_dot_product && a.k_plane_stride < a.ldk * (int64_t)a.nb_faces)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: gradient planes overlap");
  if (!(a.wavenumber >= 0.0))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: wavenumber must be >= 0");
  const bool tabulated = a.nr > 1 && a.nz > 1;
  const bool finite_k = a.wavenumber > 0.0 && std::isfinite(a.wavenumber);
  if (finite_k && tabulated && (!a.r_range_dev || !a.z_range_dev || !a.table_dev))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: tabulation pointers missing");
  if (finite_k && !tabulated && a.tabulation_nb_integration_points <= 0)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: nb_integration_points <= 0");
  const TabView T{a.tabulation_nb_integration_points, a.tabulation_grid_shape, a.nr, a.nz, a.r_range_dev,
                  a.z_range_dev, a.table_dev, a.table32_dev, 0.0, 0.0, a.r_inv_den_dev, a.z_inv_den_dev, 0.0};
  // the caller picks the variant (delhommeau.py:467-487: the legacy method
  // takes low_freq before the wavenumber rules apply)
  const int gf_sing = a.gf_singularities;
  if (gf_sing < kHighFreq || gf_sing > kLowFreqWithRankinePart)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_assemble_finite_depth: unknown gf_singularities");
  dim3 grid(ceil_div(a.n, kRows), ceil_div(a.nb_faces, kTileJ));
  cudaStream_t s = (cudaStream_t)stream;
  {
    TimedLaunch tl(kKAssemble, s);
    if (a.out_dtype == BEM_DTYPE_C128)
      assemble_finite_depth_kernel<double2><<<grid, kRows, 0, s>>>(a, T, depth, method == 0 ? 1 : 0, prony_dev, nexp,
                                                                   gf_sing);
    else
      assemble_finite_depth_kernel<float2><<<grid, kRows, 0, s>>>(a, T, depth, method == 0 ? 1 : 0, prony_dev, nexp,
                                                                  gf_sing);
  }
  count_launches(1);
  BEM_CUDA_CHECK(cudaGetLastError());
  return BEM_OK;
}
