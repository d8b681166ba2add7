// ORACLE — test infrastructure only.
//
// CPU restatement of the infinite-depth path of Capytaine's libDelhommeau
// (Fortran 90 + OpenMP).  Only the test suite, the smoke check and the CPU
// baseline leg of the benchmark load this library; the product path never
// does.  Every function names the reference routine it follows, by
// file:line inside libs/libDelhommeau/src of the capytaine project.
//
// Fidelity notes (Fortran semantics that change numbers):
//  * Literals without a kind suffix are default REAL (single precision) in
//    Fortran, so PI and EULER_GAMMA are float values promoted to double
//    (constants.f90:26-28), and thresholds such as 1e-3, 1e-4, 1e-5, 1e-7,
//    1e-8, 1e-10 compare against float-rounded values.
//  * NORM2 follows gfortran's scaled accumulation, HYPOT is libm hypot.
//  * NINT rounds half away from zero (lround), INT truncates.
//  * exp(z)E1(z) is evaluated in single-precision complex arithmetic with the
//    range-reduced (Smith) complex division that gfortran emits
//    (Delhommeau_integrals.f90:104-151).
//  * Built with -ffp-contract=off so every operation rounds on its own.
#include <cmath>
#include <vector>
#include <cstdint>
#include <cstring>
#include <climits>
#include <omp.h>
#include <complex>

namespace {

using f32 = float;
using f64 = double;

// constants.f90:22-32
const f64 ZERO = 0.0;
const f64 ONE = 1.0;
const f64 PI = (f64)(f32)3.141592653588979;          // default-real literal
const f64 MINUS_ONE_OVER_FOURPI = -ONE / (4 * PI);
const f64 EULER_GAMMA = (f64)(f32)0.5772156649;      // default-real literal
const f64 LOG_2 = std::log(2.0);
constexpr int NB_TAB = 5;
// constants.f90:40-52
constexpr int LEGACY_GRID = 0;
constexpr int SCALED_NEMOH3_GRID = 1;
constexpr int HIGH_FREQ = 0;
constexpr int LOW_FREQ = 1;
constexpr int LOW_FREQ_WITH_RANKINE_PART = 2;

inline f64 lit(f32 x) { return (f64)x; }  // promote a default-real literal

// ---------------------------------------------------------------------------
// Small complex types with explicit Fortran-like arithmetic.
struct c32 { f32 re, im; };
struct c64 { f64 re, im; };

inline c32 cadd(c32 a, c32 b) { return {a.re + b.re, a.im + b.im}; }
inline c32 cmul(c32 a, c32 b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline c32 radd(f32 r, c32 b) { return {r + b.re, b.im}; }
inline c32 rmul(f32 r, c32 b) { return {r * b.re, r * b.im}; }
// Range-reduced complex division (Smith), as emitted by gfortran.
template <class T, class C>
inline C smith_div(T a, T b, T c, T d) {
  if (std::fabs(c) < std::fabs(d)) {
    T ratio = c / d;
    T div = (c * ratio) + d;
    T tr = (a * ratio) + b;
    T ti = (b * ratio) - a;
    return C{tr / div, ti / div};
  } else {
    T ratio = d / c;
    T div = (d * ratio) + c;
    T tr = (b * ratio) + a;
    T ti = b - (a * ratio);
    return C{tr / div, ti / div};
  }
}
inline c32 cdiv(c32 x, c32 y) { return smith_div<f32, c32>(x.re, x.im, y.re, y.im); }
inline c64 cdiv64(c64 x, c64 y) { return smith_div<f64, c64>(x.re, x.im, y.re, y.im); }
inline c32 clog32(c32 z) {
  // LOG of a COMPLEX(4) value: gfortran calls the C library's clogf.
  std::complex<float> w = std::log(std::complex<float>(z.re, z.im));
  return {w.real(), w.imag()};
}

// gfortran NORM2: scaled sum of squares.
inline f64 norm2(const f64* x, int n) {
  f64 scale = 0.0, result = 1.0;
  for (int i = 0; i < n; ++i) {
    if (x[i] != 0.0) {
      f64 ax = std::fabs(x[i]);
      if (scale < ax) {
        f64 v = scale / ax;
        result = 1.0 + result * v * v;
        scale = ax;
      } else {
        f64 v = ax / scale;
        result += v * v;
      }
    }
  }
  return scale * std::sqrt(result);
}
inline f64 norm2_3(f64 a, f64 b, f64 c) { f64 v[3] = {a, b, c}; return norm2(v, 3); }
inline f64 norm2_2(f64 a, f64 b) { f64 v[2] = {a, b}; return norm2(v, 2); }

// Fortran NINT / INT to default integer, saturating non-finite values the way
// the subsequent clamp to [2, n-1] treats them.
inline int f_nint(f64 x) {
  if (!(x == x)) return INT_MIN;
  if (x >= 2147483647.0) return INT_MAX;
  if (x <= -2147483648.0) return INT_MIN;
  return (int)std::lround(x);
}
inline int f_int(f64 x) {
  if (!(x == x)) return INT_MIN;
  if (x >= 2147483647.0) return INT_MAX;
  if (x <= -2147483648.0) return INT_MIN;
  return (int)x;
}

// ---------------------------------------------------------------------------
// Delhommeau_integrals.f90:104-151  exp(z)*E1(z) in single precision.
c64 exp_e1(c64 zz) {
  c32 z{(f32)zz.re, (f32)zz.im};
  c32 g;
  if (z.re < -16.0f) {                       // case 1
    c32 y = cdiv(c32{1.0f, 0.0f}, z);
    c32 t = rmul(-120.0f, y);                // y*(-120.)
    t = cmul(y, radd(24.0f, t));
    t = cmul(y, radd(-6.0f, t));
    t = cmul(y, radd(2.0f, t));
    t = cmul(y, radd(-1.0f, t));
    g = cmul(y, radd(1.0f, t));
  } else if (std::fabs(z.im) > 10.0f) {      // case 3
    c32 a = cdiv(c32{0.711093f, 0.0f}, radd(0.415775f, z));
    c32 b = cdiv(c32{0.278518f, 0.0f}, radd(2.29428f, z));
    c32 c = cdiv(c32{0.010389f, 0.0f}, radd(6.2900f, z));
    g = cadd(cadd(a, b), c);
  } else if (z.re > -0.5f) {                 // case 2
    c32 p1 = rmul(0.97087007e-05f, z);
    p1 = cmul(z, radd(0.763297e-03f, p1));
    p1 = cmul(z, radd(0.206543e-01f, p1));
    p1 = cmul(z, radd(0.23721365e+00f, p1));
    p1 = radd(0.1e+01f, p1);
    c32 p2 = rmul(-0.51801555e-03f, z);
    p2 = cmul(z, radd(0.19387339e-02f, p2));
    p2 = cmul(z, radd(-0.3000591e-01f, p2));
    p2 = cmul(z, radd(0.41806426e-01f, p2));
    p2 = cmul(z, radd(-0.149545886e+01f, p2));
    p2 = radd(0.99999207e+00f, p2);
    c32 q = rmul(0.2989204e-03f, z);
    q = cmul(z, radd(-0.8700861e-03f, q));
    q = cmul(z, radd(0.12982719e-01f, q));
    q = cmul(z, radd(-0.66786033e-01f, q));
    q = cmul(z, radd(0.28388363e+00f, q));
    q = cmul(z, radd(-0.76273617e+00f, q));
    q = radd(0.1e+01f, q);
    c32 num = cadd(cmul(clog32(z), p1), rmul(0.5772156649e+00f, p2));
    c32 r = cdiv(num, q);
    g = c32{-r.re, -r.im};
  } else {                                   // case 4
    const f32 s = (z.im < 0.0f) ? 1.0f : -1.0f;  // conjugate coefficients when Im z >= 0
    const c32 A[8] = {{1.000000f, s * 1.3935496e-06f}, {15.82958f, -s * 20.14222f},
                      {-70.52863f, -s * 227.9511f},    {-985.4221f, -s * 226.6272f},
                      {-1202.318f, s * 1580.907f},     {953.2441f, s * 1342.447f},
                      {417.3716f, -s * 196.6665f},     {-9.881266f, -s * 24.24952f}};
    const c32 B[9] = {{1.000000f, 0.0f},             {16.83184f, -s * 20.14481f},
                      {-55.66969f, -s * 248.1167f},  {-1068.640f, -s * 434.4707f},
                      {-2082.250f, s * 1522.471f},   {383.3455f, s * 2730.378f},
                      {1216.791f, s * 351.7189f},    {115.3926f, -s * 161.2647f},
                      {-3.777369f, -s * 4.510900f}};
    c32 num = cmul(A[0], z);
    for (int i = 1; i < 8; ++i) {
      num = cadd(num, A[i]);
      if (i < 7) num = cmul(num, z);
    }
    c32 den = cmul(B[0], z);
    for (int i = 1; i < 9; ++i) {
      den = cadd(den, B[i]);
      if (i < 8) den = cmul(den, z);
    }
    g = cdiv(num, den);
  }
  return c64{(f64)g.re, (f64)g.im};
}

// Delhommeau_integrals.f90:43-100
void numerical_integration(f64 r, f64 z, int nb_integration_points, f64* out) {
  f64 I[NB_TAB] = {0, 0, 0, 0, 0};
  int n = (nb_integration_points % 2 == 0) ? nb_integration_points + 1 : nb_integration_points;
  for (int k = 1; k <= n; ++k) {
    f64 km1 = (f64)(f32)((f32)k - 1.0f);
    f64 nm1 = (f64)(f32)((f32)n - 1.0f);
    f64 theta = -PI / 2 + PI * km1 / nm1;
    f64 three_nm1 = (f64)(3.0f * (f32)nm1);
    f64 delta_theta;
    if (k == 1 || k == n) delta_theta = PI / three_nm1;
    else if (k % 2 == 0) delta_theta = 4 * PI / three_nm1;
    else delta_theta = 2 * PI / three_nm1;
    f64 cos_theta = std::cos(theta);
    c64 zeta{z, r * cos_theta};
    c64 exp_zeta;
    if (zeta.re <= -30.0) {
      exp_zeta = {0.0, 0.0};
    } else {
      f64 e = std::exp(zeta.re);
      exp_zeta = {e * std::cos(zeta.im), e * std::sin(zeta.im)};
    }
    c64 e1 = exp_e1(zeta);
    // ii*pi*exp_zeta = (0, pi) * exp_zeta
    c64 ipe{0.0 * exp_zeta.re - PI * exp_zeta.im, 0.0 * exp_zeta.im + PI * exp_zeta.re};
    c64 jzeta{e1.re + ipe.re, e1.im + ipe.im};
    c64 inv = cdiv64(c64{1.0, 0.0}, zeta);
    c64 jm{jzeta.re - inv.re, jzeta.im - inv.im};
    I[0] = I[0] + delta_theta * jzeta.re;
    I[1] = I[1] + delta_theta * jm.re;
    I[2] = I[2] + delta_theta * exp_zeta.re;
    I[3] = I[3] - delta_theta * cos_theta * jm.im;
    I[4] = I[4] - delta_theta * cos_theta * exp_zeta.im;
  }
  I[0] = I[0] / PI;
  I[1] = I[1] / PI;
  I[3] = I[3] / PI;
  for (int i = 0; i < NB_TAB; ++i) out[i] = 2 * I[i];
}

// Delhommeau_integrals.f90:157-186
void asymptotic_approximations(f64 r, f64 z, f64* out) {
  f64 one_over_r = 1 / std::fmax(r, lit(1e-10f));
  f64 one_over_r1 = 1 / std::hypot(r, z);
  f64 expz_sqr = std::exp(z) * std::sqrt(2 * PI * one_over_r);
  f64 cos_kr = std::cos(r - PI / 4);
  f64 sin_kr = std::sin(r - PI / 4);
  f64 r13 = one_over_r1 * one_over_r1 * one_over_r1;
  out[0] = -expz_sqr * sin_kr + z * r13 - one_over_r1;
  out[1] = -expz_sqr * sin_kr + z * r13;
  out[2] = expz_sqr * cos_kr;
  out[3] = -expz_sqr * (cos_kr - sin_kr * one_over_r / 2) + r * r13;
  out[4] = -expz_sqr * (sin_kr + cos_kr * one_over_r / 2);
  for (int i = 0; i < NB_TAB; ++i) out[i] = 2 * out[i];
}

// Delhommeau_integrals.f90:208-243
void default_r_spacing(int nr, f64 rmax, int method, f64* out) {
  const int nr_ref = 676, index_of_1_ref = 81;
  if (nr <= 0) return;
  out[0] = 0.0;
  if (method == LEGACY_GRID) {
    for (int i = 2; i <= nr; ++i) {
      f32 a = std::pow(10.0f, ((f32)i - 1.0f) / 5.0f - 6.0f);
      f32 b = (f32)std::abs(i - 32) / 3.0f + 4.0f / 3.0f;
      out[i - 1] = (f64)std::fmin(a, b);
    }
  } else {
    int index_of_1 = (int)std::lround((f32)((f32)nr * 1.0f / (f32)nr_ref * (f32)index_of_1_ref));
    for (int i = 1; i <= nr; ++i) {
      if (i < index_of_1) {
        f32 e = -10.0f * (1.0f - (f32)(i - 1) / (f32)(index_of_1 - 1));
        out[i - 1] = (f64)std::pow(10.0f, e);
      } else {
        out[i - 1] = (rmax - 1.0) / (f64)(nr - index_of_1) * (f64)(i - index_of_1) + 1.0;
      }
    }
  }
}

// Delhommeau_integrals.f90:247-270
void default_z_spacing(int nz, f64 zmin, int method, f64* out) {
  if (nz <= 0) return;
  if (method == LEGACY_GRID) {
    for (int j = 1; j <= nz; ++j) {
      f32 a = std::pow(10.0f, (f32)j / 5.0f - 6.0f);
      f32 b = std::pow(10.0f, (f32)j / 8.0f - 4.5f);
      out[j - 1] = -(f64)std::fmin(a, b);
    }
    if (nz == 46) out[45] = -16.0;
  } else {
    f64 dz = (std::log10(std::fabs(zmin)) + 10.0) / (f64)nz;
    for (int j = 1; j <= nz; ++j) {
      out[j - 1] = -std::fmin(std::pow(10.0, dz * (f64)j - 10.0), std::fabs(zmin));
    }
  }
}

// Delhommeau_integrals.f90:301-335 (1-based result)
int nearest_r_index(f64 r, const f64* r_range, int nr, int method) {
  if (method == LEGACY_GRID) {
    if (r < lit(1e-6f)) return 1;
    if (r < 1.0) return f_int(5 * (std::log10(r) + 6) + 1);
    return f_int(3 * r + 28);
  }
  const int nr_ref = 676, index_of_1_ref = 81;
  int index_of_1 = (int)std::lround((f32)(nr * index_of_1_ref) / (f32)nr_ref);
  f64 rmax = r_range[nr - 1];
  if (r < lit(1e-10f)) return 1;
  if (r < 1.0) return f_nint((std::log10(r) / 10.0 + 1.0) * (f64)(index_of_1 - 1) + 1);
  return f_nint((r - 1) * (f64)(nr - index_of_1) / (rmax - 1) + (f64)index_of_1);
}

// Delhommeau_integrals.f90:339-363 (1-based result)
int nearest_z_index(f64 z, const f64* z_range, int nz, int method) {
  f64 absz = std::fabs(z);
  if (method == LEGACY_GRID) {
    if (absz > lit(1e-2f)) return f_int(8 * (std::log10(absz) + 4.5));
    return f_int(5 * (std::log10(absz) + 6));
  }
  f64 dz = (std::log10(std::fabs(z_range[nz - 1])) + 10.0) / (f64)nz;
  return f_nint((std::log10(absz) + 10) / dz);
}

inline f64 pl2(f64 u1, f64 u2, f64 u3, f64 xu) { return ((xu - u1) * (xu - u2)) / ((u3 - u1) * (u3 - u2)); }

// Table layout: C-contiguous (nr, nz, 5), value(i, j, k) at (i*nz + j)*5 + k.
// Delhommeau_integrals.f90:274-297 and 367-402
void pick_in_default_tabulation(f64 r, f64 z, int method, const f64* r_range, int nr, const f64* z_range,
                                int nz, const f64* tab, f64* out) {
  int i = nearest_r_index(r, r_range, nr, method);
  i = i < nr - 1 ? i : nr - 1;
  i = i > 2 ? i : 2;
  int j = nearest_z_index(z, z_range, nz, method);
  j = j < nz - 1 ? j : nz - 1;
  j = j > 2 ? j : 2;
  // 0-based centre indices
  int ic = i - 1, jc = j - 1;
  const f64 r1 = r_range[ic - 1], r2 = r_range[ic], r3 = r_range[ic + 1];
  const f64 z1 = z_range[jc - 1], z2 = z_range[jc], z3 = z_range[jc + 1];
  f64 xl[3] = {pl2(r2, r3, r1, r), pl2(r3, r1, r2, r), pl2(r1, r2, r3, r)};
  f64 zl[3] = {pl2(z2, z3, z1, z), pl2(z3, z1, z2, z), pl2(z1, z2, z3, z)};
  for (int k = 0; k < NB_TAB; ++k) {
    f64 v[3];
    for (int a = 0; a < 3; ++a) {
      const f64* row = tab + ((size_t)(ic - 1 + a) * nz + (jc - 1)) * NB_TAB + k;
      v[a] = row[0] * zl[0] + row[NB_TAB] * zl[1] + row[2 * NB_TAB] * zl[2];
    }
    out[k] = xl[0] * v[0] + xl[1] * v[1] + xl[2] * v[2];
  }
}

struct Tabulation {
  int npts;
  int grid;
  const f64* r_range;
  int nr;
  const f64* z_range;
  int nz;
  const f64* tab;
};

// Green_wave.f90:162-271
void wave_part_infinite_depth(const f64* x0i, const f64* x0j, f64 k, const Tabulation& T, int gf_sing,
                              c64& G, c64* nablaG) {
  f64 r = k * norm2_2(x0i[0] - x0j[0], x0i[1] - x0j[1]);
  f64 z = k * (x0i[2] + x0j[2]);
  f64 r1 = std::hypot(r, z);
  f64 drdx1, drdx2;
  const f64 eps = 2.220446049250313e-16;  // EPSILON(1d0)
  if (std::fabs(r) > 16 * eps) {
    drdx1 = k * k * (x0i[0] - x0j[0]) / r;
    drdx2 = k * k * (x0i[1] - x0j[1]) / r;
  } else {
    drdx1 = ZERO;
    drdx2 = ZERO;
  }
  f64 dzdx3 = k;
  f64 I[NB_TAB];
  if (T.nz <= 1 || T.nr <= 1) {
    numerical_integration(r, z, T.npts, I);
  } else if (std::fabs(z) < std::fabs(T.z_range[T.nz - 1]) && r < T.r_range[T.nr - 1]) {
    pick_in_default_tabulation(r, z, T.grid, T.r_range, T.nr, T.z_range, T.nz, T.tab, I);
  } else {
    asymptotic_approximations(r, z, I);
  }
  if (gf_sing == LOW_FREQ || gf_sing == LOW_FREQ_WITH_RANKINE_PART) {
    G = {I[0], I[2]};
    c64 dGdr{I[3], I[4]};
    nablaG[0] = {drdx1 * dGdr.re, drdx1 * dGdr.im};
    nablaG[1] = {drdx2 * dGdr.re, drdx2 * dGdr.im};
    if (gf_sing == LOW_FREQ) {
      nablaG[2] = {dzdx3 * (G.re + 2 / r1), dzdx3 * G.im};
    } else {
      nablaG[2] = {dzdx3 * G.re, dzdx3 * G.im};
    }
  } else {  // HIGH_FREQ
    G = {I[1], I[2]};
    c64 dGdr{I[3], I[4]};
    f64 r13 = r1 * r1 * r1;
    nablaG[0] = {drdx1 * dGdr.re - 2 * drdx1 * r / r13, drdx1 * dGdr.im};
    nablaG[1] = {drdx2 * dGdr.re - 2 * drdx2 * r / r13, drdx2 * dGdr.im};
    nablaG[2] = {dzdx3 * G.re - 2 * dzdx3 * z / r13, dzdx3 * G.im};
  }
  G = {k * G.re, k * G.im};
  for (int c = 0; c < 3; ++c) nablaG[c] = {k * nablaG[c].re, k * nablaG[c].im};
}

// Green_wave.f90:128-158
void integral_of_singularity_on_free_surface(f64 face_area, f64 k, c64& int_G, c64* int_nablaG) {
  f64 re = (1 - std::log(k * k * face_area / PI)) + 2 * (EULER_GAMMA - LOG_2);
  f64 im = -2 * PI;
  f64 ka = k * face_area;
  int_G = {ka * re, ka * im};
  int_nablaG[0] = {0.0, 0.0};
  int_nablaG[1] = {0.0, 0.0};
  int_nablaG[2] = {k * (int_G.re + 4 * std::sqrt(PI * face_area)), k * int_G.im};
}

// Green_wave.f90:50-124
void integral_of_wave_part_infinite_depth(const f64* x, const f64* face_center, f64 face_area, int nq,
                                          const f64* quad_points /* (nq,3) */, const f64* quad_weights, f64 k,
                                          const Tabulation& T, int gf_sing, bool deriv_first, c64& int_G,
                                          c64* int_nablaG) {
  f64 r = k * norm2_2(x[0] - face_center[0], x[1] - face_center[1]);
  f64 z = k * (x[2] + face_center[2]);
  if (std::fabs(r) < lit(1e-10f) && std::fabs(z) < lit(1e-10f)) {
    integral_of_singularity_on_free_surface(face_area, k, int_G, int_nablaG);
  } else {
    int_G = {0, 0};
    for (int c = 0; c < 3; ++c) int_nablaG[c] = {0, 0};
    for (int q = 0; q < nq; ++q) {
      c64 G, nG[3];
      wave_part_infinite_depth(x, quad_points + 3 * q, k, T, gf_sing, G, nG);
      f64 w = quad_weights[q];
      int_G = {int_G.re + G.re * w, int_G.im + G.im * w};
      for (int c = 0; c < 3; ++c) int_nablaG[c] = {int_nablaG[c].re + nG[c].re * w, int_nablaG[c].im + nG[c].im * w};
    }
  }
  if (!deriv_first) {
    int_nablaG[0] = {-int_nablaG[0].re, -int_nablaG[0].im};
    int_nablaG[1] = {-int_nablaG[1].re, -int_nablaG[1].im};
  }
}

// Green_Rankine.f90:68-157
void exact_integral_of_Rankine(const f64* M, const f64* nodes /* (4,3) */, const f64* c, const f64* n,
                               f64 area, f64 R, bool deriv_first, f64& int_G, f64* int_nabla_G) {
  (void)area;
  static const int next_node[4] = {1, 2, 3, 0};
  f64 GZ = (M[0] - c[0]) * n[0] + (M[1] - c[1]) * n[1] + (M[2] - c[2]) * n[2];
  f64 RR[4], DRX[4][3];
  for (int L = 0; L < 4; ++L) {
    f64 d[3] = {M[0] - nodes[3 * L], M[1] - nodes[3 * L + 1], M[2] - nodes[3 * L + 2]};
    RR[L] = norm2(d, 3);
    for (int a = 0; a < 3; ++a) DRX[L][a] = d[a] / RR[L];
  }
  int_G = ZERO;
  int_nabla_G[0] = int_nabla_G[1] = int_nabla_G[2] = ZERO;
  const f64 sgn = std::copysign(ONE, GZ);
  const f64 aGZ = std::fabs(GZ);
  for (int L = 0; L < 4; ++L) {
    const int Ln = next_node[L];
    f64 e[3] = {nodes[3 * Ln] - nodes[3 * L], nodes[3 * Ln + 1] - nodes[3 * L + 1], nodes[3 * Ln + 2] - nodes[3 * L + 2]};
    f64 DK = norm2(e, 3);
    if (DK >= lit(1e-3f) * R) {
      f64 PJ[3] = {e[0] / DK, e[1] / DK, e[2] / DK};
      f64 GYX[3] = {n[1] * PJ[2] - n[2] * PJ[1], n[2] * PJ[0] - n[0] * PJ[2], n[0] * PJ[1] - n[1] * PJ[0]};
      f64 GY = (M[0] - nodes[3 * L]) * GYX[0] + (M[1] - nodes[3 * L + 1]) * GYX[1] + (M[2] - nodes[3 * L + 2]) * GYX[2];
      f64 S = RR[Ln] + RR[L];
      f64 ANT = 2 * GY * DK;
      f64 DNT = S * S - DK * DK + 2 * aGZ * S;
      f64 ANL = S + DK;
      f64 DNL = S - DK;
      f64 ALDEN = std::log(ANL / DNL);
      f64 AT = (aGZ >= lit(1e-4f) * R) ? std::atan(ANT / DNT) : 0.0;
      f64 ANLX[3], ANTX[3], DNTX[3];
      for (int a = 0; a < 3; ++a) {
        ANLX[a] = DRX[Ln][a] + DRX[L][a];
        ANTX[a] = 2 * DK * GYX[a];
      }
      for (int a = 0; a < 3; ++a) DNTX[a] = 2 * (S + aGZ) * ANLX[a] + 2 * sgn * S * n[a];
      if (std::fabs(GY) < lit(1e-5f)) {
        int_G = int_G - 2 * AT * aGZ;
      } else {
        int_G = int_G + GY * ALDEN - 2 * AT * aGZ;
      }
      const f64 c1 = GY * (DNL - ANL) / (ANL * DNL);
      const f64 den = ANT * ANT + DNT * DNT;
      for (int a = 0; a < 3; ++a) {
        int_nabla_G[a] = int_nabla_G[a] + ALDEN * GYX[a] - 2 * sgn * AT * n[a] + c1 * ANLX[a] -
                         2 * aGZ * (ANTX[a] * DNT - DNTX[a] * ANT) / den;
      }
    }
  }
  if (!deriv_first) {
    for (int a = 0; a < 3; ++a) int_nabla_G[a] = -int_nabla_G[a];
  }
}

// Green_Rankine.f90:161-198
void one_point_integral_of_Rankine(const f64* M, const f64* c, f64 area, bool deriv_first, f64& int_G,
                                   f64* int_nabla_G) {
  f64 vo[3] = {c[0] - M[0], c[1] - M[1], c[2] - M[2]};
  f64 ro = norm2(vo, 3);
  if (ro > lit(1e-7f)) {
    int_G = area / ro;
    f64 ro2 = ro * ro;
    for (int a = 0; a < 3; ++a) int_nabla_G[a] = vo[a] * int_G / ro2;
  } else {
    int_G = ZERO;
    int_nabla_G[0] = int_nabla_G[1] = int_nabla_G[2] = ZERO;
  }
  if (!deriv_first) {
    for (int a = 0; a < 3; ++a) int_nabla_G[a] = -int_nabla_G[a];
  }
}

// Green_Rankine.f90:28-64
void integral_of_Rankine(const f64* M, const f64* nodes, const f64* c, const f64* n, f64 area, f64 R,
                         bool deriv_first, f64& int_G, f64* int_nabla_G) {
  f64 r0 = norm2_3(M[0] - c[0], M[1] - c[1], M[2] - c[2]);
  if (r0 > 7 * R) {
    one_point_integral_of_Rankine(M, c, area, deriv_first, int_G, int_nabla_G);
  } else {
    exact_integral_of_Rankine(M, nodes, c, n, area, R, deriv_first, int_G, int_nabla_G);
  }
}

// Green_Rankine.f90:202-243, 247-296, 300-338
void integral_of_reflected_Rankine(const f64* M, const f64* nodes, const f64* c, const f64* n, f64 area, f64 R,
                                   bool deriv_first, f64 c0, f64 c1, f64& int_G, f64* int_nabla_G) {
  f64 r1 = std::hypot(norm2_2(M[0] - c[0], M[1] - c[1]), c0 * M[2] + c1 - c[2]);
  f64 Mr[3] = {M[0], M[1], c0 * M[2] + c1};
  if (r1 > 7 * R) {
    one_point_integral_of_Rankine(Mr, c, area, true, int_G, int_nabla_G);
  } else {
    exact_integral_of_Rankine(Mr, nodes, c, n, area, R, true, int_G, int_nabla_G);
  }
  int_nabla_G[2] = c0 * int_nabla_G[2];
  if (!deriv_first) {
    int_nabla_G[0] = -int_nabla_G[0];
    int_nabla_G[1] = -int_nabla_G[1];
    if (c0 > 0) int_nabla_G[2] = -int_nabla_G[2];
  }
}

// Green_Rankine.f90:300-338: one-point term at the image c0 z + c1 of M.
void one_point_integral_of_reflected_Rankine(const f64* M, const f64* c, f64 area, bool deriv_first, f64 c0, f64 c1,
                                             f64& int_G, f64* int_nabla_G) {
  f64 Mr[3] = {M[0], M[1], c0 * M[2] + c1};
  one_point_integral_of_Rankine(Mr, c, area, true, int_G, int_nabla_G);
  int_nabla_G[2] = c0 * int_nabla_G[2];
  if (!deriv_first) {
    int_nabla_G[0] = -int_nabla_G[0];
    int_nabla_G[1] = -int_nabla_G[1];
    if (c0 > 0) int_nabla_G[2] = -int_nabla_G[2];
  }
}

// Green_wave.f90:283-290: image of a point through the sea bottom z = -depth.
inline void bottom_image(const f64* x, f64 depth, f64* y) {
  y[0] = x[0];
  y[1] = x[1];
  y[2] = -x[2] - 2 * depth;
}

// Green_wave.f90:311-425: four infinite-depth wave terms (point and face, each
// possibly reflected through the sea bottom), scaled by Delhommeau's factor.
void integral_of_wave_parts_finite_depth(const f64* x, const f64* face_center, f64 face_area, int nq,
                                         const f64* quad_points, const f64* quad_weights, f64 k, f64 depth,
                                         const Tabulation& T, int gf_sing, bool deriv_first, c64& int_G,
                                         c64* int_nablaG) {
  f64 x_sym[3], c_sym[3];
  bottom_image(x, depth, x_sym);
  bottom_image(face_center, depth, c_sym);
  std::vector<f64> q_sym(3 * (size_t)nq);
  for (int q = 0; q < nq; ++q) bottom_image(quad_points + 3 * q, depth, q_sym.data() + 3 * q);
  int_G = {0, 0};
  for (int a = 0; a < 3; ++a) int_nablaG[a] = {0, 0};
  // (point, face, gradient's z component flipped?)
  struct Term { const f64* p; const f64* c; const f64* q; bool flip_z; };
  const Term terms[4] = {
      {x, face_center, quad_points, false},
      {x_sym, face_center, quad_points, deriv_first},
      {x, c_sym, q_sym.data(), !deriv_first},
      {x_sym, c_sym, q_sym.data(), true},
  };
  for (const Term& t : terms) {
    c64 g, ng[3];
    integral_of_wave_part_infinite_depth(t.p, t.c, face_area, nq, t.q, quad_weights, k, T, gf_sing, deriv_first, g,
                                         ng);
    if (t.flip_z) ng[2] = {-ng[2].re, -ng[2].im};
    int_G = {int_G.re + g.re, int_G.im + g.im};
    for (int a = 0; a < 3; ++a) int_nablaG[a] = {int_nablaG[a].re + ng[a].re, int_nablaG[a].im + ng[a].im};
  }
  const f64 amh = k * depth;
  const f64 akh = amh * std::tanh(amh);
  const f64 A = (amh + akh) * (amh + akh) / (4 * amh * (amh * amh - akh * akh + akh));
  int_G = {A * int_G.re, A * int_G.im};
  for (int a = 0; a < 3; ++a) int_nablaG[a] = {A * int_nablaG[a].re, A * int_nablaG[a].im};
}

// Green_wave.f90:427-508: each exponential (lambda_k, a_k) of the Prony
// decomposition as four Rankine terms at images of M, weighted a_k / 2.
void integral_of_prony_decomp_finite_depth(const f64* x, const f64* nodes, const f64* c, const f64* n, f64 area,
                                           f64 R, f64 depth, int nexp, const f64* lambdas, const f64* amplitudes,
                                           bool deriv_first, f64& int_G, f64* int_nablaG) {
  int_G = ZERO;
  int_nablaG[0] = int_nablaG[1] = int_nablaG[2] = ZERO;
  for (int e = 0; e < nexp; ++e) {
    const f64 lam = lambdas[e], a = amplitudes[e];
    const f64 coefs[4][2] = {{ONE, depth * lam - 2 * depth},
                             {-ONE, -depth * lam},
                             {-ONE, depth * lam - 4 * depth},
                             {ONE, -depth * lam + 2 * depth}};
    for (const auto& cc : coefs) {
      f64 g, dg[3];
      integral_of_reflected_Rankine(x, nodes, c, n, area, R, deriv_first, cc[0], cc[1], g, dg);
      int_G = int_G + a / 2 * g;
      for (int d = 0; d < 3; ++d) int_nablaG[d] = int_nablaG[d] + a / 2 * dg[d];
    }
  }
}

struct MeshArgs {
  int n;                 // collocation points
  const f64* colloc;     // (n,3)
  const f64* dot_normals;// (n,3) if adjoint else (N,3)
  int N;                 // faces
  const f64* vertices;   // (V,3)
  const int32_t* faces;  // (N,4), 0-based
  const f64* centers;    // (N,3)
  const f64* normals;    // (N,3)
  const f64* areas;      // (N)
  const f64* radii;      // (N)
  int nq;
  const f64* quad_points;  // (N,nq,3)
  const f64* quad_weights; // (N,nq)
};

inline void gather_nodes(const MeshArgs& m, int J, f64* nodes) {
  for (int L = 0; L < 4; ++L) {
    int v = m.faces[4 * J + L];
    nodes[3 * L] = m.vertices[3 * v];
    nodes[3 * L + 1] = m.vertices[3 * v + 1];
    nodes[3 * L + 2] = m.vertices[3 * v + 2];
  }
}

}  // namespace

extern "C" {

int oracle_nb_tabulated_values() { return NB_TAB; }
double oracle_pi() { return PI; }

void oracle_exp_e1(double re, double im, double* out2) {
  c64 r = exp_e1(c64{re, im});
  out2[0] = r.re;
  out2[1] = r.im;
}

void oracle_numerical_integration(double r, double z, int npts, double* out5) {
  numerical_integration(r, z, npts, out5);
}

void oracle_asymptotic_approximations(double r, double z, double* out5) { asymptotic_approximations(r, z, out5); }

void oracle_default_r_spacing(int nr, double rmax, int method, double* out) { default_r_spacing(nr, rmax, method, out); }

void oracle_default_z_spacing(int nz, double zmin, int method, double* out) { default_z_spacing(nz, zmin, method, out); }

int oracle_nearest_r_index(double r, const double* r_range, int nr, int method) {
  return nearest_r_index(r, r_range, nr, method);
}

int oracle_nearest_z_index(double z, const double* z_range, int nz, int method) {
  return nearest_z_index(z, z_range, nz, method);
}

// Delhommeau_integrals.f90:190-204; output C-contiguous (nr, nz, 5).
void oracle_construct_tabulation(const double* r_range, int nr, const double* z_range, int nz, int npts,
                                 double* out, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < nr; ++i) {
    for (int j = 0; j < nz; ++j) {
      numerical_integration(r_range[i], z_range[j], npts, out + ((size_t)i * nz + j) * NB_TAB);
    }
  }
}

void oracle_pick_in_default_tabulation(double r, double z, int method, const double* r_range, int nr,
                                       const double* z_range, int nz, const double* tab, double* out5) {
  pick_in_default_tabulation(r, z, method, r_range, nr, z_range, nz, tab, out5);
}

// Green_wave.f90:162-271 on a list of point pairs (interface.f90:29-70).
void oracle_wave_part_infinite_depth(int npairs, const double* x0i, const double* x0j, double k, int npts, int grid,
                                     const double* r_range, int nr, const double* z_range, int nz,
                                     const double* tab, int gf_sing, double* G /* (npairs,2) */,
                                     double* nablaG /* (npairs,3,2) */) {
  Tabulation T{npts, grid, r_range, nr, z_range, nz, tab};
  for (int p = 0; p < npairs; ++p) {
    c64 g, ng[3];
    wave_part_infinite_depth(x0i + 3 * p, x0j + 3 * p, k, T, gf_sing, g, ng);
    G[2 * p] = g.re;
    G[2 * p + 1] = g.im;
    for (int c = 0; c < 3; ++c) {
      nablaG[6 * p + 2 * c] = ng[c].re;
      nablaG[6 * p + 2 * c + 1] = ng[c].im;
    }
  }
}

// Rankine integrals for a list of (point, face) pairs; used by unit tests.
void oracle_integral_of_rankine(int npairs, const double* points, const double* nodes /* (npairs,4,3) */,
                                const double* centers, const double* normals, const double* areas,
                                const double* radii, int deriv_first, int reflected, double* G,
                                double* nablaG /* (npairs,3) */) {
  for (int p = 0; p < npairs; ++p) {
    if (reflected)
      integral_of_reflected_Rankine(points + 3 * p, nodes + 12 * p, centers + 3 * p, normals + 3 * p, areas[p],
                                    radii[p], deriv_first != 0, -1.0, 0.0, G[p], nablaG + 3 * p);
    else
      integral_of_Rankine(points + 3 * p, nodes + 12 * p, centers + 3 * p, normals + 3 * p, areas[p], radii[p],
                          deriv_first != 0, G[p], nablaG + 3 * p);
  }
}

// matrices.f90:28-325 (infinite depth only).
// S: complex128 Fortran-order (n, N); K: complex128 Fortran-order (kdim, n, N), kdim = 1 or 3.
// Returns 0 on success, -1 when depth is finite (not part of this restatement).
int oracle_build_matrices(int n, const double* colloc, const double* dot_normals, int N, const double* vertices,
                          const int32_t* faces, const double* centers, const double* normals, const double* areas,
                          const double* radii, int nq, const double* quad_points, const double* quad_weights,
                          double wavenumber, double depth, int npts, int grid, const double* r_range, int nr,
                          const double* z_range, int nz, const double* tab, int gf_sing, int adjoint, int kdim,
                          double* S, double* K, int nthreads) {
  if (std::isfinite(depth)) return -1;
  MeshArgs m{n, colloc, dot_normals, N, vertices, faces, centers, normals, areas, radii, nq, quad_points, quad_weights};
  Tabulation T{npts, grid, r_range, nr, z_range, nz, tab};
  const bool deriv_first = adjoint != 0;
  const bool finite_wavenumber = (ZERO < wavenumber) && std::isfinite(wavenumber);
  const f64 sign_refl = (gf_sing == HIGH_FREQ) ? -ONE : ONE;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic)
  for (int J = 0; J < N; ++J) {
    f64 nodes[12];
    gather_nodes(m, J, nodes);
    const f64* cJ = centers + 3 * J;
    const f64* nJ = normals + 3 * J;
    for (int I = 0; I < n; ++I) {
      const f64* M = colloc + 3 * I;
      c64 int_G{0, 0};
      c64 int_nablaG[3] = {{0, 0}, {0, 0}, {0, 0}};
      f64 gR, nR[3];
      integral_of_Rankine(M, nodes, cJ, nJ, areas[J], radii[J], deriv_first, gR, nR);
      int_G.re = int_G.re + gR;
      for (int a = 0; a < 3; ++a) int_nablaG[a].re = int_nablaG[a].re + nR[a];
      integral_of_reflected_Rankine(M, nodes, cJ, nJ, areas[J], radii[J], deriv_first, -ONE, ZERO, gR, nR);
      int_G.re = int_G.re + sign_refl * gR;
      for (int a = 0; a < 3; ++a) int_nablaG[a].re = int_nablaG[a].re + sign_refl * nR[a];
      if (gf_sing == LOW_FREQ_WITH_RANKINE_PART) int_nablaG[2].re = int_nablaG[2].re + 2 * wavenumber * gR;
      if (finite_wavenumber) {
        c64 gW, nW[3];
        integral_of_wave_part_infinite_depth(M, cJ, areas[J], nq, quad_points + (size_t)3 * nq * J,
                                             quad_weights + (size_t)nq * J, wavenumber, T, gf_sing, deriv_first,
                                             gW, nW);
        int_G = {int_G.re + gW.re, int_G.im + gW.im};
        for (int a = 0; a < 3; ++a) int_nablaG[a] = {int_nablaG[a].re + nW[a].re, int_nablaG[a].im + nW[a].im};
      }
      size_t idx = (size_t)I + (size_t)n * J;
      S[2 * idx] = MINUS_ONE_OVER_FOURPI * int_G.re;
      S[2 * idx + 1] = MINUS_ONE_OVER_FOURPI * int_G.im;
      if (kdim == 1) {
        const f64* dn = adjoint ? dot_normals + 3 * I : dot_normals + 3 * J;
        f64 re = dn[0] * int_nablaG[0].re + dn[1] * int_nablaG[1].re + dn[2] * int_nablaG[2].re;
        f64 im = dn[0] * int_nablaG[0].im + dn[1] * int_nablaG[1].im + dn[2] * int_nablaG[2].im;
        K[2 * idx] = MINUS_ONE_OVER_FOURPI * re;
        K[2 * idx + 1] = MINUS_ONE_OVER_FOURPI * im;
      } else {
        for (int a = 0; a < 3; ++a) {
          K[2 * (3 * idx + a)] = MINUS_ONE_OVER_FOURPI * int_nablaG[a].re;
          K[2 * (3 * idx + a) + 1] = MINUS_ONE_OVER_FOURPI * int_nablaG[a].im;
        }
      }
    }
  }
  return 0;
}

// matrices.f90:28-325, finite depth with Delhommeau's method (finite_depth_method
// 0 = legacy: one-point free-surface image, 1 = newer).  prony: lambdas then
// amplitudes (2 x nexp).  Same outputs as oracle_build_matrices.
int oracle_build_matrices_finite_depth(int n, const double* colloc, const double* dot_normals, int N,
                                       const double* vertices, const int32_t* faces, const double* centers,
                                       const double* normals, const double* areas, const double* radii, int nq,
                                       const double* quad_points, const double* quad_weights, double wavenumber,
                                       double depth, int npts, int grid, const double* r_range, int nr,
                                       const double* z_range, int nz, const double* tab, int method, int nexp,
                                       const double* prony, int gf_sing, int adjoint, int kdim, double* S, double* K,
                                       int nthreads) {
  if (!std::isfinite(depth) || depth <= 0) return -1;
  MeshArgs m{n, colloc, dot_normals, N, vertices, faces, centers, normals, areas, radii, nq, quad_points, quad_weights};
  Tabulation T{npts, grid, r_range, nr, z_range, nz, tab};
  const bool deriv_first = adjoint != 0;
  const bool finite_wavenumber = (ZERO < wavenumber) && std::isfinite(wavenumber);
  const f64 sign_refl = (gf_sing == HIGH_FREQ) ? -ONE : ONE;
  const f64* lambdas = prony;
  const f64* amplitudes = prony + nexp;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic)
  for (int J = 0; J < N; ++J) {
    f64 nodes[12];
    gather_nodes(m, J, nodes);
    const f64* cJ = centers + 3 * J;
    const f64* nJ = normals + 3 * J;
    for (int I = 0; I < n; ++I) {
      const f64* M = colloc + 3 * I;
      c64 int_G{0, 0};
      c64 int_nablaG[3] = {{0, 0}, {0, 0}, {0, 0}};
      f64 gR, nR[3];
      auto add_real = [&](f64 coef, f64 g, const f64* dg) {
        int_G.re = int_G.re + coef * g;
        for (int a = 0; a < 3; ++a) int_nablaG[a].re = int_nablaG[a].re + coef * dg[a];
      };
      integral_of_Rankine(M, nodes, cJ, nJ, areas[J], radii[J], deriv_first, gR, nR);
      add_real(ONE, gR, nR);
      if (method == 0)
        one_point_integral_of_reflected_Rankine(M, cJ, areas[J], deriv_first, -ONE, ZERO, gR, nR);
      else
        integral_of_reflected_Rankine(M, nodes, cJ, nJ, areas[J], radii[J], deriv_first, -ONE, ZERO, gR, nR);
      add_real(sign_refl, gR, nR);
      if (gf_sing == LOW_FREQ_WITH_RANKINE_PART) int_nablaG[2].re = int_nablaG[2].re + 2 * wavenumber * gR;
      // images through the sea bottom, and through both boundaries
      integral_of_reflected_Rankine(M, nodes, cJ, nJ, areas[J], radii[J], deriv_first, -ONE, -2 * depth, gR, nR);
      add_real(ONE, gR, nR);
      one_point_integral_of_reflected_Rankine(M, cJ, areas[J], deriv_first, ONE, -2 * depth, gR, nR);
      add_real(sign_refl, gR, nR);
      one_point_integral_of_reflected_Rankine(M, cJ, areas[J], deriv_first, ONE, 2 * depth, gR, nR);
      add_real(sign_refl, gR, nR);
      one_point_integral_of_reflected_Rankine(M, cJ, areas[J], deriv_first, -ONE, -4 * depth, gR, nR);
      add_real(sign_refl, gR, nR);
      if (finite_wavenumber) {
        c64 gW, nW[3];
        integral_of_wave_parts_finite_depth(M, cJ, areas[J], nq, quad_points + (size_t)3 * nq * J,
                                            quad_weights + (size_t)nq * J, wavenumber, depth, T, gf_sing, deriv_first,
                                            gW, nW);
        int_G = {int_G.re + gW.re, int_G.im + gW.im};
        for (int a = 0; a < 3; ++a) int_nablaG[a] = {int_nablaG[a].re + nW[a].re, int_nablaG[a].im + nW[a].im};
      }
      integral_of_prony_decomp_finite_depth(M, nodes, cJ, nJ, areas[J], radii[J], depth, nexp, lambdas, amplitudes,
                                            deriv_first, gR, nR);
      add_real(ONE, gR, nR);
      size_t idx = (size_t)I + (size_t)n * J;
      S[2 * idx] = MINUS_ONE_OVER_FOURPI * int_G.re;
      S[2 * idx + 1] = MINUS_ONE_OVER_FOURPI * int_G.im;
      if (kdim == 1) {
        const f64* dn = adjoint ? dot_normals + 3 * I : dot_normals + 3 * J;
        f64 re = dn[0] * int_nablaG[0].re + dn[1] * int_nablaG[1].re + dn[2] * int_nablaG[2].re;
        f64 im = dn[0] * int_nablaG[0].im + dn[1] * int_nablaG[1].im + dn[2] * int_nablaG[2].im;
        K[2 * idx] = MINUS_ONE_OVER_FOURPI * re;
        K[2 * idx + 1] = MINUS_ONE_OVER_FOURPI * im;
      } else {
        for (int a = 0; a < 3; ++a) {
          K[2 * (3 * idx + a)] = MINUS_ONE_OVER_FOURPI * int_nablaG[a].re;
          K[2 * (3 * idx + a) + 1] = MINUS_ONE_OVER_FOURPI * int_nablaG[a].im;
        }
      }
    }
  }
  return 0;
}

// Green_wave.f90:311-425 at one (point, face) pair; out: G (re, im), gradient (3 x (re, im)).
void oracle_wave_parts_finite_depth(const double* x, const double* face_center, double face_area, int nq,
                                    const double* quad_points, const double* quad_weights, double k, double depth,
                                    int npts, int grid, const double* r_range, int nr, const double* z_range, int nz,
                                    const double* tab, int gf_sing, int deriv_first, double* out8) {
  Tabulation T{npts, grid, r_range, nr, z_range, nz, tab};
  c64 g, ng[3];
  integral_of_wave_parts_finite_depth(x, face_center, face_area, nq, quad_points, quad_weights, k, depth, T, gf_sing,
                                      deriv_first != 0, g, ng);
  out8[0] = g.re;
  out8[1] = g.im;
  for (int a = 0; a < 3; ++a) {
    out8[2 + 2 * a] = ng[a].re;
    out8[3 + 2 * a] = ng[a].im;
  }
}

// Green_wave.f90:50-124 at one (point, face) pair, same output layout.
void oracle_wave_part_integral_infinite_depth(const double* x, const double* face_center, double face_area, int nq,
                                              const double* quad_points, const double* quad_weights, double k,
                                              int npts, int grid, const double* r_range, int nr,
                                              const double* z_range, int nz, const double* tab, int gf_sing,
                                              int deriv_first, double* out8) {
  Tabulation T{npts, grid, r_range, nr, z_range, nz, tab};
  c64 g, ng[3];
  integral_of_wave_part_infinite_depth(x, face_center, face_area, nq, quad_points, quad_weights, k, T, gf_sing,
                                       deriv_first != 0, g, ng);
  out8[0] = g.re;
  out8[1] = g.im;
  for (int a = 0; a < 3; ++a) {
    out8[2 + 2 * a] = ng[a].re;
    out8[3 + 2 * a] = ng[a].im;
  }
}

// Green_wave.f90:427-508 at one (point, face) pair; out: G, gradient (4 reals).
void oracle_prony_decomp_finite_depth(const double* x, const double* nodes, const double* c, const double* n,
                                      double area, double R, double depth, int nexp, const double* prony,
                                      int deriv_first, double* out4) {
  f64 g, dg[3];
  integral_of_prony_decomp_finite_depth(x, nodes, c, n, area, R, depth, nexp, prony, prony + nexp, deriv_first != 0,
                                        g, dg);
  out4[0] = g;
  out4[1] = dg[0];
  out4[2] = dg[1];
  out4[3] = dg[2];
}

// matrices.f90:329-364.  centers: (m,3) of the first m faces; K layout as above with (n, N) extents.
void oracle_add_diagonal_term(int n, int N, const double* centers, const double* dot_normals, double free_surface,
                              int kdim, double* K) {
  int m = n < N ? n : N;
  for (int i = 0; i < m; ++i) {
    f64 coef = (std::fabs(centers[3 * i + 2] - free_surface) < lit(1e-8f)) ? ONE : ONE / 2;
    size_t idx = (size_t)i + (size_t)n * i;
    if (kdim == 1) {
      K[2 * idx] = K[2 * idx] + coef;
    } else {
      for (int a = 0; a < 3; ++a) K[2 * (3 * idx + a)] = K[2 * (3 * idx + a)] + coef * dot_normals[3 * i + a];
    }
  }
}

// matrices.f90:368-432.  Real outputs (the reference keeps complex storage and takes the real part).
void oracle_add_rankine_term_only(int n, const double* colloc, const double* dot_normals, int N,
                                  const double* vertices, const int32_t* faces, const double* centers,
                                  const double* normals, const double* areas, const double* radii, int adjoint,
                                  int kdim, double* S, double* K, int nthreads) {
  MeshArgs m{n, colloc, dot_normals, N, vertices, faces, centers, normals, areas, radii, 1, nullptr, nullptr};
  const bool deriv_first = adjoint != 0;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic)
  for (int J = 0; J < N; ++J) {
    f64 nodes[12];
    gather_nodes(m, J, nodes);
    for (int I = 0; I < n; ++I) {
      f64 gR, nR[3];
      integral_of_Rankine(colloc + 3 * I, nodes, centers + 3 * J, normals + 3 * J, areas[J], radii[J], deriv_first,
                          gR, nR);
      size_t idx = (size_t)I + (size_t)n * J;
      S[idx] = S[idx] + MINUS_ONE_OVER_FOURPI * gR;
      if (kdim == 1) {
        const f64* dn = adjoint ? dot_normals + 3 * I : dot_normals + 3 * J;
        K[idx] = K[idx] + MINUS_ONE_OVER_FOURPI * (dn[0] * nR[0] + dn[1] * nR[1] + dn[2] * nR[2]);
      } else {
        for (int a = 0; a < 3; ++a) K[3 * idx + a] = K[3 * idx + a] + MINUS_ONE_OVER_FOURPI * nR[a];
      }
    }
  }
}

}  // extern "C"
