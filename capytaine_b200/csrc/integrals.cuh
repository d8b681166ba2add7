// Delhommeau integrals on the device: exp(z)E1(z) in float32 complex arithmetic
// and the Simpson integration over theta (libs/libDelhommeau/src/
// Delhommeau_integrals.f90:43-153).  Included by the tabulation builder (compiled
// without FMA contraction) and by the assembly kernels (direct integration when
// no tabulation is given).
#pragma once
#include "common.cuh"

namespace bem {
namespace {

struct cf {
  float re, im;
};
__device__ __forceinline__ cf cf_add(cf a, cf b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cf cf_mul(cf a, cf b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cf cf_radd(float r, cf b) { return {r + b.re, b.im}; }
__device__ __forceinline__ cf cf_rmul(float r, cf b) { return {r * b.re, r * b.im}; }
// Range-reduced (Smith) complex division, the form gfortran emits.
template <class T>
__device__ __forceinline__ void smith(T a, T b, T c, T d, T& x, T& y) {
  if (fabs(c) < fabs(d)) {
    T ratio = c / d;
    T div = (c * ratio) + d;
    T tr = (a * ratio) + b;
    T ti = (b * ratio) - a;
    x = tr / div;
    y = ti / div;
  } else {
    T ratio = d / c;
    T div = (d * ratio) + c;
    T tr = (b * ratio) + a;
    T ti = b - (a * ratio);
    x = tr / div;
    y = ti / div;
  }
}
__device__ __forceinline__ cf cf_div(cf p, cf q) {
  cf r;
  smith<float>(p.re, p.im, q.re, q.im, r.re, r.im);
  return r;
}

// exp(z) E1(z), Delhommeau thesis p.367-369 (Delhommeau_integrals.f90:104-151).
__device__ inline c64d exp_e1(double zr, double zi) {
  cf z{(float)zr, (float)zi};
  cf g;
  if (z.re < -16.0f) {
    cf y = cf_div(cf{1.0f, 0.0f}, z);
    cf t = cf_rmul(-120.0f, y);
    t = cf_mul(y, cf_radd(24.0f, t));
    t = cf_mul(y, cf_radd(-6.0f, t));
    t = cf_mul(y, cf_radd(2.0f, t));
    t = cf_mul(y, cf_radd(-1.0f, t));
    g = cf_mul(y, cf_radd(1.0f, t));
  } else if (fabsf(z.im) > 10.0f) {
    cf a = cf_div(cf{0.711093f, 0.0f}, cf_radd(0.415775f, z));
    cf b = cf_div(cf{0.278518f, 0.0f}, cf_radd(2.29428f, z));
    cf c = cf_div(cf{0.010389f, 0.0f}, cf_radd(6.2900f, z));
    g = cf_add(cf_add(a, b), c);
  } else if (z.re > -0.5f) {
    cf p1 = cf_rmul(0.97087007e-05f, z);
    p1 = cf_mul(z, cf_radd(0.763297e-03f, p1));
    p1 = cf_mul(z, cf_radd(0.206543e-01f, p1));
    p1 = cf_mul(z, cf_radd(0.23721365e+00f, p1));
    p1 = cf_radd(0.1e+01f, p1);
    cf p2 = cf_rmul(-0.51801555e-03f, z);
    p2 = cf_mul(z, cf_radd(0.19387339e-02f, p2));
    p2 = cf_mul(z, cf_radd(-0.3000591e-01f, p2));
    p2 = cf_mul(z, cf_radd(0.41806426e-01f, p2));
    p2 = cf_mul(z, cf_radd(-0.149545886e+01f, p2));
    p2 = cf_radd(0.99999207e+00f, p2);
    cf q = cf_rmul(0.2989204e-03f, z);
    q = cf_mul(z, cf_radd(-0.8700861e-03f, q));
    q = cf_mul(z, cf_radd(0.12982719e-01f, q));
    q = cf_mul(z, cf_radd(-0.66786033e-01f, q));
    q = cf_mul(z, cf_radd(0.28388363e+00f, q));
    q = cf_mul(z, cf_radd(-0.76273617e+00f, q));
    q = cf_radd(0.1e+01f, q);
    // Complex logarithm of a float value: modulus rounded to float, then the
    // float-rounded log and argument evaluated in double precision.  This
    // tracks the host C library's clogf (what gfortran calls for LOG of a
    // COMPLEX(4)) to a few 1e-9 over the whole default tabulation.
    const float modulus = (float)sqrt((double)z.re * (double)z.re + (double)z.im * (double)z.im);
    cf lz{(float)log((double)modulus), (float)atan2((double)z.im, (double)z.re)};
    cf num = cf_add(cf_mul(lz, p1), cf_rmul(0.5772156649e+00f, p2));
    cf r = cf_div(num, q);
    g = cf{-r.re, -r.im};
  } else {
    const float s = (z.im < 0.0f) ? 1.0f : -1.0f;
    const cf A[8] = {{1.000000f, s * 1.3935496e-06f}, {15.82958f, -s * 20.14222f},
                     {-70.52863f, -s * 227.9511f},    {-985.4221f, -s * 226.6272f},
                     {-1202.318f, s * 1580.907f},     {953.2441f, s * 1342.447f},
                     {417.3716f, -s * 196.6665f},     {-9.881266f, -s * 24.24952f}};
    const cf B[9] = {{1.000000f, 0.0f},            {16.83184f, -s * 20.14481f},
                     {-55.66969f, -s * 248.1167f}, {-1068.640f, -s * 434.4707f},
                     {-2082.250f, s * 1522.471f},  {383.3455f, s * 2730.378f},
                     {1216.791f, s * 351.7189f},   {115.3926f, -s * 161.2647f},
                     {-3.777369f, -s * 4.510900f}};
    cf num = cf_mul(A[0], z);
#pragma unroll
    for (int i = 1; i < 8; ++i) {
      num = cf_add(num, A[i]);
      if (i < 7) num = cf_mul(num, z);
    }
    cf den = cf_mul(B[0], z);
#pragma unroll
    for (int i = 1; i < 9; ++i) {
      den = cf_add(den, B[i]);
      if (i < 8) den = cf_mul(den, z);
    }
    g = cf_div(num, den);
  }
  return c64d{(double)g.re, (double)g.im};
}

}  // namespace

// Simpson integration over theta (Delhommeau_integrals.f90:43-100).
__device__ inline void numerical_integration_device(double r, double z, int nb_integration_points, double* out) {
  double I0 = 0, I1 = 0, I2 = 0, I3 = 0, I4 = 0;
  const int n = (nb_integration_points % 2 == 0) ? nb_integration_points + 1 : nb_integration_points;
  const double nm1 = (double)((float)n - 1.0f);
  const double three_nm1 = (double)(3.0f * (float)nm1);
  for (int k = 1; k <= n; ++k) {
    const double km1 = (double)((float)k - 1.0f);
    const double theta = -kPI / 2 + kPI * km1 / nm1;
    double delta_theta;
    if (k == 1 || k == n) delta_theta = kPI / three_nm1;
    else if (k % 2 == 0) delta_theta = 4 * kPI / three_nm1;
    else delta_theta = 2 * kPI / three_nm1;
    const double cos_theta = cos(theta);
    const double zr = z, zi = r * cos_theta;
    double er = 0.0, ei = 0.0;
    if (!(zr <= -30.0)) {
      double s, c;
      sincos(zi, &s, &c);
      const double e = exp(zr);
      er = e * c;
      ei = e * s;
    }
    const c64d e1 = exp_e1(zr, zi);
    const double jr = e1.re + (0.0 * er - kPI * ei);
    const double ji = e1.im + (0.0 * ei + kPI * er);
    double invr, invi;
    smith<double>(1.0, 0.0, zr, zi, invr, invi);
    const double jmr = jr - invr, jmi = ji - invi;
    I0 = I0 + delta_theta * jr;
    I1 = I1 + delta_theta * jmr;
    I2 = I2 + delta_theta * er;
    I3 = I3 - delta_theta * cos_theta * jmi;
    I4 = I4 - delta_theta * cos_theta * ei;
  }
  out[0] = 2 * (I0 / kPI);
  out[1] = 2 * (I1 / kPI);
  out[2] = 2 * I2;
  out[3] = 2 * (I3 / kPI);
  out[4] = 2 * I4;
}

}  // namespace bem
