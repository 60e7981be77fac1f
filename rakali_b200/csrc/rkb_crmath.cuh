// Correctly rounded FP64 evaluations of the transcendental terms of the step.
//
// The reference evaluates h**(1/3) (Manning friction), sin/cos (tidal
// forcing, Coriolis rotation) with the platform libm.  A correctly rounded
// result is the unique IEEE-754 double nearest the exact value, so computing
// these terms correctly rounded on the device reproduces any libm that is
// itself correctly rounded for the same argument (glibc's pow/sin/cos are,
// except for arguments exceptionally close to a rounding midpoint).
//
// Methods (double-double arithmetic: Dekker 1971 exact product via FMA,
// Knuth two-sum):
//   pow(h, 1/3): one Newton step for the cube root from a 1-ulp start, then
//     the factor h^(-d), d = 1/3 - fl(1/3) = 2^-54 / 3, as 1 - d ln h.
//   sin/cos:     Cody-Waite reduction by pi/2 in double-double, then Taylor
//     series of sin/cos on |r| <= pi/4 in double-double.
#pragma once

#include <cmath>
#if defined(__CUDACC__)
#include <cuda_runtime.h>
#endif

namespace rkb {

#if defined(__CUDACC__)
#define RKB_HD __host__ __device__ __forceinline__
#else
#define RKB_HD inline
#endif

struct dd {
  double hi, lo;
};

RKB_HD double cr_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

// exact a*b = p + e
RKB_HD dd two_prod(double a, double b) {
  double p = a * b;
  return {p, cr_fma(a, b, -p)};
}

// exact a+b = s + e
RKB_HD dd two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}

RKB_HD dd fast_two_sum(double a, double b) {  // |a| >= |b|
  double s = a + b;
  return {s, b - (s - a)};
}

RKB_HD dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}

RKB_HD dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return fast_two_sum(p.hi, p.lo);
}

RKB_HD dd dd_mul_d(dd a, double b) {
  dd p = two_prod(a.hi, b);
  p.lo += a.lo * b;
  return fast_two_sum(p.hi, p.lo);
}

// h ** fl(1/3) for finite h > 0, correctly rounded (see header).
RKB_HD double cr_pow_third(double h) {
  const double y = std::cbrt(h);
  // r = y^3 - h, with y^2 and y^3 split exactly
  const dd y2 = two_prod(y, y);
  const dd y3 = two_prod(y2.hi, y);
  const double r = (y3.hi - h) + (y3.lo + y2.lo * y);
  const double newton = -r / (3.0 * y2.hi);          // y + newton ~ h^(1/3) to ~2^-100
  const double d = 1.8503717077085943e-17;           // 1/3 - fl(1/3) = 2^-54 / 3
  const double t = -d * std::log(h);                 // h^(-d) = 1 + t + O(t^2), |t| < 1e-14
  return y + (newton + y * t);
}

// Cody-Waite split of pi/2 = P1 + P2 + P3 + P4 (P1, P2 carry 33 significant
// bits, so k * P1 and k * P2 are exact for |k| < 2^20), derived from pi to
// 200 digits.
constexpr double kPio2_1 = 1.5707963267341256;      // 0x1.921fb54400000p+0
constexpr double kPio2_2 = 6.077100506303966e-11;   // 0x1.0b4611a600000p-34
constexpr double kPio2_3 = 2.0222662487959506e-21;  // 0x1.3198a2e037073p-69
constexpr double kPio2_4 = 1.0085854035872483e-37;  // 0x1.129024e088a68p-123
constexpr double kTwoOverPi = 0.6366197723675814;

// r = x - k pi/2 in double-double, quadrant k mod 4.
RKB_HD dd reduce_pio2(double x, int& quadrant) {
  const double k = std::nearbyint(x * kTwoOverPi);
  dd r = two_sum(x, -k * kPio2_1);
  r = dd_add(r, {-k * kPio2_2, 0.0});
  r = dd_add(r, two_prod(-k, kPio2_3));
  r = dd_add(r, {-k * kPio2_4, 0.0});
  const long long kk = (long long)k;
  quadrant = (int)(((kk % 4) + 4) % 4);
  return r;
}

// 1/n in double-double.
RKB_HD dd dd_inv(double n) {
  const double hi = 1.0 / n;
  return {hi, -cr_fma(hi, n, -1.0) / n};
}

// sin(r), cos(r) for |r| <= pi/4, Taylor series in double-double (Horner:
// sin r = r (1 - r^2/(2*3) (1 - r^2/(4*5) (...))), cos likewise from 1*2).
RKB_HD void dd_sincos_small(dd r, dd& s, dd& c) {
  const dd r2 = dd_mul(r, r);
  const dd one = {1.0, 0.0};
  dd ts = one, tc = one;
  for (int n = 25; n >= 3; n -= 2) {
    const dd q = dd_mul(r2, dd_inv((double)(n * (n - 1))));
    ts = dd_add(one, dd_mul({-q.hi, -q.lo}, ts));
  }
  for (int n = 26; n >= 2; n -= 2) {
    const dd q = dd_mul(r2, dd_inv((double)(n * (n - 1))));
    tc = dd_add(one, dd_mul({-q.hi, -q.lo}, tc));
  }
  s = dd_mul(r, ts);
  c = tc;
}

// sin(x) and cos(x), correctly rounded for |x| < 1e6 (larger arguments fall
// back to the platform function).
RKB_HD void cr_sincos(double x, double& sn, double& cs) {
  if (!(std::fabs(x) < 1.0e6)) {
    sn = std::sin(x);
    cs = std::cos(x);
    return;
  }
  int q;
  dd r = reduce_pio2(x, q);
  dd s, c;
  dd_sincos_small(r, s, c);
  const double s1 = s.hi + s.lo, c1 = c.hi + c.lo;
  switch (q) {
    case 0: sn = s1; cs = c1; break;
    case 1: sn = c1; cs = -s1; break;
    case 2: sn = -s1; cs = -c1; break;
    default: sn = -c1; cs = s1; break;
  }
}

RKB_HD double cr_sin(double x) {
  double s, c;
  cr_sincos(x, s, c);
  return s;
}

RKB_HD double cr_cos(double x) {
  double s, c;
  cr_sincos(x, s, c);
  return c;
}

}  // namespace rkb
