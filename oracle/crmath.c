/*
 * Correctly rounded h**(1/3), sin and cos for the oracle (test
 * infrastructure only).
 *
 * The reference evaluates these with the Fortran intrinsics, whose last bit
 * depends on the platform libm (glibc on CPU builds, the CUDA math library
 * on GPU builds); glibc itself misrounds about 0.1% of arguments.  The only
 * platform-independent value is the correctly rounded one, which is what the
 * oracle uses.  Methods: double-double arithmetic (Dekker's exact product via
 * fma, Knuth's two-sum); one Newton step for the cube root; Cody-Waite
 * reduction by pi/2 and Taylor series for sin/cos.
 */
#include <math.h>

#include "swe_oracle.h"

typedef struct {
  double hi, lo;
} ddv;

static ddv tp(double a, double b) {
  ddv r;
  r.hi = a * b;
  r.lo = fma(a, b, -r.hi);
  return r;
}

static ddv ts(double a, double b) {
  ddv r;
  double s = a + b, bb = s - a;
  r.hi = s;
  r.lo = (a - (s - bb)) + (b - bb);
  return r;
}

static ddv fts(double a, double b) {
  ddv r;
  r.hi = a + b;
  r.lo = b - (r.hi - a);
  return r;
}

static ddv add(ddv a, ddv b) {
  ddv s = ts(a.hi, b.hi), t = ts(a.lo, b.lo);
  s.lo += t.hi;
  s = fts(s.hi, s.lo);
  s.lo += t.lo;
  return fts(s.hi, s.lo);
}

static ddv mul(ddv a, ddv b) {
  ddv p = tp(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return fts(p.hi, p.lo);
}

static ddv mk(double hi, double lo) {
  ddv r;
  r.hi = hi;
  r.lo = lo;
  return r;
}

double orc_cr_pow_third(double h) {
  /* cube root y ~ h^(1/3) to ~1 ulp, refined by one Newton step in
   * double-double, then times h^(-d) = 1 - d ln h, d = 1/3 - fl(1/3) */
  double y = cbrt(h);
  ddv y2 = tp(y, y);
  ddv y3 = tp(y2.hi, y);
  double r = (y3.hi - h) + (y3.lo + y2.lo * y);
  double newton = -r / (3.0 * y2.hi);
  double t = -1.8503717077085943e-17 * log(h);
  return y + (newton + y * t);
}

/* pi/2 split: the first two parts carry 33 significant bits (derived from
 * pi to 200 digits) */
static const double P1 = 1.5707963267341256;
static const double P2 = 6.077100506303966e-11;
static const double P3 = 2.0222662487959506e-21;
static const double P4 = 1.0085854035872483e-37;

static ddv inv(double n) {
  double hi = 1.0 / n;
  return mk(hi, -fma(hi, n, -1.0) / n);
}

void orc_cr_sincos(double x, double *sn, double *cs) {
  if (!(fabs(x) < 1.0e6)) {
    *sn = sin(x);
    *cs = cos(x);
    return;
  }
  double k = nearbyint(x * 0.6366197723675814);
  ddv r = ts(x, -k * P1);
  r = add(r, mk(-k * P2, 0.0));
  r = add(r, tp(-k, P3));
  r = add(r, mk(-k * P4, 0.0));
  long long kk = (long long)k;
  int q = (int)(((kk % 4) + 4) % 4);
  ddv r2 = mul(r, r), one = mk(1.0, 0.0), tsn = one, tcs = one;
  for (int n = 25; n >= 3; n -= 2) {
    ddv c = mul(r2, inv((double)(n * (n - 1))));
    tsn = add(one, mul(mk(-c.hi, -c.lo), tsn));
  }
  for (int n = 26; n >= 2; n -= 2) {
    ddv c = mul(r2, inv((double)(n * (n - 1))));
    tcs = add(one, mul(mk(-c.hi, -c.lo), tcs));
  }
  ddv s = mul(r, tsn);
  double s1 = s.hi + s.lo, c1 = tcs.hi + tcs.lo;
  switch (q) {
    case 0: *sn = s1; *cs = c1; break;
    case 1: *sn = c1; *cs = -s1; break;
    case 2: *sn = -s1; *cs = -c1; break;
    default: *sn = -c1; *cs = s1; break;
  }
}

double orc_cr_sin(double x) {
  double s, c;
  orc_cr_sincos(x, &s, &c);
  return s;
}

double orc_cr_cos(double x) {
  double s, c;
  orc_cr_sincos(x, &s, &c);
  return c;
}
