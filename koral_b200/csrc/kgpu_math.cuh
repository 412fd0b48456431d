// Powers of the solver's hot path without a general pow: products and
// square roots carried to double-double accuracy (the error-free
// transformations of Dekker and Knuth: a*b = p + e exactly with
// e = fma(a, b, -p); a + b = s + t exactly) and rounded once at the end.
// The double-double value is within about 2^-100 of the exact power, so
// the rounded result is the correctly rounded power except in the rare
// cases where the exact value lies within that distance of a rounding
// boundary.  A correctly rounded result is what the host C library's pow
// returns too wherever its own error (below 0.52 ulp) does not cross such a
// boundary, so these agree with the reference's pow far more often than a
// general device pow does (whose error bound is 2 ulp), at a small fraction
// of its cost.  Only +, -, *, /, sqrt and fma are used: the same bits on
// the host and on the device.
//
// The hot path uses pw2 (the squares of the M1 closure's closed forms) and
// pw4 (the Planck term T^4).  pw_m3p5 (the Kramers term) and the quarter
// powers (the entropy at Gamma = 13/9) are as accurate but were measured
// slower inside the implicit solve than the library pow (their divisions
// and square roots add code to an instruction-fetch-bound kernel), so the
// solver keeps pow for those; they remain for kgpu_eval_powers.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define KM_HD __host__ __device__ inline
#else
#define KM_HD inline
#endif

namespace kgpu {

// double-double number hi + lo, |lo| <= ulp(hi)/2
struct DD {
  double hi, lo;
};

KM_HD DD dd_two_prod(double a, double b) {
  const double p = a * b;
  return DD{p, fma(a, b, -p)};
}

// renormalises hi + lo when |hi| >= |lo| (Dekker's fast two-sum)
KM_HD DD dd_fast(double hi, double lo) {
  const double s = hi + lo;
  return DD{s, lo - (s - hi)};
}

KM_HD DD dd_mul(DD a, DD b) {
  DD p = dd_two_prod(a.hi, b.hi);
  const double c = a.hi * b.lo + a.lo * b.hi;
  return dd_fast(p.hi, p.lo + c);
}

KM_HD DD dd_mul_d(DD a, double b) {
  DD p = dd_two_prod(a.hi, b);
  return dd_fast(p.hi, p.lo + a.lo * b);
}

// sqrt of a double to double-double accuracy: s = sqrt(a) rounded, then one
// Newton correction (a - s^2) / (2 s) with a - s^2 exact by fma
KM_HD DD dd_sqrt(double a) {
  const double s = sqrt(a);
  const double r = fma(-s, s, a);
  return dd_fast(s, r / (2. * s));
}

// sqrt of a double-double
KM_HD DD dd_sqrt_dd(DD a) {
  const double s = sqrt(a.hi);
  const double r = fma(-s, s, a.hi) + a.lo;
  return dd_fast(s, r / (2. * s));
}

// 1 / a to double-double accuracy: q rounded, then one correction
KM_HD DD dd_recip(DD a) {
  const double q = 1. / a.hi;
  const double r = fma(-q, a.hi, 1.) - q * a.lo;
  return dd_fast(q, q * r);
}

// x^2: one product, already correctly rounded
KM_HD double pw2(double x) { return x * x; }

// the double-double forms keep their accuracy while every partial power
// stays a normal number: |log2 x| * |exponent| well inside 1000
KM_HD bool pw_in_range(double x, double y) {
  if (!(x > 0. && x < INFINITY)) return false;
  const int e = ilogb(x);
  return (double)(e < 0 ? -e : e) * (fabs(y) + 1.) < 900.;
}

// x^4 = (x^2)^2 with x^2 kept exact as a double-double
KM_HD double pw4(double x) {
  if (!pw_in_range(fabs(x), 4.)) return pow(x, 4.);
  const DD t = dd_two_prod(x, x);
  const DD q = dd_mul(t, t);
  return q.hi + q.lo;
}

// x^-3.5 = 1 / (x^3 sqrt(x))
KM_HD double pw_m3p5(double x) {
  if (!pw_in_range(x, 3.5)) return pow(x, -3.5);
  const DD x2 = dd_two_prod(x, x);
  const DD x3 = dd_mul_d(x2, x);
  const DD r = dd_mul(x3, dd_sqrt(x));
  const DD q = dd_recip(r);
  return q.hi + q.lo;
}

// x^(k/4) for an integer k in [-64, 64], x > 0: x^(k div 4) by repeated
// double-double products times the fourth root to the power k mod 4
KM_HD double pw_quarter(double x, int k) {
  const bool neg = k < 0;
  int m = neg ? -k : k;
  const int whole = m >> 2, frac = m & 3;
  DD acc{1., 0.};
  DD base{x, 0.};
  for (int w = whole; w; w >>= 1) {   // binary powering, at most 5 squarings
    if (w & 1) acc = dd_mul(acc, base);
    if (w > 1) base = dd_mul(base, base);
  }
  if (frac) {
    const DD r2 = dd_sqrt(x);          // x^(1/2)
    const DD r4 = dd_sqrt_dd(r2);      // x^(1/4)
    DD f = frac == 2 ? r2 : r4;
    if (frac == 3) f = dd_mul(r2, r4);
    acc = dd_mul(acc, f);
  }
  if (neg) acc = dd_recip(acc);
  return acc.hi + acc.lo;
}

// x^y where 4 y is an integer of at most 64 in magnitude (the quarter
// powers above), else the library pow; the test on y is exact
KM_HD double pw_any(double x, double y) {
  const double q = 4. * y;
  if (q >= -64. && q <= 64. && q == (double)(int)q && pw_in_range(x, y)) return pw_quarter(x, (int)q);
  return pow(x, y);
}

}  // namespace kgpu
