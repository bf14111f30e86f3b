// Correctly rounded pow(x, 0.25) and pow(x, 0.2) for x >= 0, host and device.
//
// The exact Riemann solver's rarefaction step control raises an error ratio
// to the powers 0.25 and 0.2 (ExactRiemannSolverBase.cpp:1298, 1305,
// 1348-1349). The reference takes them from the host C library's pow, whose
// result is the correctly rounded one on all but about 6e-4 of the arguments
// the solver reaches (glibc's pow has a worst-case error of 0.52 ulp);
// CUDA's double pow has a looser bound (2 ulp). A step size that differs in
// its last bit changes the integrated rarefaction in its last bits and,
// where it changes which steps are accepted, the secant iterates after it.
// Both the GPU and the host build of the solver therefore use these
// functions, which return the correctly rounded result everywhere, so the
// GPU's solves are bit-identical to the host build's and differ from the
// reference only where the C library rounds the other way.
//
// Method (written for this library; no library pow's constants or steps):
//  * x^(1/4) = sqrt(sqrt(x)) carried in double-double. After x = y 2^(4q)
//    with y in [0.5, 8), s = sqrt(y) is refined by its exact remainder
//    y - s^2 (one fma), then t = sqrt(s) by (s - t^2 + s_lo) / (2t). The
//    pair t + t_lo holds y^(1/4) to about 2^-100 relative, so rounding
//    t + t_lo once gives the correctly rounded value except on arguments
//    within ~2^-95 relative of a rounding midpoint (none of those is an
//    exact case: a double's fourth root is either exact or irrational).
//  * x^0.2: 0.2 as a double is 1/5 + d with d = 2^-54/5, so
//    x^0.2 = x^(1/5) (1 + e), e = d ln x + (d ln x)^2 / 2 (|d ln x| < 1e-14).
//    After x = y 2^(5q) with y in [0.5, 16), a seed r0 = exp(log(y) / 5)
//    (accurate to a few ulp; no pow, so this header can also stand in for
//    the C library's pow) takes one Newton step on r^5 = y
//    with r0^5 formed in double-double: r = r0 - (r0^5 - y) / (5 r0^4),
//    quadratically accurate to ~2^-100; the (1 + e) factor is applied to the
//    double-double value before the single final rounding. The seed and
//    ln x only need a few correct bits, so the host's and the device's
//    exp and log give the same final result.
// Zero maps to zero, +inf to +inf, NaN and negative x to NaN, as pow does
// for these exponents.
#pragma once
#include <math.h>

#include "physics.cuh"

namespace m2c {
namespace crp {

// a*b = p + e exactly (fma form).
M2C_HD void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = fma(a, b, -p);
}

// a+b = s + e exactly (Knuth's branch-free form).
M2C_HD void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// (ah + al) * (bh + bl) as a double-double (relative error ~2^-104).
M2C_HD void dd_mul(double ah, double al, double bh, double bl, double& h, double& l) {
  double p, e;
  two_prod(ah, bh, p, e);
  e = e + (ah * bl + al * bh);
  two_sum(p, e, h, l);
}

// Split x > 0 finite as y * 2^(k*q) with y in [0.5, 2^k): frexp then move
// the exponent's remainder modulo k into y.
M2C_HD double split_exponent(double x, int k, int& q) {
  int ex;
  const double m = frexp(x, &ex);  // x = m 2^ex, m in [0.5, 1)
  int r = ex % k;
  if (r < 0) r += k;
  q = (ex - r) / k;
  return ldexp(m, r);
}

}  // namespace crp

// Correctly rounded x^0.25.
M2C_HD double cr_pow_quarter(double x) {
  if (!(x > 0.0) || x == INFINITY) return (x == 0.0 || x == INFINITY) ? x : NAN;
  int q;
  const double y = crp::split_exponent(x, 4, q);
  const double s = sqrt(y);
  const double s_lo = fma(-s, s, y) / (2.0 * s);  // y - s^2 is exact
  const double t = sqrt(s);
  const double t_lo = (fma(-t, t, s) + s_lo) / (2.0 * t);
  return ldexp(t + t_lo, q);
}

// Correctly rounded x^0.2 (0.2 the double nearest 1/5).
M2C_HD double cr_pow_fifth(double x) {
  if (!(x > 0.0) || x == INFINITY) return (x == 0.0 || x == INFINITY) ? x : NAN;
  int q;
  const double y = crp::split_exponent(x, 5, q);
  const double r0 = exp(0.2 * log(y));  // seed: a few ulp from y^(1/5)
  double h2, l2, h4, l4, h5, l5;
  crp::two_prod(r0, r0, h2, l2);
  crp::dd_mul(h2, l2, h2, l2, h4, l4);
  crp::dd_mul(h4, l4, r0, 0.0, h5, l5);
  // residual r0^5 - y: h5 - y is exact (Sterbenz: h5 is within a few ulp of y)
  const double res = (h5 - y) + l5;
  const double corr = res / (5.0 * h4);
  // (r0 - corr) (1 + e), e from d ln x with d = 0.2 - 1/5 = 2^-54 / 5
  const double dl = (0x1p-54 / 5.0) * log(x);
  const double e = dl + 0.5 * dl * dl;
  const double lo = (r0 * e - corr) - corr * e;
  return ldexp(r0 + lo, q);
}

}  // namespace m2c
