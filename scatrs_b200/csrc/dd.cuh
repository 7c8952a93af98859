// Double-double arithmetic (an unevaluated sum hi + lo of two doubles, about 106 bits) for the
// spheroid T-matrix's surface integrals, whose outgoing terms cancel by many orders of
// magnitude. The building blocks are the published error-free transformations: Knuth's
// two-sum, Dekker's fast two-sum, and the product error from one fused multiply-add; the
// compound operations follow the usual double-double constructions (addition with both error
// terms carried, division by two correction steps, square root by one Newton step), and the
// elementary functions reduce their argument with multi-part constants and sum Taylor series.
// Usable on the host (Gauss-Legendre rules) and the device; needs IEEE double with a
// correctly rounded fma and no reassociation.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace sb {
namespace ddm {

#define DD_FN __host__ __device__ __forceinline__

struct dd {
  double hi, lo;
};

DD_FN dd mkdd(double h, double l = 0.0) { return dd{h, l}; }

DD_FN dd two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  return dd{s, (a - (s - bb)) + (b - bb)};
}
DD_FN dd fast_two_sum(double a, double b) {  // |a| >= |b| or a == 0
  const double s = a + b;
  return dd{s, b - (s - a)};
}
DD_FN dd two_prod(double a, double b) {
  const double p = a * b;
  return dd{p, fma(a, b, -p)};
}

DD_FN dd operator+(dd x, dd y) {
  dd s = two_sum(x.hi, y.hi);
  const dd t = two_sum(x.lo, y.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
DD_FN dd operator-(dd x) { return dd{-x.hi, -x.lo}; }
DD_FN dd operator-(dd x, dd y) { return x + (-y); }
DD_FN dd operator+(dd x, double y) {
  dd s = two_sum(x.hi, y);
  s.lo += x.lo;
  return fast_two_sum(s.hi, s.lo);
}
DD_FN dd operator-(dd x, double y) { return x + (-y); }
// Products: the exact error of hi * hi from one fma, the cross terms folded into it by two
// more.
DD_FN dd operator*(dd x, dd y) {
  const double p = x.hi * y.hi;
  double e = fma(x.hi, y.hi, -p);
  e = fma(x.hi, y.lo, e);
  e = fma(x.lo, y.hi, e);
  return fast_two_sum(p, e);
}
DD_FN dd operator*(dd x, double y) {
  const double p = x.hi * y;
  double e = fma(x.hi, y, -p);
  e = fma(x.lo, y, e);
  return fast_two_sum(p, e);
}
// x + y with one two-sum (the low parts added in double): its error is about 2^-106 of
// max(|x|, |y|) rather than of |x + y|, which sums whose accuracy is measured against the
// size of their terms can afford.
DD_FN dd add_terms(dd x, dd y) {
  dd s = two_sum(x.hi, y.hi);
  s.lo += x.lo + y.lo;
  return fast_two_sum(s.hi, s.lo);
}
DD_FN dd operator/(dd x, double y) {
  const double q1 = x.hi / y;
  const dd r = x - two_prod(q1, y);
  const double q2 = r.hi / y;
  const dd r2 = r - two_prod(q2, y);
  const double q3 = r2.hi / y;
  return fast_two_sum(q1, q2) + q3;
}
DD_FN dd operator/(dd x, dd y) {
  const double q1 = x.hi / y.hi;
  const dd r = x - y * q1;
  const double q2 = r.hi / y.hi;
  const dd r2 = r - y * q2;
  const double q3 = r2.hi / y.hi;
  return fast_two_sum(q1, q2) + q3;
}
DD_FN dd ldexp_dd(dd x, int e) { return dd{ldexp(x.hi, e), ldexp(x.lo, e)}; }

DD_FN dd dd_sqrt(dd x) {
  if (!(x.hi > 0.0)) return dd{0.0, 0.0};
  const double s = sqrt(x.hi);
  const dd r = x - two_prod(s, s);
  return fast_two_sum(s, r.hi / (2.0 * s));
}
DD_FN dd dd_sqrt(double x) { return dd_sqrt(dd{x, 0.0}); }

// x - k c for a constant c = c0 + c1 + c2 given in three parts, for an integer-valued k of at
// most 2^26 or so. pi/2 and ln 2 in three parts:
#define DD_PIO2 1.5707963267948966, 6.123233995736766e-17, -1.4973849048591698e-33
#define DD_LN2 0.6931471805599453, 2.3190468138462996e-17, 5.707708438416212e-34
DD_FN dd reduce(dd x, double k, double c0, double c1, double c2) {
  dd r = x - two_prod(k, c0);
  r = r - two_prod(k, c1);
  return r + (-(k * c2));
}

// sin and cos of |r| <= pi/4 by their Taylor series in nested (Horner) form, 14 factors each:
// the first omitted term is below 4e-33 of the result.
DD_FN void sincos_reduced(dd r, dd* s, dd* c) {
  const dd r2 = r * r;
  dd ts = mkdd(1.0), tc = mkdd(1.0);
  for (int k = 14; k >= 1; --k) {
    ts = mkdd(1.0) - (r2 * ts) / (double)((2 * k) * (2 * k + 1));
    tc = mkdd(1.0) - (r2 * tc) / (double)((2 * k - 1) * (2 * k));
  }
  *s = r * ts;
  *c = tc;
}

DD_FN void dd_sincos(dd x, dd* s, dd* c) {
  const double k = rint(x.hi / 1.5707963267948966);
  const dd r = reduce(x, k, DD_PIO2);
  dd sr, cr;
  sincos_reduced(r, &sr, &cr);
  const long long q = ((long long)k) & 3;
  if (q == 0) {
    *s = sr;
    *c = cr;
  } else if (q == 1) {
    *s = cr;
    *c = -sr;
  } else if (q == 2) {
    *s = -sr;
    *c = -cr;
  } else {
    *s = -cr;
    *c = sr;
  }
}

// e^x: x = k ln 2 + r, e^r from e^(r / 256) - 1 (Taylor, 10 terms) squared eight times as
// (1 + u)^2 - 1 = u (2 + u), then scaled by 2^k.
DD_FN dd dd_exp(dd x) {
  if (x.hi > 709.0) return dd{INFINITY, 0.0};
  if (x.hi < -745.0) return dd{0.0, 0.0};
  const double k = rint(x.hi / 0.6931471805599453);
  const dd r = ldexp_dd(reduce(x, k, DD_LN2), -8);
  dd t = mkdd(1.0);
  for (int j = 10; j >= 2; --j) t = mkdd(1.0) + (r * t) / (double)j;
  dd u = r * t;  // e^r' - 1
  for (int i = 0; i < 8; ++i) u = u * (u + 2.0);
  return ldexp_dd(u + 1.0, (int)k);
}

DD_FN void dd_sinhcosh(dd x, dd* sh, dd* ch) {
  const dd e = dd_exp(x);
  const dd ie = mkdd(1.0) / e;
  *sh = ldexp_dd(e - ie, -1);
  *ch = ldexp_dd(e + ie, -1);
}

// Complex double-double.
struct cdd {
  dd re, im;
};
DD_FN cdd mkc(dd re, dd im) { return cdd{re, im}; }
DD_FN cdd mkc(double re, double im = 0.0) { return cdd{mkdd(re), mkdd(im)}; }
DD_FN cdd operator+(cdd a, cdd b) { return cdd{a.re + b.re, a.im + b.im}; }
DD_FN cdd operator-(cdd a, cdd b) { return cdd{a.re - b.re, a.im - b.im}; }
DD_FN cdd operator-(cdd a) { return cdd{-a.re, -a.im}; }
DD_FN cdd operator*(cdd a, cdd b) {
  return cdd{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
DD_FN cdd operator*(cdd a, dd s) { return cdd{a.re * s, a.im * s}; }
DD_FN cdd operator*(cdd a, double s) { return cdd{a.re * s, a.im * s}; }
DD_FN cdd times_i(cdd a) { return cdd{-a.im, a.re}; }
// Complex operations with add_terms.
DD_FN cdd add_terms(cdd a, cdd b) { return cdd{add_terms(a.re, b.re), add_terms(a.im, b.im)}; }
DD_FN cdd sub_terms(cdd a, cdd b) { return cdd{add_terms(a.re, -b.re), add_terms(a.im, -b.im)}; }
DD_FN cdd mul_terms(cdd a, cdd b) {
  return cdd{add_terms(a.re * b.re, -(a.im * b.im)), add_terms(a.re * b.im, a.im * b.re)};
}
DD_FN dd norm2(cdd a) { return a.re * a.re + a.im * a.im; }
// 1 / a, scaled by a power of two first so that |a|^2 neither overflows nor underflows.
DD_FN cdd inv(cdd a) {
  const double m = fmax(fabs(a.re.hi), fabs(a.im.hi));
  const int e = m > 0.0 ? ilogb(m) : 0;
  const cdd b{ldexp_dd(a.re, -e), ldexp_dd(a.im, -e)};
  const dd d = norm2(b);
  return cdd{ldexp_dd(b.re / d, -e), ldexp_dd(-b.im / d, -e)};
}

// sin z and cos z of a complex argument.
DD_FN void c_sincos(cdd z, cdd* s, cdd* c) {
  dd sr, cr, sh, ch;
  dd_sincos(z.re, &sr, &cr);
  dd_sinhcosh(z.im, &sh, &ch);
  *s = cdd{sr * ch, cr * sh};
  *c = cdd{cr * ch, -(sr * sh)};
}

#undef DD_FN

}  // namespace ddm
}  // namespace sb
