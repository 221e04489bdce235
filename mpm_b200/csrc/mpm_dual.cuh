// mpm_dual.cuh -- forward-mode (tangent) arithmetic: a value with its
// derivatives with respect to NT parameters.  Every operation propagates the
// derivatives by the chain rule; comparisons look at the value only, so a
// branch taken by the value arithmetic is taken the same way here and the
// derivative is that of the branch taken (the derivative of a piecewise
// function away from its switch points).
#pragma once

#include <cmath>

#include "mpm_math.cuh"

namespace mpm_b200 {

constexpr int NT = 2;  // parameters differentiated at once

struct Dual {
  double v;
  double d[NT];
  MPM_HD Dual() : v(0.0) {
#pragma unroll
    for (int k = 0; k < NT; ++k) d[k] = 0.0;
  }
  MPM_HD Dual(double x) : v(x) {
#pragma unroll
    for (int k = 0; k < NT; ++k) d[k] = 0.0;
  }
  MPM_HD Dual& operator+=(const Dual& b) {
    v += b.v;
#pragma unroll
    for (int k = 0; k < NT; ++k) d[k] += b.d[k];
    return *this;
  }
  MPM_HD Dual& operator-=(const Dual& b) {
    v -= b.v;
#pragma unroll
    for (int k = 0; k < NT; ++k) d[k] -= b.d[k];
    return *this;
  }
  MPM_HD Dual& operator*=(const Dual& b);
  MPM_HD Dual& operator/=(const Dual& b);
};

MPM_HD Dual operator-(const Dual& a) {
  Dual r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < NT; ++k) r.d[k] = -a.d[k];
  return r;
}
MPM_HD Dual operator+(const Dual& a, const Dual& b) {
  Dual r = a;
  r += b;
  return r;
}
MPM_HD Dual operator-(const Dual& a, const Dual& b) {
  Dual r = a;
  r -= b;
  return r;
}
MPM_HD Dual operator*(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < NT; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
MPM_HD Dual operator/(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v / b.v;
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int k = 0; k < NT; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
MPM_HD Dual operator+(const Dual& a, double b) { return a + Dual(b); }
MPM_HD Dual operator+(double a, const Dual& b) { return Dual(a) + b; }
MPM_HD Dual operator-(const Dual& a, double b) { return a - Dual(b); }
MPM_HD Dual operator-(double a, const Dual& b) { return Dual(a) - b; }
MPM_HD Dual operator*(const Dual& a, double b) {
  Dual r;
  r.v = a.v * b;
#pragma unroll
  for (int k = 0; k < NT; ++k) r.d[k] = a.d[k] * b;
  return r;
}
MPM_HD Dual operator*(double a, const Dual& b) { return b * a; }
MPM_HD Dual operator/(const Dual& a, double b) { return a / Dual(b); }
MPM_HD Dual operator/(double a, const Dual& b) { return Dual(a) / b; }
MPM_HD Dual& Dual::operator*=(const Dual& b) {
  *this = *this * b;
  return *this;
}
MPM_HD Dual& Dual::operator/=(const Dual& b) {
  *this = *this / b;
  return *this;
}

#define MPM_DUAL_CMP(op)                                                      \
  MPM_HD bool operator op(const Dual& a, const Dual& b) { return a.v op b.v; } \
  MPM_HD bool operator op(const Dual& a, double b) { return a.v op b; }        \
  MPM_HD bool operator op(double a, const Dual& b) { return a op b.v; }
MPM_DUAL_CMP(<)
MPM_DUAL_CMP(>)
MPM_DUAL_CMP(<=)
MPM_DUAL_CMP(>=)
MPM_DUAL_CMP(==)
MPM_DUAL_CMP(!=)
#undef MPM_DUAL_CMP

// f(a) with derivative f'(a) * da
MPM_HD Dual chain(const Dual& a, double f, double df) {
  Dual r;
  r.v = f;
#pragma unroll
  for (int k = 0; k < NT; ++k) r.d[k] = df * a.d[k];
  return r;
}
// sqrt: the derivative at 0 is taken as 0 (a norm of a zero vector)
MPM_HD Dual sqrt(const Dual& a) {
  const double s = ::sqrt(a.v);
  return chain(a, s, s > 0.0 ? 0.5 / s : 0.0);
}
MPM_HD Dual sin(const Dual& a) { return chain(a, ::sin(a.v), ::cos(a.v)); }
MPM_HD Dual cos(const Dual& a) { return chain(a, ::cos(a.v), -::sin(a.v)); }
MPM_HD Dual tan(const Dual& a) {
  const double t = ::tan(a.v);
  return chain(a, t, 1.0 + t * t);
}
MPM_HD Dual acos(const Dual& a) {
  const double q = 1.0 - a.v * a.v;
  return chain(a, ::acos(a.v), q > 0.0 ? -1.0 / ::sqrt(q) : 0.0);
}
MPM_HD Dual pow(const Dual& a, double e) {
  const double p = ::pow(a.v, e);
  return chain(a, p, a.v != 0.0 ? e * p / a.v : 0.0);
}
MPM_HD Dual pow(const Dual& a, const Dual& e) { return pow(a, e.v); }  // constant exponents only
MPM_HD Dual fabs(const Dual& a) { return a.v < 0.0 ? -a : a; }
MPM_HD bool isfinite(const Dual& a) { return a.v - a.v == 0.0; }
MPM_HD void sin_cos(const Dual& x, Dual* sn, Dual* cs) {
  double s, c;
  sin_cos(x.v, &s, &c);
  *sn = chain(x, s, c);
  *cs = chain(x, c, -s);
}
MPM_HD double value(const Dual& a) { return a.v; }

// Within MPM_LODE_CORNER_TOL of a triaxial corner of the MohrCoulomb surface
// (distance 1 - cos^2 3 theta) the Lode angle's derivative is taken as zero
// (values are unchanged): theta is acos of a ratio, so d theta / d sigma
// grows without bound at the corner.
#ifndef MPM_LODE_CORNER_TOL
#define MPM_LODE_CORNER_TOL 1e-8
#endif
template <>
MPM_HD Dual lode_corner<Dual>(const Dual& x, double dist_to_corner) {
  return dist_to_corner < MPM_LODE_CORNER_TOL ? Dual(x.v) : x;
}

template <>
MPM_HD Dual huge_value<Dual>() {
  return Dual(1.7976931348623157e308);
}

// the invariants of a Dual state are evaluated in Dual (not rounded to FP64)
template <>
struct HighPrecision<Dual> {
  using T = Dual;
};

}  // namespace mpm_b200
