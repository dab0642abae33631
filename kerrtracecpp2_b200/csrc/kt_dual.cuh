// kt_dual.cuh -- forward-mode dual numbers for the differentiable tracer.
//
// Dual<N> carries a value and N tangents: x = v + sum_i d[i] e_i with
// e_i e_j = 0.  Arithmetic follows the first-order chain rule; sqrt and
// sincos use the library's own correctly rounded sqrt and ktm_sincos for the
// value.  Comparisons look at the value only, so branches taken on a Dual are
// the branches of the primal computation.
#pragma once

#include "kt_physics.cuh"

namespace kt {

template <int N>
struct Dual {
  double v;
  double d[N];

  KT_HD Dual() {}
  KT_HD Dual(double x) : v(x) {
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
  // Independent variable i of N.
  KT_HD static Dual var(double x, int i) {
    Dual r(x);
    r.d[i] = 1.0;
    return r;
  }
};

// Value of a double or a Dual.
KT_HD double val(double x) { return x; }
template <int N>
KT_HD double val(const Dual<N>& x) { return x.v; }

template <int N>
KT_HD Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
KT_HD Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
KT_HD Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
KT_HD Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
KT_HD Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v / b.v;
  const double ib = 1.0 / b.v;
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
// Mixed with double.
template <int N>
KT_HD Dual<N> operator+(const Dual<N>& a, double b) {
  Dual<N> r = a;
  r.v = a.v + b;
  return r;
}
template <int N>
KT_HD Dual<N> operator+(double a, const Dual<N>& b) { return b + a; }
template <int N>
KT_HD Dual<N> operator-(const Dual<N>& a, double b) {
  Dual<N> r = a;
  r.v = a.v - b;
  return r;
}
template <int N>
KT_HD Dual<N> operator-(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a - b.v;
  for (int i = 0; i < N; ++i) r.d[i] = -b.d[i];
  return r;
}
template <int N>
KT_HD Dual<N> operator*(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v * b;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
  return r;
}
template <int N>
KT_HD Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N>
KT_HD Dual<N> operator/(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v / b;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] / b;
  return r;
}
template <int N>
KT_HD Dual<N> operator/(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a / b.v;
  // d(a/b) = -(a/b)/b db; for a reciprocal (a = 1) -(1/b)^2 db without a
  // second division (the value, which the primal branches on, is a / b.v
  // either way)
  const double s = (a == 1.0) ? -(r.v * r.v) : -r.v / b.v;
  for (int i = 0; i < N; ++i) r.d[i] = s * b.d[i];
  return r;
}

template <int N>
KT_HD bool operator<(const Dual<N>& a, double b) { return a.v < b; }
template <int N>
KT_HD bool operator>(const Dual<N>& a, double b) { return a.v > b; }
template <int N>
KT_HD bool operator<=(const Dual<N>& a, double b) { return a.v <= b; }
template <int N>
KT_HD bool operator>=(const Dual<N>& a, double b) { return a.v >= b; }

// Elementary functions on doubles and Duals under one name.
KT_HD double sm_sqrt(double x) { return sqrt(x); }
template <int N>
KT_HD Dual<N> sm_sqrt(const Dual<N>& x) {
  Dual<N> r;
  r.v = sqrt(x.v);
  const double s = 0.5 / r.v;
  for (int i = 0; i < N; ++i) r.d[i] = x.d[i] * s;
  return r;
}

// The mixed-precision bundle's variants (not compared bit for bit): the
// value's reciprocal and sincos from mx_rcp and mx_sincos.
KT_HD double sm_rcp_fast(double x) { return mx_rcp<double>(x); }
template <int N>
KT_HD Dual<N> sm_rcp_fast(const Dual<N>& x) {
  Dual<N> r;
  r.v = mx_rcp<double>(x.v);
  const double s = -r.v * r.v;
  for (int i = 0; i < N; ++i) r.d[i] = s * x.d[i];
  return r;
}
KT_HD void sm_sincos_fast(double x, double* s, double* c) { mx_sincos(x, s, c); }
template <int N>
KT_HD void sm_sincos_fast(const Dual<N>& x, Dual<N>* s, Dual<N>* c) {
  double sv, cv;
  mx_sincos(x.v, &sv, &cv);
  s->v = sv;
  c->v = cv;
  for (int i = 0; i < N; ++i) {
    s->d[i] = cv * x.d[i];
    c->d[i] = -sv * x.d[i];
  }
}

KT_HD void sm_sincos(double x, double* s, double* c) { ktm_sincos(x, s, c); }
template <int N>
KT_HD void sm_sincos(const Dual<N>& x, Dual<N>* s, Dual<N>* c) {
  double sv, cv;
  ktm_sincos(x.v, &sv, &cv);
  s->v = sv;
  c->v = cv;
  for (int i = 0; i < N; ++i) {
    s->d[i] = cv * x.d[i];
    c->d[i] = -sv * x.d[i];
  }
}

KT_HD double sm_abs(double x) { return fabs(x); }
template <int N>
KT_HD Dual<N> sm_abs(const Dual<N>& x) { return x.v < 0.0 ? -x : x; }

}  // namespace kt
