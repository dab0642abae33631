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

// Hyper-dual numbers x = v + a e1 + b e2 + c e1 e2 with e1^2 = e2^2 = 0
// (Fike and Alonso, "The development of hyper-dual numbers for exact
// second-derivative calculations", AIAA 2011-886): f(x) = f(v) + f'(v) a e1 +
// f'(v) b e2 + (f'(v) c + f''(v) a b) e1 e2, so evaluating g at x0 + e1 u +
// e2 w gives g's second directional derivative D^2 g[u, w] in the e1 e2 part.
// Only the operations of the BL Hamiltonian gradient are defined.  The
// values follow the primal's operations (comparisons look at v).
struct HDual {
  double v, a, b, c;
  KT_HD HDual() {}
  KT_HD HDual(double x) : v(x), a(0.0), b(0.0), c(0.0) {}
  KT_HD HDual(double x, double da, double db, double dc) : v(x), a(da), b(db), c(dc) {}
};
KT_HD double val(const HDual& x) { return x.v; }
KT_HD HDual operator+(const HDual& x, const HDual& y) {
  return HDual(x.v + y.v, x.a + y.a, x.b + y.b, x.c + y.c);
}
KT_HD HDual operator-(const HDual& x, const HDual& y) {
  return HDual(x.v - y.v, x.a - y.a, x.b - y.b, x.c - y.c);
}
KT_HD HDual operator-(const HDual& x) { return HDual(-x.v, -x.a, -x.b, -x.c); }
KT_HD HDual operator*(const HDual& x, const HDual& y) {
  return HDual(x.v * y.v, x.a * y.v + x.v * y.a, x.b * y.v + x.v * y.b,
               x.c * y.v + x.v * y.c + x.a * y.b + x.b * y.a);
}
KT_HD HDual operator+(const HDual& x, double y) { return HDual(x.v + y, x.a, x.b, x.c); }
KT_HD HDual operator+(double x, const HDual& y) { return y + x; }
KT_HD HDual operator-(const HDual& x, double y) { return HDual(x.v - y, x.a, x.b, x.c); }
KT_HD HDual operator-(double x, const HDual& y) { return HDual(x - y.v, -y.a, -y.b, -y.c); }
KT_HD HDual operator*(const HDual& x, double y) { return HDual(x.v * y, x.a * y, x.b * y, x.c * y); }
KT_HD HDual operator*(double x, const HDual& y) { return y * x; }
KT_HD HDual operator/(const HDual& x, double y) { return HDual(x.v / y, x.a / y, x.b / y, x.c / y); }
// x / y: the value x / y.v; f(y) = x / y, f' = -f / y, f'' = -2 f' / y
KT_HD HDual operator/(double x, const HDual& y) {
  const double f = x / y.v;
  const double iy = 1.0 / y.v;
  const double f1 = -f * iy;
  const double f2 = -2.0 * f1 * iy;
  return HDual(f, f1 * y.a, f1 * y.b, f1 * y.c + f2 * y.a * y.b);
}
KT_HD bool operator<(const HDual& x, double y) { return x.v < y; }
KT_HD bool operator>(const HDual& x, double y) { return x.v > y; }
KT_HD bool operator<=(const HDual& x, double y) { return x.v <= y; }
KT_HD bool operator>=(const HDual& x, double y) { return x.v >= y; }
KT_HD void sm_sincos(const HDual& x, HDual* s, HDual* c) {
  double sv, cv;
  ktm_sincos(x.v, &sv, &cv);
  const double ab = x.a * x.b;
  *s = HDual(sv, cv * x.a, cv * x.b, cv * x.c - sv * ab);
  *c = HDual(cv, -sv * x.a, -sv * x.b, -sv * x.c - cv * ab);
}

}  // namespace kt
