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

// One evaluation carrying a Dual<1> (tangent d) and two hyper-duals (pairs
// a[k], b[k] with cross part c[k], k = 0, 1) that share a value:
//   x = v + d e + sum_k (a_k e1k + b_k e2k + c_k e1k e2k),
// products of different infinitesimals dropped.  Each part follows, operation
// for operation, the rule of the type it stands for (the d part Dual<1>'s,
// the others HDual's), so its results equal those of the three separate
// evaluations bit for bit, at the cost of one value and one reciprocal.
struct BDual {
  double v, d, a[2], b[2], c[2];
  KT_HD BDual() {}
  KT_HD BDual(double x) : v(x), d(0.0) {
    for (int k = 0; k < 2; ++k) a[k] = b[k] = c[k] = 0.0;
  }
};
KT_HD double val(const BDual& x) { return x.v; }
KT_HD BDual operator+(const BDual& x, const BDual& y) {
  BDual r;
  r.v = x.v + y.v;
  r.d = x.d + y.d;
  for (int k = 0; k < 2; ++k) {
    r.a[k] = x.a[k] + y.a[k];
    r.b[k] = x.b[k] + y.b[k];
    r.c[k] = x.c[k] + y.c[k];
  }
  return r;
}
KT_HD BDual operator-(const BDual& x, const BDual& y) {
  BDual r;
  r.v = x.v - y.v;
  r.d = x.d - y.d;
  for (int k = 0; k < 2; ++k) {
    r.a[k] = x.a[k] - y.a[k];
    r.b[k] = x.b[k] - y.b[k];
    r.c[k] = x.c[k] - y.c[k];
  }
  return r;
}
KT_HD BDual operator-(const BDual& x) {
  BDual r;
  r.v = -x.v;
  r.d = -x.d;
  for (int k = 0; k < 2; ++k) {
    r.a[k] = -x.a[k];
    r.b[k] = -x.b[k];
    r.c[k] = -x.c[k];
  }
  return r;
}
KT_HD BDual operator*(const BDual& x, const BDual& y) {
  BDual r;
  r.v = x.v * y.v;
  r.d = x.d * y.v + x.v * y.d;
  for (int k = 0; k < 2; ++k) {
    r.a[k] = x.a[k] * y.v + x.v * y.a[k];
    r.b[k] = x.b[k] * y.v + x.v * y.b[k];
    r.c[k] = x.c[k] * y.v + x.v * y.c[k] + x.a[k] * y.b[k] + x.b[k] * y.a[k];
  }
  return r;
}
KT_HD BDual operator+(const BDual& x, double y) {
  BDual r = x;
  r.v = x.v + y;
  return r;
}
KT_HD BDual operator+(double x, const BDual& y) { return y + x; }
KT_HD BDual operator-(const BDual& x, double y) {
  BDual r = x;
  r.v = x.v - y;
  return r;
}
KT_HD BDual operator-(double x, const BDual& y) {
  BDual r = -y;
  r.v = x - y.v;
  return r;
}
KT_HD BDual operator*(const BDual& x, double y) {
  BDual r;
  r.v = x.v * y;
  r.d = x.d * y;
  for (int k = 0; k < 2; ++k) {
    r.a[k] = x.a[k] * y;
    r.b[k] = x.b[k] * y;
    r.c[k] = x.c[k] * y;
  }
  return r;
}
KT_HD BDual operator*(double x, const BDual& y) { return y * x; }
KT_HD BDual operator/(const BDual& x, double y) {
  BDual r;
  r.v = x.v / y;
  r.d = x.d / y;
  for (int k = 0; k < 2; ++k) {
    r.a[k] = x.a[k] / y;
    r.b[k] = x.b[k] / y;
    r.c[k] = x.c[k] / y;
  }
  return r;
}
// x / y: the d part as Dual<1>'s division, the pairs as HDual's
KT_HD BDual operator/(double x, const BDual& y) {
  BDual r;
  r.v = x / y.v;
  const double s = (x == 1.0) ? -(r.v * r.v) : -r.v / y.v;
  r.d = s * y.d;
  const double iy = 1.0 / y.v;
  const double f1 = -r.v * iy;
  const double f2 = -2.0 * f1 * iy;
  for (int k = 0; k < 2; ++k) {
    r.a[k] = f1 * y.a[k];
    r.b[k] = f1 * y.b[k];
    r.c[k] = f1 * y.c[k] + f2 * y.a[k] * y.b[k];
  }
  return r;
}
KT_HD bool operator<(const BDual& x, double y) { return x.v < y; }
KT_HD bool operator>(const BDual& x, double y) { return x.v > y; }
KT_HD bool operator<=(const BDual& x, double y) { return x.v <= y; }
KT_HD bool operator>=(const BDual& x, double y) { return x.v >= y; }
KT_HD void sm_sincos(const BDual& x, BDual* s, BDual* c) {
  double sv, cv;
  ktm_sincos(x.v, &sv, &cv);
  s->v = sv;
  c->v = cv;
  s->d = cv * x.d;
  c->d = -sv * x.d;
  for (int k = 0; k < 2; ++k) {
    const double ab = x.a[k] * x.b[k];
    s->a[k] = cv * x.a[k];
    s->b[k] = cv * x.b[k];
    s->c[k] = cv * x.c[k] - sv * ab;
    c->a[k] = -sv * x.a[k];
    c->b[k] = -sv * x.b[k];
    c->c[k] = -sv * x.c[k] - cv * ab;
  }
}

}  // namespace kt
