// gg_dual.cuh -- forward-mode dual numbers for the differentiable render.
//
// Dual<N> carries a value and its derivatives along N directions.  The
// adjoint kernels (gg_adjoint.cu) use it for the Jacobians of the crossing
// step and of the camera's initial state, and gg_vjp.cuh for the dual form
// of the stage product (the check beside the hand-written reverse pass), by
// running the same templated physics (kerr_geometry / kerr_contract) on
// Dual<N> instead of double.  Only the operations that code uses are defined.
#pragma once

#include <cuda_runtime.h>

namespace gg {

template <int N>
struct Dual {
  double v;
  double d[N];
  GG_DEV Dual() : v(0.0) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
  GG_DEV Dual(double x) : v(x) {  // NOLINT: constants convert implicitly
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
  GG_DEV static Dual var(double x, int dir) {
    Dual r(x);
    r.d[dir] = 1.0;
    return r;
  }
};

template <int N>
GG_DEV Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
GG_DEV Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
GG_DEV Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
GG_DEV Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
GG_DEV Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  const double ib = 1.0 / b.v;
  r.v = a.v * ib;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <int N>
GG_DEV Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N>
GG_DEV Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N>
GG_DEV Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N>
GG_DEV Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
GG_DEV Dual<N> operator*(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v * b;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
  return r;
}
template <int N>
GG_DEV Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N>
GG_DEV Dual<N> operator/(const Dual<N>& a, double b) { return a * (1.0 / b); }
template <int N>
GG_DEV Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }

template <int N>
GG_DEV Dual<N> rcp(const Dual<N>& x) { return 1.0 / x; }

template <int N>
GG_DEV Dual<N> sqrt(const Dual<N>& x) {
  Dual<N> r;
  r.v = ::sqrt(x.v);
  const double k = 0.5 / r.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = x.d[i] * k;
  return r;
}

template <int N>
GG_DEV Dual<N> log(const Dual<N>& x) {
  Dual<N> r;
  r.v = ::log(x.v);
  const double k = 1.0 / x.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = x.d[i] * k;
  return r;
}

// x^p for a constant exponent p (x > 0)
template <int N>
GG_DEV Dual<N> pow(const Dual<N>& x, double p) {
  Dual<N> r;
  r.v = ::pow(x.v, p);
  const double k = p * r.v / x.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = x.d[i] * k;
  return r;
}

template <int N>
GG_DEV void sincos(const Dual<N>& x, Dual<N>* s, Dual<N>* c) {
  double sv, cv;
  ::sincos(x.v, &sv, &cv);
  s->v = sv;
  c->v = cv;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    s->d[i] = cv * x.d[i];
    c->d[i] = -sv * x.d[i];
  }
}

template <int N>
GG_DEV Dual<N> dmax(const Dual<N>& a, double b) { return a.v >= b ? a : Dual<N>(b); }

}  // namespace gg
