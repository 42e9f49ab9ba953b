// gg_counting.hpp -- a double that tallies the arithmetic done with it.
//
// TEST INFRASTRUCTURE ONLY.  Instantiating the oracle's metric and RK45
// templates with CountingDouble counts the floating-point operations of one
// reference RK45 attempt (the algorithmic work unit of the roofline).  Each
// +, -, *, / and unary minus counts one op of its kind; library functions
// count one call of their kind.
#pragma once

#include <cmath>
#include <cstdint>

namespace ggo {

struct OpCounts {
  uint64_t add = 0, mul = 0, div = 0, neg = 0, sqrt = 0, sin = 0, cos = 0, pow = 0, exp = 0,
           other = 0;
};

inline OpCounts& op_counts() {
  static thread_local OpCounts c;
  return c;
}

struct CountingDouble {
  double v;
  CountingDouble() : v(0.0) {}
  CountingDouble(double x) : v(x) {}  // NOLINT: implicit on purpose
};

using CD = CountingDouble;
inline CD operator+(CD a, CD b) { op_counts().add++; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { op_counts().add++; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { op_counts().mul++; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { op_counts().div++; return CD(a.v / b.v); }
inline CD operator-(CD a) { op_counts().neg++; return CD(-a.v); }
inline bool operator<(CD a, CD b) { return a.v < b.v; }
inline bool operator>(CD a, CD b) { return a.v > b.v; }
inline bool operator<=(CD a, CD b) { return a.v <= b.v; }
inline bool operator>=(CD a, CD b) { return a.v >= b.v; }
inline bool operator==(CD a, CD b) { return a.v == b.v; }
inline CD sqrt(CD a) { op_counts().sqrt++; return CD(std::sqrt(a.v)); }
inline CD sin(CD a) { op_counts().sin++; return CD(std::sin(a.v)); }
inline CD cos(CD a) { op_counts().cos++; return CD(std::cos(a.v)); }
inline CD pow(CD a, CD b) { op_counts().pow++; return CD(std::pow(a.v, b.v)); }
inline CD exp(CD a) { op_counts().exp++; return CD(std::exp(a.v)); }
inline CD fabs(CD a) { return CD(std::fabs(a.v)); }
inline CD fmax(CD a, CD b) { op_counts().other++; return CD(std::fmax(a.v, b.v)); }
inline CD fmod(CD a, CD b) { op_counts().other++; return CD(std::fmod(a.v, b.v)); }
inline bool isfinite(CD a) { return std::isfinite(a.v); }

}  // namespace ggo
