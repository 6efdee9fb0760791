// Forward-mode dual numbers for the CPU adjoint tests (test infrastructure).
//
// The pointwise microphysics routines are templates on their real type; run
// with Dual they return, next to each value, its derivatives with respect to
// up to NDIR seeded inputs, following the branches the double evaluation
// takes at the same point. Their Jacobian-transpose products are the exact
// reference for the hand-written adjoints. Ties of fmin/fmax go to the first
// argument (a <= b for fmin, a >= b for fmax), as in the adjoints.
#pragma once

#include <cmath>

namespace shield {

// the double versions stay visible next to the Dual overloads below
using std::fabs;
using std::fmax;
using std::fmin;
using std::sqrt;

constexpr int NDIR = 24;

// ABS = true gives the magnitude dual: every derivative contribution is
// accumulated in absolute value, so d[i] bounds the size of the terms that
// make up the derivative (the scale of its rounding error), not the
// derivative itself.
template <bool ABS>
struct DualT {
  double v;
  double d[NDIR];
  DualT() : v(0.0) {
    for (int i = 0; i < NDIR; ++i) d[i] = 0.0;
  }
  DualT(double x) : v(x) {  // NOLINT: constants promote implicitly
    for (int i = 0; i < NDIR; ++i) d[i] = 0.0;
  }
  static DualT seed(double x, int i) {
    DualT r(x);
    r.d[i] = 1.0;
    return r;
  }
};
using Dual = DualT<false>;
using ADual = DualT<true>;

template <bool A>
inline DualT<A> scale_add(const DualT<A>& a, double ca, const DualT<A>& b, double cb, double v) {
  DualT<A> r;
  r.v = v;
  if (A) {
    ca = std::fabs(ca);
    cb = std::fabs(cb);
  }
  for (int i = 0; i < NDIR; ++i) r.d[i] = ca * a.d[i] + cb * b.d[i];
  return r;
}
template <bool A>
inline DualT<A> chain(const DualT<A>& a, double da, double v) {
  DualT<A> r;
  r.v = v;
  if (A) da = std::fabs(da);
  for (int i = 0; i < NDIR; ++i) r.d[i] = da * a.d[i];
  return r;
}

template <bool A>
inline DualT<A> operator+(const DualT<A>& a, const DualT<A>& b) { return scale_add(a, 1.0, b, 1.0, a.v + b.v); }
template <bool A>
inline DualT<A> operator-(const DualT<A>& a, const DualT<A>& b) { return scale_add(a, 1.0, b, -1.0, a.v - b.v); }
template <bool A>
inline DualT<A> operator*(const DualT<A>& a, const DualT<A>& b) { return scale_add(a, b.v, b, a.v, a.v * b.v); }
template <bool A>
inline DualT<A> operator/(const DualT<A>& a, const DualT<A>& b) {
  const double q = a.v / b.v;
  return scale_add(a, 1.0 / b.v, b, -q / b.v, q);
}
template <bool A>
inline DualT<A> operator-(const DualT<A>& a) { return chain(a, -1.0, -a.v); }
template <bool A>
inline DualT<A> operator+(const DualT<A>& a, double b) { return chain(a, 1.0, a.v + b); }
template <bool A>
inline DualT<A> operator+(double a, const DualT<A>& b) { return chain(b, 1.0, a + b.v); }
template <bool A>
inline DualT<A> operator-(const DualT<A>& a, double b) { return chain(a, 1.0, a.v - b); }
template <bool A>
inline DualT<A> operator-(double a, const DualT<A>& b) { return chain(b, -1.0, a - b.v); }
template <bool A>
inline DualT<A> operator*(const DualT<A>& a, double b) { return chain(a, b, a.v * b); }
template <bool A>
inline DualT<A> operator*(double a, const DualT<A>& b) { return chain(b, a, a * b.v); }
template <bool A>
inline DualT<A> operator/(const DualT<A>& a, double b) { return chain(a, 1.0 / b, a.v / b); }
template <bool A>
inline DualT<A> operator/(double a, const DualT<A>& b) {
  const double q = a / b.v;
  return chain(b, -q / b.v, q);
}

#define SHIELD_DUAL_CMP(op)                                                                 \
  template <bool A>                                                                         \
  inline bool operator op(const DualT<A>& a, const DualT<A>& b) { return a.v op b.v; }      \
  template <bool A>                                                                         \
  inline bool operator op(const DualT<A>& a, double b) { return a.v op b; }                 \
  template <bool A>                                                                         \
  inline bool operator op(double a, const DualT<A>& b) { return a op b.v; }
SHIELD_DUAL_CMP(<)
SHIELD_DUAL_CMP(>)
SHIELD_DUAL_CMP(<=)
SHIELD_DUAL_CMP(>=)
#undef SHIELD_DUAL_CMP

template <bool A>
inline DualT<A> sqrt(const DualT<A>& a) {
  const double s = std::sqrt(a.v);
  return chain(a, 0.5 / s, s);
}
template <bool A>
inline DualT<A> fabs(const DualT<A>& a) { return a.v >= 0.0 ? a : -a; }
template <bool A>
inline DualT<A> fmin(const DualT<A>& a, const DualT<A>& b) { return a.v <= b.v ? a : b; }
template <bool A>
inline DualT<A> fmin(const DualT<A>& a, double b) { return a.v <= b ? a : DualT<A>(b); }
template <bool A>
inline DualT<A> fmin(double a, const DualT<A>& b) { return a <= b.v ? DualT<A>(a) : b; }
template <bool A>
inline DualT<A> fmax(const DualT<A>& a, const DualT<A>& b) { return a.v >= b.v ? a : b; }
template <bool A>
inline DualT<A> fmax(const DualT<A>& a, double b) { return a.v >= b ? a : DualT<A>(b); }
template <bool A>
inline DualT<A> fmax(double a, const DualT<A>& b) { return a >= b.v ? DualT<A>(a) : b; }
template <bool A>
inline DualT<A> xexp(const DualT<A>& a) {
  const double e = std::exp(a.v);
  return chain(a, e, e);
}
template <bool A>
inline DualT<A> xlog(const DualT<A>& a) { return chain(a, 1.0 / a.v, std::log(a.v)); }
template <bool A>
inline DualT<A> xpow(const DualT<A>& a, const DualT<A>& b) {
  const double p = std::pow(a.v, b.v);
  DualT<A> r = chain(a, p * b.v / a.v, p);
  if (a.v > 0.0)
    for (int i = 0; i < NDIR; ++i) r.d[i] += p * std::log(a.v) * b.d[i];
  return r;
}
template <bool A>
inline DualT<A> xpow(const DualT<A>& a, double b) {
  const double p = std::pow(a.v, b);
  return chain(a, p * b / a.v, p);
}
template <bool A>
inline DualT<A> dim(const DualT<A>& x, const DualT<A>& y) { return (x.v - y.v > 0.0) ? x - y : DualT<A>(0.0); }
template <bool A>
inline DualT<A> dim(double x, const DualT<A>& y) { return (x - y.v > 0.0) ? x - y : DualT<A>(0.0); }
template <bool A>
inline DualT<A> dim(const DualT<A>& x, double y) { return (x.v - y > 0.0) ? x - y : DualT<A>(0.0); }
template <bool A>
inline DualT<A> sq(const DualT<A>& x) { return x * x; }

}  // namespace shield
