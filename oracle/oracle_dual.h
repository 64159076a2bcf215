/*
 * oracle_dual.h -- TEST INFRASTRUCTURE ONLY (see oracle_common.h).
 *
 * A forward-mode dual number (value, derivative) in double precision.  The
 * oracle's transport is templated on OLAM's `real`; instantiated on Dual it
 * computes, besides the FP64 step, the exact directional derivative of the
 * step (the tangent-linear map) along the derivative parts of its inputs.
 * Comparisons act on the value, so every branch of a min / max / sign test
 * takes the side the FP64 step takes, and the derivative is that of the
 * branch taken: the Jacobian of the step wherever it is differentiable.
 */
#ifndef OLAM_ORACLE_DUAL_H
#define OLAM_ORACLE_DUAL_H

#include <cmath>

namespace oracle {

struct Dual {
  double v = 0.0, d = 0.0;
  Dual() = default;
  Dual(double x) : v(x), d(0.0) {}  // NOLINT: implicit, as a real literal converts
  Dual(double x, double dx) : v(x), d(dx) {}
  explicit operator double() const { return v; }
  explicit operator float() const { return (float)v; }
  Dual& operator+=(const Dual& o) { v += o.v; d += o.d; return *this; }
  Dual& operator-=(const Dual& o) { v -= o.v; d -= o.d; return *this; }
  Dual& operator*=(const Dual& o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
  Dual& operator/=(const Dual& o) { *this = Dual(v / o.v, (d * o.v - v * o.d) / (o.v * o.v)); return *this; }
};

inline Dual operator+(Dual a, const Dual& b) { return a += b; }
inline Dual operator-(Dual a, const Dual& b) { return a -= b; }
inline Dual operator*(Dual a, const Dual& b) { return a *= b; }
inline Dual operator/(Dual a, const Dual& b) { return a /= b; }
inline Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
inline bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
inline bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }

// |a| for every real type of the oracle
inline float abs_(float a) { return std::fabs(a); }
inline double abs_(double a) { return std::fabs(a); }
inline Dual abs_(const Dual& a) { return a.v < 0.0 ? -a : a; }

}  // namespace oracle

#endif
