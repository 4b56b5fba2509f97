// Forward-mode dual numbers for the pointwise physics (host and device).
//
// Dual<K> carries a float64 value and K directional derivatives.  The
// equation and boundary-condition code (dg_physics.cuh) is written over a
// scalar type T, so instantiating it with Dual<K> differentiates exactly the
// arithmetic the float64 right-hand side performs: comparisons and clamps act
// on the value (a clamped quantity gets derivative 0), sqrt and division use
// their derivatives at the value.  Dual<1> gives Jacobian-vector products;
// Dual<M> seeded with the unit vectors gives full M x M Jacobians.
#pragma once

#include <math.h>

#include "dg_physics.cuh"

namespace apollo {

template <int K>
struct Dual {
  double v;
  double d[K];

  APOLLO_HD Dual() : v(0.0) {
#pragma unroll
    for (int k = 0; k < K; ++k) d[k] = 0.0;
  }
  // a constant (implicit, so that mixed double/Dual expressions work)
  APOLLO_HD Dual(double x) : v(x) {
#pragma unroll
    for (int k = 0; k < K; ++k) d[k] = 0.0;
  }

  APOLLO_HD friend Dual operator+(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
  }
  APOLLO_HD friend Dual operator-(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
  }
  APOLLO_HD friend Dual operator-(const Dual& a) {
    Dual r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
  }
  APOLLO_HD friend Dual operator*(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
  }
  APOLLO_HD friend Dual operator/(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
  }
  APOLLO_HD friend bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
  APOLLO_HD friend bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
  APOLLO_HD friend bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
  APOLLO_HD friend bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
  APOLLO_HD friend bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
  APOLLO_HD friend bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }
  // sqrt(a)' = a' / (2 sqrt(a)); the derivative of sqrt(0) is taken as 0
  APOLLO_HD friend Dual sqrt(const Dual& a) {
    Dual r;
    r.v = ::sqrt(a.v);
    const double s = r.v > 0.0 ? 0.5 / r.v : 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * s;
    return r;
  }
  APOLLO_HD friend Dual fabs(const Dual& a) { return a.v < 0.0 ? -a : a; }
  // piecewise constant: derivative 0
  APOLLO_HD friend Dual abs_int(const Dual& a) { return Dual(::apollo::abs_int(a.v)); }
};

}  // namespace apollo
