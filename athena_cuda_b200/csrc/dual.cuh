// dual.cuh -- forward-mode (tangent-linear) scalar for the MHD step.
//
// A Dual carries a value and one directional derivative.  Instantiating the
// per-cell physics (mhd_physics.cuh) and the generic step kernels
// (step_generic.cuh) with Dual instead of double gives the discrete
// tangent-linear model of the step: the value part performs exactly the
// double arithmetic of the plain step (same operations, same order), the
// tangent part its derivative along the seeded direction.
//
// Branches (limiters, upwind selections, the HLLE fallback, max/min) test the
// value part only, so the tangent is the derivative of the branch the plain
// step takes ("frozen" branches); the adjoint kernels (mhd_adjoint.cuh) make
// the same choices, which is what makes them exact transposes of each other.
//
// Non-differentiable points: sqrt(0) is given a zero derivative.  Exact zeros
// under a square root come from field-free regions (|B| = 0, where the
// eigenvector formulas switch branch) and from squares of the tiny fields that
// numerical diffusion leaks into them (|B| ~ 1e-160 squares to 0.0); in both
// the derivative of the square root is unbounded while that of the function it
// belongs to (|B|, the Alfven speed) is not.  fabs(0) differentiates as +x,
// and MAX/MIN pick the operand the value comparison picks.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define ATHB_DHD __host__ __device__ __forceinline__
#define ATHB_MEM __host__ __device__ __forceinline__   // member functions
#else
#define ATHB_DHD static inline
#define ATHB_MEM inline
#endif

namespace athb {

struct Dual {
  double v, t;
  ATHB_MEM Dual() : v(0.0), t(0.0) {}
  ATHB_MEM Dual(double x) : v(x), t(0.0) {}
  ATHB_MEM Dual(double x, double dx) : v(x), t(dx) {}
};

ATHB_DHD Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.t + b.t); }
ATHB_DHD Dual operator+(Dual a, double b) { return Dual(a.v + b, a.t); }
ATHB_DHD Dual operator+(double a, Dual b) { return Dual(a + b.v, b.t); }
ATHB_DHD Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.t - b.t); }
ATHB_DHD Dual operator-(Dual a, double b) { return Dual(a.v - b, a.t); }
ATHB_DHD Dual operator-(double a, Dual b) { return Dual(a - b.v, -b.t); }
ATHB_DHD Dual operator-(Dual a) { return Dual(-a.v, -a.t); }
ATHB_DHD Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.t * b.v + a.v * b.t); }
ATHB_DHD Dual operator*(Dual a, double b) { return Dual(a.v * b, a.t * b); }
ATHB_DHD Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.t); }
ATHB_DHD Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual(q, (a.t - q * b.t) / b.v);
}
ATHB_DHD Dual operator/(Dual a, double b) { return Dual(a.v / b, a.t / b); }
ATHB_DHD Dual operator/(double a, Dual b) {
  const double q = a / b.v;
  return Dual(q, -q * b.t / b.v);
}
ATHB_DHD Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
ATHB_DHD Dual& operator-=(Dual& a, Dual b) { a = a - b; return a; }
ATHB_DHD Dual& operator*=(Dual& a, Dual b) { a = a * b; return a; }

ATHB_DHD bool operator<(Dual a, Dual b) { return a.v < b.v; }
ATHB_DHD bool operator>(Dual a, Dual b) { return a.v > b.v; }
ATHB_DHD bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
ATHB_DHD bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
ATHB_DHD bool operator==(Dual a, Dual b) { return a.v == b.v; }
ATHB_DHD bool operator<(Dual a, double b) { return a.v < b; }
ATHB_DHD bool operator>(Dual a, double b) { return a.v > b; }
ATHB_DHD bool operator<=(Dual a, double b) { return a.v <= b; }
ATHB_DHD bool operator>=(Dual a, double b) { return a.v >= b; }
ATHB_DHD bool operator==(Dual a, double b) { return a.v == b; }

// the plain functions stay visible next to the Dual overloads, so that
// unqualified sqrt / fabs in templated code pick them for double arguments
using ::fabs;
using ::sqrt;
ATHB_DHD Dual sqrt(Dual a) {
  const double s = ::sqrt(a.v);
  return Dual(s, s > 0.0 ? a.t / (2.0 * s) : 0.0);
}
ATHB_DHD Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }

// the same value with no derivative
ATHB_DHD Dual no_tangent(Dual a) { return Dual(a.v, 0.0); }

// value of a scalar of either kind
ATHB_DHD double value_of(double a) { return a; }
ATHB_DHD double value_of(Dual a) { return a.v; }

}  // namespace athb
