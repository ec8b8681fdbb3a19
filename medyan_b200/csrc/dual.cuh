// dual.cuh — forward-mode (dual-number) arithmetic for directional
// derivatives of the force and energy formulas.
//
// A Dual carries a value and its derivative along one direction of the
// coordinates: positions x + eps v enter as Dual{x, v}, and every formula of
// potentials.cuh / excl.cuh evaluated on them returns Dual{f(x), df/deps}.
// Applied to the forces this is the Hessian-vector product (dF/deps = -H v),
// to the parameter gradients the mixed derivative v . d2E/dx dtheta, both
// exact to rounding (no finite-difference step). Branches (clamps, the
// in-plane test, the reference's special cases) follow the value, as the
// derivative of a piecewise formula does inside each piece.
#pragma once

#include <cmath>

#include "device_math.cuh"

namespace mb {

// Dual and its functions live in their own namespace: sqrt, atan, exp, fabs
// on a Dual are found by argument-dependent lookup only, so the double
// versions stay the ones every other call in namespace mb resolves to.
namespace ad {

struct Dual {
    double v, d;
    __host__ __device__ Dual() : v(0.0), d(0.0) {}
    __host__ __device__ Dual(double x) : v(x), d(0.0) {}  // a constant
    __host__ __device__ Dual(double x, double dx) : v(x), d(dx) {}
    __host__ __device__ explicit operator double() const { return v; }
    __device__ Dual& operator+=(const Dual& b) {
        v += b.v;
        d += b.d;
        return *this;
    }
    __device__ Dual& operator-=(const Dual& b) {
        v -= b.v;
        d -= b.d;
        return *this;
    }
};

__device__ __forceinline__ Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual operator+(const Dual& a, double b) { return Dual(a.v + b, a.d); }
__device__ __forceinline__ Dual operator+(double a, const Dual& b) { return Dual(a + b.v, b.d); }
__device__ __forceinline__ Dual operator-(const Dual& a, double b) { return Dual(a.v - b, a.d); }
__device__ __forceinline__ Dual operator-(double a, const Dual& b) { return Dual(a - b.v, -b.d); }
__device__ __forceinline__ Dual operator*(const Dual& a, double b) { return Dual(a.v * b, a.d * b); }
__device__ __forceinline__ Dual operator*(double a, const Dual& b) { return Dual(a * b.v, a * b.d); }
__device__ __forceinline__ Dual operator/(const Dual& a, double b) { return Dual(a.v / b, a.d / b); }
__device__ __forceinline__ Dual operator/(double a, const Dual& b) {
    const double q = a / b.v;
    return Dual(q, -q * b.d / b.v);
}

__device__ __forceinline__ bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator<(const Dual& a, double b) { return a.v < b; }
__device__ __forceinline__ bool operator>(const Dual& a, double b) { return a.v > b; }
__device__ __forceinline__ bool operator<(double a, const Dual& b) { return a < b.v; }
__device__ __forceinline__ bool operator>(double a, const Dual& b) { return a > b.v; }

// d sqrt(u) = du / (2 sqrt(u)), d atan(u) = du / (1 + u^2), d exp(u) = exp(u) du
__device__ __forceinline__ Dual sqrt(const Dual& a) {
    const double s = ::sqrt(a.v);
    return Dual(s, a.d / (2.0 * s));
}
__device__ __forceinline__ Dual atan(const Dual& a) { return Dual(::atan(a.v), a.d / (1.0 + a.v * a.v)); }
__device__ __forceinline__ Dual exp(const Dual& a) {
    const double e = ::exp(a.v);
    return Dual(e, e * a.d);
}
__device__ __forceinline__ Dual fabs(const Dual& a) { return a.v < 0.0 ? -a : a; }
__device__ __forceinline__ bool isinf(const Dual& a) { return ::isinf(a.v) || ::isinf(a.d); }
__device__ __forceinline__ bool isnan(const Dual& a) { return ::isnan(a.v) || ::isnan(a.d); }

}  // namespace ad

using ad::Dual;

// Positions carrying a direction: DV3 = T3<Dual>.
using DV3 = T3<Dual>;

__device__ __forceinline__ DV3 dual3(const V3& x, const V3& v) {
    return DV3{Dual(x.x, v.x), Dual(x.y, v.y), Dual(x.z, v.z)};
}

// b - a for dual positions (the arithmetic type is Dual as well).
template <class R>
__device__ __forceinline__ T3<R> diff(const DV3& a, const DV3& b) {
    return T3<R>{b.x - a.x, b.y - a.y, b.z - a.z};
}

__device__ __forceinline__ DV3 midpoint(const DV3& v1, const DV3& v2, double alpha) {
    const double beta = 1 - alpha;
    return DV3{v1.x * beta + alpha * v2.x, v1.y * beta + alpha * v2.y, v1.z * beta + alpha * v2.z};
}

}  // namespace mb
