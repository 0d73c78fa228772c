// dual.hpp -- TEST INFRASTRUCTURE ONLY.
//
// Forward-mode derivative numbers for the CPU restatement: a value and its derivative along one
// direction of the inputs.  `World<DualOf<V>>` runs the restatement with values of type V and
// carries with every quantity its derivative along that direction (the tangent), in double,
// exactly, with no step size:
//
//   Dual   = DualOf<double>: the derivative of the FP64 method;
//   Dual32 = DualOf<float>:  the derivative of the FP32 program itself.  Its values are the float
//          restatement's bit for bit (every value operation is the float one), hence the CUDA
//          library's in EXACT arithmetic, so it takes every branch the library's run takes;
//   DualOf<float, float>:    the same values with each derivative operation rounded to float, as a
//          single-precision derivative code carries it (how far that drifts from Dual32 measures
//          the conditioning an FP32 adjoint meets).
//
// Tests check the CUDA library's adjoint (step_backward, the transposed derivative) with the
// identity <g, J d> = <J^T g, d>.  Branches (the pressure clamp, approach-only viscosity, wall
// clamps, solver stops) follow the value, as the adjoint follows the forward's branches; floor,
// round and ceil have derivative zero; the square root of zero takes derivative zero (the only
// zero lengths are a particle's offset to itself, whose derivative is zero too).
#pragma once

#include <cmath>
#include <cstdint>
#include <type_traits>

template <class V, class D = double> struct DualOf {
    V v = V(0);
    D d = D(0);
    DualOf() = default;
    DualOf(double x) : v(V(x)) {}  // constants carry no derivative
    DualOf(double x, double dx) : v(V(x)), d(D(dx)) {}
    explicit operator double() const { return double(v); }
    explicit operator float() const { return float(v); }
    explicit operator int() const { return int(v); }
    explicit operator unsigned() const { return unsigned(v); }
    explicit operator long() const { return long(v); }
    explicit operator unsigned long() const { return (unsigned long)(v); }
    explicit operator long long() const { return (long long)(v); }

    static DualOf of(V x, D dx) {
        DualOf r;
        r.v = x;
        r.d = dx;
        return r;
    }
    DualOf& operator+=(DualOf b) { return *this = *this + b; }
    DualOf& operator-=(DualOf b) { return *this = *this - b; }
    DualOf& operator*=(DualOf b) { return *this = *this * b; }
    DualOf& operator/=(DualOf b) { return *this = *this / b; }

    // hidden friends: found through the dual operand, the other one converts
    friend DualOf operator+(DualOf a, DualOf b) { return of(a.v + b.v, a.d + b.d); }
    friend DualOf operator-(DualOf a, DualOf b) { return of(a.v - b.v, a.d - b.d); }
    friend DualOf operator-(DualOf a) { return of(-a.v, -a.d); }
    friend DualOf operator*(DualOf a, DualOf b) { return of(a.v * b.v, a.d * D(b.v) + D(a.v) * b.d); }
    friend DualOf operator/(DualOf a, DualOf b) {
        D bv = D(b.v);
        return of(a.v / b.v, (a.d * bv - D(a.v) * b.d) / (bv * bv));
    }
    friend bool operator<(DualOf a, DualOf b) { return a.v < b.v; }
    friend bool operator>(DualOf a, DualOf b) { return a.v > b.v; }
    friend bool operator<=(DualOf a, DualOf b) { return a.v <= b.v; }
    friend bool operator>=(DualOf a, DualOf b) { return a.v >= b.v; }
    friend bool operator==(DualOf a, DualOf b) { return a.v == b.v; }
    friend bool operator!=(DualOf a, DualOf b) { return a.v != b.v; }

    friend DualOf osqrt(DualOf x) {
        V r = std::sqrt(x.v);
        return of(r, r > V(0) ? x.d / (D(2) * D(r)) : D(0));
    }
    friend DualOf ofloor(DualOf x) { return of(std::floor(x.v), D(0)); }
    friend DualOf oceil(DualOf x) { return of(std::ceil(x.v), D(0)); }
    friend DualOf oround(DualOf x) { return of(std::round(x.v), D(0)); }
    friend DualOf ofabs(DualOf x) { return x.v < V(0) ? -x : x; }
    friend bool oisnan(DualOf x) { return std::isnan(x.v); }
    friend bool oisfinite(DualOf x) { return std::isfinite(x.v); }
};

using Dual = DualOf<double>;
using Dual32 = DualOf<float>;

template <class R> struct is_dual : std::false_type {};
template <class V, class D> struct is_dual<DualOf<V, D>> : std::true_type {};
