// dual.hpp -- TEST INFRASTRUCTURE ONLY.
//
// Forward-mode derivative numbers for the CPU restatement: a double value and its derivative
// along one direction of the inputs.  `World<Dual>` runs the restatement in FP64 and carries
// with every quantity its derivative along that direction (the tangent), exactly, with no step
// size.  Tests check the CUDA library's adjoint (step_backward, the transposed derivative) with
// the identity <g, J d> = <J^T g, d>.  Branches (the pressure clamp, approach-only viscosity, wall
// clamps, solver stops) follow the value, as the adjoint follows the forward's branches; floor,
// round and ceil have derivative zero; the square root of zero takes derivative zero (the only
// zero lengths are a particle's offset to itself, whose derivative is zero too).
#pragma once

#include <cmath>
#include <cstdint>

struct Dual {
    double v = 0.0, d = 0.0;
    Dual() = default;
    Dual(double x) : v(x) {}  // constants carry no derivative
    Dual(double x, double dx) : v(x), d(dx) {}
    explicit operator double() const { return v; }
    explicit operator float() const { return float(v); }
    explicit operator int() const { return int(v); }
    explicit operator unsigned() const { return unsigned(v); }
    explicit operator long() const { return long(v); }
    explicit operator unsigned long() const { return (unsigned long)(v); }
    explicit operator long long() const { return (long long)(v); }
    Dual& operator+=(Dual b) { d += b.d; v += b.v; return *this; }
    Dual& operator-=(Dual b) { d -= b.d; v -= b.v; return *this; }
    Dual& operator*=(Dual b) { d = d * b.v + v * b.d; v *= b.v; return *this; }
    Dual& operator/=(Dual b) { *this = Dual(v / b.v, (d * b.v - v * b.d) / (b.v * b.v)); return *this; }
};

inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b) { return Dual(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
inline bool operator!=(Dual a, Dual b) { return a.v != b.v; }

inline Dual osqrt(Dual x) {
    double r = std::sqrt(x.v);
    return Dual(r, r > 0.0 ? x.d / (2.0 * r) : 0.0);
}
inline Dual ofloor(Dual x) { return Dual(std::floor(x.v)); }
inline Dual oceil(Dual x) { return Dual(std::ceil(x.v)); }
inline Dual oround(Dual x) { return Dual(std::round(x.v)); }
inline Dual ofabs(Dual x) { return x.v < 0.0 ? -x : x; }
inline bool oisnan(Dual x) { return std::isnan(x.v); }
inline bool oisfinite(Dual x) { return std::isfinite(x.v); }
