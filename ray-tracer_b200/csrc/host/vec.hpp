#pragma once
// Double-precision 3-vectors for the host side (scene compile, BVH build, camera
// set-up). The host keeps the reference's double arithmetic so that the compiled
// scene and the BVH are bit-identical to the reference's
// (include/raytracer/math/vec3.hpp:17); only the flattened device copy is fp32.
#include <cmath>
#include <limits>

namespace rtg {

constexpr double kPi = 3.14159265358979323846;
constexpr double kInf = std::numeric_limits<double>::infinity();

struct D3 {
  double x = 0, y = 0, z = 0;
  constexpr D3() = default;
  constexpr D3(double a, double b, double c) : x(a), y(b), z(c) {}
  explicit constexpr D3(double s) : x(s), y(s), z(s) {}
  constexpr double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  constexpr double& at(int i) { return i == 0 ? x : (i == 1 ? y : z); }
  constexpr bool operator==(const D3&) const = default;
  bool finite() const { return std::isfinite(x) && std::isfinite(y) && std::isfinite(z); }
  constexpr bool zero() const { return x == 0 && y == 0 && z == 0; }
};

constexpr D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
constexpr D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
constexpr D3 operator-(D3 a) { return {-a.x, -a.y, -a.z}; }
constexpr D3 operator*(D3 a, D3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
constexpr D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
constexpr D3 operator*(double s, D3 a) { return {a.x * s, a.y * s, a.z * s}; }
// Division multiplies by the reciprocal, as the reference's Vec3::operator/= does.
constexpr D3 operator/(D3 a, double s) { return a * (1.0 / s); }
constexpr double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
constexpr D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
constexpr double len2(D3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline double len(D3 a) { return std::sqrt(len2(a)); }
inline D3 dmin(D3 a, D3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
inline D3 dmax(D3 a, D3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }

// Guarded normalisation (same threshold as the reference's normalize_or,
// include/raytracer/math/vec3.hpp:85-89): tiny or non-finite input -> fallback.
inline D3 unit_or(D3 v, D3 fallback) {
  constexpr double kTinyLength = 1e-9;
  const double l2 = len2(v);
  if (!(l2 > kTinyLength * kTinyLength) || !std::isfinite(l2)) return fallback;
  return v / std::sqrt(l2);
}
inline D3 unit(D3 v) { return unit_or(v, D3{}); }

// Axis-aligned box; default is empty (+inf/-inf).
struct Box {
  D3 lo{kInf}, hi{-kInf};
  bool empty() const { return lo.x > hi.x || lo.y > hi.y || lo.z > hi.z; }
  void grow(D3 p) { lo = dmin(lo, p); hi = dmax(hi, p); }
  void grow(const Box& b) { lo = dmin(lo, b.lo); hi = dmax(hi, b.hi); }
  D3 center() const { return 0.5 * (lo + hi); }
  double area() const {
    if (empty()) return 0;
    const D3 e = hi - lo;
    return 2 * (e.x * e.y + e.y * e.z + e.z * e.x);
  }
  int widest_axis() const {
    const D3 e = empty() ? D3{} : hi - lo;
    return (e.x >= e.y && e.x >= e.z) ? 0 : (e.y >= e.z ? 1 : 2);
  }
};

}  // namespace rtg
