#pragma once
// fp32 vector maths, the per-sample PCG32 stream, sampling routines and robust
// ray spawning for the sm_100a kernels.
//
// RNG: the stream for sample s of pixel p is keyed exactly as the reference's
// Rng::for_sample (include/raytracer/math/rng.hpp:10-46): SplitMix64 finaliser
// over (seed, pixel, sample), PCG32 (O'Neill 2014) with a 64-bit state and a
// per-stream increment. The integer outputs are bit-identical to the CPU's and
// are drawn in the same order; only the mapping to [0, 1) differs (24 bits here,
// so a float can never round up to 1).
#include <cstdint>

#include "device/layout.h"

namespace rtg {

__device__ __forceinline__ float3 f3(float a, float b, float c) { return make_float3(a, b, c); }
__device__ __forceinline__ float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float max3(float3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
__device__ __forceinline__ bool is_zero3(float3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }

// Pinned rounding, for the code that decides hits: the hit tests, the slab
// set-up and the camera ray. Every product and sum is an explicit fmaf or an
// __fmul_rn / __fadd_rn / __fsub_rn, which the compiler never fuses, so the bits
// do not depend on the kernel the code is inlined into. (Left to contract freely,
// the counting and non-counting instances of the closest-hit kernel rounded a few
// hits differently.)
__device__ __forceinline__ float3 sub3p(float3 a, float3 b) {
  return f3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}
__device__ __forceinline__ float3 add3p(float3 a, float3 b) {
  return f3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z));
}
__device__ __forceinline__ float dot3p(float3 a, float3 b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, __fmul_rn(a.x, b.x))); }
__device__ __forceinline__ float3 cross3p(float3 a, float3 b) {
  return f3(fmaf(a.y, b.z, -__fmul_rn(a.z, b.y)), fmaf(a.z, b.x, -__fmul_rn(a.x, b.z)),
            fmaf(a.x, b.y, -__fmul_rn(a.y, b.x)));
}

// Normalise (pinned rounding), or return `fallback` for (near-)zero or non-finite input.
__device__ __forceinline__ float3 unit_or(float3 v, float3 fallback) {
  const float l2 = dot3p(v, v);
  if (!(l2 > 1e-30f) || !isfinite(l2)) return fallback;
  const float s = rsqrtf(l2);
  return f3(__fmul_rn(v.x, s), __fmul_rn(v.y, s), __fmul_rn(v.z, s));
}

__device__ __forceinline__ float3 reflect3(float3 v, float3 n) { return v - (2.f * dot3(v, n)) * n; }

// Snell refraction of unit `v` through unit `n` (facing against v), eta = n_i / n_t.
__device__ __forceinline__ bool refract3(float3 v, float3 n, float eta, float3& out) {
  const float cos_i = fminf(-dot3(v, n), 1.f);
  const float sin2_t = eta * eta * (1.f - cos_i * cos_i);
  if (sin2_t > 1.f) return false;
  const float cos_t = sqrtf(1.f - sin2_t);
  out = eta * v + (eta * cos_i - cos_t) * n;
  return true;
}

__device__ __forceinline__ float schlick(float cos_theta, float eta) {
  float r0 = (1.f - eta) / (1.f + eta);
  r0 *= r0;
  const float m = 1.f - cos_theta;
  const float m2 = m * m;
  return r0 + (1.f - r0) * (m2 * m2 * m);
}

// ---------------------------------------------------------------------------
// PCG32 stream keyed on (seed, pixel, sample)
__host__ __device__ __forceinline__ std::uint64_t mix64(std::uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct Pcg {
  std::uint64_t state, inc;

  __device__ __forceinline__ std::uint32_t next() {
    const std::uint64_t old = state;
    state = old * 6364136223846793005ull + inc;
    const std::uint32_t x = static_cast<std::uint32_t>(((old >> 18u) ^ old) >> 27u);
    const std::uint32_t r = static_cast<std::uint32_t>(old >> 59u);
    return __funnelshift_r(x, x, r);  // rotate right by r
  }
  // Uniform in [0, 1) from the top 24 bits of one draw.
  __device__ __forceinline__ float uniform() { return static_cast<float>(next() >> 8) * 0x1p-24f; }
  // Uniform integer in [0, n): floor(u32 * n / 2^32), which equals the CPU's
  // floor(double(u32) / 2^32 * n) exactly for n < 2^21.
  __device__ __forceinline__ std::uint32_t below(std::uint32_t n) {
    return static_cast<std::uint32_t>((static_cast<std::uint64_t>(next()) * n) >> 32);
  }

  __device__ static __forceinline__ Pcg seeded(std::uint64_t seed, std::uint64_t stream) {
    Pcg p{0, (stream << 1u) | 1u};
    p.next();
    p.state += seed;
    p.next();
    return p;
  }
  __device__ static __forceinline__ Pcg for_sample(std::uint64_t seed, std::uint64_t pixel, std::uint64_t sample) {
    const std::uint64_t h = mix64(seed ^ mix64(pixel ^ mix64(sample)));
    return seeded(h, mix64(h));
  }
};

// ---------------------------------------------------------------------------
// Sampling (each follows the matching reference routine and draw order,
// include/raytracer/math/sampling.hpp:13-78).
__device__ __forceinline__ float2 unit_disk(Pcg& rng) {
  const float r = sqrtf(rng.uniform());
  float s, c;
  sincospif(2.f * rng.uniform(), &s, &c);
  return make_float2(__fmul_rn(r, c), __fmul_rn(r, s));
}

__device__ __forceinline__ float3 unit_vector(Pcg& rng) {
  const float z = 1.f - 2.f * rng.uniform();
  const float r = sqrtf(fmaxf(0.f, 1.f - z * z));
  float s, c;
  sincospif(2.f * rng.uniform(), &s, &c);
  return f3(r * c, r * s, z);
}

__device__ __forceinline__ float3 cosine_hemisphere(Pcg& rng) {
  const float2 d = unit_disk(rng);
  return f3(d.x, d.y, sqrtf(fmaxf(0.f, 1.f - d.x * d.x - d.y * d.y)));
}

// Uniform direction in the cone 1 - cos(theta) <= one_minus_cos_max around +Z.
// Written in terms of 1 - cos so narrow cones keep their precision in fp32.
__device__ __forceinline__ float3 uniform_cone(Pcg& rng, float one_minus_cos_max) {
  const float s = rng.uniform() * one_minus_cos_max;  // 1 - cos(theta)
  const float cos_t = 1.f - s;
  const float sin_t = sqrtf(fmaxf(0.f, s * (2.f - s)));
  float sp, cp;
  sincospif(2.f * rng.uniform(), &sp, &cp);
  return f3(sin_t * cp, sin_t * sp, cos_t);
}

// Uniform barycentrics (b1, b2) on a triangle (square-root parameterisation).
__device__ __forceinline__ float2 uniform_triangle(Pcg& rng) {
  const float su = sqrtf(rng.uniform());
  return make_float2(1.f - su, rng.uniform() * su);
}

// Orthonormal basis around unit w (Duff et al. 2017, "Building an Orthonormal
// Basis, Revisited", JCGT 6(1)).
struct Frame {
  float3 u, v, w;
  __device__ __forceinline__ explicit Frame(float3 n) : w(n) {
    const float sign = copysignf(1.f, n.z);
    const float a = -1.f / (sign + n.z);
    const float b = n.x * n.y * a;
    u = f3(1.f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    v = f3(b, sign + n.y * n.y * a, -n.y);
  }
  __device__ __forceinline__ float3 to_world(float3 a) const { return a.x * u + a.y * v + a.z * w; }
};

// ---------------------------------------------------------------------------
// Robust spawn point: move p off the surface along n (which must point to the
// side the new ray leaves towards) by a fixed number of float ulps, or by a
// small absolute amount near the origin. Wächter and Binder, "A Fast and Robust
// Method for Avoiding Self-Intersection", Ray Tracing Gems (2019), ch. 6. The
// fp32 replacement for the reference's 1.6e-6 * max(1, |p|) offset
// (include/raytracer/math/ray.hpp:41-58), which is below an fp32 ulp at the
// 555-unit scale of a Cornell room.
__device__ __forceinline__ float ulp_step(float p, float n, float scaled_n) {
  const int step = static_cast<int>(256.f * n);
  const float moved = __int_as_float(__float_as_int(p) + (p < 0.f ? -step : step));
  return fabsf(p) < (1.f / 32.f) ? p + scaled_n : moved;
}
__device__ __forceinline__ float3 spawn_point(float3 p, float3 n) {
  constexpr float kNearScale = 1.f / 65536.f;
  return f3(ulp_step(p.x, n.x, kNearScale * n.x), ulp_step(p.y, n.y, kNearScale * n.y),
            ulp_step(p.z, n.z, kNearScale * n.z));
}
// Spawn for direction `dir` from a surface with geometric normal `gn`.
__device__ __forceinline__ float3 spawn_towards(float3 p, float3 gn, float3 dir) {
  return spawn_point(p, dot3(dir, gn) > 0.f ? gn : -gn);
}

// The reference's shadow-ray shortening distance, 4 * 1.6e-6 * max(1, |p|inf)
// (src/rendering/integrator.cpp:69-70), which is ~100 fp32 ulps of |p|.
__device__ __forceinline__ float shadow_margin(float3 p) {
  const float m = fmaxf(fmaxf(fabsf(p.x), fabsf(p.y)), fmaxf(fabsf(p.z), 1.f));
  return 4.f * 1.6e-6f * m;
}

}  // namespace rtg
