#pragma once
// Surface reconstruction, materials, background and next-event estimation.
//
// Each routine restates a reference routine in fp32 with the same branch
// structure and RNG draw order:
//   finalize            include/raytracer/geometry/shapes.hpp:49-58, 82-97, 129-142
//   texture / scatter   src/materials/material.cpp:14-74
//   emission / BRDF     src/materials/material.cpp:76-100
//   background          src/core/scene.cpp:10-14
//   light sample        src/rendering/integrator.cpp:14-91
#include "device/trace.cuh"

namespace rtg {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kInvPiF = 0.318309886183790671538f;

struct Surface {
  float3 p;        // hit point
  float3 gn;       // geometric normal, facing the incoming ray
  float3 n;        // shading normal, facing the incoming ray
  bool front;      // hit the side the outward normal points to
  bool is_plane;
  std::uint32_t material;  // absolute index into the material pool
};

// The hit point is rebuilt from the surface (barycentrics, or a projection onto
// the sphere or plane) rather than taken as o + t d: far from the ray origin that
// sum carries an absolute error of ulps of |o|, which can exceed the spawn offset
// and put the point behind the surface (Waechter and Binder's method assumes a
// surface-accurate point).
__device__ __forceinline__ Surface make_surface(const RtgSceneDev& sc, float3 o, float3 d, const RayHit& h) {
  Surface s;
  s.p = o + h.t * d;
  s.is_plane = (h.word & kHitPlaneBit) != 0 && h.word != kHitMiss;
  if (s.is_plane) {
    const DevPlane pl = sc.planes[h.word & ~kHitPlaneBit];
    const float3 nrm = f3(pl.normal);
    s.p = s.p - dot3(s.p - f3(pl.point), nrm) * nrm;
    s.front = dot3(d, nrm) < 0.f;
    s.gn = s.front ? nrm : -nrm;
    s.n = s.gn;
    s.material = __float_as_uint(pl.point.w);
    return s;
  }
  const int slot = static_cast<int>(h.word);
  const float4 p0 = __ldg(&sc.prims[3 * slot]);
  const float4 p1 = __ldg(&sc.prims[3 * slot + 1]);
  const float4 p2 = __ldg(&sc.prims[3 * slot + 2]);  // with the others, not after the kind test
  const std::uint32_t mword = __ldg(&sc.slot_material[slot]);
  s.material = mword & 0x7FFFFFFFu;
  if (__float_as_uint(p0.w) & kSphereBit) {
    const float3 outward = unit_or((s.p - f3(p0)) * (1.f / p1.x), f3(0.f, 1.f, 0.f));
    s.p = f3(p0) + p1.x * outward;
    s.front = dot3(d, outward) < 0.f;
    s.gn = s.front ? outward : -outward;
    s.n = s.gn;
    return s;
  }
  s.p = f3(p0) + h.b1 * f3(p1) + h.b2 * f3(p2);
  const float3 ng = unit_or(cross3(f3(p1), f3(p2)), f3(0.f, 0.f, 0.f));
  s.front = dot3(d, ng) < 0.f;
  s.gn = s.front ? ng : -ng;
  s.n = s.gn;
  if (mword & 0x80000000u) {
    const float4 n0 = __ldg(&sc.slot_normals[3 * slot]);
    const float4 n1 = __ldg(&sc.slot_normals[3 * slot + 1]);
    const float4 n2 = __ldg(&sc.slot_normals[3 * slot + 2]);
    const float w0 = 1.f - h.b1 - h.b2;
    const float3 ns = unit_or(w0 * f3(n0) + h.b1 * f3(n1) + h.b2 * f3(n2), ng);
    s.n = s.front ? ns : -ns;
    // Keep the shading normal in the geometric normal's hemisphere.
    if (dot3(s.n, s.gn) <= 0.f) s.n = s.gn;
  }
  return s;
}

__device__ __forceinline__ float3 background(const RtgSceneDev& sc, float3 d) {
  if (sc.bg_solid) return sc.bg_top * sc.bg_intensity;
  const float t = 0.5f * (unit_or(d, f3(0.f, 0.f, 0.f)).y + 1.f);
  return (sc.bg_bottom * (1.f - t) + sc.bg_top * t) * sc.bg_intensity;
}

__device__ __forceinline__ float3 albedo_at(const DevMaterial& m, float3 p) {
  const float scale = m.head.y;
  if (scale <= 0.f) return f3(m.colour_a);
  // The 1e-4 offset keeps surfaces lying on a cell boundary from flickering.
  const int parity = static_cast<int>(floorf(p.x * scale + 1e-4f)) + static_cast<int>(floorf(p.y * scale + 1e-4f)) +
                     static_cast<int>(floorf(p.z * scale + 1e-4f));
  return (parity & 1) ? f3(m.colour_b) : f3(m.colour_a);
}

__device__ __forceinline__ std::uint32_t kind_of(const DevMaterial& m) { return __float_as_uint(m.head.x); }

__device__ __forceinline__ float3 emitted(const DevMaterial& m, bool front) {
  if (kind_of(m) != kEmissive) return f3(0.f, 0.f, 0.f);
  return (front || m.head.w != 0.f) ? f3(m.emit) : f3(0.f, 0.f, 0.f);
}

struct Scatter {
  float3 dir, weight;
  bool specular;
};

// Samples the outgoing direction; false when the path is absorbed.
__device__ __forceinline__ bool scatter(const DevMaterial& m, float3 d, const Surface& s, Pcg& rng, Scatter& out) {
  const std::uint32_t kind = kind_of(m);
  if (kind == kLambertian) {
    out.dir = Frame(s.n).to_world(cosine_hemisphere(rng));
    if (dot3(out.dir, s.gn) <= 0.f) return false;  // smooth normals can dip below the surface
    out.weight = albedo_at(m, s.p);
    out.specular = false;
    return true;
  }
  if (kind == kMetal) {
    const float3 in = unit_or(d, f3(0.f, 0.f, 0.f));
    float3 r = reflect3(in, s.n);
    const float rough = m.head.z;
    if (rough > 0.f) {
      const float3 fuzz = unit_vector(rng);
      r = unit_or(unit_or(r, f3(0.f, 0.f, 0.f)) + rough * fuzz, f3(0.f, 0.f, 0.f));
    }
    if (dot3(r, s.gn) <= 0.f) return false;
    out.dir = r;
    out.weight = f3(m.colour_a);
    out.specular = true;
    return true;
  }
  if (kind == kDielectric) {
    const float ior = m.head.z;
    const float eta = s.front ? 1.f / ior : ior;
    const float3 in = unit_or(d, f3(0.f, 0.f, 0.f));
    const float cos_i = fminf(-dot3(in, s.n), 1.f);
    float3 refr;
    const bool can = refract3(in, s.n, eta, refr);
    // Reflect with probability F (one draw, only when refraction is possible).
    if (!can || rng.uniform() < schlick(cos_i, eta)) out.dir = reflect3(in, s.n);
    else out.dir = unit_or(refr, f3(0.f, 0.f, 0.f));
    out.weight = f3(m.colour_a);
    out.specular = true;
    return true;
  }
  return false;  // emitters absorb
}

// Lambertian BRDF * cos for light sampling; zero for other materials.
__device__ __forceinline__ float3 brdf_cos(const DevMaterial& m, const Surface& s, float3 wi) {
  if (kind_of(m) != kLambertian) return f3(0.f, 0.f, 0.f);
  const float c = dot3(s.n, wi);
  if (c <= 0.f || dot3(s.gn, wi) <= 0.f) return f3(0.f, 0.f, 0.f);
  return albedo_at(m, s.p) * (c * kInvPiF);
}

// brdf_cos for a Lambertian surface of albedo `albedo` (the only non-specular
// scatter), from the scatter weight instead of the material record.
__device__ __forceinline__ float3 lambert_cos(float3 albedo, const Surface& s, float3 wi) {
  const float c = dot3(s.n, wi);
  if (c <= 0.f || dot3(s.gn, wi) <= 0.f) return f3(0.f, 0.f, 0.f);
  return albedo * (c * kInvPiF);
}

struct LightSample {
  float3 wi;
  float dist;
  float3 li_over_pdf;  // incident radiance / pdf (I / d^2 for point lights)
  float pdf;           // solid-angle pdf of wi (0 for point lights: a delta)
  bool valid;
};

// Visibility ray for a light sample: from the surface point offset to the
// light's side, aimed at the sampled point on the light and stopping short of
// it by the reference's margin. Aiming at the point (rather than reusing wi from
// the un-offset point) keeps the ray from clipping the light itself when the
// offset is larger than the margin, e.g. near the rim of a sphere light.
struct ShadowRay {
  float3 o, d;
  float tmax;
};
__device__ __forceinline__ ShadowRay shadow_ray(const Surface& s, const LightSample& ls) {
  ShadowRay r;
  r.o = spawn_towards(s.p, s.gn, ls.wi);
  const float3 target = s.p + ls.dist * ls.wi;
  const float3 span = target - r.o;
  const float len = sqrtf(dot3(span, span));
  r.d = len > 0.f ? span * (1.f / len) : ls.wi;
  r.tmax = fmaxf(len - shadow_margin(target), 0.f);
  return r;
}

// One sample of one light as seen from s.p (no shadow test). The record's
// fields are read only for the light's kind, which keeps registers free.
__device__ __forceinline__ LightSample sample_light(const DevLight* __restrict__ Lp, const Surface& s, Pcg& rng) {
  LightSample out{};
  out.valid = false;
  const float4 q0 = __ldg(&Lp->q0);
  const std::uint32_t kind = __float_as_uint(q0.w);
  const float3 p = s.p;
  if (kind == kLightPoint) {
    const float3 dv = f3(q0) - p;
    const float d2 = dot3(dv, dv);
    if (d2 < 1e-16f) return out;
    out.dist = sqrtf(d2);
    out.wi = dv * (1.f / out.dist);
    out.li_over_pdf = f3(__ldg(&Lp->q1)) * (1.f / d2);
    out.pdf = 0.f;
    out.valid = true;
    return out;
  }
  if (kind == kLightSphere) {
    const float4 q1 = __ldg(&Lp->q1);
    const float3 c = f3(q0);
    const float r = q1.x, r2 = q1.y, area = q1.z;
    const bool two_sided = q1.w != 0.f;
    const float3 emit = f3(__ldg(&Lp->q2));
    const float3 oc = c - p;
    const float d2 = dot3(oc, oc);
    if (d2 <= r2) {
      // Inside the sphere: area-sample its surface (only two-sided emitters light their inside).
      if (!two_sided) return out;
      const float3 nl = unit_vector(rng);
      const float3 dv = c + r * nl - p;
      const float dd2 = dot3(dv, dv);
      if (dd2 < 1e-16f) return out;
      out.dist = sqrtf(dd2);
      out.wi = dv * (1.f / out.dist);
      const float cos_l = fabsf(dot3(nl, out.wi));
      if (cos_l < 1e-9f) return out;
      out.li_over_pdf = emit * (cos_l * area / dd2);
      out.pdf = dd2 / (cos_l * area);
      out.valid = true;
      return out;
    }
    // Cone of directions subtended by the sphere; 1 - cos written without cancellation.
    const float x = r2 / d2;
    const float one_minus_cos = x / (1.f + sqrtf(1.f - x));
    const float3 axis = oc * rsqrtf(d2);
    out.wi = Frame(axis).to_world(uniform_cone(rng, one_minus_cos));
    float t;
    if (!sphere_test(p, out.wi, c, f3(0.f, 0.f, 0.f), r, 0.f, __int_as_float(0x7f800000), t)) return out;  // grazing miss
    out.dist = t;
    out.li_over_pdf = emit * (2.f * kPiF * one_minus_cos);
    out.pdf = 1.f / (2.f * kPiF * one_minus_cos);
    out.valid = true;
    return out;
  }
  // Triangle: uniform area sample converted to solid angle.
  const float4 q1 = __ldg(&Lp->q1), q2 = __ldg(&Lp->q2);
  const float3 v0 = f3(q0), v1 = f3(q1), v2 = f3(q2);
  const float area = q1.w;
  const bool two_sided = q2.w != 0.f;
  const float2 b = uniform_triangle(rng);
  const float3 q = (1.f - b.x - b.y) * v0 + b.x * v1 + b.y * v2;
  const float3 dv = q - p;
  const float d2 = dot3(dv, dv);
  if (d2 < 1e-16f) return out;
  out.dist = sqrtf(d2);
  out.wi = dv * (1.f / out.dist);
  const float cos_signed = -dot3(f3(__ldg(&Lp->q3)), out.wi);
  if (cos_signed <= 0.f && !two_sided) return out;
  const float cos_l = fabsf(cos_signed);
  if (cos_l < 1e-9f) return out;
  out.li_over_pdf = f3(__ldg(&Lp->q4)) * (cos_l * area / d2);
  out.pdf = d2 / (cos_l * area);
  out.valid = true;
  return out;
}

// Solid-angle pdf with which sample_light would have produced direction d from
// o toward the emitter the ray hit (slot h.word, distance h.t, surface s): the
// same cone / area cases as above, seen from the ray origin. Multiple importance
// sampling weighs a BSDF-sampled hit on a light with it.
__device__ __forceinline__ float light_pdf_of_hit(const RtgSceneDev& sc, float3 o, float3 d, const RayHit& h,
                                                  const Surface& s) {
  const int slot = static_cast<int>(h.word);
  const float4 p0 = __ldg(&sc.prims[3 * slot]);
  const float4 p1 = __ldg(&sc.prims[3 * slot + 1]);
  const float cos_l = fabsf(dot3(s.gn, d));
  if (__float_as_uint(p0.w) & kSphereBit) {
    const float r2 = p1.y;  // radius squared (p1.x holds the radius)
    const float3 oc = f3(p0) - o;
    const float d2 = dot3(oc, oc);
    if (d2 <= r2) return cos_l > 0.f ? h.t * h.t / (cos_l * 4.f * kPiF * r2) : 0.f;
    const float x = r2 / d2;
    return 1.f / (2.f * kPiF * (x / (1.f + sqrtf(1.f - x))));
  }
  const float4 p2 = __ldg(&sc.prims[3 * slot + 2]);
  const float3 c = cross3(f3(p1), f3(p2));
  const float area = 0.5f * sqrtf(dot3(c, c));
  return cos_l > 0.f && area > 0.f ? h.t * h.t / (cos_l * area) : 0.f;
}

// Power heuristic (Veach, beta = 2) of the strategy with pdf a against one with pdf b.
__device__ __forceinline__ float power_heuristic(float a, float b) {
  const float a2 = a * a, b2 = b * b;
  return a2 + b2 > 0.f ? a2 / (a2 + b2) : 0.f;
}

}  // namespace rtg
