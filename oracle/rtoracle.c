/*
 * Oracle (test infrastructure only; see rtoracle.h). Restates, in C and double
 * precision, the reference renderer's hot path with the same operation order so
 * that its results match the reference bit for bit on the same compiled scene:
 *
 *   RNG            include/raytracer/math/rng.hpp:10-46
 *   sampling, ONB  include/raytracer/math/sampling.hpp:13-78
 *   vectors        include/raytracer/math/vec3.hpp:65-106
 *   spawn offset   include/raytracer/math/ray.hpp:41-58
 *   slab test      include/raytracer/math/aabb.hpp:41-67
 *   shapes         include/raytracer/geometry/shapes.hpp:25-160
 *   BVH traversal  include/raytracer/geometry/bvh.hpp:75-132
 *   scene queries  src/core/scene.cpp:10-14, 152-234
 *   camera         include/raytracer/core/camera.hpp:54-62
 *   materials      src/materials/material.cpp:14-100
 *   integrators    src/rendering/integrator.cpp:14-198
 *   sample loop    src/rendering/renderer.cpp:28-50
 *   tone map       src/rendering/tonemap.cpp:15-37
 *
 * One addition is not the reference's: multiple importance sampling
 * (light_sampling == 2), the GPU renderer's opt-in estimator, restated here so
 * that its weights can be checked sample by sample. With light_sampling 0 or 1
 * the code paths are the reference's.
 */
#include "rtoracle.h"

#include <math.h>
#include <stdint.h>
#include <string.h>

#define PI 3.14159265358979323846
#define INV_PI (1.0 / PI)
#define RAY_TMIN 1e-6
#define NO_PRIM 0xFFFFFFFFu

typedef struct { double x, y, z; } v3;

static inline v3 V(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 scl(v3 a, double s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 dvs(v3 a, double s) { return scl(a, 1.0 / s); } /* Vec3 / s multiplies by 1/s */
static inline v3 neg(v3 a) { return V(-a.x, -a.y, -a.z); }
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double len2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static inline double len(v3 a) { return sqrt(len2(a)); }
static inline int is_zero(v3 a) { return a.x == 0 && a.y == 0 && a.z == 0; }
static inline int finite3(v3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
static inline double maxc(v3 a) { return a.x > a.y ? (a.x > a.z ? a.x : a.z) : (a.y > a.z ? a.y : a.z); }
static inline v3 unit_or(v3 v, v3 fb) {
  const double eps = 1e-9;
  const double l2 = len2(v);
  if (!(l2 > eps * eps) || !isfinite(l2)) return fb;
  return dvs(v, sqrt(l2));
}
static inline v3 unit(v3 v) { return unit_or(v, V(0, 0, 0)); }
static inline v3 reflect(v3 v, v3 n) { return sub(v, scl(n, 2 * dot(v, n))); }
static int refract(v3 uv, v3 n, double eta, v3* out) {
  const double cos_i = fmin(dot(neg(uv), n), 1.0);
  const double sin2_t = eta * eta * (1.0 - cos_i * cos_i);
  if (sin2_t > 1.0) return 0;
  const double cos_t = sqrt(1.0 - sin2_t);
  *out = add(scl(uv, eta), scl(n, eta * cos_i - cos_t));
  return 1;
}
static inline v3 at(const double* p) { return V(p[0], p[1], p[2]); }

/* ---------------------------------------------------------------- RNG */
static inline uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
typedef struct { uint64_t state, inc; } rng_t;
static inline uint32_t rng_u32(rng_t* r) {
  const uint64_t old = r->state;
  r->state = old * 6364136223846793005ull + r->inc;
  const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
  const uint32_t rot = (uint32_t)(old >> 59u);
  return (xs >> rot) | (xs << ((-rot) & 31u));
}
static inline rng_t rng_new(uint64_t seed, uint64_t stream) {
  rng_t r = {0, (stream << 1u) | 1u};
  rng_u32(&r);
  r.state += seed;
  rng_u32(&r);
  return r;
}
static inline rng_t rng_for_sample(uint64_t seed, uint64_t pixel, uint64_t sample) {
  const uint64_t h = splitmix(seed ^ splitmix(pixel ^ splitmix(sample)));
  return rng_new(h, splitmix(h));
}
static inline double uni(rng_t* r) { return rng_u32(r) * (1.0 / 4294967296.0); }
static inline uint32_t below(rng_t* r, uint32_t n) { return (uint32_t)(uni(r) * n); }

void ro_rng(uint64_t seed, uint64_t pixel, uint64_t sample, uint32_t* out, int32_t n) {
  rng_t r = rng_for_sample(seed, pixel, sample);
  for (int32_t i = 0; i < n; ++i) out[i] = rng_u32(&r);
}

/* ---------------------------------------------------------------- sampling */
typedef struct { v3 u, v, w; } onb_t;
static onb_t onb(v3 n) {
  onb_t b;
  b.w = n;
  const double sign = copysign(1.0, n.z);
  const double a = -1.0 / (sign + n.z);
  const double bb = n.x * n.y * a;
  b.u = V(1.0 + sign * n.x * n.x * a, sign * bb, -sign * n.x);
  b.v = V(bb, sign + n.y * n.y * a, -n.y);
  return b;
}
static inline v3 to_world(const onb_t* b, v3 a) { return add(add(scl(b->u, a.x), scl(b->v, a.y)), scl(b->w, a.z)); }

static v3 random_unit_vector(rng_t* r) {
  const double z = 1 - 2 * uni(r);
  const double rr = sqrt(fmax(0.0, 1 - z * z));
  const double phi = 2 * PI * uni(r);
  return V(rr * cos(phi), rr * sin(phi), z);
}
static void random_in_unit_disk(rng_t* r, double* x, double* y) {
  const double rr = sqrt(uni(r));
  const double phi = 2 * PI * uni(r);
  *x = rr * cos(phi);
  *y = rr * sin(phi);
}
static v3 cosine_hemisphere(rng_t* r) {
  double dx, dy;
  random_in_unit_disk(r, &dx, &dy);
  return V(dx, dy, sqrt(fmax(0.0, 1 - dx * dx - dy * dy)));
}
static v3 uniform_cone(rng_t* r, double cos_max) {
  const double cos_t = 1 - uni(r) * (1 - cos_max);
  const double sin_t = sqrt(fmax(0.0, 1 - cos_t * cos_t));
  const double phi = 2 * PI * uni(r);
  return V(sin_t * cos(phi), sin_t * sin(phi), cos_t);
}
static void uniform_triangle(rng_t* r, double* b1, double* b2) {
  const double su = sqrt(uni(r));
  *b1 = 1 - su;
  *b2 = uni(r) * su;
}

/* ---------------------------------------------------------------- scene access */
#define PRIM(s, i) ((s)->prims + 24 * (size_t)(i))
#define PLANE(s, i) ((s)->planes + 8 * (size_t)(i))
#define NODE(s, i) ((s)->nodes + 10 * (size_t)(i))
#define MAT(s, i) ((s)->materials + 16 * (size_t)(i))

typedef struct { v3 o, d; } ray_t;

typedef struct {
  double t;
  v3 p, normal, gn;
  int front;
  uint32_t material, prim;
  int is_plane;
} hit_t;

static inline double spawn_offset(v3 p) {
  double m = fabs(p.x);
  if (fabs(p.y) > m) m = fabs(p.y);
  if (fabs(p.z) > m) m = fabs(p.z);
  if (1.0 > m) m = 1.0;
  return 1e-7 * m * 16;
}
static inline v3 offset_origin(v3 p, v3 gn, v3 dir) {
  const double d = spawn_offset(p);
  return dot(dir, gn) > 0 ? add(p, scl(gn, d)) : sub(p, scl(gn, d));
}

static void set_face(hit_t* h, v3 dir, v3 outward) {
  h->front = dot(dir, outward) < 0;
  h->gn = h->front ? outward : neg(outward);
  h->normal = h->gn;
}

/* Sphere::hit_t */
static int sphere_hit_t(const double* p, const ray_t* r, double tmin, double tmax, double* tout) {
  const v3 c = V(p[3], p[4], p[5]);
  const double radius = p[6];
  const v3 oc = sub(c, r->o);
  const double a = len2(r->d);
  if (a == 0) return 0;
  const double h = dot(r->d, oc);
  const double cc = len2(oc) - radius * radius;
  const v3 vv = sub(oc, scl(r->d, h / a));
  const double disc = a * (radius * radius - len2(vv));
  if (disc < 0) return 0;
  const double sq = sqrt(disc);
  const double q = h + copysign(sq, h);
  double t0 = cc / q, t1 = q / a;
  if (q == 0) { t0 = t1 = h / a; }
  if (t0 > t1) { const double x = t0; t0 = t1; t1 = x; }
  double t = t0;
  if (!(tmin < t && t < tmax)) {
    t = t1;
    if (!(tmin < t && t < tmax)) return 0;
  }
  *tout = t;
  return 1;
}

/* Triangle::hit_t (Moller-Trumbore) */
static int tri_hit_t(const double* p, const ray_t* r, double tmin, double tmax, double* tout, double* b1o, double* b2o) {
  const v3 v0 = at(p + 3), v1 = at(p + 6), v2 = at(p + 9);
  const v3 e1 = sub(v1, v0), e2 = sub(v2, v0);
  const v3 pvec = cross(r->d, e2);
  const double det = dot(e1, pvec);
  if (fabs(det) < 1e-14) return 0;
  const double inv_det = 1.0 / det;
  const v3 tvec = sub(r->o, v0);
  const double b1 = dot(tvec, pvec) * inv_det;
  if (b1 < 0 || b1 > 1) return 0;
  const v3 qvec = cross(tvec, e1);
  const double b2 = dot(r->d, qvec) * inv_det;
  if (b2 < 0 || b1 + b2 > 1) return 0;
  const double t = dot(e2, qvec) * inv_det;
  if (!(tmin < t && t < tmax)) return 0;
  *tout = t;
  *b1o = b1;
  *b2o = b2;
  return 1;
}

static int prim_hit_t(const ro_scene* s, uint32_t i, const ray_t* r, double tmin, double tmax, double* t, double* b1,
                      double* b2) {
  const double* p = PRIM(s, i);
  if (p[0] == 0) return sphere_hit_t(p, r, tmin, tmax, t);
  return tri_hit_t(p, r, tmin, tmax, t, b1, b2);
}

static void prim_finalize(const ro_scene* s, uint32_t i, const ray_t* r, double t, double b1, double b2, hit_t* h) {
  const double* p = PRIM(s, i);
  h->t = t;
  h->p = add(r->o, scl(r->d, t));
  if (p[0] == 0) {
    const v3 outward = dvs(sub(h->p, at(p + 3)), p[6]);
    set_face(h, r->d, outward);
  } else {
    const v3 v0 = at(p + 3), v1 = at(p + 6), v2 = at(p + 9);
    const v3 ng = unit(cross(sub(v1, v0), sub(v2, v0)));
    set_face(h, r->d, ng);
    if (p[2] != 0) {
      const v3 ns = unit_or(add(add(scl(at(p + 12), 1 - b1 - b2), scl(at(p + 15), b1)), scl(at(p + 18), b2)), ng);
      h->normal = h->front ? ns : neg(ns);
      if (dot(h->normal, h->gn) <= 0) h->normal = h->gn;
    }
  }
  h->material = (uint32_t)p[1];
  h->prim = i;
  h->is_plane = 0;
}

/* Plane::intersect */
static int plane_intersect(const ro_scene* s, uint64_t i, const ray_t* r, double tmin, double tmax, hit_t* h) {
  const double* pl = PLANE(s, i);
  const v3 n = at(pl + 3);
  const double denom = dot(n, r->d);
  if (fabs(denom) < 1e-12) return 0;
  const double t = dot(sub(at(pl), r->o), n) / denom;
  if (!(tmin < t && t < tmax)) return 0;
  h->t = t;
  h->p = add(r->o, scl(r->d, t));
  set_face(h, r->d, n);
  h->material = (uint32_t)pl[6];
  return 1;
}

/* AABB::hit slab test, NaN => inside */
static int slab(double lo, double hi, double o, double inv, double* tmin, double* tmax) {
  double t0 = (lo - o) * inv;
  double t1 = (hi - o) * inv;
  if (t0 != t0 || t1 != t1) return 1;
  if (t0 > t1) { const double x = t0; t0 = t1; t1 = x; }
  *tmin = t0 > *tmin ? t0 : *tmin;
  *tmax = t1 < *tmax ? t1 : *tmax;
  return *tmin <= *tmax;
}
static int box_hit(const double* nd, v3 o, v3 inv, double tmin, double tmax) {
  return slab(nd[0], nd[3], o.x, inv.x, &tmin, &tmax) && slab(nd[1], nd[4], o.y, inv.y, &tmin, &tmax) &&
         slab(nd[2], nd[5], o.z, inv.z, &tmin, &tmax);
}

static int intersect_planes(const ro_scene* s, const ray_t* r, double tmin, double* tmax, hit_t* rec) {
  int hit = 0;
  for (uint64_t i = 0; i < s->n_planes; ++i) {
    hit_t tmp;
    if (plane_intersect(s, i, r, tmin, *tmax, &tmp)) {
      tmp.prim = (uint32_t)i;
      tmp.is_plane = 1;
      *rec = tmp;
      *tmax = tmp.t;
      hit = 1;
    }
  }
  return hit;
}

/* Scene::intersect_brute */
static int intersect_brute(const ro_scene* s, const ray_t* r, double tmin, double tmax0, hit_t* rec) {
  double tmax = tmax0;
  const int plane_hit = intersect_planes(s, r, tmin, &tmax, rec);
  double best_t = tmax, bb1 = 0, bb2 = 0;
  uint32_t best = NO_PRIM;
  for (uint64_t i = 0; i < s->n_prims; ++i) {
    double th, b1 = 0, b2 = 0;
    if (prim_hit_t(s, (uint32_t)i, r, tmin, best_t, &th, &b1, &b2)) {
      best_t = th;
      bb1 = b1;
      bb2 = b2;
      best = (uint32_t)i;
    }
  }
  if (best != NO_PRIM) {
    prim_finalize(s, best, r, best_t, bb1, bb2, rec);
    return 1;
  }
  return plane_hit;
}

/* Scene::intersect with Bvh::closest */
static int intersect(const ro_scene* s, const ray_t* r, double tmin, double tmax0, hit_t* rec) {
  if (!s->use_bvh) return intersect_brute(s, r, tmin, tmax0, rec);
  double tmax = tmax0;
  const int plane_hit = intersect_planes(s, r, tmin, &tmax, rec);
  double best_t = tmax, bb1 = 0, bb2 = 0;
  uint32_t best = NO_PRIM;
  if (s->n_nodes) {
    const v3 inv = V(1.0 / r->d.x, 1.0 / r->d.y, 1.0 / r->d.z);
    const int negd[3] = {inv.x < 0, inv.y < 0, inv.z < 0};
    uint32_t stack[64];
    int sp = 0;
    uint32_t idx = 0;
    double t_max = tmax;
    for (;;) {
      const double* n = NODE(s, idx);
      if (box_hit(n, r->o, inv, tmin, t_max)) {
        const uint32_t count = (uint32_t)n[7];
        if (count > 0) {
          const uint32_t first = (uint32_t)n[6];
          for (uint32_t k = 0; k < count; ++k) {
            const uint32_t pi = s->order[first + k];
            double th, b1 = 0, b2 = 0;
            double t = t_max;
            if (prim_hit_t(s, pi, r, tmin, t_max, &th, &b1, &b2)) {
              best_t = th;
              bb1 = b1;
              bb2 = b2;
              best = pi;
              t = th;
            }
            if (t < t_max) t_max = t;
          }
        } else {
          const uint32_t right = (uint32_t)n[6];
          const int axis = (int)n[8];
          if (negd[axis]) { stack[sp++] = idx + 1; idx = right; }
          else { stack[sp++] = right; idx = idx + 1; }
          continue;
        }
      }
      if (sp == 0) break;
      idx = stack[--sp];
    }
  }
  if (best != NO_PRIM) {
    prim_finalize(s, best, r, best_t, bb1, bb2, rec);
    return 1;
  }
  return plane_hit;
}

/* Scene::occluded */
static int occluded(const ro_scene* s, const ray_t* r, double tmax) {
  const double tmin = RAY_TMIN;
  hit_t tmp;
  for (uint64_t i = 0; i < s->n_planes; ++i)
    if (plane_intersect(s, i, r, tmin, tmax, &tmp)) return 1;
  double th, b1, b2;
  if (!s->use_bvh) {
    for (uint64_t i = 0; i < s->n_prims; ++i)
      if (prim_hit_t(s, (uint32_t)i, r, tmin, tmax, &th, &b1, &b2)) return 1;
    return 0;
  }
  if (!s->n_nodes) return 0;
  const v3 inv = V(1.0 / r->d.x, 1.0 / r->d.y, 1.0 / r->d.z);
  uint32_t stack[64];
  int sp = 0;
  uint32_t idx = 0;
  for (;;) {
    const double* n = NODE(s, idx);
    if (box_hit(n, r->o, inv, tmin, tmax)) {
      const uint32_t count = (uint32_t)n[7];
      if (count > 0) {
        const uint32_t first = (uint32_t)n[6];
        for (uint32_t k = 0; k < count; ++k)
          if (prim_hit_t(s, s->order[first + k], r, tmin, tmax, &th, &b1, &b2) && th < tmax) return 1;
      } else {
        stack[sp++] = (uint32_t)n[6];
        idx = idx + 1;
        continue;
      }
    }
    if (sp == 0) break;
    idx = stack[--sp];
  }
  return 0;
}

/* ---------------------------------------------------------------- materials */
static v3 texture(const double* m, v3 p) {
  const double scale = m[7];
  if (scale <= 0) return at(m + 1);
  const double off = 1e-4;
  const long long parity = (long long)floor(p.x * scale + off) + (long long)floor(p.y * scale + off) +
                           (long long)floor(p.z * scale + off);
  return (parity & 1) ? at(m + 4) : at(m + 1);
}
static v3 emission(const double* m) { return m[0] == 3 ? scl(at(m + 1), m[10]) : V(0, 0, 0); }
static v3 emitted(const double* m, int front) {
  if (m[0] == 3 && (front || m[11] != 0)) return scl(at(m + 1), m[10]);
  return V(0, 0, 0);
}
static double schlick(double c, double eta) {
  double r0 = (1 - eta) / (1 + eta);
  r0 *= r0;
  const double m = 1 - c;
  return r0 + (1 - r0) * m * m * m * m * m;
}

typedef struct { v3 dir, weight; int specular; } scatter_t;

static int scatter(const double* m, const ray_t* in, const hit_t* rec, rng_t* rng, scatter_t* out) {
  const int kind = (int)m[0];
  if (kind == 0) {
    const onb_t b = onb(rec->normal);
    out->dir = to_world(&b, cosine_hemisphere(rng));
    if (dot(out->dir, rec->gn) <= 0) return 0;
    out->weight = texture(m, rec->p);
    out->specular = 0;
    return 1;
  }
  if (kind == 1) {
    const v3 unit_in = unit(in->d);
    v3 d = reflect(unit_in, rec->normal);
    if (m[8] > 0) d = unit(add(unit(d), scl(random_unit_vector(rng), m[8])));
    if (dot(d, rec->gn) <= 0) return 0;
    out->dir = d;
    out->weight = at(m + 1);
    out->specular = 1;
    return 1;
  }
  if (kind == 2) {
    const double eta = rec->front ? (1.0 / m[9]) : m[9];
    const v3 unit_in = unit(in->d);
    const double cos_i = fmin(dot(neg(unit_in), rec->normal), 1.0);
    v3 refr;
    const int can = refract(unit_in, rec->normal, eta, &refr);
    if (!can || uni(rng) < schlick(cos_i, eta)) out->dir = reflect(unit_in, rec->normal);
    else out->dir = unit(refr);
    out->weight = at(m + 1);
    out->specular = 1;
    return 1;
  }
  return 0;
}

static v3 eval_brdf_cos(const double* m, const hit_t* rec, v3 wi) {
  if (m[0] != 0) return V(0, 0, 0);
  const double c = dot(rec->normal, wi);
  if (c <= 0 || dot(rec->gn, wi) <= 0) return V(0, 0, 0);
  return scl(texture(m, rec->p), c * INV_PI);
}

static v3 background(const ro_scene* s, v3 d) {
  const double* b = s->background;
  const v3 top = at(b + 1), bottom = at(b + 4);
  if (b[0] != 0) return scl(top, b[7]);
  const double t = 0.5 * (unit(d).y + 1.0);
  return scl(add(scl(bottom, 1 - t), scl(top, t)), b[7]);
}

/* ---------------------------------------------------------------- integrators */
typedef struct { uint64_t rays, shadow, rr, invalid; } counters_t;

/* pdf_out, wi_out (may be NULL): the solid-angle pdf of the sampled direction (0
 * for a point light) and the direction itself, for the MIS extension's weights. */
static v3 sample_one_light(const ro_scene* s, uint32_t li, const hit_t* rec, const double* mat, rng_t* rng,
                           counters_t* st, double* pdf_out, v3* wi_out) {
  double pdf_l = 0;
  const v3 p = rec->p;
  v3 wi;
  double dist = 0;
  v3 rad;
  const uint32_t kind = s->lights[2 * li], index = s->lights[2 * li + 1];
  if (kind == 0) {
    const double* L = s->point_lights + 6 * (size_t)index;
    const v3 d = sub(at(L), p);
    const double d2 = len2(d);
    if (d2 < 1e-16) return V(0, 0, 0);
    dist = sqrt(d2);
    wi = dvs(d, dist);
    rad = dvs(at(L + 3), d2);
  } else {
    const double* pr = PRIM(s, index);
    const double* lm = MAT(s, (uint32_t)pr[1]);
    if (pr[0] == 0) {
      const v3 c = at(pr + 3);
      const double radius = pr[6];
      const v3 oc = sub(c, p);
      const double d2 = len2(oc);
      const double r2 = radius * radius;
      if (d2 <= r2 * (1 + 1e-9)) {
        if (lm[11] == 0) return V(0, 0, 0);
        const v3 nl = random_unit_vector(rng);
        const v3 d = sub(add(c, scl(nl, radius)), p);
        const double dd2 = len2(d);
        if (dd2 < 1e-16) return V(0, 0, 0);
        dist = sqrt(dd2);
        wi = dvs(d, dist);
        const double cos_l = fabs(dot(nl, wi));
        if (cos_l < 1e-9) return V(0, 0, 0);
        const double area = 4 * PI * radius * radius;
        rad = scl(emission(lm), cos_l * area / dd2);
        pdf_l = dd2 / (cos_l * area);
      } else {
        const double x = r2 / d2;
        const double omc = x / (1 + sqrt(1 - x));
        const double cos_max = 1 - omc;
        const onb_t b = onb(dvs(oc, sqrt(d2)));
        wi = to_world(&b, uniform_cone(rng, cos_max));
        const ray_t lr = {p, wi};
        double th;
        if (!sphere_hit_t(pr, &lr, 0, INFINITY, &th)) return V(0, 0, 0);
        dist = th;
        const double pdf = 1 / (2 * PI * omc);
        rad = dvs(emission(lm), pdf);
        pdf_l = pdf;
      }
    } else {
      double b1, b2;
      uniform_triangle(rng, &b1, &b2);
      const v3 v0 = at(pr + 3), v1 = at(pr + 6), v2 = at(pr + 9);
      const v3 q = add(add(scl(v0, 1 - b1 - b2), scl(v1, b1)), scl(v2, b2));
      const v3 d = sub(q, p);
      const double d2 = len2(d);
      if (d2 < 1e-16) return V(0, 0, 0);
      dist = sqrt(d2);
      wi = dvs(d, dist);
      const v3 nl = unit(cross(sub(v1, v0), sub(v2, v0)));
      const double cos_signed = -dot(nl, wi);
      if (cos_signed <= 0 && lm[11] == 0) return V(0, 0, 0);
      const double cos_l = fabs(cos_signed);
      if (cos_l < 1e-9) return V(0, 0, 0);
      const double area = 0.5 * len(cross(sub(v1, v0), sub(v2, v0)));
      const double pdf = d2 / (cos_l * area);
      rad = dvs(emission(lm), pdf);
      pdf_l = pdf;
    }
  }
  if (pdf_out) *pdf_out = pdf_l;
  if (wi_out) *wi_out = wi;
  const v3 f = eval_brdf_cos(mat, rec, wi);
  if (is_zero(f) || is_zero(rad)) return V(0, 0, 0);
  const v3 origin = offset_origin(p, rec->gn, wi);
  const v3 target = add(p, scl(wi, dist));
  double tmax = len(sub(target, origin)) - 4 * spawn_offset(target);
  if (tmax < 0) tmax = 0;
  st->shadow++;
  const ray_t sr = {origin, wi};
  if (occluded(s, &sr, tmax)) return V(0, 0, 0);
  return mul(f, rad);
}

static int is_sampled_light(const ro_scene* s, const hit_t* rec) {
  if (rec->is_plane || rec->prim == NO_PRIM) return 0;
  return !is_zero(emission(MAT(s, (uint32_t)PRIM(s, rec->prim)[1])));
}

/* MIS extension: power heuristic (Veach, beta = 2) of pdf a against pdf b. */
static double power_heuristic(double a, double b) {
  const double a2 = a * a, b2 = b * b;
  return a2 + b2 > 0 ? a2 / (a2 + b2) : 0;
}

/* MIS extension: the solid-angle pdf with which light sampling would have chosen
 * direction ray.d from ray.o toward the emitter that `rec` hit. */
static double light_pdf_of_hit(const ro_scene* s, const ray_t* ray, const hit_t* rec) {
  const double* pr = PRIM(s, rec->prim);
  const double cos_l = fabs(dot(rec->gn, ray->d));
  if (pr[0] == 0) {
    const double r = pr[6], r2 = r * r;
    const v3 oc = sub(at(pr + 3), ray->o);
    const double d2 = len2(oc);
    if (d2 <= r2) return cos_l > 0 ? rec->t * rec->t / (cos_l * 4 * PI * r2) : 0;
    const double x = r2 / d2;
    return 1 / (2 * PI * (x / (1 + sqrt(1 - x))));
  }
  const v3 v0 = at(pr + 3), v1 = at(pr + 6), v2 = at(pr + 9);
  const double area = 0.5 * len(cross(sub(v1, v0), sub(v2, v0)));
  return cos_l > 0 && area > 0 ? rec->t * rec->t / (cos_l * area) : 0;
}

static v3 path_trace(const ro_scene* s, ray_t ray, rng_t* rng, counters_t* st) {
  v3 L = V(0, 0, 0), beta = V(1, 1, 1);
  int specular_bounce = 1;
  const int mis = s->light_sampling == 2;
  double pdf_prev = 0; /* MIS: cosine pdf of the direction the last diffuse bounce sampled */
  for (int depth = 0; depth < s->max_depth; ++depth) {
    hit_t rec;
    st->rays++;
    if (!intersect(s, &ray, RAY_TMIN, INFINITY, &rec)) {
      L = add(L, mul(beta, background(s, ray.d)));
      break;
    }
    const double* mat = MAT(s, rec.material);
    const v3 le = emitted(mat, rec.front);
    if (!is_zero(le) && (specular_bounce || !s->light_sampling || !is_sampled_light(s, &rec))) {
      L = add(L, mul(beta, le));
    } else if (!is_zero(le) && mis) {
      const double w = power_heuristic(pdf_prev, light_pdf_of_hit(s, &ray, &rec) / (double)s->n_lights);
      L = add(L, scl(mul(beta, le), w));
    }
    scatter_t sr;
    if (!scatter(mat, &ray, &rec, rng, &sr)) break;
    if (s->light_sampling && !sr.specular && s->n_lights > 0) {
      const uint32_t n = (uint32_t)s->n_lights;
      const uint32_t li = below(rng, n);
      double pdf_l = 0;
      v3 wi = V(0, 0, 0);
      const v3 c = sample_one_light(s, li, &rec, mat, rng, st, &pdf_l, &wi);
      double w = 1; /* a point light (pdf 0) cannot be hit by BSDF sampling */
      if (mis && pdf_l > 0) w = power_heuristic(pdf_l / (double)n, dot(rec.normal, wi) * INV_PI);
      L = add(L, scl(mul(beta, c), (double)n * w));
    }
    if (mis && !sr.specular) pdf_prev = dot(rec.normal, sr.dir) * INV_PI;
    beta = mul(beta, sr.weight);
    specular_bounce = sr.specular;
    if (is_zero(beta)) break;
    if (depth + 1 >= s->rr_min_depth) {
      double q = maxc(beta);
      q = q < 0.05 ? 0.05 : (q > 0.95 ? 0.95 : q);
      if (uni(rng) >= q) {
        st->rr++;
        break;
      }
      beta = dvs(beta, q);
    }
    ray.o = offset_origin(rec.p, rec.gn, sr.dir);
    ray.d = sr.dir;
  }
  return L;
}

static v3 direct_trace(const ro_scene* s, ray_t ray, rng_t* rng, counters_t* st, int depth) {
  st->rays++;
  hit_t rec;
  if (!intersect(s, &ray, RAY_TMIN, INFINITY, &rec)) return background(s, ray.d);
  const double* mat = MAT(s, rec.material);
  v3 L = emitted(mat, rec.front);
  if (depth >= s->max_depth) return L;
  const int kind = (int)mat[0];
  if (kind == 0) {
    for (uint32_t li = 0; li < s->n_lights; ++li)
      L = add(L, sample_one_light(s, li, &rec, mat, rng, st, NULL, NULL));
    return L;
  }
  if (kind == 1) {
    scatter_t sr;
    if (scatter(mat, &ray, &rec, rng, &sr)) {
      const ray_t nr = {offset_origin(rec.p, rec.gn, sr.dir), sr.dir};
      L = add(L, mul(at(mat + 1), direct_trace(s, nr, rng, st, depth + 1)));
    }
    return L;
  }
  if (kind == 2) {
    const v3 in = unit(ray.d);
    const double eta = rec.front ? 1.0 / mat[9] : mat[9];
    const double cos_i = fmin(dot(neg(in), rec.normal), 1.0);
    v3 refr;
    const int can = refract(in, rec.normal, eta, &refr);
    const double F = can ? schlick(cos_i, eta) : 1.0;
    const v3 rd = reflect(in, rec.normal);
    const ray_t r1 = {offset_origin(rec.p, rec.gn, rd), rd};
    L = add(L, mul(scl(at(mat + 1), F), direct_trace(s, r1, rng, st, depth + 1)));
    if (can) {
      const v3 td = unit(refr);
      const ray_t r2 = {offset_origin(rec.p, rec.gn, td), td};
      L = add(L, mul(scl(at(mat + 1), 1 - F), direct_trace(s, r2, rng, st, depth + 1)));
    }
    return L;
  }
  return L;
}

static v3 radiance(const ro_scene* s, ray_t r, rng_t* rng, counters_t* st) {
  if (s->integrator == 0) return path_trace(s, r, rng, st);
  if (s->integrator == 1) return direct_trace(s, r, rng, st, 0);
  st->rays++;
  hit_t rec;
  if (!intersect(s, &r, RAY_TMIN, INFINITY, &rec)) return V(0, 0, 0);
  const v3 n = rec.front ? rec.normal : neg(rec.normal);
  return scl(add(n, V(1, 1, 1)), 0.5);
}

static ray_t camera_ray(const ro_scene* s, int i, int j, double sx, double sy, rng_t* rng) {
  const double* c = s->camera;
  const v3 origin = at(c), corner = at(c + 3), du = at(c + 6), dv = at(c + 9), u = at(c + 12), v = at(c + 15);
  const v3 target = add(add(corner, scl(du, i + sx)), scl(dv, j + sy));
  v3 o = origin;
  if (c[18] > 0) {
    double dx, dy;
    random_in_unit_disk(rng, &dx, &dy);
    o = add(origin, scl(add(scl(u, dx), scl(v, dy)), c[18]));
  }
  ray_t r = {o, unit(sub(target, o))};
  return r;
}

/* ---------------------------------------------------------------- exports */
void ro_closest(const ro_scene* s, const double* rays, int64_t n, int32_t brute, double* t, int32_t* prim,
                int32_t* is_plane, double* gn) {
  for (int64_t i = 0; i < n; ++i) {
    const double* r = rays + 8 * i;
    const ray_t ray = {V(r[0], r[1], r[2]), V(r[4], r[5], r[6])};
    hit_t rec;
    memset(&rec, 0, sizeof rec);
    rec.prim = NO_PRIM;
    const int h = brute ? intersect_brute(s, &ray, r[3], r[7], &rec) : intersect(s, &ray, r[3], r[7], &rec);
    if (t) t[i] = h ? rec.t : 0;
    if (prim) prim[i] = h ? (int32_t)rec.prim : -1;
    if (is_plane) is_plane[i] = h ? rec.is_plane : 0;
    if (gn) {
      gn[3 * i] = h ? rec.gn.x : 0;
      gn[3 * i + 1] = h ? rec.gn.y : 0;
      gn[3 * i + 2] = h ? rec.gn.z : 0;
    }
  }
}

void ro_occluded(const ro_scene* s, const double* rays, int64_t n, uint8_t* out) {
  for (int64_t i = 0; i < n; ++i) {
    const double* r = rays + 8 * i;
    const ray_t ray = {V(r[0], r[1], r[2]), V(r[4], r[5], r[6])};
    out[i] = (uint8_t)occluded(s, &ray, r[7]);
  }
}

void ro_camera(const ro_scene* s, const double* pix, int64_t n, uint64_t pixel_for_rng, double* out) {
  for (int64_t k = 0; k < n; ++k) {
    rng_t rng = rng_for_sample(s->seed, pixel_for_rng, (uint64_t)k);
    const ray_t r = camera_ray(s, (int)pix[4 * k], (int)pix[4 * k + 1], pix[4 * k + 2], pix[4 * k + 3], &rng);
    out[6 * k] = r.o.x; out[6 * k + 1] = r.o.y; out[6 * k + 2] = r.o.z;
    out[6 * k + 3] = r.d.x; out[6 * k + 4] = r.d.y; out[6 * k + 5] = r.d.z;
  }
}

void ro_sample(const ro_scene* s, int32_t x, int32_t y, uint32_t sample, double* rgb) {
  counters_t st = {0, 0, 0, 0};
  const uint64_t pixel = (uint64_t)y * (uint64_t)s->width + (uint64_t)x;
  rng_t rng = rng_for_sample(s->seed, pixel, sample);
  const double jx = uni(&rng);
  const double jy = uni(&rng);
  const ray_t r = camera_ray(s, x, y, jx, jy, &rng);
  const v3 L = radiance(s, r, &rng, &st);
  rgb[0] = L.x;
  rgb[1] = L.y;
  rgb[2] = L.z;
}

void ro_render_rows(const ro_scene* s, int32_t y0, int32_t y1, uint32_t s0, uint32_t s1, double* sum, double* sumsq,
                    uint64_t* stats) {
  counters_t st = {0, 0, 0, 0};
  for (int32_t y = y0; y < y1; ++y)
    for (int32_t x = 0; x < s->width; ++x) {
      const uint64_t pixel = (uint64_t)y * (uint64_t)s->width + (uint64_t)x;
      v3 acc = V(0, 0, 0), acc2 = V(0, 0, 0);
      double* ps = sum + 3 * pixel;
      double* pq = sumsq + 3 * pixel;
      acc = V(ps[0], ps[1], ps[2]);
      acc2 = V(pq[0], pq[1], pq[2]);
      for (uint32_t smp = s0; smp < s1; ++smp) {
        rng_t rng = rng_for_sample(s->seed, pixel, smp);
        const double jx = uni(&rng);
        const double jy = uni(&rng);
        const ray_t r = camera_ray(s, x, y, jx, jy, &rng);
        v3 L = radiance(s, r, &rng, &st);
        if (!finite3(L) || L.x < 0 || L.y < 0 || L.z < 0) {
          st.invalid++;
          L = V(0, 0, 0);
        }
        acc = add(acc, L);
        acc2 = add(acc2, mul(L, L));
      }
      ps[0] = acc.x; ps[1] = acc.y; ps[2] = acc.z;
      pq[0] = acc2.x; pq[1] = acc2.y; pq[2] = acc2.z;
    }
  if (stats) {
    stats[0] += st.rays;
    stats[1] += st.shadow;
    stats[2] += st.rr;
    stats[3] += st.invalid;
  }
}

static double aces(double x) {
  const double a = 2.51, b = 0.03, c = 2.43, d = 0.59, e = 0.14;
  const double v = (x * (a * x + b)) / (x * (c * x + d) + e);
  return v < 0 ? 0 : (v > 1 ? 1 : v);
}
static uint8_t srgb8(double v) {
  v = v < 0 ? 0 : (v > 1 ? 1 : v);
  double s = v <= 0.0031308 ? 12.92 * v : 1.055 * pow(v, 1.0 / 2.4) - 0.055;
  s = s < 0 ? 0 : (s > 1 ? 1 : s);
  return (uint8_t)lround(s * 255.0);
}

void ro_tone_map_srgb8(const double* rgb, int64_t n, int32_t op, double exposure, uint8_t* out) {
  for (int64_t i = 0; i < n; ++i) {
    v3 c = scl(at(rgb + 3 * i), exposure);
    if (!finite3(c)) c = V(0, 0, 0);
    double ch[3] = {c.x, c.y, c.z};
    for (int k = 0; k < 3; ++k) {
      double v = ch[k];
      if (op == 0) v = v < 0 ? 0 : (v > 1 ? 1 : v);
      else if (op == 1) v = v / (1 + v);
      else v = aces(v);
      out[3 * i + k] = srgb8(v);
    }
  }
}
