#pragma once
// Ray queries against one scene's BVH + planes, in fp32.
//
// Semantics follow the reference's Scene::intersect / intersect_brute / occluded
// (src/core/scene.cpp:152-234) and Bvh::closest / Bvh::any
// (include/raytracer/geometry/bvh.hpp:75-132): planes are tested linearly first and
// shrink t_max; the BVH is walked depth first; a primitive is accepted only if
// t_min < t < t_max (strict), so among equal distances the first tested wins.
// The closest-hit walk visits the child whose box the ray enters first (the
// reference orders by the sign of the direction on the split axis); that visits
// fewer nodes, and only changes which of two primitives at exactly the same
// distance is reported.
//
// Traversal stack: the top kStackSmem entries of each thread's stack live in
// shared memory (laid out [entry][thread] so a warp's pushes hit 32 distinct
// banks); deeper entries spill to a small local array. The reference caps BVH
// depth at 60, so 64 entries always suffice.
#include "device/dmath.cuh"

namespace rtg {

constexpr int kStackDepth = 64;

struct RayHit {
  float t;
  std::uint32_t word;  // slot, kHitPlaneBit | plane, or kHitMiss
  float b1, b2;
};

struct TraceCount {
  std::uint32_t nodes = 0, prims = 0, spheres = 0;
  __device__ __forceinline__ void add_prim(std::uint32_t id) {
    ++prims;
    spheres += (id & kSphereBit) ? 1u : 0u;
  }
};

// Precomputed per-ray slab-test terms: t = box * inv - o * inv.
struct SlabRay {
  float3 inv, ooi;
  int neg[3];
  __device__ __forceinline__ SlabRay(float3 o, float3 d) {
    // A zero direction component becomes a tiny one so 0 * inf never appears;
    // the slab on that axis then spans everything or nothing, as it should.
    auto safe = [](float c) { return fabsf(c) < 1e-20f ? copysignf(1e-20f, c) : c; };
    inv = f3(1.f / safe(d.x), 1.f / safe(d.y), 1.f / safe(d.z));
    ooi = f3(__fmul_rn(o.x, inv.x), __fmul_rn(o.y, inv.y), __fmul_rn(o.z, inv.z));
    neg[0] = d.x < 0.f;
    neg[1] = d.y < 0.f;
    neg[2] = d.z < 0.f;
  }
};

// Both children's slab tests from one node; returns entry distances.
// `second_first` (when given) is set when child 1's box is entered before child 0's.
__device__ __forceinline__ void node_boxes(const DevNode* __restrict__ node, const SlabRay& r, float tmin, float tmax,
                                           bool& hit0, bool& hit1, int4& link, bool* second_first = nullptr) {
  const float4 a = __ldg(&node->xy0);
  const float4 b = __ldg(&node->xy1);
  const float4 c = __ldg(&node->zz);
  link = __ldg(&node->link);
  const float ax0 = fmaf(a.x, r.inv.x, -r.ooi.x), ax1 = fmaf(a.y, r.inv.x, -r.ooi.x);
  const float ay0 = fmaf(a.z, r.inv.y, -r.ooi.y), ay1 = fmaf(a.w, r.inv.y, -r.ooi.y);
  const float az0 = fmaf(c.x, r.inv.z, -r.ooi.z), az1 = fmaf(c.y, r.inv.z, -r.ooi.z);
  const float bx0 = fmaf(b.x, r.inv.x, -r.ooi.x), bx1 = fmaf(b.y, r.inv.x, -r.ooi.x);
  const float by0 = fmaf(b.z, r.inv.y, -r.ooi.y), by1 = fmaf(b.w, r.inv.y, -r.ooi.y);
  const float bz0 = fmaf(c.z, r.inv.z, -r.ooi.z), bz1 = fmaf(c.w, r.inv.z, -r.ooi.z);
  const float a_in = fmaxf(fmaxf(fminf(ax0, ax1), fminf(ay0, ay1)), fmaxf(fminf(az0, az1), tmin));
  const float a_out = fminf(fminf(fmaxf(ax0, ax1), fmaxf(ay0, ay1)), fminf(fmaxf(az0, az1), tmax));
  const float b_in = fmaxf(fmaxf(fminf(bx0, bx1), fminf(by0, by1)), fmaxf(fminf(bz0, bz1), tmin));
  const float b_out = fminf(fminf(fmaxf(bx0, bx1), fmaxf(by0, by1)), fminf(fmaxf(bz0, bz1), tmax));
  hit0 = a_in <= a_out;
  hit1 = b_in <= b_out;
  if (second_first) *second_first = b_in < a_in;
}

// Barycentric slack of the fp32 triangle test. Without it, a ray through the edge
// two triangles share can round outside both and pass through the surface: with
// the Cornell camera, pixel centres on the image diagonal met the back wall's
// diagonal edge that way. The reference, in double, hits one of the two.
constexpr float kEdgeSlack = 1e-6f;

// Möller-Trumbore, two-sided (include/raytracer/geometry/shapes.hpp:110-127).
// `k` is dot(r, e1 x e2) for the residual r that rounding v0 to fp32 lost: the
// distance to the plane through the double-precision v0 is (dot(e2, qv) - k) / det.
// For hits close to the ray origin that rounding, not the arithmetic, dominates
// the error of t. Rounding is pinned (dmath.cuh) so every kernel gets the same hit.
__device__ __forceinline__ bool tri_test(float3 o, float3 d, float3 v0, float3 e1, float3 e2, float k, float tmin,
                                         float tmax, float& t, float& b1, float& b2) {
  const float3 pv = cross3p(d, e2);
  const float det = dot3p(e1, pv);
  if (fabsf(det) < 1e-14f) return false;
  const float inv_det = 1.f / det;
  const float3 tv = sub3p(o, v0);
  const float u = __fmul_rn(dot3p(tv, pv), inv_det);
  if (u < -kEdgeSlack || u > 1.f + kEdgeSlack) return false;
  const float3 qv = cross3p(tv, e1);
  const float v = __fmul_rn(dot3p(d, qv), inv_det);
  if (v < -kEdgeSlack || __fadd_rn(u, v) > 1.f + kEdgeSlack) return false;
  const float tt = __fmul_rn(__fsub_rn(dot3p(e2, qv), k), inv_det);
  if (!(tmin < tt && tt < tmax)) return false;
  t = tt;
  b1 = u;
  b2 = v;
  return true;
}

// Ray-sphere with the Haines et al. precision fixes ("Precision Improvements for
// Ray/Sphere Intersection", Ray Tracing Gems ch. 7), as the reference's
// Sphere::hit_t (include/raytracer/geometry/shapes.hpp:25-46). `rc` is what
// rounding the centre to fp32 lost; adding it after the subtraction gives the
// offset to the double-precision centre. Rounding is pinned (dmath.cuh).
__device__ __forceinline__ bool sphere_test(float3 o, float3 d, float3 c, float3 rc, float radius, float tmin,
                                            float tmax, float& t) {
  const float3 oc = add3p(sub3p(c, o), rc);
  const float a = dot3p(d, d);
  if (a == 0.f) return false;
  const float h = dot3p(d, oc);
  const float cc = fmaf(-radius, radius, dot3p(oc, oc));
  const float s = h / a;
  const float3 perp = f3(fmaf(-s, d.x, oc.x), fmaf(-s, d.y, oc.y), fmaf(-s, d.z, oc.z));
  const float disc = __fmul_rn(a, fmaf(radius, radius, -dot3p(perp, perp)));
  if (disc < 0.f) return false;
  const float q = __fadd_rn(h, copysignf(sqrtf(disc), h));
  float t0 = cc / q, t1 = q / a;
  if (q == 0.f) t0 = t1 = h / a;
  if (t0 > t1) { const float s = t0; t0 = t1; t1 = s; }
  float tt = t0;
  if (!(tmin < tt && tt < tmax)) {
    tt = t1;
    if (!(tmin < tt && tt < tmax)) return false;
  }
  t = tt;
  return true;
}

// normal.w holds the plane offset that rounding the point to fp32 lost. Rounding
// is pinned (dmath.cuh).
__device__ __forceinline__ bool plane_test(const DevPlane& pl, float3 o, float3 d, float tmin, float tmax, float& t) {
  const float3 n = f3(pl.normal);
  const float denom = dot3p(n, d);
  if (fabsf(denom) < 1e-12f) return false;
  const float tt = __fadd_rn(dot3p(sub3p(f3(pl.point), o), n), pl.normal.w) / denom;
  if (!(tmin < tt && tt < tmax)) return false;
  t = tt;
  return true;
}

// Tests one primitive slot; updates the best hit when closer.
__device__ __forceinline__ std::uint32_t prim_slot_test(const float4* __restrict__ prims, int slot, float3 o, float3 d,
                                                        float tmin, RayHit& best) {
  // All three rows at once: waiting for the kind bit before fetching the third
  // row put a second memory round trip on every triangle test.
  const float4 p0 = __ldg(&prims[3 * slot]);
  const float4 p1 = __ldg(&prims[3 * slot + 1]);
  const float4 p2 = __ldg(&prims[3 * slot + 2]);
  const std::uint32_t id = __float_as_uint(p0.w);
  float t, b1 = 0.f, b2 = 0.f;
  bool hit;
  if (id & kSphereBit) {
    hit = sphere_test(o, d, f3(p0), f3(p2), p1.x, tmin, best.t, t);
  } else {
    hit = tri_test(o, d, f3(p0), f3(p1), f3(p2), p1.w, tmin, best.t, t, b1, b2);
  }
  if (hit) {
    best.t = t;
    best.word = static_cast<std::uint32_t>(slot);
    best.b1 = b1;
    best.b2 = b2;
  }
  return id;
}

template <int kStackSmem, int kBlock, int kDepth = kStackDepth>
struct TraversalStack {
  int* smem;  // this thread's column: entry k at smem[k * kBlock]
  int spill[kDepth - kStackSmem];
  int sp = 0;
  __device__ __forceinline__ explicit TraversalStack(int* base) : smem(base + threadIdx.x) {}
  __device__ __forceinline__ void push(int v) {
    if (sp < kStackSmem) smem[sp * kBlock] = v;
    else spill[sp - kStackSmem] = v;
    ++sp;
  }
  __device__ __forceinline__ bool pop(int& v) {
    if (sp == 0) return false;
    --sp;
    v = sp < kStackSmem ? smem[sp * kBlock] : spill[sp - kStackSmem];
    return true;
  }
};

// Closest hit over planes then BVH. `stack_base` is the block's shared stack area.
template <int kStackSmem, int kBlock, bool kCount>
__device__ __forceinline__ RayHit closest_hit(const RtgSceneDev& sc, float3 o, float3 d, float tmin, float tmax,
                                              int* stack_base, TraceCount& cnt) {
  RayHit best{tmax, kHitMiss, 0.f, 0.f};
  for (int i = 0; i < sc.n_planes; ++i) {
    float t;
    if (plane_test(sc.planes[i], o, d, tmin, best.t, t)) {
      best.t = t;
      best.word = kHitPlaneBit | static_cast<std::uint32_t>(i);
    }
  }
  if (sc.root == INT32_MIN) return best;  // no bounded primitives
  const SlabRay sr(o, d);
  TraversalStack<kStackSmem, kBlock> st(stack_base);
  int cur = sc.root;
  while (true) {
    if (cur >= 0) {
      if (kCount) cnt.nodes++;
      bool h0, h1, right_first;
      int4 link;
      node_boxes(sc.nodes + cur, sr, tmin, best.t, h0, h1, link, &right_first);
      if (h0 && h1) {
        st.push(right_first ? link.x : link.y);
        cur = right_first ? link.y : link.x;
        continue;
      }
      if (h0) { cur = link.x; continue; }
      if (h1) { cur = link.y; continue; }
    } else {
      int slot = ~cur;
      while (true) {
        const std::uint32_t id = prim_slot_test(sc.prims, slot, o, d, tmin, best);
        if (kCount) cnt.add_prim(id);
        if (id & kLastInLeaf) break;
        ++slot;
      }
    }
    if (!st.pop(cur)) break;
  }
  return best;
}

// Slab tests of a four-wide node's children: entry distances and hit flags.
__device__ __forceinline__ void node4_boxes(const DevNode4* __restrict__ nd, const SlabRay& r, float tmin, float tmax,
                                            float in[4], bool hit[4], int link[4]) {
  const float4 lx = __ldg(&nd->lo_x), hx = __ldg(&nd->hi_x);
  const float4 ly = __ldg(&nd->lo_y), hy = __ldg(&nd->hi_y);
  const float4 lz = __ldg(&nd->lo_z), hz = __ldg(&nd->hi_z);
  const int4 lk = __ldg(&nd->link);
  const float lox[4] = {lx.x, lx.y, lx.z, lx.w}, hix[4] = {hx.x, hx.y, hx.z, hx.w};
  const float loy[4] = {ly.x, ly.y, ly.z, ly.w}, hiy[4] = {hy.x, hy.y, hy.z, hy.w};
  const float loz[4] = {lz.x, lz.y, lz.z, lz.w}, hiz[4] = {hz.x, hz.y, hz.z, hz.w};
  link[0] = lk.x;
  link[1] = lk.y;
  link[2] = lk.z;
  link[3] = lk.w;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float x0 = fmaf(lox[k], r.inv.x, -r.ooi.x), x1 = fmaf(hix[k], r.inv.x, -r.ooi.x);
    const float y0 = fmaf(loy[k], r.inv.y, -r.ooi.y), y1 = fmaf(hiy[k], r.inv.y, -r.ooi.y);
    const float z0 = fmaf(loz[k], r.inv.z, -r.ooi.z), z1 = fmaf(hiz[k], r.inv.z, -r.ooi.z);
    in[k] = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
    const float out = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tmax));
    hit[k] = in[k] <= out && link[k] != kNoChild;
  }
}

// Any hit over planes then the four-wide BVH (order does not matter: first hit wins).
template <int kStackSmem, int kBlock, bool kCount>
__device__ __forceinline__ bool any_hit4(const RtgSceneDev& sc, float3 o, float3 d, float tmin, float tmax,
                                         int* stack_base, TraceCount& cnt) {
  for (int i = 0; i < sc.n_planes; ++i) {
    float t;
    if (plane_test(sc.planes[i], o, d, tmin, tmax, t)) return true;
  }
  if (sc.root4 == INT32_MIN) return false;
  const SlabRay sr(o, d);
  TraversalStack<kStackSmem, kBlock, kWideStackDepth> st(stack_base);
  int cur = sc.root4;
  RayHit probe{tmax, kHitMiss, 0.f, 0.f};
  while (true) {
    if (cur >= 0) {
      if (kCount) cnt.nodes++;
      float in[4];
      bool hit[4];
      int link[4];
      node4_boxes(sc.nodes4 + cur, sr, tmin, tmax, in, hit, link);
      int next = INT32_MIN;
#pragma unroll
      for (int k = 3; k >= 0; --k) {
        if (!hit[k]) continue;
        if (next != INT32_MIN) st.push(next);
        next = link[k];
      }
      if (next != INT32_MIN) {
        cur = next;
        continue;
      }
    } else {
      int slot = ~cur;
      while (true) {
        const std::uint32_t id = prim_slot_test(sc.prims, slot, o, d, tmin, probe);
        if (kCount) cnt.add_prim(id);
        if (probe.word != kHitMiss) return true;
        if (id & kLastInLeaf) break;
        ++slot;
      }
    }
    if (!st.pop(cur)) break;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Compressed eight-wide tree (DevNode8; Ylitie, Karras and Laine, HPG 2017).
//
// A ray visits a node's children in the order of their slots XOR its direction
// octant, which the slot assignment makes roughly front to back. The traversal
// stack holds groups of children still to visit: the node index of the group's
// first interior child and one word with the node's interior-slot mask (bits
// 8-15) and the visit-order bits of the children left (bits 0-7). A node visit
// pushes at most the rest of its group, so the stack needs one entry per level.
// Leaf children hit at a node are tested at once, in visit order, before the
// walk descends.

struct Wide8Ray {
  float3 o, inv;
  std::uint32_t oct;  // bit k set: the direction is negative along axis k
  __device__ __forceinline__ Wide8Ray(float3 origin, float3 d) : o(origin) {
    // As SlabRay: a zero component becomes a tiny one of the same sign.
    auto safe = [](float c) { return fabsf(c) < 1e-20f ? copysignf(1e-20f, c) : c; };
    inv = f3(1.f / safe(d.x), 1.f / safe(d.y), 1.f / safe(d.z));
    oct = (inv.x < 0.f ? 1u : 0u) | (inv.y < 0.f ? 2u : 0u) | (inv.z < 0.f ? 4u : 0u);
  }
};

// Byte k (0-3) of `w` as a float, exactly: 2^23 + b built by a byte permute, then 2^23 subtracted.
__device__ __forceinline__ float quant_byte(std::uint32_t w, int k) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | static_cast<unsigned>(k))) - 8388608.f;
}

struct Node8Hits {
  std::uint32_t inner;  // visit-order bits of interior children hit
  std::uint32_t leaves; // visit-order bits of leaf children hit
  std::uint32_t imask;  // interior slots of the node
  uint4 b;              // child_base, prim_base, meta 0-3, meta 4-7
};

// Slab tests of a node's eight children against [tmin, tmax].
__device__ __forceinline__ Node8Hits node8_hits(const DevNode8* __restrict__ nd, const Wide8Ray& r, float tmin,
                                                float tmax) {
  const float4 a = __ldg(&nd->a);
  Node8Hits h;
  h.b = __ldg(&nd->b);
  const uint4 q0 = __ldg(&nd->qlo_xy), q1 = __ldg(&nd->qlo_z_hi_x), q2 = __ldg(&nd->qhi_yz);
  const std::uint32_t ew = __float_as_uint(a.w);
  h.imask = ew >> 24;
  // Node space: t = q * (scale / d) + (p - o) / d per axis.
  const float ax = __fmul_rn(__uint_as_float((ew & 0xFFu) << 23), r.inv.x);
  const float ay = __fmul_rn(__uint_as_float(((ew >> 8) & 0xFFu) << 23), r.inv.y);
  const float az = __fmul_rn(__uint_as_float(((ew >> 16) & 0xFFu) << 23), r.inv.z);
  const float bx = __fmul_rn(__fsub_rn(a.x, r.o.x), r.inv.x), by = __fmul_rn(__fsub_rn(a.y, r.o.y), r.inv.y);
  const float bz = __fmul_rn(__fsub_rn(a.z, r.o.z), r.inv.z);
  // Near and far planes per axis: lo bytes when the direction is positive.
  const bool px = !(r.oct & 1u), py = !(r.oct & 2u), pz = !(r.oct & 4u);
  const std::uint32_t nx0 = px ? q0.x : q1.z, nx1 = px ? q0.y : q1.w, fx0 = px ? q1.z : q0.x, fx1 = px ? q1.w : q0.y;
  const std::uint32_t ny0 = py ? q0.z : q2.x, ny1 = py ? q0.w : q2.y, fy0 = py ? q2.x : q0.z, fy1 = py ? q2.y : q0.w;
  const std::uint32_t nz0 = pz ? q1.x : q2.z, nz1 = pz ? q1.y : q2.w, fz0 = pz ? q2.z : q1.x, fz1 = pz ? q2.w : q1.y;
  h.inner = h.leaves = 0u;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int k = j & 3;
    const float tnx = fmaf(quant_byte(j < 4 ? nx0 : nx1, k), ax, bx);
    const float tny = fmaf(quant_byte(j < 4 ? ny0 : ny1, k), ay, by);
    const float tnz = fmaf(quant_byte(j < 4 ? nz0 : nz1, k), az, bz);
    const float tfx = fmaf(quant_byte(j < 4 ? fx0 : fx1, k), ax, bx);
    const float tfy = fmaf(quant_byte(j < 4 ? fy0 : fy1, k), ay, by);
    const float tfz = fmaf(quant_byte(j < 4 ? fz0 : fz1, k), az, bz);
    const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin));
    const float tf = fminf(fminf(tfx, tfy), fminf(tfz, tmax));
    if (tn <= tf) {
      const std::uint32_t bit = 1u << (static_cast<std::uint32_t>(j) ^ r.oct);
      if ((h.imask >> j) & 1u) h.inner |= bit;
      else h.leaves |= bit;
    }
  }
  return h;
}

// First slot of the leaf child in `slot` of a node.
__device__ __forceinline__ int leaf8_first(const uint4& b, std::uint32_t slot) {
  return static_cast<int>(b.y + (((slot < 4 ? b.z : b.w) >> (8 * (slot & 3u))) & 0xFFu));
}

template <int kStackSmem, int kBlock>
struct GroupStack {
  uint2* smem;  // this thread's column: entry k at smem[k * kBlock]
  uint2 spill[kWide8StackDepth - kStackSmem];
  int sp = 0;
  __device__ __forceinline__ explicit GroupStack(uint2* base) : smem(base + threadIdx.x) {}
  __device__ __forceinline__ void push(std::uint32_t base, std::uint32_t mask) {
    const uint2 v = make_uint2(base, mask);
    if (sp < kStackSmem) smem[sp * kBlock] = v;
    else spill[sp - kStackSmem] = v;
    ++sp;
  }
  __device__ __forceinline__ bool pop(std::uint32_t& base, std::uint32_t& mask) {
    if (sp == 0) return false;
    --sp;
    const uint2 v = sp < kStackSmem ? smem[sp * kBlock] : spill[sp - kStackSmem];
    base = v.x;
    mask = v.y;
    return true;
  }
};

// Closest hit over planes then the eight-wide tree. `stack_base` is the block's
// shared group-stack area (kStackSmem * kBlock entries).
template <int kStackSmem, int kBlock, bool kCount>
__device__ __forceinline__ RayHit closest_hit8(const RtgSceneDev& sc, float3 o, float3 d, float tmin, float tmax,
                                               uint2* stack_base, TraceCount& cnt) {
  RayHit best{tmax, kHitMiss, 0.f, 0.f};
  for (int i = 0; i < sc.n_planes; ++i) {
    float t;
    if (plane_test(sc.planes[i], o, d, tmin, best.t, t)) {
      best.t = t;
      best.word = kHitPlaneBit | static_cast<std::uint32_t>(i);
    }
  }
  if (sc.root8 == INT32_MIN) return best;
  if (sc.root8 < 0) {
    for (int slot = ~sc.root8;; ++slot) {
      const std::uint32_t id = prim_slot_test(sc.prims, slot, o, d, tmin, best);
      if (kCount) cnt.add_prim(id);
      if (id & kLastInLeaf) break;
    }
    return best;
  }
  const Wide8Ray r(o, d);
  GroupStack<kStackSmem, kBlock> st(stack_base);
  // The root as the one interior child (slot 0) of a group.
  std::uint32_t g_base = static_cast<std::uint32_t>(sc.root8), g_mask = (1u << r.oct) | (1u << 8);
  while (true) {
    if ((g_mask & 0xFFu) == 0u) {
      if (!st.pop(g_base, g_mask)) break;
      continue;
    }
    const std::uint32_t pos = static_cast<std::uint32_t>(__ffs(g_mask & 0xFFu) - 1);
    g_mask &= ~(1u << pos);
    const std::uint32_t slot = pos ^ r.oct;
    const std::uint32_t node = g_base + __popc((g_mask >> 8) & ((1u << slot) - 1u));
    if (g_mask & 0xFFu) st.push(g_base, g_mask);
    if (kCount) cnt.nodes++;
    const Node8Hits h = node8_hits(sc.nodes8 + node, r, tmin, best.t);
    for (std::uint32_t lh = h.leaves; lh; lh &= lh - 1u) {
      const std::uint32_t ls = static_cast<std::uint32_t>(__ffs(lh) - 1) ^ r.oct;
      for (int s = leaf8_first(h.b, ls);; ++s) {
        const std::uint32_t id = prim_slot_test(sc.prims, s, o, d, tmin, best);
        if (kCount) cnt.add_prim(id);
        if (id & kLastInLeaf) break;
      }
    }
    g_base = h.b.x;
    g_mask = h.inner | (h.imask << 8);
  }
  return best;
}

// Any hit over planes then the eight-wide tree (first hit wins).
template <int kStackSmem, int kBlock, bool kCount>
__device__ __forceinline__ bool any_hit8(const RtgSceneDev& sc, float3 o, float3 d, float tmin, float tmax,
                                         uint2* stack_base, TraceCount& cnt) {
  for (int i = 0; i < sc.n_planes; ++i) {
    float t;
    if (plane_test(sc.planes[i], o, d, tmin, tmax, t)) return true;
  }
  if (sc.root8 == INT32_MIN) return false;
  RayHit probe{tmax, kHitMiss, 0.f, 0.f};
  if (sc.root8 < 0) {
    for (int slot = ~sc.root8;; ++slot) {
      const std::uint32_t id = prim_slot_test(sc.prims, slot, o, d, tmin, probe);
      if (kCount) cnt.add_prim(id);
      if (probe.word != kHitMiss) return true;
      if (id & kLastInLeaf) return false;
    }
  }
  const Wide8Ray r(o, d);
  GroupStack<kStackSmem, kBlock> st(stack_base);
  std::uint32_t g_base = static_cast<std::uint32_t>(sc.root8), g_mask = (1u << r.oct) | (1u << 8);
  while (true) {
    if ((g_mask & 0xFFu) == 0u) {
      if (!st.pop(g_base, g_mask)) break;
      continue;
    }
    const std::uint32_t pos = static_cast<std::uint32_t>(__ffs(g_mask & 0xFFu) - 1);
    g_mask &= ~(1u << pos);
    const std::uint32_t slot = pos ^ r.oct;
    const std::uint32_t node = g_base + __popc((g_mask >> 8) & ((1u << slot) - 1u));
    if (g_mask & 0xFFu) st.push(g_base, g_mask);
    if (kCount) cnt.nodes++;
    const Node8Hits h = node8_hits(sc.nodes8 + node, r, tmin, tmax);
    for (std::uint32_t lh = h.leaves; lh; lh &= lh - 1u) {
      const std::uint32_t ls = static_cast<std::uint32_t>(__ffs(lh) - 1) ^ r.oct;
      for (int s = leaf8_first(h.b, ls);; ++s) {
        const std::uint32_t id = prim_slot_test(sc.prims, s, o, d, tmin, probe);
        if (kCount) cnt.add_prim(id);
        if (probe.word != kHitMiss) return true;
        if (id & kLastInLeaf) break;
      }
    }
    g_base = h.b.x;
    g_mask = h.inner | (h.imask << 8);
  }
  return false;
}

// Brute force over the scene's slots. Ties go to the lower primitive id, which
// reproduces the reference's index-order loop (src/core/scene.cpp:200-215).
template <bool kCount>
__device__ __forceinline__ RayHit closest_brute(const RtgSceneDev& sc, float3 o, float3 d, float tmin, float tmax,
                                                TraceCount& cnt) {
  RayHit best{tmax, kHitMiss, 0.f, 0.f};
  for (int i = 0; i < sc.n_planes; ++i) {
    float t;
    if (plane_test(sc.planes[i], o, d, tmin, best.t, t)) {
      best.t = t;
      best.word = kHitPlaneBit | static_cast<std::uint32_t>(i);
    }
  }
  std::uint32_t best_id = 0xFFFFFFFFu;
  const float plane_t = best.t;
  float tb = tmax < plane_t ? tmax : plane_t;
  bool have = false;
  for (int slot = sc.slot_begin; slot < sc.slot_end; ++slot) {
    const float4 p0 = __ldg(&sc.prims[3 * slot]);
    const float4 p1 = __ldg(&sc.prims[3 * slot + 1]);
    const std::uint32_t id = __float_as_uint(p0.w);
    if (kCount) cnt.add_prim(id);
    float t, b1 = 0.f, b2 = 0.f;
    bool hit;
    // Accept t == current best too, so a lower id can take over an exact tie.
    const float limit = have ? __int_as_float(__float_as_int(tb) + 1) : tb;
    const float4 p2 = __ldg(&sc.prims[3 * slot + 2]);
    if (id & kSphereBit) {
      hit = sphere_test(o, d, f3(p0), f3(p2), p1.x, tmin, limit, t);
    } else {
      hit = tri_test(o, d, f3(p0), f3(p1), f3(p2), p1.w, tmin, limit, t, b1, b2);
    }
    if (!hit) continue;
    const std::uint32_t pid = id & kIdMask;
    if (have && (t > tb || (t == tb && pid > best_id))) continue;
    have = true;
    tb = t;
    best_id = pid;
    best.t = t;
    best.word = static_cast<std::uint32_t>(slot);
    best.b1 = b1;
    best.b2 = b2;
  }
  return best;
}

// Recomputes the winning primitive's distance (and barycentrics) in double from
// its fp32 record, for the ray-query API: fp32 loses digits of t for near-tangent
// sphere and grazing triangle hits. Which primitive wins stays the fp32 decision.
__device__ __forceinline__ void refine_hit(const RtgSceneDev& sc, float3 of, float3 df, RayHit& h) {
  if (h.word == kHitMiss || !sc.prims64) return;
  const double ox = of.x, oy = of.y, oz = of.z, dx = df.x, dy = df.y, dz = df.z;
  double t = h.t, b1 = h.b1, b2 = h.b2;
  if (h.word & kHitPlaneBit) {
    const double* pl = sc.planes64 + 6 * (h.word & ~kHitPlaneBit);
    const double nx = pl[3], ny = pl[4], nz = pl[5];
    const double denom = nx * dx + ny * dy + nz * dz;
    t = ((pl[0] - ox) * nx + (pl[1] - oy) * ny + (pl[2] - oz) * nz) / denom;
  } else {
    const int slot = static_cast<int>(h.word);
    const double* g = sc.prims64 + 9 * slot;
    if (__float_as_uint(sc.prims[3 * slot].w) & kSphereBit) {
      const double r = g[3];
      const double ocx = g[0] - ox, ocy = g[1] - oy, ocz = g[2] - oz;
      const double a = dx * dx + dy * dy + dz * dz;
      const double hh = dx * ocx + dy * ocy + dz * ocz;
      const double cc = ocx * ocx + ocy * ocy + ocz * ocz - r * r;
      const double px = ocx - hh / a * dx, py = ocy - hh / a * dy, pz = ocz - hh / a * dz;
      const double disc = a * (r * r - (px * px + py * py + pz * pz));
      if (disc >= 0) {
        const double q = hh + copysign(sqrt(disc), hh);
        const double t0 = q != 0 ? cc / q : hh / a, t1 = q != 0 ? q / a : hh / a;
        t = fabs(t0 - h.t) < fabs(t1 - h.t) ? t0 : t1;  // the root the fp32 test chose
      }
    } else {
      const double e1x = g[3] - g[0], e1y = g[4] - g[1], e1z = g[5] - g[2];
      const double e2x = g[6] - g[0], e2y = g[7] - g[1], e2z = g[8] - g[2];
      const double pvx = dy * e2z - dz * e2y, pvy = dz * e2x - dx * e2z, pvz = dx * e2y - dy * e2x;
      const double det = e1x * pvx + e1y * pvy + e1z * pvz;
      const double tvx = ox - g[0], tvy = oy - g[1], tvz = oz - g[2];
      const double qvx = tvy * e1z - tvz * e1y, qvy = tvz * e1x - tvx * e1z, qvz = tvx * e1y - tvy * e1x;
      const double inv = 1.0 / det;
      b1 = (tvx * pvx + tvy * pvy + tvz * pvz) * inv;
      b2 = (dx * qvx + dy * qvy + dz * qvz) * inv;
      t = (e2x * qvx + e2y * qvy + e2z * qvz) * inv;
    }
  }
  if (isfinite(t) && fabs(t - h.t) <= 1e-3 * fabs(static_cast<double>(h.t))) {
    h.t = static_cast<float>(t);
    h.b1 = static_cast<float>(b1);
    h.b2 = static_cast<float>(b2);
  }
}

__device__ __forceinline__ bool any_brute(const RtgSceneDev& sc, float3 o, float3 d, float tmin, float tmax) {
  for (int i = 0; i < sc.n_planes; ++i) {
    float t;
    if (plane_test(sc.planes[i], o, d, tmin, tmax, t)) return true;
  }
  RayHit probe{tmax, kHitMiss, 0.f, 0.f};
  for (int slot = sc.slot_begin; slot < sc.slot_end; ++slot) {
    prim_slot_test(sc.prims, slot, o, d, tmin, probe);
    if (probe.word != kHitMiss) return true;
  }
  return false;
}

}  // namespace rtg
