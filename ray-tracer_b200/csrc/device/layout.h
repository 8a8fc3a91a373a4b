#pragma once
// Device-resident scene and wavefront layouts (fp32), shared by the host
// flattener and the sm_100a kernels. Every array is a run of 16-byte aligned
// float4/uint4 records so a warp's loads coalesce into full sectors and each
// record is one vectorised load.
//
// Geometry pools can hold many scenes back to back (batched and served modes):
// node links and primitive slots are absolute indices into the pools, so a scene
// is just a root node plus per-scene tables in RtgSceneDev.
#include <cstdint>

#if defined(__CUDACC__)
#include <cuda_runtime.h>
#else
#include <vector_functions.h>
#include <vector_types.h>
#endif

namespace rtg {

// Two-child BVH node: both children's boxes are stored in the parent so one
// 64-byte fetch tests two boxes. Child link >= 0: interior node index; < 0: leaf
// whose primitives are the slots ~link, ~link + 1, ... up to the first slot that
// carries kLastInLeaf.
struct alignas(16) DevNode {
  float4 xy0;   // child 0: lo.x, hi.x, lo.y, hi.y
  float4 xy1;   // child 1: lo.x, hi.x, lo.y, hi.y
  float4 zz;    // child 0: lo.z, hi.z; child 1: lo.z, hi.z
  int4 link;    // x: child 0 link, y: child 1 link, z: split axis << 16, w: unused
};

// Four-child BVH node, collapsed from the binary tree (same leaves): the four
// children's boxes as SoA float4s (component k is child k), then their links with
// the same meaning as DevNode's; an unused child has kNoChild. One 128-byte node
// replaces up to three binary nodes. Any-hit (shadow) queries walk this tree: they
// stop at the first hit, so a wide node's four tests pay off; closest-hit queries
// walk the binary tree, which measured faster for them.
struct alignas(16) DevNode4 {
  float4 lo_x, hi_x, lo_y, hi_y, lo_z, hi_z;
  int4 link;
  int4 pad;
};
constexpr std::int32_t kNoChild = INT32_MIN;

// Compressed eight-child BVH node, 80 bytes (after Ylitie, Karras and Laine,
// "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs",
// HPG 2017), collapsed from the binary tree with the same leaves. Child boxes
// are stored as 8-bit offsets from the node origin `p` in units of a power of two
// per axis, rounded outward, so a decoded box always encloses the child's fp32
// box. An unused child has lo = 255, hi = 0 on every axis (never hit).
//  a: p.x, p.y, p.z; w bits: e_x | e_y << 8 | e_z << 16 | imask << 24, where e is a
//     biased float exponent (scale = 2^(e - 127)) and imask bit s marks child
//     slot s as an interior node
//  b: x = child_base (first interior child; interior children are stored
//     contiguously in slot order), y = prim_base (first primitive slot of the
//     leaf children), z/w = meta bytes 0-3 / 4-7: for an interior child its index
//     among the interior children, for a leaf child the offset of its first slot
//     from prim_base (the leaf runs to the slot carrying kLastInLeaf)
//  qlo_xy: x, y = lo.x bytes of children 0-3, 4-7; z, w = lo.y bytes
//  qlo_z_hi_x: x, y = lo.z bytes; z, w = hi.x bytes
//  qhi_yz: x, y = hi.y bytes; z, w = hi.z bytes
// Child slots are assigned by the direction of each child's centre from the
// node's centre (slot bit k set: positive along axis k), so a ray visiting slots
// in the order s ^ octant meets the children roughly front to back.
struct alignas(16) DevNode8 {
  float4 a;
  uint4 b;
  uint4 qlo_xy;
  uint4 qlo_z_hi_x;
  uint4 qhi_yz;
};
static_assert(sizeof(DevNode8) == 80, "DevNode8 must be 80 bytes");
// Leaf children of one node start within this many slots of its prim_base.
constexpr int kWide8MaxLeafOffset = 255;
// Traversal stack entries an eight-wide walk may need (one group per level; the
// builder rejects deeper trees).
constexpr int kWide8StackDepth = 64;
// Traversal stack entries a 4-wide walk may need: 3 per level (the binary tree's
// depth cap of 60 bounds the four-wide depth) plus the current one.
constexpr int kWideStackDepth = 3 * 61 + 1;

// Primitive slot (leaf order): three float4.
//  triangle: p0 = (v0, id), p1 = (e1 = v1 - v0, k), p2 = (e2 = v2 - v0, 0), where
//            k = dot(v0 - fp32(v0), e1 x e2) in double: the plane offset the
//            rounding of v0 lost (the distance test subtracts it)
//  sphere:   p0 = (centre, id | kSphereBit), p1 = (radius, radius^2, 0, 0),
//            p2 = (centre - fp32(centre), 0): the rounding residual of the centre
// `id` is the scene-local primitive id (the reference's hit id), stored as bits.
constexpr std::uint32_t kSphereBit = 0x80000000u;
constexpr std::uint32_t kLastInLeaf = 0x40000000u;  // set on the last primitive slot of a leaf
constexpr std::uint32_t kIdMask = 0x3FFFFFFFu;

// Hit word written by the closest-hit kernel (float4.y as bits):
constexpr std::uint32_t kHitMiss = 0xFFFFFFFFu;
constexpr std::uint32_t kHitPlaneBit = 0x40000000u;  // low bits = plane index within the scene
// Otherwise the word is the primitive slot (absolute, < 2^30).

enum DevMaterialKind : std::uint32_t { kLambertian = 0, kMetal = 1, kDielectric = 2, kEmissive = 3 };

struct alignas(16) DevMaterial {
  float4 head;      // x: kind (bits), y: checker scale, z: roughness | ior, w: two-sided (0/1)
  float4 colour_a;  // lambertian albedo a | metal albedo | dielectric tint | emissive colour
  float4 colour_b;  // lambertian albedo b (checker)
  float4 emit;      // emitted radiance colour * intensity (0 unless emissive)
};

enum DevLightKind : std::uint32_t { kLightPoint = 0, kLightSphere = 1, kLightTriangle = 2 };

struct alignas(16) DevLight {
  float4 q0;  // point: (position, kind); sphere: (centre, kind); triangle: (v0, kind)
  float4 q1;  // point: (intensity, 0);   sphere: (r, r^2, area, two_sided); triangle: (v1, area)
  float4 q2;  // sphere: (emission, 0);   triangle: (v2, two_sided)
  float4 q3;  // triangle: (unit normal, 0)
  float4 q4;  // triangle: (emission, 0)
};

struct alignas(16) DevPlane {
  float4 point;   // xyz, w = material index (bits)
  float4 normal;  // unit xyz, w = dot(point - fp32(point), normal): the offset rounding the point lost
};

// One scene as the kernels see it. Pointers are device addresses.
struct alignas(16) RtgSceneDev {
  const DevNode* nodes;
  const float4* prims;        // 3 per slot
  const std::uint32_t* slot_material;  // per slot: material index | smooth flag << 31
  const float4* slot_normals; // 3 per slot (n0, n1, n2); only read for smooth triangles
  const DevPlane* planes;
  const DevMaterial* materials;
  const DevLight* lights;
  std::int32_t root;          // >= 0: node; < 0: ~slot of a root leaf; INT32_MIN: no bounded primitives
  std::int32_t n_planes;
  std::int32_t n_lights;
  std::int32_t slot_begin;    // this scene's slots are [slot_begin, slot_end)
  std::int32_t slot_end;
  // camera
  float3 cam_origin, cam_corner, cam_du, cam_dv, cam_u, cam_v;
  float lens_radius;
  // settings
  std::int32_t width, height, max_depth, rr_min_depth;
  std::int32_t integrator;    // 0 path, 1 direct, 2 normals
  std::int32_t light_sampling;  // 0 off, 1 NEE, 2 NEE with MIS
  std::int32_t use_bvh;
  std::uint32_t pad0;
  std::uint64_t seed;
  // background
  float3 bg_top, bg_bottom;
  float bg_intensity;
  std::int32_t bg_solid;
  // framebuffer of the render this descriptor belongs to (per pixel)
  double* fb_sum;             // 4 doubles per pixel: running sum r, g, b, (unused)
  double* fb_sumsq;           // 4 doubles per pixel: running sum of squares
  std::uint32_t* fb_count;    // samples accumulated per pixel
  std::uint64_t* stats;       // [0] invalid samples
  // Double-precision originals for the ray-query API's distance refinement
  // (null unless that API has been used on the scene): per slot 9 doubles
  // (sphere: centre, radius; triangle: v0, v1, v2); per plane 6 (point, normal).
  const double* prims64;
  const double* planes64;
  // 4-wide copy of the same tree (any-hit queries).
  const DevNode4* nodes4;
  std::int32_t root4;         // as root, for nodes4
  std::int32_t root8;         // as root, for nodes8
  // Compressed 8-wide copy of the same tree (closest-hit queries).
  const DevNode8* nodes8;
};

// A segment is one pass of one render: samples [pass_s0, pass_s0 + pass_spp) of every
// pixel of a job. The continuous wavefront schedules segments; the host appends
// them (and new jobs) between iterations, so passes and requests overlap.
struct alignas(16) DevSegment {
  std::uint32_t job;          // descriptor index
  std::uint32_t pass_s0;      // first sample index of the pass
  std::uint32_t pass_spp;     // samples per pixel in this pass
  std::uint32_t pad;
  std::uint64_t count;        // pixels * pass_spp camera samples
  std::uint64_t sample_base;  // radiance slot of (pixel 0, sample pass_s0); sample s of pixel p
                              // is at sample_base + p * pass_spp + (s - pass_s0)
};

// Device-side progress of one segment slot (zeroed when the slot is assigned).
struct alignas(16) SegmentProgress {
  std::uint64_t generated;    // camera samples handed to the wavefront
  std::uint32_t done;         // samples whose path (and last shadow ray) finished
  std::uint32_t pad;
};

constexpr int kMaxSegments = 4096;  // segment slots (the path record carries the slot)
constexpr int kMaxGen = 256;        // segments open for generation at once

// Generation order written by the host between iterations: segment slots in
// priority order. The plan kernel hands free pool slots to them greedily.
struct alignas(16) GenTable {
  std::uint32_t n;
  std::uint32_t snapshot_slots;  // segment slots [0, this) copied into each snapshot
  std::uint32_t pad[2];
  std::uint32_t slot[kMaxGen];
};

// Where this iteration's new paths come from (written by the plan kernel):
// new path j belongs to the first entry k with end[k] > j, and is local sample
// start[k] + j - end[k - 1] of segment seg[k].
struct alignas(16) GenPlan {
  std::uint32_t n;
  std::uint32_t n_new;
  std::uint32_t pad[2];
  std::uint32_t end[kMaxGen];
  std::uint32_t seg[kMaxGen];
  std::uint64_t start[kMaxGen];
};

// Path-state stream record, four float4 (SoA): one element per live path.
//  a = (origin, sample id bits)         b = (direction, meta bits)
//  c = (throughput, segment slot bits)  d = PCG32 state (lo, hi) and increment (lo, hi)
// meta: depth (bits 0-11) | flags (bits 12-15) | job (bits 16-31)
constexpr std::uint32_t kFlagSpecular = 1u << 12;
constexpr std::uint32_t kMetaDepthMask = 0xFFFu;
constexpr int kMetaSceneShift = 16;
constexpr int kMaxJobs = 65536;  // job descriptors addressable from the path record

// Wavefront counters in device memory.
struct alignas(16) WaveCounters {
  std::uint32_t live[2];      // live paths at the start of an iteration (parity)
  std::uint32_t n_extend;     // paths traced this iteration (live + new)
  std::uint32_t n_shadow;     // shadow rays queued this iteration
  std::uint32_t fetch[4];     // persistent-kernel work-fetch cursors
  std::uint64_t iteration;    // plan launches so far (selects the snapshot ring slot)
  std::uint64_t generated;    // camera samples generated so far
  std::uint64_t rays;         // closest-hit rays traced
  std::uint64_t shadow_rays;
  std::uint64_t rr_terminated;
  std::uint64_t invalid_samples;
  std::uint64_t node_visits;  // closest-hit kernel; filled only by the counting kernel variants
  std::uint64_t prim_tests;
  std::uint64_t sphere_tests; // of which spheres (32-byte reads; triangles read 48)
  std::uint64_t shadow_node_visits;  // any-hit kernel, same meaning
  std::uint64_t shadow_prim_tests;
  std::uint64_t shadow_sphere_tests;
  std::uint32_t error;        // non-zero: a bounds check failed (index recorded in error_info)
  std::uint32_t error_info;
};

// What the plan kernel copies to pinned host memory at the start of each
// iteration: the counters and segment progress as the previous iteration left them.
struct alignas(16) WaveSnapshot {
  WaveCounters c;
  SegmentProgress seg[kMaxSegments];
};

}  // namespace rtg
