#include "host/flatten.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <thread>

namespace rtg {

namespace {

std::uint32_t bits_of(float f) {
  std::uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
float float_of(std::uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// One float step toward -inf / +inf (std::nextafterf for finite f, by bits).
float step_down(float f) {
  if (f == 0.f) return -std::numeric_limits<float>::denorm_min();
  return float_of(f > 0.f ? bits_of(f) - 1u : bits_of(f) + 1u);
}
float step_up(float f) {
  if (f == 0.f) return std::numeric_limits<float>::denorm_min();
  return float_of(f > 0.f ? bits_of(f) + 1u : bits_of(f) - 1u);
}

// Round a double down / up to the nearest float, then widen by a few float ulps
// so the fp32 slab test (whose FMA form rounds once per plane) never culls a box
// that a primitive inside it would have been hit in.
float down(double v) {
  float f = static_cast<float>(v);
  if (static_cast<double>(f) > v) f = step_down(f);
  f -= std::fabs(f) * 0x1p-22f;
  return step_down(f);
}
float up(double v) {
  float f = static_cast<float>(v);
  if (static_cast<double>(f) < v) f = step_up(f);
  f += std::fabs(f) * 0x1p-22f;
  return step_up(f);
}

// Threads one flatten call may use (its max_threads argument; set for the call).
thread_local std::size_t t_flatten_threads = 16;

std::size_t flatten_threads() {
  return std::min<std::size_t>({std::max(1u, std::thread::hardware_concurrency()), 16, t_flatten_threads});
}

// Runs body(begin, end) over [0, n) in contiguous chunks on up to
// flatten_threads() threads (one chunk inline when n is small). Used for the
// per-slot and per-node loops, whose iterations write disjoint records.
template <class F>
void parallel_chunks(std::size_t n, F&& body) {
  const std::size_t workers = std::min<std::size_t>(flatten_threads(), (n + 8191) / 8192);
  if (workers <= 1) {
    body(std::size_t(0), n);
    return;
  }
  std::vector<std::thread> pool;
  const std::size_t chunk = (n + workers - 1) / workers;
  for (std::size_t w = 1; w < workers; ++w) {
    const std::size_t b = std::min(n, w * chunk), e = std::min(n, b + chunk);
    pool.emplace_back([&body, b, e] { body(b, e); });
  }
  body(std::size_t(0), std::min(n, chunk));
  for (auto& t : pool) t.join();
}

// A node box rounded outward to fp32 (lo down, hi up).
struct FBox {
  float lo[3], hi[3];
};
FBox outward(const Box& b) {
  return FBox{{down(b.lo.x), down(b.lo.y), down(b.lo.z)}, {up(b.hi.x), up(b.hi.y), up(b.hi.z)}};
}

float4 f4(D3 v, float w = 0.f) { return make_float4(float(v.x), float(v.y), float(v.z), w); }
float3 f3h(D3 v) { return make_float3(float(v.x), float(v.y), float(v.z)); }

DevMaterial material_record(const Material& m) {
  DevMaterial r{};
  if (const auto* l = std::get_if<Lambertian>(&m)) {
    r.head = make_float4(float_of(kLambertian), float(l->albedo.checker_scale), 0.f, 0.f);
    r.colour_a = f4(l->albedo.a);
    r.colour_b = f4(l->albedo.b);
  } else if (const auto* me = std::get_if<Metal>(&m)) {
    r.head = make_float4(float_of(kMetal), 0.f, float(me->roughness), 0.f);
    r.colour_a = f4(me->albedo);
  } else if (const auto* d = std::get_if<Dielectric>(&m)) {
    r.head = make_float4(float_of(kDielectric), 0.f, float(d->ior), 0.f);
    r.colour_a = f4(d->tint);
  } else {
    const auto& e = std::get<Emissive>(m);
    r.head = make_float4(float_of(kEmissive), 0.f, 0.f, e.two_sided ? 1.f : 0.f);
    r.colour_a = f4(e.color);
    r.emit = f4(e.color * e.intensity);
  }
  return r;
}

// Collapses the binary tree into four-child nodes: starting from an interior
// node's two children, the interior child with the largest surface area is
// replaced by its own children until there are four (or only leaves). Leaves
// keep their slot ranges. Four-wide nodes are numbered in the depth-first order
// of the binary nodes they start from, which the device build computes with a
// scan instead of a serial walk.
void build_wide(const BinaryBvh& bvh, const RecordVector<FBox>& fbox, FlatScene& f) {
  f.nodes4.clear();
  f.depth4 = 0;
  if (bvh.nodes.empty()) {
    f.root4 = kNoRoot;
    return;
  }
  if (bvh.nodes[0].leaf()) {
    f.root4 = ~static_cast<std::int32_t>(bvh.nodes[0].first);
    return;
  }
  // Topology first (indices only), then the boxes. A four-wide node's children
  // are recorded under the binary node it starts from, so numbering the starts
  // in binary (depth-first) order needs no sort, and disjoint subtrees can be
  // collapsed on different threads.
  struct Kids {
    std::uint32_t bin[4];
    int n;  // 0: this binary node starts no four-wide node
  };
  std::vector<Kids> kids_of(bvh.nodes.size());
  // The four-wide node starting at binary node `bin`; push(c) gets each interior
  // child, which starts a four-wide node of its own.
  auto expand = [&](std::uint32_t bin, auto&& push) {
    Kids k{};
    k.bin[k.n++] = bin + 1;
    k.bin[k.n++] = bvh.nodes[bin].first;
    while (k.n < 4) {
      int pick = -1;
      double pick_area = -1;
      for (int q = 0; q < k.n; ++q) {
        const BinaryNode& c = bvh.nodes[k.bin[q]];
        if (c.leaf()) continue;
        const double a = c.box.area();
        if (a > pick_area) {
          pick_area = a;
          pick = q;
        }
      }
      if (pick < 0) break;
      const std::uint32_t b = k.bin[pick];
      k.bin[pick] = b + 1;
      k.bin[k.n++] = bvh.nodes[b].first;
    }
    for (int q = 0; q < k.n; ++q)
      if (!bvh.nodes[k.bin[q]].leaf()) push(k.bin[q]);
    kids_of[bin] = k;
  };
  // Breadth first from the root until about 256 subtrees are open, then each of
  // those depth first as its own task.
  std::vector<std::pair<std::uint32_t, int>> open{{0u, 1}};
  std::size_t head = 0;
  int depth4 = 0;
  while (head < open.size() && open.size() - head < 256) {
    const auto [bin, depth] = open[head++];
    depth4 = std::max(depth4, depth);
    expand(bin, [&, depth = depth](std::uint32_t c) { open.push_back({c, depth + 1}); });
  }
  std::atomic<std::size_t> next_task{head};
  std::mutex depth_lock;
  auto subtrees = [&] {
    int deepest = 0;
    std::vector<std::pair<std::uint32_t, int>> work;
    for (std::size_t t; (t = next_task.fetch_add(1)) < open.size();) {
      work.assign(1, open[t]);
      while (!work.empty()) {
        const auto [bin, depth] = work.back();
        work.pop_back();
        deepest = std::max(deepest, depth);
        expand(bin, [&, depth = depth](std::uint32_t c) { work.push_back({c, depth + 1}); });
      }
    }
    std::lock_guard<std::mutex> g(depth_lock);
    depth4 = std::max(depth4, deepest);
  };
  const std::size_t tasks = open.size() - head;
  const std::size_t workers = std::min<std::size_t>(flatten_threads(), (tasks + 15) / 16);
  std::vector<std::thread> pool;
  for (std::size_t w = 1; w < workers; ++w) pool.emplace_back(subtrees);
  subtrees();
  for (auto& t : pool) t.join();
  f.depth4 = depth4;
  std::vector<std::int32_t> wide_index(bvh.nodes.size(), -1);
  std::vector<std::uint32_t> start;  // four-wide node i starts from binary node start[i]
  for (std::size_t b = 0; b < bvh.nodes.size(); ++b)
    if (kids_of[b].n) {
      wide_index[b] = static_cast<std::int32_t>(start.size());
      start.push_back(static_cast<std::uint32_t>(b));
    }
  f.nodes4.resize(start.size());
  parallel_chunks(start.size(), [&](std::size_t i0, std::size_t i1) {
    for (std::size_t i = i0; i < i1; ++i) {
      const Kids& k = kids_of[start[i]];
      float lo[3][4], hi[3][4];
      std::int32_t link[4];
      for (int q = 0; q < 4; ++q) {
        if (q >= k.n) {
          for (int a = 0; a < 3; ++a) lo[a][q] = hi[a][q] = 0.f;
          link[q] = kNoChild;
          continue;
        }
        const FBox& b = fbox[k.bin[q]];
        for (int a = 0; a < 3; ++a) {
          lo[a][q] = b.lo[a];
          hi[a][q] = b.hi[a];
        }
        const BinaryNode& c = bvh.nodes[k.bin[q]];
        link[q] = c.leaf() ? ~static_cast<std::int32_t>(c.first) : wide_index[k.bin[q]];
      }
      DevNode4& d = f.nodes4[i];
      d.lo_x = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
      d.hi_x = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
      d.lo_y = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
      d.hi_y = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
      d.lo_z = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
      d.hi_z = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
      d.link = make_int4(link[0], link[1], link[2], link[3]);
      d.pad = make_int4(0, 0, 0, 0);
    }
  });
  f.root4 = 0;
  if (3 * f.depth4 + 1 > kWideStackDepth)
    throw std::runtime_error("BVH deeper than the traversal stack allows");
}

}  // namespace

void slot_record(const Prim& p, std::uint32_t id, float4* rows, float4* normals, std::uint32_t& material) {
  std::uint32_t word = id;
  normals[0] = normals[1] = normals[2] = make_float4(0.f, 0.f, 0.f, 0.f);
  // What rounding the position to fp32 lost, kept so the distance can be
  // corrected where it is computed (the stored fp32 values are as before).
  const D3 a32{double(float(p.a.x)), double(float(p.a.y)), double(float(p.a.z))};
  const D3 residual = p.a - a32;
  if (p.kind == Prim::kSphere) {
    word |= kSphereBit;
    rows[0] = f4(p.a, float_of(word));
    rows[1] = make_float4(float(p.b.x), float(p.b.x * p.b.x), 0.f, 0.f);
    rows[2] = f4(residual);
  } else {
    // The triangle's plane offset that v0's rounding lost: t gains
    // -dot(residual, e1 x e2) / det, with the edges as stored.
    const float4 e1 = f4(p.b - p.a), e2 = f4(p.c - p.a);
    const D3 n = cross(D3{e1.x, e1.y, e1.z}, D3{e2.x, e2.y, e2.z});
    rows[0] = f4(p.a, float_of(word));
    rows[1] = make_float4(e1.x, e1.y, e1.z, float(dot(residual, n)));
    rows[2] = e2;
    if (p.smooth) {
      normals[0] = f4(p.n0);
      normals[1] = f4(p.n1);
      normals[2] = f4(p.n2);
    }
  }
  material = p.material | ((p.kind == Prim::kTriangle && p.smooth) ? 0x80000000u : 0u);
}

void flatten_tables(const CompiledScene& s, FlatScene& f) {
  f.planes.clear();
  f.materials.clear();
  f.lights.clear();
  for (const PlanePrim& pl : s.planes) {
    DevPlane dp;
    dp.point = f4(pl.point, float_of(pl.material));
    dp.normal = f4(pl.normal);
    // The plane offset its point's rounding lost, along the stored normal.
    const D3 p32{double(float(pl.point.x)), double(float(pl.point.y)), double(float(pl.point.z))};
    dp.normal.w = float(dot(pl.point - p32, D3{dp.normal.x, dp.normal.y, dp.normal.z}));
    f.planes.push_back(dp);
  }
  for (const Material& m : s.materials) f.materials.push_back(material_record(m));

  for (const LightEntry& le : s.lights) {
    DevLight L{};
    if (le.kind == LightEntry::kPoint) {
      const PointLight& pl = s.point_lights[le.index];
      L.q0 = f4(pl.position, float_of(kLightPoint));
      L.q1 = f4(pl.intensity);
    } else {
      const Prim& p = s.prims[le.index];
      const Material& m = s.materials[p.material];
      const auto& e = std::get<Emissive>(m);
      const D3 emit = e.color * e.intensity;
      if (p.kind == Prim::kSphere) {
        L.q0 = f4(p.a, float_of(kLightSphere));
        L.q1 = make_float4(float(p.b.x), float(p.b.x * p.b.x), float(p.area()), e.two_sided ? 1.f : 0.f);
        L.q2 = f4(emit);
      } else {
        L.q0 = f4(p.a, float_of(kLightTriangle));
        L.q1 = f4(p.b, float(p.area()));
        L.q2 = f4(p.c, e.two_sided ? 1.f : 0.f);
        L.q3 = f4(unit(cross(p.b - p.a, p.c - p.a)));
        L.q4 = f4(emit);
      }
    }
    f.lights.push_back(L);
  }
}

FlatScene flatten(const CompiledScene& s, bool wide8, unsigned max_threads) {
  struct Cap {
    std::size_t old = t_flatten_threads;
    explicit Cap(unsigned n) { t_flatten_threads = n ? n : 16; }
    ~Cap() { t_flatten_threads = old; }
  } cap(max_threads);
  FlatScene f;
  const BinaryBvh& bvh = s.bvh;

  // Primitive slots in leaf order; mark the last slot of every leaf.
  const std::size_t nslots = bvh.order.size();
  if (s.prims.size() > kIdMask) throw std::runtime_error("too many primitives for the device layout");
  std::vector<std::uint8_t> last(nslots, 0);
  for (const BinaryNode& n : bvh.nodes)
    if (n.leaf()) last[n.first + n.count - 1] = 1;
  f.prims.resize(nslots * 3);  // every slot_record writes all three rows and normals
  f.slot_material.resize(nslots);
  f.slot_normals.resize(nslots * 3);
  f.slot_prim.resize(nslots);
  parallel_chunks(nslots, [&](std::size_t k0, std::size_t k1) {
    for (std::size_t k = k0; k < k1; ++k) {
      const std::uint32_t id = bvh.order[k];
      slot_record(s.prims[id], id, &f.prims[3 * k], &f.slot_normals[3 * k], f.slot_material[k]);
      if (last[k]) f.prims[3 * k].w = float_of(bits_of(f.prims[3 * k].w) | kLastInLeaf);
      f.slot_prim[k] = id;
    }
  });

  // Interior nodes in depth-first order -> DevNode indices.
  std::vector<std::int32_t> dev_index(bvh.nodes.size(), -1);
  std::int32_t ninterior = 0;
  for (std::size_t i = 0; i < bvh.nodes.size(); ++i)
    if (!bvh.nodes[i].leaf()) dev_index[i] = ninterior++;
  auto link_of = [&](std::size_t child) -> std::int32_t {
    const BinaryNode& c = bvh.nodes[child];
    return c.leaf() ? ~static_cast<std::int32_t>(c.first) : dev_index[child];
  };
  // Every node's box rounded outward once; both device trees copy from here.
  RecordVector<FBox> fbox(bvh.nodes.size());  // every entry written below
  parallel_chunks(bvh.nodes.size(), [&](std::size_t i0, std::size_t i1) {
    for (std::size_t i = i0; i < i1; ++i) fbox[i] = outward(bvh.nodes[i].box);
  });
  f.nodes.resize(static_cast<std::size_t>(ninterior));
  parallel_chunks(bvh.nodes.size(), [&](std::size_t i0, std::size_t i1) {
  for (std::size_t i = i0; i < i1; ++i) {
    const BinaryNode& n = bvh.nodes[i];
    if (n.leaf()) continue;
    const FBox& L = fbox[i + 1];
    const FBox& R = fbox[n.first];
    DevNode& d = f.nodes[static_cast<std::size_t>(dev_index[i])];
    d.xy0 = make_float4(L.lo[0], L.hi[0], L.lo[1], L.hi[1]);
    d.xy1 = make_float4(R.lo[0], R.hi[0], R.lo[1], R.hi[1]);
    d.zz = make_float4(L.lo[2], L.hi[2], R.lo[2], R.hi[2]);
    d.link = make_int4(link_of(i + 1), link_of(n.first), static_cast<int>(n.axis) << 16, 0);
  }
  });
  if (!bvh.nodes.empty()) f.root = link_of(0);
  build_wide(bvh, fbox, f);
  if (wide8) add_wide8(f);

  flatten_tables(s, f);
  return f;
}

void add_wide8(FlatScene& f) {
  const std::size_t nslots = f.slot_prim.size();
  std::vector<std::uint8_t> last(nslots);
  for (std::size_t k = 0; k < nslots; ++k) last[k] = (bits_of(f.prims[3 * k].w) & kLastInLeaf) ? 1 : 0;
  Wide8 w = build_wide8(f.nodes.data(), f.nodes.size(), f.root, last.data(), nslots);
  f.nodes8 = std::move(w.nodes);
  f.root8 = w.root;
  bool identity = true;
  for (std::size_t k = 0; k < nslots && identity; ++k) identity = w.old_of[k] == k;
  if (identity) return;
  RecordVector<float4> prims(f.prims.size()), normals(f.slot_normals.size());
  std::vector<std::uint32_t> material(nslots), prim(nslots);
  parallel_chunks(nslots, [&](std::size_t k0, std::size_t k1) {
    for (std::size_t k = k0; k < k1; ++k) {
      const std::size_t o = w.old_of[k];
      for (int r = 0; r < 3; ++r) {
        prims[3 * k + r] = f.prims[3 * o + r];
        normals[3 * k + r] = f.slot_normals[3 * o + r];
      }
      material[k] = f.slot_material[o];
      prim[k] = f.slot_prim[o];
    }
  });
  f.prims = std::move(prims);
  f.slot_normals = std::move(normals);
  f.slot_material = std::move(material);
  f.slot_prim = std::move(prim);
  for (DevNode& n : f.nodes) {
    n.link.x = remap_link(n.link.x, w.new_of);
    n.link.y = remap_link(n.link.y, w.new_of);
  }
  for (DevNode4& n : f.nodes4) {
    n.link.x = remap_link(n.link.x, w.new_of);
    n.link.y = remap_link(n.link.y, w.new_of);
    n.link.z = remap_link(n.link.z, w.new_of);
    n.link.w = remap_link(n.link.w, w.new_of);
  }
  f.root = remap_link(f.root, w.new_of);
  f.root4 = remap_link(f.root4, w.new_of);
}

void describe(const CompiledScene& s, const RenderSettings& r, RtgSceneDev& d) {
  CameraFrame c;
  c.setup(s.camera_desc, r.width, r.height);
  d.cam_origin = f3h(c.origin);
  d.cam_corner = f3h(c.corner);
  d.cam_du = f3h(c.du);
  d.cam_dv = f3h(c.dv);
  d.cam_u = f3h(c.u);
  d.cam_v = f3h(c.v);
  d.lens_radius = float(c.lens_radius);
  d.width = r.width;
  d.height = r.height;
  d.max_depth = r.max_depth;
  d.rr_min_depth = r.rr_min_depth;
  d.integrator = static_cast<std::int32_t>(r.integrator);
  d.light_sampling = r.light_sampling ? (r.mis ? 2 : 1) : 0;
  d.use_bvh = r.use_bvh ? 1 : 0;
  d.seed = r.seed;
  d.bg_top = f3h(s.background.top);
  d.bg_bottom = f3h(s.background.bottom);
  d.bg_intensity = float(s.background.intensity);
  d.bg_solid = s.background.kind == Background::Kind::Solid ? 1 : 0;
}

}  // namespace rtg
