#include "host/compiled_scene.hpp"

#include <algorithm>
#include <array>
#include <filesystem>
#include <stdexcept>
#include <thread>

#include "host/mesh.hpp"

namespace rtg {

Box Prim::bounds() const {
  Box out;
  if (kind == kSphere) {
    const D3 r{std::fabs(b.x)};
    out.lo = a - r;
    out.hi = a + r;
    return out;
  }
  out.grow(a);
  out.grow(b);
  out.grow(c);
  // Flat (axis-aligned) triangles get a little thickness so no slab is empty.
  const D3 pad{1e-9};
  out.lo = out.lo - pad;
  out.hi = out.hi + pad;
  return out;
}

double Prim::area() const {
  if (kind == kSphere) return 4 * kPi * b.x * b.x;
  return 0.5 * len(cross(b - a, c - a));
}

void CameraFrame::setup(const CameraDesc& d, int width, int height) {
  const double aspect = double(width) / double(height);
  origin = d.look_from;
  const D3 view = d.look_at - d.look_from;
  w = unit_or(-view, D3{0, 0, 1});
  D3 up = unit_or(d.vup, D3{0, 1, 0});
  // A view direction parallel to vup needs another up vector.
  if (std::fabs(dot(up, w)) > 0.999999) up = std::fabs(w.y) < 0.9 ? D3{0, 1, 0} : D3{0, 0, 1};
  u = unit(cross(up, w));
  v = cross(w, u);
  const double focus = d.focus_dist > 0 ? d.focus_dist : std::fmax(len(view), 1e-3);
  const double theta = std::clamp(d.vfov_deg, 0.1, 179.0) * kPi / 180;
  const double half_h = std::tan(theta / 2);
  const double vp_h = 2 * half_h * focus;
  const double vp_w = vp_h * aspect;
  const D3 span_u = vp_w * u;
  const D3 span_v = -vp_h * v;  // rows go down the image
  du = span_u / double(width);
  dv = span_v / double(height);
  corner = origin - focus * w - span_u / 2 - span_v / 2;
  lens_radius = d.aperture / 2;
}

namespace {

constexpr double kMinTriangleArea = 1e-14;  // smaller triangles are dropped as degenerate

// Runs body(begin, end) over [0, n) in contiguous chunks on the host cores, with
// at least `grain` items per worker.
template <class F>
void parallel_for(std::size_t n, F&& body, std::size_t grain = 1024) {
  const std::size_t workers = std::min<std::size_t>({16, std::max(1u, std::thread::hardware_concurrency()),
                                                     (n + grain - 1) / grain});
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

}  // namespace

CompiledScene compile_scene(const SceneDesc& desc, BvhBuild where) {
  CompiledScene s;
  s.settings = desc.render;
  s.background = desc.background;
  s.camera_desc = desc.camera;
  s.camera.setup(desc.camera, desc.render.width, desc.render.height);
  for (const auto& m : desc.materials) s.materials.push_back(m.material);

  auto material_index = [&](const std::string& name) -> std::uint32_t {
    for (std::size_t i = 0; i < desc.materials.size(); ++i)
      if (desc.materials[i].name == name) return static_cast<std::uint32_t>(i);
    throw std::runtime_error("unknown material '" + name + "'");
  };

  auto add_tri = [&](const Prim& t) {
    if (t.area() < kMinTriangleArea) {  // degenerate: cannot be hit reliably
      s.info.degenerate_skipped++;
      return;
    }
    s.prims.push_back(t);
    s.info.triangles++;
  };
  auto flat_tri = [](D3 v0, D3 v1, D3 v2, std::uint32_t mat) {
    Prim t;
    t.kind = Prim::kTriangle;
    t.a = v0; t.b = v1; t.c = v2;
    t.material = mat;
    return t;
  };

  for (const ObjectDesc& obj : desc.objects) {
    const std::uint32_t mat = material_index(obj.material);
    if (const auto* sp = std::get_if<SphereDesc>(&obj.shape)) {
      Prim p;
      p.kind = Prim::kSphere;
      p.a = sp->center;
      p.b = D3{sp->radius, 0, 0};
      p.material = mat;
      s.prims.push_back(p);
      s.info.spheres++;
    } else if (const auto* pl = std::get_if<PlaneDesc>(&obj.shape)) {
      s.planes.push_back({pl->point, unit_or(pl->normal, D3{0, 1, 0}), mat});
      s.info.planes++;
    } else if (const auto* t = std::get_if<TriangleDesc>(&obj.shape)) {
      add_tri(flat_tri(t->v0, t->v1, t->v2, mat));
    } else if (const auto* q = std::get_if<QuadDesc>(&obj.shape)) {
      const D3 o = q->corner;
      add_tri(flat_tri(o, o + q->u, o + q->u + q->v, mat));
      add_tri(flat_tri(o, o + q->u + q->v, o + q->v, mat));
    } else if (const auto* bx = std::get_if<BoxDesc>(&obj.shape)) {
      const D3 mid = 0.5 * (bx->min + bx->max);
      const Placement place{{1, 1, 1}, bx->rotate_y, mid};
      const D3 half = 0.5 * (bx->max - bx->min);
      auto corner = [&](double sx, double sy, double sz) { return place.point(D3{sx * half.x, sy * half.y, sz * half.z}); };
      // Corners indexed by bits (x, y, z) in the order below; each face lists
      // its corners counter-clockwise from outside, split into two triangles.
      const D3 k[8] = {corner(-1, -1, -1), corner(1, -1, -1), corner(1, 1, -1), corner(-1, 1, -1),
                       corner(-1, -1, 1),  corner(1, -1, 1),  corner(1, 1, 1),  corner(-1, 1, 1)};
      static const int kFaces[6][4] = {{4, 5, 6, 7}, {1, 0, 3, 2}, {5, 1, 2, 6},
                                       {0, 4, 7, 3}, {7, 6, 2, 3}, {0, 1, 5, 4}};
      for (const auto& f : kFaces) {
        add_tri(flat_tri(k[f[0]], k[f[1]], k[f[2]], mat));
        add_tri(flat_tri(k[f[0]], k[f[2]], k[f[3]], mat));
      }
    } else {
      const auto& md = std::get<MeshDesc>(obj.shape);
      IndexedMesh mesh;
      if (md.source == MeshDesc::Source::Icosphere) {
        mesh = icosphere(md.subdivisions);
      } else if (md.source == MeshDesc::Source::Torus) {
        const int sv = md.segments_v > 0 ? md.segments_v : std::max(3, md.segments / 2);
        mesh = torus(md.major_radius, md.minor_radius, md.segments, sv);
      } else {
        std::filesystem::path p(md.path);
        if (p.is_relative() && !desc.base_dir.empty()) p = std::filesystem::path(desc.base_dir) / p;
        mesh = load_obj_file(p.string());
      }
      if (md.smooth && mesh.normals.empty()) mesh.smooth_normals();
      const Placement place{md.scale, md.rotate_y, md.translate};
      const bool smooth = md.smooth && !mesh.normals.empty();
      // Every vertex is placed once (the same arithmetic the per-corner placement
      // does), then the faces are filled on all host cores: each chunk counts its
      // non-degenerate faces, and writes them at its offset, in face order.
      std::vector<D3> pos(mesh.positions.size()), nrm(smooth ? mesh.normals.size() : 0);
      parallel_for(pos.size(), [&](std::size_t i0, std::size_t i1) {
        for (std::size_t i = i0; i < i1; ++i) pos[i] = place.point(mesh.positions[i]);
        for (std::size_t i = i0; i < std::min(i1, nrm.size()); ++i) nrm[i] = place.normal(mesh.normals[i]);
      });
      auto face_prim = [&](const std::array<std::uint32_t, 3>& f) {
        Prim t = flat_tri(pos[f[0]], pos[f[1]], pos[f[2]], mat);
        if (smooth) {
          t.n0 = nrm[f[0]];
          t.n1 = nrm[f[1]];
          t.n2 = nrm[f[2]];
          t.smooth = true;
        }
        return t;
      };
      const std::size_t nf = mesh.faces.size();
      const std::size_t chunks = std::min<std::size_t>(64, (nf + 4095) / 4096);
      std::vector<std::size_t> kept(chunks + 1, 0);
      std::vector<std::uint8_t> keep(nf);
      auto chunk_range = [&](std::size_t c) { return std::pair{nf * c / chunks, nf * (c + 1) / chunks}; };
      parallel_for(chunks, [&](std::size_t c0, std::size_t c1) {
        for (std::size_t c = c0; c < c1; ++c) {
          const auto [f0, f1] = chunk_range(c);
          for (std::size_t i = f0; i < f1; ++i) {
            // Prim::area() of the face, from the placed vertices.
            const auto& f = mesh.faces[i];
            keep[i] = 0.5 * len(cross(pos[f[1]] - pos[f[0]], pos[f[2]] - pos[f[0]])) >= kMinTriangleArea;
            kept[c + 1] += keep[i];
          }
        }
      }, 1);
      for (std::size_t c = 0; c < chunks; ++c) kept[c + 1] += kept[c];
      const std::size_t base = s.prims.size();
      s.prims.resize(base + kept[chunks]);
      parallel_for(chunks, [&](std::size_t c0, std::size_t c1) {
        for (std::size_t c = c0; c < c1; ++c) {
          const auto [f0, f1] = chunk_range(c);
          std::size_t at = base + kept[c];
          for (std::size_t i = f0; i < f1; ++i)
            if (keep[i]) s.prims[at++] = face_prim(mesh.faces[i]);
        }
      }, 1);
      s.info.triangles += kept[chunks];
      s.info.degenerate_skipped += nf - kept[chunks];
    }
  }

  for (const auto& l : desc.lights) {
    s.lights.push_back({LightEntry::kPoint, static_cast<std::uint32_t>(s.point_lights.size())});
    s.point_lights.push_back({l.position, l.intensity});
  }
  for (std::size_t i = 0; i < s.prims.size(); ++i)
    if (!emission_of(s.materials[s.prims[i].material]).zero())
      s.lights.push_back({LightEntry::kEmitter, static_cast<std::uint32_t>(i)});
  s.info.lights = s.lights.size();

  if (where == BvhBuild::Defer || (where == BvhBuild::Auto && s.prims.size() >= kGpuBuildMinPrims)) {
    s.bvh_built = false;
    return s;
  }
  std::vector<Box> boxes;
  boxes.reserve(s.prims.size());
  for (const Prim& p : s.prims) boxes.push_back(p.bounds());
  s.bvh.build(boxes, 4);
  s.info.bvh = s.bvh.stats;
  return s;
}

}  // namespace rtg
