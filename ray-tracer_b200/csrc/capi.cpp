// C ABI (include/rtg.h) over the host engine. Exceptions never cross the
// boundary: each entry point maps them to an RTG_ERR_* code and keeps the
// message for rtg_last_error.
#include "rtg.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <deque>
#include <exception>
#include <stdexcept>
#include <unordered_map>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>

#include "device/noalloc.h"
#include "device/probe.h"
#include "host/alloc_count.hpp"
#include "host/autotune.hpp"
#include "host/engine.hpp"
#include "host/scene_io.hpp"
#include "host/flatten.hpp"

namespace rtg {
std::vector<std::uint8_t> encode_png(const std::uint8_t* rgb, int width, int height);
}

struct rtg_host_scene {
  std::shared_ptr<const rtg::CompiledScene> scene;  // shared with every context it is uploaded to
  // Reference-layout arrays behind rtg_scene_view, made on its first call.
  mutable std::once_flag view_once;
  mutable std::vector<double> prims, planes, nodes, point_lights, materials;
  mutable std::vector<std::uint32_t> lights;
};

struct rtg_context {
  std::unique_ptr<rtg::Engine> engine;
  std::string error;
  bool busy = false;
  // Settings of the last plain render (for rtg_image_rgb8 with tone_map < 0).
  std::vector<rtg::RenderSettings> last_settings;
  // Serving: events not yet handed out, the admission budget and what the open
  // requests hold against it.
  std::deque<rtg_request_event> pending;
  std::uint64_t serve_budget = 16ull << 30;
  std::uint64_t serve_reserve = 2ull << 30;
  std::uint64_t serve_used = 0;
  std::unordered_map<int, std::uint64_t> footprint;
  std::unordered_map<int, rtg::RenderSettings> request_settings;
};

namespace {

thread_local std::string g_validate_message;

rtg::RenderSettings from_c(const rtg_settings& c) {
  rtg::RenderSettings s;
  s.width = c.width;
  s.height = c.height;
  s.spp = c.spp;
  s.max_depth = c.max_depth;
  s.rr_min_depth = c.rr_min_depth;
  s.integrator = static_cast<rtg::Integrator>(c.integrator);
  s.light_sampling = c.light_sampling != 0;
  s.mis = c.light_sampling == 2;
  s.tone_map = static_cast<rtg::ToneMap>(c.tone_map);
  s.seed = c.seed;
  s.exposure = c.exposure;
  s.threads = c.threads;
  s.tile_size = c.tile_size;
  s.use_bvh = c.use_bvh != 0;
  return s;
}

rtg_settings to_c(const rtg::RenderSettings& s) {
  rtg_settings c{};
  c.width = s.width;
  c.height = s.height;
  c.spp = s.spp;
  c.max_depth = s.max_depth;
  c.rr_min_depth = s.rr_min_depth;
  c.integrator = static_cast<int32_t>(s.integrator);
  c.light_sampling = s.light_sampling ? (s.mis ? 2 : 1) : 0;
  c.tone_map = static_cast<int32_t>(s.tone_map);
  c.seed = s.seed;
  c.exposure = s.exposure;
  c.threads = s.threads;
  c.tile_size = s.tile_size;
  c.use_bvh = s.use_bvh ? 1 : 0;
  return c;
}

rtg_progress to_c(const rtg::RenderProgress& p) {
  rtg_progress c{};
  c.pass = p.pass;
  c.spp_done = p.spp_done;
  c.spp_target = p.spp_target;
  c.finished = p.finished ? 1 : 0;
  c.cancelled = p.cancelled ? 1 : 0;
  c.elapsed_ms = p.elapsed_ms;
  c.rays = p.rays;
  return c;
}

// Range checks of validate_scene (src/io/scene_io.cpp:389-397) for settings
// passed directly through the ABI.
const char* settings_problem(const rtg_settings& c) {
  if (c.integrator < 0 || c.integrator > 2) return "render.integrator: expected path, direct or normals";
  if (c.tone_map < 0 || c.tone_map > 2) return "render.tone_map: expected clamp, reinhard or aces";
  return nullptr;
}

const char* settings_problem(const rtg::RenderSettings& s) {
  if (s.width < 1 || s.width > 8192) return "render.width: must be in [1, 8192]";
  if (s.height < 1 || s.height > 8192) return "render.height: must be in [1, 8192]";
  if (s.spp < 1 || s.spp > 1000000) return "render.spp: must be in [1, 1000000]";
  if (s.max_depth < 1 || s.max_depth > 1000) return "render.max_depth: must be in [1, 1000]";
  if (s.rr_min_depth < 0) return "render.rr_min_depth: must be >= 0";
  if (!(s.exposure > 0) || !std::isfinite(s.exposure)) return "render.exposure: must be > 0";
  return nullptr;
}

template <class F>
int guarded(rtg_context* ctx, F&& body) {
  if (!ctx) return RTG_ERR_INVALID;
  try {
    ctx->error.clear();
    return body();
  } catch (const rtg::SceneError& e) {
    ctx->error = e.what();
    return RTG_ERR_SCENE;
  } catch (const rtg::CudaFailure& e) {
    ctx->error = e.what();
    return std::strstr(e.what(), "device error flag") ? RTG_ERR_DEVICE : RTG_ERR_CUDA;
  } catch (const std::invalid_argument& e) {
    ctx->error = e.what();
    return RTG_ERR_INVALID;
  } catch (const std::length_error& e) {  // a fixed table is full
    ctx->error = e.what();
    return RTG_ERR_LIMIT;
  } catch (const std::logic_error& e) {   // the call conflicts with work in flight
    ctx->error = e.what();
    return RTG_ERR_BUSY;
  } catch (const std::exception& e) {
    ctx->error = e.what();
    return RTG_ERR_SCENE;
  }
}

struct BusyGuard {
  rtg_context* ctx;
  explicit BusyGuard(rtg_context* c) : ctx(c) { ctx->busy = true; }
  ~BusyGuard() { ctx->busy = false; }
};

}  // namespace

extern "C" {

const char* rtg_validate(const char* scene_json) {
  g_validate_message.clear();
  if (!scene_json) {
    g_validate_message = "scene: null input";
    return g_validate_message.c_str();
  }
  try {
    const rtg::SceneDesc d = rtg::parse_scene(scene_json);
    const auto errors = rtg::validate_scene(d);
    if (!errors.empty()) g_validate_message = errors.front();
  } catch (const std::exception& e) {
    g_validate_message = e.what();
  }
  return g_validate_message.c_str();
}

int64_t rtg_scene_dump(const char* scene_json, char* out, size_t cap) {
  if (!scene_json) return RTG_ERR_INVALID;
  try {
    const std::string s = rtg::scene_to_json(rtg::parse_scene(scene_json)).serialize(2);
    if (out && cap) {
      const std::size_t n = std::min(cap - 1, s.size());
      std::memcpy(out, s.data(), n);
      out[n] = '\0';
    }
    return static_cast<int64_t>(s.size());
  } catch (const std::exception&) {
    return RTG_ERR_SCENE;
  }
}

namespace {

// The compiled scene in the reference's own layout (rtg_scene_view's arrays).
void build_view_arrays(const rtg_host_scene& hs) {
  const rtg::CompiledScene& s = *hs.scene;
  for (const rtg::Prim& p : s.prims) {
    const rtg::D3 v[6] = {p.a, p.b, p.c, p.n0, p.n1, p.n2};
    hs.prims.push_back(p.kind == rtg::Prim::kSphere ? 0.0 : 1.0);
    hs.prims.push_back(p.material);
    hs.prims.push_back(p.smooth ? 1.0 : 0.0);
    for (const rtg::D3& q : v) {
      hs.prims.push_back(q.x);
      hs.prims.push_back(q.y);
      hs.prims.push_back(q.z);
    }
    hs.prims.insert(hs.prims.end(), 3, 0.0);
  }
  for (const rtg::PlanePrim& pl : s.planes) {
    const double r[8] = {pl.point.x, pl.point.y, pl.point.z, pl.normal.x, pl.normal.y, pl.normal.z, double(pl.material), 0};
    hs.planes.insert(hs.planes.end(), r, r + 8);
  }
  for (const rtg::BinaryNode& n : s.bvh.nodes) {
    const double r[10] = {n.box.lo.x, n.box.lo.y, n.box.lo.z, n.box.hi.x, n.box.hi.y, n.box.hi.z,
                          double(n.first), double(n.count), double(n.axis), 0};
    hs.nodes.insert(hs.nodes.end(), r, r + 10);
  }
  for (const rtg::LightEntry& l : s.lights) {
    hs.lights.push_back(l.kind == rtg::LightEntry::kPoint ? 0u : 1u);
    hs.lights.push_back(l.index);
  }
  for (const rtg::PointLight& pl : s.point_lights) {
    const double r[6] = {pl.position.x, pl.position.y, pl.position.z, pl.intensity.x, pl.intensity.y, pl.intensity.z};
    hs.point_lights.insert(hs.point_lights.end(), r, r + 6);
  }
  for (const rtg::Material& m : s.materials) {
    double r[16] = {0};
    if (const auto* l = std::get_if<rtg::Lambertian>(&m)) {
      r[0] = 0;
      r[1] = l->albedo.a.x; r[2] = l->albedo.a.y; r[3] = l->albedo.a.z;
      r[4] = l->albedo.b.x; r[5] = l->albedo.b.y; r[6] = l->albedo.b.z;
      r[7] = l->albedo.checker_scale;
    } else if (const auto* me = std::get_if<rtg::Metal>(&m)) {
      r[0] = 1;
      r[1] = me->albedo.x; r[2] = me->albedo.y; r[3] = me->albedo.z;
      r[8] = me->roughness;
    } else if (const auto* di = std::get_if<rtg::Dielectric>(&m)) {
      r[0] = 2;
      r[1] = di->tint.x; r[2] = di->tint.y; r[3] = di->tint.z;
      r[9] = di->ior;
    } else {
      const auto& e = std::get<rtg::Emissive>(m);
      r[0] = 3;
      r[1] = e.color.x; r[2] = e.color.y; r[3] = e.color.z;
      r[10] = e.intensity;
      r[11] = e.two_sided ? 1 : 0;
    }
    hs.materials.insert(hs.materials.end(), r, r + 16);
  }
}

}  // namespace

int rtg_compile(const char* scene_json, const char* base_dir, rtg_host_scene** out, char* err, size_t err_cap) {
  return rtg_compile_flags(scene_json, base_dir, 0, out, err, err_cap);
}

int rtg_compile_flags(const char* scene_json, const char* base_dir, uint32_t flags, rtg_host_scene** out, char* err,
                      size_t err_cap) {
  if (!scene_json || !out || (flags & ~uint32_t(RTG_COMPILE_DEFER_BVH | RTG_COMPILE_AUTO_BVH)) ||
      (flags == (RTG_COMPILE_DEFER_BVH | RTG_COMPILE_AUTO_BVH)))
    return RTG_ERR_INVALID;
  *out = nullptr;
  auto fail = [&](const char* msg) {
    if (err && err_cap) {
      const std::size_t n = std::min(err_cap - 1, std::strlen(msg));
      std::memcpy(err, msg, n);
      err[n] = '\0';
    }
  };
  try {
    rtg::SceneDesc d = rtg::parse_scene(scene_json);
    if (base_dir) d.base_dir = base_dir;
    auto hs = std::make_unique<rtg_host_scene>();
    const rtg::BvhBuild where = (flags & RTG_COMPILE_DEFER_BVH)  ? rtg::BvhBuild::Defer
                                : (flags & RTG_COMPILE_AUTO_BVH) ? rtg::BvhBuild::Auto
                                                                 : rtg::BvhBuild::Host;
    hs->scene = std::make_shared<const rtg::CompiledScene>(rtg::compile_scene(d, where));
    *out = hs.release();
    return RTG_OK;
  } catch (const std::exception& e) {
    fail(e.what());
    return RTG_ERR_SCENE;
  }
}

void rtg_host_scene_free(rtg_host_scene* scene) { delete scene; }

int64_t rtg_host_scene_layout(const rtg_host_scene* hs, int32_t part, void* out, uint64_t cap) {
  if (!hs) return RTG_ERR_INVALID;
  try {
    if (!hs->scene->bvh_built) return RTG_ERR_INVALID;
    const rtg::FlatScene f = rtg::flatten(*hs->scene, true);
    const std::int32_t roots[5] = {f.root, f.root4, static_cast<std::int32_t>(f.slot_prim.size()), 0, f.root8};
    const void* src = nullptr;
    std::size_t bytes = 0;
    switch (part) {
      case RTG_LAYOUT_NODES: src = f.nodes.data(); bytes = f.nodes.size() * sizeof(rtg::DevNode); break;
      case RTG_LAYOUT_NODES4: src = f.nodes4.data(); bytes = f.nodes4.size() * sizeof(rtg::DevNode4); break;
      case RTG_LAYOUT_NODES8: src = f.nodes8.data(); bytes = f.nodes8.size() * sizeof(rtg::DevNode8); break;
      case RTG_LAYOUT_PRIMS: src = f.prims.data(); bytes = f.prims.size() * sizeof(float4); break;
      case RTG_LAYOUT_SLOT_MATERIAL: src = f.slot_material.data(); bytes = f.slot_material.size() * 4; break;
      case RTG_LAYOUT_SLOT_NORMALS: src = f.slot_normals.data(); bytes = f.slot_normals.size() * sizeof(float4); break;
      case RTG_LAYOUT_PLANES: src = f.planes.data(); bytes = f.planes.size() * sizeof(rtg::DevPlane); break;
      case RTG_LAYOUT_MATERIALS: src = f.materials.data(); bytes = f.materials.size() * sizeof(rtg::DevMaterial); break;
      case RTG_LAYOUT_LIGHTS: src = f.lights.data(); bytes = f.lights.size() * sizeof(rtg::DevLight); break;
      case RTG_LAYOUT_SLOT_PRIM: src = f.slot_prim.data(); bytes = f.slot_prim.size() * 4; break;
      case RTG_LAYOUT_ROOTS: src = roots; bytes = sizeof(roots); break;
      default: return RTG_ERR_INVALID;
    }
    if (out && bytes) std::memcpy(out, src, std::min<std::size_t>(bytes, cap));
    return static_cast<int64_t>(bytes);
  } catch (const std::exception&) {
    return RTG_ERR_INVALID;
  }
}

int rtg_host_scene_view(const rtg_host_scene* hs, rtg_scene_view* out) {
  if (!hs || !out) return RTG_ERR_INVALID;
  std::call_once(hs->view_once, [hs] { build_view_arrays(*hs); });
  const rtg::CompiledScene& s = *hs->scene;
  *out = rtg_scene_view{};
  out->n_prims = s.prims.size();
  out->n_planes = s.planes.size();
  out->n_nodes = s.bvh.nodes.size();
  out->n_order = s.bvh.order.size();
  out->n_lights = s.lights.size();
  out->n_point_lights = s.point_lights.size();
  out->n_materials = s.materials.size();
  out->prims = hs->prims.data();
  out->planes = hs->planes.data();
  out->nodes = hs->nodes.data();
  out->order = s.bvh.order.data();
  out->lights = hs->lights.data();
  out->point_lights = hs->point_lights.data();
  out->materials = hs->materials.data();
  const rtg::CameraFrame& c = s.camera;
  const rtg::D3 cv[6] = {c.origin, c.corner, c.du, c.dv, c.u, c.v};
  for (int k = 0; k < 6; ++k) {
    out->camera[3 * k] = cv[k].x;
    out->camera[3 * k + 1] = cv[k].y;
    out->camera[3 * k + 2] = cv[k].z;
  }
  out->camera[18] = c.lens_radius;
  const rtg::Background& b = s.background;
  const double bg[8] = {b.kind == rtg::Background::Kind::Solid ? 1.0 : 0.0, b.top.x, b.top.y, b.top.z,
                        b.bottom.x, b.bottom.y, b.bottom.z, b.intensity};
  std::memcpy(out->background, bg, sizeof bg);
  out->settings = to_c(s.settings);
  out->degenerate_skipped = s.info.degenerate_skipped;
  out->bvh_max_depth = s.info.bvh.max_depth;
  out->bvh_leaves = s.info.bvh.leaves;
  out->bvh_max_leaf = s.info.bvh.max_leaf;
  out->bvh_sah_cost = s.info.bvh.sah_cost;
  return RTG_OK;
}

int rtg_scene_upload(rtg_context* ctx, const rtg_host_scene* scene, rtg_scene_id* out) {
  return guarded(ctx, [&]() {
    if (!scene || !out) throw std::invalid_argument("null argument");
    *out = ctx->engine->add_scene(scene->scene);
    return RTG_OK;
  });
}

int rtg_scene_upload_gpu_bvh(rtg_context* ctx, const rtg_host_scene* scene, rtg_scene_id* out) {
  return guarded(ctx, [&]() {
    if (!scene || !out) throw std::invalid_argument("null argument");
    *out = ctx->engine->add_scene_gpu_bvh(scene->scene);
    return RTG_OK;
  });
}

int64_t rtg_scene_layout(rtg_context* ctx, rtg_scene_id scene, int32_t part, void* out, uint64_t cap) {
  int64_t bytes = 0;
  const int rc = guarded(ctx, [&]() {
    if (ctx->busy) return RTG_ERR_BUSY;
    const rtg::GpuScene& g = ctx->engine->scene(scene);
    const std::int32_t roots[5] = {g.root, g.root4, g.n_slots, g.device_built ? 1 : 0, g.root8};
    const void* src = nullptr;
    bool on_device = true;
    const int64_t slots = g.n_slots;
    switch (part) {
      case RTG_LAYOUT_NODES: src = g.nodes; bytes = int64_t(g.n_interior) * int64_t(sizeof(rtg::DevNode)); break;
      case RTG_LAYOUT_NODES4: src = g.nodes4; bytes = int64_t(g.n_wide) * int64_t(sizeof(rtg::DevNode4)); break;
      case RTG_LAYOUT_NODES8: src = g.nodes8; bytes = int64_t(g.n_wide8) * int64_t(sizeof(rtg::DevNode8)); break;
      case RTG_LAYOUT_PRIMS: src = g.prims; bytes = slots * 3 * int64_t(sizeof(float4)); break;
      case RTG_LAYOUT_SLOT_MATERIAL: src = g.slot_material; bytes = slots * int64_t(sizeof(uint32_t)); break;
      case RTG_LAYOUT_SLOT_NORMALS: src = g.slot_normals; bytes = slots * 3 * int64_t(sizeof(float4)); break;
      case RTG_LAYOUT_PLANES: src = g.planes; bytes = int64_t(g.n_planes) * int64_t(sizeof(rtg::DevPlane)); break;
      case RTG_LAYOUT_MATERIALS:
        src = g.materials;
        bytes = int64_t(g.host->materials.size()) * int64_t(sizeof(rtg::DevMaterial));
        break;
      case RTG_LAYOUT_LIGHTS: src = g.lights; bytes = int64_t(g.n_lights) * int64_t(sizeof(rtg::DevLight)); break;
      case RTG_LAYOUT_SLOT_PRIM:
        src = g.slot_prim.data();
        on_device = false;
        bytes = slots * int64_t(sizeof(uint32_t));
        break;
      case RTG_LAYOUT_ROOTS:
        src = roots;
        on_device = false;
        bytes = int64_t(sizeof(roots));
        break;
      default: throw std::invalid_argument("unknown layout part " + std::to_string(part));
    }
    const std::size_t n = static_cast<std::size_t>(std::min<uint64_t>(cap, uint64_t(bytes)));
    if (out && n) {
      if (on_device) {
        cudaStream_t st = ctx->engine->stream();
        const cudaError_t e1 = cudaMemcpyAsync(out, src, n, cudaMemcpyDeviceToHost, st);
        const cudaError_t e2 = cudaStreamSynchronize(st);
        if (e1 != cudaSuccess || e2 != cudaSuccess)
          throw rtg::CudaFailure(std::string("layout read-back: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
      } else {
        std::memcpy(out, src, n);
      }
    }
    return RTG_OK;
  });
  return rc < 0 ? rc : bytes;
}

int rtg_scene_upload_batch(rtg_context* ctx, int32_t n, const rtg_host_scene* const* scenes, rtg_scene_id* out) {
  return guarded(ctx, [&]() {
    if (n < 0 || (n > 0 && (!scenes || !out))) throw std::invalid_argument("null argument");
    std::vector<std::shared_ptr<const rtg::CompiledScene>> list;
    for (int32_t k = 0; k < n; ++k) {
      if (!scenes[k]) throw std::invalid_argument("null scene in batch");
      list.push_back(scenes[k]->scene);
    }
    const std::vector<int> ids = ctx->engine->add_scenes(list);
    for (int32_t k = 0; k < n; ++k) out[k] = ids[static_cast<std::size_t>(k)];
    return RTG_OK;
  });
}

int rtg_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int rtg_context_create(int device, rtg_context** out) {
  if (!out) return RTG_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return RTG_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return RTG_ERR_INVALID;
  auto ctx = std::make_unique<rtg_context>();
  try {
    ctx->engine = std::make_unique<rtg::Engine>(device);
  } catch (const std::exception&) {
    return RTG_ERR_CUDA;
  }
  *out = ctx.release();
  return RTG_OK;
}

void rtg_context_destroy(rtg_context* ctx) { delete ctx; }

const char* rtg_last_error(const rtg_context* ctx) { return ctx ? ctx->error.c_str() : "null context"; }

int rtg_scene_load_json(rtg_context* ctx, const char* scene_json, const char* base_dir, rtg_scene_id* out) {
  return guarded(ctx, [&]() {
    if (!scene_json || !out) throw std::invalid_argument("null argument");
    rtg::SceneDesc d = rtg::parse_scene(scene_json);
    if (base_dir) d.base_dir = base_dir;
    *out = ctx->engine->add_scene(
        std::make_shared<const rtg::CompiledScene>(rtg::compile_scene(d, rtg::BvhBuild::Auto)));
    return RTG_OK;
  });
}

int rtg_scene_load_file(rtg_context* ctx, const char* path, rtg_scene_id* out) {
  return guarded(ctx, [&]() {
    if (!path || !out) throw std::invalid_argument("null argument");
    const rtg::SceneDesc d = rtg::load_scene(path);
    *out = ctx->engine->add_scene(
        std::make_shared<const rtg::CompiledScene>(rtg::compile_scene(d, rtg::BvhBuild::Auto)));
    return RTG_OK;
  });
}

int rtg_scene_settings(rtg_context* ctx, rtg_scene_id scene, rtg_settings* out) {
  return guarded(ctx, [&]() {
    if (!out) throw std::invalid_argument("null argument");
    *out = to_c(ctx->engine->scene(scene).host->settings);
    return RTG_OK;
  });
}

int rtg_scene_get_info(rtg_context* ctx, rtg_scene_id scene, rtg_scene_info* out) {
  return guarded(ctx, [&]() {
    if (!out) throw std::invalid_argument("null argument");
    const rtg::GpuScene& g = ctx->engine->scene(scene);
    const rtg::BuildInfo& i = g.host->info;
    const rtg::BvhStats& b = g.bvh;
    *out = rtg_scene_info{};
    out->primitives = g.host->prims.size();
    out->triangles = i.triangles;
    out->spheres = i.spheres;
    out->planes = i.planes;
    out->degenerate_skipped = i.degenerate_skipped;
    out->lights = i.lights;
    out->bvh_nodes = b.nodes;
    out->bvh_leaves = b.leaves;
    out->bvh_max_depth = b.max_depth;
    out->bvh_max_leaf = b.max_leaf;
    out->device_bytes = g.device_bytes;
    out->bvh_build_ms = b.build_ms;
    out->bvh_sah_cost = b.sah_cost;
    return RTG_OK;
  });
}

int rtg_scene_release(rtg_context* ctx, rtg_scene_id scene) {
  return guarded(ctx, [&]() {
    if (ctx->busy) return RTG_ERR_BUSY;
    ctx->engine->release_scene(scene);
    return RTG_OK;
  });
}

int rtg_render(rtg_context* ctx, rtg_scene_id scene, const rtg_settings* settings, const rtg_render_options* opts,
               rtg_pass_fn on_pass, void* user, const volatile int32_t* cancel, rtg_progress* out) {
  return guarded(ctx, [&]() {
    if (ctx->busy) return RTG_ERR_BUSY;
    if (settings)
      if (const char* bad = settings_problem(*settings)) throw rtg::SceneError(bad);
    const rtg::RenderSettings s = settings ? from_c(*settings) : ctx->engine->scene(scene).host->settings;
    if (const char* bad = settings_problem(s)) throw rtg::SceneError(bad);
    rtg::RenderOptions o;
    if (opts) {
      o.progressive = opts->progressive != 0;
      o.max_pass_spp = opts->max_pass_spp;
    }
    BusyGuard guard(ctx);
    ctx->last_settings.assign(1, s);
    rtg::PassCallback cb;
    if (on_pass) cb = [&](const rtg::RenderProgress& p) {
      const rtg_progress c = to_c(p);
      on_pass(user, &c);
    };
    if (ctx->engine->open_requests() > 0) {
      ctx->error = "rtg_render: serving requests are open on this context";
      return RTG_ERR_BUSY;
    }
    const rtg::RenderProgress p = ctx->engine->render(scene, s, o, cb, cancel);
    if (out) *out = to_c(p);
    return RTG_OK;
  });
}

int rtg_render_batch(rtg_context* ctx, int32_t n, const rtg_scene_id* scenes, const rtg_settings* settings,
                     const rtg_render_options* opts, const volatile int32_t* cancel, rtg_progress* out) {
  return guarded(ctx, [&]() {
    if (ctx->busy) return RTG_ERR_BUSY;
    if (n <= 0 || n > 65535 || !scenes) throw std::invalid_argument("batch needs 1..65535 jobs");
    std::vector<rtg::Engine::BatchJob> jobs;
    for (int32_t j = 0; j < n; ++j) {
      if (settings)
        if (const char* bad = settings_problem(settings[j])) throw rtg::SceneError(bad);
      const rtg::RenderSettings s = settings ? from_c(settings[j]) : ctx->engine->scene(scenes[j]).host->settings;
      if (const char* bad = settings_problem(s)) throw rtg::SceneError(bad);
      jobs.push_back({scenes[j], s});
    }
    rtg::RenderOptions o;
    if (opts) {
      o.progressive = opts->progressive != 0;
      o.max_pass_spp = opts->max_pass_spp;
    }
    BusyGuard guard(ctx);
    ctx->last_settings.clear();
    for (const auto& j : jobs) ctx->last_settings.push_back(j.settings);
    if (ctx->engine->open_requests() > 0) {
      ctx->error = "rtg_render_batch: serving requests are open on this context";
      return RTG_ERR_BUSY;
    }
    const std::vector<rtg::RenderProgress> p = ctx->engine->render_batch(jobs, o, cancel);
    if (out)
      for (int32_t j = 0; j < n; ++j) out[j] = to_c(p[static_cast<std::size_t>(j)]);
    return RTG_OK;
  });
}

int rtg_framebuffer_mean(rtg_context* ctx, int32_t job, double* rgb) {
  return guarded(ctx, [&]() {
    if (!rgb) throw std::invalid_argument("null argument");
    ctx->engine->read_mean(job, rgb);
    return RTG_OK;
  });
}

int rtg_framebuffer_moments(rtg_context* ctx, int32_t job, double* sum, double* sumsq, uint32_t* count) {
  return guarded(ctx, [&]() {
    ctx->engine->read_moments(job, sum, sumsq, count);
    return RTG_OK;
  });
}

namespace {

// The tone map and exposure an image of `job` uses: the render's settings when
// tone_map < 0 (normals: clamp, exposure 1, as Renderer::image), else the given ones.
void image_op(const rtg_context* ctx, int32_t job, int32_t tone_map, double exposure, rtg::ToneMap& op, double& ex) {
  op = rtg::ToneMap::Clamp;
  ex = exposure;
  if (tone_map < 0) {
    const std::size_t j = job < 0 ? 0 : static_cast<std::size_t>(job);
    if (j >= ctx->last_settings.size()) throw std::invalid_argument("no render for job");
    const rtg::RenderSettings& s = ctx->last_settings[j];
    if (s.integrator == rtg::Integrator::Normals) {
      ex = 1.0;
    } else {
      op = s.tone_map;
      ex = s.exposure;
    }
  } else {
    if (tone_map > 2) throw std::invalid_argument("tone_map must be 0, 1 or 2");
    op = static_cast<rtg::ToneMap>(tone_map);
  }
}

}  // namespace

int rtg_image_rgb8(rtg_context* ctx, int32_t job, int32_t tone_map, double exposure, uint8_t* rgb) {
  return guarded(ctx, [&]() {
    if (!rgb) throw std::invalid_argument("null argument");
    rtg::ToneMap op;
    double ex;
    image_op(ctx, job, tone_map, exposure, op, ex);
    ctx->engine->read_image(job, op, ex, rgb);
    return RTG_OK;
  });
}

int rtg_images_rgb8(rtg_context* ctx, int32_t n, const int32_t* jobs, int32_t tone_map, double exposure,
                    uint8_t* const* rgb) {
  return guarded(ctx, [&]() {
    if (n < 0 || (n > 0 && (!jobs || !rgb))) throw std::invalid_argument("null argument");
    std::vector<rtg::ToneMap> ops(static_cast<std::size_t>(n));
    std::vector<double> exs(static_cast<std::size_t>(n));
    std::vector<int> js(static_cast<std::size_t>(n));
    for (int32_t k = 0; k < n; ++k) {
      if (!rgb[k]) throw std::invalid_argument("null argument");
      image_op(ctx, jobs[k], tone_map, exposure, ops[k], exs[k]);
      js[k] = jobs[k];
    }
    ctx->engine->read_images(n, js.data(), ops.data(), exs.data(), rgb);
    return RTG_OK;
  });
}

int rtg_render_stats(rtg_context* ctx, rtg_stats* out) {
  return guarded(ctx, [&]() {
    if (!out) throw std::invalid_argument("null argument");
    const rtg::RenderStats& s = ctx->engine->stats();
    *out = rtg_stats{};
    out->camera_samples = s.camera_samples;
    out->rays = s.rays;
    out->shadow_rays = s.shadow_rays;
    out->rr_terminated = s.rr_terminated;
    out->invalid_samples = s.invalid_samples;
    out->passes = s.passes;
    out->iterations = s.iterations;
    out->node_visits = s.node_visits;
    out->prim_tests = s.prim_tests;
    out->extend_launches = s.extend_launches;
    out->sphere_tests = s.sphere_tests;
    out->shadow_node_visits = s.shadow_node_visits;
    out->shadow_prim_tests = s.shadow_prim_tests;
    out->shadow_sphere_tests = s.shadow_sphere_tests;
    out->kernel_launches = s.kernel_launches;
    out->elapsed_ms = s.elapsed_ms;
    out->device_ms = s.device_ms;
    out->extend_ms = s.extend_ms;
    out->shade_ms = s.shade_ms;
    out->shadow_ms = s.shadow_ms;
    out->accumulate_ms = s.accumulate_ms;
    out->direct_ms = s.direct_ms;
    out->plan_ms = s.plan_ms;
    return RTG_OK;
  });
}

int rtg_trace_closest(rtg_context* ctx, rtg_scene_id scene, const float* rays, uint64_t n, int32_t brute, float* t,
                      int32_t* prim, int32_t* is_plane, float* bary) {
  return guarded(ctx, [&]() {
    if (!rays && n) throw std::invalid_argument("null rays");
    ctx->engine->trace_closest(scene, rays, n, brute != 0, t, prim, is_plane, bary);
    return RTG_OK;
  });
}

int rtg_trace_any(rtg_context* ctx, rtg_scene_id scene, const float* rays, uint64_t n, int32_t brute,
                  uint8_t* occluded) {
  return guarded(ctx, [&]() {
    if ((!rays || !occluded) && n) throw std::invalid_argument("null argument");
    ctx->engine->trace_any(scene, rays, n, brute != 0, occluded);
    return RTG_OK;
  });
}

int rtg_trace_closest_noalloc(rtg_context* ctx, rtg_scene_id scene, const float* rays, uint64_t n, int32_t brute,
                              float* t, int32_t* prim, int32_t* is_plane, float* bary) {
  static_assert(RTG_NOALLOC_MAX_RAYS == rtg::kNoAllocMaxRays, "header and scratch sizes disagree");
  return guarded(ctx, [&]() {
    if (!rays && n) throw std::invalid_argument("null rays");
    if (n > rtg::kNoAllocMaxRays) {
      ctx->error = "rtg_trace_closest_noalloc: " + std::to_string(n) + " rays exceed the limit of " +
                   std::to_string(rtg::kNoAllocMaxRays) + " per call (RTG_NOALLOC_MAX_RAYS)";
      return RTG_ERR_LIMIT;
    }
    const rtg::RtgSceneDev d = ctx->engine->query_descriptor(scene, brute != 0);
    const cudaError_t e = rtg::noalloc_trace_closest(ctx->engine->device(), d, rays, n, brute,
                                                     ctx->engine->config().shape.closest_tree, t, prim, is_plane,
                                                     bary, ctx->engine->stream());
    if (e != cudaSuccess) throw rtg::CudaFailure(std::string("rtg_trace_closest_noalloc: ") + cudaGetErrorString(e));
    return RTG_OK;
  });
}

uint64_t rtg_allocation_count(void) { return rtg::allocation_count(); }

int rtg_probe_read_bandwidth(rtg_context* ctx, uint64_t bytes, int32_t reps, int32_t l1, double* gbs) {
  return guarded(ctx, [&]() {
    if (!gbs) throw std::invalid_argument("null argument");
    if (reps < 1) throw std::invalid_argument("reps must be >= 1");
    if (l1 && (bytes < 4096 || bytes > (128u << 10))) throw std::invalid_argument("l1: bytes must be in [4 KiB, 128 KiB]");
    if (!l1 && bytes < (1u << 20)) throw std::invalid_argument("bytes must be >= 1 MiB");
    if (ctx->busy) return RTG_ERR_BUSY;
    cudaError_t e = cudaSetDevice(ctx->engine->device());
    if (e == cudaSuccess) e = rtg::probe_read_bandwidth(bytes, reps, l1 != 0, ctx->engine->stream(), gbs);
    if (e != cudaSuccess) throw rtg::CudaFailure(std::string("rtg_probe_read_bandwidth: ") + cudaGetErrorString(e));
    return RTG_OK;
  });
}

int rtg_get_tuning(rtg_context* ctx, rtg_tuning* out) {
  return guarded(ctx, [&]() {
    if (!out) throw std::invalid_argument("null argument");
    const rtg::EngineConfig& c = ctx->engine->config();
    *out = rtg_tuning{};
    out->pool_paths = c.pool_paths;
    out->block = static_cast<uint32_t>(c.shape.extend_block);
    out->max_pass_samples = c.max_pass_samples;
    out->extend_blocks = c.shape.extend_blocks;
    out->shade_blocks = c.shape.shade_blocks;
    out->shadow_blocks = c.shape.shadow_blocks;
    out->time_kernels = c.time_kernels ? 1 : 0;
    out->count_traversal = c.count_traversal ? 1 : 0;
    out->backlog_pools = c.backlog_pools;
    out->chained = c.shape.chained ? 1 : 0;
    out->serve_budget_bytes = ctx->serve_budget;
    out->serve_reserve_bytes = ctx->serve_reserve;
    out->refine_hits = c.refine_hits ? 1 : 0;
    out->closest_tree = c.shape.closest_tree;
    out->shadow_tree = c.shape.shadow_tree;
    return RTG_OK;
  });
}

int rtg_set_tuning(rtg_context* ctx, const rtg_tuning* in) {
  return guarded(ctx, [&]() {
    if (!in) throw std::invalid_argument("null argument");
    if (ctx->busy) return RTG_ERR_BUSY;
    if (in->block != 64 && in->block != 128 && in->block != 256) throw std::invalid_argument("block must be 64, 128 or 256");
    if (in->pool_paths < 1024 || in->pool_paths > (1u << 23)) throw std::invalid_argument("pool_paths must be in [1024, 2^23]");
    if (in->max_pass_samples < 1 || in->max_pass_samples > (1ull << 31)) throw std::invalid_argument("max_pass_samples must be in [1, 2^31]");
    if (in->backlog_pools < 1 || in->backlog_pools > 64) throw std::invalid_argument("backlog_pools must be in [1, 64]");
    if (in->closest_tree != 2 && in->closest_tree != 8) throw std::invalid_argument("closest_tree must be 2 or 8");
    if (in->shadow_tree != 4 && in->shadow_tree != 8) throw std::invalid_argument("shadow_tree must be 4 or 8");
    if (in->serve_reserve_bytes > (in->serve_budget_bytes ? in->serve_budget_bytes : ctx->serve_budget))
      throw std::invalid_argument("serve_reserve_bytes exceeds the budget");
    rtg::EngineConfig& c = ctx->engine->config();
    const bool realloc = c.pool_paths != in->pool_paths || c.max_pass_samples != in->max_pass_samples;
    if (realloc && ctx->engine->open_requests() > 0) {
      ctx->error = "rtg_set_tuning: the pool cannot change while serving requests are open";
      return RTG_ERR_BUSY;
    }
    c.pool_paths = in->pool_paths;
    c.shape.extend_block = static_cast<int>(in->block);
    c.max_pass_samples = in->max_pass_samples;
    c.shape.extend_blocks = in->extend_blocks;
    c.shape.shade_blocks = in->shade_blocks;
    c.shape.shadow_blocks = in->shadow_blocks;
    c.time_kernels = in->time_kernels != 0;
    c.count_traversal = in->count_traversal != 0;
    c.backlog_pools = in->backlog_pools;
    c.shape.chained = in->chained != 0;
    c.refine_hits = in->refine_hits != 0;
    c.shape.closest_tree = in->closest_tree;
    c.shape.shadow_tree = in->shadow_tree;
    if (in->serve_budget_bytes) ctx->serve_budget = in->serve_budget_bytes;
    ctx->serve_reserve = in->serve_reserve_bytes;
    if (realloc) ctx->engine->reset_wave();
    return RTG_OK;
  });
}

int rtg_autotune(rtg_context* ctx, int32_t n, const rtg_scene_id* scenes, const rtg_settings* settings,
                 const rtg_render_options* opts, int32_t use_cache, rtg_tuning* chosen, double* msamples_per_s,
                 int32_t* from_cache) {
  return guarded(ctx, [&]() {
    if (ctx->busy) return RTG_ERR_BUSY;
    if (n <= 0 || n > 65535 || !scenes) throw std::invalid_argument("autotune needs 1..65535 jobs");
    if (ctx->engine->open_requests() > 0) {
      ctx->error = "rtg_autotune: serving requests are open on this context";
      return RTG_ERR_BUSY;
    }
    std::vector<rtg::Engine::BatchJob> jobs;
    for (int32_t j = 0; j < n; ++j) {
      if (settings)
        if (const char* bad = settings_problem(settings[j])) throw rtg::SceneError(bad);
      const rtg::RenderSettings s = settings ? from_c(settings[j]) : ctx->engine->scene(scenes[j]).host->settings;
      if (const char* bad = settings_problem(s)) throw rtg::SceneError(bad);
      jobs.push_back({scenes[j], s});
    }
    rtg::RenderOptions o;
    if (opts) {
      o.progressive = opts->progressive != 0;
      o.max_pass_spp = opts->max_pass_spp;
    }
    BusyGuard guard(ctx);
    const rtg::AutotuneResult r = rtg::autotune(*ctx->engine, jobs, o, use_cache != 0);
    if (msamples_per_s) *msamples_per_s = r.msamples_per_s;
    if (from_cache) *from_cache = r.from_cache ? 1 : 0;
    ctx->last_settings.clear();  // the probe renders replaced the last frames
    if (chosen) return rtg_get_tuning(ctx, chosen);
    return RTG_OK;
  });
}

int rtg_request_submit(rtg_context* ctx, rtg_scene_id scene, const rtg_settings* settings,
                       const rtg_render_options* opts, int32_t priority, rtg_request_id* out) {
  return guarded(ctx, [&]() {
    if (!out) throw std::invalid_argument("null argument");
    if (ctx->busy) return RTG_ERR_BUSY;
    if (settings)
      if (const char* bad = settings_problem(*settings)) throw rtg::SceneError(bad);
    rtg::JobSpec spec;
    spec.scene_id = scene;
    spec.settings = settings ? from_c(*settings) : ctx->engine->scene(scene).host->settings;
    if (const char* bad = settings_problem(spec.settings)) throw rtg::SceneError(bad);
    if (opts) {
      spec.opts.progressive = opts->progressive != 0;
      spec.opts.max_pass_spp = opts->max_pass_spp;
    }
    spec.priority = priority;
    const std::uint64_t bytes = ctx->engine->request_bytes(spec);
    const std::uint64_t limit = priority > 0 ? ctx->serve_budget - ctx->serve_reserve : ctx->serve_budget;
    if (ctx->serve_used + bytes > limit) {
      ctx->error = "rtg_request_submit: " + std::to_string(bytes) + " bytes would exceed the serving budget (" +
                   std::to_string(ctx->serve_used) + " of " + std::to_string(limit) + " in use at priority " +
                   std::to_string(priority) + ")";
      return RTG_ERR_LIMIT;
    }
    // Map the whole admission budget into the pool before the first request, so
    // later framebuffer allocations are suballocations and never stall on the driver.
    ctx->engine->reserve_pool(static_cast<std::size_t>(ctx->serve_budget));
    const int h = ctx->engine->submit(spec);
    ctx->footprint[h] = bytes;
    ctx->serve_used += bytes;
    ctx->request_settings[h] = spec.settings;
    *out = h;
    return RTG_OK;
  });
}

int rtg_serve_pump(rtg_context* ctx, double budget_ms, int32_t return_on_event, rtg_request_event* events,
                   int32_t cap, int32_t* n) {
  return guarded(ctx, [&]() {
    if (!n || (cap > 0 && !events)) throw std::invalid_argument("null argument");
    if (ctx->busy) return RTG_ERR_BUSY;
    *n = 0;
    if (ctx->pending.empty() || !return_on_event) {
      std::vector<rtg::Engine::PassEvent> ev;
      ctx->engine->pump(budget_ms, return_on_event != 0, ev);
      for (const auto& e : ev) {
        rtg_request_event c{};
        c.request = e.request;
        c.progress = to_c(e.progress);
        ctx->pending.push_back(c);
      }
    }
    while (*n < cap && !ctx->pending.empty()) {
      events[(*n)++] = ctx->pending.front();
      ctx->pending.pop_front();
    }
    return RTG_OK;
  });
}

int rtg_request_cancel(rtg_context* ctx, rtg_request_id request) {
  return guarded(ctx, [&]() {
    ctx->engine->cancel_request(request);
    return RTG_OK;
  });
}

int rtg_request_release(rtg_context* ctx, rtg_request_id request) {
  return guarded(ctx, [&]() {
    if (!ctx->engine->request_exists(request)) throw std::invalid_argument("unknown request " + std::to_string(request));
    const rtg::RenderProgress& p = ctx->engine->request_progress(request);
    if (!p.finished && !p.cancelled) {
      ctx->error = "rtg_request_release: request " + std::to_string(request) + " is still rendering";
      return RTG_ERR_BUSY;
    }
    try {
      ctx->engine->release_request(request);
    } catch (const std::logic_error& e) {
      ctx->error = e.what();
      return RTG_ERR_BUSY;
    }
    ctx->serve_used -= ctx->footprint[request];
    ctx->footprint.erase(request);
    ctx->request_settings.erase(request);
    return RTG_OK;
  });
}

int rtg_request_progress(rtg_context* ctx, rtg_request_id request, rtg_progress* out) {
  return guarded(ctx, [&]() {
    if (!out) throw std::invalid_argument("null argument");
    *out = to_c(ctx->engine->request_progress(request));
    return RTG_OK;
  });
}

int rtg_request_mean(rtg_context* ctx, rtg_request_id request, double* rgb) {
  return guarded(ctx, [&]() {
    if (!rgb) throw std::invalid_argument("null argument");
    ctx->engine->read_mean_frame(ctx->engine->request_frame(request), rgb);
    return RTG_OK;
  });
}

int rtg_request_image_rgb8(rtg_context* ctx, rtg_request_id request, int32_t tone_map, double exposure, uint8_t* rgb) {
  return guarded(ctx, [&]() {
    if (!rgb) throw std::invalid_argument("null argument");
    const rtg::GpuFrame& f = ctx->engine->request_frame(request);
    rtg::ToneMap op = rtg::ToneMap::Clamp;
    double ex = exposure;
    if (tone_map < 0) {
      const rtg::RenderSettings& s = ctx->request_settings.at(request);
      if (s.integrator == rtg::Integrator::Normals) {
        ex = 1.0;
      } else {
        op = s.tone_map;
        ex = s.exposure;
      }
    } else {
      if (tone_map > 2) throw std::invalid_argument("tone_map must be 0, 1 or 2");
      op = static_cast<rtg::ToneMap>(tone_map);
    }
    ctx->engine->read_image_frame(f, op, ex, rgb);
    return RTG_OK;
  });
}

int rtg_serve_prepare(rtg_context* ctx) {
  return guarded(ctx, [&]() {
    ctx->engine->reserve_pool(static_cast<std::size_t>(ctx->serve_budget));
    return RTG_OK;
  });
}

int rtg_serve_footprint(rtg_context* ctx, uint64_t* bytes, int32_t* open_requests, int32_t* rendering) {
  return guarded(ctx, [&]() {
    if (bytes) *bytes = ctx->serve_used;
    if (open_requests) *open_requests = static_cast<int32_t>(ctx->engine->open_requests());
    if (rendering) *rendering = static_cast<int32_t>(ctx->engine->requests_rendering());
    return RTG_OK;
  });
}

int64_t rtg_encode_png(const uint8_t* rgb, int32_t width, int32_t height, uint8_t* out, size_t cap) {
  try {
    const std::vector<std::uint8_t> png = rtg::encode_png(rgb, width, height);
    if (out) {
      if (cap < png.size()) return RTG_ERR_LIMIT;
      std::memcpy(out, png.data(), png.size());
    }
    return static_cast<int64_t>(png.size());
  } catch (const std::exception&) {
    return RTG_ERR_INVALID;
  }
}

}  // extern "C"
