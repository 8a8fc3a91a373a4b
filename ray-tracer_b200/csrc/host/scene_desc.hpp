#pragma once
// Editable scene description: what the scene JSON and the editor talk about.
//
// Field names, defaults and meaning follow the reference's SceneDesc and
// RenderSettings (include/raytracer/core/scene_desc.hpp:20-102,
// include/raytracer/core/camera.hpp:9-17, include/raytracer/materials/material.hpp:14-56)
// so that the same JSON produces the same scene. One extension: torus meshes may
// carry `segments_v` (0 = the reference's segments / 2).
#include <cstdint>
#include <string>
#include <variant>
#include <vector>

#include "host/vec.hpp"

namespace rtg {

enum class Integrator : std::uint8_t { Path = 0, Direct = 1, Normals = 2 };
enum class ToneMap : std::uint8_t { Clamp = 0, Reinhard = 1, Aces = 2 };

struct CameraDesc {
  D3 look_from{0, 0, 0};
  D3 look_at{0, 0, -1};
  D3 vup{0, 1, 0};
  double vfov_deg = 40;
  double aperture = 0;
  double focus_dist = 0;
  bool operator==(const CameraDesc&) const = default;
};

struct RenderSettings {
  int width = 640;
  int height = 360;
  int spp = 64;
  int max_depth = 8;
  int rr_min_depth = 3;
  Integrator integrator = Integrator::Path;
  bool light_sampling = true;
  std::uint64_t seed = 1;
  ToneMap tone_map = ToneMap::Aces;
  double exposure = 1.0;
  int threads = 0;      // CPU worker count in the reference; ignored on the GPU
  int tile_size = 16;   // CPU tile edge in the reference; ignored on the GPU
  bool use_bvh = true;  // false selects the brute-force kernel
  // Multiple importance sampling of next-event estimation and BSDF sampling (power
  // heuristic). No counterpart in the reference, which lists it as future work;
  // off by default, and only with light_sampling.
  bool mis = false;
  bool operator==(const RenderSettings&) const = default;
};

struct Background {
  enum class Kind : std::uint8_t { Gradient = 0, Solid = 1 } kind = Kind::Gradient;
  D3 top{0.5, 0.7, 1.0};
  D3 bottom{1, 1, 1};
  double intensity = 1;
  bool operator==(const Background&) const = default;
};

// --- materials --------------------------------------------------------------
struct Texture {
  D3 a{0.5};
  D3 b{0.5};
  double checker_scale = 0;
  bool operator==(const Texture&) const = default;
};
struct Lambertian { Texture albedo; bool operator==(const Lambertian&) const = default; };
struct Metal { D3 albedo{0.9}; double roughness = 0; bool operator==(const Metal&) const = default; };
struct Dielectric { double ior = 1.5; D3 tint{1}; bool operator==(const Dielectric&) const = default; };
struct Emissive {
  D3 color{1};
  double intensity = 1;
  bool two_sided = false;
  bool operator==(const Emissive&) const = default;
};
using Material = std::variant<Lambertian, Metal, Dielectric, Emissive>;

inline D3 emission_of(const Material& m) {
  if (const auto* e = std::get_if<Emissive>(&m)) return e->color * e->intensity;
  return {};
}

// --- shapes -----------------------------------------------------------------
struct SphereDesc { D3 center; double radius = 1; bool operator==(const SphereDesc&) const = default; };
struct PlaneDesc { D3 point; D3 normal{0, 1, 0}; bool operator==(const PlaneDesc&) const = default; };
struct TriangleDesc { D3 v0, v1{1, 0, 0}, v2{0, 1, 0}; bool operator==(const TriangleDesc&) const = default; };
struct QuadDesc { D3 corner; D3 u{1, 0, 0}, v{0, 0, 1}; bool operator==(const QuadDesc&) const = default; };
struct BoxDesc { D3 min{-0.5}, max{0.5}; double rotate_y = 0; bool operator==(const BoxDesc&) const = default; };
struct MeshDesc {
  enum class Source : std::uint8_t { Icosphere = 0, Torus = 1, ObjFile = 2 } source = Source::Icosphere;
  int subdivisions = 3;
  double major_radius = 1, minor_radius = 0.35;
  int segments = 48;
  int segments_v = 0;  // extension: 0 => max(3, segments / 2) as in the reference
  std::string path;
  bool smooth = true;
  D3 scale{1, 1, 1};
  double rotate_y = 0;
  D3 translate{0, 0, 0};
  bool operator==(const MeshDesc&) const = default;
};

struct ObjectDesc {
  std::string name;
  std::string material;
  std::variant<SphereDesc, PlaneDesc, TriangleDesc, QuadDesc, BoxDesc, MeshDesc> shape;
  bool operator==(const ObjectDesc&) const = default;
};

struct PointLightDesc {
  std::string name;
  D3 position;
  D3 intensity{10};
  bool operator==(const PointLightDesc&) const = default;
};

struct NamedMaterial {
  std::string name;
  Material material;
  bool operator==(const NamedMaterial&) const = default;
};

struct SceneDesc {
  std::string name = "untitled";
  CameraDesc camera;
  RenderSettings render;
  Background background;
  std::vector<NamedMaterial> materials;
  std::vector<ObjectDesc> objects;
  std::vector<PointLightDesc> lights;
  std::string base_dir;  // resolves relative OBJ paths; not serialised

  const NamedMaterial* find_material(const std::string& n) const {
    for (const auto& m : materials)
      if (m.name == n) return &m;
    return nullptr;
  }
  bool operator==(const SceneDesc& o) const {
    return name == o.name && camera == o.camera && render == o.render && background == o.background &&
           materials == o.materials && objects == o.objects && lights == o.lights;
  }
};

}  // namespace rtg
