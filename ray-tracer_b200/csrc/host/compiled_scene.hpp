#pragma once
// Render-ready scene on the host, in double precision.
//
// compile_scene() flattens a SceneDesc exactly as the reference's Scene::compile
// does (src/core/scene.cpp:31-137): objects in order; quads -> 2 triangles,
// boxes -> 12, meshes -> their faces; degenerate triangles dropped; planes kept
// out of the BVH; the light list is point lights first, then emissive primitives
// in primitive order. Primitive ids (indices into `prims`) are therefore the
// reference's hit ids. The device copy is produced from this by flatten.hpp.
#include <cstdint>
#include <string>
#include <vector>

#include "host/bvh_build.hpp"
#include "host/scene_desc.hpp"

namespace rtg {

struct Prim {
  enum Kind : std::uint8_t { kSphere = 0, kTriangle = 1 } kind = kTriangle;
  bool smooth = false;            // triangle has vertex normals
  std::uint32_t material = 0;
  D3 a, b, c;                     // sphere: a = centre, b.x = radius; triangle: v0, v1, v2
  D3 n0, n1, n2;                  // vertex normals (smooth triangles)
  Box bounds() const;
  double area() const;            // 4 pi r^2 or |e1 x e2| / 2
};

struct PlanePrim {
  D3 point, normal;  // unit normal
  std::uint32_t material = 0;
};

struct PointLight {
  D3 position, intensity;
};

struct LightEntry {
  enum Kind : std::uint8_t { kPoint = 0, kEmitter = 1 } kind;
  std::uint32_t index;  // into point_lights or prims
};

// Thin-lens camera, set up as the reference's Camera::setup
// (include/raytracer/core/camera.hpp:29-51). Pixel (0, 0) is top-left.
struct CameraFrame {
  D3 origin, corner, du, dv, u{1, 0, 0}, v{0, 1, 0}, w{0, 0, 1};
  double lens_radius = 0;
  void setup(const CameraDesc& d, int width, int height);
};

struct BuildInfo {
  std::size_t triangles = 0, spheres = 0, planes = 0, degenerate_skipped = 0, lights = 0;
  BvhStats bvh;
};

struct CompiledScene {
  CameraDesc camera_desc;  // kept so a render at another resolution can redo the set-up
  CameraFrame camera;
  RenderSettings settings;
  Background background;
  std::vector<Material> materials;
  std::vector<Prim> prims;
  std::vector<PlanePrim> planes;
  std::vector<PointLight> point_lights;
  std::vector<LightEntry> lights;
  BinaryBvh bvh;
  bool bvh_built = true;  // false: compiled without the BVH (built on the GPU at upload)
  BuildInfo info;
};

// Scenes from this many primitives up build their BVH faster on the GPU than on
// the host (latency of the GPU build's level passes against the host build's work).
constexpr std::size_t kGpuBuildMinPrims = 32768;

// Where the BVH is built: in the compile (Host); at upload, on the GPU from
// kGpuBuildMinPrims primitives up and on the host below (Defer: `bvh` stays empty
// here); or chosen by size here (Auto: small scenes built now, large ones deferred).
enum class BvhBuild { Host, Defer, Auto };
CompiledScene compile_scene(const SceneDesc& desc, BvhBuild where = BvhBuild::Host);

}  // namespace rtg
