#pragma once
// GPU render engine: resident scenes, the wavefront path pool, framebuffers and
// the progressive pass loop.
//
// The pass schedule, progress record and callback contract are the reference
// Renderer's (src/rendering/renderer.cpp:58-105, include/raytracer/rendering/renderer.hpp:25-56):
// pass sizes min(remaining, max(1, done), max_pass_spp) => 1, 1, 2, 4, 8, ...;
// the callback runs on the calling thread between passes with no kernel of this
// render in flight; cancellation is checked between wavefront iterations and a
// cancelled pass is dropped whole, so every pixel keeps the same sample count.
#include <chrono>
#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "device/wave.h"
#include "host/compiled_scene.hpp"
#include "host/flatten.hpp"

namespace rtg {

struct CudaFailure : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct RenderOptions {
  bool progressive = true;
  int max_pass_spp = 32;
};

struct RenderProgress {
  int pass = 0;
  std::uint32_t spp_done = 0;
  int spp_target = 0;
  double elapsed_ms = 0;
  std::uint64_t rays = 0;  // closest-hit + shadow rays so far
  bool finished = false;
  bool cancelled = false;
};

struct RenderStats {
  std::uint64_t camera_samples = 0, rays = 0, shadow_rays = 0, rr_terminated = 0, invalid_samples = 0, passes = 0;
  std::uint64_t iterations = 0, node_visits = 0, prim_tests = 0, sphere_tests = 0, kernel_launches = 0;
  std::uint64_t shadow_node_visits = 0, shadow_prim_tests = 0, shadow_sphere_tests = 0;
  double elapsed_ms = 0;
  double device_ms = 0;  // CUDA events on the engine stream around the whole render
  // Summed CUDA-event time of each kernel family (when kernel timing is on).
  double extend_ms = 0, shade_ms = 0, shadow_ms = 0, accumulate_ms = 0, direct_ms = 0;
  std::uint64_t extend_launches = 0;
};

// One uploaded scene: device copy of the flattened arrays plus the host compile.
struct GpuScene {
  CompiledScene host;
  std::vector<std::uint32_t> slot_prim;  // slot -> primitive id (ray API)
  std::int32_t root = kNoRoot;
  std::int32_t n_slots = 0, n_planes = 0, n_lights = 0;
  DevNode* nodes = nullptr;
  float4* prims = nullptr;
  std::uint32_t* slot_material = nullptr;
  float4* slot_normals = nullptr;
  DevPlane* planes = nullptr;
  DevMaterial* materials = nullptr;
  DevLight* lights = nullptr;
  double* prims64 = nullptr;   // ray-query refinement geometry (lazily uploaded)
  double* planes64 = nullptr;
  std::size_t device_bytes = 0;
};

// Per-render device framebuffer.
struct GpuFrame {
  int width = 0, height = 0;
  double* sum = nullptr;
  double* sumsq = nullptr;
  std::uint32_t* count = nullptr;
  std::uint64_t* stats = nullptr;
  std::size_t bytes() const { return std::size_t(width) * height * (64 + 4) + 8; }
};

using PassCallback = std::function<void(const RenderProgress&)>;

struct EngineConfig {
  std::uint32_t pool_paths = 1u << 20;     // wavefront path slots
  std::uint64_t max_pass_samples = 1ull << 27;  // radiance slots per pass
  LaunchShape shape;
  bool time_kernels = false;               // CUDA events around every launch
  bool count_traversal = false;            // node / primitive counters
};

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  int device() const { return device_; }
  // Frees the wavefront pool so the next render allocates it with the current config.
  void reset_wave();
  cudaStream_t stream() const { return stream_; }
  EngineConfig& config() { return cfg_; }

  int add_scene(CompiledScene scene);
  void release_scene(int id);
  GpuScene& scene(int id);
  bool has_scene(int id) const { return scenes_.count(id) != 0; }

  // Plain renderer: one scene per launch sequence.
  RenderProgress render(int scene_id, const RenderSettings& settings, const RenderOptions& opts,
                        const PassCallback& on_pass, const volatile std::int32_t* cancel);

  // Batched renderer: every job's passes share one persistent wavefront; pass p of
  // all jobs that still need samples runs as one pass.
  struct BatchJob {
    int scene_id;
    RenderSettings settings;
  };
  std::vector<RenderProgress> render_batch(const std::vector<BatchJob>& jobs, const RenderOptions& opts,
                                           const volatile std::int32_t* cancel);

  // Results of the last render (plain) or of job `j` of the last batch.
  const GpuFrame& frame(int job = -1) const;
  void read_mean(int job, double* rgb) const;
  void read_moments(int job, double* sum, double* sumsq, std::uint32_t* count) const;
  void read_image(int job, ToneMap op, double exposure, std::uint8_t* rgb) const;
  const RenderStats& stats() const { return stats_; }

  // Ray queries against one scene: rays = n x 8 floats (o, tmin, d, tmax).
  void trace_closest(int scene_id, const float* rays, std::uint64_t n, bool brute, float* t, std::int32_t* prim,
                     std::int32_t* is_plane, float* bary);
  void trace_any(int scene_id, const float* rays, std::uint64_t n, bool brute, std::uint8_t* occluded);
  // Descriptor of one scene for a ray query (a host struct; allocates nothing).
  RtgSceneDev query_descriptor(int scene_id, bool brute);

 private:
  struct Wave;
  void ensure_wave(std::uint64_t pass_samples);
  GpuFrame make_frame(int w, int h);
  void free_frame(GpuFrame& f);
  RtgSceneDev job_descriptor(const GpuScene& sc, const RenderSettings& s, const GpuFrame& f) const;
  // Runs one pass over the jobs in `table_host` (already staged); returns false if cancelled.
  bool run_pass(std::vector<RtgSceneDev>& jobs, const std::vector<std::uint32_t>& ids, std::uint64_t total,
                bool direct, const volatile std::int32_t* cancel);

  void finish_timing();  // records the end event and fills stats_.device_ms

  int device_;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev_begin_ = nullptr, ev_end_ = nullptr;
  EngineConfig cfg_;
  std::unordered_map<int, std::unique_ptr<GpuScene>> scenes_;
  int next_scene_ = 1;
  std::unique_ptr<Wave> wave_;
  std::vector<GpuFrame> frames_;  // frames of the last render / batch
  RenderStats stats_;
};

}  // namespace rtg
