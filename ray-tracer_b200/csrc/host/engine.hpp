#pragma once
// GPU render engine: resident scenes, the continuous wavefront, framebuffers and
// the progressive pass schedule.
//
// Every render is a job; every pass of a job is a segment. Segments of any number
// of jobs share one persistent pool of path slots: the host appends segments (and
// jobs) between iterations and the device hands free slots to them in priority
// order, so the pool stays full across pass boundaries, between the jobs of a
// batch and between requests that arrive while others render. A job's finished
// segments are folded into its framebuffer strictly in pass order, so results are
// bit-identical whatever else shares the wavefront.
//
// The pass schedule, progress record and callback contract are the reference
// Renderer's (src/rendering/renderer.cpp:58-105, include/raytracer/rendering/renderer.hpp:25-56):
// pass sizes min(remaining, max(1, done), max_pass_spp) => 1, 1, 2, 4, 8, ...;
// the callback runs on the calling thread after each pass, when the framebuffer
// holds exactly the passes reported so far (later passes may be tracing, but they
// touch only their own radiance slots); cancellation is checked between
// wavefront iterations and unfinished passes are dropped whole, so every pixel
// keeps the same sample count.
#include <chrono>
#include <cstdint>
#include <deque>
#include <functional>
#include <map>
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
  double extend_ms = 0, shade_ms = 0, shadow_ms = 0, accumulate_ms = 0, direct_ms = 0, plan_ms = 0;
  std::uint64_t extend_launches = 0;
};

// One uploaded scene: device copy of the flattened arrays plus the host compile.
struct GpuScene {
  std::shared_ptr<const CompiledScene> host;  // shared with the caller's host scene (not copied)
  std::vector<std::uint32_t> slot_prim;  // slot -> primitive id (ray API)
  std::int32_t root = kNoRoot;
  std::int32_t n_slots = 0, n_planes = 0, n_lights = 0;
  std::int32_t n_interior = 0, n_wide = 0, n_wide8 = 0;  // DevNode / DevNode4 / DevNode8 records
  void* block = nullptr;       // one device allocation holding the arrays below
  DevNode* nodes = nullptr;
  DevNode4* nodes4 = nullptr;  // four-wide copy of the tree (any-hit queries)
  std::int32_t root4 = kNoRoot;
  DevNode8* nodes8 = nullptr;  // compressed eight-wide copy (built when an eight-wide walk is selected)
  std::int32_t root8 = kNoRoot;
  bool has_wide8 = false;      // uploaded with the eight-wide tree (and its slot order)
  float4* prims = nullptr;
  std::uint32_t* slot_material = nullptr;
  float4* slot_normals = nullptr;
  DevPlane* planes = nullptr;
  DevMaterial* materials = nullptr;
  DevLight* lights = nullptr;
  double* prims64 = nullptr;   // ray-query refinement geometry (lazily uploaded)
  double* planes64 = nullptr;
  std::size_t device_bytes = 0;
  int jobs_open = 0;           // jobs in the wavefront that use this scene
  BvhStats bvh;                // of the tree on the device (host or device build)
  bool device_built = false;   // the BVH was built on the GPU
};

// Per-job device framebuffer.
struct GpuFrame {
  int width = 0, height = 0;
  double* sum = nullptr;
  double* sumsq = nullptr;
  std::uint32_t* count = nullptr;
  std::uint64_t* stats = nullptr;
  std::size_t bytes() const { return std::size_t(width) * height * (64 + 4) + 32; }
};

using PassCallback = std::function<void(const RenderProgress&)>;

struct EngineConfig {
  std::uint32_t pool_paths = 1u << 20;          // wavefront path slots (<= 2^23)
  std::uint64_t max_pass_samples = 1ull << 27;  // radiance slots shared by the open segments
  std::uint32_t backlog_pools = 3;              // keep this many pools of samples open for generation
  LaunchShape shape;
  bool time_kernels = false;                    // CUDA events around every launch
  bool count_traversal = false;                 // node / primitive counters
  // Ray queries (trace_closest and the no-alloc variant) report the winning
  // primitive's distance recomputed in double; off: the fp32 traversal's own t,
  // exactly what the wavefront's closest-hit stage hands to shading.
  bool refine_hits = true;
};

// A render request for the scheduler.
struct JobSpec {
  int scene_id = 0;
  RenderSettings settings;
  RenderOptions opts;
  int priority = 0;  // lower is served first (previews before finals)
};

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  int device() const { return device_; }
  // Frees the wavefront pool so the next render allocates it with the current config.
  // Requires an idle wavefront.
  void reset_wave();
  cudaStream_t stream() const { return stream_; }
  EngineConfig& config() { return cfg_; }
  // Scenes uploaded now get the eight-wide tree: an eight-wide walk is selected.
  bool wants_wide8() const { return cfg_.shape.closest_tree == 8 || cfg_.shape.shadow_tree == 8; }

  // Host-built scenes are flattened on the host. Scenes compiled without a BVH
  // (BvhBuild::Defer / Auto) get it built on the GPU (add_scene_gpu_bvh) from
  // kGpuBuildMinPrims primitives up, and on the host below that; either way the tree
  // is the same.
  int add_scene(std::shared_ptr<const CompiledScene> scene);
  // Builds the scene's BVH on the GPU (device/bvh_gpu.h), whether or not the host
  // compile holds one, and derives the device layout there.
  int add_scene_gpu_bvh(std::shared_ptr<const CompiledScene> scene);
  // Several scenes at once: flattened in parallel on the host, then copied.
  std::vector<int> add_scenes(const std::vector<std::shared_ptr<const CompiledScene>>& scenes);
  void release_scene(int id);
  GpuScene& scene(int id);
  bool has_scene(int id) const { return scenes_.count(id) != 0; }

  // Plain renderer: one job; its passes overlap in the wavefront.
  RenderProgress render(int scene_id, const RenderSettings& settings, const RenderOptions& opts,
                        const PassCallback& on_pass, const volatile std::int32_t* cancel);

  // Batched renderer: every job's passes share the wavefront.
  struct BatchJob {
    int scene_id;
    RenderSettings settings;
  };
  std::vector<RenderProgress> render_batch(const std::vector<BatchJob>& jobs, const RenderOptions& opts,
                                           const volatile std::int32_t* cancel, const PassCallback& on_pass = {});

  // Results of the last render (plain) or of job `j` of the last batch.
  const GpuFrame& frame(int job = -1) const;
  void read_mean(int job, double* rgb) const;
  void read_moments(int job, double* sum, double* sumsq, std::uint32_t* count) const;
  void read_image(int job, ToneMap op, double exposure, std::uint8_t* rgb) const;
  // Several jobs' images: every resolve, then one device-to-host copy into pinned
  // memory and one synchronisation, then copies out to rgb[k] on the host cores.
  void read_images(int n, const int* jobs, const ToneMap* ops, const double* exposures, std::uint8_t* const* rgb);
  void read_mean_frame(const GpuFrame& f, double* rgb) const;
  void read_image_frame(const GpuFrame& f, ToneMap op, double exposure, std::uint8_t* rgb) const;
  const RenderStats& stats() const { return stats_; }

  // ---- serving: requests live in the wavefront across calls ----
  // Opens a request; it starts tracing on the next pump. Returns its handle (> 0).
  int submit(const JobSpec& spec);
  struct PassEvent {
    int request;
    RenderProgress progress;
  };
  // Runs wavefront iterations until `budget_ms` of host time has passed, an event
  // is ready and `return_on_event` is set, or no request has work left. Appends
  // the pass events (in completion order) to `events`.
  void pump(double budget_ms, bool return_on_event, std::vector<PassEvent>& events);
  void cancel_request(int request);
  // Frees a finished or cancelled request's framebuffer.
  void release_request(int request);
  bool request_exists(int request) const { return jobs_.count(request) != 0; }
  const GpuFrame& request_frame(int request) const;
  const RenderProgress& request_progress(int request) const;
  // Footprint a request adds on the device (framebuffer + radiance of one pass).
  std::size_t request_bytes(const JobSpec& spec) const;
  std::size_t open_requests() const { return serve_open_; }
  // Maps `bytes` of device memory into the engine's pool ahead of time, so
  // framebuffer allocations of arriving requests never wait for the driver.
  void reserve_pool(std::size_t bytes);
  std::size_t requests_rendering() const;
  bool wave_idle() const { return jobs_.empty() || all_jobs_drained(); }

  // Ray queries against one scene: rays = n x 8 floats (o, tmin, d, tmax).
  void trace_closest(int scene_id, const float* rays, std::uint64_t n, bool brute, float* t, std::int32_t* prim,
                     std::int32_t* is_plane, float* bary);
  void trace_any(int scene_id, const float* rays, std::uint64_t n, bool brute, std::uint8_t* occluded);
  // Descriptor of one scene for a ray query (a host struct; allocates nothing).
  RtgSceneDev query_descriptor(int scene_id, bool brute);

 private:
  struct Wave;
  struct Job {
    int handle = 0;
    int desc_slot = -1;
    int scene_id = 0;
    RenderSettings settings;
    RenderOptions opts;
    int priority = 0;
    std::uint64_t seq = 0;          // submission order
    GpuFrame frame;
    std::uint64_t pixels = 0;
    std::uint32_t target = 0, issued = 0, done = 0;
    int passes_issued = 0;
    RenderProgress prog;
    std::deque<int> segs;           // issued segment slots, pass order
    bool cancelled = false;
    bool direct = false;
    bool serving = false;           // owned by the serving API (else by a render call)
    PassCallback on_pass;
    std::chrono::steady_clock::time_point t0;
    bool drained() const { return segs.empty() && (cancelled || done >= target); }
  };
  struct Seg {
    bool used = false;
    int job = 0;                    // job handle
    DevSegment d{};
    std::uint64_t rad_begin = 0;
    bool in_gen = false;
    bool complete = false;
    bool abandoned = false;         // its job was cancelled: drop the result
    std::uint64_t done = 0, generated = 0;  // last snapshot
    std::uint64_t assigned_at = 0;  // first iteration whose plan sees the slot's records
    std::uint64_t closed_at = 0;    // first iteration whose plan no longer lists it (cancelled)
  };

  int add_flat(std::shared_ptr<const CompiledScene> scene, FlatScene flat);
  // Byte offsets of a flattened scene's arrays in its device block (and in its
  // pinned staging copy): nodes, nodes4, prims, slot_material, slot_normals,
  // planes, materials, lights, nodes8, each 256-byte aligned.
  static constexpr int kSceneParts = 9;
  struct StagedParts {
    std::size_t at[kSceneParts], bytes[kSceneParts], total;
  };
  static StagedParts staged_parts(const FlatScene& f);
  // The host copy into pinned staging, as pieces of at most 1 MiB so that one
  // large scene is copied by many threads.
  struct StagePiece {
    unsigned char* dst;
    const unsigned char* src;
    std::size_t bytes;
  };
  static void stage_pieces(const FlatScene& f, const StagedParts& p, unsigned char* dst, std::vector<StagePiece>& out);
  static void copy_pieces(const std::vector<StagePiece>& pieces);  // on the host cores
  static void stage_flat(const FlatScene& f, const StagedParts& p, unsigned char* dst);
  // Allocates the scene's device block, queues its copy from `staged` (pinned,
  // laid out by `p`) and registers the scene.
  int register_flat(std::shared_ptr<const CompiledScene> scene, FlatScene flat, const StagedParts& p,
                    const unsigned char* staged);
  // One of the two pinned upload buffers, grown to `bytes`, once its previous copy
  // is done; the caller records upload_ev_[b] after queuing its copy from it.
  // want >= 0 picks that buffer instead of alternating (batch uploads use buffer 0,
  // so only one buffer grows to a whole batch).
  unsigned char* upload_staging(std::size_t bytes, int& b, int want = -1);
  void ensure_wave();
  GpuFrame make_frame(int w, int h);
  void free_frame(GpuFrame& f);
  RtgSceneDev job_descriptor(const GpuScene& sc, const RenderSettings& s, const GpuFrame& f) const;

  // Scheduler.
  int open_job(const JobSpec& spec, bool serving, PassCallback cb);
  void close_job(Job& j);
  bool all_jobs_drained() const;
  std::uint32_t next_pass_size(const Job& j) const;
  bool issue_pass(Job& j);          // false if no radiance space or slot is free now
  void refill();
  bool run_direct_pass(Job& j);     // false if no radiance space is free now
  void process_snapshot(std::uint64_t iter, std::vector<PassEvent>* events);
  void retire_segments(Job& j, std::vector<PassEvent>* events);
  void launch_one_iteration();
  void drain(const volatile std::int32_t* cancel, std::vector<PassEvent>* events, double budget_ms,
             bool return_on_event);
  void abort_all();                 // drop every open segment (after a cancel) and reset the pool
  void stage(void* dst, const void* src, std::size_t n);
  void write_gen_table();
  void begin_stats();
  void end_stats();
  void finish_timing();  // records the end event and fills stats_.device_ms

  int device_;
  cudaStream_t stream_ = nullptr;
  // GPU BVH builds run here, beside the wavefront: their per-level
  // synchronisation waits for the build alone, not for queued render iterations.
  cudaStream_t build_stream_ = nullptr;
  cudaMemPool_t pool_ = nullptr;  // framebuffers and read-back staging
  // Pinned staging for scene uploads (two alternating buffers).
  unsigned char* upload_host_[2] = {nullptr, nullptr};
  std::size_t upload_cap_[2] = {0, 0};
  cudaEvent_t upload_ev_[2] = {nullptr, nullptr};
  bool upload_pending_[2] = {false, false};
  // Pinned read-back buffer of read_images (grown on demand).
  unsigned char* readback_host_ = nullptr;
  std::size_t readback_cap_ = 0;
  int upload_next_ = 0;
  std::size_t pool_reserved_ = 0;
  bool bvh_preloaded_ = false;
  cudaEvent_t ev_begin_ = nullptr, ev_end_ = nullptr;
  EngineConfig cfg_;
  std::unordered_map<int, std::unique_ptr<GpuScene>> scenes_;
  int next_scene_ = 1;
  std::unique_ptr<Wave> wave_;
  std::vector<GpuFrame> frames_;  // frames of the last render / batch
  std::vector<int> rendering_;    // handles of the render / batch in progress (pass callbacks read these)
  std::vector<RenderSettings> frame_settings_;
  RenderStats stats_;
  std::map<int, Job> jobs_;        // open jobs by handle
  std::vector<Seg> segs_;          // by segment slot
  int next_job_ = 1;
  std::uint64_t job_seq_ = 0;
  std::size_t serve_open_ = 0;
  int mis_jobs_ = 0;               // open jobs with multiple importance sampling
  bool gen_dirty_ = false;
  WaveCounters last_counters_{};   // from the latest snapshot
  WaveCounters base_counters_{};   // at the start of the current render
};

}  // namespace rtg
