/*
 * rtg — C ABI of the B200 path-tracing hot path.
 *
 * Plain C types only (no CUDA or C++ types cross this boundary). Every function
 * returns RTG_OK (0) or a negative RTG_ERR_* code; the message of the last
 * failure on a context is available from rtg_last_error(ctx). A context owns one
 * CUDA stream on one device and is driven by one host thread at a time.
 *
 * Each entry point names the reference interface it replaces
 * (Kaushlendra-Kumar/ray-tracer, paths relative to that project).
 */
#ifndef RTG_H
#define RTG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RTG_OK 0
#define RTG_ERR_INVALID (-1)   /* bad argument or unknown id */
#define RTG_ERR_SCENE (-2)     /* scene JSON rejected (parse or validation); message names the field */
#define RTG_ERR_CUDA (-3)      /* CUDA runtime failure */
#define RTG_ERR_NO_DEVICE (-4) /* no usable CUDA device */
#define RTG_ERR_DEVICE (-5)    /* a kernel reported an error through its status word */
#define RTG_ERR_BUSY (-6)      /* another render is running on this context */
#define RTG_ERR_LIMIT (-7)     /* a size exceeds a documented maximum */

typedef struct rtg_context rtg_context;
typedef int32_t rtg_scene_id;

/* RenderSettings (include/raytracer/core/scene_desc.hpp:20-35). threads and
 * tile_size are accepted for compatibility and ignored on the GPU. */
typedef struct rtg_settings {
  int32_t width, height, spp, max_depth, rr_min_depth;
  int32_t integrator; /* 0 path, 1 direct, 2 normals */
  int32_t light_sampling; /* 0 off, 1 next-event estimation, 2 NEE + multiple importance
                           * sampling with BSDF sampling (power heuristic; no reference
                           * counterpart: its docs/performance.md lists MIS as future work) */
  int32_t tone_map;   /* 0 clamp, 1 reinhard, 2 aces */
  uint64_t seed;
  double exposure;
  int32_t threads, tile_size;
  int32_t use_bvh;    /* 0: brute-force intersection */
  int32_t reserved;
} rtg_settings;

/* RenderOptions (include/raytracer/rendering/renderer.hpp:41-44). */
typedef struct rtg_render_options {
  int32_t progressive;  /* passes of 1, 1, 2, 4, ... samples */
  int32_t max_pass_spp; /* cap on samples per pass (reference default 32) */
} rtg_render_options;

/* RenderProgress (include/raytracer/rendering/renderer.hpp:25-33). */
typedef struct rtg_progress {
  int32_t pass;
  uint32_t spp_done;
  int32_t spp_target;
  int32_t finished;
  int32_t cancelled;
  int32_t reserved;
  double elapsed_ms;
  uint64_t rays; /* closest-hit + shadow rays so far */
} rtg_progress;

/* RenderStatsSnapshot (include/raytracer/rendering/renderer.hpp:35-39), plus the
 * device counters behind the roofline figures. */
typedef struct rtg_stats {
  uint64_t camera_samples, rays, shadow_rays, rr_terminated, invalid_samples, passes;
  uint64_t iterations, node_visits, prim_tests, sphere_tests, extend_launches; /* closest-hit kernel */
  uint64_t shadow_node_visits, shadow_prim_tests, shadow_sphere_tests;         /* any-hit kernel */
  uint64_t kernel_launches; /* every kernel of this library launched by the render */
  double elapsed_ms;        /* host wall time of the render call */
  double device_ms;         /* CUDA-event time on the context's stream, first to last launch */
  double extend_ms, shade_ms, shadow_ms, accumulate_ms, direct_ms; /* per-kernel event time (time_kernels) */
  double plan_ms;           /* generation-plan kernel (time_kernels) */
} rtg_stats;

/* SceneBuildInfo (include/raytracer/core/scene.hpp:24-27) and BvhBuildStats
 * (include/raytracer/geometry/bvh.hpp:28-32). */
typedef struct rtg_scene_info {
  uint64_t primitives, triangles, spheres, planes, degenerate_skipped, lights;
  uint64_t bvh_nodes, bvh_leaves, bvh_max_depth, bvh_max_leaf, device_bytes;
  double bvh_build_ms, bvh_sah_cost;
} rtg_scene_info;

/* Called on the rendering thread after each pass, when the framebuffer holds
 * exactly the passes reported so far: the framebuffer accessors below may be
 * called from inside it (later passes may be tracing meanwhile; they do not touch
 * the framebuffer until the callback returns).
 * ProgressFn (include/raytracer/rendering/renderer.hpp:46-48). */
typedef void (*rtg_pass_fn)(void* user, const rtg_progress* progress);

/* ---- scene-level entry points (the editor / WASM FFI, apps/rt_wasm.cpp:117-128) ---- */

/* "" if the scene parses and validates, else the first problem
 * (rt_validate, apps/rt_wasm.cpp:117-126; parse_scene + validate_scene,
 * src/io/scene_io.cpp:380-492). The returned string lives until the next call
 * on the same thread. */
const char* rtg_validate(const char* scene_json);

/* Normalised scene JSON (scene_to_json, src/io/scene_io.cpp:321-378): the CLI's
 * --dump-scene. Writes at most cap bytes including the terminator; returns the
 * full length (excluding the terminator) or a negative error. */
int64_t rtg_scene_dump(const char* scene_json, char* out, size_t cap);

/* ---- host-side compile (no GPU needed) ---- */

/* A compiled scene held on the host: Scene::compile (src/core/scene.cpp:31-137)
 * including the binned-SAH BVH build (src/geometry/bvh.cpp:133-163). */
typedef struct rtg_host_scene rtg_host_scene;

/* Parse + validate + compile. On RTG_ERR_SCENE the message goes to err (cap bytes). */
int rtg_compile(const char* scene_json, const char* base_dir, rtg_host_scene** out, char* err, size_t err_cap);
/* rtg_compile with flags. RTG_COMPILE_DEFER_BVH leaves the BVH out of the host
 * compile (Bvh::build, src/geometry/bvh.cpp:133-163, is skipped; the view below
 * then has no nodes): rtg_scene_upload builds the same tree at upload, on the GPU
 * for scenes of 32,768 primitives or more and on the host below that, where the
 * host is faster. */
#define RTG_COMPILE_DEFER_BVH 1u
/* RTG_COMPILE_AUTO_BVH: the compile builds the tree itself for scenes under 32,768
 * primitives and defers it to the GPU build for larger ones, so the host work stays
 * on the compiling thread (not on the thread that uploads). */
#define RTG_COMPILE_AUTO_BVH 2u
int rtg_compile_flags(const char* scene_json, const char* base_dir, uint32_t flags, rtg_host_scene** out, char* err,
                      size_t err_cap);
void rtg_host_scene_free(rtg_host_scene* scene);

/* Read-only view of a compiled scene in the reference's own layout and order
 * (double precision): primitives in Scene::primitives order, planes, BVH nodes in
 * the depth-first array of Bvh::nodes() with Bvh::prim_indices(), the light list
 * (point lights first, then emitters), materials and the camera. Arrays stay
 * valid until rtg_host_scene_free. Record layouts:
 *   prims        24 doubles: kind (0 sphere, 1 triangle), material, smooth,
 *                a(3), b(3), c(3), n0(3), n1(3), n2(3), 0, 0, 0
 *                (sphere: a = centre, b.x = radius; triangle: v0, v1, v2)
 *   planes        8 doubles: point(3), unit normal(3), material, 0
 *   nodes        10 doubles: lo(3), hi(3), first, count (0 = interior), axis, 0
 *   lights        2 uint32: kind (0 point, 1 emitter), index
 *   point_lights  6 doubles: position(3), intensity(3)
 *   materials    16 doubles: kind (0 lambertian, 1 metal, 2 dielectric, 3 emissive),
 *                a(3) (albedo | metal albedo | tint | emitter colour), b(3) (checker
 *                albedo 2), checker_scale, roughness, ior, intensity, two_sided, 0...
 *   camera       19 doubles: origin(3), corner(3), du(3), dv(3), u(3), v(3), lens radius
 *   background    8 doubles: kind (0 gradient, 1 solid), top(3), bottom(3), intensity */
typedef struct rtg_scene_view {
  uint64_t n_prims, n_planes, n_nodes, n_order, n_lights, n_point_lights, n_materials;
  const double* prims;
  const double* planes;
  const double* nodes;
  const uint32_t* order;
  const uint32_t* lights;
  const double* point_lights;
  const double* materials;
  double camera[19];
  double background[8];
  rtg_settings settings;
  uint64_t degenerate_skipped, bvh_max_depth, bvh_leaves, bvh_max_leaf;
  double bvh_sah_cost;
} rtg_scene_view;
int rtg_host_scene_view(const rtg_host_scene* scene, rtg_scene_view* out);

/* ---- context ---- */
int rtg_context_create(int device, rtg_context** out);
void rtg_context_destroy(rtg_context* ctx);
const char* rtg_last_error(const rtg_context* ctx);
int rtg_device_count(void);

/* ---- scenes (Scene::compile, src/core/scene.cpp:31-137; load_scene / parse_scene,
 *      src/io/scene_io.cpp:480-502) ---- */

/* Parse, validate, compile and upload. The BVH is built on the host for scenes under
 * 32,768 primitives and on the GPU for larger ones (RTG_COMPILE_AUTO_BVH): the same
 * tree either way. base_dir resolves relative OBJ paths (may be NULL). */
int rtg_scene_load_json(rtg_context* ctx, const char* scene_json, const char* base_dir, rtg_scene_id* out);
int rtg_scene_load_file(rtg_context* ctx, const char* path, rtg_scene_id* out);
/* Flatten a host-compiled scene to the device layout and copy it to HBM. The
 * host scene stays owned by the caller. */
int rtg_scene_upload(rtg_context* ctx, const rtg_host_scene* scene, rtg_scene_id* out);
/* Uploads n host scenes at once: they are flattened for the device in parallel
 * on the host cores, then copied. out receives n ids (no counterpart in the
 * reference: the batched form). */
int rtg_scene_upload_batch(rtg_context* ctx, int32_t n, const rtg_host_scene* const* scenes, rtg_scene_id* out);
/* Uploads a host scene with its BVH built on the GPU: the binned-SAH tree of
 * Bvh::build (src/geometry/bvh.cpp:28-163), node for node, and the device layout
 * derived from it there (byte-identical to what rtg_scene_upload makes from a host
 * build). Large host scenes compiled with RTG_COMPILE_DEFER_BVH take this path in
 * rtg_scene_upload too. It replaces the host build for scenes that are not
 * resident yet, where that build dominates the time to the first pass. Builds run
 * on their own high-priority stream, beside any render in flight. */
int rtg_scene_upload_gpu_bvh(rtg_context* ctx, const rtg_host_scene* scene, rtg_scene_id* out);
/* Reads back one part of a scene's device layout (tests and tools; no reference
 * counterpart). Copies min(cap, size) bytes to out (out may be NULL) and returns
 * the part's full size in bytes, or a negative error. */
enum {
  RTG_LAYOUT_NODES = 0,         /* DevNode, 64 B each (interior nodes, depth-first) */
  RTG_LAYOUT_NODES4 = 1,        /* DevNode4, 128 B each */
  RTG_LAYOUT_PRIMS = 2,         /* 3 float4 per slot */
  RTG_LAYOUT_SLOT_MATERIAL = 3, /* uint32 per slot */
  RTG_LAYOUT_SLOT_NORMALS = 4,  /* 3 float4 per slot */
  RTG_LAYOUT_PLANES = 5,
  RTG_LAYOUT_MATERIALS = 6,
  RTG_LAYOUT_LIGHTS = 7,
  RTG_LAYOUT_SLOT_PRIM = 8,     /* uint32 per slot: primitive id */
  RTG_LAYOUT_ROOTS = 9,         /* int32[5]: root link, four-wide root link, slots, built on the GPU,
                                 * eight-wide root link */
  RTG_LAYOUT_NODES8 = 10        /* DevNode8, 80 B each (compressed eight-wide nodes, breadth-first) */
};
int64_t rtg_scene_layout(rtg_context* ctx, rtg_scene_id scene, int32_t part, void* out, uint64_t cap);
/* No counterpart in the reference. The device layout a host-compiled scene gets
 * at upload with an eight-wide walk selected (so with the eight-wide tree and its
 * slot order), computed on the host without a GPU (tests and tools): the same
 * parts and record formats as rtg_scene_layout (the built-on-GPU flag of ROOTS is 0).
 * Copies min(cap, size) bytes to out (out may be NULL) and returns the part's full
 * size in bytes; RTG_ERR_INVALID for an unknown part or a scene compiled without
 * its BVH. */
int64_t rtg_host_scene_layout(const rtg_host_scene* scene, int32_t part, void* out, uint64_t cap);
/* The scene file's own render settings. */
int rtg_scene_settings(rtg_context* ctx, rtg_scene_id scene, rtg_settings* out);
int rtg_scene_get_info(rtg_context* ctx, rtg_scene_id scene, rtg_scene_info* out);
int rtg_scene_release(rtg_context* ctx, rtg_scene_id scene);

/* ---- rendering (Renderer::render, src/rendering/renderer.cpp:58-105) ---- */

/* Blocking progressive render. `cancel` may be set to non-zero from any thread;
 * the render stops at the next wavefront iteration, drops the partial pass and
 * reports cancelled. `settings` may be NULL (use the scene's); `opts` may be NULL
 * (progressive, 32). */
int rtg_render(rtg_context* ctx, rtg_scene_id scene, const rtg_settings* settings, const rtg_render_options* opts,
               rtg_pass_fn on_pass, void* user, const volatile int32_t* cancel, rtg_progress* out);

/* Batched render: n jobs traced by one shared wavefront per pass (no reference
 * counterpart; each job's image equals its plain render bit for bit). */
int rtg_render_batch(rtg_context* ctx, int32_t n, const rtg_scene_id* scenes, const rtg_settings* settings,
                     const rtg_render_options* opts, const volatile int32_t* cancel, rtg_progress* out);

/* Results of the last render (job = -1 or 0) or of job j of the last batch.
 * Framebuffer::mean (include/raytracer/rendering/framebuffer.hpp:35-38): w*h*3 doubles. */
int rtg_framebuffer_mean(rtg_context* ctx, int32_t job, double* rgb);
/* Running sums: 4 doubles per pixel each (r, g, b, 0) and a sample count per pixel. */
int rtg_framebuffer_moments(rtg_context* ctx, int32_t job, double* sum, double* sumsq, uint32_t* count);
/* Renderer::image (src/rendering/renderer.cpp:107-110): tone-mapped sRGB8, w*h*3.
 * tone_map < 0 uses the render's settings (normals: clamp, exposure 1). */
int rtg_image_rgb8(rtg_context* ctx, int32_t job, int32_t tone_map, double exposure, uint8_t* rgb);
/* rtg_image_rgb8 for n jobs at once (no reference counterpart; Renderer::image
 * per job): image of jobs[k] into rgb[k]. All images are resolved on the device,
 * copied to the host in one transfer with one synchronisation, then copied out on
 * the host cores. tone_map and exposure as rtg_image_rgb8, for every job. */
int rtg_images_rgb8(rtg_context* ctx, int32_t n, const int32_t* jobs, int32_t tone_map, double exposure,
                    uint8_t* const* rgb);
int rtg_render_stats(rtg_context* ctx, rtg_stats* out);

/* ---- ray queries (Scene::intersect / intersect_brute / occluded,
 *      src/core/scene.cpp:176-234) ---- */

/* rays: n records of 8 floats (ox, oy, oz, tmin, dx, dy, dz, tmax). Outputs per
 * ray: t, primitive id (reference numbering; -1 on a miss; the plane index when
 * is_plane), is_plane, barycentrics (b1, b2). Output pointers may be NULL. */
int rtg_trace_closest(rtg_context* ctx, rtg_scene_id scene, const float* rays, uint64_t n, int32_t brute, float* t,
                      int32_t* prim, int32_t* is_plane, float* bary);
int rtg_trace_any(rtg_context* ctx, rtg_scene_id scene, const float* rays, uint64_t n, int32_t brute,
                  uint8_t* occluded);

/* No counterpart in the reference. rtg_trace_closest for callers that must not
 * allocate device memory during the call: a loop sharing the GPU with other
 * streams (freeing device memory synchronises the whole device), or a host that
 * pre-reserves all device memory in its own pool. Same arguments; at most
 * RTG_NOALLOC_MAX_RAYS rays per call (RTG_ERR_LIMIT beyond). The call makes the
 * context's GPU current (it stays current afterwards). Its rays and results pass
 * through one static device array of about 13 MiB that the library reserves on
 * every GPU it runs on until the process exits. The first call on a device sets
 * that array up (make it before any stream capture). All calls share the array,
 * so calls whose GPU work overlaps (other streams or contexts on the same
 * device) race. Ids and planes are those of rtg_trace_closest. t is refined in
 * double only when the scene's double-precision copy is already resident (after
 * an rtg_trace_closest call on the same scene with refine_hits on); otherwise it
 * is the fp32 traversal's own t, as with refine_hits = 0, since this entry point
 * never uploads that copy itself. */
#define RTG_NOALLOC_MAX_RAYS 262144
int rtg_trace_closest_noalloc(rtg_context* ctx, rtg_scene_id scene, const float* rays, uint64_t n, int32_t brute,
                              float* t, int32_t* prim, int32_t* is_plane, float* bary);

/* No counterpart in the reference. How many memory allocations (device, pooled
 * and pinned host) the library has asked CUDA for in this process so far: a
 * diagnostic for callers that must not allocate, to check an entry point. */
uint64_t rtg_allocation_count(void);

/* No counterpart in the reference. Measures read bandwidth on the context's GPU:
 * a zero-filled buffer of `bytes` (allocated for the call) is read `reps` times
 * per launch with 16-byte loads by a grid that fills every SM; *gbs receives the
 * best of five launches in GB/s. l1 = 0: loads bypass L1 and the grid shares the
 * buffer (>= 1 MiB); well under the L2 size (126 MB on B200) that is the L2 read
 * bandwidth, far above it the HBM read bandwidth. l1 = 1: L1-cached loads, every
 * block reads the whole buffer (4 KiB to 128 KiB), so it is the aggregate L1 read
 * bandwidth. BVH traversal's node and primitive fetches are served from L1 and
 * L2, so these bound it, not HBM. */
int rtg_probe_read_bandwidth(rtg_context* ctx, uint64_t bytes, int32_t reps, int32_t l1, double* gbs);

/* ---- engine tuning (no reference counterpart) ---- */
typedef struct rtg_tuning {
  uint32_t pool_paths;       /* wavefront path slots (default 1 << 20) */
  uint32_t block;            /* threads per block of the wavefront kernels: 64, 128, 256 */
  uint64_t max_pass_samples; /* radiance slots shared by all passes in flight (default 1 << 27) */
  int32_t extend_blocks, shade_blocks, shadow_blocks; /* 0 = occupancy-derived persistent grid */
  int32_t time_kernels;      /* CUDA events around each kernel (rtg_stats.*_ms) */
  int32_t count_traversal;   /* node / primitive counters (rtg_stats.node_visits, prim_tests) */
  uint32_t backlog_pools;    /* samples kept open for generation, in pools (default 3) */
  uint32_t chained;          /* programmatic dependent launch between wavefront kernels (default 1) */
  uint64_t serve_budget_bytes; /* admission limit of the open requests' device footprint */
  uint64_t serve_reserve_bytes; /* part of that budget only priority-0 requests (previews) may use */
  int32_t refine_hits;       /* ray queries report t recomputed in double for the winning primitive
                              * (default 1); 0: the fp32 traversal's own t, the value the renderer's
                              * closest-hit stage hands to shading */
  int32_t closest_tree;      /* closest-hit walk: 2 the binary tree (default), 8 the compressed eight-wide tree */
  int32_t shadow_tree;       /* any-hit walk: 4 the four-wide tree (default), 8 the compressed eight-wide tree.
                              * Scenes get the eight-wide tree (and its slot order) when they are uploaded
                              * while either walk is 8; rendering or querying a scene without it with an
                              * eight-wide walk selected returns RTG_ERR_INVALID. */
  int32_t reserved;
} rtg_tuning;
int rtg_get_tuning(rtg_context* ctx, rtg_tuning* out);
int rtg_set_tuning(rtg_context* ctx, const rtg_tuning* in);
/* Picks pool_paths and block for a batch of renders (settings = NULL: each
 * scene's own) by timing a reduced copy of it (1/16 of the samples) under each
 * candidate, and applies the winner. Cached per GPU and workload signature in
 * $RTG_TUNE_CACHE (default $HOME/.cache/rtg/tuning.txt) when use_cache is set.
 * chosen, msamples_per_s and from_cache may be NULL. */
int rtg_autotune(rtg_context* ctx, int32_t n, const rtg_scene_id* scenes, const rtg_settings* settings,
                 const rtg_render_options* opts, int32_t use_cache, rtg_tuning* chosen, double* msamples_per_s,
                 int32_t* from_cache);

/* ---- serving (no reference counterpart: the reference renders one scene per
 * Renderer). Requests on resident scenes share one continuous wavefront with each
 * other: a request's passes are folded into its own framebuffer in pass order, so
 * its image is bit-identical to rendering it alone with rtg_render. Lower
 * priority values get free path slots first (previews before finals). ---- */
typedef int32_t rtg_request_id;
typedef struct rtg_request_event {
  rtg_request_id request;
  int32_t reserved;
  rtg_progress progress; /* after the pass that just finished */
} rtg_request_event;

/* Admission by footprint: RTG_ERR_LIMIT (and nothing opened) when the request's
 * framebuffer plus its first pass's radiance would take the open requests past
 * rtg_tuning.serve_budget_bytes, or, for priority > 0, past that budget less
 * serve_reserve_bytes (so previews are never locked out by finals).
 * settings = NULL: the scene's own. The request starts tracing on the next
 * rtg_serve_pump. */
int rtg_request_submit(rtg_context* ctx, rtg_scene_id scene, const rtg_settings* settings,
                       const rtg_render_options* opts, int32_t priority, rtg_request_id* out);
/* Runs the wavefront for up to budget_ms of host time, or until the first pass
 * event when return_on_event is set, or until no request has work. Writes up to
 * cap events in completion order (*n of them); events that do not fit are kept
 * for the next call. */
int rtg_serve_pump(rtg_context* ctx, double budget_ms, int32_t return_on_event, rtg_request_event* events,
                   int32_t cap, int32_t* n);
/* Stops a request; passes already reported stay in its framebuffer. */
int rtg_request_cancel(rtg_context* ctx, rtg_request_id request);
/* Frees a finished or cancelled request (RTG_ERR_BUSY while passes are in flight). */
int rtg_request_release(rtg_context* ctx, rtg_request_id request);
int rtg_request_progress(rtg_context* ctx, rtg_request_id request, rtg_progress* out);
/* The request's framebuffer: means (3 doubles per pixel) or the tone-mapped RGB8
 * image (tone_map < 0: the request's own settings, as rtg_image_rgb8). */
int rtg_request_mean(rtg_context* ctx, rtg_request_id request, double* rgb);
int rtg_request_image_rgb8(rtg_context* ctx, rtg_request_id request, int32_t tone_map, double exposure, uint8_t* rgb);
/* Maps the admission budget's worth of device memory into the context's pool
 * (rtg_request_submit does it on first use otherwise): a server calls it once at
 * start-up so no request's first allocation waits for the driver. */
int rtg_serve_prepare(rtg_context* ctx);
/* Device bytes the open requests hold against the admission budget, the number
 * of open requests, and how many of them still have passes to render or in flight. */
int rtg_serve_footprint(rtg_context* ctx, uint64_t* bytes, int32_t* open_requests, int32_t* rendering);

/* ---- image output (encode_png / write_image, src/io/image_io.cpp:45-70) ---- */
/* PNG bytes of an RGB8 image into out (cap bytes); returns the PNG size, or a
 * negative error. Pass out = NULL to query the size. */
int64_t rtg_encode_png(const uint8_t* rgb, int32_t width, int32_t height, uint8_t* out, size_t cap);

#ifdef __cplusplus
}
#endif

#endif /* RTG_H */
