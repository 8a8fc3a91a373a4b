#pragma once
// Host-visible launch interface of the sm_100a kernels (kernels.cu). Plain C++:
// no CUDA syntax, so the C++20 host code can include it.
#include <cstdint>

#include <cuda_runtime_api.h>

#include "device/layout.h"

namespace rtg {

// Device buffers of one continuous wavefront (a pool of `capacity` path slots)
// and the segment tables it draws new paths from.
struct WaveBuffers {
  float4* st_a[2];
  float4* st_b[2];
  float4* st_c[2];
  uint4* st_d[2];
  float* st_e[2];  // pdf of the direction a diffuse bounce sampled (read only by MIS jobs)
  float4* hits;
  float4* sh_a;
  float4* sh_b;
  float4* sh_c;
  float4* radiance;            // one float4 per sample of every open segment
  WaveCounters* cnt;
  const RtgSceneDev* jobs;     // job descriptors, indexed by job slot
  const DevSegment* segs;      // indexed by segment slot
  SegmentProgress* seg_prog;   // indexed by segment slot
  const GenTable* gen;         // host-written generation order
  GenPlan* plan;               // this iteration's generation plan
  WaveSnapshot* ring;          // pinned, host-mapped snapshot ring
  std::uint32_t ring_size;
  std::uint32_t capacity;      // at most 2^23 path slots
};

struct LaunchShape {
  int extend_blocks = 0, shade_blocks = 0, shadow_blocks = 0;  // 0 = derived from the SM count
  int extend_block = 128;  // 64, 128 or 256
  bool chained = true;     // programmatic dependent launch between the wavefront kernels
  bool mis = false;        // a job with multiple importance sampling is open (shade kernel variant)
  int closest_tree = 2;    // closest-hit walk: 2 the binary tree, 8 the compressed eight-wide tree
  int shadow_tree = 4;     // any-hit walk: 4 the four-wide tree, 8 the compressed eight-wide tree
};

enum class Stage { Plan, Extend, Shade, Shadow };

// One stage of a wavefront iteration on `stream`; `parity` alternates 0/1
// between iterations. The stages must run in the order plan, extend, shade, shadow.
cudaError_t launch_stage(Stage stage, const WaveBuffers& wb, int parity, const LaunchShape& shape, bool count_traversal,
                         cudaStream_t stream);

// One wavefront iteration (plan, generate+extend, shade, shadow) on `stream`.
cudaError_t launch_iteration(const WaveBuffers& wb, int parity, const LaunchShape& shape, bool count_traversal,
                             cudaStream_t stream);

// Per-pixel reduction of a finished segment into its job's framebuffer.
cudaError_t launch_accumulate(const RtgSceneDev* job_dev, std::uint64_t pixels, const DevSegment& seg,
                              const float4* radiance, cudaStream_t stream);

// Direct (Whitted) integrator over one whole segment: whole samples per thread
// (depth-first with an explicit stack). Writes each sample's radiance slot.
cudaError_t launch_direct(const RtgSceneDev* job_dev, const DevSegment& seg, float4* radiance, WaveCounters* cnt,
                          bool wide8, cudaStream_t stream);

// Framebuffer means (mean_out, 3 doubles per pixel) and/or their tone-mapped
// sRGB encoding (rgb8, 3 bytes per pixel); either output may be null.
cudaError_t launch_resolve(const double* fb_sum, const std::uint32_t* fb_count, std::uint64_t pixels, int tone_map,
                           double exposure, std::uint8_t* rgb8, double* mean_out, cudaStream_t stream);

// Ray queries for parity tests and the ray API. rays: 2 float4 per ray
// (origin, tmin), (direction, tmax). closest -> float4 (t, word, b1, b2) per ray.
// tree: 8 walks the eight-wide tree; otherwise the binary tree (closest hit) or
// the four-wide tree (any hit).
cudaError_t launch_ray_closest(const RtgSceneDev* job_dev, const float4* rays, std::uint32_t n, float4* out,
                               int brute, int tree, cudaStream_t stream);
cudaError_t launch_ray_any(const RtgSceneDev* job_dev, const float4* rays, std::uint32_t n, std::uint32_t* out,
                           int brute, int tree, cudaStream_t stream);

}  // namespace rtg
