#pragma once
// Host-visible launch interface of the sm_100a kernels (kernels.cu). Plain C++:
// no CUDA syntax, so the C++20 host code can include it.
#include <cstdint>

#include <cuda_runtime_api.h>

#include "device/layout.h"

namespace rtg {

// Device buffers of one wavefront (a pool of `capacity` path slots).
struct WaveBuffers {
  float4* st_a[2];
  float4* st_b[2];
  float4* st_c[2];
  uint4* st_d[2];
  float4* hits;
  float4* sh_a;
  float4* sh_b;
  float4* sh_c;
  float4* radiance;   // one float4 per sample of the current pass
  WaveCounters* cnt;
  std::uint32_t capacity;
};

// One pass: which descriptors (jobs) have work, and where their work begins.
struct PassTable {
  const RtgSceneDev* jobs;         // device array of job descriptors
  const std::uint32_t* job_ids;    // device: jobs with work in this pass
  const std::uint64_t* job_begin;  // device: first work index of each (strictly increasing)
  std::int32_t n;
};

struct LaunchShape {
  int extend_blocks = 0, shade_blocks = 0, shadow_blocks = 0;  // 0 = derived from the SM count
  int extend_block = 128;  // 64, 128 or 256
};

enum class Stage { Extend, Shade, Shadow };

// One stage of a wavefront iteration on `stream`; `parity` alternates 0/1
// between iterations. The stages must run in the order extend, shade, shadow.
cudaError_t launch_stage(Stage stage, const WaveBuffers& wb, const PassTable& pt, int parity, const LaunchShape& shape,
                         bool count_traversal, cudaStream_t stream);

// One wavefront iteration (generate+extend, shade, shadow) on `stream`.
cudaError_t launch_iteration(const WaveBuffers& wb, const PassTable& pt, int parity, const LaunchShape& shape,
                             bool count_traversal, cudaStream_t stream);

// Per-pixel reduction of a finished pass into the job's framebuffer.
cudaError_t launch_accumulate(const RtgSceneDev* job_dev, const RtgSceneDev& job_host, const float4* radiance,
                              cudaStream_t stream);

// Direct (Whitted) integrator: whole samples per thread (depth-first with an
// explicit stack). Writes each sample's radiance into `radiance`.
cudaError_t launch_direct(const PassTable& pt, std::uint64_t total_work, float4* radiance, WaveCounters* cnt,
                          cudaStream_t stream);

// Tone map + sRGB encode of a job's framebuffer means into rgb8 (w * h * 3).
cudaError_t launch_resolve(const RtgSceneDev* job_dev, std::uint64_t pixels, int tone_map, double exposure,
                           std::uint8_t* rgb8, double* mean_out, cudaStream_t stream);

// Ray queries for parity tests and the ray API. rays: 2 float4 per ray
// (origin, tmin), (direction, tmax). closest -> float4 (t, word, b1, b2) per ray.
cudaError_t launch_ray_closest(const RtgSceneDev* job_dev, const float4* rays, std::uint32_t n, float4* out,
                               int brute, cudaStream_t stream);
cudaError_t launch_ray_any(const RtgSceneDev* job_dev, const float4* rays, std::uint32_t n, std::uint32_t* out,
                           int brute, cudaStream_t stream);

}  // namespace rtg
