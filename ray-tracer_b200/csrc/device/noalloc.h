#pragma once
// Closest-hit ray query that allocates no device memory (see noalloc.cu).
#include <cstdint>

#include <cuda_runtime_api.h>

#include "device/layout.h"

namespace rtg {

// Largest ray batch one call accepts; fixes the size of the static device scratch.
constexpr std::uint64_t kNoAllocMaxRays = 1ull << 18;

// Traces `n` rays (host array, 8 floats each: origin, tmin, direction, tmax) against
// the scene described by `job` on `device`, through the static scratch array, and
// writes the per-ray results straight into the caller's host arrays (any of which
// may be null). tree 8 walks the eight-wide tree, otherwise the binary tree.
// Returns cudaErrorInvalidValue when n exceeds kNoAllocMaxRays.
cudaError_t noalloc_trace_closest(int device, const RtgSceneDev& job, const float* rays, std::uint64_t n, int brute,
                                  int tree, float* t, std::int32_t* prim, std::int32_t* is_plane, float* bary,
                                  cudaStream_t stream);

}  // namespace rtg
