#pragma once
// Engine autotuner: picks the wavefront pool size (1M to 8M path slots) and block size for a workload
// by rendering a reduced copy of it (every job at 1/16 of its samples) under each
// candidate and keeping the fastest by device time. Results are cached per GPU
// (name, SM count) and per workload signature (scene sizes, resolutions, sample
// counts, depths, integrators), in a text file: $RTG_TUNE_CACHE, else
// $HOME/.cache/rtg/tuning.txt.
#include <cstdint>
#include <string>
#include <vector>

#include "host/engine.hpp"

namespace rtg {

struct AutotuneResult {
  std::uint32_t pool_paths = 0;
  int block = 0;
  double msamples_per_s = 0;  // of the winning candidate on the reduced workload
  bool from_cache = false;
  int candidates_tried = 0;
  std::string key;
};

std::string workload_signature(Engine& e, const std::vector<Engine::BatchJob>& jobs);

// Leaves the winning configuration applied to the engine.
AutotuneResult autotune(Engine& e, const std::vector<Engine::BatchJob>& jobs, const RenderOptions& opts,
                        bool use_cache);

}  // namespace rtg
