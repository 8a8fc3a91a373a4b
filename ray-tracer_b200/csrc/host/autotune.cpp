#include "host/autotune.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <sys/stat.h>

namespace rtg {

namespace {

std::uint64_t fnv1a(std::uint64_t h, std::uint64_t v) {
  for (int k = 0; k < 8; ++k) {
    h ^= (v >> (8 * k)) & 0xFF;
    h *= 1099511628211ull;
  }
  return h;
}

std::string cache_path() {
  if (const char* p = std::getenv("RTG_TUNE_CACHE")) return p;
  const char* home = std::getenv("HOME");
  return std::string(home ? home : "/tmp") + "/.cache/rtg/tuning.txt";
}

void make_parent_dirs(const std::string& path) {
  for (std::size_t k = 1; k < path.size(); ++k)
    if (path[k] == '/') mkdir(path.substr(0, k).c_str(), 0755);
}

bool cache_lookup(const std::string& key, AutotuneResult& r) {
  std::ifstream in(cache_path());
  std::string line;
  bool found = false;
  while (std::getline(in, line)) {  // the last entry for a key wins
    std::istringstream ss(line);
    std::string k;
    AutotuneResult t;
    if (!(ss >> k >> t.pool_paths >> t.block >> t.msamples_per_s)) continue;
    if (k != key) continue;
    r = t;
    found = true;
  }
  return found;
}

void cache_store(const std::string& key, const AutotuneResult& r) {
  const std::string path = cache_path();
  make_parent_dirs(path);
  std::ofstream out(path, std::ios::app);
  if (out) out << key << ' ' << r.pool_paths << ' ' << r.block << ' ' << r.msamples_per_s << '\n';
}

}  // namespace

std::string workload_signature(Engine& e, const std::vector<Engine::BatchJob>& jobs) {
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, e.device());
  std::uint64_t h = 1469598103934665603ull;
  for (const auto& j : jobs) {
    const GpuScene& s = e.scene(j.scene_id);
    for (std::uint64_t v : {std::uint64_t(s.n_slots), std::uint64_t(s.n_planes), std::uint64_t(s.n_lights),
                            std::uint64_t(j.settings.width), std::uint64_t(j.settings.height),
                            std::uint64_t(j.settings.spp), std::uint64_t(j.settings.max_depth),
                            std::uint64_t(j.settings.rr_min_depth), std::uint64_t(j.settings.integrator)})
      h = fnv1a(h, v);
  }
  std::string name = prop.name;
  std::replace(name.begin(), name.end(), ' ', '_');
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s|sm%d|%016llx", name.c_str(), prop.multiProcessorCount,
                static_cast<unsigned long long>(h));
  return buf;
}

AutotuneResult autotune(Engine& e, const std::vector<Engine::BatchJob>& jobs, const RenderOptions& opts,
                        bool use_cache) {
  AutotuneResult best;
  best.key = workload_signature(e, jobs);
  EngineConfig& cfg = e.config();
  auto apply = [&](std::uint32_t pool, int block) {
    if (cfg.pool_paths != pool) {
      cfg.pool_paths = pool;
      e.reset_wave();
    }
    cfg.shape.extend_block = block;
  };
  if (use_cache && cache_lookup(best.key, best)) {
    best.key = workload_signature(e, jobs);
    best.from_cache = true;
    apply(best.pool_paths, best.block);
    return best;
  }
  std::vector<Engine::BatchJob> probe = jobs;
  for (auto& j : probe) j.settings.spp = std::max(1, j.settings.spp / 16);
  const bool timed = cfg.time_kernels, counted = cfg.count_traversal;
  cfg.time_kernels = cfg.count_traversal = false;
  const std::uint32_t pools[] = {1u << 20, 1u << 21, 1u << 22, 6u << 20, 1u << 23};
  const int blocks[] = {128, 256};
  for (std::uint32_t pool : pools) {
    for (int block : blocks) {
      apply(pool, block);
      e.render_batch(probe, opts, nullptr);  // warm: allocations, caches
      e.render_batch(probe, opts, nullptr);
      const RenderStats& st = e.stats();
      const double rate = st.camera_samples / std::max(1e-9, st.device_ms * 1e-3) / 1e6;
      best.candidates_tried++;
      if (rate > best.msamples_per_s) {
        best.msamples_per_s = rate;
        best.pool_paths = pool;
        best.block = block;
      }
    }
  }
  cfg.time_kernels = timed;
  cfg.count_traversal = counted;
  apply(best.pool_paths, best.block);
  cache_store(best.key, best);
  return best;
}

}  // namespace rtg
