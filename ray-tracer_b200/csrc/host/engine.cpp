#include "host/engine.hpp"

#include "host/alloc_count.hpp"

#include "device/bvh_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <exception>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>

namespace rtg {

namespace {
std::atomic<std::uint64_t> g_allocations{0};
}  // namespace

void count_allocation() { g_allocations.fetch_add(1, std::memory_order_relaxed); }
std::uint64_t allocation_count() { return g_allocations.load(std::memory_order_relaxed); }

namespace {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaFailure(std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(expr) check((expr), #expr)

template <class T>
T* dev_alloc(std::size_t n) {
  void* p = nullptr;
  count_allocation();
  CK(cudaMalloc(&p, std::max<std::size_t>(n, 1) * sizeof(T)));
  return static_cast<T*>(p);
}

// Stream-ordered allocation from the engine's own pool: never synchronises with
// kernels in flight, and freed blocks stay mapped for reuse.
template <class T>
T* dev_alloc_async(std::size_t n, cudaMemPool_t pool, cudaStream_t s) {
  void* p = nullptr;
  count_allocation();
  CK(cudaMallocFromPoolAsync(&p, std::max<std::size_t>(n, 1) * sizeof(T), pool, s));
  return static_cast<T*>(p);
}

template <class T>
T* dev_upload(const std::vector<T>& v, cudaStream_t s, std::size_t& bytes) {
  T* p = dev_alloc<T>(v.size());
  if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  bytes += std::max<std::size_t>(v.size(), 1) * sizeof(T);
  return p;
}

void dev_free(void* p) {
  if (p) cudaFree(p);
}

// Returns a scene's device memory; the flattened arrays are one stream-ordered
// allocation from the engine's pool, freed in stream order (no device sync).
void free_scene_arrays(GpuScene& s, cudaStream_t stream) {
  if (s.block) cudaFreeAsync(s.block, stream);
  s.block = nullptr;
  dev_free(s.prims64); dev_free(s.planes64);
}

constexpr int kRing = 8;   // snapshot / staging slots (iterations in flight at most)
constexpr int kLag = 2;    // iterations queued ahead of the snapshot being read
constexpr std::size_t kStageBytes = std::size_t(1) << 20;  // host->device staging per iteration
constexpr std::size_t kStagePiece = std::size_t(1) << 20;  // batch upload: bytes per host copy task
constexpr int kJobSlots = 4096;  // job descriptors resident at once

}  // namespace

struct Engine::Wave {
  WaveBuffers wb{};
  RtgSceneDev* jobs_dev = nullptr;
  DevSegment* segs_dev = nullptr;
  SegmentProgress* prog_dev = nullptr;
  GenTable* gen_dev = nullptr;
  GenPlan* plan_dev = nullptr;
  WaveSnapshot* ring = nullptr;        // pinned, device-mapped
  unsigned char* staging = nullptr;    // pinned, kRing * kStageBytes
  std::uint64_t stage_it = ~0ull;      // iteration the current staging slot belongs to
  std::size_t stage_used = 0;
  cudaEvent_t plan_ev[kRing]{};
  bool plan_recorded[kRing]{};
  cudaEvent_t tev[10]{};
  std::uint64_t it = 0;                // iterations launched (the device's `iteration`)
  std::uint64_t seen = 0;              // next snapshot to read: the one plan(seen) wrote
  std::uint64_t rad_cap = 0;
  std::map<std::uint64_t, std::uint64_t> rad_free;  // free radiance ranges: begin -> length
  std::vector<int> free_jobs;          // descriptor slots, popped from the back
  std::vector<int> free_segs;
  std::uint32_t snapshot_slots = 0;
  std::uint32_t hi_slot = 0;           // segment slots ever used are below this
  std::uint64_t stall = 0;             // snapshots without a finished sample while work is open
  std::uint64_t last_done_sum = 0;

  std::uint64_t rad_in_free = 0;       // radiance slots in rad_free
  bool rad_alloc(std::uint64_t n, std::uint64_t& at) {
    for (auto itr = rad_free.begin(); itr != rad_free.end(); ++itr) {
      if (itr->second < n) continue;
      at = itr->first;
      const std::uint64_t rest = itr->second - n;
      rad_free.erase(itr);
      if (rest) rad_free.emplace(at + n, rest);
      rad_in_free -= n;
      return true;
    }
    return false;
  }
  void rad_release(std::uint64_t at, std::uint64_t n) {
    rad_in_free += n;
    auto nx = rad_free.lower_bound(at);
    if (nx != rad_free.end() && at + n == nx->first) {
      n += nx->second;
      nx = rad_free.erase(nx);
    }
    if (nx != rad_free.begin()) {
      auto pv = std::prev(nx);
      if (pv->first + pv->second == at) {
        pv->second += n;
        return;
      }
    }
    rad_free.emplace(at, n);
  }
};

Engine::Engine(int device) : device_(device) {
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  // Highest priority: a build's short kernels take SM slots ahead of the
  // wavefront's queued blocks, so a cold scene does not wait behind renders.
  int least = 0, greatest = 0;
  CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  CK(cudaStreamCreateWithPriority(&build_stream_, cudaStreamNonBlocking, greatest));
  CK(cudaEventCreate(&ev_begin_));
  CK(cudaEventCreate(&ev_end_));
  for (auto& e : upload_ev_) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  CK(cudaMemPoolCreate(&pool_, &props));
  // Keep freed framebuffers mapped: requests come and go at hundreds per second.
  std::uint64_t keep = ~0ull;
  CK(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep));
}

void Engine::finish_timing() {
  CK(cudaEventRecord(ev_end_, stream_));
  CK(cudaEventSynchronize(ev_end_));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, ev_begin_, ev_end_));
  stats_.device_ms = ms;
}

Engine::~Engine() {
  cudaSetDevice(device_);
  cudaStreamSynchronize(stream_);
  for (auto& f : frames_) free_frame(f);
  for (auto& kv : jobs_) free_frame(kv.second.frame);
  cudaStreamSynchronize(stream_);
  for (auto& kv : scenes_) free_scene_arrays(*kv.second, stream_);
  cudaStreamSynchronize(stream_);
  jobs_.clear();
  reset_wave();
  cudaEventDestroy(ev_begin_);
  cudaEventDestroy(ev_end_);
  for (int b = 0; b < 2; ++b) {
    cudaEventDestroy(upload_ev_[b]);
    if (upload_host_[b]) cudaFreeHost(upload_host_[b]);
  }
  if (readback_host_) cudaFreeHost(readback_host_);
  cudaStreamSynchronize(build_stream_);
  cudaStreamDestroy(build_stream_);
  cudaStreamDestroy(stream_);
  cudaMemPoolDestroy(pool_);
}

void Engine::reset_wave() {
  if (!jobs_.empty()) throw std::logic_error("the wavefront has open jobs");
  cudaStreamSynchronize(stream_);
  if (wave_) {
    WaveBuffers& b = wave_->wb;
    for (int i = 0; i < 2; ++i) { dev_free(b.st_a[i]); dev_free(b.st_b[i]); dev_free(b.st_c[i]); dev_free(b.st_d[i]); dev_free(b.st_e[i]); }
    dev_free(b.hits); dev_free(b.sh_a); dev_free(b.sh_b); dev_free(b.sh_c); dev_free(b.radiance); dev_free(b.cnt);
    dev_free(wave_->jobs_dev); dev_free(wave_->segs_dev); dev_free(wave_->prog_dev);
    dev_free(wave_->gen_dev); dev_free(wave_->plan_dev);
    if (wave_->ring) cudaFreeHost(wave_->ring);
    if (wave_->staging) cudaFreeHost(wave_->staging);
    for (auto& e : wave_->plan_ev) if (e) cudaEventDestroy(e);
    for (auto& e : wave_->tev) if (e) cudaEventDestroy(e);
    wave_.reset();
  }
  segs_.clear();
}

int Engine::add_scene(std::shared_ptr<const CompiledScene> scene) {
  if (!scene->bvh_built) {
    if (scene->prims.size() >= kGpuBuildMinPrims) return add_scene_gpu_bvh(std::move(scene));
    // Small scene: the host builds the same tree faster than the GPU build's
    // level-by-level passes can start and finish.
    auto built = std::make_shared<CompiledScene>(*scene);
    std::vector<Box> boxes;
    boxes.reserve(built->prims.size());
    for (const Prim& p : built->prims) boxes.push_back(p.bounds());
    built->bvh.build(boxes, 4);
    built->info.bvh = built->bvh.stats;
    built->bvh_built = true;
    FlatScene flat = flatten(*built, wants_wide8());
    return add_flat(std::move(built), std::move(flat));
  }
  FlatScene flat = flatten(*scene, wants_wide8());
  return add_flat(std::move(scene), std::move(flat));
}

std::vector<int> Engine::add_scenes(const std::vector<std::shared_ptr<const CompiledScene>>& scenes) {
  // Flatten on all host cores (one scene per task), then copy in order.
  for (const auto& sc : scenes)
    if (!sc->bvh_built) {
      // Scenes without a host BVH are built on the GPU, one after another.
      std::vector<int> ids;
      ids.reserve(scenes.size());
      for (const auto& x : scenes) ids.push_back(add_scene(x));
      return ids;
    }
  std::vector<FlatScene> flats(scenes.size());
  const bool wide8 = wants_wide8();
  // Largest scenes first, so none of them starts last and sets the finish.
  std::vector<std::size_t> by_size(scenes.size());
  for (std::size_t k = 0; k < scenes.size(); ++k) by_size[k] = k;
  std::stable_sort(by_size.begin(), by_size.end(), [&](std::size_t a, std::size_t b) {
    return scenes[a]->prims.size() > scenes[b]->prims.size();
  });
  std::atomic<std::size_t> next{0};
  std::exception_ptr failed;
  std::mutex failed_lock;
  auto work = [&] {
    for (std::size_t i; (i = next.fetch_add(1)) < scenes.size();) {
      const std::size_t k = by_size[i];
      try {
        // The workers already use every core: only the largest scenes, which
        // start first and set the finish, split their own loops.
        const std::size_t np = scenes[k]->prims.size();
        flats[k] = flatten(*scenes[k], wide8, np >= 100000 ? 4u : np >= 32768 ? 2u : 1u);
      } catch (...) {
        std::lock_guard<std::mutex> g(failed_lock);
        if (!failed) failed = std::current_exception();
      }
    }
  };
  const std::size_t workers = std::min<std::size_t>(scenes.size(), std::max(1u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (std::size_t w = 1; w < workers; ++w) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  if (failed) std::rethrow_exception(failed);
  // All scenes go through one pinned staging buffer, filled on all host cores
  // (the copy into pinned memory was the serial part of the upload), then one
  // device block and one copy per scene.
  CK(cudaSetDevice(device_));
  std::vector<StagedParts> parts(scenes.size());
  std::vector<std::size_t> offset(scenes.size());
  std::size_t total = 0;
  for (std::size_t k = 0; k < scenes.size(); ++k) {
    parts[k] = staged_parts(flats[k]);
    offset[k] = total;
    total += parts[k].total;
  }
  int b = 0;
  unsigned char* host = upload_staging(std::max<std::size_t>(total, 1), b, 0);
  // The copy into pinned memory, in pieces over all scenes' parts.
  std::vector<StagePiece> pieces;
  for (std::size_t k = 0; k < scenes.size(); ++k) stage_pieces(flats[k], parts[k], host + offset[k], pieces);
  copy_pieces(pieces);
  std::vector<int> ids;
  ids.reserve(scenes.size());
  for (std::size_t k = 0; k < scenes.size(); ++k)
    ids.push_back(register_flat(scenes[k], std::move(flats[k]), parts[k], host + offset[k]));
  CK(cudaEventRecord(upload_ev_[b], stream_));
  upload_pending_[b] = true;
  return ids;
}

Engine::StagedParts Engine::staged_parts(const FlatScene& f) {
  StagedParts p{};
  const std::size_t bytes[kSceneParts] = {f.nodes.size() * sizeof(DevNode), f.nodes4.size() * sizeof(DevNode4),
                                          f.prims.size() * sizeof(float4), f.slot_material.size() * sizeof(std::uint32_t),
                                          f.slot_normals.size() * sizeof(float4), f.planes.size() * sizeof(DevPlane),
                                          f.materials.size() * sizeof(DevMaterial), f.lights.size() * sizeof(DevLight),
                                          f.nodes8.size() * sizeof(DevNode8)};
  p.total = 0;
  for (int k = 0; k < kSceneParts; ++k) {
    p.bytes[k] = bytes[k];
    p.at[k] = p.total;
    p.total += (std::max<std::size_t>(bytes[k], 1) + 255) & ~std::size_t(255);
  }
  return p;
}

void Engine::stage_pieces(const FlatScene& f, const StagedParts& p, unsigned char* dst, std::vector<StagePiece>& out) {
  const void* src[kSceneParts] = {f.nodes.data(), f.nodes4.data(), f.prims.data(), f.slot_material.data(),
                                  f.slot_normals.data(), f.planes.data(), f.materials.data(), f.lights.data(),
                                  f.nodes8.data()};
  for (int q = 0; q < kSceneParts; ++q)
    for (std::size_t o = 0; o < p.bytes[q]; o += kStagePiece)
      out.push_back({dst + p.at[q] + o, static_cast<const unsigned char*>(src[q]) + o,
                     std::min(kStagePiece, p.bytes[q] - o)});
}

void Engine::copy_pieces(const std::vector<StagePiece>& pieces) {
  std::atomic<std::size_t> next{0};
  auto copy = [&] {
    for (std::size_t k; (k = next.fetch_add(1)) < pieces.size();) std::memcpy(pieces[k].dst, pieces[k].src, pieces[k].bytes);
  };
  // A thread per 4 pieces at most: small scenes are copied inline.
  const std::size_t workers =
      std::min<std::size_t>({std::max(1u, std::thread::hardware_concurrency()), 16, (pieces.size() + 3) / 4});
  std::vector<std::thread> pool;
  for (std::size_t w = 1; w < workers; ++w) pool.emplace_back(copy);
  copy();
  for (auto& t : pool) t.join();
}

void Engine::stage_flat(const FlatScene& f, const StagedParts& p, unsigned char* dst) {
  std::vector<StagePiece> pieces;
  stage_pieces(f, p, dst, pieces);
  copy_pieces(pieces);
}

int Engine::add_flat(std::shared_ptr<const CompiledScene> scene, FlatScene flat) {
  // One device allocation and one copy per scene, through a pinned staging
  // buffer: the copy runs while the caller flattens the next scene (two buffers
  // alternate), and the flattened vectors can go at once.
  CK(cudaSetDevice(device_));
  const StagedParts p = staged_parts(flat);
  int b = 0;
  unsigned char* host = upload_staging(p.total, b);
  stage_flat(flat, p, host);
  const int id = register_flat(std::move(scene), std::move(flat), p, host);
  CK(cudaEventRecord(upload_ev_[b], stream_));
  upload_pending_[b] = true;
  return id;
}

int Engine::register_flat(std::shared_ptr<const CompiledScene> scene, FlatScene flat, const StagedParts& p,
                          const unsigned char* staged) {
  CK(cudaSetDevice(device_));
  auto gs = std::make_unique<GpuScene>();
  gs->root = flat.root;
  gs->n_slots = static_cast<std::int32_t>(flat.slot_prim.size());
  gs->n_planes = static_cast<std::int32_t>(flat.planes.size());
  gs->n_lights = static_cast<std::int32_t>(flat.lights.size());
  gs->root4 = flat.root4;
  gs->n_interior = static_cast<std::int32_t>(flat.nodes.size());
  gs->n_wide = static_cast<std::int32_t>(flat.nodes4.size());
  gs->root8 = flat.root8;
  gs->n_wide8 = static_cast<std::int32_t>(flat.nodes8.size());
  gs->has_wide8 = wants_wide8();
  void* block = nullptr;
  count_allocation();
  CK(cudaMallocFromPoolAsync(&block, p.total, pool_, stream_));
  CK(cudaMemcpyAsync(block, staged, p.total, cudaMemcpyHostToDevice, stream_));
  auto at = [&](int k) { return static_cast<void*>(static_cast<unsigned char*>(block) + p.at[k]); };
  gs->block = block;
  gs->nodes = static_cast<DevNode*>(at(0));
  gs->nodes4 = static_cast<DevNode4*>(at(1));
  gs->prims = static_cast<float4*>(at(2));
  gs->slot_material = static_cast<std::uint32_t*>(at(3));
  gs->slot_normals = static_cast<float4*>(at(4));
  gs->planes = static_cast<DevPlane*>(at(5));
  gs->materials = static_cast<DevMaterial*>(at(6));
  gs->lights = static_cast<DevLight*>(at(7));
  gs->nodes8 = static_cast<DevNode8*>(at(8));
  gs->device_bytes = p.total;
  gs->slot_prim = std::move(flat.slot_prim);
  gs->bvh = scene->info.bvh;
  gs->host = std::move(scene);
  const int id = next_scene_++;
  scenes_[id] = std::move(gs);
  return id;
}

unsigned char* Engine::upload_staging(std::size_t bytes, int& b, int want) {
  if (want >= 0) {
    b = want;
  } else {
    b = upload_next_;
    upload_next_ ^= 1;
  }
  if (upload_pending_[b]) CK(cudaEventSynchronize(upload_ev_[b]));
  upload_pending_[b] = false;
  if (upload_cap_[b] < bytes) {
    if (upload_host_[b]) CK(cudaFreeHost(upload_host_[b]));
    upload_host_[b] = nullptr;
    upload_cap_[b] = 0;
    count_allocation();
    CK(cudaMallocHost(reinterpret_cast<void**>(&upload_host_[b]), bytes));
    upload_cap_[b] = bytes;
  }
  return upload_host_[b];
}

int Engine::add_scene_gpu_bvh(std::shared_ptr<const CompiledScene> scene) {
  CK(cudaSetDevice(device_));
  const CompiledScene& s = *scene;
  if (s.prims.size() > kIdMask) throw std::runtime_error("too many primitives for the device layout");
  const std::size_t np = s.prims.size();
  FlatScene tables;
  flatten_tables(s, tables);

  // Inputs in primitive order, converted on the host cores into one pinned buffer:
  // boxes (double), slot rows, normals, material words, the ids of primitives
  // with a usable box, then the tables. One copy takes them all to the GPU.
  auto pad = [](std::size_t bytes) { return (std::max<std::size_t>(bytes, 1) + 255) & ~std::size_t(255); };
  const std::size_t in_bytes[8] = {np * 6 * sizeof(double), np * 3 * sizeof(float4), np * 3 * sizeof(float4),
                                   np * sizeof(std::uint32_t), np * sizeof(std::uint32_t),
                                   tables.planes.size() * sizeof(DevPlane),
                                   tables.materials.size() * sizeof(DevMaterial),
                                   tables.lights.size() * sizeof(DevLight)};
  std::size_t in_at[9];
  in_at[0] = 0;
  for (int k = 0; k < 8; ++k) in_at[k + 1] = in_at[k] + pad(in_bytes[k]);
  const std::size_t staged = in_at[8];
  int b = 0;
  unsigned char* host = upload_staging(staged, b);
  auto* boxes = reinterpret_cast<double*>(host + in_at[0]);
  auto* rows = reinterpret_cast<float4*>(host + in_at[1]);
  auto* normals = reinterpret_cast<float4*>(host + in_at[2]);
  auto* material = reinterpret_cast<std::uint32_t*>(host + in_at[3]);
  auto* items = reinterpret_cast<std::uint32_t*>(host + in_at[4]);
  std::vector<std::uint8_t> usable(np);
  {
    const std::size_t workers = std::min<std::size_t>({16, std::max(1u, std::thread::hardware_concurrency()),
                                                       (np + 16383) / 16384});
    auto body = [&](std::size_t i0, std::size_t i1) {
      for (std::size_t i = i0; i < i1; ++i) {
        const Prim& p = s.prims[i];
        const Box bx = p.bounds();
        double* d = boxes + 6 * i;
        d[0] = bx.lo.x; d[1] = bx.lo.y; d[2] = bx.lo.z;
        d[3] = bx.hi.x; d[4] = bx.hi.y; d[5] = bx.hi.z;
        usable[i] = !(bx.empty() || !bx.lo.finite() || !bx.hi.finite());
        slot_record(p, static_cast<std::uint32_t>(i), rows + 3 * i, normals + 3 * i, material[i]);
      }
    };
    std::vector<std::thread> pool;
    const std::size_t chunk = workers > 1 ? (np + workers - 1) / workers : np;
    for (std::size_t w = 1; w < workers; ++w)
      pool.emplace_back(body, std::min(np, w * chunk), std::min(np, (w + 1) * chunk));
    body(0, std::min(np, chunk));
    for (auto& t : pool) t.join();
  }
  std::uint32_t n_items = 0;
  for (std::size_t i = 0; i < np; ++i)
    if (usable[i]) items[n_items++] = static_cast<std::uint32_t>(i);
  std::memcpy(host + in_at[5], tables.planes.data(), in_bytes[5]);
  std::memcpy(host + in_at[6], tables.materials.data(), in_bytes[6]);
  std::memcpy(host + in_at[7], tables.lights.data(), in_bytes[7]);

  // Device copy of the inputs plus room for the slot -> primitive map.
  void* in_block = nullptr;
  count_allocation();
  CK(cudaMallocFromPoolAsync(&in_block, staged + pad(np * sizeof(std::uint32_t)), pool_, build_stream_));
  struct FreeInput {
    void* p;
    cudaStream_t s;
    ~FreeInput() { cudaFreeAsync(p, s); }
  } free_input{in_block, build_stream_};
  auto* dev_in = static_cast<unsigned char*>(in_block);
  CK(cudaMemcpyAsync(dev_in, host, staged, cudaMemcpyHostToDevice, build_stream_));
  CK(cudaEventRecord(upload_ev_[b], build_stream_));
  upload_pending_[b] = true;
  auto* order = reinterpret_cast<std::uint32_t*>(dev_in + staged);

  GpuBvhInput in;
  in.n_items = n_items;
  in.boxes = reinterpret_cast<const double*>(dev_in + in_at[0]);
  in.rows = reinterpret_cast<const float4*>(dev_in + in_at[1]);
  in.normals = reinterpret_cast<const float4*>(dev_in + in_at[2]);
  in.material = reinterpret_cast<const std::uint32_t*>(dev_in + in_at[3]);
  in.items = reinterpret_cast<const std::uint32_t*>(dev_in + in_at[4]);
  GpuBvhBuilder builder(build_stream_, pool_);
  const GpuBvhCounts c = builder.build(in);

  // The layout in the binary tree's leaf order, in scratch first: the
  // eight-wide tree is built from it on the host (the same function as for a
  // host-built scene, so the bytes agree) and sets the final slot order.
  const std::size_t scratch_bytes[7] = {std::size_t(c.interior) * sizeof(DevNode), std::size_t(c.wide) * sizeof(DevNode4),
                                        std::size_t(n_items) * 3 * sizeof(float4), std::size_t(n_items) * sizeof(std::uint32_t),
                                        std::size_t(n_items) * 3 * sizeof(float4), std::size_t(n_items) * sizeof(std::uint32_t),
                                        std::size_t(n_items) * sizeof(std::uint32_t)};
  std::size_t sat[7], scratch_total = 0;
  for (int k = 0; k < 7; ++k) {
    sat[k] = scratch_total;
    scratch_total += pad(scratch_bytes[k]);
  }
  void* scratch = nullptr;
  count_allocation();
  CK(cudaMallocFromPoolAsync(&scratch, scratch_total, pool_, build_stream_));
  struct FreeScratch {
    void* p;
    cudaStream_t s;
    ~FreeScratch() { cudaFreeAsync(p, s); }
  } free_scratch{scratch, build_stream_};
  auto* sb = static_cast<unsigned char*>(scratch);
  auto* s_nodes = reinterpret_cast<DevNode*>(sb + sat[0]);
  auto* s_nodes4 = reinterpret_cast<DevNode4*>(sb + sat[1]);
  auto* s_prims = reinterpret_cast<float4*>(sb + sat[2]);
  auto* s_material = reinterpret_cast<std::uint32_t*>(sb + sat[3]);
  auto* s_normals = reinterpret_cast<float4*>(sb + sat[4]);
  auto* s_old_of = reinterpret_cast<std::uint32_t*>(sb + sat[5]);
  auto* s_new_of = reinterpret_cast<std::uint32_t*>(sb + sat[6]);
  builder.emit(in, s_nodes, s_nodes4, s_prims, s_material, s_normals, order);
  const bool want8 = wants_wide8();
  std::vector<DevNode> bin_nodes;
  std::vector<std::uint32_t> row0_w, prim_of_slot(n_items);
  if (n_items)
    CK(cudaMemcpyAsync(prim_of_slot.data(), order, n_items * sizeof(std::uint32_t), cudaMemcpyDeviceToHost,
                       build_stream_));
  if (want8) {
    bin_nodes.resize(static_cast<std::size_t>(c.interior));
    row0_w.resize(n_items);
    if (c.interior)
      CK(cudaMemcpyAsync(bin_nodes.data(), s_nodes, scratch_bytes[0], cudaMemcpyDeviceToHost, build_stream_));
    if (n_items)  // the w word of each slot's first row: its primitive id and leaf-end mark
      CK(cudaMemcpy2DAsync(row0_w.data(), sizeof(std::uint32_t), reinterpret_cast<const unsigned char*>(s_prims) + 12,
                           3 * sizeof(float4), sizeof(std::uint32_t), n_items, cudaMemcpyDeviceToHost, build_stream_));
    CK(cudaStreamSynchronize(build_stream_));
  }
  Wide8 w8;
  if (want8) {
    std::vector<std::uint8_t> last(n_items);
    for (std::size_t k = 0; k < n_items; ++k) last[k] = (row0_w[k] & kLastInLeaf) ? 1 : 0;
    const std::int32_t bin_root = n_items ? c.root : kNoRoot;
    w8 = build_wide8(bin_nodes.data(), bin_nodes.size(), bin_root, last.data(), n_items);
  } else {
    // The binary tree's own slot order, no eight-wide tree.
    w8.old_of.resize(n_items);
    for (std::size_t k = 0; k < n_items; ++k) w8.old_of[k] = static_cast<std::uint32_t>(k);
    w8.new_of = w8.old_of;
    w8.root = kNoRoot;
  }

  // The scene's arrays, in add_flat's order, in one allocation.
  const std::size_t part_bytes[kSceneParts] = {
      std::size_t(c.interior) * sizeof(DevNode), std::size_t(c.wide) * sizeof(DevNode4),
      std::size_t(n_items) * 3 * sizeof(float4), std::size_t(n_items) * sizeof(std::uint32_t),
      std::size_t(n_items) * 3 * sizeof(float4), in_bytes[5], in_bytes[6], in_bytes[7],
      w8.nodes.size() * sizeof(DevNode8)};
  std::size_t at[kSceneParts], total = 0;
  for (int k = 0; k < kSceneParts; ++k) {
    at[k] = total;
    total += pad(part_bytes[k]);
  }
  void* block = nullptr;
  count_allocation();
  CK(cudaMallocFromPoolAsync(&block, total, pool_, build_stream_));
  // Freed again if anything below throws; handed to the scene at the end.
  struct FreeBlock {
    void* p;
    cudaStream_t s;
    ~FreeBlock() {
      if (p) cudaFreeAsync(p, s);
    }
  } free_block{block, build_stream_};
  auto* dst = static_cast<unsigned char*>(block);
  auto gs = std::make_unique<GpuScene>();
  gs->block = block;
  gs->nodes = reinterpret_cast<DevNode*>(dst + at[0]);
  gs->nodes4 = reinterpret_cast<DevNode4*>(dst + at[1]);
  gs->prims = reinterpret_cast<float4*>(dst + at[2]);
  gs->slot_material = reinterpret_cast<std::uint32_t*>(dst + at[3]);
  gs->slot_normals = reinterpret_cast<float4*>(dst + at[4]);
  gs->planes = reinterpret_cast<DevPlane*>(dst + at[5]);
  gs->materials = reinterpret_cast<DevMaterial*>(dst + at[6]);
  gs->lights = reinterpret_cast<DevLight*>(dst + at[7]);
  gs->nodes8 = reinterpret_cast<DevNode8*>(dst + at[8]);
  for (int k : {0, 1})
    if (part_bytes[k])
      CK(cudaMemcpyAsync(dst + at[k], sb + sat[k], part_bytes[k], cudaMemcpyDeviceToDevice, build_stream_));
  if (want8) {
    if (n_items) {
      CK(cudaMemcpyAsync(s_old_of, w8.old_of.data(), n_items * sizeof(std::uint32_t), cudaMemcpyHostToDevice, build_stream_));
      CK(cudaMemcpyAsync(s_new_of, w8.new_of.data(), n_items * sizeof(std::uint32_t), cudaMemcpyHostToDevice, build_stream_));
    }
    if (part_bytes[8])
      CK(cudaMemcpyAsync(gs->nodes8, w8.nodes.data(), part_bytes[8], cudaMemcpyHostToDevice, build_stream_));
    CK(apply_slot_order(s_old_of, s_new_of, n_items, s_prims, s_normals, s_material, gs->prims, gs->slot_normals,
                        gs->slot_material, gs->nodes, c.interior, gs->nodes4, c.wide, build_stream_));
  } else {
    // The slots stay in the binary tree's order.
    for (int k : {2, 3, 4})
      if (part_bytes[k])
        CK(cudaMemcpyAsync(dst + at[k], sb + sat[k], part_bytes[k], cudaMemcpyDeviceToDevice, build_stream_));
  }
  for (int k = 5; k < 8; ++k)
    if (part_bytes[k]) CK(cudaMemcpyAsync(dst + at[k], dev_in + in_at[k], part_bytes[k], cudaMemcpyDeviceToDevice, build_stream_));
  CK(cudaStreamSynchronize(build_stream_));
  gs->slot_prim.resize(n_items);
  for (std::size_t k = 0; k < n_items; ++k) gs->slot_prim[k] = prim_of_slot[w8.old_of[k]];

  gs->root = n_items ? remap_link(c.root, w8.new_of) : kNoRoot;
  gs->root4 = n_items ? remap_link(c.root4, w8.new_of) : kNoRoot;
  gs->root8 = w8.root;
  gs->n_wide8 = static_cast<std::int32_t>(w8.nodes.size());
  gs->has_wide8 = want8;
  gs->n_slots = static_cast<std::int32_t>(n_items);
  gs->n_interior = c.interior;
  gs->n_wide = c.wide;
  gs->n_planes = static_cast<std::int32_t>(tables.planes.size());
  gs->n_lights = static_cast<std::int32_t>(tables.lights.size());
  gs->device_bytes = total;
  gs->bvh.nodes = static_cast<std::size_t>(c.nodes);
  gs->bvh.leaves = static_cast<std::size_t>(c.leaves);
  gs->bvh.max_depth = static_cast<std::size_t>(c.max_depth);
  gs->bvh.max_leaf = static_cast<std::size_t>(c.max_leaf);
  gs->bvh.build_ms = c.build_ms;
  gs->device_built = true;
  free_block.p = nullptr;
  gs->host = std::move(scene);
  const int id = next_scene_++;
  scenes_[id] = std::move(gs);
  return id;
}

void Engine::release_scene(int id) {
  auto it = scenes_.find(id);
  if (it == scenes_.end()) throw std::invalid_argument("unknown scene id " + std::to_string(id));
  if (it->second->jobs_open > 0) throw std::logic_error("scene " + std::to_string(id) + " is used by an open request");
  free_scene_arrays(*it->second, stream_);
  scenes_.erase(it);
}

GpuScene& Engine::scene(int id) {
  auto it = scenes_.find(id);
  if (it == scenes_.end()) throw std::invalid_argument("unknown scene id " + std::to_string(id));
  return *it->second;
}

void Engine::ensure_wave() {
  if (wave_) return;
  CK(cudaSetDevice(device_));
  if (cfg_.pool_paths < 32 || cfg_.pool_paths > (1u << 23)) throw std::invalid_argument("pool_paths must be in [32, 2^23]");
  wave_ = std::make_unique<Wave>();
  Wave& W = *wave_;
  WaveBuffers& b = W.wb;
  const std::uint32_t P = cfg_.pool_paths;
  b.capacity = P;
  for (int i = 0; i < 2; ++i) {
    b.st_a[i] = dev_alloc<float4>(P);
    b.st_b[i] = dev_alloc<float4>(P);
    b.st_c[i] = dev_alloc<float4>(P);
    b.st_d[i] = dev_alloc<uint4>(P);
    b.st_e[i] = dev_alloc<float>(P);
  }
  b.hits = dev_alloc<float4>(P);
  b.sh_a = dev_alloc<float4>(P);
  b.sh_b = dev_alloc<float4>(P);
  b.sh_c = dev_alloc<float4>(P);
  W.rad_cap = std::max<std::uint64_t>(1, std::min<std::uint64_t>(cfg_.max_pass_samples, 0xFFFFFFFFull));
  b.radiance = dev_alloc<float4>(W.rad_cap);
  W.rad_free.emplace(0, W.rad_cap);
  W.rad_in_free = W.rad_cap;
  b.cnt = dev_alloc<WaveCounters>(1);
  W.jobs_dev = dev_alloc<RtgSceneDev>(kJobSlots);
  W.segs_dev = dev_alloc<DevSegment>(kMaxSegments);
  W.prog_dev = dev_alloc<SegmentProgress>(kMaxSegments);
  W.gen_dev = dev_alloc<GenTable>(1);
  W.plan_dev = dev_alloc<GenPlan>(1);
  CK(cudaMemset(b.cnt, 0, sizeof(WaveCounters)));
  CK(cudaMemset(W.prog_dev, 0, sizeof(SegmentProgress) * kMaxSegments));
  CK(cudaMemset(W.gen_dev, 0, sizeof(GenTable)));
  CK(cudaMemset(W.plan_dev, 0, sizeof(GenPlan)));
  count_allocation();
  CK(cudaHostAlloc(reinterpret_cast<void**>(&W.ring), sizeof(WaveSnapshot) * kRing, cudaHostAllocMapped));
  WaveSnapshot* ring_dev = nullptr;
  CK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&ring_dev), W.ring, 0));
  count_allocation();
  CK(cudaMallocHost(reinterpret_cast<void**>(&W.staging), kStageBytes * kRing));
  for (auto& e : W.plan_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto& e : W.tev) CK(cudaEventCreate(&e));
  b.jobs = W.jobs_dev;
  b.segs = W.segs_dev;
  b.seg_prog = W.prog_dev;
  b.gen = W.gen_dev;
  b.plan = W.plan_dev;
  b.ring = ring_dev;
  b.ring_size = kRing;
  for (int k = kJobSlots - 1; k >= 0; --k) W.free_jobs.push_back(k);
  for (int k = kMaxSegments - 1; k >= 0; --k) W.free_segs.push_back(k);
  segs_.assign(kMaxSegments, Seg{});
  CK(cudaDeviceSynchronize());
}

GpuFrame Engine::make_frame(int w, int h) {
  GpuFrame f;
  f.width = w;
  f.height = h;
  const std::size_t px = std::size_t(w) * std::size_t(h);
  f.sum = dev_alloc_async<double>(px * 4, pool_, stream_);
  f.sumsq = dev_alloc_async<double>(px * 4, pool_, stream_);
  f.count = dev_alloc_async<std::uint32_t>(px, pool_, stream_);
  f.stats = dev_alloc_async<std::uint64_t>(4, pool_, stream_);
  CK(cudaMemsetAsync(f.sum, 0, px * 4 * sizeof(double), stream_));
  CK(cudaMemsetAsync(f.sumsq, 0, px * 4 * sizeof(double), stream_));
  CK(cudaMemsetAsync(f.count, 0, px * sizeof(std::uint32_t), stream_));
  CK(cudaMemsetAsync(f.stats, 0, 4 * sizeof(std::uint64_t), stream_));
  return f;
}

void Engine::free_frame(GpuFrame& f) {
  for (void* p : {static_cast<void*>(f.sum), static_cast<void*>(f.sumsq), static_cast<void*>(f.count),
                  static_cast<void*>(f.stats)})
    if (p) cudaFreeAsync(p, stream_);
  f = GpuFrame{};
}

RtgSceneDev Engine::job_descriptor(const GpuScene& sc, const RenderSettings& s, const GpuFrame& f) const {
  if (wants_wide8() && !sc.has_wide8)
    throw std::invalid_argument("scene was uploaded without the eight-wide tree: select the eight-wide walk "
                                "(rtg_tuning closest_tree / shadow_tree = 8) before uploading it");
  RtgSceneDev d{};
  describe(*sc.host, s, d);
  d.nodes = sc.nodes;
  d.prims = sc.prims;
  d.slot_material = sc.slot_material;
  d.slot_normals = sc.slot_normals;
  d.planes = sc.planes;
  d.materials = sc.materials;
  d.lights = sc.lights;
  d.root = sc.root;
  d.nodes4 = sc.nodes4;
  d.root4 = sc.root4;
  d.nodes8 = sc.nodes8;
  d.root8 = sc.root8;
  d.n_planes = sc.n_planes;
  d.n_lights = sc.n_lights;
  d.slot_begin = 0;
  d.slot_end = sc.n_slots;
  d.prims64 = sc.prims64;
  d.planes64 = sc.planes64;
  d.fb_sum = f.sum;
  d.fb_sumsq = f.sumsq;
  d.fb_count = f.count;
  d.stats = f.stats;
  return d;
}

// ---------------------------------------------------------------------------
// Host->device writes of the scheduler go through a pinned staging slot that
// belongs to the next iteration, so they never wait for the stream.
void Engine::stage(void* dst, const void* src, std::size_t n) {
  Wave& W = *wave_;
  const int r = static_cast<int>(W.it % kRing);
  if (W.stage_it != W.it) {
    if (W.plan_recorded[r]) CK(cudaEventSynchronize(W.plan_ev[r]));  // its last copies have run
    W.stage_it = W.it;
    W.stage_used = 0;
  }
  const std::size_t at = (W.stage_used + 15) & ~std::size_t(15);
  if (at + n > kStageBytes) {
    // Burst larger than a staging slot: fall back to a synchronous copy.
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice));
    return;
  }
  unsigned char* p = W.staging + std::size_t(r) * kStageBytes + at;
  std::memcpy(p, src, n);
  CK(cudaMemcpyAsync(dst, p, n, cudaMemcpyHostToDevice, stream_));
  W.stage_used = at + n;
}

void Engine::write_gen_table() {
  Wave& W = *wave_;
  // Open segments still generating, in priority order: previews before finals,
  // then earlier passes before later ones (a new render's first pass overtakes
  // the later passes of renders already running), then submission order.
  std::vector<int> open;
  std::uint32_t hi = 0;
  for (int k = 0; k < static_cast<int>(W.hi_slot); ++k) {
    Seg& s = segs_[k];
    if (!s.used) continue;
    hi = static_cast<std::uint32_t>(k + 1);
    s.in_gen = false;
    if (s.complete || s.abandoned || s.generated >= s.d.count) continue;
    open.push_back(k);
  }
  std::sort(open.begin(), open.end(), [&](int a, int b) {
    const Job& ja = jobs_.at(segs_[a].job);
    const Job& jb = jobs_.at(segs_[b].job);
    if (ja.priority != jb.priority) return ja.priority < jb.priority;
    if (segs_[a].d.pass_s0 != segs_[b].d.pass_s0) return segs_[a].d.pass_s0 < segs_[b].d.pass_s0;
    return ja.seq < jb.seq;
  });
  GenTable g{};
  g.n = static_cast<std::uint32_t>(std::min<std::size_t>(open.size(), kMaxGen));
  for (std::uint32_t k = 0; k < g.n; ++k) {
    g.slot[k] = static_cast<std::uint32_t>(open[k]);
    segs_[open[k]].in_gen = true;
  }
  g.snapshot_slots = hi;
  W.snapshot_slots = hi;
  stage(W.gen_dev, &g, offsetof(GenTable, slot) + sizeof(std::uint32_t) * std::max<std::uint32_t>(g.n, 1));
  gen_dirty_ = false;
}

int Engine::open_job(const JobSpec& spec, bool serving, PassCallback cb) {
  ensure_wave();
  Wave& W = *wave_;
  GpuScene& sc = scene(spec.scene_id);
  if (W.free_jobs.empty()) throw std::length_error("too many open renders");
  Job j;
  j.handle = next_job_++;
  j.desc_slot = W.free_jobs.back();
  W.free_jobs.pop_back();
  j.scene_id = spec.scene_id;
  j.settings = spec.settings;
  j.opts = spec.opts;
  j.priority = spec.priority;
  j.seq = job_seq_++;
  j.pixels = std::uint64_t(spec.settings.width) * std::uint64_t(spec.settings.height);
  j.target = static_cast<std::uint32_t>(spec.settings.spp);
  j.direct = spec.settings.integrator == Integrator::Direct;
  j.serving = serving;
  j.on_pass = std::move(cb);
  j.t0 = std::chrono::steady_clock::now();
  j.prog.spp_target = spec.settings.spp;
  j.frame = make_frame(spec.settings.width, spec.settings.height);
  const RtgSceneDev d = job_descriptor(sc, spec.settings, j.frame);
  stage(W.jobs_dev + j.desc_slot, &d, sizeof(d));
  sc.jobs_open++;
  if (j.settings.light_sampling && j.settings.mis) ++mis_jobs_;
  const int h = j.handle;
  jobs_.emplace(h, std::move(j));
  return h;
}

void Engine::close_job(Job& j) {
  Wave& W = *wave_;
  W.free_jobs.push_back(j.desc_slot);
  if (j.settings.light_sampling && j.settings.mis) --mis_jobs_;
  auto it = scenes_.find(j.scene_id);
  if (it != scenes_.end()) it->second->jobs_open--;
}

bool Engine::all_jobs_drained() const {
  for (const auto& kv : jobs_)
    if (!kv.second.drained()) return false;
  return true;
}

std::uint32_t Engine::next_pass_size(const Job& j) const {
  std::uint32_t k = j.target - j.issued;
  if (j.opts.progressive) {
    const std::uint32_t grow = std::max<std::uint32_t>(1u, j.issued);
    const std::uint32_t cap = static_cast<std::uint32_t>(std::max(1, j.opts.max_pass_spp));
    k = std::min({k, grow, cap});
  }
  const std::uint64_t fit = std::max<std::uint64_t>(1, wave_->rad_cap / std::max<std::uint64_t>(1, j.pixels));
  return static_cast<std::uint32_t>(std::min<std::uint64_t>(k, fit));
}

bool Engine::issue_pass(Job& j) {
  Wave& W = *wave_;
  const std::uint32_t k = next_pass_size(j);
  const std::uint64_t count = j.pixels * k;
  if (W.free_segs.empty()) return false;
  // Lower-priority work leaves an eighth of the radiance slots to priority 0.
  if (j.priority > 0 && W.rad_in_free < count + W.rad_cap / 8) return false;
  std::uint64_t at = 0;
  if (!W.rad_alloc(count, at)) return false;
  const int slot = W.free_segs.back();
  W.free_segs.pop_back();
  W.hi_slot = std::max<std::uint32_t>(W.hi_slot, static_cast<std::uint32_t>(slot + 1));
  Seg& s = segs_[slot];
  s = Seg{};
  s.used = true;
  s.job = j.handle;
  s.d.job = static_cast<std::uint32_t>(j.desc_slot);
  s.d.pass_s0 = j.issued;
  s.d.pass_spp = k;
  s.d.count = count;
  s.d.sample_base = at;
  s.rad_begin = at;
  s.assigned_at = W.it;
  const SegmentProgress zero{};
  stage(W.segs_dev + slot, &s.d, sizeof(s.d));
  stage(W.prog_dev + slot, &zero, sizeof(zero));
  j.issued += k;
  j.passes_issued++;
  j.segs.push_back(slot);
  gen_dirty_ = true;
  return true;
}

bool Engine::run_direct_pass(Job& j) {
  Wave& W = *wave_;
  const std::uint32_t k = next_pass_size(j);
  const std::uint64_t count = j.pixels * k;
  std::uint64_t at = 0;
  if (!W.rad_alloc(count, at)) return false;  // retried once radiance space frees up
  DevSegment d{};
  d.job = static_cast<std::uint32_t>(j.desc_slot);
  d.pass_s0 = j.issued;
  d.pass_spp = k;
  d.count = count;
  d.sample_base = at;
  const bool timed = cfg_.time_kernels;
  if (timed) CK(cudaEventRecord(W.tev[8], stream_));
  CK(launch_direct(W.jobs_dev + j.desc_slot, d, W.wb.radiance, W.wb.cnt, cfg_.shape.closest_tree == 8, stream_));
  if (timed) CK(cudaEventRecord(W.tev[9], stream_));
  CK(launch_accumulate(W.jobs_dev + j.desc_slot, j.pixels, d, W.wb.radiance, stream_));
  stats_.kernel_launches += 2;
  // Reported once it has run, so progress times are device-complete.
  CK(cudaStreamSynchronize(stream_));
  if (timed) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, W.tev[8], W.tev[9]));
    stats_.direct_ms += ms;
  }
  W.rad_release(at, count);
  WaveCounters c{};
  CK(cudaMemcpy(&c, W.wb.cnt, sizeof(c), cudaMemcpyDeviceToHost));
  if (c.error) throw CudaFailure("device error flag " + std::to_string(c.error) +
                                 (c.error == 2 ? " (direct integrator branch stack overflow)" : ""));
  last_counters_ = c;
  j.issued += k;
  j.passes_issued++;
  j.done += k;
  j.prog.pass++;
  j.prog.spp_done = j.done;
  j.prog.finished = j.done >= j.target;
  j.prog.elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - j.t0).count();
  j.prog.rays = (c.rays - base_counters_.rays) + (c.shadow_rays - base_counters_.shadow_rays);
  stats_.passes++;
  return true;
}

void Engine::refill() {
  Wave& W = *wave_;
  // Samples not yet finished in the open segments, per priority level.
  std::map<int, std::uint64_t> backlog;
  for (int k = 0; k < static_cast<int>(W.hi_slot); ++k) {
    const Seg& s = segs_[k];
    if (!s.used || s.complete || s.abandoned) continue;
    backlog[jobs_.at(s.job).priority] += s.d.count - std::min<std::uint64_t>(s.done, s.d.count);
  }
  const std::uint64_t target = std::uint64_t(cfg_.backlog_pools) * W.wb.capacity;
  while (true) {
    Job* best = nullptr;
    for (auto& kv : jobs_) {
      Job& j = kv.second;
      if (j.cancelled || j.issued >= j.target) continue;
      if (!best || j.priority < best->priority ||
          (j.priority == best->priority &&
           (j.passes_issued < best->passes_issued || (j.passes_issued == best->passes_issued && j.seq < best->seq))))
        best = &j;
    }
    if (!best) return;
    if (best->direct) {
      // One whole pass per call, so cancellation is checked between passes.
      if (run_direct_pass(*best) && best->on_pass) best->on_pass(best->prog);
      return;
    }
    // Enough samples are open ahead of this job: wait. A priority-0 job (a plain
    // or batched render, a preview) gets its first pass at once regardless.
    std::uint64_t ahead = 0;
    for (const auto& kv : backlog)
      if (kv.first <= best->priority) ahead += kv.second;
    if (ahead >= target && !(best->priority == 0 && best->segs.empty())) return;
    const std::uint64_t before = best->issued;
    if (!issue_pass(*best)) return;
    backlog[best->priority] += best->pixels * (best->issued - before);
  }
}

// Folds finished segments at the head of a job into its framebuffer (pass order)
// and reports each pass.
void Engine::retire_segments(Job& j, std::vector<PassEvent>* events) {
  Wave& W = *wave_;
  auto free_seg = [&](int slot) {
    Seg& s = segs_[slot];
    W.rad_release(s.rad_begin, s.d.count);
    s = Seg{};
    W.free_segs.push_back(slot);
    gen_dirty_ = true;
  };
  if (j.cancelled) {
    for (auto it = j.segs.begin(); it != j.segs.end();) {
      if (segs_[*it].complete) {
        free_seg(*it);
        it = j.segs.erase(it);
      } else {
        ++it;
      }
    }
    return;
  }
  while (!j.segs.empty() && segs_[j.segs.front()].complete) {
    const int slot = j.segs.front();
    const Seg& s = segs_[slot];
    const bool timed = cfg_.time_kernels;
    if (timed) CK(cudaEventRecord(W.tev[8], stream_));
    CK(launch_accumulate(W.jobs_dev + j.desc_slot, j.pixels, s.d, W.wb.radiance, stream_));
    stats_.kernel_launches++;
    if (timed) {
      CK(cudaEventRecord(W.tev[9], stream_));
      CK(cudaEventSynchronize(W.tev[9]));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, W.tev[8], W.tev[9]));
      stats_.accumulate_ms += ms;
    }
    j.done += s.d.pass_spp;
    free_seg(slot);
    j.segs.pop_front();
    stats_.passes++;
    j.prog.pass++;
    j.prog.spp_done = j.done;
    j.prog.finished = j.done >= j.target;
    j.prog.elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - j.t0).count();
    j.prog.rays = (last_counters_.rays - base_counters_.rays) + (last_counters_.shadow_rays - base_counters_.shadow_rays);
    if (events) events->push_back(PassEvent{j.handle, j.prog});
    if (j.on_pass) j.on_pass(j.prog);
  }
}

void Engine::process_snapshot(std::uint64_t iter, std::vector<PassEvent>* events) {
  Wave& W = *wave_;
  const int r = static_cast<int>(iter % kRing);
  CK(cudaEventSynchronize(W.plan_ev[r]));
  const WaveSnapshot& S = W.ring[r];
  if (S.c.error) {
    const std::uint32_t e = S.c.error;
    throw CudaFailure("device error flag " + std::to_string(e) +
                      (e == 3 ? " (generation table names segment slot " + std::to_string(S.c.error_info) + ")" : ""));
  }
  last_counters_ = S.c;
  std::uint64_t done_sum = 0;
  bool open = false;
  int max_depth = 1;
  const std::uint32_t ns = std::min<std::uint32_t>(W.snapshot_slots, kMaxSegments);
  for (std::uint32_t k = 0; k < ns; ++k) {
    Seg& s = segs_[k];
    // A slot assigned after this plan ran has no data in it yet.
    if (!s.used || s.complete || iter < s.assigned_at) continue;
    s.done = S.seg[k].done;
    s.generated = S.seg[k].generated;
    done_sum += s.done;
    open = true;
    max_depth = std::max(max_depth, jobs_.at(s.job).settings.max_depth);
    if (s.abandoned ? (iter >= s.closed_at && s.done >= s.generated) : s.done >= s.d.count) {
      s.complete = true;
      gen_dirty_ = true;
    } else if (s.in_gen && s.generated >= s.d.count) {
      gen_dirty_ = true;  // fully generated: leaves the table
    }
  }
  // Watchdog: a path lives at most max_depth iterations, so open work that
  // finishes nothing for much longer than that means the wavefront is stuck.
  if (open && done_sum == W.last_done_sum) {
    if (++W.stall > static_cast<std::uint64_t>(max_depth) + kRing + 64)
      throw CudaFailure("wavefront stalled: no sample finished for " + std::to_string(W.stall) + " iterations");
  } else {
    W.stall = 0;
  }
  W.last_done_sum = done_sum;
  for (auto& kv : jobs_) retire_segments(kv.second, events);
}

void Engine::launch_one_iteration() {
  Wave& W = *wave_;
  if (gen_dirty_) write_gen_table();
  const int par = static_cast<int>(W.it & 1);
  const int r = static_cast<int>(W.it % kRing);
  const bool timed = cfg_.time_kernels;
  const bool count = cfg_.count_traversal;
  const Stage stages[4] = {Stage::Plan, Stage::Extend, Stage::Shade, Stage::Shadow};
  LaunchShape shape = cfg_.shape;
  shape.mis = mis_jobs_ > 0;
  for (int k = 0; k < 4; ++k) {
    if (timed) CK(cudaEventRecord(W.tev[2 * k], stream_));
    CK(launch_stage(stages[k], W.wb, par, shape, count, stream_));
    if (timed) CK(cudaEventRecord(W.tev[2 * k + 1], stream_));
  }
  // After the whole iteration, so no event sits between chained kernels; the
  // plan's snapshot and this slot's staged copies are complete once it fires.
  CK(cudaEventRecord(W.plan_ev[r], stream_));
  W.plan_recorded[r] = true;
  if (timed) {
    CK(cudaEventSynchronize(W.tev[7]));
    float ms[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; ++k) CK(cudaEventElapsedTime(&ms[k], W.tev[2 * k], W.tev[2 * k + 1]));
    stats_.plan_ms += ms[0];
    stats_.extend_ms += ms[1];
    stats_.shade_ms += ms[2];
    stats_.shadow_ms += ms[3];
  }
  stats_.extend_launches++;
  stats_.kernel_launches += 4;
  stats_.iterations++;
  W.it++;
}

void Engine::drain(const volatile std::int32_t* cancel, std::vector<PassEvent>* events, double budget_ms,
                   bool return_on_event) {
  Wave& W = *wave_;
  const auto t0 = std::chrono::steady_clock::now();
  const std::size_t events0 = events ? events->size() : 0;
  while (true) {
    if (cancel && *cancel) return;
    refill();
    if (all_jobs_drained()) return;
    launch_one_iteration();
    while (W.seen + kLag < W.it) process_snapshot(W.seen++, events);
    if (return_on_event && events && events->size() > events0) return;
    if (budget_ms < std::numeric_limits<double>::infinity() &&
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() >= budget_ms)
      return;
  }
}

void Engine::abort_all() {
  Wave& W = *wave_;
  CK(cudaStreamSynchronize(stream_));
  WaveCounters c{};
  CK(cudaMemcpy(&c, W.wb.cnt, sizeof(c), cudaMemcpyDeviceToHost));
  c.live[0] = c.live[1] = 0;
  c.n_extend = c.n_shadow = 0;
  CK(cudaMemcpy(W.wb.cnt, &c, sizeof(c), cudaMemcpyHostToDevice));
  for (int k = 0; k < kMaxSegments; ++k)
    if (segs_[k].used) {
      segs_[k] = Seg{};
      W.free_segs.push_back(k);
    }
  W.rad_free.clear();
  W.rad_free.emplace(0, W.rad_cap);
  W.rad_in_free = W.rad_cap;
  for (auto& kv : jobs_) kv.second.segs.clear();
  W.seen = W.it;
  W.stall = 0;
  W.last_done_sum = 0;
  gen_dirty_ = true;
  write_gen_table();
}

void Engine::begin_stats() {
  stats_ = RenderStats{};
  CK(cudaStreamSynchronize(stream_));
  CK(cudaMemcpy(&base_counters_, wave_->wb.cnt, sizeof(base_counters_), cudaMemcpyDeviceToHost));
  last_counters_ = base_counters_;
  CK(cudaEventRecord(ev_begin_, stream_));
}

void Engine::end_stats() {
  finish_timing();
  WaveCounters end{};
  CK(cudaMemcpy(&end, wave_->wb.cnt, sizeof(end), cudaMemcpyDeviceToHost));
  if (end.error) throw CudaFailure("device error flag " + std::to_string(end.error));
  const WaveCounters& b = base_counters_;
  stats_.rays = end.rays - b.rays;
  stats_.shadow_rays = end.shadow_rays - b.shadow_rays;
  stats_.rr_terminated = end.rr_terminated - b.rr_terminated;
  stats_.node_visits = end.node_visits - b.node_visits;
  stats_.prim_tests = end.prim_tests - b.prim_tests;
  stats_.sphere_tests = end.sphere_tests - b.sphere_tests;
  stats_.shadow_node_visits = end.shadow_node_visits - b.shadow_node_visits;
  stats_.shadow_prim_tests = end.shadow_prim_tests - b.shadow_prim_tests;
  stats_.shadow_sphere_tests = end.shadow_sphere_tests - b.shadow_sphere_tests;
}

// ---------------------------------------------------------------------------
RenderProgress Engine::render(int scene_id, const RenderSettings& settings, const RenderOptions& opts,
                              const PassCallback& on_pass, const volatile std::int32_t* cancel) {
  std::vector<RenderProgress> p =
      render_batch({BatchJob{scene_id, settings}}, opts, cancel, on_pass);
  return p[0];
}

std::vector<RenderProgress> Engine::render_batch(const std::vector<BatchJob>& batch, const RenderOptions& opts,
                                                 const volatile std::int32_t* cancel, const PassCallback& on_pass) {
  CK(cudaSetDevice(device_));
  if (serve_open_ > 0) throw std::logic_error("serving requests are open on this context");
  for (auto& f : frames_) free_frame(f);
  frames_.clear();
  frame_settings_.clear();
  ensure_wave();
  begin_stats();
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<int> handles;
  handles.reserve(batch.size());
  for (const BatchJob& b : batch) {
    JobSpec spec;
    spec.scene_id = b.scene_id;
    spec.settings = b.settings;
    spec.opts = opts;
    handles.push_back(open_job(spec, false, on_pass));
  }
  rendering_ = handles;
  bool cancelled = false;
  try {
    drain(cancel, nullptr, std::numeric_limits<double>::infinity(), false);
    cancelled = cancel && *cancel && !all_jobs_drained();
  } catch (...) {
    rendering_.clear();
    abort_all();
    for (int h : handles) {
      Job& j = jobs_.at(h);
      free_frame(j.frame);
      close_job(j);
      jobs_.erase(h);
    }
    throw;
  }
  if (cancelled) abort_all();
  std::vector<RenderProgress> out;
  std::uint64_t samples = 0, invalid = 0;
  if (cancelled)
    for (int h : handles) {
      Job& j = jobs_.at(h);
      if (j.prog.finished) continue;
      j.prog.cancelled = true;
      j.prog.spp_done = j.done;
      if (j.on_pass) j.on_pass(j.prog);
    }
  rendering_.clear();
  for (int h : handles) {
    Job& j = jobs_.at(h);
    out.push_back(j.prog);
    samples += j.pixels * j.done;
    frames_.push_back(j.frame);
    frame_settings_.push_back(j.settings);
    close_job(j);
    jobs_.erase(h);
  }
  end_stats();
  for (const GpuFrame& f : frames_) {
    std::uint64_t inv = 0;
    CK(cudaMemcpy(&inv, f.stats, sizeof(inv), cudaMemcpyDeviceToHost));
    invalid += inv;
  }
  stats_.camera_samples = samples;
  stats_.invalid_samples = invalid;
  stats_.elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  for (auto& p : out) p.rays = stats_.rays + stats_.shadow_rays;
  return out;
}

// ---- serving ----
std::size_t Engine::request_bytes(const JobSpec& spec) const {
  const std::uint64_t px = std::uint64_t(spec.settings.width) * std::uint64_t(spec.settings.height);
  const std::uint32_t first = spec.opts.progressive ? 1u : static_cast<std::uint32_t>(spec.settings.spp);
  return static_cast<std::size_t>(px * (64 + 4) + 32 + px * first * sizeof(float4));
}

int Engine::submit(const JobSpec& spec) {
  CK(cudaSetDevice(device_));
  const int h = open_job(spec, true, nullptr);
  serve_open_++;
  return h;
}

void Engine::pump(double budget_ms, bool return_on_event, std::vector<PassEvent>& events) {
  CK(cudaSetDevice(device_));
  if (!wave_) return;
  drain(nullptr, &events, budget_ms, return_on_event);
}

void Engine::cancel_request(int request) {
  auto it = jobs_.find(request);
  if (it == jobs_.end() || !it->second.serving) throw std::invalid_argument("unknown request " + std::to_string(request));
  Job& j = it->second;
  if (j.cancelled || j.prog.finished) return;
  j.cancelled = true;
  j.prog.cancelled = true;
  for (int slot : j.segs) {
    Seg& s = segs_[slot];
    if (s.complete) continue;
    s.abandoned = true;
    s.closed_at = wave_->it;  // the next plan no longer lists it
  }
  gen_dirty_ = true;
  retire_segments(j, nullptr);
}

void Engine::release_request(int request) {
  auto it = jobs_.find(request);
  if (it == jobs_.end() || !it->second.serving) throw std::invalid_argument("unknown request " + std::to_string(request));
  Job& j = it->second;
  if (!j.drained()) throw std::logic_error("request " + std::to_string(request) + " is still rendering");
  free_frame(j.frame);
  close_job(j);
  jobs_.erase(it);
  serve_open_--;
}

void Engine::reserve_pool(std::size_t bytes) {
  CK(cudaSetDevice(device_));
  if (!bvh_preloaded_) {
    gpu_bvh_preload();
    bvh_preloaded_ = true;
  }
  if (bytes <= pool_reserved_) return;
  void* p = nullptr;
  count_allocation();
  CK(cudaMallocFromPoolAsync(&p, bytes, pool_, stream_));
  CK(cudaFreeAsync(p, stream_));
  CK(cudaStreamSynchronize(stream_));
  pool_reserved_ = bytes;
}

std::size_t Engine::requests_rendering() const {
  std::size_t n = 0;
  for (const auto& kv : jobs_)
    if (kv.second.serving && !kv.second.drained()) ++n;
  return n;
}

const GpuFrame& Engine::request_frame(int request) const {
  auto it = jobs_.find(request);
  if (it == jobs_.end() || !it->second.serving) throw std::invalid_argument("unknown request " + std::to_string(request));
  return it->second.frame;
}

const RenderProgress& Engine::request_progress(int request) const {
  auto it = jobs_.find(request);
  if (it == jobs_.end() || !it->second.serving) throw std::invalid_argument("unknown request " + std::to_string(request));
  return it->second.prog;
}

// ---- framebuffer reads ----
const GpuFrame& Engine::frame(int job) const {
  const std::size_t j = job < 0 ? 0 : static_cast<std::size_t>(job);
  if (!rendering_.empty()) {  // inside a pass callback: the render in progress
    if (j >= rendering_.size()) throw std::invalid_argument("no framebuffer for job " + std::to_string(job));
    return jobs_.at(rendering_[j]).frame;
  }
  if (j >= frames_.size()) throw std::invalid_argument("no framebuffer for job " + std::to_string(job));
  return frames_[j];
}

void Engine::read_mean(int job, double* rgb) const { read_mean_frame(frame(job), rgb); }

void Engine::read_moments(int job, double* sum, double* sumsq, std::uint32_t* count) const {
  const GpuFrame& f = frame(job);
  const std::uint64_t px = std::uint64_t(f.width) * f.height;
  if (sum) CK(cudaMemcpyAsync(sum, f.sum, px * 4 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  if (sumsq) CK(cudaMemcpyAsync(sumsq, f.sumsq, px * 4 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  if (count) CK(cudaMemcpyAsync(count, f.count, px * sizeof(std::uint32_t), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
}

void Engine::read_image(int job, ToneMap op, double exposure, std::uint8_t* rgb) const {
  read_image_frame(frame(job), op, exposure, rgb);
}

void Engine::read_mean_frame(const GpuFrame& f, double* rgb) const {
  const std::uint64_t px = std::uint64_t(f.width) * f.height;
  double* tmp = dev_alloc_async<double>(px * 3, pool_, stream_);
  CK(launch_resolve(f.sum, f.count, px, 0, 1.0, nullptr, tmp, stream_));
  CK(cudaMemcpyAsync(rgb, tmp, px * 3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  CK(cudaFreeAsync(tmp, stream_));
  CK(cudaStreamSynchronize(stream_));
}

void Engine::read_image_frame(const GpuFrame& f, ToneMap op, double exposure, std::uint8_t* rgb) const {
  const std::uint64_t px = std::uint64_t(f.width) * f.height;
  std::uint8_t* tmp = dev_alloc_async<std::uint8_t>(px * 3, pool_, stream_);
  CK(launch_resolve(f.sum, f.count, px, static_cast<int>(op), exposure, tmp, nullptr, stream_));
  CK(cudaMemcpyAsync(rgb, tmp, px * 3, cudaMemcpyDeviceToHost, stream_));
  CK(cudaFreeAsync(tmp, stream_));
  CK(cudaStreamSynchronize(stream_));
}

void Engine::read_images(int n, const int* jobs, const ToneMap* ops, const double* exposures, std::uint8_t* const* rgb) {
  CK(cudaSetDevice(device_));
  if (n <= 0) return;
  std::vector<const GpuFrame*> fr(static_cast<std::size_t>(n));
  std::vector<std::size_t> at(static_cast<std::size_t>(n) + 1, 0), bytes(static_cast<std::size_t>(n));
  for (int k = 0; k < n; ++k) {
    fr[k] = &frame(jobs[k]);
    bytes[k] = std::uint64_t(fr[k]->width) * fr[k]->height * 3;
    at[k + 1] = at[k] + ((bytes[k] + 255) & ~std::size_t(255));
  }
  const std::size_t total = at[n];
  if (total == 0) return;
  std::uint8_t* dev = dev_alloc_async<std::uint8_t>(total, pool_, stream_);
  for (int k = 0; k < n; ++k)
    CK(launch_resolve(fr[k]->sum, fr[k]->count, std::uint64_t(fr[k]->width) * fr[k]->height, static_cast<int>(ops[k]),
                      exposures[k], dev + at[k], nullptr, stream_));
  if (readback_cap_ < total) {
    CK(cudaStreamSynchronize(stream_));
    if (readback_host_) CK(cudaFreeHost(readback_host_));
    readback_host_ = nullptr;
    readback_cap_ = 0;
    count_allocation();
    CK(cudaMallocHost(reinterpret_cast<void**>(&readback_host_), total));
    readback_cap_ = total;
  }
  CK(cudaMemcpyAsync(readback_host_, dev, total, cudaMemcpyDeviceToHost, stream_));
  CK(cudaFreeAsync(dev, stream_));
  CK(cudaStreamSynchronize(stream_));
  // Out of pinned memory into the caller's buffers, one image per task.
  std::atomic<int> next{0};
  auto copy = [&] {
    for (int k; (k = next.fetch_add(1)) < n;) std::memcpy(rgb[k], readback_host_ + at[k], bytes[k]);
  };
  const int workers = std::min(n, static_cast<int>(std::min(16u, std::max(1u, std::thread::hardware_concurrency()))));
  std::vector<std::thread> pool;
  for (int w = 1; w < workers; ++w) pool.emplace_back(copy);
  copy();
  for (auto& t : pool) t.join();
}

// ---------------------------------------------------------------------------
void Engine::trace_closest(int scene_id, const float* rays, std::uint64_t n, bool brute, float* t, std::int32_t* prim,
                           std::int32_t* is_plane, float* bary) {
  CK(cudaSetDevice(device_));
  GpuScene& sc = scene(scene_id);
  if (n == 0) return;
  if (n > 0xFFFFFFFFull) throw std::invalid_argument("too many rays in one call");
  if (!sc.prims64 && cfg_.refine_hits) {
    // Double originals in slot order, for the reported distance only.
    std::vector<double> g(std::max<std::size_t>(1, sc.slot_prim.size()) * 9, 0.0);
    for (std::size_t k = 0; k < sc.slot_prim.size(); ++k) {
      const Prim& p = sc.host->prims[sc.slot_prim[k]];
      const D3 v[3] = {p.a, p.kind == Prim::kSphere ? D3{p.b.x, 0, 0} : p.b, p.c};
      for (int j = 0; j < 3; ++j) {
        g[9 * k + 3 * j] = v[j].x;
        g[9 * k + 3 * j + 1] = v[j].y;
        g[9 * k + 3 * j + 2] = v[j].z;
      }
    }
    std::vector<double> pl(std::max<std::size_t>(1, sc.host->planes.size()) * 6, 0.0);
    for (std::size_t k = 0; k < sc.host->planes.size(); ++k) {
      const PlanePrim& q = sc.host->planes[k];
      const double r[6] = {q.point.x, q.point.y, q.point.z, q.normal.x, q.normal.y, q.normal.z};
      std::copy(r, r + 6, pl.begin() + 6 * k);
    }
    std::size_t bytes = 0;
    sc.prims64 = dev_upload(g, stream_, bytes);
    sc.planes64 = dev_upload(pl, stream_, bytes);
    CK(cudaStreamSynchronize(stream_));
  }
  RenderSettings s = sc.host->settings;
  s.use_bvh = !brute;
  RtgSceneDev d = job_descriptor(sc, s, GpuFrame{});
  if (!cfg_.refine_hits) d.prims64 = d.planes64 = nullptr;
  RtgSceneDev* dd = dev_alloc<RtgSceneDev>(1);
  float4* in = dev_alloc<float4>(2 * n);
  float4* out = dev_alloc<float4>(n);
  CK(cudaMemcpyAsync(dd, &d, sizeof(d), cudaMemcpyHostToDevice, stream_));
  CK(cudaMemcpyAsync(in, rays, n * 8 * sizeof(float), cudaMemcpyHostToDevice, stream_));
  CK(launch_ray_closest(dd, in, static_cast<std::uint32_t>(n), out, brute ? 1 : 0, cfg_.shape.closest_tree, stream_));
  std::vector<float4> host(n);
  CK(cudaMemcpyAsync(host.data(), out, n * sizeof(float4), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  dev_free(dd);
  dev_free(in);
  dev_free(out);
  for (std::uint64_t i = 0; i < n; ++i) {
    std::uint32_t w;
    std::memcpy(&w, &host[i].y, 4);
    const bool miss = w == kHitMiss;
    const bool plane = !miss && (w & kHitPlaneBit);
    if (t) t[i] = miss ? 0.f : host[i].x;
    if (prim) prim[i] = miss ? -1 : (plane ? static_cast<std::int32_t>(w & ~kHitPlaneBit) : static_cast<std::int32_t>(sc.slot_prim[w]));
    if (is_plane) is_plane[i] = plane ? 1 : 0;
    if (bary) {
      bary[2 * i] = host[i].z;
      bary[2 * i + 1] = host[i].w;
    }
  }
}

void Engine::trace_any(int scene_id, const float* rays, std::uint64_t n, bool brute, std::uint8_t* occluded) {
  CK(cudaSetDevice(device_));
  GpuScene& sc = scene(scene_id);
  if (n == 0) return;
  if (n > 0xFFFFFFFFull) throw std::invalid_argument("too many rays in one call");
  RenderSettings s = sc.host->settings;
  s.use_bvh = !brute;
  const RtgSceneDev d = job_descriptor(sc, s, GpuFrame{});
  RtgSceneDev* dd = dev_alloc<RtgSceneDev>(1);
  float4* in = dev_alloc<float4>(2 * n);
  std::uint32_t* out = dev_alloc<std::uint32_t>(n);
  CK(cudaMemcpyAsync(dd, &d, sizeof(d), cudaMemcpyHostToDevice, stream_));
  CK(cudaMemcpyAsync(in, rays, n * 8 * sizeof(float), cudaMemcpyHostToDevice, stream_));
  CK(launch_ray_any(dd, in, static_cast<std::uint32_t>(n), out, brute ? 1 : 0, cfg_.shape.shadow_tree, stream_));
  std::vector<std::uint32_t> host(n);
  CK(cudaMemcpyAsync(host.data(), out, n * sizeof(std::uint32_t), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  dev_free(dd);
  dev_free(in);
  dev_free(out);
  for (std::uint64_t i = 0; i < n; ++i) occluded[i] = host[i] ? 1 : 0;
}

}  // namespace rtg

namespace rtg {

RtgSceneDev Engine::query_descriptor(int scene_id, bool brute) {
  GpuScene& sc = scene(scene_id);
  RenderSettings s = sc.host->settings;
  s.use_bvh = !brute;
  RtgSceneDev d = job_descriptor(sc, s, GpuFrame{});
  if (!cfg_.refine_hits) d.prims64 = d.planes64 = nullptr;
  return d;
}

}  // namespace rtg
