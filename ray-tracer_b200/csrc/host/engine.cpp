#include "host/engine.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

namespace rtg {

namespace {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaFailure(std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(expr) check((expr), #expr)

template <class T>
T* dev_alloc(std::size_t n) {
  void* p = nullptr;
  CK(cudaMalloc(&p, std::max<std::size_t>(n, 1) * sizeof(T)));
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

std::uint32_t pass_size(std::uint32_t done, std::uint32_t target, const RenderOptions& o) {
  std::uint32_t k = target - done;
  if (o.progressive) {
    const std::uint32_t grow = std::max<std::uint32_t>(1u, done);
    const std::uint32_t cap = static_cast<std::uint32_t>(std::max(1, o.max_pass_spp));
    k = std::min({k, grow, cap});
  }
  return k;
}

constexpr int kRing = 8;  // pinned counter snapshots in flight
constexpr int kLag = 2;   // iterations queued ahead of the termination check

}  // namespace

struct Engine::Wave {
  WaveBuffers wb{};
  std::uint64_t radiance_cap = 0;
  RtgSceneDev* jobs_dev = nullptr;
  std::size_t jobs_cap = 0;
  std::uint32_t* ids_dev = nullptr;
  std::uint64_t* begin_dev = nullptr;
  std::size_t table_cap = 0;
  WaveCounters* ring = nullptr;  // pinned host
  cudaEvent_t ring_ev[kRing]{};
  cudaEvent_t tev[8]{};
};

Engine::Engine(int device) : device_(device) {
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  CK(cudaEventCreate(&ev_begin_));
  CK(cudaEventCreate(&ev_end_));
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
  for (auto& kv : scenes_) {
    GpuScene& s = *kv.second;
    dev_free(s.nodes); dev_free(s.prims); dev_free(s.slot_material); dev_free(s.slot_normals);
    dev_free(s.planes); dev_free(s.materials); dev_free(s.lights);
    dev_free(s.prims64); dev_free(s.planes64);
  }
  reset_wave();
  cudaEventDestroy(ev_begin_);
  cudaEventDestroy(ev_end_);
  cudaStreamDestroy(stream_);
}

void Engine::reset_wave() {
  cudaStreamSynchronize(stream_);
  if (wave_) {
    WaveBuffers& b = wave_->wb;
    for (int i = 0; i < 2; ++i) { dev_free(b.st_a[i]); dev_free(b.st_b[i]); dev_free(b.st_c[i]); dev_free(b.st_d[i]); }
    dev_free(b.hits); dev_free(b.sh_a); dev_free(b.sh_b); dev_free(b.sh_c); dev_free(b.radiance); dev_free(b.cnt);
    dev_free(wave_->jobs_dev); dev_free(wave_->ids_dev); dev_free(wave_->begin_dev);
    if (wave_->ring) cudaFreeHost(wave_->ring);
    for (auto& e : wave_->ring_ev) if (e) cudaEventDestroy(e);
    for (auto& e : wave_->tev) if (e) cudaEventDestroy(e);
    wave_.reset();
  }
}

int Engine::add_scene(CompiledScene scene) {
  CK(cudaSetDevice(device_));
  auto gs = std::make_unique<GpuScene>();
  FlatScene flat = flatten(scene);
  gs->root = flat.root;
  gs->n_slots = static_cast<std::int32_t>(flat.slot_prim.size());
  gs->n_planes = static_cast<std::int32_t>(flat.planes.size());
  gs->n_lights = static_cast<std::int32_t>(flat.lights.size());
  std::size_t bytes = 0;
  gs->nodes = dev_upload(flat.nodes, stream_, bytes);
  gs->prims = dev_upload(flat.prims, stream_, bytes);
  gs->slot_material = dev_upload(flat.slot_material, stream_, bytes);
  gs->slot_normals = dev_upload(flat.slot_normals, stream_, bytes);
  gs->planes = dev_upload(flat.planes, stream_, bytes);
  gs->materials = dev_upload(flat.materials, stream_, bytes);
  gs->lights = dev_upload(flat.lights, stream_, bytes);
  gs->device_bytes = bytes;
  gs->slot_prim = std::move(flat.slot_prim);
  gs->host = std::move(scene);
  CK(cudaStreamSynchronize(stream_));  // the host vectors die with `flat`
  const int id = next_scene_++;
  scenes_[id] = std::move(gs);
  return id;
}

void Engine::release_scene(int id) {
  auto it = scenes_.find(id);
  if (it == scenes_.end()) throw std::invalid_argument("unknown scene id " + std::to_string(id));
  cudaStreamSynchronize(stream_);
  GpuScene& s = *it->second;
  dev_free(s.nodes); dev_free(s.prims); dev_free(s.slot_material); dev_free(s.slot_normals);
  dev_free(s.planes); dev_free(s.materials); dev_free(s.lights);
    dev_free(s.prims64); dev_free(s.planes64);
  scenes_.erase(it);
}

GpuScene& Engine::scene(int id) {
  auto it = scenes_.find(id);
  if (it == scenes_.end()) throw std::invalid_argument("unknown scene id " + std::to_string(id));
  return *it->second;
}

void Engine::ensure_wave(std::uint64_t pass_samples) {
  if (!wave_) {
    wave_ = std::make_unique<Wave>();
    WaveBuffers& b = wave_->wb;
    const std::uint32_t P = cfg_.pool_paths;
    b.capacity = P;
    for (int i = 0; i < 2; ++i) {
      b.st_a[i] = dev_alloc<float4>(P);
      b.st_b[i] = dev_alloc<float4>(P);
      b.st_c[i] = dev_alloc<float4>(P);
      b.st_d[i] = dev_alloc<uint4>(P);
    }
    b.hits = dev_alloc<float4>(P);
    b.sh_a = dev_alloc<float4>(P);
    b.sh_b = dev_alloc<float4>(P);
    b.sh_c = dev_alloc<float4>(P);
    b.cnt = dev_alloc<WaveCounters>(1);
    CK(cudaMallocHost(reinterpret_cast<void**>(&wave_->ring), sizeof(WaveCounters) * kRing));
    for (auto& e : wave_->ring_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : wave_->tev) CK(cudaEventCreate(&e));
  }
  if (pass_samples > wave_->radiance_cap) {
    dev_free(wave_->wb.radiance);
    wave_->wb.radiance = dev_alloc<float4>(pass_samples);
    wave_->radiance_cap = pass_samples;
  }
}

GpuFrame Engine::make_frame(int w, int h) {
  GpuFrame f;
  f.width = w;
  f.height = h;
  const std::size_t px = std::size_t(w) * std::size_t(h);
  f.sum = dev_alloc<double>(px * 4);
  f.sumsq = dev_alloc<double>(px * 4);
  f.count = dev_alloc<std::uint32_t>(px);
  f.stats = dev_alloc<std::uint64_t>(4);
  CK(cudaMemsetAsync(f.sum, 0, px * 4 * sizeof(double), stream_));
  CK(cudaMemsetAsync(f.sumsq, 0, px * 4 * sizeof(double), stream_));
  CK(cudaMemsetAsync(f.count, 0, px * sizeof(std::uint32_t), stream_));
  CK(cudaMemsetAsync(f.stats, 0, 4 * sizeof(std::uint64_t), stream_));
  return f;
}

void Engine::free_frame(GpuFrame& f) {
  dev_free(f.sum); dev_free(f.sumsq); dev_free(f.count); dev_free(f.stats);
  f = GpuFrame{};
}

RtgSceneDev Engine::job_descriptor(const GpuScene& sc, const RenderSettings& s, const GpuFrame& f) const {
  RtgSceneDev d{};
  describe(sc.host, s, d);
  d.nodes = sc.nodes;
  d.prims = sc.prims;
  d.slot_material = sc.slot_material;
  d.slot_normals = sc.slot_normals;
  d.planes = sc.planes;
  d.materials = sc.materials;
  d.lights = sc.lights;
  d.root = sc.root;
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

bool Engine::run_pass(std::vector<RtgSceneDev>& jobs, const std::vector<std::uint32_t>& ids, std::uint64_t total,
                      bool direct, const volatile std::int32_t* cancel) {
  Wave& W = *wave_;
  // Stage descriptors and the pass table.
  if (jobs.size() > W.jobs_cap) {
    dev_free(W.jobs_dev);
    W.jobs_dev = dev_alloc<RtgSceneDev>(jobs.size());
    W.jobs_cap = jobs.size();
  }
  if (ids.size() > W.table_cap) {
    dev_free(W.ids_dev);
    dev_free(W.begin_dev);
    W.ids_dev = dev_alloc<std::uint32_t>(ids.size());
    W.begin_dev = dev_alloc<std::uint64_t>(ids.size());
    W.table_cap = ids.size();
  }
  std::vector<std::uint64_t> begin(ids.size());
  std::uint64_t acc = 0;
  for (std::size_t k = 0; k < ids.size(); ++k) {
    begin[k] = acc;
    acc += jobs[ids[k]].work_count;
  }
  CK(cudaMemcpyAsync(W.jobs_dev, jobs.data(), jobs.size() * sizeof(RtgSceneDev), cudaMemcpyHostToDevice, stream_));
  CK(cudaMemcpyAsync(W.ids_dev, ids.data(), ids.size() * sizeof(std::uint32_t), cudaMemcpyHostToDevice, stream_));
  CK(cudaMemcpyAsync(W.begin_dev, begin.data(), begin.size() * sizeof(std::uint64_t), cudaMemcpyHostToDevice, stream_));
  PassTable pt{W.jobs_dev, W.ids_dev, W.begin_dev, static_cast<std::int32_t>(ids.size())};

  WaveCounters init{};
  init.total_work = total;
  CK(cudaMemcpyAsync(W.wb.cnt, &init, sizeof(init), cudaMemcpyHostToDevice, stream_));
  const bool timed = cfg_.time_kernels;
  bool cancelled = false;

  if (direct) {
    if (timed) CK(cudaEventRecord(W.tev[0], stream_));
    CK(launch_direct(pt, total, W.wb.radiance, W.wb.cnt, stream_));
    stats_.kernel_launches += 1;
    if (timed) {
      CK(cudaEventRecord(W.tev[1], stream_));
      CK(cudaEventSynchronize(W.tev[1]));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, W.tev[0], W.tev[1]));
      stats_.direct_ms += ms;
    }
  } else {
    // Generous bound on iterations: every path needs at most max_depth of them
    // and the pool refills at least once per max_depth iterations.
    int max_depth = 1;
    for (std::uint32_t id : ids) max_depth = std::max(max_depth, jobs[id].max_depth);
    const std::uint64_t fills = total / W.wb.capacity + 2;
    const std::uint64_t it_cap = fills * static_cast<std::uint64_t>(max_depth + 2) * 4 + 64;
    std::uint64_t it = 0;
    bool done = false;
    while (!done) {
      if (it > it_cap) throw CudaFailure("wavefront did not drain (iteration bound exceeded)");
      const int par = static_cast<int>(it & 1);
      if (timed) {
        float ms[3] = {0, 0, 0};
        const Stage stages[3] = {Stage::Extend, Stage::Shade, Stage::Shadow};
        for (int k = 0; k < 3; ++k) {
          CK(cudaEventRecord(W.tev[2 * k], stream_));
          CK(launch_stage(stages[k], W.wb, pt, par, cfg_.shape, cfg_.count_traversal, stream_));
          CK(cudaEventRecord(W.tev[2 * k + 1], stream_));
        }
        CK(cudaEventSynchronize(W.tev[5]));
        for (int k = 0; k < 3; ++k) CK(cudaEventElapsedTime(&ms[k], W.tev[2 * k], W.tev[2 * k + 1]));
        stats_.extend_ms += ms[0];
        stats_.shade_ms += ms[1];
        stats_.shadow_ms += ms[2];
        stats_.extend_launches++;
      } else {
        CK(launch_iteration(W.wb, pt, par, cfg_.shape, cfg_.count_traversal, stream_));
      }
      stats_.kernel_launches += 3;
      const int slot = static_cast<int>(it % kRing);
      CK(cudaMemcpyAsync(&W.ring[slot], W.wb.cnt, sizeof(WaveCounters), cudaMemcpyDeviceToHost, stream_));
      CK(cudaEventRecord(W.ring_ev[slot], stream_));
      stats_.iterations++;
      if (it >= static_cast<std::uint64_t>(kLag)) {
        const std::uint64_t j = it - kLag;
        CK(cudaEventSynchronize(W.ring_ev[j % kRing]));
        const WaveCounters& c = W.ring[j % kRing];
        if (c.error) throw CudaFailure("device error flag " + std::to_string(c.error));
        if (c.live[(j + 1) & 1] == 0 && c.next_work >= c.total_work) done = true;
      }
      ++it;
      if (cancel && *cancel) {
        cancelled = true;
        break;
      }
    }
  }
  if (!cancelled) {
    if (timed) CK(cudaEventRecord(W.tev[6], stream_));
    for (std::uint32_t id : ids) CK(launch_accumulate(W.jobs_dev + id, jobs[id], W.wb.radiance, stream_));
    stats_.kernel_launches += ids.size();
    if (timed) CK(cudaEventRecord(W.tev[7], stream_));
  }
  CK(cudaStreamSynchronize(stream_));
  if (timed && !cancelled) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, W.tev[6], W.tev[7]));
    stats_.accumulate_ms += ms;
  }
  WaveCounters end{};
  CK(cudaMemcpy(&end, W.wb.cnt, sizeof(end), cudaMemcpyDeviceToHost));
  if (end.error) throw CudaFailure("device error flag " + std::to_string(end.error) +
                                   (end.error == 2 ? " (direct integrator branch stack overflow)" : ""));
  stats_.rays += end.rays;
  stats_.shadow_rays += end.shadow_rays;
  stats_.rr_terminated += end.rr_terminated;
  stats_.node_visits += end.node_visits;
  stats_.prim_tests += end.prim_tests;
  stats_.sphere_tests += end.sphere_tests;
  stats_.shadow_node_visits += end.shadow_node_visits;
  stats_.shadow_prim_tests += end.shadow_prim_tests;
  stats_.shadow_sphere_tests += end.shadow_sphere_tests;
  stats_.passes++;
  return !cancelled;
}

RenderProgress Engine::render(int scene_id, const RenderSettings& settings, const RenderOptions& opts,
                              const PassCallback& on_pass, const volatile std::int32_t* cancel) {
  CK(cudaSetDevice(device_));
  GpuScene& sc = scene(scene_id);
  for (auto& f : frames_) free_frame(f);
  frames_.clear();
  stats_ = RenderStats{};
  const auto t0 = std::chrono::steady_clock::now();

  frames_.push_back(make_frame(settings.width, settings.height));
  std::vector<RtgSceneDev> jobs(1, job_descriptor(sc, settings, frames_[0]));
  CK(cudaEventRecord(ev_begin_, stream_));

  const std::uint64_t pixels = std::uint64_t(settings.width) * std::uint64_t(settings.height);
  const std::uint32_t target = static_cast<std::uint32_t>(settings.spp);
  const bool direct = settings.integrator == Integrator::Direct;
  RenderProgress prog;
  prog.spp_target = settings.spp;
  std::uint32_t done = 0;
  while (done < target) {
    std::uint32_t k = pass_size(done, target, opts);
    const std::uint64_t fit = std::max<std::uint64_t>(1, cfg_.max_pass_samples / std::max<std::uint64_t>(1, pixels));
    k = static_cast<std::uint32_t>(std::min<std::uint64_t>(k, fit));
    ensure_wave(pixels * k);
    RtgSceneDev& J = jobs[0];
    J.pass_s0 = done;
    J.pass_spp = k;
    J.work_begin = 0;
    J.work_count = pixels * k;
    J.sample_base = 0;
    const bool complete = run_pass(jobs, {0u}, pixels * k, direct, cancel);
    prog.pass++;
    prog.elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    prog.rays = stats_.rays + stats_.shadow_rays;
    if (complete) done += k;
    stats_.camera_samples = pixels * done;
    stats_.elapsed_ms = prog.elapsed_ms;
    if (!complete || (cancel && *cancel)) {
      prog.cancelled = true;
      prog.spp_done = done;
      if (on_pass) on_pass(prog);
      break;
    }
    prog.spp_done = done;
    prog.finished = done >= target;
    if (on_pass) on_pass(prog);
  }
  finish_timing();
  std::uint64_t invalid = 0;
  CK(cudaMemcpy(&invalid, frames_[0].stats, sizeof(invalid), cudaMemcpyDeviceToHost));
  stats_.invalid_samples = invalid;
  stats_.elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return prog;
}

std::vector<RenderProgress> Engine::render_batch(const std::vector<BatchJob>& batch, const RenderOptions& opts,
                                                 const volatile std::int32_t* cancel) {
  CK(cudaSetDevice(device_));
  for (auto& f : frames_) free_frame(f);
  frames_.clear();
  stats_ = RenderStats{};
  const auto t0 = std::chrono::steady_clock::now();
  const std::size_t n = batch.size();
  std::vector<RtgSceneDev> jobs;
  jobs.reserve(n);
  for (std::size_t j = 0; j < n; ++j) {
    frames_.push_back(make_frame(batch[j].settings.width, batch[j].settings.height));
    jobs.push_back(job_descriptor(scene(batch[j].scene_id), batch[j].settings, frames_.back()));
  }
  CK(cudaEventRecord(ev_begin_, stream_));
  std::vector<RenderProgress> prog(n);
  std::vector<std::uint32_t> done(n, 0);
  for (std::size_t j = 0; j < n; ++j) prog[j].spp_target = batch[j].settings.spp;
  // Direct-integrator jobs run through their own kernel; everything else shares the wavefront.
  for (int direct_group = 0; direct_group < 2; ++direct_group) {
    while (true) {
      std::vector<std::uint32_t> ids;
      std::uint64_t total = 0;
      for (std::size_t j = 0; j < n; ++j) {
        const RenderSettings& s = batch[j].settings;
        const bool is_direct = s.integrator == Integrator::Direct;
        if (is_direct != (direct_group == 1)) continue;
        const std::uint32_t target = static_cast<std::uint32_t>(s.spp);
        if (done[j] >= target) continue;
        const std::uint64_t pixels = std::uint64_t(s.width) * std::uint64_t(s.height);
        std::uint32_t k = pass_size(done[j], target, opts);
        const std::uint64_t fit = std::max<std::uint64_t>(1, cfg_.max_pass_samples / std::max<std::uint64_t>(1, pixels));
        k = static_cast<std::uint32_t>(std::min<std::uint64_t>(k, fit));
        // Keep one batched pass within the radiance buffer; later passes pick up the rest.
        if (!ids.empty() && total + pixels * k > cfg_.max_pass_samples) continue;
        RtgSceneDev& J = jobs[j];
        J.pass_s0 = done[j];
        J.pass_spp = k;
        J.work_begin = total;
        J.work_count = pixels * k;
        J.sample_base = total;
        ids.push_back(static_cast<std::uint32_t>(j));
        total += pixels * k;
      }
      if (ids.empty()) break;
      ensure_wave(total);
      const bool complete = run_pass(jobs, ids, total, direct_group == 1, cancel);
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      for (std::uint32_t id : ids) {
        if (complete) done[id] += jobs[id].pass_spp;
        prog[id].pass++;
        prog[id].spp_done = done[id];
        prog[id].elapsed_ms = ms;
        prog[id].finished = done[id] >= static_cast<std::uint32_t>(batch[id].settings.spp);
      }
      if (!complete || (cancel && *cancel)) {
        for (auto& p : prog) p.cancelled = !p.finished;
        finish_timing();
        stats_.elapsed_ms = ms;
        return prog;
      }
    }
  }
  finish_timing();
  std::uint64_t samples = 0, invalid = 0;
  for (std::size_t j = 0; j < n; ++j) {
    std::uint64_t inv = 0;
    CK(cudaMemcpy(&inv, frames_[j].stats, sizeof(inv), cudaMemcpyDeviceToHost));
    invalid += inv;
    samples += std::uint64_t(batch[j].settings.width) * batch[j].settings.height * done[j];
  }
  stats_.camera_samples = samples;
  stats_.invalid_samples = invalid;
  stats_.elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  for (auto& p : prog) p.rays = stats_.rays + stats_.shadow_rays;
  return prog;
}

const GpuFrame& Engine::frame(int job) const {
  const std::size_t j = job < 0 ? 0 : static_cast<std::size_t>(job);
  if (j >= frames_.size()) throw std::invalid_argument("no framebuffer for job " + std::to_string(job));
  return frames_[j];
}

void Engine::read_mean(int job, double* rgb) const {
  const GpuFrame& f = frame(job);
  const std::uint64_t px = std::uint64_t(f.width) * f.height;
  double* tmp = dev_alloc<double>(px * 3);
  // The resolve kernel reads the framebuffer through a descriptor.
  RtgSceneDev d{};
  d.width = f.width;
  d.height = f.height;
  d.fb_sum = f.sum;
  d.fb_sumsq = f.sumsq;
  d.fb_count = f.count;
  RtgSceneDev* dd = dev_alloc<RtgSceneDev>(1);
  CK(cudaMemcpyAsync(dd, &d, sizeof(d), cudaMemcpyHostToDevice, stream_));
  CK(launch_resolve(dd, px, 0, 1.0, nullptr, tmp, stream_));
  CK(cudaMemcpyAsync(rgb, tmp, px * 3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  dev_free(tmp);
  dev_free(dd);
}

void Engine::read_moments(int job, double* sum, double* sumsq, std::uint32_t* count) const {
  const GpuFrame& f = frame(job);
  const std::uint64_t px = std::uint64_t(f.width) * f.height;
  if (sum) CK(cudaMemcpyAsync(sum, f.sum, px * 4 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  if (sumsq) CK(cudaMemcpyAsync(sumsq, f.sumsq, px * 4 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  if (count) CK(cudaMemcpyAsync(count, f.count, px * sizeof(std::uint32_t), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
}

void Engine::read_image(int job, ToneMap op, double exposure, std::uint8_t* rgb) const {
  const GpuFrame& f = frame(job);
  const std::uint64_t px = std::uint64_t(f.width) * f.height;
  std::uint8_t* tmp = dev_alloc<std::uint8_t>(px * 3);
  RtgSceneDev d{};
  d.width = f.width;
  d.height = f.height;
  d.fb_sum = f.sum;
  d.fb_sumsq = f.sumsq;
  d.fb_count = f.count;
  RtgSceneDev* dd = dev_alloc<RtgSceneDev>(1);
  CK(cudaMemcpyAsync(dd, &d, sizeof(d), cudaMemcpyHostToDevice, stream_));
  CK(launch_resolve(dd, px, static_cast<int>(op), exposure, tmp, nullptr, stream_));
  CK(cudaMemcpyAsync(rgb, tmp, px * 3, cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  dev_free(tmp);
  dev_free(dd);
}

void Engine::trace_closest(int scene_id, const float* rays, std::uint64_t n, bool brute, float* t, std::int32_t* prim,
                           std::int32_t* is_plane, float* bary) {
  CK(cudaSetDevice(device_));
  GpuScene& sc = scene(scene_id);
  if (n == 0) return;
  if (n > 0xFFFFFFFFull) throw std::invalid_argument("too many rays in one call");
  if (!sc.prims64) {
    // Double originals in slot order, for the reported distance only.
    std::vector<double> g(std::max<std::size_t>(1, sc.slot_prim.size()) * 9, 0.0);
    for (std::size_t k = 0; k < sc.slot_prim.size(); ++k) {
      const Prim& p = sc.host.prims[sc.slot_prim[k]];
      const D3 v[3] = {p.a, p.kind == Prim::kSphere ? D3{p.b.x, 0, 0} : p.b, p.c};
      for (int j = 0; j < 3; ++j) {
        g[9 * k + 3 * j] = v[j].x;
        g[9 * k + 3 * j + 1] = v[j].y;
        g[9 * k + 3 * j + 2] = v[j].z;
      }
    }
    std::vector<double> pl(std::max<std::size_t>(1, sc.host.planes.size()) * 6, 0.0);
    for (std::size_t k = 0; k < sc.host.planes.size(); ++k) {
      const PlanePrim& q = sc.host.planes[k];
      const double r[6] = {q.point.x, q.point.y, q.point.z, q.normal.x, q.normal.y, q.normal.z};
      std::copy(r, r + 6, pl.begin() + 6 * k);
    }
    std::size_t bytes = 0;
    sc.prims64 = dev_upload(g, stream_, bytes);
    sc.planes64 = dev_upload(pl, stream_, bytes);
    CK(cudaStreamSynchronize(stream_));
  }
  RenderSettings s = sc.host.settings;
  s.use_bvh = !brute;
  const RtgSceneDev d = job_descriptor(sc, s, GpuFrame{});
  RtgSceneDev* dd = dev_alloc<RtgSceneDev>(1);
  float4* in = dev_alloc<float4>(2 * n);
  float4* out = dev_alloc<float4>(n);
  CK(cudaMemcpyAsync(dd, &d, sizeof(d), cudaMemcpyHostToDevice, stream_));
  CK(cudaMemcpyAsync(in, rays, n * 8 * sizeof(float), cudaMemcpyHostToDevice, stream_));
  CK(launch_ray_closest(dd, in, static_cast<std::uint32_t>(n), out, brute ? 1 : 0, stream_));
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
  RenderSettings s = sc.host.settings;
  s.use_bvh = !brute;
  const RtgSceneDev d = job_descriptor(sc, s, GpuFrame{});
  RtgSceneDev* dd = dev_alloc<RtgSceneDev>(1);
  float4* in = dev_alloc<float4>(2 * n);
  std::uint32_t* out = dev_alloc<std::uint32_t>(n);
  CK(cudaMemcpyAsync(dd, &d, sizeof(d), cudaMemcpyHostToDevice, stream_));
  CK(cudaMemcpyAsync(in, rays, n * 8 * sizeof(float), cudaMemcpyHostToDevice, stream_));
  CK(launch_ray_any(dd, in, static_cast<std::uint32_t>(n), out, brute ? 1 : 0, stream_));
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
  RenderSettings s = sc.host.settings;
  s.use_bvh = !brute;
  return job_descriptor(sc, s, GpuFrame{});
}

}  // namespace rtg
