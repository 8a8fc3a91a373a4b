// Wavefront path tracer for sm_100a.
//
// One iteration of the wavefront over a pool of path slots:
//   k_plan    — one block: decides which open segments (passes of renders) the
//               free slots go to, in the host's priority order, and copies the
//               counters and segment progress to the pinned snapshot ring;
//   k_extend  — fills free slots with new camera paths (thin-lens generation,
//               src/rendering/renderer.cpp:33-37 + include/raytracer/core/camera.hpp:54-62)
//               and finds every live path's closest hit (Scene::intersect).
//   k_shade   — emission, material sampling, next-event estimation and Russian
//               roulette for each hit (src/rendering/integrator.cpp:97-139); continuing
//               paths are stream-compacted into the other state buffer and shadow
//               rays into the shadow queue with one atomic per warp (ballot + popc).
//   k_shadow  — any-hit test of each shadow ray (Scene::occluded); unoccluded ones
//               add their contribution to the sample's radiance slot.
// Every path owns one radiance slot addressed by (segment, pixel, sample-in-pass);
// all adds to it happen in path order from kernels that are stream-ordered, so
// the result does not depend on queue order, batch composition or timing. Paths
// that end count themselves done in their segment's progress record; once a
// segment is done, k_accumulate folds each pixel's samples into the double
// framebuffer in sample order (Framebuffer::add,
// include/raytracer/rendering/framebuffer.hpp:31), passes of one render in order.
//
// Path state, hits and shadow rays are written and read once per iteration and
// outgrow L2 at the pool sizes used, so they go through cache-streaming loads and
// stores (__ldcs / __stcs) and leave L1/L2 to the BVH nodes and primitives.
//
// Work distribution: persistent warps fetch 32 items at a time from a cursor in
// WaveCounters (Aila & Laine, "Understanding the Efficiency of Ray Traversal on
// GPUs", HPG 2009), so uneven traversal costs balance across SMs.
#include <cfloat>
#include <type_traits>

#include "device/shade.cuh"
#include "device/wave.h"

namespace rtg {

namespace {

constexpr float kRayTMin = 1e-6f;  // include/raytracer/math/ray.hpp:45
constexpr int kStackSmem = 8;  // stack entries per thread in shared memory (8 measured 1% faster than 16 or 24)
constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ std::uint64_t ld_u64(std::uint32_t lo, std::uint32_t hi) {
  return static_cast<std::uint64_t>(lo) | (static_cast<std::uint64_t>(hi) << 32);
}

__device__ __forceinline__ void warp_add_u64(std::uint64_t v, std::uint64_t* dst) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFull, v, off);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(reinterpret_cast<unsigned long long*>(dst), static_cast<unsigned long long>(v));
}

// Programmatic dependent launch: each wavefront kernel lets the next one be
// scheduled at once (its blocks take SM slots as this grid's blocks exit) and
// waits for the previous grid's completion and memory before touching any data.
__device__ __forceinline__ void chain_to_previous_grid() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Warp-wide fetch of the next 32 work items from `cursor`.
__device__ __forceinline__ std::uint32_t warp_fetch(std::uint32_t* cursor) {
  std::uint32_t base = 0;
  if ((threadIdx.x & 31) == 0) base = atomicAdd(cursor, 32u);
  return __shfl_sync(kFull, base, 0);
}

struct CameraSample {
  float3 o, d;
  Pcg rng;
  std::uint32_t sample;  // radiance slot
};

// Camera ray for local sample `local` of a segment, numbered pixel-major
// (local = pixel * pass_spp + (s - pass_s0)): a warp's new paths are samples of
// the same few pixels, which keeps their walks (and their later bounces) coherent;
// numbering sample-major measured 17% slower in the closest-hit stage.
// Jitter (2 draws), then the lens (2 draws). A segment holds fewer than 2^32 samples.
// The ray's rounding is pinned (explicit FMAs and unfused products), so every
// instance of the kernel generates the same bits.
__device__ __forceinline__ CameraSample camera_sample(const RtgSceneDev& J, const DevSegment& S, std::uint64_t local) {
  CameraSample cs;
  const std::uint32_t spp = S.pass_spp;
  const std::uint32_t l32 = static_cast<std::uint32_t>(local);
  const std::uint32_t pixel = l32 / spp;
  const std::uint32_t s = S.pass_s0 + (l32 - pixel * spp);
  const std::uint32_t px = static_cast<std::uint32_t>(pixel % static_cast<std::uint32_t>(J.width));
  const std::uint32_t py = static_cast<std::uint32_t>(pixel / static_cast<std::uint32_t>(J.width));
  cs.rng = Pcg::for_sample(J.seed, pixel, s);
  const float jx = cs.rng.uniform();
  const float jy = cs.rng.uniform();
  const float sx = __fadd_rn(static_cast<float>(px), jx), sy = __fadd_rn(static_cast<float>(py), jy);
  const float3 target = f3(fmaf(sy, J.cam_dv.x, fmaf(sx, J.cam_du.x, J.cam_corner.x)),
                           fmaf(sy, J.cam_dv.y, fmaf(sx, J.cam_du.y, J.cam_corner.y)),
                           fmaf(sy, J.cam_dv.z, fmaf(sx, J.cam_du.z, J.cam_corner.z)));
  cs.o = J.cam_origin;
  if (J.lens_radius > 0.f) {
    const float2 dk = unit_disk(cs.rng);
    const float lr = J.lens_radius;
    cs.o = f3(fmaf(lr, fmaf(dk.y, J.cam_v.x, __fmul_rn(dk.x, J.cam_u.x)), cs.o.x),
              fmaf(lr, fmaf(dk.y, J.cam_v.y, __fmul_rn(dk.x, J.cam_u.y)), cs.o.y),
              fmaf(lr, fmaf(dk.y, J.cam_v.z, __fmul_rn(dk.x, J.cam_u.z)), cs.o.z));
  }
  cs.d = unit_or(sub3p(target, cs.o), f3(0.f, 0.f, 0.f));
  cs.sample = static_cast<std::uint32_t>(S.sample_base + local);
  return cs;
}

// ---------------------------------------------------------------------------
// Inclusive scan over one block of kMaxGen threads (warp shuffles, then the warp
// totals); `tot` is a kMaxGen / 32 scratch array and receives the block total.
__device__ __forceinline__ std::uint32_t plan_scan(std::uint32_t v, std::uint32_t* tot, std::uint32_t& total) {
  constexpr int kWarps = kMaxGen / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const std::uint32_t y = __shfl_up_sync(kFull, v, off);
    if (lane >= off) v += y;
  }
  if (lane == 31) tot[w] = v;
  __syncthreads();
  if (w == 0) {
    std::uint32_t x = lane < kWarps ? tot[lane] : 0u;
#pragma unroll
    for (int off = 1; off < kWarps; off <<= 1) {
      const std::uint32_t y = __shfl_up_sync(kFull, x, off);
      if (lane >= off) x += y;
    }
    if (lane < kWarps) tot[lane] = x;
  }
  __syncthreads();
  total = tot[kWarps - 1];
  return v + (w > 0 ? tot[w - 1] : 0u);
}

// Generation plan: free slots go to the open segments greedily in the host's
// order. One block of kMaxGen threads, one table entry each.
__global__ void __launch_bounds__(kMaxGen) k_plan(WaveBuffers wb, int par) {
  __shared__ std::uint32_t tot_rem[kMaxGen / 32], tot_flag[kMaxGen / 32];
  chain_to_previous_grid();
  WaveCounters* C = wb.cnt;
  const int t = threadIdx.x;
  const std::uint32_t live = C->live[par];
  const std::uint32_t room = wb.capacity - live;
  const std::uint32_t ng = min(wb.gen->n, static_cast<std::uint32_t>(kMaxGen));
  // Snapshot of the state the previous iteration left, before this plan changes it.
  const std::uint64_t iter = C->iteration;
  WaveSnapshot* snap = wb.ring + (iter % wb.ring_size);
  const std::uint32_t ns = min(wb.gen->snapshot_slots, static_cast<std::uint32_t>(kMaxSegments));
  for (std::uint32_t k = t; k < ns; k += kMaxGen) snap->seg[k] = wb.seg_prog[k];
  if (t == 0) snap->c = *C;
  std::uint32_t slot = 0, rem = 0;
  std::uint64_t gen0 = 0;
  if (t < static_cast<int>(ng)) {
    slot = wb.gen->slot[t];
    if (slot < static_cast<std::uint32_t>(kMaxSegments)) {
      gen0 = wb.seg_prog[slot].generated;
      const std::uint64_t count = wb.segs[slot].count;
      const std::uint64_t r = count > gen0 ? count - gen0 : 0;
      rem = r < room ? static_cast<std::uint32_t>(r) : room;
    } else {
      atomicExch(&C->error, 3u);
      C->error_info = slot;
    }
  }
  // Inclusive scan of rem (each <= room <= 2^23, so the sum fits 32 bits).
  std::uint32_t total = 0, n_plan = 0;
  const std::uint32_t excl = plan_scan(rem, tot_rem, total) - rem;
  const std::uint32_t take = excl >= room ? 0u : min(rem, room - excl);
  const std::uint32_t flag = take > 0 ? 1u : 0u;
  const std::uint32_t fpos = plan_scan(flag, tot_flag, n_plan);
  if (flag) {
    const std::uint32_t k = fpos - 1;
    wb.plan->end[k] = excl + take;
    wb.plan->seg[k] = slot;
    wb.plan->start[k] = gen0;
    wb.seg_prog[slot].generated = gen0 + take;
  }
  if (t == 0) {
    const std::uint32_t n_new = total < room ? total : room;
    wb.plan->n = n_plan;
    wb.plan->n_new = n_new;
    C->n_extend = live + n_new;
    C->live[par ^ 1] = 0;
    C->n_shadow = 0;
    C->fetch[0] = 0;
    C->fetch[1] = 0;
    C->fetch[2] = 0;
    C->generated += n_new;
    C->iteration = iter + 1;
  }
}

// ---------------------------------------------------------------------------
// Closest hit of one ray: the eight-wide tree (kWide8) or the binary tree, or
// brute force when the job asks for it.
template <int kBlock, bool kCount, bool kWide8, class Stack>
__device__ __forceinline__ RayHit trace_closest(const RtgSceneDev& J, float3 o, float3 d, float tmin, Stack* stack,
                                                TraceCount& tc) {
  if (!J.use_bvh) return closest_brute<kCount>(J, o, d, tmin, FLT_MAX, tc);
  if constexpr (kWide8) return closest_hit8<kStackSmem, kBlock, kCount>(J, o, d, tmin, FLT_MAX, stack, tc);
  else return closest_hit<kStackSmem, kBlock, kCount>(J, o, d, tmin, FLT_MAX, stack, tc);
}

// Any hit of one shadow ray below tmax: the eight-wide or the four-wide tree.
template <int kBlock, bool kCount, bool kWide8, class Stack>
__device__ __forceinline__ bool trace_any(const RtgSceneDev& J, float3 o, float3 d, float tmin, float tmax,
                                          Stack* stack, TraceCount& tc) {
  if (!J.use_bvh) return any_brute(J, o, d, tmin, tmax);
  if constexpr (kWide8) return any_hit8<kStackSmem, kBlock, kCount>(J, o, d, tmin, tmax, stack, tc);
  else return any_hit4<kStackSmem, kBlock, kCount>(J, o, d, tmin, tmax, stack, tc);
}

// Per-thread traversal stack entries in shared memory: groups (two words) for
// the eight-wide walk, node links for the binary and four-wide walks.
template <bool kWide8>
using StackEntry = std::conditional_t<kWide8, uint2, int>;

template <int kBlock, bool kCount, bool kWide8>
__global__ void __launch_bounds__(kBlock) k_extend(WaveBuffers wb, int par) {
  __shared__ StackEntry<kWide8> stack[kStackSmem * kBlock];
  chain_to_previous_grid();
  WaveCounters* C = wb.cnt;
  const std::uint32_t live = C->live[par];
  const std::uint32_t n = C->n_extend;
  const GenPlan& P = *wb.plan;
  float4* const A = wb.st_a[par];
  float4* const B = wb.st_b[par];
  TraceCount tc;
  std::uint64_t rays = 0;
  while (true) {
    const std::uint32_t base = warp_fetch(&C->fetch[0]);
    if (base >= n) break;
    const std::uint32_t i = base + (threadIdx.x & 31);
    if (i >= n) continue;
    float3 o, d;
    std::uint32_t job;
    if (i >= live) {
      // New path j: plan entry k is the first with end[k] > j.
      const std::uint32_t j = i - live;
      int lo = 0, hi = static_cast<int>(P.n) - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (P.end[mid] > j) hi = mid;
        else lo = mid + 1;
      }
      const std::uint32_t seg = P.seg[lo];
      const std::uint64_t local = P.start[lo] + (j - (lo > 0 ? P.end[lo - 1] : 0u));
      const DevSegment S = wb.segs[seg];
      job = S.job;
      const CameraSample cs = camera_sample(wb.jobs[job], S, local);
      o = cs.o;
      d = cs.d;
      __stcs(&A[i], make_float4(o.x, o.y, o.z, __uint_as_float(cs.sample)));
      // Camera rays count as a specular bounce (no NEE double-count guard).
      __stcs(&B[i], make_float4(d.x, d.y, d.z, __uint_as_float(kFlagSpecular | (job << kMetaSceneShift))));
      __stcs(&wb.st_c[par][i], make_float4(1.f, 1.f, 1.f, __uint_as_float(seg)));
      __stcs(&wb.st_d[par][i], make_uint4(static_cast<std::uint32_t>(cs.rng.state), static_cast<std::uint32_t>(cs.rng.state >> 32),
                                   static_cast<std::uint32_t>(cs.rng.inc), static_cast<std::uint32_t>(cs.rng.inc >> 32)));
      wb.radiance[cs.sample] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
      const float4 a = __ldcs(&A[i]);
      const float4 b = __ldcs(&B[i]);
      o = f3(a);
      d = f3(b);
      job = __float_as_uint(b.w) >> kMetaSceneShift;
    }
    const RtgSceneDev& J = wb.jobs[job];
    const RayHit h = trace_closest<kBlock, kCount, kWide8>(J, o, d, kRayTMin, stack, tc);
    __stcs(&wb.hits[i], make_float4(h.t, __uint_as_float(h.word), h.b1, h.b2));
    ++rays;
  }
  warp_add_u64(rays, &C->rays);
  if (kCount) {
    warp_add_u64(tc.nodes, &C->node_visits);
    warp_add_u64(tc.prims, &C->prim_tests);
    warp_add_u64(tc.spheres, &C->sphere_tests);
  }
}

// ---------------------------------------------------------------------------
// 64 registers (8 blocks of 128 per SM) with a few spills measured 4% faster than 80.
// kMis: some open job uses multiple importance sampling. Without one, the MIS code
// is compiled out and the kernel keeps its registers for the common path.
template <int kBlock, bool kMis>
__global__ void __launch_bounds__(kBlock, 1024 / kBlock) k_shade(WaveBuffers wb, int par) {
  constexpr int kWarps = kBlock / 32;
  // Per-round queue counts and bases, double-buffered by round parity: a round
  // writes one buffer while the other may still be read, so no barrier is needed
  // at the end of a round.
  __shared__ std::uint32_t s_cnt[2][2][kWarps];
  __shared__ std::uint32_t s_base[2][2];
  int rb = 0;
  chain_to_previous_grid();
  WaveCounters* C = wb.cnt;
  const std::uint32_t n = C->n_extend;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float4* const A = wb.st_a[par];
  const float4* const B = wb.st_b[par];
  const float4* const Cc = wb.st_c[par];
  const uint4* const D = wb.st_d[par];
  std::uint64_t rr_killed = 0;
  // Uniform work per path: blocks stride over the hits in order (no fetch atomics).
  for (std::uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    const std::uint32_t i = base + threadIdx.x;
    bool cont = false, shadow = false;
    float3 o_next = f3(0.f, 0.f, 0.f), d_next = o_next, beta = o_next, sh_o = o_next, sh_d = o_next, sh_c = o_next;
    float sh_tmax = 0.f;
    std::uint32_t sample = 0, meta_next = 0, job = 0, seg = 0;
    float pdf_next = -1.f;  // set when the next hit may need a MIS weight
    Pcg rng{0, 0};
    if (i < n) {
      const float4 a = __ldcs(&A[i]), b = __ldcs(&B[i]), c = __ldcs(&Cc[i]), hv = __ldcs(&wb.hits[i]);
      const uint4 r = __ldcs(&D[i]);
      const float3 o = f3(a), d = f3(b);
      sample = __float_as_uint(a.w);
      const std::uint32_t meta = __float_as_uint(b.w);
      const std::uint32_t depth = meta & kMetaDepthMask;
      const bool specular_bounce = (meta & kFlagSpecular) != 0;
      job = meta >> kMetaSceneShift;
      seg = __float_as_uint(c.w);
      beta = f3(c);
      rng.state = ld_u64(r.x, r.y);
      rng.inc = ld_u64(r.z, r.w);
      const RtgSceneDev& J = wb.jobs[job];
      const RayHit h{hv.x, __float_as_uint(hv.y), hv.z, hv.w};
      float4* const slot = &wb.radiance[sample];
      if (J.integrator == 2) {
        // Normals view: outward shading normal mapped to [0, 1]; black on a miss.
        if (h.word != kHitMiss) {
          const Surface s = make_surface(J, o, d, h);
          const float3 nn = s.front ? s.n : -s.n;
          *slot = make_float4(0.5f * (nn.x + 1.f), 0.5f * (nn.y + 1.f), 0.5f * (nn.z + 1.f), 0.f);
        }
      } else if (h.word == kHitMiss) {
        const float3 bg = beta * background(J, d);
        const float4 acc = *slot;
        *slot = make_float4(acc.x + bg.x, acc.y + bg.y, acc.z + bg.z, 0.f);
      } else {
        const Surface s = make_surface(J, o, d, h);
        const DevMaterial m = J.materials[s.material];
        const float3 le = emitted(m, s.front);
        // A light reached by a diffuse bounce was already counted by NEE. With
        // MIS both count, each weighted by the power heuristic against the other.
        if (!is_zero3(le)) {
          float w = 1.f;
          if (!specular_bounce && J.light_sampling && !s.is_plane)
            w = kMis && J.light_sampling == 2
                    ? power_heuristic(__ldcs(&wb.st_e[par][i]),
                                      light_pdf_of_hit(J, o, d, h, s) / static_cast<float>(J.n_lights))
                    : 0.f;
          if (w > 0.f) {
            const float3 add = beta * le * w;
            const float4 acc = *slot;
            *slot = make_float4(acc.x + add.x, acc.y + add.y, acc.z + add.z, 0.f);
          }
        }
        Scatter sr;
        if (scatter(m, d, s, rng, sr)) {
          if (J.light_sampling && !sr.specular && J.n_lights > 0) {
            const std::uint32_t nl = static_cast<std::uint32_t>(J.n_lights);
            const LightSample ls = sample_light(J.lights + rng.below(nl), s, rng);
            if (ls.valid) {
              // Only a Lambertian scatter is non-specular: its weight is the albedo.
              const float3 f = lambert_cos(sr.weight, s, ls.wi);
              if (!is_zero3(f) && !is_zero3(ls.li_over_pdf)) {
                const ShadowRay sray = shadow_ray(s, ls);
                sh_o = sray.o;
                sh_d = sray.d;
                sh_tmax = sray.tmax;
                float w = 1.f;  // a point light (pdf 0) cannot be hit by BSDF sampling
                if (kMis && J.light_sampling == 2 && ls.pdf > 0.f)
                  w = power_heuristic(ls.pdf / static_cast<float>(nl), dot3(s.n, ls.wi) * kInvPiF);
                sh_c = beta * (f * ls.li_over_pdf) * (static_cast<float>(nl) * w);
                shadow = true;
              }
            }
          }
          beta = beta * sr.weight;
          bool alive = !is_zero3(beta);
          if (alive && depth + 1 >= static_cast<std::uint32_t>(J.rr_min_depth)) {
            const float q = fminf(fmaxf(max3(beta), 0.05f), 0.95f);
            if (rng.uniform() >= q) {
              alive = false;
              ++rr_killed;
            } else {
              beta = beta * (1.f / q);
            }
          }
          if (alive && depth + 1 < static_cast<std::uint32_t>(J.max_depth)) {
            cont = true;
            o_next = spawn_towards(s.p, s.gn, sr.dir);
            d_next = sr.dir;
            meta_next = (depth + 1) | (sr.specular ? kFlagSpecular : 0u) | (job << kMetaSceneShift);
            // Cosine-hemisphere pdf of this bounce, for the MIS weight at the next hit.
            if (kMis && J.light_sampling == 2 && !sr.specular) pdf_next = dot3(s.n, sr.dir) * kInvPiF;
          }
        }
      }
    }
    // Appends aggregated per block: one atomic per queue per 256 paths.
    const unsigned mc = __ballot_sync(kFull, cont), ms = __ballot_sync(kFull, shadow);
    if (lane == 0) {
      s_cnt[rb][0][warp] = __popc(mc);
      s_cnt[rb][1][warp] = __popc(ms);
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      std::uint32_t total = 0;
      for (int w = 0; w < kWarps; ++w) {
        const std::uint32_t c = s_cnt[rb][threadIdx.x][w];
        s_cnt[rb][threadIdx.x][w] = total;
        total += c;
      }
      s_base[rb][threadIdx.x] = total ? atomicAdd(threadIdx.x == 0 ? &C->live[par ^ 1] : &C->n_shadow, total) : 0u;
    }
    __syncthreads();
    const unsigned below = (1u << lane) - 1u;
    const std::uint32_t cpos = s_base[rb][0] + s_cnt[rb][0][warp] + __popc(mc & below);
    const std::uint32_t spos = s_base[rb][1] + s_cnt[rb][1][warp] + __popc(ms & below);
    // The next round writes the other buffer; the one after writes this one again
    // only after its first barrier, which every thread reaches after these reads.
    rb ^= 1;
    // A path that ends here is done once this iteration's shadow stage has run:
    // count it in its segment (one atomic per segment present in the warp).
    const bool fin = i < n && !cont;
    const unsigned same = __match_any_sync(kFull, fin ? seg : 0xFFFFFFFFu);
    if (fin && (threadIdx.x & 31) == static_cast<unsigned>(__ffs(same) - 1))
      atomicAdd(&wb.seg_prog[seg].done, static_cast<std::uint32_t>(__popc(same)));
    if (cont) {
      __stcs(&wb.st_a[par ^ 1][cpos], make_float4(o_next.x, o_next.y, o_next.z, __uint_as_float(sample)));
      __stcs(&wb.st_b[par ^ 1][cpos], make_float4(d_next.x, d_next.y, d_next.z, __uint_as_float(meta_next)));
      __stcs(&wb.st_c[par ^ 1][cpos], make_float4(beta.x, beta.y, beta.z, __uint_as_float(seg)));
      __stcs(&wb.st_d[par ^ 1][cpos], make_uint4(static_cast<std::uint32_t>(rng.state), static_cast<std::uint32_t>(rng.state >> 32),
                                          static_cast<std::uint32_t>(rng.inc), static_cast<std::uint32_t>(rng.inc >> 32)));
      if (kMis && pdf_next >= 0.f) __stcs(&wb.st_e[par ^ 1][cpos], pdf_next);
    }
    if (shadow) {
      __stcs(&wb.sh_a[spos], make_float4(sh_o.x, sh_o.y, sh_o.z, __uint_as_float(sample)));
      __stcs(&wb.sh_b[spos], make_float4(sh_d.x, sh_d.y, sh_d.z, sh_tmax));
      __stcs(&wb.sh_c[spos], make_float4(sh_c.x, sh_c.y, sh_c.z, __uint_as_float(job)));
    }
  }
  warp_add_u64(rr_killed, &C->rr_terminated);
}

// ---------------------------------------------------------------------------
template <int kBlock, bool kCount, bool kWide8>
__global__ void __launch_bounds__(kBlock) k_shadow(WaveBuffers wb) {
  __shared__ StackEntry<kWide8> stack[kStackSmem * kBlock];
  chain_to_previous_grid();
  WaveCounters* C = wb.cnt;
  const std::uint32_t n = C->n_shadow;
  TraceCount tc;
  std::uint64_t rays = 0;
  while (true) {
    const std::uint32_t base = warp_fetch(&C->fetch[2]);
    if (base >= n) break;
    const std::uint32_t i = base + (threadIdx.x & 31);
    if (i >= n) continue;
    const float4 a = __ldcs(&wb.sh_a[i]), b = __ldcs(&wb.sh_b[i]), c = __ldcs(&wb.sh_c[i]);
    const RtgSceneDev& J = wb.jobs[__float_as_uint(c.w)];
    const float3 o = f3(a), d = f3(b);
    const bool blocked = trace_any<kBlock, kCount, kWide8>(J, o, d, kRayTMin, b.w, stack, tc);
    ++rays;
    if (!blocked) {
      float4* const slot = &wb.radiance[__float_as_uint(a.w)];
      const float4 acc = *slot;
      *slot = make_float4(acc.x + c.x, acc.y + c.y, acc.z + c.z, 0.f);
    }
  }
  warp_add_u64(rays, &C->shadow_rays);
  if (kCount) {
    warp_add_u64(tc.nodes, &C->shadow_node_visits);
    warp_add_u64(tc.prims, &C->shadow_prim_tests);
    warp_add_u64(tc.spheres, &C->shadow_sphere_tests);
  }
}

// ---------------------------------------------------------------------------
// Whitted-style direct integrator (src/rendering/integrator.cpp:141-174): every
// light at diffuse hits, recursion through metal, and a deterministic Fresnel
// split at dielectrics. The recursion becomes a depth-first walk with an explicit
// stack of pending refraction branches, which keeps the reference's RNG draw order.
constexpr int kDirectStack = 48;

struct Pending {
  float3 o, d, w;
  int depth;
};

template <int kBlock, bool kWide8>
__device__ __forceinline__ float3 direct_light_all(const RtgSceneDev& J, const DevMaterial& m, const Surface& s,
                                                   Pcg& rng, StackEntry<kWide8>* stack, TraceCount& tc,
                                                   std::uint64_t& shadow_rays) {
  float3 sum = f3(0.f, 0.f, 0.f);
  for (int li = 0; li < J.n_lights; ++li) {
    const LightSample ls = sample_light(J.lights + li, s, rng);
    if (!ls.valid) continue;
    const float3 f = brdf_cos(m, s, ls.wi);
    if (is_zero3(f) || is_zero3(ls.li_over_pdf)) continue;
    const ShadowRay sr = shadow_ray(s, ls);
    ++shadow_rays;
    const bool blocked = trace_any<kBlock, false, kWide8>(J, sr.o, sr.d, kRayTMin, sr.tmax, stack, tc);
    if (!blocked) sum = sum + f * ls.li_over_pdf;
  }
  return sum;
}

template <int kBlock, bool kWide8>
__global__ void __launch_bounds__(kBlock) k_direct(const RtgSceneDev* __restrict__ job, DevSegment seg, float4* radiance,
                                                   WaveCounters* C) {
  __shared__ StackEntry<kWide8> stack[kStackSmem * kBlock];
  TraceCount tc;
  std::uint64_t rays = 0, shadow_rays = 0;
  const RtgSceneDev& J = *job;
  const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * kBlock;
  for (std::uint64_t w = static_cast<std::uint64_t>(blockIdx.x) * kBlock + threadIdx.x; w < seg.count; w += stride) {
    CameraSample cs = camera_sample(J, seg, w);
    Pending todo[kDirectStack];
    int sp = 0;
    Pending cur{cs.o, cs.d, f3(1.f, 1.f, 1.f), 0};
    float3 L = f3(0.f, 0.f, 0.f);
    bool overflow = false;
    while (true) {
      ++rays;
      const RayHit h = trace_closest<kBlock, false, kWide8>(J, cur.o, cur.d, kRayTMin, stack, tc);
      bool next = false;
      if (h.word == kHitMiss) {
        L = L + cur.w * background(J, cur.d);
      } else {
        const Surface s = make_surface(J, cur.o, cur.d, h);
        const DevMaterial m = J.materials[s.material];
        L = L + cur.w * emitted(m, s.front);
        if (cur.depth < J.max_depth) {
          const std::uint32_t kind = kind_of(m);
          if (kind == kLambertian) {
            L = L + cur.w * direct_light_all<kBlock, kWide8>(J, m, s, cs.rng, stack, tc, shadow_rays);
          } else if (kind == kMetal) {
            Scatter sr;
            if (scatter(m, cur.d, s, cs.rng, sr)) {
              cur = Pending{spawn_towards(s.p, s.gn, sr.dir), sr.dir, cur.w * f3(m.colour_a), cur.depth + 1};
              next = true;
            }
          } else if (kind == kDielectric) {
            const float ior = m.head.z;
            const float3 in = unit_or(cur.d, f3(0.f, 0.f, 0.f));
            const float eta = s.front ? 1.f / ior : ior;
            const float cos_i = fminf(-dot3(in, s.n), 1.f);
            float3 refr;
            const bool can = refract3(in, s.n, eta, refr);
            const float F = can ? schlick(cos_i, eta) : 1.f;
            const float3 tint = f3(m.colour_a);
            if (can) {
              if (sp < kDirectStack) {
                const float3 td = unit_or(refr, f3(0.f, 0.f, 0.f));
                todo[sp++] = Pending{spawn_towards(s.p, s.gn, td), td, cur.w * tint * (1.f - F), cur.depth + 1};
              } else {
                overflow = true;
              }
            }
            const float3 rd = reflect3(in, s.n);
            cur = Pending{spawn_towards(s.p, s.gn, rd), rd, cur.w * tint * F, cur.depth + 1};
            next = true;
          }
        }
      }
      if (next) continue;
      if (sp == 0) break;
      cur = todo[--sp];
    }
    if (overflow) atomicExch(&C->error, 2u);
    radiance[cs.sample] = make_float4(L.x, L.y, L.z, 0.f);
  }
  warp_add_u64(rays, &C->rays);
  warp_add_u64(shadow_rays, &C->shadow_rays);
}

// ---------------------------------------------------------------------------
__global__ void k_accumulate(const RtgSceneDev* __restrict__ job, DevSegment seg, const float4* __restrict__ radiance) {
  const RtgSceneDev& J = *job;
  const std::uint64_t pixels = static_cast<std::uint64_t>(J.width) * static_cast<std::uint64_t>(J.height);
  const std::uint64_t p = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  std::uint64_t bad = 0;
  if (p < pixels) {
    const std::uint32_t k = seg.pass_spp;
    const float4* src = radiance + seg.sample_base + p * k;
    double s0 = J.fb_sum[4 * p], s1 = J.fb_sum[4 * p + 1], s2 = J.fb_sum[4 * p + 2];
    double q0 = J.fb_sumsq[4 * p], q1 = J.fb_sumsq[4 * p + 1], q2 = J.fb_sumsq[4 * p + 2];
    for (std::uint32_t j = 0; j < k; ++j) {
      const float4 v = src[j];
      double r = v.x, g = v.y, b = v.z;
      // A non-finite or negative sample would poison the pixel: record it as black.
      if (!isfinite(r) || !isfinite(g) || !isfinite(b) || r < 0 || g < 0 || b < 0) {
        r = g = b = 0;
        ++bad;
      }
      s0 += r; s1 += g; s2 += b;
      q0 += r * r; q1 += g * g; q2 += b * b;
    }
    J.fb_sum[4 * p] = s0; J.fb_sum[4 * p + 1] = s1; J.fb_sum[4 * p + 2] = s2;
    J.fb_sumsq[4 * p] = q0; J.fb_sumsq[4 * p + 1] = q1; J.fb_sumsq[4 * p + 2] = q2;
    J.fb_count[p] += k;
  }
  warp_add_u64(bad, J.stats);
}

// Tone map (src/rendering/tonemap.cpp:15-53) in double: exposure, operator, exact
// sRGB transfer function, round half away from zero to 8 bits.
__device__ __forceinline__ double aces_curve(double x) {
  const double a = 2.51, b = 0.03, c = 2.43, d = 0.59, e = 0.14;
  const double v = (x * (a * x + b)) / (x * (c * x + d) + e);
  return v < 0 ? 0 : (v > 1 ? 1 : v);
}
__device__ __forceinline__ std::uint8_t srgb8(double v) {
  v = v < 0 ? 0 : (v > 1 ? 1 : v);
  double s = v <= 0.0031308 ? 12.92 * v : 1.055 * pow(v, 1.0 / 2.4) - 0.055;
  s = s < 0 ? 0 : (s > 1 ? 1 : s);
  return static_cast<std::uint8_t>(llround(s * 255.0));
}

__global__ void k_resolve(const double* __restrict__ fb_sum, const std::uint32_t* __restrict__ fb_count,
                          std::uint64_t pixels, int op, double exposure, std::uint8_t* rgb8, double* mean_out) {
  const std::uint64_t p = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= pixels) return;
  const std::uint32_t n = fb_count[p];
  double c[3] = {0, 0, 0};
  if (n) {
    const double inv = 1.0 / static_cast<double>(n);
    for (int k = 0; k < 3; ++k) c[k] = fb_sum[4 * p + k] * inv;
  }
  if (mean_out)
    for (int k = 0; k < 3; ++k) mean_out[3 * p + k] = c[k];
  if (!rgb8) return;
  double t[3];
  bool finite = true;
  for (int k = 0; k < 3; ++k) {
    t[k] = c[k] * exposure;
    finite = finite && isfinite(t[k]);
  }
  for (int k = 0; k < 3; ++k) {
    double v = finite ? t[k] : 0.0;
    if (op == 0) v = v < 0 ? 0 : (v > 1 ? 1 : v);
    else if (op == 1) v = v / (1 + v);
    else v = aces_curve(v);
    rgb8[3 * p + k] = srgb8(v);
  }
}

// ---------------------------------------------------------------------------
// `tree` picks the walk: 8 the eight-wide tree; otherwise the binary tree
// (closest hit) or the four-wide tree (any hit).
template <int kBlock>
__global__ void __launch_bounds__(kBlock) k_ray_closest(const RtgSceneDev* __restrict__ job, const float4* __restrict__ rays,
                                                        std::uint32_t n, float4* out, int brute, int tree) {
  __shared__ uint2 stack[kStackSmem * kBlock];
  const std::uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const float4 a = rays[2 * i], b = rays[2 * i + 1];
  TraceCount tc;
  RayHit h;
  if (brute) h = closest_brute<false>(*job, f3(a), f3(b), a.w, b.w, tc);
  else if (tree == 8) h = closest_hit8<kStackSmem, kBlock, false>(*job, f3(a), f3(b), a.w, b.w, stack, tc);
  else h = closest_hit<kStackSmem, kBlock, false>(*job, f3(a), f3(b), a.w, b.w, reinterpret_cast<int*>(stack), tc);
  refine_hit(*job, f3(a), f3(b), h);
  out[i] = make_float4(h.t, __uint_as_float(h.word), h.b1, h.b2);
}

template <int kBlock>
__global__ void __launch_bounds__(kBlock) k_ray_any(const RtgSceneDev* __restrict__ job, const float4* __restrict__ rays,
                                                    std::uint32_t n, std::uint32_t* out, int brute, int tree) {
  __shared__ uint2 stack[kStackSmem * kBlock];
  const std::uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const float4 a = rays[2 * i], b = rays[2 * i + 1];
  TraceCount tc;
  bool hit;
  if (brute) hit = any_brute(*job, f3(a), f3(b), a.w, b.w);
  else if (tree == 8) hit = any_hit8<kStackSmem, kBlock, false>(*job, f3(a), f3(b), a.w, b.w, stack, tc);
  else hit = any_hit4<kStackSmem, kBlock, false>(*job, f3(a), f3(b), a.w, b.w, reinterpret_cast<int*>(stack), tc);
  out[i] = hit ? 1u : 0u;
}

// Blocks per SM the persistent kernels are launched with (occupancy-derived, cached).
template <class K>
int persistent_blocks(K kernel, int block) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

// Persistent grid sizes per kernel variant: [counting][eight-wide].
struct BlockCounts {
  int extend[2][2] = {}, shadow[2][2] = {}, shade = 0, shade_mis = 0;
};

template <int kBlock>
const BlockCounts& block_counts() {
  static BlockCounts bc = [] {
    BlockCounts b;
    b.extend[0][0] = persistent_blocks(k_extend<kBlock, false, false>, kBlock);
    b.extend[0][1] = persistent_blocks(k_extend<kBlock, false, true>, kBlock);
    b.extend[1][0] = persistent_blocks(k_extend<kBlock, true, false>, kBlock);
    b.extend[1][1] = persistent_blocks(k_extend<kBlock, true, true>, kBlock);
    b.shade = persistent_blocks(k_shade<kBlock, false>, kBlock);
    b.shade_mis = persistent_blocks(k_shade<kBlock, true>, kBlock);
    b.shadow[0][0] = persistent_blocks(k_shadow<kBlock, false, false>, kBlock);
    b.shadow[0][1] = persistent_blocks(k_shadow<kBlock, false, true>, kBlock);
    b.shadow[1][0] = persistent_blocks(k_shadow<kBlock, true, false>, kBlock);
    b.shadow[1][1] = persistent_blocks(k_shadow<kBlock, true, true>, kBlock);
    return b;
  }();
  return bc;
}

// Launch with programmatic stream serialization (when enabled) so the kernel's
// blocks are scheduled while the previous wavefront kernel drains.
template <class... KArgs, class... Args>
cudaError_t launch_chained(void (*kernel)(KArgs...), int grid, int block, bool pdl, cudaStream_t stream,
                           Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(static_cast<unsigned>(grid));
  cfg.blockDim = dim3(static_cast<unsigned>(block));
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <int kBlock, bool kCount, bool kWide8>
cudaError_t launch_extend(int blocks, bool pdl, cudaStream_t stream, const WaveBuffers& wb, int par) {
  return launch_chained(k_extend<kBlock, kCount, kWide8>, blocks, kBlock, pdl, stream, wb, par);
}

template <int kBlock, bool kCount, bool kWide8>
cudaError_t launch_shadow(int blocks, bool pdl, cudaStream_t stream, const WaveBuffers& wb) {
  return launch_chained(k_shadow<kBlock, kCount, kWide8>, blocks, kBlock, pdl, stream, wb);
}

template <int kBlock>
cudaError_t stage_impl(Stage stage, const WaveBuffers& wb, int par, const LaunchShape& shape, bool count,
                       cudaStream_t stream) {
  const BlockCounts& bc = block_counts<kBlock>();
  const bool pdl = shape.chained;
  switch (stage) {
    case Stage::Plan:
      return launch_chained(k_plan, 1, kMaxGen, pdl, stream, wb, par);
    case Stage::Extend: {
      const bool w8 = shape.closest_tree == 8;
      const int blocks = shape.extend_blocks ? shape.extend_blocks : bc.extend[count][w8];
      if (count) return w8 ? launch_extend<kBlock, true, true>(blocks, pdl, stream, wb, par)
                           : launch_extend<kBlock, true, false>(blocks, pdl, stream, wb, par);
      return w8 ? launch_extend<kBlock, false, true>(blocks, pdl, stream, wb, par)
                : launch_extend<kBlock, false, false>(blocks, pdl, stream, wb, par);
    }
    case Stage::Shade: {
      const int blocks = shape.shade_blocks ? shape.shade_blocks : (shape.mis ? bc.shade_mis : bc.shade);
      return shape.mis ? launch_chained(k_shade<kBlock, true>, blocks, kBlock, pdl, stream, wb, par)
                       : launch_chained(k_shade<kBlock, false>, blocks, kBlock, pdl, stream, wb, par);
    }
    case Stage::Shadow: {
      const bool w8 = shape.shadow_tree == 8;
      const int blocks = shape.shadow_blocks ? shape.shadow_blocks : bc.shadow[count][w8];
      if (count) return w8 ? launch_shadow<kBlock, true, true>(blocks, pdl, stream, wb)
                           : launch_shadow<kBlock, true, false>(blocks, pdl, stream, wb);
      return w8 ? launch_shadow<kBlock, false, true>(blocks, pdl, stream, wb)
                : launch_shadow<kBlock, false, false>(blocks, pdl, stream, wb);
    }
  }
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_stage(Stage stage, const WaveBuffers& wb, int parity, const LaunchShape& shape, bool count_traversal,
                         cudaStream_t stream) {
  switch (shape.extend_block) {
    case 64: return stage_impl<64>(stage, wb, parity, shape, count_traversal, stream);
    case 256: return stage_impl<256>(stage, wb, parity, shape, count_traversal, stream);
    default: return stage_impl<128>(stage, wb, parity, shape, count_traversal, stream);
  }
}

cudaError_t launch_iteration(const WaveBuffers& wb, int parity, const LaunchShape& shape, bool count_traversal,
                             cudaStream_t stream) {
  for (Stage st : {Stage::Plan, Stage::Extend, Stage::Shade, Stage::Shadow}) {
    const cudaError_t e = launch_stage(st, wb, parity, shape, count_traversal, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_accumulate(const RtgSceneDev* job_dev, std::uint64_t pixels, const DevSegment& seg,
                              const float4* radiance, cudaStream_t stream) {
  const unsigned blocks = static_cast<unsigned>((pixels + 255) / 256);
  k_accumulate<<<blocks, 256, 0, stream>>>(job_dev, seg, radiance);
  return cudaGetLastError();
}

cudaError_t launch_direct(const RtgSceneDev* job_dev, const DevSegment& seg, float4* radiance, WaveCounters* cnt,
                          bool wide8, cudaStream_t stream) {
  static int blocks[2] = {0, 0};
  if (wide8) {
    if (!blocks[1]) blocks[1] = persistent_blocks(k_direct<128, true>, 128);
    k_direct<128, true><<<blocks[1], 128, 0, stream>>>(job_dev, seg, radiance, cnt);
  } else {
    if (!blocks[0]) blocks[0] = persistent_blocks(k_direct<128, false>, 128);
    k_direct<128, false><<<blocks[0], 128, 0, stream>>>(job_dev, seg, radiance, cnt);
  }
  return cudaGetLastError();
}

cudaError_t launch_resolve(const double* fb_sum, const std::uint32_t* fb_count, std::uint64_t pixels, int tone_map,
                           double exposure, std::uint8_t* rgb8, double* mean_out, cudaStream_t stream) {
  if (pixels == 0) return cudaSuccess;
  const unsigned blocks = static_cast<unsigned>((pixels + 255) / 256);
  k_resolve<<<blocks, 256, 0, stream>>>(fb_sum, fb_count, pixels, tone_map, exposure, rgb8, mean_out);
  return cudaGetLastError();
}

cudaError_t launch_ray_closest(const RtgSceneDev* job_dev, const float4* rays, std::uint32_t n, float4* out, int brute,
                               int tree, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  k_ray_closest<128><<<(n + 127) / 128, 128, 0, stream>>>(job_dev, rays, n, out, brute, tree);
  return cudaGetLastError();
}

cudaError_t launch_ray_any(const RtgSceneDev* job_dev, const float4* rays, std::uint32_t n, std::uint32_t* out, int brute,
                           int tree, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  k_ray_any<128><<<(n + 127) / 128, 128, 0, stream>>>(job_dev, rays, n, out, brute, tree);
  return cudaGetLastError();
}

}  // namespace rtg
