// BVH build on the GPU (see bvh_gpu.h for the scheme).
//
// This file is compiled with --fmad=false: the SAH costs, box areas and bin
// indices must round exactly as the host's (and the reference's) double
// arithmetic does, and a fused multiply-add would round once where they round
// twice. The build follows src/geometry/bvh.cpp:28-163 of the reference: 16
// bins per axis, traversal cost 1, leaves of <= 4 primitives (<= 16 when no
// split is cheaper), depth cap 60, the middle split when every centroid
// coincides or a partition leaves one side empty, and std::partition.
#include "device/bvh_gpu.h"
#include "host/alloc_count.hpp"

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

namespace rtg {

namespace {

constexpr int kBins = 16;
constexpr int kDepthCap = 60;
constexpr int kSmallItems = 32;          // a warp builds a node this small, and its subtree, whole
constexpr int kChunk = 256;              // primitives per warp in the level passes (8 per lane)
constexpr int kBinWords = 3 * kBins * 7; // per large node: 3 axes x 16 bins x (6 box keys + count)
constexpr int kMaxLevels = 64;
constexpr int kWarpsPerBlock = 4;

#define BVH_CK(x)                                                                      \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess)                                                             \
      throw std::runtime_error(std::string("CUDA (bvh build): ") + cudaGetErrorString(e_)); \
  } while (0)

// Counters the build shares between kernels and with the host.
struct LevelCount {
  int tasks;   // large nodes of a level
  int chunks;  // their 256-primitive chunks
};
struct Counters {
  int nodes;          // node ids handed out
  int small_roots;    // nodes built whole by one warp
  int error;          // 1: a leaf of more than 65535 primitives; 2: partition counts disagree
  int leaves, max_leaf, max_depth;
  int interior;       // interior nodes (root's interior subtree size)
  int wide_total;
  LevelCount lvl[2];  // by level parity: the level being created
  int wide_cnt[kMaxLevels + 2];
  int wide_off[kMaxLevels + 2];
};

// Doubles as integers whose signed order is the doubles' order, so atomicMin /
// atomicMax on the keys take box unions exactly.
__device__ __forceinline__ long long key_of(double x) {
  const long long b = __double_as_longlong(x);
  return b >= 0 ? b : (b ^ 0x7FFFFFFFFFFFFFFFLL);
}
__device__ __forceinline__ double value_of(long long k) {
  return __longlong_as_double(k >= 0 ? k : (k ^ 0x7FFFFFFFFFFFFFFFLL));
}
constexpr long long kKeyPosInf = 0x7FF0000000000000LL;   // key_of(+inf)
constexpr long long kKeyNegInf = -0x7FF0000000000001LL;  // key_of(-inf) = 0x800FFFFFFFFFFFFF

__device__ __forceinline__ double box_area(const double lo[3], const double hi[3]) {
  if (lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]) return 0.0;
  const double ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
  return 2.0 * (ex * ey + ey * ez + ez * ex);
}

__device__ __forceinline__ int bin_of(double c, double lo, double inv_width) {
  const int b = static_cast<int>((c - lo) * inv_width);
  return min(max(b, 0), kBins - 1);
}

__device__ __forceinline__ int widest_axis(const double lo[3], const double hi[3]) {
  const double ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
  return (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
}

__device__ __forceinline__ void load_box(const double* boxes, unsigned id, double lo[3], double hi[3]) {
  const double2* b = reinterpret_cast<const double2*>(boxes + 6ull * id);
  const double2 a = __ldg(b), m = __ldg(b + 1), z = __ldg(b + 2);
  lo[0] = a.x; lo[1] = a.y; lo[2] = m.x;
  hi[0] = m.y; hi[1] = z.x; hi[2] = z.y;
}

__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  return v;
}

// One float step toward -inf / +inf by bits (std::nextafterf for finite f).
__device__ __forceinline__ float step_down(float f) {
  if (f == 0.f) return -__int_as_float(1);
  const unsigned u = __float_as_uint(f);
  return __uint_as_float(f > 0.f ? u - 1u : u + 1u);
}
__device__ __forceinline__ float step_up(float f) {
  if (f == 0.f) return __int_as_float(1);
  const unsigned u = __float_as_uint(f);
  return __uint_as_float(f > 0.f ? u + 1u : u - 1u);
}
// A node bound rounded outward to fp32 and widened, exactly as the host flattener
// does it (flatten.cpp down / up).
__device__ __forceinline__ float round_down(double v) {
  float f = __double2float_rn(v);
  if (static_cast<double>(f) > v) f = step_down(f);
  f -= fabsf(f) * 0x1p-22f;
  return step_down(f);
}
__device__ __forceinline__ float round_up(double v) {
  float f = __double2float_rn(v);
  if (static_cast<double>(f) < v) f = step_up(f);
  f += fabsf(f) * 0x1p-22f;
  return step_up(f);
}

}  // namespace

// Device pointers of one build's scratch memory.
struct GpuBvhBuilder::State {
  std::uint32_t n = 0, nn = 0, max_level_tasks = 0, max_chunks = 0;
  Counters* counters = nullptr;
  Counters* host_counters = nullptr;  // pinned copy
  std::uint32_t* items = nullptr;     // working order (becomes the leaf order)
  std::uint32_t* scratch = nullptr;   // partition partner positions
  // per node
  double* box = nullptr;              // 6 per node
  long long* key = nullptr;           // 12 per node: box lo, box hi, centroid lo, centroid hi (large nodes)
  int* left = nullptr;
  int* right = nullptr;
  std::uint32_t* first = nullptr;
  std::uint32_t* count = nullptr;
  int* depth = nullptr;
  int* axis = nullptr;
  int* size = nullptr;
  int* isize = nullptr;
  int* dfs = nullptr;
  int* idfs = nullptr;
  int* sub = nullptr;                 // small subtree root, or -1
  int* local = nullptr;               // preorder index inside the small subtree
  int* ilocal = nullptr;              // interior preorder index inside the small subtree
  int* tasks = nullptr;               // large nodes, level after level
  int* small_roots = nullptr;
  // per level of large nodes, by parity
  long long* bins[2] = {};
  int* task_chunk0[2] = {};
  int* task_nchunks[2] = {};
  int* need_part[2] = {};
  int* part_t[2] = {};
  int* part_m[2] = {};
  int* part_axis[2] = {};
  int* part_bin[2] = {};
  double* part_lo[2] = {};
  double* part_inv[2] = {};
  int* chunk_task[2] = {};
  std::uint32_t* chunk_start[2] = {};
  int* cnt_lf[2] = {};
  int* cnt_rt[2] = {};
  int* base_lf[2] = {};
  int* base_rt[2] = {};
  // four-wide collapse
  int* wide_list = nullptr;
  int* wide_kids = nullptr;           // 4 per binary node
  std::uint32_t* wflag = nullptr;     // by depth-first index
  std::uint32_t* wscan = nullptr;
  std::uint32_t* scan_sums = nullptr;
  std::uint8_t* last = nullptr;       // last slot of a leaf
  std::vector<std::pair<int, int>> levels;  // (first task, tasks) of each level
};

namespace {

__device__ __forceinline__ double pos_inf() { return __longlong_as_double(0x7FF0000000000000LL); }

// Pointers and sizes the level kernels share. `parity` is the level's parity;
// the *_next arrays belong to the level the kernels create.
struct LevelArgs {
  const double* boxes;
  std::uint32_t* items;
  std::uint32_t* scratch;
  double* box;
  long long* key;
  int* left;
  int* right;
  std::uint32_t* first;
  std::uint32_t* count;
  int* depth;
  int* axis;
  int* sub;
  const int* tasks_cur;  // this level's large nodes
  int* tasks_next;       // the next level's
  int* small_roots;
  Counters* counters;
  int n_tasks, n_chunks, parity;
  long long* bins;
  int* need_part;
  int* part_t;
  int* part_m;
  int* part_axis;
  int* part_bin;
  double* part_lo;
  double* part_inv;
  int* task_chunk0;
  int* task_nchunks;
  int* chunk_task;
  std::uint32_t* chunk_start;
  int* cnt_lf;
  int* cnt_rt;
  int* base_lf;
  int* base_rt;
  long long* bins_next;
  int* task_chunk0_next;
  int* task_nchunks_next;
  int* chunk_task_next;
  std::uint32_t* chunk_start_next;
};

// One bin of one axis as a lane holds it.
struct BinData {
  double lo[3], hi[3];
  unsigned n;
};

__device__ __forceinline__ void bin_clear(BinData& e) {
  const double inf = pos_inf();
  for (int k = 0; k < 3; ++k) {
    e.lo[k] = inf;
    e.hi[k] = -inf;
  }
  e.n = 0;
}

__device__ __forceinline__ void note_leaf(Counters* c, std::uint32_t n, int d) {
  if (n > 0xFFFFu) atomicOr(&c->error, 1);
  atomicAdd(&c->leaves, 1);
  atomicMax(&c->max_leaf, static_cast<int>(n));
  atomicMax(&c->max_depth, d);
}

// Registers node c (primitives [first, first + n) of the working order, at
// `depth`) as a large node of the next level, with its chunks, or as the root
// of a subtree that one warp builds whole. Called by all 32 lanes of a warp.
__device__ void enqueue_node(const LevelArgs& a, int c, std::uint32_t first, std::uint32_t n, int depth) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
    a.first[c] = first;
    a.count[c] = n;
    a.depth[c] = depth;
    a.sub[c] = -1;
    a.left[c] = -1;
    a.right[c] = -1;
  }
  if (n > static_cast<std::uint32_t>(kSmallItems)) {
    const int nch = static_cast<int>((n + kChunk - 1) / kChunk);
    int slot = 0, c0 = 0;
    if (lane == 0) {
      slot = atomicAdd(&a.counters->lvl[a.parity ^ 1].tasks, 1);
      c0 = atomicAdd(&a.counters->lvl[a.parity ^ 1].chunks, nch);
      a.tasks_next[slot] = c;
      a.task_chunk0_next[slot] = c0;
      a.task_nchunks_next[slot] = nch;
    }
    slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
    c0 = __shfl_sync(0xFFFFFFFFu, c0, 0);
    // Empty bounds (lo +inf, hi -inf for the box and the centroids) and bins.
    if (lane < 12) a.key[12ll * c + lane] = (lane % 6) < 3 ? kKeyPosInf : kKeyNegInf;
    long long* g = a.bins_next + static_cast<long long>(slot) * kBinWords;
    for (int i = lane; i < kBinWords; i += 32) {
      const int f = i % 7;
      g[i] = f < 3 ? kKeyPosInf : (f < 6 ? kKeyNegInf : 0);
    }
    for (int j = lane; j < nch; j += 32) {
      a.chunk_task_next[c0 + j] = slot;
      a.chunk_start_next[c0 + j] = first + static_cast<std::uint32_t>(j) * kChunk;
    }
  } else if (lane == 0) {
    a.small_roots[atomicAdd(&a.counters->small_roots, 1)] = c;
  }
}

// The root: node 0 over every primitive. Launched with one warp; `a.parity` is 1
// so that the root lands in level 0's arrays.
__global__ void k_init(LevelArgs a, std::uint32_t n, int* dfs, int* idfs) {
  if (blockIdx.x != 0) return;
  if (threadIdx.x == 0) {
    a.counters->nodes = 1;
    dfs[0] = 0;
    idfs[0] = 0;
  }
  enqueue_node(a, 0, 0, n, 0);
}

// Box and centroid bounds of each large node: one warp per 256-primitive chunk.
__global__ void __launch_bounds__(128) k_bounds(LevelArgs a) {
  const int w = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= a.n_chunks) return;
  const int t = a.tasks_cur[a.chunk_task[w]];
  const std::uint32_t start = a.chunk_start[w];
  const std::uint32_t end = min(start + static_cast<std::uint32_t>(kChunk), a.first[t] + a.count[t]);
  const double inf = pos_inf();
  double lo[3] = {inf, inf, inf}, hi[3] = {-inf, -inf, -inf};
  double clo[3] = {inf, inf, inf}, chi[3] = {-inf, -inf, -inf};
  for (int j = 0; j < kChunk / 32; ++j) {
    const std::uint32_t pos = start + static_cast<std::uint32_t>(j * 32 + lane);
    if (pos >= end) break;
    double bl[3], bh[3];
    load_box(a.boxes, a.items[pos], bl, bh);
    for (int k = 0; k < 3; ++k) {
      lo[k] = fmin(lo[k], bl[k]);
      hi[k] = fmax(hi[k], bh[k]);
      const double c = 0.5 * (bl[k] + bh[k]);
      clo[k] = fmin(clo[k], c);
      chi[k] = fmax(chi[k], c);
    }
  }
  for (int k = 0; k < 3; ++k) {
    lo[k] = warp_min(lo[k]);
    hi[k] = warp_max(hi[k]);
    clo[k] = warp_min(clo[k]);
    chi[k] = warp_max(chi[k]);
  }
  if (lane == 0) {
    long long* key = a.key + 12ll * t;
    for (int k = 0; k < 3; ++k) {
      atomicMin(&key[k], key_of(lo[k]));
      atomicMax(&key[3 + k], key_of(hi[k]));
      atomicMin(&key[6 + k], key_of(clo[k]));
      atomicMax(&key[9 + k], key_of(chi[k]));
    }
  }
}

// Bin boxes and counts of each large node (16 bins per axis over the centroid
// bounds): warp-private bins in shared memory, then merged with atomics.
__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_bins(LevelArgs a) {
  __shared__ long long s_bins[kWarpsPerBlock][kBinWords];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * kWarpsPerBlock + wib;
  if (w >= a.n_chunks) return;
  const int lt = a.chunk_task[w];
  const int t = a.tasks_cur[lt];
  if (a.depth[t] >= kDepthCap) return;  // becomes a leaf
  const long long* key = a.key + 12ll * t;
  double clo[3], inv[3];
  bool use[3];
  for (int k = 0; k < 3; ++k) {
    clo[k] = value_of(key[6 + k]);
    const double chi = value_of(key[9 + k]);
    use[k] = chi > clo[k];
    inv[k] = use[k] ? kBins / (chi - clo[k]) : 0.0;
  }
  long long* s = s_bins[wib];
  for (int i = lane; i < kBinWords; i += 32) {
    const int f = i % 7;
    s[i] = f < 3 ? kKeyPosInf : (f < 6 ? kKeyNegInf : 0);
  }
  __syncwarp();
  // Each lane takes 8 consecutive primitives (neighbours in the working order
  // are usually neighbours in space) and merges a run of primitives that fall in
  // the same bin before it touches shared memory.
  const std::uint32_t start = a.chunk_start[w];
  const std::uint32_t end = min(start + static_cast<std::uint32_t>(kChunk), a.first[t] + a.count[t]);
  constexpr int kPerLane = kChunk / 32;
  int run_bin[3] = {-1, -1, -1};
  BinData run[3];
  auto flush = [&](int k) {
    if (run_bin[k] < 0) return;
    long long* e = s + 7 * (k * kBins + run_bin[k]);
    for (int m = 0; m < 3; ++m) {
      atomicMin(&e[m], key_of(run[k].lo[m]));
      atomicMax(&e[3 + m], key_of(run[k].hi[m]));
    }
    atomicAdd(reinterpret_cast<unsigned long long*>(&e[6]), static_cast<unsigned long long>(run[k].n));
  };
  for (int j = 0; j < kPerLane; ++j) {
    const std::uint32_t pos = start + static_cast<std::uint32_t>(lane * kPerLane + j);
    if (pos >= end) break;
    double bl[3], bh[3];
    load_box(a.boxes, a.items[pos], bl, bh);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (!use[k]) continue;
      const int b = bin_of(0.5 * (bl[k] + bh[k]), clo[k], inv[k]);
      if (b != run_bin[k]) {
        flush(k);
        run_bin[k] = b;
        bin_clear(run[k]);
      }
      for (int m = 0; m < 3; ++m) {
        run[k].lo[m] = fmin(run[k].lo[m], bl[m]);
        run[k].hi[m] = fmax(run[k].hi[m], bh[m]);
      }
      ++run[k].n;
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) flush(k);
  __syncwarp();
  long long* g = a.bins + static_cast<long long>(lt) * kBinWords;
  for (int q = lane; q < 3 * kBins; q += 32) {
    const long long* e = s + 7 * q;
    if (e[6] == 0) continue;
    long long* ge = g + 7 * q;
    atomicAdd(reinterpret_cast<unsigned long long*>(&ge[6]), static_cast<unsigned long long>(e[6]));
    for (int m = 0; m < 3; ++m) {
      atomicMin(&ge[m], e[m]);
      atomicMax(&ge[3 + m], e[3 + m]);
    }
  }
}

// The reference's SAH sweep over one axis's 16 bins (src/geometry/bvh.cpp:62-88),
// with lane b of each 16-lane half holding bin b of that half's axis. The prefix
// and suffix unions are scans (min / max and integer sums give the same values
// in any order), every lane prices the plane after its bin, and the cheapest plane
// wins with the lowest bin on ties, which is the first strictly cheaper plane of
// the reference's loop. On return every lane of the half holds the axis's result
// (cost +inf when no plane separates anything) and the primitives left of it.
__device__ void half_sweep(const BinData& d, double area_floor, double& cost, int& bin, unsigned& left_n) {
  const unsigned full = 0xFFFFFFFFu;
  const int b = threadIdx.x & 15;
  double pl[3], ph[3], sl[3], sh[3];
  unsigned pn = d.n, sn = d.n;
  for (int k = 0; k < 3; ++k) {
    pl[k] = sl[k] = d.lo[k];
    ph[k] = sh[k] = d.hi[k];
  }
  for (int o = 1; o < 16; o <<= 1) {
    double ul[3], uh[3], dl[3], dh[3];
    for (int k = 0; k < 3; ++k) {
      ul[k] = __shfl_up_sync(full, pl[k], o, 16);
      uh[k] = __shfl_up_sync(full, ph[k], o, 16);
      dl[k] = __shfl_down_sync(full, sl[k], o, 16);
      dh[k] = __shfl_down_sync(full, sh[k], o, 16);
    }
    const unsigned un = __shfl_up_sync(full, pn, o, 16), dn = __shfl_down_sync(full, sn, o, 16);
    if (b >= o) {
      for (int k = 0; k < 3; ++k) {
        pl[k] = fmin(pl[k], ul[k]);
        ph[k] = fmax(ph[k], uh[k]);
      }
      pn += un;
    }
    if (b + o < 16) {
      for (int k = 0; k < 3; ++k) {
        sl[k] = fmin(sl[k], dl[k]);
        sh[k] = fmax(sh[k], dh[k]);
      }
      sn += dn;
    }
  }
  double rl[3], rh[3];
  for (int k = 0; k < 3; ++k) {
    rl[k] = __shfl_down_sync(full, sl[k], 1, 16);
    rh[k] = __shfl_down_sync(full, sh[k], 1, 16);
  }
  const unsigned rn = __shfl_down_sync(full, sn, 1, 16);
  cost = pos_inf();
  if (b < kBins - 1 && pn != 0 && rn != 0)
    cost = 1.0 + (box_area(pl, ph) * double(pn) + box_area(rl, rh) * double(rn)) / area_floor;
  bin = b;
  left_n = pn;
  for (int o = 8; o >= 1; o >>= 1) {
    const double oc = __shfl_xor_sync(full, cost, o, 16);
    const int ob = __shfl_xor_sync(full, bin, o, 16);
    const unsigned ol = __shfl_xor_sync(full, left_n, o, 16);
    if (oc < cost || (oc == cost && ob < bin)) {
      cost = oc;
      bin = ob;
      left_n = ol;
    }
  }
}

// The best split over the three axes, on every lane: r0 holds axis 0 (lanes
// 0-15) and axis 1 (lanes 16-31), r1 axis 2 (lanes 0-15). Axes in order, the
// first strictly cheaper wins; an axis whose centroids coincide is skipped.
__device__ void warp_best_split(const BinData& r0, const BinData& r1, const bool use[3], double parent_area,
                                double& best_cost, int& best_axis, int& best_bin, unsigned& best_left) {
  const unsigned full = 0xFFFFFFFFu;
  const double area_floor = parent_area < 1e-30 ? 1e-30 : parent_area;
  double c0, c1;
  int b0, b1;
  unsigned l0, l1;
  half_sweep(r0, area_floor, c0, b0, l0);
  half_sweep(r1, area_floor, c1, b1, l1);
  const double cost[3] = {__shfl_sync(full, c0, 0), __shfl_sync(full, c0, 16), __shfl_sync(full, c1, 0)};
  const int bin[3] = {__shfl_sync(full, b0, 0), __shfl_sync(full, b0, 16), __shfl_sync(full, b1, 0)};
  const unsigned left[3] = {__shfl_sync(full, l0, 0), __shfl_sync(full, l0, 16), __shfl_sync(full, l1, 0)};
  best_cost = pos_inf();
  best_axis = -1;
  best_bin = -1;
  best_left = 0;
  for (int ax = 0; ax < 3; ++ax)
    if (use[ax] && cost[ax] < best_cost) {
      best_cost = cost[ax];
      best_axis = ax;
      best_bin = bin[ax];
      best_left = left[ax];
    }
}

// One warp per large node: box from the keys, SAH decision, children.
__global__ void __launch_bounds__(128) k_decide(LevelArgs a) {
  const int i = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (i >= a.n_tasks) return;
  const int t = a.tasks_cur[i];
  const long long* key = a.key + 12ll * t;
  double lo[3], hi[3], clo[3], chi[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = value_of(key[k]);
    hi[k] = value_of(key[3 + k]);
    clo[k] = value_of(key[6 + k]);
    chi[k] = value_of(key[9 + k]);
  }
  if (lane == 0)
    for (int k = 0; k < 3; ++k) {
      a.box[6ll * t + k] = lo[k];
      a.box[6ll * t + 3 + k] = hi[k];
    }
  const std::uint32_t n = a.count[t], f0 = a.first[t];
  const int d = a.depth[t];
  bool leaf = n <= 4 || d >= kDepthCap;
  int split_axis = -1;
  std::uint32_t mid = 0;
  bool part = false;
  int best_bin = -1;
  if (!leaf) {
    bool use[3];
    for (int k = 0; k < 3; ++k) use[k] = chi[k] > clo[k];
    const long long* g = a.bins + static_cast<long long>(i) * kBinWords;
    BinData r[2];
    for (int round = 0; round < 2; ++round) {
      bin_clear(r[round]);
      if (round == 1 && lane >= 16) continue;
      const long long* e = g + 7 * ((round == 0 ? (lane >> 4) : 2) * kBins + (lane & 15));
      for (int k = 0; k < 3; ++k) {
        r[round].lo[k] = value_of(e[k]);
        r[round].hi[k] = value_of(e[3 + k]);
      }
      r[round].n = static_cast<unsigned>(e[6]);
    }
    double best_cost;
    unsigned left_n;
    warp_best_split(r[0], r[1], use, box_area(lo, hi), best_cost, split_axis, best_bin, left_n);
    if (split_axis < 0) {
      mid = n / 2;  // every centroid coincides
      split_axis = widest_axis(clo, chi);
    } else if (best_cost >= double(n) && n <= 16) {
      leaf = true;
    } else if (left_n == 0 || left_n == n) {
      mid = n / 2;  // rounding put everything on one side
    } else {
      mid = left_n;
      part = true;
    }
  }
  if (leaf) {
    if (lane == 0) {
      a.left[t] = -1;
      a.right[t] = -1;
      a.axis[t] = 0;
      a.need_part[i] = 0;
      note_leaf(a.counters, n, d);
    }
    return;
  }
  int c = 0;
  if (lane == 0) {
    a.axis[t] = split_axis;
    a.need_part[i] = part ? 1 : 0;
    if (part) {
      a.part_t[i] = static_cast<int>(mid);
      a.part_axis[i] = split_axis;
      a.part_bin[i] = best_bin;
      a.part_lo[i] = clo[split_axis];
      a.part_inv[i] = kBins / (chi[split_axis] - clo[split_axis]);
    }
    c = atomicAdd(&a.counters->nodes, 2);
    a.left[t] = c;
    a.right[t] = c + 1;
  }
  c = __shfl_sync(0xFFFFFFFFu, c, 0);
  enqueue_node(a, c, f0, mid, d + 1);
  enqueue_node(a, c + 1, f0 + mid, n - mid, d + 1);
}

__device__ __forceinline__ bool goes_left(const LevelArgs& a, int lt, std::uint32_t id) {
  const int ax = a.part_axis[lt];
  const double* b = a.boxes + 6ull * id;
  const double c = 0.5 * (__ldg(b + ax) + __ldg(b + 3 + ax));
  return bin_of(c, a.part_lo[lt], a.part_inv[lt]) <= a.part_bin[lt];
}

// Partition, pass 1: per chunk, primitives on the left that belong on the right
// ("left-false") and primitives on the right that belong on the left.
__global__ void __launch_bounds__(128) k_pcount(LevelArgs a) {
  const int w = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= a.n_chunks) return;
  const int lt = a.chunk_task[w];
  if (!a.need_part[lt]) return;
  const int t = a.tasks_cur[lt];
  const std::uint32_t f0 = a.first[t], start = a.chunk_start[w];
  const std::uint32_t end = min(start + static_cast<std::uint32_t>(kChunk), f0 + a.count[t]);
  const std::uint32_t split = f0 + static_cast<std::uint32_t>(a.part_t[lt]);
  unsigned lf = 0, rt = 0;
  for (int j = 0; j < kChunk / 32; ++j) {
    const std::uint32_t pos = start + static_cast<std::uint32_t>(j * 32 + lane);
    if (pos >= end) break;
    const bool l = goes_left(a, lt, a.items[pos]);
    if (pos < split) lf += !l;
    else rt += l;
  }
  lf = __reduce_add_sync(0xFFFFFFFFu, lf);
  rt = __reduce_add_sync(0xFFFFFFFFu, rt);
  if (lane == 0) {
    a.cnt_lf[w] = static_cast<int>(lf);
    a.cnt_rt[w] = static_cast<int>(rt);
  }
}

// Partition, pass 2: one warp per node scans its chunks' counts.
__global__ void __launch_bounds__(128) k_pscan(LevelArgs a) {
  const int i = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (i >= a.n_tasks || !a.need_part[i]) return;
  const int c0 = a.task_chunk0[i], nch = a.task_nchunks[i];
  int carry_lf = 0, carry_rt = 0;
  for (int b = 0; b < nch; b += 32) {
    const bool ok = b + lane < nch;
    const int c = c0 + b + lane;
    const int vl = ok ? a.cnt_lf[c] : 0, vr = ok ? a.cnt_rt[c] : 0;
    int il = vl, ir = vr;
    for (int o = 1; o < 32; o <<= 1) {
      const int xl = __shfl_up_sync(0xFFFFFFFFu, il, o), xr = __shfl_up_sync(0xFFFFFFFFu, ir, o);
      if (lane >= o) {
        il += xl;
        ir += xr;
      }
    }
    if (ok) {
      a.base_lf[c] = carry_lf + il - vl;
      a.base_rt[c] = carry_rt + ir - vr;
    }
    carry_lf += __shfl_sync(0xFFFFFFFFu, il, 31);
    carry_rt += __shfl_sync(0xFFFFFFFFu, ir, 31);
  }
  if (lane == 0) {
    a.part_m[i] = carry_lf;
    if (carry_lf != carry_rt) atomicOr(&a.counters->error, 2);
  }
}

// Partition, pass 3: the k-th right-side primitive that belongs on the left,
// counted from the right end, records its position at scratch[first + k].
__global__ void __launch_bounds__(128) k_pranks(LevelArgs a) {
  const int w = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= a.n_chunks) return;
  const int lt = a.chunk_task[w];
  if (!a.need_part[lt]) return;
  const int t = a.tasks_cur[lt];
  const std::uint32_t f0 = a.first[t], start = a.chunk_start[w];
  const std::uint32_t end = min(start + static_cast<std::uint32_t>(kChunk), f0 + a.count[t]);
  const std::uint32_t split = f0 + static_cast<std::uint32_t>(a.part_t[lt]);
  const int m = a.part_m[lt];
  int run = a.base_rt[w];
  for (int j = 0; j < kChunk / 32; ++j) {
    const std::uint32_t pos = start + static_cast<std::uint32_t>(j * 32 + lane);
    bool rt = false;
    if (pos < end && pos >= split) rt = goes_left(a, lt, a.items[pos]);
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, rt);
    if (rt) {
      const int r = m - 1 - (run + __popc(bal & ((1u << lane) - 1u)));
      if (r >= 0 && r < m) a.scratch[f0 + static_cast<std::uint32_t>(r)] = pos;
    }
    run += __popc(bal);
  }
}

// Partition, pass 4: the k-th left-side primitive that belongs on the right
// trades places with the position recorded at scratch[first + k] (Hoare's
// scheme, as std::partition runs it).
__global__ void __launch_bounds__(128) k_pswap(LevelArgs a) {
  const int w = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= a.n_chunks) return;
  const int lt = a.chunk_task[w];
  if (!a.need_part[lt]) return;
  const int t = a.tasks_cur[lt];
  const std::uint32_t f0 = a.first[t], start = a.chunk_start[w];
  const std::uint32_t end = min(start + static_cast<std::uint32_t>(kChunk), f0 + a.count[t]);
  const std::uint32_t split = f0 + static_cast<std::uint32_t>(a.part_t[lt]);
  const int m = a.part_m[lt];
  int run = a.base_lf[w];
  for (int j = 0; j < kChunk / 32; ++j) {
    const std::uint32_t pos = start + static_cast<std::uint32_t>(j * 32 + lane);
    bool lf = false;
    std::uint32_t mine = 0;
    if (pos < end && pos < split) {
      mine = a.items[pos];
      lf = !goes_left(a, lt, mine);
    }
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, lf);
    if (lf) {
      const int k = run + __popc(bal & ((1u << lane) - 1u));
      if (k < m) {
        const std::uint32_t q = a.scratch[f0 + static_cast<std::uint32_t>(k)];
        if (q >= split && q < f0 + a.count[t]) {  // always true; keeps the swap in the node's range
          a.items[pos] = a.items[q];
          a.items[q] = mine;
        }
      }
    }
    run += __popc(bal);
  }
}

}  // namespace

namespace {

constexpr int kSmallNodes = 2 * kSmallItems - 1;

struct SmallArgs {
  const double* boxes;
  std::uint32_t* items;
  double* box;
  int* left;
  int* right;
  std::uint32_t* first;
  std::uint32_t* count;
  int* depth;
  int* axis;
  int* size;
  int* isize;
  int* sub;
  int* local;
  int* ilocal;
  const int* small_roots;
  int n_small;
  Counters* counters;
};

// One warp's workspace: the subtree's primitives (position = lane), its nodes in
// preorder, and the stack of nodes still to build. Bins live in registers (one
// lane per axis and bin).
struct SmallWarp {
  double box[kSmallItems][6];
  double cen[kSmallItems][3];
  std::uint32_t id[kSmallItems];
  double nbox[kSmallNodes][6];
  int nl[kSmallNodes], nr[kSmallNodes], nfirst[kSmallNodes], ncount[kSmallNodes], naxis[kSmallNodes];
  int ndepth[kSmallNodes], nsize[kSmallNodes], nisize[kSmallNodes], nilocal[kSmallNodes];
  int stk_lo[kSmallItems], stk_hi[kSmallItems], stk_depth[kSmallItems], stk_parent[kSmallItems], stk_side[kSmallItems];
};

// Position of the k-th highest set bit of `mask` (k = 0: the highest).
__device__ __forceinline__ int kth_highest(unsigned mask, int k) {
  for (int j = 0; j < k; ++j) mask &= ~(1u << (31 - __clz(mask)));
  return 31 - __clz(mask);
}

// Builds the whole subtree under each node of at most kSmallItems primitives, one
// warp per node, exactly as the recursive build would: nodes are made in
// preorder (left subtree before right), each with the same bounds, SAH decision
// and partition as at the large levels.
__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_small(SmallArgs a) {
  __shared__ SmallWarp s_all[kWarpsPerBlock];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * kWarpsPerBlock + wib;
  if (w >= a.n_small) return;
  SmallWarp& s = s_all[wib];
  const int r = a.small_roots[w];
  const std::uint32_t b0 = a.first[r];
  const int n = static_cast<int>(a.count[r]);
  const double inf = pos_inf();
  if (lane < n) {
    const std::uint32_t id = a.items[b0 + lane];
    double bl[3], bh[3];
    load_box(a.boxes, id, bl, bh);
    s.id[lane] = id;
    for (int k = 0; k < 3; ++k) {
      s.box[lane][k] = bl[k];
      s.box[lane][3 + k] = bh[k];
      s.cen[lane][k] = 0.5 * (bl[k] + bh[k]);
    }
  }
  if (lane == 0) {
    s.stk_lo[0] = 0;
    s.stk_hi[0] = n;
    s.stk_depth[0] = a.depth[r];
    s.stk_parent[0] = -1;
    s.stk_side[0] = 0;
  }
  int top = 1, m = 0;
  bool overflow = false;
  __syncwarp();
  while (top > 0) {
    --top;
    const int lo = s.stk_lo[top], hi = s.stk_hi[top], d = s.stk_depth[top];
    const int parent = s.stk_parent[top], side = s.stk_side[top];
    __syncwarp();
    const int me = m++;
    if (lane == 0 && parent >= 0) {
      if (side == 0) s.nl[parent] = me;
      else s.nr[parent] = me;
    }
    const int cnt = hi - lo;
    const bool act = lane >= lo && lane < hi;
    double bl[3], bh[3], cl[3], ch[3];
    for (int k = 0; k < 3; ++k) {
      bl[k] = warp_min(act ? s.box[lane][k] : inf);
      bh[k] = warp_max(act ? s.box[lane][3 + k] : -inf);
      cl[k] = warp_min(act ? s.cen[lane][k] : inf);
      ch[k] = warp_max(act ? s.cen[lane][k] : -inf);
    }
    if (lane == 0) {
      for (int k = 0; k < 3; ++k) {
        s.nbox[me][k] = bl[k];
        s.nbox[me][3 + k] = bh[k];
      }
      s.ndepth[me] = d;
      s.nfirst[me] = lo;
      s.ncount[me] = cnt;
    }
    int kind = 0;  // 0 leaf, 1 middle split, 2 SAH partition
    int sp_axis = 0, sp_bin = -1, mid = lo;
    if (!(cnt <= 4 || d >= kDepthCap)) {
      // Lane (axis, bin) bins the node's primitives itself: round 0 covers axes
      // 0 and 1 (lanes 0-15, 16-31), round 1 axis 2 (lanes 0-15).
      bool use[3];
      double inv[3];
      for (int k = 0; k < 3; ++k) {
        use[k] = ch[k] > cl[k];
        inv[k] = use[k] ? kBins / (ch[k] - cl[k]) : 0.0;
      }
      BinData r[2];
      for (int round = 0; round < 2; ++round) {
        BinData& e = r[round];
        bin_clear(e);
        const int ax = round == 0 ? (lane >> 4) : 2, b = lane & 15;
        if ((round == 1 && lane >= 16) || !use[ax]) continue;
        for (int p = lo; p < hi; ++p) {
          if (bin_of(s.cen[p][ax], cl[ax], inv[ax]) != b) continue;
          for (int k = 0; k < 3; ++k) {
            e.lo[k] = fmin(e.lo[k], s.box[p][k]);
            e.hi[k] = fmax(e.hi[k], s.box[p][3 + k]);
          }
          ++e.n;
        }
      }
      double best_cost;
      int best_axis, best_bin;
      unsigned left_n;
      warp_best_split(r[0], r[1], use, box_area(bl, bh), best_cost, best_axis, best_bin, left_n);
      if (best_axis < 0) {
        kind = 1;
        sp_axis = widest_axis(cl, ch);
        mid = lo + cnt / 2;
      } else if (!(best_cost >= double(cnt) && cnt <= 16)) {
        sp_axis = best_axis;
        sp_bin = best_bin;
        if (left_n == 0 || left_n == static_cast<unsigned>(cnt)) {
          kind = 1;
          mid = lo + cnt / 2;
        } else {
          kind = 2;
          mid = lo + static_cast<int>(left_n);
        }
      }
      // Two more stack entries always fit (at most 29 for 32 primitives); the
      // check only keeps shared memory safe.
      if (kind != 0 && top + 2 > kSmallItems) {
        kind = 0;
        overflow = true;
      }
    }
    if (kind == 0) {
      if (lane == 0) {
        s.nl[me] = -1;
        s.nr[me] = -1;
        s.naxis[me] = 0;
      }
      continue;
    }
    if (lane == 0) s.naxis[me] = sp_axis;
    if (kind == 2) {
      const double inv = kBins / (ch[sp_axis] - cl[sp_axis]);
      const bool goes_left = act && bin_of(s.cen[lane][sp_axis], cl[sp_axis], inv) <= sp_bin;
      const unsigned lf = __ballot_sync(0xFFFFFFFFu, act && lane < mid && !goes_left);
      const unsigned rt = __ballot_sync(0xFFFFFFFFu, act && lane >= mid && goes_left);
      const int q = (lf & (1u << lane)) ? kth_highest(rt, __popc(lf & ((1u << lane) - 1u))) : -1;
      if (q >= lo && q < hi) {
        const std::uint32_t id = s.id[lane];
        s.id[lane] = s.id[q];
        s.id[q] = id;
        for (int k = 0; k < 6; ++k) {
          const double v = s.box[lane][k];
          s.box[lane][k] = s.box[q][k];
          s.box[q][k] = v;
        }
        for (int k = 0; k < 3; ++k) {
          const double v = s.cen[lane][k];
          s.cen[lane][k] = s.cen[q][k];
          s.cen[q][k] = v;
        }
      }
    }
    if (lane == 0) {
      s.stk_lo[top] = mid;
      s.stk_hi[top] = hi;
      s.stk_depth[top] = d + 1;
      s.stk_parent[top] = me;
      s.stk_side[top] = 1;
      s.stk_lo[top + 1] = lo;
      s.stk_hi[top + 1] = mid;
      s.stk_depth[top + 1] = d + 1;
      s.stk_parent[top + 1] = me;
      s.stk_side[top + 1] = 0;
    }
    top += 2;
    __syncwarp();
  }
  __syncwarp();
  int base = 0;
  if (lane == 0) {
    // Children follow their parent in preorder, so a reverse sweep sees them first.
    int leaves = 0, max_leaf = 0, max_depth = 0;
    for (int i = m - 1; i >= 0; --i) {
      if (s.nl[i] < 0) {
        s.nsize[i] = 1;
        s.nisize[i] = 0;
        ++leaves;
        max_leaf = max(max_leaf, s.ncount[i]);
        max_depth = max(max_depth, s.ndepth[i]);
      } else {
        s.nsize[i] = 1 + s.nsize[s.nl[i]] + s.nsize[s.nr[i]];
        s.nisize[i] = 1 + s.nisize[s.nl[i]] + s.nisize[s.nr[i]];
      }
    }
    int c = 0;
    for (int i = 0; i < m; ++i) s.nilocal[i] = s.nl[i] >= 0 ? c++ : -1;
    atomicAdd(&a.counters->leaves, leaves);
    atomicMax(&a.counters->max_leaf, max_leaf);
    atomicMax(&a.counters->max_depth, max_depth);
    if (overflow) atomicOr(&a.counters->error, 4);
    if (m > 1) base = atomicAdd(&a.counters->nodes, m - 1);
  }
  base = __shfl_sync(0xFFFFFFFFu, base, 0);
  __syncwarp();
  for (int i = lane; i < m; i += 32) {
    const int g = i == 0 ? r : base + i - 1;
    for (int k = 0; k < 6; ++k) a.box[6ll * g + k] = s.nbox[i][k];
    a.left[g] = s.nl[i] < 0 ? -1 : (s.nl[i] == 0 ? r : base + s.nl[i] - 1);
    a.right[g] = s.nr[i] < 0 ? -1 : (s.nr[i] == 0 ? r : base + s.nr[i] - 1);
    a.first[g] = b0 + static_cast<std::uint32_t>(s.nfirst[i]);
    a.count[g] = static_cast<std::uint32_t>(s.ncount[i]);
    a.depth[g] = s.ndepth[i];
    a.axis[g] = s.naxis[i];
    a.size[g] = s.nsize[i];
    a.isize[g] = s.nisize[i];
    a.sub[g] = r;
    a.local[g] = i;
    a.ilocal[g] = s.nilocal[i];
  }
  if (lane < n) a.items[b0 + lane] = s.id[lane];
}

}  // namespace

namespace {

struct TreeArgs {
  const double* box;
  const int* left;
  const int* right;
  const std::uint32_t* first;
  const std::uint32_t* count;
  const int* axis;
  int* size;
  int* isize;
  int* dfs;
  int* idfs;
  const int* sub;
  const int* local;
  const int* ilocal;
  Counters* counters;
};

// Subtree sizes of one level's large nodes (their children are done already).
__global__ void k_sizes(TreeArgs a, const int* tasks, int n) {
  const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n) return;
  const int t = tasks[i], l = a.left[t], r = a.right[t];
  if (l < 0) {
    a.size[t] = 1;
    a.isize[t] = 0;
  } else {
    a.size[t] = 1 + a.size[l] + a.size[r];
    a.isize[t] = 1 + a.isize[l] + a.isize[r];
  }
}

// Depth-first indices (all nodes, and interior nodes only) of one level's
// children: left follows its parent, right follows the left subtree.
__global__ void k_dfs(TreeArgs a, const int* tasks, int n) {
  const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n) return;
  const int t = tasks[i], l = a.left[t], r = a.right[t];
  if (l < 0) return;
  a.dfs[l] = a.dfs[t] + 1;
  a.dfs[r] = a.dfs[t] + 1 + a.size[l];
  a.idfs[l] = a.idfs[t] + 1;
  a.idfs[r] = a.idfs[t] + 1 + a.isize[l];
}

// Nodes inside warp-built subtrees: offsets from their subtree root.
__global__ void k_small_dfs(TreeArgs a, int capacity) {
  const int id = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  if (id >= capacity || id >= a.counters->nodes) return;
  const int root = a.sub[id];
  if (root < 0 || a.local[id] == 0) return;
  a.dfs[id] = a.dfs[root] + a.local[id];
  if (a.ilocal[id] >= 0) a.idfs[id] = a.idfs[root] + a.ilocal[id];
}

__global__ void k_finish(TreeArgs a) {
  if (blockIdx.x == 0 && threadIdx.x == 0) a.counters->interior = a.left[0] >= 0 ? a.isize[0] : 0;
}

struct WideArgs {
  const double* box;
  const int* left;
  const int* right;
  const int* dfs;
  int* wide_list;
  int* wide_kids;
  std::uint32_t* wflag;
  Counters* counters;
};

__global__ void k_wide_init(WideArgs a) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  a.counters->wide_off[0] = 0;
  if (a.left[0] >= 0) {
    a.wide_list[0] = 0;
    a.counters->wide_cnt[0] = 1;
  }
}

// One level of the four-wide collapse: each node starting a four-wide node takes
// its two children and replaces the interior child of largest surface area by
// its own children until there are four (flatten.cpp build_wide); the interior
// children then start the next level's four-wide nodes.
__global__ void k_wide(WideArgs a, int level) {
  const int cnt = a.counters->wide_cnt[level], off = a.counters->wide_off[level];
  if (blockIdx.x == 0 && threadIdx.x == 0) a.counters->wide_off[level + 1] = off + cnt;
  for (int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x); i < cnt;
       i += static_cast<int>(gridDim.x * blockDim.x)) {
    const int b = a.wide_list[off + i];
    int kid[4] = {a.left[b], a.right[b], -1, -1};
    int nk = 2;
    while (nk < 4) {
      int pick = -1;
      double pick_area = -1;
      for (int q = 0; q < nk; ++q) {
        const int c = kid[q];
        if (a.left[c] < 0) continue;
        const double* cb = a.box + 6ll * c;
        const double area = box_area(cb, cb + 3);
        if (area > pick_area) {
          pick_area = area;
          pick = q;
        }
      }
      if (pick < 0) break;
      const int c = kid[pick];
      kid[pick] = a.left[c];
      kid[nk++] = a.right[c];
    }
    for (int q = 0; q < 4; ++q) a.wide_kids[4ll * b + q] = q < nk ? kid[q] : -1;
    const int at = a.dfs[b];
    if (at >= 0 && at < a.counters->nodes) a.wflag[at] = 1;
    for (int q = 0; q < nk; ++q)
      if (a.left[kid[q]] >= 0) a.wide_list[off + cnt + atomicAdd(&a.counters->wide_cnt[level + 1], 1)] = kid[q];
  }
}

// Exclusive scan of n 32-bit flags: per-block scans, a scan of the block sums,
// then the block offsets added.
constexpr int kScanBlock = 1024;

__global__ void __launch_bounds__(kScanBlock) k_scan_block(const std::uint32_t* in, std::uint32_t* out,
                                                           std::uint32_t* sums, int n) {
  __shared__ std::uint32_t warp_sum[32];
  const int i = static_cast<int>(blockIdx.x) * kScanBlock + static_cast<int>(threadIdx.x);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const std::uint32_t v = i < n ? in[i] : 0u;
  std::uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const std::uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sum[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const std::uint32_t t = warp_sum[lane];
    std::uint32_t y = t;
    for (int o = 1; o < 32; o <<= 1) {
      const std::uint32_t z = __shfl_up_sync(0xFFFFFFFFu, y, o);
      if (lane >= o) y += z;
    }
    warp_sum[lane] = y - t;
    if (lane == 31) sums[blockIdx.x] = y;
  }
  __syncthreads();
  if (i < n) out[i] = warp_sum[wid] + x - v;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_sums(std::uint32_t* sums, int nb) {
  __shared__ std::uint32_t warp_sum[32];
  __shared__ std::uint32_t carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += kScanBlock) {
    const int i = base + static_cast<int>(threadIdx.x);
    const std::uint32_t v = i < nb ? sums[i] : 0u;
    std::uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const std::uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      const std::uint32_t t = warp_sum[lane];
      std::uint32_t y = t;
      for (int o = 1; o < 32; o <<= 1) {
        const std::uint32_t z = __shfl_up_sync(0xFFFFFFFFu, y, o);
        if (lane >= o) y += z;
      }
      warp_sum[lane] = y - t;
    }
    __syncthreads();
    const std::uint32_t c = carry;
    if (i < nb) sums[i] = c + warp_sum[wid] + x - v;
    __syncthreads();
    if (threadIdx.x == kScanBlock - 1) carry = c + warp_sum[wid] + x;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanBlock) k_scan_add(std::uint32_t* out, const std::uint32_t* sums, int n) {
  const int i = static_cast<int>(blockIdx.x) * kScanBlock + static_cast<int>(threadIdx.x);
  if (i < n) out[i] += sums[blockIdx.x];
}

struct EmitArgs {
  TreeArgs t;
  const std::uint32_t* items;
  const float4* rows;
  const float4* normals;
  const std::uint32_t* material;
  const int* wide_list;
  const int* wide_kids;
  const std::uint32_t* wscan;
  std::uint8_t* last;
  DevNode* nodes;
  DevNode4* nodes4;
  float4* prims;
  std::uint32_t* slot_material;
  float4* slot_normals;
  std::uint32_t* order;
  int capacity;
};

__device__ __forceinline__ std::int32_t binary_link(const TreeArgs& t, int c) {
  return t.left[c] >= 0 ? t.idfs[c] : ~static_cast<std::int32_t>(t.first[c]);
}

__global__ void k_mark_last(EmitArgs a) {
  const int id = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  if (id >= a.capacity || id >= a.t.counters->nodes || a.t.left[id] >= 0) return;
  a.last[a.t.first[id] + a.t.count[id] - 1] = 1;
}

// Binary nodes at their interior depth-first index: both children's boxes rounded
// outward to fp32, links, split axis.
__global__ void k_emit_nodes(EmitArgs a) {
  const int id = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  if (id >= a.capacity || id >= a.t.counters->nodes) return;
  const int l = a.t.left[id], r = a.t.right[id];
  if (l < 0) return;
  const double* L = a.t.box + 6ll * l;
  const double* R = a.t.box + 6ll * r;
  DevNode d;
  d.xy0 = make_float4(round_down(L[0]), round_up(L[3]), round_down(L[1]), round_up(L[4]));
  d.xy1 = make_float4(round_down(R[0]), round_up(R[3]), round_down(R[1]), round_up(R[4]));
  d.zz = make_float4(round_down(L[2]), round_up(L[5]), round_down(R[2]), round_up(R[5]));
  d.link = make_int4(binary_link(a.t, l), binary_link(a.t, r), a.t.axis[id] << 16, 0);
  const int at = a.t.idfs[id];
  if (at >= 0 && at < a.t.counters->interior) a.nodes[at] = d;
}

// Slots in leaf order, gathered from the per-primitive records.
__global__ void k_emit_slots(EmitArgs a, std::uint32_t n) {
  const std::uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const std::uint32_t id = a.items[k];
  float4 r0 = a.rows[3ull * id];
  if (a.last[k]) r0.w = __uint_as_float(__float_as_uint(r0.w) | kLastInLeaf);
  a.prims[3ull * k] = r0;
  a.prims[3ull * k + 1] = a.rows[3ull * id + 1];
  a.prims[3ull * k + 2] = a.rows[3ull * id + 2];
  a.slot_normals[3ull * k] = a.normals[3ull * id];
  a.slot_normals[3ull * k + 1] = a.normals[3ull * id + 1];
  a.slot_normals[3ull * k + 2] = a.normals[3ull * id + 2];
  a.slot_material[k] = a.material[id];
  a.order[k] = id;
}

// Four-wide nodes at their index: the rank of their binary node in depth-first
// order among the binary nodes that start a four-wide node.
__global__ void k_emit_wide(EmitArgs a, int n_wide) {
  const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n_wide) return;
  const int b = a.wide_list[i];
  float lo[3][4], hi[3][4];
  std::int32_t link[4];
  for (int q = 0; q < 4; ++q) {
    const int c = a.wide_kids[4ll * b + q];
    if (c < 0) {
      for (int k = 0; k < 3; ++k) lo[k][q] = hi[k][q] = 0.f;
      link[q] = kNoChild;
      continue;
    }
    const double* cb = a.t.box + 6ll * c;
    for (int k = 0; k < 3; ++k) {
      lo[k][q] = round_down(cb[k]);
      hi[k][q] = round_up(cb[3 + k]);
    }
    const int at = a.t.dfs[c];
    link[q] = a.t.left[c] >= 0 ? (at >= 0 && at < a.t.counters->nodes ? static_cast<std::int32_t>(a.wscan[at]) : kNoChild)
                               : ~static_cast<std::int32_t>(a.t.first[c]);
  }
  DevNode4 d;
  d.lo_x = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
  d.hi_x = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
  d.lo_y = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
  d.hi_y = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
  d.lo_z = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
  d.hi_z = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
  d.link = make_int4(link[0], link[1], link[2], link[3]);
  d.pad = make_int4(0, 0, 0, 0);
  const int at = a.t.dfs[b];
  if (at < 0 || at >= a.t.counters->nodes) return;
  const std::uint32_t slot = a.wscan[at];
  if (slot < static_cast<std::uint32_t>(n_wide)) a.nodes4[slot] = d;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side

namespace {

int blocks_for(long long threads, int per_block) {
  return static_cast<int>(std::max<long long>(1, (threads + per_block - 1) / per_block));
}

}  // namespace

void gpu_bvh_preload() {
  cudaFuncAttributes a;
  const void* kernels[] = {
      reinterpret_cast<const void*>(k_init),       reinterpret_cast<const void*>(k_bounds),
      reinterpret_cast<const void*>(k_bins),       reinterpret_cast<const void*>(k_decide),
      reinterpret_cast<const void*>(k_pcount),     reinterpret_cast<const void*>(k_pscan),
      reinterpret_cast<const void*>(k_pranks),     reinterpret_cast<const void*>(k_pswap),
      reinterpret_cast<const void*>(k_small),      reinterpret_cast<const void*>(k_sizes),
      reinterpret_cast<const void*>(k_dfs),        reinterpret_cast<const void*>(k_small_dfs),
      reinterpret_cast<const void*>(k_finish),     reinterpret_cast<const void*>(k_wide_init),
      reinterpret_cast<const void*>(k_wide),       reinterpret_cast<const void*>(k_scan_block),
      reinterpret_cast<const void*>(k_scan_sums),  reinterpret_cast<const void*>(k_scan_add),
      reinterpret_cast<const void*>(k_mark_last),  reinterpret_cast<const void*>(k_emit_nodes),
      reinterpret_cast<const void*>(k_emit_slots), reinterpret_cast<const void*>(k_emit_wide)};
  for (const void* k : kernels) BVH_CK(cudaFuncGetAttributes(&a, k));
}

GpuBvhBuilder::~GpuBvhBuilder() { release(); }

void GpuBvhBuilder::release() {
  for (int i = 0; i < n_blocks_; ++i) cudaFreeAsync(blocks_[i], stream_);
  n_blocks_ = 0;
  delete st_;
  st_ = nullptr;
}

void* GpuBvhBuilder::alloc(std::size_t bytes) {
  if (n_blocks_ >= static_cast<int>(sizeof(blocks_) / sizeof(blocks_[0])))
    throw std::logic_error("bvh build: too many scratch blocks");
  void* p = nullptr;
  count_allocation();
  BVH_CK(cudaMallocFromPoolAsync(&p, std::max<std::size_t>(bytes, 256), pool_, stream_));
  blocks_[n_blocks_++] = p;
  return p;
}

GpuBvhCounts GpuBvhBuilder::build(const GpuBvhInput& in) {
  release();
  counts_ = GpuBvhCounts{};
  const std::uint32_t n = in.n_items;
  if (n == 0) return counts_;
  if (n > (1u << 30)) throw std::runtime_error("too many primitives for the device BVH build");
  st_ = new State;
  State& s = *st_;
  s.n = n;
  s.nn = 2 * n;
  s.max_level_tasks = n / (kSmallItems + 1) + 2;
  s.max_chunks = n / kChunk + s.max_level_tasks + 8;

  // Carve every scratch array out of one pool allocation.
  std::vector<std::pair<void**, std::size_t>> parts;
  auto add = [&](auto*& p, std::size_t count) {
    parts.push_back({reinterpret_cast<void**>(&p), count * sizeof(*p)});
  };
  const std::size_t nn = s.nn, lt = s.max_level_tasks, mc = s.max_chunks;
  add(s.counters, 1);
  add(s.items, n);
  add(s.scratch, n);
  add(s.box, 6 * nn);
  add(s.key, 12 * nn);
  for (int** p : {&s.left, &s.right, &s.depth, &s.axis, &s.size, &s.isize, &s.dfs, &s.idfs, &s.sub, &s.local,
                  &s.ilocal, &s.tasks})
    add(*p, nn);
  add(s.first, nn);
  add(s.count, nn);
  add(s.small_roots, n);
  for (int q = 0; q < 2; ++q) {
    add(s.bins[q], lt * kBinWords);
    for (int** p : {&s.task_chunk0[q], &s.task_nchunks[q], &s.need_part[q], &s.part_t[q], &s.part_m[q],
                    &s.part_axis[q], &s.part_bin[q]})
      add(*p, lt);
    add(s.part_lo[q], lt);
    add(s.part_inv[q], lt);
    for (int** p : {&s.chunk_task[q], &s.cnt_lf[q], &s.cnt_rt[q], &s.base_lf[q], &s.base_rt[q]}) add(*p, mc);
    add(s.chunk_start[q], mc);
  }
  add(s.wide_list, n + 1);
  add(s.wide_kids, 4 * nn);
  add(s.wflag, nn);
  add(s.wscan, nn);
  add(s.scan_sums, nn / kScanBlock + 2);
  add(s.last, n);
  std::size_t total = 0;
  for (auto& p : parts) total += (p.second + 255) & ~std::size_t(255);
  auto* base = static_cast<unsigned char*>(alloc(total));
  std::size_t at = 0;
  for (auto& p : parts) {
    *p.first = base + at;
    at += (p.second + 255) & ~std::size_t(255);
  }

  cudaEvent_t ev[2];
  BVH_CK(cudaEventCreate(&ev[0]));
  BVH_CK(cudaEventCreate(&ev[1]));
  struct EventGuard {
    cudaEvent_t* e;
    ~EventGuard() {
      cudaEventDestroy(e[0]);
      cudaEventDestroy(e[1]);
    }
  } guard{ev};
  BVH_CK(cudaEventRecord(ev[0], stream_));
  BVH_CK(cudaMemsetAsync(s.counters, 0, sizeof(Counters), stream_));
  BVH_CK(cudaMemcpyAsync(s.items, in.items, n * sizeof(std::uint32_t), cudaMemcpyDeviceToDevice, stream_));

  Counters host{};
  auto read_counters = [&] {
    BVH_CK(cudaMemcpyAsync(&host, s.counters, sizeof(Counters), cudaMemcpyDeviceToHost, stream_));
    BVH_CK(cudaStreamSynchronize(stream_));
    if (host.error & 1) throw std::runtime_error("BVH leaf too large");
    if (host.error) throw std::runtime_error("device BVH build: inconsistent partition");
  };
  auto level_args = [&](int parity, int lb, int nt, int nc) {
    LevelArgs a{};
    a.boxes = in.boxes;
    a.items = s.items;
    a.scratch = s.scratch;
    a.box = s.box;
    a.key = s.key;
    a.left = s.left;
    a.right = s.right;
    a.first = s.first;
    a.count = s.count;
    a.depth = s.depth;
    a.axis = s.axis;
    a.sub = s.sub;
    a.tasks_cur = s.tasks + lb;
    a.tasks_next = s.tasks + lb + nt;
    a.small_roots = s.small_roots;
    a.counters = s.counters;
    a.n_tasks = nt;
    a.n_chunks = nc;
    a.parity = parity;
    const int p = parity, q = parity ^ 1;
    a.bins = s.bins[p];
    a.need_part = s.need_part[p];
    a.part_t = s.part_t[p];
    a.part_m = s.part_m[p];
    a.part_axis = s.part_axis[p];
    a.part_bin = s.part_bin[p];
    a.part_lo = s.part_lo[p];
    a.part_inv = s.part_inv[p];
    a.task_chunk0 = s.task_chunk0[p];
    a.task_nchunks = s.task_nchunks[p];
    a.chunk_task = s.chunk_task[p];
    a.chunk_start = s.chunk_start[p];
    a.cnt_lf = s.cnt_lf[p];
    a.cnt_rt = s.cnt_rt[p];
    a.base_lf = s.base_lf[p];
    a.base_rt = s.base_rt[p];
    a.bins_next = s.bins[q];
    a.task_chunk0_next = s.task_chunk0[q];
    a.task_nchunks_next = s.task_nchunks[q];
    a.chunk_task_next = s.chunk_task[q];
    a.chunk_start_next = s.chunk_start[q];
    return a;
  };

  // The root lands in level 0 (parity 0) as a large node, or as a warp subtree.
  k_init<<<1, 32, 0, stream_>>>(level_args(1, 0, 0, 0), n, s.dfs, s.idfs);
  BVH_CK(cudaGetLastError());
  read_counters();
  int lb = 0, nt = host.lvl[0].tasks, nc = host.lvl[0].chunks;
  for (int level = 0; nt > 0; ++level) {
    if (level >= kMaxLevels) throw std::logic_error("device BVH build: too many levels");
    const int p = level & 1;
    const LevelArgs a = level_args(p, lb, nt, nc);
    k_bounds<<<blocks_for(32ll * nc, 128), 128, 0, stream_>>>(a);
    k_bins<<<blocks_for(nc, kWarpsPerBlock), kWarpsPerBlock * 32, 0, stream_>>>(a);
    BVH_CK(cudaMemsetAsync(&s.counters->lvl[p ^ 1], 0, sizeof(LevelCount), stream_));
    k_decide<<<blocks_for(32ll * nt, 128), 128, 0, stream_>>>(a);
    k_pcount<<<blocks_for(32ll * nc, 128), 128, 0, stream_>>>(a);
    k_pscan<<<blocks_for(32ll * nt, 128), 128, 0, stream_>>>(a);
    k_pranks<<<blocks_for(32ll * nc, 128), 128, 0, stream_>>>(a);
    k_pswap<<<blocks_for(32ll * nc, 128), 128, 0, stream_>>>(a);
    BVH_CK(cudaGetLastError());
    s.levels.push_back({lb, nt});
    read_counters();
    lb += nt;
    nt = host.lvl[p ^ 1].tasks;
    nc = host.lvl[p ^ 1].chunks;
    if (nt > static_cast<int>(s.max_level_tasks) || nc > static_cast<int>(s.max_chunks))
      throw std::logic_error("device BVH build: level overflow");
  }

  SmallArgs sa{};
  sa.boxes = in.boxes;
  sa.items = s.items;
  sa.box = s.box;
  sa.left = s.left;
  sa.right = s.right;
  sa.first = s.first;
  sa.count = s.count;
  sa.depth = s.depth;
  sa.axis = s.axis;
  sa.size = s.size;
  sa.isize = s.isize;
  sa.sub = s.sub;
  sa.local = s.local;
  sa.ilocal = s.ilocal;
  sa.small_roots = s.small_roots;
  sa.n_small = host.small_roots;
  sa.counters = s.counters;
  if (sa.n_small > 0) k_small<<<blocks_for(sa.n_small, kWarpsPerBlock), kWarpsPerBlock * 32, 0, stream_>>>(sa);

  TreeArgs ta{};
  ta.box = s.box;
  ta.left = s.left;
  ta.right = s.right;
  ta.first = s.first;
  ta.count = s.count;
  ta.axis = s.axis;
  ta.size = s.size;
  ta.isize = s.isize;
  ta.dfs = s.dfs;
  ta.idfs = s.idfs;
  ta.sub = s.sub;
  ta.local = s.local;
  ta.ilocal = s.ilocal;
  ta.counters = s.counters;
  for (auto it = s.levels.rbegin(); it != s.levels.rend(); ++it)
    k_sizes<<<blocks_for(it->second, 128), 128, 0, stream_>>>(ta, s.tasks + it->first, it->second);
  for (const auto& lv : s.levels) k_dfs<<<blocks_for(lv.second, 128), 128, 0, stream_>>>(ta, s.tasks + lv.first, lv.second);
  k_small_dfs<<<blocks_for(s.nn, 256), 256, 0, stream_>>>(ta, static_cast<int>(s.nn));
  k_finish<<<1, 32, 0, stream_>>>(ta);
  BVH_CK(cudaGetLastError());
  read_counters();
  if (host.nodes > static_cast<int>(s.nn)) throw std::logic_error("device BVH build: node overflow");

  // Four-wide collapse, one launch per level (at most one per binary level).
  BVH_CK(cudaMemsetAsync(s.wflag, 0, std::size_t(host.nodes) * sizeof(std::uint32_t), stream_));
  WideArgs wa{s.box, s.left, s.right, s.dfs, s.wide_list, s.wide_kids, s.wflag, s.counters};
  k_wide_init<<<1, 32, 0, stream_>>>(wa);
  const int wide_levels = std::min(host.max_depth + 1, kMaxLevels);
  const int wide_grid = std::min(blocks_for(host.interior, 256), 148 * 8);
  for (int w = 0; w < wide_levels; ++w) k_wide<<<wide_grid, 256, 0, stream_>>>(wa, w);
  const int nb = blocks_for(host.nodes, kScanBlock);
  k_scan_block<<<nb, kScanBlock, 0, stream_>>>(s.wflag, s.wscan, s.scan_sums, host.nodes);
  k_scan_sums<<<1, kScanBlock, 0, stream_>>>(s.scan_sums, nb);
  k_scan_add<<<nb, kScanBlock, 0, stream_>>>(s.wscan, s.scan_sums, host.nodes);
  BVH_CK(cudaGetLastError());
  BVH_CK(cudaEventRecord(ev[1], stream_));
  read_counters();
  BVH_CK(cudaEventElapsedTime(&counts_.build_ms, ev[0], ev[1]));

  counts_.nodes = host.nodes;
  counts_.interior = host.interior;
  counts_.leaves = host.leaves;
  counts_.max_leaf = host.max_leaf;
  counts_.max_depth = host.max_depth;
  counts_.levels = static_cast<std::int32_t>(s.levels.size());
  int wide = 0, depth4 = 0;
  for (int w = 0; w < kMaxLevels; ++w) {
    wide += host.wide_cnt[w];
    if (host.wide_cnt[w] > 0) depth4 = w + 1;
  }
  if (host.wide_cnt[wide_levels] != 0) throw std::logic_error("device BVH build: four-wide levels left over");
  counts_.wide = wide;
  counts_.depth4 = depth4;
  counts_.root = host.interior > 0 ? 0 : ~0;
  counts_.root4 = host.interior > 0 ? 0 : ~0;
  if (3 * depth4 + 1 > kWideStackDepth) throw std::runtime_error("BVH deeper than the traversal stack allows");
  return counts_;
}

void GpuBvhBuilder::emit(const GpuBvhInput& in, DevNode* nodes, DevNode4* nodes4, float4* prims,
                         std::uint32_t* slot_material, float4* slot_normals, std::uint32_t* order) {
  if (in.n_items == 0 || !st_) return;
  State& s = *st_;
  EmitArgs e{};
  e.t.box = s.box;
  e.t.left = s.left;
  e.t.right = s.right;
  e.t.first = s.first;
  e.t.count = s.count;
  e.t.axis = s.axis;
  e.t.size = s.size;
  e.t.isize = s.isize;
  e.t.dfs = s.dfs;
  e.t.idfs = s.idfs;
  e.t.sub = s.sub;
  e.t.local = s.local;
  e.t.ilocal = s.ilocal;
  e.t.counters = s.counters;
  e.items = s.items;
  e.rows = in.rows;
  e.normals = in.normals;
  e.material = in.material;
  e.wide_list = s.wide_list;
  e.wide_kids = s.wide_kids;
  e.wscan = s.wscan;
  e.last = s.last;
  e.nodes = nodes;
  e.nodes4 = nodes4;
  e.prims = prims;
  e.slot_material = slot_material;
  e.slot_normals = slot_normals;
  e.order = order;
  e.capacity = static_cast<int>(s.nn);
  BVH_CK(cudaMemsetAsync(s.last, 0, s.n, stream_));
  k_mark_last<<<blocks_for(counts_.nodes, 256), 256, 0, stream_>>>(e);
  if (counts_.interior > 0) k_emit_nodes<<<blocks_for(counts_.nodes, 256), 256, 0, stream_>>>(e);
  k_emit_slots<<<blocks_for(s.n, 256), 256, 0, stream_>>>(e, s.n);
  if (counts_.wide > 0) k_emit_wide<<<blocks_for(counts_.wide, 256), 256, 0, stream_>>>(e, counts_.wide);
  BVH_CK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Slot order of the eight-wide tree

namespace {

__device__ __forceinline__ std::int32_t remap_leaf(std::int32_t link, const std::uint32_t* new_of, std::uint32_t n) {
  if (link >= 0 || link == INT32_MIN) return link;
  const std::uint32_t old = static_cast<std::uint32_t>(~link);
  return old < n ? ~static_cast<std::int32_t>(new_of[old]) : link;
}

__global__ void k_gather_slots(const std::uint32_t* old_of, std::uint32_t n, const float4* prims_in,
                               const float4* normals_in, const std::uint32_t* material_in, float4* prims,
                               float4* normals, std::uint32_t* material) {
  const std::uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const std::uint32_t o = old_of[k];
  if (o >= n) return;
  for (int r = 0; r < 3; ++r) {
    prims[3 * k + r] = prims_in[3 * o + r];
    normals[3 * k + r] = normals_in[3 * o + r];
  }
  material[k] = material_in[o];
}

__global__ void k_remap_links(const std::uint32_t* new_of, std::uint32_t n, DevNode* nodes, std::int32_t n_nodes,
                              DevNode4* nodes4, std::int32_t n_wide) {
  const std::int32_t i = static_cast<std::int32_t>(blockIdx.x * blockDim.x + threadIdx.x);
  if (i < n_nodes) {
    int4 l = nodes[i].link;
    l.x = remap_leaf(l.x, new_of, n);
    l.y = remap_leaf(l.y, new_of, n);
    nodes[i].link = l;
  }
  if (i < n_wide) {
    int4 l = nodes4[i].link;
    l.x = remap_leaf(l.x, new_of, n);
    l.y = remap_leaf(l.y, new_of, n);
    l.z = remap_leaf(l.z, new_of, n);
    l.w = remap_leaf(l.w, new_of, n);
    nodes4[i].link = l;
  }
}

}  // namespace

cudaError_t apply_slot_order(const std::uint32_t* old_of, const std::uint32_t* new_of, std::uint32_t n_slots,
                             const float4* prims_in, const float4* normals_in, const std::uint32_t* material_in,
                             float4* prims, float4* normals, std::uint32_t* material, DevNode* nodes,
                             std::int32_t n_nodes, DevNode4* nodes4, std::int32_t n_wide, cudaStream_t stream) {
  if (n_slots) {
    k_gather_slots<<<(n_slots + 255) / 256, 256, 0, stream>>>(old_of, n_slots, prims_in, normals_in, material_in,
                                                              prims, normals, material);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const std::int32_t n = n_nodes > n_wide ? n_nodes : n_wide;
  if (n > 0) k_remap_links<<<(n + 255) / 256, 256, 0, stream>>>(new_of, n_slots, nodes, n_nodes, nodes4, n_wide);
  return cudaGetLastError();
}

}  // namespace rtg
