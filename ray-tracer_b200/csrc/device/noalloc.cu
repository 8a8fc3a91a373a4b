// Closest-hit ray query for callers that must not allocate device memory.
//
// rtg_trace_closest stages its rays, its results and the scene descriptor in
// buffers it cudaMallocs and cudaFrees on every call. Some callers cannot do
// that: a render loop sharing the GPU with other streams (cudaFree synchronises
// the whole device), or a host that reserves all device memory up front in its
// own pool and forbids further allocations. This variant keeps every byte it
// needs in one file-scope device array, sized for kNoAllocMaxRays rays, that the
// CUDA module reserves on each GPU where it is loaded (with lazy module loading:
// at this file's first use on that GPU) and that stays until the process exits.
// It makes no allocation and no free during a call; it does copy from pageable
// host memory and waits for the context's stream before returning.
//
// Set-up: every call first makes its context's device current (cudaSetDevice;
// the device stays current after the call returns). The first call on a device
// then looks up the array's device address there with cudaGetSymbolAddress and
// caches it for that device; make that first call before starting any stream
// capture. Every call, on every context, shares the one array and leaves its
// contents behind: a call copies its rays in and writes every result slot it
// reads back, so nothing has to start at zero, but two calls whose work overlaps
// on the GPU (different streams or contexts on the same device) race on the
// array and corrupt each other's results.
//
// The reported distance is the fp32 traversal's own unless the scene's
// double-precision copy is already resident (uploaded by an earlier
// rtg_trace_closest call with distance refinement on); this call never uploads
// that copy itself, since that would allocate.
#include <mutex>

#include "device/noalloc.h"
#include "device/trace.cuh"

namespace rtg {

namespace {

// Scratch layout: descriptor, then per-ray input and output columns.
constexpr std::uint64_t kDescBytes = 1024;
constexpr std::uint64_t kRaysOff = kDescBytes;                                  // 2 float4 per ray
constexpr std::uint64_t kTOff = kRaysOff + kNoAllocMaxRays * 32;                // float
constexpr std::uint64_t kPrimOff = kTOff + kNoAllocMaxRays * 4;                 // int32
constexpr std::uint64_t kPlaneOff = kPrimOff + kNoAllocMaxRays * 4;             // int32
constexpr std::uint64_t kBaryOff = kPlaneOff + kNoAllocMaxRays * 4;             // 2 float
constexpr std::uint64_t kScratchBytes = kBaryOff + kNoAllocMaxRays * 8;         // 13 MiB + 1 KiB
static_assert(sizeof(RtgSceneDev) <= kDescBytes, "descriptor does not fit its scratch slot");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Device address of g_scratch on `device`. The symbol lookup answers for the
// current device, so the cache entry is only written when `device` is current.
cudaError_t scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    int current = -1;
    const cudaError_t ge = cudaGetDevice(&current);
    if (ge != cudaSuccess) return ge;
    if (current != device) return cudaErrorInvalidDevice;
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

constexpr int kBlock = 128;
constexpr int kStack = 16;

__global__ void __launch_bounds__(kBlock) k_ray_closest_scratch(unsigned char* scratch, std::uint32_t n, int brute,
                                                                int tree) {
  __shared__ uint2 stack[kStack * kBlock];
  const std::uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const RtgSceneDev& job = *reinterpret_cast<const RtgSceneDev*>(scratch);
  const float4* rays = reinterpret_cast<const float4*>(scratch + kRaysOff);
  const float4 a = rays[2 * i], b = rays[2 * i + 1];
  TraceCount tc;
  RayHit h;
  if (brute) h = closest_brute<false>(job, f3(a), f3(b), a.w, b.w, tc);
  else if (tree == 8) h = closest_hit8<kStack, kBlock, false>(job, f3(a), f3(b), a.w, b.w, stack, tc);
  else h = closest_hit<kStack, kBlock, false>(job, f3(a), f3(b), a.w, b.w, reinterpret_cast<int*>(stack), tc);
  refine_hit(job, f3(a), f3(b), h);
  const bool miss = h.word == kHitMiss;
  const bool plane = !miss && (h.word & kHitPlaneBit);
  std::int32_t id = -1;
  if (plane) id = static_cast<std::int32_t>(h.word & ~kHitPlaneBit);
  else if (!miss) id = static_cast<std::int32_t>(__float_as_uint(job.prims[3 * h.word].w) & kIdMask);
  reinterpret_cast<float*>(scratch + kTOff)[i] = miss ? 0.f : h.t;
  reinterpret_cast<std::int32_t*>(scratch + kPrimOff)[i] = id;
  reinterpret_cast<std::int32_t*>(scratch + kPlaneOff)[i] = plane ? 1 : 0;
  reinterpret_cast<float2*>(scratch + kBaryOff)[i] = make_float2(h.b1, h.b2);
}

}  // namespace

cudaError_t noalloc_trace_closest(int device, const RtgSceneDev& job, const float* rays, std::uint64_t n, int brute,
                                  int tree, float* t, std::int32_t* prim, std::int32_t* is_plane, float* bary,
                                  cudaStream_t stream) {
  if (n > kNoAllocMaxRays) return cudaErrorInvalidValue;
  if (n == 0) return cudaSuccess;
  // The scratch address, the kernel launch and the copies all belong to the
  // context's device: make it current first (it stays current after the call).
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return e;
  unsigned char* s = nullptr;
  e = scratch_address(device, &s);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(s, &job, sizeof(job), cudaMemcpyHostToDevice, stream)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(s + kRaysOff, rays, n * 32, cudaMemcpyHostToDevice, stream)) != cudaSuccess) return e;
  const unsigned blocks = static_cast<unsigned>((n + kBlock - 1) / kBlock);
  k_ray_closest_scratch<<<blocks, kBlock, 0, stream>>>(s, static_cast<std::uint32_t>(n), brute, tree);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (t && (e = cudaMemcpyAsync(t, s + kTOff, n * 4, cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
  if (prim && (e = cudaMemcpyAsync(prim, s + kPrimOff, n * 4, cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
  if (is_plane && (e = cudaMemcpyAsync(is_plane, s + kPlaneOff, n * 4, cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
    return e;
  if (bary && (e = cudaMemcpyAsync(bary, s + kBaryOff, n * 8, cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
  return cudaStreamSynchronize(stream);
}

}  // namespace rtg
