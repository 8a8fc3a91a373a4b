#pragma once
// BVH build on the GPU: the reference's binned-SAH tree (src/geometry/bvh.cpp:28-163),
// built from primitive boxes in HBM, then laid out for the traversal kernels.
//
// The tree is the one the host build makes, node for node: every split decision
// depends only on which primitives a node holds (box unions, bin counts and SAH
// costs, all in double without fused multiply-adds), and the reference's
// std::partition is reproduced exactly. That partition is Hoare's two-pointer
// scheme, so the k-th primitive from the left that belongs on the right trades
// places with the k-th primitive from the right that belongs on the left; both
// ranks come from prefix counts, which the GPU computes in parallel. The device
// layout that results (DevNode, DevNode4, slots) is byte-identical to
// flatten()'s output for the same scene.
//
// Work is split by size. Nodes with more than 32 primitives are built level by
// level: warps reduce 256-primitive chunks into per-node bounds and bins with
// atomics on order-preserving integer keys of the doubles, one warp per node runs
// the SAH sweep (16 lanes per axis), and the partition runs as count / scan / rank
// / swap passes. A node with at most 32 primitives is built whole, with all its
// descendants, by one warp in shared memory. Depth-first numbering is then
// derived from subtree sizes.
#include <cstdint>

#include <cuda_runtime.h>

#include "device/layout.h"

namespace rtg {

// Inputs, indexed by primitive id, all in device memory.
struct GpuBvhInput {
  std::uint32_t n_items = 0;            // primitives with a finite, non-empty box
  const double* boxes = nullptr;        // 6 per primitive: lo xyz, hi xyz
  const std::uint32_t* items = nullptr; // ids of those primitives, ascending
  const float4* rows = nullptr;         // 3 per primitive: slot rows (flatten.hpp slot_record)
  const float4* normals = nullptr;      // 3 per primitive
  const std::uint32_t* material = nullptr; // 1 per primitive
};

// What the build found; the caller sizes the layout arrays from it.
struct GpuBvhCounts {
  std::int32_t interior = 0;  // DevNode records
  std::int32_t wide = 0;      // DevNode4 records
  std::int32_t root = INT32_MIN, root4 = INT32_MIN;
  std::int32_t nodes = 0, leaves = 0, max_leaf = 0, max_depth = 0, depth4 = 0;
  std::int32_t levels = 0;    // level-by-level passes over large nodes
  float build_ms = 0;         // device time of the tree build (CUDA events)
};

// Loads the build kernels onto the current device now (they are otherwise loaded
// on first launch, which would stall the first build by milliseconds).
void gpu_bvh_preload();

// Owns the scratch memory of one build (from `pool`, stream-ordered).
// Moves an emitted layout to another slot order (the one the compressed
// eight-wide tree needs, wide8.hpp): slot k of the output takes old slot
// old_of[k] of the inputs (prims and normals 3 rows per slot, material 1 word),
// and the leaf links of `nodes` (n_nodes DevNode) and `nodes4` (n_wide DevNode4)
// become ~new_of[old start]. Indices are range-checked; stream-ordered.
cudaError_t apply_slot_order(const std::uint32_t* old_of, const std::uint32_t* new_of, std::uint32_t n_slots,
                             const float4* prims_in, const float4* normals_in, const std::uint32_t* material_in,
                             float4* prims, float4* normals, std::uint32_t* material, DevNode* nodes,
                             std::int32_t n_nodes, DevNode4* nodes4, std::int32_t n_wide, cudaStream_t stream);

class GpuBvhBuilder {
 public:
  GpuBvhBuilder(cudaStream_t stream, cudaMemPool_t pool) : stream_(stream), pool_(pool) {}
  ~GpuBvhBuilder();
  GpuBvhBuilder(const GpuBvhBuilder&) = delete;
  GpuBvhBuilder& operator=(const GpuBvhBuilder&) = delete;

  // Builds the tree and its four-wide collapse; synchronises the stream once per
  // level of large nodes and at the end. Throws std::runtime_error on a leaf of
  // more than 65535 primitives or a tree deeper than the traversal stack allows.
  GpuBvhCounts build(const GpuBvhInput& in);

  // Writes the device layout: counts.interior nodes, counts.wide four-wide nodes
  // and n_items slots (prims 3 per slot, slot_material, slot_normals 3 per slot,
  // order = slot -> primitive id). Stream-ordered; no synchronisation.
  void emit(const GpuBvhInput& in, DevNode* nodes, DevNode4* nodes4, float4* prims, std::uint32_t* slot_material,
            float4* slot_normals, std::uint32_t* order);

 private:
  void* alloc(std::size_t bytes);
  void release();

  cudaStream_t stream_;
  cudaMemPool_t pool_;
  void* blocks_[24] = {};
  int n_blocks_ = 0;
  struct State;
  State* st_ = nullptr;
  GpuBvhCounts counts_;
};

}  // namespace rtg
