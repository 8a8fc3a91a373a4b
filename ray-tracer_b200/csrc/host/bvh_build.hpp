#pragma once
// Host BVH construction: top-down binned SAH over primitive boxes, in double.
//
// The build steps and constants are the reference's (src/geometry/bvh.cpp:13-163:
// 16 bins, traversal cost 1, leaf <= 4 or <= 16 when a split is not cheaper, depth
// cap 60, count split when all centroids coincide), so the tree has the same
// topology and leaf contents. That keeps primitive test order, and therefore
// tie-breaking between equal-distance hits, the same as the CPU renderer's. The
// device layout (flatten.hpp) is derived from this tree.
#include <cstdint>
#include <vector>

#include "host/vec.hpp"

namespace rtg {

struct BinaryNode {
  Box box;
  std::uint32_t first = 0;  // leaf: first slot in `order`; interior: right child
  std::uint32_t count = 0;  // primitives in a leaf; 0 for interior nodes
  std::uint8_t axis = 0;    // interior: split axis (front-to-back ordering)
  bool leaf() const { return count > 0; }
};

struct BvhStats {
  std::size_t nodes = 0, leaves = 0, max_depth = 0, max_leaf = 0;
  double build_ms = 0, sah_cost = 0;
};

struct BinaryBvh {
  std::vector<BinaryNode> nodes;    // depth first; left child of i is i + 1
  std::vector<std::uint32_t> order; // primitive ids in leaf order
  BvhStats stats;

  void build(const std::vector<Box>& prim_boxes, int max_leaf = 4);
  bool check(const std::vector<Box>& prim_boxes) const;  // containment + coverage
};

}  // namespace rtg
