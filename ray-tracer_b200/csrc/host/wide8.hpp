#pragma once
// The compressed eight-wide BVH (DevNode8) and the primitive slot order it needs.
//
// The eight-wide tree is collapsed from the binary device tree (DevNode), whose
// fp32 child boxes it quantises, so a scene whose binary tree was built on the
// host and one whose tree was built on the GPU — byte-identical binary layouts —
// get byte-identical eight-wide layouts from the same function.
//
// Its leaves refer to slots by an 8-bit offset from their node's prim_base, so the
// leaf children of every eight-wide node must sit in consecutive slots. The slot
// order that gives this (leaf children of each node, nodes in breadth-first order)
// replaces the binary tree's leaf order for every per-slot array of the scene; the
// binary and four-wide trees' leaf links are remapped to it. A leaf keeps its
// primitives, in their order, and its last-in-leaf mark.
#include <cstdint>
#include <vector>

#include "device/layout.h"

namespace rtg {

struct Wide8 {
  std::vector<DevNode8> nodes;
  std::int32_t root = INT32_MIN;      // 0; or ~slot of a root leaf (new order); INT32_MIN: no primitives
  std::vector<std::uint32_t> old_of;  // new slot -> old slot
  std::vector<std::uint32_t> new_of;  // old slot -> new slot
  int depth = 0;                      // eight-wide levels (the traversal stack holds one entry per level)
};

// `nodes`/`root`: the binary device tree (links and slots in its own order);
// `last[k]`: old slot k is the last of its leaf. Deterministic (serial).
Wide8 build_wide8(const DevNode* nodes, std::size_t n_nodes, std::int32_t root, const std::uint8_t* last,
                  std::size_t n_slots);

// A leaf or interior link of the binary/four-wide trees moved to the new slot order.
inline std::int32_t remap_link(std::int32_t link, const std::vector<std::uint32_t>& new_of) {
  return link >= 0 || link == INT32_MIN ? link : ~static_cast<std::int32_t>(new_of[static_cast<std::size_t>(~link)]);
}

}  // namespace rtg
