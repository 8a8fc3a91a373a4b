#pragma once
// CompiledScene (double, reference order) -> device layout (fp32 records).
//
// The node array keeps the host tree's topology: every interior node becomes one
// DevNode holding both children's boxes, rounded outward to fp32 so the boxes
// still enclose what they enclosed in double. A leaf's primitives occupy
// consecutive slots (one streaming read per leaf); the last slot of each leaf
// carries kLastInLeaf, so leaves need no count. Leaves are placed in the order the
// compressed eight-wide tree needs (wide8.hpp): the leaf children of each of its
// nodes side by side.
#include <cstdint>
#include <memory>
#include <new>
#include <utility>
#include <vector>

#include "device/layout.h"
#include "host/compiled_scene.hpp"
#include "host/wide8.hpp"

namespace rtg {

constexpr std::int32_t kNoRoot = INT32_MIN;

// Allocator whose resize leaves new elements uninitialised: the large record
// arrays below are written in full by flatten's parallel loops, so filling them
// with zeros first only adds a serial pass over fresh pages.
template <class T>
struct Uninit : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = Uninit<U>;
  };
  Uninit() = default;
  template <class U>
  Uninit(const Uninit<U>&) noexcept {}
  template <class U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
template <class T>
using RecordVector = std::vector<T, Uninit<T>>;

struct FlatScene {
  RecordVector<DevNode> nodes;
  RecordVector<float4> prims;               // 3 per slot
  std::vector<std::uint32_t> slot_material; // material | smooth << 31 (scene-local material index)
  RecordVector<float4> slot_normals;        // 3 per slot
  std::vector<std::uint32_t> slot_prim;     // slot -> primitive id
  std::vector<DevPlane> planes;             // material scene-local
  std::vector<DevMaterial> materials;
  std::vector<DevLight> lights;
  std::int32_t root = kNoRoot;              // >= 0 node; < 0: ~slot of a root leaf; kNoRoot: none
  // The same tree collapsed to four children per node (any-hit queries).
  std::vector<DevNode4> nodes4;
  std::int32_t root4 = kNoRoot;
  int depth4 = 0;
  // The same tree as compressed eight-child nodes (closest-hit queries); the
  // slot arrays above are in the order it needs.
  std::vector<DevNode8> nodes8;
  std::int32_t root8 = kNoRoot;
};

// wide8: also build the compressed eight-wide tree and move the slots to its
// order (add_wide8); without it nodes8 stays empty and root8 kNoRoot.
// max_threads bounds the threads this call uses (0: up to 16, or the core
// count); callers flattening many scenes at once give each a small share.
FlatScene flatten(const CompiledScene& s, bool wide8, unsigned max_threads = 0);

// Builds the eight-wide tree from f.nodes / f.root and moves every per-slot array
// of f (and the binary and four-wide trees' leaf links) to its slot order.
void add_wide8(FlatScene& f);

// One primitive's device records, indexed by primitive rather than slot: its three
// slot rows (id bits set, no last-in-leaf bit), its three vertex normals (zero
// unless smooth) and its material word. flatten() writes these in leaf order; the
// device BVH build uploads them in primitive order and gathers them there.
void slot_record(const Prim& p, std::uint32_t id, float4* rows, float4* normals, std::uint32_t& material);

// The planes, materials and light list of a scene (f.planes, f.materials, f.lights).
void flatten_tables(const CompiledScene& s, FlatScene& f);

// Camera (set up for r's resolution), settings and background of a descriptor;
// pointers and pass fields are filled in by the engine.
void describe(const CompiledScene& s, const RenderSettings& r, RtgSceneDev& d);

}  // namespace rtg
