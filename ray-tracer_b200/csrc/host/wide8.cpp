#include "host/wide8.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace rtg {

namespace {

// One child of an eight-wide node under construction: a binary link and its
// fp32 box as stored in the binary parent. `wrap` marks a leaf that is placed in
// a node of its own (its start would be too far from its node's prim_base).
struct Child {
  std::int32_t link;
  float lo[3], hi[3];
  bool wrap = false;
};

void binary_children(const DevNode& n, Child out[2]) {
  out[0] = Child{n.link.x, {n.xy0.x, n.xy0.z, n.zz.x}, {n.xy0.y, n.xy0.w, n.zz.y}};
  out[1] = Child{n.link.y, {n.xy1.x, n.xy1.z, n.zz.z}, {n.xy1.y, n.xy1.w, n.zz.w}};
}

double surface_area(const Child& c) {
  const double x = double(c.hi[0]) - c.lo[0], y = double(c.hi[1]) - c.lo[1], z = double(c.hi[2]) - c.lo[2];
  return 2.0 * (x * y + y * z + z * x);
}

// Children of an eight-wide node that starts at binary interior node `b`: the two
// binary children, then the interior child with the largest surface area is
// replaced by its own two children until there are eight or only leaves.
int collapse(const DevNode* nodes, std::int32_t b, Child kids[8]) {
  binary_children(nodes[b], kids);
  int n = 2;
  while (n < 8) {
    int pick = -1;
    double best = -1.0;
    for (int q = 0; q < n; ++q) {
      if (kids[q].link < 0) continue;
      const double a = surface_area(kids[q]);
      if (a > best) {
        best = a;
        pick = q;
      }
    }
    if (pick < 0) break;
    Child two[2];
    binary_children(nodes[kids[pick].link], two);
    kids[pick] = two[0];
    kids[n++] = two[1];
  }
  return n;
}

// Biased float exponent e of the per-axis scale 2^(e - 127): the smallest with
// extent / scale <= 255 (normal range only).
int axis_exponent(double extent) {
  if (!(extent > 0)) return 1;
  int e = static_cast<int>(std::ceil(std::log2(extent / 255.0))) + 127;
  e = std::clamp(e, 1, 254);
  while (e > 1 && extent / std::ldexp(1.0, e - 1 - 127) <= 255.0) --e;
  while (e < 254 && extent / std::ldexp(1.0, e - 127) > 255.0) ++e;
  return e;
}

// Greedy assignment of children to slots by direction from the node's centre:
// slot s favours the corner (+/-1, +/-1, +/-1) with bit k set = positive along
// axis k. The cheapest (child, slot) pair is taken first; ties go to the lower
// child, then the lower slot.
void assign_slots(const Child* kids, int n, const float nlo[3], const float nhi[3], int slot_of[8]) {
  double cost[8][8];
  for (int i = 0; i < n; ++i) {
    double d[3];
    for (int a = 0; a < 3; ++a)
      d[a] = 0.5 * (double(kids[i].lo[a]) + kids[i].hi[a]) - 0.5 * (double(nlo[a]) + nhi[a]);
    for (int s = 0; s < 8; ++s) {
      double dot = 0;
      for (int a = 0; a < 3; ++a) dot += ((s >> a) & 1 ? d[a] : -d[a]);
      cost[i][s] = -dot;
    }
  }
  bool child_done[8] = {}, slot_used[8] = {};
  for (int round = 0; round < n; ++round) {
    int bi = -1, bs = -1;
    for (int i = 0; i < n; ++i) {
      if (child_done[i]) continue;
      for (int s = 0; s < 8; ++s) {
        if (slot_used[s]) continue;
        if (bi < 0 || cost[i][s] < cost[bi][bs]) {
          bi = i;
          bs = s;
        }
      }
    }
    child_done[bi] = slot_used[bs] = true;
    slot_of[bi] = bs;
  }
}

std::uint32_t pack4(const std::uint8_t* q, int first) {
  return static_cast<std::uint32_t>(q[first]) | static_cast<std::uint32_t>(q[first + 1]) << 8 |
         static_cast<std::uint32_t>(q[first + 2]) << 16 | static_cast<std::uint32_t>(q[first + 3]) << 24;
}

}  // namespace

Wide8 build_wide8(const DevNode* nodes, std::size_t n_nodes, std::int32_t root, const std::uint8_t* last,
                  std::size_t n_slots) {
  Wide8 w;
  w.old_of.resize(n_slots);
  w.new_of.resize(n_slots);
  if (root == INT32_MIN || root < 0) {
    // No bounded primitives, or one leaf holds them all: the slot order stays.
    for (std::size_t k = 0; k < n_slots; ++k) w.old_of[k] = w.new_of[k] = static_cast<std::uint32_t>(k);
    w.root = root;
    return w;
  }
  if (static_cast<std::size_t>(root) >= n_nodes) throw std::runtime_error("wide8: root out of range");

  // Pending nodes in breadth-first order: a binary interior node to collapse, or
  // one wrapped leaf.
  struct Pending {
    Child origin;  // link >= 0: binary interior node; < 0: a wrapped leaf
    int depth;
  };
  std::vector<Pending> queue;
  queue.push_back({Child{root, {}, {}}, 1});
  std::size_t next_slot = 0;
  auto leaf_size = [&](std::int32_t link) {
    std::size_t k = static_cast<std::size_t>(~link), n = 1;
    while (k < n_slots && !last[k]) {
      ++k;
      ++n;
    }
    if (k >= n_slots) throw std::runtime_error("wide8: leaf runs past the last slot");
    return n;
  };
  for (std::size_t qi = 0; qi < queue.size(); ++qi) {
    const Pending p = queue[qi];
    w.depth = std::max(w.depth, p.depth);
    Child kids[8];
    int n = 0;
    if (p.origin.link >= 0) {
      if (static_cast<std::size_t>(p.origin.link) >= n_nodes) throw std::runtime_error("wide8: link out of range");
      n = collapse(nodes, p.origin.link, kids);
    } else {
      kids[0] = p.origin;
      kids[0].wrap = false;
      n = 1;
    }
    float nlo[3], nhi[3];
    for (int a = 0; a < 3; ++a) {
      nlo[a] = kids[0].lo[a];
      nhi[a] = kids[0].hi[a];
      for (int i = 1; i < n; ++i) {
        nlo[a] = std::min(nlo[a], kids[i].lo[a]);
        nhi[a] = std::max(nhi[a], kids[i].hi[a]);
      }
    }
    int slot_of[8];
    assign_slots(kids, n, nlo, nhi, slot_of);
    int kid_in[8];
    for (int s = 0; s < 8; ++s) kid_in[s] = -1;
    for (int i = 0; i < n; ++i) kid_in[slot_of[i]] = i;

    // Leaf children in slot order get consecutive slots from prim_base; one that
    // would start too far away becomes a node of its own.
    std::uint32_t meta[8] = {};
    std::uint32_t imask = 0;
    std::size_t offset = 0;
    for (int s = 0; s < 8; ++s) {
      const int i = kid_in[s];
      if (i < 0 || kids[i].link >= 0) continue;
      if (offset > static_cast<std::size_t>(kWide8MaxLeafOffset)) {
        kids[i].wrap = true;
        continue;
      }
      meta[s] = static_cast<std::uint32_t>(offset);
      offset += leaf_size(kids[i].link);
    }
    const std::uint32_t prim_base = static_cast<std::uint32_t>(next_slot);
    for (int s = 0; s < 8; ++s) {
      const int i = kid_in[s];
      if (i < 0 || kids[i].link >= 0 || kids[i].wrap) continue;
      const std::size_t start = static_cast<std::size_t>(~kids[i].link), size = leaf_size(kids[i].link);
      for (std::size_t k = 0; k < size; ++k) {
        w.old_of[next_slot] = static_cast<std::uint32_t>(start + k);
        w.new_of[start + k] = static_cast<std::uint32_t>(next_slot);
        ++next_slot;
      }
    }
    // Interior children (and wrapped leaves) in slot order, contiguous from child_base.
    const std::uint32_t child_base = static_cast<std::uint32_t>(queue.size());
    std::uint32_t rank = 0;
    for (int s = 0; s < 8; ++s) {
      const int i = kid_in[s];
      if (i < 0 || (kids[i].link < 0 && !kids[i].wrap)) continue;
      imask |= 1u << s;
      meta[s] = rank++;
      queue.push_back({kids[i], p.depth + 1});
    }

    // Quantised child boxes, rounded outward.
    int e[3];
    double scale[3];
    for (int a = 0; a < 3; ++a) {
      e[a] = axis_exponent(double(nhi[a]) - double(nlo[a]));
      scale[a] = std::ldexp(1.0, e[a] - 127);
    }
    std::uint8_t qlo[3][8], qhi[3][8];
    for (int s = 0; s < 8; ++s) {
      const int i = kid_in[s];
      for (int a = 0; a < 3; ++a) {
        if (i < 0) {
          qlo[a][s] = 255;
          qhi[a][s] = 0;
          continue;
        }
        const double lo = std::floor((double(kids[i].lo[a]) - nlo[a]) / scale[a]);
        const double hi = std::ceil((double(kids[i].hi[a]) - nlo[a]) / scale[a]);
        if (lo < 0 || hi > 255 || lo > hi) throw std::runtime_error("wide8: child box outside its node");
        qlo[a][s] = static_cast<std::uint8_t>(lo);
        qhi[a][s] = static_cast<std::uint8_t>(hi);
      }
    }
    DevNode8 d;
    const std::uint32_t ew = static_cast<std::uint32_t>(e[0]) | static_cast<std::uint32_t>(e[1]) << 8 |
                             static_cast<std::uint32_t>(e[2]) << 16 | imask << 24;
    float ewf;
    std::memcpy(&ewf, &ew, 4);
    d.a = make_float4(nlo[0], nlo[1], nlo[2], ewf);
    std::uint8_t mb[8];
    for (int s = 0; s < 8; ++s) mb[s] = static_cast<std::uint8_t>(meta[s]);
    d.b = make_uint4(child_base, prim_base, pack4(mb, 0), pack4(mb, 4));
    d.qlo_xy = make_uint4(pack4(qlo[0], 0), pack4(qlo[0], 4), pack4(qlo[1], 0), pack4(qlo[1], 4));
    d.qlo_z_hi_x = make_uint4(pack4(qlo[2], 0), pack4(qlo[2], 4), pack4(qhi[0], 0), pack4(qhi[0], 4));
    d.qhi_yz = make_uint4(pack4(qhi[1], 0), pack4(qhi[1], 4), pack4(qhi[2], 0), pack4(qhi[2], 4));
    w.nodes.push_back(d);
  }
  if (next_slot != n_slots) throw std::runtime_error("wide8: leaves do not cover every slot");
  if (w.depth > kWide8StackDepth) throw std::runtime_error("BVH deeper than the eight-wide traversal stack allows");
  w.root = 0;
  return w;
}

}  // namespace rtg
