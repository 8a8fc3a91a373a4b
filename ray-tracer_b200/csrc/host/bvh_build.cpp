#include "host/bvh_build.hpp"

#include <algorithm>
#include <array>
#include <chrono>
#include <stdexcept>

namespace rtg {

namespace {

constexpr int kBinCount = 16;
constexpr double kNodeCost = 1.0;      // one node visit relative to one primitive test
constexpr std::size_t kDepthCap = 60;  // keeps the traversal stack within 64 entries

struct Item {
  Box box;
  D3 centre;
  std::uint32_t id;
};

int bin_index(double c, double lo, double inv_width) {
  const int b = static_cast<int>((c - lo) * inv_width);
  return std::clamp(b, 0, kBinCount - 1);
}

class SahBuilder {
 public:
  SahBuilder(std::vector<Item>& items, BinaryBvh& out, std::size_t leaf_cap)
      : items_(items), out_(out), leaf_cap_(leaf_cap) {}

  void node(std::size_t lo, std::size_t hi, std::size_t depth) {
    const std::size_t me = out_.nodes.size();
    out_.nodes.emplace_back();
    Box box, cbox;
    for (std::size_t i = lo; i < hi; ++i) {
      box.grow(items_[i].box);
      cbox.grow(items_[i].centre);
    }
    out_.nodes[me].box = box;
    out_.stats.max_depth = std::max(out_.stats.max_depth, depth);
    const std::size_t n = hi - lo;
    if (n <= leaf_cap_ || depth >= kDepthCap) return leaf(me, lo, n);

    // Evaluate the kBinCount - 1 bin boundaries on every axis.
    int split_axis = -1, split_bin = -1;
    double split_cost = kInf;
    const double parent_area = box.area();
    for (int axis = 0; axis < 3; ++axis) {
      const double clo = cbox.lo[axis], chi = cbox.hi[axis];
      if (!(chi > clo)) continue;
      std::array<Box, kBinCount> bin_box{};
      std::array<std::size_t, kBinCount> bin_n{};
      const double inv_width = kBinCount / (chi - clo);
      for (std::size_t i = lo; i < hi; ++i) {
        const auto b = static_cast<std::size_t>(bin_index(items_[i].centre[axis], clo, inv_width));
        bin_n[b]++;
        bin_box[b].grow(items_[i].box);
      }
      // Suffix (right-side) areas and counts, then a prefix sweep.
      std::array<double, kBinCount> right_area{};
      std::array<std::size_t, kBinCount> right_n{};
      Box acc;
      std::size_t cnt = 0;
      for (int b = kBinCount - 1; b > 0; --b) {
        const auto ub = static_cast<std::size_t>(b);
        acc.grow(bin_box[ub]);
        cnt += bin_n[ub];
        right_area[ub] = acc.area();
        right_n[ub] = cnt;
      }
      acc = Box{};
      cnt = 0;
      for (int b = 0; b < kBinCount - 1; ++b) {
        const auto ub = static_cast<std::size_t>(b);
        acc.grow(bin_box[ub]);
        cnt += bin_n[ub];
        const std::size_t rn = right_n[ub + 1];
        if (cnt == 0 || rn == 0) continue;
        const double cost = kNodeCost + (acc.area() * double(cnt) + right_area[ub + 1] * double(rn)) /
                                            std::max(parent_area, 1e-30);
        if (cost < split_cost) {
          split_cost = cost;
          split_axis = axis;
          split_bin = b;
        }
      }
    }

    std::size_t mid;
    if (split_axis < 0) {
      // Every centroid coincides: no plane separates them, split by count.
      mid = lo + n / 2;
      split_axis = cbox.widest_axis();
    } else {
      if (split_cost >= double(n) && n <= 16) return leaf(me, lo, n);
      const double clo = cbox.lo[split_axis];
      const double inv_width = kBinCount / (cbox.hi[split_axis] - clo);
      const auto first = items_.begin() + static_cast<std::ptrdiff_t>(lo);
      const auto last = items_.begin() + static_cast<std::ptrdiff_t>(hi);
      const auto cut = std::partition(first, last, [&](const Item& it) {
        return bin_index(it.centre[split_axis], clo, inv_width) <= split_bin;
      });
      mid = static_cast<std::size_t>(cut - items_.begin());
      if (mid == lo || mid == hi) mid = lo + n / 2;  // rounding put everything on one side
    }

    out_.nodes[me].axis = static_cast<std::uint8_t>(split_axis);
    node(lo, mid, depth + 1);
    const std::size_t right = out_.nodes.size();
    node(mid, hi, depth + 1);
    out_.nodes[me].first = static_cast<std::uint32_t>(right);
    out_.nodes[me].count = 0;
  }

 private:
  void leaf(std::size_t me, std::size_t lo, std::size_t n) {
    if (n > 0xFFFF) throw std::runtime_error("BVH leaf too large");
    out_.nodes[me].first = static_cast<std::uint32_t>(lo);
    out_.nodes[me].count = static_cast<std::uint32_t>(n);
    out_.stats.leaves++;
    out_.stats.max_leaf = std::max(out_.stats.max_leaf, n);
  }

  std::vector<Item>& items_;
  BinaryBvh& out_;
  std::size_t leaf_cap_;
};

}  // namespace

void BinaryBvh::build(const std::vector<Box>& prim_boxes, int max_leaf) {
  const auto t0 = std::chrono::steady_clock::now();
  nodes.clear();
  order.clear();
  stats = {};
  std::vector<Item> items;
  items.reserve(prim_boxes.size());
  for (std::size_t i = 0; i < prim_boxes.size(); ++i) {
    const Box& b = prim_boxes[i];
    if (b.empty() || !b.lo.finite() || !b.hi.finite()) continue;  // nothing to hit
    items.push_back({b, b.center(), static_cast<std::uint32_t>(i)});
  }
  if (items.empty()) return;
  const std::size_t cap = static_cast<std::size_t>(std::max(1, max_leaf));
  nodes.reserve(2 * items.size() / cap + 1);
  SahBuilder(items, *this, cap).node(0, items.size(), 0);
  order.resize(items.size());
  for (std::size_t i = 0; i < items.size(); ++i) order[i] = items[i].id;

  const double root_area = std::max(nodes[0].box.area(), 1e-30);
  for (const BinaryNode& n : nodes) stats.sah_cost += n.box.area() / root_area * (n.leaf() ? double(n.count) : kNodeCost);
  stats.nodes = nodes.size();
  stats.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

bool BinaryBvh::check(const std::vector<Box>& prim_boxes) const {
  auto inside = [](const Box& outer, const Box& inner) {
    const double e = 1e-9;
    return inner.lo.x >= outer.lo.x - e && inner.lo.y >= outer.lo.y - e && inner.lo.z >= outer.lo.z - e &&
           inner.hi.x <= outer.hi.x + e && inner.hi.y <= outer.hi.y + e && inner.hi.z <= outer.hi.z + e;
  };
  std::vector<int> seen(prim_boxes.size(), 0);
  for (std::size_t i = 0; i < nodes.size(); ++i) {
    const BinaryNode& n = nodes[i];
    if (n.leaf()) {
      for (std::uint32_t k = 0; k < n.count; ++k) {
        const std::uint32_t p = order[n.first + k];
        if (!inside(n.box, prim_boxes[p])) return false;
        seen[p]++;
      }
    } else {
      if (n.first >= nodes.size() || n.first <= i) return false;
      if (!inside(n.box, nodes[i + 1].box) || !inside(n.box, nodes[n.first].box)) return false;
    }
  }
  for (std::size_t p = 0; p < prim_boxes.size(); ++p)
    if (seen[p] != (prim_boxes[p].empty() ? 0 : 1)) return false;
  return true;
}

}  // namespace rtg
