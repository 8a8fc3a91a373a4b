#include "host/bvh_build.hpp"

#include <algorithm>
#include <array>
#include <chrono>
#include <future>
#include <stdexcept>
#include <thread>

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

// Large nodes bin on several threads and their two subtrees build concurrently.
// Box unions (min/max) and counts do not depend on the order they are taken in,
// and each subtree's nodes are numbered locally and spliced into the depth-first
// order afterwards, so the tree is the same as a single-threaded build's.
constexpr std::size_t kParallelItems = 16384;   // subtrees at least this big may build concurrently
constexpr std::size_t kParallelBinItems = 65536; // nodes at least this big bin on several threads
constexpr std::size_t kMaxTasks = 16;

struct Subtree {
  std::vector<BinaryNode> nodes;
  BvhStats stats;
};

// Runs body(t, begin, end) on `parts` contiguous chunks of [lo, hi) concurrently.
template <class F>
void chunked(std::size_t lo, std::size_t hi, std::size_t parts, F&& body) {
  std::vector<std::thread> pool;
  const std::size_t n = hi - lo, step = (n + parts - 1) / parts;
  for (std::size_t t = 1; t < parts; ++t) {
    const std::size_t b = std::min(hi, lo + t * step), e = std::min(hi, b + step);
    pool.emplace_back([&body, t, b, e] { body(t, b, e); });
  }
  body(std::size_t(0), lo, std::min(hi, lo + step));
  for (auto& th : pool) th.join();
}

class SahBuilder {
 public:
  SahBuilder(std::vector<Item>& items, std::size_t leaf_cap) : items_(items), leaf_cap_(leaf_cap) {
    workers_ = std::min<std::size_t>(kMaxTasks, std::max(1u, std::thread::hardware_concurrency()));
  }

  // Builds the subtree over items [lo, hi) into `out` (indices local to `out`).
  void node(std::size_t lo, std::size_t hi, std::size_t depth, Subtree& out, std::size_t tasks) {
    const std::size_t me = out.nodes.size();
    out.nodes.emplace_back();
    const std::size_t n = hi - lo;
    const std::size_t parts = (n >= kParallelBinItems && tasks > 1) ? std::min<std::size_t>(tasks, 16) : 1;
    Box box, cbox;
    if (parts > 1) {
      std::vector<Box> pb(parts), pc(parts);
      chunked(lo, hi, parts, [&](std::size_t t, std::size_t b, std::size_t e) {
        for (std::size_t i = b; i < e; ++i) {
          pb[t].grow(items_[i].box);
          pc[t].grow(items_[i].centre);
        }
      });
      for (std::size_t t = 0; t < parts; ++t) {
        box.grow(pb[t]);
        cbox.grow(pc[t]);
      }
    } else {
      for (std::size_t i = lo; i < hi; ++i) {
        box.grow(items_[i].box);
        cbox.grow(items_[i].centre);
      }
    }
    out.nodes[me].box = box;
    out.stats.max_depth = std::max(out.stats.max_depth, depth);
    if (n <= leaf_cap_ || depth >= kDepthCap) return leaf(out, me, lo, n);

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
      if (parts > 1) {
        std::vector<std::array<Box, kBinCount>> pbox(parts);
        std::vector<std::array<std::size_t, kBinCount>> pn(parts);
        chunked(lo, hi, parts, [&](std::size_t t, std::size_t b, std::size_t e) {
          pn[t].fill(0);
          for (std::size_t i = b; i < e; ++i) {
            const auto k = static_cast<std::size_t>(bin_index(items_[i].centre[axis], clo, inv_width));
            pn[t][k]++;
            pbox[t][k].grow(items_[i].box);
          }
        });
        for (std::size_t t = 0; t < parts; ++t)
          for (std::size_t k = 0; k < kBinCount; ++k) {
            bin_n[k] += pn[t][k];
            bin_box[k].grow(pbox[t][k]);
          }
      } else {
        for (std::size_t i = lo; i < hi; ++i) {
          const auto b = static_cast<std::size_t>(bin_index(items_[i].centre[axis], clo, inv_width));
          bin_n[b]++;
          bin_box[b].grow(items_[i].box);
        }
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
      if (split_cost >= double(n) && n <= 16) return leaf(out, me, lo, n);
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

    out.nodes[me].axis = static_cast<std::uint8_t>(split_axis);
    out.nodes[me].count = 0;
    if (tasks > 1 && mid - lo >= kParallelItems && hi - mid >= kParallelItems) {
      // Both halves concurrently, each into its own list, then spliced in order.
      Subtree left, right;
      const std::size_t lt = tasks / 2, rt = tasks - lt;
      auto done = std::async(std::launch::async, [&] { node(lo, mid, depth + 1, left, lt); });
      node(mid, hi, depth + 1, right, rt);
      done.get();
      splice(out, left);
      out.nodes[me].first = static_cast<std::uint32_t>(out.nodes.size());
      splice(out, right);
      return;
    }
    node(lo, mid, depth + 1, out, tasks);
    const std::size_t right = out.nodes.size();
    node(mid, hi, depth + 1, out, tasks);
    out.nodes[me].first = static_cast<std::uint32_t>(right);
  }

  std::size_t workers() const { return workers_; }

 private:
  void leaf(Subtree& out, std::size_t me, std::size_t lo, std::size_t n) {
    if (n > 0xFFFF) throw std::runtime_error("BVH leaf too large");
    out.nodes[me].first = static_cast<std::uint32_t>(lo);
    out.nodes[me].count = static_cast<std::uint32_t>(n);
    out.stats.leaves++;
    out.stats.max_leaf = std::max(out.stats.max_leaf, n);
  }

  // Appends a subtree built with local indices; its interior links move by the offset.
  static void splice(Subtree& out, const Subtree& sub) {
    const auto base = static_cast<std::uint32_t>(out.nodes.size());
    for (BinaryNode nd : sub.nodes) {
      if (!nd.leaf()) nd.first += base;
      out.nodes.push_back(nd);
    }
    out.stats.leaves += sub.stats.leaves;
    out.stats.max_leaf = std::max(out.stats.max_leaf, sub.stats.max_leaf);
    out.stats.max_depth = std::max(out.stats.max_depth, sub.stats.max_depth);
  }

  std::vector<Item>& items_;
  std::size_t leaf_cap_;
  std::size_t workers_ = 1;
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
  SahBuilder builder(items, cap);
  Subtree tree;
  tree.nodes.reserve(2 * items.size() / cap + 1);
  builder.node(0, items.size(), 0, tree, builder.workers());
  nodes = std::move(tree.nodes);
  stats.leaves = tree.stats.leaves;
  stats.max_leaf = tree.stats.max_leaf;
  stats.max_depth = tree.stats.max_depth;
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
