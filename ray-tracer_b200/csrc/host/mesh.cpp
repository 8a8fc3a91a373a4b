#include "host/mesh.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace rtg {

void IndexedMesh::smooth_normals() {
  normals.assign(positions.size(), D3{});
  // Un-normalised face normals are twice the face area: summing them weights by area.
  for (const auto& f : faces) {
    const D3 p0 = positions[f[0]], p1 = positions[f[1]], p2 = positions[f[2]];
    const D3 fn = cross(p1 - p0, p2 - p0);
    for (const std::uint32_t v : f) normals[v] = normals[v] + fn;
  }
  for (D3& n : normals) n = unit_or(n, D3{0, 1, 0});
}

D3 Placement::point(D3 p) const {
  const D3 s = p * scale;
  const double ang = rotate_y_deg * kPi / 180;
  const double c = std::cos(ang), sn = std::sin(ang);
  return D3{c * s.x + sn * s.z, s.y, -sn * s.x + c * s.z} + translate;
}

D3 Placement::normal(D3 n) const {
  const D3 s{n.x / scale.x, n.y / scale.y, n.z / scale.z};
  const double ang = rotate_y_deg * kPi / 180;
  const double c = std::cos(ang), sn = std::sin(ang);
  return unit_or(D3{c * s.x + sn * s.z, s.y, -sn * s.x + c * s.z}, n);
}

IndexedMesh icosphere(int subdivisions) {
  IndexedMesh m;
  // The 12 vertices of a regular icosahedron are the cyclic permutations of
  // (0, +-1, +-phi); faces are listed counter-clockwise seen from outside.
  const double phi = (1 + std::sqrt(5.0)) / 2;
  m.positions = {{-1, phi, 0}, {1, phi, 0}, {-1, -phi, 0}, {1, -phi, 0}, {0, -1, phi}, {0, 1, phi},
                 {0, -1, -phi}, {0, 1, -phi}, {phi, 0, -1}, {phi, 0, 1}, {-phi, 0, -1}, {-phi, 0, 1}};
  for (D3& p : m.positions) p = unit(p);
  m.faces = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
             {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
             {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
  for (int level = 0; level < subdivisions; ++level) {
    // Each edge gets one midpoint vertex, created the first time the edge is
    // met while walking the faces in order (so vertex numbering is stable).
    // Open-addressing table edge -> midpoint vertex, at most half full. A key
    // is never 0: an edge's larger endpoint index is at least 1.
    int bits = 1;
    while ((std::size_t(1) << bits) < m.faces.size() * 4) ++bits;
    const std::size_t mask = (std::size_t(1) << bits) - 1;
    std::vector<std::uint64_t> keys(mask + 1, 0);
    std::vector<std::uint32_t> mids(mask + 1, 0);
    auto midpoint = [&](std::uint32_t a, std::uint32_t b) -> std::uint32_t {
      const std::uint64_t key = (std::uint64_t(std::min(a, b)) << 32) | std::max(a, b);
      std::size_t h = static_cast<std::size_t>((key * 0x9E3779B97F4A7C15ull) >> (64 - bits));
      while (keys[h] != 0) {
        if (keys[h] == key) return mids[h];
        h = (h + 1) & mask;
      }
      m.positions.push_back(unit(m.positions[a] + m.positions[b]));
      const auto id = static_cast<std::uint32_t>(m.positions.size() - 1);
      keys[h] = key;
      mids[h] = id;
      return id;
    };
    std::vector<std::array<std::uint32_t, 3>> finer;
    finer.reserve(m.faces.size() * 4);
    for (const auto& f : m.faces) {
      const std::uint32_t ab = midpoint(f[0], f[1]);
      const std::uint32_t bc = midpoint(f[1], f[2]);
      const std::uint32_t ca = midpoint(f[2], f[0]);
      finer.push_back({f[0], ab, ca});
      finer.push_back({f[1], bc, ab});
      finer.push_back({f[2], ca, bc});
      finer.push_back({ab, bc, ca});
    }
    m.faces.swap(finer);
  }
  m.normals = m.positions;  // a unit sphere's normal is its position
  return m;
}

IndexedMesh torus(double major, double minor, int seg_u, int seg_v) {
  IndexedMesh m;
  const int nu = std::max(3, seg_u), nv = std::max(3, seg_v);
  m.positions.reserve(std::size_t(nu) * std::size_t(nv));
  m.normals.reserve(std::size_t(nu) * std::size_t(nv));
  for (int i = 0; i < nu; ++i) {
    const double u = 2 * kPi * i / nu;
    const D3 ring{std::cos(u), 0, std::sin(u)};
    for (int j = 0; j < nv; ++j) {
      const double v = 2 * kPi * j / nv;
      const D3 n = std::cos(v) * ring + D3{0, std::sin(v), 0};
      m.positions.push_back(major * ring + minor * n);
      m.normals.push_back(n);
    }
  }
  auto vid = [&](int i, int j) { return static_cast<std::uint32_t>((i % nu) * nv + (j % nv)); };
  m.faces.reserve(std::size_t(nu) * std::size_t(nv) * 2);
  for (int i = 0; i < nu; ++i)
    for (int j = 0; j < nv; ++j) {
      // Two triangles per (u, v) cell, wound so cross(e1, e2) points outward.
      m.faces.push_back({vid(i, j), vid(i, j + 1), vid(i + 1, j)});
      m.faces.push_back({vid(i + 1, j), vid(i, j + 1), vid(i + 1, j + 1)});
    }
  return m;
}

namespace {

[[noreturn]] void obj_fail(int line, const std::string& what) {
  throw std::runtime_error("OBJ line " + std::to_string(line) + ": " + what);
}

// Resolves a 1-based (or negative, relative) OBJ index against `count` entries.
std::uint32_t obj_index(long v, std::size_t count, int line) {
  long idx = v > 0 ? v - 1 : static_cast<long>(count) + v;
  if (v == 0 || idx < 0 || static_cast<std::size_t>(idx) >= count) obj_fail(line, "index out of range");
  return static_cast<std::uint32_t>(idx);
}

}  // namespace

IndexedMesh parse_obj_text(const std::string& text) {
  IndexedMesh m;
  std::vector<D3> vn;
  // File normals survive only if every face corner names one and each position
  // always names the same one; otherwise the compiler computes smooth normals.
  std::vector<long> normal_for;  // per position, -1 = none yet
  bool consistent = true;
  std::istringstream in(text);
  std::string raw;
  int line = 0;
  while (std::getline(in, raw)) {
    ++line;
    std::istringstream ls(raw);
    std::string tag;
    if (!(ls >> tag) || tag[0] == '#') continue;
    if (tag == "v") {
      D3 p;
      if (!(ls >> p.x >> p.y >> p.z)) obj_fail(line, "bad vertex");
      m.positions.push_back(p);
      normal_for.push_back(-1);
    } else if (tag == "vn") {
      D3 n;
      if (!(ls >> n.x >> n.y >> n.z)) obj_fail(line, "bad normal");
      vn.push_back(unit_or(n, D3{0, 1, 0}));
    } else if (tag == "f") {
      std::vector<std::uint32_t> poly;
      std::string tok;
      while (ls >> tok) {
        // v, v/vt, v//vn or v/vt/vn
        const auto s1 = tok.find('/');
        long pi = 0, ni = 0;
        bool with_normal = false;
        try {
          pi = std::stol(tok.substr(0, s1));
          if (s1 != std::string::npos) {
            const auto s2 = tok.find('/', s1 + 1);
            if (s2 != std::string::npos && s2 + 1 < tok.size()) {
              ni = std::stol(tok.substr(s2 + 1));
              with_normal = true;
            }
          }
        } catch (const std::exception&) {
          obj_fail(line, "bad face corner '" + tok + "'");
        }
        const std::uint32_t p = obj_index(pi, m.positions.size(), line);
        if (with_normal) {
          const long n = static_cast<long>(obj_index(ni, vn.size(), line));
          if (normal_for[p] < 0) normal_for[p] = n;
          else if (normal_for[p] != n) consistent = false;
        } else {
          consistent = false;
        }
        poly.push_back(p);
      }
      if (poly.size() < 3) obj_fail(line, "face has < 3 vertices");
      for (std::size_t k = 1; k + 1 < poly.size(); ++k) m.faces.push_back({poly[0], poly[k], poly[k + 1]});
    }
  }
  if (consistent && !vn.empty() && !m.faces.empty()) {
    m.normals.assign(m.positions.size(), D3{0, 1, 0});
    for (std::size_t i = 0; i < m.positions.size(); ++i)
      if (normal_for[i] >= 0) m.normals[i] = vn[static_cast<std::size_t>(normal_for[i])];
  }
  return m;
}

IndexedMesh load_obj_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open OBJ file: " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return parse_obj_text(ss.str());
}

}  // namespace rtg
