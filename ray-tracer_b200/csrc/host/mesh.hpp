#pragma once
// Indexed triangle meshes for procedural and OBJ geometry, generated with the
// reference's vertex and face ordering (src/geometry/mesh.cpp:10-88), because the
// face order becomes the primitive order and therefore the hit ids.
#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "host/vec.hpp"

namespace rtg {

struct IndexedMesh {
  std::vector<D3> positions;
  std::vector<D3> normals;  // per vertex; empty or positions.size()
  std::vector<std::array<std::uint32_t, 3>> faces;
  void smooth_normals();    // area-weighted vertex normals
};

// Scale, then rotate about +Y (degrees), then translate; normals use the
// inverse transpose of the linear part.
struct Placement {
  D3 scale{1, 1, 1};
  double rotate_y_deg = 0;
  D3 translate{0, 0, 0};
  D3 point(D3 p) const;
  D3 normal(D3 n) const;
};

IndexedMesh icosphere(int subdivisions);                          // unit radius, 20 * 4^s faces
IndexedMesh torus(double major, double minor, int seg_u, int seg_v);
IndexedMesh parse_obj_text(const std::string& text);              // v / vn / f, fan triangulation
IndexedMesh load_obj_file(const std::string& path);

}  // namespace rtg
