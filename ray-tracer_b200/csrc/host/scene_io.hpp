#pragma once
// Scene JSON <-> SceneDesc, with the reference's schema, defaults, validation
// ranges and field-path error messages (src/io/scene_io.cpp:101-502,
// include/raytracer/io/scene_io.hpp:13-30).
#include <stdexcept>
#include <string>
#include <vector>

#include "host/json.hpp"
#include "host/scene_desc.hpp"

namespace rtg {

// Any problem in a scene description; the message names the offending field
// ("objects[2].radius: must be > 0").
struct SceneError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

SceneDesc scene_from_json(const JsonValue& root);   // parse + validate
SceneDesc parse_scene(const std::string& text);      // JSON text -> SceneDesc
SceneDesc load_scene(const std::string& path);       // file -> SceneDesc (sets base_dir)
JsonValue scene_to_json(const SceneDesc& s);
std::vector<std::string> validate_scene(const SceneDesc& s);

const char* integrator_name(Integrator i);
const char* tone_map_name(ToneMap t);

}  // namespace rtg
