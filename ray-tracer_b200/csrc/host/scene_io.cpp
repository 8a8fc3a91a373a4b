// Scene JSON <-> SceneDesc, driven by one declarative schema.
//
// Each record of a scene file (camera, render, background, the four material
// kinds, the six object kinds, a point light) is described by a table of its
// fields: JSON key, value kind, whether it is required, and how the value goes
// into and out of the description. Reading walks a table in order, so the first
// bad field in table order is the one reported; writing walks the same table
// (or a record's own write order) and skips fields whose `written` test fails.
// Validation is a second table per record: range checks with their messages,
// finiteness and colour checks of vector fields, evaluated over a SceneDesc (the
// CLI validates again after its command-line overrides).
//
// The schema itself — keys, defaults, kinds, ranges, the order problems are
// found in and every message — is the reference's contract for scene files
// (src/io/scene_io.cpp:101-473, include/raytracer/core/scene_desc.hpp:20-102), so
// that the same files are accepted and rejected with the same words.
// tests/test_scene_schema.py holds the reference CLI's own answers for a corpus
// of scenes and checks them byte for byte.
#include "host/scene_io.hpp"

#include <cmath>
#include <filesystem>
#include <fstream>
#include <span>
#include <sstream>
#include <utility>

namespace rtg {

namespace {

// ---------------------------------------------------------------------------
// Values

enum class Kind : std::uint8_t { Number, Integer, Flag, Text, Vector };

struct Value {
  double num = 0;
  int integer = 0;
  bool flag = false;
  std::string text;
  D3 vec;
};

std::string field_path(const std::string& at, const char* key) {
  return at.empty() ? std::string(key) : at + "." + key;
}

[[noreturn]] void reject(const std::string& at, const std::string& what) {
  throw SceneError((at.empty() ? std::string("scene") : at) + ": " + what);
}

// Decodes a present JSON value as `kind`; `at` is its field path.
Value decode(const JsonValue& v, Kind kind, const std::string& at) {
  Value out;
  switch (kind) {
    case Kind::Number:
      if (!v.is_number()) reject(at, "expected a number");
      out.num = v.number();
      break;
    case Kind::Integer: {
      if (!v.is_number()) reject(at, "expected an integer");
      const double d = v.number();
      if (d != std::floor(d) || std::fabs(d) > 2e9) reject(at, "expected an integer");
      out.integer = static_cast<int>(d);
      break;
    }
    case Kind::Flag:
      if (!v.is_bool()) reject(at, "expected true/false");
      out.flag = v.boolean();
      break;
    case Kind::Text:
      if (!v.is_string()) reject(at, "expected a string");
      out.text = v.str();
      break;
    case Kind::Vector:
      if (v.is_number()) {  // a scalar s stands for [s, s, s]
        out.vec = D3{v.number()};
        break;
      }
      if (!v.is_list() || v.list().size() != 3) reject(at, "expected [x, y, z]");
      for (int k = 0; k < 3; ++k) {
        const JsonValue& e = v.list()[static_cast<std::size_t>(k)];
        if (!e.is_number()) reject(at, "expected [x, y, z] of numbers");
        out.vec.at(k) = e.number();
      }
      break;
  }
  return out;
}

JsonValue vec_json(D3 v) { return JsonList{v.x, v.y, v.z}; }

// Named choices of an enumerated text field: "expected a, b or c" when unknown.
template <class E>
struct Choice {
  const char* name;
  E value;
};

template <class E, std::size_t N>
E choose(const Choice<E> (&options)[N], const std::string& text, const std::string& at) {
  for (const auto& o : options)
    if (text == o.name) return o.value;
  std::string list;
  for (std::size_t i = 0; i < N; ++i) list += (i == 0 ? "" : (i + 1 == N ? " or " : ", ")) + std::string(options[i].name);
  reject(at, "expected " + list);
}

template <class E, std::size_t N>
const char* choice_name(const Choice<E> (&options)[N], E value) {
  for (const auto& o : options)
    if (o.value == value) return o.name;
  return options[0].name;
}

constexpr Choice<Integrator> kIntegrators[] = {
    {"path", Integrator::Path}, {"direct", Integrator::Direct}, {"normals", Integrator::Normals}};
constexpr Choice<ToneMap> kToneMaps[] = {
    {"clamp", ToneMap::Clamp}, {"reinhard", ToneMap::Reinhard}, {"aces", ToneMap::Aces}};
constexpr Choice<Background::Kind> kBackgrounds[] = {
    {"gradient", Background::Kind::Gradient}, {"solid", Background::Kind::Solid}};
constexpr Choice<MeshDesc::Source> kMeshSources[] = {
    {"icosphere", MeshDesc::Source::Icosphere}, {"torus", MeshDesc::Source::Torus}, {"obj", MeshDesc::Source::ObjFile}};

// ---------------------------------------------------------------------------
// Field tables

// One field of record type R. `put` stores a decoded value (`at` is the field's
// path, for enumeration errors); `get` gives it back for writing. `read_if` and
// `written` gate the field on the record's other fields (null: always).
template <class R>
struct Field {
  const char* key;
  Kind kind;
  bool required;
  void (*put)(R&, Value&&, const std::string& at);
  JsonValue (*get)(const R&);
  bool (*read_if)(const R&) = nullptr;
  bool (*written)(const R&) = nullptr;
};

// Reads the fields of `table` from `j` (a map) into `rec`, in table order.
template <class R>
void read_fields(std::span<const Field<R>> table, const JsonValue& j, const std::string& at, R& rec) {
  for (const Field<R>& f : table) {
    if (f.read_if && !f.read_if(rec)) continue;
    const std::string where = field_path(at, f.key);
    const JsonValue* v = j.get(f.key);
    if (!v) {
      if (f.required) reject(where, "required");
      continue;
    }
    f.put(rec, decode(*v, f.kind, where), where);
  }
}

template <class R>
void write_fields(std::span<const Field<R>> table, const R& rec, JsonValue& j) {
  for (const Field<R>& f : table)
    if (!f.written || f.written(rec)) j[f.key] = f.get(rec);
}

// A map record: rejects anything else with "<path>: expected an object".
const JsonValue& record(const JsonValue& j, const std::string& at) {
  if (!j.is_map()) reject(at, "expected an object");
  return j;
}

const Field<CameraDesc> kCameraFields[] = {
    {"look_from", Kind::Vector, false, [](CameraDesc& c, Value&& v, const std::string&) { c.look_from = v.vec; },
     [](const CameraDesc& c) { return vec_json(c.look_from); }},
    {"look_at", Kind::Vector, false, [](CameraDesc& c, Value&& v, const std::string&) { c.look_at = v.vec; },
     [](const CameraDesc& c) { return vec_json(c.look_at); }},
    {"vup", Kind::Vector, false, [](CameraDesc& c, Value&& v, const std::string&) { c.vup = v.vec; },
     [](const CameraDesc& c) { return vec_json(c.vup); }},
    {"vfov", Kind::Number, false, [](CameraDesc& c, Value&& v, const std::string&) { c.vfov_deg = v.num; },
     [](const CameraDesc& c) { return JsonValue(c.vfov_deg); }},
    {"aperture", Kind::Number, false, [](CameraDesc& c, Value&& v, const std::string&) { c.aperture = v.num; },
     [](const CameraDesc& c) { return JsonValue(c.aperture); }},
    {"focus_dist", Kind::Number, false, [](CameraDesc& c, Value&& v, const std::string&) { c.focus_dist = v.num; },
     [](const CameraDesc& c) { return JsonValue(c.focus_dist); }},
};

const Field<RenderSettings> kRenderFields[] = {
    {"width", Kind::Integer, false, [](RenderSettings& r, Value&& v, const std::string&) { r.width = v.integer; },
     [](const RenderSettings& r) { return JsonValue(r.width); }},
    {"height", Kind::Integer, false, [](RenderSettings& r, Value&& v, const std::string&) { r.height = v.integer; },
     [](const RenderSettings& r) { return JsonValue(r.height); }},
    {"spp", Kind::Integer, false, [](RenderSettings& r, Value&& v, const std::string&) { r.spp = v.integer; },
     [](const RenderSettings& r) { return JsonValue(r.spp); }},
    {"max_depth", Kind::Integer, false, [](RenderSettings& r, Value&& v, const std::string&) { r.max_depth = v.integer; },
     [](const RenderSettings& r) { return JsonValue(r.max_depth); }},
    {"rr_min_depth", Kind::Integer, false,
     [](RenderSettings& r, Value&& v, const std::string&) { r.rr_min_depth = v.integer; },
     [](const RenderSettings& r) { return JsonValue(r.rr_min_depth); }},
    {"light_sampling", Kind::Flag, false,
     [](RenderSettings& r, Value&& v, const std::string&) { r.light_sampling = v.flag; },
     [](const RenderSettings& r) { return JsonValue(r.light_sampling); }},
    // Schema extension (no reference counterpart): written only when set.
    {"mis", Kind::Flag, false, [](RenderSettings& r, Value&& v, const std::string&) { r.mis = v.flag; },
     [](const RenderSettings&) { return JsonValue(true); }, nullptr, [](const RenderSettings& r) { return r.mis; }},
    // The seed is read as a 32-bit integer (and sign-extended), as the reference's loader reads it.
    {"seed", Kind::Integer, false,
     [](RenderSettings& r, Value&& v, const std::string&) { r.seed = static_cast<std::uint64_t>(v.integer); },
     [](const RenderSettings& r) { return JsonValue(r.seed); }},
    {"exposure", Kind::Number, false, [](RenderSettings& r, Value&& v, const std::string&) { r.exposure = v.num; },
     [](const RenderSettings& r) { return JsonValue(r.exposure); }},
    {"threads", Kind::Integer, false, [](RenderSettings& r, Value&& v, const std::string&) { r.threads = v.integer; },
     [](const RenderSettings& r) { return JsonValue(r.threads); }},
    {"tile_size", Kind::Integer, false,
     [](RenderSettings& r, Value&& v, const std::string&) { r.tile_size = v.integer; },
     [](const RenderSettings& r) { return JsonValue(r.tile_size); }},
    {"use_bvh", Kind::Flag, false, [](RenderSettings& r, Value&& v, const std::string&) { r.use_bvh = v.flag; },
     [](const RenderSettings& r) { return JsonValue(r.use_bvh); }},
    {"integrator", Kind::Text, false,
     [](RenderSettings& r, Value&& v, const std::string& at) { r.integrator = choose(kIntegrators, v.text, at); },
     [](const RenderSettings& r) { return JsonValue(choice_name(kIntegrators, r.integrator)); }},
    {"tone_map", Kind::Text, false,
     [](RenderSettings& r, Value&& v, const std::string& at) { r.tone_map = choose(kToneMaps, v.text, at); },
     [](const RenderSettings& r) { return JsonValue(choice_name(kToneMaps, r.tone_map)); }},
};
// The normalised file lists the render block in this order.
constexpr const char* kRenderWriteOrder[] = {"width", "height", "spp", "max_depth", "rr_min_depth", "integrator",
                                             "light_sampling", "mis", "seed", "tone_map", "exposure", "threads",
                                             "tile_size", "use_bvh"};

bool is_solid(const Background& b) { return b.kind == Background::Kind::Solid; }

// A solid background keeps its colour in `top` and reads it from "color".
const Field<Background> kBackgroundFields[] = {
    {"type", Kind::Text, false,
     [](Background& b, Value&& v, const std::string& at) { b.kind = choose(kBackgrounds, v.text, at); },
     [](const Background& b) { return JsonValue(choice_name(kBackgrounds, b.kind)); }},
    {"color", Kind::Vector, false, [](Background& b, Value&& v, const std::string&) { b.top = v.vec; },
     [](const Background& b) { return vec_json(b.top); }, is_solid, is_solid},
    {"top", Kind::Vector, false, [](Background& b, Value&& v, const std::string&) { b.top = v.vec; },
     [](const Background& b) { return vec_json(b.top); }, [](const Background& b) { return !is_solid(b); },
     [](const Background& b) { return !is_solid(b); }},
    {"bottom", Kind::Vector, false, [](Background& b, Value&& v, const std::string&) { b.bottom = v.vec; },
     [](const Background& b) { return vec_json(b.bottom); }, nullptr, [](const Background& b) { return !is_solid(b); }},
    {"intensity", Kind::Number, false, [](Background& b, Value&& v, const std::string&) { b.intensity = v.num; },
     [](const Background& b) { return JsonValue(b.intensity); }},
};

const Field<PointLightDesc> kLightFields[] = {
    {"name", Kind::Text, false, [](PointLightDesc& l, Value&& v, const std::string&) { l.name = std::move(v.text); },
     [](const PointLightDesc& l) { return JsonValue(l.name); }},
    {"position", Kind::Vector, true, [](PointLightDesc& l, Value&& v, const std::string&) { l.position = v.vec; },
     [](const PointLightDesc& l) { return vec_json(l.position); }},
    {"intensity", Kind::Vector, false, [](PointLightDesc& l, Value&& v, const std::string&) { l.intensity = v.vec; },
     [](const PointLightDesc& l) { return vec_json(l.intensity); }},
};

// ---------------------------------------------------------------------------
// Kinds of a variant: the schema of each alternative (its type names, fields
// and validation rules) is a specialisation of Schema<T>.

template <class T>
struct Schema;

// Validation rule of record type R. Check: `ok` must hold, else `message`.
// Finite: the vector must be finite. Colour: finite, and no component below 0.
template <class R>
struct Rule {
  enum Kind : std::uint8_t { Check, Finite, Colour } kind;
  const char* field;  // appended to the record's path; "" names the record itself
  const char* message = nullptr;
  bool (*ok)(const R&) = nullptr;
  D3 (*vec)(const R&) = nullptr;
};

template <class R>
Rule<R> check(const char* field, const char* message, bool (*ok)(const R&)) {
  return Rule<R>{Rule<R>::Check, field, message, ok, nullptr};
}
template <class R>
Rule<R> finite(const char* field, D3 (*vec)(const R&)) {
  return Rule<R>{Rule<R>::Finite, field, nullptr, nullptr, vec};
}
template <class R>
Rule<R> colour(const char* field, D3 (*vec)(const R&)) {
  return Rule<R>{Rule<R>::Colour, field, nullptr, nullptr, vec};
}

// Appends every problem of `rec` (at path `at`) to `out`, in rule order.
template <class R>
void apply_rules(std::span<const Rule<R>> rules, const R& rec, const std::string& at, std::vector<std::string>& out) {
  for (const Rule<R>& r : rules) {
    const std::string where = *r.field ? field_path(at, r.field) : at;
    if (r.kind == Rule<R>::Check) {
      if (!r.ok(rec)) out.push_back(where + ": " + r.message);
      continue;
    }
    const D3 v = r.vec(rec);
    if (!v.finite()) out.push_back(where + ": must be finite");
    if (r.kind == Rule<R>::Colour && (v.x < 0 || v.y < 0 || v.z < 0))
      out.push_back(where + ": colour components must be >= 0");
  }
}

bool finite_positive(double x) { return x > 0 && std::isfinite(x); }

template <>
struct Schema<Lambertian> {
  static constexpr const char* names[] = {"lambertian", "diffuse"};
  static inline const Field<Lambertian> fields[] = {
      {"albedo", Kind::Vector, false,
       [](Lambertian& m, Value&& v, const std::string&) { m.albedo.a = m.albedo.b = v.vec; },
       [](const Lambertian& m) { return vec_json(m.albedo.a); }},
      // Absent: the second checker colour is the first (set together above).
      {"albedo2", Kind::Vector, false, [](Lambertian& m, Value&& v, const std::string&) { m.albedo.b = v.vec; },
       [](const Lambertian& m) { return vec_json(m.albedo.b); }, nullptr,
       [](const Lambertian& m) { return m.albedo.checker_scale > 0; }},
      {"checker_scale", Kind::Number, false,
       [](Lambertian& m, Value&& v, const std::string&) { m.albedo.checker_scale = v.num; },
       [](const Lambertian& m) { return JsonValue(m.albedo.checker_scale); }, nullptr,
       [](const Lambertian& m) { return m.albedo.checker_scale > 0; }},
  };
  static inline const Rule<Lambertian> rules[] = {
      colour<Lambertian>("albedo", [](const Lambertian& m) { return m.albedo.a; }),
      colour<Lambertian>("albedo2", [](const Lambertian& m) { return m.albedo.b; }),
      check<Lambertian>("checker_scale", "must be >= 0", [](const Lambertian& m) { return !(m.albedo.checker_scale < 0); }),
  };
};

template <>
struct Schema<Metal> {
  static constexpr const char* names[] = {"metal"};
  static inline const Field<Metal> fields[] = {
      {"albedo", Kind::Vector, false, [](Metal& m, Value&& v, const std::string&) { m.albedo = v.vec; },
       [](const Metal& m) { return vec_json(m.albedo); }},
      {"roughness", Kind::Number, false, [](Metal& m, Value&& v, const std::string&) { m.roughness = v.num; },
       [](const Metal& m) { return JsonValue(m.roughness); }},
  };
  static inline const Rule<Metal> rules[] = {
      colour<Metal>("albedo", [](const Metal& m) { return m.albedo; }),
      check<Metal>("roughness", "must be in [0, 1]", [](const Metal& m) { return !(m.roughness < 0 || m.roughness > 1); }),
  };
};

template <>
struct Schema<Dielectric> {
  static constexpr const char* names[] = {"dielectric", "glass"};
  static inline const Field<Dielectric> fields[] = {
      {"ior", Kind::Number, false, [](Dielectric& m, Value&& v, const std::string&) { m.ior = v.num; },
       [](const Dielectric& m) { return JsonValue(m.ior); }},
      {"tint", Kind::Vector, false, [](Dielectric& m, Value&& v, const std::string&) { m.tint = v.vec; },
       [](const Dielectric& m) { return vec_json(m.tint); }},
  };
  static inline const Rule<Dielectric> rules[] = {
      check<Dielectric>("ior", "must be in [1, 4]", [](const Dielectric& m) { return m.ior >= 1.0 && m.ior <= 4.0; }),
      colour<Dielectric>("tint", [](const Dielectric& m) { return m.tint; }),
  };
};

template <>
struct Schema<Emissive> {
  static constexpr const char* names[] = {"emissive", "light"};
  static inline const Field<Emissive> fields[] = {
      {"color", Kind::Vector, false, [](Emissive& m, Value&& v, const std::string&) { m.color = v.vec; },
       [](const Emissive& m) { return vec_json(m.color); }},
      {"intensity", Kind::Number, false, [](Emissive& m, Value&& v, const std::string&) { m.intensity = v.num; },
       [](const Emissive& m) { return JsonValue(m.intensity); }},
      {"two_sided", Kind::Flag, false, [](Emissive& m, Value&& v, const std::string&) { m.two_sided = v.flag; },
       [](const Emissive&) { return JsonValue(true); }, nullptr, [](const Emissive& m) { return m.two_sided; }},
  };
  static inline const Rule<Emissive> rules[] = {
      colour<Emissive>("color", [](const Emissive& m) { return m.color; }),
      check<Emissive>("intensity", "must be >= 0", [](const Emissive& m) { return m.intensity >= 0 && std::isfinite(m.intensity); }),
  };
};

template <>
struct Schema<SphereDesc> {
  static constexpr const char* names[] = {"sphere"};
  static inline const Field<SphereDesc> fields[] = {
      {"center", Kind::Vector, true, [](SphereDesc& s, Value&& v, const std::string&) { s.center = v.vec; },
       [](const SphereDesc& s) { return vec_json(s.center); }},
      {"radius", Kind::Number, false, [](SphereDesc& s, Value&& v, const std::string&) { s.radius = v.num; },
       [](const SphereDesc& s) { return JsonValue(s.radius); }},
  };
  static inline const Rule<SphereDesc> rules[] = {
      finite<SphereDesc>("center", [](const SphereDesc& s) { return s.center; }),
      check<SphereDesc>("radius", "must be > 0", [](const SphereDesc& s) { return finite_positive(s.radius); }),
  };
};

template <>
struct Schema<PlaneDesc> {
  static constexpr const char* names[] = {"plane"};
  static inline const Field<PlaneDesc> fields[] = {
      {"point", Kind::Vector, false, [](PlaneDesc& p, Value&& v, const std::string&) { p.point = v.vec; },
       [](const PlaneDesc& p) { return vec_json(p.point); }},
      {"normal", Kind::Vector, false, [](PlaneDesc& p, Value&& v, const std::string&) { p.normal = v.vec; },
       [](const PlaneDesc& p) { return vec_json(p.normal); }},
  };
  static inline const Rule<PlaneDesc> rules[] = {
      finite<PlaneDesc>("point", [](const PlaneDesc& p) { return p.point; }),
      finite<PlaneDesc>("normal", [](const PlaneDesc& p) { return p.normal; }),
      check<PlaneDesc>("normal", "must be non-zero", [](const PlaneDesc& p) { return !(len(p.normal) < 1e-9); }),
  };
};

template <>
struct Schema<TriangleDesc> {
  static constexpr const char* names[] = {"triangle"};
  static inline const Field<TriangleDesc> fields[] = {
      {"v0", Kind::Vector, true, [](TriangleDesc& t, Value&& v, const std::string&) { t.v0 = v.vec; },
       [](const TriangleDesc& t) { return vec_json(t.v0); }},
      {"v1", Kind::Vector, true, [](TriangleDesc& t, Value&& v, const std::string&) { t.v1 = v.vec; },
       [](const TriangleDesc& t) { return vec_json(t.v1); }},
      {"v2", Kind::Vector, true, [](TriangleDesc& t, Value&& v, const std::string&) { t.v2 = v.vec; },
       [](const TriangleDesc& t) { return vec_json(t.v2); }},
  };
  static inline const Rule<TriangleDesc> rules[] = {
      finite<TriangleDesc>("v0", [](const TriangleDesc& t) { return t.v0; }),
      finite<TriangleDesc>("v1", [](const TriangleDesc& t) { return t.v1; }),
      finite<TriangleDesc>("v2", [](const TriangleDesc& t) { return t.v2; }),
      check<TriangleDesc>("", "triangle is degenerate",
                          [](const TriangleDesc& t) { return !(len(cross(t.v1 - t.v0, t.v2 - t.v0)) < 1e-12); }),
  };
};

template <>
struct Schema<QuadDesc> {
  static constexpr const char* names[] = {"quad"};
  static inline const Field<QuadDesc> fields[] = {
      {"corner", Kind::Vector, true, [](QuadDesc& q, Value&& v, const std::string&) { q.corner = v.vec; },
       [](const QuadDesc& q) { return vec_json(q.corner); }},
      {"u", Kind::Vector, true, [](QuadDesc& q, Value&& v, const std::string&) { q.u = v.vec; },
       [](const QuadDesc& q) { return vec_json(q.u); }},
      {"v", Kind::Vector, true, [](QuadDesc& q, Value&& v, const std::string&) { q.v = v.vec; },
       [](const QuadDesc& q) { return vec_json(q.v); }},
  };
  static inline const Rule<QuadDesc> rules[] = {
      finite<QuadDesc>("corner", [](const QuadDesc& q) { return q.corner; }),
      finite<QuadDesc>("u", [](const QuadDesc& q) { return q.u; }),
      finite<QuadDesc>("v", [](const QuadDesc& q) { return q.v; }),
      check<QuadDesc>("", "quad is degenerate (u parallel to v)",
                      [](const QuadDesc& q) { return !(len(cross(q.u, q.v)) < 1e-12); }),
  };
};

template <>
struct Schema<BoxDesc> {
  static constexpr const char* names[] = {"box"};
  static inline const Field<BoxDesc> fields[] = {
      {"min", Kind::Vector, true, [](BoxDesc& b, Value&& v, const std::string&) { b.min = v.vec; },
       [](const BoxDesc& b) { return vec_json(b.min); }},
      {"max", Kind::Vector, true, [](BoxDesc& b, Value&& v, const std::string&) { b.max = v.vec; },
       [](const BoxDesc& b) { return vec_json(b.max); }},
      {"rotate_y", Kind::Number, false, [](BoxDesc& b, Value&& v, const std::string&) { b.rotate_y = v.num; },
       [](const BoxDesc& b) { return JsonValue(b.rotate_y); }},
  };
  static inline const Rule<BoxDesc> rules[] = {
      finite<BoxDesc>("min", [](const BoxDesc& b) { return b.min; }),
      finite<BoxDesc>("max", [](const BoxDesc& b) { return b.max; }),
      check<BoxDesc>("", "box max must exceed min on every axis",
                     [](const BoxDesc& b) { return b.max.x > b.min.x && b.max.y > b.min.y && b.max.z > b.min.z; }),
  };
};

bool mesh_is(const MeshDesc& m, MeshDesc::Source s) { return m.source == s; }

template <>
struct Schema<MeshDesc> {
  static constexpr const char* names[] = {"mesh"};
  static inline const Field<MeshDesc> fields[] = {
      {"source", Kind::Text, false,
       [](MeshDesc& m, Value&& v, const std::string& at) { m.source = choose(kMeshSources, v.text, at); },
       [](const MeshDesc& m) { return JsonValue(choice_name(kMeshSources, m.source)); }},
      {"subdivisions", Kind::Integer, false, [](MeshDesc& m, Value&& v, const std::string&) { m.subdivisions = v.integer; },
       [](const MeshDesc& m) { return JsonValue(m.subdivisions); }, nullptr,
       [](const MeshDesc& m) { return mesh_is(m, MeshDesc::Source::Icosphere); }},
      {"major_radius", Kind::Number, false, [](MeshDesc& m, Value&& v, const std::string&) { m.major_radius = v.num; },
       [](const MeshDesc& m) { return JsonValue(m.major_radius); }, nullptr,
       [](const MeshDesc& m) { return mesh_is(m, MeshDesc::Source::Torus); }},
      {"minor_radius", Kind::Number, false, [](MeshDesc& m, Value&& v, const std::string&) { m.minor_radius = v.num; },
       [](const MeshDesc& m) { return JsonValue(m.minor_radius); }, nullptr,
       [](const MeshDesc& m) { return mesh_is(m, MeshDesc::Source::Torus); }},
      {"segments", Kind::Integer, false, [](MeshDesc& m, Value&& v, const std::string&) { m.segments = v.integer; },
       [](const MeshDesc& m) { return JsonValue(m.segments); }, nullptr,
       [](const MeshDesc& m) { return mesh_is(m, MeshDesc::Source::Torus); }},
      // Schema extension: the torus's minor segment count (0 keeps segments / 2).
      {"segments_v", Kind::Integer, false, [](MeshDesc& m, Value&& v, const std::string&) { m.segments_v = v.integer; },
       [](const MeshDesc& m) { return JsonValue(m.segments_v); }, nullptr,
       [](const MeshDesc& m) { return mesh_is(m, MeshDesc::Source::Torus) && m.segments_v > 0; }},
      {"path", Kind::Text, false, [](MeshDesc& m, Value&& v, const std::string&) { m.path = std::move(v.text); },
       [](const MeshDesc& m) { return JsonValue(m.path); }, nullptr,
       [](const MeshDesc& m) { return mesh_is(m, MeshDesc::Source::ObjFile); }},
      {"smooth", Kind::Flag, false, [](MeshDesc& m, Value&& v, const std::string&) { m.smooth = v.flag; },
       [](const MeshDesc& m) { return JsonValue(m.smooth); }},
      {"scale", Kind::Vector, false, [](MeshDesc& m, Value&& v, const std::string&) { m.scale = v.vec; },
       [](const MeshDesc& m) { return vec_json(m.scale); }},
      {"rotate_y", Kind::Number, false, [](MeshDesc& m, Value&& v, const std::string&) { m.rotate_y = v.num; },
       [](const MeshDesc& m) { return JsonValue(m.rotate_y); }},
      {"translate", Kind::Vector, false, [](MeshDesc& m, Value&& v, const std::string&) { m.translate = v.vec; },
       [](const MeshDesc& m) { return vec_json(m.translate); }},
  };
  static inline const Rule<MeshDesc> rules[] = {
      check<MeshDesc>("subdivisions", "must be in [0, 7]",
                      [](const MeshDesc& m) { return m.subdivisions >= 0 && m.subdivisions <= 7; }),
      check<MeshDesc>("segments", "must be in [3, 2048]", [](const MeshDesc& m) { return m.segments >= 3 && m.segments <= 2048; }),
      check<MeshDesc>("segments_v", "must be in [3, 2048]",
                      [](const MeshDesc& m) { return m.segments_v == 0 || (m.segments_v >= 3 && m.segments_v <= 2048); }),
      check<MeshDesc>("", "torus radii must be > 0", [](const MeshDesc& m) { return m.major_radius > 0 && m.minor_radius > 0; }),
      check<MeshDesc>("path", "required for obj meshes",
                      [](const MeshDesc& m) { return !(m.source == MeshDesc::Source::ObjFile && m.path.empty()); }),
      finite<MeshDesc>("scale", [](const MeshDesc& m) { return m.scale; }),
      finite<MeshDesc>("translate", [](const MeshDesc& m) { return m.translate; }),
      check<MeshDesc>("scale", "components must be non-zero",
                      [](const MeshDesc& m) { return !(std::fabs(m.scale.x * m.scale.y * m.scale.z) < 1e-12); }),
  };
};

template <class T>
bool named(const std::string& type) {
  for (const char* n : Schema<T>::names)
    if (type == n) return true;
  return false;
}

// Reads the alternative of variant V named `type` (false if none is).
template <class V, std::size_t I = 0>
bool read_kind(const std::string& type, const JsonValue& j, const std::string& at, V& out) {
  if constexpr (I == std::variant_size_v<V>) {
    return false;
  } else {
    using T = std::variant_alternative_t<I, V>;
    if (!named<T>(type)) return read_kind<V, I + 1>(type, j, at, out);
    T rec;
    read_fields<T>(Schema<T>::fields, j, at, rec);
    out = std::move(rec);
    return true;
  }
}

template <class V>
void write_kind(const V& v, JsonValue& j) {
  std::visit([&](const auto& rec) {
    using T = std::decay_t<decltype(rec)>;
    j["type"] = Schema<T>::names[0];
    write_fields<T>(Schema<T>::fields, rec, j);
  }, v);
}

template <class V>
void check_kind(const V& v, const std::string& at, std::vector<std::string>& out) {
  std::visit([&](const auto& rec) {
    using T = std::decay_t<decltype(rec)>;
    apply_rules<T>(Schema<T>::rules, rec, at, out);
  }, v);
}

// ---------------------------------------------------------------------------
// Records with their own framing

Material read_material(const JsonValue& j, const std::string& at) {
  record(j, at);
  const std::string where = field_path(at, "type");
  const JsonValue* t = j.get("type");
  if (!t) reject(where, "required");
  const std::string type = decode(*t, Kind::Text, where).text;
  Material m;
  if (!read_kind(type, j, at, m)) reject(where, "unknown material type '" + type + "'");
  return m;
}

// Objects read type, name and material before their shape's fields, and write
// the material last.
ObjectDesc read_object(const JsonValue& j, const std::string& at) {
  record(j, at);
  auto text = [&](const char* key, bool required, const std::string& fallback) {
    const std::string where = field_path(at, key);
    const JsonValue* v = j.get(key);
    if (!v) {
      if (required) reject(where, "required");
      return fallback;
    }
    return decode(*v, Kind::Text, where).text;
  };
  ObjectDesc o;
  const std::string type = text("type", true, "");
  o.name = text("name", false, type);
  o.material = text("material", true, "");
  if (!read_kind(type, j, at, o.shape)) reject(field_path(at, "type"), "unknown object type '" + type + "'");
  return o;
}

JsonValue write_object(const ObjectDesc& o) {
  JsonValue j;
  std::visit([&](const auto& rec) {
    using T = std::decay_t<decltype(rec)>;
    j["type"] = Schema<T>::names[0];
    j["name"] = o.name;
    write_fields<T>(Schema<T>::fields, rec, j);
  }, o.shape);
  j["material"] = o.material;
  return j;
}

PointLightDesc read_light(const JsonValue& j, const std::string& at, std::size_t index) {
  record(j, at);
  const std::string where = field_path(at, "type");
  if (const JsonValue* t = j.get("type"); t && decode(*t, Kind::Text, where).text != "point")
    reject(where, "only 'point' lights are supported (use emissive materials for area lights)");
  PointLightDesc l;
  l.name = "light" + std::to_string(index);
  read_fields<PointLightDesc>(kLightFields, j, at, l);
  return l;
}

// ---------------------------------------------------------------------------
// Whole-scene validation rules

const Rule<RenderSettings> kRenderRules[] = {
    check<RenderSettings>("width", "must be in [1, 8192]", [](const RenderSettings& r) { return r.width >= 1 && r.width <= 8192; }),
    check<RenderSettings>("height", "must be in [1, 8192]", [](const RenderSettings& r) { return r.height >= 1 && r.height <= 8192; }),
    check<RenderSettings>("spp", "must be in [1, 1000000]", [](const RenderSettings& r) { return r.spp >= 1 && r.spp <= 1'000'000; }),
    check<RenderSettings>("max_depth", "must be in [1, 1000]",
                          [](const RenderSettings& r) { return r.max_depth >= 1 && r.max_depth <= 1000; }),
    check<RenderSettings>("rr_min_depth", "must be >= 0", [](const RenderSettings& r) { return r.rr_min_depth >= 0; }),
    check<RenderSettings>("threads", "must be in [0, 1024]", [](const RenderSettings& r) { return r.threads >= 0 && r.threads <= 1024; }),
    check<RenderSettings>("tile_size", "must be in [1, 1024]",
                          [](const RenderSettings& r) { return r.tile_size >= 1 && r.tile_size <= 1024; }),
    check<RenderSettings>("exposure", "must be > 0", [](const RenderSettings& r) { return finite_positive(r.exposure); }),
};

const Rule<CameraDesc> kCameraRules[] = {
    finite<CameraDesc>("look_from", [](const CameraDesc& c) { return c.look_from; }),
    finite<CameraDesc>("look_at", [](const CameraDesc& c) { return c.look_at; }),
    check<CameraDesc>("", "look_from and look_at must differ",
                      [](const CameraDesc& c) { return !(len(c.look_at - c.look_from) < 1e-9); }),
    check<CameraDesc>("vfov", "must be in (0, 180)", [](const CameraDesc& c) { return c.vfov_deg > 0 && c.vfov_deg < 180; }),
    check<CameraDesc>("aperture", "must be >= 0", [](const CameraDesc& c) { return !(c.aperture < 0); }),
    check<CameraDesc>("focus_dist", "must be >= 0", [](const CameraDesc& c) { return !(c.focus_dist < 0); }),
};

const Rule<Background> kBackgroundRules[] = {
    colour<Background>("top", [](const Background& b) { return b.top; }),
    colour<Background>("bottom", [](const Background& b) { return b.bottom; }),
};

const Rule<PointLightDesc> kLightRules[] = {
    finite<PointLightDesc>("position", [](const PointLightDesc& l) { return l.position; }),
    colour<PointLightDesc>("intensity", [](const PointLightDesc& l) { return l.intensity; }),
};

constexpr const char* kTopLevelKeys[] = {"name", "camera", "render", "background", "materials",
                                         "objects", "lights", "$schema", "description"};

}  // namespace

const char* integrator_name(Integrator i) { return choice_name(kIntegrators, i); }
const char* tone_map_name(ToneMap t) { return choice_name(kToneMaps, t); }

SceneDesc scene_from_json(const JsonValue& root) {
  record(root, "");
  for (const auto& kv : root.map()) {
    bool known = false;
    for (const char* k : kTopLevelKeys) known = known || kv.first == k;
    if (!known) reject("", "unknown top-level key '" + kv.first + "'");
  }
  SceneDesc s;
  if (const JsonValue* v = root.get("name")) s.name = decode(*v, Kind::Text, "name").text;
  if (const JsonValue* v = root.get("camera")) read_fields<CameraDesc>(kCameraFields, record(*v, "camera"), "camera", s.camera);
  if (const JsonValue* v = root.get("render")) read_fields<RenderSettings>(kRenderFields, record(*v, "render"), "render", s.render);
  if (const JsonValue* v = root.get("background"))
    read_fields<Background>(kBackgroundFields, record(*v, "background"), "background", s.background);
  if (const JsonValue* v = root.get("materials")) {
    if (!v->is_map()) reject("materials", "expected an object of name -> material");
    for (const auto& kv : v->map()) s.materials.push_back({kv.first, read_material(kv.second, "materials." + kv.first)});
  }
  if (const JsonValue* v = root.get("objects")) {
    if (!v->is_list()) reject("objects", "expected an array");
    for (std::size_t i = 0; i < v->list().size(); ++i)
      s.objects.push_back(read_object(v->list()[i], "objects[" + std::to_string(i) + "]"));
  }
  if (const JsonValue* v = root.get("lights")) {
    if (!v->is_list()) reject("lights", "expected an array");
    for (std::size_t i = 0; i < v->list().size(); ++i)
      s.lights.push_back(read_light(v->list()[i], "lights[" + std::to_string(i) + "]", i));
  }
  const std::vector<std::string> problems = validate_scene(s);
  if (!problems.empty()) {
    std::string msg = problems.front();
    if (problems.size() > 1) msg += " (and " + std::to_string(problems.size() - 1) + " more problem(s))";
    throw SceneError(msg);
  }
  return s;
}

JsonValue scene_to_json(const SceneDesc& s) {
  JsonValue j;
  j["name"] = s.name;
  write_fields<CameraDesc>(kCameraFields, s.camera, j["camera"]);
  JsonValue& r = j["render"];
  for (const char* key : kRenderWriteOrder)
    for (const Field<RenderSettings>& f : kRenderFields)
      if (std::string(f.key) == key && (!f.written || f.written(s.render))) r[key] = f.get(s.render);
  write_fields<Background>(kBackgroundFields, s.background, j["background"]);
  JsonValue mats = JsonMap{};
  for (const auto& m : s.materials) write_kind(m.material, mats[m.name]);
  j["materials"] = std::move(mats);
  JsonList objs;
  for (const auto& o : s.objects) objs.push_back(write_object(o));
  j["objects"] = std::move(objs);
  JsonList lights;
  for (const auto& l : s.lights) {
    JsonValue lj;
    lj["type"] = "point";
    write_fields<PointLightDesc>(kLightFields, l, lj);
    lights.push_back(std::move(lj));
  }
  j["lights"] = std::move(lights);
  return j;
}

std::vector<std::string> validate_scene(const SceneDesc& s) {
  std::vector<std::string> out;
  apply_rules<RenderSettings>(kRenderRules, s.render, "render", out);
  apply_rules<CameraDesc>(kCameraRules, s.camera, "camera", out);
  apply_rules<Background>(kBackgroundRules, s.background, "background", out);
  for (std::size_t i = 0; i < s.materials.size(); ++i) {
    const std::string at = "materials." + s.materials[i].name;
    if (s.materials[i].name.empty()) out.push_back("materials: material names must be non-empty");
    for (std::size_t k = 0; k < i; ++k)
      if (s.materials[k].name == s.materials[i].name) out.push_back(at + ": duplicate material name");
    check_kind(s.materials[i].material, at, out);
  }
  for (std::size_t i = 0; i < s.objects.size(); ++i) {
    const std::string at = "objects[" + std::to_string(i) + "]";
    if (!s.find_material(s.objects[i].material))
      out.push_back(at + ".material: unknown material '" + s.objects[i].material + "'");
    check_kind(s.objects[i].shape, at, out);
  }
  for (std::size_t i = 0; i < s.lights.size(); ++i)
    apply_rules<PointLightDesc>(kLightRules, s.lights[i], "lights[" + std::to_string(i) + "]", out);
  return out;
}

SceneDesc parse_scene(const std::string& text) {
  try {
    return scene_from_json(JsonValue::parse(text));
  } catch (const JsonError& e) {
    throw SceneError(e.what());
  }
}

SceneDesc load_scene(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw SceneError("cannot open scene file: " + path);
  std::stringstream text;
  text << f.rdbuf();
  SceneDesc s = parse_scene(text.str());
  s.base_dir = std::filesystem::path(path).parent_path().string();
  return s;
}

}  // namespace rtg
