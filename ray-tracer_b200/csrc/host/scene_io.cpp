#include "host/scene_io.hpp"

#include <cmath>
#include <filesystem>
#include <fstream>
#include <sstream>

namespace rtg {

const char* integrator_name(Integrator i) {
  switch (i) {
    case Integrator::Direct: return "direct";
    case Integrator::Normals: return "normals";
    default: return "path";
  }
}
const char* tone_map_name(ToneMap t) {
  switch (t) {
    case ToneMap::Clamp: return "clamp";
    case ToneMap::Reinhard: return "reinhard";
    default: return "aces";
  }
}

namespace {

// Typed field access on one JSON object; errors carry the dotted field path.
class Fields {
 public:
  Fields(const JsonValue& v, std::string where) : v_(v), where_(std::move(where)) {
    if (!v_.is_map()) throw SceneError((where_.empty() ? std::string("scene") : where_) + ": expected an object");
  }
  std::string path(const std::string& key) const { return where_.empty() ? key : where_ + "." + key; }
  const JsonValue* find(const std::string& key) const { return v_.get(key); }

  double num(const std::string& key, double fallback) const {
    const JsonValue* f = find(key);
    if (!f) return fallback;
    if (!f->is_number()) throw SceneError(path(key) + ": expected a number");
    return f->number();
  }
  int integer(const std::string& key, int fallback) const {
    const JsonValue* f = find(key);
    if (!f) return fallback;
    if (!f->is_number()) throw SceneError(path(key) + ": expected an integer");
    const double d = f->number();
    if (d != std::floor(d) || std::fabs(d) > 2e9) throw SceneError(path(key) + ": expected an integer");
    return static_cast<int>(d);
  }
  bool flag(const std::string& key, bool fallback) const {
    const JsonValue* f = find(key);
    if (!f) return fallback;
    if (!f->is_bool()) throw SceneError(path(key) + ": expected true/false");
    return f->boolean();
  }
  std::string text(const std::string& key, const std::string& fallback) const {
    const JsonValue* f = find(key);
    if (!f) return fallback;
    if (!f->is_string()) throw SceneError(path(key) + ": expected a string");
    return f->str();
  }
  std::string required_text(const std::string& key) const {
    if (!find(key)) throw SceneError(path(key) + ": required");
    return text(key, "");
  }
  // [x, y, z], or a scalar s meaning [s, s, s].
  D3 vec(const std::string& key, D3 fallback) const {
    const JsonValue* f = find(key);
    if (!f) return fallback;
    if (f->is_number()) return D3{f->number()};
    if (!f->is_list() || f->list().size() != 3) throw SceneError(path(key) + ": expected [x, y, z]");
    D3 out;
    for (int i = 0; i < 3; ++i) {
      const JsonValue& e = f->list()[static_cast<std::size_t>(i)];
      if (!e.is_number()) throw SceneError(path(key) + ": expected [x, y, z] of numbers");
      out.at(i) = e.number();
    }
    return out;
  }
  D3 required_vec(const std::string& key) const {
    if (!find(key)) throw SceneError(path(key) + ": required");
    return vec(key, {});
  }

 private:
  const JsonValue& v_;
  std::string where_;
};

JsonValue vjson(D3 v) { return JsonList{v.x, v.y, v.z}; }

Material material_from(const Fields& f) {
  const std::string type = f.required_text("type");
  if (type == "lambertian" || type == "diffuse") {
    Lambertian m;
    m.albedo.a = f.vec("albedo", D3{0.5});
    m.albedo.b = f.vec("albedo2", m.albedo.a);
    m.albedo.checker_scale = f.num("checker_scale", 0);
    return m;
  }
  if (type == "metal") return Metal{f.vec("albedo", D3{0.9}), f.num("roughness", 0)};
  if (type == "dielectric" || type == "glass") return Dielectric{f.num("ior", 1.5), f.vec("tint", D3{1})};
  if (type == "emissive" || type == "light")
    return Emissive{f.vec("color", D3{1}), f.num("intensity", 1), f.flag("two_sided", false)};
  throw SceneError(f.path("type") + ": unknown material type '" + type + "'");
}

JsonValue material_to(const Material& m) {
  JsonValue j;
  if (const auto* l = std::get_if<Lambertian>(&m)) {
    j["type"] = "lambertian";
    j["albedo"] = vjson(l->albedo.a);
    if (l->albedo.checker_scale > 0) {
      j["albedo2"] = vjson(l->albedo.b);
      j["checker_scale"] = l->albedo.checker_scale;
    }
  } else if (const auto* me = std::get_if<Metal>(&m)) {
    j["type"] = "metal";
    j["albedo"] = vjson(me->albedo);
    j["roughness"] = me->roughness;
  } else if (const auto* d = std::get_if<Dielectric>(&m)) {
    j["type"] = "dielectric";
    j["ior"] = d->ior;
    j["tint"] = vjson(d->tint);
  } else {
    const auto& e = std::get<Emissive>(m);
    j["type"] = "emissive";
    j["color"] = vjson(e.color);
    j["intensity"] = e.intensity;
    if (e.two_sided) j["two_sided"] = true;
  }
  return j;
}

ObjectDesc object_from(const Fields& f) {
  ObjectDesc o;
  const std::string type = f.required_text("type");
  o.name = f.text("name", type);
  o.material = f.required_text("material");
  if (type == "sphere") {
    o.shape = SphereDesc{f.required_vec("center"), f.num("radius", 1)};
  } else if (type == "plane") {
    o.shape = PlaneDesc{f.vec("point", {}), f.vec("normal", {0, 1, 0})};
  } else if (type == "triangle") {
    o.shape = TriangleDesc{f.required_vec("v0"), f.required_vec("v1"), f.required_vec("v2")};
  } else if (type == "quad") {
    o.shape = QuadDesc{f.required_vec("corner"), f.required_vec("u"), f.required_vec("v")};
  } else if (type == "box") {
    o.shape = BoxDesc{f.required_vec("min"), f.required_vec("max"), f.num("rotate_y", 0)};
  } else if (type == "mesh") {
    MeshDesc m;
    const std::string src = f.text("source", "icosphere");
    if (src == "icosphere") m.source = MeshDesc::Source::Icosphere;
    else if (src == "torus") m.source = MeshDesc::Source::Torus;
    else if (src == "obj") m.source = MeshDesc::Source::ObjFile;
    else throw SceneError(f.path("source") + ": expected icosphere, torus or obj");
    m.subdivisions = f.integer("subdivisions", m.subdivisions);
    m.major_radius = f.num("major_radius", m.major_radius);
    m.minor_radius = f.num("minor_radius", m.minor_radius);
    m.segments = f.integer("segments", m.segments);
    m.segments_v = f.integer("segments_v", 0);
    m.path = f.text("path", "");
    m.smooth = f.flag("smooth", true);
    m.scale = f.vec("scale", {1, 1, 1});
    m.rotate_y = f.num("rotate_y", 0);
    m.translate = f.vec("translate", {0, 0, 0});
    o.shape = m;
  } else {
    throw SceneError(f.path("type") + ": unknown object type '" + type + "'");
  }
  return o;
}

JsonValue object_to(const ObjectDesc& o) {
  JsonValue j;
  if (const auto* s = std::get_if<SphereDesc>(&o.shape)) {
    j["type"] = "sphere"; j["name"] = o.name; j["center"] = vjson(s->center); j["radius"] = s->radius;
  } else if (const auto* p = std::get_if<PlaneDesc>(&o.shape)) {
    j["type"] = "plane"; j["name"] = o.name; j["point"] = vjson(p->point); j["normal"] = vjson(p->normal);
  } else if (const auto* t = std::get_if<TriangleDesc>(&o.shape)) {
    j["type"] = "triangle"; j["name"] = o.name;
    j["v0"] = vjson(t->v0); j["v1"] = vjson(t->v1); j["v2"] = vjson(t->v2);
  } else if (const auto* q = std::get_if<QuadDesc>(&o.shape)) {
    j["type"] = "quad"; j["name"] = o.name;
    j["corner"] = vjson(q->corner); j["u"] = vjson(q->u); j["v"] = vjson(q->v);
  } else if (const auto* b = std::get_if<BoxDesc>(&o.shape)) {
    j["type"] = "box"; j["name"] = o.name;
    j["min"] = vjson(b->min); j["max"] = vjson(b->max); j["rotate_y"] = b->rotate_y;
  } else {
    const auto& m = std::get<MeshDesc>(o.shape);
    j["type"] = "mesh"; j["name"] = o.name;
    if (m.source == MeshDesc::Source::Icosphere) {
      j["source"] = "icosphere"; j["subdivisions"] = m.subdivisions;
    } else if (m.source == MeshDesc::Source::Torus) {
      j["source"] = "torus"; j["major_radius"] = m.major_radius; j["minor_radius"] = m.minor_radius;
      j["segments"] = m.segments;
      if (m.segments_v > 0) j["segments_v"] = m.segments_v;
    } else {
      j["source"] = "obj"; j["path"] = m.path;
    }
    j["smooth"] = m.smooth;
    j["scale"] = vjson(m.scale);
    j["rotate_y"] = m.rotate_y;
    j["translate"] = vjson(m.translate);
  }
  j["material"] = o.material;
  return j;
}

}  // namespace

SceneDesc scene_from_json(const JsonValue& root) {
  SceneDesc s;
  const Fields top(root, "");
  static const char* const kTopKeys[] = {"name", "camera", "render", "background", "materials",
                                         "objects", "lights", "$schema", "description"};
  for (const auto& kv : root.map()) {
    bool known = false;
    for (const char* k : kTopKeys) known = known || kv.first == k;
    if (!known) throw SceneError("scene: unknown top-level key '" + kv.first + "'");
  }
  s.name = top.text("name", s.name);

  if (const JsonValue* cj = top.find("camera")) {
    const Fields c(*cj, "camera");
    s.camera.look_from = c.vec("look_from", s.camera.look_from);
    s.camera.look_at = c.vec("look_at", s.camera.look_at);
    s.camera.vup = c.vec("vup", s.camera.vup);
    s.camera.vfov_deg = c.num("vfov", s.camera.vfov_deg);
    s.camera.aperture = c.num("aperture", 0);
    s.camera.focus_dist = c.num("focus_dist", 0);
  }

  if (const JsonValue* rj = top.find("render")) {
    const Fields c(*rj, "render");
    RenderSettings& R = s.render;
    R.width = c.integer("width", R.width);
    R.height = c.integer("height", R.height);
    R.spp = c.integer("spp", R.spp);
    R.max_depth = c.integer("max_depth", R.max_depth);
    R.rr_min_depth = c.integer("rr_min_depth", R.rr_min_depth);
    R.light_sampling = c.flag("light_sampling", R.light_sampling);
    R.mis = c.flag("mis", R.mis);  // schema extension (no reference counterpart)
    // The seed goes through a 32-bit integer read, as in the reference loader.
    R.seed = static_cast<std::uint64_t>(c.integer("seed", static_cast<int>(R.seed)));
    R.exposure = c.num("exposure", R.exposure);
    R.threads = c.integer("threads", R.threads);
    R.tile_size = c.integer("tile_size", R.tile_size);
    R.use_bvh = c.flag("use_bvh", R.use_bvh);
    const std::string integ = c.text("integrator", integrator_name(R.integrator));
    if (integ == "path") R.integrator = Integrator::Path;
    else if (integ == "direct") R.integrator = Integrator::Direct;
    else if (integ == "normals") R.integrator = Integrator::Normals;
    else throw SceneError("render.integrator: expected path, direct or normals");
    const std::string tm = c.text("tone_map", tone_map_name(R.tone_map));
    if (tm == "clamp") R.tone_map = ToneMap::Clamp;
    else if (tm == "reinhard") R.tone_map = ToneMap::Reinhard;
    else if (tm == "aces") R.tone_map = ToneMap::Aces;
    else throw SceneError("render.tone_map: expected clamp, reinhard or aces");
  }

  if (const JsonValue* bj = top.find("background")) {
    const Fields b(*bj, "background");
    const std::string kind = b.text("type", "gradient");
    if (kind == "gradient") s.background.kind = Background::Kind::Gradient;
    else if (kind == "solid") s.background.kind = Background::Kind::Solid;
    else throw SceneError("background.type: expected gradient or solid");
    s.background.top = b.vec(kind == "solid" ? "color" : "top", s.background.top);
    s.background.bottom = b.vec("bottom", s.background.bottom);
    s.background.intensity = b.num("intensity", 1);
  }

  if (const JsonValue* mj = top.find("materials")) {
    if (!mj->is_map()) throw SceneError("materials: expected an object of name -> material");
    for (const auto& kv : mj->map())
      s.materials.push_back({kv.first, material_from(Fields(kv.second, "materials." + kv.first))});
  }

  if (const JsonValue* oj = top.find("objects")) {
    if (!oj->is_list()) throw SceneError("objects: expected an array");
    const auto& l = oj->list();
    for (std::size_t i = 0; i < l.size(); ++i)
      s.objects.push_back(object_from(Fields(l[i], "objects[" + std::to_string(i) + "]")));
  }

  if (const JsonValue* lj = top.find("lights")) {
    if (!lj->is_list()) throw SceneError("lights: expected an array");
    const auto& l = lj->list();
    for (std::size_t i = 0; i < l.size(); ++i) {
      const Fields f(l[i], "lights[" + std::to_string(i) + "]");
      if (f.text("type", "point") != "point")
        throw SceneError(f.path("type") + ": only 'point' lights are supported (use emissive materials for area lights)");
      s.lights.push_back({f.text("name", "light" + std::to_string(i)), f.required_vec("position"),
                          f.vec("intensity", D3{10})});
    }
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
  JsonValue& c = j["camera"];
  c["look_from"] = vjson(s.camera.look_from);
  c["look_at"] = vjson(s.camera.look_at);
  c["vup"] = vjson(s.camera.vup);
  c["vfov"] = s.camera.vfov_deg;
  c["aperture"] = s.camera.aperture;
  c["focus_dist"] = s.camera.focus_dist;

  JsonValue& r = j["render"];
  const RenderSettings& R = s.render;
  r["width"] = R.width;
  r["height"] = R.height;
  r["spp"] = R.spp;
  r["max_depth"] = R.max_depth;
  r["rr_min_depth"] = R.rr_min_depth;
  r["integrator"] = integrator_name(R.integrator);
  r["light_sampling"] = R.light_sampling;
  if (R.mis) r["mis"] = true;
  r["seed"] = R.seed;
  r["tone_map"] = tone_map_name(R.tone_map);
  r["exposure"] = R.exposure;
  r["threads"] = R.threads;
  r["tile_size"] = R.tile_size;
  r["use_bvh"] = R.use_bvh;

  JsonValue& b = j["background"];
  if (s.background.kind == Background::Kind::Solid) {
    b["type"] = "solid";
    b["color"] = vjson(s.background.top);
  } else {
    b["type"] = "gradient";
    b["top"] = vjson(s.background.top);
    b["bottom"] = vjson(s.background.bottom);
  }
  b["intensity"] = s.background.intensity;

  JsonValue mats = JsonMap{};
  for (const auto& m : s.materials) mats[m.name] = material_to(m.material);
  j["materials"] = std::move(mats);

  JsonList objs;
  for (const auto& o : s.objects) objs.push_back(object_to(o));
  j["objects"] = std::move(objs);

  JsonList lights;
  for (const auto& l : s.lights) {
    JsonValue lj;
    lj["type"] = "point";
    lj["name"] = l.name;
    lj["position"] = vjson(l.position);
    lj["intensity"] = vjson(l.intensity);
    lights.push_back(std::move(lj));
  }
  j["lights"] = std::move(lights);
  return j;
}

std::vector<std::string> validate_scene(const SceneDesc& s) {
  std::vector<std::string> out;
  auto finite = [&](D3 v, const std::string& where) {
    if (!v.finite()) out.push_back(where + ": must be finite");
  };
  auto colour = [&](D3 v, const std::string& where) {
    finite(v, where);
    if (v.x < 0 || v.y < 0 || v.z < 0) out.push_back(where + ": colour components must be >= 0");
  };
  const RenderSettings& R = s.render;
  if (R.width < 1 || R.width > 8192) out.push_back("render.width: must be in [1, 8192]");
  if (R.height < 1 || R.height > 8192) out.push_back("render.height: must be in [1, 8192]");
  if (R.spp < 1 || R.spp > 1'000'000) out.push_back("render.spp: must be in [1, 1000000]");
  if (R.max_depth < 1 || R.max_depth > 1000) out.push_back("render.max_depth: must be in [1, 1000]");
  if (R.rr_min_depth < 0) out.push_back("render.rr_min_depth: must be >= 0");
  if (R.threads < 0 || R.threads > 1024) out.push_back("render.threads: must be in [0, 1024]");
  if (R.tile_size < 1 || R.tile_size > 1024) out.push_back("render.tile_size: must be in [1, 1024]");
  if (!(R.exposure > 0) || !std::isfinite(R.exposure)) out.push_back("render.exposure: must be > 0");

  finite(s.camera.look_from, "camera.look_from");
  finite(s.camera.look_at, "camera.look_at");
  if (len(s.camera.look_at - s.camera.look_from) < 1e-9) out.push_back("camera: look_from and look_at must differ");
  if (!(s.camera.vfov_deg > 0 && s.camera.vfov_deg < 180)) out.push_back("camera.vfov: must be in (0, 180)");
  if (s.camera.aperture < 0) out.push_back("camera.aperture: must be >= 0");
  if (s.camera.focus_dist < 0) out.push_back("camera.focus_dist: must be >= 0");
  colour(s.background.top, "background.top");
  colour(s.background.bottom, "background.bottom");

  for (std::size_t i = 0; i < s.materials.size(); ++i) {
    const NamedMaterial& nm = s.materials[i];
    const std::string at = "materials." + nm.name;
    if (nm.name.empty()) out.push_back("materials: material names must be non-empty");
    for (std::size_t k = 0; k < i; ++k)
      if (s.materials[k].name == nm.name) out.push_back(at + ": duplicate material name");
    if (const auto* l = std::get_if<Lambertian>(&nm.material)) {
      colour(l->albedo.a, at + ".albedo");
      colour(l->albedo.b, at + ".albedo2");
      if (l->albedo.checker_scale < 0) out.push_back(at + ".checker_scale: must be >= 0");
    } else if (const auto* m = std::get_if<Metal>(&nm.material)) {
      colour(m->albedo, at + ".albedo");
      if (m->roughness < 0 || m->roughness > 1) out.push_back(at + ".roughness: must be in [0, 1]");
    } else if (const auto* d = std::get_if<Dielectric>(&nm.material)) {
      if (!(d->ior >= 1.0 && d->ior <= 4.0)) out.push_back(at + ".ior: must be in [1, 4]");
      colour(d->tint, at + ".tint");
    } else {
      const auto& e = std::get<Emissive>(nm.material);
      colour(e.color, at + ".color");
      if (!(e.intensity >= 0) || !std::isfinite(e.intensity)) out.push_back(at + ".intensity: must be >= 0");
    }
  }

  for (std::size_t i = 0; i < s.objects.size(); ++i) {
    const ObjectDesc& o = s.objects[i];
    const std::string at = "objects[" + std::to_string(i) + "]";
    if (!s.find_material(o.material)) out.push_back(at + ".material: unknown material '" + o.material + "'");
    if (const auto* sp = std::get_if<SphereDesc>(&o.shape)) {
      finite(sp->center, at + ".center");
      if (!(sp->radius > 0) || !std::isfinite(sp->radius)) out.push_back(at + ".radius: must be > 0");
    } else if (const auto* pl = std::get_if<PlaneDesc>(&o.shape)) {
      finite(pl->point, at + ".point");
      finite(pl->normal, at + ".normal");
      if (len(pl->normal) < 1e-9) out.push_back(at + ".normal: must be non-zero");
    } else if (const auto* t = std::get_if<TriangleDesc>(&o.shape)) {
      finite(t->v0, at + ".v0");
      finite(t->v1, at + ".v1");
      finite(t->v2, at + ".v2");
      if (len(cross(t->v1 - t->v0, t->v2 - t->v0)) < 1e-12) out.push_back(at + ": triangle is degenerate");
    } else if (const auto* q = std::get_if<QuadDesc>(&o.shape)) {
      finite(q->corner, at + ".corner");
      finite(q->u, at + ".u");
      finite(q->v, at + ".v");
      if (len(cross(q->u, q->v)) < 1e-12) out.push_back(at + ": quad is degenerate (u parallel to v)");
    } else if (const auto* b = std::get_if<BoxDesc>(&o.shape)) {
      finite(b->min, at + ".min");
      finite(b->max, at + ".max");
      if (!(b->max.x > b->min.x && b->max.y > b->min.y && b->max.z > b->min.z))
        out.push_back(at + ": box max must exceed min on every axis");
    } else {
      const auto& m = std::get<MeshDesc>(o.shape);
      if (m.subdivisions < 0 || m.subdivisions > 7) out.push_back(at + ".subdivisions: must be in [0, 7]");
      if (m.segments < 3 || m.segments > 2048) out.push_back(at + ".segments: must be in [3, 2048]");
      if (m.segments_v != 0 && (m.segments_v < 3 || m.segments_v > 2048))
        out.push_back(at + ".segments_v: must be in [3, 2048]");
      if (!(m.major_radius > 0) || !(m.minor_radius > 0)) out.push_back(at + ": torus radii must be > 0");
      if (m.source == MeshDesc::Source::ObjFile && m.path.empty()) out.push_back(at + ".path: required for obj meshes");
      finite(m.scale, at + ".scale");
      finite(m.translate, at + ".translate");
      if (std::fabs(m.scale.x * m.scale.y * m.scale.z) < 1e-12) out.push_back(at + ".scale: components must be non-zero");
    }
  }

  for (std::size_t i = 0; i < s.lights.size(); ++i) {
    finite(s.lights[i].position, "lights[" + std::to_string(i) + "].position");
    colour(s.lights[i].intensity, "lights[" + std::to_string(i) + "].intensity");
  }
  return out;
}

SceneDesc parse_scene(const std::string& text) {
  JsonValue j;
  try {
    j = JsonValue::parse(text);
  } catch (const JsonError& e) {
    throw SceneError(e.what());
  }
  try {
    return scene_from_json(j);
  } catch (const JsonError& e) {
    throw SceneError(e.what());
  }
}

SceneDesc load_scene(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw SceneError("cannot open scene file: " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  SceneDesc s = parse_scene(ss.str());
  s.base_dir = std::filesystem::path(path).parent_path().string();
  return s;
}

}  // namespace rtg
