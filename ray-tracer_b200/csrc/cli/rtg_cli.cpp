// rtg — GPU command-line renderer with the reference CLI's flags, exit codes and
// streaming protocol (apps/rt_cli.cpp:1-209), written against the C ABI (rtg.h):
//
//   rtg scene.json -o out.png [overrides...]
//   rtg - --stream < scene.json        (scene on stdin, progressive frames on stdout)
//
// Streaming protocol on stdout:
//   FRAME <json header>\n<png bytes>     one per progressive pass; header has "bytes"
//   DONE <json stats>\n                  render finished or was cancelled
//   ERROR <json {"message": ...}>\n      scene could not be loaded/validated
// Exit codes: 0 done, 1 usage, 2 scene error, 3 output error, 130 cancelled.
#include <atomic>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <optional>
#include <sstream>
#include <string>
#include <vector>

#include "rtg.h"

namespace {

volatile std::int32_t g_cancel = 0;
extern "C" void on_signal(int) { g_cancel = 1; }

void usage() {
  std::cerr << "usage: rtg <scene.json | -> [options]\n"
               "  -o, --output FILE      output image (.png or .ppm), default render.png\n"
               "  --width N --height N   override resolution\n"
               "  --spp N                samples per pixel\n"
               "  --max-depth N          maximum bounces\n"
               "  --integrator NAME      path | direct | normals\n"
               "  --threads N            accepted for compatibility (ignored on the GPU)\n"
               "  --tile N               accepted for compatibility (ignored on the GPU)\n"
               "  --seed N               RNG seed\n"
               "  --exposure X           exposure multiplier\n"
               "  --no-bvh               brute-force intersection (reference)\n"
               "  --gpu-bvh              build the BVH on the GPU instead of the host (same tree)\n"
               "  --no-light-sampling    disable next-event estimation\n"
               "  --mis                  weight NEE and BSDF sampling by multiple importance sampling\n"
               "  --single-pass          render all samples in one pass\n"
               "  --max-pass N           cap samples per progressive pass (default 32)\n"
               "  --stream               write progressive PNG frames to stdout\n"
               "  --save-every-pass      rewrite the output image after every pass\n"
               "  --snapshot-dir DIR     also save each pass as DIR/spp_NNNNN.png\n"
               "  --validate             only parse + validate the scene\n"
               "  --dump-scene           print the normalised scene JSON and exit\n"
               "  --device N             CUDA device (default 0)\n"
               "  -q, --quiet            no progress output\n";
}

std::string json_str(const std::string& s) {
  std::string o = "\"";
  for (const unsigned char c : s) {
    if (c == '"') o += "\\\"";
    else if (c == '\\') o += "\\\\";
    else if (c == '\n') o += "\\n";
    else if (c < 0x20) {
      char b[8];
      std::snprintf(b, sizeof b, "\\u%04x", c);
      o += b;
    } else o.push_back(static_cast<char>(c));
  }
  return o + "\"";
}

bool ends_with(const std::string& s, const char* suf) {
  const std::size_t n = std::strlen(suf);
  return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

std::vector<std::uint8_t> png_of(const std::vector<std::uint8_t>& rgb, int w, int h) {
  const std::int64_t n = rtg_encode_png(rgb.data(), w, h, nullptr, 0);
  std::vector<std::uint8_t> out(n > 0 ? static_cast<std::size_t>(n) : 0);
  if (n > 0) rtg_encode_png(rgb.data(), w, h, out.data(), out.size());
  return out;
}

bool write_image(const std::string& path, const std::vector<std::uint8_t>& rgb, int w, int h) {
  std::ofstream f(path, std::ios::binary);
  if (!f) return false;
  if (ends_with(path, ".ppm")) {
    f << "P6\n" << w << ' ' << h << "\n255\n";
    f.write(reinterpret_cast<const char*>(rgb.data()), static_cast<std::streamsize>(rgb.size()));
  } else if (ends_with(path, ".png")) {
    const auto png = png_of(rgb, w, h);
    f.write(reinterpret_cast<const char*>(png.data()), static_cast<std::streamsize>(png.size()));
  } else {
    return false;
  }
  return static_cast<bool>(f);
}

struct PassState {
  rtg_context* ctx;
  int width, height;
  bool stream, quiet, save_every;
  std::string output, snapshot_dir;
  bool write_failed = false;
};

void on_pass(void* user, const rtg_progress* p) {
  auto* st = static_cast<PassState*>(user);
  std::vector<std::uint8_t> rgb(static_cast<std::size_t>(st->width) * st->height * 3);
  const bool need_image = st->stream || st->save_every || (!st->snapshot_dir.empty() && !p->cancelled);
  if (need_image) rtg_image_rgb8(st->ctx, -1, -1, 1.0, rgb.data());
  if (st->stream) {
    const auto png = png_of(rgb, st->width, st->height);
    char hdr[512];
    std::snprintf(hdr, sizeof hdr,
                  "FRAME {\"pass\":%d,\"spp_done\":%u,\"spp_target\":%d,\"elapsed_ms\":%f,\"rays\":%llu,\"width\":%d,"
                  "\"height\":%d,\"finished\":%s,\"cancelled\":%s,\"bytes\":%zu}\n",
                  p->pass, p->spp_done, p->spp_target, p->elapsed_ms, static_cast<unsigned long long>(p->rays),
                  st->width, st->height, p->finished ? "true" : "false", p->cancelled ? "true" : "false", png.size());
    std::fwrite(hdr, 1, std::strlen(hdr), stdout);
    std::fwrite(png.data(), 1, png.size(), stdout);
    std::fflush(stdout);
  }
  if (st->save_every && !write_image(st->output, rgb, st->width, st->height)) st->write_failed = true;
  if (!st->snapshot_dir.empty() && !p->cancelled) {
    char name[40];
    std::snprintf(name, sizeof name, "/spp_%05u.png", p->spp_done);
    write_image(st->snapshot_dir + name, rgb, st->width, st->height);
  }
  if (!st->quiet)
    std::cerr << "\r  pass " << p->pass << ": " << p->spp_done << "/" << p->spp_target << " spp, "
              << static_cast<long>(p->elapsed_ms) << " ms" << std::flush;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    usage();
    return 1;
  }
  std::string scene_path, output = "render.png", snapshot_dir;
  std::optional<int> width, height, spp, max_depth, max_pass;
  std::optional<long long> seed;
  std::optional<double> exposure;
  std::optional<std::string> integrator;
  bool no_bvh = false, gpu_bvh = false, no_nee = false, mis = false, single_pass = false, stream = false, quiet = false;
  bool validate_only = false, dump = false, save_every = false;
  int device = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) {
        std::cerr << "missing value for " << a << "\n";
        std::exit(1);
      }
      return argv[++i];
    };
    auto next_int = [&]() {
      const std::string v = next();
      try {
        return std::stoi(v);
      } catch (...) {
        std::cerr << "invalid integer for " << a << ": " << v << "\n";
        std::exit(1);
      }
    };
    if (a == "-o" || a == "--output") output = next();
    else if (a == "--width") width = next_int();
    else if (a == "--height") height = next_int();
    else if (a == "--spp") spp = next_int();
    else if (a == "--max-depth") max_depth = next_int();
    else if (a == "--threads" || a == "--tile") (void)next_int();
    else if (a == "--max-pass") max_pass = next_int();
    else if (a == "--seed") seed = next_int();
    else if (a == "--exposure") exposure = std::stod(next());
    else if (a == "--integrator") integrator = next();
    else if (a == "--device") device = next_int();
    else if (a == "--no-bvh") no_bvh = true;
    else if (a == "--gpu-bvh") gpu_bvh = true;
    else if (a == "--no-light-sampling") no_nee = true;
    else if (a == "--mis") mis = true;
    else if (a == "--single-pass") single_pass = true;
    else if (a == "--stream") stream = true;
    else if (a == "--save-every-pass") save_every = true;
    else if (a == "--snapshot-dir") snapshot_dir = next();
    else if (a == "--validate") validate_only = true;
    else if (a == "--dump-scene") dump = true;
    else if (a == "-q" || a == "--quiet") quiet = true;
    else if (a == "-h" || a == "--help") {
      usage();
      return 0;
    } else if (!a.empty() && a[0] == '-' && a != "-") {
      std::cerr << "unknown option " << a << "\n";
      usage();
      return 1;
    } else scene_path = a;
  }
  if (scene_path.empty()) {
    usage();
    return 1;
  }
  std::signal(SIGINT, on_signal);
  std::signal(SIGTERM, on_signal);

  auto scene_error = [&](const std::string& msg) {
    if (stream) std::cout << "ERROR {\"message\":" << json_str(msg) << "}\n" << std::flush;
    std::cerr << "error: " << msg << "\n";
    return 2;
  };

  std::string text, base_dir;
  if (scene_path == "-") {
    text.assign(std::istreambuf_iterator<char>(std::cin), std::istreambuf_iterator<char>());
  } else {
    std::ifstream f(scene_path, std::ios::binary);
    if (!f) return scene_error("cannot open scene file: " + scene_path);
    std::stringstream ss;
    ss << f.rdbuf();
    text = ss.str();
    const auto slash = scene_path.find_last_of('/');
    base_dir = slash == std::string::npos ? "" : scene_path.substr(0, slash);
  }

  char err[1024] = {0};
  rtg_host_scene* host = nullptr;
  // The tree is built where it is faster (host for small scenes, GPU for large);
  // --gpu-bvh always builds it on the GPU.
  if (rtg_compile_flags(text.c_str(), base_dir.c_str(), gpu_bvh ? RTG_COMPILE_DEFER_BVH : RTG_COMPILE_AUTO_BVH, &host,
                        err, sizeof err) != RTG_OK)
    return scene_error(err);
  rtg_scene_view view{};
  rtg_host_scene_view(host, &view);
  rtg_settings s = view.settings;
  if (width) s.width = *width;
  if (height) s.height = *height;
  if (spp) s.spp = *spp;
  if (max_depth) s.max_depth = *max_depth;
  if (seed) s.seed = static_cast<std::uint64_t>(*seed);
  if (exposure) s.exposure = *exposure;
  if (no_bvh) s.use_bvh = 0;
  if (mis && s.light_sampling) s.light_sampling = 2;
  if (no_nee) s.light_sampling = 0;
  if (integrator) {
    if (*integrator == "path") s.integrator = 0;
    else if (*integrator == "direct") s.integrator = 1;
    else if (*integrator == "normals") s.integrator = 2;
    else {
      rtg_host_scene_free(host);
      return scene_error("--integrator: expected path, direct or normals");
    }
  }
  if (dump) {
    const std::int64_t n = rtg_scene_dump(text.c_str(), nullptr, 0);
    std::string out(static_cast<std::size_t>(n > 0 ? n : 0) + 1, '\0');
    rtg_scene_dump(text.c_str(), out.data(), out.size());
    std::cout << out.c_str() << "\n";
    rtg_host_scene_free(host);
    return 0;
  }
  if (validate_only) {
    std::cerr << "scene OK: " << view.n_prims << " primitives, " << view.n_planes << " planes\n";
    rtg_host_scene_free(host);
    return 0;
  }

  rtg_context* ctx = nullptr;
  if (rtg_context_create(device, &ctx) != RTG_OK) {
    rtg_host_scene_free(host);
    std::cerr << "error: no usable CUDA device\n";
    return 2;
  }
  rtg_scene_id sid = 0;
  if ((gpu_bvh ? rtg_scene_upload_gpu_bvh(ctx, host, &sid) : rtg_scene_upload(ctx, host, &sid)) != RTG_OK) {
    const std::string msg = rtg_last_error(ctx);
    rtg_context_destroy(ctx);
    rtg_host_scene_free(host);
    return scene_error(msg);
  }
  if (!quiet) {
    rtg_scene_info info{};
    rtg_scene_get_info(ctx, sid, &info);
    std::cerr << "scene: " << info.spheres << " spheres, " << info.triangles << " triangles, " << info.planes
              << " planes, " << info.lights << " lights\nBVH: " << info.bvh_nodes << " nodes, depth "
              << info.bvh_max_depth << ", built in " << info.bvh_build_ms << " ms\n"
              << "rendering " << s.width << "x" << s.height << " @ " << s.spp << " spp on GPU " << device << "\n";
  }
  rtg_render_options opts{single_pass ? 0 : 1, max_pass ? *max_pass : 32};
  PassState st{ctx, s.width, s.height, stream, quiet, save_every, output, snapshot_dir};
  rtg_progress fin{};
  if (rtg_render(ctx, sid, &s, &opts, on_pass, &st, &g_cancel, &fin) != RTG_OK) {
    const std::string msg = rtg_last_error(ctx);
    rtg_context_destroy(ctx);
    rtg_host_scene_free(host);
    return scene_error(msg);
  }
  if (!quiet) std::cerr << "\n";

  int code = fin.cancelled ? 130 : 0;
  std::vector<std::uint8_t> rgb(static_cast<std::size_t>(s.width) * s.height * 3);
  rtg_image_rgb8(ctx, -1, -1, 1.0, rgb.data());
  if (!stream || output != "render.png") {
    if (!write_image(output, rgb, s.width, s.height) || st.write_failed) {
      std::cerr << "error: cannot write " << output << " (use .png or .ppm)\n";
      code = 3;
    }
  }
  rtg_stats stats{};
  rtg_render_stats(ctx, &stats);
  const double mrays = stats.elapsed_ms > 0 ? (double(stats.rays + stats.shadow_rays) / 1e3) / stats.elapsed_ms : 0;
  char done[512];
  std::snprintf(done, sizeof done,
                "{\"cancelled\":%s,\"spp_done\":%u,\"elapsed_ms\":%f,\"rays\":%llu,\"shadow_rays\":%llu,"
                "\"mrays_per_sec\":%f,\"invalid_samples\":%llu,\"device\":%d}",
                fin.cancelled ? "true" : "false", fin.spp_done, stats.elapsed_ms,
                static_cast<unsigned long long>(stats.rays), static_cast<unsigned long long>(stats.shadow_rays), mrays,
                static_cast<unsigned long long>(stats.invalid_samples), device);
  if (stream) std::cout << "DONE " << done << "\n" << std::flush;
  if (!quiet)
    std::cerr << (fin.cancelled ? "cancelled" : "done") << " in " << stats.elapsed_ms << " ms, "
              << (stats.rays + stats.shadow_rays) << " rays (" << mrays << " Mrays/s) -> "
              << (!stream || output != "render.png" ? output : "stdout") << "\n";
  rtg_context_destroy(ctx);
  rtg_host_scene_free(host);
  return code;
}
