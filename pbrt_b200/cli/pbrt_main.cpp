// pbrt — the command-line renderer (the reference's src/main.rs with src/config.rs), on the GPU.
//
//   pbrt --input scene.stage [--output output.png] [--near 0.0001] [--far 1000] [--fov 90]
//        [--output_width 800] [--output_height 600] [--max_depth 3] [--samples_ppx 5]
//        [--integrator path|naive|normal] [--threads N] [--renderer st|mt]
//        [--lens_radius R] [--focal_distance F]
//        [--device 0] [--seed 1] [--rr_start 0] [--bvh_bins 8] [--bvh_max_leaf 1] [--no_loader_lights 1]
//
// Options come in `--name value` pairs (Config::new, config.rs:131-170); defaults are
// default_config's (config.rs:112-129). --threads and --renderer are accepted and ignored
// (the GPU renders every pixel); --lens_radius and --focal_distance are accepted and ignored
// as in the reference, whose thin lens takes its radius and focal length from the scene file.
// The options after --lens_radius/--focal_distance are this renderer's own. Mesh files named
// in the scene are read relative to the working directory, as the reference reads them.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/pbrt_b200.h"

namespace {

struct Config {
  std::string input, output = "output.png";
  double near = 0.0001, far = 1000.0, fov_deg = 90.0;
  uint32_t width = 800, height = 600, max_depth = 3, spp = 5;
  uint32_t integrator = PBRT_INTEGRATOR_PATH;
  int device = 0;
  uint64_t seed = 1;
  uint32_t rr_start = 0, bvh_bins = 8, bvh_max_leaf = 1, no_loader_lights = 0;
};

[[noreturn]] void die(const std::string& m) {
  std::fprintf(stderr, "pbrt: %s\n", m.c_str());
  std::exit(1);
}

double to_f(const std::string& k, const std::string& v) {
  char* end = nullptr;
  const double x = std::strtod(v.c_str(), &end);
  if (v.empty() || *end) die("bad value for " + k + ": " + v);
  return x;
}

uint64_t to_u(const std::string& k, const std::string& v) {
  char* end = nullptr;
  const unsigned long long x = std::strtoull(v.c_str(), &end, 10);
  if (v.empty() || *end || v[0] == '-') die("bad value for " + k + ": " + v);
  return x;
}

Config parse(int argc, char** argv) {
  Config c;
  if ((argc - 1) % 2) die(std::string("found trailing parameter ") + argv[argc - 1]);
  for (int i = 1; i + 1 < argc; i += 2) {
    const std::string k = argv[i], v = argv[i + 1];
    if (k == "--input") c.input = v;
    else if (k == "--output") c.output = v;
    else if (k == "--near") c.near = to_f(k, v);
    else if (k == "--far") c.far = to_f(k, v);
    else if (k == "--fov") c.fov_deg = to_f(k, v);
    else if (k == "--output_width") c.width = uint32_t(to_u(k, v));
    else if (k == "--output_height") c.height = uint32_t(to_u(k, v));
    else if (k == "--max_depth") c.max_depth = uint32_t(to_u(k, v));
    else if (k == "--samples_ppx") c.spp = uint32_t(to_u(k, v));
    else if (k == "--threads" || k == "--renderer" || k == "--lens_radius" || k == "--focal_distance") (void)v;
    else if (k == "--integrator") {
      if (v == "path") c.integrator = PBRT_INTEGRATOR_PATH;
      else if (v == "naive") c.integrator = PBRT_INTEGRATOR_NAIVE;
      else if (v == "normal") c.integrator = PBRT_INTEGRATOR_NORMAL;
      else c.integrator = PBRT_INTEGRATOR_PATH;  // parse_integrator's default arm (config.rs:75-90)
    } else if (k == "--device") c.device = int(to_u(k, v));
    else if (k == "--seed") c.seed = to_u(k, v);
    else if (k == "--rr_start") c.rr_start = uint32_t(to_u(k, v));
    else if (k == "--bvh_bins") c.bvh_bins = uint32_t(to_u(k, v));
    else if (k == "--bvh_max_leaf") c.bvh_max_leaf = uint32_t(to_u(k, v));
    else if (k == "--no_loader_lights") c.no_loader_lights = uint32_t(to_u(k, v));
    else die("Unknown option " + k);
  }
  if (c.input.empty()) die("--input is required");
  return c;
}

}  // namespace

int main(int argc, char** argv) {
  const Config c = parse(argc, argv);
  std::ifstream f(c.input, std::ios::binary);
  if (!f) die("cannot read " + c.input);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();

  pbrt_ctx* ctx = nullptr;
  if (pbrt_ctx_create(c.device, &ctx) != PBRT_OK) die("no CUDA device " + std::to_string(c.device));
  pbrt_stage_options o{};
  o.width = c.width;
  o.height = c.height;
  o.fov_deg = c.fov_deg;
  o.near = c.near;
  o.far = c.far;
  o.no_loader_lights = c.no_loader_lights;
  o.bvh_bins = c.bvh_bins;
  o.bvh_max_leaf = c.bvh_max_leaf;
  pbrt_scene* scene = nullptr;
  pbrt_render_params p{};
  if (pbrt_scene_load(ctx, text.c_str(), &o, &scene, &p.camera) != PBRT_OK) die(pbrt_last_error(ctx));
  p.spp = c.spp;
  p.max_depth = c.max_depth;
  p.rr_start = c.rr_start;
  p.seed = c.seed;
  p.integrator = c.integrator;
  std::vector<double> film(size_t(c.width) * c.height * 3);
  if (pbrt_render(scene, &p, film.data()) != PBRT_OK) die(pbrt_last_error(ctx));
  std::vector<uint8_t> rgba(size_t(c.width) * c.height * 4);
  pbrt_film_to_rgba8(film.data(), c.width, c.height, rgba.data());
  if (pbrt_write_png(c.output.c_str(), rgba.data(), c.width, c.height) != PBRT_OK) die("cannot write " + c.output);
  pbrt_scene_destroy(scene);
  pbrt_ctx_destroy(ctx);
  std::printf("%s: %ux%u, %u samples per pixel -> %s\n", c.input.c_str(), c.width, c.height, c.spp, c.output.c_str());
  return 0;
}
