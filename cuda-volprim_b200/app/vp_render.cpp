// vp_render: the reference renderer's command line on the C ABI (include/volprim_b200.h) -- the
// C++ host side of the drop-in.  It takes the options of app::Config::parse
// (src/thesis/host/app/config.cpp:15-50) plus the scene and camera the reference wires in code:
//
//   --output PATH            EXR output (default output.exr; vertically flipped as the reference's
//                            Image::save -> saveExr, include/thesis/host/params/image.h:136-145)
//   --width N --height N     image size (default 1000 x 750)
//   --samples_per_pixel N    spp (default 1)
//   --env_map PATH           Radiance .hdr environment (default: constant white)
//   --seed N                 launch seed (default 42)
//   --max-depth N --rr-depth N --rr-max-survival F --firefly-clamp F --filter-width F
//   --phase-g F              Henyey-Greenstein g (default 0.85)
//   --ris [--ris-candidates N]   product RIS NEE (default: MIS)
//   --measure-caps           print the device counters (hits per ray, point overlap)
//   --adaptive-threshold F [--adaptive-min-samples N]   adaptive sampling (the reference's
//                            compile-time ADAPTIVE_THRESHOLD / ADAPTIVE_MIN_SAMPLES,
//                            device/core/constants.cuh:196-211; default off, 32)
//   --ply PATH               Gaussian PLY (x y z rot_0..3 scale_0..2 albedo_0..2 sigma_t_0);
//                            default: main.cpp's single purple Gaussian at the origin
//   --sigma-multiplier F     density multiplier (ply.cpp:116; default 1)
//   --albedo R G B           albedo override for the PLY (ply.cpp:84-105)
//   --eye X Y Z --lookat X Y Z --up X Y Z --vfov DEG   pinhole camera (default: the reference's
//                            getDefaultCamera, eye (0,0,-1) looking at the origin, vfov 90)
//   --ortho-height H         orthographic camera of that viewport height instead
//   --engine wavefront|warp|megakernel   --precision auto|fast|accurate
//   --mitsuba-scene INIT_PY ARGS_JSON   the multi-view harness (test/test_runner.cpp
//                            run_multiview_test with the cameras of a Mitsuba scene description,
//                            test/scenes/cloud_validation.cpp:52-62): every camera, orthographic,
//                            at its own resolution, to OUTPUT_DIR/NNNN.exr (NNNN = position among
//                            the cameras rendered); --camera N keeps camera N only (the
//                            reference's SG_CAM); --output-dir DIR (default multiview);
//                            --list-cameras prints the parsed cameras and exits (no GPU needed)
//   --raygen/--miss/--anyhit/--launch_params/--module_blob NAME   accepted and ignored (they name
//                            OptiX programs; this library has one compiled path)
//   --denoise                accepted; the OptiX AI denoiser is not part of this library, so the
//                            image is written undenoised with a warning
// Exit status 0 on success; on failure the library's message and status 1 (the reference exits
// through try_unwrap_or_exit, include/thesis/host/utils/result.h:89-97).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <string>
#include <vector>

#include "mitsuba_scene.h"
#include "volprim_b200.h"

namespace {

[[noreturn]] void die(const std::string& what) {
  std::fprintf(stderr, "vp_render: %s\n", what.c_str());
  std::exit(1);
}

void ok(vp_status s, const char* what) {
  if (s != VP_OK) die(std::string(what) + ": " + vp_last_error_string());
}

struct Args {
  std::string output = "output.exr", env_map, ply;
  uint32_t width = 1000, height = 750, spp = 1, seed = 42, max_depth = 128, rr_depth = 12, ris_k = 6;
  float rr_max_survival = 0.99f, firefly = 0.f, filter = 0.f, phase_g = 0.85f, sigma = 1.f, vfov = 90.f,
        ortho_h = 0.f, adaptive = 0.f;
  uint32_t adaptive_min = 32;
  float eye[3] = {0.f, 0.f, -1.f}, lookat[3] = {0.f, 0.f, 0.f}, up[3] = {0.f, 1.f, 0.f};
  float albedo[3] = {-1.f, -1.f, -1.f};
  bool ris = false, measure = false;
  int engine = VP_ENGINE_WAVEFRONT, precision = VP_PRECISION_AUTO;
  std::string mitsuba_py, mitsuba_json, output_dir = "multiview";
  int camera_index = -1;
  bool list_cameras = false;
};

Args parse(int argc, char** argv) {
  Args a;
  auto need = [&](int& i, int k) {
    if (i + k >= argc) die(std::string("option ") + argv[i] + " needs " + std::to_string(k) + " value(s)");
  };
  auto u32 = [&](const char* s) {
    char* end = nullptr;
    const unsigned long v = std::strtoul(s, &end, 10);
    if (!end || *end) die(std::string("not an unsigned integer: ") + s);
    return (uint32_t)v;
  };
  auto f32 = [&](const char* s) {
    char* end = nullptr;
    const float v = std::strtof(s, &end);
    if (!end || *end) die(std::string("not a number: ") + s);
    return v;
  };
  for (int i = 1; i < argc; ++i) {
    const std::string o = argv[i];
    if (o == "--output") need(i, 1), a.output = argv[++i];
    else if (o == "--width") need(i, 1), a.width = u32(argv[++i]);
    else if (o == "--height") need(i, 1), a.height = u32(argv[++i]);
    else if (o == "--samples_per_pixel") need(i, 1), a.spp = u32(argv[++i]);
    else if (o == "--env_map") need(i, 1), a.env_map = argv[++i];
    else if (o == "--seed") need(i, 1), a.seed = u32(argv[++i]);
    else if (o == "--max-depth") need(i, 1), a.max_depth = u32(argv[++i]);
    else if (o == "--rr-depth") need(i, 1), a.rr_depth = u32(argv[++i]);
    else if (o == "--rr-max-survival") need(i, 1), a.rr_max_survival = f32(argv[++i]);
    else if (o == "--firefly-clamp") need(i, 1), a.firefly = f32(argv[++i]);
    else if (o == "--adaptive-threshold") need(i, 1), a.adaptive = f32(argv[++i]);
    else if (o == "--adaptive-min-samples") need(i, 1), a.adaptive_min = u32(argv[++i]);
    else if (o == "--filter-width") need(i, 1), a.filter = f32(argv[++i]);
    else if (o == "--phase-g") need(i, 1), a.phase_g = f32(argv[++i]);
    else if (o == "--raygen" || o == "--miss" || o == "--anyhit" || o == "--launch_params" ||
             o == "--module_blob") need(i, 1), ++i;
    else if (o == "--denoise") std::fprintf(stderr, "vp_render: --denoise is not supported; writing the raw image\n");
    else if (o == "--ris") a.ris = true;
    else if (o == "--ris-candidates") need(i, 1), a.ris_k = u32(argv[++i]);
    else if (o == "--measure-caps") a.measure = true;
    else if (o == "--ply") need(i, 1), a.ply = argv[++i];
    else if (o == "--sigma-multiplier") need(i, 1), a.sigma = f32(argv[++i]);
    else if (o == "--albedo") {
      need(i, 3);
      for (float& v : a.albedo) v = f32(argv[++i]);
    } else if (o == "--eye" || o == "--lookat" || o == "--up") {
      need(i, 3);
      float* dst = o == "--eye" ? a.eye : o == "--lookat" ? a.lookat : a.up;
      for (int k = 0; k < 3; ++k) dst[k] = f32(argv[++i]);
    } else if (o == "--vfov") need(i, 1), a.vfov = f32(argv[++i]);
    else if (o == "--ortho-height") need(i, 1), a.ortho_h = f32(argv[++i]);
    else if (o == "--mitsuba-scene") {
      need(i, 2);
      a.mitsuba_py = argv[++i];
      a.mitsuba_json = argv[++i];
    } else if (o == "--output-dir") need(i, 1), a.output_dir = argv[++i];
    else if (o == "--camera") need(i, 1), a.camera_index = (int)u32(argv[++i]);
    else if (o == "--list-cameras") a.list_cameras = true;
    else if (o == "--engine") {
      need(i, 1);
      const std::string v = argv[++i];
      a.engine = v == "wavefront" ? VP_ENGINE_WAVEFRONT : v == "warp" ? VP_ENGINE_WARP
               : v == "megakernel" ? VP_ENGINE_MEGAKERNEL : (die("unknown engine " + v), 0);
    } else if (o == "--precision") {
      need(i, 1);
      const std::string v = argv[++i];
      a.precision = v == "auto" ? VP_PRECISION_AUTO : v == "fast" ? VP_PRECISION_FAST
                  : v == "accurate" ? VP_PRECISION_ACCURATE : (die("unknown precision " + v), 0);
    } else if (o == "--help" || o == "-h") {
      std::printf("see the header of vp_render.cpp for the options\n");
      std::exit(0);
    } else {
      die("unknown option " + o);
    }
  }
  if (a.max_depth == 0) die("--max-depth must be positive");
  if (!(a.phase_g >= -0.999f && a.phase_g <= 0.999f)) die("--phase-g must be in [-0.999, 0.999]");
  if (!(a.rr_max_survival >= 0.f && a.rr_max_survival <= 1.f)) die("--rr-max-survival must be in [0, 1]");
  if (!(a.firefly >= 0.f)) die("--firefly-clamp must be non-negative");
  if (!(a.adaptive >= 0.f)) die("--adaptive-threshold must be non-negative");
  if (!(a.filter >= 0.f)) die("--filter-width must be non-negative");
  if (a.width == 0 || a.height == 0 || a.spp == 0) die("--width, --height and --samples_per_pixel must be positive");
  if ((a.list_cameras || a.camera_index >= 0) && a.mitsuba_py.empty())
    die("--list-cameras and --camera need --mitsuba-scene");
  return a;
}

// The cameras the multi-view harness renders: all, or the one --camera names.
std::vector<vpapp::MitsubaCamera> harness_cameras(const Args& a) {
  vpapp::MitsubaScene ms;
  std::string err;
  if (!vpapp::parse_mitsuba_scene(a.mitsuba_py, a.mitsuba_json, ms, err)) die(err);
  if (a.camera_index < 0) return ms.cameras;
  if (a.camera_index >= (int)ms.cameras.size())
    die("--camera " + std::to_string(a.camera_index) + " out of range (" + std::to_string(ms.cameras.size()) +
        " cameras)");
  return {ms.cameras[(size_t)a.camera_index]};
}

}  // namespace

int main(int argc, char** argv) {
  const Args a = parse(argc, argv);
  std::vector<vpapp::MitsubaCamera> views;
  if (!a.mitsuba_py.empty()) views = harness_cameras(a);
  if (a.list_cameras) {
    for (size_t i = 0; i < views.size(); ++i) {
      const auto& c = views[i];
      const vp_camera cam = vpapp::mitsuba_orthographic_camera(c);
      std::printf("%zu %s %ux%u origin %.9g %.9g %.9g target %.9g %.9g %.9g up %.9g %.9g %.9g ortho_height %.9g\n",
                  i, c.name.c_str(), c.width, c.height, c.origin[0], c.origin[1], c.origin[2], c.target[0],
                  c.target[1], c.target[2], c.up[0], c.up[1], c.up[2], cam.ortho_height);
    }
    return 0;
  }
  vp_context* ctx = nullptr;
  ok(vp_context_create(0, &ctx), "vp_context_create");

  // scene: a PLY, or main.cpp's default (one purple Gaussian at the origin, scale 0.5, sigma_t 0.5)
  vp_host_gaussians hg{};
  const float dm[3] = {0.f, 0.f, 0.f}, ds[3] = {0.5f, 0.5f, 0.5f}, dq[4] = {1.f, 0.f, 0.f, 0.f}, dd[1] = {0.5f},
              da[3] = {0.5f, 0.f, 0.5f};
  vp_gaussians g{1, dm, ds, dq, dd, da, 0, VP_MEMORY_HOST};
  if (!a.ply.empty()) {
    ok(vp_ply_load(a.ply.c_str(), a.albedo, &hg), "vp_ply_load");
    g = vp_gaussians{hg.count, hg.mean, hg.log_scale, hg.quat_wxyz, hg.density, hg.albedo, 1, VP_MEMORY_HOST};
  }
  vp_scene* scene = nullptr;
  ok(vp_scene_create(ctx, &g, a.sigma, &scene), "vp_scene_create");
  if (!a.ply.empty()) vp_host_gaussians_free(&hg);

  vp_env* env = nullptr;
  if (!a.env_map.empty()) {
    float* rgb = nullptr;
    uint32_t w = 0, h = 0;
    ok(vp_hdr_load(a.env_map.c_str(), &rgb, &w, &h), "vp_hdr_load");
    ok(vp_env_create(ctx, rgb, w, h, 3, VP_MEMORY_HOST, &env), "vp_env_create");
    vp_host_free(rgb);
  } else {
    ok(vp_env_create_constant(ctx, 1.f, 1.f, 1.f, &env), "vp_env_create_constant");
  }

  vp_camera cam{};
  std::memcpy(cam.eye, a.eye, sizeof(cam.eye));
  std::memcpy(cam.lookat, a.lookat, sizeof(cam.lookat));
  std::memcpy(cam.up, a.up, sizeof(cam.up));
  cam.vfov_deg = a.vfov;
  cam.orthographic = a.ortho_h > 0.f ? 1 : 0;
  cam.ortho_height = a.ortho_h > 0.f ? a.ortho_h : 2.f;

  vp_render_params p;
  ok(vp_render_params_default(&p), "vp_render_params_default");
  p.width = a.width, p.height = a.height, p.spp = a.spp, p.seed = a.seed;
  p.max_bounces = a.max_depth, p.rr_depth = a.rr_depth, p.rr_max_survival = a.rr_max_survival;
  p.hg_g = a.phase_g, p.firefly_clamp = a.firefly, p.pixel_filter_stddev = a.filter;
  p.nee_mode = a.ris ? VP_NEE_RIS : VP_NEE_MIS;
  p.ris_candidates = a.ris_k;
  p.engine = a.engine, p.precision = a.precision;
  p.measure = a.measure ? VP_MEASURE_COUNTERS : 0;
  p.adaptive_threshold = a.adaptive, p.adaptive_min_samples = a.adaptive_min;

  if (!views.empty()) {  // the multi-view harness: one render per camera, the scene built once
    std::error_code ec;
    std::filesystem::create_directories(a.output_dir, ec);
    if (ec) die("cannot create " + a.output_dir + ": " + ec.message());
    for (size_t i = 0; i < views.size(); ++i) {
      const vp_camera vc = vpapp::mitsuba_orthographic_camera(views[i]);
      p.width = views[i].width, p.height = views[i].height;
      std::vector<float> img(4ull * p.width * p.height);
      vp_render_stats vs{};
      ok(vp_render(scene, env, &vc, &p, img.data(), VP_MEMORY_HOST, &vs), "vp_render");
      char name[32];
      std::snprintf(name, sizeof(name), "%04zu.exr", i);
      const std::string path = (std::filesystem::path(a.output_dir) / name).string();
      ok(vp_exr_save(path.c_str(), img.data(), p.width, p.height, 1), "vp_exr_save");
      std::printf("camera %zu (%s) %ux%u x %u spp (%.3f ms on the device) -> %s\n", i, views[i].name.c_str(), p.width,
                  p.height, p.spp, vs.ms_kernels, path.c_str());
    }
    vp_env_destroy(env);
    vp_scene_destroy(scene);
    vp_context_destroy(ctx);
    return 0;
  }

  std::vector<float> rgba(4ull * a.width * a.height);
  vp_render_stats st{};
  const auto t0 = std::chrono::steady_clock::now();
  ok(vp_render(scene, env, &cam, &p, rgba.data(), VP_MEMORY_HOST, &st), "vp_render");
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ok(vp_exr_save(a.output.c_str(), rgba.data(), a.width, a.height, 1), "vp_exr_save");
  vp_scene_info info{};
  ok(vp_scene_info_get(scene, &info), "vp_scene_info_get");
  std::printf("rendered %ux%u x %u spp of %u Gaussians in %.3f s (%.3f ms on the device, %.2f Mpaths/s) -> %s\n",
              a.width, a.height, a.spp, info.count, secs, st.ms_kernels,
              (double)st.paths / (st.ms_kernels * 1e-3) / 1e6, a.output.c_str());
  if (st.paths_skipped)
    std::printf("adaptive sampling: %llu of %llu paths skipped\n", (unsigned long long)st.paths_skipped,
                (unsigned long long)(st.paths + st.paths_skipped));
  if (a.measure)
    std::printf("max hits per ray %u, max point overlap %u, crossings %llu, shadow rays %llu\n", st.max_hits_per_ray,
                st.max_point_overlap, (unsigned long long)st.crossings, (unsigned long long)st.shadow_rays);
  vp_env_destroy(env);
  vp_scene_destroy(scene);
  vp_context_destroy(ctx);
  return 0;
}
