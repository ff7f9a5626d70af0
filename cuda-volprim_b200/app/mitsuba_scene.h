// Cameras of a Mitsuba scene description, for the multi-view harness of vp_render.
//
// Reads what the reference's parser reads (src/thesis/host/utils/mitsuba_parser.cpp:14-211):
//   - args.json: "cam_res": N sets every camera's default resolution to N x N (800 x 800 without
//     it); a file that cannot be opened is an error;
//   - __init__.py: 'extent': X (the orthographic extent, 3.0 without it; reported, not used by
//     the camera build, as in the reference), and camera blocks, line by line:
//       'cam_0007': {              starts a camera (resolution back to the defaults)
//       'width': 900, 'height': 600    override its resolution
//       ... T().look_at(           starts the look-at block, which ends at the first line
//       origin=[x, y, z], target=[x, y, z], up=[x, y, z]   holding "),"; a camera is kept when
//       ),                         the block names all three vectors
//     no camera is an error.
// Numbers are the reference's [-0-9.e+]+ tokens.  Each camera becomes an orthographic vp_camera
// of viewport height 2 / aspect (a 2-unit wide film, Mitsuba's [-1, 1] square;
// createOrthographicCamera, mitsuba_parser.cpp:213-225).
#pragma once

#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <iterator>
#include <regex>
#include <sstream>
#include <string>
#include <vector>

#include "volprim_b200.h"

namespace vpapp {

struct MitsubaCamera {
  std::string name;
  float origin[3], target[3], up[3];
  uint32_t width, height;
};

struct MitsubaScene {
  std::vector<MitsubaCamera> cameras;
  float orthographic_extent = 3.0f;
  uint32_t default_width = 800, default_height = 800;
};

namespace detail {

inline const char* kNum = R"(([-\d.e+]+))";

// The three numbers of `key=[a, b, c]` in text; false when absent or not numbers.
inline bool vec3_after(const std::string& text, const char* key, float out[3]) {
  const std::regex re(std::string(key) + R"(=\[)" + kNum + R"(,\s*)" + kNum + R"(,\s*)" + kNum + R"(\])");
  std::smatch m;
  if (!std::regex_search(text, m, re)) return false;
  for (int k = 0; k < 3; ++k) {
    const std::string s = m[k + 1].str();
    char* end = nullptr;
    out[k] = std::strtof(s.c_str(), &end);
    if (end == s.c_str()) return false;
  }
  return true;
}

inline bool read_file(const std::string& path, std::string& out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return true;
}

}  // namespace detail

// Parses init_py + args_json into `out`; on failure returns false with a message in `err`.
inline bool parse_mitsuba_scene(const std::string& init_py, const std::string& args_json, MitsubaScene& out,
                                std::string& err) {
  out = MitsubaScene{};
  std::string json, py;
  if (!detail::read_file(args_json, json)) {
    err = "failed to open args.json: " + args_json;
    return false;
  }
  std::smatch m;
  if (std::regex_search(json, m, std::regex(R"#("cam_res":\s*(\d+))#"))) {
    out.default_width = out.default_height = static_cast<uint32_t>(std::strtoul(m[1].str().c_str(), nullptr, 10));
  }
  if (!detail::read_file(init_py, py)) {
    err = "failed to open Mitsuba config file: " + init_py;
    return false;
  }
  if (std::regex_search(py, m, std::regex(R"('extent':\s*([\d.e+-]+))"))) out.orthographic_extent = std::strtof(m[1].str().c_str(), nullptr);

  const std::regex cam_start(R"('(cam_\d+)':\s*\{)"), width_re(R"('width':\s*(\d+))"),
      height_re(R"('height':\s*(\d+))");
  enum { kIdle, kInCamera, kInLookAt } state = kIdle;
  MitsubaCamera cur{};
  std::string block;
  std::istringstream lines(py);
  std::string line;
  while (std::getline(lines, line)) {
    if (std::regex_search(line, m, cam_start)) {
      cur = MitsubaCamera{};
      cur.name = m[1].str();
      cur.width = out.default_width;
      cur.height = out.default_height;
      state = kInCamera;
      continue;
    }
    if (state == kInCamera) {
      if (std::regex_search(line, m, width_re)) {
        cur.width = static_cast<uint32_t>(std::strtoul(m[1].str().c_str(), nullptr, 10));
        continue;
      }
      if (std::regex_search(line, m, height_re)) {
        cur.height = static_cast<uint32_t>(std::strtoul(m[1].str().c_str(), nullptr, 10));
        continue;
      }
      if (line.find("T().look_at(") != std::string::npos) {
        state = kInLookAt;
        block.clear();
      }
    }
    if (state == kInLookAt) {
      block += line + "\n";
      if (line.find("),") != std::string::npos) {
        MitsubaCamera c = cur;
        if (detail::vec3_after(block, "origin", c.origin) && detail::vec3_after(block, "target", c.target) &&
            detail::vec3_after(block, "up", c.up))
          out.cameras.push_back(c);
        state = kInCamera;
        block.clear();
      }
    }
  }
  if (out.cameras.empty()) {
    err = "no cameras found in Mitsuba config " + init_py;
    return false;
  }
  return true;
}

// Orthographic camera of a 2-unit wide film: viewport height 2 / (width / height).
inline vp_camera mitsuba_orthographic_camera(const MitsubaCamera& c) {
  vp_camera cam{};
  for (int k = 0; k < 3; ++k) cam.eye[k] = c.origin[k], cam.lookat[k] = c.target[k], cam.up[k] = c.up[k];
  const float aspect = static_cast<float>(c.width) / static_cast<float>(c.height);
  cam.ortho_height = 2.0f / aspect;
  cam.vfov_deg = 90.0f;
  cam.orthographic = 1;
  return cam;
}

}  // namespace vpapp
