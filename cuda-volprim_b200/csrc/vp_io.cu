// Asset IO on the host: Gaussian PLY files, Radiance RGBE (.hdr) environment maps and OpenEXR
// images -- the reference's loaders and writer (src/thesis/host/utils/io/ply.cpp, hdr.cpp,
// exr.cpp), which use miniply and tinyexr; here the formats are read and written directly from
// their published specifications (PLY: Turk 1994; Radiance picture format: Ward; OpenEXR file
// layout: ILM), with the reference's semantics:
//  - PLY: the "vertex" element's 14 properties x y z, rot_0..3 (w, x, y, z), scale_0..2 (log),
//    albedo_0..2, sigma_t_0 (the Gaussian's total mass); any numeric property type; ascii and
//    binary (either endianness); elements before "vertex" are skipped, list properties included;
//    an albedo override replaces the file's albedo when all three components are >= 0
//    (ply.cpp:84-105).  Scale, rotation and density validation happen in vp_scene_create.
//  - HDR: "#?RADIANCE" / "#?RGBE" magic, FORMAT=32-bit_rle_rgbe, "-Y H +X W" orientation, new
//    run-length scanlines (0x02 0x02 W_hi W_lo, four RLE channels) and raw scanlines; texel =
//    byte * 2^(exponent - 136) (hdr.cpp:30-43); the first scanline is row 0.
//  - EXR: single-part scanline file, uncompressed, FLOAT channels B, G, R (exr.cpp:41-90), with an
//    optional vertical flip.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "vp_internal.h"

namespace vp {
namespace {

// ---- PLY ------------------------------------------------------------------------------------
enum class PlyType { I8, U8, I16, U16, I32, U32, F32, F64, Bad };

PlyType ply_type(const std::string& t) {
  if (t == "char" || t == "int8") return PlyType::I8;
  if (t == "uchar" || t == "uint8") return PlyType::U8;
  if (t == "short" || t == "int16") return PlyType::I16;
  if (t == "ushort" || t == "uint16") return PlyType::U16;
  if (t == "int" || t == "int32") return PlyType::I32;
  if (t == "uint" || t == "uint32") return PlyType::U32;
  if (t == "float" || t == "float32") return PlyType::F32;
  if (t == "double" || t == "float64") return PlyType::F64;
  return PlyType::Bad;
}

size_t ply_size(PlyType t) {
  switch (t) {
    case PlyType::I8: case PlyType::U8: return 1;
    case PlyType::I16: case PlyType::U16: return 2;
    case PlyType::I32: case PlyType::U32: case PlyType::F32: return 4;
    case PlyType::F64: return 8;
    default: return 0;
  }
}

struct PlyProp {
  std::string name;
  PlyType type = PlyType::Bad;
  bool is_list = false;
  PlyType count_type = PlyType::Bad;
};

struct PlyElement {
  std::string name;
  uint64_t count = 0;
  std::vector<PlyProp> props;
};

// Reads one binary value of type t (the file's byte order) as double.
double read_bin(const unsigned char* p, PlyType t, bool swap) {
  unsigned char b[8];
  const size_t n = ply_size(t);
  for (size_t i = 0; i < n; ++i) b[i] = swap ? p[n - 1 - i] : p[i];
  switch (t) {
    case PlyType::I8: { int8_t v; std::memcpy(&v, b, 1); return v; }
    case PlyType::U8: { uint8_t v; std::memcpy(&v, b, 1); return v; }
    case PlyType::I16: { int16_t v; std::memcpy(&v, b, 2); return v; }
    case PlyType::U16: { uint16_t v; std::memcpy(&v, b, 2); return v; }
    case PlyType::I32: { int32_t v; std::memcpy(&v, b, 4); return v; }
    case PlyType::U32: { uint32_t v; std::memcpy(&v, b, 4); return v; }
    case PlyType::F32: { float v; std::memcpy(&v, b, 4); return v; }
    case PlyType::F64: { double v; std::memcpy(&v, b, 8); return v; }
    default: return 0.0;
  }
}

bool host_little_endian() {
  const uint16_t one = 1;
  unsigned char c;
  std::memcpy(&c, &one, 1);
  return c == 1;
}

constexpr int kPlyProps = 14;
const char* const kPlyNames[kPlyProps] = {"x", "y", "z", "rot_0", "rot_1", "rot_2", "rot_3",
                                          "scale_0", "scale_1", "scale_2", "albedo_0", "albedo_1",
                                          "albedo_2", "sigma_t_0"};

vp_status ply_load(const char* path, const float* albedo_override, vp_host_gaussians* out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("Failed to open PLY file: ") + path);
  std::string line;
  std::getline(f, line);
  if (line.rfind("ply", 0) != 0) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("not a PLY file: ") + path);
  int format = -1;  // 0 ascii, 1 binary little endian, 2 binary big endian
  std::vector<PlyElement> elems;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::istringstream ss(line);
    std::string kw;
    ss >> kw;
    if (kw == "format") {
      std::string fmt;
      ss >> fmt;
      format = fmt == "ascii" ? 0 : fmt == "binary_little_endian" ? 1 : fmt == "binary_big_endian" ? 2 : -1;
      if (format < 0) return fail(VP_ERROR_INVALID_ARGUMENT, "unknown PLY format '" + fmt + "'");
    } else if (kw == "element") {
      PlyElement e;
      ss >> e.name >> e.count;
      elems.push_back(e);
    } else if (kw == "property") {
      if (elems.empty()) return fail(VP_ERROR_INVALID_ARGUMENT, "PLY property before any element");
      PlyProp p;
      std::string t;
      ss >> t;
      if (t == "list") {
        std::string ct, it;
        ss >> ct >> it >> p.name;
        p.is_list = true;
        p.count_type = ply_type(ct);
        p.type = ply_type(it);
        if (p.count_type == PlyType::Bad || p.type == PlyType::Bad)
          return fail(VP_ERROR_INVALID_ARGUMENT, "bad PLY list property types in '" + line + "'");
      } else {
        p.type = ply_type(t);
        ss >> p.name;
        if (p.type == PlyType::Bad) return fail(VP_ERROR_INVALID_ARGUMENT, "bad PLY property type '" + t + "'");
      }
      elems.back().props.push_back(p);
    } else if (kw == "end_header") {
      break;
    }
  }
  if (format < 0) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("PLY file without a format line: ") + path);
  const bool swap = (format == 1) != host_little_endian() && format != 0;
  size_t vi = elems.size();
  for (size_t i = 0; i < elems.size(); ++i)
    if (elems[i].name == "vertex") {
      vi = i;
      break;
    }
  if (vi == elems.size()) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("PLY file '") + path + "' has no 'vertex' element");
  const PlyElement& V = elems[vi];
  int col[kPlyProps];
  for (int k = 0; k < kPlyProps; ++k) {
    col[k] = -1;
    for (size_t j = 0; j < V.props.size(); ++j)
      if (!V.props[j].is_list && V.props[j].name == kPlyNames[k]) col[k] = (int)j;
    if (col[k] < 0)
      return fail(VP_ERROR_INVALID_ARGUMENT,
                  std::string("PLY file '") + path + "' missing required property '" + kPlyNames[k] + "'");
  }
  if (V.count > 0x03FFFFFFull) return fail(VP_ERROR_LIMIT, "PLY vertex count above 2^26");
  const uint32_t n = (uint32_t)V.count;
  std::vector<double> row(V.props.size());
  std::vector<float> vals((size_t)n * kPlyProps);
  // Skip or read the elements in file order.
  auto read_row_ascii = [&](const PlyElement& e, std::vector<double>* dst) -> bool {
    for (size_t j = 0; j < e.props.size(); ++j) {
      const PlyProp& p = e.props[j];
      if (p.is_list) {
        double cnt;
        if (!(f >> cnt)) return false;
        for (uint64_t k = 0; k < (uint64_t)cnt; ++k) {
          double tmp;
          if (!(f >> tmp)) return false;
        }
      } else {
        double v;
        if (!(f >> v)) return false;
        if (dst) (*dst)[j] = v;
      }
    }
    return true;
  };
  auto read_row_bin = [&](const PlyElement& e, std::vector<double>* dst) -> bool {
    unsigned char buf[8];
    for (size_t j = 0; j < e.props.size(); ++j) {
      const PlyProp& p = e.props[j];
      if (p.is_list) {
        const size_t cs = ply_size(p.count_type);
        if (!f.read(reinterpret_cast<char*>(buf), (std::streamsize)cs)) return false;
        const uint64_t cnt = (uint64_t)read_bin(buf, p.count_type, swap);
        f.seekg((std::streamoff)(cnt * ply_size(p.type)), std::ios::cur);
        if (!f) return false;
      } else {
        const size_t s = ply_size(p.type);
        if (!f.read(reinterpret_cast<char*>(buf), (std::streamsize)s)) return false;
        if (dst) (*dst)[j] = read_bin(buf, p.type, swap);
      }
    }
    return true;
  };
  for (size_t ei = 0; ei <= vi; ++ei) {
    const PlyElement& e = elems[ei];
    const bool want = ei == vi;
    // A binary element of fixed-size scalar rows before the vertex element is skipped in one seek.
    bool fixed = format != 0 && !want;
    size_t row_bytes = 0;
    for (const PlyProp& p : e.props) {
      if (p.is_list) fixed = false;
      row_bytes += ply_size(p.type);
    }
    if (fixed) {
      f.seekg((std::streamoff)(e.count * row_bytes), std::ios::cur);
      if (!f) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("truncated PLY file: ") + path);
      continue;
    }
    for (uint64_t r = 0; r < e.count; ++r) {
      const bool ok = format == 0 ? read_row_ascii(e, want ? &row : nullptr) : read_row_bin(e, want ? &row : nullptr);
      if (!ok) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("truncated PLY file: ") + path);
      if (want)
        for (int k = 0; k < kPlyProps; ++k) vals[(size_t)r * kPlyProps + k] = (float)row[col[k]];
    }
  }
  const bool override_albedo = albedo_override && albedo_override[0] >= 0.f && albedo_override[1] >= 0.f &&
                               albedo_override[2] >= 0.f;
  vp_host_gaussians g{};
  g.count = n;
  const size_t bytes3 = sizeof(float) * 3ull * (n ? n : 1), bytes4 = sizeof(float) * 4ull * (n ? n : 1),
               bytes1 = sizeof(float) * (n ? n : 1);
  g.mean = static_cast<float*>(std::malloc(bytes3));
  g.log_scale = static_cast<float*>(std::malloc(bytes3));
  g.quat_wxyz = static_cast<float*>(std::malloc(bytes4));
  g.density = static_cast<float*>(std::malloc(bytes1));
  g.albedo = static_cast<float*>(std::malloc(bytes3));
  if (!g.mean || !g.log_scale || !g.quat_wxyz || !g.density || !g.albedo) {
    vp_host_gaussians_free(&g);
    return fail(VP_ERROR_OUT_OF_MEMORY, "host allocation failed");
  }
  for (uint32_t i = 0; i < n; ++i) {
    const float* v = &vals[(size_t)i * kPlyProps];
    for (int k = 0; k < 3; ++k) {
      g.mean[3 * i + k] = v[k];
      g.log_scale[3 * i + k] = v[7 + k];
      g.albedo[3 * i + k] = override_albedo ? albedo_override[k] : v[10 + k];
    }
    for (int k = 0; k < 4; ++k) g.quat_wxyz[4 * i + k] = v[3 + k];
    g.density[i] = v[13];
  }
  *out = g;
  return VP_OK;
}

vp_status ply_save(const char* path, const vp_host_gaussians* g) {
  std::ofstream f(path, std::ios::binary);
  if (!f) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("cannot write ") + path);
  f << "ply\nformat binary_little_endian 1.0\nelement vertex " << g->count << "\n";
  for (const char* name : kPlyNames) f << "property float " << name << "\n";
  f << "end_header\n";
  const bool swap = !host_little_endian();
  for (uint32_t i = 0; i < g->count; ++i) {
    float v[kPlyProps];
    for (int k = 0; k < 3; ++k) {
      v[k] = g->mean[3 * i + k];
      v[7 + k] = g->log_scale[3 * i + k];
      v[10 + k] = g->albedo ? g->albedo[3 * i + k] : 0.f;
    }
    for (int k = 0; k < 4; ++k) v[3 + k] = g->quat_wxyz[4 * i + k];
    v[13] = g->density[i];
    for (float x : v) {
      unsigned char b[4];
      std::memcpy(b, &x, 4);
      if (swap) std::swap(b[0], b[3]), std::swap(b[1], b[2]);
      f.write(reinterpret_cast<const char*>(b), 4);
    }
  }
  if (!f) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("write failed: ") + path);
  return VP_OK;
}

// ---- Radiance RGBE ---------------------------------------------------------------------------
void rgbe_to_rgb(const uint8_t* c, float* out) {
  if (c[3] == 0) {
    out[0] = out[1] = out[2] = 0.0f;
    return;
  }
  const float s = std::ldexp(1.0f, (int)c[3] - 136);
  out[0] = (float)c[0] * s;
  out[1] = (float)c[1] * s;
  out[2] = (float)c[2] * s;
}

vp_status hdr_load(const char* path, float** rgb, uint32_t* width, uint32_t* height) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("Failed to open HDR file: ") + path);
  std::string line;
  std::getline(f, line);
  if (line != "#?RADIANCE" && line != "#?RGBE") return fail(VP_ERROR_INVALID_ARGUMENT, "not a Radiance HDR file (bad magic)");
  bool format = false;
  while (std::getline(f, line) && !line.empty()) {
    if (line.rfind("FORMAT=", 0) == 0) {
      if (line != "FORMAT=32-bit_rle_rgbe") return fail(VP_ERROR_UNSUPPORTED, "unsupported HDR " + line);
      format = true;
    }
  }
  if (!format) return fail(VP_ERROR_INVALID_ARGUMENT, "HDR file missing FORMAT line");
  std::getline(f, line);
  char ya[4] = {0}, xa[4] = {0};
  long H = 0, W = 0;
  if (std::sscanf(line.c_str(), "%2s %ld %2s %ld", ya, &H, xa, &W) != 4 || std::string(ya) != "-Y" ||
      std::string(xa) != "+X" || H <= 0 || W <= 0)
    return fail(VP_ERROR_UNSUPPORTED, "HDR resolution line must be '-Y <height> +X <width>': " + line);
  std::vector<char> rest((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  const uint8_t* p = reinterpret_cast<const uint8_t*>(rest.data());
  const uint8_t* end = p + rest.size();
  float* img = static_cast<float*>(std::malloc(sizeof(float) * 3ull * (size_t)W * (size_t)H));
  if (!img) return fail(VP_ERROR_OUT_OF_MEMORY, "host allocation failed");
  std::vector<uint8_t> line4(4ull * (size_t)W);
  auto bad = [&](const char* why) {
    std::free(img);
    return fail(VP_ERROR_INVALID_ARGUMENT, std::string("corrupt HDR scanline data: ") + why);
  };
  for (long y = 0; y < H; ++y) {
    const bool rle = W >= 8 && W <= 0x7FFF && end - p >= 4 && p[0] == 2 && p[1] == 2 && (p[2] & 0x80) == 0;
    if (rle) {
      if (((long)p[2] << 8 | p[3]) != W) return bad("scanline width mismatch");
      p += 4;
      for (int c = 0; c < 4; ++c) {  // channel planes R, G, B, E
        long x = 0;
        while (x < W) {
          if (p >= end) return bad("truncated");
          const uint8_t code = *p++;
          if (code > 128) {
            const long run = code & 0x7F;
            if (x + run > W || p >= end) return bad("run overflows the scanline");
            for (long k = 0; k < run; ++k) line4[4 * (x + k) + c] = *p;
            ++p;
            x += run;
          } else {
            if (code == 0 || x + code > W || end - p < code) return bad("literal overflows the scanline");
            for (long k = 0; k < code; ++k) line4[4 * (x + k) + c] = p[k];
            p += code;
            x += code;
          }
        }
      }
    } else {
      if (end - p >= 4 && p[0] == 1 && p[1] == 1 && p[2] == 1) {
        std::free(img);
        return fail(VP_ERROR_UNSUPPORTED, "old-style run-length HDR scanlines are not supported");
      }
      if (end - p < 4 * W) return bad("truncated raw scanline");
      std::memcpy(line4.data(), p, 4ull * (size_t)W);
      p += 4 * W;
    }
    for (long x = 0; x < W; ++x) rgbe_to_rgb(&line4[4 * x], img + 3 * ((size_t)y * W + x));
  }
  *rgb = img;
  *width = (uint32_t)W;
  *height = (uint32_t)H;
  return VP_OK;
}

// ---- OpenEXR ---------------------------------------------------------------------------------
void put_i32(std::string& s, int32_t v) {
  char b[4];
  for (int i = 0; i < 4; ++i) b[i] = (char)((uint32_t)v >> (8 * i) & 0xFF);
  s.append(b, 4);
}
void put_u64(std::string& s, uint64_t v) {
  char b[8];
  for (int i = 0; i < 8; ++i) b[i] = (char)(v >> (8 * i) & 0xFF);
  s.append(b, 8);
}
void put_f32(std::string& s, float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  put_i32(s, (int32_t)u);
}
void put_attr(std::string& s, const char* name, const char* type, const std::string& value) {
  s.append(name);
  s.push_back('\0');
  s.append(type);
  s.push_back('\0');
  put_i32(s, (int32_t)value.size());
  s += value;
}

vp_status exr_save(const char* path, const float* rgba, uint32_t W, uint32_t H, int flip) {
  std::string hdr;
  put_i32(hdr, 20000630);  // magic
  put_i32(hdr, 2);         // version 2, single-part scanline
  std::string ch;
  for (const char* c : {"B", "G", "R"}) {  // channels in alphabetical order
    ch.append(c);
    ch.push_back('\0');
    put_i32(ch, 2);  // FLOAT
    ch.append(4, '\0');  // pLinear + reserved
    put_i32(ch, 1);
    put_i32(ch, 1);
  }
  ch.push_back('\0');
  put_attr(hdr, "channels", "chlist", ch);
  put_attr(hdr, "compression", "compression", std::string(1, '\0'));
  std::string box;
  put_i32(box, 0);
  put_i32(box, 0);
  put_i32(box, (int32_t)W - 1);
  put_i32(box, (int32_t)H - 1);
  put_attr(hdr, "dataWindow", "box2i", box);
  put_attr(hdr, "displayWindow", "box2i", box);
  put_attr(hdr, "lineOrder", "lineOrder", std::string(1, '\0'));
  std::string par;
  put_f32(par, 1.0f);
  put_attr(hdr, "pixelAspectRatio", "float", par);
  std::string swc;
  put_f32(swc, 0.0f);
  put_f32(swc, 0.0f);
  put_attr(hdr, "screenWindowCenter", "v2f", swc);
  put_attr(hdr, "screenWindowWidth", "float", par);
  hdr.push_back('\0');
  const uint64_t block = 8ull + 12ull * W;  // y, size, 3 channels x W floats
  const uint64_t first = hdr.size() + 8ull * H;
  for (uint32_t y = 0; y < H; ++y) put_u64(hdr, first + (uint64_t)y * block);
  std::ofstream f(path, std::ios::binary);
  if (!f) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("cannot write ") + path);
  f.write(hdr.data(), (std::streamsize)hdr.size());
  std::string row;
  for (uint32_t y = 0; y < H; ++y) {
    row.clear();
    put_i32(row, (int32_t)y);
    put_i32(row, (int32_t)(12u * W));
    const uint32_t src = flip ? H - 1 - y : y;
    for (int c : {2, 1, 0})  // B, G, R
      for (uint32_t x = 0; x < W; ++x) put_f32(row, rgba[4ull * ((size_t)src * W + x) + c]);
    f.write(row.data(), (std::streamsize)row.size());
  }
  if (!f) return fail(VP_ERROR_INVALID_ARGUMENT, std::string("write failed: ") + path);
  return VP_OK;
}

}  // namespace
}  // namespace vp

using namespace vp;

extern "C" {

vp_status vp_ply_load(const char* path, const float* albedo_override, vp_host_gaussians* out) {
  if (!path || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  std::memset(out, 0, sizeof(*out));
  return ply_load(path, albedo_override, out);
}

vp_status vp_ply_save(const char* path, const vp_host_gaussians* g) {
  if (!path || !g || (g->count && (!g->mean || !g->log_scale || !g->quat_wxyz || !g->density)))
    return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  return ply_save(path, g);
}

vp_status vp_host_gaussians_free(vp_host_gaussians* g) {
  if (!g) return VP_OK;
  std::free(g->mean);
  std::free(g->log_scale);
  std::free(g->quat_wxyz);
  std::free(g->density);
  std::free(g->albedo);
  std::memset(g, 0, sizeof(*g));
  return VP_OK;
}

vp_status vp_hdr_load(const char* path, float** out_rgb, uint32_t* width, uint32_t* height) {
  if (!path || !out_rgb || !width || !height) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out_rgb = nullptr;
  return hdr_load(path, out_rgb, width, height);
}

vp_status vp_host_free(void* p) {
  std::free(p);
  return VP_OK;
}

vp_status vp_exr_save(const char* path, const float* rgba, uint32_t width, uint32_t height, int32_t flip_vertical) {
  if (!path || !rgba || width == 0 || height == 0) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument or empty image");
  return exr_save(path, rgba, width, height, flip_vertical);
}

}  // extern "C"
