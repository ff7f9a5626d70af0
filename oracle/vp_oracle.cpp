// ORACLE — test infrastructure only.  A CPU restatement of the reference renderer's per-ray
// hot path (kfernandez31/cuda-volprim), used by tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg as the checker.  Nothing in the product links or calls this file.
//
// Two parts:
//  1. FP64 closed-form transmittance: exp(-sum over Gaussians of the 3-sigma-truncated chord
//     optical depth), brute force over all Gaussians -- the formula of
//     experiments/mitsuba-reference/cloud_bruteforce_transmittance.py:48-60 -- and the
//     absorption-only image it implies (bounce-0 analytic direct term x environment), replaying
//     the reference's PCG32 jitter stream per (pixel, sample).
//  2. FP32 restatement of the full path tracer in the reference's operation order:
//       Primitive precompute / transforms / inv_cdf / inv_cdf_span / optical_depth / pdf
//         (include/thesis/device/params/primitive.h:70-318),
//       UnitQuaternion (include/thesis/common/geometry/quat.h:55-71),
//       point_inside_bvh_bound / exit_from_inside / compute_exit_from_entry
//         (include/thesis/common/geometry/intersection.h:56-173),
//       sampling stages, phase, env_is, transmittance (device/core/sampling.cuh:74-583),
//       russian_roulette / finalize_sample / escape / NEE (device/entry/path_stages.cuh:25-226),
//       the raygen loop (device/entry/raygen.cuh:72-230), PCG32 (device/core/random.cuh:16-72),
//       camera (include/thesis/device/params/camera.h:33-57, host/params/camera.h:32-111),
//       env CDF build + lookup (include/thesis/host/params/environment_map.h:45-101,
//         device/params/environment_map.h:36-61).
//     OptiX traversal order is replaced by ascending entry distance (the reference's order is
//     unspecified).  rng_mode 0 draws the free flights from the path's PCG32 in that order as
//     the reference does; rng_mode 1 keys them by (bounce key, Gaussian index) and samples the
//     environment through per-row alias tables, as the GPU engines do, so GPU and oracle paths
//     can be compared sample by sample.
//  The reference's erfinvf (CUDA) has no libm counterpart: erfinv here is a Newton iteration on
//  double-precision std::erf, rounded to float.
#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace {

// ---------------------------------------------------------------------------------------------
// FP32 vector ops in the reference's order (include/thesis/common/utils/math.h)
// ---------------------------------------------------------------------------------------------
struct F3 {
  float x, y, z;
};
inline F3 mk(float x, float y, float z) { return F3{x, y, z}; }
inline F3 operator+(F3 a, F3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 operator-(F3 a) { return mk(-a.x, -a.y, -a.z); }
inline F3 operator-(F3 a, F3 b) { return a + (-b); }
inline F3 operator*(F3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline F3 operator*(float s, F3 a) { return a * s; }
inline F3 operator*(F3 a, F3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float rcp(float x) { return 1.0f / x; }
inline float dot(F3 a, F3 b) { return std::fmaf(a.x, b.x, std::fmaf(a.y, b.y, a.z * b.z)); }
inline float length2(F3 v) { return dot(v, v); }
inline float rsqrt_(float x) { return 1.0f / std::sqrt(x); }
inline F3 normalize(F3 v) { return v * rsqrt_(length2(v)); }
inline F3 cross(F3 a, F3 b) {
  return mk(std::fmaf(a.y, b.z, -(a.z * b.y)), std::fmaf(a.z, b.x, -(a.x * b.z)),
            std::fmaf(a.x, b.y, -(a.y * b.x)));
}
inline F3 fma3(float a, F3 b, F3 c) {
  return mk(std::fmaf(a, b.x, c.x), std::fmaf(a, b.y, c.y), std::fmaf(a, b.z, c.z));
}
inline float maxc(F3 v) { return std::max(std::max(v.x, v.y), v.z); }
inline float sumc(F3 v) { return v.x + v.y + v.z; }
inline F3 lerp(F3 a, F3 b, float t) {
  return mk(std::fmaf(t, b.x - a.x, a.x), std::fmaf(t, b.y - a.y, a.y), std::fmaf(t, b.z - a.z, a.z));
}
inline F3 midpoint(F3 a, F3 b) { return lerp(a, b, 0.5f); }

constexpr float PI_F = 3.14159265358979323846f;
constexpr float TWO_PI_F = 2.0f * PI_F;
constexpr float ONE_OVER_PI_F = 1.0f / PI_F;
constexpr float ONE_OVER_TWO_PI_F = 1.0f / (2.0f * PI_F);
constexpr float ONE_OVER_FOUR_PI_F = 1.0f / (4.0f * PI_F);
constexpr float ROOT_TWO_F = 1.41421356237309504880f;
constexpr float ONE_OVER_ROOT_TWO_F = 1.0f / ROOT_TWO_F;
constexpr float ROOT_TWO_PI_F = 2.5066282746f;
constexpr float ROOT_HALF_PI_F = ROOT_TWO_PI_F * 0.5f;
constexpr float ONE_OVER_TWO_PI_POW_3_2_F = 0.0634936359f;
constexpr float GAUSSIAN_EXTENT_F = 3.0f;
constexpr float GAUSSIAN_DIAMETER_F = 6.0f;
constexpr float INF_F = 1e20f;
constexpr float RAY_SEGMENT_MIN_LENGTH = 1e-6f;
constexpr float MAX_OPTICAL_DEPTH = 88.0f;
constexpr float MIN_THROUGHPUT = 1e-4f;

float erfinv_f(float x) {  // float(erfinv(x)) via Newton on double erf
  if (x >= 1.0f) return INFINITY;
  if (x <= -1.0f) return -INFINITY;
  const double y = x;
  // initial guess (Giles-style log form), then Newton steps on erf(z) - y
  double w = -std::log((1.0 - y) * (1.0 + y));
  double z = (w < 5.0) ? (y * (1.0 + 0.2 * w)) : (std::copysign(std::sqrt(w), y));
  for (int it = 0; it < 60; ++it) {
    const double f = std::erf(z) - y;
    const double df = 1.1283791670955126 * std::exp(-z * z);
    if (df == 0.0) break;
    const double dz = f / df;
    z -= dz;
    if (std::fabs(dz) < 1e-17 * (1.0 + std::fabs(z))) break;
  }
  return static_cast<float>(z);
}

// ---------------------------------------------------------------------------------------------
// Primitive (primitive.h:27-318) + UnitQuaternion (quat.h)
// ---------------------------------------------------------------------------------------------
struct Quat {
  float s;
  F3 u;
  F3 rotate(F3 v) const {  // v + 2s(u x v) + 2u x (u x v)
    const F3 uv = cross(u, v);
    const F3 uuv = cross(u, uv);
    return fma3(2.0f, fma3(s, uv, uuv), v);
  }
};

struct Prim {
  F3 center;
  Quat rot;  // conjugate of the forward rotation
  F3 rcp_scale;
  float dnf, icf;
  F3 albedo;
  float mass;
  F3 scale;
  F3 pos_local(F3 p) const { return rot.rotate(p - center) * rcp_scale; }
  F3 dir_local(F3 d) const { return rot.rotate(d) * rcp_scale; }
  float pdf(F3 pos) const {
    const F3 l = pos_local(pos);
    return std::exp(-0.5f * length2(l)) * dnf;
  }
  float inv_cdf(F3 o, F3 d, float tau) const {
    const F3 w = dir_local(d), p = pos_local(o);
    const float w_len2 = length2(w);
    const float w_inv_len = rsqrt_(w_len2);
    const float wp = dot(w, p) * w_inv_len;
    const float pp = length2(p);
    const float diff = std::fmaf(-wp, wp, pp);
    const float K = w_inv_len * std::exp(-0.5f * diff) * icf;
    const float raw = std::erf(wp * ONE_OVER_ROOT_TWO_F) + tau * rcp(K);
    if (raw > 1.0f) return INF_F;
    const float arg = std::min(std::max(raw, -1.0f), 1.0f);
    return (ROOT_TWO_F * erfinv_f(arg) - wp) * w_inv_len;
  }
  float inv_cdf_span(F3 o, F3 d, float t_offset, float tau) const {
    const F3 w = dir_local(d), p = pos_local(o);
    const float w_len2 = length2(w);
    const float w_inv_len = rsqrt_(w_len2);
    const float w_len = w_len2 * w_inv_len;
    const float wp = dot(w, p) * w_inv_len;
    const float pp = length2(p);
    const float diff = std::fmaf(-wp, wp, pp);
    const float K = w_inv_len * std::exp(-0.5f * diff) * icf;
    const float wp_off = std::fmaf(t_offset, w_len, wp);
    const float raw = std::erf(wp_off * ONE_OVER_ROOT_TWO_F) + tau * rcp(K);
    if (raw > 1.0f) return INF_F;
    const float arg = std::min(std::max(raw, -1.0f), 1.0f);
    return (ROOT_TWO_F * erfinv_f(arg) - wp) * w_inv_len;
  }
  float optical_depth(F3 o, F3 d, float t0, float t1) const {
    if (t1 - t0 <= RAY_SEGMENT_MIN_LENGTH) return 0.0f;
    const F3 w = dir_local(d), p = pos_local(o);
    const float w_inv_len = rsqrt_(length2(w));
    const float t0s = std::max(0.0f, t0);
    const float t1s = std::max(t0s + RAY_SEGMENT_MIN_LENGTH, t1);
    const F3 wn = w * w_inv_len;
    const F3 p_start = p + t0s * w;
    const float t_limit = std::min(std::max((t1s - t0s) * rcp(w_inv_len), 0.0f), GAUSSIAN_DIAMETER_F);
    const float B = dot(wn, p_start);
    const float C = length2(p_start);
    const float perp2 = std::fmaf(-B, B, C);
    const float e_term = std::exp(-0.5f * perp2);
    const float G = ROOT_TWO_PI_F * w_inv_len;
    const float Bs = B * ONE_OVER_ROOT_TWO_F;
    const float lo = std::erf(Bs);
    const float up = std::erf(std::fmaf(t_limit, ONE_OVER_ROOT_TWO_F, Bs));
    const float et = (up - lo) * 0.5f;
    return mass * G * e_term * et * dnf;
  }
};

inline bool point_inside(F3 point, const Prim& p) {  // intersection.h:56-61
  const F3 l = p.pos_local(point);
  return length2(l) <= GAUSSIAN_EXTENT_F * GAUSSIAN_EXTENT_F;
}
inline float exit_from_inside(F3 o, F3 d, const Prim& p) {  // intersection.h:115-126
  const F3 w = p.dir_local(d), q = p.pos_local(o);
  const float a = length2(w), b = dot(q, w);
  const float c = length2(q) - 9.0f;
  const float disc = std::fmaf(-a, c, b * b);
  return (-b + std::sqrt(disc)) * rcp(a);
}
inline float exit_from_entry(F3 o, F3 d, float t_entry, const Prim& p, float w_len2) {  // :142-173
  const F3 entry = o + t_entry * d;
  const F3 q = p.pos_local(entry);
  const F3 w = p.dir_local(d);
  const float pw = dot(q, w);
  return t_entry + (-2.0f * pw * rcp(w_len2));
}
// Entry distance of the 3-sigma ellipsoid (what OptiX's sphere intersector reports for the
// 3x-scaled instance): stable quadratic of intersection.h:66-101 with radius^2 = 9.
inline bool entry_3sigma(F3 o, F3 d, const Prim& p, float& t_entry) {
  const F3 w = p.dir_local(d), q = p.pos_local(o);
  const float a = length2(w);
  if (a < 1e-12f) return false;
  const float a_inv = rcp(a);
  const float b = -dot(q, w);
  const float delta = 9.0f - length2(fma3(b * a_inv, w, q));
  if (delta < 1e-12f) return false;
  const float c = length2(q) - 9.0f;
  const float qq = b + std::copysign(std::sqrt(a * delta), b);
  const float t1 = c * rcp(qq), t2 = qq * a_inv;
  const float te = std::min(t1, t2);
  if (!(te > 0.0f) || te >= INF_F) return false;  // OptiX reports front-face entries in (0, tmax)
  t_entry = te;
  return true;
}

// ---------------------------------------------------------------------------------------------
// RNG (random.cuh:16-72)
// ---------------------------------------------------------------------------------------------
struct Pcg {
  uint64_t state, inc;
  uint32_t next() {
    const uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = static_cast<uint32_t>(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
  }
  float uniform() { return static_cast<float>(next()) / static_cast<float>(UINT32_MAX); }
};
inline uint64_t seq_hash(uint64_t x) {
  x = x * 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x = x * 0x94d049bb133111ebULL;
  x ^= x >> 31;
  return x;
}
inline Pcg pcg_init(uint64_t seed, uint64_t seq) {
  Pcg r{0u, (seq << 1u) | 1u};
  r.next();
  r.state += seed;
  r.next();
  return r;
}
inline uint32_t keyed_u32(uint64_t key, uint32_t idx) {  // GPU keyed free-flight draw
  uint64_t z = key ^ (static_cast<uint64_t>(idx) * 0x9E3779B97F4A7C15ULL);
  z ^= z >> 30;
  z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27;
  z *= 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return static_cast<uint32_t>(z >> 32);
}

// ---------------------------------------------------------------------------------------------
// scene, camera, environment
// ---------------------------------------------------------------------------------------------
struct Camera {
  F3 eye, p00, du, dv, view_dir;
  int ortho;
};

void build_camera(const float* eye, const float* lookat, const float* up, float vfov, float ortho_h,
                  int ortho, uint32_t W, uint32_t H, Camera& c) {
  const F3 lf = mk(eye[0], eye[1], eye[2]), la = mk(lookat[0], lookat[1], lookat[2]),
           vup = mk(up[0], up[1], up[2]);
  const float fw = static_cast<float>(W), fh = static_cast<float>(H);
  if (!ortho) {
    const float theta = vfov * (PI_F / 180.0f);
    const float h = std::tan(0.5f * theta);
    const F3 w = normalize(lf - la);
    const F3 u = normalize(cross(vup, w));
    const F3 v = cross(w, u);
    const float focal = std::sqrt(length2(lf - la));
    const float aspect = fw * rcp(fh);
    const float vh = 2.0f * h * focal;
    const float vw = vh * aspect;
    const F3 vu = u * vw, vv = (-v) * vh;
    const F3 du = vu * rcp(fw), dv = vv * rcp(fh);
    const F3 ul = lf - focal * w - midpoint(vu, vv);
    const F3 p00 = ul + midpoint(du, dv);
    c = Camera{lf, p00 - lf, du, dv, mk(0.f, 0.f, 1.f), 0};
  } else {
    const F3 vd = normalize(la - lf);
    const F3 right = normalize(cross(vd, vup));
    const F3 upv = cross(right, vd);
    const float aspect = fw * rcp(fh);
    const float vh = ortho_h, vw = vh * aspect;
    const F3 vu = right * vw, vv = upv * vh;
    const F3 du = vu * rcp(fw), dv = vv * rcp(fh);
    const F3 ul = lf - midpoint(vu, vv);
    const F3 p00 = ul + midpoint(du, dv);
    c = Camera{lf, p00 - lf, du, dv, vd, 1};
  }
}

// Camera ray of (pixel, sample) with the reference's jitter draws (raygen.cuh:82-99).
inline void camera_ray(const Camera& c, float filter_stddev, uint32_t px, uint32_t py, Pcg& rng, F3& o, F3& d) {
  float jx, jy;
  if (filter_stddev > 0.0f) {
    const float u1 = std::max(rng.uniform(), 1e-7f);
    const float u2 = rng.uniform();
    const float r = filter_stddev * std::sqrt(-2.0f * std::log(u1));
    const float th = TWO_PI_F * u2;
    jx = std::min(std::max(r * std::cos(th), -2.0f), 2.0f);
    jy = std::min(std::max(r * std::sin(th), -2.0f), 2.0f);
  } else {
    jx = rng.uniform() - 0.5f;
    jy = rng.uniform() - 0.5f;
  }
  const float x = static_cast<float>(px) + jx, y = static_cast<float>(py) + jy;
  const F3 off = fma3(x, c.du, fma3(y, c.dv, c.p00));
  if (c.ortho) {
    o = c.eye + off;
    d = c.view_dir;
  } else {
    o = c.eye;
    d = normalize(off);
  }
}

struct Env {
  uint32_t W = 0, H = 0;
  std::vector<float> rgba;         // W*H*4
  std::vector<float> joint, cond_cdf, marg_cdf;  // reference CDF (FP32 build)
  float total = 0.f;
  std::vector<float> alias_cond_p, alias_marg_p;  // GPU alias tables (FP64 build)
  std::vector<uint32_t> alias_cond_a, alias_marg_a;
  double total64 = 0.0;
};

void vose(uint32_t n, const double* w, double sum, float* prob, uint32_t* alias) {
  if (!(sum > 0.0)) {
    for (uint32_t u = 0; u < n; ++u) prob[u] = 1.0f, alias[u] = u;
    return;
  }
  std::vector<double> p(n);
  std::vector<uint32_t> small, large;
  const double scale = static_cast<double>(n) / sum;
  for (uint32_t u = 0; u < n; ++u) {
    p[u] = w[u] * scale;
    if (p[u] < 1.0) small.push_back(u);
    else large.push_back(u);
  }
  while (!small.empty() && !large.empty()) {
    const uint32_t l = small.back();
    small.pop_back();
    const uint32_t g = large.back();
    large.pop_back();
    prob[l] = static_cast<float>(p[l]);
    alias[l] = g;
    p[g] = (p[g] + p[l]) - 1.0;
    if (p[g] < 1.0) small.push_back(g);
    else large.push_back(g);
  }
  while (!large.empty()) {
    const uint32_t g = large.back();
    large.pop_back();
    prob[g] = 1.0f, alias[g] = g;
  }
  while (!small.empty()) {
    const uint32_t l = small.back();
    small.pop_back();
    prob[l] = 1.0f, alias[l] = l;
  }
}

void build_env(const float* data, uint32_t W, uint32_t H, uint32_t ch, Env& e) {
  e.W = W;
  e.H = H;
  const size_t n = static_cast<size_t>(W) * H;
  e.rgba.assign(n * 4, 0.f);
  e.joint.assign(n, 0.f);
  e.cond_cdf.assign(n, 0.f);
  e.marg_cdf.assign(H, 0.f);
  std::vector<double> w64(n), rows(H, 0.0);
  for (size_t i = 0; i < n; ++i) {
    const float* px = data + i * ch;
    const float r = px[0], g = ch >= 2 ? px[1] : r, b = ch >= 3 ? px[2] : r, a = ch >= 4 ? px[3] : 1.f;
    e.rgba[4 * i] = r, e.rgba[4 * i + 1] = g, e.rgba[4 * i + 2] = b, e.rgba[4 * i + 3] = a;
  }
  // Reference FP32 CDF (environment_map.h:45-101).
  for (uint32_t v = 0; v < H; ++v) {
    const float theta = (static_cast<float>(v) + 0.5f) / static_cast<float>(H) * PI_F;
    const float st = std::sin(theta);
    float row = 0.f;
    for (uint32_t u = 0; u < W; ++u) {
      const size_t i = static_cast<size_t>(v) * W + u;
      const float lum = 0.2126f * e.rgba[4 * i] + 0.7152f * e.rgba[4 * i + 1] + 0.0722f * e.rgba[4 * i + 2];
      const float wt = lum * st;
      e.joint[i] = wt;
      row += wt;
      e.cond_cdf[i] = row;
    }
    if (row > 0.f) {
      const float inv = 1.0f / row;
      for (uint32_t u = 0; u < W; ++u) e.cond_cdf[static_cast<size_t>(v) * W + u] *= inv;
    } else {
      for (uint32_t u = 0; u < W; ++u)
        e.cond_cdf[static_cast<size_t>(v) * W + u] = (static_cast<float>(u) + 1.0f) / static_cast<float>(W);
    }
    e.marg_cdf[v] = row;
  }
  float total = 0.f;
  for (uint32_t v = 0; v < H; ++v) {
    total += e.marg_cdf[v];
    e.marg_cdf[v] = total;
  }
  e.total = total;
  if (total > 0.f) {
    const float inv = 1.0f / total;
    for (uint32_t v = 0; v < H; ++v) e.marg_cdf[v] *= inv;
  } else {
    for (uint32_t v = 0; v < H; ++v) e.marg_cdf[v] = (static_cast<float>(v) + 1.0f) / static_cast<float>(H);
  }
  // GPU alias tables (FP64 weights, per-row + marginal Vose).
  for (uint32_t v = 0; v < H; ++v) {
    const double theta = (static_cast<double>(v) + 0.5) / static_cast<double>(H) * 3.14159265358979323846;
    for (uint32_t u = 0; u < W; ++u) {
      const size_t i = static_cast<size_t>(v) * W + u;
      const double lum = 0.2126 * e.rgba[4 * i] + 0.7152 * e.rgba[4 * i + 1] + 0.0722 * e.rgba[4 * i + 2];
      w64[i] = lum * std::sin(theta);
      rows[v] += w64[i];
    }
  }
  e.alias_cond_p.assign(n, 1.f);
  e.alias_cond_a.assign(n, 0u);
  e.alias_marg_p.assign(H, 1.f);
  e.alias_marg_a.assign(H, 0u);
  for (uint32_t v = 0; v < H; ++v)
    vose(W, w64.data() + static_cast<size_t>(v) * W, rows[v], e.alias_cond_p.data() + static_cast<size_t>(v) * W,
         e.alias_cond_a.data() + static_cast<size_t>(v) * W);
  double tot = 0.0;
  for (uint32_t v = 0; v < H; ++v) tot += rows[v];
  e.total64 = tot;
  vose(H, rows.data(), tot, e.alias_marg_p.data(), e.alias_marg_a.data());
}

// Bilinear wrap-U / clamp-V lat-long lookup (environment_map.h:36-61; FP32 filter weights).
F3 env_lookup(const Env& e, F3 dir) {
  const float theta = std::atan2(dir.z, dir.x);
  const float phi = std::acos(std::min(std::max(dir.y, -1.0f), 1.0f));
  float u = std::fmaf(theta, ONE_OVER_TWO_PI_F, 0.5f);
  const float v = phi * ONE_OVER_PI_F;
  u = u - std::floor(u);
  const float x = u * static_cast<float>(e.W) - 0.5f, y = v * static_cast<float>(e.H) - 0.5f;
  const float xf = std::floor(x), yf = std::floor(y);
  const float fx = x - xf, fy = y - yf;
  const int W = static_cast<int>(e.W), H = static_cast<int>(e.H);
  int i0 = static_cast<int>(xf), j0 = static_cast<int>(yf);
  int i1 = i0 + 1, j1 = j0 + 1;
  i0 = ((i0 % W) + W) % W;
  i1 = ((i1 % W) + W) % W;
  j0 = std::min(std::max(j0, 0), H - 1);
  j1 = std::min(std::max(j1, 0), H - 1);
  auto T = [&](int i, int j, int c) { return e.rgba[4 * (static_cast<size_t>(j) * W + i) + c]; };
  const float gx = 1.f - fx, gy = 1.f - fy;
  float out[3];
  for (int c = 0; c < 3; ++c)
    out[c] = gy * (gx * T(i0, j0, c) + fx * T(i1, j0, c)) + fy * (gx * T(i0, j1, c) + fx * T(i1, j1, c));
  return mk(out[0], out[1], out[2]);
}

int upper_bound(const float* cdf, int n, float u) {  // env_is::upper_bound (sampling.cuh:160-171)
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (cdf[mid] <= u) lo = mid + 1;
    else hi = mid;
  }
  return std::min(lo, n - 1);
}

inline uint32_t alias_pick(const float* p, const uint32_t* a, uint32_t n, uint32_t r) {
  const uint64_t x = static_cast<uint64_t>(r) * n;
  const uint32_t idx = static_cast<uint32_t>(x >> 32);
  const float coin = static_cast<float>(static_cast<uint32_t>(x)) * 2.3283064365386963e-10f;
  return coin < p[idx] ? idx : a[idx];
}

struct EnvSample {
  F3 wo;
  float pdf;
};

EnvSample env_sample(const Env& e, Pcg& rng, bool alias) {  // env_is::sample (sampling.cuh:173-216)
  const uint32_t r0 = rng.next(), r1 = rng.next();
  const float u0 = static_cast<float>(r0) / static_cast<float>(UINT32_MAX);
  const float u1 = static_cast<float>(r1) / static_cast<float>(UINT32_MAX);
  const float total = alias ? static_cast<float>(e.total64) : e.total;
  if (total <= 0.f || e.W == 0 || e.H == 0) {
    const float z = std::fmaf(-2.0f, u0, 1.0f);
    const float r = std::sqrt(std::max(0.0f, std::fmaf(-z, z, 1.0f)));
    const float phi = TWO_PI_F * u1;
    return {mk(r * std::cos(phi), r * std::sin(phi), z), ONE_OVER_FOUR_PI_F};
  }
  const int W = static_cast<int>(e.W), H = static_cast<int>(e.H);
  int v, u;
  if (alias) {
    v = static_cast<int>(alias_pick(e.alias_marg_p.data(), e.alias_marg_a.data(), e.H, r0));
    u = static_cast<int>(alias_pick(e.alias_cond_p.data() + static_cast<size_t>(v) * W,
                                    e.alias_cond_a.data() + static_cast<size_t>(v) * W, e.W, r1));
  } else {
    v = upper_bound(e.marg_cdf.data(), H, u0);
    u = upper_bound(e.cond_cdf.data() + static_cast<size_t>(v) * W, W, u1);
  }
  const float jx = rng.uniform(), jy = rng.uniform();
  const float un = (static_cast<float>(u) + jx) * rcp(static_cast<float>(W));
  const float vn = (static_cast<float>(v) + jy) * rcp(static_cast<float>(H));
  const float theta = std::fmaf(2.0f * PI_F, un, -PI_F);
  const float polar = vn * PI_F;
  const float sp = std::sin(polar);
  const F3 wo = mk(sp * std::cos(theta), std::cos(polar), sp * std::sin(theta));
  const float joint = e.joint[static_cast<size_t>(v) * W + u];
  const float p_uv = (joint * rcp(total)) * static_cast<float>(W * H);
  const float jac = 2.0f * PI_F * PI_F * sp;
  return {wo, sp > 0.f ? p_uv * rcp(jac) : 0.f};
}

float env_pdf(const Env& e, F3 wo, bool alias) {  // env_is::pdf (sampling.cuh:218-246)
  const float total = alias ? static_cast<float>(e.total64) : e.total;
  if (total <= 0.f || e.W == 0 || e.H == 0) return ONE_OVER_FOUR_PI_F;
  const int W = static_cast<int>(e.W), H = static_cast<int>(e.H);
  const float theta = std::atan2(wo.z, wo.x);
  const float polar = std::acos(std::min(std::max(wo.y, -1.0f), 1.0f));
  const float un = std::fmaf(theta, ONE_OVER_TWO_PI_F, 0.5f);
  const float vn = polar * ONE_OVER_PI_F;
  int u = static_cast<int>(un * static_cast<float>(W));
  int v = static_cast<int>(vn * static_cast<float>(H));
  u = u < 0 ? 0 : (u >= W ? W - 1 : u);
  v = v < 0 ? 0 : (v >= H ? H - 1 : v);
  const float joint = e.joint[static_cast<size_t>(v) * W + u];
  const float sp = std::sin(polar);
  if (joint <= 0.f || sp <= 0.f) return 0.f;
  const float p_uv = (joint * rcp(total)) * static_cast<float>(W * H);
  return p_uv * rcp(2.0f * PI_F * PI_F * sp);
}

// ---------------------------------------------------------------------------------------------
// CPU BVH over the 3-sigma boxes: returns a candidate superset for ray and point queries, so the
// algorithm above runs exactly as with brute force over all Gaussians.
// ---------------------------------------------------------------------------------------------
struct Box {
  double lo[3], hi[3];
};
struct Bvh {
  struct Node {
    Box b;
    int left = -1, right = -1;
    uint32_t first = 0, count = 0;
  };
  std::vector<Node> nodes;
  std::vector<uint32_t> idx;
  std::vector<Box> boxes;
  bool enabled = false;

  void build(const std::vector<Box>& bx) {
    boxes = bx;
    idx.resize(bx.size());
    std::iota(idx.begin(), idx.end(), 0u);
    nodes.clear();
    nodes.reserve(2 * bx.size() + 1);
    build_rec(0, static_cast<uint32_t>(bx.size()));
    enabled = true;
  }
  int build_rec(uint32_t first, uint32_t count) {
    Node nd;
    for (int k = 0; k < 3; ++k) nd.b.lo[k] = INFINITY, nd.b.hi[k] = -INFINITY;
    double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = first; i < first + count; ++i) {
      const Box& b = boxes[idx[i]];
      for (int k = 0; k < 3; ++k) {
        nd.b.lo[k] = std::min(nd.b.lo[k], b.lo[k]);
        nd.b.hi[k] = std::max(nd.b.hi[k], b.hi[k]);
        const double c = 0.5 * (b.lo[k] + b.hi[k]);
        clo[k] = std::min(clo[k], c);
        chi[k] = std::max(chi[k], c);
      }
    }
    const int me = static_cast<int>(nodes.size());
    nodes.push_back(nd);
    if (count <= 4) {
      nodes[me].first = first;
      nodes[me].count = count;
      return me;
    }
    int ax = 0;
    for (int k = 1; k < 3; ++k)
      if (chi[k] - clo[k] > chi[ax] - clo[ax]) ax = k;
    const uint32_t mid = first + count / 2;
    std::nth_element(idx.begin() + first, idx.begin() + mid, idx.begin() + first + count, [&](uint32_t a, uint32_t b) {
      const double ca = boxes[a].lo[ax] + boxes[a].hi[ax], cb = boxes[b].lo[ax] + boxes[b].hi[ax];
      return ca < cb || (ca == cb && a < b);
    });
    const int l = build_rec(first, mid - first);
    const int r = build_rec(mid, first + count - mid);
    nodes[me].left = l;
    nodes[me].right = r;
    return me;
  }
  static bool ray_box(const Box& b, const double o[3], const double inv[3]) {
    double t0 = 0.0, t1 = INFINITY;
    for (int k = 0; k < 3; ++k) {
      double a = (b.lo[k] - o[k]) * inv[k], c = (b.hi[k] - o[k]) * inv[k];
      if (a > c) std::swap(a, c);
      if (std::isnan(a)) a = -INFINITY;
      if (std::isnan(c)) c = INFINITY;
      t0 = std::max(t0, a);
      t1 = std::min(t1, c);
    }
    return t0 <= t1;
  }
  void ray(F3 of, F3 df, std::vector<uint32_t>& out) const {
    const double o[3] = {of.x, of.y, of.z};
    const double dd[3] = {df.x, df.y, df.z};
    double inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = 1.0 / (std::fabs(dd[k]) < 1e-300 ? std::copysign(1e-300, dd[k]) : dd[k]);
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const Node& n = nodes[stack[--sp]];
      if (!ray_box(n.b, o, inv)) continue;
      if (n.left < 0) {
        for (uint32_t i = n.first; i < n.first + n.count; ++i) out.push_back(idx[i]);
      } else {
        stack[sp++] = n.left;
        stack[sp++] = n.right;
      }
    }
  }
  void point(F3 p, std::vector<uint32_t>& out) const {
    const double x[3] = {p.x, p.y, p.z};
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const Node& n = nodes[stack[--sp]];
      bool in = true;
      for (int k = 0; k < 3; ++k) in = in && x[k] >= n.b.lo[k] && x[k] <= n.b.hi[k];
      if (!in) continue;
      if (n.left < 0) {
        for (uint32_t i = n.first; i < n.first + n.count; ++i) out.push_back(idx[i]);
      } else {
        stack[sp++] = n.left;
        stack[sp++] = n.right;
      }
    }
  }
};

// Morton code of the reference's host sort (include/thesis/host/utils/math.h:103-131).
inline uint32_t expand_bits(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}
inline uint32_t morton3d(F3 pos, F3 scene_min, F3 inv_extent) {
  const F3 n = (pos - scene_min) * inv_extent;
  auto q = [](float x) { return static_cast<uint32_t>(std::min(std::max(x, 0.0f), 1.0f) * 1023.0f); };
  return (expand_bits(q(n.z)) << 2) | (expand_bits(q(n.y)) << 1) | expand_bits(q(n.x));
}

struct Scene {
  std::vector<Prim> prims;
  std::vector<uint32_t> orig;  // scene order -> caller's index (keys the free-flight draws)
  // FP64 geometry for the closed-form oracle.
  std::vector<double> c64, W64, norm64;  // centre, whitening matrix (row-major 3x3), M/(2 pi prod s)
  std::vector<Box> boxes;
  Bvh bvh;
};

struct Params {
  uint32_t width, height, spp, seed, max_bounces, rr_depth;
  float rr_max_survival, hg_g, firefly_clamp, filter_stddev;
  int32_t nee_mode;  // 0 MIS, 1 phase, 2 RIS, 3 none
  uint32_t ris_k;
  int32_t rng_mode;  // 0 reference sequential, 1 keyed (GPU)
  // HG pre-fold
  int hg_iso;
  float hg_g_eff, hg_one_plus_g2, hg_one_minus_g2, hg_neg_inv_2g, hg_coeff;
};

void fold_hg(Params& p) {  // renderer.cpp:224-235
  const float g = p.hg_g, ag = g < 0.f ? -g : g;
  p.hg_iso = ag < 1e-3f;
  p.hg_g_eff = -g;
  const float g2 = g * g;
  p.hg_one_plus_g2 = 1.0f + g2;
  p.hg_one_minus_g2 = 1.0f - g2;
  p.hg_neg_inv_2g = p.hg_iso ? 0.0f : (-0.5f / p.hg_g_eff);
  p.hg_coeff = ONE_OVER_FOUR_PI_F * p.hg_one_minus_g2;
}

float hg_eval_cos(const Params& P, float c) {
  if (P.hg_iso) return ONE_OVER_FOUR_PI_F;
  const float denom = std::fmaf(-2.0f * P.hg_g, c, P.hg_one_plus_g2);
  const float is = rsqrt_(denom);
  return P.hg_coeff * (is * is * is);
}
void onb(F3 n, F3& tx, F3& ty) {
  const float sign = std::copysign(1.0f, n.z);
  const float a = -1.0f / (sign + n.z);
  const float b = n.x * n.y * a;
  tx = mk(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
  ty = mk(b, sign + n.y * n.y * a, -n.y);
}
F3 hg_sample(const Params& P, F3 wi, Pcg& rng, float& pdf) {
  const float u0 = rng.uniform(), u1 = rng.uniform();
  float ct;
  if (P.hg_iso) {
    ct = std::fmaf(-2.0f, u0, 1.0f);
  } else {
    const float g = P.hg_g_eff;
    const float inner = std::fmaf(-2.0f, u0, 1.0f);
    const float denom = std::fmaf(g, inner, 1.0f);
    const float sq = P.hg_one_minus_g2 * rcp(denom);
    ct = P.hg_neg_inv_2g * std::fmaf(-sq, sq, P.hg_one_plus_g2);
  }
  const float st = std::sqrt(std::max(0.0f, 1.0f - ct * ct));
  const float phi = TWO_PI_F * u1;
  const F3 wl = mk(st * std::cos(phi), st * std::sin(phi), ct);
  F3 ex, ey;
  onb(wi, ex, ey);
  pdf = hg_eval_cos(P, ct);
  return wl.x * ex + wl.y * ey + wl.z * wi;
}

// ---------------------------------------------------------------------------------------------
// the path (raygen.cuh:72-230)
// ---------------------------------------------------------------------------------------------
struct Tracer {
  const Scene& S;
  const Env& E;
  const Camera& C;
  const Params& P;
  std::vector<uint32_t> cand;
  double scan_s = 0.0;  // thread time in the bounce-0 origin-inside scan (timed renders only)
  bool time_scan = false;

  void candidates_ray(F3 o, F3 d) {
    cand.clear();
    if (S.bvh.enabled) {
      S.bvh.ray(o, d, cand);
      std::sort(cand.begin(), cand.end());
    } else {
      cand.resize(S.prims.size());
      std::iota(cand.begin(), cand.end(), 0u);
    }
  }
  void candidates_point(F3 p) {
    cand.clear();
    if (S.bvh.enabled) {
      S.bvh.point(p, cand);
      std::sort(cand.begin(), cand.end());
    } else {
      cand.resize(S.prims.size());
      std::iota(cand.begin(), cand.end(), 0u);
    }
  }

  // compute_transmittance_to_env (sampling.cuh:548-583)
  float transmittance(F3 o, F3 d, const std::vector<uint32_t>& active) {
    float acc = 0.f;
    for (uint32_t i : active) {
      const Prim& p = S.prims[i];
      const float te = exit_from_inside(o, d, p);
      if (te > 0.f && te < INF_F) {
        acc += p.optical_depth(o, d, 0.f, te);
        if (acc >= MAX_OPTICAL_DEPTH) return 0.f;
      }
    }
    candidates_ray(o, d);
    for (uint32_t i : cand) {
      const Prim& p = S.prims[i];
      float t_entry;
      if (!entry_3sigma(o, d, p, t_entry)) continue;
      const F3 w = p.dir_local(d);
      const float t_exit = exit_from_entry(o, d, t_entry, p, length2(w));
      if (t_exit > t_entry && t_exit < INF_F) acc += p.optical_depth(o, d, t_entry, t_exit);
    }
    return std::exp(-acc);
  }

  F3 albedo_at(F3 pos, const std::vector<uint32_t>& active) {  // evaluate_albedo (:257-283)
    F3 a = mk(0.f, 0.f, 0.f);
    float w = 0.f;
    for (uint32_t i : active) {
      const Prim& p = S.prims[i];
      const float wt = p.mass * p.pdf(pos);
      a = a + p.albedo * wt;
      w += wt;
    }
    if (w <= 0.f) return mk(0.f, 0.f, 0.f);
    return a * rcp(w);
  }

  F3 trace(uint32_t px, uint32_t py, uint64_t sample) {
    const uint64_t pix = static_cast<uint64_t>(py) * P.width + px;
    Pcg rng = pcg_init(P.seed, seq_hash(pix * P.spp + sample));
    F3 o, d;
    camera_ray(C, P.filter_stddev, px, py, rng, o, d);
    F3 thr = mk(1.f, 1.f, 1.f), rad = mk(0.f, 0.f, 0.f);
    std::vector<uint32_t> active, origin_inside, next_active;
    struct Hit {
      float t;
      uint32_t i;
    };
    std::vector<Hit> hits;
    const bool alias = P.rng_mode == 1;
    for (uint32_t bounce = 0; bounce < P.max_bounces; ++bounce) {
      if (bounce == 0) {  // build_origin_inside_set (:322-341)
        const double ts = time_scan ? omp_get_wtime() : 0.0;
        active.clear();
        for (uint32_t i = 0; i < S.prims.size(); ++i)
          if (point_inside(o, S.prims[i])) active.push_back(i);
        if (time_scan) scan_s += omp_get_wtime() - ts;
      }
      origin_inside = active;
      hits.clear();  // collect_hits (:287-305), canonical order = ascending entry distance
      candidates_ray(o, d);
      for (uint32_t i : cand) {
        float te;
        if (entry_3sigma(o, d, S.prims[i], te)) hits.push_back({te, i});
      }
      std::sort(hits.begin(), hits.end(), [](const Hit& a, const Hit& b) { return a.t < b.t || (a.t == b.t && a.i < b.i); });
      bool scattered = false;
      float tmin = INF_F;
      uint64_t key = 0;
      if (alias) {
        const uint32_t hi = rng.next(), lo = rng.next();
        key = (static_cast<uint64_t>(hi) << 32) | lo;
      }
      auto tau_of = [&](uint32_t i) {
        float chi;
        if (alias) chi = static_cast<float>(keyed_u32(key, S.orig[i])) * 2.3283064365386963e-10f;
        else chi = rng.uniform();
        return -std::log(std::max(1.0f - chi, 1e-10f));
      };
      if (!(hits.empty() && active.empty())) {
        // argmin_scatter_distance (:350-415)
        for (uint32_t i : active) {
          const Prim& p = S.prims[i];
          const float te = exit_from_inside(o, d, p);
          const float ts = p.inv_cdf(o, d, tau_of(i));
          if (ts >= 0.f && ts < tmin && ts <= te) tmin = ts;
        }
        for (const Hit& h : hits) {
          const Prim& p = S.prims[h.i];
          const float tau = tau_of(h.i);
          float ts = p.inv_cdf_span(o, d, h.t, tau);
          if (ts >= 0.f && ts < h.t) ts = h.t;
          if (ts >= 0.f && ts < tmin) {
            const F3 w = p.dir_local(d);
            const float te = exit_from_entry(o, d, h.t, p, length2(w));
            if (ts <= te) tmin = ts;
          }
        }
        scattered = tmin < INF_F;
      }
      F3 pos = o, dir_next = d;
      if (scattered) {
        // rebuild_active_set_at_scatter (:422-458)
        next_active.clear();
        for (uint32_t i : active) {
          const float te = exit_from_inside(o, d, S.prims[i]);
          if (tmin <= te) next_active.push_back(i);
        }
        for (const Hit& h : hits) {
          if (h.t > tmin) continue;
          const Prim& p = S.prims[h.i];
          const F3 w = p.dir_local(d);
          const float te = exit_from_entry(o, d, h.t, p, length2(w));
          if (tmin <= te && std::find(next_active.begin(), next_active.end(), h.i) == next_active.end())
            next_active.push_back(h.i);
        }
        active = next_active;
        pos = o + tmin * d;
        float pdf;
        dir_next = hg_sample(P, d, rng, pdf);
      } else {
        active.clear();
      }
      if (bounce == 0) {  // analytic direct (raygen.cuh:148-160)
        const float T = transmittance(o, d, origin_inside);
        rad = rad + thr * T * env_lookup(E, d);
      }
      if (!scattered) {
        if (P.nee_mode == 3 && bounce > 0) rad = rad + thr * env_lookup(E, d);
        break;
      }
      const F3 albedo = albedo_at(pos, active);
      const F3 base = thr * albedo;
      if (P.nee_mode == 0) {
        float pa;
        const F3 wa = hg_sample(P, d, rng, pa);
        const float pb_a = env_pdf(E, wa, alias);
        const float sa = pa + pb_a;
        const float w_a = sa > 0.f ? pa / sa : 0.f;
        const F3 ea = env_lookup(E, wa);
        const float Ta = transmittance(pos, wa, active);
        rad = rad + base * ea * Ta * w_a;
        const EnvSample b = env_sample(E, rng, alias);
        const float ph_b = hg_eval_cos(P, dot(d, b.wo));
        const float sb = b.pdf + ph_b;
        const float w_b = sb > 0.f ? b.pdf / sb : 0.f;
        const F3 eb = env_lookup(E, b.wo);
        const float Tb = transmittance(pos, b.wo, active);
        rad = rad + base * eb * Tb * w_b * ph_b * rcp(b.pdf);
      } else if (P.nee_mode == 1) {
        float pa;
        const F3 wa = hg_sample(P, d, rng, pa);
        const F3 ea = env_lookup(E, wa);
        rad = rad + base * ea * transmittance(pos, wa, active);
      } else if (P.nee_mode == 2) {
        const F3 luma = mk(0.2126f, 0.7152f, 0.0722f);
        float wsum = 0.f;
        F3 ydir = mk(0.f, 0.f, 0.f), yenv = mk(0.f, 0.f, 0.f);
        for (uint32_t k = 0; k < P.ris_k; ++k) {
          const EnvSample c = env_sample(E, rng, alias);
          if (c.pdf <= 0.f) continue;
          const F3 ec = env_lookup(E, c.wo);
          const float lc = dot(ec, luma);
          const float w = hg_eval_cos(P, dot(d, c.wo)) * lc * rcp(c.pdf);
          if (!(w > 0.f)) continue;
          wsum += w;
          if (rng.uniform() * wsum < w) ydir = c.wo, yenv = ec;
        }
        if (wsum > 0.f) {
          const float ly = dot(yenv, luma);
          if (ly > 0.f) {
            const float T = transmittance(pos, ydir, active);
            const float Wr = wsum * rcp(static_cast<float>(P.ris_k));
            rad = rad + base * (yenv * rcp(ly)) * T * Wr;
          }
        }
      }
      thr = thr * albedo;
      if (bounce >= P.rr_depth) {
        const float ps = std::min(P.rr_max_survival, maxc(thr));
        if (rng.uniform() > ps || ps <= 0.f) break;
        thr = thr * rcp(ps);
      }
      if (maxc(thr) < MIN_THROUGHPUT) break;
      if (!std::isfinite(sumc(thr))) break;
      o = pos;
      d = dir_next;
    }
    if (P.firefly_clamp > 0.f) {
      const float lum = dot(rad, mk(0.2126f, 0.7152f, 0.0722f));
      if (lum > P.firefly_clamp) rad = rad * (P.firefly_clamp * rcp(lum));
    }
    if (!std::isfinite(sumc(rad))) rad = mk(0.f, 0.f, 0.f);
    return rad;
  }
};

// ---------------------------------------------------------------------------------------------
// FP64 closed-form transmittance (cloud_bruteforce_transmittance.py:48-60)
// ---------------------------------------------------------------------------------------------
double tau64(const Scene& S, const double o[3], const double d[3], const std::vector<uint32_t>* cand) {
  double tau = 0.0;
  const size_t n = cand ? cand->size() : S.prims.size();
  for (size_t k = 0; k < n; ++k) {
    const size_t i = cand ? (*cand)[k] : k;
    const double* c = &S.c64[3 * i];
    const double* W = &S.W64[9 * i];
    const double D[3] = {o[0] - c[0], o[1] - c[1], o[2] - c[2]};
    double p[3], w[3];
    for (int r = 0; r < 3; ++r) {
      p[r] = W[3 * r] * D[0] + W[3 * r + 1] * D[1] + W[3 * r + 2] * D[2];
      w[r] = W[3 * r] * d[0] + W[3 * r + 1] * d[1] + W[3 * r + 2] * d[2];
    }
    const double a = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    const double pw = p[0] * w[0] + p[1] * w[1] + p[2] * w[2];
    const double pp = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
    const double b = 2.0 * pw;
    const double disc = b * b - 4.0 * a * (pp - 9.0);
    if (!(disc > 0.0)) continue;
    const double sq = std::sqrt(disc);
    const double ta = (-b - sq) / (2.0 * a), tb = (-b + sq) / (2.0 * a);
    const double t0 = std::max(ta, 0.0), t1 = tb;
    if (!(t1 > t0)) continue;
    const double tc = -pw / a;
    const double perp2 = pp - pw * pw / a;
    const double wl = std::sqrt(a);
    const double contrib = S.norm64[i] * std::exp(-0.5 * perp2) / wl * 0.5 *
                           (std::erf((t1 - tc) * wl / std::sqrt(2.0)) - std::erf((t0 - tc) * wl / std::sqrt(2.0)));
    tau += std::max(contrib, 0.0);
  }
  return tau;
}

}  // namespace

// =============================================================================================
// C ABI of the oracle (ctypes from oracle/oracle.py)
// =============================================================================================
extern "C" {

struct OrScene;

// Primitive records in the reference's 80-byte layout (primitive.h:47-61):
// center[3], rot_quat (s, u[3]) = conjugate, rcp_scale[3], density_norm_factor,
// inv_cdf_factor, albedo[3], optical_thickness, scale[3]  -> 20 floats per Gaussian.
void* or_scene_create(uint32_t n, const float* mean, const float* scale, const float* quat_wxyz,
                      const float* density, const float* albedo, float sigma_multiplier,
                      int scale_is_log, int use_bvh, float* out_records /* 20n or NULL */) {
  auto* S = new Scene();
  S->prims.resize(n);
  S->c64.resize(3ull * n);
  S->W64.resize(9ull * n);
  S->norm64.resize(n);
  S->boxes.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    float sx = scale[3 * i], sy = scale[3 * i + 1], sz = scale[3 * i + 2];
    if (scale_is_log) sx = std::exp(sx), sy = std::exp(sy), sz = std::exp(sz);
    const float w = quat_wxyz[4 * i], x = quat_wxyz[4 * i + 1], y = quat_wxyz[4 * i + 2], z = quat_wxyz[4 * i + 3];
    // UnitQuaternion::from (quat.h:55-58): rlength(float4(w,x,y,z))
    const float r = 1.0f / std::sqrt(std::fmaf(w, w, std::fmaf(x, x, std::fmaf(y, y, z * z))));
    const float qw = w * r, qx = x * r, qy = y * r, qz = z * r;
    auto clampa = [](float v) { return !std::isfinite(v) ? 0.f : (v < 0.f ? 0.f : (v > 1.f ? 1.f : v)); };
    Prim& p = S->prims[i];
    p.center = mk(mean[3 * i], mean[3 * i + 1], mean[3 * i + 2]);
    p.rot = Quat{qw, mk(-qx, -qy, -qz)};  // from_forward_quat stores the conjugate
    p.scale = mk(sx, sy, sz);
    p.rcp_scale = mk(rcp(sx), rcp(sy), rcp(sz));
    p.dnf = ONE_OVER_TWO_PI_POW_3_2_F * (p.rcp_scale.x * p.rcp_scale.y * p.rcp_scale.z);
    p.mass = density[i] * sigma_multiplier;
    p.icf = p.mass * p.dnf * ROOT_HALF_PI_F;
    p.albedo = albedo ? mk(clampa(albedo[3 * i]), clampa(albedo[3 * i + 1]), clampa(albedo[3 * i + 2])) : mk(0.f, 0.f, 0.f);
    if (out_records) {
      float* o = out_records + 20ull * i;
      const float v[20] = {p.center.x, p.center.y, p.center.z, p.rot.s, p.rot.u.x, p.rot.u.y, p.rot.u.z,
                           p.rcp_scale.x, p.rcp_scale.y, p.rcp_scale.z, p.dnf, p.icf, p.albedo.x, p.albedo.y,
                           p.albedo.z, p.mass, p.scale.x, p.scale.y, p.scale.z, 0.f};
      std::memcpy(o, v, sizeof(v));
    }
    // FP64 geometry from the same inputs.
    const double dw = qw, dx = qx, dy = qy, dz = qz;
    const double R[3][3] = {{1 - 2 * (dy * dy + dz * dz), 2 * (dx * dy - dw * dz), 2 * (dx * dz + dw * dy)},
                            {2 * (dx * dy + dw * dz), 1 - 2 * (dx * dx + dz * dz), 2 * (dy * dz - dw * dx)},
                            {2 * (dx * dz - dw * dy), 2 * (dy * dz + dw * dx), 1 - 2 * (dx * dx + dy * dy)}};
    const double s[3] = {sx, sy, sz};
    for (int rr = 0; rr < 3; ++rr)
      for (int cc = 0; cc < 3; ++cc) S->W64[9ull * i + 3 * rr + cc] = R[cc][rr] / s[rr];
    S->c64[3ull * i] = mean[3 * i];
    S->c64[3ull * i + 1] = mean[3 * i + 1];
    S->c64[3ull * i + 2] = mean[3 * i + 2];
    S->norm64[i] = static_cast<double>(density[i]) * static_cast<double>(sigma_multiplier) /
                   (2.0 * 3.14159265358979323846 * s[0] * s[1] * s[2]);
    Box& b = S->boxes[i];
    for (int k = 0; k < 3; ++k) {
      const double e = 3.0 * std::sqrt(std::pow(R[k][0] * s[0], 2) + std::pow(R[k][1] * s[1], 2) + std::pow(R[k][2] * s[2], 2));
      const double pad = e * 1e-4 + 1e-6;
      b.lo[k] = mean[3 * i + k] - e - pad;
      b.hi[k] = mean[3 * i + k] + e + pad;
    }
  }
  // The reference renders the Gaussians in its host Morton order (renderer.cpp:91-121: 30-bit
  // codes of the centres over their bounds); its origin-inside scan draws in that order.  Ties
  // keep the caller's order here (the reference's std::sort leaves them unspecified).
  S->orig.resize(n);
  std::iota(S->orig.begin(), S->orig.end(), 0u);
  if (n > 1) {
    F3 mn = mk(FLT_MAX, FLT_MAX, FLT_MAX), mx = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (const Prim& p : S->prims) {
      mn = mk(std::min(mn.x, p.center.x), std::min(mn.y, p.center.y), std::min(mn.z, p.center.z));
      mx = mk(std::max(mx.x, p.center.x), std::max(mx.y, p.center.y), std::max(mx.z, p.center.z));
    }
    const F3 ext = mx - mn;
    const F3 inv = mk(1.0f / std::max(ext.x, 1e-30f), 1.0f / std::max(ext.y, 1e-30f), 1.0f / std::max(ext.z, 1e-30f));
    std::vector<uint32_t> code(n);
    for (uint32_t i = 0; i < n; ++i) code[i] = morton3d(S->prims[i].center, mn, inv);
    std::stable_sort(S->orig.begin(), S->orig.end(), [&](uint32_t a, uint32_t b) { return code[a] < code[b]; });
    Scene T;
    T.prims.resize(n), T.c64.resize(3ull * n), T.W64.resize(9ull * n), T.norm64.resize(n), T.boxes.resize(n);
    for (uint32_t k = 0; k < n; ++k) {
      const uint32_t i = S->orig[k];
      T.prims[k] = S->prims[i];
      T.norm64[k] = S->norm64[i];
      T.boxes[k] = S->boxes[i];
      for (int c = 0; c < 3; ++c) T.c64[3ull * k + c] = S->c64[3ull * i + c];
      for (int c = 0; c < 9; ++c) T.W64[9ull * k + c] = S->W64[9ull * i + c];
    }
    S->prims.swap(T.prims), S->c64.swap(T.c64), S->W64.swap(T.W64), S->norm64.swap(T.norm64), S->boxes.swap(T.boxes);
  }
  if (use_bvh) S->bvh.build(S->boxes);
  return S;
}

void or_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

// Whitened position and direction of (pos, dir) for the caller's Gaussian `index`, and
// point_inside_bvh_bound(pos): out7 = pos_local[3], dir_local[3], inside.
void or_transform(void* sv, uint32_t index, const float* pos, const float* dir, float* out7) {
  const Scene& S = *static_cast<Scene*>(sv);
  uint32_t k = 0;
  while (k < S.orig.size() && S.orig[k] != index) ++k;
  const Prim& p = S.prims[k];
  const F3 a = p.pos_local(mk(pos[0], pos[1], pos[2])), b = p.dir_local(mk(dir[0], dir[1], dir[2]));
  out7[0] = a.x, out7[1] = a.y, out7[2] = a.z, out7[3] = b.x, out7[4] = b.y, out7[5] = b.z;
  out7[6] = point_inside(mk(pos[0], pos[1], pos[2]), p) ? 1.0f : 0.0f;
}

uint32_t or_morton3d(const float* pos, const float* scene_min, const float* inv_extent) {
  return morton3d(mk(pos[0], pos[1], pos[2]), mk(scene_min[0], scene_min[1], scene_min[2]),
                  mk(inv_extent[0], inv_extent[1], inv_extent[2]));
}

// Scene order (the reference's Morton order) as caller indices.
void or_scene_order(void* sv, uint32_t* out) {
  const Scene& S = *static_cast<Scene*>(sv);
  std::copy(S.orig.begin(), S.orig.end(), out);
}

void* or_env_create(const float* rgb, uint32_t W, uint32_t H, uint32_t ch) {
  auto* e = new Env();
  build_env(rgb, W, H, ch, *e);
  return e;
}
void or_env_destroy(void* e) { delete static_cast<Env*>(e); }

// Env tables: joint[W*H], marg_cdf[H], cond_cdf[W*H], total; alias (p, a) for rows and marginal.
void or_env_tables(void* ev, float* joint, float* marg_cdf, float* cond_cdf, float* total, float* alias_cond_p,
                   uint32_t* alias_cond_a, float* alias_marg_p, uint32_t* alias_marg_a, double* total64) {
  const Env& e = *static_cast<Env*>(ev);
  const size_t n = static_cast<size_t>(e.W) * e.H;
  if (joint) std::memcpy(joint, e.joint.data(), n * 4);
  if (marg_cdf) std::memcpy(marg_cdf, e.marg_cdf.data(), e.H * 4);
  if (cond_cdf) std::memcpy(cond_cdf, e.cond_cdf.data(), n * 4);
  if (total) *total = e.total;
  if (alias_cond_p) std::memcpy(alias_cond_p, e.alias_cond_p.data(), n * 4);
  if (alias_cond_a) std::memcpy(alias_cond_a, e.alias_cond_a.data(), n * 4);
  if (alias_marg_p) std::memcpy(alias_marg_p, e.alias_marg_p.data(), e.H * 4);
  if (alias_marg_a) std::memcpy(alias_marg_a, e.alias_marg_a.data(), e.H * 4);
  if (total64) *total64 = e.total64;
}

// Env lookup for n directions -> rgb[3n].
void or_env_lookup(void* ev, const float* dirs, uint32_t n, float* out) {
  const Env& e = *static_cast<Env*>(ev);
  for (uint32_t i = 0; i < n; ++i) {
    const F3 c = env_lookup(e, mk(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
    out[3 * i] = c.x, out[3 * i + 1] = c.y, out[3 * i + 2] = c.z;
  }
}

// Camera build -> 16 floats: eye[3], p00_rel[3], du[3], dv[3], view_dir[3], ortho.
void or_camera(const float* eye, const float* lookat, const float* up, float vfov, float ortho_h, int ortho,
               uint32_t W, uint32_t H, float* out16) {
  Camera c;
  build_camera(eye, lookat, up, vfov, ortho_h, ortho, W, H, c);
  const float v[16] = {c.eye.x, c.eye.y, c.eye.z, c.p00.x, c.p00.y, c.p00.z, c.du.x, c.du.y,
                       c.du.z, c.dv.x, c.dv.y, c.dv.z, c.view_dir.x, c.view_dir.y, c.view_dir.z,
                       static_cast<float>(c.ortho)};
  std::memcpy(out16, v, sizeof(v));
}

// Camera rays of (pixel, sample) pairs: origins[3n], dirs[3n] (the reference's jitter stream).
void or_camera_rays(const float* cam16, uint32_t W, uint32_t spp, uint32_t seed, float filter_stddev,
                    const uint32_t* px, const uint32_t* py, const uint32_t* sample, uint32_t n, float* o,
                    float* d) {
  Camera c{mk(cam16[0], cam16[1], cam16[2]), mk(cam16[3], cam16[4], cam16[5]), mk(cam16[6], cam16[7], cam16[8]),
           mk(cam16[9], cam16[10], cam16[11]), mk(cam16[12], cam16[13], cam16[14]), static_cast<int>(cam16[15])};
  for (uint32_t i = 0; i < n; ++i) {
    const uint64_t pix = static_cast<uint64_t>(py[i]) * W + px[i];
    Pcg rng = pcg_init(seed, seq_hash(pix * spp + sample[i]));
    F3 oo, dd;
    camera_ray(c, filter_stddev, px[i], py[i], rng, oo, dd);
    o[3 * i] = oo.x, o[3 * i + 1] = oo.y, o[3 * i + 2] = oo.z;
    d[3 * i] = dd.x, d[3 * i + 1] = dd.y, d[3 * i + 2] = dd.z;
  }
}

// PCG32 stream: first `count` outputs of init(seed, sequence) (no hash applied).
void or_pcg32(uint64_t seed, uint64_t sequence, uint32_t count, uint32_t* out) {
  Pcg r = pcg_init(seed, sequence);
  for (uint32_t i = 0; i < count; ++i) out[i] = r.next();
}
uint64_t or_seq_hash(uint64_t x) { return seq_hash(x); }

// FP64 closed-form transmittance of n rays over [0, inf).
void or_transmittance_fp64(void* sv, const float* o, const float* d, uint32_t n, double* out_T, double* out_tau) {
  const Scene& S = *static_cast<Scene*>(sv);
#pragma omp parallel
  {
    std::vector<uint32_t> cand;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      const double oo[3] = {o[3 * i], o[3 * i + 1], o[3 * i + 2]}, dd[3] = {d[3 * i], d[3 * i + 1], d[3 * i + 2]};
      double tau;
      if (S.bvh.enabled) {
        cand.clear();
        S.bvh.ray(mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]), cand);
        tau = tau64(S, oo, dd, &cand);
      } else {
        tau = tau64(S, oo, dd, nullptr);
      }
      if (out_tau) out_tau[i] = tau;
      if (out_T) out_T[i] = std::exp(-tau);
    }
  }
}

// FP32 reference-order transmittance (compute_transmittance_to_env with the origin-inside set
// from a full scan) of n rays.
void or_transmittance_fp32(void* sv, const float* o, const float* d, uint32_t n, float* out_T) {
  const Scene& S = *static_cast<Scene*>(sv);
  Env e;
  Camera c{};
  Params p{};
#pragma omp parallel
  {
    Tracer t{S, e, c, p, {}};
    std::vector<uint32_t> active;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      const F3 oo = mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), dd = mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
      active.clear();
      for (uint32_t k = 0; k < S.prims.size(); ++k)
        if (point_inside(oo, S.prims[k])) active.push_back(k);
      out_T[i] = t.transmittance(oo, dd, active);
    }
  }
}

// evaluate_albedo (sampling.cuh:257-283) over the Gaussians containing each point
// (point_inside_bvh_bound), FP32; out_rgb[3n], out_count[n].
void or_albedo_at(void* sv, const float* pts, uint32_t n, float* out_rgb, uint32_t* out_count) {
  const Scene& S = *static_cast<Scene*>(sv);
  Env e;
  Camera c{};
  Params p{};
#pragma omp parallel
  {
    Tracer t{S, e, c, p, {}};
    std::vector<uint32_t> active;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      const F3 x = mk(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
      t.candidates_point(x);
      active.clear();
      for (uint32_t k : t.cand)
        if (point_inside(x, S.prims[k])) active.push_back(k);
      const F3 a = t.albedo_at(x, active);
      out_rgb[3 * i] = a.x, out_rgb[3 * i + 1] = a.y, out_rgb[3 * i + 2] = a.z;
      out_count[i] = static_cast<uint32_t>(active.size());
    }
  }
}

// Absorption-only image in FP64: mean over samples [0, spp) of T(camera ray) x env(dir) with the
// reference's jitter stream.  out_rgb: W*H*3 doubles.
void or_render_absorption_fp64(void* sv, void* ev, const float* cam16, uint32_t W, uint32_t H, uint32_t spp,
                               uint32_t seed, double* out_rgb) {
  const Scene& S = *static_cast<Scene*>(sv);
  const Env& E = *static_cast<Env*>(ev);
  Camera c{mk(cam16[0], cam16[1], cam16[2]), mk(cam16[3], cam16[4], cam16[5]), mk(cam16[6], cam16[7], cam16[8]),
           mk(cam16[9], cam16[10], cam16[11]), mk(cam16[12], cam16[13], cam16[14]), static_cast<int>(cam16[15])};
#pragma omp parallel
  {
    std::vector<uint32_t> cand;
#pragma omp for schedule(dynamic, 16)
    for (int64_t pix = 0; pix < static_cast<int64_t>(W) * H; ++pix) {
      const uint32_t px = static_cast<uint32_t>(pix % W), py = static_cast<uint32_t>(pix / W);
      double acc[3] = {0, 0, 0};
      for (uint32_t s = 0; s < spp; ++s) {
        Pcg rng = pcg_init(seed, seq_hash(static_cast<uint64_t>(pix) * spp + s));
        F3 o, d;
        camera_ray(c, 0.0f, px, py, rng, o, d);
        const double oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
        double tau;
        if (S.bvh.enabled) {
          cand.clear();
          S.bvh.ray(o, d, cand);
          tau = tau64(S, oo, dd, &cand);
        } else {
          tau = tau64(S, oo, dd, nullptr);
        }
        const double T = std::exp(-tau);
        const F3 env = env_lookup(E, d);
        acc[0] += T * env.x, acc[1] += T * env.y, acc[2] += T * env.z;
      }
      for (int k = 0; k < 3; ++k) out_rgb[3 * pix + k] = acc[k] / spp;
    }
  }
}

// Full FP32 path tracer over pixel rows [y0, y1) (all columns), samples [s0, s1) of a
// params.spp-sample render.  out_rgb: (y1-y0)*W*3 floats holding the per-pixel mean over those
// samples.  params: uint32 fields then floats, see oracle.py.  Returns elapsed seconds.
double or_render(void* sv, void* ev, const float* cam16, const uint32_t* pu, const float* pf, uint32_t y0,
                 uint32_t y1, uint32_t s0, uint32_t s1, int n_threads, float* out_rgb) {
  const Scene& S = *static_cast<Scene*>(sv);
  const Env& E = *static_cast<Env*>(ev);
  Camera c{mk(cam16[0], cam16[1], cam16[2]), mk(cam16[3], cam16[4], cam16[5]), mk(cam16[6], cam16[7], cam16[8]),
           mk(cam16[9], cam16[10], cam16[11]), mk(cam16[12], cam16[13], cam16[14]), static_cast<int>(cam16[15])};
  Params P{};
  P.width = pu[0], P.height = pu[1], P.spp = pu[2], P.seed = pu[3], P.max_bounces = pu[4], P.rr_depth = pu[5];
  P.nee_mode = static_cast<int32_t>(pu[6]), P.ris_k = pu[7], P.rng_mode = static_cast<int32_t>(pu[8]);
  P.rr_max_survival = pf[0], P.hg_g = pf[1], P.firefly_clamp = pf[2], P.filter_stddev = pf[3];
  fold_hg(P);
  const uint32_t W = P.width;
  if (n_threads > 0) omp_set_num_threads(n_threads);
  const double t0 = omp_get_wtime();
#pragma omp parallel
  {
    Tracer t{S, E, c, P, {}};
#pragma omp for schedule(dynamic, 64)
    for (int64_t k = 0; k < static_cast<int64_t>(y1 - y0) * W; ++k) {
      const uint32_t px = static_cast<uint32_t>(k % W), py = y0 + static_cast<uint32_t>(k / W);
      double acc[3] = {0, 0, 0};
      for (uint32_t s = s0; s < s1; ++s) {
        const F3 L = t.trace(px, py, s);
        acc[0] += L.x, acc[1] += L.y, acc[2] += L.z;
      }
      const double inv = 1.0 / static_cast<double>(s1 - s0);
      for (int j = 0; j < 3; ++j) out_rgb[3 * k + j] = static_cast<float>(acc[j] * inv);
    }
  }
  return omp_get_wtime() - t0;
}

// The same path tracer over a list of n pixels (px[i], py[i]), samples [s0, s1) each: the CPU
// baseline's bounded sample of a workload.  out_rgb: n*3 per-pixel means.  out_times[0] = the
// threads' total time in trace(), out_times[1] = their time in the bounce-0 origin-inside scan
// (build_origin_inside_set, sampling.cuh:322-341: every Gaussian, every camera path).  Returns
// elapsed seconds.
double or_render_pixels(void* sv, void* ev, const float* cam16, const uint32_t* pu, const float* pf,
                        const uint32_t* px, const uint32_t* py, uint32_t n, uint32_t s0, uint32_t s1, int n_threads,
                        float* out_rgb, double* out_times) {
  const Scene& S = *static_cast<Scene*>(sv);
  const Env& E = *static_cast<Env*>(ev);
  Camera c{mk(cam16[0], cam16[1], cam16[2]), mk(cam16[3], cam16[4], cam16[5]), mk(cam16[6], cam16[7], cam16[8]),
           mk(cam16[9], cam16[10], cam16[11]), mk(cam16[12], cam16[13], cam16[14]), static_cast<int>(cam16[15])};
  Params P{};
  P.width = pu[0], P.height = pu[1], P.spp = pu[2], P.seed = pu[3], P.max_bounces = pu[4], P.rr_depth = pu[5];
  P.nee_mode = static_cast<int32_t>(pu[6]), P.ris_k = pu[7], P.rng_mode = static_cast<int32_t>(pu[8]);
  P.rr_max_survival = pf[0], P.hg_g = pf[1], P.firefly_clamp = pf[2], P.filter_stddev = pf[3];
  fold_hg(P);
  if (n_threads > 0) omp_set_num_threads(n_threads);
  double trace_total = 0.0, scan_total = 0.0;
  const double t0 = omp_get_wtime();
#pragma omp parallel reduction(+ : trace_total, scan_total)
  {
    Tracer t{S, E, c, P, {}};
    t.time_scan = true;
    const double tt = omp_get_wtime();
#pragma omp for schedule(dynamic, 4)
    for (int64_t k = 0; k < static_cast<int64_t>(n); ++k) {
      double acc[3] = {0, 0, 0};
      for (uint32_t s = s0; s < s1; ++s) {
        const F3 L = t.trace(px[k], py[k], s);
        acc[0] += L.x, acc[1] += L.y, acc[2] += L.z;
      }
      const double inv = 1.0 / static_cast<double>(s1 - s0);
      for (int j = 0; j < 3; ++j) out_rgb[3 * k + j] = static_cast<float>(acc[j] * inv);
    }
    trace_total += omp_get_wtime() - tt;
    scan_total += t.scan_s;
  }
  const double el = omp_get_wtime() - t0;
  if (out_times) {
    out_times[0] = trace_total;
    out_times[1] = scan_total;
  }
  return el;
}

// Adaptive-sampling test of one pixel (raygen.cuh:52-67, constants.cuh:202-211): with at least
// max(min_samples, 2) samples, converged when max over channels of
// sqrt(M2 * rcp(n - 1)) * rcp(max(mean, 1e-6)) is below the threshold; threshold <= 0 is off.
// max(a, b) is a > b ? a : b, as the reference's math::max.
static bool adaptive_converged(float threshold, uint32_t min_samples, uint32_t n, const float* mean,
                               const float* m2) {
  if (!(threshold > 0.0f) || n < min_samples || n < 2u) return false;
  auto mx = [](float a, float b) { return a > b ? a : b; };
  const float inv_n1 = 1.0f / static_cast<float>(n - 1u);
  float e[3];
  for (int k = 0; k < 3; ++k) e[k] = std::sqrt(m2[k] * inv_n1) * (1.0f / mx(mean[k], 1e-6f));
  return mx(mx(e[0], e[1]), e[2]) < threshold;
}

// One Welford step for the k-th sample (k = 1, 2, ...; raygen.cuh:214-222):
//   delta1 = L - mean;  mean += delta1 * rcp(k);  M2 += delta1 * (L - mean)
static inline void welford_update(float* m, float* q, const float* L, uint32_t k) {
  const float n_inv = 1.0f / static_cast<float>(k);
  for (int j = 0; j < 3; ++j) {
    const float d1 = L[j] - m[j];
    m[j] = m[j] + d1 * n_inv;
    q[j] = q[j] + d1 * (L[j] - m[j]);
  }
}

// io6 = mean[3], M2[3], updated by sample L3 as sample number k.
void or_welford_step(const float* L3, uint32_t k, float* io6) { welford_update(io6, io6 + 3, L3, k); }

// Flags of the adaptive-sampling test over n pixels' Welford states (mean3, m2_3, count).
void or_adaptive_converged(const float* mean3, const float* m2_3, const uint32_t* count, uint32_t n,
                           float threshold, uint32_t min_samples, uint8_t* out) {
  for (uint32_t i = 0; i < n; ++i)
    out[i] = adaptive_converged(threshold, min_samples, count[i], mean3 + 3ull * i, m2_3 + 3ull * i) ? 1 : 0;
}

// Progressive FP32 render into a Welford image (raygen.cuh:31-67 and :210-242): samples
// [s0, s1) in batches of `batch`; before each batch a pixel whose state passes the adaptive test
// skips it; otherwise each sample updates mean and M2 (welford_update) and the count, in sample
// order.  mean3 / m2_3 / count hold the whole image (W*H pixels) and are updated in place.  Returns
// elapsed seconds.
double or_render_welford(void* sv, void* ev, const float* cam16, const uint32_t* pu, const float* pf, uint32_t s0,
                         uint32_t s1, uint32_t batch, float threshold, uint32_t min_samples, int n_threads,
                         float* mean3, float* m2_3, uint32_t* count) {
  const Scene& S = *static_cast<Scene*>(sv);
  const Env& E = *static_cast<Env*>(ev);
  Camera c{mk(cam16[0], cam16[1], cam16[2]), mk(cam16[3], cam16[4], cam16[5]), mk(cam16[6], cam16[7], cam16[8]),
           mk(cam16[9], cam16[10], cam16[11]), mk(cam16[12], cam16[13], cam16[14]), static_cast<int>(cam16[15])};
  Params P{};
  P.width = pu[0], P.height = pu[1], P.spp = pu[2], P.seed = pu[3], P.max_bounces = pu[4], P.rr_depth = pu[5];
  P.nee_mode = static_cast<int32_t>(pu[6]), P.ris_k = pu[7], P.rng_mode = static_cast<int32_t>(pu[8]);
  P.rr_max_survival = pf[0], P.hg_g = pf[1], P.firefly_clamp = pf[2], P.filter_stddev = pf[3];
  fold_hg(P);
  const uint32_t W = P.width;
  if (batch == 0) batch = s1 - s0;
  if (n_threads > 0) omp_set_num_threads(n_threads);
  const double t0 = omp_get_wtime();
#pragma omp parallel
  {
    Tracer t{S, E, c, P, {}};
#pragma omp for schedule(dynamic, 16)
    for (int64_t k = 0; k < static_cast<int64_t>(P.height) * W; ++k) {
      const uint32_t px = static_cast<uint32_t>(k % W), py = static_cast<uint32_t>(k / W);
      float* m = mean3 + 3 * k;
      float* q = m2_3 + 3 * k;
      for (uint32_t b0 = s0; b0 < s1; b0 += batch) {
        const uint32_t b1 = std::min(s1, b0 + batch);
        if (adaptive_converged(threshold, min_samples, count[k], m, q)) continue;
        for (uint32_t s = b0; s < b1; ++s) {
          const F3 L = t.trace(px, py, s);
          const float Lc[3] = {L.x, L.y, L.z};
          welford_update(m, q, Lc, count[k] + (s - b0) + 1u);
        }
        count[k] += b1 - b0;
      }
    }
  }
  return omp_get_wtime() - t0;
}

// Candidate Gaussians of n rays over [0, inf): the caller's indices of every Gaussian whose padded
// 3-sigma box the ray meets (CPU BVH; all Gaussians without one).  Two passes: with idx == NULL
// it writes counts[n]; then, with offsets[n] = exclusive prefix sums of counts, it fills idx.
void or_ray_candidates(void* sv, const float* o, const float* d, uint32_t n, uint32_t* counts,
                       const uint64_t* offsets, uint32_t* idx) {
  const Scene& S = *static_cast<Scene*>(sv);
#pragma omp parallel
  {
    std::vector<uint32_t> cand;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      cand.clear();
      if (S.bvh.enabled) {
        S.bvh.ray(mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]), cand);
      } else {
        cand.resize(S.prims.size());
        std::iota(cand.begin(), cand.end(), 0u);
      }
      if (!idx) {
        counts[i] = static_cast<uint32_t>(cand.size());
      } else {
        uint32_t* out = idx + offsets[i];
        for (size_t k = 0; k < cand.size(); ++k) out[k] = S.orig[cand[k]];
      }
    }
  }
}

// FP64 sums of the absorption-plus-emission model per ray: S = sum tau_i and C = sum tau_i e_i
// (tau_i as tau64: the 3-sigma chord over [0, inf)), over every Gaussian except the caller's
// index `exclude` (-1: none).  emission: [3 * count] in the caller's order; out_S[n], out_C[3n].
void or_emission_sums(void* sv, const float* emission, const float* o, const float* d, uint32_t n, int64_t exclude,
                      double* out_S, double* out_C) {
  const Scene& S = *static_cast<Scene*>(sv);
#pragma omp parallel
  {
    std::vector<uint32_t> cand, one(1);
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      const double oo[3] = {o[3 * i], o[3 * i + 1], o[3 * i + 2]}, dd[3] = {d[3 * i], d[3 * i + 1], d[3 * i + 2]};
      cand.clear();
      if (S.bvh.enabled) {
        S.bvh.ray(mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]), cand);
      } else {
        cand.resize(S.prims.size());
        std::iota(cand.begin(), cand.end(), 0u);
      }
      double s = 0.0, c[3] = {0.0, 0.0, 0.0};
      for (uint32_t k : cand) {
        const uint32_t orig = S.orig[k];
        if (static_cast<int64_t>(orig) == exclude) continue;
        one[0] = k;
        const double t = tau64(S, oo, dd, &one);
        s += t;
        for (int ch = 0; ch < 3; ++ch) c[ch] += t * emission[3ull * orig + ch];
      }
      out_S[i] = s;
      for (int ch = 0; ch < 3; ++ch) out_C[3 * i + ch] = c[ch];
    }
  }
}

int or_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
