// ORACLE pin (test infrastructure only): a C-ABI shim over the reference's OWN host-compilable
// headers, compiled from the reference's include/ tree by oracle/Makefile into _ref/libref_pin.so.
// It exposes the reference's Primitive constructor and whitening transforms
// (include/thesis/device/params/primitive.h:70-122), the 3-sigma containment test
// (include/thesis/common/geometry/intersection.h:56-61), the host camera build
// (include/thesis/host/params/camera.h:32-150) and the Morton code
// (include/thesis/host/utils/math.h:103-131), so the oracle's restatement of them can be checked
// against the reference's code itself.  It also returns the test runner's geometric validation
// scenes (test/scenes/geometric_validation.cpp, compiled in), exposes the adaptive-sampling constants
// (device/core/constants.cuh:196-211) and evaluates the raygen's Welford update and convergence
// test (device/entry/raygen.cuh:52-67, 214-222: a few lines of a device-only file, written out
// here) with the reference's own float3 operators and math::rcp / sqrt / max.  The device-only
// parts of the path (OptiX programs, sampling.cuh) need the OptiX SDK and are not built here.
// <cstdint> first: the reference's own build provides it through its precompiled header.
#include <cstdint>

#include "thesis/device/params/primitive.h"
#include "thesis/common/geometry/intersection.h"
#include "thesis/host/params/camera.h"
#include "thesis/host/utils/math.h"
#include "device/core/constants.cuh"
#include "scenes/geometric_validation.h"

#include <cstring>

using thesis::common::geometry::UnitQuaternion;
using thesis::device::params::Primitive;

extern "C" {

// out20: center[3], rot_quat(s, u[3]) (stored conjugate), rcp_scale[3], density_norm_factor,
// inv_cdf_factor, albedo[3], optical_thickness, scale[3], 0
void ref_primitive(const float* mean3, const float* scale3, const float* quat_wxyz, const float* albedo3,
                   float optical_thickness, float* out20) {
  const Primitive p = Primitive::from_forward_quat(
      make_float3(mean3[0], mean3[1], mean3[2]),
      UnitQuaternion::from(quat_wxyz[0], quat_wxyz[1], quat_wxyz[2], quat_wxyz[3]),
      make_float3(scale3[0], scale3[1], scale3[2]), make_float3(albedo3[0], albedo3[1], albedo3[2]),
      optical_thickness);
  const float v[20] = {p.center_.x, p.center_.y, p.center_.z, p.rot_quat_.s_, p.rot_quat_.u_.x,
                       p.rot_quat_.u_.y, p.rot_quat_.u_.z, p.rcp_scale_.x, p.rcp_scale_.y, p.rcp_scale_.z,
                       p.density_norm_factor_, p.inv_cdf_factor_, p.albedo_.x, p.albedo_.y, p.albedo_.z,
                       p.optical_thickness_, p.scale_.x, p.scale_.y, p.scale_.z, 0.0f};
  std::memcpy(out20, v, sizeof(v));
}

// Whitened position and direction + point_inside_bvh_bound for one Gaussian.
// out7: pos_local[3], dir_local[3], inside (0/1)
void ref_transform(const float* mean3, const float* scale3, const float* quat_wxyz, float optical_thickness,
                   const float* pos3, const float* dir3, float* out7) {
  const Primitive p = Primitive::from_forward_quat(
      make_float3(mean3[0], mean3[1], mean3[2]),
      UnitQuaternion::from(quat_wxyz[0], quat_wxyz[1], quat_wxyz[2], quat_wxyz[3]),
      make_float3(scale3[0], scale3[1], scale3[2]), make_float3(0.f, 0.f, 0.f), optical_thickness);
  const float3 a = p.transform_pos_local(make_float3(pos3[0], pos3[1], pos3[2]));
  const float3 b = p.transform_dir_local(make_float3(dir3[0], dir3[1], dir3[2]));
  const bool in = thesis::common::geometry::point_inside_bvh_bound(make_float3(pos3[0], pos3[1], pos3[2]), p);
  const float v[7] = {a.x, a.y, a.z, b.x, b.y, b.z, in ? 1.0f : 0.0f};
  std::memcpy(out7, v, sizeof(v));
}

// out16: eye[3], pixel00_relative[3], pixel_du[3], pixel_dv[3], view_direction[3], ortho
void ref_camera(const float* eye3, const float* lookat3, const float* up3, float vfov_deg, float ortho_height,
                int orthographic, unsigned width, unsigned height, float* out16) {
  const auto o = make_float3(eye3[0], eye3[1], eye3[2]);
  const auto t = make_float3(lookat3[0], lookat3[1], lookat3[2]);
  const auto u = make_float3(up3[0], up3[1], up3[2]);
  const auto cam = orthographic
                       ? thesis::host::params::Camera::createOrthographic(width, height, o, t, u, ortho_height)
                       : thesis::host::params::Camera::createPerspective(width, height, o, t, u, vfov_deg);
  const auto& d = cam.device_camera();
  const float v[16] = {d.eye_.x, d.eye_.y, d.eye_.z, d.pixel00_relative_.x, d.pixel00_relative_.y,
                       d.pixel00_relative_.z, d.pixel_du_.x, d.pixel_du_.y, d.pixel_du_.z, d.pixel_dv_.x,
                       d.pixel_dv_.y, d.pixel_dv_.z, d.view_direction_.x, d.view_direction_.y,
                       d.view_direction_.z, d.is_orthographic_ ? 1.0f : 0.0f};
  std::memcpy(out16, v, sizeof(v));
}

unsigned ref_morton3d(const float* pos3, const float* scene_min3, const float* inv_extent3) {
  return thesis::host::utils::math::morton3D(make_float3(pos3[0], pos3[1], pos3[2]),
                                             make_float3(scene_min3[0], scene_min3[1], scene_min3[2]),
                                             make_float3(inv_extent3[0], inv_extent3[1], inv_extent3[2]));
}

// The test runner's geometric validation and stress scenes (test/scenes/geometric_validation.cpp,
// compiled from the reference's source beside this file): the number of scenes, then scene i's
// name (NUL-terminated, at most name_cap bytes) and, for its first `cap` Gaussians, 14 floats
// each: centre[3], forward rotation (w, x, y, z) (the stored rotation is its conjugate), scale[3],
// albedo[3], optical thickness.  Returns the scene's Gaussian count.
int ref_validation_scene_count() { return static_cast<int>(thesis::test::scenes::get_all_test_scenes().size()); }

int ref_validation_scene(int i, char* name, int name_cap, float* out14, int cap) {
  const auto scenes = thesis::test::scenes::get_all_test_scenes();
  if (i < 0 || i >= static_cast<int>(scenes.size())) return -1;
  const auto& sc = scenes[static_cast<size_t>(i)];
  std::strncpy(name, sc.name.c_str(), static_cast<size_t>(name_cap) - 1);
  name[name_cap - 1] = '\0';
  const int n = static_cast<int>(sc.primitives.size());
  for (int j = 0; j < n && j < cap; ++j) {
    const Primitive& p = sc.primitives[static_cast<size_t>(j)];
    const float v[14] = {p.center_.x, p.center_.y, p.center_.z, p.rot_quat_.s_, -p.rot_quat_.u_.x,
                         -p.rot_quat_.u_.y, -p.rot_quat_.u_.z, p.scale_.x, p.scale_.y, p.scale_.z,
                         p.albedo_.x, p.albedo_.y, p.albedo_.z, p.optical_thickness_};
    std::memcpy(out14 + 14 * j, v, sizeof(v));
  }
  return n;
}

// out4: ENABLE_ADAPTIVE_SAMPLING (0/1), ADAPTIVE_MIN_SAMPLES, ADAPTIVE_THRESHOLD,
// ADAPTIVE_MIN_LUMINANCE
void ref_adaptive_constants(float* out4) {
  namespace k = thesis::device::consts;
  out4[0] = k::ENABLE_ADAPTIVE_SAMPLING ? 1.0f : 0.0f;
  out4[1] = static_cast<float>(k::ADAPTIVE_MIN_SAMPLES);
  out4[2] = k::ADAPTIVE_THRESHOLD;
  out4[3] = k::ADAPTIVE_MIN_LUMINANCE;
}

// The convergence statistic of raygen.cuh:56-63 for a pixel with prev_count >= 2 samples:
// out4 = per-channel error (3) and its max.
void ref_adaptive_error(const float* mean3, const float* m2_3, unsigned prev_count, float* out4) {
  namespace m = thesis::common::math;
  const auto mean = make_float3(mean3[0], mean3[1], mean3[2]);
  const auto M2 = make_float3(m2_3[0], m2_3[1], m2_3[2]);
  const auto variance = M2 * m::rcp(static_cast<float>(prev_count - 1));
  const auto std_dev = m::sqrt(variance);
  const auto lum = thesis::device::consts::ADAPTIVE_MIN_LUMINANCE;
  const auto safe_mean = make_float3(m::max(mean.x, lum), m::max(mean.y, lum), m::max(mean.z, lum));
  const auto err = std_dev / safe_mean;
  out4[0] = err.x, out4[1] = err.y, out4[2] = err.z, out4[3] = m::max(err);
}

// One Welford step of raygen.cuh:214-222 for sample number k (1-based): io6 = mean[3], M2[3].
void ref_welford_step(const float* L3, unsigned k, float* io6) {
  namespace m = thesis::common::math;
  const auto radiance = make_float3(L3[0], L3[1], L3[2]);
  auto mean = make_float3(io6[0], io6[1], io6[2]);
  auto M2 = make_float3(io6[3], io6[4], io6[5]);
  const auto n_inv = m::rcp(static_cast<float>(k));
  const auto delta1 = radiance - mean;
  mean += delta1 * n_inv;
  const auto delta2 = radiance - mean;
  M2 += delta1 * delta2;
  io6[0] = mean.x, io6[1] = mean.y, io6[2] = mean.z, io6[3] = M2.x, io6[4] = M2.y, io6[5] = M2.z;
}

}  // extern "C"
