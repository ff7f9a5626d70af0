// One path vertex of the integrator (device/entry/raygen.cuh:115-208 with
// device/entry/path_stages.cuh:25-226), split from the queries so the persistent warp engine
// and the wavefront engine run the same shading code: given the outcome of the free-flight
// argmin of this bounce (scatter distance and the albedo there), draw the phase sample, build
// the transmittance queries of the bounce (the bounce-0 analytic direct term and the NEE shadow
// rays) with their radiance weights, apply the escape rule, throughput update and Russian
// roulette.  Random numbers are drawn in the reference's order: [free-flight key] -> phase
// sample (sampling.cuh:537) -> NEE (path_stages.cuh:148-226) -> roulette (:25-37).
#pragma once

#include "vp_device.cuh"

namespace vp {

struct PathState {
  float3 o, d, thr, rad;
  Pcg32 rng;
  uint32_t bounce;
};

struct ShadowSet {  // transmittance queries of one bounce: rad += w[k] * T(o[k], d[k])
  float3 o[3], d[3], w[3];
  // The Gaussian whose free flight put the query's origin there (the NEE rays start inside it),
  // or kNoGauss: the transmittance query evaluates it first and stops at once when its chord
  // alone reaches MAX_OPTICAL_DEPTH.
  uint32_t seed[3];
  int n;
};

// First random draws of a bounce: the 64-bit key of the keyed free-flight draws.
__device__ __forceinline__ uint64_t draw_bounce_key(Pcg32& rng) {
  const uint32_t hi = rng.next();
  const uint32_t lo = rng.next();
  return ((uint64_t)hi << 32) | lo;
}

__device__ __forceinline__ PathState start_path(const CameraView& C, const ParamsView& P, uint32_t px,
                                                uint32_t py, uint64_t sample_index) {
  PathState s;
  const uint64_t pix = (uint64_t)py * P.width + px;
  s.rng = pcg_init(P.seed, seq_hash(pix * (uint64_t)P.spp_total + sample_index));  // raygen.cuh:82-86
  camera_ray(C, P, px, py, s.rng, s.o, s.d);
  s.thr = f3(1.f, 1.f, 1.f);
  s.rad = f3(0.f, 0.f, 0.f);
  s.bounce = 0;
  return s;
}

// Returns true when the path continues (s.o / s.d then hold the next ray); the caller adds
// sh.w[k] * T(sh.o[k], sh.d[k]) to s.rad for k < sh.n either way.  scatter_gauss is the Gaussian
// whose free flight gave tstar (kNoGauss if unknown).
__device__ __forceinline__ bool shade_bounce(const EnvView& E, const ParamsView& P, PathState& s,
                                             bool scattered, float tstar, float3 albedo, ShadowSet& sh,
                                             uint32_t scatter_gauss = kNoGauss) {
  sh.n = 0;
  float3 pos = s.o, dir_next = s.d;
  if (scattered) {
    pos = fma3(tstar, s.d, s.o);  // ray.at(t)
    float pdf;
    dir_next = hg_sample(P, s.d, s.rng, pdf);
  }
  if (s.bounce == 0) {  // Rao-Blackwellised direct term (raygen.cuh:148-160)
    sh.o[0] = s.o;
    sh.d[0] = s.d;
    sh.w[0] = mul(s.thr, env_lookup(E, s.d));
    sh.seed[0] = kNoGauss;
    sh.n = 1;
  }
  if (!scattered) {  // accumulate_escape_radiance (path_stages.cuh:122-146)
    if (P.nee_mode == VP_NEE_NONE && s.bounce > 0) s.rad = add(s.rad, mul(s.thr, env_lookup(E, s.d)));
    return false;
  }
  const float3 base = mul(s.thr, albedo);
  if (P.nee_mode != VP_NEE_NONE && (base.x != 0.f || base.y != 0.f || base.z != 0.f)) {
    // accumulate_nee_direct (path_stages.cuh:148-226); a zero `base` adds nothing and the path
    // ends below, so its draws are skipped.
    if (P.nee_mode == VP_NEE_MIS) {
      float pdf_a;
      const float3 wa = hg_sample(P, s.d, s.rng, pdf_a);
      const float w_a = mis_balance(pdf_a, env_pdf(E, wa));
      const float3 c_a = mul(mul(base, env_lookup(E, wa)), w_a);
      float pdf_b;
      const float3 wb = env_sample(E, s.rng, pdf_b);
      const float ph_b = hg_eval(P, s.d, wb);
      const float w_b = mis_balance(pdf_b, ph_b);
      const float3 c_b = mul(mul(base, env_lookup(E, wb)), w_b * ph_b * __frcp_rn(pdf_b));
      sh.o[sh.n] = pos, sh.d[sh.n] = wa, sh.w[sh.n] = c_a, sh.seed[sh.n] = scatter_gauss;
      ++sh.n;
      sh.o[sh.n] = pos, sh.d[sh.n] = wb, sh.w[sh.n] = c_b, sh.seed[sh.n] = scatter_gauss;
      ++sh.n;
    } else if (P.nee_mode == VP_NEE_PHASE) {
      float pdf;
      const float3 wp = hg_sample(P, s.d, s.rng, pdf);
      sh.o[sh.n] = pos, sh.d[sh.n] = wp, sh.w[sh.n] = mul(base, env_lookup(E, wp)), sh.seed[sh.n] = scatter_gauss;
      ++sh.n;
    } else {  // VP_NEE_RIS: product RIS over ris_k env-IS candidates, 1 shadow ray
      const float3 luma = f3(0.2126f, 0.7152f, 0.0722f);
      float wsum = 0.f;
      float3 y_dir = f3(0.f, 0.f, 0.f), y_env = f3(0.f, 0.f, 0.f);
      for (uint32_t k = 0; k < P.ris_k; ++k) {
        float cpdf;
        const float3 cw = env_sample(E, s.rng, cpdf);
        if (cpdf <= 0.f) continue;
        const float3 env_c = env_lookup(E, cw);
        const float lum_c = dot3(env_c, luma);
        const float w = hg_eval(P, s.d, cw) * lum_c * __frcp_rn(cpdf);
        if (!(w > 0.f)) continue;
        wsum += w;
        if (s.rng.uniform() * wsum < w) {
          y_dir = cw;
          y_env = env_c;
        }
      }
      if (wsum > 0.f) {
        const float lum_y = dot3(y_env, luma);
        if (lum_y > 0.f) {
          const float W_ris = wsum * __frcp_rn((float)P.ris_k);
          sh.o[sh.n] = pos, sh.d[sh.n] = y_dir, sh.w[sh.n] = mul(mul(base, mul(y_env, __frcp_rn(lum_y))), W_ris);
          sh.seed[sh.n] = scatter_gauss;
          ++sh.n;
        }
      }
    }
  }
  s.thr = mul(s.thr, albedo);
  if (s.bounce >= P.rr_depth) {  // russian_roulette (path_stages.cuh:25-37)
    const float p_survive = fminf(P.rr_max_survival, fmax3(s.thr));
    if (s.rng.uniform() > p_survive || p_survive <= 0.f) return false;
    s.thr = mul(s.thr, __frcp_rn(p_survive));
  }
  if (fmax3(s.thr) < kMinThroughput) return false;  // raygen.cuh:197-199
  if (!isfinite(sum3(s.thr))) return false;          // raygen.cuh:201-204
  s.o = pos;
  s.d = dir_next;
  s.bounce += 1;
  return s.bounce < P.max_bounces;
}

// finalize_sample (path_stages.cuh:52-62)
__device__ __forceinline__ float3 finalize_sample(const ParamsView& P, float3 rad) {
  if (P.firefly_clamp > 0.f) {
    const float lum = dot3(rad, f3(0.2126f, 0.7152f, 0.0722f));
    if (lum > P.firefly_clamp) rad = mul(rad, P.firefly_clamp * __frcp_rn(lum));
  }
  if (!isfinite(sum3(rad))) rad = f3(0.f, 0.f, 0.f);
  return rad;
}

// Adaptive-sampling test on a pixel's Welford state before a batch (raygen.cuh:52-67 with
// constants.cuh:202-211): converged when every channel's sample standard deviation
// sqrt(M2 / (n - 1)) is below threshold x max(mean, 1e-6).  The reference's float3 divisions
// are multiplications by a round-to-nearest reciprocal; they are written out here with the _rn
// intrinsics so that no contraction changes a rounding.  Its max is `a > b ? a : b`
// (math.h:218-226), kept for the same answer when a rounding makes M2 a tiny negative number
// (a NaN error).  n >= 2 keeps n - 1 non-zero when the caller's minimum is 0 or 1.
constexpr float kAdaptiveMinLuminance = 1e-6f;
__device__ __forceinline__ bool pixel_converged(const ParamsView& P, uint32_t n, float4 mean, float4 m2) {
  if (!(P.adaptive_threshold > 0.0f) || n < P.adaptive_min_samples || n < 2u) return false;
  auto mx = [](float a, float b) { return a > b ? a : b; };
  const float inv_n1 = __frcp_rn((float)(n - 1u));
  auto err = [&](float m2c, float mc) {
    return __fmul_rn(__fsqrt_rn(__fmul_rn(m2c, inv_n1)), __frcp_rn(mx(mc, kAdaptiveMinLuminance)));
  };
  return mx(mx(err(m2.x, mean.x), err(m2.y, mean.y)), err(m2.z, mean.z)) < P.adaptive_threshold;
}

// One Welford step of a pixel's mean (and, with kM2, M2) for its k-th sample (k = 1, 2, ...;
// raygen.cuh:214-222): delta1 = L - mean, mean += delta1 * rcp(k), M2 += delta1 * (L - mean).
template <bool kM2>
__device__ __forceinline__ void welford_step(float3& m, float3& m2, float3 L, uint32_t k) {
  const float n_inv = __frcp_rn((float)k);
  const float3 d1 = sub(L, m);
  m = add(m, mul(d1, n_inv));
  if constexpr (kM2) m2 = add(m2, mul(d1, sub(L, m)));
}

}  // namespace vp
