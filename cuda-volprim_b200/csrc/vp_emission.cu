// Absorption-plus-emission image and its hand-written adjoint (the differentiation form; the
// reference renderer has no emission and no gradients).
//
// Image model.  Along a camera ray x(t) = o + t d, Gaussian i contributes the closed-form optical
// depth tau_i of its 3-sigma chord over [0, inf) -- the same truncated-chord sum as the
// transmittance query (Primitive::optical_depth, primitive.h:249-318) -- and emits RGB e_i per
// unit optical depth.  With S = sum_i tau_i, C = sum_i tau_i e_i and T = exp(-S):
//
//     L = (1 - T) C / S + T env(d)        (L = env(d) when S = 0)
//
// which is the exact emission-absorption integral int T(t) sigma(t) c(t) dt + T env when the
// emission-to-extinction ratio c(t) along the ray equals its tau-weighted mean C / S (exact for a
// single Gaussian, for disjoint chords of equal colour, and in the optically thin limit, where
// L -> sum_i tau_i e_i).  It depends on the Gaussians only through the order-independent sums S
// and C, so a ray's Gaussians are visited in any order and no hit list is sorted or stored.
// Limitation: no occlusion between Gaussians -- a Gaussian behind an opaque one still colours the
// pixel with its tau-weighted share; only the background term is attenuated.
//
// Adjoint.  For one ray with upstream gradient G = dLoss/dL (RGB):
//     dL/dS = C (T - a) / S - T env,  a = (1 - T) / S,      dL/dC = a
//     g_tau_i = G . (dL/dS + a e_i),   dLoss/de_i = G a tau_i
// and tau_i is differentiated in closed form through the whitening p = W (o - mu), w = W d,
// W = diag(1/s) R(q)^T (see tau_grad below).  The backward kernel traverses each ray twice --
// once for S and C, once to scatter per-Gaussian gradients -- instead of storing hit lists.
// Per Gaussian it accumulates 16 floats (float4 atomics, internal order): dLoss/dW (9),
// sum g_tau dtau/dp (3, for the mean), sum g_tau tau (1, for density and the scale
// normaliser), dLoss/de (3); a finishing kernel maps them to mean / scale / quaternion /
// density / emission gradients in the caller's order.
#include <cstring>
#include <type_traits>
#include <vector>

#include "vp_internal.h"
#include "vp_traverse.cuh"

namespace vp {
namespace {

// Warp-cooperative visit of every Gaussian whose 3-sigma chord overlaps [0, inf) of the ray.  The
// warp walks the BVH32 with the first hit child of each inner node kept in registers and the
// others on the warp's shared-memory stack (no ordering: the image model is order-independent).
// At a leaf (packed with the leaves next on the stack while they fit in 32 lanes), lane j takes the
// j-th Gaussian of the ranges laid end to end: box pre-test, chord set-up, then f(pi, g, ch) on
// that lane alone.
template <bool kAcc, class F>
__device__ void warp_visit(const SceneView& S, uint32_t* stack, float3 o, float3 d, uint32_t& status, F&& f) {
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const RayBox rb = ray_box(o, d);
  int sp = 0;
  uint32_t ref = S.wide_root;
  bool have = true;
  while (true) {
    if (!have) {
      if (sp == 0) break;
      ref = stack[--sp];
      __syncwarp();
    }
    have = false;
    if (ref_is_leaf(ref)) {
      // leaves next on the stack join this step while their Gaussians fit in the 32 lanes
      int total = (int)wide_leaf_count(ref);
      uint32_t pi = wide_leaf_first(ref) + (uint32_t)lane;
      while (VP_LEAF_PACK && sp > 0) {
        const uint32_t r2 = stack[sp - 1];
        if (!ref_is_leaf(r2)) break;
        const int c2 = (int)wide_leaf_count(r2);
        if (total + c2 > 32) break;
        --sp;
        if (lane >= total && lane < total + c2) pi = wide_leaf_first(r2) + (uint32_t)(lane - total);
        total += c2;
      }
      __syncwarp();
      if (lane < total) {
        float tb;
        if (slab(rb, __ldg(S.pbox + 2u * pi), __ldg(S.pbox + 2u * pi + 1u), 0.0f, kInf, tb)) {
          const PrimGeo g = load_geo(S.prims, pi);
          Chord ch;
          if (chord_setup<kAcc>(g, o, d, ch) && ch.t_out > 0.0f) f(pi, g, ch);
        }
      }
    } else {
      const float4* node = S.wide + (size_t)ref * 64u;
      const float4 lo = __ldg(node + lane);
      const float4 hi = __ldg(node + 32 + lane);
      const uint32_t cref = __float_as_uint(lo.w);
      float tnear = 0.f;
      const bool hit = (cref != kEmptyRef) && slab(rb, lo, hi, 0.0f, kInf, tnear);
      const unsigned m = __ballot_sync(kFull, hit);
      const int nh = __popc(m);
      if (nh > 0) {
        if ((uint32_t)(sp + nh) > S.stack_cap) {  // cannot happen for a BVH of the recorded depth
          status |= kStatusStackOverflow;
          break;
        }
        const int first = __ffs(m) - 1;
        if (hit && lane != first) stack[sp + __popc(m & lt_mask) - 1] = cref;
        sp += nh - 1;
        ref = __shfl_sync(kFull, cref, first);
        have = true;
      }
    }
    __syncwarp();
  }
  __syncwarp();
}

// tau of one chord over [max(t_in, 0), t_out] (0 for a segment below RAY_SEGMENT_MIN_LENGTH).
template <bool kAcc>
__device__ __forceinline__ float chord_tau0(const Chord& ch, float icf) {
  return chord_tau<kAcc>(ch.tc, ch.rw, ch.d2, ch.h, chord_u0(ch, 0.0f), fmaxf(ch.t_in, 0.0f), ch.t_out, icf,
                         ch.d2lo);
}

// The ray of (pixel, sample): the renderer's jittered camera ray (raygen.cuh:82-99).
__device__ __forceinline__ void pixel_ray(const CameraView& C, const ParamsView& P, uint32_t pix, uint32_t s,
                                          float3& o, float3& d) {
  const uint32_t px = pix % P.width, py = pix / P.width;
  Pcg32 rng = pcg_init(P.seed, seq_hash((uint64_t)pix * (uint64_t)P.spp_total + s));
  camera_ray(C, P, px, py, rng, o, d);
}

struct RaySums {
  float S, r, g, b;  // sum tau, sum tau * e (RGB)
};

template <bool kAcc>
__device__ RaySums ray_sums(const SceneView& S, const float4* __restrict__ emis, uint32_t* stack, float3 o, float3 d,
                            uint32_t& status, unsigned long long& crossings) {
  float s = 0.f, r = 0.f, g = 0.f, b = 0.f;
  unsigned int nc = 0;
  warp_visit<kAcc>(S, stack, o, d, status, [&](uint32_t pi, const PrimGeo& geo, const Chord& ch) {
    const float tau = chord_tau0<kAcc>(ch, geo.icf);
    const float4 e = __ldg(emis + pi);
    s += tau;
    r = fmaf(tau, e.x, r);
    g = fmaf(tau, e.y, g);
    b = fmaf(tau, e.z, b);
    ++nc;
  });
  for (int off = 16; off > 0; off >>= 1) nc += __shfl_xor_sync(kFull, nc, off);
  crossings += nc;
  return RaySums{warp_sum(s), warp_sum(r), warp_sum(g), warp_sum(b)};
}

// (1 - T) / S and (T - (1 - T) / S) / S for S >= 0, with their series below 1e-3.
__device__ __forceinline__ void opacity_terms(float S, float& T, float& a, float& q) {
  T = expf(-S);
  if (S < 1e-3f) {
    a = 1.0f - S * (0.5f - S * (1.0f / 6.0f));
    q = -0.5f + S * (1.0f / 3.0f - S * 0.125f);
  } else {
    a = -expm1f(-S) / S;
    q = (T - a) / S;
  }
}

__device__ __forceinline__ float3 ray_radiance(const RaySums& rs, float3 env) {
  float T, a, q;
  opacity_terms(rs.S, T, a, q);
  return f3(fmaf(a, rs.r, T * env.x), fmaf(a, rs.g, T * env.y), fmaf(a, rs.b, T * env.z));
}

// Resident 256-thread blocks per SM the FP32 emission kernels' register budgets are sized for
// (64 registers; the ACCURATE float-pair variants keep 2, which holds their ~100 registers).  On the differentiation workload 4 blocks take the
// forward from 56.5 to 49.2 ms and the adjoint from 127 to 114 ms against the compiler's own
// budgets (76 and 80 registers: 3 blocks).
#ifndef VP_EMIS_FWD_BLOCKS
#define VP_EMIS_FWD_BLOCKS 4
#endif
#ifndef VP_EMIS_BWD_BLOCKS
#define VP_EMIS_BWD_BLOCKS 4
#endif

template <bool kAcc>
__global__ void __launch_bounds__(256, kAcc ? 2 : VP_EMIS_FWD_BLOCKS) k_emis_forward(SceneView S, EnvView E, CameraView C, ParamsView P,
                                                      const float4* __restrict__ emis, float4* __restrict__ out,
                                                      unsigned int* work, Counters* ctr) {
  extern __shared__ uint32_t stacks[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* stack = stacks + warp * S.stack_cap;
  const uint32_t n_pix = P.width * P.height;
  uint32_t status = 0;
  unsigned long long crossings = 0;
  while (true) {
    uint32_t pix = 0;
    if (lane == 0) pix = atomicAdd(work, 1u);
    pix = __shfl_sync(kFull, pix, 0);
    if (pix >= n_pix) break;
    float3 sum = f3(0.f, 0.f, 0.f);
    for (uint32_t s = 0; s < P.spp_total; ++s) {
      float3 o, d;
      pixel_ray(C, P, pix, s, o, d);
      const RaySums rs = ray_sums<kAcc>(S, emis, stack, o, d, status, crossings);
      sum = add(sum, ray_radiance(rs, env_lookup(E, d)));
    }
    const float inv = 1.0f / (float)P.spp_total;
    if (lane == 0) out[pix] = make_float4(sum.x * inv, sum.y * inv, sum.z * inv, 1.0f);
    if (status) break;
  }
  if (lane == 0) {
    if (status) atomicOr(&ctr->status, status);
    if (P.measure) atomicAdd(&ctr->crossings, crossings);
  }
}

// dtau/dp and dtau/dw of one chord, with tau itself, where p = W (x0 - mu), w = W d and x0 is a
// point of the ray taken as fixed:
//   tau = icf |w|^-1 exp(-d2/2) [erf(h/sqrt2) - erf(u/sqrt2)],  h = sqrt(9 - d2),
//   A = w.w, B = p.w, d2 = p.p - B^2/A, u = B/sqrt(A) when the segment starts at x0 (origin inside
//   the chord, x0 = o), else u = -h.  The boundary terms of the moving 3-sigma limits enter through
//   h: icf |w|^-1 exp(-d2/2) sqrt(2/pi) exp(-h^2/2) = icf |w|^-1 sqrt(2/pi) exp(-9/2).
// For a ray that enters the chord (t_in >= 0) tau depends on the line only, so x0 is the closest
// approach o + t_c d: then |p| <= 3 and no term carries the camera's lever arm |o - mu| / s (which
// would make the accumulated dLoss/dW cancel to a few digits).  For an origin inside the chord,
// x0 = o, already within 3 whitened units.  v returns x0 - mu, formed as the chord set-up forms it
// (o - mu exact as a float pair, plus t_c d).  FP32; under kAcc p and d2 are float pairs, as in
// chord_accurate.  Returns false (no contribution) for a segment below RAY_SEGMENT_MIN_LENGTH.
template <bool kAcc>
__device__ __forceinline__ bool tau_grad(const PrimGeo& g, const Chord& ch, float3 o, float3 d, float& tau,
                                         float3& v, float3& dp, float3& dw) {
  const float t0 = fmaxf(ch.t_in, 0.0f);
  if (ch.t_out - t0 <= kSegmentMin) return false;
  const bool inside = !(ch.t_in >= 0.0f);
  float Dh[3], Dl[3];
  two_sum(o.x, -g.a.x, Dh[0], Dl[0]);
  two_sum(o.y, -g.a.y, Dh[1], Dl[1]);
  two_sum(o.z, -g.a.z, Dh[2], Dl[2]);
  const float t = inside ? 0.0f : ch.tc;
  const float dd[3] = {d.x, d.y, d.z};
  float vh[3], vl[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float pr, pe, sm, se;
    two_prod(t, dd[k], pr, pe);
    two_sum(Dh[k], pr, sm, se);
    fast_two_sum(sm, __fadd_rn(se, __fadd_rn(pe, Dl[k])), vh[k], vl[k]);
  }
  const float W[9] = {g.a.w, g.b.x, g.b.y, g.b.z, g.b.w, g.c.x, g.c.y, g.c.z, g.c.w};
  float px, py, pz, pp, pplo = 0.0f;
  if constexpr (kAcc) {
    FF p3[3];
    mat_vec_ff(W, vh, vl, p3);
    const FF n2 = norm2_ff(p3);
    px = p3[0].hi, py = p3[1].hi, pz = p3[2].hi;
    pp = n2.hi;
    pplo = n2.lo;
  } else {
    const float3 pv = whiten(g, f3(vh[0] + vl[0], vh[1] + vl[1], vh[2] + vl[2]));
    px = pv.x, py = pv.y, pz = pv.z;
    pp = dot3(pv, pv);
  }
  const float3 w3 = whiten(g, d);
  const float wx = w3.x, wy = w3.y, wz = w3.z;
  const float A = dot3(w3, w3), B = fmaf(px, wx, fmaf(py, wy, pz * wz));
  const float rA = __frcp_rn(A), rw = __frsqrt_rn(A);
  // d2 = p.p - B^2 / A; at the closest approach B = 0 up to rounding, so the pair's low part
  // carries the bits that matter on grazing chords
  const float d2 = __fadd_rn(fmaf(-B * B, rA, pp), pplo);
  if (!(d2 < 9.0f)) return false;
  const float h = sqrtf(9.0f - d2);
  const float u = inside ? B * rw : -h;
  const float E = expf(-0.5f * d2);
  const float base = g.icf * rw;
  const float k2pi = 0.79788456080286535588f, kis2 = 0.70710678118654752440f;
  const float D = inside ? erff(h * kis2) - erff(u * kis2) : 2.0f * erff(h * kis2);
  const float tt = base * E * D;
  const float dtau_dh = (inside ? 1.0f : 2.0f) * base * k2pi * 0.011108996538242306f;
  const float dtau_dd2 = -0.5f * tt - dtau_dh * 0.5f / h;
  const float dtau_du = inside ? -base * E * k2pi * expf(-0.5f * u * u) : 0.0f;
  const float gP = dtau_dd2;
  const float gB = dtau_dd2 * (-2.0f * B * rA) + dtau_du * rw;
  const float gA = -0.5f * tt * rA + dtau_dd2 * B * B * rA * rA - dtau_du * 0.5f * B * rA * rw;
  tau = tt;
  v = f3(vh[0] + vl[0], vh[1] + vl[1], vh[2] + vl[2]);
  dp = f3(2.0f * gP * px + gB * wx, 2.0f * gP * py + gB * wy, 2.0f * gP * pz + gB * wz);
  dw = f3(2.0f * gA * wx + gB * px, 2.0f * gA * wy + gB * py, 2.0f * gA * wz + gB * pz);
  return true;
}

template <bool kAcc>
__global__ void __launch_bounds__(256, kAcc ? 2 : VP_EMIS_BWD_BLOCKS) k_emis_backward(SceneView S, EnvView E, CameraView C, ParamsView P,
                                                       const float4* __restrict__ emis,
                                                       const float4* __restrict__ dl_dpix, float4* __restrict__ acc,
                                                       unsigned int* work, Counters* ctr) {
  extern __shared__ uint32_t stacks[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* stack = stacks + warp * S.stack_cap;
  const uint32_t n_pix = P.width * P.height;
  const float inv_spp = 1.0f / (float)P.spp_total;
  uint32_t status = 0;
  unsigned long long crossings = 0;
  while (true) {
    uint32_t pix = 0;
    if (lane == 0) pix = atomicAdd(work, 1u);
    pix = __shfl_sync(kFull, pix, 0);
    if (pix >= n_pix) break;
    const float4 gp = __ldg(dl_dpix + pix);
    if (gp.x == 0.0f && gp.y == 0.0f && gp.z == 0.0f) continue;  // nothing flows back (e.g. a crop)
    const float3 G = f3(gp.x * inv_spp, gp.y * inv_spp, gp.z * inv_spp);
    for (uint32_t s = 0; s < P.spp_total; ++s) {
      float3 o, d;
      pixel_ray(C, P, pix, s, o, d);
      const RaySums rs = ray_sums<kAcc>(S, emis, stack, o, d, status, crossings);
      const float3 env = env_lookup(E, d);
      float T, a, q;
      opacity_terms(rs.S, T, a, q);
      const float gS = G.x * fmaf(rs.r, q, -T * env.x) + G.y * fmaf(rs.g, q, -T * env.y) +
                       G.z * fmaf(rs.b, q, -T * env.z);
      const float3 gC = mul(G, a);
      warp_visit<kAcc>(S, stack, o, d, status, [&](uint32_t pi, const PrimGeo& geo, const Chord& ch) {
        float tau;
        float3 v, dp, dw;
        if (!tau_grad<kAcc>(geo, ch, o, d, tau, v, dp, dw)) return;
        const float4 e = __ldg(emis + pi);
        const float gt = gS + gC.x * e.x + gC.y * e.y + gC.z * e.z;
        const float3 gp3 = mul(dp, gt), gw3 = mul(dw, gt);
        // dLoss/dW_kl = gp_k v_l + gw_k d_l
        float4* a4 = acc + 4u * pi;
        atomicAdd(a4 + 0, make_float4(fmaf(gp3.x, v.x, gw3.x * d.x), fmaf(gp3.x, v.y, gw3.x * d.y),
                                      fmaf(gp3.x, v.z, gw3.x * d.z), fmaf(gp3.y, v.x, gw3.y * d.x)));
        atomicAdd(a4 + 1, make_float4(fmaf(gp3.y, v.y, gw3.y * d.y), fmaf(gp3.y, v.z, gw3.y * d.z),
                                      fmaf(gp3.z, v.x, gw3.z * d.x), fmaf(gp3.z, v.y, gw3.z * d.y)));
        atomicAdd(a4 + 2, make_float4(fmaf(gp3.z, v.z, gw3.z * d.z), gp3.x, gp3.y, gp3.z));
        atomicAdd(a4 + 3, make_float4(gt * tau, gC.x * tau, gC.y * tau, gC.z * tau));
      });
    }
    if (status) break;
  }
  if (lane == 0) {
    if (status) atomicOr(&ctr->status, status);
    if (P.measure) atomicAdd(&ctr->crossings, crossings);
  }
}

// Per-Gaussian accumulators (internal order) -> gradients of the caller's parameters (caller
// order), added to out[].  W_kl = R_lk / s_k with R = R(q / |q|) (the build's rotation matrix) and
// icf proportional to density / (s_x s_y s_z):
//   dL/dmu = -W^T sum(g dtau/dp);  dL/ds_k = -(sum_l gW_kl W_kl + gK) / s_k;
//   dL/dR_lk = gW_kl / s_k -> dL/dq_hat -> dL/dq = (g - q_hat (q_hat . g)) / |q|;
//   dL/ddensity = gK / density.
__global__ void k_emis_finish(uint32_t n, const uint32_t* __restrict__ perm, const float4* __restrict__ prims,
                              const float4* __restrict__ raw, const float4* __restrict__ acc, int scale_is_log,
                              float* __restrict__ g_mean, float* __restrict__ g_scale, float* __restrict__ g_quat,
                              float* __restrict__ g_dens, float* __restrict__ g_emis) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = perm[i];
  const float4 a0 = acc[4 * i], a1 = acc[4 * i + 1], a2 = acc[4 * i + 2], a3 = acc[4 * i + 3];
  const float gW[3][3] = {{a0.x, a0.y, a0.z}, {a0.w, a1.x, a1.y}, {a1.z, a1.w, a2.x}};
  const float gP[3] = {a2.y, a2.z, a2.w};
  const float gK = a3.x;
  const float4 r0 = prims[4 * i], r1 = prims[4 * i + 1], r2 = prims[4 * i + 2];
  const float W[3][3] = {{r0.w, r1.x, r1.y}, {r1.z, r1.w, r2.x}, {r2.y, r2.z, r2.w}};
  const float4 q4 = raw[2 * i], sd = raw[2 * i + 1];
  for (int l = 0; l < 3; ++l) g_mean[3 * c + l] += -(W[0][l] * gP[0] + W[1][l] * gP[1] + W[2][l] * gP[2]);
  float s[3] = {sd.x, sd.y, sd.z};
  if (scale_is_log)
    for (int k = 0; k < 3; ++k) s[k] = expf(s[k]);
  for (int k = 0; k < 3; ++k) {
    const float gs = -(gW[k][0] * W[k][0] + gW[k][1] * W[k][1] + gW[k][2] * W[k][2] + gK) / s[k];
    g_scale[3 * c + k] += scale_is_log ? gs * s[k] : gs;
  }
  // dL/dR_lk = gW_kl / s_k
  float gR[3][3];
  for (int l = 0; l < 3; ++l)
    for (int k = 0; k < 3; ++k) gR[l][k] = gW[k][l] / s[k];
  const float qn = sqrtf(q4.x * q4.x + q4.y * q4.y + q4.z * q4.z + q4.w * q4.w);
  const float w = q4.x / qn, x = q4.y / qn, y = q4.z / qn, z = q4.w / qn;
  // R(q) = [[1-2(y2+z2), 2(xy-wz), 2(xz+wy)], [2(xy+wz), 1-2(x2+z2), 2(yz-wx)], [2(xz-wy), 2(yz+wx), 1-2(x2+y2)]]
  const float gw = 2.0f * (-z * gR[0][1] + y * gR[0][2] + z * gR[1][0] - x * gR[1][2] - y * gR[2][0] + x * gR[2][1]);
  const float gx = 2.0f * (y * gR[0][1] + z * gR[0][2] + y * gR[1][0] - 2.0f * x * gR[1][1] - w * gR[1][2] +
                           z * gR[2][0] + w * gR[2][1] - 2.0f * x * gR[2][2]);
  const float gy = 2.0f * (-2.0f * y * gR[0][0] + x * gR[0][1] + w * gR[0][2] + x * gR[1][0] + z * gR[1][2] -
                           w * gR[2][0] + z * gR[2][1] - 2.0f * y * gR[2][2]);
  const float gz = 2.0f * (-2.0f * z * gR[0][0] - w * gR[0][1] + x * gR[0][2] + w * gR[1][0] - 2.0f * z * gR[1][1] +
                           y * gR[1][2] + x * gR[2][0] + y * gR[2][1]);
  const float dotq = w * gw + x * gx + y * gy + z * gz;
  g_quat[4 * c + 0] += (gw - w * dotq) / qn;
  g_quat[4 * c + 1] += (gx - x * dotq) / qn;
  g_quat[4 * c + 2] += (gy - y * dotq) / qn;
  g_quat[4 * c + 3] += (gz - z * dotq) / qn;
  g_dens[c] += gK / sd.w;
  if (g_emis) {
    g_emis[3 * c + 0] += a3.y;
    g_emis[3 * c + 1] += a3.z;
    g_emis[3 * c + 2] += a3.w;
  }
}

__global__ void k_set_emission(uint32_t n, const uint32_t* __restrict__ perm, const float* __restrict__ rgb,
                               float4* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = perm[i];
  out[i] = make_float4(rgb[3 * c], rgb[3 * c + 1], rgb[3 * c + 2], 0.0f);
}

template <class K>
int blocks_per_sm(K kernel, int threads, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem) != cudaSuccess) b = 1;
  return b < 1 ? 1 : b;
}

vp_status ensure_emission(vp_scene* s) {
  if (s->emis) return VP_OK;
  vp_status r;
  if ((r = dev_alloc(&s->emis, s->info.count, s->ctx->stream))) return r;
  VP_CUDA(cudaMemsetAsync(s->emis, 0, 16ull * s->info.count, s->ctx->stream));
  s->info.device_bytes += 16ull * s->info.count;
  return VP_OK;
}

struct Common {
  CameraView cv;
  ParamsView P;
  size_t smem;
};

vp_status prepare(vp_scene* s, vp_env* e, const vp_camera* cam, const vp_render_params* p, Common& c) {
  if (!s || !e || !cam || !p) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (s->ctx != e->ctx) return fail(VP_ERROR_INVALID_ARGUMENT, "objects belong to different contexts");
  if (s->info.count == 0) return fail(VP_ERROR_INVALID_ARGUMENT, "the emission model needs a scene with Gaussians");
  if (p->width == 0 || p->height == 0 || p->spp == 0)
    return fail(VP_ERROR_INVALID_ARGUMENT, "width, height and spp must be positive");
  if ((uint64_t)p->width * p->height >= (1ull << 32)) return fail(VP_ERROR_LIMIT, "image too large");
  VP_CUDA(cudaSetDevice(s->ctx->device));
  build_camera(*cam, p->width, p->height, c.cv);
  c.P = make_params(*p, s);
  c.smem = (size_t)8 * s->view.stack_cap * 4u;
  if (c.smem > 200 * 1024) return fail(VP_ERROR_LIMIT, "BVH too deep for the shared-memory stack");
  vp_status r;
  if ((r = ensure_emission(s))) return r;
  return VP_OK;
}

vp_status finish_stats(vp_context* ctx, const vp_render_params* p, uint32_t launches, vp_render_stats* stats) {
  VP_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  VP_CUDA(cudaEventSynchronize(ctx->ev1));
  Counters c{};
  VP_CUDA(cudaMemcpy(&c, ctx->counters, sizeof(c), cudaMemcpyDeviceToHost));
  if (stats) {
    float ms = 0.f;
    VP_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    std::memset(stats, 0, sizeof(*stats));
    stats->ms_kernels = ms;
    stats->paths = (uint64_t)p->width * p->height * p->spp;
    stats->crossings = c.crossings;
    stats->device_status = c.status;
    stats->launches = launches;
  }
  if (c.status) return fail(VP_ERROR_DEVICE_STATUS, "an emission kernel raised device status " + std::to_string(c.status));
  return VP_OK;
}

}  // namespace
}  // namespace vp

using namespace vp;

extern "C" {

vp_status vp_scene_set_emission(vp_scene* s, const float* rgb, int32_t memory) {
  if (!s) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (s->info.count == 0) return fail(VP_ERROR_INVALID_ARGUMENT, "the emission model needs a scene with Gaussians");
  if (!rgb) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (memory != VP_MEMORY_HOST && memory != VP_MEMORY_DEVICE) return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind");
  VP_CUDA(cudaSetDevice(s->ctx->device));
  cudaStream_t st = s->ctx->stream;
  const uint32_t n = s->info.count;
  vp_status r;
  if ((r = ensure_emission(s))) return r;
  const float* src = rgb;
  float* tmp = nullptr;
  if (memory == VP_MEMORY_HOST) {
    if ((r = dev_alloc(&tmp, 3ull * n, st))) return r;
    VP_CUDA(cudaMemcpyAsync(tmp, rgb, 12ull * n, cudaMemcpyHostToDevice, st));
    src = tmp;
  }
  k_set_emission<<<(n + 255) / 256, 256, 0, st>>>(n, s->perm, src, s->emis);
  const cudaError_t e = cudaGetLastError();
  if (tmp) dev_free(tmp, st);
  if (e != cudaSuccess) return cuda_fail(e, "k_set_emission");
  VP_CUDA(cudaStreamSynchronize(st));
  return VP_OK;
}

vp_status vp_render_emission(vp_scene* s, vp_env* e, const vp_camera* cam, const vp_render_params* p,
                             float* out_rgba, int32_t memory, vp_render_stats* stats) {
  if (!out_rgba) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (memory != VP_MEMORY_HOST && memory != VP_MEMORY_DEVICE) return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind");
  Common c;
  vp_status r;
  if ((r = prepare(s, e, cam, p, c))) return r;
  vp_context* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  const size_t n_pix = (size_t)p->width * p->height;
  float4* out = reinterpret_cast<float4*>(out_rgba);
  float4* tmp = nullptr;
  if (memory == VP_MEMORY_HOST) {
    if ((r = dev_alloc(&tmp, n_pix, st))) return r;
    out = tmp;
  }
  VP_CUDA(cudaMemsetAsync(ctx->counters, 0, sizeof(Counters), st));
  VP_CUDA(cudaMemsetAsync(ctx->work_counter, 0, sizeof(unsigned int), st));
  VP_CUDA(cudaEventRecord(ctx->ev0, st));
  auto kern = c.P.accurate ? k_emis_forward<true> : k_emis_forward<false>;
  if (c.smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem));
  const int blocks = ctx->sm_count * blocks_per_sm(kern, 256, c.smem);
  kern<<<blocks, 256, c.smem, st>>>(s->view, e->view, c.cv, c.P, s->emis, out, ctx->work_counter, ctx->counters);
  VP_CUDA(cudaGetLastError());
  r = finish_stats(ctx, p, 1, stats);
  if (tmp) {
    if (r == VP_OK) {
      const cudaError_t ce = cudaMemcpy(out_rgba, tmp, 16ull * n_pix, cudaMemcpyDeviceToHost);
      if (ce != cudaSuccess) r = cuda_fail(ce, "vp_render_emission read-back");
    }
    dev_free(tmp, st);
    cudaStreamSynchronize(st);
  }
  return r;
}

vp_status vp_render_emission_backward(vp_scene* s, vp_env* e, const vp_camera* cam, const vp_render_params* p,
                                      const float* dloss_drgba, int32_t memory, vp_gaussian_grads* grads,
                                      vp_render_stats* stats) {
  if (!dloss_drgba || !grads || !grads->mean || !grads->scale || !grads->quat_wxyz || !grads->density)
    return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (memory != VP_MEMORY_HOST && memory != VP_MEMORY_DEVICE) return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind");
  if (grads->memory != VP_MEMORY_HOST && grads->memory != VP_MEMORY_DEVICE)
    return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind of the gradient arrays");
  Common c;
  vp_status r;
  if ((r = prepare(s, e, cam, p, c))) return r;
  vp_context* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t n = s->info.count;
  const size_t n_pix = (size_t)p->width * p->height;
  // scratch: per-Gaussian accumulators, the staged upstream gradient, staged outputs
  float4* acc = nullptr;
  float4* dl = nullptr;
  float* gout = nullptr;  // 14 n floats: mean 3n, scale 3n, quat 4n, density n, emission 3n
  const float4* dsrc = reinterpret_cast<const float4*>(dloss_drgba);
  auto cleanup = [&]() {
    dev_free(acc, st);
    dev_free(dl, st);
    dev_free(gout, st);
    cudaStreamSynchronize(st);
  };
  if ((r = dev_alloc(&acc, 4ull * n, st))) return r;
  if (memory == VP_MEMORY_HOST) {
    if ((r = dev_alloc(&dl, n_pix, st))) return cleanup(), r;
    VP_CUDA(cudaMemcpyAsync(dl, dloss_drgba, 16ull * n_pix, cudaMemcpyHostToDevice, st));
    dsrc = dl;
  }
  const bool host_out = grads->memory == VP_MEMORY_HOST;
  float *gm = grads->mean, *gs = grads->scale, *gq = grads->quat_wxyz, *gd = grads->density, *ge = grads->emission;
  if (host_out) {
    if ((r = dev_alloc(&gout, 14ull * n, st))) return cleanup(), r;
    VP_CUDA(cudaMemsetAsync(gout, 0, 56ull * n, st));
    gm = gout;
    gs = gout + 3ull * n;
    gq = gout + 6ull * n;
    gd = gout + 10ull * n;
    ge = grads->emission ? gout + 11ull * n : nullptr;
  }
  VP_CUDA(cudaMemsetAsync(acc, 0, 64ull * n, st));
  VP_CUDA(cudaMemsetAsync(ctx->counters, 0, sizeof(Counters), st));
  VP_CUDA(cudaMemsetAsync(ctx->work_counter, 0, sizeof(unsigned int), st));
  VP_CUDA(cudaEventRecord(ctx->ev0, st));
  auto kern = c.P.accurate ? k_emis_backward<true> : k_emis_backward<false>;
  if (c.smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem));
  const int blocks = ctx->sm_count * blocks_per_sm(kern, 256, c.smem);
  kern<<<blocks, 256, c.smem, st>>>(s->view, e->view, c.cv, c.P, s->emis, dsrc, acc, ctx->work_counter, ctx->counters);
  VP_CUDA(cudaGetLastError());
  k_emis_finish<<<(n + 255) / 256, 256, 0, st>>>(n, s->perm, s->prims, s->raw, acc, s->scale_is_log, gm, gs, gq, gd, ge);
  VP_CUDA(cudaGetLastError());
  r = finish_stats(ctx, p, 2, stats);
  if (r == VP_OK && host_out) {
    std::vector<float> h(14ull * n);
    const cudaError_t ce = cudaMemcpy(h.data(), gout, 56ull * n, cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) {
      r = cuda_fail(ce, "vp_render_emission_backward read-back");
    } else {
      for (size_t k = 0; k < 3ull * n; ++k) grads->mean[k] += h[k];
      for (size_t k = 0; k < 3ull * n; ++k) grads->scale[k] += h[3ull * n + k];
      for (size_t k = 0; k < 4ull * n; ++k) grads->quat_wxyz[k] += h[6ull * n + k];
      for (size_t k = 0; k < 1ull * n; ++k) grads->density[k] += h[10ull * n + k];
      if (grads->emission)
        for (size_t k = 0; k < 3ull * n; ++k) grads->emission[k] += h[11ull * n + k];
    }
  }
  cleanup();
  return r;
}

}  // extern "C"
