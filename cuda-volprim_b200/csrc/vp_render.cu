// The path integrator on the device, in two engines over the same per-Gaussian math:
//
//  * WARP (default): a persistent kernel where each warp owns one path at a time and all 32
//    lanes cooperate on each of its queries.  A query walks the 32-wide BVH with the warp's
//    stack in shared memory: at an inner node every lane slab-tests one child and the hits are
//    pushed nearest-on-top (warp vote + shuffle rank); at a leaf every lane sets up the chord of
//    one Gaussian and the overlapping ones are compacted into the warp's hit buffer in shared
//    memory; full buffers of 32 are then evaluated one entry per lane (erf/erfinv/exp) and
//    reduced with shuffles.  Path control is warp-uniform, so the SIMT divergence of a
//    per-pixel megakernel between traversal, shading and termination does not arise.
//  * MEGAKERNEL: the straightforward per-pixel megakernel of the same method -- one thread per
//    pixel, thread-private stack traversal of the binary LBVH -- kept as the baseline.
//
// Path loop = __raygen__rg (device/entry/raygen.cuh:72-230) with the stages of
// device/entry/path_stages.cuh:25-226 and device/core/sampling.cuh:322-583:
//   per bounce: free-flight argmin over every Gaussian the ray overlaps (ADT) -> phase sample
//   -> [bounce 0: analytic camera transmittance x env] -> escape / albedo at the scatter point
//   -> NEE (MIS / phase / RIS) with shadow-ray transmittance -> Russian roulette.
// The origin-inside set, hit buffer and active-set rebuild of the reference are not stored:
// every query recovers them from the geometry (a Gaussian is "origin-inside" iff its chord
// starts at t <= 0; the active set at a point is the set of ellipsoids containing it), so no
// per-ray capacity limit exists.
#include <algorithm>

#include "vp_internal.h"

namespace vp {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kHitCap = 64;    // hit-buffer entries per warp (a leaf adds <= 32 to < 32)
constexpr int kBinStack = 128; // thread-private stack of the binary traversal

__device__ __forceinline__ float3 safe_inv(float3 d) {
  auto inv1 = [](float x) { return 1.0f / (fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x); };
  return f3(inv1(d.x), inv1(d.y), inv1(d.z));
}

__device__ __forceinline__ bool slab(float3 o, float3 inv, float4 lo, float4 hi, float t_lo,
                                     float t_hi, float& tnear) {
  const float tx0 = (lo.x - o.x) * inv.x, tx1 = (hi.x - o.x) * inv.x;
  const float ty0 = (lo.y - o.y) * inv.y, ty1 = (hi.y - o.y) * inv.y;
  const float tz0 = (lo.z - o.z) * inv.z, tz1 = (hi.z - o.z) * inv.z;
  const float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), t_lo));
  const float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), t_hi));
  tnear = tn;
  return tn <= tf;
}

__device__ __forceinline__ bool box_contains(float4 lo, float4 hi, float3 p) {
  return p.x >= lo.x && p.x <= hi.x && p.y >= lo.y && p.y <= hi.y && p.z >= lo.z && p.z <= hi.z;
}

// ------------------------------------------------------------------------------------------
// warp engine
// ------------------------------------------------------------------------------------------
struct WarpSmem {
  uint32_t* st_ref;
  float* st_t;
  uint32_t* hb_idx;
  float *hb_tc, *hb_rw, *hb_d2, *hb_h, *hb_u0, *hb_tin, *hb_tout, *hb_icf;
};

__device__ __forceinline__ size_t warp_smem_bytes(uint32_t stack_cap) {
  return (size_t)stack_cap * 8u + (size_t)kHitCap * 9u * 4u;
}

__device__ __forceinline__ WarpSmem carve(unsigned char* base, uint32_t stack_cap) {
  WarpSmem w;
  w.st_ref = reinterpret_cast<uint32_t*>(base);
  w.st_t = reinterpret_cast<float*>(base + 4u * stack_cap);
  float* hb = reinterpret_cast<float*>(base + 8u * stack_cap);
  w.hb_idx = reinterpret_cast<uint32_t*>(hb);
  w.hb_tc = hb + 1 * kHitCap;
  w.hb_rw = hb + 2 * kHitCap;
  w.hb_d2 = hb + 3 * kHitCap;
  w.hb_h = hb + 4 * kHitCap;
  w.hb_u0 = hb + 5 * kHitCap;
  w.hb_tin = hb + 6 * kHitCap;
  w.hb_tout = hb + 7 * kHitCap;
  w.hb_icf = hb + 8 * kHitCap;
  return w;
}

enum QueryKind { kArgmin = 0, kTau = 1 };

struct WarpStats {
  unsigned long long crossings = 0, nodes = 0, leaves = 0, prim_tests = 0, geo_loads = 0;
  unsigned int max_hits = 0;
};

// One ray query of the warp: kArgmin returns the smallest accepted free-flight distance over
// every Gaussian whose chord overlaps [0, t) (kInf = escape); kTau returns the optical depth
// over [0, inf), stopping once it reaches MAX_OPTICAL_DEPTH.
template <bool kAcc, int kKind>
__device__ float warp_ray_query(const SceneView& S, const WarpSmem& W, float3 o, float3 d,
                                uint64_t key, uint32_t& status, WarpStats& ws, bool measure) {
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const float3 inv = safe_inv(d);
  float t_hi = kInf;
  float acc = 0.0f;
  int sp = 1, hb = 0;
  unsigned int hits_seen = 0;
  if (lane == 0) {
    W.st_ref[0] = S.wide_root;
    W.st_t[0] = 0.0f;
  }
  __syncwarp();

  auto process = [&](int base, int cnt) {
    float v = (kKind == kArgmin) ? kInf : 0.0f;
    if (lane < cnt) {
      const int e = base + lane;
      const float tc = W.hb_tc[e], rw = W.hb_rw[e], d2 = W.hb_d2[e], h = W.hb_h[e], u0 = W.hb_u0[e];
      const float tin = W.hb_tin[e], tout = W.hb_tout[e], icf = W.hb_icf[e];
      if (kKind == kArgmin) {
        const uint32_t orig = __ldg(S.perm + W.hb_idx[e]);
        v = chord_free_flight(tc, rw, d2, h, u0, tin, tout, icf, free_flight_tau(key, orig));
      } else {
        v = chord_tau(tc, rw, d2, h, u0, fmaxf(tin, 0.0f), tout, icf);
      }
    }
    if (kKind == kArgmin) t_hi = fminf(t_hi, warp_min(v));
    else acc += warp_sum(v);
    if (measure) ws.crossings += (unsigned)cnt;
  };

  while (sp > 0) {
    --sp;
    const uint32_t ref = W.st_ref[sp];
    const float tn = W.st_t[sp];
    __syncwarp();
    if (tn > t_hi) continue;
    if (ref_is_leaf(ref)) {
      const uint32_t first = wide_leaf_first(ref), count = wide_leaf_count(ref);
      if (measure) {
        ws.leaves++;
        ws.prim_tests += count;
      }
      bool hit = false;
      Chord ch;
      float icf = 0.f;
      const uint32_t pi = first + (uint32_t)lane;
      bool boxed = false;
      if ((uint32_t)lane < count) {  // the Gaussian's own 3-sigma box first (32 B), then its record
        float tb;
        boxed = slab(o, inv, __ldg(S.pbox + 2u * pi), __ldg(S.pbox + 2u * pi + 1u), 0.0f, t_hi, tb);
      }
      if (boxed) {
        const PrimGeo g = load_geo(S.prims, pi);
        if (chord_setup<kAcc>(g, o, d, ch) && ch.t_out > 0.0f && ch.t_in <= t_hi) {
          hit = true;
          icf = g.icf;
        }
      }
      if (measure) ws.geo_loads += __popc(__ballot_sync(kFull, boxed));
      const unsigned m = __ballot_sync(kFull, hit);
      if (hit) {
        const int pos = hb + __popc(m & lt_mask);
        W.hb_idx[pos] = pi;
        W.hb_tc[pos] = ch.tc;
        W.hb_rw[pos] = ch.rw;
        W.hb_d2[pos] = ch.d2;
        W.hb_h[pos] = ch.h;
        W.hb_u0[pos] = chord_u0(ch, 0.0f);
        W.hb_tin[pos] = ch.t_in;
        W.hb_tout[pos] = ch.t_out;
        W.hb_icf[pos] = icf;
      }
      hb += __popc(m);
      hits_seen += __popc(m);
      __syncwarp();
      // Evaluate the buffered chords after every leaf that produced any: the argmin bound t_hi
      // and the shadow ray's optical depth must be current for pruning and early exit.
      if (hb > 0) {
        const int cnt = min(hb, 32);
        process(hb - cnt, cnt);
        hb -= cnt;
        __syncwarp();
        if (kKind == kTau && acc >= kMaxOpticalDepth) break;
      }
    } else {
      if (measure) ws.nodes++;
      const float4* node = S.wide + (size_t)ref * 64u;
      const float4 lo = __ldg(node + lane);
      const float4 hi = __ldg(node + 32 + lane);
      const uint32_t cref = __float_as_uint(lo.w);
      float tnear = 0.f;
      const bool hit = (cref != kEmptyRef) && slab(o, inv, lo, hi, 0.0f, t_hi, tnear);
      const unsigned m = __ballot_sync(kFull, hit);
      const int nh = __popc(m);
      if (nh > 0) {
        if ((uint32_t)(sp + nh) > S.stack_cap) {  // cannot happen for a BVH of the recorded depth
          status |= kStatusStackOverflow;
          break;
        }
        int rank = 0;  // farther children sit deeper in the stack
        for (unsigned mm = m; mm; mm &= mm - 1u) {
          const int j = __ffs(mm) - 1;
          const float tj = __shfl_sync(kFull, tnear, j);
          rank += (tj > tnear || (tj == tnear && j < lane)) ? 1 : 0;
        }
        if (hit) {
          W.st_ref[sp + rank] = cref;
          W.st_t[sp + rank] = tnear;
        }
        sp += nh;
      }
      __syncwarp();
    }
  }
  if (!(kKind == kTau && acc >= kMaxOpticalDepth) && hb > 0) process(0, hb);
  __syncwarp();
  if (measure) ws.max_hits = max(ws.max_hits, hits_seen);
  return (kKind == kArgmin) ? t_hi : acc;
}

// Albedo at a point: sigma_t * pdf weighted mean over the ellipsoids containing it
// (evaluate_albedo, sampling.cuh:257-283, over the active set of rebuild_active_set_at_scatter,
// :422-458).  Also returns the overlap count.
template <bool kAcc>
__device__ float3 warp_albedo(const SceneView& S, const WarpSmem& W, float3 x, uint32_t& overlap,
                              uint32_t& status, WarpStats& ws, bool measure) {
  const int lane = threadIdx.x & 31;
  float aw = 0.f, ar = 0.f, ag = 0.f, ab = 0.f;
  unsigned int cnt = 0;
  int sp = 1;
  if (lane == 0) W.st_ref[0] = S.wide_root;
  __syncwarp();
  while (sp > 0) {
    --sp;
    const uint32_t ref = W.st_ref[sp];
    __syncwarp();
    if (ref_is_leaf(ref)) {
      const uint32_t first = wide_leaf_first(ref), count = wide_leaf_count(ref);
      if (measure) {
        ws.leaves++;
        ws.prim_tests += count;
      }
      const uint32_t pi = first + lane;
      const bool boxed = (uint32_t)lane < count &&
                         box_contains(__ldg(S.pbox + 2u * pi), __ldg(S.pbox + 2u * pi + 1u), x);
      if (measure) ws.geo_loads += __popc(__ballot_sync(kFull, boxed));
      if (boxed) {
        const PrimGeo g = load_geo(S.prims, pi);
        float r2;
        if constexpr (kAcc) {
          const double Dx = (double)x.x - g.a.x, Dy = (double)x.y - g.a.y, Dz = (double)x.z - g.a.z;
          const double yx = g.a.w * Dx + g.b.x * Dy + g.b.y * Dz;
          const double yy = g.b.z * Dx + g.b.w * Dy + g.c.x * Dz;
          const double yz = g.c.y * Dx + g.c.z * Dy + g.c.w * Dz;
          r2 = (float)(yx * yx + yy * yy + yz * yz);
        } else {
          const float3 y = whiten(g, sub(x, f3(g.a.x, g.a.y, g.a.z)));
          r2 = dot3(y, y);
        }
        if (r2 <= kExtent2) {  // point_inside_bvh_bound (intersection.h:56-61)
          const float wgt = g.icf * expf(-0.5f * r2);
          const float3 al = load_albedo(S.prims, pi);
          aw += wgt;
          ar += wgt * al.x;
          ag += wgt * al.y;
          ab += wgt * al.z;
          ++cnt;
        }
      }
    } else {
      if (measure) ws.nodes++;
      const float4* node = S.wide + (size_t)ref * 64u;
      const float4 lo = __ldg(node + lane);
      const float4 hi = __ldg(node + 32 + lane);
      const uint32_t cref = __float_as_uint(lo.w);
      const bool hit = (cref != kEmptyRef) && box_contains(lo, hi, x);
      const unsigned m = __ballot_sync(kFull, hit);
      const int nh = __popc(m);
      if ((uint32_t)(sp + nh) > S.stack_cap) {
        status |= kStatusStackOverflow;
        break;
      }
      if (hit) W.st_ref[sp + __popc(m & ((1u << lane) - 1u))] = cref;
      sp += nh;
      __syncwarp();
    }
  }
  __syncwarp();
  aw = warp_sum(aw);
  ar = warp_sum(ar);
  ag = warp_sum(ag);
  ab = warp_sum(ab);
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(kFull, cnt, o);
  overlap = cnt;
  if (!(aw > 0.f)) return f3(0.f, 0.f, 0.f);
  const float r = __frcp_rn(aw);
  return f3(ar * r, ag * r, ab * r);
}

struct PathStats {
  unsigned long long bounces = 0, scatters = 0, shadow = 0;
  unsigned int max_overlap = 0;
};

// ---- the path loop, shared by both engines through a query policy ------------------------
template <class Q>
__device__ float3 trace_path(const SceneView& S, const EnvView& E, const CameraView& C,
                             const ParamsView& P, Q& q, uint32_t px, uint32_t py,
                             uint64_t sample_index, PathStats& ps) {
  const uint64_t pix = (uint64_t)py * P.width + px;
  Pcg32 rng = pcg_init(P.seed, seq_hash(pix * (uint64_t)P.spp_total + sample_index));
  float3 o, d;
  camera_ray(C, P, px, py, rng, o, d);
  float3 thr = f3(1.f, 1.f, 1.f), rad = f3(0.f, 0.f, 0.f);
  for (uint32_t bounce = 0; bounce < P.max_bounces; ++bounce) {
    const uint32_t khi = rng.next();
    const uint32_t klo = rng.next();
    const uint64_t key = ((uint64_t)khi << 32) | klo;
    // Stage 1-3 of sample_scattering_event: ADT argmin over every overlapped Gaussian.  In a
    // scene whose albedo is 0 everywhere a scatter ends the path with zero contribution, so
    // the camera-ray argmin is skipped there (the bounce-0 direct term below is the image).
    float tstar = kInf;
    if (!(bounce == 0 && S.albedo_all_zero)) tstar = q.argmin(o, d, key);
    const bool scattered = tstar < kInf;
    if (P.measure) {
      ps.bounces++;
      if (scattered) ps.scatters++;
    }
    float3 pos = o, dir_next = d;
    if (scattered) {
      pos = fma3(tstar, d, o);  // ray.at(t) = o + t d
      float pdf;
      dir_next = hg_sample(P, d, rng, pdf);
    }
    // Transmittance queries of this bounce (the bounce-0 camera ray and the NEE shadow rays)
    // are collected first and traced in one loop below: they draw no random numbers, so the
    // PCG32 stream is the reference's, and the query code exists once in the kernel.
    float3 sh_o[3], sh_d[3], sh_w[3];
    int ns = 0;
    if (bounce == 0) {  // Rao-Blackwellised direct term (raygen.cuh:148-160)
      sh_o[0] = o;
      sh_d[0] = d;
      sh_w[0] = mul(thr, env_lookup(E, d));
      ns = 1;
    }
    float3 albedo = f3(0.f, 0.f, 0.f);
    if (!scattered) {  // accumulate_escape_radiance (path_stages.cuh:368-386)
      if (P.nee_mode == VP_NEE_NONE && bounce > 0) rad = add(rad, mul(thr, env_lookup(E, d)));
    } else {
      uint32_t overlap = 0;
      albedo = q.albedo(pos, overlap);
      if (P.measure) ps.max_overlap = max(ps.max_overlap, overlap);
      const float3 base = mul(thr, albedo);
      if (P.nee_mode != VP_NEE_NONE && (base.x != 0.f || base.y != 0.f || base.z != 0.f)) {
        // accumulate_nee_direct (path_stages.cuh:394-472); shadow rays start at the scatter point.
        if (P.nee_mode == VP_NEE_MIS) {
          float pdf_a;
          const float3 wa = hg_sample(P, d, rng, pdf_a);
          const float w_a = mis_balance(pdf_a, env_pdf(E, wa));
          const float3 c_a = mul(mul(base, env_lookup(E, wa)), w_a);
          float pdf_b;
          const float3 wb = env_sample(E, rng, pdf_b);
          const float ph_b = hg_eval(P, d, wb);
          const float w_b = mis_balance(pdf_b, ph_b);
          const float3 c_b = mul(mul(base, env_lookup(E, wb)), w_b * ph_b * __frcp_rn(pdf_b));
          sh_o[ns] = pos, sh_d[ns] = wa, sh_w[ns] = c_a;
          ++ns;
          sh_o[ns] = pos, sh_d[ns] = wb, sh_w[ns] = c_b;
          ++ns;
        } else if (P.nee_mode == VP_NEE_PHASE) {
          float pdf;
          const float3 ws_ = hg_sample(P, d, rng, pdf);
          sh_o[ns] = pos, sh_d[ns] = ws_, sh_w[ns] = mul(base, env_lookup(E, ws_));
          ++ns;
        } else {  // VP_NEE_RIS: product RIS over ris_k env-IS candidates, 1 shadow ray
          const float3 luma = f3(0.2126f, 0.7152f, 0.0722f);
          float wsum = 0.f;
          float3 y_dir = f3(0.f, 0.f, 0.f), y_env = f3(0.f, 0.f, 0.f);
          for (uint32_t k = 0; k < P.ris_k; ++k) {
            float cpdf;
            const float3 cw = env_sample(E, rng, cpdf);
            if (cpdf <= 0.f) continue;
            const float3 env_c = env_lookup(E, cw);
            const float lum_c = dot3(env_c, luma);
            const float w = hg_eval(P, d, cw) * lum_c * __frcp_rn(cpdf);
            if (!(w > 0.f)) continue;
            wsum += w;
            if (rng.uniform() * wsum < w) {
              y_dir = cw;
              y_env = env_c;
            }
          }
          if (wsum > 0.f) {
            const float lum_y = dot3(y_env, luma);
            if (lum_y > 0.f) {
              const float W_ris = wsum * __frcp_rn((float)P.ris_k);
              sh_o[ns] = pos, sh_d[ns] = y_dir, sh_w[ns] = mul(mul(base, mul(y_env, __frcp_rn(lum_y))), W_ris);
              ++ns;
            }
          }
        }
      }
    }
#pragma unroll 1
    for (int k = 0; k < ns; ++k) {  // compute_transmittance_to_env (sampling.cuh:548-583)
      rad = add(rad, mul(sh_w[k], q.transmittance(sh_o[k], sh_d[k])));
      if (P.measure) ps.shadow++;
    }
    if (!scattered) break;
    thr = mul(thr, albedo);
    if (bounce >= P.rr_depth) {  // russian_roulette (path_stages.cuh:25-37)
      const float p_survive = fminf(P.rr_max_survival, fmax3(thr));
      if (rng.uniform() > p_survive || p_survive <= 0.f) break;
      thr = mul(thr, __frcp_rn(p_survive));
    }
    if (fmax3(thr) < kMinThroughput) break;
    if (!isfinite(sum3(thr))) break;
    o = pos;
    d = dir_next;
  }
  // finalize_sample (path_stages.cuh:52-62)
  if (P.firefly_clamp > 0.f) {
    const float lum = dot3(rad, f3(0.2126f, 0.7152f, 0.0722f));
    if (lum > P.firefly_clamp) rad = mul(rad, P.firefly_clamp * __frcp_rn(lum));
  }
  if (!isfinite(sum3(rad))) rad = f3(0.f, 0.f, 0.f);
  return rad;
}

template <bool kAcc>
struct WarpQueries {
  const SceneView& S;
  const WarpSmem& W;
  uint32_t& status;
  WarpStats& ws;
  bool measure;
  __device__ float argmin(float3 o, float3 d, uint64_t key) {
    return warp_ray_query<kAcc, kArgmin>(S, W, o, d, key, status, ws, measure);
  }
  __device__ float transmittance(float3 o, float3 d) {
    const float tau = warp_ray_query<kAcc, kTau>(S, W, o, d, 0ull, status, ws, measure);
    return tau >= kMaxOpticalDepth ? 0.0f : expf(-tau);
  }
  __device__ float3 albedo(float3 x, uint32_t& overlap) {
    return warp_albedo<kAcc>(S, W, x, overlap, status, ws, measure);
  }
};

__device__ __forceinline__ void flush_stats(Counters* c, const PathStats& ps, const WarpStats& ws,
                                            uint32_t status, bool measure) {
  if (status) atomicOr(&c->status, status);
  if (!measure) return;
  atomicAdd(&c->bounces, ps.bounces);
  atomicAdd(&c->scatters, ps.scatters);
  atomicAdd(&c->shadow_rays, ps.shadow);
  atomicAdd(&c->crossings, ws.crossings);
  atomicAdd(&c->nodes, ws.nodes);
  atomicAdd(&c->leaves, ws.leaves);
  atomicAdd(&c->prim_tests, ws.prim_tests);
  atomicAdd(&c->geo_loads, ws.geo_loads);
  atomicMax(&c->max_hits, ws.max_hits);
  atomicMax(&c->max_overlap, ps.max_overlap);
}

// Persistent warp-per-path kernel: warps pull pixels from a global counter; each pixel runs
// samples [spp_offset, spp_offset + spp_count) in order and Welford-updates mean/count.
template <bool kAcc>
__global__ void __launch_bounds__(256) k_render_warp(SceneView S, EnvView E, CameraView C,
                                                     ParamsView P, float4* __restrict__ mean,
                                                     uint32_t* __restrict__ count,
                                                     uint32_t spp_offset, uint32_t spp_count,
                                                     unsigned int* __restrict__ work,
                                                     Counters* __restrict__ ctr) {
  extern __shared__ unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpSmem W = carve(smem + warp * warp_smem_bytes(S.stack_cap), S.stack_cap);
  const uint32_t n_pix = P.width * P.height;
  uint32_t status = 0;
  WarpStats ws;
  PathStats ps;
  WarpQueries<kAcc> q{S, W, status, ws, P.measure != 0};
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(work, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= n_pix) break;
    const uint32_t px = item % P.width, py = item / P.width;
    const uint32_t prev = count[item];
    const float4 m4 = mean[item];
    float3 m = f3(m4.x, m4.y, m4.z);
    for (uint32_t s = 0; s < spp_count; ++s) {
      const float3 L = trace_path(S, E, C, P, q, px, py, (uint64_t)spp_offset + s, ps);
      const float n_inv = __frcp_rn((float)(prev + s + 1u));
      m = add(m, mul(sub(L, m), n_inv));  // Welford mean (raygen.cuh:214-219)
    }
    if (lane == 0) {
      mean[item] = make_float4(m.x, m.y, m.z, 0.f);
      count[item] = prev + spp_count;
    }
    if (status) break;
  }
  if (lane == 0) flush_stats(ctr, ps, ws, status, P.measure != 0);
}

// ------------------------------------------------------------------------------------------
// megakernel (thread per pixel, binary LBVH)
// ------------------------------------------------------------------------------------------
template <bool kAcc>
struct ThreadQueries {
  const SceneView& S;
  uint32_t& status;
  WarpStats& ws;
  bool measure;

  template <int kKind>
  __device__ float ray(float3 o, float3 d, uint64_t key) {
    const float3 inv = safe_inv(d);
    uint32_t stack[kBinStack];
    int sp = 0;
    float t_hi = kInf, acc = 0.f;
    uint32_t node = S.bin_root;
    unsigned int hits = 0;
    while (true) {
      if (measure) ws.nodes++;
      const float4* nd = S.bin + 4u * node;
      const float4 ll = __ldg(nd), lh = __ldg(nd + 1), rl = __ldg(nd + 2), rh = __ldg(nd + 3);
      const uint32_t refs[2] = {__float_as_uint(ll.w), __float_as_uint(rl.w)};
      float tn[2];
      bool hit[2];
      hit[0] = refs[0] != kEmptyRef && slab(o, inv, ll, lh, 0.f, t_hi, tn[0]);
      hit[1] = refs[1] != kEmptyRef && slab(o, inv, rl, rh, 0.f, t_hi, tn[1]);
      uint32_t next_inner[2];
      int n_inner = 0;
      for (int c = 0; c < 2; ++c) {
        if (!hit[c]) continue;
        if (ref_is_leaf(refs[c])) {
          const uint32_t pi = refs[c] & ~kLeafBit;
          if (measure) ws.geo_loads++;
          const PrimGeo g = load_geo(S.prims, pi);
          Chord ch;
          if (chord_setup<kAcc>(g, o, d, ch) && ch.t_out > 0.f && ch.t_in <= t_hi) {
            ++hits;
            if (measure) ws.crossings++;
            const float u0 = chord_u0(ch, 0.f);
            if (kKind == kArgmin) {
              const float ts = chord_free_flight(ch.tc, ch.rw, ch.d2, ch.h, u0, ch.t_in, ch.t_out, g.icf,
                                                 free_flight_tau(key, __ldg(S.perm + pi)));
              t_hi = fminf(t_hi, ts);
            } else {
              acc += chord_tau(ch.tc, ch.rw, ch.d2, ch.h, u0, fmaxf(ch.t_in, 0.f), ch.t_out, g.icf);
            }
          }
        } else {
          next_inner[n_inner++] = c;
        }
      }
      if (kKind == kTau && acc >= kMaxOpticalDepth) break;
      if (n_inner == 2) {  // nearer first
        const int nearc = tn[0] <= tn[1] ? 0 : 1;
        if (sp >= kBinStack) {
          status |= kStatusStackOverflow;
          break;
        }
        stack[sp++] = refs[1 - nearc];
        node = refs[nearc];
        continue;
      }
      if (n_inner == 1) {
        node = refs[next_inner[0]];
        continue;
      }
      // pop, skipping nodes that can no longer matter is done on the next visit's slab test
      if (sp == 0) break;
      node = stack[--sp];
    }
    if (measure) ws.max_hits = max(ws.max_hits, hits);
    return (kKind == kArgmin) ? t_hi : acc;
  }
  __device__ float argmin(float3 o, float3 d, uint64_t key) { return ray<kArgmin>(o, d, key); }
  __device__ float transmittance(float3 o, float3 d) {
    const float tau = ray<kTau>(o, d, 0ull);
    return tau >= kMaxOpticalDepth ? 0.0f : expf(-tau);
  }
  __device__ float3 albedo(float3 x, uint32_t& overlap) {
    uint32_t stack[kBinStack];
    int sp = 0;
    uint32_t node = S.bin_root;
    float aw = 0.f;
    float3 a = f3(0.f, 0.f, 0.f);
    uint32_t cnt = 0;
    while (true) {
      if (measure) ws.nodes++;
      const float4* nd = S.bin + 4u * node;
      const float4 bl[2] = {__ldg(nd), __ldg(nd + 2)};
      const float4 bh[2] = {__ldg(nd + 1), __ldg(nd + 3)};
      int n_inner = 0;
      uint32_t inner[2];
      for (int c = 0; c < 2; ++c) {
        const uint32_t r = __float_as_uint(bl[c].w);
        if (r == kEmptyRef || !box_contains(bl[c], bh[c], x)) continue;
        if (ref_is_leaf(r)) {
          const uint32_t pi = r & ~kLeafBit;
          if (measure) ws.geo_loads++;
          const PrimGeo g = load_geo(S.prims, pi);
          float r2;
          if constexpr (kAcc) {
            const double Dx = (double)x.x - g.a.x, Dy = (double)x.y - g.a.y, Dz = (double)x.z - g.a.z;
            const double yx = g.a.w * Dx + g.b.x * Dy + g.b.y * Dz;
            const double yy = g.b.z * Dx + g.b.w * Dy + g.c.x * Dz;
            const double yz = g.c.y * Dx + g.c.z * Dy + g.c.w * Dz;
            r2 = (float)(yx * yx + yy * yy + yz * yz);
          } else {
            const float3 y = whiten(g, sub(x, f3(g.a.x, g.a.y, g.a.z)));
            r2 = dot3(y, y);
          }
          if (r2 <= kExtent2) {
            const float wgt = g.icf * expf(-0.5f * r2);
            aw += wgt;
            a = add(a, mul(load_albedo(S.prims, pi), wgt));
            ++cnt;
          }
        } else {
          inner[n_inner++] = r;
        }
      }
      if (n_inner == 2) {
        if (sp >= kBinStack) {
          status |= kStatusStackOverflow;
          break;
        }
        stack[sp++] = inner[1];
        node = inner[0];
        continue;
      }
      if (n_inner == 1) {
        node = inner[0];
        continue;
      }
      if (sp == 0) break;
      node = stack[--sp];
    }
    overlap = cnt;
    if (!(aw > 0.f)) return f3(0.f, 0.f, 0.f);
    return mul(a, __frcp_rn(aw));
  }
};

template <bool kAcc>
__global__ void __launch_bounds__(128) k_render_mega(SceneView S, EnvView E, CameraView C, ParamsView P,
                                                     float4* __restrict__ mean, uint32_t* __restrict__ count,
                                                     uint32_t spp_offset, uint32_t spp_count,
                                                     Counters* __restrict__ ctr) {
  const uint32_t px = blockIdx.x * 16 + (threadIdx.x & 15);
  const uint32_t py = blockIdx.y * 8 + (threadIdx.x >> 4);
  uint32_t status = 0;
  WarpStats ws;
  PathStats ps;
  const bool inside = px < P.width && py < P.height;
  if (inside) {
    ThreadQueries<kAcc> q{S, status, ws, P.measure != 0};
    const uint32_t item = py * P.width + px;
    const uint32_t prev = count[item];
    const float4 m4 = mean[item];
    float3 m = f3(m4.x, m4.y, m4.z);
    for (uint32_t s = 0; s < spp_count; ++s) {
      const float3 L = trace_path(S, E, C, P, q, px, py, (uint64_t)spp_offset + s, ps);
      const float n_inv = __frcp_rn((float)(prev + s + 1u));
      m = add(m, mul(sub(L, m), n_inv));
    }
    mean[item] = make_float4(m.x, m.y, m.z, 0.f);
    count[item] = prev + spp_count;
  }
  if (status) atomicOr(&ctr->status, status);
  if (P.measure && inside) flush_stats(ctr, ps, ws, 0u, true);
}

// ------------------------------------------------------------------------------------------
// transmittance queries
// ------------------------------------------------------------------------------------------
template <bool kAcc>
__global__ void __launch_bounds__(256) k_tau_warp(SceneView S, const float* __restrict__ org,
                                                  const float* __restrict__ dir, uint32_t n,
                                                  float* __restrict__ out, unsigned int* __restrict__ work,
                                                  Counters* __restrict__ ctr) {
  extern __shared__ unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpSmem W = carve(smem + warp * warp_smem_bytes(S.stack_cap), S.stack_cap);
  uint32_t status = 0;
  WarpStats ws;
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(work, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= n) break;
    const float3 o = f3(org[3 * item], org[3 * item + 1], org[3 * item + 2]);
    const float3 d = f3(dir[3 * item], dir[3 * item + 1], dir[3 * item + 2]);
    const float tau = warp_ray_query<kAcc, kTau>(S, W, o, d, 0ull, status, ws, false);
    if (lane == 0) out[item] = tau >= kMaxOpticalDepth ? 0.0f : expf(-tau);
    if (status) break;
  }
  if (lane == 0 && status) atomicOr(&ctr->status, status);
}

template <bool kAcc>
__global__ void k_tau_thread(SceneView S, const float* __restrict__ org, const float* __restrict__ dir,
                             uint32_t n, float* __restrict__ out, Counters* __restrict__ ctr) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t status = 0;
  WarpStats ws;
  ThreadQueries<kAcc> q{S, status, ws, false};
  out[i] = q.transmittance(f3(org[3 * i], org[3 * i + 1], org[3 * i + 2]),
                           f3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]));
  if (status) atomicOr(&ctr->status, status);
}

// albedo / overlap queries at points (evaluate_albedo over the containing ellipsoids)
template <bool kAcc>
__global__ void __launch_bounds__(256) k_albedo_warp(SceneView S, const float* __restrict__ pts, uint32_t n,
                                                     float* __restrict__ rgb, uint32_t* __restrict__ cnt,
                                                     unsigned int* __restrict__ work, Counters* __restrict__ ctr) {
  extern __shared__ unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpSmem W = carve(smem + warp * warp_smem_bytes(S.stack_cap), S.stack_cap);
  uint32_t status = 0;
  WarpStats ws;
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(work, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= n) break;
    uint32_t ov = 0;
    const float3 a = warp_albedo<kAcc>(S, W, f3(pts[3 * item], pts[3 * item + 1], pts[3 * item + 2]), ov, status,
                                       ws, false);
    if (lane == 0) {
      rgb[3 * item] = a.x;
      rgb[3 * item + 1] = a.y;
      rgb[3 * item + 2] = a.z;
      cnt[item] = ov;
    }
    if (status) break;
  }
  if (lane == 0 && status) atomicOr(&ctr->status, status);
}

template <bool kAcc>
__global__ void k_albedo_thread(SceneView S, const float* __restrict__ pts, uint32_t n, float* __restrict__ rgb,
                                uint32_t* __restrict__ cnt, Counters* __restrict__ ctr) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t status = 0;
  WarpStats ws;
  ThreadQueries<kAcc> q{S, status, ws, false};
  uint32_t ov = 0;
  const float3 a = q.albedo(f3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), ov);
  rgb[3 * i] = a.x;
  rgb[3 * i + 1] = a.y;
  rgb[3 * i + 2] = a.z;
  cnt[i] = ov;
  if (status) atomicOr(&ctr->status, status);
}

// normalize_accumulator_kernel (device/kernels/normalize_accumulator.cu:16-25)
__global__ void k_normalize(float4* __restrict__ out, const float4* __restrict__ in, size_t n, float s) {
  const size_t stride = (size_t)blockDim.x * gridDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float4 v = __ldg(in + i);
    out[i] = make_float4(v.x * s, v.y * s, v.z * s, v.w * s);
  }
}

template <class K>
int occupancy_blocks(K kernel, int threads, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem) != cudaSuccess) b = 1;
  return b < 1 ? 1 : b;
}

}  // namespace

vp_status launch_render(vp_scene* s, vp_env* e, const CameraView& cam, const ParamsView& P,
                        int32_t engine, vp_image* img, uint32_t spp_offset, uint32_t spp_count) {
  vp_context* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  if (engine == VP_ENGINE_WARP) {
    const int threads = 256;
    const size_t smem = (size_t)(threads / 32) * (s->view.stack_cap * 8u + kHitCap * 9u * 4u);
    if (smem > 200 * 1024) return fail(VP_ERROR_LIMIT, "BVH too deep for the warp engine's shared-memory stack");
    VP_CUDA(cudaMemsetAsync(ctx->work_counter, 0, sizeof(unsigned int), st));
    if (P.accurate) {
      if (smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(k_render_warp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const int blocks = ctx->sm_count * occupancy_blocks(k_render_warp<true>, threads, smem);
      k_render_warp<true><<<blocks, threads, smem, st>>>(s->view, e->view, cam, P, img->mean, img->count,
                                                        spp_offset, spp_count, ctx->work_counter, ctx->counters);
    } else {
      if (smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(k_render_warp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const int blocks = ctx->sm_count * occupancy_blocks(k_render_warp<false>, threads, smem);
      k_render_warp<false><<<blocks, threads, smem, st>>>(s->view, e->view, cam, P, img->mean, img->count,
                                                         spp_offset, spp_count, ctx->work_counter, ctx->counters);
    }
  } else if (engine == VP_ENGINE_MEGAKERNEL) {
    const dim3 grid((P.width + 15) / 16, (P.height + 7) / 8);
    if (P.accurate)
      k_render_mega<true><<<grid, 128, 0, st>>>(s->view, e->view, cam, P, img->mean, img->count, spp_offset,
                                               spp_count, ctx->counters);
    else
      k_render_mega<false><<<grid, 128, 0, st>>>(s->view, e->view, cam, P, img->mean, img->count, spp_offset,
                                                spp_count, ctx->counters);
  } else {
    return fail(VP_ERROR_INVALID_ARGUMENT, "unknown engine");
  }
  VP_CUDA(cudaGetLastError());
  return VP_OK;
}

vp_status launch_transmittance(vp_scene* s, const float* o, const float* d, uint32_t n, bool accurate,
                               int32_t engine, float* out) {
  vp_context* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  if (n == 0) return VP_OK;
  if (engine == VP_ENGINE_WARP) {
    const int threads = 256;
    const size_t smem = (size_t)(threads / 32) * (s->view.stack_cap * 8u + kHitCap * 9u * 4u);
    VP_CUDA(cudaMemsetAsync(ctx->work_counter, 0, sizeof(unsigned int), st));
    if (accurate) {
      if (smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(k_tau_warp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const int blocks = ctx->sm_count * occupancy_blocks(k_tau_warp<true>, threads, smem);
      k_tau_warp<true><<<blocks, threads, smem, st>>>(s->view, o, d, n, out, ctx->work_counter, ctx->counters);
    } else {
      if (smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(k_tau_warp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const int blocks = ctx->sm_count * occupancy_blocks(k_tau_warp<false>, threads, smem);
      k_tau_warp<false><<<blocks, threads, smem, st>>>(s->view, o, d, n, out, ctx->work_counter, ctx->counters);
    }
  } else if (engine == VP_ENGINE_MEGAKERNEL) {
    if (accurate) k_tau_thread<true><<<(n + 127) / 128, 128, 0, st>>>(s->view, o, d, n, out, ctx->counters);
    else k_tau_thread<false><<<(n + 127) / 128, 128, 0, st>>>(s->view, o, d, n, out, ctx->counters);
  } else {
    return fail(VP_ERROR_INVALID_ARGUMENT, "unknown engine");
  }
  VP_CUDA(cudaGetLastError());
  return VP_OK;
}

vp_status launch_albedo(vp_scene* s, const float* pts, uint32_t n, bool accurate, int32_t engine, float* rgb,
                        uint32_t* cnt) {
  vp_context* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  if (n == 0) return VP_OK;
  if (engine == VP_ENGINE_WARP) {
    const int threads = 256;
    const size_t smem = (size_t)(threads / 32) * (s->view.stack_cap * 8u + kHitCap * 9u * 4u);
    VP_CUDA(cudaMemsetAsync(ctx->work_counter, 0, sizeof(unsigned int), st));
    if (accurate) {
      if (smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(k_albedo_warp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const int blocks = ctx->sm_count * occupancy_blocks(k_albedo_warp<true>, threads, smem);
      k_albedo_warp<true><<<blocks, threads, smem, st>>>(s->view, pts, n, rgb, cnt, ctx->work_counter, ctx->counters);
    } else {
      if (smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(k_albedo_warp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const int blocks = ctx->sm_count * occupancy_blocks(k_albedo_warp<false>, threads, smem);
      k_albedo_warp<false><<<blocks, threads, smem, st>>>(s->view, pts, n, rgb, cnt, ctx->work_counter, ctx->counters);
    }
  } else if (engine == VP_ENGINE_MEGAKERNEL) {
    if (accurate) k_albedo_thread<true><<<(n + 127) / 128, 128, 0, st>>>(s->view, pts, n, rgb, cnt, ctx->counters);
    else k_albedo_thread<false><<<(n + 127) / 128, 128, 0, st>>>(s->view, pts, n, rgb, cnt, ctx->counters);
  } else {
    return fail(VP_ERROR_INVALID_ARGUMENT, "unknown engine");
  }
  VP_CUDA(cudaGetLastError());
  return VP_OK;
}

vp_status launch_normalize(const float4* in, float4* out, size_t n, float scale, cudaStream_t st) {
  if (n == 0) return VP_OK;
  const size_t blocks = std::min<size_t>((n + 255) / 256, 1024);
  k_normalize<<<(unsigned)blocks, 256, 0, st>>>(out, in, n, scale);
  VP_CUDA(cudaGetLastError());
  return VP_OK;
}

}  // namespace vp
