// Warp-cooperative BVH32 queries and thread-private binary-LBVH queries over the per-Gaussian
// math of vp_device.cuh, shared by the persistent warp engine, the plain megakernel and the
// wavefront engine.
#pragma once

#include <type_traits>

#include "vp_internal.h"

namespace vp {

constexpr unsigned kFull = 0xFFFFFFFFu;
#ifndef VP_HIT_CAP
#define VP_HIT_CAP 128
#endif
constexpr int kHitCap = VP_HIT_CAP;  // hit-buffer entries per warp (retained chords + one step's new ones)

// Leaf packing in the warp traversals (1 = on): a leaf step also takes the leaves next on the
// stack while their Gaussians fit in the 32 lanes.
#ifndef VP_LEAF_PACK
#define VP_LEAF_PACK 1
#endif

// Stack discipline of the argmin traversal (the free-flight minimum, and so every result, is the
// same either way): 0 = the hit children are ranked by entry distance and stacked farther-deeper;
// 1 (default) = they are stacked in lane order (the nearest continues, as in transmittance) and
// each pop takes the nearest entry within the bound among the top 32 of the stack.  On the 500k
// showcase 1 visits 13.0 instead of 14.3 inner nodes and 98 instead of 110 boxes per bounce, and
// the extend stage takes 124 instead of 137 ms per 16-spp step (ranking costs a pass over the hit
// children at every inner node; the windowed minimum costs one redux.sync per pop).
#ifndef VP_ARGMIN_BEST_FIRST
#define VP_ARGMIN_BEST_FIRST 1
#endif

// Resident 256-thread blocks per SM the warp engine's register budget is sized for.
#ifndef VP_WARP_MIN_BLOCKS
#define VP_WARP_MIN_BLOCKS 4
#endif

__device__ __forceinline__ float3 safe_inv(float3 d) {
  auto inv1 = [](float x) { return 1.0f / (fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x); };
  return f3(inv1(d.x), inv1(d.y), inv1(d.z));
}

// Per-ray constants of the slab test.  With kFma each plane distance is one FMA,
// t = b (1/d) - o (1/d); against (b - o)(1/d) this moves a plane by a few ulps of o (as the
// subtraction's own rounding does), and the 3-sigma boxes are padded far beyond that.  It holds
// three more registers through the traversal: the argmin kernels (64 registers) take it, the
// transmittance kernel (48 registers, five blocks per SM) keeps the subtraction form, which
// measured faster there (the extra registers raised its spills from 52 to 84 B).
struct RayBox {
  float3 o, inv, oinv;
};
__device__ __forceinline__ RayBox ray_box(float3 o, float3 d) {
  RayBox r;
  r.o = o;
  r.inv = safe_inv(d);
  r.oinv = f3(o.x * r.inv.x, o.y * r.inv.y, o.z * r.inv.z);
  return r;
}

// Three-operand minimum / maximum (PTX ISA 8.8, sm_100a).
__device__ __forceinline__ float fmax3f(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ float fmin3f(float a, float b, float c) {
  float d;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}

template <bool kFma = true>
__device__ __forceinline__ bool slab(const RayBox& r, float4 lo, float4 hi, float t_lo, float t_hi, float& tnear) {
  float tx0, tx1, ty0, ty1, tz0, tz1;
  if constexpr (kFma) {
    tx0 = fmaf(lo.x, r.inv.x, -r.oinv.x), tx1 = fmaf(hi.x, r.inv.x, -r.oinv.x);
    ty0 = fmaf(lo.y, r.inv.y, -r.oinv.y), ty1 = fmaf(hi.y, r.inv.y, -r.oinv.y);
    tz0 = fmaf(lo.z, r.inv.z, -r.oinv.z), tz1 = fmaf(hi.z, r.inv.z, -r.oinv.z);
  } else {
    tx0 = (lo.x - r.o.x) * r.inv.x, tx1 = (hi.x - r.o.x) * r.inv.x;
    ty0 = (lo.y - r.o.y) * r.inv.y, ty1 = (hi.y - r.o.y) * r.inv.y;
    tz0 = (lo.z - r.o.z) * r.inv.z, tz1 = (hi.z - r.o.z) * r.inv.z;
  }
  const float tn = fmax3f(fminf(tx0, tx1), fminf(ty0, ty1), fmaxf(fminf(tz0, tz1), t_lo));
  const float tf = fmin3f(fmaxf(tx0, tx1), fmaxf(ty0, ty1), fminf(fmaxf(tz0, tz1), t_hi));
  tnear = tn;
  return tn <= tf;
}

__device__ __forceinline__ bool box_contains(float4 lo, float4 hi, float3 p) {
  return p.x >= lo.x && p.x <= hi.x && p.y >= lo.y && p.y <= hi.y && p.z >= lo.z && p.z <= hi.z;
}

// ------------------------------------------------------------------------------------------
// warp engine
// ------------------------------------------------------------------------------------------
// Per-warp shared memory: the traversal stack and the hit buffer of the chords the argmin retains
// for the scatter-point albedo (the transmittance and point queries keep none).
struct WarpSmem {
  uint32_t* st_ref;
  float* st_t;
  uint32_t* hb_idx;
  float *hb_tc, *hb_rw, *hb_d2, *hb_tin, *hb_tout, *hb_icf;
  int hit_cap;
  uint32_t st_cap;     // stack entries
  bool root_staged;    // the BVH32 root's child boxes sit at the start of dynamic shared memory
};

// VP_STAGE_ROOT: the wavefront traversal kernels copy the BVH32 root (which every query visits
// first) into shared memory once per block and read it from there instead of through L1
// (measured on the 500k showcase: extend -1.7%, shadow -0.5% per step).
#ifndef VP_STAGE_ROOT
#define VP_STAGE_ROOT 1
#endif
constexpr size_t kRootStageBytes = VP_STAGE_ROOT ? 64u * sizeof(float4) : 0u;
extern __shared__ __align__(16) unsigned char vp_dyn_smem[];  // every kernel's dynamic shared memory

// All threads of the block call it, before any warp traverses.
__device__ __forceinline__ void stage_root(const float4* wide, uint32_t root) {
  float4* r = reinterpret_cast<float4*>(vp_dyn_smem);
  for (int i = threadIdx.x; i < 64; i += blockDim.x) r[i] = __ldg(wide + (size_t)root * 64u + i);
  __syncthreads();
}

__host__ __device__ __forceinline__ size_t warp_smem_bytes(uint32_t stack_cap, int hit_cap) {
  return (size_t)stack_cap * 8u + (size_t)hit_cap * 7u * 4u;
}

__device__ __forceinline__ WarpSmem carve(unsigned char* base, uint32_t stack_cap, int hit_cap) {
  WarpSmem w;
  w.st_ref = reinterpret_cast<uint32_t*>(base);
  w.st_t = reinterpret_cast<float*>(base + 4u * stack_cap);
  float* hb = reinterpret_cast<float*>(base + 8u * stack_cap);
  w.hb_idx = reinterpret_cast<uint32_t*>(hb);
  w.hb_tc = hb + 1 * hit_cap;
  w.hb_rw = hb + 2 * hit_cap;
  w.hb_d2 = hb + 3 * hit_cap;
  w.hb_tin = hb + 4 * hit_cap;
  w.hb_tout = hb + 5 * hit_cap;
  w.hb_icf = hb + 6 * hit_cap;
  w.hit_cap = hit_cap;
  w.st_cap = stack_cap;
  w.root_staged = false;
  return w;
}

enum QueryKind { kArgmin = 0, kTau = 1 };

__device__ __forceinline__ float tau_value(float v) { return v; }
__device__ __forceinline__ float tau_value(FF v) { return __fadd_rn(v.hi, v.lo); }

// Squared whitened radius |W (x - c)|^2 of a point (point_inside_bvh_bound, intersection.h:56-61).
// kAcc: x - c exact as a float pair and the product as float pairs.
template <bool kAcc>
__device__ __forceinline__ float point_r2(const PrimGeo& g, float3 x) {
  if constexpr (kAcc) {
    float Dh[3], Dl[3];
    two_sum(x.x, -g.a.x, Dh[0], Dl[0]);
    two_sum(x.y, -g.a.y, Dh[1], Dl[1]);
    two_sum(x.z, -g.a.z, Dh[2], Dl[2]);
    const float W[9] = {g.a.w, g.b.x, g.b.y, g.b.z, g.b.w, g.c.x, g.c.y, g.c.z, g.c.w};
    FF y[3];
    mat_vec_ff(W, Dh, Dl, y);
    const FF r2 = norm2_ff(y);
    return __fadd_rn(r2.hi, r2.lo);
  } else {
    const float3 y = whiten(g, sub(x, f3(g.a.x, g.a.y, g.a.z)));
    return dot3(y, y);
  }
}

struct WarpStats {
  unsigned long long crossings = 0, nodes = 0, leaves = 0;
  unsigned long long kind_nodes[3] = {0, 0, 0}, kind_leaves[3] = {0, 0, 0};
  unsigned long long kind_prims[3] = {0, 0, 0}, kind_geo[3] = {0, 0, 0};  // boxes tested, records loaded
  unsigned int max_hits = 0;
  unsigned long long* hist = nullptr;  // Counters::hits_hist when the kernel measures
};

// Albedo at the scatter point, when the argmin query could derive it from its own chords, and
// the Gaussian whose free flight was the minimum (scene order; kNoGauss on escape).
struct ScatterAlbedo {
  float3 albedo;
  uint32_t overlap;
  uint32_t gauss;
  bool valid;
};

// Optical depth of the seed Gaussian's chord along a shadow ray from its origin: the first term of
// a transmittance query, also evaluated ahead of the query, one thread per ray, by the shading
// kernels (a ray whose seed chord alone reaches MAX_OPTICAL_DEPTH then never enters the query).
template <bool kAcc>
__device__ __forceinline__ float seed_chord_tau(const SceneView& S, uint32_t seed, float3 o, float3 d) {
  const PrimGeo g = load_geo(S.prims, seed);
  Chord ch;
  if (chord_setup<kAcc>(g, o, d, ch) && ch.t_out > 0.0f)
    return chord_tau<kAcc>(ch.tc, ch.rw, ch.d2, ch.h, chord_u0(ch, 0.0f), fmaxf(ch.t_in, 0.0f), ch.t_out, g.icf,
                           ch.d2lo);
  return 0.0f;
}

// One ray query of the warp: kArgmin returns the smallest accepted free-flight distance over
// every Gaussian whose chord overlaps [0, t) (kInf = escape); kTau returns the optical depth
// over [0, inf), stopping once it reaches MAX_OPTICAL_DEPTH.
//
// With `sa` (kArgmin only) the overlapping chords with t_in <= t stay in the hit buffer, and after
// the traversal the albedo at the scatter distance t* is the sigma_t * pdf-weighted mean over
// the chords containing t* -- the reference's rebuilt active set (sampling.cuh:422-458) and
// evaluate_albedo (:257-283), with the whitened radius from the chord frame,
// |y|^2 = d2 + ((t* - t_c)|w|)^2.  Every Gaussian containing the scatter point was processed (its
// chord starts before t* <= t), so the set is complete; if the retained chords outgrow the
// buffer, sa->valid stays false and the caller runs the point query instead.
//
// The optical depth is summed over the warp in FP32 after every leaf step (for the stop at
// MAX_OPTICAL_DEPTH); under kAcc each lane also keeps a compensated float-pair sum of its own
// chords, reduced once at the end, so thousands of overlapping chords keep the 1e-5
// transmittance bound.
//
// A kTau query whose origin lies inside a known Gaussian (`seed`, the one whose free flight put
// the path there) evaluates that chord first (or takes its value, seed_tau, when the caller
// evaluated it already): in a dense medium it alone usually reaches MAX_OPTICAL_DEPTH and the
// traversal is skipped; otherwise the traversal skips it at its leaf.
template <bool kAcc, int kKind>
__device__ float warp_ray_query(const SceneView& S, const WarpSmem& W, float3 o, float3 d,
                                uint64_t key, uint32_t& status, WarpStats& ws, bool measure,
                                ScatterAlbedo* sa = nullptr, uint32_t seed = kNoGauss, float seed_tau = -1.0f) {
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const RayBox rb = ray_box(o, d);
  float t_hi = kInf;
  float acc = 0.0f;
  FF lane_tau = {0.0f, 0.0f};  // kAcc: this lane's chords as a compensated float pair
  auto tau_total = [&]() -> float {
    if constexpr (kAcc) return warp_sum_ff(lane_tau);
    else return acc;
  };
  uint32_t arg = kNoGauss;  // kArgmin: the Gaussian of the current minimum
  if (kKind == kTau && seed != kNoGauss) {
    float v = 0.0f;  // seed_tau >= 0: evaluated ahead of the query (seed_chord_tau)
    if (lane == 0) v = seed_tau >= 0.0f ? seed_tau : seed_chord_tau<kAcc>(S, seed, o, d);
    acc = __shfl_sync(kFull, v, 0);
    if (kAcc) lane_tau.hi = v;  // v is 0 on lanes other than 0
    if (measure) ws.crossings += 1;
    if (acc >= kMaxOpticalDepth) {
      if (measure) {
        ws.max_hits = max(ws.max_hits, 1u);
        if (ws.hist && lane == 0) atomicAdd(ws.hist + 16 * kTau + 1, 1ull);
      }
      return tau_total();
    }
  }
  int sp = 0, hb = 0, kept = 0;  // retained chords [0, kept); hb == kept between leaves
  // best-first pops while the stack holds at most bf_limit entries (negative: never, for a warp
  // stack without the argmin's extra room)
  const int bf_limit = min((int)kArgminBestFirstStack, (int)W.st_cap - (int)S.stack_cap - 64);
  bool keep = (kKind == kArgmin) && sa != nullptr;
  unsigned int hits_seen = 0;
  // The node to visit next is kept in registers (the nearest hit child of the last inner node);
  // only its siblings go through the shared-memory stack.
  uint32_t ref = S.wide_root;
  float tn = 0.0f;
  bool have = true;

  // Drop retained chords that start beyond the current bound (they cannot contain t*).
  auto compact = [&]() {
    int w = 0;
    for (int base = 0; base < kept; base += 32) {
      const int e = base + lane;
      const bool keepit = e < kept && W.hb_tin[e] <= t_hi;
      uint32_t idx = 0;
      float f[6];
      if (keepit) {
        idx = W.hb_idx[e];
        f[0] = W.hb_tc[e], f[1] = W.hb_rw[e], f[2] = W.hb_d2[e];
        f[3] = W.hb_tin[e], f[4] = W.hb_tout[e], f[5] = W.hb_icf[e];
      }
      const unsigned m = __ballot_sync(kFull, keepit);
      __syncwarp();
      if (keepit) {
        const int p = w + __popc(m & lt_mask);
        W.hb_idx[p] = idx;
        W.hb_tc[p] = f[0], W.hb_rw[p] = f[1], W.hb_d2[p] = f[2];
        W.hb_tin[p] = f[3], W.hb_tout[p] = f[4], W.hb_icf[p] = f[5];
      }
      w += __popc(m);
      __syncwarp();
    }
    kept = hb = w;
  };

  while (true) {
    if (!have) {
      if (sp == 0) break;
      if (kKind == kArgmin && VP_ARGMIN_BEST_FIRST && sp <= bf_limit) {
        // the argmin's bound shrinks: pop the nearest entry within it among the top 32 of the
        // stack (lane j looks at the j-th entry from the top); the top entry fills its place.
        // Such pops can leave older entries below newer ones, so the stack is not bounded by the
        // depth-first bound; above bf_limit the traversal pops depth-first (the branch below),
        // which from any state adds at most one depth-first bound, and the warp's stack holds
        // bf_limit + 32 + that bound.
        const int e = sp - 1 - lane;
        const float te = e >= 0 ? W.st_t[e] + 0.0f : kInf;  // + 0: -0 -> +0, so bits order as values
        const unsigned key = (e >= 0 && te <= t_hi) ? __float_as_uint(te) : 0xFFFFFFFFu;
        const unsigned mn = __reduce_min_sync(kFull, key);
        if (mn == 0xFFFFFFFFu) {  // the whole window lies beyond the bound
          sp = max(sp - 32, 0);
          __syncwarp();
          continue;
        }
        const int es = sp - 1 - (__ffs(__ballot_sync(kFull, key == mn)) - 1);
        ref = W.st_ref[es];
        tn = __uint_as_float(mn);
        __syncwarp();
        if (lane == 0 && es != sp - 1) {
          W.st_ref[es] = W.st_ref[sp - 1];
          W.st_t[es] = W.st_t[sp - 1];
        }
        --sp;
        __syncwarp();
      } else {
        if constexpr (kKind == kArgmin) {
          // the argmin's bound shrinks: pop the topmost entry within it, skipping culled ones in
          // one step (lane j looks at the j-th entry from the top)
          const int e = sp - 1 - lane;
          const unsigned bm = __ballot_sync(kFull, e >= 0 && W.st_t[max(e, 0)] <= t_hi);
          if (bm == 0u) {
            sp = max(sp - 32, 0);
            __syncwarp();
            continue;
          }
          sp -= __ffs(bm);
        } else {
          --sp;
        }
        ref = W.st_ref[sp];
        tn = W.st_t[sp];
        __syncwarp();
      }
    }
    have = false;
    if (tn > t_hi) continue;
    if (ref_is_leaf(ref)) {
      // Leaf packing: the leaves next on the stack join this step while their Gaussians fit in
      // the warp's 32 lanes (lane -> Gaussian: the ranges laid end to end).
      int total = (int)wide_leaf_count(ref);
      uint32_t pi = wide_leaf_first(ref) + (uint32_t)lane;
      int packed = 1;
      while (VP_LEAF_PACK && sp > 0) {
        const uint32_t r2 = W.st_ref[sp - 1];
        if (!ref_is_leaf(r2)) break;
        const int c2 = (int)wide_leaf_count(r2);
        if (total + c2 > 32) break;
        const float t2 = W.st_t[sp - 1];
        --sp;
        if (t2 > t_hi) continue;  // culled, as it would be when popped
        if (lane >= total && lane < total + c2) pi = wide_leaf_first(r2) + (uint32_t)(lane - total);
        total += c2;
        ++packed;
      }
      __syncwarp();
      if (measure) {
        ws.leaves += packed;
        ws.kind_leaves[kKind] += packed;
        ws.kind_prims[kKind] += total;
      }
      bool hit = false;
      Chord ch;
      float icf = 0.f;
      bool boxed = false;
      if (lane < total && pi != seed) {  // the Gaussian's own 3-sigma box first (32 B), then its record
        float tb;
        boxed = slab<kKind == kArgmin>(rb, __ldg(S.pbox + 2u * pi), __ldg(S.pbox + 2u * pi + 1u), 0.0f, t_hi, tb);
      }
      if (boxed) {
        const PrimGeo g = load_geo(S.prims, pi);
        if (chord_setup<kAcc>(g, o, d, ch) && ch.t_out > 0.0f && ch.t_in <= t_hi) {
          hit = true;
          icf = g.icf;
        }
      }
      if (measure) ws.kind_geo[kKind] += __popc(__ballot_sync(kFull, boxed));
      const unsigned m = __ballot_sync(kFull, hit);
      if constexpr (kKind == kTau) {
        // Transmittance keeps no chords: each lane evaluates its own and the warp sums them
        // (no hit-buffer round trip through shared memory).  Evaluating at once, even with few
        // lanes busy, keeps the MAX_OPTICAL_DEPTH stop as early as possible: collecting the box
        // hits of several leaf steps to evaluate them with full warps was measured slower on the
        // showcase (+9% shadow time: 37% more boxes tested per shadow ray before the stop).
        if (m != 0u) {
          const float v = hit ? chord_tau<kAcc>(ch.tc, ch.rw, ch.d2, ch.h, chord_u0(ch, 0.0f), fmaxf(ch.t_in, 0.0f),
                                                ch.t_out, icf, ch.d2lo)
                              : 0.0f;
          acc += warp_sum(v);
          if (kAcc) ff_accumulate(lane_tau, v);
          hits_seen += __popc(m);
          if (measure) ws.crossings += (unsigned)__popc(m);
          if (acc >= kMaxOpticalDepth) break;
        }
        continue;
      }
      // The argmin: each lane evaluates its own chord's free flight and the warp takes the
      // minimum (the argmin does not depend on the order of the chords); the chords that can
      // still contain the scatter point (t_in <= t_hi) are retained for its albedo.
      if (m != 0u) {
        float v = kInf;
        if (hit) {
          const uint32_t orig = __ldg(S.perm + pi);
          v = chord_free_flight<kAcc>(ch.tc, ch.rw, ch.d2, ch.h, chord_u0(ch, 0.0f), ch.t_in, ch.t_out, icf,
                                      free_flight_tau<kAcc>(key, orig), ch.d2lo);
        }
        // free flights are >= 0 (+ 0 turns -0 into +0), so their bits order as their values and
        // one redux.sync takes the warp minimum
        v += 0.0f;
        const float mn = __uint_as_float(__reduce_min_sync(kFull, __float_as_uint(v)));
        if (mn < t_hi) {
          const unsigned wm = __ballot_sync(kFull, v == mn);
          arg = __shfl_sync(kFull, pi, __ffs(wm) - 1);
          t_hi = mn;
        }
        hits_seen += __popc(m);
        if (measure) ws.crossings += (unsigned)__popc(m);
        if (keep) {
          const bool ret = hit && ch.t_in <= t_hi;
          const unsigned rm = __ballot_sync(kFull, ret);
          const int nr = __popc(rm);
          if (nr != 0 && hb + nr > W.hit_cap) {  // make room: drop chords that start beyond t_hi
            compact();
            if (hb + nr > W.hit_cap) {  // still full: stop retaining, the caller will query the point
              keep = false;
              kept = hb = 0;
            }
          }
          if (keep) {
            if (ret) {
              const int pos = hb + __popc(rm & lt_mask);
              W.hb_idx[pos] = pi;
              W.hb_tc[pos] = ch.tc;
              W.hb_rw[pos] = ch.rw;
              W.hb_d2[pos] = ch.d2;
              W.hb_tin[pos] = ch.t_in;
              W.hb_tout[pos] = ch.t_out;
              W.hb_icf[pos] = icf;
            }
            hb += nr;
            kept = hb;
          }
          __syncwarp();
        }
      }
    } else {
      if (measure) {
        ws.nodes++;
        ws.kind_nodes[kKind]++;
      }
      float4 lo, hi;
      if (VP_STAGE_ROOT && W.root_staged && ref == S.wide_root) {
        const float4* r = reinterpret_cast<const float4*>(vp_dyn_smem);
        lo = r[lane];
        hi = r[32 + lane];
      } else {
        const float4* node = S.wide + (size_t)ref * 64u;
        lo = __ldg(node + lane);
        hi = __ldg(node + 32 + lane);
      }
      const uint32_t cref = __float_as_uint(lo.w);
      float tnear = 0.f;
      const bool hit = (cref != kEmptyRef) && slab<kKind == kArgmin>(rb, lo, hi, 0.0f, t_hi, tnear);
      const unsigned m = __ballot_sync(kFull, hit);
      const int nh = __popc(m);
      if (nh > 0) {
        if ((uint32_t)(sp + nh) > W.st_cap) {  // cannot happen for a BVH of the recorded depth
          status |= kStatusStackOverflow;
          break;
        }
        // The traversal continues into the nearest child.  The argmin (without best-first pops)
        // stacks the others by distance (farther deeper; rank nh-1 is the nearest), so its
        // culling at the best t* pops the near ones first.  Transmittance sums every chord
        // whatever the order: in lane order (the nearest child picked by a warp min, a fixed few
        // instructions) or, for scenes whose rays need many overlapping Gaussians to reach
        // MAX_OPTICAL_DEPTH (S.tau_nearest), ranked like the argmin so the stop comes sooner.
        int rank = 0;
        int src;
        const bool ranked = kKind == kArgmin ? !VP_ARGMIN_BEST_FIRST : (kKind == kTau && S.tau_nearest != 0u);
        if (!ranked) {
          const unsigned key = hit ? __float_as_uint(tnear + 0.0f) : 0xFFFFFFFFu;  // tnear >= 0: bit order
          const unsigned mn = __reduce_min_sync(kFull, key);
          src = __ffs(__ballot_sync(kFull, hit && key == mn)) - 1;
          rank = __popc(m & lt_mask & ~(1u << src));
        } else {
          for (unsigned mm = m; mm; mm &= mm - 1u) {
            const int j = __ffs(mm) - 1;
            const float tj = __shfl_sync(kFull, tnear, j);
            rank += (tj > tnear || (tj == tnear && j < lane)) ? 1 : 0;
          }
          src = __ffs(__ballot_sync(kFull, hit && rank == nh - 1)) - 1;
        }
        const bool nearest = lane == src;
        if (hit && !nearest) {
          W.st_ref[sp + rank] = cref;
          W.st_t[sp + rank] = tnear;
        }
        sp += nh - 1;
        ref = __shfl_sync(kFull, cref, src);
        tn = __shfl_sync(kFull, tnear, src);
        have = true;
      }
      __syncwarp();
    }
  }
  __syncwarp();
  if (measure) {
    ws.max_hits = max(ws.max_hits, hits_seen);
    if (ws.hist && lane == 0) atomicAdd(ws.hist + 16 * kKind + hits_bin(hits_seen), 1ull);
  }
  if constexpr (kKind == kArgmin) {
    if (sa != nullptr) {
      sa->valid = false;
      sa->gauss = t_hi < kInf ? arg : kNoGauss;
      if (keep && t_hi < kInf) {
        const float ts = t_hi;
        float aw = 0.f, ar = 0.f, ag = 0.f, ab = 0.f;
        unsigned int cnt = 0;
        for (int base = 0; base < kept; base += 32) {
          const int e = base + lane;
          if (e < kept && W.hb_tin[e] <= ts && ts <= W.hb_tout[e]) {
            const float u = (ts - W.hb_tc[e]) / W.hb_rw[e];
            const float wgt = W.hb_icf[e] * vexp<kAcc>(-0.5f * fmaf(u, u, W.hb_d2[e]));
            const float3 al = load_albedo(S.prims, W.hb_idx[e]);
            aw += wgt;
            ar += wgt * al.x;
            ag += wgt * al.y;
            ab += wgt * al.z;
            ++cnt;
          }
        }
        aw = warp_sum(aw);
        ar = warp_sum(ar);
        ag = warp_sum(ag);
        ab = warp_sum(ab);
        for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(kFull, cnt, off);
        const float r = aw > 0.f ? __frcp_rn(aw) : 0.f;
        sa->albedo = aw > 0.f ? f3(ar * r, ag * r, ab * r) : f3(0.f, 0.f, 0.f);
        sa->overlap = cnt;
        sa->valid = true;
      }
    }
  }
  __syncwarp();
  if constexpr (kKind == kArgmin) return t_hi;
  else return tau_total();
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
        ws.kind_leaves[2]++;
        ws.kind_prims[2] += count;
      }
      const uint32_t pi = first + lane;
      const bool boxed = (uint32_t)lane < count &&
                         box_contains(__ldg(S.pbox + 2u * pi), __ldg(S.pbox + 2u * pi + 1u), x);
      if (measure) ws.kind_geo[2] += __popc(__ballot_sync(kFull, boxed));
      if (boxed) {
        const PrimGeo g = load_geo(S.prims, pi);
        const float r2 = point_r2<kAcc>(g, x);
        if (r2 <= kExtent2) {  // point_inside_bvh_bound (intersection.h:56-61)
          const float wgt = g.icf * vexp<kAcc>(-0.5f * r2);
          const float3 al = load_albedo(S.prims, pi);
          aw += wgt;
          ar += wgt * al.x;
          ag += wgt * al.y;
          ab += wgt * al.z;
          ++cnt;
        }
      }
    } else {
      if (measure) {
        ws.nodes++;
        ws.kind_nodes[2]++;
      }
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


template <bool kAcc>
struct ThreadQueries {
  const SceneView& S;
  uint32_t& status;
  WarpStats& ws;
  bool measure;

  template <int kKind>
  __device__ float ray(float3 o, float3 d, uint64_t key) {
    const RayBox rb = ray_box(o, d);
    uint32_t stack[kBinStack];
    int sp = 0;
    float t_hi = kInf;
    std::conditional_t<kAcc, FF, float> acc{};  // compensated float-pair optical-depth sum under kAcc
    uint32_t node = S.bin_root;
    unsigned int hits = 0;
    while (true) {
      if (measure) ws.nodes++;
      const float4* nd = S.bin + 4u * node;
      const float4 ll = __ldg(nd), lh = __ldg(nd + 1), rl = __ldg(nd + 2), rh = __ldg(nd + 3);
      const uint32_t refs[2] = {__float_as_uint(ll.w), __float_as_uint(rl.w)};
      float tn[2];
      bool hit[2];
      hit[0] = refs[0] != kEmptyRef && slab(rb, ll, lh, 0.f, t_hi, tn[0]);
      hit[1] = refs[1] != kEmptyRef && slab(rb, rl, rh, 0.f, t_hi, tn[1]);
      uint32_t next_inner[2];
      int n_inner = 0;
      for (int c = 0; c < 2; ++c) {
        if (!hit[c]) continue;
        if (ref_is_leaf(refs[c])) {
          const uint32_t pi = refs[c] & ~kLeafBit;
          if (measure) {
            ws.kind_prims[kKind]++;
            ws.kind_geo[kKind]++;
          }
          const PrimGeo g = load_geo(S.prims, pi);
          Chord ch;
          if (chord_setup<kAcc>(g, o, d, ch) && ch.t_out > 0.f && ch.t_in <= t_hi) {
            ++hits;
            if (measure) ws.crossings++;
            const float u0 = chord_u0(ch, 0.f);
            if (kKind == kArgmin) {
              const float ts = chord_free_flight<kAcc>(ch.tc, ch.rw, ch.d2, ch.h, u0, ch.t_in, ch.t_out, g.icf,
                                                 free_flight_tau<kAcc>(key, __ldg(S.perm + pi)), ch.d2lo);
              t_hi = fminf(t_hi, ts);
            } else {
              const float v = chord_tau<kAcc>(ch.tc, ch.rw, ch.d2, ch.h, u0, fmaxf(ch.t_in, 0.f), ch.t_out, g.icf,
                                              ch.d2lo);
              if constexpr (kAcc) ff_accumulate(acc, v);
              else acc += v;
            }
          }
        } else {
          next_inner[n_inner++] = c;
        }
      }
      if (kKind == kTau && tau_value(acc) >= kMaxOpticalDepth) break;
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
    if (measure) {
      ws.max_hits = max(ws.max_hits, hits);
      if (ws.hist) atomicAdd(ws.hist + 16 * kKind + hits_bin(hits), 1ull);
    }
    return (kKind == kArgmin) ? t_hi : tau_value(acc);
  }
  __device__ float argmin(float3 o, float3 d, uint64_t key, ScatterAlbedo* sa) {
    sa->valid = false;  // the plain megakernel evaluates the albedo with its own point query
    sa->gauss = kNoGauss;
    return ray<kArgmin>(o, d, key);
  }
  __device__ float transmittance(float3 o, float3 d, uint32_t /*seed: the plain megakernel traverses*/ = kNoGauss) {
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
          if (measure) {
            ws.kind_prims[2]++;
            ws.kind_geo[2]++;
          }
          const PrimGeo g = load_geo(S.prims, pi);
          const float r2 = point_r2<kAcc>(g, x);
          if (r2 <= kExtent2) {
            const float wgt = g.icf * vexp<kAcc>(-0.5f * r2);
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

}  // namespace vp
