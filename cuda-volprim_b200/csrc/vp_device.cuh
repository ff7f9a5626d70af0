// Device-side data model and per-(ray, Gaussian) math shared by every kernel of the path.
//
// The reference evaluates each Gaussian through the `Primitive` methods
// (include/thesis/device/params/primitive.h:98-318), the ellipsoid helpers
// (include/thesis/common/geometry/intersection.h:56-173) and the sampling stages
// (device/core/sampling.cuh:74-583).  Here the same closed forms are written around one
// better-conditioned quantity, the ray's closest approach to the Gaussian centre in whitened
// space:
//   whitening   y = W (x - c),  W = diag(1/s) R(q)^T            (primitive.h:98-104)
//   w = W d,  t_c = -(W(o-c) . w) / |w|^2,  p_perp = W(o - c + t_c d),  d2 = |p_perp|^2
//   3-sigma chord: h = sqrt(9 - d2), t in [t_c - h/|w|, t_c + h/|w|]  (intersection.h:66-173)
//   optical depth over whitened arc [u0, h]:
//     tau = icf / |w| * exp(-d2/2) * (erf(h/sqrt2) - erf(u0/sqrt2))   (primitive.h:249-318)
//   free flight (span-restricted inverse CDF) for threshold tau:
//     u* = sqrt2 erfinv(erf(u0/sqrt2) + tau / K),  K = icf/|w| exp(-d2/2),
//     t = t_c + u*/|w|                                               (primitive.h:140-246)
// with icf = M (2 pi)^(-3/2) / prod(s) * sqrt(pi/2) (the reference's inv_cdf_factor_).
// Computing p_perp from o - c + t_c d in world space avoids the cancellation of the
// reference's p + t w form (|p| ~ distance/scale), which bounds FP32 transmittance accuracy
// well above 1e-5.  Everything here is FP32.  The ACCURATE variant carries the closest-approach
// vector, p_perp and d2 as unevaluated float pairs (hi + lo, built from the error-free TwoSum and
// FMA TwoProduct transforms), so 9 - d2 and the half-chord keep their bits on grazing chords,
// and sums optical depth in float pairs too.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vp {

// ---- constants (device/core/constants.cuh, include/thesis/common/utils/math.h) ----------
constexpr float kInf = 1e20f;               // consts::INF_F
constexpr float kExtent2 = 9.0f;            // GAUSSIAN_EXTENT_F^2 (3-sigma support)
constexpr float kMaxOpticalDepth = 88.0f;   // consts::MAX_OPTICAL_DEPTH
constexpr float kSegmentMin = 1e-6f;        // consts::RAY_SEGMENT_MIN_LENGTH
constexpr float kMinThroughput = 1e-4f;     // consts::MIN_THROUGHPUT
constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 2.0f * kPi;
constexpr float kInvPi = 1.0f / kPi;
constexpr float kInvTwoPi = 1.0f / (2.0f * kPi);
constexpr float kInvFourPi = 1.0f / (4.0f * kPi);  // consts::PHASE_VALUE
constexpr float kSqrt2 = 1.41421356237309504880f;
constexpr float kInvSqrt2 = 1.0f / 1.41421356237309504880f;

// Child-reference encoding of both BVHs.
constexpr uint32_t kEmptyRef = 0xFFFFFFFFu;
constexpr uint32_t kNoGauss = 0xFFFFFFFFu;  // no Gaussian (scene order)
constexpr uint32_t kLeafBit = 0x80000000u;
// Thread-private stack of the binary-tree traversal (megakernel); the scene build keeps the
// binary tree's height below it.
constexpr int kBinStack = 128;
__host__ __device__ inline bool ref_is_leaf(uint32_t r) { return (r & kLeafBit) != 0u; }
// BVH32 leaf: bit31 | (count-1) << 26 | first
__host__ __device__ inline uint32_t wide_leaf_ref(uint32_t first, uint32_t count) {
  return kLeafBit | ((count - 1u) << 26) | first;
}
__host__ __device__ inline uint32_t wide_leaf_first(uint32_t r) { return r & 0x03FFFFFFu; }
__host__ __device__ inline uint32_t wide_leaf_count(uint32_t r) { return ((r >> 26) & 31u) + 1u; }

// The argmin traversal pops best-first while its stack holds at most this many entries.
constexpr uint32_t kArgminBestFirstStack = 64;

// Device error words (raised instead of trapping; read back by the host).
constexpr uint32_t kStatusStackOverflow = 1u;
constexpr uint32_t kStatusBadInput = 2u;

// ---- views -------------------------------------------------------------------------------
// Per-Gaussian hot record, 64 B = four float4 (the reference's hot 64 B, primitive.h:47-61,
// with the quaternion + 1/scale folded into the whitening matrix W):
//   a = (c.x, c.y, c.z, W00)  b = (W01, W02, W10, W11)
//   c = (W12, W20, W21, W22)  d = (icf, albedo.r, albedo.g, albedo.b)
struct SceneView {
  const float4* prims;   // 4 float4 per Gaussian, in BVH (Morton) order
  const uint32_t* perm;  // Morton order -> caller's index (keys the free-flight draws)
  const float4* wide;    // BVH32: node k = 32 lo float4 then 32 hi float4; lo.w = child ref
  const float4* bin;     // binary LBVH: node i = (l_lo, l_hi, r_lo, r_hi); lo.w = child ref
  const float4* pbox;    // per Gaussian (Morton order): 3-sigma box lo, hi (2 float4)
  uint32_t count;
  uint32_t wide_root;    // ref of the BVH32 root (a node index; 0)
  uint32_t bin_root;     // ref of the binary root
  uint32_t stack_cap;    // per-warp stack entries a depth-first BVH32 traversal can need
  uint32_t argmin_cap;   // per-warp stack entries of the argmin traversal: stack_cap +
                         // kArgminBestFirstStack + 64 (best-first pops need room beyond the
                         // depth-first bound; see warp_ray_query)
  int32_t albedo_all_zero;
  uint32_t tau_nearest;  // transmittance stacks hit children nearest first (VP_TAU_ORDER_NEAREST)
};

struct CameraView {
  float3 eye, p00, du, dv, view_dir;
  int32_t ortho;
};

struct EnvView {
  const float4* texels;  // width*height RGBA, row-major (row = polar angle)
  const float2* cond;    // per texel: (alias probability, alias index bits) within its row
  const float2* marg;    // per row: (alias probability, alias row bits)
  const float* joint;    // per texel luminance * sin(theta_row)
  uint32_t width, height;
  float total;           // sum of joint (0 -> uniform-sphere fallback)
  float inv_total;
};

struct ParamsView {
  uint32_t width, height, spp_total, seed, max_bounces, rr_depth;
  float rr_max_survival, firefly_clamp, filter_stddev;
  int32_t nee_mode;
  uint32_t ris_k;
  int32_t hg_iso;
  float hg_g, hg_g_eff, hg_one_plus_g2, hg_one_minus_g2, hg_neg_inv_2g, hg_phase_coeff;
  int32_t accurate;
  int32_t measure;
  float adaptive_threshold;  // 0: adaptive sampling off
  uint32_t adaptive_min_samples;
};

struct Counters {  // device-side statistics (only touched when ParamsView::measure)
  unsigned long long bounces, scatters, crossings, shadow_rays, nodes, leaves;
  // per query kind (argmin, transmittance, albedo): inner nodes, leaves, Gaussian boxes tested,
  // Gaussian records loaded
  unsigned long long kind_nodes[3], kind_leaves[3], kind_prims[3], kind_geo[3];
  unsigned int max_hits, max_overlap, status;
  unsigned long long skipped;  // paths of converged pixels not traced (adaptive sampling)
  unsigned long long hits_hist[2][16];  // queries by chords evaluated, power-of-two bins (argmin, tau)
};

// Power-of-two bin of a per-query chord count: 0 -> 0, [2^(k-1), 2^k) -> k, >= 2^14 -> 15.
__device__ __forceinline__ int hits_bin(unsigned int n) { return n == 0u ? 0 : min(15, 32 - __clz(n)); }

// ---- small vector helpers ----------------------------------------------------------------
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 mul(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 mul(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) {  // math::dot order (math.h)
  return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z));
}
__device__ __forceinline__ float fmax3(float3 v) { return fmaxf(fmaxf(v.x, v.y), v.z); }
__device__ __forceinline__ float sum3(float3 v) { return v.x + v.y + v.z; }
__device__ __forceinline__ float3 fma3(float a, float3 b, float3 c) {
  return f3(fmaf(a, b.x, c.x), fmaf(a, b.y, c.y), fmaf(a, b.z, c.z));
}

// ---- float pairs: a value carried as an unevaluated sum hi + lo of two floats --------------
// Error-free transforms (Knuth's TwoSum, Dekker's FastTwoSum, the FMA TwoProduct) with IEEE
// round-to-nearest intrinsics, which the compiler neither contracts nor reassociates.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}
__device__ __forceinline__ void fast_two_sum(float a, float b, float& s, float& e) {  // |a| >= |b|
  s = __fadd_rn(a, b);
  e = __fsub_rn(b, __fsub_rn(s, a));
}
__device__ __forceinline__ void two_prod(float a, float b, float& p, float& e) {
  p = __fmul_rn(a, b);
  e = __fmaf_rn(a, b, -p);
}
struct FF {
  float hi, lo;
};
// hi + lo of a + b, with a and b float pairs
__device__ __forceinline__ FF ff_add(FF a, FF b) {
  float s, e;
  two_sum(a.hi, b.hi, s, e);
  FF r;
  fast_two_sum(s, __fadd_rn(e, __fadd_rn(a.lo, b.lo)), r.hi, r.lo);
  return r;
}
// acc += v (float), compensated
__device__ __forceinline__ void ff_accumulate(FF& acc, float v) {
  float s, e;
  two_sum(acc.hi, v, s, e);
  acc.hi = s;
  acc.lo = __fadd_rn(acc.lo, e);
}
// W x for x = xh + xl, as float pairs per component: sum_j W_ij xh_j exactly (TwoProduct +
// TwoSum) plus the first-order terms W_ij xl_j.
__device__ __forceinline__ void mat_vec_ff(const float (&W)[9], const float (&xh)[3], const float (&xl)[3],
                                           FF (&y)[3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float s, lo;
    two_prod(W[3 * i], xh[0], s, lo);
    lo = __fmaf_rn(W[3 * i], xl[0], lo);
#pragma unroll
    for (int j = 1; j < 3; ++j) {
      float p, pe, s2, se;
      two_prod(W[3 * i + j], xh[j], p, pe);
      two_sum(s, p, s2, se);
      s = s2;
      lo = __fadd_rn(lo, __fadd_rn(se, __fmaf_rn(W[3 * i + j], xl[j], pe)));
    }
    fast_two_sum(s, lo, y[i].hi, y[i].lo);
  }
}
// |y|^2 of a float-pair vector, as a float pair
__device__ __forceinline__ FF norm2_ff(const FF (&y)[3]) {
  float s, lo;
  two_prod(y[0].hi, y[0].hi, s, lo);
  lo = __fmaf_rn(2.0f * y[0].hi, y[0].lo, lo);
#pragma unroll
  for (int i = 1; i < 3; ++i) {
    float p, pe, s2, se;
    two_prod(y[i].hi, y[i].hi, p, pe);
    two_sum(s, p, s2, se);
    s = s2;
    lo = __fadd_rn(lo, __fadd_rn(se, __fmaf_rn(2.0f * y[i].hi, y[i].lo, pe)));
  }
  FF r;
  fast_two_sum(s, lo, r.hi, r.lo);
  return r;
}

// ---- RNG: PCG32 + 64-bit mixer, restated from device/core/random.cuh:16-58 ----------------
struct Pcg32 {
  uint64_t state, inc;
  __device__ __forceinline__ uint32_t next() {
    const uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    const uint32_t xorshifted = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = static_cast<uint32_t>(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
  }
  // float(next) / float(UINT32_MAX): float(UINT32_MAX) rounds to 2^32, so this is exact
  // scaling by 2^-32 (random.cuh:51-53); the value can equal 1.0.
  __device__ __forceinline__ float uniform() { return __uint2float_rn(next()) * 2.3283064365386963e-10f; }
};

__device__ __forceinline__ uint64_t seq_hash(uint64_t x) {  // random::hash (random.cuh:33-39)
  x = x * 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 27;
  x = x * 0x94d049bb133111ebULL;
  x ^= x >> 31;
  return x;
}

__device__ __forceinline__ Pcg32 pcg_init(uint64_t seed, uint64_t sequence) {  // random::init
  Pcg32 r;
  r.state = 0u;
  r.inc = (sequence << 1u) | 1u;
  r.next();
  r.state += seed;
  r.next();
  return r;
}

// Free-flight threshold of one Gaussian at one bounce, keyed by (bounce key, caller index).
// The reference draws these from the path's PCG32 in hit-buffer order, which is OptiX
// traversal order (sampling.cuh:348-349,356-377); keying the draw by Gaussian index instead
// makes the argmin independent of visit order, so a warp can reduce it in any order.
__device__ __forceinline__ uint32_t keyed_u32(uint64_t key, uint32_t idx) {
  uint64_t z = key ^ (static_cast<uint64_t>(idx) * 0x9E3779B97F4A7C15ULL);
  z ^= z >> 30;
  z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27;
  z *= 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return static_cast<uint32_t>(z >> 32);
}
// exp / log of the per-Gaussian terms: CUDA's full-accuracy functions for ACCURATE, the
// hardware-approximation intrinsics for FAST (the reference builds with -use_fast_math, which
// maps expf/logf to these, cmake/OptiX-IR.cmake:40-88).
template <bool kAcc>
__device__ __forceinline__ float vexp(float x) {
  if constexpr (kAcc) return expf(x);
  else return __expf(x);
}
template <bool kAcc>
__device__ __forceinline__ float vlog(float x) {
  if constexpr (kAcc) return logf(x);
  else return __logf(x);
}

// tau = -log(max(1 - chi, 1e-10)), chi uniform (sample_free_flight_tau, sampling.cuh:310-313)
template <bool kAcc>
__device__ __forceinline__ float free_flight_tau(uint64_t key, uint32_t idx) {
  const float chi = __uint2float_rn(keyed_u32(key, idx)) * 2.3283064365386963e-10f;
  return -vlog<kAcc>(fmaxf(1.0f - chi, 1e-10f));
}

// ---- Gaussian record access ----------------------------------------------------------------
struct PrimGeo {  // the record minus albedo
  float4 a, b, c;
  float icf;
};
__device__ __forceinline__ PrimGeo load_geo(const float4* __restrict__ prims, uint32_t i) {
  PrimGeo g;
  g.a = __ldg(prims + 4u * i + 0u);
  g.b = __ldg(prims + 4u * i + 1u);
  g.c = __ldg(prims + 4u * i + 2u);
  g.icf = __ldg(reinterpret_cast<const float*>(prims + 4u * i + 3u));
  return g;
}
__device__ __forceinline__ float3 load_albedo(const float4* __restrict__ prims, uint32_t i) {
  const float4 d = __ldg(prims + 4u * i + 3u);
  return f3(d.y, d.z, d.w);
}
__device__ __forceinline__ float3 whiten(const PrimGeo& g, float3 v) {
  return f3(fmaf(g.a.w, v.x, fmaf(g.b.x, v.y, g.b.y * v.z)),
            fmaf(g.b.z, v.x, fmaf(g.b.w, v.y, g.c.x * v.z)),
            fmaf(g.c.y, v.x, fmaf(g.c.z, v.y, g.c.w * v.z)));
}

// Chord of a ray through a Gaussian's 3-sigma ellipsoid, in the closest-approach frame.
struct Chord {
  float tc;    // ray parameter of the closest whitened approach
  float rw;    // 1 / |W d|
  float d2;    // squared whitened distance of closest approach
  float h;     // whitened half-chord sqrt(9 - d2)
  float t_in, t_out;
  float d2lo;  // ACCURATE: low part of d2 (d2 + d2lo is the float-pair value); 0 otherwise
};

// FP32 set-up.  o - c is split into hi + lo parts (TwoSum) so the world-space closest-approach
// vector keeps the bits the subtraction would round away.
__device__ __forceinline__ bool chord_fast(const PrimGeo& g, float3 o, float3 d, Chord& ch) {
  float3 dh, dl;
  {
    const float cx = g.a.x, cy = g.a.y, cz = g.a.z;
    dh.x = o.x - cx; { const float bb = dh.x - o.x; dl.x = (o.x - (dh.x - bb)) + (-cx - bb); }
    dh.y = o.y - cy; { const float bb = dh.y - o.y; dl.y = (o.y - (dh.y - bb)) + (-cy - bb); }
    dh.z = o.z - cz; { const float bb = dh.z - o.z; dl.z = (o.z - (dh.z - bb)) + (-cz - bb); }
  }
  const float3 w = whiten(g, d);
  const float3 q = whiten(g, dh);
  const float a2 = dot3(w, w);
  const float ra = __frcp_rn(a2);
  const float qw = dot3(q, w);
  // Early miss: the closest-approach distance is also |q|^2 - (q.w)^2 / |w|^2.  Its FP32 error is
  // a few ulps of |q|^2 (cancellation), so a lane above 9 + 1e-5 |q|^2 + 1e-4 is a miss for the
  // exact test below as well (inf and NaN never reject); the rest go through the compensated
  // closest-approach frame, so the chords are the same with or without this test.
  {
    const float qq = dot3(q, q);
    if (fmaf(-qw * qw, ra, qq) > fmaf(1e-5f, qq, kExtent2 + 1e-4f)) return false;
  }
  const float tc = -qw * ra;
  const float3 r = add(fma3(tc, d, dh), dl);
  const float3 pp = whiten(g, r);
  const float d2 = dot3(pp, pp);
  if (!(d2 < kExtent2)) return false;
  const float h = sqrtf(kExtent2 - d2);
  const float rw = rsqrtf(a2);
  ch.tc = tc;
  ch.rw = rw;
  ch.d2 = d2;
  ch.h = h;
  ch.t_in = fmaf(-h, rw, tc);
  ch.t_out = fmaf(h, rw, tc);
  ch.d2lo = 0.0f;
  return true;
}

// ACCURATE set-up, FP32 with float pairs.  o - c is exact as hi + lo (TwoSum); the closest
// approach r = (o - c) + t_c d is formed as a float pair (TwoProduct of t_c d, TwoSum with the
// hi part), p_perp = W r and d2 = |p_perp|^2 as float pairs; 9 - d2 is then exact up to the
// pair's rounding, and h = sqrt(9 - d2) gets its first-order correction.  t_c itself needs no
// extra bits: an error in it moves r along d, which changes d2 only to second order.
__device__ __forceinline__ bool chord_accurate(const PrimGeo& g, float3 o, float3 d, Chord& ch) {
  float Dh[3], Dl[3];
  two_sum(o.x, -g.a.x, Dh[0], Dl[0]);
  two_sum(o.y, -g.a.y, Dh[1], Dl[1]);
  two_sum(o.z, -g.a.z, Dh[2], Dl[2]);
  const float3 w = whiten(g, d);
  const float3 q = whiten(g, f3(Dh[0], Dh[1], Dh[2]));
  const float a2 = dot3(w, w);
  const float ra = __frcp_rn(a2);
  const float qw = dot3(q, w);
  {  // the FAST path's conservative early miss (same chords with or without it)
    const float qq = dot3(q, q);
    if (fmaf(-qw * qw, ra, qq) > fmaf(1e-5f, qq, kExtent2 + 1e-4f)) return false;
  }
  const float tc = -qw * ra;
  const float dd[3] = {d.x, d.y, d.z};
  float rh[3], rl[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float p, pe, s, se;
    two_prod(tc, dd[k], p, pe);
    two_sum(Dh[k], p, s, se);
    fast_two_sum(s, __fadd_rn(se, __fadd_rn(pe, Dl[k])), rh[k], rl[k]);
  }
  const float W[9] = {g.a.w, g.b.x, g.b.y, g.b.z, g.b.w, g.c.x, g.c.y, g.c.z, g.c.w};
  FF pp[3];
  mat_vec_ff(W, rh, rl, pp);
  const FF d2 = norm2_ff(pp);
  if (!(d2.hi < kExtent2)) return false;
  float m, me;
  two_sum(kExtent2, -d2.hi, m, me);
  me = __fsub_rn(me, d2.lo);
  if (!(m + me > 0.0f)) return false;
  const float hs = __fsqrt_rn(m);
  const float h = __fmaf_rn(me, __fdividef(0.5f, hs), hs);
  const float rw = __frsqrt_rn(a2);
  ch.tc = tc;
  ch.rw = rw;
  ch.d2 = d2.hi;
  ch.h = h;
  ch.t_in = fmaf(-h, rw, tc);
  ch.t_out = fmaf(h, rw, tc);
  ch.d2lo = d2.lo;
  return true;
}

template <bool kAccurate>
__device__ __forceinline__ bool chord_setup(const PrimGeo& g, float3 o, float3 d, Chord& ch) {
  if constexpr (kAccurate) return chord_accurate(g, o, d, ch);
  else return chord_fast(g, o, d, ch);
}

// Whitened arc-length at which the segment [max(t_in, t_lo), t_out] starts.
__device__ __forceinline__ float chord_u0(const Chord& ch, float t_lo) {
  return (ch.t_in >= t_lo) ? -ch.h : (t_lo - ch.tc) / ch.rw;
}

// erf(b/sqrt2) - erf(a/sqrt2) for a <= b, using erfc when both are positive (no cancellation
// near erf -> 1).
__device__ __forceinline__ float erf_diff(float a, float b) {
  if (a >= 0.0f) return erfcf(a * kInvSqrt2) - erfcf(b * kInvSqrt2);
  if (a == -b) return 2.0f * erff(b * kInvSqrt2);  // the whole chord, entered from outside (erf is odd)
  return erff(b * kInvSqrt2) - erff(a * kInvSqrt2);
}

// Optical depth of one Gaussian over the ray segment [max(t_in, t_lo), t_out]
// (Primitive::optical_depth, primitive.h:249-318; zero below RAY_SEGMENT_MIN_LENGTH).
// exp(-(d2 + d2lo) / 2) for a float-pair d2 (first order in the low part).
template <bool kAcc>
__device__ __forceinline__ float gauss_d2(float d2, float d2lo) {
  const float e = vexp<kAcc>(-0.5f * d2);
  if constexpr (kAcc) return __fmaf_rn(e, -0.5f * d2lo, e);
  else return e;
}

template <bool kAcc>
__device__ __forceinline__ float chord_tau(float tc, float rw, float d2, float h, float u0,
                                           float t_start, float t_out, float icf, float d2lo = 0.0f) {
  (void)tc;
  if (t_out - t_start <= kSegmentMin) return 0.0f;
  return icf * rw * gauss_d2<kAcc>(d2, d2lo) * erf_diff(u0, h);
}

// Analog free flight inside one Gaussian, restricted to t >= segment start, with the
// reference's acceptance rules (argmin_scatter_distance, sampling.cuh:350-415): +inf when the
// remaining mass is below tau (primitive.h:174,235); an entry hit's FP undershoot below its
// entry is clamped to the entry (sampling.cuh:392-394); valid only in [0, t_out].
template <bool kAcc>
__device__ __forceinline__ float chord_free_flight(float tc, float rw, float d2, float h,
                                                   float u0, float t_in, float t_out, float icf,
                                                   float tau, float d2lo = 0.0f) {
  (void)h;
  const float K = icf * rw * gauss_d2<kAcc>(d2, d2lo);
  const float raw = erff(u0 * kInvSqrt2) + tau / K;
  if (!(raw <= 1.0f)) return kInf;  // raw > 1 (or NaN): no scatter in this Gaussian
  const float arg = fmaxf(raw, -1.0f);
  float ts = fmaf(kSqrt2 * erfinvf(arg), rw, tc);
  if (t_in > 0.0f && ts >= 0.0f && ts < t_in) ts = t_in;
  if (ts >= 0.0f && ts <= t_out && ts < kInf) return ts;
  return kInf;
}

// ---- phase function (Henyey-Greenstein), sampling.cuh:74-134 -----------------------------
__device__ __forceinline__ float hg_eval_cos(const ParamsView& P, float cos_theta) {
  if (P.hg_iso) return kInvFourPi;
  const float denom = fmaf(-2.0f * P.hg_g, cos_theta, P.hg_one_plus_g2);
  const float is = rsqrtf(denom);
  return P.hg_phase_coeff * (is * is * is);
}
__device__ __forceinline__ float hg_eval(const ParamsView& P, float3 wi, float3 wo) {
  return hg_eval_cos(P, dot3(wi, wo));
}
__device__ __forceinline__ void onb_from_normal(float3 n, float3& tx, float3& ty) {
  const float sign = copysignf(1.0f, n.z);
  const float a = -1.0f / (sign + n.z);
  const float b = n.x * n.y * a;
  tx = f3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
  ty = f3(b, sign + n.y * n.y * a, -n.y);
}
__device__ __forceinline__ float3 hg_sample(const ParamsView& P, float3 wi, Pcg32& rng,
                                            float& pdf) {
  const float u0 = rng.uniform();
  const float u1 = rng.uniform();
  float cos_theta;
  if (P.hg_iso) {
    cos_theta = fmaf(-2.0f, u0, 1.0f);
  } else {
    const float g = P.hg_g_eff;
    const float inner = fmaf(-2.0f, u0, 1.0f);
    const float denom = fmaf(g, inner, 1.0f);
    const float sq = P.hg_one_minus_g2 / denom;
    cos_theta = P.hg_neg_inv_2g * fmaf(-sq, sq, P.hg_one_plus_g2);
  }
  const float sin_theta = sqrtf(fmaxf(0.0f, 1.0f - cos_theta * cos_theta));
  float sp, cp;
  sincosf(kTwoPi * u1, &sp, &cp);
  float3 ex, ey;
  onb_from_normal(wi, ex, ey);
  const float lx = sin_theta * cp, ly = sin_theta * sp;
  pdf = hg_eval_cos(P, cos_theta);
  return f3(lx * ex.x + ly * ey.x + cos_theta * wi.x, lx * ex.y + ly * ey.y + cos_theta * wi.y,
            lx * ex.z + ly * ey.z + cos_theta * wi.z);
}

// ---- environment map -----------------------------------------------------------------------
// Bilinear lat-long lookup with wrap in u and clamp in v, as the reference's tex2D on a
// normalised-coordinate, linear-filtered texture (device/params/environment_map.h:36-61,
// host/cuda/texture.h:75-79).  Filter weights are full FP32 (the texture unit's are 8-bit).
__device__ __forceinline__ float3 env_lookup(const EnvView& E, float3 dir) {
  const float theta = atan2f(dir.z, dir.x);
  const float phi = acosf(fminf(fmaxf(dir.y, -1.0f), 1.0f));
  float u = fmaf(theta, kInvTwoPi, 0.5f);
  const float v = phi * kInvPi;
  u = u - floorf(u);
  const float x = u * (float)E.width - 0.5f;
  const float y = v * (float)E.height - 0.5f;
  const float xf = floorf(x), yf = floorf(y);
  const float fx = x - xf, fy = y - yf;
  int i0 = (int)xf, j0 = (int)yf;
  int i1 = i0 + 1, j1 = j0 + 1;
  const int W = (int)E.width, H = (int)E.height;
  i0 = ((i0 % W) + W) % W;
  i1 = ((i1 % W) + W) % W;
  j0 = min(max(j0, 0), H - 1);
  j1 = min(max(j1, 0), H - 1);
  const float4 t00 = __ldg(E.texels + (size_t)j0 * W + i0);
  const float4 t01 = __ldg(E.texels + (size_t)j0 * W + i1);
  const float4 t10 = __ldg(E.texels + (size_t)j1 * W + i0);
  const float4 t11 = __ldg(E.texels + (size_t)j1 * W + i1);
  const float gx = 1.0f - fx, gy = 1.0f - fy;
  return f3(gy * (gx * t00.x + fx * t01.x) + fy * (gx * t10.x + fx * t11.x),
            gy * (gx * t00.y + fx * t01.y) + fy * (gx * t10.y + fx * t11.y),
            gy * (gx * t00.z + fx * t01.z) + fy * (gx * t10.z + fx * t11.z));
}

__device__ __forceinline__ uint32_t alias_pick(const float2* __restrict__ table, uint32_t n,
                                               uint32_t r) {
  const uint64_t x = static_cast<uint64_t>(r) * n;
  const uint32_t idx = static_cast<uint32_t>(x >> 32);
  const float coin = __uint2float_rn(static_cast<uint32_t>(x)) * 2.3283064365386963e-10f;
  const float2 e = __ldg(table + idx);
  return coin < e.x ? idx : __float_as_uint(e.y);
}

// Environment importance sampling (env_is::sample, sampling.cuh:173-216): texel chosen in
// proportion to luminance * sin(theta) -- here by a marginal alias table over rows and a
// per-row alias table, O(1) instead of two binary searches -- then a continuous position
// inside the texel.  Draw count and pdf are the reference's.
__device__ __forceinline__ float3 env_sample(const EnvView& E, Pcg32& rng, float& pdf) {
  const uint32_t r0 = rng.next();
  const uint32_t r1 = rng.next();
  if (!(E.total > 0.0f) || E.width == 0u || E.height == 0u) {
    const float u0 = __uint2float_rn(r0) * 2.3283064365386963e-10f;
    const float u1 = __uint2float_rn(r1) * 2.3283064365386963e-10f;
    const float z = fmaf(-2.0f, u0, 1.0f);
    const float r = sqrtf(fmaxf(0.0f, fmaf(-z, z, 1.0f)));
    float sp, cp;
    sincosf(kTwoPi * u1, &sp, &cp);
    pdf = kInvFourPi;
    return f3(r * cp, r * sp, z);
  }
  const uint32_t W = E.width, H = E.height;
  const uint32_t v = alias_pick(E.marg, H, r0);
  const uint32_t u = alias_pick(E.cond + (size_t)v * W, W, r1);
  const float jx = rng.uniform();
  const float jy = rng.uniform();
  const float u_norm = ((float)u + jx) / (float)W;
  const float v_norm = ((float)v + jy) / (float)H;
  const float theta = fmaf(2.0f * kPi, u_norm, -kPi);
  const float polar = v_norm * kPi;
  float sin_p, cos_p, sin_t, cos_t;
  sincosf(polar, &sin_p, &cos_p);
  sincosf(theta, &sin_t, &cos_t);
  const float joint = __ldg(E.joint + (size_t)v * W + u);
  const float p_uv = (joint * E.inv_total) * (float)(W * H);
  const float jac = 2.0f * kPi * kPi * sin_p;
  pdf = (sin_p > 0.0f) ? p_uv / jac : 0.0f;
  return f3(sin_p * cos_t, cos_p, sin_p * sin_t);
}

__device__ __forceinline__ float env_pdf(const EnvView& E, float3 wo) {  // env_is::pdf
  if (!(E.total > 0.0f) || E.width == 0u || E.height == 0u) return kInvFourPi;
  const int W = (int)E.width, H = (int)E.height;
  const float theta = atan2f(wo.z, wo.x);
  const float polar = acosf(fminf(fmaxf(wo.y, -1.0f), 1.0f));
  const float u_norm = fmaf(theta, kInvTwoPi, 0.5f);
  const float v_norm = polar * kInvPi;
  int u = (int)(u_norm * (float)W);
  int v = (int)(v_norm * (float)H);
  u = u < 0 ? 0 : (u >= W ? W - 1 : u);
  v = v < 0 ? 0 : (v >= H ? H - 1 : v);
  const float joint = __ldg(E.joint + (size_t)v * W + u);
  const float sin_p = sinf(polar);
  if (joint <= 0.0f || sin_p <= 0.0f) return 0.0f;
  const float p_uv = (joint * E.inv_total) * (float)(W * H);
  return p_uv / (2.0f * kPi * kPi * sin_p);
}

__device__ __forceinline__ float mis_balance(float a, float b) {
  const float s = a + b;
  return (s > 0.0f) ? a / s : 0.0f;
}

// ---- camera (device/params/camera.h:33-57, random.cuh:55-72) ------------------------------
// IEEE-rounded operations only (no contraction, correctly rounded normalisation) so the
// host oracle reproduces every camera ray bit for bit.
__device__ __forceinline__ void camera_ray(const CameraView& C, const ParamsView& P, uint32_t px,
                                           uint32_t py, Pcg32& rng, float3& o, float3& d) {
  float jx, jy;
  if (P.filter_stddev > 0.0f) {
    const float u1 = fmaxf(rng.uniform(), 1e-7f);
    const float u2 = rng.uniform();
    const float r = P.filter_stddev * sqrtf(-2.0f * logf(u1));
    float s, c;
    sincosf(kTwoPi * u2, &s, &c);
    jx = fminf(fmaxf(r * c, -2.0f), 2.0f);
    jy = fminf(fmaxf(r * s, -2.0f), 2.0f);
  } else {
    jx = __fsub_rn(rng.uniform(), 0.5f);
    jy = __fsub_rn(rng.uniform(), 0.5f);
  }
  const float x = __fadd_rn((float)px, jx);
  const float y = __fadd_rn((float)py, jy);
  const float3 off = f3(fmaf(x, C.du.x, fmaf(y, C.dv.x, C.p00.x)),
                        fmaf(x, C.du.y, fmaf(y, C.dv.y, C.p00.y)),
                        fmaf(x, C.du.z, fmaf(y, C.dv.z, C.p00.z)));
  if (C.ortho) {
    o = f3(__fadd_rn(C.eye.x, off.x), __fadd_rn(C.eye.y, off.y), __fadd_rn(C.eye.z, off.z));
    d = C.view_dir;
  } else {
    const float l2 = fmaf(off.x, off.x, fmaf(off.y, off.y, __fmul_rn(off.z, off.z)));
    const float inv = __fdiv_rn(1.0f, __fsqrt_rn(l2));
    o = C.eye;
    d = f3(__fmul_rn(off.x, inv), __fmul_rn(off.y, inv), __fmul_rn(off.z, inv));
  }
}

// ---- warp helpers -------------------------------------------------------------------------
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}
// Sum of the lanes' float pairs, as a float.
__device__ __forceinline__ float warp_sum_ff(FF v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    FF w;
    w.hi = __shfl_xor_sync(0xFFFFFFFFu, v.hi, o);
    w.lo = __shfl_xor_sync(0xFFFFFFFFu, v.lo, o);
    v = ff_add(v, w);
  }
  return __fadd_rn(v.hi, v.lo);
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  return v;
}

}  // namespace vp
