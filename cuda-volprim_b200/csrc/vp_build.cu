// Scene build on the device: per-Gaussian precompute, 3-sigma ellipsoid bounds, 63-bit Morton
// codes, radix sort, then two binary trees over the sorted boxes -- a Karras radix tree with a
// bottom-up refit (the thread-per-ray megakernel's tree) and a PLOC agglomerative clustering
// (the warp engines' tree) -- and the collapse of the latter to a 32-wide BVH, whose depth-first
// leaf order becomes the scene order of the Gaussians.
//
// Replaces the reference's host Morton sort + OptiX unit-sphere GAS / instance IAS build
// (src/thesis/host/app/renderer.cpp:85-173, include/thesis/host/utils/math.h:103-131,
// include/thesis/host/optix/acceleration_structure.h:23-87) and the Primitive precompute
// (include/thesis/device/params/primitive.h:70-87) plus PLY-load validation
// (src/thesis/host/utils/io/ply.cpp:124-172).

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "vp_internal.h"

namespace vp {
namespace {

struct ErrorWords {
  int bad_scale, bad_density, bad_center;  // lowest failing index (INT_MAX = none)
  unsigned int any_albedo;                 // 1 if some albedo component > 0
  unsigned int opaque_cores;               // Gaussians opaque at their core (vp_tau_order AUTO)
};

// A Gaussian is "opaque at its core" when the optical depth through its centre along its thinnest
// direction, M / (2 pi s_mid s_max), is at least this (4 x MAX_OPTICAL_DEPTH).
constexpr float kOpaqueCoreTau = 4.0f * kMaxOpticalDepth;

__device__ __forceinline__ float clamp_albedo(float v) {
  if (!isfinite(v)) return 0.0f;
  if (v < 0.0f) return 0.0f;
  if (v > 1.0f) return 1.0f;
  return v;
}

// One thread per Gaussian: the reference's Primitive constructor arithmetic in FP32 (host
// order; IEEE division/sqrt), the whitening matrix W = diag(1/s) R(q)^T and the 3-sigma
// ellipsoid's axis-aligned bound (from renderer.cpp:142-157's local-to-world TRS with 3x scale).
__global__ void k_precompute(uint32_t n, const float* __restrict__ mean,
                             const float* __restrict__ scale, const float* __restrict__ quat,
                             const float* __restrict__ density, const float* __restrict__ albedo,
                             int scale_is_log, float sigma_multiplier, float4* __restrict__ rec,
                             float4* __restrict__ lo, float4* __restrict__ hi,
                             ErrorWords* __restrict__ err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float cx = mean[3 * i], cy = mean[3 * i + 1], cz = mean[3 * i + 2];
  float sx = scale[3 * i], sy = scale[3 * i + 1], sz = scale[3 * i + 2];
  if (scale_is_log) {
    sx = expf(sx);
    sy = expf(sy);
    sz = expf(sz);
  }
  const float qw = quat[4 * i], qx = quat[4 * i + 1], qy = quat[4 * i + 2], qz = quat[4 * i + 3];
  // UnitQuaternion::from: rlength(float4(w,x,y,z)) = 1 / sqrt(fma(w,w,fma(x,x,fma(y,y,z*z))))
  const float qr = __fdiv_rn(1.0f, __fsqrt_rn(fmaf(qw, qw, fmaf(qx, qx, fmaf(qy, qy, __fmul_rn(qz, qz))))));
  const float w = __fmul_rn(qw, qr), x = __fmul_rn(qx, qr), y = __fmul_rn(qy, qr), z = __fmul_rn(qz, qr);
  const float M = __fmul_rn(density[i], sigma_multiplier);  // ply.cpp:116
  float ar = 0.f, ag = 0.f, ab = 0.f;
  if (albedo) {
    ar = clamp_albedo(albedo[3 * i]);
    ag = clamp_albedo(albedo[3 * i + 1]);
    ab = clamp_albedo(albedo[3 * i + 2]);
  }
  if (ar > 0.f || ag > 0.f || ab > 0.f) atomicOr(&err->any_albedo, 1u);
  const bool scale_ok = sx > 0.f && sy > 0.f && sz > 0.f && isfinite(sx) && isfinite(sy) && isfinite(sz);
  if (!scale_ok) atomicMin(&err->bad_scale, (int)i);
  if (!(M > 0.f) || !isfinite(M)) atomicMin(&err->bad_density, (int)i);
  if (!isfinite(cx) || !isfinite(cy) || !isfinite(cz) || !isfinite(w) || !isfinite(x) ||
      !isfinite(y) || !isfinite(z))
    atomicMin(&err->bad_center, (int)i);
  {
    const float smax = fmaxf(sx, fmaxf(sy, sz)), smin = fminf(sx, fminf(sy, sz));
    const float smid = sx + sy + sz - smax - smin;
    const bool core = scale_ok && M >= kOpaqueCoreTau * 6.28318531f * smid * smax;
    const unsigned am = __activemask();
    const unsigned cm = __ballot_sync(am, core);
    if (cm && (int)(threadIdx.x & 31) == __ffs(am) - 1) atomicAdd(&err->opaque_cores, (unsigned)__popc(cm));
  }
  // Primitive ctor (primitive.h:80-87): rcp_scale, density_norm_factor, inv_cdf_factor.
  const float rx = __fdiv_rn(1.0f, sx), ry = __fdiv_rn(1.0f, sy), rz = __fdiv_rn(1.0f, sz);
  const float dnf = __fmul_rn(0.0634936359f, __fmul_rn(__fmul_rn(rx, ry), rz));
  const float icf = __fmul_rn(__fmul_rn(M, dnf), 1.2533141373f);
  // Forward rotation matrix R(q) (include/thesis/host/utils/math.h:52-97 without scale) as float
  // pairs: each product of two quaternion components is exact as a TwoProduct pair, so every
  // entry carries ~44 bits, and W = diag(rcp_scale) R^T is rounded to FP32 once.
  auto sq2 = [](float a, float b, float c, float d, float sgn) {  // a*b + sgn*c*d as a float pair
    float p, pe, q, qe, s, se;
    two_prod(a, b, p, pe);
    two_prod(c, d, q, qe);
    if (sgn < 0.f) q = -q, qe = -qe;
    two_sum(p, q, s, se);
    FF r;
    fast_two_sum(s, __fadd_rn(se, __fadd_rn(pe, qe)), r.hi, r.lo);
    return r;
  };
  auto one_minus_2 = [](FF v) {  // 1 - 2 v
    float s, se;
    two_sum(1.0f, -2.0f * v.hi, s, se);
    FF r;
    fast_two_sum(s, __fsub_rn(se, 2.0f * v.lo), r.hi, r.lo);
    return r;
  };
  auto twice = [](FF v) { return FF{2.0f * v.hi, 2.0f * v.lo}; };
  FF R[3][3];
  R[0][0] = one_minus_2(sq2(y, y, z, z, 1.f));
  R[0][1] = twice(sq2(x, y, w, z, -1.f));
  R[0][2] = twice(sq2(x, z, w, y, 1.f));
  R[1][0] = twice(sq2(x, y, w, z, 1.f));
  R[1][1] = one_minus_2(sq2(x, x, z, z, 1.f));
  R[1][2] = twice(sq2(y, z, w, x, -1.f));
  R[2][0] = twice(sq2(x, z, w, y, -1.f));
  R[2][1] = twice(sq2(y, z, w, x, 1.f));
  R[2][2] = one_minus_2(sq2(x, x, y, y, 1.f));
  const float rs[3] = {rx, ry, rz};
  const float ss[3] = {sx, sy, sz};
  float W[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      float p, pe;
      two_prod(rs[r], R[c][r].hi, p, pe);
      W[r][c] = __fadd_rn(p, __fmaf_rn(rs[r], R[c][r].lo, pe));
    }
  rec[4 * i + 0] = make_float4(cx, cy, cz, W[0][0]);
  rec[4 * i + 1] = make_float4(W[0][1], W[0][2], W[1][0], W[1][1]);
  rec[4 * i + 2] = make_float4(W[1][2], W[2][0], W[2][1], W[2][2]);
  rec[4 * i + 3] = make_float4(icf, ar, ag, ab);
  float e[3];
  const float cen[3] = {cx, cy, cz};
  for (int k = 0; k < 3; ++k) {
    const float a0 = R[k][0].hi * ss[0], a1 = R[k][1].hi * ss[1], a2 = R[k][2].hi * ss[2];
    // 3-sigma half extent along world axis k, padded (1e-5 relative, far above the few-ulp error
    // of this FP32 evaluation) so FP32 chord tests never escape it; the box is rounded outward.
    e[k] = __fadd_ru(__fmul_ru(3.0f * sqrtf(fmaf(a0, a0, fmaf(a1, a1, a2 * a2))), 1.0f + 1e-5f),
                     1e-7f * (1.0f + fabsf(cen[k])));
  }
  lo[i] = make_float4(__fsub_rd(cx, e[0]), __fsub_rd(cy, e[1]), __fsub_rd(cz, e[2]), 0.f);
  hi[i] = make_float4(__fadd_ru(cx, e[0]), __fadd_ru(cy, e[1]), __fadd_ru(cz, e[2]), 0.f);
}

__device__ __forceinline__ unsigned int f2ord(float f) {
  const unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned int u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// Bounds of the Gaussian centres (Morton frame, as computeBounds in math.h:135-160) and of
// the 3-sigma boxes (scene bounds).
__global__ void k_bounds(uint32_t n, const float* __restrict__ mean, const float4* __restrict__ lo,
                         const float4* __restrict__ hi, unsigned int* __restrict__ out12) {
  float cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
  float bmn[3] = {INFINITY, INFINITY, INFINITY}, bmx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    for (int k = 0; k < 3; ++k) {
      const float c = mean[3 * i + k];
      cmn[k] = fminf(cmn[k], c);
      cmx[k] = fmaxf(cmx[k], c);
    }
    const float4 l = lo[i], h = hi[i];
    bmn[0] = fminf(bmn[0], l.x); bmn[1] = fminf(bmn[1], l.y); bmn[2] = fminf(bmn[2], l.z);
    bmx[0] = fmaxf(bmx[0], h.x); bmx[1] = fmaxf(bmx[1], h.y); bmx[2] = fmaxf(bmx[2], h.z);
  }
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      cmn[k] = fminf(cmn[k], __shfl_xor_sync(0xFFFFFFFFu, cmn[k], o));
      cmx[k] = fmaxf(cmx[k], __shfl_xor_sync(0xFFFFFFFFu, cmx[k], o));
      bmn[k] = fminf(bmn[k], __shfl_xor_sync(0xFFFFFFFFu, bmn[k], o));
      bmx[k] = fmaxf(bmx[k], __shfl_xor_sync(0xFFFFFFFFu, bmx[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int k = 0; k < 3; ++k) {
      atomicMin(&out12[k], f2ord(cmn[k]));
      atomicMax(&out12[3 + k], f2ord(cmx[k]));
      atomicMin(&out12[6 + k], f2ord(bmn[k]));
      atomicMax(&out12[9 + k], f2ord(bmx[k]));
    }
  }
}

__device__ __forceinline__ uint64_t expand21(uint64_t v) {  // 21 bits -> every third of 63
  v &= 0x1FFFFFull;
  v = (v | (v << 32)) & 0x1F00000000FFFFull;
  v = (v | (v << 16)) & 0x1F0000FF0000FFull;
  v = (v | (v << 8)) & 0x100F00F00F00F00Full;
  v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

// 63-bit Morton code of each centre (21 bits per axis; the reference uses 10 bits per axis on
// the host, math.h:117-131 -- more bits keep 2M-Gaussian scenes from collapsing into shared
// codes).
__global__ void k_morton(uint32_t n, const float* __restrict__ mean, const unsigned int* __restrict__ b,
                         uint64_t* __restrict__ codes, uint32_t* __restrict__ idx) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t code = 0;
  for (int k = 0; k < 3; ++k) {
    const float mn = ord2f(b[k]), mx = ord2f(b[3 + k]);
    const float inv = 1.0f / fmaxf(mx - mn, 1e-30f);
    const float t = fminf(fmaxf((mean[3 * i + k] - mn) * inv, 0.0f), 1.0f);
    const uint64_t q = (uint64_t)(t * 2097151.0f);
    code |= expand21(q) << k;  // x lowest bit, then y, then z (math.h:128)
  }
  codes[i] = code;
  idx[i] = i;
}

// Records and 3-sigma boxes in scene order (order[i] = caller index of scene position i).
__global__ void k_gather(uint32_t n, const uint32_t* __restrict__ order, const float4* __restrict__ rec_in,
                         const float4* __restrict__ lo_in, const float4* __restrict__ hi_in,
                         float4* __restrict__ rec_out, float4* __restrict__ pbox) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = order[i];
  for (int k = 0; k < 4; ++k) rec_out[4 * i + k] = rec_in[4 * s + k];
  pbox[2 * i] = lo_in[s];
  pbox[2 * i + 1] = hi_in[s];
}

// 3-sigma boxes in Morton order: the input of both tree builders.
__global__ void k_gather_boxes(uint32_t n, const uint32_t* __restrict__ order, const float4* __restrict__ lo_in,
                               const float4* __restrict__ hi_in, float4* __restrict__ lo_out,
                               float4* __restrict__ hi_out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = order[i];
  lo_out[i] = make_float4(lo_in[s].x, lo_in[s].y, lo_in[s].z, 0.f);
  hi_out[i] = make_float4(hi_in[s].x, hi_in[s].y, hi_in[s].z, 0.f);
}

__global__ void k_gather_raw(uint32_t n, const uint32_t* __restrict__ order, const float* __restrict__ scale,
                             const float* __restrict__ quat, const float* __restrict__ density,
                             float4* __restrict__ raw) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = order[i];
  raw[2 * i] = make_float4(quat[4 * s], quat[4 * s + 1], quat[4 * s + 2], quat[4 * s + 3]);
  raw[2 * i + 1] = make_float4(scale[3 * s], scale[3 * s + 1], scale[3 * s + 2], density[s]);
}

__device__ __forceinline__ int karras_delta(const uint64_t* __restrict__ codes, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint64_t a = codes[i], b = codes[j];
  if (a == b) return 64 + __clz(i ^ j);
  return __clzll(a ^ b);
}

// Karras 2012 ("Maximizing parallelism in the construction of BVHs, octrees, and k-d trees"):
// one thread per internal node of the binary radix tree over the sorted codes.
__global__ void k_karras(int n, const uint64_t* __restrict__ codes, uint32_t* __restrict__ left,
                         uint32_t* __restrict__ right, uint32_t* __restrict__ first,
                         uint32_t* __restrict__ last, uint32_t* __restrict__ parent_int,
                         uint32_t* __restrict__ parent_leaf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (karras_delta(codes, n, i, i + 1) - karras_delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = karras_delta(codes, n, i, i - d);
  int lmax = 2;
  while (karras_delta(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (karras_delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = karras_delta(codes, n, i, j);
  int s = 0, t = l;
  do {
    t = (t + 1) >> 1;
    if (karras_delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int gamma = i + s * d + min(d, 0);
  const int lo_i = min(i, j), hi_i = max(i, j);
  uint32_t lref, rref;
  if (lo_i == gamma) {
    lref = kLeafBit | (uint32_t)gamma;
    parent_leaf[gamma] = i;
  } else {
    lref = (uint32_t)gamma;
    parent_int[gamma] = i;
  }
  if (hi_i == gamma + 1) {
    rref = kLeafBit | (uint32_t)(gamma + 1);
    parent_leaf[gamma + 1] = i;
  } else {
    rref = (uint32_t)(gamma + 1);
    parent_int[gamma + 1] = i;
  }
  left[i] = lref;
  right[i] = rref;
  first[i] = lo_i;
  last[i] = hi_i;
}

// Box of a binary-tree child and the number of Gaussians under it (internal nodes keep the count
// in hi.w).
__device__ __forceinline__ uint32_t child_box(uint32_t ref, const float4* plo, const float4* phi,
                                              const float4* nlo, const float4* nhi, float4& l, float4& h) {
  if (ref_is_leaf(ref)) {
    const uint32_t p = ref & ~kLeafBit;
    l = plo[p];
    h = phi[p];
    return 1u;
  }
  l = __ldcg(nlo + ref);
  h = __ldcg(nhi + ref);
  return __float_as_uint(h.w);
}

// Bottom-up refit: the second thread to reach an internal node unions its children.
__global__ void k_refit(int n, const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                        const uint32_t* __restrict__ parent_int, const uint32_t* __restrict__ parent_leaf,
                        const float4* __restrict__ plo, const float4* __restrict__ phi,
                        float4* nlo, float4* nhi, unsigned int* flags) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || n < 2) return;
  uint32_t node = parent_leaf[k];
  while (true) {
    __threadfence();
    if (atomicAdd(&flags[node], 1u) == 0u) return;
    __threadfence();
    float4 al, ah, bl, bh;
    const uint32_t ca = child_box(left[node], plo, phi, nlo, nhi, al, ah);
    const uint32_t cb = child_box(right[node], plo, phi, nlo, nhi, bl, bh);
    __stcg(nlo + node, make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.f));
    __stcg(nhi + node, make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), __uint_as_float(ca + cb)));
    if (node == 0u) return;
    node = parent_int[node];
  }
}

// Binary-LBVH node records for the thread-per-ray megakernel: (l_lo, l_hi, r_lo, r_hi), child
// refs in l_lo.w / r_lo.w (leaf bit | scene-order Gaussian index: pos maps Morton order to it).
__global__ void k_binary_nodes(int n, const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                               const float4* __restrict__ plo, const float4* __restrict__ phi,
                               const float4* __restrict__ nlo, const float4* __restrict__ nhi,
                               const uint32_t* __restrict__ pos, float4* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  auto scene_ref = [&](uint32_t r) { return ref_is_leaf(r) ? (kLeafBit | pos[r & ~kLeafBit]) : r; };
  float4 al, ah, bl, bh;
  child_box(left[i], plo, phi, nlo, nhi, al, ah);
  child_box(right[i], plo, phi, nlo, nhi, bl, bh);
  al.w = __uint_as_float(scene_ref(left[i]));
  bl.w = __uint_as_float(scene_ref(right[i]));
  ah.w = 0.f;
  bh.w = 0.f;
  out[4 * i + 0] = al;
  out[4 * i + 1] = ah;
  out[4 * i + 2] = bl;
  out[4 * i + 3] = bh;
}

// ------------------------------------------------------------------------------------------
// PLOC: Meister & Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume Hierarchy
// Construction" (IEEE TVCG 2018).  Clusters start as the Morton-sorted Gaussian boxes; every pass,
// each cluster finds the neighbour within kPlocRadius positions whose union box has the smallest
// surface area, mutual nearest neighbours merge into a new binary node (at the lower position),
// and the cluster array is compacted in order.  Node ids are handed out in merge order, so the
// root is node n - 2.
// ------------------------------------------------------------------------------------------
constexpr int kPlocRadius = 32;
constexpr int kPlocBlock = 256;

// A cluster is (lo.xyz, ref bits in lo.w) and (hi.xyz, Gaussian count bits in hi.w); refs are
// binary node ids or kLeafBit | Morton position.
__global__ void k_ploc_init(uint32_t n, const float4* __restrict__ plo, const float4* __restrict__ phi,
                            float4* __restrict__ cl, float4* __restrict__ ch) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 l = plo[i], h = phi[i];
  l.w = __uint_as_float(kLeafBit | i);
  h.w = __uint_as_float(1u);
  cl[i] = l;
  ch[i] = h;
}

// Surface area of the union of two boxes; the same value whichever box comes first, and NaN
// (from non-finite extents) ordered as +inf, so the pair order below is a total order and the
// globally smallest pair is always mutual (every pass merges at least once).
__device__ __forceinline__ float union_area(float4 al, float4 ah, float4 bl, float4 bh) {
  const float dx = fmaxf(ah.x, bh.x) - fminf(al.x, bl.x);
  const float dy = fmaxf(ah.y, bh.y) - fminf(al.y, bl.y);
  const float dz = fmaxf(ah.z, bh.z) - fminf(al.z, bl.z);
  const float a = 2.f * (dx * dy + dy * dz + dz * dx);
  return a == a ? a : INFINITY;
}

// The pass kernels take the live cluster count from ctr_in = (clusters, nodes made so far), written
// by the previous pass, so a run of passes needs no host round trip; grids cover an upper bound.
__global__ void __launch_bounds__(kPlocBlock) k_ploc_nn(const uint32_t* __restrict__ ctr_in,
                                                        const float4* __restrict__ cl,
                                                        const float4* __restrict__ ch, uint32_t* __restrict__ nn) {
  __shared__ float4 sl[kPlocBlock + 2 * kPlocRadius], sh[kPlocBlock + 2 * kPlocRadius];
  const uint32_t m = ctr_in[0];
  if (m < 2u) return;
  const int b0 = (int)(blockIdx.x * kPlocBlock);
  if (b0 >= (int)m) return;
  for (int k = threadIdx.x; k < kPlocBlock + 2 * kPlocRadius; k += blockDim.x) {
    const int g = b0 - kPlocRadius + k;
    if (g >= 0 && g < (int)m) {
      sl[k] = cl[g];
      sh[k] = ch[g];
    }
  }
  __syncthreads();
  const int i = b0 + (int)threadIdx.x;
  if (i >= (int)m) return;
  const int c = (int)threadIdx.x + kPlocRadius;
  const float4 al = sl[c], ah = sh[c];
  float best = INFINITY;
  int bj = -1;
  for (int k = -kPlocRadius; k <= kPlocRadius; ++k) {
    const int j = i + k;
    if (k == 0 || j < 0 || j >= (int)m) continue;
    const float a = union_area(al, ah, sl[c + k], sh[c + k]);
    // pair order: area, then buddy pairs (2k, 2k + 1) first -- so equal boxes pair up in halves
    // instead of chaining -- then the pair's lower position, then its upper position
    bool take = bj < 0 || a < best;
    if (!take && a == best) {
      const int lo_new = min(i, j), lo_old = min(i, bj);
      const bool bud_new = !(lo_new & 1) && max(i, j) == lo_new + 1;
      const bool bud_old = !(lo_old & 1) && max(i, bj) == lo_old + 1;
      take = (bud_new != bud_old) ? bud_new
                                  : (lo_new < lo_old || (lo_new == lo_old && max(i, j) < max(i, bj)));
    }
    if (take) {
      best = a;
      bj = j;
    }
  }
  nn[i] = (uint32_t)bj;
}

// f[i] = merge << 32 | keep: the lower cluster of a mutual pair creates the node (merge) and keeps
// its position; the upper one is absorbed (keep = 0).
// Entries in [m, bound) are 0 so that the scan may run over the grid's upper bound; a lone
// cluster (m == 1) just keeps its place.
__global__ void k_ploc_flags(uint32_t bound, const uint32_t* __restrict__ ctr_in, const uint32_t* __restrict__ nn,
                             unsigned long long* __restrict__ f) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= bound) return;
  const uint32_t m = ctr_in[0];
  if (i >= m || m < 2u) {
    f[i] = (i == 0u && m == 1u) ? 1ull : 0ull;
    return;
  }
  const uint32_t j = nn[i];
  const bool mutual = nn[j] == i;
  const unsigned long long merge = (mutual && i < j) ? 1ull : 0ull;
  const unsigned long long keep = (mutual && i > j) ? 0ull : 1ull;
  f[i] = (merge << 32) | keep;
}

// Writes the merged nodes (Gaussian count in nhi.w, height in nlo.w) and the compacted clusters;
// ctr_out = (clusters left, nodes made).
__global__ void k_ploc_write(const uint32_t* __restrict__ ctr_in, uint32_t* __restrict__ ctr_out,
                             const uint32_t* __restrict__ nn, const unsigned long long* __restrict__ f,
                             const unsigned long long* __restrict__ x, const float4* __restrict__ cl,
                             const float4* __restrict__ ch, float4* __restrict__ ol, float4* __restrict__ oh,
                             uint32_t* __restrict__ left, uint32_t* __restrict__ right, float4* __restrict__ nlo,
                             float4* __restrict__ nhi) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t m = ctr_in[0], node_base = ctr_in[1];
  if (i >= m) return;
  const unsigned long long fi = f[i], xi = x[i];
  if (i == m - 1u) {
    ctr_out[0] = (uint32_t)(xi & 0xFFFFFFFFull) + (uint32_t)(fi & 1ull);
    ctr_out[1] = node_base + (uint32_t)((xi >> 32) + (fi >> 32));
  }
  if (!(fi & 1ull)) return;
  float4 l = cl[i], h = ch[i];
  if (fi >> 32) {
    const uint32_t j = nn[i];
    const float4 bl = cl[j], bh = ch[j];
    const uint32_t node = node_base + (uint32_t)(xi >> 32);
    const uint32_t lref = __float_as_uint(l.w), rref = __float_as_uint(bl.w);
    left[node] = lref;
    right[node] = rref;
    // node height (leaf refs 0) in nlo.w: the children were made in earlier passes
    const uint32_t hl = ref_is_leaf(lref) ? 0u : __float_as_uint(nlo[lref].w);
    const uint32_t hr = ref_is_leaf(rref) ? 0u : __float_as_uint(nlo[rref].w);
    l = make_float4(fminf(l.x, bl.x), fminf(l.y, bl.y), fminf(l.z, bl.z), __uint_as_float(node));
    h = make_float4(fmaxf(h.x, bh.x), fmaxf(h.y, bh.y), fmaxf(h.z, bh.z),
                    __uint_as_float(__float_as_uint(h.w) + __float_as_uint(bh.w)));
    nlo[node] = make_float4(l.x, l.y, l.z, __uint_as_float(1u + max(hl, hr)));
    nhi[node] = h;
  }
  const uint32_t p = (uint32_t)(xi & 0xFFFFFFFFull);
  ol[p] = l;
  oh[p] = h;
}

struct CollapseItem {
  uint32_t bin;     // binary internal node to expand
  uint32_t slot;    // BVH32 node slot it becomes
  uint32_t offset;  // scene position of its first Gaussian (depth-first leaf order)
  uint32_t pad;
};

__device__ __forceinline__ float box_area(float4 l, float4 h) {
  const float dx = fmaxf(h.x - l.x, 0.f), dy = fmaxf(h.y - l.y, 0.f), dz = fmaxf(h.z - l.z, 0.f);
  return 2.f * (dx * dy + dy * dz + dz * dx);
}

__device__ __forceinline__ uint32_t ref_count(uint32_t r, const float4* __restrict__ nhi) {
  return ref_is_leaf(r) ? 1u : __float_as_uint(nhi[r].w);
}

// ------------------------------------------------------------------------------------------
// SAH-optimal collapse (the dynamic programme of Ylitie, Karras & Laine, "Efficient Incoherent Ray
// Traversal on GPUs Through Compressed Wide BVHs", HPG 2017, with 32 slots per node).  For each
// binary node v and slot budget i, C(v, i) is the least expected traversal cost of representing
// v's subtree with at most i child slots of the enclosing BVH32 node:
//   C(v, 1) = min(leaf: A(v) (c_leaf + c_box n(v)) if n(v) <= leaf_max,  node: A(v) c_node + D(v, 32))
//   D(v, i) = min over 2 <= k <= i, 1 <= j < k of C(left, j) + C(right, k - j)
//   C(v, i) = min(C(v, 1), D(v, i))
// with A the surface area.  A Gaussian is a leaf of cost A (c_leaf + c_box).  The costs weigh an
// inner-node step against a leaf range (leaf packing shares warp steps between ranges) and a box
// test: c_node = 1, c_leaf = 0.5, c_box = 0.05 (measured on the showcase: c_leaf 0.3 or 1.0 and
// c_box 0.02 are within 0.3 %).
// ------------------------------------------------------------------------------------------
constexpr float kDpNode = 1.0f, kDpLeaf = 0.5f, kDpBox = 0.05f;

struct DpTables {
  float* cost;       // [ni * 32]: C(v, i) at v * 32 + i - 1
  uint8_t* split;    // [ni * 32]: j of the best split into exactly i slots
  uint8_t* best;     // [ni * 32]: the k <= i of D(v, i)
  uint32_t* single;  // [ni]: bit i - 1 set when C(v, i) uses one slot
  uint8_t* leaf;     // [ni]: the one slot of C(v, 1) is a leaf
};

// Parent links of a binary tree (internal children in parent[], Gaussians in parent_leaf[]).
__global__ void k_parents(uint32_t ni, const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                          uint32_t* __restrict__ parent, uint32_t* __restrict__ parent_leaf) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= ni) return;
  const uint32_t c[2] = {left[v], right[v]};
  for (int k = 0; k < 2; ++k) {
    if (ref_is_leaf(c[k])) parent_leaf[c[k] & ~kLeafBit] = v;
    else parent[c[k]] = v;
  }
}

__device__ __forceinline__ void dp_child(uint32_t ref, const float4* __restrict__ plo, const float4* __restrict__ phi,
                                         const float* cost, float (&C)[32]) {
  if (ref_is_leaf(ref)) {
    const uint32_t p = ref & ~kLeafBit;
    const float c = box_area(plo[p], phi[p]) * (kDpLeaf + kDpBox);
    for (int i = 0; i < 32; ++i) C[i] = c;
  } else {
    for (int i = 0; i < 32; ++i) C[i] = __ldcg(cost + (size_t)ref * 32u + i);
  }
}

// Bottom-up: one thread per Gaussian walks to the root; the second arrival at a node computes it.
__global__ void k_dp_cost(uint32_t n, uint32_t root, const uint32_t* __restrict__ left,
                          const uint32_t* __restrict__ right, const float4* __restrict__ plo,
                          const float4* __restrict__ phi, const float4* __restrict__ nlo,
                          const float4* __restrict__ nhi, const uint32_t* __restrict__ parent,
                          const uint32_t* __restrict__ parent_leaf, unsigned int* flags, DpTables T,
                          uint32_t leaf_max) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t v = parent_leaf[k];
  while (true) {
    __threadfence();
    if (atomicAdd(&flags[v], 1u) == 0u) return;
    __threadfence();
    float Cl[32], Cr[32], D[33];
    dp_child(left[v], plo, phi, T.cost, Cl);
    dp_child(right[v], plo, phi, T.cost, Cr);
    float dprev = INFINITY;
    uint32_t kprev = 2;
    for (int i = 2; i <= 32; ++i) {
      float b = INFINITY;
      int bj = 1;
      for (int j = 1; j < i; ++j) {
        const float c = Cl[j - 1] + Cr[i - j - 1];
        if (c < b) {
          b = c;
          bj = j;
        }
      }
      T.split[(size_t)v * 32u + i - 1] = (uint8_t)bj;
      if (i == 2 || b < dprev) {
        dprev = b;
        kprev = (uint32_t)i;
      }
      D[i] = dprev;
      T.best[(size_t)v * 32u + i - 1] = (uint8_t)kprev;
    }
    const float4 l = nlo[v], h = nhi[v];
    const float A = box_area(l, h);
    const uint32_t count = __float_as_uint(h.w);
    const float c_node = fmaf(A, kDpNode, D[32]);
    const float c_leaf = count <= leaf_max ? A * fmaf(kDpBox, (float)count, kDpLeaf) : INFINITY;
    const bool is_leaf = count <= leaf_max && c_leaf <= c_node;  // a leaf fits in one warp step
    const float c1 = fminf(c_leaf, c_node);
    uint32_t mask = 1u;
    __stcg(T.cost + (size_t)v * 32u, c1);
    for (int i = 2; i <= 32; ++i) {
      const bool one = c1 <= D[i];
      if (one) mask |= 1u << (i - 1);
      __stcg(T.cost + (size_t)v * 32u + i - 1, one ? c1 : D[i]);
    }
    T.single[v] = mask;
    T.leaf[v] = is_leaf ? 1 : 0;
    if (v == root) return;
    v = parent[v];
  }
}

// Collapse of a binary tree (Gaussian counts in nhi.w) into 32-wide nodes, level by level:
//  - greedy (kDp false): starting from the binary node's two children, repeatedly replace the
//    largest-area child holding more than kLeafMax Gaussians by its two children until 32 slots
//    are used; children with <= kLeafMax Gaussians become leaves, larger ones the next level's
//    nodes;
//  - SAH-optimal (kDp true): replay the choices of k_dp_cost for a budget of 32 slots.
// Every child carries the scene position of its first Gaussian in depth-first leaf order (left
// subtree first), so a leaf is one contiguous range of the scene order; pos[Morton position]
// receives each Gaussian's scene position.  The level's item count is read on the device
// (*n_items_dev), so levels run back to back with upper-bound grids.  Nodes beyond max_nodes are
// not written: the build then sees *overflow set and falls back to the greedy collapse.
template <bool kDp>
__global__ void k_collapse(const unsigned int* __restrict__ n_items_dev, const CollapseItem* __restrict__ in,
                           CollapseItem* __restrict__ out, unsigned int* __restrict__ out_count,
                           unsigned int* __restrict__ slot_counter, const uint32_t* __restrict__ left,
                           const uint32_t* __restrict__ right, const float4* __restrict__ plo,
                           const float4* __restrict__ phi, const float4* __restrict__ nlo,
                           const float4* __restrict__ nhi, float4* __restrict__ wide, uint32_t kLeafMax,
                           uint32_t* __restrict__ pos, unsigned int* __restrict__ leaf_counter, DpTables T,
                           uint32_t max_nodes, unsigned int* __restrict__ overflow) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *n_items_dev) return;
  const CollapseItem it = in[t];
  uint32_t refs[32], offs[32];
  uint32_t leafmask = 0;  // kDp: internal refs that are leaves
  int cnt = 0;
  if constexpr (kDp) {
    // expansion stack of (ref, slot budget, offset); the budgets on it sum to <= 32
    uint32_t sv[32], so[32];
    uint8_t si[32];
    int sp = 0;
    {
      const uint32_t v = it.bin;
      const uint32_t kk = T.best[(size_t)v * 32u + 31u], j = T.split[(size_t)v * 32u + kk - 1u];
      sv[sp] = right[v], si[sp] = (uint8_t)(kk - j), so[sp] = it.offset + ref_count(left[v], nhi), ++sp;
      sv[sp] = left[v], si[sp] = (uint8_t)j, so[sp] = it.offset, ++sp;
    }
    while (sp > 0 && cnt < 32) {
      --sp;
      const uint32_t v = sv[sp], i = si[sp], off = so[sp];
      if (ref_is_leaf(v) || i == 1u || ((T.single[v] >> (i - 1u)) & 1u)) {
        if (!ref_is_leaf(v) && T.leaf[v]) leafmask |= 1u << cnt;
        refs[cnt] = v;
        offs[cnt] = off;
        ++cnt;
        continue;
      }
      const uint32_t kk = T.best[(size_t)v * 32u + i - 1u], j = T.split[(size_t)v * 32u + kk - 1u];
      sv[sp] = right[v], si[sp] = (uint8_t)(kk - j), so[sp] = off + ref_count(left[v], nhi), ++sp;
      sv[sp] = left[v], si[sp] = (uint8_t)j, so[sp] = off, ++sp;
    }
  } else {
    cnt = 2;
    refs[0] = left[it.bin];
    refs[1] = right[it.bin];
    offs[0] = it.offset;
    offs[1] = it.offset + ref_count(refs[0], nhi);
    while (cnt < 32) {
      int best = -1;
      float best_a = -1.f;
      for (int c = 0; c < cnt; ++c) {
        const uint32_t r = refs[c];
        if (ref_is_leaf(r)) continue;
        if (ref_count(r, nhi) <= kLeafMax) continue;
        const float a = box_area(nlo[r], nhi[r]);
        if (a > best_a) {
          best_a = a;
          best = c;
        }
      }
      if (best < 0) break;
      const uint32_t r = refs[best];
      refs[best] = left[r];
      refs[cnt] = right[r];
      offs[cnt] = offs[best] + ref_count(left[r], nhi);
      ++cnt;
    }
    for (int c = 0; c < cnt; ++c)
      if (!ref_is_leaf(refs[c]) && ref_count(refs[c], nhi) <= kLeafMax) leafmask |= 1u << c;
  }
  float4* node = wide + (size_t)it.slot * 64u;
  for (int c = 0; c < 32; ++c) {
    float4 l, h;
    uint32_t wref;
    if (c >= cnt) {
      l = make_float4(INFINITY, INFINITY, INFINITY, __uint_as_float(kEmptyRef));
      h = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
      node[c] = l;
      node[32 + c] = h;
      continue;
    }
    const uint32_t r = refs[c];
    if (ref_is_leaf(r)) {
      const uint32_t p = r & ~kLeafBit;
      l = plo[p];
      h = phi[p];
      pos[p] = offs[c];
      wref = wide_leaf_ref(offs[c], 1u);
      atomicAdd(leaf_counter, 1u);
    } else {
      l = nlo[r];
      h = nhi[r];
      const uint32_t count = ref_count(r, nhi);
      if ((leafmask >> c) & 1u) {
        wref = wide_leaf_ref(offs[c], count);
        atomicAdd(leaf_counter, 1u);
        // depth-first walk of the leaf's subtree (<= 32 Gaussians, so <= 32 stacked refs)
        uint32_t st[32];
        int sp = 0;
        uint32_t k = offs[c];
        st[sp++] = r;
        while (sp > 0) {
          const uint32_t v = st[--sp];
          if (ref_is_leaf(v)) {
            pos[v & ~kLeafBit] = k++;
          } else {
            st[sp++] = right[v];
            st[sp++] = left[v];
          }
        }
      } else {
        const uint32_t slot = atomicAdd(slot_counter, 1u);
        if (slot >= max_nodes) {  // over the node budget: no write; the build falls back
          atomicOr(overflow, 1u);
          wref = kEmptyRef;
        } else {
          const uint32_t q = atomicAdd(out_count, 1u);
          out[q] = CollapseItem{r, slot, offs[c], 0u};
          wref = slot;
        }
      }
    }
    l.w = __uint_as_float(wref);
    h.w = 0.f;
    node[c] = l;
    node[32 + c] = h;
  }
}

// Scene order from the collapse's positions: order[pos[m]] = Morton order's caller index.
__global__ void k_compose(uint32_t n, const uint32_t* __restrict__ morton_order, const uint32_t* __restrict__ pos,
                          uint32_t* __restrict__ order) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  order[pos[i]] = morton_order[i];
}

__global__ void k_iota(uint32_t n, uint32_t* __restrict__ v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

// Root of a scene with <= 32 Gaussians: one node holding one leaf.
__global__ void k_single_leaf_root(uint32_t n, const float4* __restrict__ plo,
                                   const float4* __restrict__ phi, float4* __restrict__ wide) {
  const int c = threadIdx.x;
  if (c >= 32) return;
  if (c == 0) {
    float4 l = make_float4(INFINITY, INFINITY, INFINITY, 0.f), h = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
    for (uint32_t i = 0; i < n; ++i) {
      const float4 a = plo[i], b = phi[i];
      l.x = fminf(l.x, a.x); l.y = fminf(l.y, a.y); l.z = fminf(l.z, a.z);
      h.x = fmaxf(h.x, b.x); h.y = fmaxf(h.y, b.y); h.z = fmaxf(h.z, b.z);
    }
    l.w = __uint_as_float(wide_leaf_ref(0u, n));
    wide[0] = l;
    wide[32] = h;
  } else {
    wide[c] = make_float4(INFINITY, INFINITY, INFINITY, __uint_as_float(kEmptyRef));
    wide[32 + c] = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
  }
}

// One-Gaussian binary "tree": a root whose left child is the Gaussian and right is empty.
__global__ void k_single_binary_root(const float4* __restrict__ plo, const float4* __restrict__ phi,
                                     float4* __restrict__ out) {
  float4 l = plo[0];
  l.w = __uint_as_float(kLeafBit | 0u);
  out[0] = l;
  out[1] = phi[0];
  out[2] = make_float4(INFINITY, INFINITY, INFINITY, __uint_as_float(kEmptyRef));
  out[3] = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
}

template <class T>
struct Scratch {  // stream-ordered temporary, freed on scope exit
  T* p = nullptr;
  cudaStream_t s;
  explicit Scratch(cudaStream_t st) : s(st) {}
  ~Scratch() { dev_free(p, s); }
};

}  // namespace

// A scene without Gaussians (the reference builds an instance AS over zero instances and every
// ray misses; test/scenes/geometric_validation.cpp empty_scene): one BVH32 root and one binary
// root whose children are all empty, and one zeroed element in each per-Gaussian array so that
// no pointer is null.  Every traversal tests the root's children, finds none, and ends.
vp_status build_empty_scene(vp_context* ctx, const vp_gaussians* g, float sigma_multiplier,
                            const vp_scene_options& opt, vp_scene* sc) {
  cudaStream_t st = ctx->stream;
  float ref_empty;
  std::memcpy(&ref_empty, &kEmptyRef, sizeof(ref_empty));
  const float4 lo_empty = make_float4(INFINITY, INFINITY, INFINITY, ref_empty);
  const float4 hi_empty = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
  float4 wide_h[64], bin_h[4];
  for (int c = 0; c < 32; ++c) wide_h[c] = lo_empty, wide_h[32 + c] = hi_empty;
  bin_h[0] = bin_h[2] = lo_empty;
  bin_h[1] = bin_h[3] = hi_empty;
  vp_status s;
  if ((s = dev_alloc(&sc->prims, 4, st)) || (s = dev_alloc(&sc->perm, 1, st)) || (s = dev_alloc(&sc->pbox, 2, st)) ||
      (s = dev_alloc(&sc->raw, 2, st)) || (s = dev_alloc(&sc->wide, 64, st)) || (s = dev_alloc(&sc->bin, 4, st)))
    return s;
  VP_CUDA(cudaMemsetAsync(sc->prims, 0, 4 * sizeof(float4), st));
  VP_CUDA(cudaMemsetAsync(sc->perm, 0, sizeof(uint32_t), st));
  VP_CUDA(cudaMemsetAsync(sc->pbox, 0, 2 * sizeof(float4), st));
  VP_CUDA(cudaMemsetAsync(sc->raw, 0, 2 * sizeof(float4), st));
  VP_CUDA(cudaMemcpyAsync(sc->wide, wide_h, sizeof(wide_h), cudaMemcpyHostToDevice, st));
  VP_CUDA(cudaMemcpyAsync(sc->bin, bin_h, sizeof(bin_h), cudaMemcpyHostToDevice, st));
  VP_CUDA(cudaStreamSynchronize(st));
  sc->ctx = ctx;
  sc->scale_is_log = g->scale_is_log ? 1 : 0;
  sc->sigma_multiplier = sigma_multiplier;
  SceneView& v = sc->view;
  v.prims = sc->prims;
  v.perm = sc->perm;
  v.wide = sc->wide;
  v.bin = sc->bin;
  v.pbox = sc->pbox;
  v.count = 0u;
  v.wide_root = 0u;
  v.bin_root = 0u;
  v.stack_cap = 31u + 2u;
  v.argmin_cap = v.stack_cap + kArgminBestFirstStack + 64u;
  v.albedo_all_zero = 1;
  v.tau_nearest = 0;
  vp_scene_info& info = sc->info;
  info = vp_scene_info{};
  info.tau_order = VP_TAU_ORDER_LANE;
  info.wide_nodes = 1;
  info.wide_depth = 1;
  info.binary_nodes = 1;
  info.wide_builder = opt.wide_builder;
  info.binary_builder = opt.binary_builder;
  info.leaf_max = opt.leaf_max;
  info.wide_collapse = opt.wide_collapse;
  info.albedo_all_zero = 1;
  info.device_bytes = 64ull + 4ull + 32ull + 32ull + 1024ull + 64ull;
  return VP_OK;
}

vp_status build_scene(vp_context* ctx, const vp_gaussians* g, float sigma_multiplier, const vp_scene_options& opt,
                      vp_scene* sc) {
  cudaStream_t st = ctx->stream;
  const uint32_t n = g->count;
  if (n >= (1u << 26)) return fail(VP_ERROR_LIMIT, "scene exceeds 2^26 Gaussians");
  if (!(sigma_multiplier > 0.f) || !std::isfinite(sigma_multiplier))
    return fail(VP_ERROR_INVALID_ARGUMENT, "sigma_multiplier must be positive and finite");
  if (n == 0) return build_empty_scene(ctx, g, sigma_multiplier, opt, sc);
  if (!g->mean || !g->scale || !g->quat_wxyz || !g->density)
    return fail(VP_ERROR_INVALID_ARGUMENT, "vp_gaussians: mean, scale, quat_wxyz and density are required");

  VP_CUDA(cudaEventRecord(ctx->ev0, st));
  // Inputs on the device.
  Scratch<float> d_mean(st), d_scale(st), d_quat(st), d_dens(st), d_alb(st);
  const float *mean = g->mean, *scale = g->scale, *quat = g->quat_wxyz, *dens = g->density,
              *alb = g->albedo;
  if (g->memory == VP_MEMORY_HOST) {
    vp_status s;
    if ((s = dev_alloc(&d_mean.p, 3ull * n, st))) return s;
    if ((s = dev_alloc(&d_scale.p, 3ull * n, st))) return s;
    if ((s = dev_alloc(&d_quat.p, 4ull * n, st))) return s;
    if ((s = dev_alloc(&d_dens.p, 1ull * n, st))) return s;
    VP_CUDA(cudaMemcpyAsync(d_mean.p, mean, 12ull * n, cudaMemcpyHostToDevice, st));
    VP_CUDA(cudaMemcpyAsync(d_scale.p, scale, 12ull * n, cudaMemcpyHostToDevice, st));
    VP_CUDA(cudaMemcpyAsync(d_quat.p, quat, 16ull * n, cudaMemcpyHostToDevice, st));
    VP_CUDA(cudaMemcpyAsync(d_dens.p, dens, 4ull * n, cudaMemcpyHostToDevice, st));
    mean = d_mean.p;
    scale = d_scale.p;
    quat = d_quat.p;
    dens = d_dens.p;
    if (alb) {
      if ((s = dev_alloc(&d_alb.p, 3ull * n, st))) return s;
      VP_CUDA(cudaMemcpyAsync(d_alb.p, alb, 12ull * n, cudaMemcpyHostToDevice, st));
      alb = d_alb.p;
    }
  } else if (g->memory != VP_MEMORY_DEVICE) {
    return fail(VP_ERROR_INVALID_ARGUMENT, "vp_gaussians.memory must be VP_MEMORY_HOST or VP_MEMORY_DEVICE");
  }

  vp_status s;
  Scratch<float4> rec0(st), lo0(st), hi0(st), plo(st), phi(st);
  Scratch<ErrorWords> errw(st);
  Scratch<unsigned int> bounds(st);
  if ((s = dev_alloc(&rec0.p, 4ull * n, st))) return s;
  if ((s = dev_alloc(&lo0.p, n, st))) return s;
  if ((s = dev_alloc(&hi0.p, n, st))) return s;
  if ((s = dev_alloc(&errw.p, 1, st))) return s;
  if ((s = dev_alloc(&bounds.p, 12, st))) return s;
  {
    ErrorWords e0{0x7FFFFFFF, 0x7FFFFFFF, 0x7FFFFFFF, 0u, 0u};
    VP_CUDA(cudaMemcpyAsync(errw.p, &e0, sizeof(e0), cudaMemcpyHostToDevice, st));
    unsigned int b0[12];
    for (int k = 0; k < 3; ++k) {
      b0[k] = 0xFFFFFFFFu;
      b0[3 + k] = 0u;
      b0[6 + k] = 0xFFFFFFFFu;
      b0[9 + k] = 0u;
    }
    VP_CUDA(cudaMemcpyAsync(bounds.p, b0, sizeof(b0), cudaMemcpyHostToDevice, st));
  }
  const int TB = 256;
  const unsigned nb = (n + TB - 1) / TB;
  k_precompute<<<nb, TB, 0, st>>>(n, mean, scale, quat, dens, alb, g->scale_is_log, sigma_multiplier,
                                  rec0.p, lo0.p, hi0.p, errw.p);
  VP_CUDA(cudaGetLastError());
  k_bounds<<<std::min(nb, 1184u), TB, 0, st>>>(n, mean, lo0.p, hi0.p, bounds.p);
  VP_CUDA(cudaGetLastError());
  ErrorWords eh{};
  unsigned int bh[12];
  VP_CUDA(cudaMemcpyAsync(&eh, errw.p, sizeof(eh), cudaMemcpyDeviceToHost, st));
  VP_CUDA(cudaMemcpyAsync(bh, bounds.p, sizeof(bh), cudaMemcpyDeviceToHost, st));
  VP_CUDA(cudaStreamSynchronize(st));
  if (eh.bad_scale != 0x7FFFFFFF)
    return fail(VP_ERROR_INVALID_ARGUMENT, "Gaussian " + std::to_string(eh.bad_scale) +
                                               ": invalid scale - all components must be finite and > 0");
  if (eh.bad_density != 0x7FFFFFFF)
    return fail(VP_ERROR_INVALID_ARGUMENT, "Gaussian " + std::to_string(eh.bad_density) +
                                               ": invalid density - must be finite and > 0");
  if (eh.bad_center != 0x7FFFFFFF)
    return fail(VP_ERROR_INVALID_ARGUMENT, "Gaussian " + std::to_string(eh.bad_center) +
                                               ": NaN/Inf in centre or rotation");

  // Morton codes + radix sort (stable: ties keep the caller's order).
  Scratch<uint64_t> codes(st);
  Scratch<uint32_t> idx(st), pos(st);
  Scratch<unsigned char> sort_tmp(st);
  if ((s = dev_alloc(&codes.p, n, st))) return s;
  if ((s = dev_alloc(&idx.p, n, st))) return s;
  if ((s = dev_alloc(&pos.p, n, st))) return s;
  k_morton<<<nb, TB, 0, st>>>(n, mean, bounds.p, codes.p, idx.p);
  VP_CUDA(cudaGetLastError());
  // Stable radix sort of the 63-bit codes (ties keep the caller's order), in place: codes become
  // the sorted codes and idx the Morton order.  The same scratch serves the clustering's scans.
  const size_t scan_bytes = exclusive_scan_tmp_bytes(n);
  const size_t tmp_bytes = std::max(radix_sort_tmp_bytes_u64(n), scan_bytes);
  if ((s = dev_alloc(&sort_tmp.p, tmp_bytes, st))) return s;
  if ((s = radix_sort_pairs(codes.p, idx.p, n, 63, sort_tmp.p, tmp_bytes, st))) return s;
  const uint64_t* codes_sorted = codes.p;
  const uint32_t* morton = idx.p;
  if ((s = dev_alloc(&plo.p, n, st))) return s;
  if ((s = dev_alloc(&phi.p, n, st))) return s;
  k_gather_boxes<<<nb, TB, 0, st>>>(n, morton, lo0.p, hi0.p, plo.p, phi.p);
  VP_CUDA(cudaGetLastError());

  // PLOC clustering: the binary tree of the BVH32 and of the megakernel unless the options ask for
  // the Karras tree for both (a BVH32 that is a single leaf needs no tree).
  const uint32_t ni = n > 1 ? n - 1 : 1;
  const uint32_t kLeafMax = opt.leaf_max;
  bool wide_ploc = n > kLeafMax && opt.wide_builder == VP_TREE_PLOC;
  bool use_ploc = n > 1u && (wide_ploc || opt.binary_builder == VP_TREE_PLOC);
  Scratch<uint32_t> pleft(st), pright(st), nn(st), totals(st);
  Scratch<float4> pnlo(st), pnhi(st), ca(st), cb(st), oa(st), ob(st);
  Scratch<unsigned long long> fl(st), sc_x(st);
  uint32_t wroot = 0u, ploc_height = 0u;
  if (use_ploc) {
    if ((s = dev_alloc(&pleft.p, ni, st))) return s;
    if ((s = dev_alloc(&pright.p, ni, st))) return s;
    if ((s = dev_alloc(&pnlo.p, ni, st))) return s;
    if ((s = dev_alloc(&pnhi.p, ni, st))) return s;
    if ((s = dev_alloc(&nn.p, n, st))) return s;
    if ((s = dev_alloc(&totals.p, 4, st))) return s;
    if ((s = dev_alloc(&ca.p, n, st))) return s;
    if ((s = dev_alloc(&cb.p, n, st))) return s;
    if ((s = dev_alloc(&oa.p, n, st))) return s;
    if ((s = dev_alloc(&ob.p, n, st))) return s;
    if ((s = dev_alloc(&fl.p, n, st))) return s;
    if ((s = dev_alloc(&sc_x.p, n, st))) return s;
    k_ploc_init<<<nb, TB, 0, st>>>(n, plo.p, phi.p, ca.p, cb.p);
    VP_CUDA(cudaGetLastError());
    {
      const uint32_t c0[4] = {n, 0u, n, 0u};
      VP_CUDA(cudaMemcpyAsync(totals.p, c0, sizeof(c0), cudaMemcpyHostToDevice, st));
    }
    // Passes run in chunks between host reads of the count; the count only falls, so the last
    // value read bounds the grids of the next chunk.
    // A chain of nested boxes (concentric Gaussians of growing size) merges about one pair per
    // pass; past kMaxPasses the build drops the clustering and uses the Karras tree instead.
    constexpr int kChunk = 16;
    constexpr int kMaxPasses = 1024;
    uint32_t m = n, made = 0u;
    int pass = 0;
    while (m > 1u && pass < kMaxPasses) {
      for (int k = 0; k < kChunk; ++k, ++pass) {
        const uint32_t* cin = totals.p + 2 * (pass & 1);
        uint32_t* cout = totals.p + 2 * ((pass + 1) & 1);
        k_ploc_nn<<<(m + kPlocBlock - 1) / kPlocBlock, kPlocBlock, 0, st>>>(cin, ca.p, cb.p, nn.p);
        VP_CUDA(cudaGetLastError());
        k_ploc_flags<<<(m + TB - 1) / TB, TB, 0, st>>>(m, cin, nn.p, fl.p);
        VP_CUDA(cudaGetLastError());
        if ((s = exclusive_scan(fl.p, sc_x.p, m, sort_tmp.p, scan_bytes, st))) return s;
        k_ploc_write<<<(m + TB - 1) / TB, TB, 0, st>>>(cin, cout, nn.p, fl.p, sc_x.p, ca.p, cb.p, oa.p, ob.p,
                                                       pleft.p, pright.p, pnlo.p, pnhi.p);
        VP_CUDA(cudaGetLastError());
        std::swap(ca.p, oa.p);
        std::swap(cb.p, ob.p);
      }
      uint32_t th[2];
      VP_CUDA(cudaMemcpyAsync(th, totals.p + 2 * (pass & 1), sizeof(th), cudaMemcpyDeviceToHost, st));
      VP_CUDA(cudaStreamSynchronize(st));
      if (th[0] >= m && m > 1u) return fail(VP_ERROR_INTERNAL, "PLOC clustering made no progress");
      if (th[0] + th[1] != n || th[1] > ni) return fail(VP_ERROR_INTERNAL, "PLOC clustering lost a cluster");
      m = th[0];
      made = th[1];
    }
    if (m > 1u) {
      use_ploc = false;
      wide_ploc = false;
    } else {
      wroot = made - 1u;  // the last merge made the root (node n - 2)
      float4 root_lo;
      VP_CUDA(cudaMemcpyAsync(&root_lo, pnlo.p + wroot, sizeof(root_lo), cudaMemcpyDeviceToHost, st));
      VP_CUDA(cudaStreamSynchronize(st));
      std::memcpy(&ploc_height, &root_lo.w, sizeof(ploc_height));
    }
  }
  // Karras radix tree + refit over the Morton order: the BVH32's source when the options ask for it,
  // and the megakernel's binary tree when they ask for it or the PLOC tree is deeper than the
  // megakernel's thread-private stack.
  Scratch<uint32_t> left(st), right(st), first(st), last(st), par_i(st), par_l(st);
  Scratch<float4> nlo(st), nhi(st);
  Scratch<unsigned int> flags(st);
  const bool bin_from_ploc = use_ploc && opt.binary_builder == VP_TREE_PLOC && ploc_height + 1u < (uint32_t)kBinStack;
  const bool need_karras = !wide_ploc || !bin_from_ploc;
  if (need_karras) {
    if ((s = dev_alloc(&left.p, ni, st))) return s;
    if ((s = dev_alloc(&right.p, ni, st))) return s;
    if ((s = dev_alloc(&first.p, ni, st))) return s;
    if ((s = dev_alloc(&last.p, ni, st))) return s;
    if ((s = dev_alloc(&par_i.p, ni, st))) return s;
    if ((s = dev_alloc(&par_l.p, n, st))) return s;
    if ((s = dev_alloc(&nlo.p, ni, st))) return s;
    if ((s = dev_alloc(&nhi.p, ni, st))) return s;
    if ((s = dev_alloc(&flags.p, ni, st))) return s;
    if (n > 1) {
      VP_CUDA(cudaMemsetAsync(flags.p, 0, sizeof(unsigned int) * ni, st));
      k_karras<<<(ni + TB - 1) / TB, TB, 0, st>>>((int)n, codes_sorted, left.p, right.p, first.p, last.p,
                                                  par_i.p, par_l.p);
      VP_CUDA(cudaGetLastError());
      k_refit<<<nb, TB, 0, st>>>((int)n, left.p, right.p, par_i.p, par_l.p, plo.p, phi.p, nlo.p, nhi.p, flags.p);
      VP_CUDA(cudaGetLastError());
    }
  }

  const uint32_t wide_root = wide_ploc ? wroot : 0u;
  const uint32_t* wl = wide_ploc ? pleft.p : left.p;
  const uint32_t* wr = wide_ploc ? pright.p : right.p;
  const float4* wlo = wide_ploc ? pnlo.p : nlo.p;
  const float4* whi = wide_ploc ? pnhi.p : nhi.p;

  // Collapse to BVH32; its depth-first leaf order defines the scene order (pos).
  // Upper bound on BVH32 nodes: childless nodes hold > L disjoint Gaussians (<= n/(L+1)), nodes
  // with one node child hold 31 leaves of their own (<= n/31), branching nodes are fewer than
  // childless ones (<= n/(L+1)).
  const uint32_t max_wide = n / 31u + 2u * (n / (kLeafMax + 1u)) + 4u;
  float4* wide = nullptr;
  if ((s = dev_alloc(&wide, 64ull * max_wide, st))) return s;
  sc->wide = wide;
  uint32_t depth = 1, wide_nodes = 1, leaves = 1;
  bool dp_used = false;
  if (n <= kLeafMax) {
    k_single_leaf_root<<<1, 32, 0, st>>>(n, plo.p, phi.p, wide);
    VP_CUDA(cudaGetLastError());
    k_iota<<<nb, TB, 0, st>>>(n, pos.p);
    VP_CUDA(cudaGetLastError());
  } else {
    // SAH-optimal slot tables (k_dp_cost) when asked for and the scene is at most 2^24 Gaussians.
    const uint32_t nint = n - 1u;
    Scratch<float> dp_cost(st);
    Scratch<uint8_t> dp_split(st), dp_best(st), dp_leaf(st);
    Scratch<uint32_t> dp_single(st), par(st), par_leaf(st);
    Scratch<unsigned int> dp_flags(st);
    DpTables T{nullptr, nullptr, nullptr, nullptr, nullptr};
    bool dp = opt.wide_collapse == VP_COLLAPSE_SAH && n <= (1u << 24);
    if (dp) {
      if ((s = dev_alloc(&dp_cost.p, 32ull * nint, st))) return s;
      if ((s = dev_alloc(&dp_split.p, 32ull * nint, st))) return s;
      if ((s = dev_alloc(&dp_best.p, 32ull * nint, st))) return s;
      if ((s = dev_alloc(&dp_leaf.p, nint, st))) return s;
      if ((s = dev_alloc(&dp_single.p, nint, st))) return s;
      if ((s = dev_alloc(&par.p, nint, st))) return s;
      if ((s = dev_alloc(&par_leaf.p, n, st))) return s;
      if ((s = dev_alloc(&dp_flags.p, nint, st))) return s;
      VP_CUDA(cudaMemsetAsync(dp_flags.p, 0, sizeof(unsigned int) * nint, st));
      k_parents<<<(nint + TB - 1) / TB, TB, 0, st>>>(nint, wl, wr, par.p, par_leaf.p);
      VP_CUDA(cudaGetLastError());
      T = DpTables{dp_cost.p, dp_split.p, dp_best.p, dp_single.p, dp_leaf.p};
      k_dp_cost<<<nb, TB, 0, st>>>(n, wide_root, wl, wr, plo.p, phi.p, wlo, whi, par.p, par_leaf.p, dp_flags.p, T,
                                   kLeafMax);
      VP_CUDA(cudaGetLastError());
    }
    Scratch<CollapseItem> qa(st), qb(st);
    Scratch<unsigned int> ctr(st), lvl(st);
    constexpr int kMaxLevels = 512;  // BVH32 depth bound (a PLOC chain of 1,024 passes stays far below)
    constexpr int kLevelChunk = 4;   // levels between host reads
    if ((s = dev_alloc(&qa.p, max_wide, st))) return s;
    if ((s = dev_alloc(&qb.p, max_wide, st))) return s;
    if ((s = dev_alloc(&ctr.p, 3, st))) return s;
    if ((s = dev_alloc(&lvl.p, kMaxLevels + 1, st))) return s;
    // A level-by-level collapse: lvl[k] = items (BVH32 nodes to fill) at level k, counted on the
    // device; the host reads the counts every kLevelChunk levels.  An SAH cut that needs more
    // nodes than the greedy bound is redone greedily.
    for (int attempt = 0; attempt < 2; ++attempt) {
      CollapseItem root{wide_root, 0u, 0u, 0u};
      VP_CUDA(cudaMemcpyAsync(qa.p, &root, sizeof(root), cudaMemcpyHostToDevice, st));
      const unsigned int c0[3] = {1u, 0u, 0u};  // next free slot, leaves, overflow
      VP_CUDA(cudaMemcpyAsync(ctr.p, c0, sizeof(c0), cudaMemcpyHostToDevice, st));
      VP_CUDA(cudaMemsetAsync(lvl.p, 0, sizeof(unsigned int) * (kMaxLevels + 1), st));
      const unsigned int one = 1u;
      VP_CUDA(cudaMemcpyAsync(lvl.p, &one, sizeof(one), cudaMemcpyHostToDevice, st));
      uint64_t bound = 1;  // upper bound of the items at the next level to launch
      int k = 0;
      bool done = false, over = false;
      while (!done) {
        for (int c = 0; c < kLevelChunk; ++c, ++k) {
          if (k >= kMaxLevels) return fail(VP_ERROR_INTERNAL, "BVH32 deeper than 512 levels");
          const unsigned grid = (unsigned)((bound + 127) / 128);
          CollapseItem* qin = (k & 1) ? qb.p : qa.p;
          CollapseItem* qout = (k & 1) ? qa.p : qb.p;
          if (dp)
            k_collapse<true><<<grid, 128, 0, st>>>(lvl.p + k, qin, qout, lvl.p + k + 1, ctr.p, wl, wr, plo.p, phi.p,
                                                   wlo, whi, wide, kLeafMax, pos.p, ctr.p + 1, T, max_wide, ctr.p + 2);
          else
            k_collapse<false><<<grid, 128, 0, st>>>(lvl.p + k, qin, qout, lvl.p + k + 1, ctr.p, wl, wr, plo.p, phi.p,
                                                    wlo, whi, wide, kLeafMax, pos.p, ctr.p + 1, T, max_wide, ctr.p + 2);
          VP_CUDA(cudaGetLastError());
          bound = std::min<uint64_t>(bound * 32u, max_wide);  // each item makes at most 32 children
        }
        unsigned int ch[3], next = 0u;
        VP_CUDA(cudaMemcpyAsync(ch, ctr.p, sizeof(ch), cudaMemcpyDeviceToHost, st));
        VP_CUDA(cudaMemcpyAsync(&next, lvl.p + k, sizeof(next), cudaMemcpyDeviceToHost, st));
        VP_CUDA(cudaStreamSynchronize(st));
        wide_nodes = ch[0];
        leaves = ch[1];
        over = ch[2] != 0u;
        bound = next;
        done = over || next == 0u;
      }
      if (!over) {
        std::vector<unsigned int> counts(k + 1);
        VP_CUDA(cudaMemcpyAsync(counts.data(), lvl.p, sizeof(unsigned int) * (k + 1), cudaMemcpyDeviceToHost, st));
        VP_CUDA(cudaStreamSynchronize(st));
        depth = 0;
        while (depth < (uint32_t)k && counts[depth] != 0u) ++depth;
        dp_used = dp;
        break;
      }
      if (!dp) return fail(VP_ERROR_INTERNAL, "BVH32 node budget exceeded");
      dp = false;
    }
  }
  // Scene order, then the records, boxes and adjoint inputs gathered into it.
  uint32_t* perm = nullptr;
  if ((s = dev_alloc(&perm, n, st))) return s;
  sc->perm = perm;
  k_compose<<<nb, TB, 0, st>>>(n, morton, pos.p, perm);
  VP_CUDA(cudaGetLastError());
  float4* prims = nullptr;
  if ((s = dev_alloc(&prims, 4ull * n, st))) return s;
  sc->prims = prims;
  float4* pbox = nullptr;
  if ((s = dev_alloc(&pbox, 2ull * n, st))) return s;
  sc->pbox = pbox;
  k_gather<<<nb, TB, 0, st>>>(n, perm, rec0.p, lo0.p, hi0.p, prims, pbox);
  VP_CUDA(cudaGetLastError());
  float4* raw = nullptr;
  if ((s = dev_alloc(&raw, 2ull * n, st))) return s;
  sc->raw = raw;
  sc->scale_is_log = g->scale_is_log ? 1 : 0;
  sc->sigma_multiplier = sigma_multiplier;
  k_gather_raw<<<nb, TB, 0, st>>>(n, perm, scale, quat, dens, raw);
  VP_CUDA(cudaGetLastError());
  float4* bin = nullptr;
  if ((s = dev_alloc(&bin, 4ull * ni, st))) return s;
  sc->bin = bin;
  uint32_t bin_root = 0u;
  if (bin_from_ploc) {
    k_binary_nodes<<<(ni + TB - 1) / TB, TB, 0, st>>>((int)n, pleft.p, pright.p, plo.p, phi.p, pnlo.p, pnhi.p, pos.p,
                                                      bin);
    bin_root = wroot;
  } else if (n > 1) {
    k_binary_nodes<<<(ni + TB - 1) / TB, TB, 0, st>>>((int)n, left.p, right.p, plo.p, phi.p, nlo.p, nhi.p, pos.p,
                                                      bin);
  } else {
    k_single_binary_root<<<1, 1, 0, st>>>(plo.p, phi.p, bin);
  }
  VP_CUDA(cudaGetLastError());
  if (wide_nodes < max_wide) {  // keep only the nodes in use
    float4* tight = nullptr;
    if ((s = dev_alloc(&tight, 64ull * wide_nodes, st))) return s;
    VP_CUDA(cudaMemcpyAsync(tight, wide, 1024ull * wide_nodes, cudaMemcpyDeviceToDevice, st));
    dev_free(wide, st);
    wide = tight;
    sc->wide = wide;
  }
  VP_CUDA(cudaEventRecord(ctx->ev1, st));
  VP_CUDA(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  VP_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));

  sc->ctx = ctx;
  SceneView& v = sc->view;
  v.prims = prims;
  v.perm = perm;
  v.wide = wide;
  v.bin = bin;
  v.pbox = pbox;
  v.count = n;
  v.wide_root = 0u;
  v.bin_root = bin_root;
  v.stack_cap = 31u * depth + 2u;
  v.argmin_cap = v.stack_cap + kArgminBestFirstStack + 64u;
  v.albedo_all_zero = eh.any_albedo ? 0 : 1;
  // AUTO: nearest first where rays need many translucent Gaussians to become opaque and the tree
  // has levels below the root's children to order (on a two-level tree the ranking pass costs
  // more than it saves)
  const int32_t tau_order = opt.tau_order != VP_TAU_ORDER_AUTO ? opt.tau_order
                            : (2ull * eh.opaque_cores < n && depth >= 3u) ? VP_TAU_ORDER_NEAREST
                                                                         : VP_TAU_ORDER_LANE;
  v.tau_nearest = tau_order == VP_TAU_ORDER_NEAREST ? 1 : 0;
  vp_scene_info& info = sc->info;
  info.count = n;
  info.wide_nodes = wide_nodes;
  info.wide_depth = depth;
  info.binary_nodes = n > 1 ? n - 1 : 1;
  info.leaves = leaves;
  info.wide_builder = n <= kLeafMax ? opt.wide_builder : (wide_ploc ? VP_TREE_PLOC : VP_TREE_LBVH);
  info.binary_builder = bin_from_ploc ? VP_TREE_PLOC : VP_TREE_LBVH;
  info.binary_height = ploc_height;
  info.leaf_max = kLeafMax;
  info.wide_collapse = dp_used ? VP_COLLAPSE_SAH : VP_COLLAPSE_GREEDY;
  info.albedo_all_zero = v.albedo_all_zero;
  info.tau_order = tau_order;
  info.build_ms = ms;
  for (int k = 0; k < 3; ++k) {
    auto o2f = [](unsigned int u) {
      unsigned int b = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
      float f;
      std::memcpy(&f, &b, 4);
      return f;
    };
    info.bounds_min[k] = o2f(bh[6 + k]);
    info.bounds_max[k] = o2f(bh[9 + k]);
  }
  // records, order, per-Gaussian boxes, adjoint inputs, BVH32, binary LBVH
  info.device_bytes = 64ull * n + 4ull * n + 32ull * n + 32ull * n + 1024ull * wide_nodes + 64ull * ni;
  return VP_OK;
}

}  // namespace vp
