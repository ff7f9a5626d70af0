// Wavefront engine: the path loop as a sequence of small persistent kernels over queues of
// paths, with the path state in device memory between stages.
//
//   generate  (thread per path)  camera ray, PCG32 stream, first free-flight key
//   per bounce, while any path is alive:
//     extend  (warp per path)    free-flight argmin over the BVH32 + albedo at the scatter point
//     shade   (thread per path)  phase sample, NEE sampling, escape rule, roulette; compacts
//                                surviving paths into the next queue and the bounce's
//                                transmittance queries into the shadow queue
//     shadow  (warp per query)   transmittance over the BVH32 with early exit at tau >= 88
//     gather  (thread per path)  radiance += weight x T in query order; finished paths write
//                                their sample
//   welford   (thread per pixel) running mean over the batch's samples in sample order
//
// Each kernel is a fraction of the fused path loop's code and registers, so more warps are
// resident per SM to hide the latency of the dependent node loads.  The reference found a
// wavefront 100x slower than its megakernel because ~352 B of per-ray sets and hit buffers
// streamed through DRAM each bounce (latex/chapters/06-optimization.tex:438-446); here no hit
// buffer or active set survives a stage (the queries rebuild them from geometry), so a path
// carries ~290 B in total and the traffic is negligible next to the traversal.  Results are
// those of the warp engine: the same shading code (vp_path.cuh), the same queries, and the
// same order of radiance accumulation.
#include <algorithm>

#include "vp_internal.h"
#include "vp_path.cuh"
#include "vp_traverse.cuh"

namespace vp {
namespace {

constexpr uint32_t kAliveBit = 1u << 18;

// Resident 256-thread blocks per SM the extend / shadow kernels' register budgets are sized for:
// 4 (64 registers) for extend; 5 (48 registers, 52 B of spills) for the FP32 shadow kernel, whose
// smaller state gains more from the extra warps than it loses to the spills (-2% shadow time on
// the showcase; extend at 5 spills 116 B and loses 9%).  The ACCURATE (float-pair) shadow kernel keeps
// the extend budget.
#ifndef VP_WF_MIN_BLOCKS
#define VP_WF_MIN_BLOCKS 4
#endif
#ifndef VP_WF_SHADOW_MIN_BLOCKS
#define VP_WF_SHADOW_MIN_BLOCKS 5
#endif
// Hit-buffer entries of the extend kernel (chords retained for the scatter-point albedo plus
// one leaf's new ones); the shadow kernel retains none and uses 32.
#ifndef VP_WF_EXTEND_HIT_CAP
#define VP_WF_EXTEND_HIT_CAP 64
#endif
constexpr int kExtendHitCap = VP_WF_EXTEND_HIT_CAP;
// Queues shorter than this are not re-sorted (the sort would cost more than it saves).
#ifndef VP_WF_SORT_MIN
#define VP_WF_SORT_MIN 65536
#endif
constexpr uint32_t kSortMinPaths = VP_WF_SORT_MIN;

__device__ __forceinline__ uint32_t meta_bounce(uint32_t m) { return m & 0xFFFFu; }
__device__ __forceinline__ uint32_t meta_nshadow(uint32_t m) { return (m >> 16) & 3u; }

__device__ __forceinline__ void store_path(const WfBuffers& b, uint32_t p, const PathState& s) {
  b.o4[p] = make_float4(s.o.x, s.o.y, s.o.z, 0.f);
  b.d4[p] = make_float4(s.d.x, s.d.y, s.d.z, 0.f);
  b.thr4[p] = make_float4(s.thr.x, s.thr.y, s.thr.z, 0.f);
  b.rad4[p] = make_float4(s.rad.x, s.rad.y, s.rad.z, 0.f);
  b.rng4[p] = make_uint4((uint32_t)s.rng.state, (uint32_t)(s.rng.state >> 32), (uint32_t)s.rng.inc,
                         (uint32_t)(s.rng.inc >> 32));
}

__device__ __forceinline__ PathState load_path(const WfBuffers& b, uint32_t p, uint32_t bounce) {
  PathState s;
  const float4 o = b.o4[p], d = b.d4[p], t = b.thr4[p], r = b.rad4[p];
  const uint4 g = b.rng4[p];
  s.o = f3(o.x, o.y, o.z);
  s.d = f3(d.x, d.y, d.z);
  s.thr = f3(t.x, t.y, t.z);
  s.rad = f3(r.x, r.y, r.z);
  s.rng.state = ((uint64_t)g.y << 32) | g.x;
  s.rng.inc = ((uint64_t)g.w << 32) | g.z;
  s.bounce = bounce;
  return s;
}

// Warp-aggregated queue append, called by all 32 lanes: returns this lane's first slot for its
// `n` (possibly 0) entries; one atomic per warp.
__device__ __forceinline__ uint32_t queue_reserve(uint32_t* counter, uint32_t n) {
  const int lane = threadIdx.x & 31;
  uint32_t incl = n;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += v;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  uint32_t base = 0;
  if (lane == 31 && total) base = atomicAdd(counter, total);
  base = __shfl_sync(kFull, base, 31);
  return base + incl - n;
}

// Path p is sample p % batch of pixel p / batch.  Without adaptive sampling every path starts
// and queue slot p holds path p.  With it, the host has cleared the counters and only the paths
// of pixels that have not converged join the queue (their order within a warp is kept).
__global__ void k_wf_generate(CameraView C, ParamsView P, uint32_t spp_offset, uint32_t batch, uint32_t n,
                              WfBuffers b, const float4* __restrict__ mean, const float4* __restrict__ m2,
                              const uint32_t* __restrict__ count, Counters* __restrict__ ctr) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool adaptive = P.adaptive_threshold > 0.0f;
  uint32_t slot = p;
  if (!adaptive) {
    if (p == 0) {
      b.ctr[0] = P.max_bounces > 0 ? n : 0u;
      b.ctr[1] = b.ctr[2] = b.ctr[3] = b.ctr[4] = 0u;
    }
    if (p >= n) return;
  } else {
    bool live = false;
    if (p < n) {
      const uint32_t pixel = p / batch;
      live = !pixel_converged(P, count[pixel], mean[pixel], m2[pixel]);
      if (!live && p % batch == 0u) atomicAdd(&ctr->skipped, (unsigned long long)batch);
    }
    slot = queue_reserve(b.ctr + 0, live ? 1u : 0u);  // all 32 lanes: blockDim is a multiple of 32
    if (!live) return;
  }
  const uint32_t pixel = p / batch, s = p % batch;
  PathState st = start_path(C, P, pixel % P.width, pixel / P.width, (uint64_t)spp_offset + s);
  const uint64_t key = draw_bounce_key(st.rng);
  store_path(b, p, st);
  b.key2[p] = make_uint2((uint32_t)key, (uint32_t)(key >> 32));
  b.meta[p] = 0u | kAliveBit;
  b.qa[slot] = p;
  b.L4[p] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// kMeasure = false compiles the statistics out (their registers would otherwise stay live
// through the traversal loop).
template <bool kAcc, bool kMeasure>
__global__ void __launch_bounds__(256, VP_WF_MIN_BLOCKS) k_wf_extend(SceneView S, ParamsView P, WfBuffers b, const uint32_t* q,
                                                   const uint32_t* count, unsigned int* work, Counters* ctr) {
  extern __shared__ unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem W = carve(smem + kRootStageBytes + warp * warp_smem_bytes(S.argmin_cap, kExtendHitCap), S.argmin_cap,
                     kExtendHitCap);
  if constexpr (VP_STAGE_ROOT) {
    stage_root(S.wide, S.wide_root);
    W.root_staged = true;
  }
  const uint32_t n = *count;
  uint32_t status = 0, max_overlap = 0;
  unsigned long long bounces = 0, scatters = 0;
  WarpStats ws;
  const bool measure = kMeasure && P.measure != 0;
  if (measure) ws.hist = &ctr->hits_hist[0][0];
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(work, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= n) break;
    const uint32_t p = __ldg(q + item);
    const float4 o = b.o4[p], d = b.d4[p];
    const uint2 k2 = b.key2[p];
    const uint32_t bounce = meta_bounce(b.meta[p]);
    const float3 of = f3(o.x, o.y, o.z), df = f3(d.x, d.y, d.z);
    float tstar = kInf;
    ScatterAlbedo sa;
    sa.valid = false;
    if (!(bounce == 0 && S.albedo_all_zero))
      tstar = warp_ray_query<kAcc, kArgmin>(S, W, of, df, ((uint64_t)k2.y << 32) | k2.x, status, ws, measure, &sa);
    float3 albedo = f3(0.f, 0.f, 0.f);
    if (tstar < kInf) {
      uint32_t ov = sa.overlap;
      albedo = sa.valid ? sa.albedo : warp_albedo<kAcc>(S, W, fma3(tstar, df, of), ov, status, ws, measure);
      max_overlap = max(max_overlap, ov);
      ++scatters;
    }
    ++bounces;
    if (lane == 0) {
      b.alb4[p] = make_float4(albedo.x, albedo.y, albedo.z, tstar);
      b.sg[p] = tstar < kInf ? sa.gauss : kNoGauss;
    }
    if (status) break;
  }
  if (lane == 0) {
    if (status) atomicOr(&ctr->status, status);
    if (measure) {
      atomicAdd(&ctr->bounces, bounces);
      atomicAdd(&ctr->scatters, scatters);
      atomicMax(&ctr->max_overlap, max_overlap);
      atomicAdd(&ctr->crossings, ws.crossings);
      atomicAdd(&ctr->nodes, ws.nodes);
      atomicAdd(&ctr->leaves, ws.leaves);
      atomicMax(&ctr->max_hits, ws.max_hits);
      for (int k = 0; k < 3; ++k) {
        atomicAdd(&ctr->kind_nodes[k], ws.kind_nodes[k]);
        atomicAdd(&ctr->kind_leaves[k], ws.kind_leaves[k]);
        atomicAdd(&ctr->kind_prims[k], ws.kind_prims[k]);
        atomicAdd(&ctr->kind_geo[k], ws.kind_geo[k]);
      }
    }
  }
}

// The shadow rays' seed chords are evaluated here, one thread per ray (seed_chord_tau): a ray
// whose seed chord alone reaches MAX_OPTICAL_DEPTH gets T = 0 and never enters the shadow queue;
// the others carry the seed's optical depth to the transmittance query in so4.w.
__global__ void __launch_bounds__(256) k_wf_shade(SceneView S, EnvView E, ParamsView P, WfBuffers b,
                                                  const uint32_t* q, const uint32_t* count, uint32_t* qnext,
                                                  uint32_t* cnext, Counters* ctr) {
  const uint32_t n = *count;
  unsigned long long shadows = 0, opaque = 0;
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  const uint32_t wid = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  // warp-uniform loop: every lane runs every iteration, so the queue appends are full-warp
  for (uint32_t base = wid * 32u; base < n; base += warps * 32u) {
    const uint32_t i = base + lane;
    const bool valid = i < n;
    uint32_t p = 0;
    int ns = 0;
    unsigned queued = 0u;  // bit k: shadow ray k enters the shadow queue
    bool alive = false;
    if (valid) {
      p = q[i];
      PathState s = load_path(b, p, meta_bounce(b.meta[p]));
      const float4 a = b.alb4[p];
      const bool scattered = a.w < kInf;
      ShadowSet sh;
      alive = shade_bounce(E, P, s, scattered, a.w, f3(a.x, a.y, a.z), sh, b.sg[p]);
      ns = sh.n;
      for (int k = 0; k < sh.n; ++k) {
        float seed_tau = -1.0f;  // no seed
        if (sh.seed[k] != kNoGauss)
          seed_tau = P.accurate ? seed_chord_tau<true>(S, sh.seed[k], sh.o[k], sh.d[k])
                                : seed_chord_tau<false>(S, sh.seed[k], sh.o[k], sh.d[k]);
        const bool opaque_k = seed_tau >= kMaxOpticalDepth;
        // .w of the origin: the seed's optical depth for the query, or T = 0 already
        b.so4[3u * p + k] = make_float4(sh.o[k].x, sh.o[k].y, sh.o[k].z, opaque_k ? 0.0f : seed_tau);
        b.sd4[3u * p + k] = make_float4(sh.d[k].x, sh.d[k].y, sh.d[k].z, __uint_as_float(sh.seed[k]));
        b.sw4[3u * p + k] = make_float4(sh.w[k].x, sh.w[k].y, sh.w[k].z, 0.f);
        if (!opaque_k) queued |= 1u << k;
        else opaque += 1;
      }
      if (alive) {
        const uint64_t key = draw_bounce_key(s.rng);
        b.key2[p] = make_uint2((uint32_t)key, (uint32_t)(key >> 32));
      }
      store_path(b, p, s);
      b.meta[p] = (s.bounce & 0xFFFFu) | ((uint32_t)sh.n << 16) | (alive ? kAliveBit : 0u);
    }
    shadows += (unsigned)ns;
    uint32_t slot = queue_reserve(b.ctr + 2, (uint32_t)__popc(queued));
    for (int k = 0; k < ns; ++k)
      if (queued & (1u << k)) b.qs[slot++] = 3u * p + k;
    const uint32_t qslot = queue_reserve(cnext, alive ? 1u : 0u);
    if (alive) qnext[qslot] = p;
  }
  if (P.measure) {
    for (int o = 16; o > 0; o >>= 1) {
      shadows += __shfl_xor_sync(0xFFFFFFFFu, shadows, o);
      opaque += __shfl_xor_sync(0xFFFFFFFFu, opaque, o);
    }
    if ((threadIdx.x & 31) == 0 && shadows) atomicAdd(&ctr->shadow_rays, shadows);
    if ((threadIdx.x & 31) == 0 && opaque) {  // transmittance queries answered by their seed chord
      atomicAdd(&ctr->crossings, opaque);
      atomicAdd(&ctr->hits_hist[1][1], opaque);
      atomicMax(&ctr->max_hits, 1u);
    }
  }
}

template <bool kAcc, bool kMeasure>
__global__ void __launch_bounds__(256, kAcc ? VP_WF_MIN_BLOCKS : VP_WF_SHADOW_MIN_BLOCKS) k_wf_shadow(SceneView S, WfBuffers b, const uint32_t* count,
                                                   unsigned int* work, Counters* ctr, int measure_i) {
  extern __shared__ unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem W = carve(smem + kRootStageBytes + warp * warp_smem_bytes(S.stack_cap, 32), S.stack_cap, 32);
  if constexpr (VP_STAGE_ROOT) {
    stage_root(S.wide, S.wide_root);
    W.root_staged = true;
  }
  const uint32_t n = *count;
  uint32_t status = 0;
  WarpStats ws;
  const bool measure = kMeasure && measure_i != 0;
  if (measure) ws.hist = &ctr->hits_hist[0][0];
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(work, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= n) break;
    const uint32_t slot = __ldg(b.qs + item);
    const float4 o = b.so4[slot], d = b.sd4[slot];
    const float tau = warp_ray_query<kAcc, kTau>(S, W, f3(o.x, o.y, o.z), f3(d.x, d.y, d.z), 0ull, status, ws,
                                                 measure, nullptr, __float_as_uint(d.w), o.w);
    if (lane == 0) b.so4[slot].w = tau >= kMaxOpticalDepth ? 0.0f : expf(-tau);
    if (status) break;
  }
  if (lane == 0) {
    if (status) atomicOr(&ctr->status, status);
    if (measure) {
      atomicAdd(&ctr->crossings, ws.crossings);
      atomicAdd(&ctr->nodes, ws.nodes);
      atomicAdd(&ctr->leaves, ws.leaves);
      atomicMax(&ctr->max_hits, ws.max_hits);
      for (int k = 0; k < 3; ++k) {
        atomicAdd(&ctr->kind_nodes[k], ws.kind_nodes[k]);
        atomicAdd(&ctr->kind_leaves[k], ws.kind_leaves[k]);
        atomicAdd(&ctr->kind_prims[k], ws.kind_prims[k]);
        atomicAdd(&ctr->kind_geo[k], ws.kind_geo[k]);
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_wf_gather(ParamsView P, WfBuffers b, const uint32_t* q,
                                                   const uint32_t* count) {
  const uint32_t n = *count;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t p = q[i];
    const uint32_t m = b.meta[p];
    const int ns = (int)meta_nshadow(m);
    const float4 r = b.rad4[p];
    float3 rad = f3(r.x, r.y, r.z);
    for (int k = 0; k < ns; ++k) {
      const float4 w = b.sw4[3u * p + k];
      rad = add(rad, mul(f3(w.x, w.y, w.z), b.so4[3u * p + k].w));
    }
    if (m & kAliveBit) {
      b.rad4[p] = make_float4(rad.x, rad.y, rad.z, 0.f);
    } else {
      const float3 L = finalize_sample(P, rad);
      b.L4[p] = make_float4(L.x, L.y, L.z, 0.f);
    }
  }
}

// Next bounce: the new queue becomes current; shadow queue and work heads restart.
__global__ void k_wf_advance(uint32_t* ctr) {
  ctr[0] = ctr[1];
  ctr[1] = 0u;
  ctr[2] = 0u;
  ctr[3] = 0u;
  ctr[4] = 0u;
}

// Welford mean over the batch's samples of each pixel, in sample order (raygen.cuh:214-242).
// With adaptive sampling it also keeps M2, and a pixel that k_wf_generate found converged (the
// same test on the same, still unchanged state) keeps its state.
__global__ void k_wf_welford(ParamsView P, WfBuffers b, uint32_t batch, uint32_t n_pix, float4* __restrict__ mean,
                             float4* __restrict__ m2, uint32_t* __restrict__ count) {
  const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= n_pix) return;
  const bool adaptive = P.adaptive_threshold > 0.0f;
  const uint32_t prev = count[pix];
  const float4 m4 = mean[pix];
  const float4 q4 = adaptive ? m2[pix] : make_float4(0.f, 0.f, 0.f, 0.f);
  if (adaptive && pixel_converged(P, prev, m4, q4)) return;
  float3 m = f3(m4.x, m4.y, m4.z), q = f3(q4.x, q4.y, q4.z);
  for (uint32_t s = 0; s < batch; ++s) {
    const float4 L = b.L4[(size_t)pix * batch + s];
    welford_step<true>(m, q, f3(L.x, L.y, L.z), prev + s + 1u);
  }
  mean[pix] = make_float4(m.x, m.y, m.z, 0.f);
  if (adaptive) m2[pix] = make_float4(q.x, q.y, q.z, 0.f);
  count[pix] = prev + batch;
}

// Morton key (10 bits per axis) of each queued path's origin over the scene bounds: sorting the
// queue by it makes neighbouring warps traverse the same BVH32 region (L1 reuse).
__device__ __forceinline__ uint32_t expand10(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_wf_sort_keys(uint32_t n, const uint32_t* __restrict__ q, const float4* __restrict__ o4,
                               float3 lo, float3 inv_ext, uint32_t* __restrict__ keys) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 o = o4[q[i]];
  auto quant = [](float x) { return (uint32_t)fminf(fmaxf(x, 0.0f), 1023.0f); };
  const uint32_t x = quant((o.x - lo.x) * inv_ext.x), y = quant((o.y - lo.y) * inv_ext.y),
                 z = quant((o.z - lo.z) * inv_ext.z);
  keys[i] = (expand10(z) << 2) | (expand10(y) << 1) | expand10(x);
}

template <class K>
int resident_blocks(K kernel, int threads, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem) != cudaSuccess) b = 1;
  return b < 1 ? 1 : b;
}

template <class T>
void carve_buf(char*& cur, T*& out, size_t count) {
  out = reinterpret_cast<T*>(cur);
  cur += (count * sizeof(T) + 255) & ~size_t(255);
}

vp_status ensure_workspace(vp_context* ctx, size_t paths) {
  WfWorkspace& w = ctx->wf;
  if (w.cap >= paths && w.base) return VP_OK;
  free_wavefront(ctx);
  const size_t per_path = 4 * 16 + 16 + 8 + 4 + 16 + 4 + 3 * 48 + 16 + 4 * 3 + 3 * 4;
  const size_t bytes = paths * per_path + 64 * 256 + 4096;
  cudaError_t e = cudaMalloc(&w.base, bytes);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    w.base = nullptr;
    return fail(VP_ERROR_OUT_OF_MEMORY, "wavefront workspace of " + std::to_string(bytes) + " bytes");
  }
  if (!w.host_count) {
    e = cudaMallocHost(&w.host_count, sizeof(uint32_t));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
  }
  char* cur = static_cast<char*>(w.base);
  WfBuffers& b = w.b;
  carve_buf(cur, b.o4, paths);
  carve_buf(cur, b.d4, paths);
  carve_buf(cur, b.thr4, paths);
  carve_buf(cur, b.rad4, paths);
  carve_buf(cur, b.rng4, paths);
  carve_buf(cur, b.key2, paths);
  carve_buf(cur, b.meta, paths);
  carve_buf(cur, b.alb4, paths);
  carve_buf(cur, b.sg, paths);
  carve_buf(cur, b.so4, 3 * paths);
  carve_buf(cur, b.sd4, 3 * paths);
  carve_buf(cur, b.sw4, 3 * paths);
  carve_buf(cur, b.L4, paths);
  carve_buf(cur, b.qa, paths);
  carve_buf(cur, b.qb, paths);
  carve_buf(cur, b.qs, 3 * paths);
  carve_buf(cur, b.sk_a, paths);
  carve_buf(cur, b.ctr, 64);
  w.cap = paths;
  const size_t tmp = radix_sort_tmp_bytes_u32(paths);
  e = cudaMalloc(&w.sort_tmp, tmp);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    free_wavefront(ctx);
    return fail(VP_ERROR_OUT_OF_MEMORY, "wavefront sort scratch");
  }
  w.sort_tmp_bytes = tmp;
  return VP_OK;
}

}  // namespace

void free_wavefront(vp_context* ctx) {
  WfWorkspace& w = ctx->wf;
  if (w.base) cudaFree(w.base);
  if (w.sort_tmp) cudaFree(w.sort_tmp);
  w.base = nullptr;
  w.sort_tmp = nullptr;
  w.sort_tmp_bytes = 0;
  w.cap = 0;
}

vp_status launch_wavefront(vp_scene* s, vp_env* e, const CameraView& cam, const ParamsView& P, vp_image* img,
                           uint32_t spp_offset, uint32_t spp_count) {
  vp_context* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t n_pix = P.width * P.height;
  const uint64_t paths64 = (uint64_t)n_pix * spp_count;
  if (paths64 == 0) return VP_OK;
  if (paths64 >= (1ull << 31) / 3) return fail(VP_ERROR_LIMIT, "batch too large for the wavefront engine");
  const uint32_t paths = (uint32_t)paths64;
  vp_status r;
  if ((r = ensure_workspace(ctx, paths))) return r;
  WfBuffers b = ctx->wf.b;
  const int threads = 256;
  const size_t smem = kRootStageBytes + (size_t)(threads / 32) * warp_smem_bytes(s->view.argmin_cap, kExtendHitCap);
  const size_t smem_sh = kRootStageBytes + (size_t)(threads / 32) * warp_smem_bytes(s->view.stack_cap, 32);
  if (smem > 200 * 1024) return fail(VP_ERROR_LIMIT, "BVH too deep for the shared-memory stack");
  auto ext = P.accurate ? (P.measure ? k_wf_extend<true, true> : k_wf_extend<true, false>)
                        : (P.measure ? k_wf_extend<false, true> : k_wf_extend<false, false>);
  auto shd = P.accurate ? (P.measure ? k_wf_shadow<true, true> : k_wf_shadow<true, false>)
                        : (P.measure ? k_wf_shadow<false, true> : k_wf_shadow<false, false>);
  if (smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(ext, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (smem_sh > 48 * 1024)
    VP_CUDA(cudaFuncSetAttribute(shd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_sh));
  const int ext_blocks = ctx->sm_count * resident_blocks(ext, threads, smem);
  const int shd_blocks = ctx->sm_count * resident_blocks(shd, threads, smem_sh);
  const int thr_blocks = ctx->sm_count * 8;
  // VP_MEASURE_STAGES: events around the extend and shadow launches of each iteration (a ring of 4 iterations,
  // read back at every poll, when the stream has drained)
  cudaEvent_t* ev = ctx->stage_ev;
  const bool timed = ctx->time_stages;
  if (timed && !ev[0])
    for (int i = 0; i < vp_context::kStageEvents; ++i) VP_CUDA(cudaEventCreate(&ev[i]));
  uint32_t pending = 0;  // iterations whose events are recorded but not yet read
  auto harvest = [&]() -> cudaError_t {
    for (uint32_t j = 0; j < pending; ++j) {
      float a = 0.f, c = 0.f;
      cudaError_t er = cudaEventElapsedTime(&a, ev[4 * j + 0], ev[4 * j + 1]);
      if (er == cudaSuccess) er = cudaEventElapsedTime(&c, ev[4 * j + 2], ev[4 * j + 3]);
      if (er != cudaSuccess) return er;
      ctx->stage_ms[0] += a;
      ctx->stage_ms[1] += c;
    }
    pending = 0;
    return cudaSuccess;
  };
  if (P.adaptive_threshold > 0.0f) VP_CUDA(cudaMemsetAsync(b.ctr, 0, 5 * sizeof(uint32_t), st));
  k_wf_generate<<<(paths + 255) / 256, 256, 0, st>>>(cam, P, spp_offset, spp_count, paths, b, img->mean, img->m2,
                                                     img->count, ctx->counters);
  VP_CUDA(cudaGetLastError());
  ctx->launches += 1;
  uint32_t* qcur = b.qa;
  uint32_t* qnext = b.qb;
  // Path origins' Morton order: the queue is re-sorted after every poll (the count is known on
  // the host then); compaction keeps most of the order in between.
  const vp_scene_info& si = s->info;
  const float3 blo = make_float3((float)si.bounds_min[0], (float)si.bounds_min[1], (float)si.bounds_min[2]);
  auto inv_ext1 = [](double a, double b) { return (float)(1024.0 / std::max(b - a, 1e-30)); };
  const float3 binv = make_float3(inv_ext1(si.bounds_min[0], si.bounds_max[0]),
                                  inv_ext1(si.bounds_min[1], si.bounds_max[1]),
                                  inv_ext1(si.bounds_min[2], si.bounds_max[2]));
  uint32_t polled = paths;
  for (uint32_t it = 0; it < P.max_bounces; ++it) {
    if (it != 0u && (it & 3u) == 0u && polled >= kSortMinPaths) {  // (camera rays share one origin)
      k_wf_sort_keys<<<(polled + 255) / 256, 256, 0, st>>>(polled, qcur, b.o4, blo, binv, b.sk_a);
      vp_status r = radix_sort_pairs(b.sk_a, qcur, polled, 30, ctx->wf.sort_tmp, ctx->wf.sort_tmp_bytes, st,
                                     &ctx->launches);
      if (r) return r;
    }
    cudaEvent_t* e4 = ev + 4 * (it & 3u);
    if (timed) VP_CUDA(cudaEventRecord(e4[0], st));
    ext<<<ext_blocks, threads, smem, st>>>(s->view, P, b, qcur, b.ctr + 0, b.ctr + 3, ctx->counters);
    if (timed) VP_CUDA(cudaEventRecord(e4[1], st));
    k_wf_shade<<<thr_blocks, threads, 0, st>>>(s->view, e->view, P, b, qcur, b.ctr + 0, qnext, b.ctr + 1,
                                               ctx->counters);
    if (timed) VP_CUDA(cudaEventRecord(e4[2], st));
    shd<<<shd_blocks, threads, smem_sh, st>>>(s->view, b, b.ctr + 2, b.ctr + 4, ctx->counters, P.measure);
    if (timed) VP_CUDA(cudaEventRecord(e4[3], st));
    k_wf_gather<<<thr_blocks, threads, 0, st>>>(P, b, qcur, b.ctr + 0);
    k_wf_advance<<<1, 1, 0, st>>>(b.ctr);
    VP_CUDA(cudaGetLastError());
    ctx->launches += 5;
    ctx->stage_launches[0] += 1;
    ctx->stage_launches[1] += 1;
    if (timed) ++pending;
    std::swap(qcur, qnext);
    if ((it & 3u) == 3u) {  // stop once no path is alive
      VP_CUDA(cudaMemcpyAsync(ctx->wf.host_count, b.ctr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      VP_CUDA(cudaStreamSynchronize(st));
      VP_CUDA(harvest());
      polled = *ctx->wf.host_count;
      if (polled == 0u) break;
    }
  }
  k_wf_welford<<<(n_pix + 255) / 256, 256, 0, st>>>(P, b, spp_count, n_pix, img->mean, img->m2, img->count);
  VP_CUDA(cudaGetLastError());
  ctx->launches += 1;
  if (timed && pending) {
    VP_CUDA(cudaStreamSynchronize(st));
    VP_CUDA(harvest());
  }
  return VP_OK;
}

}  // namespace vp
