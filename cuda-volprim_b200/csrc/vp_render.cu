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
#include <type_traits>

#include "vp_internal.h"
#include "vp_path.cuh"
#include "vp_traverse.cuh"

namespace vp {
namespace {

struct PathStats {
  unsigned long long bounces = 0, scatters = 0, shadow = 0;
  unsigned int max_overlap = 0;
};

// ---- the path loop, shared by the warp engine and the megakernel through a query policy -----
template <class Q>
__device__ float3 trace_path(const SceneView& S, const EnvView& E, const CameraView& C,
                             const ParamsView& P, Q& q, uint32_t px, uint32_t py,
                             uint64_t sample_index, PathStats& ps) {
  PathState s = start_path(C, P, px, py, sample_index);
  bool alive = P.max_bounces > 0;
  while (alive) {
    const uint64_t key = draw_bounce_key(s.rng);
    // Stages 1-3 of sample_scattering_event (sampling.cuh:474-540): ADT argmin over every
    // overlapped Gaussian, with the albedo of the rebuilt active set.  In a scene whose albedo
    // is 0 everywhere a scatter ends the path with zero contribution, so the camera-ray argmin
    // is skipped there (the bounce-0 direct term is the whole image).
    float tstar = kInf;
    ScatterAlbedo sa;
    sa.valid = false;
    if (!(s.bounce == 0 && S.albedo_all_zero)) tstar = q.argmin(s.o, s.d, key, &sa);
    const bool scattered = tstar < kInf;
    float3 albedo = f3(0.f, 0.f, 0.f);
    if (scattered) {
      uint32_t overlap = sa.overlap;
      albedo = sa.valid ? sa.albedo : q.albedo(fma3(tstar, s.d, s.o), overlap);
      if (P.measure) ps.max_overlap = max(ps.max_overlap, overlap);
    }
    if (P.measure) {
      ps.bounces++;
      if (scattered) ps.scatters++;
    }
    ShadowSet sh;
    alive = shade_bounce(E, P, s, scattered, tstar, albedo, sh, scattered ? sa.gauss : kNoGauss);
#pragma unroll 1
    for (int k = 0; k < sh.n; ++k) {  // compute_transmittance_to_env (sampling.cuh:548-583)
      s.rad = add(s.rad, mul(sh.w[k], q.transmittance(sh.o[k], sh.d[k], sh.seed[k])));
      if (P.measure) ps.shadow++;
    }
  }
  return finalize_sample(P, s.rad);
}

template <bool kAcc>
struct WarpQueries {
  const SceneView& S;
  const WarpSmem& W;
  uint32_t& status;
  WarpStats& ws;
  bool measure;
  __device__ float argmin(float3 o, float3 d, uint64_t key, ScatterAlbedo* sa) {
    return warp_ray_query<kAcc, kArgmin>(S, W, o, d, key, status, ws, measure, sa);
  }
  __device__ float transmittance(float3 o, float3 d, uint32_t seed = kNoGauss) {
    const float tau = warp_ray_query<kAcc, kTau>(S, W, o, d, 0ull, status, ws, measure, nullptr, seed);
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
  for (int k = 0; k < 3; ++k) {
    atomicAdd(&c->kind_nodes[k], ws.kind_nodes[k]);
    atomicAdd(&c->kind_leaves[k], ws.kind_leaves[k]);
    atomicAdd(&c->kind_prims[k], ws.kind_prims[k]);
    atomicAdd(&c->kind_geo[k], ws.kind_geo[k]);
  }
  atomicMax(&c->max_hits, ws.max_hits);
  atomicMax(&c->max_overlap, ps.max_overlap);
}

// Persistent warp-per-path kernel: warps pull pixels from a global counter; each pixel runs
// samples [spp_offset, spp_offset + spp_count) in order and Welford-updates mean/count.
// kAdaptive also keeps M2 and skips converged pixels (M2 stays out of the registers of the
// plain variant, whose sample loop has none to spare).
template <bool kAcc, bool kMeasure, bool kAdaptive>
__global__ void __launch_bounds__(256, VP_WARP_MIN_BLOCKS) k_render_warp(SceneView S, EnvView E, CameraView C,
                                                     ParamsView P, float4* __restrict__ mean,
                                                     float4* __restrict__ m2, uint32_t* __restrict__ count,
                                                     uint32_t spp_offset, uint32_t spp_count,
                                                     unsigned int* __restrict__ work,
                                                     Counters* __restrict__ ctr) {
  extern __shared__ unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpSmem W = carve(smem + warp * warp_smem_bytes(S.argmin_cap, kHitCap), S.argmin_cap, kHitCap);
  const uint32_t n_pix = P.width * P.height;
  uint32_t status = 0;
  WarpStats ws;
  if (kMeasure && P.measure != 0) ws.hist = &ctr->hits_hist[0][0];
  PathStats ps;
  WarpQueries<kAcc> q{S, W, status, ws, kMeasure && P.measure != 0};
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(work, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= n_pix) break;
    const uint32_t px = item % P.width, py = item / P.width;
    const uint32_t prev = count[item];
    const float4 m4 = mean[item];
    float3 m = f3(m4.x, m4.y, m4.z), m2c = f3(0.f, 0.f, 0.f);
    if constexpr (kAdaptive) {
      const float4 q4 = m2[item];
      if (pixel_converged(P, prev, m4, q4)) {  // the same state on every lane: a warp-uniform skip
        if (lane == 0) atomicAdd(&ctr->skipped, (unsigned long long)spp_count);
        continue;
      }
      m2c = f3(q4.x, q4.y, q4.z);
    }
    for (uint32_t s = 0; s < spp_count; ++s) {
      const float3 L = trace_path(S, E, C, P, q, px, py, (uint64_t)spp_offset + s, ps);
      welford_step<kAdaptive>(m, m2c, L, prev + s + 1u);
    }
    if (lane == 0) {
      mean[item] = make_float4(m.x, m.y, m.z, 0.f);
      if constexpr (kAdaptive) m2[item] = make_float4(m2c.x, m2c.y, m2c.z, 0.f);
      count[item] = prev + spp_count;
    }
    if (status) break;
  }
  if (lane == 0) flush_stats(ctr, ps, ws, status, kMeasure && P.measure != 0);
}

// ------------------------------------------------------------------------------------------
// megakernel (thread per pixel, binary LBVH)
// ------------------------------------------------------------------------------------------
template <bool kAcc, bool kAdaptive>
__global__ void __launch_bounds__(128) k_render_mega(SceneView S, EnvView E, CameraView C, ParamsView P,
                                                     float4* __restrict__ mean, float4* __restrict__ m2,
                                                     uint32_t* __restrict__ count,
                                                     uint32_t spp_offset, uint32_t spp_count,
                                                     Counters* __restrict__ ctr) {
  const uint32_t px = blockIdx.x * 16 + (threadIdx.x & 15);
  const uint32_t py = blockIdx.y * 8 + (threadIdx.x >> 4);
  uint32_t status = 0;
  WarpStats ws;  // no hit histogram here: the baseline kernel keeps its registers
  PathStats ps;
  const bool inside = px < P.width && py < P.height;
  if (inside) {
    ThreadQueries<kAcc> q{S, status, ws, P.measure != 0};
    const uint32_t item = py * P.width + px;
    const uint32_t prev = count[item];
    const float4 m4 = mean[item];
    const float4 q4 = kAdaptive ? m2[item] : make_float4(0.f, 0.f, 0.f, 0.f);
    if (kAdaptive && pixel_converged(P, prev, m4, q4)) {
      atomicAdd(&ctr->skipped, (unsigned long long)spp_count);
    } else {
      float3 m = f3(m4.x, m4.y, m4.z), m2c = f3(q4.x, q4.y, q4.z);
      for (uint32_t s = 0; s < spp_count; ++s) {
        const float3 L = trace_path(S, E, C, P, q, px, py, (uint64_t)spp_offset + s, ps);
        welford_step<kAdaptive>(m, m2c, L, prev + s + 1u);
      }
      mean[item] = make_float4(m.x, m.y, m.z, 0.f);
      if constexpr (kAdaptive) m2[item] = make_float4(m2c.x, m2c.y, m2c.z, 0.f);
      count[item] = prev + spp_count;
    }
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
  const WarpSmem W = carve(smem + warp * warp_smem_bytes(S.stack_cap, 32), S.stack_cap, 32);
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
  const WarpSmem W = carve(smem + warp * warp_smem_bytes(S.stack_cap, 32), S.stack_cap, 32);
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
    const size_t smem = (size_t)(threads / 32) * warp_smem_bytes(s->view.argmin_cap, kHitCap);
    if (smem > 200 * 1024) return fail(VP_ERROR_LIMIT, "BVH too deep for the warp engine's shared-memory stack");
    VP_CUDA(cudaMemsetAsync(ctx->work_counter, 0, sizeof(unsigned int), st));
    const bool adaptive = P.adaptive_threshold > 0.0f;
    auto pick = [&](auto acc) {
      constexpr bool kA = decltype(acc)::value;
      return adaptive ? (P.measure ? k_render_warp<kA, true, true> : k_render_warp<kA, false, true>)
                      : (P.measure ? k_render_warp<kA, true, false> : k_render_warp<kA, false, false>);
    };
    auto kern = P.accurate ? pick(std::true_type{}) : pick(std::false_type{});
    if (smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int blocks = ctx->sm_count * occupancy_blocks(kern, threads, smem);
    kern<<<blocks, threads, smem, st>>>(s->view, e->view, cam, P, img->mean, img->m2, img->count, spp_offset, spp_count,
                                        ctx->work_counter, ctx->counters);
  } else if (engine == VP_ENGINE_MEGAKERNEL) {
    const dim3 grid((P.width + 15) / 16, (P.height + 7) / 8);
    const bool adaptive = P.adaptive_threshold > 0.0f;
    auto kern = P.accurate ? (adaptive ? k_render_mega<true, true> : k_render_mega<true, false>)
                           : (adaptive ? k_render_mega<false, true> : k_render_mega<false, false>);
    kern<<<grid, 128, 0, st>>>(s->view, e->view, cam, P, img->mean, img->m2, img->count, spp_offset, spp_count,
                               ctx->counters);
  } else {
    return fail(VP_ERROR_INVALID_ARGUMENT, "unknown engine");
  }
  ctx->launches += 1;
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
    const size_t smem = (size_t)(threads / 32) * warp_smem_bytes(s->view.stack_cap, 32);
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
    const size_t smem = (size_t)(threads / 32) * warp_smem_bytes(s->view.stack_cap, 32);
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
