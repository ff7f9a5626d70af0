// extern "C" entry points of include/volprim_b200.h: argument checking, object lifetime, the
// host restatement of the reference's camera build and render-parameter folding, and the
// batch loop of Renderer::render (src/thesis/host/app/renderer.cpp:341-376).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "vp_internal.h"

namespace vp {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }
vp_status fail(vp_status code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
vp_status cuda_fail(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return e == cudaErrorMemoryAllocation ? VP_ERROR_OUT_OF_MEMORY : VP_ERROR_CUDA;
}

// ---- host float3 arithmetic in the reference's operation order (math.h) --------------------
namespace hm {
struct V {
  float x, y, z;
};
inline V mk(float x, float y, float z) { return V{x, y, z}; }
inline V add(V a, V b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V sub(V a, V b) { return mk(a.x + (-b.x), a.y + (-b.y), a.z + (-b.z)); }
inline V neg(V a) { return mk(-a.x, -a.y, -a.z); }
inline V muls(V a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline float dot(V a, V b) { return std::fmaf(a.x, b.x, std::fmaf(a.y, b.y, a.z * b.z)); }
inline float rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline V normalize(V v) { return muls(v, rsqrt(dot(v, v))); }
inline float length(V v) { return std::sqrt(dot(v, v)); }
inline V cross(V a, V b) {
  return mk(std::fmaf(a.y, b.z, -(a.z * b.y)), std::fmaf(a.z, b.x, -(a.x * b.z)),
            std::fmaf(a.x, b.y, -(a.y * b.x)));
}
inline V lerp(V a, V b, float t) {
  return mk(std::fmaf(t, b.x - a.x, a.x), std::fmaf(t, b.y - a.y, a.y), std::fmaf(t, b.z - a.z, a.z));
}
inline V midpoint(V a, V b) { return lerp(a, b, 0.5f); }
inline float3 f3(V v) { return make_float3(v.x, v.y, v.z); }
}  // namespace hm

void build_camera(const vp_camera& cam, uint32_t width, uint32_t height, CameraView& out) {
  using namespace hm;
  const V lookfrom = mk(cam.eye[0], cam.eye[1], cam.eye[2]);
  const V lookat = mk(cam.lookat[0], cam.lookat[1], cam.lookat[2]);
  const V vup = mk(cam.up[0], cam.up[1], cam.up[2]);
  const float fw = static_cast<float>(width), fh = static_cast<float>(height);
  if (!cam.orthographic) {  // buildPerspective (host/params/camera.h:40-70)
    const float theta = cam.vfov_deg * (3.14159265358979323846f / 180.0f);
    const float h = std::tan(0.5f * theta);
    const V w = normalize(sub(lookfrom, lookat));
    const V u = normalize(cross(vup, w));
    const V v = cross(w, u);
    const float focal = length(sub(lookfrom, lookat));
    const float aspect = fw * (1.0f / fh);
    const float vh = 2.0f * h * focal;
    const float vw = vh * aspect;
    const V vu = muls(u, vw);
    const V vv = muls(neg(v), vh);
    const V du = muls(vu, 1.0f / fw);
    const V dv = muls(vv, 1.0f / fh);
    const V ul = sub(sub(lookfrom, muls(w, focal)), midpoint(vu, vv));
    const V p00 = add(ul, midpoint(du, dv));
    out.ortho = 0;
    out.eye = f3(lookfrom);
    out.p00 = f3(sub(p00, lookfrom));
    out.du = f3(du);
    out.dv = f3(dv);
    out.view_dir = make_float3(0.f, 0.f, 1.f);
  } else {  // buildOrthographic (host/params/camera.h:72-111)
    const V view_dir = normalize(sub(lookat, lookfrom));
    const V right = normalize(cross(view_dir, vup));
    const V up = cross(right, view_dir);
    const float aspect = fw * (1.0f / fh);
    const float vh = cam.ortho_height;
    const float vw = vh * aspect;
    const V vu = muls(right, vw);
    const V vv = muls(up, vh);
    const V du = muls(vu, 1.0f / fw);
    const V dv = muls(vv, 1.0f / fh);
    const V ul = sub(lookfrom, midpoint(vu, vv));
    const V p00 = add(ul, midpoint(du, dv));
    out.ortho = 1;
    out.eye = f3(lookfrom);
    out.p00 = f3(sub(p00, lookfrom));
    out.du = f3(du);
    out.dv = f3(dv);
    out.view_dir = f3(view_dir);
  }
}

ParamsView make_params(const vp_render_params& p, const vp_scene* s) {
  ParamsView P{};
  P.width = p.width;
  P.height = p.height;
  P.spp_total = p.spp;
  P.seed = p.seed;
  P.max_bounces = p.max_bounces;
  P.rr_depth = p.rr_depth;
  P.rr_max_survival = p.rr_max_survival;
  P.firefly_clamp = p.firefly_clamp;
  P.filter_stddev = p.pixel_filter_stddev;
  P.nee_mode = p.nee_mode;
  P.ris_k = p.ris_candidates;
  // Henyey-Greenstein pre-fold (renderer.cpp:224-235): eval uses +g, sample uses -g.
  const float g = p.hg_g;
  const float abs_g = g < 0.0f ? -g : g;
  P.hg_iso = abs_g < 1e-3f ? 1 : 0;
  P.hg_g = g;
  P.hg_g_eff = -g;
  const float g2 = g * g;
  P.hg_one_plus_g2 = 1.0f + g2;
  P.hg_one_minus_g2 = 1.0f - g2;
  P.hg_neg_inv_2g = P.hg_iso ? 0.0f : (-0.5f / P.hg_g_eff);
  P.hg_phase_coeff = (1.0f / (4.0f * 3.14159265358979323846f)) * P.hg_one_minus_g2;
  P.accurate = p.precision == VP_PRECISION_ACCURATE ||
               (p.precision == VP_PRECISION_AUTO && s->view.albedo_all_zero);
  P.measure = p.measure & VP_MEASURE_COUNTERS;
  P.adaptive_threshold = p.adaptive_threshold;
  P.adaptive_min_samples = p.adaptive_min_samples;
  return P;
}

vp_status check_params(const vp_render_params* p) {
  if (!p) return fail(VP_ERROR_INVALID_ARGUMENT, "params is NULL");
  if (p->width == 0 || p->height == 0) return fail(VP_ERROR_INVALID_ARGUMENT, "image size must be positive");
  if ((uint64_t)p->width * p->height >= (1ull << 31)) return fail(VP_ERROR_LIMIT, "image too large");
  if (p->spp == 0) return fail(VP_ERROR_INVALID_ARGUMENT, "spp must be positive");
  if (p->nee_mode < VP_NEE_MIS || p->nee_mode > VP_NEE_NONE) return fail(VP_ERROR_INVALID_ARGUMENT, "unknown nee_mode");
  if (p->nee_mode == VP_NEE_RIS && p->ris_candidates == 0)
    return fail(VP_ERROR_INVALID_ARGUMENT, "ris_candidates must be positive");
  if (p->engine != VP_ENGINE_WARP && p->engine != VP_ENGINE_MEGAKERNEL && p->engine != VP_ENGINE_WAVEFRONT)
    return fail(VP_ERROR_INVALID_ARGUMENT, "unknown engine");
  if (p->precision < VP_PRECISION_AUTO || p->precision > VP_PRECISION_ACCURATE)
    return fail(VP_ERROR_INVALID_ARGUMENT, "unknown precision");
  if (!(p->hg_g > -1.0f && p->hg_g < 1.0f)) return fail(VP_ERROR_INVALID_ARGUMENT, "hg_g must be in (-1, 1)");
  if (!(p->adaptive_threshold >= 0.0f && p->adaptive_threshold <= 3.402823466e38f))
    return fail(VP_ERROR_INVALID_ARGUMENT, "adaptive_threshold must be finite and non-negative");
  return VP_OK;
}

__global__ void k_camera_rays(CameraView C, ParamsView P, const uint32_t* __restrict__ px,
                              const uint32_t* __restrict__ py, const uint32_t* __restrict__ sample, uint32_t n,
                              float* __restrict__ o, float* __restrict__ d) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t pix = (uint64_t)py[i] * P.width + px[i];
  Pcg32 rng = pcg_init(P.seed, seq_hash(pix * (uint64_t)P.spp_total + sample[i]));
  float3 oo, dd;
  camera_ray(C, P, px[i], py[i], rng, oo, dd);
  o[3 * i] = oo.x, o[3 * i + 1] = oo.y, o[3 * i + 2] = oo.z;
  d[3 * i] = dd.x, d[3 * i + 1] = dd.y, d[3 * i + 2] = dd.z;
}

__global__ void k_mean_to_rgba(const float4* __restrict__ mean, float4* __restrict__ out, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 m = mean[i];
  out[i] = make_float4(m.x, m.y, m.z, 1.0f);
}

}  // namespace vp

using namespace vp;

extern "C" {

const char* vp_last_error_string(void) { return g_last_error.c_str(); }

vp_status vp_version(int32_t* major, int32_t* minor) {
  if (!major || !minor) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL output");
  *major = VP_VERSION_MAJOR;
  *minor = VP_VERSION_MINOR;
  return VP_OK;
}

vp_status vp_context_create(int32_t device, vp_context** out) {
  if (!out) return fail(VP_ERROR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  int n = 0;
  VP_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(VP_ERROR_INVALID_ARGUMENT, "device index out of range");
  VP_CUDA(cudaSetDevice(device));
  auto* c = new (std::nothrow) vp_context();
  if (!c) return fail(VP_ERROR_OUT_OF_MEMORY, "host allocation failed");
  c->device = device;
  cudaError_t e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  if (e == cudaSuccess) e = cudaMalloc(&c->counters, sizeof(Counters));
  if (e == cudaSuccess) e = cudaMalloc(&c->work_counter, sizeof(unsigned int));
  if (e != cudaSuccess) {
    vp_context_destroy(c);
    return cuda_fail(e, "vp_context_create");
  }
  *out = c;
  return VP_OK;
}

vp_status vp_context_destroy(vp_context* c) {
  if (!c) return VP_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->counters) cudaFree(c->counters);
  if (c->work_counter) cudaFree(c->work_counter);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (cudaEvent_t ev : c->stage_ev)
    if (ev) cudaEventDestroy(ev);
  free_wavefront(c);
  if (c->wf.host_count) cudaFreeHost(c->wf.host_count);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return VP_OK;
}

vp_status vp_context_stream(vp_context* c, void** out) {
  if (!c || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = c->stream;
  return VP_OK;
}

vp_status vp_context_synchronize(vp_context* c) {
  if (!c) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL context");
  VP_CUDA(cudaStreamSynchronize(c->stream));
  return VP_OK;
}

vp_status vp_context_sm_count(vp_context* c, int32_t* out) {
  if (!c || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = c->sm_count;
  return VP_OK;
}

// Default BVH32 collapse of vp_scene_options_default.
#ifndef VP_DEFAULT_COLLAPSE
#define VP_DEFAULT_COLLAPSE VP_COLLAPSE_SAH
#endif

vp_status vp_scene_options_default(vp_scene_options* out) {
  if (!out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = vp_scene_options{VP_TREE_PLOC, VP_TREE_PLOC, 24u, VP_DEFAULT_COLLAPSE, VP_TAU_ORDER_AUTO};
  return VP_OK;
}

vp_status vp_scene_create_ex(vp_context* ctx, const vp_gaussians* g, float sigma_multiplier,
                             const vp_scene_options* options, vp_scene** out) {
  if (!ctx || !g || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  vp_scene_options opt;
  vp_scene_options_default(&opt);
  if (options) opt = *options;
  auto builder_ok = [](int32_t b) { return b == VP_TREE_PLOC || b == VP_TREE_LBVH; };
  if (!builder_ok(opt.wide_builder) || !builder_ok(opt.binary_builder))
    return fail(VP_ERROR_INVALID_ARGUMENT, "vp_scene_options: builders must be VP_TREE_PLOC or VP_TREE_LBVH");
  if (opt.wide_collapse != VP_COLLAPSE_GREEDY && opt.wide_collapse != VP_COLLAPSE_SAH)
    return fail(VP_ERROR_INVALID_ARGUMENT, "vp_scene_options.wide_collapse must be VP_COLLAPSE_GREEDY or VP_COLLAPSE_SAH");
  if (opt.leaf_max < 1u || opt.leaf_max > 32u)
    return fail(VP_ERROR_INVALID_ARGUMENT, "vp_scene_options.leaf_max must be in [1, 32]");
  if (opt.tau_order < VP_TAU_ORDER_AUTO || opt.tau_order > VP_TAU_ORDER_NEAREST)
    return fail(VP_ERROR_INVALID_ARGUMENT, "vp_scene_options.tau_order must be a vp_tau_order");
  VP_CUDA(cudaSetDevice(ctx->device));
  auto* s = new (std::nothrow) vp_scene();
  if (!s) return fail(VP_ERROR_OUT_OF_MEMORY, "host allocation failed");
  s->ctx = ctx;
  const vp_status st = build_scene(ctx, g, sigma_multiplier, opt, s);
  if (st != VP_OK) {
    const std::string msg = g_last_error;
    vp_scene_destroy(s);
    g_last_error = msg;
    return st;
  }
  *out = s;
  return VP_OK;
}

vp_status vp_scene_create(vp_context* ctx, const vp_gaussians* g, float sigma_multiplier, vp_scene** out) {
  return vp_scene_create_ex(ctx, g, sigma_multiplier, nullptr, out);
}

vp_status vp_scene_info_get(vp_scene* s, vp_scene_info* out) {
  if (!s || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = s->info;
  return VP_OK;
}

vp_status vp_scene_destroy(vp_scene* s) {
  if (!s) return VP_OK;
  cudaStream_t st = s->ctx ? s->ctx->stream : nullptr;
  dev_free(s->prims, st);
  dev_free(s->perm, st);
  dev_free(s->wide, st);
  dev_free(s->bin, st);
  dev_free(s->pbox, st);
  dev_free(s->raw, st);
  dev_free(s->emis, st);
  if (st) cudaStreamSynchronize(st);
  delete s;
  return VP_OK;
}

vp_status vp_env_create(vp_context* ctx, const float* rgb, uint32_t w, uint32_t h, uint32_t channels,
                        int32_t memory, vp_env** out) {
  if (!ctx || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  VP_CUDA(cudaSetDevice(ctx->device));
  auto* e = new (std::nothrow) vp_env();
  if (!e) return fail(VP_ERROR_OUT_OF_MEMORY, "host allocation failed");
  e->ctx = ctx;
  const vp_status st = build_env(ctx, rgb, w, h, channels, memory, e);
  if (st != VP_OK) {
    const std::string msg = g_last_error;
    vp_env_destroy(e);
    g_last_error = msg;
    return st;
  }
  *out = e;
  return VP_OK;
}

vp_status vp_env_create_constant(vp_context* ctx, float r, float g, float b, vp_env** out) {
  const float rgb[6] = {r, g, b, r, g, b};
  return vp_env_create(ctx, rgb, 2, 1, 3, VP_MEMORY_HOST, out);
}

vp_status vp_env_build_ms(vp_env* e, double* out) {
  if (!e || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = e->build_ms;
  return VP_OK;
}

vp_status vp_env_read_tables(vp_env* e, uint32_t* out_w, uint32_t* out_h, float* cond_prob, uint32_t* cond_alias,
                             float* marg_prob, uint32_t* marg_alias, float* joint, float* out_total) {
  if (!e || !e->ctx) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  const uint32_t W = e->view.width, H = e->view.height;
  if (out_w) *out_w = W;
  if (out_h) *out_h = H;
  if (out_total) *out_total = e->view.total;
  const size_t n = (size_t)W * H;
  VP_CUDA(cudaSetDevice(e->ctx->device));
  cudaStream_t st = e->ctx->stream;
  std::vector<float2> cond(cond_prob || cond_alias ? n : 0), marg(marg_prob || marg_alias ? H : 0);
  if (!cond.empty()) VP_CUDA(cudaMemcpyAsync(cond.data(), e->cond, n * sizeof(float2), cudaMemcpyDeviceToHost, st));
  if (!marg.empty()) VP_CUDA(cudaMemcpyAsync(marg.data(), e->marg, H * sizeof(float2), cudaMemcpyDeviceToHost, st));
  if (joint) VP_CUDA(cudaMemcpyAsync(joint, e->joint, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  VP_CUDA(cudaStreamSynchronize(st));
  for (size_t i = 0; i < cond.size(); ++i) {
    if (cond_prob) cond_prob[i] = cond[i].x;
    if (cond_alias) std::memcpy(cond_alias + i, &cond[i].y, sizeof(uint32_t));
  }
  for (size_t i = 0; i < marg.size(); ++i) {
    if (marg_prob) marg_prob[i] = marg[i].x;
    if (marg_alias) std::memcpy(marg_alias + i, &marg[i].y, sizeof(uint32_t));
  }
  return VP_OK;
}

vp_status vp_env_destroy(vp_env* e) {
  if (!e) return VP_OK;
  cudaStream_t st = e->ctx ? e->ctx->stream : nullptr;
  dev_free(e->texels, st);
  dev_free(e->cond, st);
  dev_free(e->marg, st);
  dev_free(e->joint, st);
  if (st) cudaStreamSynchronize(st);
  delete e;
  return VP_OK;
}

vp_status vp_render_params_default(vp_render_params* p) {
  if (!p) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  std::memset(p, 0, sizeof(*p));
  p->width = 1000;  // Config defaults (config.h:30-47)
  p->height = 750;
  p->spp = 1;
  p->seed = 42;
  p->max_bounces = 128;
  p->rr_depth = 12;
  p->rr_max_survival = 0.99f;
  p->hg_g = 0.85f;
  p->firefly_clamp = 0.0f;
  p->pixel_filter_stddev = 0.0f;
  p->nee_mode = VP_NEE_MIS;
  p->ris_candidates = 6;
  p->batch_spp = 16;  // BATCH_SIZE (renderer.cpp:32)
  p->engine = VP_ENGINE_WAVEFRONT;
  p->precision = VP_PRECISION_AUTO;
  p->measure = 0;
  p->adaptive_threshold = 0.0f;   // ADAPTIVE_THRESHOLD (constants.cuh:207): off
  p->adaptive_min_samples = 32;   // ADAPTIVE_MIN_SAMPLES (constants.cuh:202)
  return VP_OK;
}

vp_status vp_image_create(vp_context* ctx, uint32_t w, uint32_t h, vp_image** out) {
  if (!ctx || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (w == 0 || h == 0 || (uint64_t)w * h >= (1ull << 31)) return fail(VP_ERROR_INVALID_ARGUMENT, "bad image size");
  VP_CUDA(cudaSetDevice(ctx->device));
  auto* im = new (std::nothrow) vp_image();
  if (!im) return fail(VP_ERROR_OUT_OF_MEMORY, "host allocation failed");
  im->ctx = ctx;
  im->width = w;
  im->height = h;
  vp_status s;
  if ((s = dev_alloc(&im->mean, (size_t)w * h, ctx->stream)) || (s = dev_alloc(&im->count, (size_t)w * h, ctx->stream))) {
    vp_image_destroy(im);
    return s;
  }
  s = vp_image_clear(im);
  if (s) {
    vp_image_destroy(im);
    return s;
  }
  *out = im;
  return VP_OK;
}

vp_status vp_image_clear(vp_image* im) {
  if (!im) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL image");
  const size_t n = (size_t)im->width * im->height;
  VP_CUDA(cudaMemsetAsync(im->mean, 0, n * sizeof(float4), im->ctx->stream));
  VP_CUDA(cudaMemsetAsync(im->count, 0, n * sizeof(uint32_t), im->ctx->stream));
  if (im->m2) VP_CUDA(cudaMemsetAsync(im->m2, 0, n * sizeof(float4), im->ctx->stream));
  im->m2_complete = true;
  return VP_OK;
}

vp_status vp_image_destroy(vp_image* im) {
  if (!im) return VP_OK;
  cudaStream_t st = im->ctx ? im->ctx->stream : nullptr;
  dev_free(im->mean, st);
  dev_free(im->m2, st);
  dev_free(im->count, st);
  if (st) cudaStreamSynchronize(st);
  delete im;
  return VP_OK;
}

vp_status vp_image_read(vp_image* im, float* out, int32_t memory) {
  if (!im || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  cudaStream_t st = im->ctx->stream;
  const size_t n = (size_t)im->width * im->height;
  if (memory == VP_MEMORY_DEVICE) {
    k_mean_to_rgba<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(im->mean, reinterpret_cast<float4*>(out), n);
    VP_CUDA(cudaGetLastError());
    VP_CUDA(cudaStreamSynchronize(st));
    return VP_OK;
  }
  if (memory != VP_MEMORY_HOST) return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind");
  float4* tmp = nullptr;
  vp_status s;
  if ((s = dev_alloc(&tmp, n, st))) return s;
  k_mean_to_rgba<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(im->mean, tmp, n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, n * sizeof(float4), cudaMemcpyDeviceToHost, st);
  dev_free(tmp, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "vp_image_read");
  return VP_OK;
}

vp_status vp_image_device_buffers(vp_image* im, void** mean, void** count) {
  if (!im || !mean || !count) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *mean = im->mean;
  *count = im->count;
  return VP_OK;
}

vp_status vp_image_read_welford(vp_image* im, float* out_m2, uint32_t* out_count, int32_t memory) {
  if (!im) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL image");
  if (memory != VP_MEMORY_HOST && memory != VP_MEMORY_DEVICE) return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind");
  if (out_m2 && !im->m2_complete)
    return fail(VP_ERROR_INVALID_ARGUMENT, "M2 is incomplete: a batch since the last clear ran without adaptive sampling");
  cudaStream_t st = im->ctx->stream;
  const size_t n = (size_t)im->width * im->height;
  const cudaMemcpyKind kind = memory == VP_MEMORY_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  VP_CUDA(cudaSetDevice(im->ctx->device));
  if (out_m2 && im->m2) {
    VP_CUDA(cudaMemcpyAsync(out_m2, im->m2, n * sizeof(float4), kind, st));
  } else if (out_m2) {  // no adaptive batch since the image was made: no samples, M2 = 0
    VP_CUDA(cudaStreamSynchronize(st));
    if (memory == VP_MEMORY_HOST) std::memset(out_m2, 0, n * sizeof(float4));
    else VP_CUDA(cudaMemsetAsync(out_m2, 0, n * sizeof(float4), st));
  }
  if (out_count) VP_CUDA(cudaMemcpyAsync(out_count, im->count, n * sizeof(uint32_t), kind, st));
  VP_CUDA(cudaStreamSynchronize(st));
  return VP_OK;
}

vp_status vp_render_accumulate(vp_scene* s, vp_env* e, const vp_camera* cam, const vp_render_params* p,
                               vp_image* im, uint32_t spp_offset, uint32_t spp_count, vp_render_stats* stats) {
  if (!s || !e || !cam || !im) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  vp_status st;
  if ((st = check_params(p))) return st;
  if (s->ctx != e->ctx || s->ctx != im->ctx) return fail(VP_ERROR_INVALID_ARGUMENT, "objects belong to different contexts");
  if (im->width != p->width || im->height != p->height) return fail(VP_ERROR_INVALID_ARGUMENT, "image size does not match params");
  if ((uint64_t)spp_offset + spp_count > p->spp) return fail(VP_ERROR_INVALID_ARGUMENT, "sample range exceeds params->spp");
  vp_context* ctx = s->ctx;
  VP_CUDA(cudaSetDevice(ctx->device));
  // Adaptive sampling reads M2, which only adaptive batches keep (the reference allocates and
  // updates it only when ENABLE_ADAPTIVE_SAMPLING is compiled in, image.h:43-57).
  if (spp_count > 0 && p->adaptive_threshold > 0.0f) {
    if (!im->m2_complete)
      return fail(VP_ERROR_INVALID_ARGUMENT,
                  "adaptive sampling needs every batch since the image's last clear to keep M2 (adaptive_threshold > 0)");
    if (!im->m2) {
      const size_t n = (size_t)im->width * im->height;
      if ((st = dev_alloc(&im->m2, n, ctx->stream))) return st;
      VP_CUDA(cudaMemsetAsync(im->m2, 0, n * sizeof(float4), ctx->stream));
    }
  } else if (spp_count > 0) {
    im->m2_complete = false;
  }
  CameraView cv;
  build_camera(*cam, p->width, p->height, cv);
  const ParamsView P = make_params(*p, s);
  ctx->launches = 0;
  ctx->time_stages = (p->measure & VP_MEASURE_STAGES) != 0;
  ctx->stage_ms[0] = ctx->stage_ms[1] = 0.0;
  ctx->stage_launches[0] = ctx->stage_launches[1] = 0;
  VP_CUDA(cudaMemsetAsync(ctx->counters, 0, sizeof(Counters), ctx->stream));
  VP_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  const uint32_t batch = p->batch_spp ? p->batch_spp : spp_count;
  for (uint32_t off = 0; off < spp_count; off += batch) {
    const uint32_t cnt = std::min(batch, spp_count - off);
    if (p->engine == VP_ENGINE_WAVEFRONT) {
      if ((st = launch_wavefront(s, e, cv, P, im, spp_offset + off, cnt))) return st;
    } else if ((st = launch_render(s, e, cv, P, p->engine, im, spp_offset + off, cnt))) {
      return st;
    }
  }
  VP_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  VP_CUDA(cudaEventSynchronize(ctx->ev1));
  Counters c{};
  VP_CUDA(cudaMemcpy(&c, ctx->counters, sizeof(c), cudaMemcpyDeviceToHost));
  if (stats) {
    float ms = 0.f;
    VP_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    std::memset(stats, 0, sizeof(*stats));
    stats->ms_kernels = ms;
    stats->paths = (uint64_t)p->width * p->height * spp_count - c.skipped;
    stats->paths_skipped = c.skipped;
    stats->bounces = c.bounces;
    stats->scatters = c.scatters;
    stats->crossings = c.crossings;
    stats->shadow_rays = c.shadow_rays;
    stats->nodes_visited = c.nodes;
    stats->leaves_visited = c.leaves;
    for (int k = 0; k < 3; ++k) {
      stats->query_nodes[k] = c.kind_nodes[k];
      stats->query_leaves[k] = c.kind_leaves[k];
      stats->query_prim_tests[k] = c.kind_prims[k];
      stats->query_geo_loads[k] = c.kind_geo[k];
      stats->prim_tests += c.kind_prims[k];
      stats->geo_loads += c.kind_geo[k];
    }
    stats->max_hits_per_ray = c.max_hits;
    stats->max_point_overlap = c.max_overlap;
    stats->device_status = c.status;
    stats->launches = ctx->launches;
    for (int q = 0; q < 2; ++q)
      for (int b = 0; b < 16; ++b) stats->hits_hist[q][b] = c.hits_hist[q][b];
    if (ctx->time_stages) {
      stats->ms_stage[0] = ctx->stage_ms[0];
      stats->ms_stage[1] = ctx->stage_ms[1];
      stats->ms_stage[2] = std::max(0.0, (double)ms - ctx->stage_ms[0] - ctx->stage_ms[1]);
      stats->stage_launches[0] = ctx->stage_launches[0];
      stats->stage_launches[1] = ctx->stage_launches[1];
      stats->stage_launches[2] = ctx->launches - ctx->stage_launches[0] - ctx->stage_launches[1];
    }
  }
  ctx->time_stages = false;
  if (c.status) return fail(VP_ERROR_DEVICE_STATUS, "a render kernel raised device status " + std::to_string(c.status));
  return VP_OK;
}

vp_status vp_render(vp_scene* s, vp_env* e, const vp_camera* cam, const vp_render_params* p, float* out,
                    int32_t memory, vp_render_stats* stats) {
  if (!s || !e || !cam || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  vp_status st;
  if ((st = check_params(p))) return st;
  vp_image* im = nullptr;
  if ((st = vp_image_create(s->ctx, p->width, p->height, &im))) return st;
  st = vp_render_accumulate(s, e, cam, p, im, 0, p->spp, stats);
  if (st == VP_OK) st = vp_image_read(im, out, memory);
  const std::string msg = g_last_error;
  vp_image_destroy(im);
  g_last_error = msg;
  return st;
}

vp_status vp_transmittance(vp_scene* s, const float* origins, const float* dirs, uint32_t n, int32_t precision,
                           int32_t engine, float* out, int32_t memory) {
  if (!s || (n > 0 && (!origins || !dirs || !out))) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (precision < VP_PRECISION_AUTO || precision > VP_PRECISION_ACCURATE) return fail(VP_ERROR_INVALID_ARGUMENT, "unknown precision");
  if (n == 0) return VP_OK;
  vp_context* ctx = s->ctx;
  VP_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const bool accurate = precision == VP_PRECISION_ACCURATE || (precision == VP_PRECISION_AUTO && s->view.albedo_all_zero);
  VP_CUDA(cudaMemsetAsync(ctx->counters, 0, sizeof(Counters), st));
  vp_status r;
  if (memory == VP_MEMORY_DEVICE) {
    if ((r = launch_transmittance(s, origins, dirs, n, accurate, engine, out))) return r;
  } else if (memory == VP_MEMORY_HOST) {
    float *o = nullptr, *d = nullptr, *t = nullptr;
    if ((r = dev_alloc(&o, 3ull * n, st)) || (r = dev_alloc(&d, 3ull * n, st)) || (r = dev_alloc(&t, n, st))) {
      dev_free(o, st);
      dev_free(d, st);
      dev_free(t, st);
      return r;
    }
    cudaError_t e = cudaMemcpyAsync(o, origins, 12ull * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, dirs, 12ull * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) r = launch_transmittance(s, o, d, n, accurate, engine, t);
    if (e == cudaSuccess && r == VP_OK) e = cudaMemcpyAsync(out, t, 4ull * n, cudaMemcpyDeviceToHost, st);
    dev_free(o, st);
    dev_free(d, st);
    dev_free(t, st);
    if (e != cudaSuccess) return cuda_fail(e, "vp_transmittance");
    if (r) return r;
  } else {
    return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind");
  }
  VP_CUDA(cudaStreamSynchronize(st));
  Counters c{};
  VP_CUDA(cudaMemcpy(&c, ctx->counters, sizeof(c), cudaMemcpyDeviceToHost));
  if (c.status) return fail(VP_ERROR_DEVICE_STATUS, "transmittance kernel raised device status " + std::to_string(c.status));
  return VP_OK;
}

vp_status vp_camera_rays(vp_context* ctx, const vp_camera* cam, const vp_render_params* p, const uint32_t* px,
                         const uint32_t* py, const uint32_t* sample, uint32_t n, float* out_o, float* out_d,
                         int32_t memory) {
  if (!ctx || !cam || !p || (n > 0 && (!px || !py || !sample || !out_o || !out_d)))
    return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (p->width == 0 || p->height == 0 || p->spp == 0) return fail(VP_ERROR_INVALID_ARGUMENT, "bad params");
  if (n == 0) return VP_OK;
  VP_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  CameraView cv;
  build_camera(*cam, p->width, p->height, cv);
  ParamsView P{};
  P.width = p->width;
  P.height = p->height;
  P.spp_total = p->spp;
  P.seed = p->seed;
  P.filter_stddev = p->pixel_filter_stddev;
  if (memory == VP_MEMORY_DEVICE) {
    k_camera_rays<<<(n + 127) / 128, 128, 0, st>>>(cv, P, px, py, sample, n, out_o, out_d);
    VP_CUDA(cudaGetLastError());
    VP_CUDA(cudaStreamSynchronize(st));
    return VP_OK;
  }
  if (memory != VP_MEMORY_HOST) return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind");
  uint32_t *dx = nullptr, *dy = nullptr, *ds = nullptr;
  float *dof = nullptr, *ddf = nullptr;
  vp_status r;
  if ((r = dev_alloc(&dx, n, st)) || (r = dev_alloc(&dy, n, st)) || (r = dev_alloc(&ds, n, st)) ||
      (r = dev_alloc(&dof, 3ull * n, st)) || (r = dev_alloc(&ddf, 3ull * n, st))) {
    dev_free(dx, st), dev_free(dy, st), dev_free(ds, st), dev_free(dof, st), dev_free(ddf, st);
    return r;
  }
  cudaError_t e = cudaMemcpyAsync(dx, px, 4ull * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dy, py, 4ull * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ds, sample, 4ull * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    k_camera_rays<<<(n + 127) / 128, 128, 0, st>>>(cv, P, dx, dy, ds, n, dof, ddf);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out_o, dof, 12ull * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out_d, ddf, 12ull * n, cudaMemcpyDeviceToHost, st);
  dev_free(dx, st), dev_free(dy, st), dev_free(ds, st), dev_free(dof, st), dev_free(ddf, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "vp_camera_rays");
  return VP_OK;
}

vp_status vp_albedo_at(vp_scene* s, const float* points, uint32_t n, int32_t precision, int32_t engine,
                       float* out_rgb, uint32_t* out_overlap, int32_t memory) {
  if (!s || (n > 0 && (!points || !out_rgb || !out_overlap))) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (precision < VP_PRECISION_AUTO || precision > VP_PRECISION_ACCURATE) return fail(VP_ERROR_INVALID_ARGUMENT, "unknown precision");
  if (n == 0) return VP_OK;
  vp_context* ctx = s->ctx;
  VP_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const bool accurate = precision == VP_PRECISION_ACCURATE || (precision == VP_PRECISION_AUTO && s->view.albedo_all_zero);
  VP_CUDA(cudaMemsetAsync(ctx->counters, 0, sizeof(Counters), st));
  vp_status r = VP_OK;
  if (memory == VP_MEMORY_DEVICE) {
    if ((r = launch_albedo(s, points, n, accurate, engine, out_rgb, out_overlap))) return r;
  } else if (memory == VP_MEMORY_HOST) {
    float *p = nullptr, *rgb = nullptr;
    uint32_t* cnt = nullptr;
    if ((r = dev_alloc(&p, 3ull * n, st)) || (r = dev_alloc(&rgb, 3ull * n, st)) || (r = dev_alloc(&cnt, n, st))) {
      dev_free(p, st);
      dev_free(rgb, st);
      dev_free(cnt, st);
      return r;
    }
    cudaError_t e = cudaMemcpyAsync(p, points, 12ull * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) r = launch_albedo(s, p, n, accurate, engine, rgb, cnt);
    if (e == cudaSuccess && r == VP_OK) e = cudaMemcpyAsync(out_rgb, rgb, 12ull * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && r == VP_OK) e = cudaMemcpyAsync(out_overlap, cnt, 4ull * n, cudaMemcpyDeviceToHost, st);
    dev_free(p, st);
    dev_free(rgb, st);
    dev_free(cnt, st);
    if (e != cudaSuccess) return cuda_fail(e, "vp_albedo_at");
    if (r) return r;
  } else {
    return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind");
  }
  VP_CUDA(cudaStreamSynchronize(st));
  Counters c{};
  VP_CUDA(cudaMemcpy(&c, ctx->counters, sizeof(c), cudaMemcpyDeviceToHost));
  if (c.status) return fail(VP_ERROR_DEVICE_STATUS, "albedo kernel raised device status " + std::to_string(c.status));
  return VP_OK;
}

vp_status vp_normalize_accumulator(vp_context* ctx, float* out, const float* acc, size_t n, float scale, void* stream) {
  if (!ctx || (n > 0 && (!out || !acc))) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  return launch_normalize(reinterpret_cast<const float4*>(acc), reinterpret_cast<float4*>(out), n, scale, st);
}

}  // extern "C"
