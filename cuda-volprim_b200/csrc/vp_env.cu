// Environment-map build on the device: RGBA texels for the bilinear lookup, the
// luminance x sin(theta) sampling weights in FP64, a Vose alias table per row and one over the
// rows.  Replaces the reference's host FP32 2-D CDF (EnvironmentMap::buildCdf,
// include/thesis/host/params/environment_map.h:45-101) and texture upload (:105-151); the
// sampled distribution and its pdf are the same (proportional to joint texel weight).
#include <cmath>
#include <vector>

#include "vp_internal.h"

namespace vp {
namespace {

// Texel weight = Rec.709 luminance x sin(theta at the row centre), environment_map.h:51-66.
__global__ void k_env_texels(uint32_t W, uint32_t H, uint32_t ch, const float* __restrict__ rgb,
                             float4* __restrict__ tex, double* __restrict__ wts,
                             float* __restrict__ joint) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)W * H) return;
  const uint32_t v = (uint32_t)(i / W);
  const float* px = rgb + i * ch;
  const float r = px[0];
  const float g = ch >= 2 ? px[1] : r;
  const float b = ch >= 3 ? px[2] : r;
  const float a = ch >= 4 ? px[3] : 1.0f;
  tex[i] = make_float4(r, g, b, a);
  const double theta = ((double)v + 0.5) / (double)H * 3.14159265358979323846;
  const double lum = 0.2126 * (double)r + 0.7152 * (double)g + 0.0722 * (double)b;
  const double wgt = lum * sin(theta);
  wts[i] = wgt;
  joint[i] = (float)wgt;
}

__global__ void k_row_sums(uint32_t W, const double* __restrict__ wts, double* __restrict__ rows) {
  const uint32_t v = blockIdx.x;
  double s = 0.0;
  for (uint32_t u = threadIdx.x; u < W; u += blockDim.x) s += wts[(size_t)v * W + u];
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) rows[v] = red[0];
}

// Vose's alias method over n weights (one thread per table), FP64 probabilities.
__device__ void vose(uint32_t n, const double* __restrict__ w, double sum, double* __restrict__ p,
                     uint32_t* __restrict__ small, uint32_t* __restrict__ large,
                     float2* __restrict__ out) {
  if (!(sum > 0.0)) {
    for (uint32_t u = 0; u < n; ++u) out[u] = make_float2(1.0f, __uint_as_float(u));
    return;
  }
  uint32_t ns = 0, nl = 0;
  const double scale = (double)n / sum;
  for (uint32_t u = 0; u < n; ++u) {
    p[u] = w[u] * scale;
    if (p[u] < 1.0) small[ns++] = u;
    else large[nl++] = u;
  }
  while (ns > 0 && nl > 0) {
    const uint32_t l = small[--ns];
    const uint32_t g = large[--nl];
    out[l] = make_float2((float)p[l], __uint_as_float(g));
    p[g] = (p[g] + p[l]) - 1.0;
    if (p[g] < 1.0) small[ns++] = g;
    else large[nl++] = g;
  }
  while (nl > 0) {
    const uint32_t g = large[--nl];
    out[g] = make_float2(1.0f, __uint_as_float(g));
  }
  while (ns > 0) {
    const uint32_t l = small[--ns];
    out[l] = make_float2(1.0f, __uint_as_float(l));
  }
}

__global__ void k_alias_rows(uint32_t W, uint32_t H, const double* __restrict__ wts,
                             const double* __restrict__ rows, double* __restrict__ p,
                             uint32_t* __restrict__ sml, uint32_t* __restrict__ lrg,
                             float2* __restrict__ cond) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= H) return;
  const size_t o = (size_t)v * W;
  vose(W, wts + o, rows[v], p + o, sml + o, lrg + o, cond + o);
}

__global__ void k_alias_marginal(uint32_t H, const double* __restrict__ rows, double* __restrict__ p,
                                 uint32_t* __restrict__ sml, uint32_t* __restrict__ lrg,
                                 float2* __restrict__ marg, double* __restrict__ total) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double s = 0.0;
  for (uint32_t v = 0; v < H; ++v) s += rows[v];
  *total = s;
  vose(H, rows, s, p, sml, lrg, marg);
}

}  // namespace

vp_status build_env(vp_context* ctx, const float* rgb, uint32_t W, uint32_t H, uint32_t ch,
                    int32_t memory, vp_env* env) {
  cudaStream_t st = ctx->stream;
  if (!rgb || W == 0 || H == 0) return fail(VP_ERROR_INVALID_ARGUMENT, "environment map is empty");
  if (ch < 1 || ch > 4) return fail(VP_ERROR_INVALID_ARGUMENT, "environment channels must be 1..4");
  if ((uint64_t)W * H >= (1ull << 31)) return fail(VP_ERROR_LIMIT, "environment map too large");
  const size_t n = (size_t)W * H;
  VP_CUDA(cudaEventRecord(ctx->ev0, st));
  vp_status s;
  float* d_rgb = nullptr;
  const float* src = rgb;
  if (memory == VP_MEMORY_HOST) {
    if ((s = dev_alloc(&d_rgb, n * ch, st))) return s;
    VP_CUDA(cudaMemcpyAsync(d_rgb, rgb, n * ch * sizeof(float), cudaMemcpyHostToDevice, st));
    src = d_rgb;
  } else if (memory != VP_MEMORY_DEVICE) {
    return fail(VP_ERROR_INVALID_ARGUMENT, "memory must be VP_MEMORY_HOST or VP_MEMORY_DEVICE");
  }
  double *wts = nullptr, *rows = nullptr, *p = nullptr, *total = nullptr;
  uint32_t *sml = nullptr, *lrg = nullptr;
  auto cleanup = [&]() {
    dev_free(d_rgb, st);
    dev_free(wts, st);
    dev_free(rows, st);
    dev_free(p, st);
    dev_free(total, st);
    dev_free(sml, st);
    dev_free(lrg, st);
  };
  if ((s = dev_alloc(&env->texels, n, st)) || (s = dev_alloc(&env->joint, n, st)) ||
      (s = dev_alloc(&env->cond, n, st)) || (s = dev_alloc(&env->marg, H, st)) ||
      (s = dev_alloc(&wts, n, st)) || (s = dev_alloc(&rows, H, st)) || (s = dev_alloc(&p, n, st)) ||
      (s = dev_alloc(&sml, n, st)) || (s = dev_alloc(&lrg, n, st)) || (s = dev_alloc(&total, 1, st))) {
    cleanup();
    return s;
  }
  k_env_texels<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(W, H, ch, src, env->texels, wts, env->joint);
  k_row_sums<<<H, 256, 0, st>>>(W, wts, rows);
  k_alias_rows<<<(H + 63) / 64, 64, 0, st>>>(W, H, wts, rows, p, sml, lrg, env->cond);
  k_alias_marginal<<<1, 1, 0, st>>>(H, rows, p, sml, lrg, env->marg, total);
  cudaError_t e = cudaGetLastError();
  double tot = 0.0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&tot, total, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, st);
  cleanup();
  if (e == cudaSuccess) e = cudaEventSynchronize(ctx->ev1);
  if (e != cudaSuccess) return cuda_fail(e, "environment build");
  float ms = 0.f;
  VP_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  env->ctx = ctx;
  env->build_ms = ms;
  EnvView& v = env->view;
  v.texels = env->texels;
  v.cond = env->cond;
  v.marg = env->marg;
  v.joint = env->joint;
  v.width = W;
  v.height = H;
  v.total = (float)tot;
  v.inv_total = tot > 0.0 ? (float)(1.0 / tot) : 0.0f;
  return VP_OK;
}

}  // namespace vp
