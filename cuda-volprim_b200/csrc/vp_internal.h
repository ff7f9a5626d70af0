// Host-side objects behind the opaque handles of include/volprim_b200.h, and the error
// plumbing shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/volprim_b200.h"
#include "vp_device.cuh"

namespace vp {

// Thread-local last error (vp_last_error_string).
void set_error(const std::string& msg);
vp_status fail(vp_status code, const std::string& msg);
vp_status cuda_fail(cudaError_t e, const char* what);

#define VP_CUDA(call)                                       \
  do {                                                      \
    cudaError_t _e = (call);                                \
    if (_e != cudaSuccess) return ::vp::cuda_fail(_e, #call); \
  } while (0)

template <class T>
vp_status dev_alloc(T** p, size_t count, cudaStream_t s) {
  *p = nullptr;
  if (count == 0) return VP_OK;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(p), count * sizeof(T), s);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    return fail(VP_ERROR_OUT_OF_MEMORY, "device allocation of " + std::to_string(count * sizeof(T)) + " bytes failed");
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
  return VP_OK;
}
template <class T>
void dev_free(T*& p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
  p = nullptr;
}

}  // namespace vp

namespace vp {
// Wavefront path state (structure of arrays, one entry per path of a launch batch) and queues.
struct WfBuffers {
  float4 *o4, *d4, *thr4, *rad4;  // ray origin / direction / throughput / radiance (.w unused)
  uint4* rng4;                    // PCG32 state (lo, hi) and increment (lo, hi)
  uint2* key2;                    // free-flight key of the next bounce
  uint32_t* meta;                 // bounce | shadow count << 16 | alive << 18
  float4* alb4;                   // albedo at the scatter point, scatter distance
  uint32_t* sg;                   // the Gaussian of the scatter (scene order) or kNoGauss
  float4 *so4, *sd4, *sw4;        // 3 transmittance queries per path: origin (.w: the seed chord's
                                  // optical depth, -1 without a seed; then T), dir (+ the
                                  // seed Gaussian's bits in .w), weight
  float4* L4;                     // finished sample radiance
  uint32_t *qa, *qb, *qs;         // path queues (current / next) and shadow-query queue
  uint32_t* sk_a;                 // sorting: the Morton keys of path origins
  uint32_t* ctr;                  // [0] paths now, [1] paths next, [2] shadow queries, [3..4] work heads
};
struct WfWorkspace {
  size_t cap = 0;  // paths
  WfBuffers b{};
  void* base = nullptr;
  void* sort_tmp = nullptr;  // radix-sort scratch for `cap` keys (radix_sort_pairs)
  size_t sort_tmp_bytes = 0;
  uint32_t* host_count = nullptr;  // pinned, for polling the active-path count
};
}  // namespace vp

struct vp_context {
  int32_t device = 0;
  int32_t sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  vp::Counters* counters = nullptr;   // device, one block of statistics per render call
  unsigned int* work_counter = nullptr;  // device, persistent-kernel work queue head
  vp::WfWorkspace wf;                 // wavefront engine buffers (grow-only)
  // launch accounting of the current render call (reset by vp_render_accumulate)
  uint32_t launches = 0;              // kernels launched
  bool time_stages = false;           // VP_MEASURE_STAGES
  double stage_ms[2] = {0.0, 0.0};    // wavefront extend, shadow
  uint32_t stage_launches[2] = {0, 0};
  static constexpr int kStageEvents = 16;  // 4 wavefront iterations x 4 events
  cudaEvent_t stage_ev[kStageEvents] = {};
};

struct vp_scene {
  vp_context* ctx = nullptr;
  vp::SceneView view{};
  float4* prims = nullptr;
  uint32_t* perm = nullptr;
  float4* wide = nullptr;
  float4* bin = nullptr;
  float4* pbox = nullptr;
  // as given by the caller, in the scene's order: quaternion (w,x,y,z), then scale (log or
  // linear, as scale_is_log says) and density -- the chain-rule inputs of the adjoint
  float4* raw = nullptr;
  float4* emis = nullptr;  // RGB emission per unit optical depth (vp_scene_set_emission)
  int32_t scale_is_log = 0;
  float sigma_multiplier = 1.0f;
  vp_scene_info info{};
};

struct vp_env {
  vp_context* ctx = nullptr;
  vp::EnvView view{};
  float4* texels = nullptr;
  float2* cond = nullptr;
  float2* marg = nullptr;
  float* joint = nullptr;
  double build_ms = 0.0;
};

struct vp_image {
  vp_context* ctx = nullptr;
  uint32_t width = 0, height = 0;
  float4* mean = nullptr;
  uint32_t* count = nullptr;
  // Welford sum of squared deviations per channel (w unused), allocated by the first batch with
  // adaptive sampling.  m2_complete: every batch since the last clear kept it.
  float4* m2 = nullptr;
  bool m2_complete = true;
};

namespace vp {
vp_status build_scene(vp_context* ctx, const vp_gaussians* g, float sigma_multiplier, const vp_scene_options& opt,
                      vp_scene* s);
vp_status build_env(vp_context* ctx, const float* rgb, uint32_t w, uint32_t h, uint32_t channels,
                    int32_t memory, vp_env* env);
// Host restatement of host::params::Camera::build (camera.h:32-111).
void build_camera(const vp_camera& cam, uint32_t width, uint32_t height, CameraView& out);
ParamsView make_params(const vp_render_params& p, const vp_scene* s);
vp_status check_params(const vp_render_params* p);
vp_status launch_render(vp_scene* s, vp_env* e, const CameraView& cam, const ParamsView& P,
                        int32_t engine, vp_image* img, uint32_t spp_offset, uint32_t spp_count);
vp_status launch_transmittance(vp_scene* s, const float* o, const float* d, uint32_t n,
                               bool accurate, int32_t engine, float* out);
vp_status launch_wavefront(vp_scene* s, vp_env* e, const CameraView& cam, const ParamsView& P, vp_image* img,
                           uint32_t spp_offset, uint32_t spp_count);
void free_wavefront(vp_context* ctx);
vp_status launch_albedo(vp_scene* s, const float* pts, uint32_t n, bool accurate, int32_t engine, float* rgb,
                        uint32_t* cnt);
vp_status launch_normalize(const float4* in, float4* out, size_t n, float scale, cudaStream_t st);

// Device-wide sort and scan (vp_sort.cu).  radix_sort_pairs sorts (key, value) pairs in place by
// the key bits [0, end_bit), stably; `tmp` holds radix_sort_tmp_bytes_*(n) bytes.  exclusive_scan
// writes the exclusive prefix sums of n counts (in may equal out); `tmp` holds
// exclusive_scan_tmp_bytes(n) bytes.  `launches`, when given, counts the kernels launched.
size_t radix_sort_tmp_bytes_u64(size_t n);
size_t radix_sort_tmp_bytes_u32(size_t n);
size_t exclusive_scan_tmp_bytes(size_t n);
vp_status radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint32_t n, int end_bit, void* tmp, size_t tmp_bytes,
                           cudaStream_t st, uint32_t* launches = nullptr);
vp_status radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, int end_bit, void* tmp, size_t tmp_bytes,
                           cudaStream_t st, uint32_t* launches = nullptr);
vp_status exclusive_scan(const uint32_t* in, uint32_t* out, size_t n, void* tmp, size_t tmp_bytes, cudaStream_t st,
                         uint32_t* launches = nullptr);
vp_status exclusive_scan(const unsigned long long* in, unsigned long long* out, size_t n, void* tmp, size_t tmp_bytes,
                         cudaStream_t st, uint32_t* launches = nullptr);
}  // namespace vp
