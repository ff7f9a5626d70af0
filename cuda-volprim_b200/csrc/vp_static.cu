// Transmittance queries that allocate no device memory.
//
// vp_transmittance stages host rays in device buffers it allocates and uses the context's
// work-queue head and status word.  Some callers cannot allocate device memory at query time:
// a plug-in inside a host application that owns the whole device-memory budget (cudaMalloc may
// fail or is not theirs to call), or a latency-bound loop where cudaMalloc / cudaFree would
// synchronise the device.  For them, vp_transmittance_static runs the same warp-per-ray
// transmittance traversal with all of its scratch -- the staged rays and results of up to
// kStaticMaxRays rays, the work-queue head and the status word -- in one file-scope
// `static __device__` array.  Every GPU that loads the library holds that array (about 1.8 MB)
// until the process exits.
//
// Use rules (repeated in include/volprim_b200.h):
//  * The first call on a device resolves the array's device address (cudaGetSymbolAddress, with
//    that device current) and caches it for the life of the process.  The cached address
//    belongs to the device's primary context:
//    like every handle of this library, it does not survive cudaDeviceReset (or a destroyed and
//    re-created primary context), so reset no device while the library is in use.
//  * Each call waits for its own work on the context's stream (cudaStreamSynchronize) before it
//    returns, and reads the status word back to the host, so no call can be stream-captured.
//  * All calls share the one array, and each call leaves its contents behind: the queue head
//    and status word are cleared at the start of every call.  Calls whose work overlaps on the
//    GPU (other streams, other host threads) race on the array and must be serialised by the
//    caller.
//  * More than kStaticMaxRays rays in one call is an error (VP_ERROR_LIMIT).
#include <mutex>

#include "vp_internal.h"
#include "vp_traverse.cuh"

namespace vp {
namespace {

constexpr uint32_t kStaticMaxRays = 65536;
constexpr size_t kHeadBytes = 256;  // [0] work-queue head, [1] status word
constexpr size_t kOrgOffset = kHeadBytes;
constexpr size_t kDirOffset = kOrgOffset + 12ull * kStaticMaxRays;
constexpr size_t kOutOffset = kDirOffset + 12ull * kStaticMaxRays;
constexpr size_t kStaticBytes = kOutOffset + 4ull * kStaticMaxRays;

static __device__ __align__(256) unsigned char g_tau_scratch[kStaticBytes];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
unsigned char* g_addr[kMaxDevices] = {};

// The array's device address on the current device (set-up once per device).
vp_status scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return fail(VP_ERROR_LIMIT, "device index beyond the static scratch table");
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_tau_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static transmittance scratch)");
    g_addr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_addr[device];
  return VP_OK;
}

// The warp-per-ray transmittance kernel with its queue head and status word in the static array.
template <bool kAcc>
__global__ void __launch_bounds__(256) k_tau_static(SceneView S, const float* __restrict__ org,
                                                    const float* __restrict__ dir, uint32_t n,
                                                    float* __restrict__ out) {
  extern __shared__ unsigned char smem[];
  unsigned int* head = reinterpret_cast<unsigned int*>(g_tau_scratch);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpSmem W = carve(smem + warp * warp_smem_bytes(S.stack_cap, 32), S.stack_cap, 32);
  uint32_t status = 0;
  WarpStats ws;
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(head, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= n) break;
    const float3 o = f3(org[3 * item], org[3 * item + 1], org[3 * item + 2]);
    const float3 d = f3(dir[3 * item], dir[3 * item + 1], dir[3 * item + 2]);
    const float tau = warp_ray_query<kAcc, kTau>(S, W, o, d, 0ull, status, ws, false);
    if (lane == 0) out[item] = tau >= kMaxOpticalDepth ? 0.0f : expf(-tau);
    if (status) break;
  }
  if (lane == 0 && status) atomicOr(head + 1, status);
}

template <class K>
int static_resident_blocks(K kernel, int threads, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem) != cudaSuccess) b = 1;
  return b < 1 ? 1 : b;
}

}  // namespace
}  // namespace vp

using namespace vp;

extern "C" vp_status vp_transmittance_static(vp_scene* s, const float* origins, const float* dirs, uint32_t n,
                                             int32_t precision, float* out_transmittance, int32_t memory) {
  if (!s || (n > 0 && (!origins || !dirs || !out_transmittance))) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (precision < VP_PRECISION_AUTO || precision > VP_PRECISION_ACCURATE) return fail(VP_ERROR_INVALID_ARGUMENT, "unknown precision");
  if (memory != VP_MEMORY_HOST && memory != VP_MEMORY_DEVICE) return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind");
  if (n > kStaticMaxRays)
    return fail(VP_ERROR_LIMIT, "vp_transmittance_static takes at most " + std::to_string(kStaticMaxRays) +
                                    " rays per call (got " + std::to_string(n) + ")");
  if (n == 0) return VP_OK;
  vp_context* ctx = s->ctx;
  VP_CUDA(cudaSetDevice(ctx->device));
  unsigned char* base = nullptr;
  vp_status r;
  if ((r = scratch_address(ctx->device, &base))) return r;
  cudaStream_t st = ctx->stream;
  const bool accurate = precision == VP_PRECISION_ACCURATE || (precision == VP_PRECISION_AUTO && s->view.albedo_all_zero);
  VP_CUDA(cudaMemsetAsync(base, 0, kHeadBytes, st));  // queue head and status start at zero
  const float* o = origins;
  const float* d = dirs;
  float* t = out_transmittance;
  if (memory == VP_MEMORY_HOST) {
    VP_CUDA(cudaMemcpyAsync(base + kOrgOffset, origins, 12ull * n, cudaMemcpyHostToDevice, st));
    VP_CUDA(cudaMemcpyAsync(base + kDirOffset, dirs, 12ull * n, cudaMemcpyHostToDevice, st));
    o = reinterpret_cast<const float*>(base + kOrgOffset);
    d = reinterpret_cast<const float*>(base + kDirOffset);
    t = reinterpret_cast<float*>(base + kOutOffset);
  }
  const int threads = 256;
  const size_t smem = (size_t)(threads / 32) * warp_smem_bytes(s->view.stack_cap, 32);
  if (smem > 200 * 1024) return fail(VP_ERROR_LIMIT, "BVH too deep for the shared-memory stack");
  auto kern = accurate ? k_tau_static<true> : k_tau_static<false>;
  if (smem > 48 * 1024) VP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int blocks = ctx->sm_count * static_resident_blocks(kern, threads, smem);
  kern<<<blocks, threads, smem, st>>>(s->view, o, d, n, t);
  VP_CUDA(cudaGetLastError());
  if (memory == VP_MEMORY_HOST)
    VP_CUDA(cudaMemcpyAsync(out_transmittance, base + kOutOffset, 4ull * n, cudaMemcpyDeviceToHost, st));
  unsigned int status = 0;
  VP_CUDA(cudaMemcpyAsync(&status, base + sizeof(unsigned int), sizeof(status), cudaMemcpyDeviceToHost, st));
  VP_CUDA(cudaStreamSynchronize(st));
  if (status) return fail(VP_ERROR_DEVICE_STATUS, "transmittance kernel raised device status " + std::to_string(status));
  return VP_OK;
}
