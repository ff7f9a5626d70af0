// Serving runtime: continuous batching of render requests over resident scenes (the serving form;
// the reference renders one configured image per process and has no counterpart).
//
// A pool of path slots runs the wavefront stages of the offline engine (vp_wavefront.cu) with
// path regeneration: every iteration
//   advance  (1 block)           carry the survivors over; hand the free slots to the admitted
//                                requests that still have unstarted paths (the schedule)
//   regen    (thread per path)   new paths: owning request from the share prefix sums, camera
//                                ray, PCG32 stream, first free-flight key -- appended to the queue
//   extend   (warp per path)     free-flight argmin + scatter albedo on the path's own scene
//   shade    (thread per path)   phase / NEE / roulette with the request's own controls
//   shadow   (warp per query)    transmittance on the query's scene
//   gather   (thread per path)   radiance += weight x T; a finished path adds its sample to its
//                                request's pixel sum, counts itself done and frees its slot
// so paths of different requests, scenes, resolutions and sample counts share every launch, and
// a request admitted while others run starts as soon as free slots reach it.  How free slots are
// shared among the requests with unstarted paths is the server's schedule (admission order by
// default; equal shares; or fewest remaining first).  A request's paths start in pixel-major
// order.  Every per-path quantity comes from the request-table entry the path
// carries, so a path computes exactly what the offline engine computes for the same (scene,
// camera, params, pixel, sample).
//
// The host side admits from a FIFO when a table entry is free and the request's accumulator fits
// the memory budget and replays the iterations as one captured CUDA graph (two iterations: the
// path queues ping-pong).  The loop is pipelined so the GPU never waits for the host: a call
// queues step k (graphs, then an asynchronous copy of the per-request done counters and the
// status word to pinned memory) and only then waits for step k-1 and harvests it, while step k
// runs.  Harvesting completes the requests whose paths have all finished: the mean (sum / spp) is
// formed on the compute stream behind step k and, for host outputs, copied on a second stream
// into pinned staging; the request is delivered (its id becomes visible to vp_server_poll) once
// those copies have landed, by a later call.  Admission writes go to pinned staging and reach the
// device table by stream-ordered copies, so every iteration sees whole table entries; an entry's
// done counter is read only from steps queued after its admission.
#include <algorithm>
#include <cstring>
#include <deque>
#include <vector>

#include "vp_internal.h"
#include "vp_path.cuh"
#include "vp_traverse.cuh"

namespace vp {
namespace {

constexpr uint32_t kAlive = 1u << 18;
constexpr int kSrvHitCap = 64;        // extend hit buffer, as the offline wavefront's
constexpr uint32_t kMaxScenes = 64;
constexpr uint32_t kMaxRequests = 1024;  // the share computation is one block

struct SrvRequest {  // device request-table entry (all zero while unused)
  CameraView cam;
  ParamsView P;
  uint32_t scene;    // resident (scene, env) pair
  uint32_t n_pix;
  uint32_t cancelled;  // set by vp_server_cancel: start no further paths
  uint32_t pad;
  unsigned long long n_paths;  // width * height * spp
  unsigned long long seq;      // admission order
  float4* sum;       // per-pixel radiance sums
};

struct SrvCtl {  // device control block of the iteration
  uint32_t free_count;  // free path slots (top of the free stack)
  uint32_t regen_m;     // paths started by the current iteration
  uint32_t regen_from;  // free-stack index of the first slot they take
  uint32_t survivors;   // paths carried over from the previous iteration
  uint32_t ctr[8];      // [0] paths this iteration, [1] next, [2] shadow queries, [3..4] work heads
  unsigned long long total_started;  // paths the lane has started (the clock of SRPT aging)
};

struct SrvPaths {  // per path slot
  float4 *o4, *d4, *thr4, *rad4, *alb4;
  uint32_t* sg;  // the Gaussian of the scatter (scene order) or kNoGauss
  uint4* rng4;
  uint2* key2;
  uint32_t* meta;  // bounce | shadow count << 16 | alive << 18
  uint32_t *req, *pix;
  float4 *so4, *sd4, *sw4;  // 3 transmittance queries per slot
  uint32_t *qa, *qb, *qs, *free_stack;
};

__device__ __forceinline__ void srv_store(const SrvPaths& b, uint32_t p, const PathState& s) {
  b.o4[p] = make_float4(s.o.x, s.o.y, s.o.z, 0.f);
  b.d4[p] = make_float4(s.d.x, s.d.y, s.d.z, 0.f);
  b.thr4[p] = make_float4(s.thr.x, s.thr.y, s.thr.z, 0.f);
  b.rad4[p] = make_float4(s.rad.x, s.rad.y, s.rad.z, 0.f);
  b.rng4[p] = make_uint4((uint32_t)s.rng.state, (uint32_t)(s.rng.state >> 32), (uint32_t)s.rng.inc,
                         (uint32_t)(s.rng.inc >> 32));
}

__device__ __forceinline__ PathState srv_load(const SrvPaths& b, uint32_t p, uint32_t bounce) {
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

// Warp-aggregated queue append (all 32 lanes call it): this lane's first slot for n entries.
__device__ __forceinline__ uint32_t srv_reserve(uint32_t* counter, uint32_t n) {
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

__global__ void k_srv_init(SrvCtl* c, uint32_t* free_stack, uint32_t slots) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    uint32_t* w = reinterpret_cast<uint32_t*>(c);
    for (uint32_t k = 0; k < sizeof(SrvCtl) / 4u; ++k) w[k] = 0u;
    c->free_count = slots;
  }
  if (i < slots) free_stack[i] = slots - 1u - i;  // pops take the lowest slots first
}

// Exclusive block-wide prefix sum (blockDim.x <= 1024); also returns the total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_tot, uint32_t& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  uint32_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    uint32_t x = lane < nw ? warp_tot[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += t;
    }
    if (lane < nw) warp_tot[lane] = x;  // inclusive over warps
  }
  __syncthreads();
  total = warp_tot[nw - 1];
  const uint32_t before = w ? warp_tot[w - 1] : 0u;
  __syncthreads();
  return before + incl - v;
}

// One block of max_requests threads, thread e = request-table entry e, shares the free slots
// among the requests with unstarted paths by the server's schedule:
//   VP_SCHEDULE_FIFO  in admission order, each request taking all it still has;
//   VP_SCHEDULE_FAIR  an equal quota ceil(free / k) to each of the k requests (capped at what each
//                     still has), then what is left over in table order;
//   VP_SCHEDULE_SRPT  fewest unstarted paths first (ties in admission order), with a fraction
//                     (srpt_reserve, default half) of the free slots kept for the oldest request
//                     that still has unstarted paths; with srpt_aging > 0 the key is the unstarted
//                     paths minus srpt_aging x the paths the lane started since the request's first
//                     iteration here (age_base, set on that iteration).
// Writes the per-entry offsets of this iteration's new paths (alloc_off, size R + 1) and their
// first pixel-major path index (alloc_start).
__global__ void k_srv_advance(SrvCtl* c, const SrvRequest* __restrict__ table, unsigned long long* __restrict__ started,
                              unsigned long long* __restrict__ age_base, uint32_t* __restrict__ alloc_off,
                              unsigned long long* __restrict__ alloc_start, int schedule, float srpt_reserve,
                              float srpt_aging, uint32_t lane, uint32_t lanes) {
  __shared__ uint32_t warp_tot[32];
  __shared__ uint32_t s_free, s_surv;
  __shared__ unsigned long long s_key[kMaxRequests], s_seq[kMaxRequests];
  __shared__ uint32_t s_by_rank[kMaxRequests];
  __shared__ unsigned long long s_oldest;
  __shared__ uint32_t s_reserve;
  const uint32_t e = threadIdx.x, R = blockDim.x;
  if (e == 0) {
    s_free = c->free_count;
    s_surv = c->ctr[1];
  }
  __syncthreads();
  const uint32_t F = s_free;
  // table entry e belongs to lane e % lanes: only that lane's kernels read or write it
  const bool mine = (e % lanes) == lane;
  const unsigned long long st0 = mine ? started[e] : 0ull;
  const unsigned long long rem64 = (mine && !table[e].cancelled) ? table[e].n_paths - st0 : 0ull;
  const uint32_t rem = (uint32_t)min(rem64, (unsigned long long)F);
  uint32_t a = 0;
  if (schedule == VP_SCHEDULE_FAIR) {
    uint32_t k = 0;
    (void)block_exclusive_scan(rem ? 1u : 0u, warp_tot, k);
    const uint32_t q = k ? (F + k - 1u) / k : 0u;
    uint32_t tot1 = 0;
    uint32_t a1 = min(rem, q);
    const uint32_t off1 = block_exclusive_scan(a1, warp_tot, tot1);
    a1 = off1 >= F ? 0u : min(a1, F - off1);
    const uint32_t F2 = tot1 >= F ? 0u : F - tot1;
    uint32_t tot2 = 0;
    const uint32_t r2 = rem - a1;
    const uint32_t off2 = block_exclusive_scan(r2, warp_tot, tot2);
    a = a1 + (off2 >= F2 ? 0u : min(r2, F2 - off2));
  } else {
    // rank every entry by its key, then hand out the free slots in rank order
    const unsigned long long seq = mine ? table[e].seq : ~0ull;
    unsigned long long srpt_key = rem64;
    if (schedule == VP_SCHEDULE_SRPT && mine && srpt_aging > 0.0f) {
      const unsigned long long now = c->total_started;
      unsigned long long base = age_base[e];
      if (base == ~0ull) {  // the request's first iteration in this lane
        base = now;
        age_base[e] = now;
      }
      const unsigned long long credit = (unsigned long long)((double)srpt_aging * (double)(now - base));
      srpt_key = rem64 > credit ? rem64 - credit : 0ull;
    }
    const unsigned long long key = rem == 0 ? ~0ull : (schedule == VP_SCHEDULE_SRPT ? srpt_key : seq);
    s_key[e] = key;
    s_seq[e] = seq;
    // SRPT: a fraction of the free slots stays with the oldest request that has unstarted paths,
    // so a large request keeps progressing while smaller ones overtake it
    uint32_t reserve = 0, Fs = F;
    if (schedule == VP_SCHEDULE_SRPT) {
      if (e == 0) {
        s_oldest = ~0ull;
        s_reserve = 0u;
      }
      __syncthreads();
      if (rem) atomicMin(&s_oldest, seq);
      __syncthreads();
      if (rem && seq == s_oldest) {
        reserve = min(rem, (uint32_t)((float)F * srpt_reserve));
        s_reserve = reserve;
      }
      __syncthreads();
      Fs = F - s_reserve;
    }
    __syncthreads();
    uint32_t rank = 0;
    for (uint32_t j = 0; j < R; ++j) {
      const unsigned long long kj = s_key[j], sj = s_seq[j];
      rank += (kj < key || (kj == key && (sj < seq || (sj == seq && j < e)))) ? 1u : 0u;
    }
    const uint32_t rest = rem - reserve;
    s_by_rank[rank] = rest;
    __syncthreads();
    uint32_t tot = 0;
    const uint32_t before = block_exclusive_scan(s_by_rank[e], warp_tot, tot);  // thread e = rank e here
    __syncthreads();
    s_by_rank[e] = before;  // offset of rank e
    __syncthreads();
    const uint32_t off = s_by_rank[rank];
    a = reserve + (off >= Fs ? 0u : min(rest, Fs - off));
  }
  uint32_t m = 0;
  const uint32_t off = block_exclusive_scan(a, warp_tot, m);
  alloc_off[e] = off;
  alloc_start[e] = st0;
  if (mine) started[e] = st0 + a;
  if (e == R - 1) alloc_off[R] = m;
  if (e == 0) {
    c->survivors = s_surv;
    c->regen_m = m;
    c->regen_from = F - m;
    c->free_count = F - m;
    c->ctr[0] = s_surv + m;
    c->ctr[1] = c->ctr[2] = c->ctr[3] = c->ctr[4] = 0u;
    c->total_started += m;
  }
}

__global__ void k_srv_regen(const SrvCtl* __restrict__ c, const SrvRequest* __restrict__ table,
                            const uint32_t* __restrict__ alloc_off, const unsigned long long* __restrict__ alloc_start,
                            uint32_t n_entries, SrvPaths b, uint32_t* __restrict__ q) {
  const uint32_t m = c->regen_m;
  const uint32_t from = c->regen_from, surv = c->survivors;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const uint32_t slot = b.free_stack[from + i];
    uint32_t lo = 0, hi = n_entries;  // the entry e with alloc_off[e] <= i < alloc_off[e + 1]
    while (hi - lo > 1u) {
      const uint32_t mid = lo + (hi - lo) / 2u;
      if (alloc_off[mid] <= i) lo = mid;
      else hi = mid;
    }
    const uint32_t e = lo;
    const SrvRequest& r = table[e];
    const unsigned long long local = alloc_start[e] + (i - alloc_off[e]);
    const uint32_t spp = r.P.spp_total;
    const uint32_t pix = (uint32_t)(local / spp), s = (uint32_t)(local % spp);
    PathState st = start_path(r.cam, r.P, pix % r.P.width, pix / r.P.width, s);
    const uint64_t key = draw_bounce_key(st.rng);
    srv_store(b, slot, st);
    b.key2[slot] = make_uint2((uint32_t)key, (uint32_t)(key >> 32));
    b.meta[slot] = kAlive;
    b.req[slot] = e;
    b.pix[slot] = pix;
    q[surv + i] = slot;
  }
}

template <bool kAcc>
__global__ void __launch_bounds__(256, 4) k_srv_extend(const SceneView* __restrict__ scenes,
                                                       const SrvRequest* __restrict__ table, SrvPaths b,
                                                       const uint32_t* __restrict__ q, SrvCtl* c, uint32_t max_cap,
                                                       Counters* ctr) {
  extern __shared__ unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpSmem W = carve(smem + warp * warp_smem_bytes(max_cap, kSrvHitCap), max_cap, kSrvHitCap);
  const uint32_t n = c->ctr[0];
  uint32_t status = 0;
  WarpStats ws;
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(&c->ctr[3], 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= n) break;
    const uint32_t p = __ldg(q + item);
    const SceneView S = scenes[table[b.req[p]].scene];
    const float4 o = b.o4[p], d = b.d4[p];
    const uint2 k2 = b.key2[p];
    const uint32_t bounce = b.meta[p] & 0xFFFFu;
    const float3 of = f3(o.x, o.y, o.z), df = f3(d.x, d.y, d.z);
    float tstar = kInf;
    ScatterAlbedo sa;
    sa.valid = false;
    if (!(bounce == 0 && S.albedo_all_zero))
      tstar = warp_ray_query<kAcc, kArgmin>(S, W, of, df, ((uint64_t)k2.y << 32) | k2.x, status, ws, false, &sa);
    float3 albedo = f3(0.f, 0.f, 0.f);
    if (tstar < kInf) {
      uint32_t ov = sa.overlap;
      albedo = sa.valid ? sa.albedo : warp_albedo<kAcc>(S, W, fma3(tstar, df, of), ov, status, ws, false);
    }
    if (lane == 0) {
      b.alb4[p] = make_float4(albedo.x, albedo.y, albedo.z, tstar);
      b.sg[p] = tstar < kInf ? sa.gauss : kNoGauss;
    }
    if (status) break;
  }
  if (lane == 0 && status) atomicOr(&ctr->status, status);
}

// As the offline engine's shade stage, the shadow rays' seed chords are evaluated here, one
// thread per ray; a ray whose seed chord alone is opaque gets T = 0 and skips the shadow queue.
__global__ void __launch_bounds__(256) k_srv_shade(const SceneView* __restrict__ scenes,
                                                   const EnvView* __restrict__ envs,
                                                   const SrvRequest* __restrict__ table, SrvPaths b,
                                                   const uint32_t* __restrict__ q, SrvCtl* c,
                                                   uint32_t* __restrict__ qnext) {
  const uint32_t n = c->ctr[0];
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  const uint32_t wid = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  for (uint32_t base = wid * 32u; base < n; base += warps * 32u) {  // warp-uniform
    const uint32_t i = base + lane;
    uint32_t p = 0;
    int ns = 0;
    unsigned queued = 0u;
    bool alive = false;
    if (i < n) {
      p = q[i];
      const SrvRequest& r = table[b.req[p]];
      PathState s = srv_load(b, p, b.meta[p] & 0xFFFFu);
      const float4 a = b.alb4[p];
      ShadowSet sh;
      alive = shade_bounce(envs[r.scene], r.P, s, a.w < kInf, a.w, f3(a.x, a.y, a.z), sh, b.sg[p]);
      ns = sh.n;
      for (int k = 0; k < sh.n; ++k) {
        float seed_tau = -1.0f;  // no seed
        if (sh.seed[k] != kNoGauss)
          seed_tau = r.P.accurate ? seed_chord_tau<true>(scenes[r.scene], sh.seed[k], sh.o[k], sh.d[k])
                                  : seed_chord_tau<false>(scenes[r.scene], sh.seed[k], sh.o[k], sh.d[k]);
        const bool opaque_k = seed_tau >= kMaxOpticalDepth;
        b.so4[3u * p + k] = make_float4(sh.o[k].x, sh.o[k].y, sh.o[k].z, opaque_k ? 0.0f : seed_tau);
        b.sd4[3u * p + k] = make_float4(sh.d[k].x, sh.d[k].y, sh.d[k].z, __uint_as_float(sh.seed[k]));
        b.sw4[3u * p + k] = make_float4(sh.w[k].x, sh.w[k].y, sh.w[k].z, 0.f);
        if (!opaque_k) queued |= 1u << k;
      }
      if (alive) {
        const uint64_t key = draw_bounce_key(s.rng);
        b.key2[p] = make_uint2((uint32_t)key, (uint32_t)(key >> 32));
      }
      srv_store(b, p, s);
      b.meta[p] = (s.bounce & 0xFFFFu) | ((uint32_t)sh.n << 16) | (alive ? kAlive : 0u);
    }
    uint32_t slot = srv_reserve(&c->ctr[2], (uint32_t)__popc(queued));
    for (int k = 0; k < ns; ++k)
      if (queued & (1u << k)) b.qs[slot++] = 3u * p + k;
    const uint32_t qslot = srv_reserve(&c->ctr[1], alive ? 1u : 0u);
    if (alive) qnext[qslot] = p;
  }
}

template <bool kAcc>
__global__ void __launch_bounds__(256, 4) k_srv_shadow(const SceneView* __restrict__ scenes,
                                                       const SrvRequest* __restrict__ table, SrvPaths b, SrvCtl* c,
                                                       uint32_t max_cap, Counters* ctr) {
  extern __shared__ unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpSmem W = carve(smem + warp * warp_smem_bytes(max_cap, 32), max_cap, 32);
  const uint32_t n = c->ctr[2];
  uint32_t status = 0;
  WarpStats ws;
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(&c->ctr[4], 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= n) break;
    const uint32_t qslot = __ldg(b.qs + item);
    const SceneView S = scenes[table[b.req[qslot / 3u]].scene];
    const float4 o = b.so4[qslot], d = b.sd4[qslot];
    const float tau = warp_ray_query<kAcc, kTau>(S, W, f3(o.x, o.y, o.z), f3(d.x, d.y, d.z), 0ull, status, ws, false,
                                                 nullptr, __float_as_uint(d.w), o.w);
    if (lane == 0) b.so4[qslot].w = tau >= kMaxOpticalDepth ? 0.0f : expf(-tau);
    if (status) break;
  }
  if (lane == 0 && status) atomicOr(&ctr->status, status);
}

__global__ void __launch_bounds__(256) k_srv_gather(const SrvRequest* __restrict__ table, SrvPaths b,
                                                    const uint32_t* __restrict__ q, SrvCtl* c,
                                                    unsigned long long* __restrict__ done) {
  const uint32_t n = c->ctr[0];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t p = q[i];
    const uint32_t m = b.meta[p];
    const int ns = (int)((m >> 16) & 3u);
    const float4 r4 = b.rad4[p];
    float3 rad = f3(r4.x, r4.y, r4.z);
    for (int k = 0; k < ns; ++k) {
      const float4 w = b.sw4[3u * p + k];
      rad = add(rad, mul(f3(w.x, w.y, w.z), b.so4[3u * p + k].w));
    }
    if (m & kAlive) {
      b.rad4[p] = make_float4(rad.x, rad.y, rad.z, 0.f);
    } else {
      const uint32_t e = b.req[p];
      const SrvRequest& r = table[e];
      const float3 L = finalize_sample(r.P, rad);
      atomicAdd(r.sum + b.pix[p], make_float4(L.x, L.y, L.z, 0.f));
      atomicAdd(done + e, 1ull);
      b.free_stack[atomicAdd(&c->free_count, 1u)] = p;
    }
  }
}

__global__ void k_srv_finish(const float4* __restrict__ sum, uint32_t n_pix, float inv_spp, float4* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_pix) return;
  const float4 s = sum[i];
  out[i] = make_float4(s.x * inv_spp, s.y * inv_spp, s.z * inv_spp, 1.0f);
}

template <class K>
int srv_blocks(K kernel, int threads, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem) != cudaSuccess) b = 1;
  return b < 1 ? 1 : b;
}

template <class T>
void srv_carve(char*& cur, T*& out, size_t count) {
  out = reinterpret_cast<T*>(cur);
  cur += (count * sizeof(T) + 255) & ~size_t(255);
}

constexpr size_t kSlotBytes = 5 * 16 + 4 + 16 + 8 + 4 + 4 + 4 + 3 * 48 + 4 * 2 + 3 * 4 + 4;

}  // namespace
}  // namespace vp

using namespace vp;

struct vp_server {
  vp_context* ctx = nullptr;
  vp_server_config cfg{};
  bool accurate = false;
  std::vector<vp_scene*> scenes;
  std::vector<vp_env*> envs;
  uint32_t max_cap = 0;         // largest depth-first stack over the scenes (transmittance)
  uint32_t max_argmin_cap = 0;  // largest argmin stack over the scenes
  // device
  SceneView* d_scenes = nullptr;
  EnvView* d_envs = nullptr;
  SrvRequest* d_table = nullptr;
  unsigned long long* d_done = nullptr;
  unsigned long long* d_started = nullptr;      // paths started per table entry
  unsigned long long* d_age_base = nullptr;     // SRPT aging: the lane's started-path clock at the
                                                // entry's first iteration (~0 until then)
  // pinned staging of the table entries (each reaches the device by a stream-ordered copy)
  SrvRequest* h_table = nullptr;
  int ext_blocks = 0, shd_blocks = 0, thr_blocks = 0;
  size_t smem_ext = 0, smem_shd = 0;
  cudaStream_t copy_stream = nullptr;  // output copies of completed requests
  // A lane: one pool of path slots with its own control block, queues, stream and graph.  Table
  // entry e belongs to lane e % lanes, so a lane's kernels read and write only entries that its
  // own stream updates.  Pipelining: two step slots per lane, each with its own events and pinned
  // copies of the done counters and the status word.
  struct Lane {
    cudaStream_t st = nullptr;
    bool own_stream = false;
    uint32_t slots = 0;
    SrvCtl* d_ctl = nullptr;
    uint32_t* d_alloc_off = nullptr;              // this iteration's new paths per entry (prefix, R + 1)
    unsigned long long* d_alloc_start = nullptr;  // their first path index per entry
    void* path_mem = nullptr;
    SrvPaths paths{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaEvent_t ev_beg[2] = {}, ev_end[2] = {}, ev_step[2] = {};
    unsigned long long* h_done_slot[2] = {};
    unsigned long long* h_started_slot[2] = {};  // paths started per entry, read with the done counts
    unsigned int* h_status = nullptr;  // [2]
    uint64_t slot_step[2] = {};
    std::deque<int> inflight;  // step slots queued and not yet harvested (oldest first)
    uint64_t step_no = 0;      // steps queued so far
    uint32_t entries = 0;      // table entries in use
    unsigned long long load = 0;  // paths of its entries in use (the admission's balance)
    double busy_ms = 0.0;      // device time of its steps
  };
  std::vector<Lane> lanes;
  // host bookkeeping
  struct Active {
    bool used = false;
    uint64_t id = 0;
    unsigned long long n_paths = 0;
    uint32_t n_pix = 0, spp = 0;
    float* out = nullptr;
    int32_t memory = 0;
    float4* sum = nullptr;
    size_t bytes = 0;
    uint64_t admit_step = 0;  // the first step of its lane queued after the admission
    uint32_t lane = 0;
    bool cancelled = false;
    uint64_t cancel_step = 0;  // the first step of its lane that sees the cancel flag
  };
  std::vector<Active> active;
  // completed requests whose outputs are still being formed / copied
  struct Delivery {
    uint64_t id;
    unsigned long long paths;
    float* host_out;  // host output: copied from the pinned staging buffer at delivery
    void* pinned;
    size_t bytes, pinned_bytes;
    size_t held;  // the request's share of the memory budget, released at delivery
  };
  struct OutBatch {
    cudaEvent_t ev;
    std::vector<Delivery> items;
  };
  std::deque<OutBatch> outs;
  std::vector<cudaEvent_t> spare_events;
  std::vector<std::pair<size_t, void*>> pinned_free;  // reusable pinned staging buffers
  std::vector<void*> pinned_all;
  uint32_t n_entries = 0;  // table entries in use (admitted, not harvested)
  struct Pending {
    uint64_t id;
    vp_request r;
  };
  std::deque<Pending> pending;
  std::vector<uint64_t> done_ids;
  uint64_t next_id = 0, admitted = 0, completed = 0, paths_completed = 0, iterations = 0;
  uint64_t cancelled = 0, alloc_failures = 0;
  uint32_t inject_alloc_failures = 0;  // host fault injection: accumulator allocations left to fail
  uint32_t n_active = 0;
  size_t bytes_fixed = 0, bytes_active = 0;
};

namespace {

size_t request_bytes(const vp_request& r) {
  size_t b = (size_t)r.params.width * r.params.height * 16u;
  if (r.memory == VP_MEMORY_HOST) b += (size_t)r.params.width * r.params.height * 16u;  // output staging
  return b;
}

void srv_free(vp_server* s) {
  if (!s) return;
  cudaSetDevice(s->ctx->device);
  for (auto& L : s->lanes)
    if (L.st) cudaStreamSynchronize(L.st);
  if (s->ctx->stream) cudaStreamSynchronize(s->ctx->stream);
  if (s->copy_stream) {
    cudaStreamSynchronize(s->copy_stream);
    cudaStreamDestroy(s->copy_stream);
  }
  for (auto& L : s->lanes) {
    for (int k = 0; k < 2; ++k) {
      if (L.ev_beg[k]) cudaEventDestroy(L.ev_beg[k]);
      if (L.ev_end[k]) cudaEventDestroy(L.ev_end[k]);
      if (L.ev_step[k]) cudaEventDestroy(L.ev_step[k]);
    }
    if (L.h_done_slot[0]) cudaFreeHost(L.h_done_slot[0]);
    if (L.h_started_slot[0]) cudaFreeHost(L.h_started_slot[0]);
    if (L.h_status) cudaFreeHost(L.h_status);
    if (L.graph_exec) cudaGraphExecDestroy(L.graph_exec);
    if (L.graph) cudaGraphDestroy(L.graph);
    cudaFree(L.d_ctl);
    cudaFree(L.d_alloc_off);
    cudaFree(L.d_alloc_start);
    cudaFree(L.path_mem);
    if (L.own_stream && L.st) cudaStreamDestroy(L.st);
  }
  for (auto& b : s->outs) cudaEventDestroy(b.ev);
  for (cudaEvent_t e : s->spare_events) cudaEventDestroy(e);
  for (void* p : s->pinned_all) cudaFreeHost(p);
  for (auto& a : s->active)
    if (a.sum) cudaFree(a.sum);
  cudaFree(s->d_scenes);
  cudaFree(s->d_envs);
  cudaFree(s->d_table);
  cudaFree(s->d_done);
  cudaFree(s->d_started);
  cudaFree(s->d_age_base);
  cudaFreeHost(s->h_table);
  delete s;
}

// One wavefront iteration of lane l with the queues in the given roles.
vp_status enqueue_iteration(vp_server* s, uint32_t l, bool even) {
  vp_server::Lane& L = s->lanes[l];
  cudaStream_t st = L.st;
  const uint32_t R = s->cfg.max_requests, nl = (uint32_t)s->lanes.size();
  uint32_t* qcur = even ? L.paths.qa : L.paths.qb;
  uint32_t* qnext = even ? L.paths.qb : L.paths.qa;
  Counters* ctr = s->ctx->counters;
  k_srv_advance<<<1, R, 0, st>>>(L.d_ctl, s->d_table, s->d_started, s->d_age_base, L.d_alloc_off,
                                 L.d_alloc_start, s->cfg.schedule, s->cfg.srpt_reserve, s->cfg.srpt_aging, l, nl);
  k_srv_regen<<<s->thr_blocks, 256, 0, st>>>(L.d_ctl, s->d_table, L.d_alloc_off, L.d_alloc_start, R, L.paths, qcur);
  if (s->accurate)
    k_srv_extend<true><<<s->ext_blocks, 256, s->smem_ext, st>>>(s->d_scenes, s->d_table, L.paths, qcur, L.d_ctl,
                                                               s->max_argmin_cap, ctr);
  else
    k_srv_extend<false><<<s->ext_blocks, 256, s->smem_ext, st>>>(s->d_scenes, s->d_table, L.paths, qcur, L.d_ctl,
                                                                s->max_argmin_cap, ctr);
  k_srv_shade<<<s->thr_blocks, 256, 0, st>>>(s->d_scenes, s->d_envs, s->d_table, L.paths, qcur, L.d_ctl, qnext);
  if (s->accurate)
    k_srv_shadow<true><<<s->shd_blocks, 256, s->smem_shd, st>>>(s->d_scenes, s->d_table, L.paths, L.d_ctl,
                                                               s->max_cap, ctr);
  else
    k_srv_shadow<false><<<s->shd_blocks, 256, s->smem_shd, st>>>(s->d_scenes, s->d_table, L.paths, L.d_ctl,
                                                                s->max_cap, ctr);
  k_srv_gather<<<s->thr_blocks, 256, 0, st>>>(s->d_table, L.paths, qcur, L.d_ctl, s->d_done);
  VP_CUDA(cudaGetLastError());
  return VP_OK;
}

// Kernel configuration and (once) the graph of two iterations; needs every scene added.
vp_status prepare_launch(vp_server* s) {
  if (s->thr_blocks) return VP_OK;
  vp_context* ctx = s->ctx;
  s->max_cap = 2;
  s->max_argmin_cap = 2;
  for (vp_scene* sc : s->scenes) {
    s->max_cap = std::max(s->max_cap, sc->view.stack_cap);
    s->max_argmin_cap = std::max(s->max_argmin_cap, sc->view.argmin_cap);
  }
  s->smem_ext = (size_t)8 * warp_smem_bytes(s->max_argmin_cap, kSrvHitCap);
  s->smem_shd = (size_t)8 * warp_smem_bytes(s->max_cap, 32);
  if (s->smem_ext > 200 * 1024) return fail(VP_ERROR_LIMIT, "BVH too deep for the shared-memory stack");
  auto ext = s->accurate ? k_srv_extend<true> : k_srv_extend<false>;
  auto shd = s->accurate ? k_srv_shadow<true> : k_srv_shadow<false>;
  if (s->smem_ext > 48 * 1024)
    VP_CUDA(cudaFuncSetAttribute(ext, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem_ext));
  if (s->smem_shd > 48 * 1024)
    VP_CUDA(cudaFuncSetAttribute(shd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem_shd));
  s->ext_blocks = ctx->sm_count * srv_blocks(ext, 256, s->smem_ext);
  s->shd_blocks = ctx->sm_count * srv_blocks(shd, 256, s->smem_shd);
  s->thr_blocks = ctx->sm_count * 8;
  if (s->cfg.use_graph) {
    for (uint32_t l = 0; l < (uint32_t)s->lanes.size(); ++l) {
      vp_server::Lane& L = s->lanes[l];
      VP_CUDA(cudaStreamBeginCapture(L.st, cudaStreamCaptureModeThreadLocal));
      vp_status r1 = enqueue_iteration(s, l, true);
      vp_status r2 = r1 == VP_OK ? enqueue_iteration(s, l, false) : r1;
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(L.st, &g);
      if (r2 != VP_OK) {
        if (g) cudaGraphDestroy(g);
        return r2;
      }
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
      L.graph = g;
      VP_CUDA(cudaGraphInstantiate(&L.graph_exec, g, 0));
    }
  }
  return VP_OK;
}

vp_status admit(vp_server* s) {
  const uint32_t R = s->cfg.max_requests, nl = (uint32_t)s->lanes.size();
  while (!s->pending.empty() && s->n_entries < R) {
    const vp_request& rq = s->pending.front().r;
    const size_t need = request_bytes(rq);
    if (s->cfg.memory_budget_bytes && s->bytes_fixed + s->bytes_active + need > s->cfg.memory_budget_bytes) break;
    // the least-loaded lane with a free entry (entry e belongs to lane e % nl)
    uint32_t lane = nl;
    for (uint32_t l = 0; l < nl; ++l)
      if (s->lanes[l].entries < (R - l + nl - 1) / nl && (lane == nl || s->lanes[l].load < s->lanes[lane].load))
        lane = l;
    if (lane == nl) break;
    uint32_t e = lane;
    while (s->active[e].used) e += nl;
    vp_server::Lane& L = s->lanes[lane];
    cudaStream_t st = L.st;
    vp_server::Active& a = s->active[e];
    const uint32_t n_pix = rq.params.width * rq.params.height;
    float4* sum = nullptr;
    cudaError_t ae = cudaErrorMemoryAllocation;
    if (s->inject_alloc_failures)
      s->inject_alloc_failures -= 1;
    else
      ae = cudaMallocAsync(reinterpret_cast<void**>(&sum), 16ull * n_pix, st);
    if (ae != cudaSuccess) {
      if (ae != cudaErrorMemoryAllocation) return cuda_fail(ae, "cudaMallocAsync");
      (void)cudaGetLastError();  // not sticky: the request stays queued
      s->alloc_failures += 1;
      if (s->n_active == 0)  // nothing admitted would release memory
        return fail(VP_ERROR_OUT_OF_MEMORY, "request accumulator: device out of memory with no request admitted");
      break;  // wait for the admitted requests to release theirs
    }
    VP_CUDA(cudaMemsetAsync(sum, 0, 16ull * n_pix, st));
    VP_CUDA(cudaMemsetAsync(s->d_done + e, 0, sizeof(unsigned long long), st));
    VP_CUDA(cudaMemsetAsync(s->d_started + e, 0, sizeof(unsigned long long), st));
    VP_CUDA(cudaMemsetAsync(s->d_age_base + e, 0xFF, sizeof(unsigned long long), st));
    SrvRequest& t = s->h_table[e];
    std::memset(&t, 0, sizeof(t));
    build_camera(rq.camera, rq.params.width, rq.params.height, t.cam);
    t.P = make_params(rq.params, s->scenes[rq.scene_id]);
    t.P.accurate = s->accurate ? 1 : 0;
    t.P.measure = 0;
    t.scene = rq.scene_id;
    t.n_pix = n_pix;
    t.n_paths = (unsigned long long)n_pix * rq.params.spp;
    t.seq = s->admitted;
    t.sum = sum;
    VP_CUDA(cudaMemcpyAsync(s->d_table + e, &t, sizeof(t), cudaMemcpyHostToDevice, st));
    a.used = true;
    a.id = s->pending.front().id;
    a.n_paths = t.n_paths;
    a.n_pix = n_pix;
    a.spp = rq.params.spp;
    a.out = rq.out_rgba;
    a.memory = rq.memory;
    a.sum = sum;
    a.bytes = need;
    a.admit_step = L.step_no;
    a.lane = lane;
    L.entries += 1;
    L.load += t.n_paths;
    s->bytes_active += need;
    s->n_active += 1;
    s->n_entries += 1;
    s->admitted += 1;
    s->pending.pop_front();
  }
  return VP_OK;
}

void* pinned_acquire(vp_server* s, size_t bytes, size_t* got) {
  size_t best = (size_t)-1;
  for (size_t i = 0; i < s->pinned_free.size(); ++i)
    if (s->pinned_free[i].first >= bytes && (best == (size_t)-1 || s->pinned_free[i].first < s->pinned_free[best].first))
      best = i;
  if (best != (size_t)-1) {
    auto pr = s->pinned_free[best];
    s->pinned_free.erase(s->pinned_free.begin() + best);
    *got = pr.first;
    return pr.second;
  }
  const size_t sz = std::max<size_t>((bytes + (1u << 20) - 1) & ~size_t((1u << 20) - 1), 1u << 20);
  void* p = nullptr;
  if (cudaMallocHost(&p, sz) != cudaSuccess) return nullptr;
  s->pinned_all.push_back(p);
  *got = sz;
  return p;
}

// Completed requests of one harvested step: the mean is formed on the compute stream (behind the
// step now running), host outputs are copied on the copy stream into pinned staging, and one event
// on the copy stream marks the batch ready for delivery.
vp_status harvest(vp_server* s, uint32_t l, int slot) {
  vp_server::Lane& L = s->lanes[l];
  cudaStream_t st = L.st, cs = s->copy_stream;
  if (L.h_status[slot])
    return fail(VP_ERROR_DEVICE_STATUS, "a serving kernel raised device status " + std::to_string(L.h_status[slot]));
  float ms = 0.f;
  VP_CUDA(cudaEventElapsedTime(&ms, L.ev_beg[slot], L.ev_end[slot]));
  L.busy_ms += ms;
  const uint32_t R = s->cfg.max_requests, nl = (uint32_t)s->lanes.size();
  const unsigned long long* done = L.h_done_slot[slot];
  const unsigned long long* started = L.h_started_slot[slot];
  vp_server::OutBatch batch{};
  struct Copy {
    float4* tmp;
    void* pinned;
    size_t bytes;
  };
  std::vector<Copy> copies;
  for (uint32_t e = l; e < R; e += nl) {  // the lane's entries
    vp_server::Active& a = s->active[e];
    if (!a.used || a.admit_step > L.slot_step[slot]) continue;
    if (a.cancelled) {
      // released once a step that saw the flag ends with every started path finished
      if (L.slot_step[slot] < a.cancel_step || done[e] < started[e]) continue;
      VP_CUDA(cudaFreeAsync(a.sum, st));
      s->bytes_active -= a.bytes;
      s->n_active -= 1;
      L.entries -= 1;
      L.load -= a.n_paths;
      a = vp_server::Active{};
      s->n_entries -= 1;
      continue;
    }
    if (done[e] < a.n_paths) continue;
    const float inv = 1.0f / (float)a.spp;
    const unsigned nb = (a.n_pix + 255u) / 256u;
    vp_server::Delivery d{a.id, a.n_paths, nullptr, nullptr, 16ull * a.n_pix, 0, a.bytes};
    if (a.memory == VP_MEMORY_DEVICE) {
      k_srv_finish<<<nb, 256, 0, st>>>(a.sum, a.n_pix, inv, reinterpret_cast<float4*>(a.out));
      VP_CUDA(cudaGetLastError());
    } else {
      float4* tmp = nullptr;
      VP_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&tmp), 16ull * a.n_pix, st));
      k_srv_finish<<<nb, 256, 0, st>>>(a.sum, a.n_pix, inv, tmp);
      VP_CUDA(cudaGetLastError());
      d.pinned = pinned_acquire(s, d.bytes, &d.pinned_bytes);
      if (!d.pinned) return fail(VP_ERROR_OUT_OF_MEMORY, "pinned staging for a request's output");
      d.host_out = a.out;
      copies.push_back({tmp, d.pinned, d.bytes});
    }
    VP_CUDA(cudaFreeAsync(a.sum, st));
    batch.items.push_back(d);
    L.entries -= 1;
    L.load -= a.n_paths;
    a = vp_server::Active{};
    s->n_entries -= 1;
  }
  if (batch.items.empty()) return VP_OK;
  if (s->spare_events.empty()) {
    cudaEvent_t ev;
    VP_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    s->spare_events.push_back(ev);
  }
  batch.ev = s->spare_events.back();
  s->spare_events.pop_back();
  VP_CUDA(cudaEventRecord(batch.ev, st));  // the finish kernels
  VP_CUDA(cudaStreamWaitEvent(cs, batch.ev, 0));
  for (const Copy& c : copies) {
    VP_CUDA(cudaMemcpyAsync(c.pinned, c.tmp, c.bytes, cudaMemcpyDeviceToHost, cs));
    VP_CUDA(cudaFreeAsync(c.tmp, cs));
  }
  VP_CUDA(cudaEventRecord(batch.ev, cs));  // finish kernels and copies
  s->outs.push_back(std::move(batch));
  return VP_OK;
}

// Hands over the output batches whose copies have landed (all of them, waiting, when `wait`).
vp_status deliver(vp_server* s, bool wait, uint32_t* n_done) {
  while (!s->outs.empty()) {
    vp_server::OutBatch& b = s->outs.front();
    if (wait) {
      VP_CUDA(cudaEventSynchronize(b.ev));
    } else {
      const cudaError_t q = cudaEventQuery(b.ev);
      if (q == cudaErrorNotReady) break;
      if (q != cudaSuccess) return cuda_fail(q, "vp_server output copy");
    }
    for (const vp_server::Delivery& d : b.items) {
      if (d.host_out) {
        std::memcpy(d.host_out, d.pinned, d.bytes);
        s->pinned_free.push_back({d.pinned_bytes, d.pinned});
      }
      s->done_ids.push_back(d.id);
      s->bytes_active -= d.held;  // its accumulator and output staging are released by now
      s->paths_completed += d.paths;
      s->completed += 1;
      s->n_active -= 1;
      *n_done += 1;
    }
    s->spare_events.push_back(b.ev);
    s->outs.pop_front();
  }
  return VP_OK;
}

}  // namespace

extern "C" {

vp_status vp_server_create(vp_context* ctx, const vp_server_config* config, vp_server** out) {
  if (!ctx || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  VP_CUDA(cudaSetDevice(ctx->device));
  auto* s = new (std::nothrow) vp_server();
  if (!s) return fail(VP_ERROR_OUT_OF_MEMORY, "host allocation failed");
  s->ctx = ctx;
  if (config) s->cfg = *config;
  vp_server_config& c = s->cfg;
  if (c.path_slots == 0) c.path_slots = 1u << 18;
  if (c.max_requests == 0) c.max_requests = 256;
  c.max_requests = (c.max_requests + 31u) & ~31u;  // the share computation runs one block of warps
  if (c.max_requests > kMaxRequests) {
    srv_free(s);
    return fail(VP_ERROR_LIMIT, "max_requests above 1024");
  }
  if (c.iterations_per_step == 0) c.iterations_per_step = 4;
  if (!(c.srpt_reserve > 0.0f)) c.srpt_reserve = 0.5f;
  if (c.srpt_reserve > 1.0f) {
    srv_free(s);
    return fail(VP_ERROR_INVALID_ARGUMENT, "srpt_reserve above 1");
  }
  c.iterations_per_step = (c.iterations_per_step + 1u) & ~1u;
  if (!(c.srpt_aging >= 0.0f) || c.srpt_aging > 1e6f) {
    srv_free(s);
    return fail(VP_ERROR_INVALID_ARGUMENT, "srpt_aging must be in [0, 1e6]");
  }
  if (c.path_slots > (1u << 28)) {
    srv_free(s);
    return fail(VP_ERROR_LIMIT, "path_slots above 2^28");
  }
  s->accurate = c.precision == VP_PRECISION_ACCURATE;
  if (c.schedule < VP_SCHEDULE_FIFO || c.schedule > VP_SCHEDULE_SRPT) {
    srv_free(s);
    return fail(VP_ERROR_INVALID_ARGUMENT, "unknown schedule");
  }
  if (c.lanes == 0) c.lanes = 1;
  if (c.lanes > 4) {
    srv_free(s);
    return fail(VP_ERROR_LIMIT, "lanes above 4");
  }
  const uint32_t R = c.max_requests, NL = c.lanes;
  const uint32_t P = ((c.path_slots / NL) + 255u) & ~255u;  // slots per lane
  s->active.resize(R);
  s->lanes.resize(NL);
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  chk(cudaMalloc(&s->d_scenes, kMaxScenes * sizeof(SceneView)));
  chk(cudaMalloc(&s->d_envs, kMaxScenes * sizeof(EnvView)));
  chk(cudaMalloc(&s->d_table, R * sizeof(SrvRequest)));
  chk(cudaMalloc(&s->d_done, R * sizeof(unsigned long long)));
  chk(cudaMalloc(&s->d_started, R * 8ull));
  chk(cudaMalloc(&s->d_age_base, R * 8ull));
  chk(cudaMallocHost(&s->h_table, R * sizeof(SrvRequest)));
  chk(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
  const size_t slot_bytes = (size_t)P * kSlotBytes + 32 * 256;
  for (uint32_t l = 0; l < NL; ++l) {
    vp_server::Lane& L = s->lanes[l];
    L.slots = P;
    if (l == 0) {
      L.st = ctx->stream;
    } else {
      chk(cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking));
      L.own_stream = e == cudaSuccess;
    }
    chk(cudaMalloc(&L.d_alloc_off, (R + 1ull) * 4ull));
    chk(cudaMalloc(&L.d_alloc_start, R * 8ull));
    chk(cudaMalloc(&L.d_ctl, sizeof(SrvCtl)));
    for (int k = 0; k < 2; ++k) {
      chk(cudaEventCreate(&L.ev_beg[k]));
      chk(cudaEventCreate(&L.ev_end[k]));
      chk(cudaEventCreateWithFlags(&L.ev_step[k], cudaEventDisableTiming));
    }
    chk(cudaMallocHost(&L.h_done_slot[0], 2ull * R * sizeof(unsigned long long)));
    chk(cudaMallocHost(&L.h_started_slot[0], 2ull * R * sizeof(unsigned long long)));
    chk(cudaMallocHost(&L.h_status, 2 * sizeof(unsigned int)));
    chk(cudaMalloc(&L.path_mem, slot_bytes));
    if (e == cudaSuccess) {
      L.h_done_slot[1] = L.h_done_slot[0] + R;
      L.h_started_slot[1] = L.h_started_slot[0] + R;
    }
  }
  if (e != cudaSuccess) {
    srv_free(s);
    return cuda_fail(e, "vp_server_create");
  }
  for (uint32_t l = 0; l < NL; ++l) {
  vp_server::Lane& L = s->lanes[l];
  char* cur = static_cast<char*>(L.path_mem);
  SrvPaths& b = L.paths;
  srv_carve(cur, b.o4, P);
  srv_carve(cur, b.d4, P);
  srv_carve(cur, b.thr4, P);
  srv_carve(cur, b.rad4, P);
  srv_carve(cur, b.alb4, P);
  srv_carve(cur, b.sg, P);
  srv_carve(cur, b.rng4, P);
  srv_carve(cur, b.key2, P);
  srv_carve(cur, b.meta, P);
  srv_carve(cur, b.req, P);
  srv_carve(cur, b.pix, P);
  srv_carve(cur, b.so4, 3ull * P);
  srv_carve(cur, b.sd4, 3ull * P);
  srv_carve(cur, b.sw4, 3ull * P);
  srv_carve(cur, b.qa, P);
  srv_carve(cur, b.qb, P);
  srv_carve(cur, b.qs, 3ull * P);
  srv_carve(cur, b.free_stack, P);
  k_srv_init<<<(P + 255) / 256, 256, 0, ctx->stream>>>(L.d_ctl, b.free_stack, P);
  }
  s->bytes_fixed = NL * slot_bytes + R * (sizeof(SrvRequest) + 36ull);
  cudaStream_t st = ctx->stream;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemsetAsync(s->d_done, 0, R * sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->d_started, 0, R * sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->d_age_base, 0xFF, R * sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->d_table, 0, R * sizeof(SrvRequest), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->counters, 0, sizeof(Counters), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    srv_free(s);
    return cuda_fail(e, "vp_server_create");
  }
  if (c.memory_budget_bytes && s->bytes_fixed > c.memory_budget_bytes) {
    srv_free(s);
    return fail(VP_ERROR_LIMIT, "memory budget below the server's path slots");
  }
  *out = s;
  return VP_OK;
}

vp_status vp_server_add_scene(vp_server* s, vp_scene* scene, vp_env* env, uint32_t* scene_id) {
  if (!s || !scene || !env || !scene_id) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (scene->ctx != s->ctx || env->ctx != s->ctx) return fail(VP_ERROR_INVALID_ARGUMENT, "objects belong to different contexts");
  if (s->thr_blocks) return fail(VP_ERROR_INVALID_ARGUMENT, "scenes must be added before the first vp_server_step");
  if (s->scenes.size() >= kMaxScenes) return fail(VP_ERROR_LIMIT, "too many resident scenes");
  const size_t need = scene->info.device_bytes;
  if (s->cfg.memory_budget_bytes && s->bytes_fixed + need > s->cfg.memory_budget_bytes)
    return fail(VP_ERROR_LIMIT, "scene does not fit the memory budget");
  const uint32_t id = (uint32_t)s->scenes.size();
  VP_CUDA(cudaSetDevice(s->ctx->device));
  VP_CUDA(cudaMemcpy(s->d_scenes + id, &scene->view, sizeof(SceneView), cudaMemcpyHostToDevice));
  VP_CUDA(cudaMemcpy(s->d_envs + id, &env->view, sizeof(EnvView), cudaMemcpyHostToDevice));
  s->scenes.push_back(scene);
  s->envs.push_back(env);
  s->bytes_fixed += need;
  *scene_id = id;
  return VP_OK;
}

vp_status vp_server_submit(vp_server* s, const vp_request* r, uint64_t* request_id) {
  if (!s || !r) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (r->scene_id >= s->scenes.size()) return fail(VP_ERROR_INVALID_ARGUMENT, "unknown scene_id");
  if (!r->out_rgba) return fail(VP_ERROR_INVALID_ARGUMENT, "out_rgba is NULL");
  if (r->memory != VP_MEMORY_HOST && r->memory != VP_MEMORY_DEVICE) return fail(VP_ERROR_INVALID_ARGUMENT, "bad memory kind");
  vp_status st;
  if ((st = check_params(&r->params))) return st;
  if (r->params.max_bounces == 0) return fail(VP_ERROR_INVALID_ARGUMENT, "max_bounces must be positive for a served request");
  if (r->params.adaptive_threshold > 0.0f)  // a request's paths are summed, not kept per pixel per batch
    return fail(VP_ERROR_INVALID_ARGUMENT, "adaptive sampling is not available for a served request");
  if (s->cfg.memory_budget_bytes && s->bytes_fixed + request_bytes(*r) > s->cfg.memory_budget_bytes)
    return fail(VP_ERROR_LIMIT, "request does not fit the memory budget");
  const uint64_t id = s->next_id++;
  s->pending.push_back({id, *r});
  if (request_id) *request_id = id;
  return VP_OK;
}

vp_status vp_server_step(vp_server* s, uint32_t* completed) {
  if (!s) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (completed) *completed = 0;
  if (s->scenes.empty()) return fail(VP_ERROR_INVALID_ARGUMENT, "no resident scene");
  VP_CUDA(cudaSetDevice(s->ctx->device));
  vp_status r;
  uint32_t nd = 0;
  if ((r = prepare_launch(s))) return r;
  if ((r = deliver(s, false, &nd))) return r;
  if ((r = admit(s))) return r;
  const uint32_t nl = (uint32_t)s->lanes.size();
  bool launched[4] = {false, false, false, false};
  for (uint32_t l = 0; l < nl; ++l) {  // queue step k of every lane with work
    vp_server::Lane& L = s->lanes[l];
    if (L.entries == 0) continue;
    cudaStream_t st = L.st;
    const int slot = L.inflight.empty() ? 0 : (L.inflight.back() ^ 1);
    VP_CUDA(cudaEventRecord(L.ev_beg[slot], st));
    for (uint32_t k = 0; k < s->cfg.iterations_per_step; k += 2) {
      if (L.graph_exec) {
        VP_CUDA(cudaGraphLaunch(L.graph_exec, st));
      } else {
        if ((r = enqueue_iteration(s, l, true))) return r;
        if ((r = enqueue_iteration(s, l, false))) return r;
      }
    }
    VP_CUDA(cudaEventRecord(L.ev_end[slot], st));
    VP_CUDA(cudaMemcpyAsync(L.h_done_slot[slot], s->d_done, s->cfg.max_requests * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, st));
    VP_CUDA(cudaMemcpyAsync(L.h_started_slot[slot], s->d_started, s->cfg.max_requests * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, st));
    VP_CUDA(cudaMemcpyAsync(L.h_status + slot, &s->ctx->counters->status, sizeof(unsigned int),
                            cudaMemcpyDeviceToHost, st));
    VP_CUDA(cudaEventRecord(L.ev_step[slot], st));
    L.slot_step[slot] = L.step_no++;
    s->iterations += s->cfg.iterations_per_step;
    L.inflight.push_back(slot);
    launched[l] = true;
  }
  // harvest each lane's step k-1 while its step k runs (every queued step of a lane that queued
  // nothing new)
  bool any_inflight = false;
  for (uint32_t l = 0; l < nl; ++l) {
    vp_server::Lane& L = s->lanes[l];
    while (L.inflight.size() > (launched[l] ? 1u : 0u)) {
      const int slot = L.inflight.front();
      L.inflight.pop_front();
      VP_CUDA(cudaEventSynchronize(L.ev_step[slot]));
      if ((r = harvest(s, l, slot))) return r;
    }
    any_inflight = any_inflight || !L.inflight.empty();
  }
  // with no step left on the GPU, wait for the outputs still being copied
  if ((r = deliver(s, !any_inflight && s->n_entries == 0, &nd))) return r;
  if (completed) *completed = nd;
  return VP_OK;
}

vp_status vp_server_cancel(vp_server* s, uint64_t request_id) {
  if (!s) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  for (auto it = s->pending.begin(); it != s->pending.end(); ++it)
    if (it->id == request_id) {
      s->pending.erase(it);
      s->cancelled += 1;
      return VP_OK;
    }
  for (uint32_t e = 0; e < s->cfg.max_requests; ++e) {
    vp_server::Active& a = s->active[e];
    if (!a.used || a.id != request_id) continue;
    if (a.cancelled) return fail(VP_ERROR_INVALID_ARGUMENT, "request already cancelled");
    VP_CUDA(cudaSetDevice(s->ctx->device));
    vp_server::Lane& L = s->lanes[a.lane];
    // stream-ordered: the lane's next queued step is the first whose advance sees the flag
    s->h_table[e].cancelled = 1u;
    VP_CUDA(cudaMemcpyAsync(&s->d_table[e].cancelled, &s->h_table[e].cancelled, sizeof(uint32_t),
                            cudaMemcpyHostToDevice, L.st));
    a.cancelled = true;
    a.cancel_step = L.step_no;
    s->cancelled += 1;
    return VP_OK;
  }
  return fail(VP_ERROR_INVALID_ARGUMENT, "unknown request id, or the request has already finished");
}

vp_status vp_server_inject_alloc_failures(vp_server* s, uint32_t n) {
  if (!s) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  s->inject_alloc_failures = n;
  return VP_OK;
}

vp_status vp_server_poll(vp_server* s, uint64_t* ids, uint32_t cap, uint32_t* n) {
  if (!s || !n || (cap && !ids)) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  const uint32_t k = (uint32_t)std::min<size_t>(cap, s->done_ids.size());
  for (uint32_t i = 0; i < k; ++i) ids[i] = s->done_ids[i];
  s->done_ids.erase(s->done_ids.begin(), s->done_ids.begin() + k);
  *n = k;
  return VP_OK;
}

vp_status vp_server_get_stats(vp_server* s, vp_server_stats* out) {
  if (!s || !out) return fail(VP_ERROR_INVALID_ARGUMENT, "NULL argument");
  std::memset(out, 0, sizeof(*out));
  out->submitted = s->next_id;
  out->admitted = s->admitted;
  out->completed = s->completed;
  out->paths_completed = s->paths_completed;
  out->iterations = s->iterations;
  out->active = s->n_active;
  out->pending = (uint32_t)s->pending.size();
  out->bytes_in_use = s->bytes_fixed + s->bytes_active;
  out->cancelled = s->cancelled;
  out->alloc_failures = s->alloc_failures;
  for (const auto& L : s->lanes) out->device_ms = std::max(out->device_ms, L.busy_ms);  // the busiest lane
  return VP_OK;
}

vp_status vp_server_destroy(vp_server* s) {
  srv_free(s);
  return VP_OK;
}

}  // extern "C"
