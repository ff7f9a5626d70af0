// Device-wide primitives of the scene build and the wavefront re-sort, written for sm_100a:
//
//   radix_sort_pairs   stable LSD radix sort of (key, value) pairs, 8-bit digits, keys of 32 or
//                      64 bits (only the digits covering [0, end_bit) are sorted)
//   exclusive_scan     exclusive prefix sum of 32- or 64-bit counts
//
// Sort pass over one 8-bit digit (tiles of 2048 items, 256 threads, 8 warps):
//   k_rs_upsweep    per-tile digit histogram (shared-memory atomics) -> hist[digit * tiles + tile]
//   exclusive_scan  over hist: digit-major order gives every (digit, tile) its first output slot
//   k_rs_scatter    each warp ranks its 256 items in index order with __match_any_sync on the
//                   digit (lanes with equal digits see one another; the rank is the number of
//                   equal-digit lanes below plus the warp's running count of that digit), the
//                   warps' counts are scanned per digit in the block, and every item goes to
//                   hist[digit, tile] + (equal digits in earlier warps) + its warp rank.  Items
//                   keep their order within a digit, so the sort is stable.
// Scan of 32- or 64-bit counts (tiles of 4096 items, 1024 threads): per-tile sums, one block
// scans the tile sums, then each tile scans itself from its offset.
#include <algorithm>

#include "vp_internal.h"

namespace vp {
namespace {

constexpr int kRsThreads = 256;
constexpr int kRsItems = 8;                          // per thread
constexpr int kRsTile = kRsThreads * kRsItems;      // 2048
constexpr int kRsWarps = kRsThreads / 32;           // 8
constexpr int kRsWarpItems = kRsTile / kRsWarps;    // 256
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096

template <class K>
__device__ __forceinline__ uint32_t digit_of(K key, int shift) {
  return static_cast<uint32_t>(key >> shift) & 0xFFu;
}

template <class K>
__global__ void __launch_bounds__(kRsThreads) k_rs_upsweep(const K* __restrict__ keys, uint32_t n, int shift,
                                                            uint32_t tiles, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0u;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * kRsTile;
#pragma unroll
  for (int k = 0; k < kRsItems; ++k) {
    const size_t i = base + (size_t)k * kRsThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[digit_of(keys[i], shift)], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

template <class K>
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const K* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                                            K* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                            uint32_t n, int shift, uint32_t tiles,
                                                            const uint32_t* __restrict__ offsets) {
  __shared__ uint32_t wcnt[kRsWarps][256];  // per warp: items of each digit (then their exclusive scan over warps)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kRsWarps * 256; i += kRsThreads) (&wcnt[0][0])[i] = 0u;
  __syncthreads();
  const size_t wbase = (size_t)blockIdx.x * kRsTile + (size_t)warp * kRsWarpItems;
  const unsigned lt = (1u << lane) - 1u;
  K key[kRsItems];
  uint32_t val[kRsItems], rank[kRsItems], dig[kRsItems];
#pragma unroll
  for (int k = 0; k < kRsItems; ++k) {  // the warp's items in index order, 32 at a time
    const size_t i = wbase + (size_t)k * 32 + lane;
    const bool valid = i < n;
    key[k] = valid ? keys_in[i] : K(0);
    val[k] = valid ? vals_in[i] : 0u;
    const uint32_t d = valid ? digit_of(key[k], shift) : 256u;  // 256: no digit (past the end)
    dig[k] = d;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
    uint32_t before = 0u;
    if (valid) before = wcnt[warp][d];
    rank[k] = before + __popc(peers & lt);
    __syncwarp();
    // the highest lane of each digit group advances the warp's count of that digit
    if (valid && (peers >> lane) == 1u) wcnt[warp][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // per digit (thread d): exclusive scan of the warps' counts
  {
    const int d = threadIdx.x;  // 256 threads = 256 digits
    uint32_t run = 0u;
#pragma unroll
    for (int w = 0; w < kRsWarps; ++w) {
      const uint32_t c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kRsItems; ++k) {
    if (dig[k] >= 256u) continue;
    const uint32_t d = dig[k];
    const size_t pos = (size_t)offsets[(size_t)d * tiles + blockIdx.x] + wcnt[warp][d] + rank[k];
    keys_out[pos] = key[k];
    vals_out[pos] = val[k];
  }
}

// ---- exclusive scan of 32- or 64-bit counts ---------------------------------------------------
template <class T>
__device__ __forceinline__ T block_scan_excl(T v, T* warp_tot, T& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  T incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    T x = lane < nw ? warp_tot[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T t = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (lane >= o) x += t;
    }
    if (lane < nw) warp_tot[lane] = x;
  }
  __syncthreads();
  total = warp_tot[nw - 1];
  const T r = (w ? warp_tot[w - 1] : T(0)) + incl - v;
  __syncthreads();
  return r;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const T* __restrict__ in, size_t n,
                                                               T* __restrict__ partial) {
  __shared__ T wt[32];
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  T s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += in[base + k];
  T total;
  (void)block_scan_excl(s, wt, total);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// One block: exclusive scan of the m tile sums in place (each thread a contiguous chunk).
template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_partials(T* __restrict__ partial, uint32_t m) {
  __shared__ T wt[32];
  const uint32_t per = (m + kScanThreads - 1) / kScanThreads;
  const uint32_t b = threadIdx.x * per, e = min(m, b + per);
  T s = 0;
  for (uint32_t i = b; i < e; ++i) s += partial[i];
  T total;
  T run = block_scan_excl(s, wt, total);
  for (uint32_t i = b; i < e; ++i) {
    const T v = partial[i];
    partial[i] = run;
    run += v;
  }
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_down(const T* in, size_t n, const T* __restrict__ partial,
                                                             T* out) {  // in may equal out
  __shared__ T wt[32];
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  T v[kScanItems], s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : T(0);
    s += v[k];
  }
  T total;
  T run = block_scan_excl(s, wt, total) + partial[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

template <class T>
vp_status exclusive_scan_t(const T* in, T* out, size_t n, void* tmp, size_t tmp_bytes, cudaStream_t st,
                           uint32_t* launches);

size_t scan_tmp_bytes(size_t n) { return ((n + kScanTile - 1) / kScanTile) * sizeof(unsigned long long) + 256; }

template <class K>
size_t sort_tmp_bytes_t(size_t n) {
  const size_t tiles = (n + kRsTile - 1) / kRsTile;
  const size_t hist = 256 * tiles;
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  return up(n * sizeof(K)) + up(n * 4) + up(hist * 4) + up(scan_tmp_bytes(hist));
}

template <class K>
vp_status sort_pairs_t(K* keys, uint32_t* vals, uint32_t n, int end_bit, void* tmp, size_t tmp_bytes,
                       cudaStream_t st, uint32_t* launches) {
  if (n <= 1) return VP_OK;
  if (tmp_bytes < sort_tmp_bytes_t<K>(n)) return fail(VP_ERROR_INTERNAL, "radix sort scratch too small");
  const uint32_t tiles = (n + kRsTile - 1) / kRsTile;
  const size_t hist_n = (size_t)256 * tiles;
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  char* p = static_cast<char*>(tmp);
  K* keys_alt = reinterpret_cast<K*>(p);
  p += up((size_t)n * sizeof(K));
  uint32_t* vals_alt = reinterpret_cast<uint32_t*>(p);
  p += up((size_t)n * 4);
  uint32_t* hist = reinterpret_cast<uint32_t*>(p);
  p += up(hist_n * 4);
  void* scan_tmp = p;
  K *kin = keys, *kout = keys_alt;
  uint32_t *vin = vals, *vout = vals_alt;
  const int passes = (end_bit + 7) / 8;
  for (int pass = 0; pass < passes; ++pass) {
    const int shift = 8 * pass;
    k_rs_upsweep<K><<<tiles, kRsThreads, 0, st>>>(kin, n, shift, tiles, hist);
    VP_CUDA(cudaGetLastError());
    vp_status r = exclusive_scan_t<uint32_t>(hist, hist, hist_n, scan_tmp, scan_tmp_bytes(hist_n), st, launches);
    if (r) return r;
    k_rs_scatter<K><<<tiles, kRsThreads, 0, st>>>(kin, vin, kout, vout, n, shift, tiles, hist);
    VP_CUDA(cudaGetLastError());
    if (launches) *launches += 2;
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  if (kin != keys) {  // an odd number of passes left the result in the scratch buffers
    VP_CUDA(cudaMemcpyAsync(keys, kin, (size_t)n * sizeof(K), cudaMemcpyDeviceToDevice, st));
    VP_CUDA(cudaMemcpyAsync(vals, vin, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
  }
  return VP_OK;
}

template <class T>
vp_status exclusive_scan_t(const T* in, T* out, size_t n, void* tmp, size_t tmp_bytes, cudaStream_t st,
                           uint32_t* launches) {
  if (n == 0) return VP_OK;
  const size_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tmp_bytes < scan_tmp_bytes(n)) return fail(VP_ERROR_INTERNAL, "scan scratch too small");
  if (tiles > (size_t)0xFFFFFFFFu) return fail(VP_ERROR_LIMIT, "scan too large");
  T* partial = static_cast<T*>(tmp);
  k_scan_reduce<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, partial);
  k_scan_partials<T><<<1, kScanThreads, 0, st>>>(partial, (uint32_t)tiles);
  k_scan_down<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, partial, out);
  VP_CUDA(cudaGetLastError());
  if (launches) *launches += 3;
  return VP_OK;
}

}  // namespace

vp_status exclusive_scan(const uint32_t* in, uint32_t* out, size_t n, void* tmp, size_t tmp_bytes, cudaStream_t st,
                         uint32_t* launches) {
  return exclusive_scan_t<uint32_t>(in, out, n, tmp, tmp_bytes, st, launches);
}
vp_status exclusive_scan(const unsigned long long* in, unsigned long long* out, size_t n, void* tmp, size_t tmp_bytes,
                         cudaStream_t st, uint32_t* launches) {
  return exclusive_scan_t<unsigned long long>(in, out, n, tmp, tmp_bytes, st, launches);
}

size_t exclusive_scan_tmp_bytes(size_t n) { return scan_tmp_bytes(n); }
size_t radix_sort_tmp_bytes_u64(size_t n) { return sort_tmp_bytes_t<uint64_t>(n); }
size_t radix_sort_tmp_bytes_u32(size_t n) { return sort_tmp_bytes_t<uint32_t>(n); }

vp_status radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint32_t n, int end_bit, void* tmp, size_t tmp_bytes,
                           cudaStream_t st, uint32_t* launches) {
  return sort_pairs_t<uint64_t>(keys, vals, n, end_bit, tmp, tmp_bytes, st, launches);
}
vp_status radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, int end_bit, void* tmp, size_t tmp_bytes,
                           cudaStream_t st, uint32_t* launches) {
  return sort_pairs_t<uint32_t>(keys, vals, n, end_bit, tmp, tmp_bytes, st, launches);
}

}  // namespace vp
