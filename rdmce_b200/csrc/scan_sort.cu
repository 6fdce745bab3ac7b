// scan_sort.cu -- hand-written device-wide exclusive scan, LSD radix sort of
// 64-bit keys and max-reduction, plus the per-device scratch cache.
//
// These replace the host-side std::sort / std::unique / prefix loops of the
// reference loader (src/graph.cc:109-145, 216-236) with HBM-bound passes.
// Radix sort: 8-bit digits; per pass one histogram kernel (tile = 4096 keys),
// one scan over the digit-major (digit, tile) counts, and one stable scatter
// that ranks keys with __match_any_sync, reorders the tile in shared memory and
// writes runs of equal digits contiguously.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace mce {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *smem_warp, T *total) {
  // smem_warp: kScanThreads/32 entries
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    T w = lane < (kScanThreads / 32) ? smem_warp[lane] : T(0);
    T s = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(kFull, s, o);
      if (lane >= o) s += y;
    }
    if (lane < (kScanThreads / 32)) smem_warp[lane] = s - w;
    if (lane == (kScanThreads / 32) - 1) smem_warp[kScanThreads / 32] = s;
  }
  __syncthreads();
  T r = x - v + smem_warp[wid];
  *total = smem_warp[kScanThreads / 32];
  __syncthreads();
  return r;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_tile_sums(const T *in, uint64_t n, T *sums) {
  __shared__ T sw[kScanThreads / 32 + 1];
  uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  T s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    uint64_t idx = base + (uint64_t)i * kScanThreads + threadIdx.x;
    if (idx < n) s += in[idx];
  }
  T total;
  block_exclusive_scan<T>(s, sw, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_tile_scan(const T *in, T *out, uint64_t n, const T *offsets,
                                                            T *d_total) {
  __shared__ T tile[kScanTile];
  __shared__ T sw[kScanThreads / 32 + 1];
  uint64_t base = (uint64_t)blockIdx.x * kScanTile;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    uint64_t idx = base + (uint64_t)i * kScanThreads + threadIdx.x;
    tile[i * kScanThreads + threadIdx.x] = idx < n ? in[idx] : T(0);
  }
  __syncthreads();
  T v[kScanItems];
  T s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    v[i] = tile[threadIdx.x * kScanItems + i];
    s += v[i];
  }
  T total;
  T pre = block_exclusive_scan<T>(s, sw, &total);
  T off = offsets ? offsets[blockIdx.x] : T(0);
  T run = pre + off;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    tile[threadIdx.x * kScanItems + i] = run;
    run += v[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    uint64_t idx = base + (uint64_t)i * kScanThreads + threadIdx.x;
    if (idx < n) out[idx] = tile[i * kScanThreads + threadIdx.x];
  }
  if (d_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *d_total = off + total;
}

template <typename T>
mce_status scan_impl(const T *in, T *out, uint64_t n, T *d_total, cudaStream_t st) {
  if (n == 0) {
    if (d_total) MCE_CUDA_TRY(cudaMemsetAsync(d_total, 0, sizeof(T), st));
    return MCE_OK;
  }
  uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    k_tile_scan<T><<<1, kScanThreads, 0, st>>>(in, out, n, nullptr, d_total); note_launch();
    MCE_CUDA_TRY(cudaGetLastError());
    return MCE_OK;
  }
  T *sums = nullptr;
  MCE_CUDA_TRY(cudaMallocAsync(&sums, tiles * sizeof(T), st));
  k_tile_sums<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, sums); note_launch();
  mce_status s = scan_impl<T>(sums, sums, tiles, (T *)nullptr, st);
  if (s == MCE_OK) {
    k_tile_scan<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, sums, d_total); note_launch();
    if (cudaGetLastError() != cudaSuccess) s = MCE_ERR_CUDA;
  }
  cudaFreeAsync(sums, st);
  return s;
}

// ---------------------------------------------------------------- radix sort

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;  // keys per thread
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadix = 256;

__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint64_t *keys, uint64_t n, int shift,
                                                             uint32_t *hist, uint32_t ntiles) {
  __shared__ uint32_t cnt[kRadix];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll 4
  for (int i = 0; i < kSortItems; i++) {
    uint64_t idx = base + (uint64_t)i * kSortThreads + threadIdx.x;
    if (idx < n) atomicAdd(&cnt[(keys[idx] >> shift) & 0xFF], 1u);
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const uint64_t *in, uint64_t *out, uint64_t n,
                                                                int shift, const uint32_t *goff,
                                                                uint32_t ntiles) {
  __shared__ uint32_t wcnt[kSortWarps][kRadix];
  __shared__ uint32_t tile_off[kRadix];
  __shared__ uint32_t sw[kSortThreads / 32 + 1];
  __shared__ uint64_t stage[kSortTile];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < kSortWarps * kRadix; d += kSortThreads) (&wcnt[0][0])[d] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
  const uint64_t seg = base + (uint64_t)wid * (32 * kSortItems);
  uint64_t key[kSortItems];
  uint32_t pos[kSortItems];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    uint64_t idx = seg + (uint64_t)j * 32 + lane;
    bool valid = idx < n;
    key[j] = valid ? in[idx] : ~0ULL;
    uint32_t d = valid ? (uint32_t)((key[j] >> shift) & 0xFF) : kRadix;
    uint32_t peers = __match_any_sync(kFull, d);
    uint32_t b = valid ? wcnt[wid][d] : 0;
    __syncwarp();
    if (valid && (peers & lt) == 0) wcnt[wid][d] = b + __popc(peers);
    __syncwarp();
    pos[j] = b + __popc(peers & lt);
  }
  __syncthreads();
  // per digit: exclusive prefix over warps; tile-local digit offsets
  {
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
      uint32_t c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
    uint32_t total;
    uint32_t pre = block_exclusive_scan<uint32_t>(run, sw, &total);
    tile_off[d] = pre;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    uint64_t idx = seg + (uint64_t)j * 32 + lane;
    if (idx < n) {
      uint32_t d = (uint32_t)((key[j] >> shift) & 0xFF);
      stage[tile_off[d] + wcnt[wid][d] + pos[j]] = key[j];
    }
  }
  __syncthreads();
  const uint64_t rem_n = n - base;
  const uint32_t valid_n = rem_n < (uint64_t)kSortTile ? (uint32_t)rem_n : (uint32_t)kSortTile;
  for (uint32_t i = threadIdx.x; i < valid_n; i += kSortThreads) {
    uint64_t k = stage[i];
    uint32_t d = (uint32_t)((k >> shift) & 0xFF);
    out[(uint64_t)goff[(uint64_t)d * ntiles + blockIdx.x] + (i - tile_off[d])] = k;
  }
}

__global__ void k_reduce_max(const uint32_t *in, uint64_t n, uint32_t *out) {
  uint32_t m = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    m = max(m, in[i]);
  m = __reduce_max_sync(kFull, m);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

std::atomic<uint64_t> g_launches{0};
std::mutex g_default_mu[64];
Scratch g_default[64];

}  // namespace

mce_status scan_exclusive_u32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total, cudaStream_t st) {
  return scan_impl<uint32_t>(in, out, n, d_total, st);
}

mce_status scan_exclusive_u64(const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *d_total, cudaStream_t st) {
  return scan_impl<uint64_t>(in, out, n, d_total, st);
}

// ---- allocation-free exclusive scan (mce_csr_offsets_static) ----
// The partial sums of the three-pass scan live in this fixed array instead of
// a buffer allocated per call: level 1 holds one sum per 2048-element tile of
// the input (at most kStaticScanMaxN / 2048 = 32768), level 2 one sum per tile
// of level 1 (at most 16).  Every entry is written before it is read, so
// nothing in it has to start at zero.  All callers on a device share it:
// calls that overlap in time on one device race.
constexpr uint64_t kStaticScanMaxN = 1ULL << 26;
constexpr uint64_t kStaticL1 = kStaticScanMaxN / kScanTile;
constexpr uint64_t kStaticL2 = kStaticL1 / kScanTile;
static_assert(kStaticL1 == 32768 && kStaticL2 == 16, "static scan layout");
static __device__ __align__(256) uint32_t g_static_scan_sums[kStaticL1 + 256];

namespace {
std::mutex g_static_scan_mu;
uint32_t *g_static_scan_addr[64];  // device address of g_static_scan_sums, per device
}  // namespace

mce_status csr_offsets_static(int device, const uint32_t *deg, uint32_t *off, uint64_t n, cudaStream_t st) {
  if (n > kStaticScanMaxN) return MCE_ERR_TOO_LARGE;
  if (!off || (n && !deg) || device < 0 || device >= 64) return MCE_ERR_INVALID_ARG;
  uint32_t *sums = nullptr;
  {
    // first call on this device: look the array up with the device current
    std::lock_guard<std::mutex> lk(g_static_scan_mu);
    if (!g_static_scan_addr[device]) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scan_sums);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return cuda_status(e == cudaSuccess ? cudaErrorInvalidSymbol : e);
      }
      g_static_scan_addr[device] = (uint32_t *)p;
    }
    sums = g_static_scan_addr[device];
  }
  if (n == 0) {
    MCE_CUDA_TRY(cudaMemsetAsync(off, 0, sizeof(uint32_t), st));
    return MCE_OK;
  }
  const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    k_tile_scan<uint32_t><<<1, kScanThreads, 0, st>>>(deg, off, n, nullptr, off + n); note_launch();
    MCE_CUDA_TRY(cudaGetLastError());
    return MCE_OK;
  }
  uint32_t *l1 = sums, *l2 = sums + kStaticL1;
  k_tile_sums<uint32_t><<<(unsigned)tiles, kScanThreads, 0, st>>>(deg, n, l1); note_launch();
  const uint64_t tiles2 = (tiles + kScanTile - 1) / kScanTile;
  if (tiles2 == 1) {
    k_tile_scan<uint32_t><<<1, kScanThreads, 0, st>>>(l1, l1, tiles, nullptr, nullptr); note_launch();
  } else {
    k_tile_sums<uint32_t><<<(unsigned)tiles2, kScanThreads, 0, st>>>(l1, tiles, l2); note_launch();
    k_tile_scan<uint32_t><<<1, kScanThreads, 0, st>>>(l2, l2, tiles2, nullptr, nullptr); note_launch();
    k_tile_scan<uint32_t><<<(unsigned)tiles2, kScanThreads, 0, st>>>(l1, l1, tiles, l2, nullptr); note_launch();
  }
  k_tile_scan<uint32_t><<<(unsigned)tiles, kScanThreads, 0, st>>>(deg, off, n, l1, off + n); note_launch();
  MCE_CUDA_TRY(cudaGetLastError());
  return MCE_OK;
}

mce_status radix_sort_u64(uint64_t *keys, uint64_t *tmp, uint64_t n, int bits, cudaStream_t st) {
  if (n < 2 || bits <= 0) return MCE_OK;
  uint64_t ntiles64 = (n + kSortTile - 1) / kSortTile;
  if (ntiles64 * kRadix >= (1ULL << 32) || n >= (1ULL << 32) * 1ULL) return MCE_ERR_TOO_LARGE;
  uint32_t ntiles = (uint32_t)ntiles64;
  uint32_t *hist = nullptr;
  MCE_CUDA_TRY(cudaMallocAsync(&hist, (uint64_t)ntiles * kRadix * sizeof(uint32_t), st));
  uint64_t *src = keys, *dst = tmp;
  mce_status s = MCE_OK;
  for (int shift = 0; shift < bits && s == MCE_OK; shift += 8) {
    k_radix_hist<<<ntiles, kSortThreads, 0, st>>>(src, n, shift, hist, ntiles); note_launch();
    s = scan_exclusive_u32(hist, hist, (uint64_t)ntiles * kRadix, nullptr, st);
    if (s != MCE_OK) break;
    k_radix_scatter<<<ntiles, kSortThreads, 0, st>>>(src, dst, n, shift, hist, ntiles); note_launch();
    if (cudaGetLastError() != cudaSuccess) s = MCE_ERR_CUDA;
    uint64_t *t = src;
    src = dst;
    dst = t;
  }
  if (s == MCE_OK && src != keys) {
    if (cudaMemcpyAsync(keys, src, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      s = MCE_ERR_CUDA;
  }
  cudaFreeAsync(hist, st);
  return s;
}

mce_status reduce_max_u32(const uint32_t *in, uint64_t n, uint32_t *d_out, cudaStream_t st) {
  MCE_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(uint32_t), st));
  if (n == 0) return MCE_OK;
  k_reduce_max<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(in, n, d_out); note_launch();
  MCE_CUDA_TRY(cudaGetLastError());
  return MCE_OK;
}

void *Scratch::get(int purpose, size_t n, mce_status *st) {
  *st = MCE_OK;
  if (purpose < 0 || purpose >= kSlots) {
    *st = MCE_ERR_INTERNAL;
    return nullptr;
  }
  if (ptr[purpose] && bytes[purpose] >= n) return ptr[purpose];
  if (ptr[purpose]) {
    if (ordered) cudaFreeAsync(ptr[purpose], ordered);
    else cudaFree(ptr[purpose]);
  }
  ptr[purpose] = nullptr;
  bytes[purpose] = 0;
  const cudaError_t e = ordered ? cudaMallocAsync(&ptr[purpose], std::max<size_t>(n, 256), ordered)
                                : cudaMalloc(&ptr[purpose], std::max<size_t>(n, 256));
  if (e != cudaSuccess) {
    cudaGetLastError();
    ptr[purpose] = nullptr;
    *st = MCE_ERR_OUT_OF_MEMORY;
    return nullptr;
  }
  bytes[purpose] = std::max<size_t>(n, 256);
  return ptr[purpose];
}

void Scratch::release() {
  bool freed = false;
  for (int i = 0; i < kSlots; i++) {
    if (ptr[i]) {
      if (ordered) cudaFreeAsync(ptr[i], ordered);
      else cudaFree(ptr[i]);
      freed = true;
    }
    ptr[i] = nullptr;
    bytes[i] = 0;
  }
  if (ordered && freed) cudaStreamSynchronize(ordered);
}

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

Scratch *default_scratch(int device) {
  Scratch *s = &g_default[device & 63];
  s->device = device;
  return s;
}
void lock_default(int device) { g_default_mu[device & 63].lock(); }
void unlock_default(int device) { g_default_mu[device & 63].unlock(); }

}  // namespace mce

extern "C" uint64_t mce_launch_count(void) { return mce::g_launches.load(); }
