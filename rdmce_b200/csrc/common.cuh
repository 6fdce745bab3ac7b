// common.cuh -- device helpers, error plumbing and the device graph view.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "internal.h"

#define MCE_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return mce::cuda_status(_e);      \
  } while (0)

#define MCE_TRY(expr)                                        \
  do {                                                       \
    mce_status _s = (expr);                                  \
    if (_s != MCE_OK) return _s;                             \
  } while (0)

namespace mce {

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kNone = 0xffffffffu;
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ULL;

inline mce_status cuda_status(cudaError_t e) {
  if (e == cudaErrorMemoryAllocation) return MCE_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorInvalidDevice)
    return MCE_ERR_NO_DEVICE;
  return MCE_ERR_CUDA;
}

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
  uint64_t z = x + kGolden;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t clique_hash(uint64_t s1, uint64_t s2, uint64_t size) {
  uint64_t rot = (s2 << 31) | (s2 >> 33);
  return mix64(s1 ^ rot ^ (size << 56));
}

__device__ __forceinline__ uint32_t lane_id() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%laneid;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ uint64_t warp_or_u64(uint64_t v) {
  uint32_t lo = __reduce_or_sync(kFull, (uint32_t)v);
  uint32_t hi = __reduce_or_sync(kFull, (uint32_t)(v >> 32));
  return ((uint64_t)hi << 32) | lo;
}

// first index in sorted a[0..n) with a[i] >= key
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *a, uint32_t n, uint32_t key) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool contains_u32(const uint32_t *a, uint32_t n, uint32_t key) {
  uint32_t i = lower_bound_u32(a, n, key);
  return i < n && __ldg(a + i) == key;
}

// Device graph view: symmetric CSR, rows sorted ascending, uint32 offsets
// (2m < 2^32, as the reference's vid_t offsets, include/graph_gpu.cuh:5-15).
struct DevGraph {
  uint32_t n;
  uint64_t m;               // undirected edges = number of roots
  const uint32_t *off;      // n + 1
  const uint32_t *adj;      // 2m
  const uint32_t *labels;   // n: id -> original label
  const uint64_t *h1;       // n: mix64(label)
  const uint64_t *h2;       // n: mix64(label ^ golden)
  const uint32_t *root_v0;  // m: roots (v0 < v1) in CSR order
  const uint32_t *root_v1;  // m
  const uint32_t *slot;     // n or null: result slot of each vertex (batched graphs)
};

// ---- device-wide primitives (scan_sort.cu) ----
// exclusive scan of n uint32 (in != out allowed or in == out); total -> *d_total if non-null
mce_status scan_exclusive_u32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total,
                              cudaStream_t st);
mce_status scan_exclusive_u64(const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *d_total,
                              cudaStream_t st);
// LSD radix sort of n 64-bit keys over bits [0, bits); result in *keys (tmp = scratch of n)
mce_status radix_sort_u64(uint64_t *keys, uint64_t *tmp, uint64_t n, int bits, cudaStream_t st);
// allocation-free CSR offsets: off[0..n] = exclusive scan of deg, off[n] = total;
// partial sums in a fixed device array (n <= 2^26); calls on one device must not overlap
mce_status csr_offsets_static(int device, const uint32_t *deg, uint32_t *off, uint64_t n, cudaStream_t st);
// reduce max of n uint32
mce_status reduce_max_u32(const uint32_t *in, uint64_t n, uint32_t *d_out, cudaStream_t st);

// Device scratch owned by one solver context: buffers keyed by purpose, grown
// on demand and kept for reuse (the role of the reference's BufferManager,
// include/context_gpu.cuh:4-32, without its worst-case sizing).
struct Scratch {
  static constexpr int kSlots = 8;
  int device = 0;
  // set: buffers are allocated and freed stream-ordered on this stream (no
  // device-wide synchronisation when one grows), for an owner whose work
  // stays on that stream (a server dispatcher)
  cudaStream_t ordered = nullptr;
  void *ptr[kSlots] = {};
  size_t bytes[kSlots] = {};
  void *get(int purpose, size_t n, mce_status *st);
  void release();
  ~Scratch() { release(); }
};
// the default per-device context used by single-graph calls, and its lock
Scratch *default_scratch(int device);
void lock_default(int device);
void unlock_default(int device);

// every kernel launch of the engine is counted (mce_launch_count)
void note_launch();

inline uint32_t grid_for(uint64_t n, uint32_t block, uint32_t cap = 148u * 64u) {
  uint64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (uint32_t)g;
}

}  // namespace mce
