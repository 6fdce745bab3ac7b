// engine.h -- device-resident graph and the entry points of the GPU pipeline.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace mce {

// A degeneracy-ordered graph resident in HBM (the role of GraphGpu,
// include/graph_gpu.cuh:5-57, plus the root list and label hashes).
struct DeviceGraph {
  uint32_t n = 0;
  uint64_t m = 0;
  uint32_t *off = nullptr;      // n + 1
  uint32_t *adj = nullptr;      // 2m
  uint32_t *labels = nullptr;   // n
  uint64_t *h1 = nullptr;       // n
  uint64_t *h2 = nullptr;       // n
  uint32_t *root_v0 = nullptr;  // m
  uint32_t *root_v1 = nullptr;  // m
  uint32_t *slot = nullptr;     // n, batched mode only
  uint32_t max_degree = 0;
  uint32_t degeneracy = 0;
  cudaStream_t stream = nullptr;
};

mce_status build_from_pairs(const uint32_t *u_d, const uint32_t *v_d, uint64_t np, int order_kind,
                            uint64_t spin_limit, cudaStream_t st, DeviceGraph *g);
mce_status finish_graph(uint32_t n, uint64_t m, const uint32_t *eu, const uint32_t *ev, const uint32_t *deg,
                        const uint32_t *labels0, int order_kind, uint64_t spin_limit, cudaStream_t st,
                        DeviceGraph *g);
mce_status build_from_csr(uint64_t n, const uint32_t *off_d, const uint32_t *adj_d, const uint32_t *labels_d,
                          int already_ordered, int order_kind, uint32_t degeneracy_hint, uint64_t spin_limit,
                          cudaStream_t st, DeviceGraph *g);
mce_status csr_to_edges(uint64_t n, const uint32_t *off, const uint32_t *adj, uint64_t m, uint32_t *deg,
                        uint32_t **eu, uint32_t **ev, cudaStream_t st);
void free_graph(DeviceGraph *g);
// Per-graph figures of a union build (build_union).
struct UnionCounts {
  std::vector<uint32_t> nv;          // vertices
  std::vector<uint64_t> ne;          // undirected edges
  std::vector<uint32_t> max_degree;
  std::vector<uint32_t> degeneracy;
};
// Disjoint union of graphs whose COO pairs are in device memory, graph i
// being pairs [pair_offsets[i], pair_offsets[i + 1]) (host offsets): labels
// are shifted into disjoint ranges (ud, vd are modified), the union is built
// as one graph, and every vertex gets its graph as result slot and its own
// label back (batch.cu).
mce_status build_union(uint32_t *ud, uint32_t *vd, const uint64_t *pair_offsets, uint32_t n_graphs, int order,
                       uint64_t spin_limit, cudaStream_t st, DeviceGraph *g, UnionCounts *counts);
// first use of a device in this process: its default stream-ordered memory
// pool keeps freed memory for reuse instead of returning it at every sync
void keep_pool_memory(int device);
// COO text file -> pairs in device memory (ingest.cu), with the reference
// parser's semantics; *u_out / *v_out are cudaMallocAsync'ed on st (free with
// cudaFreeAsync)
mce_status parse_text_device(const char *path, cudaStream_t st, uint32_t **u_out, uint32_t **v_out,
                             uint64_t *n_out);

struct EnumConfig {
  uint32_t warps_per_block = 0;
  uint32_t blocks_per_sm = 0;
  uint32_t share_bound = 24;
  uint32_t reg_share_bound = 0;  // 0 = default
  int expand_r = 1;
  int sharing = 1;
  int stats = 0;  // count nodes and word-ops (a slower kernel instance)
  uint64_t root_begin = 0, root_end = 0;
  uint64_t spin_limit = 0;
  const uint64_t *root_list = nullptr;  // device: explicit root ids (per-root mode)
  uint64_t n_root_list = 0;
  unsigned long long *per_root_count = nullptr;     // device, n_root_list
  unsigned long long *per_root_checksum = nullptr;  // device, n_root_list
  uint32_t n_slots = 1;
  uint32_t hist_len = MCE_HIST_LEN;
  uint32_t max_blocks = 0;  // cap on the grid (0 = whole GPU); the server shares the GPU
  uint32_t slab_kib = 0;    // cap on the per-warp slab in KiB (0 = 4096)
  uint32_t heavy_warps = 0; // cap on the large-scratch pass's warps (0 = as memory allows)
};

// The enumeration settings a caller's options select (every entry point maps
// mce_options through this one function).
inline EnumConfig config_from_options(const mce_options &o) {
  EnumConfig c;
  c.warps_per_block = o.warps_per_block;
  c.blocks_per_sm = o.blocks_per_sm;
  c.share_bound = o.share_bound ? o.share_bound : 24;
  c.reg_share_bound = o.reg_share_bound;
  c.expand_r = o.expand_r;
  c.sharing = (o.flags & MCE_FLAG_NO_SHARING) ? 0 : 1;
  c.stats = (o.flags & MCE_FLAG_STATS) ? 1 : 0;
  c.root_begin = o.root_begin;
  c.root_end = o.root_end;
  c.spin_limit = o.spin_limit ? o.spin_limit : (1ULL << 34);
  c.slab_kib = o.slab_kib;
  c.heavy_warps = o.heavy_warps;
  return c;
}

// True when two configs would produce the same launch plan (a captured
// launch can be replayed for the second).
inline bool same_plan_settings(const EnumConfig &a, const EnumConfig &b) {
  return a.warps_per_block == b.warps_per_block && a.blocks_per_sm == b.blocks_per_sm &&
         a.share_bound == b.share_bound && a.reg_share_bound == b.reg_share_bound && a.expand_r == b.expand_r &&
         a.sharing == b.sharing && a.stats == b.stats && a.spin_limit == b.spin_limit && a.slab_kib == b.slab_kib &&
         a.heavy_warps == b.heavy_warps && a.hist_len == b.hist_len && a.n_slots == b.n_slots;
}

struct EnumStats {
  uint64_t roots = 0;
  uint64_t heavy_roots = 0;
  uint64_t shared_tasks = 0;
  uint64_t nodes = 0, word_ops = 0, build_bytes = 0;
  uint64_t cycles[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  uint64_t max_item[2] = {0, 0};  // longest root, longest task (cycles)
  uint32_t error = 0;
  float ms_setup = 0, ms_enum = 0;
  float ms_heavy = 0;  // device time of the deferred-root pass (part of ms_enum)
  uint64_t launches = 0;
  uint32_t blocks_per_sm = 0;  // resident 8-warp blocks per SM the solve ran with
};

// Per-slot results written by the enumeration kernels.
struct SlotResult {
  unsigned long long count;
  unsigned long long checksum;
  unsigned int max_size;
  unsigned int pad;
};

struct Scratch;

// Kernel parameters of one enumeration launch.
struct EnumParams {
  DevGraph g;
  uint64_t rb, re;                       // root range [rb, re) (range mode)
  const uint32_t *heavy_list;            // large-scratch pass: work indices of the deferred roots
  uint64_t n_heavy;                      // entries in heavy_list
  const uint64_t *root_list;             // list mode: root ids (else the range [rb, re))
  uint64_t n_list;                       // entries in root_list
  unsigned long long *next;              // claim counter
  char *slab;
  uint64_t slab_bytes;                   // per warp
  uint32_t *heavy_out;                   // deferred roots' work indices (heavy_cap entries)
  uint32_t heavy_cap;
  unsigned int *heavy_n;
  unsigned long long *heavy_need;
  int push_heavy;
  SlotResult *slots;
  unsigned long long *hist;
  uint32_t hist_len;
  unsigned long long *per_root_count;
  unsigned long long *per_root_checksum;
  int expand_r;
  int sharing;                           // root-down exposure through the task pool
  int stats;                             // count search-tree nodes and row word-ops
  uint32_t share_bound;                  // expose only levels with |P| >= this (general tier)
  uint32_t reg_share_bound;              // the same inside the register tiers
  uint32_t nwarps;
  uint64_t spin_limit;                   // bound on every device-side wait
  unsigned int *error;
  unsigned long long *stat_roots;
  unsigned long long *stat_tasks;
  unsigned long long *stat_nodes;
  unsigned long long *stat_wops;
  unsigned long long *stat_bbytes;       // algorithmic ego-network build bytes (stats mode)
  unsigned long long *stat_cycles;       // per phase: build, 64-bit tier, general tier, spawn, idle, queue, 32-bit tier
  unsigned long long *stat_max_item;     // [2]: longest root, longest task, in cycles
  unsigned int *active;                  // warps holding work
  // task pool: blocks of block_bytes, a free ring and a ready ring (one cell per block)
  char *pool;
  uint32_t block_bytes;
  uint32_t pool_mask;
  uint32_t *free_slot, *ready_slot;
  unsigned long long *free_seq, *ready_seq;
  unsigned long long *free_head, *free_tail, *ready_head, *ready_tail;
};


// A planned enumeration: scratch allocated, launch shape fixed.  Launch may be
// captured into a CUDA graph; finish reads the control words and runs the
// large-scratch pass for deferred roots.
struct EnumPlan {
  EnumParams params{};
  uint32_t blocks = 0, threads = 0;
  size_t smem = 0;
  uint64_t nwarps = 0, nwork = 0;
  bool fits_all = false;  // every root fits the normal slab: no deferred pass possible
  uint32_t pool_blocks = 0;
  uint32_t heavy_warps = 0;  // cap on the large-scratch pass (0 = as memory allows)
  int build = 4;             // which register-budget build of the kernel (enum_dispatch.cu)
  uint32_t sms = 0;          // multiprocessors of the device
  void *ctl = nullptr;
  Scratch *scr = nullptr;
};

// Enumerate; results accumulate into slots[n_slots] and hist[n_slots * hist_len]
// (device buffers the caller zeroed).
mce_status enumerate(const DeviceGraph &g, const EnumConfig &cfg, Scratch *scr, cudaStream_t st, SlotResult *slots,
                     unsigned long long *hist, EnumStats *stats);
mce_status enum_plan(const DeviceGraph &g, const EnumConfig &cfg, Scratch *scr, SlotResult *slots,
                     unsigned long long *hist, EnumPlan *plan);
mce_status enum_launch(const EnumPlan &plan, cudaStream_t st);
mce_status enum_finish(const EnumPlan &plan, cudaStream_t st, EnumStats *stats);
// the kernel build a blocks_per_sm setting runs (0 = the default build)
int enum_build_for(uint32_t blocks_per_sm);

// The autotuner's record for one workload: the enumeration time of each
// kernel build (3, 4, 5 blocks of 8 warps per SM), -1 while untried.  Solves
// of the workload try the builds in turn (4, 5, 3); later ones use the
// fastest.  A counting solve (MCE_FLAG_STATS, a slower kernel instance) is
// never a trial.
struct TuneRecord {
  float ms[3] = {-1.f, -1.f, -1.f};
};
// blocks per SM for the next solve; *mode = 1 for a trial, 2 for the choice
uint32_t tune_pick(const TuneRecord &t, bool counting, uint32_t *mode);
void tune_record(TuneRecord &t, uint32_t blocks_per_sm, float ms);
// the three register-budget builds of enum.cu (3, 4, 5 blocks of 8 warps per SM)
#define MCE_DECLARE_ENUM_BUILD(b)                                                                         \
  mce_status enum_plan_b##b(const DeviceGraph &g, const EnumConfig &cfg, Scratch *scr, SlotResult *slots, \
                            unsigned long long *hist, EnumPlan *plan);                                    \
  mce_status enum_launch_b##b(const EnumPlan &plan, cudaStream_t st);                                     \
  mce_status enum_finish_b##b(const EnumPlan &plan, cudaStream_t st, EnumStats *stats);
MCE_DECLARE_ENUM_BUILD(3)
MCE_DECLARE_ENUM_BUILD(4)
MCE_DECLARE_ENUM_BUILD(5)
#undef MCE_DECLARE_ENUM_BUILD
mce_status probe_int_peak(int device, double *word_ops_per_s);

}  // namespace mce
