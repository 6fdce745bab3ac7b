// batch.cu -- many independent graphs enumerated in one persistent launch.
//
// No reference counterpart (the reference solves one graph per process).  The
// graphs are shifted into disjoint label ranges and built as one union graph
// on the GPU; maximal cliques of a disjoint union are exactly the cliques of
// its parts, so one root space and one launch cover every graph.  Each vertex
// carries a result slot (its graph), labels are mapped back to the graph's own
// labels for the checksum, and the launch -- memsets, the persistent kernel and
// the copy of the per-graph results -- is captured once into a CUDA graph and
// replayed on later solves.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"

struct mce_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  mce::DeviceGraph g;
  uint32_t n_graphs = 0;
  std::vector<uint32_t> nv;
  std::vector<uint64_t> ne;
  mce::Scratch scr;
  // captured launch
  cudaGraphExec_t exec = nullptr;
  mce::EnumConfig exec_cfg;  // the settings the captured launch was planned with
  mce::TuneRecord tune;      // the autotuner's timings of the kernel builds for this batch
  uint32_t tune_mode = 0;    // how the captured launch's blocks per SM were chosen
  mce::EnumPlan plan;
  mce::SlotResult *slots_h = nullptr;  // pinned
  unsigned long long *hist_h = nullptr;
  size_t hist_h_len = 0;
};

namespace mce {
namespace {

__global__ void k_graph_max_label(const uint32_t *u, const uint32_t *v, const uint64_t *poff, uint32_t ng,
                                  uint32_t *gmax) {
  // one block per graph
  for (uint32_t gi = blockIdx.x; gi < ng; gi += gridDim.x) {
    uint32_t m = 0;
    for (uint64_t i = poff[gi] + threadIdx.x; i < poff[gi + 1]; i += blockDim.x) m = max(m, max(u[i], v[i]));
    m = __reduce_max_sync(kFull, m);
    if ((threadIdx.x & 31) == 0) atomicMax(&gmax[gi], m);
  }
}

__global__ void k_plus_one(uint32_t *a, uint32_t n, const uint64_t *poff) {
  // graphs without pairs take no label range
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    a[i] = poff[i + 1] > poff[i] ? a[i] + 1 : 0;
}

__global__ void k_shift_pairs(uint32_t *u, uint32_t *v, const uint64_t *poff, uint32_t ng, const uint32_t *base) {
  for (uint32_t gi = blockIdx.x; gi < ng; gi += gridDim.x) {
    const uint32_t b = base[gi];
    for (uint64_t i = poff[gi] + threadIdx.x; i < poff[gi + 1]; i += blockDim.x) {
      u[i] += b;
      v[i] += b;
    }
  }
}

// union label -> (graph, own label); recompute the label hashes
__global__ void k_local_labels(uint32_t *labels, uint64_t *h1, uint64_t *h2, uint32_t *slot, uint32_t n,
                               const uint32_t *base, uint32_t ng) {
  for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    const uint32_t l = labels[x];
    uint32_t lo = 0, hi = ng;  // last gi with base[gi] <= l
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) >> 1;
      if (base[mid] <= l) lo = mid;
      else hi = mid;
    }
    // several empty graphs can share a base; take the last non-empty one
    const uint32_t own = l - base[lo];
    labels[x] = own;
    slot[x] = lo;
    h1[x] = mix64((uint64_t)own);
    h2[x] = mix64((uint64_t)own ^ kGolden);
  }
}

__global__ void k_count_per_graph(const uint32_t *slot, uint32_t n, const uint32_t *root_v0, uint64_t m,
                                  unsigned int *nv, unsigned long long *ne) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n || i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (i < n) atomicAdd(&nv[slot[i]], 1u);
    if (i < m) atomicAdd(&ne[slot[root_v0[i]]], 1ULL);
  }
}

// Per graph: largest degree and largest number of later neighbours.  In the
// union's degeneracy order each graph's vertices keep its own peel order (the
// graphs never interact), so the largest later-neighbour count of a graph's
// vertices is that graph's degeneracy.
__global__ void k_graph_degrees(const uint32_t *off, const uint32_t *adj, uint32_t n, const uint32_t *slot,
                                unsigned int *maxdeg, unsigned int *degen) {
  for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    const uint32_t b = off[x], e = off[x + 1];
    uint32_t lo = b, hi = e;  // first neighbour above x
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (adj[mid] <= x) lo = mid + 1;
      else hi = mid;
    }
    atomicMax(&maxdeg[slot[x]], e - b);
    atomicMax(&degen[slot[x]], e - lo);
  }
}

}  // namespace

mce_status build_union(uint32_t *ud, uint32_t *vd, const uint64_t *pair_offsets, uint32_t n_graphs, int order,
                       uint64_t spin_limit, cudaStream_t st, DeviceGraph *g, UnionCounts *counts) {
  const uint64_t np = pair_offsets[n_graphs];
  uint32_t *gmax = nullptr, *base = nullptr;
  uint64_t *pd = nullptr;
  struct Free {
    cudaStream_t st;
    std::vector<void *> p;
    ~Free() {
      for (void *q : p)
        if (q) cudaFreeAsync(q, st);
    }
  } fr{st, {}};
  if (cudaMallocAsync(&pd, (n_graphs + 1) * 8ULL, st) != cudaSuccess ||
      cudaMallocAsync(&gmax, (n_graphs + 1) * 4ULL, st) != cudaSuccess ||
      cudaMallocAsync(&base, (n_graphs + 1) * 4ULL, st) != cudaSuccess)
    return MCE_ERR_OUT_OF_MEMORY;
  fr.p = {pd, gmax, base};
  MCE_CUDA_TRY(cudaMemcpyAsync(pd, pair_offsets, (n_graphs + 1) * 8ULL, cudaMemcpyHostToDevice, st));
  MCE_CUDA_TRY(cudaMemsetAsync(gmax, 0, (n_graphs + 1) * 4ULL, st));
  const uint32_t gb = std::min<uint32_t>(n_graphs, 148 * 32);
  k_graph_max_label<<<gb, 256, 0, st>>>(ud, vd, pd, n_graphs, gmax); note_launch();
  k_plus_one<<<grid_for(n_graphs, 256), 256, 0, st>>>(gmax, n_graphs, pd); note_launch();
  // label_base = exclusive prefix of (max label + 1); the total must fit in 31 bits
  MCE_TRY(scan_exclusive_u32(gmax, base, n_graphs, base + n_graphs, st));
  {
    std::vector<uint32_t> gm(n_graphs);
    MCE_CUDA_TRY(cudaMemcpyAsync(gm.data(), gmax, n_graphs * 4ULL, cudaMemcpyDeviceToHost, st));
    MCE_CUDA_TRY(cudaStreamSynchronize(st));
    uint64_t sum = 0;
    for (uint32_t x : gm) sum += x;
    if (sum >= (1ULL << 31)) return MCE_ERR_TOO_LARGE;
  }
  k_shift_pairs<<<gb, 256, 0, st>>>(ud, vd, pd, n_graphs, base); note_launch();
  MCE_TRY(build_from_pairs(ud, vd, np, order, spin_limit, st, g));
  unsigned int *nvd = nullptr, *mdd = nullptr, *dgd = nullptr;
  unsigned long long *ned = nullptr;
  if (cudaMallocAsync(&g->slot, std::max<uint32_t>(g->n, 1) * 4ULL, st) != cudaSuccess ||
      cudaMallocAsync(&nvd, n_graphs * 4ULL, st) != cudaSuccess ||
      cudaMallocAsync(&mdd, n_graphs * 4ULL, st) != cudaSuccess ||
      cudaMallocAsync(&dgd, n_graphs * 4ULL, st) != cudaSuccess ||
      cudaMallocAsync(&ned, n_graphs * 8ULL, st) != cudaSuccess)
    return MCE_ERR_OUT_OF_MEMORY;
  fr.p.push_back(nvd);
  fr.p.push_back(mdd);
  fr.p.push_back(dgd);
  fr.p.push_back(ned);
  cudaMemsetAsync(nvd, 0, n_graphs * 4ULL, st);
  cudaMemsetAsync(mdd, 0, n_graphs * 4ULL, st);
  cudaMemsetAsync(dgd, 0, n_graphs * 4ULL, st);
  cudaMemsetAsync(ned, 0, n_graphs * 8ULL, st);
  k_local_labels<<<grid_for(g->n, 256), 256, 0, st>>>(g->labels, g->h1, g->h2, g->slot, g->n, base, n_graphs);
  note_launch();
  k_count_per_graph<<<grid_for(std::max<uint64_t>(g->n, g->m), 256), 256, 0, st>>>(g->slot, g->n, g->root_v0, g->m,
                                                                                  nvd, ned);
  note_launch();
  k_graph_degrees<<<grid_for(g->n, 256), 256, 0, st>>>(g->off, g->adj, g->n, g->slot, mdd, dgd);
  note_launch();
  counts->nv.resize(n_graphs);
  counts->ne.resize(n_graphs);
  counts->max_degree.resize(n_graphs);
  counts->degeneracy.resize(n_graphs);
  MCE_CUDA_TRY(cudaMemcpyAsync(counts->nv.data(), nvd, n_graphs * 4ULL, cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaMemcpyAsync(counts->ne.data(), ned, n_graphs * 8ULL, cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaMemcpyAsync(counts->max_degree.data(), mdd, n_graphs * 4ULL, cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaMemcpyAsync(counts->degeneracy.data(), dgd, n_graphs * 4ULL, cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaGetLastError());
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  return MCE_OK;
}

}  // namespace mce

using namespace mce;

extern "C" {

mce_status mce_batch_create(const uint32_t *u, const uint32_t *v, const uint64_t *pair_offsets, uint32_t n_graphs,
                            const mce_options *opt, mce_batch **out) {
  if (!out || !pair_offsets || n_graphs == 0) return MCE_ERR_INVALID_ARG;
  *out = nullptr;
  const uint64_t np = pair_offsets[n_graphs];
  if (np && (!u || !v)) return MCE_ERR_INVALID_ARG;
  if (pair_offsets[0] != 0) return MCE_ERR_INVALID_ARG;
  for (uint32_t i = 0; i < n_graphs; i++)
    if (pair_offsets[i + 1] < pair_offsets[i]) return MCE_ERR_INVALID_ARG;
  mce_options o;
  if (opt) o = *opt;
  else mce_default_options(&o);
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return MCE_ERR_NO_DEVICE;
  }
  MCE_CUDA_TRY(cudaSetDevice(o.device));
  keep_pool_memory(o.device);
  mce_batch *b = new (std::nothrow) mce_batch();
  if (!b) return MCE_ERR_OUT_OF_MEMORY;
  b->device = o.device;
  b->scr.device = o.device;
  b->n_graphs = n_graphs;
  auto fail = [&](mce_status s) {
    mce_batch_free(b);
    return s;
  };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(MCE_ERR_CUDA);
  cudaStream_t st = b->stream;
  uint32_t *ud = nullptr, *vd = nullptr;
  const size_t pb = std::max<uint64_t>(np, 1) * 4;
  if (cudaMallocAsync(&ud, pb, st) != cudaSuccess || cudaMallocAsync(&vd, pb, st) != cudaSuccess) {
    if (ud) cudaFreeAsync(ud, st);
    return fail(MCE_ERR_OUT_OF_MEMORY);
  }
  mce_status s = MCE_OK;
  if (np && (cudaMemcpyAsync(ud, u, np * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
             cudaMemcpyAsync(vd, v, np * 4, cudaMemcpyHostToDevice, st) != cudaSuccess))
    s = MCE_ERR_CUDA;
  UnionCounts uc;
  if (s == MCE_OK)
    s = build_union(ud, vd, pair_offsets, n_graphs, o.order, o.spin_limit ? o.spin_limit : (1ULL << 34), st, &b->g,
                    &uc);
  cudaFreeAsync(ud, st);
  cudaFreeAsync(vd, st);
  if (s != MCE_OK) return fail(s);
  b->nv = std::move(uc.nv);
  b->ne = std::move(uc.ne);
  *out = b;
  return MCE_OK;
}

mce_status mce_batch_solve(mce_batch *b, const mce_options *opt, mce_batch_graph_result *results, uint64_t *hist,
                           uint32_t hist_len, double *enumerate_ms) {
  if (!b || !results || (hist && hist_len == 0)) return MCE_ERR_INVALID_ARG;
  MCE_CUDA_TRY(cudaSetDevice(b->device));
  mce_options o;
  if (opt) o = *opt;
  else mce_default_options(&o);
  const uint32_t hl = hist ? hist_len : 1;
  cudaStream_t st = b->stream;
  const uint32_t ng = b->n_graphs;
  mce_status s = MCE_OK;
  const size_t slot_bytes = sizeof(SlotResult) * ng;
  const size_t hist_bytes = sizeof(unsigned long long) * (size_t)ng * hl;
  char *res = (char *)b->scr.get(0, slot_bytes + hist_bytes, &s);
  if (!res) return s;
  SlotResult *slots = (SlotResult *)res;
  unsigned long long *hd = (unsigned long long *)(res + slot_bytes);
  // the captured launch bakes in the plan: capture again when any option
  // that feeds the plan differs from the captured one's
  EnumConfig cfg = config_from_options(o);
  cfg.root_begin = cfg.root_end = 0;
  cfg.n_slots = ng;
  cfg.hist_len = hl;
  // the autotuner (o.blocks_per_sm == 0): successive solves of the batch try
  // the kernel builds in turn, then keep the fastest (each change re-captures)
  uint32_t tune_mode = 0;
  if (!o.blocks_per_sm) cfg.blocks_per_sm = tune_pick(b->tune, (o.flags & MCE_FLAG_STATS) != 0, &tune_mode);
  const bool rebuild = !b->exec || !same_plan_settings(cfg, b->exec_cfg);
  if (rebuild) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    if (b->slots_h) cudaFreeHost(b->slots_h);
    if (b->hist_h) cudaFreeHost(b->hist_h);
    b->slots_h = nullptr;
    b->hist_h = nullptr;
    MCE_CUDA_TRY(cudaMallocHost(&b->slots_h, slot_bytes));
    MCE_CUDA_TRY(cudaMallocHost(&b->hist_h, hist_bytes));
    MCE_TRY(enum_plan(b->g, cfg, &b->scr, slots, hd, &b->plan));
    // capture: clear results, run the persistent kernel, copy results out
    cudaGraph_t graph = nullptr;
    MCE_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(res, 0, slot_bytes + hist_bytes, st);
    mce_status ls = enum_launch(b->plan, st);
    cudaMemcpyAsync(b->slots_h, slots, slot_bytes, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(b->hist_h, hd, hist_bytes, cudaMemcpyDeviceToHost, st);
    cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (ls != MCE_OK) {
      if (graph) cudaGraphDestroy(graph);
      return ls;
    }
    if (ce != cudaSuccess) return MCE_ERR_CUDA;
    ce = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
      b->exec = nullptr;
      return MCE_ERR_CUDA;
    }
    b->exec_cfg = cfg;
  }
  cudaEvent_t e0, e1;
  MCE_CUDA_TRY(cudaEventCreate(&e0));
  MCE_CUDA_TRY(cudaEventCreate(&e1));
  cudaEventRecord(e0, st);
  cudaError_t ce = cudaGraphLaunch(b->exec, st);
  cudaEventRecord(e1, st);
  if (ce != cudaSuccess) s = MCE_ERR_CUDA;
  EnumStats stats;
  if (s == MCE_OK) s = enum_finish(b->plan, st, &stats);
  if (s == MCE_OK && stats.heavy_roots) {
    // deferred roots ran after the captured copy: copy the results again
    if (cudaMemcpyAsync(b->slots_h, slots, slot_bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(b->hist_h, hd, hist_bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      s = MCE_ERR_CUDA;
  }
  float ms = 0;
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (enumerate_ms) *enumerate_ms = ms;
  if (s != MCE_OK) return s;
  if (tune_mode == 1) tune_record(b->tune, cfg.blocks_per_sm, ms);
  for (uint32_t i = 0; i < ng; i++) {
    results[i].count = b->slots_h[i].count;
    results[i].checksum = b->slots_h[i].checksum;
    results[i].max_size = b->slots_h[i].max_size;
    results[i].num_vertices = b->nv[i];
    results[i].num_edges = b->ne[i];
  }
  if (hist) std::memcpy(hist, b->hist_h, hist_bytes);
  return MCE_OK;
}

void mce_batch_free(mce_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->stream) cudaStreamSynchronize(b->stream);
  free_graph(&b->g);
  if (b->slots_h) cudaFreeHost(b->slots_h);
  if (b->hist_h) cudaFreeHost(b->hist_h);
  b->scr.release();
  if (b->stream) {
    cudaStreamSynchronize(b->stream);
    cudaStreamDestroy(b->stream);
  }
  delete b;
}

}  // extern "C"
