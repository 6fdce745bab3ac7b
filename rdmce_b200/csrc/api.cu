// api.cu -- the C ABI (include/rdmce.h): graph handles, solve, results.
//
// Replaces MceGpuSolver / BkSolverWrapper (src/mce_gpu.cu:9-22,
// src/kernels/BkPivotBitBalance.cuh:611-678) and Graph's loaders
// (src/graph.cc:64-213).  Every entry point returns a status; nothing exits.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "hostio.h"

struct mce_graph {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  mce::DeviceGraph g;
  double ms_h2d = 0, ms_pre = 0;
};

namespace mce {

// The graph builders allocate their sort buffers stream-ordered
// (cudaMallocAsync) from the device's default pool, whose release threshold
// is 0: at every synchronisation the freed memory goes back to the driver and
// the next build maps gigabytes again, which costs more than the build.  The
// first time this process uses a device, its default pool is told to keep
// freed memory for reuse (an attribute of this process's pool; it ends with
// the process).
void keep_pool_memory(int device) {
  static std::mutex mu;
  static std::vector<bool> done;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)done.size() <= device) done.resize(device + 1, false);
  if (done[device]) return;
  done[device] = true;
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
}

namespace {

constexpr uint64_t kDefaultSpin = 1ULL << 34;

mce_options defaults() {
  mce_options o;
  std::memset(&o, 0, sizeof(o));
  o.device = 0;
  o.order = MCE_ORDER_DEGENERACY;
  o.share_bound = 24;
  o.expand_r = 1;
  return o;
}

const mce_options &opts_or_default(const mce_options *opt, mce_options &tmp) {
  if (opt) return *opt;
  tmp = defaults();
  return tmp;
}

mce_status set_device(int device) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return MCE_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return MCE_ERR_INVALID_ARG;
  MCE_CUDA_TRY(cudaSetDevice(device));
  keep_pool_memory(device);
  return MCE_OK;
}

uint64_t spin_of(const mce_options &o) { return o.spin_limit ? o.spin_limit : kDefaultSpin; }

mce_status new_handle(const mce_options &o, mce_graph **out) {
  MCE_TRY(set_device(o.device));
  mce_graph *h = new (std::nothrow) mce_graph();
  if (!h) return MCE_ERR_OUT_OF_MEMORY;
  h->device = o.device;
  h->own_stream = o.stream == nullptr;
  if (o.stream) {
    h->stream = (cudaStream_t)o.stream;
  } else if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return MCE_ERR_CUDA;
  }
  *out = h;
  return MCE_OK;
}

void destroy_handle(mce_graph *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  free_graph(&h->g);
  cudaStreamSynchronize(h->stream);
  if (h->own_stream) cudaStreamDestroy(h->stream);
  delete h;
}

struct Timer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

}  // namespace

mce_status graph_from_device_pairs(const uint32_t *ud, const uint32_t *vd, uint64_t n, const mce_options &o,
                                   mce_graph *h) {
  Timer t;
  mce_status s = build_from_pairs(ud, vd, n, o.order, spin_of(o), h->stream, &h->g);
  h->ms_pre = t.ms();
  return s;
}

}  // namespace mce

using namespace mce;

extern "C" {

const char *mce_version(void) { return "rdmce_b200 0.1 (sm_100a)"; }

mce_status mce_probe_int_peak(int device, double *word_ops_per_s) {
  if (!word_ops_per_s) return MCE_ERR_INVALID_ARG;
  MCE_TRY(set_device(device));
  return probe_int_peak(device, word_ops_per_s);
}

mce_status mce_csr_offsets_static(int device, const uint32_t *degree_device, uint32_t *rowoffset_device,
                                  uint64_t n, void *stream) {
  // size check first: an oversized request returns before touching the device
  if (n > MCE_STATIC_SCAN_MAX_N) return MCE_ERR_TOO_LARGE;
  if (!rowoffset_device || (n && !degree_device)) return MCE_ERR_INVALID_ARG;
  MCE_TRY(set_device(device));
  return csr_offsets_static(device, degree_device, rowoffset_device, n, (cudaStream_t)stream);
}

void mce_default_options(mce_options *opt) {
  if (opt) *opt = defaults();
}

const char *mce_status_str(mce_status s) {
  switch (s) {
    case MCE_OK: return "ok";
    case MCE_ERR_INVALID_ARG: return "invalid argument";
    case MCE_ERR_CAPACITY: return "output buffer too small";
    case MCE_ERR_IO: return "file I/O error";
    case MCE_ERR_FORMAT: return "malformed graph input";
    case MCE_ERR_NO_DEVICE: return "no usable CUDA device";
    case MCE_ERR_CUDA: return "CUDA runtime error";
    case MCE_ERR_OUT_OF_MEMORY: return "out of memory";
    case MCE_ERR_TIMEOUT: return "a bounded device wait expired";
    case MCE_ERR_TOO_LARGE: return "graph exceeds 32-bit CSR limits";
    case MCE_ERR_BUSY: return "server busy";
    case MCE_ERR_NOT_FOUND: return "unknown request";
    case MCE_ERR_INTERNAL: return "internal error";
  }
  return "unknown status";
}

mce_status mce_graph_from_coo_device(const uint32_t *u_device, const uint32_t *v_device, uint64_t n_pairs,
                                     const mce_options *opt, mce_graph **out) {
  if (!out || (n_pairs && (!u_device || !v_device))) return MCE_ERR_INVALID_ARG;
  *out = nullptr;
  mce_options tmp;
  const mce_options &o = opts_or_default(opt, tmp);
  mce_graph *h = nullptr;
  MCE_TRY(new_handle(o, &h));
  mce_status s = graph_from_device_pairs(u_device, v_device, n_pairs, o, h);
  if (s != MCE_OK) {
    destroy_handle(h);
    return s;
  }
  *out = h;
  return MCE_OK;
}

mce_status mce_graph_from_coo(const uint32_t *u, const uint32_t *v, uint64_t n_pairs, const mce_options *opt,
                              mce_graph **out) {
  if (!out || (n_pairs && (!u || !v))) return MCE_ERR_INVALID_ARG;
  *out = nullptr;
  mce_options tmp;
  const mce_options &o = opts_or_default(opt, tmp);
  mce_graph *h = nullptr;
  MCE_TRY(new_handle(o, &h));
  Timer t;
  uint32_t *ud = nullptr, *vd = nullptr;
  mce_status s = MCE_OK;
  const size_t bytes = std::max<uint64_t>(n_pairs, 1) * 4;
  if (cudaMallocAsync(&ud, bytes, h->stream) != cudaSuccess || cudaMallocAsync(&vd, bytes, h->stream) != cudaSuccess)
    s = MCE_ERR_OUT_OF_MEMORY;
  if (s == MCE_OK && n_pairs) {
    if (cudaMemcpyAsync(ud, u, n_pairs * 4, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(vd, v, n_pairs * 4, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      s = MCE_ERR_CUDA;
  }
  h->ms_h2d = t.ms();
  if (s == MCE_OK) s = graph_from_device_pairs(ud, vd, n_pairs, o, h);
  if (ud) cudaFreeAsync(ud, h->stream);
  if (vd) cudaFreeAsync(vd, h->stream);
  if (s != MCE_OK) {
    cudaGetLastError();
    destroy_handle(h);
    return s;
  }
  *out = h;
  return MCE_OK;
}

mce_status mce_graph_from_csr(uint64_t n, const uint32_t *rowoffset, const uint32_t *colidx, const uint32_t *labels,
                              int already_ordered, const mce_options *opt, mce_graph **out) {
  if (!out || !rowoffset || (rowoffset[n] && !colidx)) return MCE_ERR_INVALID_ARG;
  *out = nullptr;
  if (n >= (1ULL << 32)) return MCE_ERR_TOO_LARGE;
  // validate on the host: monotone offsets, ids in range, rows strictly increasing
  for (uint64_t x = 0; x < n; x++) {
    if (rowoffset[x + 1] < rowoffset[x]) return MCE_ERR_FORMAT;
    for (uint32_t e = rowoffset[x]; e < rowoffset[x + 1]; e++) {
      if (colidx[e] >= n || colidx[e] == x) return MCE_ERR_FORMAT;
      if (e > rowoffset[x] && colidx[e] <= colidx[e - 1]) return MCE_ERR_FORMAT;
    }
  }
  if (rowoffset[n] & 1) return MCE_ERR_FORMAT;
  mce_options tmp;
  const mce_options &o = opts_or_default(opt, tmp);
  mce_graph *h = nullptr;
  MCE_TRY(new_handle(o, &h));
  const uint64_t m2 = rowoffset[n];
  uint32_t *od = nullptr, *ad = nullptr, *ld = nullptr;
  mce_status s = MCE_OK;
  Timer t;
  if (cudaMallocAsync(&od, (n + 1) * 4, h->stream) != cudaSuccess ||
      cudaMallocAsync(&ad, std::max<uint64_t>(m2, 1) * 4, h->stream) != cudaSuccess ||
      (labels && cudaMallocAsync(&ld, std::max<uint64_t>(n, 1) * 4, h->stream) != cudaSuccess))
    s = MCE_ERR_OUT_OF_MEMORY;
  if (s == MCE_OK) {
    if (cudaMemcpyAsync(od, rowoffset, (n + 1) * 4, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        (m2 && cudaMemcpyAsync(ad, colidx, m2 * 4, cudaMemcpyHostToDevice, h->stream) != cudaSuccess) ||
        (labels && n && cudaMemcpyAsync(ld, labels, n * 4, cudaMemcpyHostToDevice, h->stream) != cudaSuccess))
      s = MCE_ERR_CUDA;
  }
  h->ms_h2d = t.ms();
  Timer t2;
  if (s == MCE_OK)
    s = build_from_csr(n, od, ad, ld, already_ordered, o.order, 0, spin_of(o), h->stream, &h->g);
  h->ms_pre = t2.ms();
  if (od) cudaFreeAsync(od, h->stream);
  if (ad) cudaFreeAsync(ad, h->stream);
  if (ld) cudaFreeAsync(ld, h->stream);
  if (s != MCE_OK) {
    cudaGetLastError();
    destroy_handle(h);
    return s;
  }
  *out = h;
  return MCE_OK;
}

mce_status mce_graph_load_file(const char *path, const mce_options *opt, mce_graph **out) {
  if (!path || !out) return MCE_ERR_INVALID_ARG;
  *out = nullptr;
  if (has_bin_suffix(path)) {
    BinGraph b;
    MCE_TRY(read_bin(path, b));
    mce_graph *h = nullptr;
    MCE_TRY(mce_graph_from_csr(b.n, b.off.data(), b.adj.data(), b.labels.data(), 1, opt, &h));
    h->g.degeneracy = (uint32_t)b.degeneracy;  // the header's value, as LoadFromBin keeps it
    *out = h;
    return MCE_OK;
  }
  // COO text: parsed on the GPU straight into the device COO buffers
  mce_options tmp;
  const mce_options &o = opts_or_default(opt, tmp);
  mce_graph *h = nullptr;
  MCE_TRY(new_handle(o, &h));
  Timer t;
  uint32_t *ud = nullptr, *vd = nullptr;
  uint64_t np = 0;
  mce_status s = parse_text_device(path, h->stream, &ud, &vd, &np);
  h->ms_h2d = t.ms();
  if (s == MCE_OK) s = graph_from_device_pairs(ud, vd, np, o, h);
  if (ud) cudaFreeAsync(ud, h->stream);
  if (vd) cudaFreeAsync(vd, h->stream);
  if (s != MCE_OK) {
    cudaGetLastError();
    destroy_handle(h);
    return s;
  }
  *out = h;
  return MCE_OK;
}

mce_status mce_parse_text_gpu(const char *path, int device, uint32_t **u, uint32_t **v, uint64_t *n_pairs) {
  if (!path || !u || !v || !n_pairs) return MCE_ERR_INVALID_ARG;
  *u = *v = nullptr;
  *n_pairs = 0;
  MCE_TRY(set_device(device));
  cudaStream_t st = nullptr;
  MCE_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  uint32_t *ud = nullptr, *vd = nullptr;
  uint64_t np = 0;
  mce_status s = parse_text_device(path, st, &ud, &vd, &np);
  if (s == MCE_OK) {
    *u = (uint32_t *)std::malloc(std::max<uint64_t>(np, 1) * 4);
    *v = (uint32_t *)std::malloc(std::max<uint64_t>(np, 1) * 4);
    if (!*u || !*v) s = MCE_ERR_OUT_OF_MEMORY;
  }
  if (s == MCE_OK && np &&
      (cudaMemcpyAsync(*u, ud, np * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
       cudaMemcpyAsync(*v, vd, np * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess))
    s = MCE_ERR_CUDA;
  if (ud) cudaFreeAsync(ud, st);
  if (vd) cudaFreeAsync(vd, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && s == MCE_OK) s = MCE_ERR_CUDA;
  cudaStreamDestroy(st);
  if (s != MCE_OK) {
    std::free(*u);
    std::free(*v);
    *u = *v = nullptr;
    return s;
  }
  *n_pairs = np;
  return MCE_OK;
}

mce_status mce_graph_info_get(const mce_graph *g, mce_graph_info *info) {
  if (!g || !info) return MCE_ERR_INVALID_ARG;
  info->num_vertices = g->g.n;
  info->num_edges = g->g.m;
  info->max_degree = g->g.max_degree;
  info->degeneracy = g->g.degeneracy;
  info->device_bytes = (uint64_t)(g->g.n + 1) * 4 + 2 * g->g.m * 4 + (uint64_t)g->g.n * (4 + 16) + g->g.m * 8;
  return MCE_OK;
}

mce_status mce_graph_export_csr(const mce_graph *g, uint32_t *rowoffset, uint32_t *colidx, uint32_t *labels) {
  if (!g) return MCE_ERR_INVALID_ARG;
  MCE_CUDA_TRY(cudaSetDevice(g->device));
  if (rowoffset)
    MCE_CUDA_TRY(cudaMemcpyAsync(rowoffset, g->g.off, (g->g.n + 1) * 4ULL, cudaMemcpyDeviceToHost, g->stream));
  if (colidx && g->g.m)
    MCE_CUDA_TRY(cudaMemcpyAsync(colidx, g->g.adj, 2 * g->g.m * 4, cudaMemcpyDeviceToHost, g->stream));
  if (labels && g->g.n)
    MCE_CUDA_TRY(cudaMemcpyAsync(labels, g->g.labels, g->g.n * 4ULL, cudaMemcpyDeviceToHost, g->stream));
  MCE_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return MCE_OK;
}

mce_status mce_graph_store_bin(const mce_graph *g, const char *path) {
  if (!g || !path) return MCE_ERR_INVALID_ARG;
  BinGraph b;
  b.n = g->g.n;
  b.m = g->g.m;
  b.max_degree = g->g.max_degree;
  b.degeneracy = g->g.degeneracy;
  b.off.resize(b.n + 1);
  b.adj.resize(2 * b.m);
  b.labels.resize(b.n);
  MCE_TRY(mce_graph_export_csr(g, b.off.data(), b.adj.data(), b.labels.data()));
  return write_bin(path, b);
}

void mce_graph_free(mce_graph *g) {
  if (!g) return;
  // a caller-supplied stream is left alone; a handle destroys only its own
  destroy_handle(g);
}

namespace mce {
namespace {

// A workload: which roots, and the settings that change the search.
uint64_t workload_key(const mce_options &o, const uint64_t *roots_h, uint64_t n_roots, bool per_root) {
  uint64_t k = mix64(o.root_begin) ^ mix64(o.root_end + 0x51ULL) ^ mix64(n_roots + 0x77ULL);
  for (uint64_t i = 0; i < n_roots; i++) k = mix64(k ^ roots_h[i]);
  k ^= mix64(((uint64_t)o.flags << 32) | ((uint64_t)o.expand_r << 8) | (per_root ? 1 : 0));
  k ^= mix64(((uint64_t)o.share_bound << 32) | o.reg_share_bound) ^ mix64(((uint64_t)o.warps_per_block << 32) |
                                                                          o.slab_kib);
  return k;
}

// The autotuner's records, process-wide: keyed by the graph's fingerprint
// (device, n, m, degeneracy, max degree) and the workload, so a graph built
// again from the same input (as each end-to-end call does) keeps its tuning.
std::mutex g_tune_mu;
std::unordered_map<uint64_t, TuneRecord> g_tune;

uint64_t tune_key(const mce_graph *g, uint64_t wkey) {
  return mix64(wkey ^ mix64(((uint64_t)g->device << 48) ^ g->g.n)) ^ mix64(g->g.m + 0x1234567ULL) ^
         mix64(((uint64_t)g->g.degeneracy << 32) | g->g.max_degree);
}

uint32_t tuned_blocks(mce_graph *g, uint64_t wkey, const mce_options &o, uint32_t *mode) {
  if (o.blocks_per_sm) {
    *mode = 0;
    return o.blocks_per_sm;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return tune_pick(g_tune[tune_key(g, wkey)], (o.flags & MCE_FLAG_STATS) != 0, mode);
}

void record_tune(mce_graph *g, uint64_t wkey, uint32_t blocks, uint32_t mode, float ms) {
  if (mode != 1) return;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_record(g_tune[tune_key(g, wkey)], blocks, ms);
}

}  // namespace
}  // namespace mce

static mce_status solve_impl(mce_graph *g, const mce_options &o, mce_result *out, const uint64_t *roots_d,
                             uint64_t n_roots, unsigned long long *cnt_d, unsigned long long *chk_d,
                             uint64_t wkey) {
  MCE_CUDA_TRY(cudaSetDevice(g->device));
  std::memset(out, 0, sizeof(*out));
  Timer t;
  cudaStream_t st = g->stream;
  mce_status s = MCE_OK;
  const size_t res_bytes = sizeof(SlotResult) + MCE_HIST_LEN * sizeof(unsigned long long);
  Scratch *scr = default_scratch(g->device);
  lock_default(g->device);
  struct Unlock {
    int d;
    ~Unlock() { unlock_default(d); }
  } unlock{g->device};
  char *res = (char *)scr->get(0, res_bytes, &s);
  if (!res) return s;
  MCE_CUDA_TRY(cudaMemsetAsync(res, 0, res_bytes, st));
  EnumConfig cfg = config_from_options(o);
  uint32_t tune_mode = 0;
  cfg.blocks_per_sm = tuned_blocks(g, wkey, o, &tune_mode);
  cfg.spin_limit = spin_of(o);
  cfg.root_list = roots_d;
  cfg.n_root_list = n_roots;
  cfg.per_root_count = cnt_d;
  cfg.per_root_checksum = chk_d;
  EnumStats stats;
  SlotResult *slot = (SlotResult *)res;
  unsigned long long *hist = (unsigned long long *)(res + sizeof(SlotResult));
  s = enumerate(g->g, cfg, scr, st, slot, hist, &stats);
  if (s != MCE_OK) return s;
  record_tune(g, wkey, cfg.blocks_per_sm, tune_mode, stats.ms_enum);
  out->blocks_per_sm = stats.blocks_per_sm;
  out->autotune = tune_mode;
  Timer t2;
  SlotResult hs;
  MCE_CUDA_TRY(cudaMemcpyAsync(&hs, slot, sizeof(hs), cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaMemcpyAsync(out->hist, hist, MCE_HIST_LEN * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  out->count = hs.count;
  out->checksum = hs.checksum;
  out->max_size = hs.max_size;
  out->degeneracy = g->g.degeneracy;
  out->max_degree = g->g.max_degree;
  out->num_vertices = g->g.n;
  out->num_edges = g->g.m;
  out->roots = stats.roots;
  out->heavy_roots = stats.heavy_roots;
  out->shared_tasks = stats.shared_tasks;
  out->nodes = stats.nodes;
  out->word_ops = stats.word_ops;
  out->build_bytes = stats.build_bytes;
  out->launches = stats.launches;
  for (int i = 0; i < 8; i++) out->warp_cycles[i] = stats.cycles[i];
  for (int i = 0; i < 2; i++) out->max_item_cycles[i] = stats.max_item[i];
  out->status_detail = stats.error;
  out->phase_ms[MCE_PHASE_H2D] = g->ms_h2d;
  out->phase_ms[MCE_PHASE_PREPROCESS] = g->ms_pre;
  out->phase_ms[MCE_PHASE_ENUMERATE] = stats.ms_enum;
  out->phase_ms[MCE_PHASE_D2H] = t2.ms();
  out->phase_ms[MCE_PHASE_TOTAL] = t.ms();
  return MCE_OK;
}

mce_status mce_solve(mce_graph *g, const mce_options *opt, mce_result *out) {
  if (!g || !out) return MCE_ERR_INVALID_ARG;
  mce_options tmp;
  const mce_options &o = opts_or_default(opt, tmp);
  return solve_impl(g, o, out, nullptr, 0, nullptr, nullptr, workload_key(o, nullptr, 0, false));
}

mce_status mce_solve_roots(mce_graph *g, const uint64_t *roots, uint64_t n_roots, const mce_options *opt,
                           uint64_t *counts, uint64_t *checksums) {
  if (!g || (n_roots && (!roots || !counts || !checksums))) return MCE_ERR_INVALID_ARG;
  if (n_roots >= (1ULL << 32)) return MCE_ERR_INVALID_ARG;
  for (uint64_t i = 0; i < n_roots; i++)
    if (roots[i] >= g->g.m) return MCE_ERR_INVALID_ARG;
  if (!n_roots) return MCE_OK;
  mce_options tmp;
  const mce_options &o = opts_or_default(opt, tmp);
  MCE_CUDA_TRY(cudaSetDevice(g->device));
  cudaStream_t st = g->stream;
  uint64_t *rd = nullptr;
  unsigned long long *cd = nullptr, *hd = nullptr;
  mce_status s = MCE_OK;
  if (cudaMallocAsync(&rd, n_roots * 8, st) != cudaSuccess || cudaMallocAsync(&cd, n_roots * 8, st) != cudaSuccess ||
      cudaMallocAsync(&hd, n_roots * 8, st) != cudaSuccess)
    s = MCE_ERR_OUT_OF_MEMORY;
  if (s == MCE_OK && cudaMemcpyAsync(rd, roots, n_roots * 8, cudaMemcpyHostToDevice, st) != cudaSuccess)
    s = MCE_ERR_CUDA;
  mce_result *r = nullptr;
  if (s == MCE_OK) {
    r = new (std::nothrow) mce_result;
    if (!r) s = MCE_ERR_OUT_OF_MEMORY;
  }
  mce_options o2 = o;
  o2.flags |= MCE_FLAG_NO_SHARING;  // a root's cliques must stay with the warp that owns it
  if (s == MCE_OK) s = solve_impl(g, o2, r, rd, n_roots, cd, hd, workload_key(o2, roots, n_roots, true));
  if (s == MCE_OK) {
    if (cudaMemcpyAsync(counts, cd, n_roots * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(checksums, hd, n_roots * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      s = MCE_ERR_CUDA;
  }
  delete r;
  if (rd) cudaFreeAsync(rd, st);
  if (cd) cudaFreeAsync(cd, st);
  if (hd) cudaFreeAsync(hd, st);
  cudaStreamSynchronize(st);
  return s;
}

mce_status mce_solve_root_list(mce_graph *g, const uint64_t *roots, uint64_t n_roots, const mce_options *opt,
                               mce_result *out) {
  if (!g || !out || (n_roots && !roots)) return MCE_ERR_INVALID_ARG;
  if (n_roots >= (1ULL << 32)) return MCE_ERR_INVALID_ARG;
  for (uint64_t i = 0; i < n_roots; i++)
    if (roots[i] >= g->g.m) return MCE_ERR_INVALID_ARG;
  mce_options tmp;
  const mce_options &o = opts_or_default(opt, tmp);
  MCE_CUDA_TRY(cudaSetDevice(g->device));
  cudaStream_t st = g->stream;
  uint64_t *rd = nullptr;
  if (cudaMallocAsync(&rd, std::max<uint64_t>(n_roots, 1) * 8, st) != cudaSuccess) return MCE_ERR_OUT_OF_MEMORY;
  mce_status s = MCE_OK;
  if (n_roots && cudaMemcpyAsync(rd, roots, n_roots * 8, cudaMemcpyHostToDevice, st) != cudaSuccess)
    s = MCE_ERR_CUDA;
  if (s == MCE_OK) s = solve_impl(g, o, out, rd, n_roots, nullptr, nullptr, workload_key(o, roots, n_roots, false));
  cudaFreeAsync(rd, st);
  cudaStreamSynchronize(st);
  return s;
}

mce_status mce_solve_coo(const uint32_t *u, const uint32_t *v, uint64_t n_pairs, const mce_options *opt,
                         mce_result *out) {
  if (!out) return MCE_ERR_INVALID_ARG;
  Timer t;
  mce_graph *g = nullptr;
  MCE_TRY(mce_graph_from_coo(u, v, n_pairs, opt, &g));
  mce_status s = mce_solve(g, opt, out);
  if (s == MCE_OK) out->phase_ms[MCE_PHASE_TOTAL] = t.ms();
  mce_graph_free(g);
  return s;
}

}  // extern "C"
