// preprocess.cu -- COO pairs -> degeneracy-ordered CSR, entirely on the GPU.
//
// Replaces the reference's single-threaded host pipeline:
//   Graph::LoadFromFile edge handling   src/graph.cc:64-152  (self-loops dropped,
//       u<v, sort+unique, dense relabel of present labels in ascending order)
//   Graph::SortByDegeneracy/ApplyOrder  src/graph.cc:281-306, 54-77
//   Graph::ConvertToCsr + LoadFromCpu   src/graph.cc:216-236, src/graph_gpu.cu:3-58
// Steps: pack (min,max) keys -> radix sort -> unique -> mark/scan dense ids ->
// degrees -> k-core peeling in synchronous rounds (one cooperative launch) ->
// relabel both edge directions -> radix sort -> CSR offsets by scan -> root
// list (v0 < v1) by flag+scan.
#include <algorithm>
#include <vector>

#include <cooperative_groups.h>

#include "common.cuh"
#include "engine.h"

namespace mce {

namespace cg = cooperative_groups;

namespace {

constexpr uint64_t kInvalidKey = ~0ULL;

__global__ void k_pack_keys(const uint32_t *u, const uint32_t *v, uint64_t n, int bits, uint64_t *keys) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a = u[i], b = v[i];
    if (a == b) {
      keys[i] = kInvalidKey;
      continue;
    }
    if (a > b) {
      uint32_t t = a;
      a = b;
      b = t;
    }
    keys[i] = ((uint64_t)a << bits) | b;
  }
}

__global__ void k_unique_flags(const uint64_t *keys, uint64_t n, uint32_t *flags) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t k = keys[i];
    flags[i] = (k != kInvalidKey && (i == 0 || keys[i - 1] != k)) ? 1u : 0u;
  }
}

__global__ void k_compact_keys(const uint64_t *keys, const uint32_t *flags, const uint32_t *pos, uint64_t n,
                               uint64_t *out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (flags[i]) out[pos[i]] = keys[i];
}

__global__ void k_mark_labels(const uint64_t *edges, uint64_t m, int bits, uint32_t *mark) {
  const uint64_t mask = (1ULL << bits) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    mark[edges[i] >> bits] = 1;
    mark[edges[i] & mask] = 1;
  }
}

__global__ void k_labels_from_marks(const uint32_t *mark, const uint32_t *id, uint64_t nl, uint32_t *labels) {
  for (uint64_t l = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; l < nl; l += (uint64_t)gridDim.x * blockDim.x)
    if (mark[l]) labels[id[l]] = (uint32_t)l;
}

// edges (label pair) -> dense ids, degrees
__global__ void k_map_edges(uint64_t *edges, uint64_t m, int bits, const uint32_t *id, uint32_t *eu,
                            uint32_t *ev, uint32_t *deg) {
  const uint64_t mask = (1ULL << bits) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a = id[edges[i] >> bits], b = id[edges[i] & mask];
    eu[i] = a;
    ev[i] = b;
    atomicAdd(&deg[a], 1u);
    atomicAdd(&deg[b], 1u);
  }
}

// unsorted symmetric adjacency for peeling
__global__ void k_fill_adj(const uint32_t *eu, const uint32_t *ev, uint64_t m, uint32_t *cursor, uint32_t *adj) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a = eu[i], b = ev[i];
    adj[atomicAdd(&cursor[a], 1u)] = b;
    adj[atomicAdd(&cursor[b], 1u)] = a;
  }
}

__global__ void k_iota(uint32_t *a, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    a[i] = (uint32_t)i;
}

// ---- k-core peeling in synchronous rounds (one cooperative launch) ----
//
// Level k: the frontier F_0 = unremoved vertices of residual degree <= k; each
// round removes its whole frontier at once and decrements the neighbours, and
// every neighbour that drops to k joins the next round's frontier.  A vertex's
// position is (global round, vertex id): every later neighbour of x is either
// in x's round or in a later one, all of which were unremoved when x's
// residual degree fell to <= k, so x has at most k later neighbours -- a
// degeneracy order.  The rounds make the order deterministic, so root ids
// (edges of the ordered CSR) are stable from run to run; the reference's
// sequential queue (graph.cc:289-304) orders vertices inside a round
// differently, which changes neither the degeneracy nor the clique set.
struct PeelCtl {
  uint32_t fcnt[3];     // frontier sizes, by round mod 3
  uint32_t rcnt[3];     // survivors of each level's scan, by level mod 3
  uint32_t rmin[3];     // smallest surviving residual degree, by level mod 3
  uint32_t degeneracy;
  uint32_t rounds;
  uint32_t levels;
  uint32_t error;       // 1: level bound exceeded (cannot happen on a consistent CSR)
};

__global__ void __launch_bounds__(256) k_peel_rounds(uint32_t n, const uint32_t *off, const uint32_t *adj,
                                                     int *deg, uint32_t *state, uint32_t *remA, uint32_t *remB,
                                                     uint32_t *frA, uint32_t *frB, PeelCtl *ctl, uint32_t max_levels) {
  cg::grid_group grid = cg::this_grid();
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t gwarp = tid >> 5, nwarps = nthreads >> 5;
  const bool leader = tid == 0;
  uint32_t k = 0, degen = 0, lev = 0, r = 0, removed = 0, nrem = n;
  uint32_t *rem_cur = remA, *rem_nxt = remB;
  while (removed < n) {
    if (lev > max_levels) {
      if (leader) atomicExch(&ctl->error, 1u);
      break;  // uniform: every thread sees the same lev
    }
    uint32_t *fr = (r & 1) ? frB : frA;
    // scan: claim residual degree <= k into F_r, keep the rest
    if (leader) {
      ctl->rcnt[(lev + 1) % 3] = 0;
      ctl->rmin[(lev + 1) % 3] = 0xffffffffu;
    }
    uint32_t local_min = 0xffffffffu;
    // warp-uniform trip count; one atomic per warp and list (every survivor
    // is appended at every level, so per-thread atomics on one counter would
    // serialise)
    for (uint64_t base = tid - lane; base < nrem; base += nthreads) {
      const uint64_t i = base + lane;
      uint32_t v = 0;
      int d = 0;
      bool claim = false, keep = false;
      if (i < nrem) {
        v = __ldcg(rem_cur + i);
        if (!__ldcg(state + v)) {
          d = __ldcg(deg + v);
          claim = d <= (int)k;
          keep = !claim;
        }
      }
      const uint32_t cm = __ballot_sync(kFull, claim), km = __ballot_sync(kFull, keep);
      uint32_t cb = 0, kb = 0;
      if (lane == 0) {
        if (cm) cb = atomicAdd(&ctl->fcnt[r % 3], (uint32_t)__popc(cm));
        if (km) kb = atomicAdd(&ctl->rcnt[lev % 3], (uint32_t)__popc(km));
      }
      cb = __shfl_sync(kFull, cb, 0);
      kb = __shfl_sync(kFull, kb, 0);
      if (claim) {
        state[v] = r + 1;
        fr[cb + __popc(cm & lanemask_lt())] = v;
      } else if (keep) {
        rem_nxt[kb + __popc(km & lanemask_lt())] = v;
        local_min = min(local_min, (uint32_t)d);
      }
    }
    local_min = __reduce_min_sync(kFull, local_min);
    if (lane == 0 && local_min != 0xffffffffu) atomicMin(&ctl->rmin[lev % 3], local_min);
    grid.sync();
    uint32_t level_claims = 0;
    for (;;) {
      const uint32_t nf = __ldcg(&ctl->fcnt[r % 3]);
      if (nf == 0) break;
      level_claims += nf;
      removed += nf;
      const uint32_t *cur = (r & 1) ? frB : frA;
      uint32_t *nxt = (r & 1) ? frA : frB;
      if (leader) ctl->fcnt[(r + 2) % 3] = 0;  // last read in round r - 1
      // Each frontier vertex's adjacency is shared by `per` warps (all the
      // grid's warps split evenly when the frontier is small: the dense
      // cores' hubs hold tens of thousands of neighbours each).
      const uint64_t per = nf < nwarps ? nwarps / nf : 1;
      for (uint64_t i = gwarp / per; i < nf; i += nwarps / per) {
        const uint32_t v = __ldcg(cur + i);
        const uint32_t e1 = off[v + 1];
        const uint32_t part = (uint32_t)(gwarp % per);
        for (uint64_t e = (uint64_t)off[v] + 32ULL * part + lane; e < e1; e += 32ULL * per) {
          const uint32_t u = adj[e];
          if (__ldcg(state + u)) continue;
          if (atomicSub(&deg[u], 1) == (int)k + 1 && atomicCAS(&state[u], 0u, r + 2) == 0u)
            nxt[atomicAdd(&ctl->fcnt[(r + 1) % 3], 1u)] = u;
        }
      }
      grid.sync();
      r++;
    }
    // F_r is empty: round index r is skipped, so no vertex of the next level
    // shares a round number with this level's
    r++;
    nrem = __ldcg(&ctl->rcnt[lev % 3]);
    const uint32_t rmin = __ldcg(&ctl->rmin[lev % 3]);
    uint32_t *t = rem_cur;
    rem_cur = rem_nxt;
    rem_nxt = t;
    if (level_claims) {
      degen = k;
      k = k + 1;
    } else {
      if (rmin == 0xffffffffu) break;
      k = max(k + 1, rmin);
    }
    lev++;
    // The next scan fills fcnt[r % 3] and the round after it fcnt[(r + 1) % 3],
    // which still holds the size of this level's last processed round; the
    // only counter still being read (fcnt of the empty round) is already zero.
    if (leader) ctl->fcnt[0] = ctl->fcnt[1] = ctl->fcnt[2] = 0;
    grid.sync();
  }
  if (leader) {
    ctl->degeneracy = degen;
    ctl->rounds = r;
    ctl->levels = lev;
  }
}

__global__ void k_round_keys(const uint32_t *state, uint32_t n, int nb, uint64_t *keys) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    keys[i] = ((uint64_t)(state[i] - 1) << nb) | i;
}

__global__ void k_order_from_round_keys(const uint64_t *keys, uint32_t n, uint64_t mask, uint32_t *order) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    order[i] = (uint32_t)(keys[i] & mask);
}

__global__ void k_rank_from_order(const uint32_t *order, uint32_t n, uint32_t *rank) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) rank[order[i]] = i;
}

// both directions of every edge under the new ids, packed (row << nb) | col
__global__ void k_relabel_keys(const uint32_t *eu, const uint32_t *ev, uint64_t m, const uint32_t *rank, int nb,
                               uint64_t *keys, uint32_t *deg_new) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a = rank[eu[i]], b = rank[ev[i]];
    keys[2 * i] = ((uint64_t)a << nb) | b;
    keys[2 * i + 1] = ((uint64_t)b << nb) | a;
    atomicAdd(&deg_new[a], 1u);
    atomicAdd(&deg_new[b], 1u);
  }
}

__global__ void k_csr_cols(const uint64_t *keys, uint64_t m2, int nb, uint32_t *adj, uint32_t *upflag) {
  const uint64_t mask = (1ULL << nb) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m2; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t r = (uint32_t)(keys[i] >> nb), c = (uint32_t)(keys[i] & mask);
    adj[i] = c;
    upflag[i] = r < c ? 1u : 0u;
  }
}

__global__ void k_roots(const uint64_t *keys, uint64_t m2, int nb, const uint32_t *upflag, const uint32_t *pos,
                        uint32_t *root_v0, uint32_t *root_v1) {
  const uint64_t mask = (1ULL << nb) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m2; i += (uint64_t)gridDim.x * blockDim.x)
    if (upflag[i]) {
      root_v0[pos[i]] = (uint32_t)(keys[i] >> nb);
      root_v1[pos[i]] = (uint32_t)(keys[i] & mask);
    }
}

__global__ void k_permute_labels(const uint32_t *labels_old, const uint32_t *rank, uint32_t n, uint32_t *labels,
                                 uint64_t *h1, uint64_t *h2) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t l = labels_old[i];
    uint32_t r = rank ? rank[i] : i;
    labels[r] = l;
    h1[r] = mix64((uint64_t)l);
    h2[r] = mix64((uint64_t)l ^ kGolden);
  }
}

__global__ void k_degree_keys(const uint32_t *deg, uint32_t n, int desc, uint64_t *keys) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t d = desc ? ~deg[i] : deg[i];
    keys[i] = ((uint64_t)d << 32) | i;
  }
}

__global__ void k_order_from_keys(const uint64_t *keys, uint32_t n, uint32_t *order) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    order[i] = (uint32_t)keys[i];
}

int bits_for(uint64_t maxval) {
  int b = 1;
  while (b < 64 && (maxval >> b) != 0) b++;
  return b;
}

template <typename T>
struct DevBuf {
  T *p = nullptr;
  cudaStream_t st = nullptr;
  mce_status alloc(size_t n, cudaStream_t s) {
    st = s;
    if (cudaMallocAsync(&p, std::max<size_t>(n, 1) * sizeof(T), s) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return MCE_ERR_OUT_OF_MEMORY;
    }
    return MCE_OK;
  }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
  }
  ~DevBuf() { release(); }
};

template <typename T>
mce_status read_scalar(const T *d, T *h, cudaStream_t st) {
  MCE_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(T), cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  return MCE_OK;
}

// k-core peeling over an unsorted symmetric CSR; fills order[] (position -> vertex)
mce_status peel(uint32_t n, const uint32_t *off, const uint32_t *adj, const uint32_t *deg0, uint32_t max_degree,
                uint32_t *order, uint32_t *degeneracy, cudaStream_t st) {
  DevBuf<int> deg;
  DevBuf<uint32_t> state, remA, remB, frA, frB;
  DevBuf<PeelCtl> ctl;
  MCE_TRY(deg.alloc(n, st));
  MCE_TRY(state.alloc(n, st));
  MCE_TRY(remA.alloc(n, st));
  MCE_TRY(remB.alloc(n, st));
  MCE_TRY(frA.alloc(n, st));
  MCE_TRY(frB.alloc(n, st));
  MCE_TRY(ctl.alloc(1, st));
  MCE_CUDA_TRY(cudaMemcpyAsync(deg.p, deg0, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  MCE_CUDA_TRY(cudaMemsetAsync(state.p, 0, n * sizeof(uint32_t), st));
  k_iota<<<grid_for(n, 256), 256, 0, st>>>(remA.p, n); note_launch();
  // the control block goes through ordinary host memory: pinning it for each
  // build (and unpinning, which synchronises the device) would stall other
  // streams' work, e.g. concurrently served requests
  PeelCtl h{};
  for (int i = 0; i < 3; i++) h.rmin[i] = 0xffffffffu;
  PeelCtl hc_buf = h;
  PeelCtl *hc = &hc_buf;
  MCE_CUDA_TRY(cudaMemcpyAsync(ctl.p, hc, sizeof(PeelCtl), cudaMemcpyHostToDevice, st));
  int dev = 0, sms = 0, per_sm = 0;
  MCE_CUDA_TRY(cudaGetDevice(&dev));
  MCE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  MCE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_peel_rounds, 256, 0));
  if (per_sm < 1) return MCE_ERR_INTERNAL;
  // a cooperative launch: every block is resident, so grid.sync() is sound
  const uint32_t blocks = (uint32_t)std::min(per_sm, 2) * (uint32_t)sms;
  uint32_t nn = n, maxl = max_degree + 2;
  int *degp = deg.p;
  uint32_t *statep = state.p, *ra = remA.p, *rb = remB.p, *fa = frA.p, *fb = frB.p;
  PeelCtl *cp = ctl.p;
  void *args[] = {&nn, (void *)&off, (void *)&adj, &degp, &statep, &ra, &rb, &fa, &fb, &cp, &maxl};
  MCE_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)k_peel_rounds, dim3(blocks), dim3(256), args, 0, st));
  note_launch();
  MCE_CUDA_TRY(cudaMemcpyAsync(hc, ctl.p, sizeof(PeelCtl), cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  h = *hc;
  if (h.error) return MCE_ERR_INTERNAL;
  *degeneracy = h.degeneracy;
  // order = vertices sorted by (round, id)
  const int nb = bits_for(n ? n - 1 : 0), rb_bits = bits_for(h.rounds);
  if (nb + rb_bits > 64) return MCE_ERR_TOO_LARGE;
  DevBuf<uint64_t> keys, tmp;
  MCE_TRY(keys.alloc(n, st));
  MCE_TRY(tmp.alloc(n, st));
  k_round_keys<<<grid_for(n, 256), 256, 0, st>>>(state.p, n, nb, keys.p); note_launch();
  MCE_TRY(radix_sort_u64(keys.p, tmp.p, n, nb + rb_bits, st));
  k_order_from_round_keys<<<grid_for(n, 256), 256, 0, st>>>(keys.p, n, (1ULL << nb) - 1, order); note_launch();
  MCE_CUDA_TRY(cudaGetLastError());
  return MCE_OK;
}

}  // namespace

namespace {

__global__ void k_pack_keys64(const uint32_t *u, const uint32_t *v, uint64_t n, uint64_t *keys) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a = u[i], b = v[i];
    if (a == b) {
      keys[i] = kInvalidKey;  // (a < b) keys never reach all-ones
      continue;
    }
    if (a > b) {
      uint32_t t = a;
      a = b;
      b = t;
    }
    keys[i] = ((uint64_t)a << 32) | b;
  }
}

__global__ void k_endpoints(const uint64_t *edges, uint64_t m, uint64_t *ends) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    ends[2 * i] = edges[i] >> 32;
    ends[2 * i + 1] = edges[i] & 0xffffffffULL;
  }
}

__global__ void k_labels_from_sorted(const uint64_t *ends, const uint32_t *flag, const uint32_t *pos, uint64_t k,
                                     uint32_t *labels) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += (uint64_t)gridDim.x * blockDim.x)
    if (flag[i]) labels[pos[i]] = (uint32_t)ends[i];
}

__device__ __forceinline__ uint32_t find_label(const uint32_t *labels, uint32_t n, uint32_t l) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (labels[mid] < l) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void k_map_edges_search(const uint64_t *edges, uint64_t m, const uint32_t *labels, uint32_t n,
                                   uint32_t *eu, uint32_t *ev, uint32_t *deg) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = find_label(labels, n, (uint32_t)(edges[i] >> 32));
    const uint32_t b = find_label(labels, n, (uint32_t)(edges[i] & 0xffffffffULL));
    eu[i] = a;
    ev[i] = b;
    atomicAdd(&deg[a], 1u);
    atomicAdd(&deg[b], 1u);
  }
}

// present labels, ascending, by sorting the 2m endpoints; ids by binary search
mce_status build_sparse_labels(const uint32_t *u, const uint32_t *v, uint64_t np, int order_kind,
                               uint64_t spin_limit, cudaStream_t st, DeviceGraph *g) {
  if (np >= (1ULL << 32)) return MCE_ERR_TOO_LARGE;
  DevBuf<uint64_t> keys, tmp;
  MCE_TRY(keys.alloc(np, st));
  MCE_TRY(tmp.alloc(np, st));
  k_pack_keys64<<<grid_for(np, 256), 256, 0, st>>>(u, v, np, keys.p); note_launch();
  MCE_TRY(radix_sort_u64(keys.p, tmp.p, np, 64, st));
  DevBuf<uint32_t> flags, pos;
  MCE_TRY(flags.alloc(np + 1, st));
  MCE_TRY(pos.alloc(np + 1, st));
  k_unique_flags<<<grid_for(np, 256), 256, 0, st>>>(keys.p, np, flags.p); note_launch();
  MCE_TRY(scan_exclusive_u32(flags.p, pos.p, np, pos.p + np, st));
  uint32_t m32 = 0;
  MCE_TRY(read_scalar(pos.p + np, &m32, st));
  const uint64_t m = m32;
  if (2 * m >= (1ULL << 32)) return MCE_ERR_TOO_LARGE;
  DevBuf<uint64_t> edges;
  MCE_TRY(edges.alloc(m, st));
  k_compact_keys<<<grid_for(np, 256), 256, 0, st>>>(keys.p, flags.p, pos.p, np, edges.p); note_launch();
  keys.release();
  tmp.release();
  flags.release();
  pos.release();
  const uint64_t k = 2 * m;
  DevBuf<uint64_t> ends, etmp;
  MCE_TRY(ends.alloc(k, st));
  MCE_TRY(etmp.alloc(k, st));
  k_endpoints<<<grid_for(m, 256), 256, 0, st>>>(edges.p, m, ends.p); note_launch();
  MCE_TRY(radix_sort_u64(ends.p, etmp.p, k, 32, st));
  etmp.release();
  DevBuf<uint32_t> f2, p2;
  MCE_TRY(f2.alloc(k + 1, st));
  MCE_TRY(p2.alloc(k + 1, st));
  k_unique_flags<<<grid_for(k, 256), 256, 0, st>>>(ends.p, k, f2.p); note_launch();
  MCE_TRY(scan_exclusive_u32(f2.p, p2.p, k, p2.p + k, st));
  uint32_t n = 0;
  MCE_TRY(read_scalar(p2.p + k, &n, st));
  DevBuf<uint32_t> labels0, eu, ev, deg;
  MCE_TRY(labels0.alloc(n, st));
  MCE_TRY(eu.alloc(m, st));
  MCE_TRY(ev.alloc(m, st));
  MCE_TRY(deg.alloc(n + 1, st));
  k_labels_from_sorted<<<grid_for(k, 256), 256, 0, st>>>(ends.p, f2.p, p2.p, k, labels0.p); note_launch();
  MCE_CUDA_TRY(cudaMemsetAsync(deg.p, 0, (n + 1) * sizeof(uint32_t), st));
  k_map_edges_search<<<grid_for(m, 256), 256, 0, st>>>(edges.p, m, labels0.p, n, eu.p, ev.p, deg.p); note_launch();
  ends.release();
  f2.release();
  p2.release();
  edges.release();
  MCE_TRY(finish_graph(n, m, eu.p, ev.p, deg.p, labels0.p, order_kind, spin_limit, st, g));
  return MCE_OK;
}

}  // namespace

mce_status build_from_pairs(const uint32_t *u, const uint32_t *v, uint64_t np, int order_kind,
                            uint64_t spin_limit, cudaStream_t st, DeviceGraph *g) {
  *g = DeviceGraph{};
  DevBuf<uint32_t> maxbuf;
  MCE_TRY(maxbuf.alloc(2, st));
  MCE_TRY(reduce_max_u32(u, np, maxbuf.p, st));
  MCE_TRY(reduce_max_u32(v, np, maxbuf.p + 1, st));
  uint32_t hm[2] = {0, 0};
  MCE_CUDA_TRY(cudaMemcpyAsync(hm, maxbuf.p, sizeof(hm), cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  const uint32_t maxlab = std::max(hm[0], hm[1]);
  // labels much sparser than the pair count (or near 2^32): sort-based relabel
  if (maxlab >= (1u << 30) || (uint64_t)maxlab > 8 * np + (1u << 20))
    return build_sparse_labels(u, v, np, order_kind, spin_limit, st, g);
  const int lb = bits_for(maxlab);
  if (2 * lb > 63) return MCE_ERR_TOO_LARGE;

  // 1) normalised (min,max) keys, sorted, unique
  DevBuf<uint64_t> keys, tmp;
  MCE_TRY(keys.alloc(np, st));
  MCE_TRY(tmp.alloc(np, st));
  k_pack_keys<<<grid_for(np, 256), 256, 0, st>>>(u, v, np, lb, keys.p); note_launch();
  MCE_TRY(radix_sort_u64(keys.p, tmp.p, np, 2 * lb, st));
  DevBuf<uint32_t> flags, pos;
  MCE_TRY(flags.alloc(np + 1, st));
  MCE_TRY(pos.alloc(np + 1, st));
  k_unique_flags<<<grid_for(np, 256), 256, 0, st>>>(keys.p, np, flags.p); note_launch();
  MCE_TRY(scan_exclusive_u32(flags.p, pos.p, np, pos.p + np, st));
  uint32_t m32 = 0;
  MCE_TRY(read_scalar(pos.p + np, &m32, st));
  const uint64_t m = m32;
  if (np > 0xffffffffULL || 2 * m >= (1ULL << 32)) return MCE_ERR_TOO_LARGE;
  DevBuf<uint64_t> edges;
  MCE_TRY(edges.alloc(m, st));
  k_compact_keys<<<grid_for(np, 256), 256, 0, st>>>(keys.p, flags.p, pos.p, np, edges.p); note_launch();
  keys.release();
  tmp.release();
  flags.release();
  pos.release();

  // 2) dense ids of present labels, ascending (src/graph.cc:123-130)
  const uint64_t nl = (uint64_t)maxlab + 1;
  DevBuf<uint32_t> mark, id;
  MCE_TRY(mark.alloc(nl + 1, st));
  MCE_TRY(id.alloc(nl + 1, st));
  MCE_CUDA_TRY(cudaMemsetAsync(mark.p, 0, nl * sizeof(uint32_t), st));
  k_mark_labels<<<grid_for(m, 256), 256, 0, st>>>(edges.p, m, lb, mark.p); note_launch();
  MCE_TRY(scan_exclusive_u32(mark.p, id.p, nl, id.p + nl, st));
  uint32_t n = 0;
  MCE_TRY(read_scalar(id.p + nl, &n, st));
  DevBuf<uint32_t> labels0, eu, ev, deg;
  MCE_TRY(labels0.alloc(n, st));
  MCE_TRY(eu.alloc(m, st));
  MCE_TRY(ev.alloc(m, st));
  MCE_TRY(deg.alloc(n + 1, st));
  k_labels_from_marks<<<grid_for(nl, 256), 256, 0, st>>>(mark.p, id.p, nl, labels0.p); note_launch();
  MCE_CUDA_TRY(cudaMemsetAsync(deg.p, 0, (n + 1) * sizeof(uint32_t), st));
  k_map_edges<<<grid_for(m, 256), 256, 0, st>>>(edges.p, m, lb, id.p, eu.p, ev.p, deg.p); note_launch();
  mark.release();
  id.release();
  edges.release();
  MCE_TRY(finish_graph(n, m, eu.p, ev.p, deg.p, labels0.p, order_kind, spin_limit, st, g));
  return MCE_OK;
}

// eu/ev: m edges on dense ids (any order, no duplicates, no self-loops);
// deg: degrees (n); labels0: original labels of the dense ids.
mce_status finish_graph(uint32_t n, uint64_t m, const uint32_t *eu, const uint32_t *ev, const uint32_t *deg,
                        const uint32_t *labels0, int order_kind, uint64_t spin_limit, cudaStream_t st,
                        DeviceGraph *g) {
  *g = DeviceGraph{};
  g->n = n;
  g->m = m;
  g->stream = st;
  if (2 * m >= (1ULL << 32)) return MCE_ERR_TOO_LARGE;
  DevBuf<uint32_t> maxd;
  MCE_TRY(maxd.alloc(1, st));
  MCE_TRY(reduce_max_u32(deg, n, maxd.p, st));
  MCE_TRY(read_scalar(maxd.p, &g->max_degree, st));

  // 3) vertex order
  DevBuf<uint32_t> order, rank;
  MCE_TRY(order.alloc(n, st));
  MCE_TRY(rank.alloc(n, st));
  g->degeneracy = g->max_degree;  // Graph::LoadFromFile leaves degeneracy_ = max degree (graph.cc:149)
  if (order_kind == MCE_ORDER_DEGENERACY && n > 0) {
    DevBuf<uint32_t> off0, cursor, adj0;
    MCE_TRY(off0.alloc(n + 1, st));
    MCE_TRY(cursor.alloc(n + 1, st));
    MCE_TRY(adj0.alloc(2 * m, st));
    MCE_TRY(scan_exclusive_u32(deg, off0.p, n, off0.p + n, st));
    MCE_CUDA_TRY(cudaMemcpyAsync(cursor.p, off0.p, (n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    k_fill_adj<<<grid_for(m, 256), 256, 0, st>>>(eu, ev, m, cursor.p, adj0.p); note_launch();
    MCE_TRY(peel(n, off0.p, adj0.p, deg, g->max_degree, order.p, &g->degeneracy, st));
  } else if ((order_kind == MCE_ORDER_DEGREE_ASC || order_kind == MCE_ORDER_DEGREE_DESC) && n > 0) {
    DevBuf<uint64_t> dk, dt;
    MCE_TRY(dk.alloc(n, st));
    MCE_TRY(dt.alloc(n, st));
    k_degree_keys<<<grid_for(n, 256), 256, 0, st>>>(deg, n, order_kind == MCE_ORDER_DEGREE_DESC, dk.p); note_launch();
    MCE_TRY(radix_sort_u64(dk.p, dt.p, n, 64, st));
    k_order_from_keys<<<grid_for(n, 256), 256, 0, st>>>(dk.p, n, order.p); note_launch();
  } else {
    k_iota<<<grid_for(n, 256), 256, 0, st>>>(order.p, n); note_launch();
  }
  k_rank_from_order<<<grid_for(n, 256), 256, 0, st>>>(order.p, n, rank.p); note_launch();
  order.release();

  // 4) relabelled symmetric edge keys -> sorted CSR
  const int nb = bits_for(n ? n - 1 : 0);
  const uint64_t m2 = 2 * m;
  DevBuf<uint64_t> keys, tmp;
  MCE_TRY(keys.alloc(m2, st));
  MCE_TRY(tmp.alloc(m2, st));
  DevBuf<uint32_t> deg_new;
  MCE_TRY(deg_new.alloc(n + 1, st));
  MCE_CUDA_TRY(cudaMemsetAsync(deg_new.p, 0, (n + 1) * sizeof(uint32_t), st));
  k_relabel_keys<<<grid_for(m, 256), 256, 0, st>>>(eu, ev, m, rank.p, nb, keys.p, deg_new.p); note_launch();
  MCE_TRY(radix_sort_u64(keys.p, tmp.p, m2, 2 * nb, st));
  tmp.release();
  MCE_CUDA_TRY(cudaMallocAsync(&g->off, (n + 1) * sizeof(uint32_t), st));
  MCE_CUDA_TRY(cudaMallocAsync(&g->adj, std::max<uint64_t>(m2, 1) * sizeof(uint32_t), st));
  MCE_TRY(scan_exclusive_u32(deg_new.p, g->off, n, g->off + n, st));
  DevBuf<uint32_t> upflag, uppos;
  MCE_TRY(upflag.alloc(m2 + 1, st));
  MCE_TRY(uppos.alloc(m2 + 1, st));
  k_csr_cols<<<grid_for(m2, 256), 256, 0, st>>>(keys.p, m2, nb, g->adj, upflag.p); note_launch();
  MCE_TRY(scan_exclusive_u32(upflag.p, uppos.p, m2, uppos.p + m2, st));
  MCE_CUDA_TRY(cudaMallocAsync(&g->root_v0, std::max<uint64_t>(m, 1) * sizeof(uint32_t), st));
  MCE_CUDA_TRY(cudaMallocAsync(&g->root_v1, std::max<uint64_t>(m, 1) * sizeof(uint32_t), st));
  k_roots<<<grid_for(m2, 256), 256, 0, st>>>(keys.p, m2, nb, upflag.p, uppos.p, g->root_v0, g->root_v1); note_launch();
  keys.release();

  // 5) labels and their hashes under the new ids
  MCE_CUDA_TRY(cudaMallocAsync(&g->labels, std::max<uint32_t>(n, 1) * sizeof(uint32_t), st));
  MCE_CUDA_TRY(cudaMallocAsync(&g->h1, std::max<uint32_t>(n, 1) * sizeof(uint64_t), st));
  MCE_CUDA_TRY(cudaMallocAsync(&g->h2, std::max<uint32_t>(n, 1) * sizeof(uint64_t), st));
  k_permute_labels<<<grid_for(n, 256), 256, 0, st>>>(labels0, rank.p, n, g->labels, g->h1, g->h2); note_launch();
  MCE_CUDA_TRY(cudaGetLastError());
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  return MCE_OK;
}

// CSR given by the caller (rows sorted).  already_ordered: use ids as given.
mce_status build_from_csr(uint64_t n, const uint32_t *off_d, const uint32_t *adj_d, const uint32_t *labels_d,
                          int already_ordered, int order_kind, uint32_t degeneracy_hint, uint64_t spin_limit,
                          cudaStream_t st, DeviceGraph *g) {
  *g = DeviceGraph{};
  uint32_t m2 = 0;
  MCE_CUDA_TRY(cudaMemcpyAsync(&m2, off_d + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  const uint64_t m = m2 / 2;
  // edges (r < c) and degrees from the CSR
  DevBuf<uint32_t> deg, eu, ev, labels0;
  MCE_TRY(deg.alloc(n + 1, st));
  MCE_TRY(labels0.alloc(n, st));
  if (labels_d)
    MCE_CUDA_TRY(cudaMemcpyAsync(labels0.p, labels_d, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  else
    k_iota<<<grid_for(n, 256), 256, 0, st>>>(labels0.p, n); note_launch();
  MCE_TRY(csr_to_edges(n, off_d, adj_d, m, deg.p, &eu.p, &ev.p, st));
  eu.st = ev.st = st;
  MCE_TRY(finish_graph((uint32_t)n, m, eu.p, ev.p, deg.p, labels0.p,
                       already_ordered ? MCE_ORDER_UNCHANGED : order_kind, spin_limit, st, g));
  if (already_ordered && degeneracy_hint) g->degeneracy = degeneracy_hint;
  return MCE_OK;
}

namespace {
__global__ void k_degrees_from_off(const uint32_t *off, uint64_t n, uint32_t *deg) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    deg[i] = off[i + 1] - off[i];
}
__global__ void k_upper_flags(const uint32_t *off, const uint32_t *adj, uint64_t n, uint32_t *flag) {
  // one warp per row
  const uint32_t lane = lane_id();
  for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n;
       r += ((uint64_t)gridDim.x * blockDim.x) >> 5)
    for (uint32_t e = off[r] + lane; e < off[r + 1]; e += 32) flag[e] = adj[e] > r ? 1u : 0u;
}
__global__ void k_upper_edges(const uint32_t *off, const uint32_t *adj, uint64_t n, const uint32_t *flag,
                              const uint32_t *pos, uint32_t *eu, uint32_t *ev) {
  const uint32_t lane = lane_id();
  for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n;
       r += ((uint64_t)gridDim.x * blockDim.x) >> 5)
    for (uint32_t e = off[r] + lane; e < off[r + 1]; e += 32)
      if (flag[e]) {
        eu[pos[e]] = (uint32_t)r;
        ev[pos[e]] = adj[e];
      }
}
}  // namespace

mce_status csr_to_edges(uint64_t n, const uint32_t *off, const uint32_t *adj, uint64_t m, uint32_t *deg,
                        uint32_t **eu, uint32_t **ev, cudaStream_t st) {
  k_degrees_from_off<<<grid_for(n, 256), 256, 0, st>>>(off, n, deg); note_launch();
  DevBuf<uint32_t> flag, pos;
  MCE_TRY(flag.alloc(2 * m + 1, st));
  MCE_TRY(pos.alloc(2 * m + 1, st));
  k_upper_flags<<<grid_for(n * 32, 256), 256, 0, st>>>(off, adj, n, flag.p); note_launch();
  MCE_TRY(scan_exclusive_u32(flag.p, pos.p, 2 * m, pos.p + 2 * m, st));
  uint32_t mu = 0;
  MCE_TRY(read_scalar(pos.p + 2 * m, &mu, st));
  if (mu != m) return MCE_ERR_FORMAT;  // not symmetric / has self-loops
  MCE_CUDA_TRY(cudaMallocAsync(eu, std::max<uint64_t>(m, 1) * sizeof(uint32_t), st));
  MCE_CUDA_TRY(cudaMallocAsync(ev, std::max<uint64_t>(m, 1) * sizeof(uint32_t), st));
  k_upper_edges<<<grid_for(n * 32, 256), 256, 0, st>>>(off, adj, n, flag.p, pos.p, *eu, *ev); note_launch();
  MCE_CUDA_TRY(cudaGetLastError());
  return MCE_OK;
}

void free_graph(DeviceGraph *g) {
  cudaStream_t st = g->stream;
  cudaFreeAsync(g->off, st);
  cudaFreeAsync(g->adj, st);
  cudaFreeAsync(g->labels, st);
  cudaFreeAsync(g->h1, st);
  cudaFreeAsync(g->h2, st);
  cudaFreeAsync(g->root_v0, st);
  cudaFreeAsync(g->root_v1, st);
  if (g->slot) cudaFreeAsync(g->slot, st);
  *g = DeviceGraph{};
}

}  // namespace mce
