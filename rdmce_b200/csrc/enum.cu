// enum.cu -- edge-rooted bitmap Bron-Kerbosch with pivot on the GPU.
//
// Method (the reference's, src/kernels/BkPivotBitBalance.cuh):
//   root = undirected edge (v0 < v1) in the degeneracy order (:428-469);
//   C = N(v0) & N(v1); P = {c in C : c > v1}, X = {c in C : c < v1};
//   an edge in no triangle is a maximal clique of size 2 (:535-539);
//   ego bitmap: row r = P[r] for r < p, then the X members; bit j = adjacency
//   to P[j]; X rows without a P neighbour are dropped (include/graph_gpu.cuh:59-107);
//   node: pivot = argmin over rows containing R of |P \ row| (:229-257),
//   branch on VP = P \ row(pivot) in ascending order; child P' = P & row(q);
//   EXPAND_R moves every i in P' with |P' \ row(i)| == 1 into R (:368-382);
//   leaf: P empty and no row contains R -> one maximal clique (:276-294).
//
// B200 design differences:
//   * each level keeps the list of rows that contain R ("active rows"), so a
//     pivot scan reads only candidate rows instead of every row with an
//     R-subset test; if the per-warp list space runs out a level inherits its
//     parent's list and falls back to the subset test (never a skipped root);
//   * ties in the pivot go to the lowest row index (canonical, matches the
//     CPU oracle's node counts);
//   * every leaf also feeds a clique-size histogram and the order-independent
//     checksum (mix64 set hash over original labels);
//   * scratch is sized per root: roots whose ego network exceeds the per-warp
//     slab are deferred to a second pass with large slabs, never skipped
//     (the reference prints and skips them, :480-487).
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace mce {

constexpr uint32_t kIdent = 0xffffffffu;  // level-0 list = all rows
constexpr uint32_t kHistCache = 128;      // per-warp shared-memory histogram bins

namespace {

struct WarpAcc {
  // lane-0 accumulators for the current result slot
  unsigned long long count, checksum;
  uint32_t max_size, slot, pending;
};

__device__ __forceinline__ void acc_flush(const EnumParams &P, WarpAcc &a, uint32_t *hcache, uint32_t lane) {
  // all lanes: flush histogram cache; lane 0: flush scalars
  __syncwarp();
  for (uint32_t b = lane; b < kHistCache; b += 32) {
    uint32_t c = hcache[b];
    if (c) {
      uint32_t bin = b < P.hist_len ? b : P.hist_len - 1;
      atomicAdd(&P.hist[(uint64_t)a.slot * P.hist_len + bin], (unsigned long long)c);
      hcache[b] = 0;
    }
  }
  if (lane == 0 && (a.count || a.max_size)) {
    atomicAdd(&P.slots[a.slot].count, a.count);
    atomicAdd(&P.slots[a.slot].checksum, a.checksum);
    atomicMax(&P.slots[a.slot].max_size, a.max_size);
  }
  a.count = 0;
  a.checksum = 0;
  a.max_size = 0;
  a.pending = 0;
  __syncwarp();
}

// lane 0 only
__device__ __forceinline__ void emit(const EnumParams &P, WarpAcc &a, uint32_t *hcache, uint32_t size, uint64_t s1,
                                     uint64_t s2) {
  a.count++;
  a.checksum += clique_hash(s1, s2, size);
  a.max_size = max(a.max_size, size);
  if (size < kHistCache) {
    hcache[size]++;
    a.pending++;
  } else {
    uint32_t bin = size < P.hist_len ? size : P.hist_len - 1;
    atomicAdd(&P.hist[(uint64_t)a.slot * P.hist_len + bin], 1ULL);
  }
}

__host__ __device__ __forceinline__ uint64_t align8(uint64_t x) { return (x + 7) & ~7ULL; }

// Layout of one root inside a warp slab (bytes).
struct RootLayout {
  uint64_t hash_off, rows_off, stack_off, alist_off, alist_cap, need;
};

__device__ __forceinline__ RootLayout layout_for(uint64_t cand_n, uint32_t p, uint32_t x, uint32_t W) {
  RootLayout L;
  L.hash_off = align8(cand_n * 4);
  L.rows_off = L.hash_off + 16ULL * p;
  L.stack_off = L.rows_off + 8ULL * (uint64_t)(p + x) * W;
  L.alist_off = L.stack_off + 8ULL * (uint64_t)(p + 2) * (3ULL * W + 4);
  L.need = L.alist_off + 4ULL * (p + x);  // at least one full-size child list
  L.alist_cap = 0;
  return L;
}

// Solve one ego network already built in the slab.  All lanes participate.
__device__ void solve_ego(const EnumParams &P, WarpAcc &acc, uint32_t *hcache, const uint64_t *rows,
                          const uint64_t *h1s, const uint64_t *h2s, uint64_t *stack, uint32_t *alist,
                          uint64_t alist_cap, uint32_t p, uint32_t nrows, uint32_t W, uint64_t s1_root,
                          uint64_t s2_root) {
  const uint32_t lane = lane_id();
  const uint64_t LREC = 3ULL * W + 4;
  // level 0: P = all p bits, R = 0, active rows = all rows
  for (uint32_t w = lane; w < W; w += 32) {
    uint32_t lo = w * 64;
    stack[w] = (p - lo >= 64) ? ~0ULL : ((1ULL << (p - lo)) - 1);
    stack[W + w] = 0;
    stack[2 * W + w] = 0;
  }
  if (lane == 0) {
    uint64_t *m = stack + 3 * W;
    m[0] = (uint64_t)kIdent | ((uint64_t)nrows << 32);
    m[1] = 0;  // atop 0, rsize 0, not lazy
    m[2] = s1_root;
    m[3] = s2_root;
  }
  __syncwarp();
  int level = 0;
  bool fresh = true;
  for (;;) {
    uint64_t *rec = stack + (uint64_t)level * LREC;
    uint64_t *Pv = rec, *VP = rec + W, *R = rec + 2 * W;
    const uint64_t m0 = rec[3 * W], m1 = rec[3 * W + 1];
    const uint32_t aoff = (uint32_t)m0, alen = (uint32_t)(m0 >> 32);
    const uint32_t atop = (uint32_t)m1, rsize = (uint32_t)(m1 >> 32) & 0x7fffffffu;
    const bool lazy = (m1 >> 63) != 0;
    if (fresh) {
      uint32_t pc = 0;
      for (uint32_t w = lane; w < W; w += 32) pc += __popcll(Pv[w]);
      pc = __reduce_add_sync(kFull, pc);
      if (pc == 0) {
        // leaf: maximal iff no active row contains R
        bool blocked;
        if (!lazy) {
          blocked = alen > 0;
        } else {
          bool hit = false;
          for (uint32_t base = 0; base < alen && !hit; base += 32) {
            uint32_t t = base + lane;
            bool h = false;
            if (t < alen) {
              uint32_t i = aoff == kIdent ? t : alist[aoff + t];
              const uint64_t *row = rows + (uint64_t)i * W;
              h = true;
              for (uint32_t w = 0; w < W; w++)
                if (R[w] & ~row[w]) {
                  h = false;
                  break;
                }
            }
            hit = __any_sync(kFull, h);
          }
          blocked = hit;
        }
        if (!blocked && lane == 0) emit(P, acc, hcache, rsize + 2, rec[3 * W + 2], rec[3 * W + 3]);
        fresh = false;
        if (level == 0) break;
        level--;
        continue;
      }
      // pivot scan over active rows
      uint32_t best_c = 0xffffffffu, best_t = 0xffffffffu;
      for (uint32_t base = 0; base < alen; base += 32) {
        uint32_t t = base + lane;
        if (t < alen) {
          uint32_t i = aoff == kIdent ? t : alist[aoff + t];
          const uint64_t *row = rows + (uint64_t)i * W;
          bool ok = true;
          if (lazy)
            for (uint32_t w = 0; w < W; w++)
              if (R[w] & ~row[w]) {
                ok = false;
                break;
              }
          if (ok) {
            uint32_t c = 0;
            for (uint32_t w = 0; w < W; w++) c += __popcll(Pv[w] & ~row[w]);
            if (c < best_c) {
              best_c = c;
              best_t = t;
            }
          }
        }
        if (__any_sync(kFull, best_c == 0)) break;
      }
      const uint32_t minc = __reduce_min_sync(kFull, best_c);
      if (minc == 0 || minc == 0xffffffffu) {
        // an X row adjacent to all of P: nothing maximal below this node
        fresh = false;
        if (level == 0) break;
        level--;
        continue;
      }
      const uint32_t tmin = __reduce_min_sync(kFull, best_c == minc ? best_t : 0xffffffffu);
      const uint32_t piv = aoff == kIdent ? tmin : alist[aoff + tmin];
      const uint64_t *prow = rows + (uint64_t)piv * W;
      for (uint32_t w = lane; w < W; w += 32) VP[w] = Pv[w] & ~prow[w];
      __syncwarp();
      fresh = false;
      continue;  // pick the first candidate at this level
    }
    // next candidate at this level: first bit of P & VP
    uint32_t q = 0xffffffffu;
    for (uint32_t wb = 0; wb < W; wb += 32) {
      uint32_t w = wb + lane;
      uint64_t val = w < W ? (Pv[w] & VP[w]) : 0;
      uint32_t bal = __ballot_sync(kFull, val != 0);
      if (bal) {
        uint32_t src = __ffs(bal) - 1;
        uint64_t vv = __shfl_sync(kFull, val, src);
        q = (wb + src) * 64 + (__ffsll((long long)vv) - 1);
        break;
      }
    }
    if (q == 0xffffffffu) {
      if (level == 0) break;
      level--;
      continue;
    }
    const uint32_t wq = q >> 6;
    const uint64_t bq = 1ULL << (q & 63);
    if (lane == 0) Pv[wq] &= ~bq;
    __syncwarp();
    // child node
    uint64_t *crec = rec + LREC;
    uint64_t *CP = crec, *CE = crec + W, *CR = crec + 2 * W;
    const uint64_t *rowq = rows + (uint64_t)q * W;
    uint32_t cpc = 0;
    for (uint32_t w = lane; w < W; w += 32) {
      uint64_t cp = Pv[w] & rowq[w];
      CP[w] = cp;
      CR[w] = R[w] | (w == wq ? bq : 0);
      CE[w] = 0;
      cpc += __popcll(cp);
    }
    cpc = __reduce_add_sync(kFull, cpc);
    __syncwarp();
    uint32_t rs = rsize + 1;
    uint64_t t1 = rec[3 * W + 2] + h1s[q], t2 = rec[3 * W + 3] + h2s[q];
    uint32_t nE = 0;
    if (P.expand_r && cpc > 1) {
      uint64_t e1 = 0, e2 = 0;
      uint32_t ne = 0;
      for (uint32_t base = 0; base < p; base += 32) {
        uint32_t i = base + lane;
        bool e = false;
        if (i < p && ((CP[i >> 6] >> (i & 63)) & 1)) {
          const uint64_t *ri = rows + (uint64_t)i * W;
          uint32_t c = 0;
          for (uint32_t w = 0; w < W && c <= 1; w++) c += __popcll(CP[w] & ~ri[w]);
          e = (c == 1);
        }
        uint32_t bal = __ballot_sync(kFull, e);
        if (bal) {
          if (lane == 0) CE[base >> 6] |= (uint64_t)bal << (base & 32);
          if (e) {
            e1 += h1s[i];
            e2 += h2s[i];
            ne++;
          }
        }
      }
      nE = __reduce_add_sync(kFull, ne);
      if (nE) {
        e1 = warp_sum_u64(e1);
        e2 = warp_sum_u64(e2);
        __syncwarp();
        for (uint32_t w = lane; w < W; w += 32) {
          uint64_t ew = CE[w];
          CP[w] &= ~ew;
          CR[w] |= ew;
        }
        rs += nE;
        t1 += e1;
        t2 += e2;
      }
    }
    __syncwarp();
    // child active rows
    uint32_t caoff, calen, catop;
    bool clazy;
    if ((uint64_t)atop + alen <= alist_cap) {
      uint32_t n2 = 0;
      const bool single = !lazy && nE == 0;
      for (uint32_t base = 0; base < alen; base += 32) {
        uint32_t t = base + lane;
        bool keep = false;
        uint32_t i = 0;
        if (t < alen) {
          i = aoff == kIdent ? t : alist[aoff + t];
          const uint64_t *row = rows + (uint64_t)i * W;
          if (single) {
            keep = (row[wq] & bq) != 0;
          } else if (!lazy) {
            keep = (row[wq] & bq) != 0;
            for (uint32_t w = 0; w < W && keep; w++) keep = (row[w] & CE[w]) == CE[w];
          } else {
            keep = true;
            for (uint32_t w = 0; w < W && keep; w++) keep = (row[w] & CR[w]) == CR[w];
          }
        }
        uint32_t bal = __ballot_sync(kFull, keep);
        if (keep) alist[atop + n2 + __popc(bal & lanemask_lt())] = i;
        n2 += __popc(bal);
      }
      caoff = atop;
      calen = n2;
      catop = atop + n2;
      clazy = false;
    } else {
      caoff = aoff;
      calen = alen;
      catop = atop;
      clazy = true;
    }
    if (lane == 0) {
      crec[3 * W] = (uint64_t)caoff | ((uint64_t)calen << 32);
      crec[3 * W + 1] = (uint64_t)catop | ((uint64_t)rs << 32) | (clazy ? (1ULL << 63) : 0);
      crec[3 * W + 2] = t1;
      crec[3 * W + 3] = t2;
    }
    __syncwarp();
    level++;
    fresh = true;
  }
}

// Candidate list C = N(v0) & N(v1) (sorted) into cand[]; returns |C| or
// 0xffffffff if more than cap.
__device__ uint32_t intersect(const DevGraph &g, uint32_t v0, uint32_t v1, uint32_t *cand, uint64_t cap) {
  const uint32_t lane = lane_id();
  const uint32_t *a = g.adj + g.off[v0], *b = g.adj + g.off[v1];
  uint32_t da = g.off[v0 + 1] - g.off[v0], db = g.off[v1 + 1] - g.off[v1];
  if (da > db) {
    const uint32_t *t = a;
    a = b;
    b = t;
    uint32_t td = da;
    da = db;
    db = td;
  }
  uint32_t nc = 0;
  for (uint32_t base = 0; base < da; base += 32) {
    uint32_t t = base + lane;
    uint32_t val = t < da ? __ldg(a + t) : 0;
    bool hit = t < da && val != v0 && val != v1 && contains_u32(b, db, val);
    uint32_t bal = __ballot_sync(kFull, hit);
    if (nc + __popc(bal) > cap) return 0xffffffffu;
    if (hit) cand[nc + __popc(bal & lanemask_lt())] = val;
    nc += __popc(bal);
  }
  __syncwarp();
  return nc;
}

// Build the ego bitmap.  Returns number of rows kept (P rows + X rows with a
// P neighbour).  rowbuf: per-warp shared buffer of 64 words.
__device__ uint32_t build_rows(const DevGraph &g, const uint32_t *cand, uint32_t x, uint32_t p, uint32_t W,
                               uint64_t *rows, uint64_t *rowbuf) {
  const uint32_t lane = lane_id();
  const uint32_t *Pl = cand + x;
  const uint32_t pmin = Pl[0], pmax = Pl[p - 1];
  uint32_t nrows = 0;
  for (uint32_t r = 0; r < p + x; r++) {
    const uint32_t u = r < p ? Pl[r] : cand[r - p];
    const uint32_t *nu = g.adj + g.off[u];
    const uint32_t du = g.off[u + 1] - g.off[u];
    uint64_t *row = rows + (uint64_t)nrows * W;
    // restrict N(u) to [pmin, pmax]
    uint32_t lo = 0, hi = 0;
    if (lane == 0) {
      lo = lower_bound_u32(nu, du, pmin);
      hi = lower_bound_u32(nu, du, pmax + 1);
    }
    lo = __shfl_sync(kFull, lo, 0);
    hi = __shfl_sync(kFull, hi, 0);
    bool any;
    if (hi - lo < p && W <= 64) {
      // lanes over N(u) slice, binary search in P, OR into shared row
      for (uint32_t w = lane; w < W; w += 32) rowbuf[w] = 0;
      __syncwarp();
      bool hit = false;
      for (uint32_t e = lo + lane; e < hi; e += 32) {
        uint32_t y = __ldg(nu + e);
        uint32_t j = lower_bound_u32(Pl, p, y);
        if (j < p && Pl[j] == y) {
          atomicOr((unsigned long long *)&rowbuf[j >> 6], 1ULL << (j & 63));
          hit = true;
        }
      }
      any = __any_sync(kFull, hit);
      __syncwarp();
      for (uint32_t w = lane; w < W; w += 32) row[w] = rowbuf[w];
    } else {
      // lanes over P, binary search in the N(u) slice
      uint64_t word = 0;
      bool hitany = false;
      const uint32_t *sl = nu + lo;
      const uint32_t sn = hi - lo;
      for (uint32_t base = 0; base < p; base += 32) {
        uint32_t j = base + lane;
        bool hit = j < p && contains_u32(sl, sn, Pl[j]);
        uint32_t bal = __ballot_sync(kFull, hit);
        hitany |= bal != 0;
        if (base & 32) {
          word |= (uint64_t)bal << 32;
          if (lane == 0) row[base >> 6] = word;
        } else {
          word = bal;
          if (base + 32 >= p && lane == 0) row[base >> 6] = word;
        }
      }
      any = hitany;
    }
    __syncwarp();
    if (r < p || any) nrows++;
  }
  return nrows;
}

__global__ void __launch_bounds__(256, 2) k_enumerate(EnumParams P) {
  extern __shared__ uint64_t smem[];
  const uint32_t lane = lane_id();
  const uint32_t wib = threadIdx.x >> 5;
  const uint64_t gwarp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint64_t *rowbuf = smem + wib * 64;
  uint32_t *hcache = (uint32_t *)(smem + (blockDim.x >> 5) * 64) + wib * kHistCache;
  for (uint32_t b = lane; b < kHistCache; b += 32) hcache[b] = 0;
  WarpAcc acc{0, 0, 0, 0, 0};
  char *slab = P.slab + gwarp * P.slab_bytes;
  const bool range_mode = P.heavy_list == nullptr && P.root_list == nullptr;
  const uint64_t total = range_mode ? P.re - P.rb : P.n_list;
  unsigned long long nroots = 0;
  __syncwarp();
  for (;;) {
    unsigned long long k = 0;
    if (lane == 0) k = atomicAdd(P.next, 1ULL);
    k = __shfl_sync(kFull, k, 0);
    if (k >= total) break;
    uint64_t r;
    if (P.heavy_list) r = P.heavy_list[k];
    else if (P.root_list) r = P.root_list[k];
    else r = P.re - 1 - k;  // heavy (late-peeled) roots first
    const uint32_t v0 = P.g.root_v0[r], v1 = P.g.root_v1[r];
    const uint32_t slot = P.g.slot ? P.g.slot[v0] : 0;
    if (slot != acc.slot) {
      acc_flush(P, acc, hcache, lane);
      acc.slot = slot;
    }
    const unsigned long long c_before = acc.count, h_before = acc.checksum;
    nroots++;
    uint32_t *cand = (uint32_t *)slab;
    const uint32_t nc = intersect(P.g, v0, v1, cand, P.slab_bytes / 4);
    bool deferred = false;
    if (nc == 0xffffffffu) {
      deferred = true;
      if (P.push_heavy && lane == 0) {
        P.heavy_out[atomicAdd(P.heavy_n, 1u)] = (uint32_t)r;
        uint32_t dmin = min(P.g.off[v0 + 1] - P.g.off[v0], P.g.off[v1 + 1] - P.g.off[v1]);
        atomicMax(P.heavy_need, (unsigned long long)layout_for(dmin, dmin, dmin, (dmin + 63) / 64).need);
      } else if (!P.push_heavy && lane == 0) {
        atomicExch(P.error, 2u);  // does not fit even the large slab
      }
    } else {
      const uint32_t x = nc ? lower_bound_u32(cand, nc, v1) : 0;
      const uint32_t p = nc - x;
      const uint64_t s1 = P.g.h1[v0] + P.g.h1[v1], s2 = P.g.h2[v0] + P.g.h2[v1];
      if (p == 0) {
        if (x == 0 && lane == 0) emit(P, acc, hcache, 2, s1, s2);
      } else {
        const uint32_t W = (p + 63) / 64;
        const RootLayout L = layout_for(nc, p, x, W);
        if (L.need > P.slab_bytes) {
          deferred = true;
          if (lane == 0) {
            if (P.push_heavy) {
              P.heavy_out[atomicAdd(P.heavy_n, 1u)] = (uint32_t)r;
              atomicMax(P.heavy_need, (unsigned long long)L.need);
            } else {
              atomicExch(P.error, 2u);
            }
          }
        } else {
          uint64_t *h1s = (uint64_t *)(slab + L.hash_off);
          uint64_t *h2s = h1s + p;
          uint64_t *rows = (uint64_t *)(slab + L.rows_off);
          uint64_t *stack = (uint64_t *)(slab + L.stack_off);
          uint32_t *alist = (uint32_t *)(slab + L.alist_off);
          const uint64_t alist_cap = (P.slab_bytes - L.alist_off) / 4;
          for (uint32_t j = lane; j < p; j += 32) {
            uint32_t y = cand[x + j];
            h1s[j] = P.g.h1[y];
            h2s[j] = P.g.h2[y];
          }
          const uint32_t nrows = build_rows(P.g, cand, x, p, W, rows, rowbuf);
          __syncwarp();
          solve_ego(P, acc, hcache, rows, h1s, h2s, stack, alist, alist_cap, p, nrows, W, s1, s2);
        }
      }
    }
    if (lane == 0 && acc.pending > (1u << 30)) acc.pending = kFull;  // force flush below
    if (__shfl_sync(kFull, acc.pending, 0) == kFull) acc_flush(P, acc, hcache, lane);
    if (P.per_root_count && lane == 0) {
      P.per_root_count[k] = deferred ? ~0ULL : acc.count - c_before;
      P.per_root_checksum[k] = acc.checksum - h_before;
    }
    __syncwarp();
  }
  acc.pending = 0;
  acc_flush(P, acc, hcache, lane);
  if (lane == 0) atomicAdd(P.stat_roots, nroots);
}

}  // namespace

struct EnumCtl {
  unsigned long long next, heavy_need, stat_roots, pad;
  unsigned int heavy_n, error, pad2[2];
};

mce_status enum_plan(const DeviceGraph &g, const EnumConfig &cfg, Scratch *scr, SlotResult *slots,
                     unsigned long long *hist, EnumPlan *plan) {
  const int device = scr->device;
  int sms = 0;
  MCE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const uint32_t wpb = cfg.warps_per_block ? std::min(cfg.warps_per_block, 8u) : 8u;
  const uint32_t bps = cfg.blocks_per_sm ? cfg.blocks_per_sm : 2u;
  EnumParams &P = plan->params;
  P = EnumParams{};
  P.g.n = g.n;
  P.g.m = g.m;
  P.g.off = g.off;
  P.g.adj = g.adj;
  P.g.labels = g.labels;
  P.g.h1 = g.h1;
  P.g.h2 = g.h2;
  P.g.root_v0 = g.root_v0;
  P.g.root_v1 = g.root_v1;
  P.g.slot = g.slot;
  P.slots = slots;
  P.hist = hist;
  P.hist_len = cfg.hist_len;
  P.expand_r = cfg.expand_r;
  P.per_root_count = cfg.per_root_count;
  P.per_root_checksum = cfg.per_root_checksum;
  mce_status s = MCE_OK;
  EnumCtl *ctl = (EnumCtl *)scr->get(1, sizeof(EnumCtl), &s);
  if (!ctl) return s;
  plan->ctl = ctl;
  P.next = &ctl->next;
  P.heavy_need = &ctl->heavy_need;
  P.heavy_n = &ctl->heavy_n;
  P.error = &ctl->error;
  P.stat_roots = &ctl->stat_roots;

  uint64_t rb = cfg.root_begin, re = cfg.root_end ? std::min<uint64_t>(cfg.root_end, g.m) : g.m;
  if (rb > re) rb = re;
  const bool list_mode = cfg.root_list != nullptr;
  const uint64_t nwork = list_mode ? cfg.n_root_list : re - rb;
  plan->nwork = nwork;

  uint32_t blocks = (uint32_t)sms * bps;
  if (cfg.max_blocks && blocks > cfg.max_blocks) blocks = cfg.max_blocks;
  // never more warps than roots
  const uint64_t want_blocks = (nwork + wpb - 1) / wpb;
  if (want_blocks < blocks) blocks = (uint32_t)std::max<uint64_t>(want_blocks, 1);
  const uint64_t nwarps = (uint64_t)blocks * wpb;
  // normal-pass slab: the largest ego network this graph can produce (p <= the
  // degeneracy, x <= the max degree), capped at 4 MB per warp and by free memory
  size_t freeb = 0, totalb = 0;
  MCE_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
  const uint64_t kcap = std::max<uint32_t>(1, std::min(g.degeneracy, g.max_degree));
  const uint64_t dcap = std::max<uint32_t>(1, g.max_degree);
  const uint64_t wcap = (kcap + 63) / 64;
  const uint64_t bound = align8(dcap * 4) + 16 * kcap + 8 * (kcap + dcap) * wcap + 8 * (kcap + 2) * (3 * wcap + 4) +
                         4 * (kcap + dcap) * 4 + 1024;
  uint64_t slab_bytes = std::min<uint64_t>(align8(bound), 4ULL << 20);
  while (slab_bytes > (64ULL << 10) && slab_bytes * nwarps > freeb / 2) slab_bytes >>= 1;
  plan->fits_all = slab_bytes >= align8(bound);
  char *slab = (char *)scr->get(2, slab_bytes * nwarps, &s);
  if (!slab) return s;
  uint32_t *heavy = nullptr;
  if (!list_mode && nwork) {
    heavy = (uint32_t *)scr->get(3, nwork * 4, &s);
    if (!heavy) return s;
  }
  P.slab = slab;
  P.slab_bytes = slab_bytes;
  P.rb = rb;
  P.re = re;
  P.root_list = list_mode ? cfg.root_list : nullptr;
  P.n_list = list_mode ? cfg.n_root_list : 0;
  P.heavy_out = heavy;
  P.push_heavy = list_mode ? 0 : 1;
  plan->blocks = blocks;
  plan->threads = wpb * 32;
  plan->smem = (size_t)wpb * 64 * 8 + (size_t)wpb * kHistCache * 4;
  plan->nwarps = nwarps;
  plan->scr = scr;
  return MCE_OK;
}

mce_status enum_launch(const EnumPlan &plan, cudaStream_t st) {
  MCE_CUDA_TRY(cudaMemsetAsync(plan.ctl, 0, sizeof(EnumCtl), st));
  if (plan.nwork) {
    k_enumerate<<<plan.blocks, plan.threads, plan.smem, st>>>(plan.params);
    MCE_CUDA_TRY(cudaGetLastError());
  }
  return MCE_OK;
}

mce_status enum_finish(const EnumPlan &plan, cudaStream_t st, EnumStats *stats) {
  EnumCtl *ctl = (EnumCtl *)plan.ctl;
  EnumCtl h{};
  MCE_CUDA_TRY(cudaMemcpyAsync(&h, ctl, sizeof(EnumCtl), cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  const uint64_t heavy_roots = h.heavy_n;
  uint64_t launches = plan.nwork ? 1 : 0;
  uint64_t roots = h.stat_roots;
  if (h.heavy_n && !h.error) {
    // heavy pass: large slabs, fewer warps
    size_t freeb = 0, totalb = 0;
    MCE_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
    const uint64_t need = align8(h.heavy_need) + 4096;
    const uint64_t hw = std::min<uint64_t>({(uint64_t)h.heavy_n, (uint64_t)(freeb * 0.8) / need, plan.nwarps});
    if (hw == 0) return MCE_ERR_OUT_OF_MEMORY;
    mce_status s = MCE_OK;
    char *big = (char *)plan.scr->get(4, need * hw, &s);
    if (!big) return s;
    EnumParams H = plan.params;
    H.slab = big;
    H.slab_bytes = need;
    H.heavy_list = plan.params.heavy_out;
    H.root_list = nullptr;
    H.n_list = h.heavy_n;
    H.push_heavy = 0;
    MCE_CUDA_TRY(cudaMemsetAsync(&ctl->next, 0, sizeof(unsigned long long), st));
    MCE_CUDA_TRY(cudaMemsetAsync(&ctl->stat_roots, 0, sizeof(unsigned long long), st));
    const uint32_t wpb = plan.threads / 32;
    const uint32_t hb = (uint32_t)((hw + wpb - 1) / wpb);
    k_enumerate<<<hb, plan.threads, plan.smem, st>>>(H);
    launches++;
    MCE_CUDA_TRY(cudaGetLastError());
    MCE_CUDA_TRY(cudaMemcpyAsync(&h, ctl, sizeof(EnumCtl), cudaMemcpyDeviceToHost, st));
    MCE_CUDA_TRY(cudaStreamSynchronize(st));
    roots = roots - heavy_roots + h.stat_roots;
  }
  if (stats) {
    stats->roots = roots;
    stats->heavy_roots = heavy_roots;
    stats->error = h.error;
    stats->launches = launches;
  }
  if (h.error == 2) return MCE_ERR_OUT_OF_MEMORY;
  if (h.error) return MCE_ERR_TIMEOUT;
  return MCE_OK;
}

mce_status enumerate(const DeviceGraph &g, const EnumConfig &cfg, Scratch *scr, cudaStream_t st, SlotResult *slots,
                     unsigned long long *hist, EnumStats *stats) {
  EnumPlan plan;
  MCE_TRY(enum_plan(g, cfg, scr, slots, hist, &plan));
  cudaEvent_t e0, e1;
  MCE_CUDA_TRY(cudaEventCreate(&e0));
  MCE_CUDA_TRY(cudaEventCreate(&e1));
  cudaEventRecord(e0, st);
  mce_status s = enum_launch(plan, st);
  if (s == MCE_OK) s = enum_finish(plan, st, stats);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (stats) stats->ms_enum = ms;
  return s;
}

}  // namespace mce
