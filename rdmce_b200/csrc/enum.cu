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
//   leaf: P empty and no row contains R -> one maximal clique (:276-294);
//   root-down exposure: the shallowest level with open candidates is handed
//   to other warps when they run dry (:87-138, :552-598).
//
// B200 design:
//   * Three tiers by subproblem size.  Nearly every search-tree node has at
//     most 32 candidate columns and 32 rows that contain R: there each lane
//     holds one row as a 32-bit word, P / VP / the active-row set are
//     warp-uniform 32-bit masks, and a node is one redux.sync (pivot argmin),
//     two ballots (EXPAND_R, the child's active rows) and a few shuffles.  Up to 64
//     columns and 128 rows, each lane holds 4 rows as 64-bit words.  Larger
//     subproblems run in the general tier (W 64-bit words per row in a global
//     scratch slab, per-level lists of active rows).  A child small enough for
//     a smaller tier has its rows compressed to its own columns (parallel bit
//     compress) and gathered, and continues there.
//   * In the 32-bit tier R is a column mask and leaves are hashed 32 at a
//     time, one per lane.  A node or child with at most 5 candidates is
//     decided in one step: its maximal cliques are the cliques K of the
//     candidates that no active row contains, and lane i tests the i-th
//     subset.  The node loop makes no calls; to expose work it steps out
//     and is resumed.
//   * Root-down exposure with self-contained tasks.  When warps are idle, a
//     busy warp turns every open candidate of the shallowest open level with
//     |P| >= tau -- outer tiers of a nested solve first -- into a task record
//     (rows restricted to the child's columns, X rows empty on them left out)
//     in a global pool, published through lock-free bounded MPMC rings.  A
//     task owns its data, so no warp ever waits on another warp's stack (the
//     reference's owner waits for its thieves, :87-138).  Every wait is bounded.
//   * Pivot ties go to the lowest row index; every leaf feeds the clique-size
//     histogram and the order-independent checksum.
//   * Roots whose ego network exceeds the per-warp slab are deferred to a
//     second pass with large slabs, never skipped (the reference prints and
//     skips them, :480-487).
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"

// This file is compiled once per register budget of the enumeration kernel:
// MCE_ENUM_BPS resident 8-warp blocks per SM (3, 4 or 5: at most 85, 64 or 51
// registers a thread).  Each build keeps its own copies of the device
// functions, so one budget never forces spills on another; enum_dispatch.cu
// picks the build per solve (the autotuner's occupancy choice).
#ifndef MCE_ENUM_BPS
#define MCE_ENUM_BPS 4
#endif
#define MCE_CAT2(a, b) a##b
#define MCE_CAT(a, b) MCE_CAT2(a, b)
#define MCE_ENUM_FN(name) MCE_CAT(name, MCE_CAT(_b, MCE_ENUM_BPS))

namespace mce {

namespace {

constexpr uint32_t kIdent = 0xffffffffu;  // level-0 list = all rows
constexpr uint32_t kHistCache = 128;      // per-warp shared-memory histogram bins
constexpr int kRPL = 4;                   // 64-bit tier: rows per lane
constexpr uint32_t kT1Rows = 32 * kRPL;   // 64-bit tier: rows per subproblem
constexpr uint32_t kT1Depth = 66;         // 64-bit tier: levels (<= 64 columns + root)
constexpr uint32_t kT0Depth = 34;         // 32-bit tier: levels (<= 32 columns + root)
constexpr uint32_t kHdr = 64;             // task record header bytes
constexpr uint32_t kLocalRec = 2048;      // per-warp local task record (64-bit-tier size)
// Default tau inside the register tiers (64 or fewer candidates): the same 24
// as the general tier measured as fast as smaller values on R-MAT inputs,
// with fewer, larger tasks, once nested tiers expose their outer levels first.
constexpr uint32_t kRegShareBound = 24;
constexpr uint32_t kShareMin = 128, kShareMax = 8192;
// 32-bit-tier nodes with this few candidates (5, 6 or 7) are decided in one
// step.  Larger limits take more nodes off the search tree but grow the node
// loop's code (the instruction cache bounds the kernel): 6 measured as fast
// as 5 where the join decision below takes most nodes, and 7 % faster where
// it does not (active rows outside P); 7 was slower.
#ifndef MCE_SMALL_P
#define MCE_SMALL_P 6
#endif
constexpr int kSmallP = MCE_SMALL_P;
static_assert(kSmallP >= 5 && kSmallP <= 7, "small-node decisions cover up to 5, 6 or 7 candidates");
// phases of the per-warp cycle accounting
// (kCycReg: the 64-bit tier; kCycT0: the 32-bit tier)
enum { kCycBuild = 0, kCycReg = 1, kCycGen = 2, kCycSpawn = 3, kCycIdle = 4, kCycQueue = 5, kCycT0 = 6, kCycPhases = 7 };

struct TaskHdr {
  uint32_t pc;     // candidate columns
  uint32_t nrows;  // rows: pc candidate rows, then the X rows
  uint32_t W;      // 64-bit words per row
  uint32_t rsize;  // |R| beyond the root edge
  uint64_t s1, s2; // label-hash sums of the clique so far (root edge included)
  uint32_t slot;   // result slot
  uint32_t pad0;
  uint64_t pad[3];
};
static_assert(sizeof(TaskHdr) == kHdr, "task header is 64 bytes");

__host__ __device__ __forceinline__ uint64_t align8(uint64_t x) { return (x + 7) & ~7ULL; }

__host__ __device__ __forceinline__ uint64_t task_bytes(uint32_t pc, uint32_t nrows, uint32_t W) {
  return kHdr + align8(4ULL * pc) + 8ULL * nrows * W;
}

// A general-tier subproblem laid out in the warp's slab.
struct Gen {
  const uint64_t *rows;
  const uint32_t *colv;
  const uint64_t *h1s, *h2s;
  uint64_t *stack;
  uint32_t *alist;
  uint64_t alist_cap;
  uint32_t pc, nrows, W;
};

// Per-warp shared memory.  All mutable per-warp state outside the tier loops
// lives here (lane 0 updates the scalars), so the small Ctx handle can be
// passed by value.
struct WarpSmem {
  uint64_t rowbuf[64];
  // 32-bit tier frames: (P, VP, active rows, R as a column mask)
  uint4 t0f[kT0Depth];
  // exchange buffer for moving a subproblem into the 32-bit tier; xh1/xh2
  // hold the label hashes of the running 32-bit-tier subproblem's columns
  uint32_t xrow[32], xcv[32];
  uint64_t xh1[32], xh2[32];
  // the running 32-bit-tier subproblem's hash sums and |R| at entry, and the
  // R masks of leaves not yet hashed
  uint64_t t0_s1, t0_s2;
  uint32_t t0_rsize;
  uint32_t pend_rm[32];
  uint64_t lchk[32];  // per-lane checksum accumulators (batched leaves)
  // a 32-bit-tier solve that stepped out to expose work: its node state
  uint32_t y_P, y_A, y_RM, y_npend;
  int y_level;
  // nodes between the 32-bit tier's checks for idle warps; doubles (up to
  // kShareMax) while checks find nothing to expose, back to kShareMin after
  // one does
  uint32_t share_period;
  uint32_t hcache[kHistCache];
  // result accumulators for the current slot
  unsigned long long count, checksum, nodes, wops, bbytes;
  uint32_t max_size, slot, pending, pad;
  unsigned long long cyc[kCycPhases];  // clock64 cycles by phase
  // The tiers enclosing the running subproblem.  A nested tier exposes their
  // open levels (shallower, so larger) before its own: the running
  // general-tier solve, and the level each enclosing tier is expanding (the
  // 64-bit tier's rows are in its T1Area).
  Gen gen;
  int t1_level, gen_level;
  uint32_t t1_pc;
  uint32_t nest;  // bit 0: a general-tier solve is running; bit 1: a 64-bit-tier solve
};

constexpr uint32_t kNestGen = 1, kNestT1 = 2;

// The 64-bit tier's frames and rows live at the tail of the warp's slab, not
// in shared memory: that tier holds few of the nodes, and shared memory kept
// small lets 4 blocks of 8 warps share an SM.
struct T1Area {
  uint64_t fP[kT1Depth], fVP[kT1Depth], fs1[kT1Depth], fs2[kT1Depth];
  uint32_t frs[kT1Depth];
  uint8_t fab[kT1Depth][32];
  uint64_t t1rows[kT1Rows];
  uint32_t t1cv[64];
};
constexpr uint32_t kT1Area = (sizeof(T1Area) + 255) & ~255u;
constexpr uint32_t kTail = kLocalRec + kT1Area;  // slab bytes reserved at its end

// Slab layout of a general-tier problem (bytes from the slab start).
struct Layout {
  uint64_t colv_off, hash_off, rows_off, stack_off, alist_off, need;
};

__host__ __device__ __forceinline__ Layout layout_for(uint64_t cand_n, uint32_t pc, uint32_t nrows, uint32_t W) {
  Layout L;
  L.colv_off = 0;
  L.hash_off = align8(4ULL * cand_n);
  L.rows_off = L.hash_off + 16ULL * pc;
  L.stack_off = L.rows_off + 8ULL * (uint64_t)nrows * W;
  // pc + 1 levels, one scratch record past the deepest, one spare
  L.alist_off = L.stack_off + 8ULL * (uint64_t)(pc + 3) * (3ULL * W + 4);
  L.need = L.alist_off + 4ULL * nrows + kTail;
  return L;
}

struct Ctx {
  const EnumParams *P;
  WarpSmem *sm;
  T1Area *ta;
  char *slab;
  uint64_t slab_bytes;
  uint32_t lane;
  bool sharing;
};

__device__ __forceinline__ unsigned long long now() { return clock64(); }

// Task records travel between SMs through reused pool blocks; read them from
// L2 (ld.global.cg) so no SM sees a stale L1 line of an earlier task.
__device__ __forceinline__ uint64_t ld_cg(const uint64_t *p) { return __ldcg((const unsigned long long *)p); }
__device__ __forceinline__ uint32_t ld_cg(const uint32_t *p) { return __ldcg((const unsigned int *)p); }

// ------------------------------------------------------------ accounting

__device__ __forceinline__ void acc_flush(const Ctx &c) {
  const EnumParams &P = *c.P;
  WarpSmem *sm = c.sm;
  __syncwarp();
  const uint64_t lc = warp_sum_u64(sm->lchk[c.lane]);
  sm->lchk[c.lane] = 0;
  if (c.lane == 0) sm->checksum += lc;
  __syncwarp();
  for (uint32_t b = c.lane; b < kHistCache; b += 32) {
    const uint32_t n = sm->hcache[b];
    if (n) {
      const uint32_t bin = b < P.hist_len ? b : P.hist_len - 1;
      atomicAdd(&P.hist[(uint64_t)sm->slot * P.hist_len + bin], (unsigned long long)n);
      sm->hcache[b] = 0;
    }
  }
  if (c.lane == 0) {
    if (sm->count || sm->max_size) {
      atomicAdd(&P.slots[sm->slot].count, sm->count);
      atomicAdd(&P.slots[sm->slot].checksum, sm->checksum);
      atomicMax(&P.slots[sm->slot].max_size, sm->max_size);
    }
    sm->count = 0;
    sm->checksum = 0;
    sm->max_size = 0;
    sm->pending = 0;
  }
  __syncwarp();
}

__device__ __forceinline__ void set_slot(const Ctx &c, uint32_t slot) {
  if (c.sm->slot != slot) {
    acc_flush(c);
    if (c.lane == 0) c.sm->slot = slot;
    __syncwarp();
  }
}

// lane 0 only
__device__ __forceinline__ void emit(const Ctx &c, uint32_t size, uint64_t s1, uint64_t s2) {
  WarpSmem *sm = c.sm;
  sm->count++;
  sm->checksum += clique_hash(s1, s2, size);
  sm->max_size = max(sm->max_size, size);
  if (size < kHistCache) {
    sm->hcache[size]++;
    sm->pending++;
  } else {
    const EnumParams &P = *c.P;
    const uint32_t bin = size < P.hist_len ? size : P.hist_len - 1;
    atomicAdd(&P.hist[(uint64_t)sm->slot * P.hist_len + bin], 1ULL);
  }
}

__device__ __forceinline__ void maybe_flush(const Ctx &c) {
  // keeps every u32 histogram bin far from overflow
  if (c.sm->pending > (1u << 30)) acc_flush(c);
}

// ------------------------------------------------------- bounded MPMC rings
// Vyukov's bounded queue: cell seq == pos means free for the producer of pos,
// seq == pos + 1 means filled for the consumer of pos.  Lane 0 only.

__device__ bool ring_push(uint32_t *slots, unsigned long long *seq, unsigned long long *tail, uint32_t mask,
                          uint32_t val, const EnumParams &P) {
  const unsigned long long pos = atomicAdd(tail, 1ULL);
  volatile unsigned long long *s = seq + (pos & mask);
  uint64_t n = 0;
  while (*s != pos) {
    if (++n > P.spin_limit) {
      atomicExch(P.error, 3u);
      return false;
    }
    __nanosleep(64);
  }
  ((volatile uint32_t *)slots)[pos & mask] = val;
  __threadfence();
  *s = pos + 1;
  return true;
}

__device__ bool ring_pop(uint32_t *slots, unsigned long long *seq, unsigned long long *head,
                         unsigned long long *tail, uint32_t mask, uint32_t *val, const EnumParams &P) {
  for (int tries = 0; tries < 8; tries++) {
    const unsigned long long h = *(volatile unsigned long long *)head;
    const unsigned long long t = *(volatile unsigned long long *)tail;
    if (h >= t) return false;
    if (atomicCAS(head, h, h + 1) == h) {
      volatile unsigned long long *s = seq + (h & mask);
      uint64_t n = 0;
      while (*s != h + 1) {
        if (++n > P.spin_limit) {
          atomicExch(P.error, 3u);
          return false;
        }
        __nanosleep(32);
      }
      __threadfence();
      *val = ((volatile uint32_t *)slots)[h & mask];
      __threadfence();
      *s = h + (unsigned long long)mask + 1;
      return true;
    }
  }
  return false;
}

// warp-uniform wrappers
__device__ __forceinline__ bool pool_alloc(const Ctx &c, uint32_t *blk) {
  const EnumParams &P = *c.P;
  uint32_t b = 0;
  bool ok = false;
  if (c.lane == 0) ok = ring_pop(P.free_slot, P.free_seq, P.free_head, P.free_tail, P.pool_mask, &b, P);
  ok = __shfl_sync(kFull, ok, 0);
  *blk = __shfl_sync(kFull, b, 0);
  return ok;
}

__device__ __forceinline__ void pool_free(const Ctx &c, uint32_t blk) {
  const EnumParams &P = *c.P;
  __syncwarp();
  if (c.lane == 0) ring_push(P.free_slot, P.free_seq, P.free_tail, P.pool_mask, blk, P);
  __syncwarp();
}

__device__ __forceinline__ void pool_publish(const Ctx &c, uint32_t blk) {
  const EnumParams &P = *c.P;
  __threadfence();
  __syncwarp();
  if (c.lane == 0) {
    __threadfence();
    ring_push(P.ready_slot, P.ready_seq, P.ready_tail, P.pool_mask, blk, P);
    atomicAdd(P.stat_tasks, 1ULL);
  }
  __syncwarp();
}

__device__ __forceinline__ char *pool_block(const EnumParams &P, uint32_t blk) {
  return P.pool + (uint64_t)blk * P.block_bytes;
}

// busy warps expose work when some warps are idle and the queue is short
__device__ __forceinline__ bool hungry(const Ctx &c) {
  const EnumParams &P = *c.P;
  uint32_t h = 0;
  if (c.lane == 0) {
    const uint32_t active = *(volatile unsigned int *)P.active;
    const unsigned long long rh = *(volatile unsigned long long *)P.ready_head;
    const unsigned long long rt = *(volatile unsigned long long *)P.ready_tail;
    const uint64_t queued = rt > rh ? rt - rh : 0;
    const uint32_t idle = P.nwarps > active ? P.nwarps - active : 0;
    h = idle > 0 && queued < idle;
  }
  return __shfl_sync(kFull, h, 0) != 0;
}

// ------------------------------------------------------- bit compression
// compress(x, m): the bits of x at the set positions of m, packed to the low
// end (Hacker's Delight 2nd ed. section 7-4, parallel-suffix form).  The plan
// depends only on m, which is warp-uniform wherever it is used.

struct CPlan {
  uint64_t m;
  uint64_t mv[6];
};

__device__ __forceinline__ CPlan compress_plan(uint64_t m) {
  CPlan p;
  p.m = m;
  uint64_t mk = ~m << 1;
#pragma unroll
  for (int i = 0; i < 6; i++) {
    uint64_t mp = mk ^ (mk << 1);
    mp ^= mp << 2;
    mp ^= mp << 4;
    mp ^= mp << 8;
    mp ^= mp << 16;
    mp ^= mp << 32;
    const uint64_t mv = mp & m;
    p.mv[i] = mv;
    m = (m ^ mv) | (mv >> (1 << i));
    mk = mk & ~mp;
  }
  return p;
}

__device__ __forceinline__ uint64_t compress_apply(uint64_t x, const CPlan &p) {
  x &= p.m;
#pragma unroll
  for (int i = 0; i < 6; i++) {
    const uint64_t t = x & p.mv[i];
    x = (x ^ t) | (t >> (1 << i));
  }
  return x;
}

// multi-word row compaction: out[0..W') = bits of row[0..W) at mask[0..W)
__device__ __forceinline__ void compress_row(const uint64_t *row, const uint64_t *mask, uint32_t W, uint64_t *out) {
  uint64_t cur = 0;
  uint32_t cb = 0, wi = 0;
  for (uint32_t w = 0; w < W; w++) {
    const uint64_t m = mask[w];
    const uint32_t n = __popcll(m);
    if (n == 0) continue;
    const uint64_t c = compress_apply(row[w], compress_plan(m));
    cur |= c << cb;
    if (cb + n >= 64) {
      out[wi++] = cur;
      cur = cb ? (c >> (64 - cb)) : 0;
      cb = cb + n - 64;
    } else {
      cb += n;
    }
  }
  if (cb) out[wi] = cur;
}

// Expose open levels of the enclosing general-tier / 64-bit-tier solve, if one
// is running; true if anything was exposed.  Defined after those tiers.
__device__ __noinline__ bool spawn_outer_gen(Ctx c);
__device__ __noinline__ bool spawn_outer_t1(Ctx c);
// Exposure for a 32-bit-tier solve that stepped out: enclosing tiers first,
// then its own levels.
struct T0;
__device__ __noinline__ bool t0_share(Ctx c, const T0 t, int level);

// ---------------------------------------------------------- 32-bit tier
// At most 32 candidate columns and 32 rows: lane l holds row l as a 32-bit
// word (rows 0..pc-1 are the column vertices, the rest X rows).  P, VP, the
// active-row set and R -- the columns added since the subproblem began -- are
// warp-uniform masks, so a child costs a few bitwise ops and two ballots.
// Label-hash sums are not carried down the tree: a leaf records its R mask,
// and every 32 leaves the lanes hash one clique each (t0_flush).

struct T0 {
  uint32_t row;
  uint32_t cv;      // vertex id of column lane
  uint64_t h1, h2;  // label hashes of column lane
};

// Hash the pending leaves, one per lane: sums of the entry sums and the R
// columns' hashes, then the clique hash, histogram and largest size.
// Out of line: it runs once per 32 leaves, and one copy keeps the hot node
// loop's code small (instruction-cache misses, not issue slots, bound it).
__device__ __noinline__ void t0_flush(Ctx c, uint32_t npend, uint64_t s10, uint64_t s20,
                                         uint32_t rsize0) {
  WarpSmem *sm = c.sm;
  const uint32_t lane = c.lane;
  __syncwarp();
  uint32_t size = 0;
  if (lane < npend) {
    uint32_t rm = sm->pend_rm[lane];
    size = rsize0 + 2 + __popc(rm);
    uint64_t a = s10, b = s20;
    while (rm) {
      const uint32_t i = __ffs(rm) - 1;
      rm &= rm - 1;
      a += sm->xh1[i];
      b += sm->xh2[i];
    }
    sm->lchk[lane] += clique_hash(a, b, size);
    if (size < kHistCache) {
      atomicAdd(&sm->hcache[size], 1u);
    } else {
      const EnumParams &P = *c.P;
      const uint32_t bin = size < P.hist_len ? size : P.hist_len - 1;
      atomicAdd(&P.hist[(uint64_t)sm->slot * P.hist_len + bin], 1ULL);
    }
  }
  const uint32_t mx = __reduce_max_sync(kFull, size);
  if (lane == 0) {
    sm->count += npend;
    sm->pending += npend;
    sm->max_size = max(sm->max_size, mx);
  }
  __syncwarp();
}

// hash sums of a frame's R mask (lanes of R contribute their column hash)
__device__ __forceinline__ void t0_sums(const Ctx &c, uint32_t rm, uint64_t *s1, uint64_t *s2) {
  const bool in = (rm >> c.lane) & 1;
  *s1 = c.sm->t0_s1 + warp_sum_u64(in ? c.sm->xh1[c.lane] : 0);
  *s2 = c.sm->t0_s2 + warp_sum_u64(in ? c.sm->xh2[c.lane] : 0);
}

// Child task of candidate q at a 32-bit-tier level, as a W = 1 record.
__device__ void t0_materialize(const Ctx &c, const T0 &t, uint32_t Pbase, uint32_t A, uint32_t q, uint32_t RM,
                               char *rec) {
  const uint32_t lane = c.lane;
  const uint32_t CP = Pbase & __shfl_sync(kFull, t.row, q);
  const uint32_t pc = __popc(CP);
  const CPlan plan = compress_plan(CP);
  uint64_t s1, s2;
  t0_sums(c, RM | (1u << q), &s1, &s2);
  uint32_t *colv = (uint32_t *)(rec + kHdr);
  uint64_t *rows = (uint64_t *)(rec + kHdr + align8(4ULL * pc));
  const uint64_t cr = compress_apply(t.row, plan);
  if ((CP >> lane) & 1) {
    const uint32_t k = __popc(CP & ((1u << lane) - 1));
    colv[k] = t.cv;
    rows[k] = cr;
  }
  const bool isx = ((A >> lane) & 1) && ((t.row >> q) & 1) && !((CP >> lane) & 1) &&
                   (CP == 0 || (t.row & CP) != 0);  // X rows empty on the child's columns left out
  const uint32_t bal = __ballot_sync(kFull, isx);
  if (isx) rows[pc + __popc(bal & lanemask_lt())] = cr;
  if (lane == 0) {
    TaskHdr *h = (TaskHdr *)rec;
    h->pc = pc;
    h->nrows = pc + __popc(bal);
    h->W = 1;
    h->rsize = c.sm->t0_rsize + __popc(RM) + 1;
    h->s1 = s1;
    h->s2 = s2;
    h->slot = c.sm->slot;
  }
  __syncwarp();
}

// expose every open candidate of the shallowest open level with |P| >= tau
// (the reference's TASK_SHARE_BOUND, BkPivotBitBalance.cuh:271-273)
__device__ bool t0_spawn(const Ctx &c, const T0 &t, int level) {
  WarpSmem *sm = c.sm;
  int l = 0;
  uint32_t open = 0;
  for (; l < level; l++) {
    const uint4 f = sm->t0f[l];
    open = f.x & f.y;
    if (open && (uint32_t)__popc(f.x) + 1 >= c.P->reg_share_bound) break;
    open = 0;
  }
  if (!open) return false;
  const uint4 f = sm->t0f[l];
  uint32_t VPl = f.y;
  // Highest candidate first: the child of q excludes every open candidate
  // below q, all still open at that point; whatever stays with this warp is
  // the lowest candidates, whose children correctly keep the exposed (later)
  // ones in P.
  while (open) {
    const uint32_t q = 31 - __clz(open);
    open &= ~(1u << q);
    uint32_t blk;
    if (!pool_alloc(c, &blk)) break;
    const uint32_t Pbase = f.x & ~(VPl & ((1u << q) - 1));
    t0_materialize(c, t, Pbase, f.z, q, f.w, pool_block(*c.P, blk));
    pool_publish(c, blk);
    VPl &= ~(1u << q);
  }
  if (c.lane == 0) sm->t0f[l].y = VPl;
  __syncwarp();
  return true;
}

// Lanes whose index has bit k set: lane s stands for the subset s of a small
// node's candidates (bit k = its k-th lowest candidate).
__device__ __forceinline__ constexpr uint32_t lanes_with_bit(int k) {
  return k == 0 ? 0xAAAAAAAAu : k == 1 ? 0xCCCCCCCCu : k == 2 ? 0xF0F0F0F0u : k == 3 ? 0xFF00FF00u : 0xFFFF0000u;
}

// A node with exactly N (3..7) candidates, decided in one step.  R + K is a
// maximal clique for exactly the cliques K of the candidates that no active
// row contains (a candidate outside K that extends K is itself such a row).
// The subsets are numbered s = 32 g + lane: the lane index carries the
// subset's lowest five candidates, the group g (one pass each, 2^(N-5) of
// them) the rest.  Whether s is a clique is read off warp-uniform masks: a
// missing edge (i, j) among the lane's candidates excludes the lanes with bits
// i and j; a missing edge from a group candidate u to candidate i excludes the
// lanes with bit i in the groups holding u; a missing edge between two group
// candidates excludes whole groups.  Rows containing s: the AND of the
// per-candidate ballots over s's members.
template <int N>
__device__ __forceinline__ void t0_small_n(const Ctx &c, const T0 &t, uint32_t P, uint32_t A, uint32_t RM,
                                           uint32_t &npend, uint64_t s10, uint64_t s20, uint32_t rsize0) {
  constexpr int NL = N < 5 ? N : 5;  // candidates carried by the lane index
  constexpr int NG = N - NL;         // candidates carried by the group
  WarpSmem *sm = c.sm;
  const uint32_t lane = c.lane;
  uint32_t qb[N], h[N], r[N - 1];
  uint32_t pm = P;
#pragma unroll
  for (int k = 0; k < N; k++) {
    qb[k] = pm & (0u - pm);
    pm ^= qb[k];
  }
  // independent collectives: rows holding each candidate, the candidates' rows
#pragma unroll
  for (int k = 0; k < N; k++) h[k] = A & __ballot_sync(kFull, (t.row & qb[k]) != 0);
#pragma unroll
  for (int k = 0; k < N - 1; k++) r[k] = __shfl_sync(kFull, t.row, __ffs(qb[k]) - 1);
  uint32_t notclique = 0;
#pragma unroll
  for (int i = 0; i < NL - 1; i++)
#pragma unroll
    for (int j = i + 1; j < NL; j++)
      if (!(r[i] & qb[j])) notclique |= lanes_with_bit(i) & lanes_with_bit(j);
  uint32_t rows = A, mask = RM;
#pragma unroll
  for (int k = 0; k < NL; k++)
    if ((lane >> k) & 1) {
      rows &= h[k];
      mask |= qb[k];
    }
  const bool lane_ok = lane < (1u << NL) && !((notclique >> lane) & 1);
#pragma unroll
  for (int g = 0; g < (1 << NG); g++) {
    bool ok = lane_ok && (g != 0 || lane != 0);
    bool group_clique = true;
    uint32_t rg = rows, mg = mask;
#pragma unroll
    for (int b = 0; b < NG; b++) {
      if (!((g >> b) & 1)) continue;
      const int u = NL + b;
      uint32_t far = 0;  // lanes holding a candidate not adjacent to u
#pragma unroll
      for (int i = 0; i < NL; i++)
        if (!(r[i] & qb[u])) far |= lanes_with_bit(i);
      ok = ok && !((far >> lane) & 1);
      rg &= h[u];
      mg |= qb[u];
#pragma unroll
      for (int b2 = b + 1; b2 < NG; b2++)
        if (((g >> b2) & 1) && !(r[u] & qb[NL + b2])) group_clique = false;
    }
    const bool out = group_clique && ok && rg == 0;
    const uint32_t E = __ballot_sync(kFull, out);
    const uint32_t pos = npend + __popc(E & lanemask_lt());
    if (out && pos < 32) sm->pend_rm[pos] = mg;
    npend += __popc(E);
    if (npend >= 32) {
      t0_flush(c, 32, s10, s20, rsize0);
      if (out && pos >= 32) sm->pend_rm[pos - 32] = mg;
      npend -= 32;
    }
  }
}

// A node with 1 to kSmallP candidates P, active rows A and R = RM, decided
// in one step: its maximal cliques go to the pending leaves.
__device__ __forceinline__ void t0_small(const Ctx &c, const T0 &t, uint32_t P, uint32_t A, uint32_t RM,
                                         uint32_t &npend, uint64_t s10, uint64_t s20, uint32_t rsize0) {
  WarpSmem *sm = c.sm;
  const uint32_t lane = c.lane;
  if ((P & (P - 1)) == 0) {
    // One candidate q: R + q is maximal iff no active row holds q (the pivot
    // step would prune on such a row, else branch on q into a leaf).
    if ((A & __ballot_sync(kFull, (t.row & P) != 0)) == 0) {
      if (lane == 0) sm->pend_rm[npend] = RM | P;
      if (++npend == 32) {
        t0_flush(c, 32, s10, s20, rsize0);
        npend = 0;
      }
    }
    return;
  }
  {
    const uint32_t lo = P & (0u - P), hi = P & ~lo;
    if (hi == (hi & (0u - hi))) {
      // Two candidates a, b.  Adjacent: R + a + b is the only maximal clique
      // below, iff no active row holds both.  Not adjacent: R + a and R + b
      // each are, iff no active row holds that vertex.  (What the pivot and
      // the two branches would find.)
      const uint32_t ra = A & __ballot_sync(kFull, (t.row & lo) != 0);
      const uint32_t rb = A & __ballot_sync(kFull, (t.row & hi) != 0);
      const uint32_t a = __ffs(lo) - 1;
      uint32_t emit_rm[2];
      uint32_t ne = 0;
      if (__shfl_sync(kFull, t.row, a) & hi) {
        if ((ra & rb) == 0) emit_rm[ne++] = RM | P;
      } else {
        if (ra == 0) emit_rm[ne++] = RM | lo;
        if (rb == 0) emit_rm[ne++] = RM | hi;
      }
      for (uint32_t k = 0; k < ne; k++) {
        if (lane == 0) sm->pend_rm[npend] = emit_rm[k];
        if (++npend == 32) {
          t0_flush(c, 32, s10, s20, rsize0);
          npend = 0;
        }
      }
      return;
    }
  }
  switch (__popc(P)) {
    case 3: t0_small_n<3>(c, t, P, A, RM, npend, s10, s20, rsize0); break;
    case 4: t0_small_n<4>(c, t, P, A, RM, npend, s10, s20, rsize0); break;
#if MCE_SMALL_P >= 6
    case 5: t0_small_n<5>(c, t, P, A, RM, npend, s10, s20, rsize0); break;
#endif
#if MCE_SMALL_P >= 7
    case 6: t0_small_n<6>(c, t, P, A, RM, npend, s10, s20, rsize0); break;
#endif
    default: t0_small_n<kSmallP < 3 ? 3 : kSmallP>(c, t, P, A, RM, npend, s10, s20, rsize0); break;
  }
}

// ------------------------------------------------ join decomposition
// A node whose active rows are all candidates (no X row contains R) has as
// its maximal cliques R + K for exactly the maximal cliques K of G[P].  Let H
// be the complement of G[P].  G[P] is the join of the complements of H's
// connected components, so its maximal cliques are the products of one
// maximal clique of each component's complement, i.e. one maximal independent
// set (in H) per component.  When every component is small, the node is
// decided without a search tree: count, histogram and largest size in closed
// form, and the checksum by walking the products, 32 lanes at a time.
//
// Components: breadth-first search with ballots (closed H-neighbourhoods
// nb = P \ row).  Component j's maximal independent sets come from the 2^s
// subsets of its s members, one per lane, and are packed into a table of at
// most 32 entries in shared memory (hash sums and size of each set).  Lane j
// holds component j's first entry and entry count.
//
// Walking the products: the first components whose entry counts multiply to
// at most 32 (Q) are carried by the lane index (each lane adds up its own
// entries once); the others form a warp-uniform mixed-radix counter, whose
// steps swap one entry per digit that moves.
constexpr int kJoinComp = 5;    // largest component decided this way
#ifndef MCE_JOIN_MIN
#define MCE_JOIN_MIN 10
#endif
constexpr int kJoinMin = MCE_JOIN_MIN;  // smallest |P| worth the decomposition

__device__ __noinline__ bool t0_join(Ctx c, T0 t, uint32_t P, uint32_t RM, uint64_t s10, uint64_t s20,
                                     uint32_t rsize0) {
  const uint32_t lane = c.lane;
  WarpSmem *sm = c.sm;
  const bool inP = (P >> lane) & 1;
  const uint32_t nb = inP ? (P & ~t.row) : 0u;  // closed non-neighbourhood in P (rows carry no self bit)
  if (__reduce_max_sync(kFull, (uint32_t)__popc(nb)) > (uint32_t)kJoinComp) return false;
  const uint32_t single = __ballot_sync(kFull, inP && nb == (1u << lane));  // adjacent to every candidate
  // components first: a node is abandoned before any set is built
  uint32_t rem = P & ~single;
  uint32_t comp = 0, ncomp = 0;  // lane j: component j's members
  #pragma unroll 1
  while (rem) {
    uint32_t C = rem & (0u - rem), fr = C;
    do {
      const uint32_t nbr = __ballot_sync(kFull, (nb & fr) != 0);
      fr = nbr & ~C;
      C |= nbr;
    } while (fr && __popc(C) <= kJoinComp);
    if (__popc(C) > kJoinComp) return false;
    if (lane == ncomp) comp = C;
    ncomp++;
    rem &= ~C;
  }
  // Scratch while the node is decided: the exchange buffer and the row buffer
  // (free inside a 32-bit-tier solve).  xrow: closed non-neighbourhoods by
  // column; rowbuf[e], rowbuf[32 + e], xcv[e]: entry e's hash sums and size.
  uint64_t *E1 = sm->rowbuf, *E2 = sm->rowbuf + 32;
  uint32_t *ES = sm->xcv;
  sm->xrow[lane] = nb;
  __syncwarp();
  uint32_t nent = 0, c_off = 0, c_r = 0;  // lane j: component j's first entry and entry count
  uint64_t total = 1;
  #pragma unroll 1
  for (uint32_t j = 0; j < ncomp; j++) {
    const uint32_t C = __shfl_sync(kFull, comp, j);
    const uint32_t ns = __popc(C);
    // lane l tests the subset l of C's members (bit k = k-th lowest member)
    uint32_t sub = 0;
    uint64_t a1 = 0, a2 = 0;
    uint32_t cm = C;
    #pragma unroll 1
    for (uint32_t k = 0; k < ns; k++) {
      const uint32_t b = cm & (0u - cm);
      cm ^= b;
      if ((lane >> k) & 1) {
        const uint32_t m = __ffs(b) - 1;
        sub |= b;
        a1 += sm->xh1[m];
        a2 += sm->xh2[m];
      }
    }
    bool ok = lane != 0 && lane < (1u << ns);
    cm = C;
    #pragma unroll 1
    for (uint32_t k = 0; k < ns; k++) {
      const uint32_t b = cm & (0u - cm);
      cm ^= b;
      const uint32_t nbk = sm->xrow[__ffs(b) - 1];
      // independent: no other member of the subset is a non-neighbour;
      // maximal: every member outside has a non-neighbour inside
      ok = ok && ((sub & b) ? (nbk & sub) == b : (nbk & sub) != 0);
    }
    const uint32_t mis = __ballot_sync(kFull, ok);
    const uint32_t r = __popc(mis);
    if (nent + r > 32) return false;
    if (ok) {
      const uint32_t e = nent + __popc(mis & lanemask_lt());
      E1[e] = a1;
      E2[e] = a2;
      ES[e] = __popc(sub);
    }
    if (lane == j) {
      c_off = nent;
      c_r = r;
    }
    nent += r;
    total *= r;
  }
  __syncwarp();
  // the part every clique shares: R and the candidates adjacent to all others
  const uint32_t base_cols = RM | single;
  const uint64_t b1 = s10 + warp_sum_u64(((base_cols >> lane) & 1) ? t.h1 : 0);
  const uint64_t b2 = s20 + warp_sum_u64(((base_cols >> lane) & 1) ? t.h2 : 0);
  const uint32_t size0 = rsize0 + 2 + __popc(base_cols);
  // sizes: the product of the components' size polynomials, lane = size - size0
  // (a component's sets leave out at least one member, so sizes stay below size0 + 32)
  uint32_t poly = lane == 0 ? 1u : 0u;
  #pragma unroll 1
  for (uint32_t j = 0; j < ncomp; j++) {
    const uint32_t off = __shfl_sync(kFull, c_off, j), r = __shfl_sync(kFull, c_r, j);
    uint32_t acc = 0;
    #pragma unroll 1
    for (uint32_t d = 0; d < r; d++) {
      const uint32_t sz = ES[off + d];
      const uint32_t v = __shfl_up_sync(kFull, poly, sz);
      if (lane >= sz) acc += v;
    }
    poly = acc;
  }
  {
    const uint32_t size = size0 + lane;
    if (poly) {
      if (size < kHistCache) {
        atomicAdd(&sm->hcache[size], poly);
      } else {
        const EnumParams &Pm = *c.P;
        const uint32_t bin = size < Pm.hist_len ? size : Pm.hist_len - 1;
        atomicAdd(&Pm.hist[(uint64_t)sm->slot * Pm.hist_len + bin], (unsigned long long)poly);
      }
    }
    const uint32_t mx = __reduce_max_sync(kFull, poly ? size : 0u);
    if (lane == 0) {
      sm->count += total;
      sm->pending += (uint32_t)total;
      sm->max_size = max(sm->max_size, mx);
    }
  }
  // lane-carried components 0 .. a - 1 (Q products): each lane's own sums
  uint32_t a = 0, Q = 1;
  #pragma unroll 1
  while (a < ncomp) {
    const uint32_t r = __shfl_sync(kFull, c_r, a);
    if (Q * r > 32) break;
    Q *= r;
    a++;
  }
  uint64_t p1 = b1, p2 = b2;
  uint32_t psz = size0;
  {
    uint32_t rest = lane;
    #pragma unroll 1
    for (uint32_t j = 0; j < a; j++) {
      const uint32_t off = __shfl_sync(kFull, c_off, j), r = __shfl_sync(kFull, c_r, j);
      const uint32_t d = rest % r;
      rest /= r;
      p1 += E1[off + d];
      p2 += E2[off + d];
      psz += ES[off + d];
    }
  }
  // counter-carried components a .. ncomp - 1: digits in lanes, sums uniform
  uint32_t dig = 0;
  uint64_t h1 = 0, h2 = 0;
  uint32_t hsz = 0;
  #pragma unroll 1
  for (uint32_t j = a; j < ncomp; j++) {
    const uint32_t off = __shfl_sync(kFull, c_off, j);
    h1 += E1[off];
    h2 += E2[off];
    hsz += ES[off];
  }
  uint64_t chk = 0;
  const bool live = lane < Q;
  #pragma unroll 1
  for (;;) {
    if (live) chk += clique_hash(p1 + h1, p2 + h2, psz + hsz);
    // next value of the counter: the lowest digit below its top moves up,
    // the digits under it wrap to their first entry
    const uint32_t can = __ballot_sync(kFull, lane >= a && lane < ncomp && dig + 1 < c_r);
    if (!can) break;
    const uint32_t jmax = __ffs(can) - 1;
    #pragma unroll 1
    for (uint32_t j = a; j <= jmax; j++) {
      const uint32_t off = __shfl_sync(kFull, c_off, j);
      const uint32_t cur = off + __shfl_sync(kFull, dig, j);
      const uint32_t nxt = j == jmax ? cur + 1 : off;
      h1 += E1[nxt] - E1[cur];
      h2 += E2[nxt] - E2[cur];
      hsz += ES[nxt] - ES[cur];
    }
    if (lane >= a && lane < jmax) dig = 0;
    if (lane == jmax) dig++;
  }
  sm->lchk[lane] += chk;
  __syncwarp();
  maybe_flush(c);
  return true;
}

// kStats: count search-tree nodes and row word-ops (a separate instance, so
// the counting costs nothing when it is off)
//
// The node loop makes no calls, which keeps its registers free.  To expose
// work it steps out instead: it saves its state and returns true; the caller
// (t0_run) exposes levels and calls it again with resume set.
template <bool kStats>
__device__ __noinline__ bool t0_solve_body(Ctx c, T0 t, uint32_t pc, uint32_t nrows, uint32_t rsize0, uint64_t s10,
                                           uint64_t s20, bool resume) {
  const uint32_t lane = c.lane;
  WarpSmem *sm = c.sm;
  const bool expand_r = c.P->expand_r != 0;
  uint32_t A, P, RM, npend;
  int level;
  if (!resume) {
    sm->xh1[lane] = t.h1;
    sm->xh2[lane] = t.h2;
    if (lane == 0) {
      sm->t0_s1 = s10;
      sm->t0_s2 = s20;
      sm->t0_rsize = rsize0;
    }
    __syncwarp();
    A = nrows >= 32 ? ~0u : ((1u << nrows) - 1);
    P = pc >= 32 ? ~0u : ((1u << pc) - 1);
    RM = 0;
    npend = 0;
    level = 0;
  } else {
    P = sm->y_P;
    A = sm->y_A;
    RM = sm->y_RM;
    npend = sm->y_npend;
    level = sm->y_level;
  }
  const uint32_t lanebit = 1u << lane;
  unsigned long long nodes = 0, wops = 0;  // uniform across lanes
  uint32_t tick = 0;
  const uint32_t period = sm->share_period;
  // A child whose candidate set comes out empty is a leaf: it is tested where
  // it is made, without a frame push, a descent and a backtrack.
  uint32_t VP = 0;
node:  // a node with candidates P, active rows A and R = RM
  if (kStats) nodes++;
  if (P == 0) {  // only a subproblem without columns starts like this
    if (A == 0) {
      if (lane == 0) sm->pend_rm[npend] = RM;
      ++npend;
    }
    goto backtrack;
  }
  if (__popc(P) <= kSmallP) {
    if (kStats) nodes++;
    t0_small(c, t, P, A, RM, npend, s10, s20, rsize0);
    goto backtrack;
  }
  if (__popc(P) >= kJoinMin && (A & ~P) == 0 && t0_join(c, t, P, RM, s10, s20, rsize0)) goto backtrack;
  {
    const uint32_t key = (A & lanebit) ? (((uint32_t)__popc(P & ~t.row) << 5) | lane) : 0xffffffffu;
    const uint32_t kmin = __reduce_min_sync(kFull, key);
    if (kStats) wops += 2 * __popc(A);  // ANDN + POPC per active row
    if ((kmin >> 5) == 0) goto backtrack;  // an X row covers P: nothing maximal below
    VP = P & ~__shfl_sync(kFull, t.row, kmin & 31);
  }
expand:  // next candidate of VP at this level
  {
    const uint32_t cand = P & VP;
    if (cand == 0) goto backtrack;
    const uint32_t q = __ffs(cand) - 1;
    P &= ~(1u << q);
    // the child's candidates and the rows holding q: two independent
    // collectives; rows holding R' = R + q (+ E) are A & those
    uint32_t P2 = P & __shfl_sync(kFull, t.row, q);
    uint32_t A2 = A & __ballot_sync(kFull, (t.row >> q) & 1);
    uint32_t M = 1u << q;
    if (expand_r && (P2 & (P2 - 1))) {
      // EXPAND_R: a candidate adjacent to every other candidate joins R at
      // once; rows carry no self bit, so that is P2 \ row == {itself}
      const uint32_t E = __ballot_sync(kFull, (P2 & ~t.row) == lanebit);
      if (kStats) wops += 2 * __popc(P2);
      if (E) {
        P2 &= ~E;
        M |= E;
        A2 &= __ballot_sync(kFull, (t.row & E) == E);
      }
    }
    if (kStats) wops += __popc(A) + 1;
    if (P2 == 0) {  // leaf child: maximal iff no row contains R + M
      if (kStats) nodes++;
      if (A2 == 0) {
        if (lane == 0) sm->pend_rm[npend] = RM | M;
        if (++npend == 32) {
          t0_flush(c, 32, s10, s20, rsize0);
          npend = 0;
        }
      }
      goto expand;
    }
    if (__popc(P2) <= kSmallP) {  // small child: decided here, no descent
      if (kStats) nodes++;
      t0_small(c, t, P2, A2, RM | M, npend, s10, s20, rsize0);
      goto expand;
    }
    // a child that is its parent's last open candidate replaces the parent
    // (no frame: the parent would only backtrack after it)
    if (cand & (cand - 1)) {
      sm->t0f[level] = make_uint4(P, VP, A, RM);
      level++;
    }
    P = P2;
    A = A2;
    RM |= M;
    if (c.sharing && ++tick >= period) {
      tick = 0;
      if (hungry(c)) {
        // step out at this fresh node; t0_run exposes work and resumes
        __syncwarp();
        if (lane == 0) {
          sm->y_P = P;
          sm->y_A = A;
          sm->y_RM = RM;
          sm->y_npend = npend;
          sm->y_level = level;
          if (kStats) {
            sm->nodes += nodes;
            sm->wops += wops;
          }
        }
        __syncwarp();
        return true;
      }
    }
    goto node;
  }
backtrack:
  if (level > 0) {
    level--;
    const uint4 f = sm->t0f[level];
    P = f.x;
    VP = f.y;
    A = f.z;
    RM = f.w;
    goto expand;
  }
  if (npend) t0_flush(c, npend, s10, s20, rsize0);
  if (kStats && lane == 0) {
    sm->nodes += nodes;
    sm->wops += wops;
  }
  __syncwarp();
  maybe_flush(c);
  return false;
}

__device__ __forceinline__ void t0_run(const Ctx &c, const T0 &t, uint32_t pc, uint32_t nrows, uint32_t rsize0,
                                       uint64_t s10, uint64_t s20) {
  bool resume = false;
  for (;;) {
    const bool out = c.P->stats ? t0_solve_body<true>(c, t, pc, nrows, rsize0, s10, s20, resume)
                                : t0_solve_body<false>(c, t, pc, nrows, rsize0, s10, s20, resume);
    if (!out) break;
    const bool any = t0_share(c, t, c.sm->y_level);
    if (c.lane == 0) c.sm->share_period = any ? kShareMin : min(c.sm->share_period * 2, kShareMax);
    __syncwarp();
    resume = true;
  }
}

// timed wrapper: cycles go to the register-tier phase, spawning excluded
__device__ __forceinline__ void t0_solve(const Ctx &c, const T0 &t, uint32_t pc, uint32_t nrows, uint32_t rsize0,
                                         uint64_t s10, uint64_t s20) {
  const unsigned long long t0 = now(), sp0 = c.sm->cyc[kCycSpawn];
  t0_run(c, t, pc, nrows, rsize0, s10, s20);
  if (c.lane == 0) c.sm->cyc[kCycT0] += (now() - t0) - (c.sm->cyc[kCycSpawn] - sp0);
}

// a W = 1 record with pc <= 32 and nrows <= 32, from a pool block (cg loads)
// or from this warp's own slab
template <bool kCoherent>
__device__ __forceinline__ void t0_load(const Ctx &c, const char *rec, T0 &t, uint32_t pc, uint32_t nrows) {
  const uint32_t *colv = (const uint32_t *)(rec + kHdr);
  const uint64_t *rows = (const uint64_t *)(rec + kHdr + align8(4ULL * pc));
  const uint32_t lane = c.lane;
  if (kCoherent) {
    t.row = lane < nrows ? (uint32_t)ld_cg(rows + lane) : 0;
    t.cv = lane < pc ? ld_cg(colv + lane) : 0;
  } else {
    t.row = lane < nrows ? (uint32_t)rows[lane] : 0;
    t.cv = lane < pc ? colv[lane] : 0;
  }
  t.h1 = lane < pc ? c.P->g.h1[t.cv] : 0;
  t.h2 = lane < pc ? c.P->g.h2[t.cv] : 0;
}

// ---------------------------------------------------------- 64-bit tier

struct T1 {
  uint64_t r[kRPL];   // rows lane, lane+32, lane+64, lane+96
  uint64_t h1a, h1b;  // label hashes of columns lane, lane+32
  uint64_t h2a, h2b;
  uint32_t cva, cvb;  // vertex ids of columns lane, lane+32
};

__device__ __forceinline__ uint64_t sel_row(const T1 &t, uint32_t j) {
  return j == 0 ? t.r[0] : j == 1 ? t.r[1] : j == 2 ? t.r[2] : t.r[3];
}
__device__ __forceinline__ uint64_t bcast_row(const T1 &t, uint32_t idx) {
  return __shfl_sync(kFull, sel_row(t, idx >> 5), idx & 31);
}

__device__ __forceinline__ void t1_hashes(const Ctx &c, T1 &t, uint32_t pc) {
  const DevGraph &g = c.P->g;
  t.h1a = c.lane < pc ? g.h1[t.cva] : 0;
  t.h2a = c.lane < pc ? g.h2[t.cva] : 0;
  t.h1b = c.lane + 32 < pc ? g.h1[t.cvb] : 0;
  t.h2b = c.lane + 32 < pc ? g.h2[t.cvb] : 0;
}

// a W = 1 record with nrows <= 128 into registers
template <bool kCoherent>
__device__ __forceinline__ void t1_load(const Ctx &c, const char *rec, T1 &t, uint32_t pc, uint32_t nrows) {
  const uint32_t *colv = (const uint32_t *)(rec + kHdr);
  const uint64_t *rows = (const uint64_t *)(rec + kHdr + align8(4ULL * pc));
#pragma unroll
  for (int j = 0; j < kRPL; j++) {
    const uint32_t idx = 32 * j + c.lane;
    t.r[j] = idx < nrows ? (kCoherent ? ld_cg(rows + idx) : rows[idx]) : 0;
  }
  t.cva = c.lane < pc ? (kCoherent ? ld_cg(colv + c.lane) : colv[c.lane]) : 0;
  t.cvb = c.lane + 32 < pc ? (kCoherent ? ld_cg(colv + c.lane + 32) : colv[c.lane + 32]) : 0;
  t1_hashes(c, t, pc);
}

// Child task of candidate q of a 64-bit-tier level, into `rec`: columns =
// Pbase & row(q), rows = active rows holding bit q, compressed to the columns.
__device__ void t1_materialize(const Ctx &c, const T1 &t, uint64_t Pbase, uint32_t ab, uint32_t q, uint32_t rsize,
                               uint64_t s1, uint64_t s2, char *rec) {
  const uint32_t lane = c.lane;
  const uint64_t CP = Pbase & bcast_row(t, q);
  const uint32_t pc = __popcll(CP);
  const CPlan plan = compress_plan(CP);
  const uint64_t hq1 = __shfl_sync(kFull, q < 32 ? t.h1a : t.h1b, q & 31);
  const uint64_t hq2 = __shfl_sync(kFull, q < 32 ? t.h2a : t.h2b, q & 31);
  uint32_t *colv = (uint32_t *)(rec + kHdr);
  uint64_t *rows = (uint64_t *)(rec + kHdr + align8(4ULL * pc));
  // candidate rows (row index == column index < 64) in column order
  if ((CP >> lane) & 1) {
    const uint32_t k = __popcll(CP & ((1ULL << lane) - 1));
    colv[k] = t.cva;
    rows[k] = compress_apply(t.r[0], plan);
  }
  if ((CP >> (lane + 32)) & 1) {
    const uint32_t k = __popcll(CP & ((1ULL << (lane + 32)) - 1));
    colv[k] = t.cvb;
    rows[k] = compress_apply(t.r[1], plan);
  }
  // X rows: active, holding bit q, not a column of the child
  uint32_t base = pc;
#pragma unroll
  for (int j = 0; j < kRPL; j++) {
    const uint32_t idx = 32 * j + lane;
    const bool act = ((ab >> j) & 1) && ((t.r[j] >> q) & 1);
    const bool isc = idx < 64 && ((CP >> idx) & 1);
    const bool isx = act && !isc && (CP == 0 || (t.r[j] & CP) != 0);  // empty X rows left out
    const uint32_t bal = __ballot_sync(kFull, isx);
    if (isx) rows[base + __popc(bal & lanemask_lt())] = compress_apply(t.r[j], plan);
    base += __popc(bal);
  }
  if (lane == 0) {
    TaskHdr *h = (TaskHdr *)rec;
    h->pc = pc;
    h->nrows = base;
    h->W = 1;
    h->rsize = rsize + 1;
    h->s1 = s1 + hq1;
    h->s2 = s2 + hq2;
    h->slot = c.sm->slot;
  }
  __syncwarp();
}

// shallowest 64-bit-tier level below `level` with open candidates and
// |P| >= tau, or -1
__device__ __forceinline__ int t1_open_level(const Ctx &c, int level) {
  const T1Area *ta = c.ta;
  for (int l = 0; l < level; l++) {
    const uint64_t Pl = ta->fP[l];
    if ((Pl & ta->fVP[l]) && (uint32_t)__popcll(Pl) + 1 >= c.P->reg_share_bound) return l;
  }
  return -1;
}

__device__ bool t1_spawn(const Ctx &c, const T1 &t, int level) {
  T1Area *ta = c.ta;
  int l = 0;
  uint64_t open = 0;
  for (; l < level; l++) {
    open = ta->fP[l] & ta->fVP[l];
    if (open && (uint32_t)__popcll(ta->fP[l]) + 1 >= c.P->reg_share_bound) break;
    open = 0;
  }
  if (!open) return false;
  const uint64_t Pl = ta->fP[l];
  uint64_t VPl = ta->fVP[l];
  const uint32_t abl = ta->fab[l][c.lane];
  const uint32_t rs = ta->frs[l];
  const uint64_t s1 = ta->fs1[l], s2 = ta->fs2[l];
  // highest open candidate first (see t0_spawn)
  while (open) {
    const uint32_t q = 63 - __clzll((long long)open);
    open &= ~(1ULL << q);
    uint32_t blk;
    if (!pool_alloc(c, &blk)) break;
    const uint64_t Pbase = Pl & ~(VPl & ((1ULL << q) - 1));
    t1_materialize(c, t, Pbase, abl, q, rs, s1, s2, pool_block(*c.P, blk));
    pool_publish(c, blk);
    VPl &= ~(1ULL << q);
  }
  if (c.lane == 0) ta->fVP[l] = VPl;
  __syncwarp();
  return true;
}

__device__ __noinline__ void t1_solve_body(Ctx c, T1 t, uint32_t pc, uint32_t nrows, uint32_t rsize0, uint64_t s10,
                                           uint64_t s20) {
  T1Area *ta = c.ta;
  const uint32_t lane = c.lane;
  WarpSmem *sm = c.sm;
  const bool expand_r = c.P->expand_r != 0;
  uint32_t ab = 0;
#pragma unroll
  for (int j = 0; j < kRPL; j++)
    if (32 * j + lane < nrows) ab |= 1u << j;
  uint64_t P = pc >= 64 ? ~0ULL : ((1ULL << pc) - 1);
  uint64_t VP = 0;
  uint32_t rsize = rsize0;
#pragma unroll
  for (int j = 0; j < kRPL; j++) ta->t1rows[32 * j + lane] = t.r[j];
  ta->t1cv[lane] = t.cva;
  ta->t1cv[lane + 32] = t.cvb;
  if (lane == 0) {
    sm->t1_pc = pc;
    sm->nest |= kNestT1;
  }
  __syncwarp();
  uint64_t s1 = s10, s2 = s20;
  unsigned long long nodes = 0, wops = 0;  // nodes uniform; wops per lane
  int level = 0;
  bool fresh = true;
  uint32_t tick = 0;
  for (;;) {
    if (fresh) {
      nodes++;
      if (P == 0) {
        if (!__any_sync(kFull, ab != 0) && lane == 0) emit(c, rsize + 2, s1, s2);
        goto backtrack;
      }
      {
        wops += 2 * __popc(ab);
        uint32_t key = 0xffffffffu;
#pragma unroll
        for (int j = 0; j < kRPL; j++)
          if ((ab >> j) & 1) key = min(key, ((uint32_t)__popcll(P & ~t.r[j]) << 8) | (32 * j + lane));
        key = __reduce_min_sync(kFull, key);
        if ((key >> 8) == 0) goto backtrack;  // an X row covers P: nothing maximal below
        VP = P & ~bcast_row(t, key & 0xff);
        fresh = false;
      }
    }
    {
      const uint64_t cand = P & VP;
      if (cand == 0) goto backtrack;
      const uint32_t q = __ffsll((long long)cand) - 1;
      P &= ~(1ULL << q);
      if (lane == 0) {
        ta->fP[level] = P;
        ta->fVP[level] = VP;
        ta->frs[level] = rsize;
        ta->fs1[level] = s1;
        ta->fs2[level] = s2;
      }
      ta->fab[level][lane] = (uint8_t)ab;
      uint64_t P2 = P & bcast_row(t, q);
      uint64_t n1 = s1 + __shfl_sync(kFull, q < 32 ? t.h1a : t.h1b, q & 31);
      uint64_t n2 = s2 + __shfl_sync(kFull, q < 32 ? t.h2a : t.h2b, q & 31);
      uint32_t rs = rsize + 1;
      uint64_t M = 1ULL << q;
      if (expand_r && __popcll(P2) > 1) {
        wops += 2 * (((P2 >> lane) & 1) + ((P2 >> (lane + 32)) & 1));
        const bool e0 = ((P2 >> lane) & 1) && __popcll(P2 & ~t.r[0]) == 1;
        const bool e1 = ((P2 >> (lane + 32)) & 1) && __popcll(P2 & ~t.r[1]) == 1;
        const uint64_t E = (uint64_t)__ballot_sync(kFull, e0) | ((uint64_t)__ballot_sync(kFull, e1) << 32);
        if (E) {
          P2 &= ~E;
          M |= E;
          rs += __popcll(E);
          n1 += warp_sum_u64((e0 ? t.h1a : 0) + (e1 ? t.h1b : 0));
          n2 += warp_sum_u64((e0 ? t.h2a : 0) + (e1 ? t.h2b : 0));
        }
      }
      uint32_t ab2 = 0;
#pragma unroll
      for (int j = 0; j < kRPL; j++)
        if (((ab >> j) & 1) && (t.r[j] & M) == M) ab2 |= 1u << j;
      wops += __popc(ab) + (lane == 0 ? 1 : 0);
      // A child with <= 32 columns and <= 32 active rows drops to the 32-bit
      // tier: rows compressed to the child's columns and gathered, columns
      // first, through the warp's exchange buffer.
      // X rows with no bit on the child's candidates never matter below a
      // child that has candidates (a pivot among them leaves VP = P, and they
      // drop out at the next step), so the handoff leaves them out
      uint32_t ab3 = ab2;
      if (P2) {
#pragma unroll
        for (int j = 0; j < kRPL; j++) {
          const uint32_t idx = 32 * j + lane;
          const bool isc = idx < 64 && ((P2 >> idx) & 1);
          if (!isc && (t.r[j] & P2) == 0) ab3 &= ~(1u << j);
        }
      }
      const uint32_t nact = __reduce_add_sync(kFull, __popc(ab3));
      if (__popcll(P2) <= 32 && nact <= 32) {
        const uint32_t pc2 = __popcll(P2);
        const CPlan plan = compress_plan(P2);
        uint32_t base = pc2;
#pragma unroll
        for (int j = 0; j < kRPL; j++) {
          const uint32_t idx = 32 * j + lane;
          const bool act = (ab3 >> j) & 1;
          const bool isc = idx < 64 && ((P2 >> idx) & 1);
          if (act && isc) {
            const uint32_t k = __popcll(P2 & ((1ULL << idx) - 1));
            sm->xrow[k] = (uint32_t)compress_apply(t.r[j], plan);
            sm->xcv[k] = j == 0 ? t.cva : t.cvb;
            sm->xh1[k] = j == 0 ? t.h1a : t.h1b;
            sm->xh2[k] = j == 0 ? t.h2a : t.h2b;
          }
          const bool isx = act && !isc;
          const uint32_t bal = __ballot_sync(kFull, isx);
          if (isx) sm->xrow[base + __popc(bal & lanemask_lt())] = (uint32_t)compress_apply(t.r[j], plan);
          base += __popc(bal);
        }
        __syncwarp();
        T0 t0;
        t0.row = lane < nact ? sm->xrow[lane] : 0;
        t0.cv = lane < pc2 ? sm->xcv[lane] : 0;
        t0.h1 = lane < pc2 ? sm->xh1[lane] : 0;
        t0.h2 = lane < pc2 ? sm->xh2[lane] : 0;
        if (lane == 0) sm->t1_level = level;
        __syncwarp();
        const unsigned long long tn = now(), spn = sm->cyc[kCycSpawn];
        t0_run(c, t0, pc2, nact, rs, n1, n2);
        if (lane == 0) {
          // the child's cycles go to the 32-bit tier (t1_solve adds the whole
          // span to the 64-bit tier afterwards)
          const unsigned long long dt = (now() - tn) - (sm->cyc[kCycSpawn] - spn);
          sm->cyc[kCycT0] += dt;
          sm->cyc[kCycReg] -= dt;
        }
        // the child may have exposed open candidates of this level
        VP = ta->fVP[level];
        // While the child ran, the levels above it were exposed only through
        // the child's own checks; offer them here as well.
        if (c.sharing && ++tick >= 4) {
          tick = 0;
          if (hungry(c)) {
            const unsigned long long ts = now();
            if (!spawn_outer_gen(c)) t1_spawn(c, t, level + 1);
            if (lane == 0) sm->cyc[kCycSpawn] += now() - ts;
            VP = ta->fVP[level];
          }
        }
        continue;  // next candidate at this level
      }
      level++;
      P = P2;
      VP = 0;
      rsize = rs;
      s1 = n1;
      s2 = n2;
      ab = ab2;
      fresh = true;
      if (c.sharing && ++tick >= 64) {
        tick = 0;
        if (hungry(c)) {
          const unsigned long long t0 = now();
          if (!spawn_outer_gen(c)) t1_spawn(c, t, level);
          if (lane == 0) sm->cyc[kCycSpawn] += now() - t0;
        }
      }
      continue;
    }
  backtrack:
    if (level == 0) break;
    level--;
    P = ta->fP[level];
    VP = ta->fVP[level];
    rsize = ta->frs[level];
    s1 = ta->fs1[level];
    s2 = ta->fs2[level];
    ab = ta->fab[level][lane];
    fresh = false;
  }
  wops = warp_sum_u64(wops);
  if (lane == 0) {
    sm->nodes += nodes;
    sm->wops += wops;
    sm->nest &= ~kNestT1;
  }
  __syncwarp();
  maybe_flush(c);
}

__device__ __forceinline__ void t1_solve(const Ctx &c, const T1 &t, uint32_t pc, uint32_t nrows, uint32_t rsize0,
                                         uint64_t s10, uint64_t s20) {
  const unsigned long long t0 = now(), sp0 = c.sm->cyc[kCycSpawn];
  t1_solve_body(c, t, pc, nrows, rsize0, s10, s20);
  if (c.lane == 0) c.sm->cyc[kCycReg] += (now() - t0) - (c.sm->cyc[kCycSpawn] - sp0);
}

// a register-tier record (W == 1) in this warp's own slab
__device__ void reg_from_local(const Ctx &c, const char *rec) {
  const TaskHdr *h = (const TaskHdr *)rec;
  const uint32_t pc = h->pc, nrows = h->nrows, rsize = h->rsize;
  const uint64_t s1 = h->s1, s2 = h->s2;
  if (pc <= 32 && nrows <= 32) {
    T0 t0;
    t0_load<false>(c, rec, t0, pc, nrows);
    __syncwarp();
    t0_solve(c, t0, pc, nrows, rsize, s1, s2);
    return;
  }
  T1 t;
  t1_load<false>(c, rec, t, pc, nrows);
  __syncwarp();
  t1_solve(c, t, pc, nrows, rsize, s1, s2);
}

// --------------------------------------------------------- general tier

// Child of candidate q at a general-tier level (record rec_l) as a task
// record in `out`: columns = Pbase & row(q), rows = active rows holding bit q
// (and all of R' when the level's list is inherited), compressed to the child
// columns.  Returns false when the record would exceed max_bytes, or, for a
// pool record (to_pool), when a warp's slab could not lay it out for the
// general tier.
__device__ bool gen_materialize(const Ctx &c, const Gen &G, const uint64_t *rec_l, uint32_t q,
                                const uint64_t *Pbase, uint64_t max_bytes, bool to_pool, char *out) {
  const uint32_t lane = c.lane, W = G.W;
  if (W > 64) return false;  // the child's column mask lives in rowbuf (64 words)
  uint64_t *CP = c.sm->rowbuf;
  const uint64_t *rowq = G.rows + (uint64_t)q * W;
  uint32_t pc = 0;
  for (uint32_t w = lane; w < W; w += 32) {
    const uint64_t v = Pbase[w] & rowq[w];
    CP[w] = v;
    pc += __popcll(v);
  }
  pc = __reduce_add_sync(kFull, pc);
  __syncwarp();
  const uint32_t Wn = (pc + 63) / 64;
  const uint64_t m0 = rec_l[3 * W], m1 = rec_l[3 * W + 1];
  const uint32_t aoff = (uint32_t)m0, alen = (uint32_t)(m0 >> 32);
  const bool lazy = (m1 >> 63) != 0;
  const uint64_t *R = rec_l + 2 * W;
  const uint32_t wq = q >> 6;
  const uint64_t bq = 1ULL << (q & 63);
  auto keep_row = [&](uint32_t i) -> bool {
    const uint64_t *row = G.rows + (uint64_t)i * W;
    if (!(row[wq] & bq)) return false;
    if (lazy)
      for (uint32_t w = 0; w < W; w++)
        if ((R[w] & row[w]) != R[w]) return false;
    return true;
  };
  auto is_col = [&](uint32_t i) -> bool { return i < G.pc && ((CP[i >> 6] >> (i & 63)) & 1); };
  // X rows empty on the child's columns are left out when it has columns
  auto hits = [&](uint32_t i) -> bool {
    if (pc == 0) return true;
    const uint64_t *row = G.rows + (uint64_t)i * W;
    for (uint32_t w = 0; w < W; w++)
      if (row[w] & CP[w]) return true;
    return false;
  };
  uint32_t nx = 0;
  for (uint32_t base = 0; base < alen; base += 32) {
    const uint32_t t = base + lane;
    bool x = false;
    if (t < alen) {
      const uint32_t i = aoff == kIdent ? t : G.alist[aoff + t];
      x = !is_col(i) && keep_row(i) && hits(i);
    }
    nx += __popc(__ballot_sync(kFull, x));
  }
  const uint32_t nrows = pc + nx;
  if (task_bytes(pc, nrows, Wn) > max_bytes) return false;
  if (to_pool && layout_for(pc, pc, nrows, Wn).need > c.slab_bytes) return false;
  uint32_t *colv = (uint32_t *)(out + kHdr);
  uint64_t *rows = (uint64_t *)(out + kHdr + align8(4ULL * pc));
  // child columns: parent candidate rows i < pc with CP bit i, in order
  for (uint32_t i = lane; i < G.pc; i += 32) {
    if (is_col(i)) {
      uint32_t k = 0;
      for (uint32_t w = 0; w < (i >> 6); w++) k += __popcll(CP[w]);
      k += __popcll(CP[i >> 6] & ((1ULL << (i & 63)) - 1));
      colv[k] = G.colv[i];
      compress_row(G.rows + (uint64_t)i * W, CP, W, rows + (uint64_t)k * Wn);
    }
  }
  uint32_t pos = pc;
  for (uint32_t base = 0; base < alen; base += 32) {
    const uint32_t t = base + lane;
    bool x = false;
    uint32_t i = 0;
    if (t < alen) {
      i = aoff == kIdent ? t : G.alist[aoff + t];
      x = !is_col(i) && keep_row(i) && hits(i);
    }
    const uint32_t bal = __ballot_sync(kFull, x);
    if (x) compress_row(G.rows + (uint64_t)i * W, CP, W, rows + (uint64_t)(pos + __popc(bal & lanemask_lt())) * Wn);
    pos += __popc(bal);
  }
  if (lane == 0) {
    TaskHdr *h = (TaskHdr *)out;
    h->pc = pc;
    h->nrows = nrows;
    h->W = Wn;
    h->rsize = ((uint32_t)(m1 >> 32) & 0x7fffffffu) + 1;
    h->s1 = rec_l[3 * W + 2] + G.h1s[q];
    h->s2 = rec_l[3 * W + 3] + G.h2s[q];
    h->slot = c.sm->slot;
  }
  __syncwarp();
  return true;
}

__device__ bool gen_spawn(const Ctx &c, const Gen &G, int level) {
  const uint32_t W = G.W, lane = c.lane;
  const uint64_t LREC = 3ULL * W + 4;
  int l = -1;
  for (int k = 0; k < level && l < 0; k++) {
    const uint64_t *rec = G.stack + (uint64_t)k * LREC;
    bool any = false;
    uint32_t pc = 0;
    for (uint32_t w = lane; w < W; w += 32) {
      any |= (rec[w] & rec[W + w]) != 0;
      pc += __popcll(rec[w]);
    }
    pc = __reduce_add_sync(kFull, pc);
    if (__any_sync(kFull, any) && pc + 1 >= c.P->share_bound) l = k;
  }
  if (l < 0) return false;
  uint64_t *rec = G.stack + (uint64_t)l * LREC;
  uint64_t *Pl = rec, *VPl = rec + W;
  // scratch record past the deepest level holds Pbase
  uint64_t *Pbase = G.stack + (uint64_t)(G.pc + 2) * LREC;
  // highest open candidate first (see t0_spawn)
  uint32_t spawned = 0;
  for (int wq = (int)W - 1; wq >= 0 && spawned < 256; wq--) {
    for (;;) {
      const uint64_t open = Pl[wq] & VPl[wq];
      if (!open) break;
      const uint32_t q = wq * 64 + (63 - __clzll((long long)open));
      uint32_t blk;
      if (!pool_alloc(c, &blk)) return spawned > 0;
      for (uint32_t w = lane; w < W; w += 32) {
        const uint64_t below = (int)w < wq ? ~0ULL : ((int)w == wq ? ((1ULL << (q & 63)) - 1) : 0);
        Pbase[w] = Pl[w] & ~(VPl[w] & below);
      }
      __syncwarp();
      const bool ok = gen_materialize(c, G, rec, q, Pbase, c.P->block_bytes, true, pool_block(*c.P, blk));
      if (!ok) {
        pool_free(c, blk);
        return spawned > 0;
      }
      pool_publish(c, blk);
      if (lane == 0) VPl[wq] &= ~(1ULL << (q & 63));
      __syncwarp();
      spawned++;
    }
  }
  return spawned > 0;
}

// Solve a general-tier ego network laid out in the slab.
__device__ __noinline__ void gen_solve_body(Ctx c, Gen G, uint32_t rsize0, uint64_t s10, uint64_t s20) {
  const uint32_t lane = c.lane, W = G.W;
  WarpSmem *sm = c.sm;
  const uint64_t LREC = 3ULL * W + 4;
  uint64_t *stack = G.stack;
  uint32_t *alist = G.alist;
  const uint64_t *rows = G.rows;
  char *local = c.slab + c.slab_bytes - kLocalRec;  // inside kTail, after the T1Area
  unsigned long long nodes = 0, wops = 0;
  if (lane == 0) {
    sm->gen = G;
    sm->nest |= kNestGen;
  }
  for (uint32_t w = lane; w < W; w += 32) {
    const uint32_t lo = w * 64;
    stack[w] = (G.pc - lo >= 64) ? ~0ULL : ((1ULL << (G.pc - lo)) - 1);
    stack[W + w] = 0;
    stack[2 * W + w] = 0;
  }
  if (lane == 0) {
    uint64_t *m = stack + 3 * W;
    m[0] = (uint64_t)kIdent | ((uint64_t)G.nrows << 32);
    m[1] = (uint64_t)rsize0 << 32;
    m[2] = s10;
    m[3] = s20;
  }
  __syncwarp();
  int level = 0;
  bool fresh = true;
  uint32_t tick = 0;
  for (;;) {
    uint64_t *rec = stack + (uint64_t)level * LREC;
    uint64_t *Pv = rec, *VP = rec + W, *R = rec + 2 * W;
    const uint64_t m0 = rec[3 * W], m1 = rec[3 * W + 1];
    const uint32_t aoff = (uint32_t)m0, alen = (uint32_t)(m0 >> 32);
    const uint32_t atop = (uint32_t)m1, rsize = (uint32_t)(m1 >> 32) & 0x7fffffffu;
    const bool lazy = (m1 >> 63) != 0;
    if (fresh) {
      nodes++;
      uint32_t pcnt = 0;
      for (uint32_t w = lane; w < W; w += 32) pcnt += __popcll(Pv[w]);
      pcnt = __reduce_add_sync(kFull, pcnt);
      if (pcnt == 0) {
        bool blocked;
        if (!lazy) {
          blocked = alen > 0;
        } else {
          bool hit = false;
          for (uint32_t base = 0; base < alen && !hit; base += 32) {
            const uint32_t t = base + lane;
            bool h = false;
            if (t < alen) {
              const uint32_t i = aoff == kIdent ? t : alist[aoff + t];
              const uint64_t *row = rows + (uint64_t)i * W;
              h = true;
              for (uint32_t w = 0; w < W && h; w++) h = (R[w] & ~row[w]) == 0;
            }
            hit = __any_sync(kFull, h);
          }
          blocked = hit;
        }
        if (!blocked && lane == 0) emit(c, rsize + 2, rec[3 * W + 2], rec[3 * W + 3]);
        fresh = false;
        if (level == 0) break;
        level--;
        continue;
      }
      uint32_t best_c = 0xffffffffu, best_t = 0xffffffffu;
      for (uint32_t base = 0; base < alen; base += 32) {
        const uint32_t t = base + lane;
        if (t < alen) {
          const uint32_t i = aoff == kIdent ? t : alist[aoff + t];
          const uint64_t *row = rows + (uint64_t)i * W;
          bool ok = true;
          if (lazy)
            for (uint32_t w = 0; w < W && ok; w++) ok = (R[w] & ~row[w]) == 0;
          if (ok) {
            uint32_t cnt = 0;
            wops += 2 * W;
            for (uint32_t w = 0; w < W; w++) cnt += __popcll(Pv[w] & ~row[w]);
            if (cnt < best_c) {
              best_c = cnt;
              best_t = t;
            }
          }
        }
        if (__any_sync(kFull, best_c == 0)) break;
      }
      const uint32_t minc = __reduce_min_sync(kFull, best_c);
      if (minc == 0 || minc == 0xffffffffu) {
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
      continue;
    }
    uint32_t q = 0xffffffffu;
    for (uint32_t wb = 0; wb < W; wb += 32) {
      const uint32_t w = wb + lane;
      const uint64_t val = w < W ? (Pv[w] & VP[w]) : 0;
      const uint32_t bal = __ballot_sync(kFull, val != 0);
      if (bal) {
        const uint32_t src = __ffs(bal) - 1;
        const uint64_t vv = __shfl_sync(kFull, val, src);
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
    uint64_t *crec = rec + LREC;
    uint64_t *CP = crec, *CE = crec + W, *CR = crec + 2 * W;
    const uint64_t *rowq = rows + (uint64_t)q * W;
    uint32_t cpc = 0;
    for (uint32_t w = lane; w < W; w += 32) {
      const uint64_t cp = Pv[w] & rowq[w];
      CP[w] = cp;
      CR[w] = R[w] | (w == wq ? bq : 0);
      CE[w] = 0;
      cpc += __popcll(cp);
    }
    cpc = __reduce_add_sync(kFull, cpc);
    __syncwarp();
    // a child small enough for the register tiers leaves the general tier here
    if (cpc <= 64 && cpc > 0) {
      uint32_t ccount = 0;
      for (uint32_t base = 0; base < alen; base += 32) {
        const uint32_t t = base + lane;
        bool keep = false;
        if (t < alen) {
          const uint32_t i = aoff == kIdent ? t : alist[aoff + t];
          const uint64_t *row = rows + (uint64_t)i * W;
          keep = (row[wq] & bq) != 0;
          if (lazy)
            for (uint32_t w = 0; w < W && keep; w++) keep = (R[w] & row[w]) == R[w];
          // an X row empty on the child's columns is left out of the record
          if (keep && !(i < G.pc && ((CP[i >> 6] >> (i & 63)) & 1))) {
            bool hit = false;
            for (uint32_t w = 0; w < W && !hit; w++) hit = (row[w] & CP[w]) != 0;
            keep = hit;
          }
        }
        ccount += __popc(__ballot_sync(kFull, keep));
      }
      if (ccount <= kT1Rows && gen_materialize(c, G, rec, q, Pv, kLocalRec, false, local)) {
        if (lane == 0) sm->gen_level = level;
        __syncwarp();
        const unsigned long long t0 = now(), sp0 = sm->cyc[kCycSpawn];
        reg_from_local(c, local);
        // the register-tier time is booked there; keep it out of this phase
        if (lane == 0) sm->cyc[kCycGen] -= (now() - t0) - (sm->cyc[kCycSpawn] - sp0);
        if (c.sharing && ++tick >= 8) {
          tick = 0;
          if (hungry(c)) {
            const unsigned long long ts = now();
            gen_spawn(c, G, level + 1);
            if (lane == 0) sm->cyc[kCycSpawn] += now() - ts;
          }
        }
        continue;  // next candidate at this level
      }
    }
    uint32_t rs = rsize + 1;
    uint64_t t1 = rec[3 * W + 2] + G.h1s[q], t2 = rec[3 * W + 3] + G.h2s[q];
    uint32_t nE = 0;
    if (c.P->expand_r && cpc > 1) {
      uint64_t e1 = 0, e2 = 0;
      uint32_t ne = 0;
      for (uint32_t base = 0; base < G.pc; base += 32) {
        const uint32_t i = base + lane;
        bool e = false;
        if (i < G.pc && ((CP[i >> 6] >> (i & 63)) & 1)) {
          const uint64_t *ri = rows + (uint64_t)i * W;
          uint32_t cc = 0;
          for (uint32_t w = 0; w < W && cc <= 1; w++) cc += __popcll(CP[w] & ~ri[w]);
          e = (cc == 1);
        }
        const uint32_t bal = __ballot_sync(kFull, e);
        if (bal) {
          if (lane == 0) CE[base >> 6] |= (uint64_t)bal << (base & 32);
          if (e) {
            e1 += G.h1s[i];
            e2 += G.h2s[i];
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
          const uint64_t ew = CE[w];
          CP[w] &= ~ew;
          CR[w] |= ew;
        }
        rs += nE;
        t1 += e1;
        t2 += e2;
      }
    }
    __syncwarp();
    uint32_t caoff, calen, catop;
    bool clazy;
    if ((uint64_t)atop + alen <= G.alist_cap) {
      uint32_t n2 = 0;
      const bool single = !lazy && nE == 0;
      const bool child_has_p = cpc > nE;  // X rows empty on P' matter only at a leaf
      for (uint32_t base = 0; base < alen; base += 32) {
        const uint32_t t = base + lane;
        bool keep = false;
        uint32_t i = 0;
        if (t < alen) {
          wops += single ? 1 : W;
          i = aoff == kIdent ? t : alist[aoff + t];
          const uint64_t *row = rows + (uint64_t)i * W;
          keep = (row[wq] & bq) != 0;
          if (!single) {
            const uint64_t *need = lazy ? CR : CE;
            for (uint32_t w = 0; w < W && keep; w++) keep = (row[w] & need[w]) == need[w];
          }
          if (keep && child_has_p && !(i < G.pc && ((CP[i >> 6] >> (i & 63)) & 1))) {
            bool hit = false;
            for (uint32_t w = 0; w < W && !hit; w++) hit = (row[w] & CP[w]) != 0;
            keep = hit;
          }
        }
        const uint32_t bal = __ballot_sync(kFull, keep);
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
    if (c.sharing && ++tick >= 8) {
      tick = 0;
      if (hungry(c)) {
        const unsigned long long ts = now();
        gen_spawn(c, G, level);
        if (lane == 0) sm->cyc[kCycSpawn] += now() - ts;
      }
    }
  }
  wops = warp_sum_u64(wops);
  if (lane == 0) {
    sm->nodes += nodes;
    sm->wops += wops;
    sm->nest &= ~kNestGen;
  }
  __syncwarp();
  maybe_flush(c);
}

__device__ __noinline__ bool spawn_outer_gen(Ctx c) {
  if (!(c.sm->nest & kNestGen)) return false;
  const Gen G = c.sm->gen;
  return gen_spawn(c, G, c.sm->gen_level + 1);
}

__device__ __noinline__ bool spawn_outer_t1(Ctx c) {
  WarpSmem *sm = c.sm;
  T1Area *ta = c.ta;
  if (!(sm->nest & kNestT1)) return false;
  if (t1_open_level(c, sm->t1_level + 1) < 0) return false;  // before loading rows
  T1 t;
#pragma unroll
  for (int j = 0; j < kRPL; j++) t.r[j] = ta->t1rows[32 * j + c.lane];
  t.cva = ta->t1cv[c.lane];
  t.cvb = ta->t1cv[c.lane + 32];
  t1_hashes(c, t, sm->t1_pc);
  return t1_spawn(c, t, sm->t1_level + 1);
}

__device__ __noinline__ bool t0_share(Ctx c, const T0 t, int level) {
  const unsigned long long ts = now();
  const bool any = spawn_outer_gen(c) || spawn_outer_t1(c) || t0_spawn(c, t, level);
  if (c.lane == 0) c.sm->cyc[kCycSpawn] += now() - ts;
  return any;
}

__device__ __forceinline__ void gen_solve(const Ctx &c, const Gen &G, uint32_t rsize0, uint64_t s10, uint64_t s20) {
  const unsigned long long t0 = now(), sp0 = c.sm->cyc[kCycSpawn];
  gen_solve_body(c, G, rsize0, s10, s20);
  if (c.lane == 0) c.sm->cyc[kCycGen] += (now() - t0) - (c.sm->cyc[kCycSpawn] - sp0);
}

// ------------------------------------------------------------ root build

// C = N(v0) & N(v1) (sorted) into cand[]; |C|, or 0xffffffff beyond cap
__device__ uint32_t intersect(const DevGraph &g, uint32_t v0, uint32_t v1, uint32_t *cand, uint64_t cap) {
  const uint32_t lane = lane_id();
  const uint32_t *a = g.adj + g.off[v0], *b = g.adj + g.off[v1];
  uint32_t da = g.off[v0 + 1] - g.off[v0], db = g.off[v1 + 1] - g.off[v1];
  if (da > db) {
    const uint32_t *t = a;
    a = b;
    b = t;
    const uint32_t td = da;
    da = db;
    db = td;
  }
  uint32_t nc = 0;
  for (uint32_t base = 0; base < da; base += 32) {
    const uint32_t t = base + lane;
    const uint32_t val = t < da ? __ldg(a + t) : 0;
    const bool hit = t < da && contains_u32(b, db, val);
    const uint32_t bal = __ballot_sync(kFull, hit);
    if (nc + __popc(bal) > cap) return 0xffffffffu;
    if (hit) cand[nc + __popc(bal & lanemask_lt())] = val;
    nc += __popc(bal);
  }
  __syncwarp();
  return nc;
}

// |N(v0) & N(v1)| and how many of those lie below v1, without storing them:
// sizes the large-scratch pass for a root whose ego network overflowed the slab.
__device__ void intersect_count(const DevGraph &g, uint32_t v0, uint32_t v1, uint32_t *nc_out, uint32_t *nx_out) {
  const uint32_t lane = lane_id();
  const uint32_t *a = g.adj + g.off[v0], *b = g.adj + g.off[v1];
  uint32_t da = g.off[v0 + 1] - g.off[v0], db = g.off[v1 + 1] - g.off[v1];
  if (da > db) {
    const uint32_t *t = a;
    a = b;
    b = t;
    const uint32_t td = da;
    da = db;
    db = td;
  }
  uint32_t nc = 0, nx = 0;
  for (uint32_t base = 0; base < da; base += 32) {
    const uint32_t t = base + lane;
    const uint32_t val = t < da ? __ldg(a + t) : 0;
    const bool hit = t < da && contains_u32(b, db, val);
    nc += __popc(__ballot_sync(kFull, hit));
    nx += __popc(__ballot_sync(kFull, hit && val < v1));
  }
  *nc_out = nc;
  *nx_out = nx;
}

// Ego bitmap rows (candidate rows, then X rows with a candidate neighbour).
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
    uint32_t lo = 0, hi = 0;
    if (lane == 0) {
      lo = lower_bound_u32(nu, du, pmin);
      hi = lower_bound_u32(nu, du, pmax + 1);
    }
    lo = __shfl_sync(kFull, lo, 0);
    hi = __shfl_sync(kFull, hi, 0);
    bool any;
    if (hi - lo < p && W <= 64) {
      for (uint32_t w = lane; w < W; w += 32) rowbuf[w] = 0;
      __syncwarp();
      bool hit = false;
      for (uint32_t e = lo + lane; e < hi; e += 32) {
        const uint32_t y = __ldg(nu + e);
        const uint32_t j = lower_bound_u32(Pl, p, y);
        if (j < p && Pl[j] == y) {
          atomicOr((unsigned long long *)&rowbuf[j >> 6], 1ULL << (j & 63));
          hit = true;
        }
      }
      any = __any_sync(kFull, hit);
      __syncwarp();
      for (uint32_t w = lane; w < W; w += 32) row[w] = rowbuf[w];
    } else {
      uint64_t word = 0;
      bool hitany = false;
      const uint32_t *sl = nu + lo;
      const uint32_t sn = hi - lo;
      for (uint32_t base = 0; base < p; base += 32) {
        const uint32_t j = base + lane;
        const bool hit = j < p && contains_u32(sl, sn, Pl[j]);
        const uint32_t bal = __ballot_sync(kFull, hit);
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

// Solve root r.  Returns false when the root does not fit this slab.
__device__ bool solve_root(const Ctx &c, uint64_t r) {
  const DevGraph &g = c.P->g;
  const uint32_t v0 = g.root_v0[r], v1 = g.root_v1[r];
  set_slot(c, g.slot ? g.slot[v0] : 0);
  uint32_t *cand = (uint32_t *)c.slab;
  const uint64_t cap = (c.slab_bytes - kTail) / 4;
  const unsigned long long tb0 = now();
  const uint32_t nc = intersect(g, v0, v1, cand, cap);
  if (nc == 0xffffffffu) {
    if (c.lane == 0) c.sm->cyc[kCycBuild] += now() - tb0;
    return false;
  }
  const uint32_t x = nc ? lower_bound_u32(cand, nc, v1) : 0;
  const uint32_t p = nc - x;
  const uint64_t s1 = g.h1[v0] + g.h1[v1], s2 = g.h2[v0] + g.h2[v1];
  const uint32_t W = (p + 63) / 64;
  const Layout L = layout_for(nc, p, p + x, W);
  if (p > 0 && L.need > c.slab_bytes) {
    if (c.lane == 0) c.sm->cyc[kCycBuild] += now() - tb0;
    return false;
  }
  if (c.P->stats) {
    // algorithmic build bytes: both endpoint lists, then every member's
    // adjacency list and its bitmap row
    uint64_t du = 0;
    if (p > 0)
      for (uint32_t j = c.lane; j < nc; j += 32) du += g.off[cand[j] + 1] - g.off[cand[j]];
    du = warp_sum_u64(du);
    if (c.lane == 0)
      c.sm->bbytes += 4ULL * ((g.off[v0 + 1] - g.off[v0]) + (g.off[v1 + 1] - g.off[v1])) +
                      (p > 0 ? 4ULL * du + 8ULL * W * nc : 0);
  }
  if (p == 0) {
    if (x == 0 && c.lane == 0) emit(c, 2, s1, s2);
    if (c.lane == 0) c.sm->cyc[kCycBuild] += now() - tb0;
    return true;
  }
  uint64_t *rows = (uint64_t *)(c.slab + L.rows_off);
  const uint32_t nrows = build_rows(g, cand, x, p, W, rows, c.sm->rowbuf);
  __syncwarp();
  if (c.lane == 0) c.sm->cyc[kCycBuild] += now() - tb0;
  if (p <= 32 && nrows <= 32) {
    T0 t0;
    t0.row = c.lane < nrows ? (uint32_t)rows[c.lane] : 0;
    t0.cv = c.lane < p ? cand[x + c.lane] : 0;
    t0.h1 = c.lane < p ? g.h1[t0.cv] : 0;
    t0.h2 = c.lane < p ? g.h2[t0.cv] : 0;
    __syncwarp();
    t0_solve(c, t0, p, nrows, 0, s1, s2);
    return true;
  }
  if (W == 1 && nrows <= kT1Rows) {
    T1 t;
#pragma unroll
    for (int j = 0; j < kRPL; j++) {
      const uint32_t idx = 32 * j + c.lane;
      t.r[j] = idx < nrows ? rows[idx] : 0;
    }
    t.cva = c.lane < p ? cand[x + c.lane] : 0;
    t.cvb = c.lane + 32 < p ? cand[x + c.lane + 32] : 0;
    t1_hashes(c, t, p);
    __syncwarp();
    t1_solve(c, t, p, nrows, 0, s1, s2);
    return true;
  }
  Gen G;
  G.rows = rows;
  G.colv = cand + x;
  uint64_t *h1s = (uint64_t *)(c.slab + L.hash_off);
  uint64_t *h2s = h1s + p;
  for (uint32_t j = c.lane; j < p; j += 32) {
    const uint32_t y = cand[x + j];
    h1s[j] = g.h1[y];
    h2s[j] = g.h2[y];
  }
  G.h1s = h1s;
  G.h2s = h2s;
  G.stack = (uint64_t *)(c.slab + L.stack_off);
  G.alist = (uint32_t *)(c.slab + L.alist_off);
  G.alist_cap = (c.slab_bytes - kTail - L.alist_off) / 4;
  G.pc = p;
  G.nrows = nrows;
  G.W = W;
  __syncwarp();
  gen_solve(c, G, 0, s1, s2);
  return true;
}

// Solve a task popped from the pool; the block goes back to the free ring as
// soon as its contents are in registers or in the slab.
__device__ __noinline__ void solve_block(Ctx c, uint32_t blk) {
  const EnumParams &P = *c.P;
  const char *rec = pool_block(P, blk);
  const uint32_t *hw = (const uint32_t *)rec;
  const uint32_t pc = ld_cg(hw + 0), nrows = ld_cg(hw + 1), W = ld_cg(hw + 2), rsize = ld_cg(hw + 3);
  const uint64_t s1 = ld_cg((const uint64_t *)(rec + 16)), s2 = ld_cg((const uint64_t *)(rec + 24));
  const uint32_t slot = ld_cg(hw + 8);
  set_slot(c, slot);
  if (W == 1 && pc <= 32 && nrows <= 32) {
    T0 t0;
    t0_load<true>(c, rec, t0, pc, nrows);
    pool_free(c, blk);
    t0_solve(c, t0, pc, nrows, rsize, s1, s2);
    return;
  }
  if (W == 1 && nrows <= kT1Rows) {
    T1 t;
    t1_load<true>(c, rec, t, pc, nrows);
    pool_free(c, blk);
    t1_solve(c, t, pc, nrows, rsize, s1, s2);
    return;
  }
  const Layout L = layout_for(pc, pc, nrows, W);
  if (L.need > c.slab_bytes) {
    if (c.lane == 0) atomicExch(P.error, 2u);
    pool_free(c, blk);
    return;
  }
  uint32_t *colv = (uint32_t *)(c.slab + L.colv_off);
  const uint32_t *scol = (const uint32_t *)(rec + kHdr);
  for (uint32_t j = c.lane; j < pc; j += 32) colv[j] = ld_cg(scol + j);
  uint64_t *rows = (uint64_t *)(c.slab + L.rows_off);
  const uint64_t *srows = (const uint64_t *)(rec + kHdr + align8(4ULL * pc));
  const uint64_t nw = (uint64_t)nrows * W;
  for (uint64_t i = c.lane; i < nw; i += 32) rows[i] = ld_cg(srows + i);
  uint64_t *h1s = (uint64_t *)(c.slab + L.hash_off);
  uint64_t *h2s = h1s + pc;
  __syncwarp();
  for (uint32_t j = c.lane; j < pc; j += 32) {
    h1s[j] = P.g.h1[colv[j]];
    h2s[j] = P.g.h2[colv[j]];
  }
  pool_free(c, blk);
  Gen G;
  G.rows = rows;
  G.colv = colv;
  G.h1s = h1s;
  G.h2s = h2s;
  G.stack = (uint64_t *)(c.slab + L.stack_off);
  G.alist = (uint32_t *)(c.slab + L.alist_off);
  G.alist_cap = (c.slab_bytes - kTail - L.alist_off) / 4;
  G.pc = pc;
  G.nrows = nrows;
  G.W = W;
  __syncwarp();
  gen_solve(c, G, rsize, s1, s2);
}

// Root k of this solve's work list: solve it, or defer it to the
// large-scratch pass (sized exactly), and record per-root values.  Not
// inlined: the persistent loop around it then keeps almost nothing live.
__device__ __noinline__ void run_root(Ctx c, uint64_t k) {
  const EnumParams &P = *c.P;
  WarpSmem *sm = c.sm;
  // wk: the root's index in this solve's work list (per-root results are
  // kept by it); the large-scratch pass walks a list of such indices
  const uint64_t wk = P.heavy_list ? P.heavy_list[k] : k;
  const uint64_t r = P.root_list ? P.root_list[wk] : P.re - 1 - wk;  // range: late-peeled roots first
  const unsigned long long c0 = sm->count, h0 = sm->checksum;
  const unsigned long long tr = now();
  const bool fit = solve_root(c, r);
  if (c.lane == 0) atomicMax(P.stat_max_item, now() - tr);
  if (!fit) {
    if (P.push_heavy) {
      // defer the root, sized exactly: the slab must hold its candidate
      // list and an ego network of p columns and up to nc rows
      uint32_t nc = 0, nx = 0;
      intersect_count(P.g, P.g.root_v0[r], P.g.root_v1[r], &nc, &nx);
      if (c.lane == 0) {
        const uint32_t slot = atomicAdd(P.heavy_n, 1u);
        if (slot < P.heavy_cap) {
          P.heavy_out[slot] = (uint32_t)wk;
          const uint32_t p = nc - nx;
          atomicMax(P.heavy_need, (unsigned long long)layout_for(nc, p, nc, (p + 63) / 64).need);
        } else {
          atomicExch(P.error, 4u);  // more deferred roots than the list holds
        }
      }
    } else if (c.lane == 0) {
      atomicExch(P.error, 2u);
    }
  }
  if (P.per_root_count) {
    // fold the per-lane checksums of batched leaves into this root's
    const uint64_t lc = warp_sum_u64(sm->lchk[c.lane]);
    sm->lchk[c.lane] = 0;
    __syncwarp();
    if (c.lane == 0) {
      sm->checksum += lc;
      if (fit) {  // a deferred root's values come from the large-scratch pass
        P.per_root_count[wk] = sm->count - c0;
        P.per_root_checksum[wk] = sm->checksum - h0;
      }
    }
  }
  __syncwarp();
}

// Wait for a task while other warps are busy.  Returns a pool block taken
// from the ready queue (the warp then counts as busy), or -1 when no work is
// left anywhere (or the wait's bound ran out: the error word says so).
//
// At most one warp per block polls the global queue at a time (the block's
// poll token); the others sleep.  A warp counts itself busy only after it has
// taken a task, so a failed attempt costs no atomic on the busy count.
// Reading the busy count before the queue: a task is published before its
// producer stops counting as busy, so "nobody busy" then "queue empty" means
// no work is left -- except for a task taken between the two reads, whose
// taker then finishes everything it exposes by itself if all others have
// left.  Exit waits for two such observations a back-off apart, which makes
// that case rare.  Not inlined, so its loop holds only a few values: idle
// polling costs no reloads of the caller's state.
__device__ __noinline__ int idle_wait(Ctx c, unsigned int *s_poll) {
  const EnumParams &P = *c.P;
  WarpSmem *sm = c.sm;
  uint64_t idle_spins = 0;
  uint32_t quiet = 0;  // consecutive "nobody busy, queue empty" observations
  for (;;) {
    int result = -2;  // -2: keep waiting
    if (c.lane == 0) {
      const unsigned long long ti0 = now();
      bool polled = false, seen = false;
      if (atomicCAS(s_poll, 0u, 1u) == 0u) {
        polled = true;
        const uint32_t act = *(volatile unsigned int *)P.active;
        __threadfence();
        const unsigned long long rh = *(volatile unsigned long long *)P.ready_head;
        const unsigned long long rt = *(volatile unsigned long long *)P.ready_tail;
        if (rh < rt) {
          seen = true;
          uint32_t b = 0;
          if (ring_pop(P.ready_slot, P.ready_seq, P.ready_head, P.ready_tail, P.pool_mask, &b, P)) {
            atomicAdd(P.active, 1u);
            result = (int)b;
          }
          quiet = 0;
        } else if (act == 0) {
          if (++quiet >= 2) result = -1;
        } else {
          quiet = 0;
        }
        atomicExch(s_poll, 0u);
      }
      if (result == -2) {
        if (++idle_spins > P.spin_limit) {
          atomicExch(P.error, 1u);
          result = -1;
        } else if (!polled || seen) {
          __nanosleep(500u + ((uint32_t)(clock64() >> 3) & 511u));
        } else {
          // back off, with jitter, so idle warps do not hammer the control words
          const uint32_t shift = idle_spins < 6 ? (uint32_t)idle_spins : 6u;
          __nanosleep((256u << shift) + ((uint32_t)(clock64() >> 3) & 1023u));
        }
      }
      sm->cyc[kCycIdle] += now() - ti0;
    }
    result = __shfl_sync(kFull, result, 0);
    if (result != -2) return result;
  }
}

__global__ void __launch_bounds__(256, MCE_ENUM_BPS) k_enumerate(const __grid_constant__ EnumParams P) {
  extern __shared__ uint64_t smem_raw[];
  Ctx c;
  c.P = &P;
  c.lane = lane_id();
  WarpSmem *sm = (WarpSmem *)smem_raw + (threadIdx.x >> 5);
  c.sm = sm;
  for (uint32_t b = c.lane; b < kHistCache; b += 32) sm->hcache[b] = 0;
  if (c.lane == 0) {
    sm->count = sm->checksum = sm->nodes = sm->wops = sm->bbytes = 0;
    sm->max_size = sm->slot = sm->pending = 0;
    sm->nest = 0;
    sm->share_period = kShareMin;
  }
  sm->lchk[c.lane] = 0;
  if (c.lane == 0) {
    for (int i = 0; i < kCycPhases; i++) sm->cyc[i] = 0;
  }
  __shared__ unsigned int s_poll;  // the block's poll token (see idle_wait)
  if (threadIdx.x == 0) s_poll = 0;
  __syncthreads();
  const uint64_t gwarp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  c.slab = P.slab + gwarp * P.slab_bytes;
  c.slab_bytes = P.slab_bytes;
  c.ta = (T1Area *)(c.slab + c.slab_bytes - kTail);
  c.sharing = P.sharing != 0;
  const uint64_t total = P.heavy_list ? P.n_heavy : (P.root_list ? P.n_list : P.re - P.rb);
  unsigned long long nroots = 0;
  // a warp counts itself busy from its first root claim until a claim fails,
  // so warps that start late (not co-resident) are never waited for
  if (c.lane == 0) atomicAdd(P.active, 1u);
  __syncwarp();
  for (;;) {
    // queued tasks first: they are the open top of the heaviest subtrees
    if (c.sharing) {
      bool got = false;
      uint32_t b = 0;
      const unsigned long long tq = now();
      if (c.lane == 0) got = ring_pop(P.ready_slot, P.ready_seq, P.ready_head, P.ready_tail, P.pool_mask, &b, P);
      got = __shfl_sync(kFull, got, 0);
      const uint32_t blk = __shfl_sync(kFull, b, 0);
      if (c.lane == 0) sm->cyc[kCycQueue] += now() - tq;
      if (got) {
        const unsigned long long tb = now();
        solve_block(c, blk);
        if (c.lane == 0) atomicMax(P.stat_max_item + 1, now() - tb);
        continue;
      }
    }
    unsigned long long k = 0;
    if (c.lane == 0) k = atomicAdd(P.next, 1ULL);
    k = __shfl_sync(kFull, k, 0);
    if (k >= total) break;
    nroots++;
    run_root(c, k);
  }
  if (c.lane == 0) atomicSub(P.active, 1u);
  if (c.sharing) {
    // roots are gone: take tasks until no warp has work left
    for (;;) {
      const int blk = idle_wait(c, &s_poll);
      if (blk < 0) break;
      const unsigned long long tb = now();
      solve_block(c, (uint32_t)blk);
      if (c.lane == 0) {
        atomicMax(P.stat_max_item + 1, now() - tb);
        atomicSub(P.active, 1u);
      }
      __syncwarp();
    }
  }
  acc_flush(c);
  if (c.lane == 0) {
    atomicAdd(P.stat_roots, nroots);
    if (P.stats) {
      atomicAdd(P.stat_nodes, sm->nodes);
      atomicAdd(P.stat_wops, sm->wops);
      atomicAdd(P.stat_bbytes, sm->bbytes);
    }
    for (int i = 0; i < kCycPhases; i++) atomicAdd(P.stat_cycles + i, sm->cyc[i]);
  }
}

// Control words; the contended ones each own a 128-byte line.
struct EnumCtl {
  alignas(128) unsigned long long next;
  alignas(128) unsigned long long free_head;
  alignas(128) unsigned long long free_tail;
  alignas(128) unsigned long long ready_head;
  alignas(128) unsigned long long ready_tail;
  alignas(128) unsigned int active;
  alignas(128) unsigned long long heavy_need, stat_roots, stat_tasks, stat_nodes, stat_wops, stat_bbytes;
  unsigned long long stat_cycles[kCycPhases];
  unsigned long long stat_max_item[2];
  unsigned int heavy_n, error;
};

// free ring full of every block, ready ring empty, counters reset
__global__ void k_pool_init(EnumCtl *ctl, uint32_t *free_slot, unsigned long long *free_seq,
                            unsigned long long *ready_seq, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    free_slot[i] = i;
    free_seq[i] = (unsigned long long)i + 1;  // filled for the consumer of position i
    ready_seq[i] = i;                        // free for the producer of position i
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    EnumCtl z{};
    z.free_tail = n;
    z.active = 0;
    *ctl = z;
  }
}

mce_status reset_ctl(const EnumPlan &plan, cudaStream_t st) {
  k_pool_init<<<grid_for(plan.pool_blocks, 256), 256, 0, st>>>((EnumCtl *)plan.ctl, plan.params.free_slot,
                                                               plan.params.free_seq, plan.params.ready_seq,
                                                               plan.pool_blocks);
  note_launch();
  MCE_CUDA_TRY(cudaGetLastError());
  return MCE_OK;
}

}  // namespace

mce_status MCE_ENUM_FN(enum_plan)(const DeviceGraph &g, const EnumConfig &cfg, Scratch *scr, SlotResult *slots,
                     unsigned long long *hist, EnumPlan *plan) {
  const int device = scr->device;
  int sms = 0;
  MCE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const uint32_t wpb = cfg.warps_per_block ? std::min(cfg.warps_per_block, 8u) : 8u;
  const uint32_t bps = cfg.blocks_per_sm ? std::min<uint32_t>(cfg.blocks_per_sm, MCE_ENUM_BPS) : MCE_ENUM_BPS;
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
  P.spin_limit = cfg.spin_limit ? cfg.spin_limit : (1ULL << 34);
  P.sharing = (cfg.sharing && cfg.per_root_count == nullptr) ? 1 : 0;
  P.stats = cfg.stats;
  P.share_bound = cfg.share_bound ? cfg.share_bound : 24;
  P.reg_share_bound = std::min(P.share_bound, cfg.reg_share_bound ? cfg.reg_share_bound : kRegShareBound);
  mce_status s = MCE_OK;
  EnumCtl *ctl = (EnumCtl *)scr->get(1, sizeof(EnumCtl), &s);
  if (!ctl) return s;
  plan->ctl = ctl;
  P.next = &ctl->next;
  P.heavy_need = &ctl->heavy_need;
  P.heavy_n = &ctl->heavy_n;
  P.error = &ctl->error;
  P.stat_roots = &ctl->stat_roots;
  P.stat_tasks = &ctl->stat_tasks;
  P.stat_nodes = &ctl->stat_nodes;
  P.stat_wops = &ctl->stat_wops;
  P.stat_bbytes = &ctl->stat_bbytes;
  P.stat_cycles = ctl->stat_cycles;
  P.stat_max_item = ctl->stat_max_item;
  P.active = &ctl->active;
  P.free_head = &ctl->free_head;
  P.free_tail = &ctl->free_tail;
  P.ready_head = &ctl->ready_head;
  P.ready_tail = &ctl->ready_tail;

  uint64_t rb = cfg.root_begin, re = cfg.root_end ? std::min<uint64_t>(cfg.root_end, g.m) : g.m;
  if (rb > re) rb = re;
  const bool list_mode = cfg.root_list != nullptr;
  const uint64_t nwork = list_mode ? cfg.n_root_list : re - rb;
  plan->nwork = nwork;

  uint32_t blocks = (uint32_t)sms * bps;
  if (cfg.max_blocks && blocks > cfg.max_blocks) blocks = cfg.max_blocks;
  if (!P.sharing) {
    const uint64_t want_blocks = (nwork + wpb - 1) / wpb;
    if (want_blocks < blocks) blocks = (uint32_t)std::max<uint64_t>(want_blocks, 1);
  }
  const uint64_t nwarps = (uint64_t)blocks * wpb;
  P.nwarps = (uint32_t)nwarps;
  // slab: the largest ego network this graph can produce (p <= degeneracy,
  // rows <= max degree), capped at 4 MB per warp and by free memory
  size_t freeb = 0, totalb = 0;
  MCE_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
  const uint64_t kcap = std::max<uint32_t>(1, std::min(g.degeneracy, g.max_degree));
  const uint64_t dcap = std::max<uint32_t>(1, g.max_degree);
  const Layout LB = layout_for(dcap, (uint32_t)kcap, (uint32_t)(kcap + dcap), (uint32_t)((kcap + 63) / 64));
  const uint64_t bound = align8(LB.need + 3ULL * (kcap + dcap) * 4);
  const uint64_t slab_cap = cfg.slab_kib ? std::max<uint64_t>(16, cfg.slab_kib) << 10 : 4ULL << 20;
  uint64_t slab_bytes = std::max<uint64_t>(std::min<uint64_t>(bound, slab_cap), 16ULL << 10);
  while (slab_bytes > (64ULL << 10) && slab_bytes * nwarps > freeb / 2) slab_bytes >>= 1;
  slab_bytes = (slab_bytes + 255) & ~255ULL;  // every warp's slab (and its T1Area) 256-byte aligned
  plan->fits_all = slab_bytes >= bound;
  char *slab = (char *)scr->get(2, slab_bytes * nwarps, &s);
  if (!slab) return s;
  // roots whose ego network overflows the slab are deferred to a second pass;
  // the list holds their work indices (a solve of more than 2^32 roots is
  // refused by the callers)
  const uint64_t heavy_cap = std::min<uint64_t>(nwork, 1ULL << 26);
  uint32_t *heavy = nullptr;
  if (nwork) {
    heavy = (uint32_t *)scr->get(3, heavy_cap * 4, &s);
    if (!heavy) return s;
  }
  // task pool: one record per block; both rings have one cell per block
  const uint32_t block_bytes =
      (uint32_t)std::min<uint64_t>(std::max<uint64_t>(4096, align8(slab_bytes / 4)), 64 << 10);
  uint32_t nblocks = 1u << 14;
  while ((uint64_t)nblocks * block_bytes > (freeb / 8) && nblocks > 1024) nblocks >>= 1;
  char *pool = (char *)scr->get(5, (uint64_t)nblocks * block_bytes, &s);
  if (!pool) return s;
  char *rings = (char *)scr->get(6, (uint64_t)nblocks * 24, &s);
  if (!rings) return s;
  P.pool = pool;
  P.block_bytes = block_bytes;
  P.pool_mask = nblocks - 1;
  P.free_seq = (unsigned long long *)rings;
  P.ready_seq = (unsigned long long *)(rings + (uint64_t)nblocks * 8);
  P.free_slot = (uint32_t *)(rings + (uint64_t)nblocks * 16);
  P.ready_slot = (uint32_t *)(rings + (uint64_t)nblocks * 20);
  plan->pool_blocks = nblocks;
  P.slab = slab;
  P.slab_bytes = slab_bytes;
  P.rb = rb;
  P.re = re;
  P.root_list = list_mode ? cfg.root_list : nullptr;
  P.n_list = list_mode ? cfg.n_root_list : 0;
  P.heavy_out = heavy;
  P.heavy_cap = (uint32_t)heavy_cap;
  P.push_heavy = 1;
  plan->heavy_warps = cfg.heavy_warps;
  plan->blocks = blocks;
  plan->sms = (uint32_t)sms;
  plan->threads = wpb * 32;
  plan->smem = (size_t)wpb * sizeof(WarpSmem);
  plan->nwarps = nwarps;
  plan->scr = scr;
  if (plan->smem > 48 * 1024)
    MCE_CUDA_TRY(cudaFuncSetAttribute(k_enumerate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan->smem));
  return MCE_OK;
}

mce_status MCE_ENUM_FN(enum_launch)(const EnumPlan &plan, cudaStream_t st) {
  MCE_TRY(reset_ctl(plan, st));
  if (plan.nwork) {
    k_enumerate<<<plan.blocks, plan.threads, plan.smem, st>>>(plan.params);
    note_launch();
    MCE_CUDA_TRY(cudaGetLastError());
  }
  return MCE_OK;
}

mce_status MCE_ENUM_FN(enum_finish)(const EnumPlan &plan, cudaStream_t st, EnumStats *stats) {
  EnumCtl *ctl = (EnumCtl *)plan.ctl;
  EnumCtl h{};
  MCE_CUDA_TRY(cudaMemcpyAsync(&h, ctl, sizeof(EnumCtl), cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  const uint64_t heavy_roots = h.heavy_n;
  uint64_t launches = plan.nwork ? 1 : 0;
  uint64_t roots = h.stat_roots;
  uint64_t tasks = h.stat_tasks, nodes = h.stat_nodes, wops = h.stat_wops, bbytes = h.stat_bbytes;
  uint64_t cycles[kCycPhases];
  for (int i = 0; i < kCycPhases; i++) cycles[i] = h.stat_cycles[i];
  uint64_t max_item[2] = {h.stat_max_item[0], h.stat_max_item[1]};
  uint32_t err = h.error;
  if (h.heavy_n && !h.error) {
    // Deferred roots: one slab per warp, each sized for the largest deferred
    // ego network; every warp of the pass shares their work (unless per-root
    // values are being attributed, which keeps each root on one warp).  Only
    // warps that get a slab are launched: with fewer slabs than a block's
    // warps, the block shrinks to that many.
    size_t freeb = 0, totalb = 0;
    MCE_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
    const uint64_t need = ((h.heavy_need + 4096) + 255) & ~255ULL;
    uint64_t hw = std::min<uint64_t>((uint64_t)(freeb * 0.7) / need, plan.nwarps);
    if (plan.heavy_warps) hw = std::min<uint64_t>(hw, plan.heavy_warps);
    hw = std::min<uint64_t>(hw, h.heavy_n);
    if (hw == 0) return MCE_ERR_OUT_OF_MEMORY;
    EnumPlan H = plan;
    const uint32_t wpb = plan.threads / 32;
    if (hw < wpb) {
      H.blocks = 1;
      H.threads = (uint32_t)hw * 32;
      H.smem = (size_t)hw * sizeof(WarpSmem);
    } else {
      H.blocks = (uint32_t)(hw / wpb);
    }
    H.nwarps = (uint64_t)H.blocks * (H.threads / 32);
    mce_status s = MCE_OK;
    char *big = (char *)plan.scr->get(4, need * H.nwarps, &s);
    if (!big) return s;
    H.params.slab = big;
    H.params.slab_bytes = need;
    H.params.heavy_list = plan.params.heavy_out;
    H.params.n_heavy = h.heavy_n;
    H.params.push_heavy = 0;
    H.params.nwarps = (uint32_t)H.nwarps;
    cudaEvent_t he0, he1;
    MCE_CUDA_TRY(cudaEventCreate(&he0));
    MCE_CUDA_TRY(cudaEventCreate(&he1));
    cudaEventRecord(he0, st);
    mce_status ls = reset_ctl(H, st);
    if (ls == MCE_OK) {
      k_enumerate<<<H.blocks, H.threads, H.smem, st>>>(H.params);
      note_launch();
      launches++;
      if (cudaGetLastError() != cudaSuccess) ls = MCE_ERR_CUDA;
    }
    cudaEventRecord(he1, st);
    EnumCtl h2{};
    if (ls == MCE_OK && cudaMemcpyAsync(&h2, ctl, sizeof(EnumCtl), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      ls = MCE_ERR_CUDA;
    if (ls == MCE_OK && cudaStreamSynchronize(st) != cudaSuccess) ls = MCE_ERR_CUDA;
    float hms = 0;
    if (ls == MCE_OK) cudaEventElapsedTime(&hms, he0, he1);
    cudaEventDestroy(he0);
    cudaEventDestroy(he1);
    if (ls != MCE_OK) return ls;
    if (stats) stats->ms_heavy = hms;
    roots = roots - heavy_roots + h2.stat_roots;
    tasks += h2.stat_tasks;
    nodes += h2.stat_nodes;
    wops += h2.stat_wops;
    bbytes += h2.stat_bbytes;
    for (int i = 0; i < kCycPhases; i++) cycles[i] += h2.stat_cycles[i];
    for (int i = 0; i < 2; i++) max_item[i] = std::max<uint64_t>(max_item[i], h2.stat_max_item[i]);
    err = h2.error;
  }
  if (stats) {
    stats->roots = roots;
    stats->heavy_roots = heavy_roots;
    stats->shared_tasks = tasks;
    stats->nodes = nodes;
    stats->word_ops = wops;
    stats->build_bytes = bbytes;
    for (int i = 0; i < kCycPhases; i++) stats->cycles[i] = cycles[i];
    for (int i = 0; i < 2; i++) stats->max_item[i] = max_item[i];
    stats->error = err;
    stats->launches = launches;
  }
  if (err == 2) return MCE_ERR_OUT_OF_MEMORY;
  if (err == 4) return MCE_ERR_CAPACITY;
  if (err) return MCE_ERR_TIMEOUT;
  return MCE_OK;
}

#if MCE_ENUM_BPS == 4
namespace {
// Integer-pipe probe: per thread, 8 independent chains of the enumeration's
// word-op mix (a 64-bit ANDN feeding a 64-bit POPC, folded back by an add).
__global__ void k_int_probe(const uint64_t *seed, uint64_t *sink, int iters) {
  uint64_t a[8];
  const uint64_t b = seed[0] ^ (threadIdx.x * 0x9E3779B97F4A7C15ULL);
#pragma unroll
  for (int i = 0; i < 8; i++) a[i] = seed[1] + (uint64_t)i * 0x632BE59BD9B4E019ULL + blockIdx.x;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] += __popcll(a[i] & ~b) | (a[i] << 7);
  }
  uint64_t x = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) x ^= a[i];
  if (x == 0x123456789ULL) sink[0] = x;  // keeps the chains live
}

}  // namespace

mce_status probe_int_peak(int device, double *word_ops_per_s) {
  MCE_CUDA_TRY(cudaSetDevice(device));
  int sms = 0;
  MCE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  uint64_t *buf = nullptr;
  MCE_CUDA_TRY(cudaMalloc(&buf, 64));
  MCE_CUDA_TRY(cudaMemset(buf, 0x5a, 64));
  const int iters = 4096, threads = 256, blocks = sms * 8;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_int_probe<<<blocks, threads>>>(buf, buf + 4, 64);
  note_launch();
  cudaEventRecord(e0);
  k_int_probe<<<blocks, threads>>>(buf, buf + 4, iters);
  note_launch();
  cudaEventRecord(e1);
  const cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  if (e != cudaSuccess || ms <= 0) return MCE_ERR_CUDA;
  // two word-ops (ANDN, POPC) per chain step
  *word_ops_per_s = 2.0 * 8.0 * iters * (double)threads * blocks / (ms * 1e-3);
  return MCE_OK;
}

#endif

}  // namespace mce
