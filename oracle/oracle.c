/*
 * oracle.c -- CPU restatement of the RDMCE hot path (TEST INFRASTRUCTURE ONLY).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this code, as the checker.  The product (rdmce_b200/) never links it.
 *
 * What it restates (reference paths relative to the RDMCE project root):
 *   - text parse:        src/graph.cc:82-104  (istream >> u >> v, bad lines skipped)
 *   - loader rules:      src/graph.cc:64-152  (self-loops dropped, u<v, sort+unique,
 *                                               dense relabel of present labels)
 *   - degeneracy order:  src/graph.cc:281-306 + ApplyOrder src/graph.cc:2-25
 *   - edge roots:        src/kernels/BkPivotBitBalance.cuh:428-469 (v0<v1, P = common
 *                        neighbours > v1, X = common neighbours < v1; an edge in no
 *                        triangle is a clique of size 2, :535-539)
 *   - ego bitmap:        include/graph_gpu.cuh:59-107 (row r = member r of P then X,
 *                        bit j = adjacency to P[j]; X rows without a P neighbour dropped)
 *   - bitmap BK:         src/kernels/BkPivotBitBalance.cuh:192-382 (pivot = argmin over
 *                        rows containing R of |P \ row|, VP = P \ row(pivot), child
 *                        P' = P & row(q), EXPAND_R moves i in P' with |P' \ row(i)| == 1
 *                        into R when |P'| > 1)
 *   - .bin container:    src/graph.cc:154-213
 *
 * The pivot tie rule here is canonical (lowest row index), which the GPU kernel
 * uses too, so node counts agree; the clique set does not depend on it.
 * Outputs beyond the reference's count: size histogram and a 64-bit checksum
 * sum over cliques of h(C) = mix64(s1 ^ rotl(s2,31) ^ (|C| << 56)) with
 * s1 = sum mix64(l), s2 = sum mix64(l ^ G) over the original labels l.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <errno.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define GOLDEN 0x9E3779B97F4A7C15ULL

struct og_graph {
  uint32_t n;
  uint64_t m;          /* undirected edges */
  uint64_t *off;       /* n+1 */
  uint32_t *adj;       /* 2m, rows sorted ascending */
  uint32_t *labels;    /* new id -> original label */
  uint32_t max_degree;
  uint32_t degeneracy;
  uint64_t *root_off;  /* lazily built: prefix over upper-degree, n+1 */
};

/* ------------------------------------------------------------------ hashing */

uint64_t og_mix64(uint64_t x) {
  uint64_t z = x + GOLDEN;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

static inline uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

static inline uint64_t finish_hash(uint64_t s1, uint64_t s2, uint64_t size) {
  return og_mix64(s1 ^ rotl64(s2, 31) ^ (size << 56));
}

uint64_t og_clique_hash(const uint32_t *labels, uint32_t size) {
  uint64_t s1 = 0, s2 = 0;
  for (uint32_t i = 0; i < size; i++) {
    s1 += og_mix64((uint64_t)labels[i]);
    s2 += og_mix64((uint64_t)labels[i] ^ GOLDEN);
  }
  return finish_hash(s1, s2, size);
}

void og_free_buf(void *p) { free(p); }

/* ------------------------------------------------------------- radix sort */

static void radix_sort_u64(uint64_t *a, uint64_t n) {
  if (n < 2) return;
  uint64_t *tmp = (uint64_t *)malloc(n * sizeof(uint64_t));
  uint64_t *src = a, *dst = tmp;
  static const int B = 16;
  size_t *cnt = (size_t *)malloc(sizeof(size_t) << B);
  for (int shift = 0; shift < 64; shift += B) {
    memset(cnt, 0, sizeof(size_t) << B);
    for (uint64_t i = 0; i < n; i++) cnt[(src[i] >> shift) & 0xFFFF]++;
    int single = 0;
    for (size_t d = 0; d < (1u << B); d++)
      if (cnt[d] == n) { single = 1; break; }
    if (single) continue;
    size_t sum = 0;
    for (size_t d = 0; d < (1u << B); d++) { size_t c = cnt[d]; cnt[d] = sum; sum += c; }
    for (uint64_t i = 0; i < n; i++) dst[cnt[(src[i] >> shift) & 0xFFFF]++] = src[i];
    uint64_t *t = src; src = dst; dst = t;
  }
  if (src != a) memcpy(a, src, n * sizeof(uint64_t));
  free(cnt);
  free(tmp);
}

/* -------------------------------------------------------------- text parse */

/* One `is >> unsigned` extraction: skip white space, optional sign, decimal
 * digits; a value above UINT32_MAX fails; a leading '-' wraps modulo 2^32. */
static int read_uint(const char *s, size_t len, size_t *pos, uint32_t *out) {
  size_t p = *pos;
  while (p < len && (s[p] == ' ' || s[p] == '\t' || s[p] == '\n' || s[p] == '\v' ||
                     s[p] == '\f' || s[p] == '\r'))
    p++;
  int neg = 0;
  if (p < len && (s[p] == '+' || s[p] == '-')) { neg = s[p] == '-'; p++; }
  if (p >= len || s[p] < '0' || s[p] > '9') { *pos = p; return 0; }
  uint64_t val = 0;
  int overflow = 0;
  while (p < len && s[p] >= '0' && s[p] <= '9') {
    if (!overflow) {
      val = val * 10 + (uint64_t)(s[p] - '0');
      if (val > 0xFFFFFFFFULL) overflow = 1;
    }
    p++;
  }
  *pos = p;
  if (overflow) return 0;
  *out = neg ? (uint32_t)(0u - (uint32_t)val) : (uint32_t)val;
  return 1;
}

int og_parse_text(const char *path, uint32_t **pu, uint32_t **pv, uint64_t *npairs) {
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  fseek(f, 0, SEEK_END);
  long len = ftell(f);
  fseek(f, 0, SEEK_SET);
  char *s = (char *)malloc((size_t)len + 1);
  if (len > 0 && fread(s, 1, (size_t)len, f) != (size_t)len) { fclose(f); free(s); return -2; }
  fclose(f);
  uint64_t cap = 1024, n = 0;
  uint32_t *u = (uint32_t *)malloc(cap * 4), *v = (uint32_t *)malloc(cap * 4);
  size_t pos = 0, L = (size_t)len;
  while (pos < L) {
    uint32_t a, b;
    int ok = read_uint(s, L, &pos, &a) && read_uint(s, L, &pos, &b);
    if (ok) {
      if (n == cap) { cap *= 2; u = realloc(u, cap * 4); v = realloc(v, cap * 4); }
      u[n] = a; v[n] = b; n++;
    }
    while (pos < L && s[pos] != '\n') pos++;
    if (pos < L) pos++;
  }
  free(s);
  *pu = u; *pv = v; *npairs = n;
  return 0;
}

/* ----------------------------------------------------------------- loader */

static og_graph *alloc_graph(uint32_t n, uint64_t m) {
  og_graph *g = (og_graph *)calloc(1, sizeof(og_graph));
  g->n = n; g->m = m;
  g->off = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
  g->adj = (uint32_t *)malloc((2 * m + 1) * sizeof(uint32_t));
  g->labels = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
  return g;
}

static void finish_stats(og_graph *g) {
  uint32_t md = 0;
  for (uint32_t x = 0; x < g->n; x++) {
    uint64_t d = g->off[x + 1] - g->off[x];
    if (d > md) md = (uint32_t)d;
  }
  g->max_degree = md;
  g->degeneracy = md; /* the loader leaves degeneracy = max degree (src/graph.cc:149) */
}

og_graph *og_from_pairs(const uint32_t *u, const uint32_t *v, uint64_t npairs) {
  uint64_t *e = (uint64_t *)malloc((npairs + 1) * sizeof(uint64_t));
  uint64_t ne = 0;
  for (uint64_t i = 0; i < npairs; i++) {
    uint32_t a = u[i], b = v[i];
    if (a == b) continue;
    if (a > b) { uint32_t t = a; a = b; b = t; }
    e[ne++] = ((uint64_t)a << 32) | b;
  }
  radix_sort_u64(e, ne);
  uint64_t m = 0;
  for (uint64_t i = 0; i < ne; i++)
    if (i == 0 || e[i] != e[i - 1]) e[m++] = e[i];
  /* present labels, ascending (label_to_id, src/graph.cc:123-130) */
  uint64_t *lab = (uint64_t *)malloc((2 * m + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < m; i++) { lab[2 * i] = e[i] >> 32; lab[2 * i + 1] = e[i] & 0xFFFFFFFFu; }
  radix_sort_u64(lab, 2 * m);
  uint64_t n = 0;
  for (uint64_t i = 0; i < 2 * m; i++)
    if (i == 0 || lab[i] != lab[i - 1]) lab[n++] = lab[i];
  og_graph *g = alloc_graph((uint32_t)n, m);
  for (uint64_t i = 0; i < n; i++) g->labels[i] = (uint32_t)lab[i];
  /* map label -> id by binary search over the sorted label list */
  uint32_t *eu = (uint32_t *)malloc((m + 1) * 4), *ev = (uint32_t *)malloc((m + 1) * 4);
  for (uint64_t i = 0; i < m; i++) {
    uint64_t keys[2] = {e[i] >> 32, e[i] & 0xFFFFFFFFu};
    uint32_t ids[2];
    for (int k = 0; k < 2; k++) {
      uint64_t lo = 0, hi = n;
      while (lo < hi) { uint64_t mid = (lo + hi) / 2; if (lab[mid] < keys[k]) lo = mid + 1; else hi = mid; }
      ids[k] = (uint32_t)lo;
    }
    eu[i] = ids[0]; ev[i] = ids[1];
    g->off[ids[0] + 1]++; g->off[ids[1] + 1]++;
  }
  for (uint64_t x = 0; x < n; x++) g->off[x + 1] += g->off[x];
  uint64_t *fill = (uint64_t *)malloc((n + 1) * sizeof(uint64_t));
  memcpy(fill, g->off, (n + 1) * sizeof(uint64_t));
  /* edges in (u,v) order: each row receives its lower neighbours first, then
   * its upper neighbours, both ascending -> rows come out sorted (graph.cc:135-145) */
  for (uint64_t i = 0; i < m; i++) {
    g->adj[fill[eu[i]]++] = ev[i];
    g->adj[fill[ev[i]]++] = eu[i];
  }
  free(fill); free(eu); free(ev); free(lab); free(e);
  finish_stats(g);
  return g;
}

og_graph *og_from_csr(uint32_t n, const uint64_t *off, const uint32_t *adj, const uint32_t *labels) {
  uint64_t m2 = off[n];
  og_graph *g = alloc_graph(n, m2 / 2);
  memcpy(g->off, off, ((size_t)n + 1) * sizeof(uint64_t));
  memcpy(g->adj, adj, m2 * sizeof(uint32_t));
  if (labels) memcpy(g->labels, labels, (size_t)n * 4);
  else for (uint32_t i = 0; i < n; i++) g->labels[i] = i;
  finish_stats(g);
  return g;
}

void og_free(og_graph *g) {
  if (!g) return;
  free(g->off); free(g->adj); free(g->labels); free(g->root_off); free(g);
}

uint32_t og_num_vertices(const og_graph *g) { return g->n; }
uint64_t og_num_edges(const og_graph *g) { return g->m; }
uint32_t og_max_degree(const og_graph *g) { return g->max_degree; }
uint32_t og_degeneracy(const og_graph *g) { return g->degeneracy; }

void og_export(const og_graph *g, uint64_t *off, uint32_t *adj, uint32_t *labels) {
  if (off) memcpy(off, g->off, ((size_t)g->n + 1) * sizeof(uint64_t));
  if (adj) memcpy(adj, g->adj, g->off[g->n] * sizeof(uint32_t));
  if (labels) memcpy(labels, g->labels, (size_t)g->n * 4);
}

/* ------------------------------------------------------------ orderings */

static int cmp_u32(const void *a, const void *b) {
  uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return x < y ? -1 : x > y;
}

int og_apply_order(og_graph *g, const uint32_t *order) {
  uint32_t n = g->n;
  uint32_t *rev = (uint32_t *)malloc(((size_t)n + 1) * 4);
  uint8_t *seen = (uint8_t *)calloc((size_t)n + 1, 1);
  for (uint32_t i = 0; i < n; i++) {
    if (order[i] >= n || seen[order[i]]) { free(rev); free(seen); return -1; }
    seen[order[i]] = 1;
    rev[order[i]] = i;
  }
  free(seen);
  uint64_t *off = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
  for (uint32_t i = 0; i < n; i++) off[i + 1] = off[i] + (g->off[order[i] + 1] - g->off[order[i]]);
  uint32_t *adj = (uint32_t *)malloc((2 * g->m + 1) * 4);
  uint32_t *lab = (uint32_t *)malloc(((size_t)n + 1) * 4);
  uint64_t *fill = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
  memcpy(fill, off, ((size_t)n + 1) * sizeof(uint64_t));
  /* transpose fill: new id i is appended to each neighbour's row in ascending
   * i, so every row comes out sorted without a per-row sort */
  for (uint32_t i = 0; i < n; i++) {
    uint32_t o = order[i];
    for (uint64_t e = g->off[o]; e < g->off[o + 1]; e++) {
      const uint32_t y = rev[g->adj[e]];
      adj[fill[y]++] = i;
    }
    lab[i] = g->labels[o];
  }
  free(fill);
  free(g->off); free(g->adj); free(g->labels); free(g->root_off);
  g->off = off; g->adj = adj; g->labels = lab; g->root_off = NULL;
  free(rev);
  return 0;
}

void og_sort_degeneracy(og_graph *g) {
  uint32_t n = g->n;
  uint32_t *order = (uint32_t *)malloc(((size_t)n + 1) * 4);
  int64_t *deg = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
  for (uint32_t x = 0; x < n; x++) deg[x] = (int64_t)(g->off[x + 1] - g->off[x]);
  uint64_t len = 0;
  int64_t k = 0;
  /* level k: append every vertex whose residual degree is exactly k in id order,
   * then cascade through the appended queue (graph.cc:289-304) */
  while (len < n) {
    uint64_t cur = len;
    k++;
    for (uint32_t x = 0; x < n; x++)
      if (deg[x] == k) order[len++] = x;
    while (cur < len) {
      uint32_t x = order[cur++];
      for (uint64_t e = g->off[x]; e < g->off[x + 1]; e++)
        if (--deg[g->adj[e]] == k) order[len++] = g->adj[e];
    }
  }
  og_apply_order(g, order);
  g->degeneracy = (uint32_t)k;
  free(order); free(deg);
}

/* The engine's own degeneracy order (rdmce_b200/csrc/preprocess.cu,
 * k_peel_rounds), restated sequentially so the oracle can number roots the way
 * the engine does.  Level k starts with a scan that claims every unclaimed
 * vertex of residual degree <= k for the current round; each round then removes
 * its whole frontier, and a neighbour whose residual degree falls to exactly k
 * is claimed for the next round.  An empty round ends the level (its index is
 * skipped); the next level is k + 1 when this one claimed anything, else the
 * smallest surviving residual degree.  Position = (round, id), so vertices of
 * one round keep ascending id order.  Same degeneracy value as the reference's
 * queue (src/graph.cc:281-306); only the order inside a round differs. */
void og_sort_gpu_rounds(og_graph *g) {
  const uint32_t n = g->n;
  int64_t *deg = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
  uint64_t *round = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t)); /* 0 = unclaimed, else round + 1 */
  uint32_t *rem = (uint32_t *)malloc(((size_t)n + 1) * 4), *rem2 = (uint32_t *)malloc(((size_t)n + 1) * 4);
  uint32_t *fr = (uint32_t *)malloc(((size_t)n + 1) * 4), *fr2 = (uint32_t *)malloc(((size_t)n + 1) * 4);
  for (uint32_t x = 0; x < n; x++) { deg[x] = (int64_t)(g->off[x + 1] - g->off[x]); rem[x] = x; }
  uint64_t nrem = n, removed = 0, r = 0;
  int64_t k = 0, degen = 0;
  while (removed < n) {
    uint64_t nf = 0, nsurv = 0;
    int64_t rmin = INT64_MAX;
    for (uint64_t i = 0; i < nrem; i++) {
      const uint32_t v = rem[i];
      if (round[v]) continue;
      if (deg[v] <= k) { round[v] = r + 1; fr[nf++] = v; }
      else { rem2[nsurv++] = v; if (deg[v] < rmin) rmin = deg[v]; }
    }
    uint64_t claims = 0;
    while (nf) {
      claims += nf;
      removed += nf;
      uint64_t nn = 0;
      for (uint64_t i = 0; i < nf; i++) {
        const uint32_t v = fr[i];
        for (uint64_t e = g->off[v]; e < g->off[v + 1]; e++) {
          const uint32_t u = g->adj[e];
          if (round[u]) continue;
          if (--deg[u] == k) { round[u] = r + 2; fr2[nn++] = u; }
        }
      }
      uint32_t *t = fr; fr = fr2; fr2 = t;
      nf = nn;
      r++;
    }
    r++; /* the empty round's index is skipped */
    { uint32_t *t = rem; rem = rem2; rem2 = t; }
    nrem = nsurv;
    if (claims) { degen = k; k++; }
    else if (rmin == INT64_MAX) break;
    else k = (k + 1 > rmin) ? k + 1 : rmin;
  }
  /* order = vertices by (round, id): a counting sort over rounds keeps ids ascending */
  uint64_t *cnt = (uint64_t *)calloc(r + 2, sizeof(uint64_t));
  for (uint32_t x = 0; x < n; x++) cnt[round[x]]++;
  uint64_t acc = 0;
  for (uint64_t i = 0; i < r + 2; i++) { uint64_t c = cnt[i]; cnt[i] = acc; acc += c; }
  uint32_t *order = (uint32_t *)malloc(((size_t)n + 1) * 4);
  for (uint32_t x = 0; x < n; x++) order[cnt[round[x]]++] = x;
  og_apply_order(g, order);
  g->degeneracy = (uint32_t)degen;
  free(order); free(cnt); free(deg); free(round); free(rem); free(rem2); free(fr); free(fr2);
}

void og_core_numbers(const og_graph *g, uint32_t *core) {
  /* bucket peeling (Batagelj-Zaversnik) */
  uint32_t n = g->n, md = 0;
  uint32_t *deg = (uint32_t *)malloc(((size_t)n + 1) * 4);
  for (uint32_t x = 0; x < n; x++) { deg[x] = (uint32_t)(g->off[x + 1] - g->off[x]); if (deg[x] > md) md = deg[x]; }
  uint32_t *bin = (uint32_t *)calloc((size_t)md + 2, 4);
  uint32_t *pos = (uint32_t *)malloc(((size_t)n + 1) * 4), *vert = (uint32_t *)malloc(((size_t)n + 1) * 4);
  for (uint32_t x = 0; x < n; x++) bin[deg[x]]++;
  uint32_t start = 0;
  for (uint32_t d = 0; d <= md; d++) { uint32_t c = bin[d]; bin[d] = start; start += c; }
  for (uint32_t x = 0; x < n; x++) { pos[x] = bin[deg[x]]; vert[pos[x]] = x; bin[deg[x]]++; }
  for (uint32_t d = md; d >= 1; d--) bin[d] = bin[d - 1];
  bin[0] = 0;
  for (uint32_t i = 0; i < n; i++) {
    uint32_t x = vert[i];
    for (uint64_t e = g->off[x]; e < g->off[x + 1]; e++) {
      uint32_t y = g->adj[e];
      if (deg[y] > deg[x]) {
        uint32_t dy = deg[y], py = pos[y], pw = bin[dy], w = vert[pw];
        if (y != w) { pos[y] = pw; vert[py] = w; pos[w] = py; vert[pw] = y; }
        bin[dy]++;
        deg[y]--;
      }
    }
  }
  for (uint32_t x = 0; x < n; x++) core[x] = deg[x];
  free(deg); free(bin); free(pos); free(vert);
}

/* ------------------------------------------------------------------ roots */

static void build_root_off(og_graph *g) {
  if (g->root_off) return;
  uint64_t *ro = (uint64_t *)malloc(((size_t)g->n + 1) * sizeof(uint64_t));
  ro[0] = 0;
  for (uint32_t x = 0; x < g->n; x++) {
    uint64_t up = 0;
    for (uint64_t e = g->off[x]; e < g->off[x + 1]; e++) up += g->adj[e] > x;
    ro[x + 1] = ro[x] + up;
  }
  g->root_off = ro;
}

static void root_of(const og_graph *g, uint64_t r, uint32_t *v0, uint32_t *v1) {
  uint64_t lo = 0, hi = g->n; /* last x with root_off[x] <= r */
  while (hi - lo > 1) {
    uint64_t mid = (lo + hi) / 2;
    if (g->root_off[mid] <= r) lo = mid; else hi = mid;
  }
  uint32_t x = (uint32_t)lo;
  uint64_t d = g->off[x + 1] - g->off[x];
  uint64_t up = g->root_off[x + 1] - g->root_off[x];
  *v0 = x;
  *v1 = g->adj[g->off[x] + (d - up) + (r - g->root_off[x])];
}

void og_root(const og_graph *g, uint64_t r, uint32_t *v0, uint32_t *v1) {
  build_root_off((og_graph *)g);
  root_of(g, r, v0, v1);
}

/* -------------------------------------------------------------- BK search */

typedef struct {
  const og_graph *g;
  int expand_r;
  uint32_t W;
  uint32_t nrows;
  uint64_t *rows; size_t rows_cap;
  uint32_t *cand; size_t cand_cap;
  uint64_t *h1, *h2; size_t h_cap;
  uint32_t *abuf; size_t acap, atop;
  uint64_t *pbuf; size_t pcap, ptop;
  uint32_t *clique; /* for og_list_cliques */
  uint32_t *rlist; size_t rlist_cap;
  uint32_t *plist; /* P members of the current root */
  uint32_t v0, v1;
  FILE *out;
  og_result *res;
  atomic_int *stop; /* og_mce_roots_timed: set at the deadline, unwinds the search */
} bk_ctx;

static void *grow(void *p, size_t *cap, size_t need, size_t elem) {
  if (need <= *cap) return p;
  size_t c = *cap ? *cap : 1024;
  while (c < need) c *= 2;
  *cap = c;
  return realloc(p, c * elem);
}

static inline uint32_t popc_vec(const uint64_t *a, uint32_t W) {
  uint32_t c = 0;
  for (uint32_t w = 0; w < W; w++) c += (uint32_t)__builtin_popcountll(a[w]);
  return c;
}

static void emit(bk_ctx *c, uint32_t size, uint64_t s1, uint64_t s2, const uint64_t *rbits) {
  og_result *r = c->res;
  r->count++;
  r->checksum += finish_hash(s1, s2, size);
  if (size < OG_HIST_LEN) r->hist[size]++;
  if (size > r->max_size) r->max_size = size;
  if (c->out) {
    uint32_t k = 0;
    c->rlist = (uint32_t *)grow(c->rlist, &c->rlist_cap, size + 2, 4);
    c->rlist[k++] = c->g->labels[c->v0];
    c->rlist[k++] = c->g->labels[c->v1];
    if (rbits)
      for (uint32_t w = 0; w < c->W; w++)
        for (uint64_t b = rbits[w]; b; b &= b - 1)
          c->rlist[k++] = c->g->labels[c->plist[w * 64 + __builtin_ctzll(b)]];
    qsort(c->rlist, k, 4, cmp_u32);
    for (uint32_t i = 0; i < k; i++) fprintf(c->out, i ? " %u" : "%u", c->rlist[i]);
    fputc('\n', c->out);
  }
}

/* Frame layout in pbuf at offset po: [P | R] (2W words) owned by the caller. */
static void bk_node(bk_ctx *c, size_t po, size_t ao, uint32_t nA, uint32_t rsize, uint64_t s1, uint64_t s2) {
  const uint32_t W = c->W;
  og_result *res = c->res;
  if (c->stop && atomic_load_explicit(c->stop, memory_order_relaxed)) return;
  res->nodes++;
  {
    const uint64_t *P = c->pbuf + po;
    if (popc_vec(P, W) == 0) {
      if (nA == 0) emit(c, rsize + 2, s1, s2, c->pbuf + po + W);
      return;
    }
  }
  /* pivot: argmin over active rows of |P \ row|, ties to the lowest row */
  uint32_t best = UINT32_MAX, piv = 0;
  {
    const uint64_t *P = c->pbuf + po;
    for (uint32_t t = 0; t < nA; t++) {
      uint32_t i = c->abuf[ao + t];
      const uint64_t *row = c->rows + (size_t)i * W;
      uint32_t cnt = 0;
      for (uint32_t w = 0; w < W; w++) cnt += (uint32_t)__builtin_popcountll(P[w] & ~row[w]);
      res->pivot_words += W;
      if (cnt < best) { best = cnt; piv = i; if (cnt == 0) break; }
    }
  }
  if (best == 0) return; /* an X vertex is adjacent to all of P: nothing maximal below */
  /* frame: VP, Pcur, child P, child R, E mask (5W words) */
  size_t base = c->ptop;
  c->ptop += 5 * (size_t)W;
  c->pbuf = (uint64_t *)grow(c->pbuf, &c->pcap, c->ptop, 8);
  {
    uint64_t *P = c->pbuf + po, *VP = c->pbuf + base, *Pc = VP + W;
    const uint64_t *prow = c->rows + (size_t)piv * W;
    for (uint32_t w = 0; w < W; w++) { VP[w] = P[w] & ~prow[w]; Pc[w] = P[w]; }
  }
  for (uint32_t wq = 0; wq < W; wq++) {
    for (;;) {
      uint64_t *VP = c->pbuf + base, *Pcur = VP + W, *CP = VP + 2 * W, *CR = VP + 3 * W, *E = VP + 4 * W;
      const uint64_t *R = c->pbuf + po + W;
      if (!VP[wq]) break;
      uint32_t b = (uint32_t)__builtin_ctzll(VP[wq]);
      VP[wq] &= VP[wq] - 1;
      uint32_t q = wq * 64 + b;
      const uint64_t *rowq = c->rows + (size_t)q * W;
      for (uint32_t w = 0; w < W; w++) { CP[w] = Pcur[w] & rowq[w]; CR[w] = R[w]; E[w] = 0; }
      Pcur[wq] &= ~(1ULL << b);
      CR[wq] |= 1ULL << b;
      uint32_t rs = rsize + 1;
      uint64_t t1 = s1 + c->h1[q], t2 = s2 + c->h2[q];
      if (c->expand_r && popc_vec(CP, W) > 1) {
        for (uint32_t w = 0; w < W; w++)
          for (uint64_t bb = CP[w]; bb; bb &= bb - 1) {
            uint32_t i = w * 64 + (uint32_t)__builtin_ctzll(bb);
            const uint64_t *ri = c->rows + (size_t)i * W;
            uint32_t cnt = 0;
            for (uint32_t x = 0; x < W; x++) cnt += (uint32_t)__builtin_popcountll(CP[x] & ~ri[x]);
            if (cnt == 1) E[w] |= 1ULL << (i & 63);
          }
        for (uint32_t w = 0; w < W; w++)
          for (uint64_t bb = E[w]; bb; bb &= bb - 1) {
            uint32_t i = w * 64 + (uint32_t)__builtin_ctzll(bb);
            rs++; t1 += c->h1[i]; t2 += c->h2[i];
          }
        for (uint32_t w = 0; w < W; w++) { CP[w] &= ~E[w]; CR[w] |= E[w]; }
      }
      /* child active rows: rows in A holding bit q and every E bit */
      E[wq] |= 1ULL << b;
      size_t a2 = c->atop;
      c->abuf = (uint32_t *)grow(c->abuf, &c->acap, a2 + nA + 1, 4);
      uint32_t n2 = 0;
      for (uint32_t t = 0; t < nA; t++) {
        uint32_t i = c->abuf[ao + t];
        const uint64_t *row = c->rows + (size_t)i * W;
        res->filter_rows++;
        if (!((row[wq] >> b) & 1)) continue;
        int ok = 1;
        for (uint32_t w = 0; w < W && ok; w++)
          if ((row[w] & E[w]) != E[w]) ok = 0;
        if (ok) c->abuf[a2 + n2++] = i;
      }
      c->atop = a2 + n2;
      /* the child frame [P | R] lives at CP (offset base + 2W) */
      bk_node(c, base + 2 * (size_t)W, a2, n2, rs, t1, t2);
      c->atop = a2;
    }
  }
  c->ptop = base;
}

static inline uint64_t lab_h1(const og_graph *g, uint32_t x) { return og_mix64((uint64_t)g->labels[x]); }
static inline uint64_t lab_h2(const og_graph *g, uint32_t x) { return og_mix64((uint64_t)g->labels[x] ^ GOLDEN); }

static void run_root(bk_ctx *c, uint32_t v0, uint32_t v1) {
  const og_graph *g = c->g;
  og_result *res = c->res;
  c->v0 = v0; c->v1 = v1;
  const uint32_t *a = g->adj + g->off[v0], *b = g->adj + g->off[v1];
  uint64_t da = g->off[v0 + 1] - g->off[v0], db = g->off[v1 + 1] - g->off[v1];
  c->cand = (uint32_t *)grow(c->cand, &c->cand_cap, (da < db ? da : db) + 1, 4);
  uint64_t i = 0, j = 0, nc = 0;
  while (i < da && j < db) {
    if (a[i] == b[j]) { c->cand[nc++] = a[i]; i++; j++; }
    else if (a[i] < b[j]) i++;
    else j++;
  }
  res->build_bytes += 4 * (da + db);
  uint64_t x = 0;
  while (x < nc && c->cand[x] < v1) x++;
  uint32_t p = (uint32_t)(nc - x);
  uint64_t s1 = lab_h1(g, v0) + lab_h1(g, v1), s2 = lab_h2(g, v0) + lab_h2(g, v1);
  res->nodes++;
  if (p == 0) {
    if (x == 0) emit(c, 2, s1, s2, NULL);
    return;
  }
  res->nodes--; /* counted again by bk_node */
  uint32_t W = (p + 63) / 64;
  c->W = W;
  const uint32_t *P = c->cand + x;
  c->plist = (uint32_t *)P;
  c->rows = (uint64_t *)grow(c->rows, &c->rows_cap, (size_t)(p + x) * W + 1, 8);
  uint32_t nrows = 0;
  for (uint64_t r = 0; r < p + x; r++) {
    uint32_t u = r < p ? P[r] : c->cand[r - p];
    uint64_t *row = c->rows + (size_t)nrows * W;
    memset(row, 0, W * 8);
    const uint32_t *nu = g->adj + g->off[u];
    uint64_t du = g->off[u + 1] - g->off[u], s = 0, t = 0;
    int any = 0;
    while (s < du && t < p) {
      if (nu[s] == P[t]) { row[t >> 6] |= 1ULL << (t & 63); any = 1; s++; t++; }
      else if (nu[s] < P[t]) s++;
      else t++;
    }
    res->build_bytes += 4 * du + 8 * (uint64_t)W;
    if (r < p || any) nrows++; /* drop X rows without a P neighbour */
  }
  c->nrows = nrows;
  c->h1 = (uint64_t *)grow(c->h1, &c->h_cap, p + 1, 8);
  c->h2 = (uint64_t *)realloc(c->h2, c->h_cap * 8);
  for (uint32_t k = 0; k < p; k++) { c->h1[k] = lab_h1(g, P[k]); c->h2[k] = lab_h2(g, P[k]); }
  c->abuf = (uint32_t *)grow(c->abuf, &c->acap, nrows + 1, 4);
  for (uint32_t k = 0; k < nrows; k++) c->abuf[k] = k;
  c->atop = nrows;
  c->ptop = 2 * (size_t)W;
  c->pbuf = (uint64_t *)grow(c->pbuf, &c->pcap, c->ptop + 5 * (size_t)W, 8);
  for (uint32_t w = 0; w < W; w++) {
    uint32_t lo = w * 64;
    c->pbuf[w] = (p - lo >= 64) ? ~0ULL : ((1ULL << (p - lo)) - 1);
    c->pbuf[W + w] = 0;
  }
  bk_node(c, 0, 0, nrows, 0, s1, s2);
}

static void ctx_free(bk_ctx *c) {
  free(c->rows); free(c->cand); free(c->h1); free(c->h2); free(c->abuf); free(c->pbuf); free(c->rlist);
}

typedef struct {
  const og_graph *g;
  uint64_t begin, end;
  const uint64_t *roots;        /* optional explicit list */
  uint64_t *counts, *checksums; /* per-root outputs for the explicit list */
  int expand_r;
  atomic_uint_fast64_t next;
  og_result *partial;
  int nthreads;
  atomic_int stop;
  atomic_int running;
  int timed;
} job_t;

typedef struct { job_t *job; int tid; } targ_t;

static void *worker(void *arg) {
  targ_t *t = (targ_t *)arg;
  job_t *J = t->job;
  bk_ctx c;
  memset(&c, 0, sizeof(c));
  c.g = J->g;
  c.expand_r = J->expand_r;
  c.res = &J->partial[t->tid];
  if (J->timed) c.stop = &J->stop;
  const uint64_t chunk = J->timed ? 1 : 16;
  uint64_t total = J->end - J->begin;
  for (;;) {
    if (J->timed && atomic_load(&J->stop)) break;
    uint64_t k0 = atomic_fetch_add(&J->next, chunk);
    if (k0 >= total) break;
    uint64_t k1 = k0 + chunk < total ? k0 + chunk : total;
    for (uint64_t k = k0; k < k1; k++) {
      uint32_t v0, v1;
      if (J->roots) {
        root_of(J->g, J->roots[k], &v0, &v1);
        uint64_t c0 = c.res->count, h0 = c.res->checksum;
        run_root(&c, v0, v1);
        J->counts[k] = c.res->count - c0;
        J->checksums[k] = c.res->checksum - h0;
      } else {
        root_of(J->g, J->begin + k, &v0, &v1);
        run_root(&c, v0, v1);
      }
    }
  }
  ctx_free(&c);
  atomic_fetch_sub(&J->running, 1);
  return NULL;
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* seconds > 0: stop the search at the deadline (partial counts are kept) */
static int run_job_until(job_t *J, int threads, double seconds, double *elapsed) {
  if (threads < 1) threads = 1;
  J->nthreads = threads;
  J->partial = (og_result *)calloc((size_t)threads, sizeof(og_result));
  atomic_init(&J->next, 0);
  atomic_init(&J->stop, 0);
  atomic_init(&J->running, threads);
  J->timed = seconds > 0;
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
  targ_t *ta = (targ_t *)malloc(sizeof(targ_t) * (size_t)threads);
  const double t0 = now_s();
  for (int i = 0; i < threads; i++) {
    ta[i].job = J; ta[i].tid = i;
    pthread_create(&th[i], NULL, worker, &ta[i]);
  }
  if (J->timed) {
    while (atomic_load(&J->running) > 0 && now_s() - t0 < seconds) {
      struct timespec ts = {0, 5 * 1000 * 1000};
      nanosleep(&ts, NULL);
    }
    atomic_store(&J->stop, 1);
  }
  for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
  if (elapsed) *elapsed = now_s() - t0;
  free(th); free(ta);
  return 0;
}

static int run_job(job_t *J, int threads) { return run_job_until(J, threads, 0.0, NULL); }

static void merge(og_result *out, const og_result *in, int k) {
  memset(out, 0, sizeof(*out));
  for (int t = 0; t < k; t++) {
    out->count += in[t].count;
    out->checksum += in[t].checksum;
    out->nodes += in[t].nodes;
    out->pivot_words += in[t].pivot_words;
    out->filter_rows += in[t].filter_rows;
    out->build_bytes += in[t].build_bytes;
    if (in[t].max_size > out->max_size) out->max_size = in[t].max_size;
    for (int s = 0; s < OG_HIST_LEN; s++) out->hist[s] += in[t].hist[s];
  }
}

int og_mce(const og_graph *g, uint64_t begin, uint64_t end, int threads, int expand_r, og_result *out) {
  build_root_off((og_graph *)g);
  if (end > g->m) end = g->m;
  if (begin > end) begin = end;
  job_t J;
  memset(&J, 0, sizeof(J));
  J.g = g; J.begin = begin; J.end = end; J.expand_r = expand_r;
  run_job(&J, threads);
  merge(out, J.partial, J.nthreads);
  free(J.partial);
  return 0;
}

int og_mce_roots(const og_graph *g, const uint64_t *roots, uint64_t nroots, int threads,
                 uint64_t *counts, uint64_t *checksums) {
  build_root_off((og_graph *)g);
  for (uint64_t k = 0; k < nroots; k++)
    if (roots[k] >= g->m) return -1;
  job_t J;
  memset(&J, 0, sizeof(J));
  J.g = g; J.begin = 0; J.end = nroots; J.roots = roots; J.counts = counts; J.checksums = checksums;
  J.expand_r = 1;
  run_job(&J, threads);
  free(J.partial);
  return 0;
}

int og_mce_root_set(const og_graph *g, const uint64_t *roots, uint64_t nroots, int threads, uint64_t *counts,
                    uint64_t *checksums, og_result *out) {
  build_root_off((og_graph *)g);
  for (uint64_t k = 0; k < nroots; k++)
    if (roots[k] >= g->m) return -1;
  uint64_t *cnt = counts ? counts : (uint64_t *)calloc(nroots ? nroots : 1, 8);
  uint64_t *chk = checksums ? checksums : (uint64_t *)calloc(nroots ? nroots : 1, 8);
  job_t J;
  memset(&J, 0, sizeof(J));
  J.g = g; J.begin = 0; J.end = nroots; J.roots = roots; J.counts = cnt; J.checksums = chk;
  J.expand_r = 1;
  run_job(&J, threads);
  merge(out, J.partial, J.nthreads);
  free(J.partial);
  if (!counts) free(cnt);
  if (!checksums) free(chk);
  return 0;
}

int og_mce_roots_timed(const og_graph *g, const uint64_t *roots, uint64_t nroots, int threads, double seconds,
                       og_result *out, uint64_t *roots_started, double *elapsed) {
  build_root_off((og_graph *)g);
  for (uint64_t k = 0; k < nroots; k++)
    if (roots[k] >= g->m) return -1;
  uint64_t *cnt = (uint64_t *)calloc(nroots ? nroots : 1, 8), *chk = (uint64_t *)calloc(nroots ? nroots : 1, 8);
  job_t J;
  memset(&J, 0, sizeof(J));
  J.g = g; J.begin = 0; J.end = nroots; J.roots = roots; J.counts = cnt; J.checksums = chk;
  J.expand_r = 1;
  run_job_until(&J, threads, seconds, elapsed);
  merge(out, J.partial, J.nthreads);
  uint64_t started = atomic_load(&J.next);
  if (roots_started) *roots_started = started < nroots ? started : nroots;
  free(J.partial); free(cnt); free(chk);
  return 0;
}

int og_list_cliques(const og_graph *g, const char *path) {
  build_root_off((og_graph *)g);
  FILE *f = fopen(path, "w");
  if (!f) return -1;
  bk_ctx c;
  memset(&c, 0, sizeof(c));
  og_result *r = (og_result *)calloc(1, sizeof(og_result));
  c.g = g; c.expand_r = 1; c.res = r; c.out = f;
  for (uint64_t k = 0; k < g->m; k++) {
    uint32_t v0, v1;
    root_of(g, k, &v0, &v1);
    run_root(&c, v0, v1);
  }
  ctx_free(&c);
  free(r);
  fclose(f);
  return 0;
}

/* ----------------------------------------------------------- .bin container */

int og_store_bin(const og_graph *g, const char *path) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  uint64_t hdr[4] = {g->n, g->m, g->max_degree, g->degeneracy};
  fwrite(hdr, 8, 4, f);
  for (uint32_t x = 0; x < g->n; x++) {
    uint64_t d = g->off[x + 1] - g->off[x];
    fwrite(&d, 8, 1, f);
    fwrite(g->adj + g->off[x], 4, d, f);
  }
  fwrite(g->labels, 4, g->n, f);
  fclose(f);
  return 0;
}

og_graph *og_load_bin(const char *path) {
  FILE *f = fopen(path, "rb");
  if (!f) return NULL;
  uint64_t hdr[4];
  if (fread(hdr, 8, 4, f) != 4) { fclose(f); return NULL; }
  og_graph *g = alloc_graph((uint32_t)hdr[0], hdr[1]);
  for (uint32_t x = 0; x < g->n; x++) {
    uint64_t d;
    if (fread(&d, 8, 1, f) != 1 || g->off[x] + d > 2 * g->m) { fclose(f); og_free(g); return NULL; }
    g->off[x + 1] = g->off[x] + d;
    if (fread(g->adj + g->off[x], 4, d, f) != d) { fclose(f); og_free(g); return NULL; }
  }
  if (fread(g->labels, 4, g->n, f) != g->n) { fclose(f); og_free(g); return NULL; }
  fclose(f);
  g->max_degree = (uint32_t)hdr[2];
  g->degeneracy = (uint32_t)hdr[3];
  return g;
}

/* Per-root ego-network sizes: p, x before and after dropping X rows with no P
 * neighbour (include/graph_gpu.cuh:90-106).  Used to size scratch tiers. */
static void root_sizes_impl(const og_graph *g, const uint64_t *list, uint64_t begin, uint64_t end, uint32_t *p_out,
                            uint32_t *x_out, uint32_t *xc_out) {
  build_root_off((og_graph *)g);
  uint32_t *cand = NULL;
  size_t cap = 0;
  for (uint64_t k = begin; k < end; k++) {
    const uint64_t r = list ? list[k] : k;
    if (r >= g->m) break;
    uint32_t v0, v1;
    root_of(g, r, &v0, &v1);
    const uint32_t *a = g->adj + g->off[v0], *b = g->adj + g->off[v1];
    uint64_t da = g->off[v0 + 1] - g->off[v0], db = g->off[v1 + 1] - g->off[v1];
    cand = (uint32_t *)grow(cand, &cap, (da < db ? da : db) + 1, 4);
    uint64_t i = 0, j = 0, nc = 0;
    while (i < da && j < db) {
      if (a[i] == b[j]) { cand[nc++] = a[i]; i++; j++; }
      else if (a[i] < b[j]) i++;
      else j++;
    }
    uint64_t x = 0;
    while (x < nc && cand[x] < v1) x++;
    uint64_t p = nc - x, xc = 0;
    if (p > 0)
      for (uint64_t k = 0; k < x; k++) {
        uint32_t u = cand[k];
        const uint32_t *nu = g->adj + g->off[u];
        uint64_t du = g->off[u + 1] - g->off[u], s = 0, t = 0;
        while (s < du && t < p) {
          if (nu[s] == cand[x + t]) { xc++; break; }
          else if (nu[s] < cand[x + t]) s++;
          else t++;
        }
      }
    p_out[k - begin] = (uint32_t)p;
    x_out[k - begin] = (uint32_t)x;
    xc_out[k - begin] = (uint32_t)xc;
  }
  free(cand);
}

void og_root_sizes(const og_graph *g, uint64_t begin, uint64_t end, uint32_t *p_out, uint32_t *x_out,
                   uint32_t *xc_out) {
  root_sizes_impl(g, NULL, begin, end < g->m ? end : g->m, p_out, x_out, xc_out);
}

void og_root_sizes_list(const og_graph *g, const uint64_t *roots, uint64_t nroots, uint32_t *p_out, uint32_t *x_out,
                        uint32_t *xc_out) {
  root_sizes_impl(g, roots, 0, nroots, p_out, x_out, xc_out);
}
