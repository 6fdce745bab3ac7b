/*
 * oracle.h -- CPU restatement of the RDMCE maximal-clique-enumeration hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls this
 * code; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do,
 * and only as the checker.  Every function cites the reference file:line whose
 * behaviour it restates (paths relative to the RDMCE project root).
 *
 * Pinned by: the reference's own CPU solver (MceSolver, src/mce.cc) compiled
 * out-of-tree into oracle/_ref by oracle/Makefile (counts, degeneracy, loader),
 * and by networkx.find_cliques fixtures under tests/golden (count, histogram,
 * checksum).
 */
#ifndef RDMCE_ORACLE_H
#define RDMCE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OG_HIST_LEN 8192

typedef struct og_graph og_graph;

typedef struct og_result {
  uint64_t count;      /* maximal cliques */
  uint64_t checksum;   /* wrapping sum of the per-clique set hash */
  uint64_t nodes;      /* search-tree nodes visited (canonical pivot rule) */
  uint64_t pivot_words;/* 64-bit row words read by pivot scans */
  uint64_t filter_rows;/* rows tested when building child active lists */
  uint64_t build_bytes;/* algorithmic bytes of candidate intersection + bitmap build */
  uint32_t max_size;
  uint32_t pad;
  uint64_t hist[OG_HIST_LEN]; /* hist[s] = number of maximal cliques of size s */
} og_result;

/* SplitMix64 output function (Steele, Lea & Flood 2014) and the clique set hash. */
uint64_t og_mix64(uint64_t x);
uint64_t og_clique_hash(const uint32_t *labels, uint32_t size);

/* Text COO parse with std::istream `>>` semantics (src/graph.cc:82-104). */
int og_parse_text(const char *path, uint32_t **u, uint32_t **v, uint64_t *npairs);
void og_free_buf(void *p);

/* Graph construction with the reference loader conventions (src/graph.cc:64-152). */
og_graph *og_from_pairs(const uint32_t *u, const uint32_t *v, uint64_t npairs);
/* Graph from an already-built symmetric CSR with sorted rows (e.g. a GPU export). */
og_graph *og_from_csr(uint32_t n, const uint64_t *off, const uint32_t *adj, const uint32_t *labels);
void og_free(og_graph *g);

uint32_t og_num_vertices(const og_graph *g);
uint64_t og_num_edges(const og_graph *g);
uint32_t og_max_degree(const og_graph *g);
uint32_t og_degeneracy(const og_graph *g);
/* Copies out CSR (off has n+1 entries, adj 2m) and labels; any pointer may be NULL. */
void og_export(const og_graph *g, uint64_t *off, uint32_t *adj, uint32_t *labels);

/* Degeneracy order exactly as Graph::SortByDegeneracy + ApplyOrder (src/graph.cc:281-306, 54-77). */
void og_sort_degeneracy(og_graph *g);
/* The engine's round-synchronous k-core peel (rdmce_b200/csrc/preprocess.cu,
 * k_peel_rounds): position = (round, id).  Gives the engine's exact CSR, so
 * root ids (edges v0 < v1 in CSR order) agree with the engine's. */
void og_sort_gpu_rounds(og_graph *g);
/* Relabel with an explicit order: new id i is old vertex order[i]. */
int og_apply_order(og_graph *g, const uint32_t *order);
/* Core number of every vertex (any valid peeling gives the same numbers). */
void og_core_numbers(const og_graph *g, uint32_t *core);

/* Roots are the undirected edges (v0 < v1) in CSR order, indices 0..m-1. */
void og_root(const og_graph *g, uint64_t r, uint32_t *v0, uint32_t *v1);

/* Enumerate all maximal cliques from roots [begin, end) with `threads` threads. */
int og_mce(const og_graph *g, uint64_t begin, uint64_t end, int threads, int expand_r, og_result *out);
/* Per-root count and checksum for an explicit root list. */
int og_mce_roots(const og_graph *g, const uint64_t *roots, uint64_t nroots, int threads,
                 uint64_t *counts, uint64_t *checksums);
/* The same over an explicit root list, also returning the merged result
 * (count, checksum, histogram, largest size); counts/checksums may be NULL. */
int og_mce_root_set(const og_graph *g, const uint64_t *roots, uint64_t nroots, int threads, uint64_t *counts,
                    uint64_t *checksums, og_result *out);
/* Time-bounded variant for CPU baselines: threads claim roots of the list
 * until `seconds` pass, then the search unwinds; `out` holds what was found
 * by then (count, histogram, nodes), `roots_started` the roots claimed. */
int og_mce_roots_timed(const og_graph *g, const uint64_t *roots, uint64_t nroots, int threads, double seconds,
                       og_result *out, uint64_t *roots_started, double *elapsed);

int og_list_cliques(const og_graph *g, const char *path);

/* Per-root ego sizes p, x (all common neighbours below v1) and x after X-row compaction. */
void og_root_sizes(const og_graph *g, uint64_t begin, uint64_t end, uint32_t *p_out, uint32_t *x_out,
                   uint32_t *xc_out);

/* The same for an explicit list of root ids. */
void og_root_sizes_list(const og_graph *g, const uint64_t *roots, uint64_t nroots, uint32_t *p_out, uint32_t *x_out,
                        uint32_t *xc_out);

/* The reference `.bin` container (src/graph.cc:154-213). */
int og_store_bin(const og_graph *g, const char *path);
og_graph *og_load_bin(const char *path);

#ifdef __cplusplus
}
#endif
#endif
