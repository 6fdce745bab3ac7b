/*
 * rdmce.h -- C ABI of the B200-native maximal-clique-enumeration engine.
 *
 * The RDMCE reference exports no C ABI: its single-GPU path is the C++ classes
 * Graph (include/graph.h:12-52) and MceGpuSolver (include/mce_gpu.cuh:15-24)
 * compiled into one executable, plus the CLI `RDMCE -i <file>` (main.cc:13-53).
 * Each entry point below names the reference interface it replaces.  A C++
 * facade with the reference's class names sits on top of this ABI in
 * rdmce_b200/csrc/rdmce_graph.h.
 *
 * Conventions
 *   - Every call returns an mce_status and never exits the process (the
 *     reference calls exit() from CUDA_CHECK, include/common.cuh:102-114).
 *   - Plain pointers and sizes only.  Host pointers unless a name says `device`.
 *   - Opaque handles are freed by their *_free function.  A handle may be used
 *     from one host thread at a time.
 *   - Device waits inside kernels are bounded; an expired wait returns
 *     MCE_ERR_TIMEOUT and leaves the CUDA context usable.
 *   - Vertex labels are the caller's uint32 ids.  Isolated vertices and
 *     vertices with only self-loops are dropped, as the reference loader does
 *     (src/graph.cc:64-152); every reported clique therefore has size >= 2.
 *   - Results are exact: count, clique-size histogram and a 64-bit checksum
 *     = sum over cliques C (mod 2^64) of mix64(s1 ^ rotl(s2,31) ^ (|C| << 56)),
 *     s1 = sum mix64(l), s2 = sum mix64(l ^ 0x9E3779B97F4A7C15) over the
 *     original labels l of C, mix64 = the SplitMix64 output function.
 */
#ifndef RDMCE_H
#define RDMCE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCE_HIST_LEN 8192  /* histogram bins: clique sizes 0..8191 */
#define MCE_PHASES 6

typedef enum mce_status {
  MCE_OK = 0,
  MCE_ERR_INVALID_ARG = 1,   /* null pointer, bad size or option */
  MCE_ERR_CAPACITY = 2,      /* caller buffer too small; the required size is reported */
  MCE_ERR_IO = 3,            /* file could not be opened, read or written */
  MCE_ERR_FORMAT = 4,        /* truncated or inconsistent .bin / CSR input */
  MCE_ERR_NO_DEVICE = 5,     /* no usable CUDA device */
  MCE_ERR_CUDA = 6,          /* a CUDA runtime call failed */
  MCE_ERR_OUT_OF_MEMORY = 7, /* device or host allocation failed */
  MCE_ERR_TIMEOUT = 8,       /* a bounded device-side wait expired */
  MCE_ERR_TOO_LARGE = 9,     /* graph exceeds the 32-bit CSR limits (2m < 2^32) */
  MCE_ERR_BUSY = 10,         /* server admission refused for now */
  MCE_ERR_NOT_FOUND = 11,    /* unknown request id */
  MCE_ERR_INTERNAL = 12
} mce_status;

/* Phase timers reported in mce_result.phase_ms (milliseconds, device events). */
enum { MCE_PHASE_H2D = 0, MCE_PHASE_PREPROCESS = 1, MCE_PHASE_SETUP = 2, MCE_PHASE_ENUMERATE = 3,
       MCE_PHASE_D2H = 4, MCE_PHASE_TOTAL = 5 };

/* Vertex order applied before enumeration (main.cc:56-88 `-o`). */
typedef enum mce_order { MCE_ORDER_DEGENERACY = 0, MCE_ORDER_UNCHANGED = 1, MCE_ORDER_DEGREE_ASC = 2,
                         MCE_ORDER_DEGREE_DESC = 3 } mce_order;

typedef struct mce_options {
  int device;                 /* CUDA ordinal (default 0) */
  int order;                  /* mce_order (default degeneracy) */
  uint32_t warps_per_block;   /* warps per block (<= 8); 0 = 8 */
  uint32_t blocks_per_sm;     /* resident 8-warp blocks per SM, 1..5, which also picks the kernel's
                                 register budget (3: 85, 4: 64, 5: 51 registers a thread).
                                 0 = autotuned: per graph and per workload (root range or root
                                 list, flags), the first three solves run 4, 5 and 3 blocks per
                                 SM in turn, timing each; later solves use the fastest. */
  uint32_t share_bound;       /* task-share bound tau; 0 = 24 (BkPivotBitBalance.cuh:6-8) */
  int expand_r;               /* aggressive node generation (mce_gpu.cuh:5); default 1 */
  uint64_t root_begin;        /* enumerate roots [root_begin, root_end); 0,0 = all roots */
  uint64_t root_end;
  uint64_t spin_limit;        /* bound on every device-side wait; 0 = default */
  void *stream;               /* cudaStream_t to run on; NULL = the engine's own stream */
  uint32_t flags;             /* MCE_FLAG_* */
  uint32_t reg_share_bound;   /* tau inside the register tiers (<= 64 columns); 0 = 24, never above share_bound */
  uint32_t slab_kib;          /* cap on each warp's scratch slab in KiB (min 16); 0 = 4096.  Roots whose
                                 ego network does not fit are solved in a second pass with larger slabs. */
  uint32_t heavy_warps;       /* cap on the warps of that second pass; 0 = as many as memory allows */
  uint32_t reserved[4];
} mce_options;

#define MCE_FLAG_NO_SHARING 1u   /* disable inter-warp task sharing (the NB ablation) */
#define MCE_FLAG_PER_ROOT   2u   /* fill per-root counts (mce_solve_roots) */
#define MCE_FLAG_QUIET      4u
#define MCE_FLAG_STATS      8u   /* count search-tree nodes and word-ops into mce_result (slower) */

typedef struct mce_result {
  uint64_t count;             /* maximal cliques */
  uint64_t checksum;          /* see header comment */
  uint32_t max_size;          /* largest clique size */
  uint32_t degeneracy;
  uint32_t max_degree;
  uint32_t status_detail;     /* nonzero: device error word (see mce_status_str) */
  uint32_t blocks_per_sm;     /* resident 8-warp blocks per SM the enumeration ran with */
  uint32_t autotune;          /* 0: blocks_per_sm was set by the caller; 1: the autotuner was
                                 trying this setting; 2: the autotuner's choice */
  uint64_t num_vertices;      /* non-isolated vertices */
  uint64_t num_edges;         /* undirected simple edges */
  uint64_t roots;             /* roots enumerated */
  uint64_t shared_tasks;      /* tasks handed between warps */
  uint64_t heavy_roots;       /* roots that went through the large-scratch pass */
  uint64_t nodes;             /* search-tree nodes visited (with MCE_FLAG_STATS, else 0) */
  uint64_t word_ops;          /* bitmap row word operations (AND/ANDN/POPC; with MCE_FLAG_STATS) */
  uint64_t build_bytes;       /* algorithmic bytes of the roots' ego-network builds (with MCE_FLAG_STATS):
                                 per root 4 (d(v0) + d(v1)) + sum over members u of P and X of
                                 (4 d(u) + 8 W), W = ceil(|P| / 64) */
  uint64_t launches;          /* enumeration kernel launches */
  uint64_t warp_cycles[8];    /* warp clock cycles by phase: [0] root build, [1] 64-bit tier,
                                 [2] general tier, [3] exposing tasks, [4] idle, [5] queue,
                                 [6] 32-bit tier, [7] reserved (0) */
  uint64_t max_item_cycles[2]; /* longest single work item, in warp clock cycles: [0] a root,
                                  [1] a task taken from another warp */
  double phase_ms[MCE_PHASES];
  uint64_t hist[MCE_HIST_LEN];
} mce_result;

typedef struct mce_graph_info {
  uint64_t num_vertices;
  uint64_t num_edges;
  uint32_t max_degree;
  uint32_t degeneracy;
  uint64_t device_bytes;      /* device memory held by the graph */
} mce_graph_info;

typedef struct mce_graph mce_graph;

void mce_default_options(mce_options *opt);
const char *mce_status_str(mce_status s);
/* Library version string. */
const char *mce_version(void);
/* Kernels the engine has launched in this process (for launch accounting). */
uint64_t mce_launch_count(void);
/* Measured throughput of the enumeration's word-op mix (64-bit ANDN + POPC),
 * in word-ops per second: the integer-pipe roof of the enumeration kernel. */
mce_status mce_probe_int_peak(int device, double *word_ops_per_s);

/* Allocation-free CSR row offsets.  No counterpart in the reference, which
 * builds offsets on the host (Graph::ConvertToCsr, src/graph.cc:216-236).
 * Both arrays are in device memory: rowoffset_device[i] = degree_device[0] +
 * ... + degree_device[i-1] for i = 0..n (n + 1 entries; the last one is the
 * total; sums are taken mod 2^32).  The engine's graph builders run the same
 * three-pass scan with a partial-sum buffer they allocate on every call; this
 * variant keeps the partial sums in a fixed 129 KiB array compiled into the
 * library and allocates nothing, on the device or the host.  It is meant for
 * callers that cannot allocate at the point of the call: a serving loop that
 * has handed all free HBM to resident graphs (cudaMalloc would fail), or code
 * whose caching allocator holds the device's whole pool, or any loop where an
 * allocation's implicit device synchronisation would stall other streams.
 *   - n > MCE_STATIC_SCAN_MAX_N (2^26 degrees) returns MCE_ERR_TOO_LARGE
 *     before anything is enqueued.
 *   - The first call on each device looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current and caches it; make
 *     that first call before any stream capture begins on the device.
 *   - Nothing has to be zeroed first: every partial sum is written before it
 *     is read, and all n + 1 offsets are written.
 *   - One array serves every caller on a device: calls that overlap in time
 *     on one device (from any stream or thread) race and corrupt each other's
 *     results.  Serialise them, e.g. by issuing them on one stream.
 *   - The work is enqueued on `stream` (a cudaStream_t, NULL = the legacy
 *     default stream); the call returns without waiting for it. */
#define MCE_STATIC_SCAN_MAX_N 67108864ull
mce_status mce_csr_offsets_static(int device, const uint32_t *degree_device, uint32_t *rowoffset_device,
                                  uint64_t n, void *stream);

/* COO pairs in host memory -> device-resident, degeneracy-ordered CSR.
 * Replaces Graph::LoadFromFile's edge handling + SortByOrder + ConvertToCsr +
 * GraphGpu::LoadFromCpu (src/graph.cc:64-152, 281-306, 216-236;
 * src/graph_gpu.cu:3-58); here sort, dedup, relabel and k-core peeling run on
 * the GPU. */
mce_status mce_graph_from_coo(const uint32_t *u, const uint32_t *v, uint64_t n_pairs,
                              const mce_options *opt, mce_graph **out);

/* Same, from COO pairs already in device memory (no host copy). */
mce_status mce_graph_from_coo_device(const uint32_t *u_device, const uint32_t *v_device, uint64_t n_pairs,
                                     const mce_options *opt, mce_graph **out);

/* A symmetric CSR with sorted rows (uint32 offsets, as Graph::ConvertToCsr
 * builds, src/graph.cc:216-236).  labels may be NULL (label = id).  If
 * already_ordered is nonzero the rows are used as given (as main.cc:26 does for
 * .bin input); otherwise the graph is reordered by `opt->order`. */
mce_status mce_graph_from_csr(uint64_t n, const uint32_t *rowoffset, const uint32_t *colidx,
                              const uint32_t *labels, int already_ordered, const mce_options *opt,
                              mce_graph **out);

/* COO text (Graph::LoadFromFile, src/graph.cc:64-152) or the reference .bin
 * container (Graph::LoadFromBin, src/graph.cc:178-213), chosen by the .bin
 * suffix exactly as main.cc:181-191 does.  Text is parsed on the GPU (the
 * file streamed to device memory, records found and converted there) and the
 * pairs go straight to the device graph build. */
mce_status mce_graph_load_file(const char *path, const mce_options *opt, mce_graph **out);

/* Write the reference .bin container (Graph::StoreIntoBin, src/graph.cc:154-176). */
mce_status mce_graph_store_bin(const mce_graph *g, const char *path);

mce_status mce_graph_info_get(const mce_graph *g, mce_graph_info *info);

/* Copy the device CSR (rowoffset n+1, colidx 2m) and labels (n) to host. */
mce_status mce_graph_export_csr(const mce_graph *g, uint32_t *rowoffset, uint32_t *colidx, uint32_t *labels);

void mce_graph_free(mce_graph *g);

/* Enumerate all maximal cliques.  Replaces MceGpuSolver::Solve /
 * BkSolverWrapper (src/mce_gpu.cu:14-22, src/kernels/BkPivotBitBalance.cuh:611-678),
 * which return only the count. */
mce_status mce_solve(mce_graph *g, const mce_options *opt, mce_result *out);

/* Per-root count and checksum for an explicit list of root ids (a root is an
 * undirected edge v0 < v1, numbered in CSR order).  For sampled-root parity. */
mce_status mce_solve_roots(mce_graph *g, const uint64_t *roots, uint64_t n_roots, const mce_options *opt,
                           uint64_t *counts, uint64_t *checksums);

/* Enumerate the maximal cliques rooted at an explicit set of roots (sampled
 * solves).  Totals only; root ids as in mce_solve_roots. */
mce_status mce_solve_root_list(mce_graph *g, const uint64_t *roots, uint64_t n_roots, const mce_options *opt,
                               mce_result *out);

/* One call: host COO -> result, everything on the device in between. */
mce_status mce_solve_coo(const uint32_t *u, const uint32_t *v, uint64_t n_pairs, const mce_options *opt,
                         mce_result *out);

/* ---- batched many-instance mode (no reference counterpart: the reference
 * solves one graph per process) ---- */
typedef struct mce_batch mce_batch;
typedef struct mce_batch_graph_result {
  uint64_t count;
  uint64_t checksum;
  uint32_t max_size;
  uint32_t num_vertices;
  uint64_t num_edges;
} mce_batch_graph_result;

/* Graph g's pairs are u[pair_offsets[g] .. pair_offsets[g+1]). */
mce_status mce_batch_create(const uint32_t *u, const uint32_t *v, const uint64_t *pair_offsets,
                            uint32_t n_graphs, const mce_options *opt, mce_batch **out);
/* hist may be NULL, else n_graphs * hist_len entries (sizes >= hist_len are
 * counted in the last bin). */
mce_status mce_batch_solve(mce_batch *b, const mce_options *opt, mce_batch_graph_result *results,
                           uint64_t *hist, uint32_t hist_len, double *enumerate_ms);
void mce_batch_free(mce_batch *b);

/* ---- serving loop (no reference counterpart) ---- */
typedef struct mce_server mce_server;
typedef struct mce_server_options {
  int device;
  uint64_t memory_budget;     /* bytes of device memory admissions may use; 0 = 60% of free */
  uint32_t max_inflight;      /* requests on the device at once, across the admitted batches; 0 = 256 */
  uint32_t reserved[5];
} mce_server_options;

mce_status mce_server_create(const mce_server_options *opt, mce_server **out);
/* Queue one request (pairs are copied).  Returns at once with its id. */
mce_status mce_server_submit(mce_server *s, const uint32_t *u, const uint32_t *v, uint64_t n_pairs,
                             uint64_t *request_id);
/* done=1 and *out filled when finished; done=0 while queued or running. */
mce_status mce_server_poll(mce_server *s, uint64_t request_id, int *done, mce_result *out,
                           double *latency_ms);
/* Device-clock span of a finished request's GPU work (upload, build, solve,
 * read-back), in milliseconds since the server was created.  Spans of
 * requests that overlap show they shared the device.  MCE_ERR_BUSY while the
 * request is queued or running. */
mce_status mce_server_request_span(mce_server *s, uint64_t request_id, double *device_start_ms,
                                   double *device_end_ms);
/* Block until every submitted request has finished. */
mce_status mce_server_drain(mce_server *s);
void mce_server_free(mce_server *s);

/* ---- synthetic generators (no reference counterpart; deterministic) ----
 * With u or v NULL the call only reports the pair count in *out_count. */
uint64_t mce_mix64(uint64_t x);
mce_status mce_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                        uint32_t *u, uint32_t *v, uint64_t capacity, uint64_t *out_count, int threads);
mce_status mce_gen_chung_lu(uint32_t n, double avg_degree, double gamma, uint64_t seed, uint32_t *u,
                            uint32_t *v, uint64_t capacity, uint64_t *out_count, int threads);
mce_status mce_gen_gnp(uint32_t n, double avg_degree, uint64_t seed, uint32_t *u, uint32_t *v,
                       uint64_t capacity, uint64_t *out_count);
mce_status mce_gen_planted(uint32_t n, uint32_t num_cliques, uint32_t size_lo, uint32_t size_hi,
                           uint64_t seed, uint32_t *u, uint32_t *v, uint64_t capacity, uint64_t *out_count);
mce_status mce_gen_batch_member(uint32_t index, uint64_t base_seed, uint32_t *u, uint32_t *v,
                                uint64_t capacity, uint64_t *out_count, uint32_t *out_n);

/* COO text parse with the reference's istream semantics (src/graph.cc:82-104).
 * Buffers are malloc'ed; release them with mce_free_host. */
mce_status mce_parse_text(const char *path, uint32_t **u, uint32_t **v, uint64_t *n_pairs);
/* The same parse on the GPU of `device` (the one mce_graph_load_file uses for
 * text), results copied back into malloc'ed host buffers (mce_free_host).
 * Replaces the text loop of Graph::LoadFromFile (src/graph.cc:82-104). */
mce_status mce_parse_text_gpu(const char *path, int device, uint32_t **u, uint32_t **v, uint64_t *n_pairs);
void mce_free_host(void *p);

#ifdef __cplusplus
}
#endif
#endif /* RDMCE_H */
