/*
 * sparx_pkt.h — C ABI of the B200 PKT k-truss engine (libsparx_pkt.so).
 *
 * Drop-in for the PKT path of alexfaisca/sparkx.  The reference computes an
 * edge's truss number with `AlgoPKT` (src/k_truss/pkt.rs) over a
 * memory-mapped CSR `GraphMemoryMap` (src/graph/mod.rs:365-378) whose
 * offsets are u64[n+1] and whose neighbour ids are u64[width]
 * (graph/mod.rs:482-489).  The result is one truss number per CSR slot, u8,
 * in slot order (pkt.rs:33,104-114,524-526).  The entry points below take
 * exactly those arrays and fill that result; every call returns a status
 * code (0 = SPARX_OK), never aborts, and never falls back to the CPU.
 *
 * Input contract (as produced by the reference's cache builders): rows
 * sorted ascending, both directions of every edge present, ids < n.
 * Self-loop slots are accepted and get truss 2 (triangles.rs:194-195,
 * impl_csc.rs:148-153).  Parallel edges (equal ids side by side in a row, the
 * reference's OneOrMany paths: impl_csc.rs:154-215, triangles.rs:172-224,
 * pkt.rs:373-395) are accepted: a triangle is one choice of a copy of each of
 * its three pairs, every copy of a pair gets the pair's truss number, and a
 * pair must appear the same number of times in both of its rows
 * (SPARX_E_INVALID_CSR otherwise).  Only the allocation-free entry point
 * rejects parallel edges (SPARX_E_MULTIGRAPH).
 */
#ifndef SPARX_PKT_H
#define SPARX_PKT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define SPARX_OK              0
#define SPARX_E_INVALID_CSR   1  /* unsorted row, asymmetric, id >= n, bad offsets */
#define SPARX_E_MULTIGRAPH    2  /* parallel edges given to the allocation-free entry point */
#define SPARX_E_OVERFLOW_U8   3  /* truss > 255 with 8-bit output (pkt.rs:508-516) */
#define SPARX_E_OOM           4  /* device memory or HBM budget exhausted */
#define SPARX_E_TIMEOUT       5  /* device-side peel exceeded its time budget */
#define SPARX_E_CUDA          6  /* CUDA runtime error (see sparx_last_error) */
#define SPARX_E_TOO_LARGE     7  /* width >= 2^32, m >= 2^28 per graph, > 65535 copies of a pair,
                                    or a multigraph support >= 2^31 */
#define SPARX_E_ARG           8  /* bad argument */
#define SPARX_E_NOT_FOUND     9  /* unknown ticket */
#define SPARX_E_CANCELLED    10  /* request cancelled before completion */
#define SPARX_E_PARSE        11  /* malformed MatrixMarket text (see sparx_last_error) */

/* ---- options ---------------------------------------------------------- */
#define SPARX_SUPPORT_WIDE 0u  /* u32 triangle counters: the defined truss */
#define SPARX_SUPPORT_U8   1u  /* the reference's AtomicU8 counters (support mod 256) */

#define SPARX_LOOP_GRAPH 0u    /* level loop on the device: CUDA graph WHILE node */
#define SPARX_LOOP_HOST  1u    /* host re-launches batches of waves (debugging) */

typedef struct sparx_pkt_opts {
  uint32_t struct_size;    /* sizeof(sparx_pkt_opts) */
  uint32_t support_mode;   /* SPARX_SUPPORT_WIDE | SPARX_SUPPORT_U8 */
  uint32_t out_bits;       /* 8 (reference layout) or 32 */
  int32_t device;          /* CUDA ordinal; -1 = current device */
  uint32_t loop;           /* SPARX_LOOP_GRAPH | SPARX_LOOP_HOST */
  uint32_t support_kernel; /* 0 = auto, 1 = balanced binary search, 2 = vertex hash */
  uint64_t timeout_ms;     /* device budget for the peel; 0 = 600000 */
} sparx_pkt_opts;

typedef struct sparx_pkt_stats {
  uint64_t n, width, m, self_loops;  /* m: distinct pairs; self_loops: self-loop slots (not split
                                        per member for a batched multigraph: 0 there) */
  uint64_t triangles;      /* sum of support / 3 (wide counters); a multigraph counts each
                              choice of copies of the three pairs */
  uint64_t max_support;    /* before the peel, after the u8 wrap in u8 mode */
  uint32_t k_max;          /* largest truss number */
  uint32_t levels;         /* non-empty peel levels */
  uint32_t waves;          /* device peel waves (sub-levels + level scans) */
  uint32_t launches;       /* kernels this call launched (graph-internal ones included) */
  double ms_upload, ms_orient, ms_support, ms_peel, ms_finalize, ms_download, ms_total;
  /* work counters behind the roofline figures */
  uint64_t support_elements;  /* shorter-out-list entries searched by the support kernel */
  uint64_t peel_elements;     /* shorter-row entries searched by the peel (all waves) */
  uint64_t peel_hits;         /* triangles found by the peel (processed or skipped) */
  uint64_t peel_scanned;      /* active-list entries read by level scans */
  uint64_t peel_edges;        /* frontier edges processed (= m minus zero-support edges) */
  uint32_t compactions;       /* rebuilds of the peel's working rows */
  uint32_t hub_maps;          /* dense neighbour -> edge maps built for the highest-degree vertices */
  uint64_t merge_iters;       /* peel warp iterations resolved by a row merge */
  uint64_t lane_iters;        /* peel warp iterations resolved by per-lane searches */
  uint64_t merge_chunks;      /* 32-entry chunks of longer rows read by the merges */
} sparx_pkt_stats;

/* Fill `opts` with defaults (wide support, u8 output, device loop). */
int sparx_pkt_default_opts(sparx_pkt_opts* opts);

/* Human-readable status text. */
const char* sparx_strerror(int status);

/* Detail of the last failing call on this thread (CUDA error text etc.). */
const char* sparx_last_error(void);

/*
 * Full PKT decomposition of one graph from HOST memory in the reference's
 * layout.  Replaces AlgoPKT::new / new_with_conf (pkt.rs:45-52,85-95), whose
 * work is compute_with_proc_mem_impl (pkt.rs:216-563).
 *   offsets    u64[n_plus_1]  (graph/mod.rs:482-485, offsets_ptr)
 *   neighbours u64[width]     (graph/mod.rs:487-489, neighbours_ptr)
 *   truss_out  u8[width] (out_bits 8) or u32[width] (out_bits 32), caller-owned
 */
int sparx_pkt_run(const uint64_t* offsets, uint64_t n_plus_1, const uint64_t* neighbours,
                  uint64_t width, void* truss_out, const sparx_pkt_opts* opts,
                  sparx_pkt_stats* stats);

/* Same, with u32 neighbour ids in host memory. */
int sparx_pkt_run_u32(const uint64_t* offsets, uint64_t n_plus_1, const uint32_t* neighbours,
                      uint64_t width, void* truss_out, const sparx_pkt_opts* opts,
                      sparx_pkt_stats* stats);

/*
 * Same, with every array already in DEVICE memory of opts->device; runs on
 * `cuda_stream` (a cudaStream_t, or NULL for the library's own stream) and
 * returns after the stream has finished the result.
 */
int sparx_pkt_run_device(const uint64_t* d_offsets, uint64_t n_plus_1,
                         const uint32_t* d_neighbours, uint64_t width, void* d_truss_out,
                         const sparx_pkt_opts* opts, sparx_pkt_stats* stats, void* cuda_stream);

/*
 * Triangle support per CSR slot, host memory in / out.  Replaces
 * Triangles::new (triangles.rs:27-32), i.e. compute_with_proc_mem_impl
 * (triangles.rs:144-243).  support_out is u32[width]; in SPARX_SUPPORT_U8 mode
 * the values are reduced mod 256 like the reference's AtomicU8 counters.
 */
int sparx_triangles_run(const uint64_t* offsets, uint64_t n_plus_1, const uint64_t* neighbours,
                        uint64_t width, uint32_t* support_out, const sparx_pkt_opts* opts,
                        sparx_pkt_stats* stats);

/*
 * k-core decomposition: the core number of every vertex.  Replaces
 * AlgoLiuEtAl::new / compute_with_proc_mem (k_core/liu_et_al.rs:45-62,190-420)
 * with its semantics: a vertex's degree is its row length (self-loop slots
 * included), isolated vertices get core 0, and peeling at level k (k >= 1)
 * removes every live vertex of degree <= k.  In SPARX_SUPPORT_U8 mode the
 * degrees are reduced mod 256 like the reference's AtomicU8 counters.
 * core_out is u8[n] (opts->out_bits == 8, the reference layout;
 * SPARX_E_OVERFLOW_U8 if a core exceeds 255) or u32[n].  stats: levels,
 * waves (sub-levels) and k_max (largest core) are filled.
 */
int sparx_kcore_run(const uint64_t* offsets, uint64_t n_plus_1, const uint64_t* neighbours,
                    uint64_t width, void* core_out, const sparx_pkt_opts* opts,
                    sparx_pkt_stats* stats);

/*
 * Local clustering coefficient of every vertex, graph transitivity and the
 * average local coefficient, from the triangle supports.  Replaces
 * ClusteringCoefficient::new / compute (clustering_coefficient.rs:41-52,93-190)
 * with its definitions: for vertex u with d distinct neighbours (a self-loop
 * counts as one), local[u] = ceil(sum of u's slot supports / 2) / (d(d-1)/2),
 * or 0 when d < 2; *transitivity = (sum of all slot supports / 3) / 2 /
 * (sum of d(d-1)/2); *average = sum of local / n.  In SPARX_SUPPORT_U8 mode the
 * slot supports are reduced mod 256 like the reference's AtomicU8 counts.  The
 * reference divides by 3 per worker thread; this is its one-thread value.
 * These are the INTENDED coefficients: the reference's compute() zeroes the
 * support counters before reading them (clustering_coefficient.rs:130-135),
 * so it returns 0 for every coefficient; this call does not reproduce that.
 * local_out is f64[n]; transitivity and average may be NULL.
 */
int sparx_clustering_run(const uint64_t* offsets, uint64_t n_plus_1, const uint64_t* neighbours,
                         uint64_t width, double* local_out, double* transitivity, double* average,
                         const sparx_pkt_opts* opts, sparx_pkt_stats* stats);

/*
 * Allocation-free PKT decomposition of one graph in DEVICE memory.  No
 * counterpart in the reference.
 *
 * For callers that must not allocate device memory when they ask for a
 * decomposition: services whose device memory is reserved up front by their
 * own pool (an allocation outside it is a fault for them), and
 * latency-critical request paths that cannot wait for or fail on cudaMalloc.
 * All scratch lives in one fixed file-scope device array of
 * SPARX_NOALLOC_SCRATCH_BYTES per device (present on every GPU that loads the
 * library, until exit); graphs needing more get SPARX_E_TOO_LARGE (roughly
 * 1.4 M CSR slots).  The call allocates no device or pinned memory, streams or
 * events.  Parallel edges return SPARX_E_MULTIGRAPH (their deduplicated rows
 * would need more scratch; sparx_pkt_run_device takes them).
 *
 * Each call looks up the array's device address on the current device
 * (cudaGetSymbolAddress); the first call on a device also loads the library's
 * device code there, so make that first call before any stream capture begins.
 * The call is host-synchronous: it reads small results back and waits for
 * `cuda_stream` several times and returns once the stream has finished the
 * result, so `cuda_stream` must not be a stream that is being captured.  All
 * calls on a device share the array and it keeps the previous call's
 * contents (each call clears what must start at zero): calls that overlap on
 * the GPU (other streams, other host threads) race and corrupt each other;
 * serialize them.  A call that fails after its first launch waits for the
 * stream before it returns, so the array is idle again.
 *   d_offsets u64[n_plus_1], d_neighbours u32[width], d_truss_out u32[width]
 *   device: CUDA ordinal (-1 = current)
 */
#define SPARX_NOALLOC_SCRATCH_BYTES (64ull << 20)
int sparx_pkt_run_device_noalloc(const uint64_t* d_offsets, uint64_t n_plus_1,
                                 const uint32_t* d_neighbours, uint64_t width, uint32_t* d_truss_out,
                                 int device, void* cuda_stream);

/* ---- input ------------------------------------------------------------- */
/*
 * MatrixMarket text -> CSR in the reference's layout, on the GPU.  Replaces
 * GraphCache::from_mtx_file (graph/cache/parser_mtx/mod.rs:34-162) with its
 * semantics: header "%%MatrixMarket matrix coordinate pattern|integer
 * symmetric|skew-symmetric|general" (case-insensitive), '%' and blank lines
 * skipped, size line "nrows ncols nnz" with nrows == ncols; every entry line
 * with at least two tokens i j (1-based; a third, the integer value, is
 * ignored) adds slot j-1 to row i-1 and, unless the header says general and
 * when i != j, slot i-1 to row j-1 (parser_mtx/producers.rs:139-240);
 * duplicates stay (parallel edges); rows are sorted ascending
 * (impl_sort.rs:10-51).  Every entry line of the text is read, whatever nnz
 * the size line declares.  An index of 0, beyond nrows or not an unsigned
 * integer returns SPARX_E_PARSE (sparx_last_error names the line).
 *   text, len          the file's bytes (host memory)
 *   offsets_out        u64[n+1], neighbours_out u64[width] (host), or NULL:
 *                      then only *n_out and *width_out are set, so a caller
 *                      can size its buffers and call again
 */
int sparx_mtx_to_csr(const char* text, uint64_t len, uint64_t* offsets_out, uint64_t offsets_cap,
                     uint64_t* neighbours_out, uint64_t neighbours_cap, uint64_t* n_out, uint64_t* width_out,
                     const sparx_pkt_opts* opts);

/* ---- tuning ------------------------------------------------------------ */
/*
 * Performance knobs of the engine (no counterpart in the reference, whose
 * only knob is its thread count).  None changes a result.  Each launch
 * picks them from a cache keyed on the degree signature of the rows it runs
 * on: key = {floor(log2(slots)), floor(log2(max degree)) + 1, eighths of the
 * slots that lie in rows of degree >= 256}; a key without an entry uses the
 * defaults below.  sparx_autotune fills the cache by measuring candidates on a
 * sample graph; the file named by the environment variable SPARX_TUNE_FILE is
 * read on first use and rewritten by each autotune.  An explicit
 * opts->support_kernel (1 or 2) overrides the tuned support form.
 */
typedef struct sparx_tuning {
  uint32_t struct_size;     /* sizeof(sparx_tuning) */
  uint32_t merge_ratio;     /* peel: merge the two rows when the longer is <= this x the shorter (8) */
  uint32_t hub_min_degree;  /* dense neighbour -> edge maps for vertices of at least this degree,
                               >= 256, or 0 for none (1024) */
  uint32_t sample_min;      /* support: longer out-lists of at least this length are narrowed
                               through 64 samples before the search (64) */
  uint32_t support_kernel;  /* 1 balanced edge form, 2 vertex form (1; 2 for keys with no
                               slots in rows of degree >= 256 and a largest degree of 64..255,
                               which is what sparx_tuning_lookup reports for such a key) */
  uint32_t compact_pct;     /* peel: rebuild the working rows once live entries fill at most
                               this percentage of them (85) */
  uint32_t hash_min_degree; /* peel: rows of at least this degree (>= 8) get a hash table that the
                               per-lane search probes instead of a binary search; 0 = none (128).
                               Skipped, with the same results, when its workspace (32 B per slot
                               plus 16 B per edge) is over a batch's budget or cannot be allocated */
  uint32_t sup_hash_min;    /* support: oriented out-lists of at least this length (>= 4) get a hash
                               table probed instead of the sampled search; 0 = none (0) */
  uint32_t relabel;         /* graphs and batched unions without parallel edges: rebuild the CSR on vertex ids
                               in (floor(log2 degree), id) order (a union's members each within their own
                               id range) before the decomposition, for locality;
                               results are returned in the caller's slot order (0; 1 for keys of
                               2^26 slots or more with a quarter of them in rows of degree >= 256) */
} sparx_tuning;

int sparx_tuning_default(sparx_tuning* t);
/* The key of a host CSR (its offsets only). */
int sparx_tuning_signature(const uint64_t* offsets, uint64_t n_plus_1, uint32_t key[3]);
/* Cached knobs for a key (*found = 0: the defaults are returned). */
int sparx_tuning_lookup(const uint32_t key[3], sparx_tuning* out, int* found);
int sparx_tuning_store(const uint32_t key[3], const sparx_tuning* t);
int sparx_tuning_clear(void);
/* Knobs and key of the last launch on this thread. */
int sparx_tuning_last(sparx_tuning* used, uint32_t key[3]);
int sparx_tuning_save(const char* path);
int sparx_tuning_load(const char* path);

/*
 * Autotune on one sample graph (host, the reference's layout): coordinate
 * descent from the defaults over the support form and sampling threshold
 * (timed by the support pass), then the hub floor, merge ratio and compaction
 * fill and row hash floor (timed by orientation + peel); `repeats` decompositions per candidate
 * (median).  Stores the winner under the sample's key and returns it.
 */
int sparx_autotune(const uint64_t* offsets, uint64_t n_plus_1, const uint64_t* neighbours, uint64_t width,
                   const sparx_pkt_opts* opts, uint32_t repeats, sparx_tuning* best, uint32_t key[3]);

/* ---- batched decomposition -------------------------------------------- */
/* One member of a batch: host arrays in the reference's layout (u64 ids) or
 * u32 ids (neighbour_bits 32).  truss_out follows opts->out_bits. */
typedef struct sparx_graph_view {
  const uint64_t* offsets;
  uint64_t n_plus_1;
  const void* neighbours;
  uint64_t width;
  uint32_t neighbour_bits; /* 64 or 32 */
  uint32_t reserved;
  void* truss_out;
} sparx_graph_view;

/*
 * Decompose `count` independent graphs.  Graphs are packed into waves under
 * `hbm_budget_bytes` (0 = 150 GB); each wave is one concatenated CSR whose
 * peel advances every member with one launch per device wave.  Per-graph
 * status goes to status_out[count] (may be NULL), per-graph stats to
 * stats_out[count] (may be NULL); the return value is the first failure.
 */
int sparx_pkt_run_batch(const sparx_graph_view* graphs, uint64_t count, uint64_t hbm_budget_bytes,
                        const sparx_pkt_opts* opts, int* status_out, sparx_pkt_stats* stats_out);

/*
 * Autotune a batch: the candidates run over the whole batch and are timed on
 * its first union (whose key receives the winner); pass a representative
 * sample that fits one union under the budget.  Results are written to the
 * members' truss_out (every candidate gives the same numbers).
 */
int sparx_autotune_batch(const sparx_graph_view* graphs, uint64_t count, uint64_t hbm_budget_bytes,
                         const sparx_pkt_opts* opts, uint32_t repeats, sparx_tuning* best, uint32_t key[3]);

/* ---- serving: continuous batching ------------------------------------ */
typedef struct sparx_server sparx_server;

/* Create a server on opts->device with an HBM budget (0 = 150 GB, capped at the
 * device's free memory).  Requests run on 4 execution lanes (the environment
 * variable SPARX_SERVE_LANES, 1..16, changes the count), each on its own
 * stream: lane 0 holds half the budget (a large graph fits there), the others
 * share the rest, and each keeps a fifth of its share to prepare requests that
 * join it.  An idle lane packs the queued requests that fit into a union sized
 * to its share; while that union's peel runs, a submitted request stops it at
 * its next wave, and the requests that fit join the union there (prepared on
 * the lane's second engine and placed behind the running members).  A union
 * takes no joins while it holds a graph of more than 2^26 slots or while its
 * waves average more than 60 us (newcomers then wait for a lane), and a union
 * without join room gets the row hash tables.  Every member's result goes back
 * as soon as its own peel ends.  A request needing
 * more than any lane holds completes with SPARX_E_OOM.  Requests stay
 * addressable by ticket until sparx_server_destroy. */
int sparx_server_create(sparx_server** out, uint64_t hbm_budget_bytes, const sparx_pkt_opts* opts);

/* Queue a decomposition; the arrays must stay valid until sparx_server_poll
 * reports it done.  *ticket identifies the request. */
int sparx_server_submit(sparx_server* s, const sparx_graph_view* graph, uint64_t* ticket);

/* Non-blocking: *done = 1 once finished; *status is that request's status. */
int sparx_server_poll(sparx_server* s, uint64_t ticket, int* done, int* status,
                      sparx_pkt_stats* stats);

/* Block until the request finishes (timeout_ms 0 = forever). */
int sparx_server_wait(sparx_server* s, uint64_t ticket, uint64_t timeout_ms, int* status,
                      sparx_pkt_stats* stats);

/* Cancel a queued (not yet admitted) request. */
int sparx_server_cancel(sparx_server* s, uint64_t ticket);

/* Served unions started, and requests that joined a union already running. */
int sparx_server_info(sparx_server* s, uint64_t* unions, uint64_t* joined);

/* Drain and free. */
int sparx_server_destroy(sparx_server* s);

#ifdef __cplusplus
}
#endif

#endif /* SPARX_PKT_H */
