/*
 * nwg_bfs.h -- C ABI of the B200 direction-optimizing BFS library
 * (libnwgr_b200.so).  Plain pointers and sizes only; every function returns
 * an int status (0 = NWG_OK, negative = error, message via nwg_last_error).
 * No exception crosses this boundary.
 *
 * Each entry point names the NWGraph interface it replaces (paths relative
 * to the NWGraph source tree).  NWGraph is header-only C++; its BFS has no
 * ABI of its own, so these functions are what a C++ wrapper (the drop-in
 * header include/nwgraph/algorithms/bfs.hpp of this repository) or a foreign
 * function interface binds to.
 *
 * Graphs are CSR: offsets (n+1 entries, uint64 or uint32) and uint32 column
 * indices, rows in any order (the bottom-up step takes the first in-neighbour
 * in row order, as the reference does).  The in-graph must be the transpose
 * of the out-graph (the reference's contract for bfs(out, in, ...)); pass
 * NULL in-pointers when the graph is symmetric and out == in.
 */
#ifndef NWG_BFS_H
#define NWG_BFS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define NWG_OK 0
#define NWG_EINVAL (-1)     /* bad argument: root >= n, alpha/beta <= 0, malformed CSR */
#define NWG_ENOMEM (-2)     /* device or pinned allocation failed */
#define NWG_ECUDA (-3)      /* CUDA runtime error */
#define NWG_ETIMEDOUT (-4)  /* a bounded device loop or wait ran out */
#define NWG_EOVERFLOW (-5)  /* a result does not fit its encoding (e.g. uint8 depth) */
#define NWG_ESTATE (-6)     /* call out of order (e.g. stats before a traversal) */

#define NWG_NULL_VERTEX 0xFFFFFFFFu /* null_vertex_v<uint32_t>(), util/util.hpp:125-132 */

/* nwg_graph_register flags */
#define NWG_REG_DEVICE 0x1u   /* arrays are device pointers, borrowed (not copied); caller keeps them alive */
#define NWG_REG_VALIDATE 0x2u /* check monotone offsets and column ids < n before upload (host arrays) */

typedef struct nwg_graph_s* nwg_graph;   /* a CSR pair resident in HBM */
typedef struct nwg_bfs_ws_s* nwg_bfs_ws; /* per-traversal device state; one traversal in flight per workspace */

#define NWG_TRACE_CAP 256

/* Per-traversal statistics, read back once after the traversal. */
typedef struct {
  int32_t status;      /* device-side status of the traversal (0 = ok) */
  uint32_t steps;      /* actions run by the level loop (top-down steps + bottom-up pulls + conversions) */
  uint32_t levels;     /* BFS levels = maximum depth + 1 */
  uint32_t td_steps;   /* top-down steps */
  uint32_t bu_steps;   /* bottom-up pulls */
  uint32_t b2q_steps;  /* bitmap-to-queue conversions */
  uint64_t reached;    /* vertices with a parent, root included */
  float device_ms;     /* device time of the traversal (CUDA events), 0 for the async API */
  uint32_t trace_len;  /* records in the trace below (<= NWG_TRACE_CAP) */
  /* one record per top-down step (dir 0) and bottom-up pull (dir 1), in order;
   * frontier = queue size entering a top-down step, or the previous awake
   * count entering a pull (bfs.hpp:205-209); found = vertices discovered */
  uint8_t trace_dir[NWG_TRACE_CAP];
  uint64_t trace_frontier[NWG_TRACE_CAP];
  uint64_t trace_found[NWG_TRACE_CAP];
  /* device clock (%globaltimer, ns since the traversal's init kernel) when
   * the level loop consumed each step's result; first_decide_ns is the first
   * decision.  Step i took trace_end_ns[i] - trace_end_ns[i-1] (i = 0:
   * minus first_decide_ns), launch gaps included. */
  uint64_t trace_end_ns[NWG_TRACE_CAP];
  uint64_t first_decide_ns;
  /* kernels the traversal launched (init, one decision per loop iteration,
   * one action per iteration but the last; a persistent small-frontier
   * action covers several steps in one launch) */
  uint32_t kernel_launches;
} nwg_bfs_stats;

/* Library version string. */
const char* nwg_version(void);

/* Copies the calling thread's last error message into buf (NUL-terminated).
 * Returns the message length. */
int nwg_last_error(char* buf, size_t len);

/* Registers a CSR pair on the current CUDA device.  Replaces the CSR access
 * that nw::graph::bfs performs on its arguments: out_graph.indices_ /
 * std::get<0>(out_graph.to_be_indexed_) (containers/compressed.hpp:67-68,
 * algorithms/bfs.hpp:168) and in_graph[u] (bfs.hpp:216).  Host arrays are
 * uploaded once (the only bulk host-to-device copy); with NWG_REG_DEVICE
 * they are borrowed in place.  in_off/in_col NULL = symmetric graph.
 * NWG_REG_VALIDATE (host arrays) checks monotone offsets, column ids < n
 * and, for a directed pair, that the in-CSR is the transpose of the
 * out-CSR; without it the caller guarantees all three. */
int nwg_graph_register(const uint64_t* out_off, const uint32_t* out_col, uint64_t n, const uint64_t* in_off,
                       const uint32_t* in_col, uint32_t flags, nwg_graph* out);

/* Same for NWGraph's default adjacency<0> layout, uint32 offsets
 * (util/defaults.hpp:23-24); offsets are widened to uint64 on the device. */
int nwg_graph_register_u32off(const uint32_t* out_off, const uint32_t* out_col, uint64_t n, const uint32_t* in_off,
                              const uint32_t* in_col, uint32_t flags, nwg_graph* out);

/* Frees the device copy (and every workspace created on it). */
int nwg_graph_release(nwg_graph g);

/* n, m (out-graph entries) and in_m of a registered graph; any may be NULL. */
int nwg_graph_info(nwg_graph g, uint64_t* n, uint64_t* m, uint64_t* in_m);

/* Direction-optimizing BFS from root; replaces nw::graph::bfs(out_graph,
 * in_graph, root, num_bins, alpha, beta) (algorithms/bfs.hpp:160-311).
 * num_bins has no GPU meaning (the device bins by degree) and is not taken.
 * parents_host: host array of n entries (pageable or pinned) or NULL;
 * parents_dev: device array of n entries or NULL; stats: NULL or filled.
 * Unreached vertices get NWG_NULL_VERTEX, the root gets itself.
 * Synchronous; thread-safe per graph (calls on one graph serialise). */
int nwg_bfs(nwg_graph g, uint32_t root, int alpha, int beta, uint32_t* parents_host, uint32_t* parents_dev,
            nwg_bfs_stats* stats);

/* nwg_bfs over k roots with each root's parents copied to host row i of
 * parents_host (k * n entries, row i = roots[i]); replaces the per-source
 * loop of NWGraph's BFS benchmark (bench/bfs.cpp:106-141), which calls
 * bfs(graph, gx, source, num_bins, alpha, beta) once per source.  Two
 * traversals are in flight: root i + 1 runs on the device while root i's
 * parents cross to the host, so with pinned host memory a call costs about
 * k copies of n * 4 bytes rather than k copies plus k traversals (pageable
 * memory works but the copies then serialise with the traversals).
 * status: NULL or k entries, each root's NWG status.  All roots are checked
 * before anything runs (NWG_EINVAL names the first bad one); otherwise every
 * root runs and the first failing root's status is returned.  Synchronous;
 * calls on one graph serialise with each other and with nwg_bfs. */
int nwg_bfs_roots(nwg_graph g, const uint32_t* roots, uint64_t k, int alpha, int beta, uint32_t* parents_host,
                  int32_t* status);

/* Workspaces for concurrent, stream-ordered traversals of one graph. */
int nwg_ws_create(nwg_graph g, nwg_bfs_ws* out);
int nwg_ws_destroy(nwg_bfs_ws ws);

/* Stream-ordered variant of nwg_bfs: enqueues the whole traversal (one CUDA
 * cooperative kernel launch, no host synchronisation) on `stream` (a cudaStream_t, NULL =
 * legacy default stream) writing parents to the device array parents_dev.
 * At most one traversal per workspace may be in flight. */
int nwg_bfs_async(nwg_bfs_ws ws, uint32_t root, int alpha, int beta, uint32_t* parents_dev, void* stream);

/* Statistics of the workspace's last traversal; synchronises with it. */
int nwg_ws_stats(nwg_bfs_ws ws, nwg_bfs_stats* stats);

/* nwg_bfs with the level loop driven from the host: the same kernels
 * launched one at a time, the decision read back after every step.  For
 * profilers (ncu cannot profile the kernels of a CUDA graph with
 * conditional nodes one by one) and debugging; slower than nwg_bfs. */
int nwg_bfs_stepped(nwg_graph g, uint32_t root, int alpha, int beta, uint32_t* parents_dev, nwg_bfs_stats* stats);

/* Top-down-only BFS (no in-graph needed); replaces the one-graph
 * nw::graph::bfs(graph, root) (algorithms/bfs.hpp:110-140). */
int nwg_bfs_topdown(nwg_graph g, uint32_t root, uint32_t* parents_host, uint32_t* parents_dev, nwg_bfs_stats* stats);

/* Failure-detection self-test (no reference counterpart).  Runs the
 * persistent small-frontier kernel's grid barrier on a grid that never
 * completes it (a wait for one block more than the grid has): every block
 * gives up after `spins` polls (1..2^24; each poll sleeps about 32 ns plus an
 * L2 round trip) and reports NWG_ETIMEDOUT, the status a traversal returns
 * when a block never arrives.  status receives that device-side status,
 * waited_ms the device time.  No fault, trap or unbounded wait is involved;
 * the context stays usable. */
int nwg_selftest_wait_timeout(uint32_t spins, int32_t* status, float* waited_ms);

/* Sum of out-degrees and count of the vertices reached in a device parents
 * array (the TEPS numerator of a traversal); both outputs may be NULL. */
int nwg_component_edges(nwg_graph g, const uint32_t* parents_dev, uint64_t* edges, uint64_t* vertices);

/* Copies a registered graph's out-CSR (and in-CSR when not symmetric) to
 * host arrays of the sizes nwg_graph_info reports; any pointer may be NULL. */
int nwg_graph_copy_csr(nwg_graph g, uint64_t* out_off, uint32_t* out_col, uint64_t* in_off, uint32_t* in_col);

/* Batched multi-source BFS (no reference counterpart: NWGraph's bfs is
 * single-source; the result equals one single-source BFS per root).  Sources
 * are packed 64 per 64-bit word, up to 256 per pass; each level pushes
 * (top-down, 64-bit atomicOr) or pulls (bottom-up, no atomics) by the rule
 * of nw::graph::bfs: pull when the frontier's out-edges exceed the
 * unexplored edges / alpha (4 suits it better than the single-source 15: a
 * multi-source pull rarely stops early).  depths_dev is a device array [k][n] of
 * uint8: depth of vertex v from root i at depths_dev[i * n + v], 255 =
 * unreached.  A source whose depths reach 255 (a graph whose diameter passes
 * 254) does not spoil the others: every other row is exact, that source's
 * row holds its depths up to 254 (255 beyond), and the call returns
 * NWG_EOVERFLOW (stats->deep_sources counts such sources; nwg_msbfs_ex
 * flags them one by one and answers them exactly in uint16).  Calls of more
 * than 256 sources keep up to four passes in flight, each on its own copy of
 * the pass state and its own stream (the extra copies are made on the first
 * such call and kept with the workspace).  Runs on `stream`
 * (NULL = the workspace's own stream) and returns when done.  A workspace
 * The passes rely on the in-CSR being the exact transpose of the out-CSR
 * (see nwg_graph_register): a pull reads the frontier words of in-
 * neighbours, and a sparse push level leaves the frontier word of a vertex
 * without out-edges unrefreshed, which a true transpose never lists as an
 * in-neighbour.  A workspace holds about 388 * n bytes of device state (three bitsets and eight level
 * bit-planes of four 64-bit words per vertex, a touched-vertex list and its
 * bitmap) plus two frontier lists of 8 * (n + m / 256 + 1) bytes: about
 * 1.7 GB for RMAT-22, 6.8 GB for RMAT-24.
 * Calls on one workspace must not overlap. */
typedef struct nwg_msbfs_ws_s* nwg_msbfs_ws;
#define NWG_MS_TRACE_CAP 64
typedef struct {
  int32_t status;
  uint32_t passes;      /* passes of up to 256 sources */
  uint32_t levels;      /* maximum depth + 1 over all sources */
  uint32_t push_levels; /* levels run top-down, summed over passes */
  uint32_t pull_levels; /* levels run bottom-up, summed over passes */
  float device_ms;      /* device time (CUDA events) */
  /* the first pass's levels: direction (0 push, 1 pull), device time,
   * out-edges of the level's frontier, (source, vertex) pairs discovered */
  uint32_t trace_len;
  uint8_t trace_pull[NWG_MS_TRACE_CAP];
  float trace_ms[NWG_MS_TRACE_CAP];
  uint64_t trace_frontier_edges[NWG_MS_TRACE_CAP];
  uint64_t trace_discovered[NWG_MS_TRACE_CAP];
  uint32_t deep_sources; /* sources whose depths reach 255 or more */
} nwg_msbfs_stats;
int nwg_msbfs_ws_create(nwg_graph g, nwg_msbfs_ws* out);
int nwg_msbfs_ws_destroy(nwg_msbfs_ws ws);
int nwg_msbfs(nwg_msbfs_ws ws, const uint32_t* roots_host, uint32_t k, uint8_t* depths_dev, int alpha, void* stream,
              nwg_msbfs_stats* stats);
/* nwg_msbfs with the row width chosen and deep sources reported per source
 * (no reference counterpart either).  depth_bytes = 1: uint8 rows as
 * nwg_msbfs writes them, but a deep source is not an error: the call returns
 * NWG_OK and deep_flags_host[i] = 1 marks each row i that stops at 254.
 * depth_bytes = 2: rows of uint16 (depths_dev[i * n + v], 0xFFFF =
 * unreached), all exact: a deep source's row comes from one single-source
 * traversal (nw::graph::bfs semantics, bfs.hpp:160-311) and its parents'
 * depths, on a workspace made and freed for the call; NWG_EOVERFLOW only if
 * a depth reaches 65535.  deep_flags_host (k bytes) may be NULL. */
int nwg_msbfs_ex(nwg_msbfs_ws ws, const uint32_t* roots_host, uint32_t k, void* depths_dev, uint32_t depth_bytes,
                 uint8_t* deep_flags_host, int alpha, void* stream, nwg_msbfs_stats* stats);

/* Ragged batch: many small graphs packed in HBM once, and a table of
 * (graph, root) traversals run in ONE persistent launch (replayed as a CUDA
 * graph).  Each block of the launch takes items from a device work counter
 * and runs an item's whole direction-optimizing level loop by itself, with
 * the item's own alpha, beta and degree threshold (warp_min, 32..256; 0 =
 * 32) -- the values the autotuner picks per graph-shape class.  No reference
 * counterpart beyond one nw::graph::bfs call per item; results are the same.
 * Registration: graph g has graph_n[g] vertices; off_concat holds each
 * graph's n + 1 offsets (starting at 0) one graph after the other, col_concat
 * each graph's columns one after the other; all host arrays, validated. */
typedef struct nwg_ragged_s* nwg_ragged;
typedef struct {
  uint32_t graph;
  uint32_t root;
  int32_t alpha;
  int32_t beta;
  uint32_t warp_min;
} nwg_ragged_item;
typedef struct {
  int32_t status;
  uint32_t steps, levels, td_steps, bu_steps, b2q_steps;
  uint64_t reached;
} nwg_ragged_result;
int nwg_ragged_register(uint32_t num_graphs, const uint64_t* graph_n, const uint64_t* off_concat,
                        const uint32_t* col_concat, nwg_ragged* out);
int nwg_ragged_release(nwg_ragged r);
int nwg_ragged_info(nwg_ragged r, uint32_t* num_graphs, uint64_t* total_n, uint64_t* nmax, uint64_t* mmax);
/* parents_dev: packed output, item i's parents (n of its graph) start at
 * item_offsets_host[i] (the running sum of the items' n, written when
 * non-NULL).  blocks_per_sm: resident blocks per SM of the persistent launch
 * (1..8, 0 = 2).  Synchronous; device_ms = device time of the launch. */
int nwg_ragged_bfs(nwg_ragged r, uint32_t num_items, const nwg_ragged_item* items, uint32_t* parents_dev,
                   uint64_t* item_offsets_host, nwg_ragged_result* results_host, uint32_t blocks_per_sm,
                   float* device_ms);

/* Serving: (graph, root) queries against registered graphs kept resident in
 * HBM, answered as depth rows: uint8 (depth per vertex, 255 = unreached; n
 * bytes of the query's graph) or, with depth_bytes = 2, uint16 (0xFFFF =
 * unreached; 2 n bytes).  A query whose depths reach 255 is answered
 * exactly in uint16 rows; in uint8 rows that query alone fails with
 * NWG_EOVERFLOW (its row then holds the depths up to 254, 255 beyond) and
 * the others coalesced with it are answered as usual.  No reference counterpart: NWGraph answers
 * one bfs call at a time; each answer equals the depths of that single-source
 * BFS.  `slots` worker threads, each with its own CUDA stream and
 * multi-source workspace, run batches concurrently: a free slot takes the
 * graph of the oldest waiting query and coalesces up to max_batch waiting
 * queries on that graph into one multi-source pass (nwg_msbfs).  Admission:
 * a query taken by a slot holds (2 * depth_bytes + 0.5) * n bytes of state
 * (its device depth row, its pinned host row and one bit per vertex in four
 * bitsets) until its
 * answer is in host memory; taken state never exceeds the budget left after
 * the slots' fixed buffers (max_batch 256 rows of the largest graph, device
 * and pinned, plus the workspace), and queries that do not fit wait.  All
 * graphs must live on one device and outlive the server. */
typedef struct nwg_server_s* nwg_server;
typedef struct {
  uint32_t slots;        /* concurrent batches (0 = 8, at most 64; fewer if the budget holds fewer) */
  uint32_t max_batch;    /* queries per multi-source pass (0 = 256, at most 256) */
  uint64_t budget_bytes; /* slots' buffers + per-query state, device and pinned host (0 = 16 GiB) */
  int32_t alpha;         /* push/pull switch of the multi-source pass (0 = 4) */
  uint32_t depth_bytes;  /* answer row bytes per vertex: 1 (uint8) or 2 (uint16); 0 = 1 */
} nwg_server_config;
typedef struct {
  uint64_t queries, batches, failed;
  double wall_s;     /* first scheduled arrival to last answer */
  double qps;        /* queries / wall_s */
  double mean_batch; /* queries per multi-source pass */
  double mean_ms, p50_ms, p99_ms, max_ms; /* latency: scheduled arrival to answer in host memory */
  uint64_t peak_state_bytes; /* most per-query state held at once */
  uint64_t budget_bytes;     /* per-query state budget left after the slots */
  uint64_t slot_bytes;       /* fixed buffers of one slot */
  uint32_t slots, peak_in_flight; /* slots created; most batches in flight at once */
  double batch_time_s;       /* summed batch times (take to answer); / wall_s = mean overlap */
} nwg_server_stats;
int nwg_server_create(const nwg_graph* graphs, uint32_t num_graphs, const nwg_server_config* cfg, nwg_server* out);
/* Stops the workers and frees the slots; no nwg_server_wait may be pending. */
int nwg_server_destroy(nwg_server s);
/* Queues one query; depths_host (n * depth_bytes bytes of the graph, or
 * NULL) receives the answer.  nwg_server_wait blocks until that query is answered and returns
 * its status; latency_us = submit to answer. */
int nwg_server_submit(nwg_server s, uint32_t graph, uint32_t root, uint8_t* depths_host, uint64_t* ticket);
int nwg_server_wait(nwg_server s, uint64_t ticket, double* latency_us);
/* Open-loop replay of a query trace: query i (graph[i], root[i]) is released
 * at arrival_us[i] (non-decreasing, microseconds from the start) whatever
 * the server's progress; returns when all are answered.  depths_host[i]
 * (or the whole array) may be NULL; latency_us[i] and batch_size[i] (may be
 * NULL) receive each query's latency from its scheduled arrival and the size
 * of the pass that answered it. */
int nwg_server_run_trace(nwg_server s, uint32_t count, const uint32_t* graph, const uint32_t* root,
                         const double* arrival_us, uint8_t* const* depths_host, double* latency_us,
                         uint32_t* batch_size, nwg_server_stats* stats);

/* Direction-optimizing BFS that allocates no device memory.  No counterpart
 * in the reference: NWGraph's bfs allocates its state per call.  For callers
 * that may not call cudaMalloc/cudaFree (both synchronise the device; latency-
 * bound services and processes whose device memory belongs to their own
 * allocator forbid them).  The caller passes device arrays: uint64 offsets
 * (n + 1), uint32 columns (16-byte aligned), optional in-CSR (NULL = the
 * out-CSR, symmetric), and parents_dev (n entries).  All scratch lives in a
 * static device array of fixed size: n <= 2^20 and m <= 2^24 (larger graphs
 * return NWG_EINVAL before any launch).  Calls share that array: calls whose
 * GPU work overlaps race, so serialise them.  The first call on a device
 * looks the array's device address up and keeps it for the life of the
 * process: do not use this entry point on a device across cudaDeviceReset,
 * which unloads the module that holds the array.  The level loop is driven
 * from the host (a small read-back per step) on `stream` (a cudaStream_t,
 * NULL = legacy default stream) and the call synchronises that stream, so
 * it must not be called while the stream is being captured into a CUDA
 * graph; it returns when the traversal is complete. */
int nwg_bfs_noalloc(const uint64_t* out_off, const uint32_t* out_col, const uint64_t* in_off, const uint32_t* in_col,
                    uint64_t n, uint32_t root, int alpha, int beta, uint32_t* parents_dev, void* stream);

/* Approximate betweenness centrality over `k` sources (Brandes): the
 * computation of nw::graph::brandes_bc<float, double>(graph, sources,
 * threads, ..., normalize) (reference: include/nwgraph/algorithms/
 * betweenness_centrality.hpp:218-324) on the out-graph: per source a BFS
 * with double path counts, then float dependencies accumulated deepest
 * level first, every reached vertex (the source included) adding its own;
 * scores divided by the largest when normalize != 0.  `lanes` sources run
 * at once (0 = 4, at most 16), one stream each.  Scores (n floats) go to
 * scores_host and/or scores_dev; float sums across sources, as in the
 * reference, so results agree with it within the reference verifier's
 * tolerance (1e-6 on normalized scores), not bit for bit. */
typedef struct {
  uint32_t sources;
  uint32_t lanes;
  uint32_t max_levels;
  float device_ms;
} nwg_bc_stats;
int nwg_bc(nwg_graph g, const uint32_t* sources, uint32_t k, int normalize, uint32_t lanes, float* scores_host,
           float* scores_dev, nwg_bc_stats* stats);

/* Graph files into the registry (read on the host, uploaded once like
 * nwg_graph_register).  The format is recognised from the content:
 *  - MatrixMarket, as NWGraph's read_mm reads it (io/mmio.hpp:60-103,
 *    172-208): coordinate general|symmetric, 1-based ids, a symmetric file
 *    contributes both directions of each off-diagonal entry, self-loops and
 *    duplicates kept, values ignored, n = max(rows, cols, largest id);
 *  - NWGraph's binary adjacency, as index_adjacency::serialize writes it
 *    (adjacency.hpp:158-162, containers/compressed.hpp:303-312; 4- or
 *    8-byte offsets, the first array = 4-byte target ids); n is taken from
 *    the offsets count (the 8-byte N_ field is not the vertex count and,
 *    with 4-byte offsets, half of it is not written from N_ at all).
 * Rows are sorted by target.  The in-CSR is the transpose, or the out-CSR
 * itself for a symmetric MatrixMarket file or with NWG_READ_SYMMETRIC. */
#define NWG_READ_SYMMETRIC 0x1u
int nwg_graph_read(const char* path, uint32_t flags, nwg_graph* out);
/* Writes a registered graph's out-CSR in NWGraph's binary adjacency format
 * (8-byte offsets), readable by index_adjacency::deserialize. */
int nwg_graph_write_nwbin(nwg_graph g, const char* path);

/* Device BFSVerifier: the checks of nw::graph::BFSVerifier(g, g_t, source,
 * parent) (reference: include/nwgraph/algorithms/bfs.hpp:44-98) on the GPU,
 * for a parent array in host OR device memory (exactly one non-NULL).  Depths
 * come from a plain top-down BFS written only for this check.  valid = 1 when
 * the reference verifier would return true; otherwise first_bad is the
 * lowest failing vertex (the one the reference stops at) and reason the
 * reference's failure: 1 source wrong, 2 wrong depths, 3 no edge from the
 * parent, 4 reachability mismatch.  Synchronous. */
typedef struct {
  int32_t valid;
  uint32_t reason;
  uint64_t first_bad;
  uint64_t reached; /* vertices reachable from the source */
  uint32_t levels;  /* BFS levels of the check's own traversal */
  float device_ms;
} nwg_verify_result;
int nwg_verify(nwg_graph g, uint32_t source, const uint32_t* parents_host, const uint32_t* parents_dev,
               nwg_verify_result* result);

/* Seeded synthetic graph generators on the device (no reference
 * counterpart: NWGraph ships no RMAT/uniform/grid generator).  Each builds a
 * symmetrized, self-loop-free, deduplicated CSR with sorted rows directly in
 * HBM and registers it (symmetric: out == in).
 * rmat: 2^scale vertices, edge_factor * 2^scale undirected draws with 32-bit
 *       cumulative quadrant thresholds ta < tab < tabc, ids permuted.
 * uniform: n vertices, n * avg_degree / 2 uniform random pairs.
 * grid: width x height 4-neighbour grid plus shortcut_pct % random pairs. */
int nwg_gen_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, uint32_t ta, uint32_t tab, uint32_t tabc,
                 nwg_graph* out);
int nwg_gen_uniform(uint64_t n, uint32_t avg_degree, uint64_t seed, nwg_graph* out);
int nwg_gen_grid(uint32_t width, uint32_t height, uint32_t shortcut_pct, uint64_t seed, nwg_graph* out);

/* `count` roots uniform on [0, n) with out-degree > 0 (seeded). */
int nwg_pick_roots(nwg_graph g, uint64_t seed, uint32_t count, uint32_t* roots_host);

#ifdef __cplusplus
}
#endif

#endif /* NWG_BFS_H */
