// Internal declarations shared by the CUDA translation units of
// libnwgr_b200.so.  Not installed; the public surface is include/nwg_bfs.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "nwg_bfs.h"

namespace nwg {

constexpr uint32_t kNull     = 0xFFFFFFFFu;
constexpr unsigned kFullMask = 0xFFFFFFFFu;

// Frontier queues.  A vertex whose out-degree is below `warp_min` goes to
// the small queue (ids; a warp expands 32 of them at once through a
// scan-based gather); any other vertex is split into chunks of `chunk`
// out-edges, one queue entry (vertex << 32 | chunk index) per chunk, and a
// warp expands one chunk at a time.  Hubs are thus spread over the whole
// grid instead of occupying one warp or CTA.
// Queue fill level of buffer q: qpos[q] packs the small-queue entry count
// (low 32 bits) and the chunk-queue entry count (high 32 bits) so one 64-bit
// atomicAdd reserves space in both; qbig[q] counts the chunked vertices.

// Actions of the device level loop (the switch node's branches).
enum Action : uint32_t {
  kActTD      = 0,  // top-down step, full grid
  kActBU      = 1,  // bottom-up pull
  kActB2Q     = 2,  // bitmap -> queue
  kActTDSmall = 3,  // top-down step on a small frontier, small grid
  kActTDCluster = 4,  // top-down step on a tiny frontier, one thread-block cluster
  kActNone    = 5,
  kNumActions = 5,
  // a bottom-up pull run as a push whose discoveries are marked in the
  // pull's discovery bitmap instead of queued (persistent kernel only)
  kActBUMark  = 6,
  // a top-down step whose discoveries are marked likewise, with their count
  // and out-degree sum (persistent kernel only)
  kActTDMark  = 7
};

struct Thresholds {
  uint32_t warp_min;     // out-degree >= warp_min -> chunked
  uint32_t chunk;        // out-edges per chunk entry (a power of two)
  uint32_t chunk_shift;  // log2(chunk)
};

// Device control block of one traversal.  Written by the init kernel, then
// advanced by the decide kernel between actions; action kernels only add to
// the accumulators and queue counters.  The header is read and written by
// the decide kernel with 16-byte vector accesses (one memory round trip).
struct alignas(16) CtrlHdr {
  uint32_t* parents;  // output array of this traversal
  uint32_t  root;
  uint32_t  alpha;
  uint32_t  beta;
  uint32_t  topdown_only;

  unsigned long long edges_to_check;  // bfs.hpp:177
  unsigned long long scout_count;     // bfs.hpp:178
  unsigned long long awake_count;     // bfs.hpp:190
  unsigned long long old_awake;       // bfs.hpp:204

  unsigned long long acc_scout;  // += out-degree of every vertex a top-down step discovers
  unsigned long long acc_awake;  // += vertices a bottom-up pull discovers

  unsigned long long qpos[2];    // [buffer] small entries | chunk entries << 32
  uint32_t           qbig[2];    // [buffer] vertices in the chunk queue
  uint32_t           nhub[2];    // [buffer] hub records whose chunk entries are still to be written
  uint32_t cur;                  // queue buffer holding the frontier
  uint32_t bm;                   // bottom-up: index of the bitmap holding the latest pull's discoveries
  uint32_t bu_mode;              // 0: first pull of a phase (front = visited), 1: later pull (front = C[bm])
  uint32_t action;               // action of the current loop iteration

  uint32_t steps, levels, td_steps, bu_steps, b2q_steps;
  int32_t  status;
  uint32_t pre_decided;  // the previous action kernel already made the next decision
  uint32_t bu_push;      // the top-down kernel's current step is a bottom-up pull run as a push
  unsigned long long reached;
  unsigned long long t_start;  // %globaltimer at init (ns)
  uint32_t trace_len;
  uint32_t max_steps;
  uint32_t scout_exact;  // scout_count is the frontier's out-degree sum (the first step, after a top-down step)
  uint32_t prev_small;   // the last step was a top-down step whose frontier had at most kSoloCap out-edges
  uint32_t mark_ok;      // kActBUMark / kActTDMark may be chosen (set by the persistent kernel in its copies)
  uint32_t b2q_then_td;  // the bitmap -> queue pass rebuilds the queue of a marking top-down step
  uint32_t pad_[2];
};
static_assert(sizeof(CtrlHdr) % 16 == 0, "the header is copied in 16-byte pieces");

// Grid barrier of the persistent small-frontier kernel.
struct GridBar {
  alignas(128) unsigned int count;  // arrivals (own 128-byte line)
  alignas(128) unsigned int gen;    // generation, polled with acquire loads (own line)
  // the persistent traversal kernel's barrier: arrivals since the launch,
  // never reset inside it (barrier k is passed when it reaches k * blocks)
  alignas(128) unsigned long long arrivals;
};

// Counters of one step of the persistent traversal kernel (k_trav), which
// rotates three of them so that a slot is cleared only when no block can
// still be reading it.
struct alignas(64) StepAcc {
  unsigned long long qpos;   // output queues' entries: small | chunk << 32
  unsigned long long scout;  // out-degree sum of the vertices a top-down step discovers
  unsigned long long awake;  // vertices a pull discovers
  uint32_t           qbig;   // chunked vertices appended
  uint32_t           nhub;   // deferred hub records appended
};

struct Ctrl {
  CtrlHdr            h;
  GridBar            bar;
  StepAcc            acc[3];
  uint32_t           kernels;  // kernel launches of the traversal when one persistent kernel ran it (else 0)
  int32_t            err;  // set with atomics by a device wait that ran out (never overwritten by the header copy)
  uint32_t           decides;  // k_decide launches of the traversal (each loop iteration launches one)
  uint8_t            trace_dir[NWG_TRACE_CAP];
  unsigned long long trace_frontier[NWG_TRACE_CAP];
  unsigned long long trace_found[NWG_TRACE_CAP];
  unsigned long long trace_end_ns[NWG_TRACE_CAP];  // %globaltimer - t_start when the step's result was consumed
  unsigned long long t_first_decide;
};

// A vertex with many chunk entries discovered by the persistent small-level
// kernel: its entries qc[pos .. pos + nc) are written by the whole grid after
// the level's barrier instead of by the one warp that claimed it.
struct HubRec {
  uint32_t v;
  uint32_t nc;
  uint64_t pos;
};

// Static parameters of the level-loop kernels (baked into the CUDA graph).
struct DobfsParams {
  const uint64_t* off;     // out-CSR offsets [n+1]
  const uint32_t* col;     // out-CSR columns [m]
  const uint64_t* in_off;  // in-CSR offsets (== off when symmetric)
  const uint32_t* in_col;
  uint64_t        n;
  uint64_t        m;
  uint32_t        nwords;  // ceil(n / 32)
  uint32_t*       V;       // visited bitmap [nwords]
  uint32_t*       C0;      // bottom-up discovery bitmaps [nwords] x 2
  uint32_t*       C1;
  const uint32_t* Z;       // in-degree-zero bitmap [nwords] (never discoverable bottom-up)
  const uint16_t* deg16;   // out-degrees saturated at 0xFFFF [n] (NULL: degrees come from off)
  uint32_t*       qs[2];  // small-degree vertex queues
  uint64_t*       qc[2];  // chunk queues
  uint64_t        qs_cap;
  uint64_t        qc_cap;
  HubRec*         hubrec[2];  // [buffer] deferred hub records (null: hubs are written by their warp)
  uint64_t        hub_cap;
  Thresholds      th;
  uint64_t        nzero;      // vertices without in-edges (0 where unknown: only a cost estimate uses it)
  uint32_t        symmetric;  // the in-CSR is the out-CSR (a pull may then run as a push)
  Ctrl*           ctrl;
};

struct GraphDev;

// Per-traversal device state.
struct Workspace {
  GraphDev*       g = nullptr;
  int             device = 0;
  uint32_t*       parents = nullptr;  // default output
  uint32_t*       V = nullptr;        // V, C0, C1 in one allocation
  uint32_t*       qbuf = nullptr;     // both small queues
  uint64_t*       cbuf = nullptr;     // both chunk queues
  HubRec*         hubbuf = nullptr;   // both deferred-hub record lists
  Ctrl*           ctrl = nullptr;     // device
  Ctrl*           ctrl_host = nullptr;  // pinned mirror for stats
  cudaStream_t    stream = nullptr;   // owned stream for the synchronous API
  cudaEvent_t     ev0 = nullptr, ev1 = nullptr;
  int             trav_grid = 0;     // blocks of the persistent traversal kernel (all resident)
  DobfsParams     params{};
  bool            ran = false;
  bool            timed = false;
};

// State of the batched multi-source BFS (nwg_msbfs.cu); sized for 256
// sources (four 64-bit words) per vertex of any graph with at most n_cap
// vertices and m_cap out-edges.
struct MsWorkspace {
  GraphDev*       g       = nullptr;  // the graph it was created for (may be null for a shared one)
  uint64_t        n_cap = 0, m_cap = 0;
  int             sm_count = 148;
  uint64_t*       vis     = nullptr;
  uint64_t*       fr[2]   = {nullptr, nullptr};
  uint64_t*       nx      = nullptr;
  uint64_t*       dp      = nullptr;  // 8 level bit-planes (depth bit j of each source), zero between passes
  uint32_t*       tlist   = nullptr;  // vertices a push level touched (sparse finalize)
  uint32_t*       tbits   = nullptr;  // their bitmap, zero between levels
  uint64_t*       list[2] = {nullptr, nullptr};  // frontier chunk entries
  uint64_t        list_cap = 0;
  void*           pass_dev  = nullptr;  // arguments and level-loop state of a pass (device)
  void*           pass_host = nullptr;  // pinned staging of the same record
  cudaGraphExec_t exec[4] = {nullptr, nullptr, nullptr, nullptr};  // pass graphs, one per word count W
  std::vector<unsigned char> last_args[4];                          // the arguments each exec was last set to
  cudaGraph_t     tmpl[4] = {nullptr, nullptr, nullptr, nullptr};  // their templates (own the nodes below)
  cudaGraphNode_t nodes[4][10] = {};                                // kernel nodes updated per pass
  int             node_occ[4][10] = {};                             // their resident blocks per SM
  bool            stepped = false;      // host-driven levels (NWG_MS_STEPPED=1), for profilers
  cudaStream_t    stream  = nullptr;
  cudaEvent_t     ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t     ev_fork = nullptr;     // the caller's stream position that the lanes start after
  std::vector<MsWorkspace*> lanes;       // further pass states for calls of more than one pass (own streams)
};

// Ragged batch (many small graphs, one persistent launch).
struct RaggedGraph {  // one packed graph (device and host copies)
  uint64_t n, m;
  uint64_t off_base;  // index of the graph's first offset in the packed offsets
  uint64_t col_base;  // index of its first column (a multiple of 4: 16-byte aligned)
  uint64_t z_base;    // index of its first in-degree-zero bitmap word
};

struct RaggedItem {  // one (graph, root) traversal
  uint32_t graph;
  uint32_t root;
  uint64_t out_base;  // index of the item's parents in the packed output
  int32_t  alpha;
  int32_t  beta;
  uint32_t warp_min;  // degree threshold of the chunked queue
  uint32_t pad;
};

struct RaggedResult {
  int32_t  status;
  uint32_t steps, levels, td_steps, bu_steps, b2q_steps;
  uint64_t reached;
};

struct RaggedParams {
  const uint64_t*     off;
  const uint32_t*     col;
  const uint32_t*     Z;
  const RaggedGraph*  graphs;
  const RaggedItem*   items;
  RaggedResult*       results;
  uint32_t*           parents;
  uint32_t            n_items;
  unsigned int*       next_item;
  unsigned char*      scratch;  // one slot per resident block
  uint64_t            slot_bytes;
  uint64_t            nmax, mmax;
};

struct RaggedDev {
  int                      device   = 0;
  int                      sm_count = 148;
  uint32_t                 ngraphs  = 0;
  uint64_t                 nmax = 0, mmax = 0, total_n = 0;
  uint64_t*                off      = nullptr;
  uint32_t*                col      = nullptr;
  uint32_t*                Z        = nullptr;
  RaggedGraph*             graphs   = nullptr;
  std::vector<RaggedGraph> graphs_host;
  // run state (sized by the last run)
  RaggedItem*              items    = nullptr;
  RaggedResult*            results  = nullptr;
  unsigned int*            counter  = nullptr;
  unsigned char*           scratch  = nullptr;
  uint64_t                 scratch_bytes = 0, items_cap = 0;
  cudaStream_t             stream   = nullptr;
  cudaEvent_t              ev0 = nullptr, ev1 = nullptr;
  cudaGraphExec_t          exec     = nullptr;
  uint32_t                 exec_items = 0, exec_slots = 0;
  uint32_t*                exec_parents = nullptr;
  std::mutex               mu;
};

struct GraphDev {
  int       device = 0;
  uint64_t  n = 0, m = 0, in_m = 0;
  uint64_t* off = nullptr;
  uint32_t* col = nullptr;
  uint64_t* in_off = nullptr;
  uint32_t* in_col = nullptr;
  uint32_t* Z = nullptr;  // in-degree-zero bitmap
  uint16_t* deg16 = nullptr;  // out-degrees saturated at 0xFFFF (2 bytes a vertex: mostly L2-resident)
  uint64_t  nzero = 0;    // its population (vertices without in-edges)
  bool      owns_out = false, owns_in = false, symmetric = true;
  int       sm_count = 148;
  // out-degree >= 64 goes to the chunk queue: 2.0% (RMAT-24) and 2.4%
  // (uniform 2^24) faster than 32 on a B200; 512-edge chunks gained nothing
  Thresholds th{64, 256, 8};
  std::mutex                mu;
  Workspace*                default_ws = nullptr;
  Workspace*                pipe_ws    = nullptr;  // second lane of nwg_bfs_roots
  std::vector<Workspace*>   workspaces;
  std::vector<MsWorkspace*> ms_workspaces;
};

// Error plumbing (nwg_api.cu).
int         set_error(int code, const std::string& msg);
int         cuda_error(cudaError_t e, const char* what);
#define NWG_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return ::nwg::cuda_error(_e, #expr); \
  } while (0)

// nwg_dobfs.cu
int  wait_probe(uint32_t spins, int32_t* status, float* waited_ms);
int  ws_init(GraphDev* g, Workspace* ws);
void ws_free(Workspace* ws);
int  ws_launch(Workspace* ws, uint32_t root, int alpha, int beta, uint32_t* parents, cudaStream_t stream,
               bool topdown_only);
int  ws_launch_stepped(Workspace* ws, uint32_t root, int alpha, int beta, uint32_t* parents, cudaStream_t stream);
int  run_stepped(const DobfsParams& params, int sm_count, uint32_t root, int alpha, int beta, uint32_t* parents,
                 cudaStream_t stream);
int  zero_indegree_into(const uint64_t* in_off, uint64_t n, uint32_t* Z, int sm_count, cudaStream_t stream);
void fill_stats(const Ctrl& c, nwg_bfs_stats* s);
int  depth_row16(Workspace* ws, uint32_t root, uint16_t* row, cudaStream_t stream);
int  build_zero_indegree(GraphDev* g, cudaStream_t stream);
int  build_deg16(GraphDev* g, cudaStream_t stream);
int  component_edges(GraphDev* g, const uint32_t* parents, uint64_t* edges, uint64_t* vertices);
int  widen_offsets(const uint32_t* src, uint64_t* dst, uint64_t count, cudaStream_t stream);

int  ragged_launch(RaggedDev* r, uint32_t n_items, uint32_t* parents_dev, uint32_t blocks_per_sm, float* ms);
int  ragged_slot_bytes(uint64_t nmax, uint64_t mmax, uint64_t* bytes);
int  zero_indegree_packed(RaggedDev* r);

// nwg_msbfs.cu
int      ms_ws_init(GraphDev* g, MsWorkspace* ws);
int      ms_ws_init_cap(GraphDev* g, uint64_t n_cap, uint64_t m_cap, MsWorkspace* ws);
uint64_t ms_ws_bytes(uint64_t n_cap, uint64_t m_cap);
void     ms_ws_free(MsWorkspace* ws);
int      ms_run_on(MsWorkspace* ws, GraphDev* g, const uint32_t* roots_host, uint32_t k, void* depths_dev,
                   uint32_t depth_bytes, uint8_t* deep_flags, int alpha, cudaStream_t stream, nwg_msbfs_stats* st,
                   cudaEvent_t end_ev = nullptr, cudaEvent_t start_ev = nullptr);
int      ms_run(MsWorkspace* ws, const uint32_t* roots_host, uint32_t k, void* depths_dev, uint32_t depth_bytes,
                uint8_t* deep_flags, int alpha, cudaStream_t stream, nwg_msbfs_stats* st, cudaEvent_t end_ev = nullptr,
                cudaEvent_t start_ev = nullptr);

// nwg_gen.cu
int gen_rmat(uint32_t scale, uint32_t ef, uint64_t seed, uint32_t ta, uint32_t tab, uint32_t tabc, GraphDev* g);
int gen_uniform(uint64_t n, uint32_t deg, uint64_t seed, GraphDev* g);
int gen_grid(uint32_t w, uint32_t h, uint32_t pct, uint64_t seed, GraphDev* g);
int pick_roots(GraphDev* g, uint64_t seed, uint32_t count, uint32_t* roots_host);

}  // namespace nwg
