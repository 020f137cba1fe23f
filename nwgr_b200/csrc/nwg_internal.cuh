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

// Degree bins of the frontier queue: a vertex is expanded by a warp-shared
// gather (S), one warp (M), one CTA (L) or the whole grid (H).
enum Bin : int { kBinS = 0, kBinM = 1, kBinL = 2, kBinH = 3, kNumBins = 4 };

// Actions of the device level loop (the switch node's branches).
enum Action : uint32_t { kActTD = 0, kActBU = 1, kActB2Q = 2, kActNone = 3, kNumActions = 3 };

struct Thresholds {
  uint32_t warp_min;  // degree >= warp_min -> bin M
  uint32_t cta_min;   // degree >= cta_min  -> bin L
  uint32_t grid_min;  // degree >= grid_min -> bin H
};

__host__ __device__ inline int degree_bin(uint64_t deg, const Thresholds& t) {
  return deg >= t.grid_min ? kBinH : deg >= t.cta_min ? kBinL : deg >= t.warp_min ? kBinM : kBinS;
}

// Device control block of one traversal.  Written by the init kernel, then
// advanced by the decide kernel between actions; action kernels only add to
// the accumulators and queue counters.
struct Ctrl {
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

  uint32_t qcount[2][kNumBins];  // entries per bin of queue buffer 0/1
  uint32_t cur;                  // queue buffer holding the frontier
  uint32_t bm;                   // bottom-up: index of the bitmap holding the latest pull's discoveries
  uint32_t bu_mode;              // 0: first pull of a phase (front = visited), 1: later pull (front = C[bm])
  uint32_t action;               // action of the current loop iteration

  uint32_t steps, levels, td_steps, bu_steps, b2q_steps;
  int32_t  status;
  unsigned long long reached;
  uint32_t trace_len;
  uint32_t max_steps;
  uint8_t            trace_dir[NWG_TRACE_CAP];
  unsigned long long trace_frontier[NWG_TRACE_CAP];
  unsigned long long trace_found[NWG_TRACE_CAP];
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
  uint32_t*       q[2][kNumBins];
  uint32_t        qcap[kNumBins];
  Thresholds      th;
  Ctrl*           ctrl;
  cudaGraphConditionalHandle h_loop;
  cudaGraphConditionalHandle h_switch;
};

struct GraphDev;

// Per-traversal device state.
struct Workspace {
  GraphDev*       g = nullptr;
  int             device = 0;
  uint32_t*       parents = nullptr;  // default output
  uint32_t*       V = nullptr;        // V, C0, C1 in one allocation
  uint32_t*       qbuf = nullptr;     // both queue buffers, all bins
  Ctrl*           ctrl = nullptr;     // device
  Ctrl*           ctrl_host = nullptr;  // pinned mirror for stats
  cudaStream_t    stream = nullptr;   // owned stream for the synchronous API
  cudaEvent_t     ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t     template_graph = nullptr;  // kept alive: init_node belongs to it
  cudaGraphExec_t exec[1] = {nullptr};     // the level loop (direction-optimizing or top-down only)
  cudaGraphNode_t init_node[1] = {nullptr};
  DobfsParams     params{};
  bool            ran = false;
  bool            timed = false;
};

struct GraphDev {
  int       device = 0;
  uint64_t  n = 0, m = 0, in_m = 0;
  uint64_t* off = nullptr;
  uint32_t* col = nullptr;
  uint64_t* in_off = nullptr;
  uint32_t* in_col = nullptr;
  uint32_t* Z = nullptr;  // in-degree-zero bitmap
  bool      owns_out = false, owns_in = false, symmetric = true;
  int       sm_count = 148;
  Thresholds th{32, 1024, 32768};
  std::mutex              mu;
  Workspace*              default_ws = nullptr;
  std::vector<Workspace*> workspaces;
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
int  ws_init(GraphDev* g, Workspace* ws);
void ws_free(Workspace* ws);
int  ws_launch(Workspace* ws, uint32_t root, int alpha, int beta, uint32_t* parents, cudaStream_t stream,
               bool topdown_only);
void fill_stats(const Ctrl& c, nwg_bfs_stats* s);
int  build_zero_indegree(GraphDev* g, cudaStream_t stream);
int  component_edges(GraphDev* g, const uint32_t* parents, uint64_t* edges, uint64_t* vertices);
int  widen_offsets(const uint32_t* src, uint64_t* dst, uint64_t count, cudaStream_t stream);

// nwg_gen.cu
int gen_rmat(uint32_t scale, uint32_t ef, uint64_t seed, uint32_t ta, uint32_t tab, uint32_t tabc, GraphDev* g);
int gen_uniform(uint64_t n, uint32_t deg, uint64_t seed, GraphDev* g);
int gen_grid(uint32_t w, uint32_t h, uint32_t pct, uint64_t seed, GraphDev* g);
int pick_roots(GraphDev* g, uint64_t seed, uint32_t count, uint32_t* roots_host);

}  // namespace nwg
