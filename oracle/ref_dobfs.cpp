// TEST INFRASTRUCTURE ONLY (the oracle).  Compiled against the UNMODIFIED
// reference header include/nwgraph/algorithms/bfs.hpp, with the project's
// TBB compatibility shim (oracle/tbb_compat) standing in for oneTBB, which is
// not installed.  Nothing in the product links this file; tests and the CPU
// baseline leg of bench.py load the resulting oracle/_ref/libnwgref.so.
//
// Exported C functions (everything else is built with hidden visibility so
// the reference's nw::graph::bfs template instances never interpose on the
// drop-in's symbols):
//   nwgref_graph_create  - build index_adjacency<0, uint64_t, uint32_t>
//                          (adjacency.hpp:66-177) from plain CSR arrays
//   nwgref_dobfs         - nw::graph::bfs(out, in, root, bins, alpha, beta)
//                          (algorithms/bfs.hpp:160-311), timed with a wall
//                          clock around the call like time_op
//                          (bench/common.hpp:155-167)
//   nwgref_bfs_serial    - nw::graph::bfs(graph, root) (algorithms/bfs.hpp:110-140)
//   nwgref_verify        - BFSVerifier(out, in, root, parents)
//                          (algorithms/bfs.hpp:44-98)
//   nwgref_bc            - brandes_bc<float, double>(out, sources, threads)
//                          (algorithms/betweenness_centrality.hpp:218-324),
//                          the parallel approximate betweenness centrality
//                          NWGraph's bench/bc.cpp:136 runs, timed with a wall clock
//   nwgref_bc_verify     - BCVerifier<float, double>(out, sources, scores)
//                          (algorithms/betweenness_centrality.hpp:59-128)
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "nwgraph/adjacency.hpp"
#include "nwgraph/algorithms/betweenness_centrality.hpp"
#include "nwgraph/algorithms/bfs.hpp"

#define NWGREF_API extern "C" __attribute__((visibility("default")))

namespace {
using ref_graph = nw::graph::index_adjacency<0, uint64_t, uint32_t>;

struct ref_pair {
  ref_graph  out;
  ref_graph  in_own;
  ref_graph* in = nullptr;  // == &out when the caller passed no in-graph
};

void fill(ref_graph& g, const uint64_t* off, const uint32_t* col, uint64_t n) {
  uint64_t m = off[n];
  std::memcpy(g.indices_.data(), off, (n + 1) * sizeof(uint64_t));
  std::memcpy(std::get<0>(g.to_be_indexed_).data(), col, m * sizeof(uint32_t));
}
}  // namespace

NWGREF_API void* nwgref_graph_create(const uint64_t* out_off, const uint32_t* out_col, const uint64_t* in_off,
                                     const uint32_t* in_col, uint64_t n) {
  auto* p = new ref_pair{ref_graph(n, out_off[n]), ref_graph(0, 0), nullptr};
  fill(p->out, out_off, out_col, n);
  if (in_off && in_col) {
    p->in_own = ref_graph(n, in_off[n]);
    fill(p->in_own, in_off, in_col, n);
    p->in = &p->in_own;
  } else {
    p->in = &p->out;
  }
  return p;
}

NWGREF_API void nwgref_graph_free(void* h) { delete static_cast<ref_pair*>(h); }

NWGREF_API int nwgref_dobfs(void* h, uint32_t root, int num_bins, int alpha, int beta, uint32_t* parents_out,
                            double* seconds_out) {
  auto* p     = static_cast<ref_pair*>(h);
  auto  start = std::chrono::high_resolution_clock::now();
  auto  par   = nw::graph::bfs(p->out, *p->in, root, num_bins, alpha, beta);
  std::chrono::duration<double> el = std::chrono::high_resolution_clock::now() - start;
  if (seconds_out) *seconds_out = el.count();
  if (parents_out) std::memcpy(parents_out, par.data(), par.size() * sizeof(uint32_t));
  return 0;
}

NWGREF_API int nwgref_bfs_serial(void* h, uint32_t root, uint32_t* parents_out) {
  auto* p   = static_cast<ref_pair*>(h);
  auto  par = nw::graph::bfs(p->out, root);
  std::memcpy(parents_out, par.data(), par.size() * sizeof(uint32_t));
  return 0;
}

NWGREF_API int nwgref_verify(void* h, uint32_t root, const uint32_t* parents, uint64_t n) {
  auto*                 p = static_cast<ref_pair*>(h);
  std::vector<uint32_t> par(parents, parents + n);
  return nw::graph::BFSVerifier(p->out, *p->in, root, par) ? 1 : 0;
}

NWGREF_API int nwgref_bc(void* h, const uint32_t* sources, uint64_t k, int threads, int normalize, float* scores_out,
                         double* seconds_out) {
  auto*                 p = static_cast<ref_pair*>(h);
  std::vector<uint32_t> src(sources, sources + k);
  auto                  start = std::chrono::high_resolution_clock::now();
  auto sc = nw::graph::brandes_bc<float, double>(p->out, src, threads, std::execution::par_unseq, std::execution::par_unseq,
                                                 normalize != 0);
  std::chrono::duration<double> el = std::chrono::high_resolution_clock::now() - start;
  if (seconds_out) *seconds_out = el.count();
  std::memcpy(scores_out, sc.data(), sc.size() * sizeof(float));
  return 0;
}

NWGREF_API int nwgref_bc_verify(void* h, const uint32_t* sources, uint64_t k, const float* scores, uint64_t n) {
  auto*                 p = static_cast<ref_pair*>(h);
  std::vector<uint32_t> src(sources, sources + k);
  std::vector<float>    sc(scores, scores + n);
  return nw::graph::BCVerifier<float, double>(p->out, src, sc) ? 1 : 0;
}

NWGREF_API int nwgref_threads() { return tbb::this_task_arena::max_concurrency(); }

// Sets the shim's thread count for subsequent calls (0 = default).
NWGREF_API void nwgref_set_threads(int t) { tbb::detail_compat::threads_override().store(t); }
