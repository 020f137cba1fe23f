// Uses the drop-in header exactly as NWGraph's bench/bfs.cpp uses the
// reference one (bench/bfs.cpp:75-76,129-130,141-143): read a MatrixMarket
// file with NWGraph's read_mm, build adjacency<1> as the out-graph and
// adjacency<0> as the in-graph, call nw::graph::bfs(graph, gx, source,
// num_bins, alpha, beta) and BFSVerifier, and the one-graph
// nw::graph::bfs(graph, source).  Parents are written to <prefix>.<root>.bin
// (uint32) and <prefix>.<root>.td.bin for the test to compare with the oracle.
//
//   dropin_test FILE.mtx PREFIX ROOT...
//   dropin_test --mutate FILE.mtx ROOT
//
// --mutate: after a first call, changes one column of the out-graph in place
// at an entry the registry's sampled fingerprint does not read, calls the
// one-graph bfs again and compares its depths with a serial BFS of the
// changed graph (prints "mutation_seen 1" when they agree).  Run with
// NWG_DROPIN_STRICT=1, which makes every call upload the graph again.
//
// Built against this repository's include/ first (so "nwgraph/algorithms/
// bfs.hpp" is the drop-in) and NWGraph's headers second.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <string>
#include <vector>

#include "nwgraph/adjacency.hpp"
#include "nwgraph/algorithms/bfs.hpp"
#include "nwgraph/edge_list.hpp"
#include "nwgraph/io/mmio.hpp"

// Depth of every vertex from the parents (unreached: -1); -2 when a parent
// chain does not reach the root.
static std::vector<long> depths_of(const std::vector<uint32_t>& parents, uint32_t root) {
  const size_t      n = parents.size();
  std::vector<long> d(n, -1);
  d[root] = 0;
  for (size_t v = 0; v < n; ++v) {
    if (parents[v] == std::numeric_limits<uint32_t>::max() || d[v] >= 0) continue;
    std::vector<size_t> chain;
    size_t              u = v;
    while (d[u] < 0 && chain.size() <= n) {
      chain.push_back(u);
      const uint32_t p = parents[u];
      if (p == std::numeric_limits<uint32_t>::max()) break;
      u = p;
    }
    long base = d[u] >= 0 ? d[u] : -2;
    for (size_t i = chain.size(); i-- > 0;) d[chain[i]] = base < 0 ? -2 : ++base;
  }
  return d;
}

template <class G>
static std::vector<long> serial_depths(const G& g, uint32_t root) {
  const auto&       idx = g.indices_;
  const auto&       col = std::get<0>(g.to_be_indexed_);
  const size_t      n   = idx.size() - 1;
  std::vector<long> d(n, -1);
  std::vector<uint32_t> q{root};
  d[root] = 0;
  for (size_t h = 0; h < q.size(); ++h) {
    const uint32_t u = q[h];
    for (auto e = idx[u]; e < idx[u + 1]; ++e)
      if (d[col[e]] < 0) {
        d[col[e]] = d[u] + 1;
        q.push_back(col[e]);
      }
  }
  return d;
}

static int mutate_check(const char* mtx, uint32_t root) {
  auto aos   = nw::graph::read_mm<nw::graph::directedness::directed>(std::string(mtx));
  auto graph = nw::graph::adjacency<1>(aos);
  auto first = nw::graph::bfs(graph, root);  // uploads the graph
  auto&        col = std::get<0>(graph.to_be_indexed_);
  const size_t m   = col.size();
  const size_t n   = graph.indices_.size() - 1;
  const size_t e   = (m - 1) / 126;  // between the fingerprint's first two samples, 0 and (m - 1) / 63
  col[e]           = (uint32_t)((col[e] + n / 2) % n);
  auto again       = nw::graph::bfs(graph, root);
  const bool seen  = depths_of(again, root) == serial_depths(graph, root);
  std::printf("mutation_seen %d changed_first %d\n", seen ? 1 : 0, depths_of(first, root) != depths_of(again, root));
  nw::graph::b200::release_all();
  return seen ? 0 : 1;
}

int main(int argc, char** argv) {
  if (argc == 4 && std::string(argv[1]) == "--mutate") return mutate_check(argv[2], (uint32_t)std::strtoul(argv[3], nullptr, 10));
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s FILE.mtx PREFIX ROOT...\n", argv[0]);
    return 2;
  }
  auto aos   = nw::graph::read_mm<nw::graph::directedness::directed>(std::string(argv[1]));
  auto graph = nw::graph::adjacency<1>(aos);
  auto gx    = nw::graph::adjacency<0>(aos);
  int  bad   = 0;
  for (int a = 3; a < argc; ++a) {
    const uint32_t root    = (uint32_t)std::strtoul(argv[a], nullptr, 10);
    auto           parents = nw::graph::bfs(graph, gx, root, 32, 15, 18);
    const bool     ok      = nw::graph::BFSVerifier(graph, gx, root, parents);
    auto           td      = nw::graph::bfs(graph, root);
    const bool     ok_td   = nw::graph::BFSVerifier(graph, gx, root, td);
    // a second call on the same graphs reuses the resident upload
    auto again = nw::graph::bfs(graph, gx, root, 32, 15, 18);
    const bool ok2 = nw::graph::BFSVerifier(graph, gx, root, again);
    std::string   base = std::string(argv[2]) + "." + std::to_string(root);
    std::ofstream(base + ".bin", std::ios::binary).write(reinterpret_cast<const char*>(parents.data()),
                                                         parents.size() * sizeof(parents[0]));
    std::ofstream(base + ".td.bin", std::ios::binary).write(reinterpret_cast<const char*>(td.data()),
                                                            td.size() * sizeof(td[0]));
    std::printf("root %u dobfs_verifier %d topdown_verifier %d repeat_verifier %d\n", root, ok, ok_td, ok2);
    bad += !(ok && ok_td && ok2);
  }
  nw::graph::b200::release_all();
  return bad ? 1 : 0;
}
