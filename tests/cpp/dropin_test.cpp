// Uses the drop-in header exactly as NWGraph's bench/bfs.cpp uses the
// reference one (bench/bfs.cpp:75-76,129-130,141-143): read a MatrixMarket
// file with NWGraph's read_mm, build adjacency<1> as the out-graph and
// adjacency<0> as the in-graph, call nw::graph::bfs(graph, gx, source,
// num_bins, alpha, beta) and BFSVerifier, and the one-graph
// nw::graph::bfs(graph, source).  Parents are written to <prefix>.<root>.bin
// (uint32) and <prefix>.<root>.td.bin for the test to compare with the oracle.
//
//   dropin_test FILE.mtx PREFIX ROOT...
//
// Built against this repository's include/ first (so "nwgraph/algorithms/
// bfs.hpp" is the drop-in) and NWGraph's headers second.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "nwgraph/adjacency.hpp"
#include "nwgraph/algorithms/bfs.hpp"
#include "nwgraph/edge_list.hpp"
#include "nwgraph/io/mmio.hpp"

int main(int argc, char** argv) {
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
