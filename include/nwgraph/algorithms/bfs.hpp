// Drop-in replacement for NWGraph's include/nwgraph/algorithms/bfs.hpp that
// runs the traversals on a B200 through libnwgr_b200.so (C ABI:
// include/nwg_bfs.h).  Put this repository's include/ directory before
// NWGraph's on the include path; every other NWGraph header still comes from
// NWGraph.  The three templates keep the reference's names, signatures and
// results:
//
//   bfs(out_graph, in_graph, root, num_bins = 32, alpha = 15, beta = 18)
//       direction-optimizing BFS (reference: algorithms/bfs.hpp:160-311);
//       nwg_bfs.  num_bins is accepted and ignored: the device bins the
//       frontier by degree, not by u % num_bins.
//   bfs(graph, root)
//       top-down BFS over out-edges only (reference: bfs.hpp:110-140);
//       nwg_bfs_topdown.
//   BFSVerifier(g, g_t, source, parent)
//       host check (reference: bfs.hpp:44-98), same rules and messages.
//
// Graph arguments must expose NWGraph's CSR members, as the reference's
// bfs itself requires (it reads out_graph.to_be_indexed_, bfs.hpp:168):
// indices_ (uint32 or uint64 offsets) and std::get<0>(to_be_indexed_)
// (32-bit vertex ids), i.e. index_adjacency / adjacency<idx>.
//
// Upload once: the first call on a graph uploads its CSR to the GPU and keeps
// it resident; later calls on the same objects reuse it.  A graph is
// recognised by its array addresses, sizes and a sampled fingerprint of its
// contents; modifying a graph in place between calls is detected by the
// fingerprint in most cases, but call nw::graph::b200::release(g) after
// mutating a graph to be certain, and before destroying it to free the
// device copy early (the registry otherwise keeps it until exit).  With the
// environment variable NWG_DROPIN_STRICT set (to anything but "0") every
// call uploads the graph again, so each call sees the graph's current
// contents as the reference's does, at the cost of one CSR upload per call.
//
// Deviations (documented): the reference cannot fail; this header throws
// std::runtime_error when the device reports an error (bad root, out of
// memory, CUDA error), and requires 32-bit vertex ids.
#ifndef NW_GRAPH_BFS_HPP
#define NW_GRAPH_BFS_HPP

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "nwg_bfs.h"
#include "nwgraph/graph_concepts.hpp"
#include "nwgraph/graph_traits.hpp"

namespace nw {
namespace graph {
namespace b200 {

inline void check(int rc) {
  if (rc != NWG_OK) {
    char buf[1024];
    nwg_last_error(buf, sizeof(buf));
    throw std::runtime_error(std::string("nwgr_b200: ") + buf);
  }
}

// One resident CSR pair per (out graph, in graph) argument pair.
class registry {
 public:
  struct key {
    const void* out_idx;
    const void* out_col;
    const void* in_idx;
    const void* in_col;
    uint64_t    n, m;
    bool        operator<(const key& o) const {
      return std::tie(out_idx, out_col, in_idx, in_col, n, m) < std::tie(o.out_idx, o.out_col, o.in_idx, o.in_col, o.n, o.m);
    }
  };

  static registry& get() {
    static registry r;
    return r;
  }

  ~registry() {
    for (auto& kv : map_) nwg_graph_release(kv.second.h);
  }

  template <class Idx>
  nwg_graph acquire(const std::vector<Idx>& out_idx, const uint32_t* out_col, const std::vector<Idx>* in_idx,
                    const uint32_t* in_col) {
    static_assert(std::is_same_v<Idx, uint32_t> || std::is_same_v<Idx, uint64_t>, "CSR offsets must be uint32 or uint64");
    const uint64_t n = out_idx.size() ? out_idx.size() - 1 : 0;
    const uint64_t m = n ? (uint64_t)out_idx[n] : 0;
    const key      k{out_idx.data(), out_col, in_idx ? in_idx->data() : nullptr, in_col, n, m};
    const uint64_t fp = fingerprint(out_idx, out_col, m) ^ (in_idx ? 0x9E3779B97F4A7C15ull * fingerprint(*in_idx, in_col, m) : 0);
    std::lock_guard<std::mutex> lk(mu_);
    auto it = map_.find(k);
    if (it != map_.end()) {
      if (it->second.fp == fp && !strict_) return it->second.h;
      nwg_graph_release(it->second.h);  // contents changed in place: upload again
      map_.erase(it);
    }
    nwg_graph h = nullptr;
    if constexpr (std::is_same_v<Idx, uint64_t>) {
      check(nwg_graph_register(out_idx.data(), out_col, n, in_idx ? in_idx->data() : nullptr, in_col, 0, &h));
    } else {
      check(nwg_graph_register_u32off(out_idx.data(), out_col, n, in_idx ? in_idx->data() : nullptr, in_col, 0, &h));
    }
    map_[k] = entry{h, fp};
    return h;
  }

  // Frees every resident graph registered with these offsets as out- or in-graph.
  void release(const void* idx_data) {
    std::lock_guard<std::mutex> lk(mu_);
    for (auto it = map_.begin(); it != map_.end();) {
      if (it->first.out_idx == idx_data || it->first.in_idx == idx_data) {
        nwg_graph_release(it->second.h);
        it = map_.erase(it);
      } else {
        ++it;
      }
    }
  }

  void release_all() {
    std::lock_guard<std::mutex> lk(mu_);
    for (auto& kv : map_) nwg_graph_release(kv.second.h);
    map_.clear();
  }

 private:
  struct entry {
    nwg_graph h;
    uint64_t  fp;
  };

  // 64 evenly spaced offsets and columns (plus the sizes), mixed.
  template <class Idx>
  static uint64_t fingerprint(const std::vector<Idx>& idx, const uint32_t* col, uint64_t m) {
    uint64_t       h = 0xCBF29CE484222325ull ^ idx.size() ^ (m << 1);
    const uint64_t n = idx.size();
    for (uint64_t s = 0; s < 64 && n; ++s) {
      const uint64_t i = (s * (n - 1)) / 63;
      h                = (h ^ (uint64_t)idx[i]) * 0x100000001B3ull;
    }
    for (uint64_t s = 0; s < 64 && m; ++s) {
      const uint64_t e = (s * (m - 1)) / 63;
      h                = (h ^ (uint64_t)col[e]) * 0x100000001B3ull;
    }
    return h;
  }

  static bool strict_from_env() {
    const char* v = std::getenv("NWG_DROPIN_STRICT");
    return v != nullptr && v[0] != '\0' && std::strcmp(v, "0") != 0;
  }

  std::mutex             mu_;
  std::map<key, entry>   map_;
  const bool             strict_ = strict_from_env();  // upload on every call
};

template <class G>
const uint32_t* columns(const G& g) {
  using col_t = std::decay_t<decltype(std::get<0>(g.to_be_indexed_))>;
  static_assert(sizeof(typename col_t::value_type) == 4, "vertex ids must be 32-bit");
  return reinterpret_cast<const uint32_t*>(std::get<0>(g.to_be_indexed_).data());
}

template <class OutGraph, class InGraph>
nwg_graph resident(const OutGraph& out_graph, const InGraph& in_graph) {
  using Idx = typename std::decay_t<decltype(out_graph.indices_)>::value_type;
  const bool same =
      static_cast<const void*>(&out_graph) == static_cast<const void*>(&in_graph) ||
      (static_cast<const void*>(out_graph.indices_.data()) == static_cast<const void*>(in_graph.indices_.data()));
  if (same) return registry::get().acquire<Idx>(out_graph.indices_, columns(out_graph), nullptr, nullptr);
  static_assert(std::is_same_v<Idx, typename std::decay_t<decltype(in_graph.indices_)>::value_type>,
                "out- and in-graph must use the same offset type");
  return registry::get().acquire<Idx>(out_graph.indices_, columns(out_graph), &in_graph.indices_, columns(in_graph));
}

// Frees the device copy of a graph (call after mutating or before destroying it).
template <class G>
void release(const G& g) {
  registry::get().release(g.indices_.data());
}

inline void release_all() { registry::get().release_all(); }

}  // namespace b200

// BFSVerifier: same rules and messages as the reference (bfs.hpp:44-98),
// written for this header.
template <adjacency_list_graph Graph, adjacency_list_graph GraphT>
bool BFSVerifier(const Graph& g, GraphT& g_t, vertex_id_t<Graph> source, std::vector<vertex_id_t<Graph>>& parent) {
  using vid             = vertex_id_t<Graph>;
  constexpr vid   none  = std::numeric_limits<vid>::max();
  const std::size_t N   = num_vertices(g);
  std::vector<vid>  depth(N, none);
  std::vector<vid>  order;
  order.reserve(N);
  depth[source] = 0;
  order.push_back(source);
  for (std::size_t head = 0; head < order.size(); ++head) {
    const vid u = order[head];
    for (auto&& e : g[u]) {
      const vid v = target(g, e);
      if (depth[v] == none) {
        depth[v] = depth[u] + 1;
        order.push_back(v);
      }
    }
  }
  for (vid u = 0; u < N; ++u) {
    if (depth[u] != none && parent[u] != none) {
      if (u == source) {
        if (!(parent[u] == u && depth[u] == 0)) {
          std::cout << "Source wrong " << u << " " << parent[u] << " " << depth[u] << std::endl;
          return false;
        }
        continue;
      }
      bool found = false;
      for (auto&& e : g_t[u]) {
        const vid v = target(g_t, e);
        if (v == parent[u]) {
          if (depth[v] != depth[u] - 1) {
            std::cout << "Wrong depths for " << u << " & " << v << std::endl;
            return false;
          }
          found = true;
          break;
        }
      }
      if (!found) {
        std::cout << "Couldn't find edge from " << parent[u] << " to " << u << std::endl;
        return false;
      }
    } else if (depth[u] != parent[u]) {
      std::cout << "Reachability mismatch " << u << " " << depth[u] << " " << parent[u] << std::endl;
      return false;
    }
  }
  return true;
}

// Top-down BFS from root over out-edges (reference: bfs.hpp:110-140).
template <adjacency_list_graph Graph>
auto bfs(const Graph& graph, vertex_id_t<Graph> root) {
  using vid = vertex_id_t<Graph>;
  static_assert(sizeof(vid) == 4, "vertex ids must be 32-bit");
  std::vector<vid> parents(num_vertices(graph));
  nwg_graph        h = b200::resident(graph, graph);
  b200::check(nwg_bfs_topdown(h, (uint32_t)root, reinterpret_cast<uint32_t*>(parents.data()), nullptr, nullptr));
  return parents;
}

// Direction-optimizing BFS (reference: bfs.hpp:160-311).
template <adjacency_list_graph OutGraph, adjacency_list_graph InGraph>
[[gnu::noinline]] auto bfs(const OutGraph& out_graph, const InGraph& in_graph, vertex_id_t<OutGraph> root,
                           int num_bins = 32, int alpha = 15, int beta = 18) {
  using vid = vertex_id_t<OutGraph>;
  static_assert(sizeof(vid) == 4, "vertex ids must be 32-bit");
  (void)num_bins;
  std::vector<vid> parents(num_vertices(out_graph));
  nwg_graph        h = b200::resident(out_graph, in_graph);
  b200::check(nwg_bfs(h, (uint32_t)root, alpha, beta, reinterpret_cast<uint32_t*>(parents.data()), nullptr, nullptr));
  return parents;
}

}  // namespace graph
}  // namespace nw

#endif  // NW_GRAPH_BFS_HPP
