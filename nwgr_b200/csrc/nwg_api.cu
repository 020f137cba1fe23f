// The extern "C" boundary of libnwgr_b200.so (declared in include/nwg_bfs.h):
// graph registration (upload once), workspaces, the synchronous and
// stream-ordered BFS entry points, and per-thread error messages.  No C++
// exception crosses this file's functions.
#include <algorithm>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "nwg_internal.cuh"

namespace nwg {

namespace {
thread_local std::string g_last_error;

// Makes `dev` current for the lifetime of the guard.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int validate_csr(const uint64_t* off, const uint32_t* col, uint64_t n, const char* which) {
  if (off[0] != 0) return set_error(NWG_EINVAL, std::string(which) + ": offsets[0] != 0");
  for (uint64_t i = 0; i < n; ++i)
    if (off[i + 1] < off[i])
      return set_error(NWG_EINVAL, std::string(which) + ": offsets not monotone at row " + std::to_string(i));
  const uint64_t m = off[n];
  for (uint64_t e = 0; e < m; ++e)
    if (col[e] >= n)
      return set_error(NWG_EINVAL, std::string(which) + ": column id " + std::to_string(col[e]) + " >= n at entry " +
                                       std::to_string(e));
  return NWG_OK;
}

// The in-CSR must be the transpose of the out-CSR (the contract of the
// reference's bfs(out_graph, in_graph, ...)): for every v, in[v] holds, as a
// multiset, exactly the u with v in out[u].  Checked by a counting sort of
// the out-edges by target and a row-by-row comparison of sorted rows; O(n + m)
// host memory.  Both CSRs have passed validate_csr.
template <typename OffT>
int validate_transpose(const OffT* out_off, const uint32_t* out_col, const OffT* in_off, const uint32_t* in_col,
                       uint64_t n) {
  const uint64_t        m = out_off[n];
  std::vector<uint64_t> start(n + 1, 0);
  for (uint64_t e = 0; e < m; ++e) start[out_col[e] + 1]++;
  for (uint64_t v = 0; v < n; ++v) start[v + 1] += start[v];
  for (uint64_t v = 0; v < n; ++v)
    if (start[v + 1] - start[v] != (uint64_t)(in_off[v + 1] - in_off[v]))
      return set_error(NWG_EINVAL, "in-graph is not the transpose of the out-graph: vertex " + std::to_string(v) +
                                       " has " + std::to_string(in_off[v + 1] - in_off[v]) + " in-edges listed, " +
                                       std::to_string(start[v + 1] - start[v]) + " out-edges pointing to it");
  std::vector<uint32_t> t(m);
  std::vector<uint64_t> pos(start.begin(), start.end() - 1);
  for (uint64_t u = 0; u < n; ++u)
    for (uint64_t e = out_off[u]; e < (uint64_t)out_off[u + 1]; ++e) t[pos[out_col[e]]++] = (uint32_t)u;
  std::vector<uint32_t> row;
  for (uint64_t v = 0; v < n; ++v) {  // t's rows are sorted already (sources visited in order)
    row.assign(in_col + in_off[v], in_col + in_off[v + 1]);
    std::sort(row.begin(), row.end());
    if (!std::equal(row.begin(), row.end(), t.begin() + start[v]))
      return set_error(NWG_EINVAL, "in-graph is not the transpose of the out-graph: in-edges of vertex " +
                                       std::to_string(v) + " differ");
  }
  return NWG_OK;
}

int validate_csr32(const uint32_t* off, const uint32_t* col, uint64_t n, const char* which) {
  if (off[0] != 0) return set_error(NWG_EINVAL, std::string(which) + ": offsets[0] != 0");
  for (uint64_t i = 0; i < n; ++i)
    if (off[i + 1] < off[i])
      return set_error(NWG_EINVAL, std::string(which) + ": offsets not monotone at row " + std::to_string(i));
  const uint64_t m = off[n];
  for (uint64_t e = 0; e < m; ++e)
    if (col[e] >= n)
      return set_error(NWG_EINVAL, std::string(which) + ": column id " + std::to_string(col[e]) + " >= n at entry " +
                                       std::to_string(e));
  return NWG_OK;
}

template <typename T>
int dev_alloc(T** p, uint64_t count) {
  if (cudaMalloc(reinterpret_cast<void**>(p), std::max<uint64_t>(count, 4) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(NWG_ENOMEM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
  }
  return NWG_OK;
}

void graph_free(GraphDev* g) {
  if (!g) return;
  DeviceGuard dg(g->device);
  for (Workspace* ws : g->workspaces) ws_free(ws);
  g->workspaces.clear();
  for (MsWorkspace* ws : g->ms_workspaces) ms_ws_free(ws);
  g->ms_workspaces.clear();
  g->default_ws = nullptr;
  g->pipe_ws    = nullptr;
  if (g->owns_out) {
    cudaFree(g->off);
    cudaFree(g->col);
  }
  if (g->owns_in) {
    cudaFree(g->in_off);
    cudaFree(g->in_col);
  }
  cudaFree(g->Z);
  cudaFree(g->deg16);
  delete g;
}

// Shared tail of both registration entry points: device-side offsets are in
// place; build the in-degree-zero bitmap and the saturated out-degrees and
// query the SM count.
int finish_register(GraphDev* g) {
  cudaDeviceProp prop;
  NWG_CUDA_TRY(cudaGetDeviceProperties(&prop, g->device));
  g->sm_count = prop.multiProcessorCount;
  int rc      = build_zero_indegree(g, nullptr);
  if (rc) return rc;
  rc = build_deg16(g, nullptr);
  if (rc) return rc;
  NWG_CUDA_TRY(cudaDeviceSynchronize());
  return NWG_OK;
}

template <typename OffT>
int register_impl(const OffT* out_off, const uint32_t* out_col, uint64_t n, const OffT* in_off,
                  const uint32_t* in_col, uint32_t flags, nwg_graph* out) {
  if (!out) return set_error(NWG_EINVAL, "out handle pointer is NULL");
  *out = nullptr;
  if (!out_off || (!out_col && n > 0)) return set_error(NWG_EINVAL, "out-graph arrays are NULL");
  if (n >= 0xFFFFFFFFull) return set_error(NWG_EINVAL, "n must be below 2^32 - 1 (uint32 vertex ids)");
  if ((in_off == nullptr) != (in_col == nullptr)) return set_error(NWG_EINVAL, "in_off and in_col must both be set or both be NULL");
  const bool device = flags & NWG_REG_DEVICE;
  auto*      g      = new (std::nothrow) GraphDev();
  if (!g) return set_error(NWG_ENOMEM, "host allocation failed");
  cudaGetDevice(&g->device);
  g->n         = n;
  g->symmetric = (in_off == nullptr) || (in_off == out_off && in_col == out_col);

  auto fail = [&](int rc) {
    graph_free(g);
    return rc;
  };

  // m and in_m
  OffT m_last = 0, in_last = 0;
  if (device) {
    if (cudaMemcpy(&m_last, out_off + n, sizeof(OffT), cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(cuda_error(cudaGetLastError(), "read out_off[n]"));
    if (!g->symmetric && cudaMemcpy(&in_last, in_off + n, sizeof(OffT), cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(cuda_error(cudaGetLastError(), "read in_off[n]"));
  } else {
    if (flags & NWG_REG_VALIDATE) {
      int rc = sizeof(OffT) == 8 ? validate_csr((const uint64_t*)out_off, out_col, n, "out-graph")
                                 : validate_csr32((const uint32_t*)out_off, out_col, n, "out-graph");
      if (rc) return fail(rc);
      if (!g->symmetric) {
        rc = sizeof(OffT) == 8 ? validate_csr((const uint64_t*)in_off, in_col, n, "in-graph")
                               : validate_csr32((const uint32_t*)in_off, in_col, n, "in-graph");
        if (!rc) rc = validate_transpose(out_off, out_col, in_off, in_col, n);
        if (rc) return fail(rc);
      }
    }
    m_last  = out_off[n];
    in_last = g->symmetric ? m_last : in_off[n];
  }
  g->m    = m_last;
  g->in_m = g->symmetric ? g->m : (uint64_t)in_last;
  if (!g->symmetric && g->in_m != g->m)
    return fail(set_error(NWG_EINVAL, "in-graph entry count differs from out-graph (not a transpose)"));

  // out-graph.  Borrowed device columns must be 16-byte aligned (the
  // top-down step reads them with 128-bit loads); otherwise they are copied.
  const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const bool col_aligned    = (reinterpret_cast<uintptr_t>(out_col) & 15) == 0;
  if (device && sizeof(OffT) == 8 && col_aligned) {
    g->off = (uint64_t*)out_off;
    g->col = (uint32_t*)out_col;
  } else {
    g->owns_out = true;
    int rc      = dev_alloc(&g->off, n + 1);
    if (!rc) rc = dev_alloc(&g->col, g->m);
    if (rc) return fail(rc);
    if (sizeof(OffT) == 8) {
      if (cudaMemcpy(g->off, out_off, (n + 1) * 8, kind) != cudaSuccess) return fail(cuda_error(cudaGetLastError(), "upload offsets"));
    } else {
      uint32_t* tmp = nullptr;
      if ((rc = dev_alloc(&tmp, n + 1))) return fail(rc);
      if (cudaMemcpy(tmp, out_off, (n + 1) * 4, kind) != cudaSuccess) {
        cudaFree(tmp);
        return fail(cuda_error(cudaGetLastError(), "upload offsets"));
      }
      rc = widen_offsets(tmp, g->off, n + 1, nullptr);
      cudaDeviceSynchronize();
      cudaFree(tmp);
      if (rc) return fail(rc);
    }
    if (g->m && cudaMemcpy(g->col, out_col, g->m * 4, kind) != cudaSuccess)
      return fail(cuda_error(cudaGetLastError(), "upload columns"));
  }
  // in-graph
  if (g->symmetric) {
    g->in_off = g->off;
    g->in_col = g->col;
  } else if (device && sizeof(OffT) == 8) {
    g->in_off = (uint64_t*)in_off;
    g->in_col = (uint32_t*)in_col;
  } else {
    g->owns_in = true;
    int rc     = dev_alloc(&g->in_off, n + 1);
    if (!rc) rc = dev_alloc(&g->in_col, g->in_m);
    if (rc) return fail(rc);
    if (sizeof(OffT) == 8) {
      if (cudaMemcpy(g->in_off, in_off, (n + 1) * 8, kind) != cudaSuccess) return fail(cuda_error(cudaGetLastError(), "upload in-offsets"));
    } else {
      uint32_t* tmp = nullptr;
      if ((rc = dev_alloc(&tmp, n + 1))) return fail(rc);
      if (cudaMemcpy(tmp, in_off, (n + 1) * 4, kind) != cudaSuccess) {
        cudaFree(tmp);
        return fail(cuda_error(cudaGetLastError(), "upload in-offsets"));
      }
      rc = widen_offsets(tmp, g->in_off, n + 1, nullptr);
      cudaDeviceSynchronize();
      cudaFree(tmp);
      if (rc) return fail(rc);
    }
    if (g->in_m && cudaMemcpy(g->in_col, in_col, g->in_m * 4, kind) != cudaSuccess)
      return fail(cuda_error(cudaGetLastError(), "upload in-columns"));
  }
  int rc = finish_register(g);
  if (rc) return fail(rc);
  *out = reinterpret_cast<nwg_graph>(g);
  return NWG_OK;
}

// Creates *slot on first use (a workspace kept with the graph) and returns it.
int get_owned_ws(GraphDev* g, Workspace** slot, Workspace** out) {
  if (!*slot) {
    auto* ws = new (std::nothrow) Workspace();
    if (!ws) return set_error(NWG_ENOMEM, "host allocation failed");
    int rc = ws_init(g, ws);
    if (rc) {
      ws_free(ws);
      return rc;
    }
    g->workspaces.push_back(ws);
    *slot = ws;
  }
  *out = *slot;
  return NWG_OK;
}

int get_default_ws(GraphDev* g, Workspace** out) { return get_owned_ws(g, &g->default_ws, out); }

int bfs_sync(GraphDev* g, uint32_t root, int alpha, int beta, uint32_t* parents_host, uint32_t* parents_dev,
             nwg_bfs_stats* stats, bool topdown_only) {
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard                 dg(g->device);
  Workspace*                  ws = nullptr;
  int                         rc = get_default_ws(g, &ws);
  if (rc) return rc;
  uint32_t* dst = parents_dev ? parents_dev : ws->parents;
  NWG_CUDA_TRY(cudaEventRecord(ws->ev0, ws->stream));
  rc = ws_launch(ws, root, alpha, beta, dst, ws->stream, topdown_only);
  if (rc) return rc;
  NWG_CUDA_TRY(cudaEventRecord(ws->ev1, ws->stream));
  if (parents_host)
    NWG_CUDA_TRY(cudaMemcpyAsync(parents_host, dst, g->n * sizeof(uint32_t), cudaMemcpyDeviceToHost, ws->stream));
  const size_t ctrl_bytes = stats ? sizeof(Ctrl) : sizeof(CtrlHdr);
  NWG_CUDA_TRY(cudaMemcpyAsync(ws->ctrl_host, ws->ctrl, ctrl_bytes, cudaMemcpyDeviceToHost, ws->stream));
  NWG_CUDA_TRY(cudaStreamSynchronize(ws->stream));
  const Ctrl& c = *ws->ctrl_host;
  if (stats) {
    fill_stats(c, stats);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ws->ev0, ws->ev1);
    stats->device_ms = ms;
  }
  if (c.h.status != 0) return set_error(c.h.status, "device traversal reported status " + std::to_string(c.h.status));
  return NWG_OK;
}

// k traversals with their parents copied to host rows, two in flight: the
// graph's default workspace and a second one take the roots in turn, each on
// its own stream, so the device-to-host copy of root i's parents runs while
// root i + 1 traverses (the traversals themselves run one after another:
// cooperative launches of a device are chained).  Before a workspace takes
// root i + 2 the host waits for its root i and reads that root's status, so
// the parents buffer and the status mirror are never overwritten in flight.
// All roots are checked before anything is launched.
int bfs_roots(GraphDev* g, const uint32_t* roots, uint64_t k, int alpha, int beta, uint32_t* parents_host,
              int32_t* status) {
  for (uint64_t i = 0; i < k; ++i)
    if (roots[i] >= g->n)
      return set_error(NWG_EINVAL, "roots[" + std::to_string(i) + "] = " + std::to_string(roots[i]) + " >= n " +
                                       std::to_string(g->n));
  if (alpha <= 0 || beta <= 0) return set_error(NWG_EINVAL, "alpha and beta must be positive");
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard                 dg(g->device);
  Workspace*                  w[2] = {nullptr, nullptr};
  int                         rc   = get_default_ws(g, &w[0]);
  if (rc) return rc;
  rc = get_owned_ws(g, &g->pipe_ws, &w[1]);
  if (rc) return rc;
  const size_t row       = g->n * sizeof(uint32_t);
  bool         busy[2]   = {false, false};
  uint64_t     which[2]  = {0, 0};
  int          first_bad = NWG_OK;
  std::string  first_msg;
  auto retire = [&](int s) -> int {  // waits for lane s's root and records its status
    if (!busy[s]) return NWG_OK;
    busy[s] = false;
    NWG_CUDA_TRY(cudaStreamSynchronize(w[s]->stream));
    const int st = w[s]->ctrl_host->h.status;
    if (status) status[which[s]] = st;
    if (st != 0 && first_bad == NWG_OK) {
      first_bad = st;
      first_msg = "root index " + std::to_string(which[s]) + ": device traversal reported status " + std::to_string(st);
    }
    return NWG_OK;
  };
  for (uint64_t i = 0; i < k; ++i) {
    const int s = (int)(i & 1);
    rc = retire(s);
    if (rc == NWG_OK) rc = ws_launch(w[s], roots[i], alpha, beta, w[s]->parents, w[s]->stream, false);
    if (rc == NWG_OK) {
      const cudaError_t e1 =
          cudaMemcpyAsync(parents_host + i * g->n, w[s]->parents, row, cudaMemcpyDeviceToHost, w[s]->stream);
      const cudaError_t e2 = e1 != cudaSuccess
                                 ? e1
                                 : cudaMemcpyAsync(w[s]->ctrl_host, w[s]->ctrl, sizeof(CtrlHdr),
                                                   cudaMemcpyDeviceToHost, w[s]->stream);
      if (e2 != cudaSuccess) rc = cuda_error(e2, "cudaMemcpyAsync(parents row / status)");
    }
    if (rc != NWG_OK) {  // the other lane's root still completes before the error returns
      const std::string msg = g_last_error;
      retire(s ^ 1);
      if (status) status[i] = rc;
      return set_error(rc, msg);
    }
    busy[s]  = true;
    which[s] = i;
  }
  rc = retire(k & 1);  // the older of the two in flight first
  if (rc == NWG_OK) rc = retire((k + 1) & 1);
  if (rc) return rc;
  if (first_bad != NWG_OK) return set_error(first_bad, first_msg);
  return NWG_OK;
}

}  // namespace

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_error(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return e == cudaErrorMemoryAllocation ? NWG_ENOMEM : NWG_ECUDA;
}

}  // namespace nwg

using namespace nwg;

#define NWG_API extern "C" __attribute__((visibility("default")))

#define NWG_GUARD_BEGIN try {
#define NWG_GUARD_END                                          \
  }                                                            \
  catch (const std::bad_alloc&) {                              \
    return set_error(NWG_ENOMEM, "host allocation failed");    \
  }                                                            \
  catch (const std::exception& ex) {                           \
    return set_error(NWG_ESTATE, ex.what());                   \
  }                                                            \
  catch (...) {                                                \
    return set_error(NWG_ESTATE, "unknown C++ exception");     \
  }

NWG_API const char* nwg_version(void) { return "nwgr_b200 0.1.0 (sm_100a)"; }

NWG_API int nwg_last_error(char* buf, size_t len) {
  if (buf && len) {
    size_t k = std::min(len - 1, g_last_error.size());
    std::memcpy(buf, g_last_error.data(), k);
    buf[k] = 0;
  }
  return (int)g_last_error.size();
}

NWG_API int nwg_graph_register(const uint64_t* out_off, const uint32_t* out_col, uint64_t n, const uint64_t* in_off,
                               const uint32_t* in_col, uint32_t flags, nwg_graph* out) {
  NWG_GUARD_BEGIN
  return register_impl<uint64_t>(out_off, out_col, n, in_off, in_col, flags, out);
  NWG_GUARD_END
}

NWG_API int nwg_graph_register_u32off(const uint32_t* out_off, const uint32_t* out_col, uint64_t n,
                                      const uint32_t* in_off, const uint32_t* in_col, uint32_t flags, nwg_graph* out) {
  NWG_GUARD_BEGIN
  return register_impl<uint32_t>(out_off, out_col, n, in_off, in_col, flags, out);
  NWG_GUARD_END
}

NWG_API int nwg_graph_release(nwg_graph h) {
  NWG_GUARD_BEGIN
  if (!h) return set_error(NWG_EINVAL, "NULL graph");
  graph_free(reinterpret_cast<GraphDev*>(h));
  return NWG_OK;
  NWG_GUARD_END
}

NWG_API int nwg_graph_info(nwg_graph h, uint64_t* n, uint64_t* m, uint64_t* in_m) {
  if (!h) return set_error(NWG_EINVAL, "NULL graph");
  auto* g = reinterpret_cast<GraphDev*>(h);
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (in_m) *in_m = g->in_m;
  return NWG_OK;
}

NWG_API int nwg_bfs(nwg_graph h, uint32_t root, int alpha, int beta, uint32_t* parents_host, uint32_t* parents_dev,
                    nwg_bfs_stats* stats) {
  NWG_GUARD_BEGIN
  if (!h) return set_error(NWG_EINVAL, "NULL graph");
  return bfs_sync(reinterpret_cast<GraphDev*>(h), root, alpha, beta, parents_host, parents_dev, stats, false);
  NWG_GUARD_END
}

NWG_API int nwg_bfs_roots(nwg_graph h, const uint32_t* roots, uint64_t k, int alpha, int beta, uint32_t* parents_host,
                          int32_t* status) {
  NWG_GUARD_BEGIN
  if (!h || (k && (!roots || !parents_host))) return set_error(NWG_EINVAL, "NULL argument");
  return bfs_roots(reinterpret_cast<GraphDev*>(h), roots, k, alpha, beta, parents_host, status);
  NWG_GUARD_END
}

NWG_API int nwg_bfs_topdown(nwg_graph h, uint32_t root, uint32_t* parents_host, uint32_t* parents_dev,
                            nwg_bfs_stats* stats) {
  NWG_GUARD_BEGIN
  if (!h) return set_error(NWG_EINVAL, "NULL graph");
  return bfs_sync(reinterpret_cast<GraphDev*>(h), root, 15, 18, parents_host, parents_dev, stats, true);
  NWG_GUARD_END
}

NWG_API int nwg_bfs_stepped(nwg_graph h, uint32_t root, int alpha, int beta, uint32_t* parents_dev,
                            nwg_bfs_stats* stats) {
  NWG_GUARD_BEGIN
  if (!h) return set_error(NWG_EINVAL, "NULL graph");
  auto*                       g = reinterpret_cast<GraphDev*>(h);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard                 dg(g->device);
  Workspace*                  ws = nullptr;
  int                         rc = get_default_ws(g, &ws);
  if (rc) return rc;
  NWG_CUDA_TRY(cudaEventRecord(ws->ev0, ws->stream));
  rc = ws_launch_stepped(ws, root, alpha, beta, parents_dev, ws->stream);
  if (rc) return rc;
  NWG_CUDA_TRY(cudaEventRecord(ws->ev1, ws->stream));
  NWG_CUDA_TRY(cudaMemcpyAsync(ws->ctrl_host, ws->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, ws->stream));
  NWG_CUDA_TRY(cudaStreamSynchronize(ws->stream));
  if (stats) {
    fill_stats(*ws->ctrl_host, stats);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ws->ev0, ws->ev1);
    stats->device_ms = ms;
  }
  const int st = ws->ctrl_host->h.status;
  if (st != 0) return set_error(st, "device traversal reported status " + std::to_string(st));
  return NWG_OK;
  NWG_GUARD_END
}

NWG_API int nwg_ws_create(nwg_graph h, nwg_bfs_ws* out) {
  NWG_GUARD_BEGIN
  if (!h || !out) return set_error(NWG_EINVAL, "NULL argument");
  auto*                       g = reinterpret_cast<GraphDev*>(h);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard                 dg(g->device);
  auto*                       ws = new Workspace();
  int                         rc = ws_init(g, ws);
  if (rc) {
    ws_free(ws);
    return rc;
  }
  g->workspaces.push_back(ws);
  *out = reinterpret_cast<nwg_bfs_ws>(ws);
  return NWG_OK;
  NWG_GUARD_END
}

NWG_API int nwg_ws_destroy(nwg_bfs_ws h) {
  NWG_GUARD_BEGIN
  if (!h) return set_error(NWG_EINVAL, "NULL workspace");
  auto*                       ws = reinterpret_cast<Workspace*>(h);
  GraphDev*                   g  = ws->g;
  std::lock_guard<std::mutex> lk(g->mu);
  g->workspaces.erase(std::remove(g->workspaces.begin(), g->workspaces.end(), ws), g->workspaces.end());
  if (g->default_ws == ws) g->default_ws = nullptr;
  ws_free(ws);
  return NWG_OK;
  NWG_GUARD_END
}

NWG_API int nwg_bfs_async(nwg_bfs_ws h, uint32_t root, int alpha, int beta, uint32_t* parents_dev, void* stream) {
  NWG_GUARD_BEGIN
  if (!h) return set_error(NWG_EINVAL, "NULL workspace");
  auto*       ws = reinterpret_cast<Workspace*>(h);
  DeviceGuard dg(ws->device);
  return ws_launch(ws, root, alpha, beta, parents_dev, reinterpret_cast<cudaStream_t>(stream), false);
  NWG_GUARD_END
}

NWG_API int nwg_ws_stats(nwg_bfs_ws h, nwg_bfs_stats* stats) {
  NWG_GUARD_BEGIN
  if (!h || !stats) return set_error(NWG_EINVAL, "NULL argument");
  auto* ws = reinterpret_cast<Workspace*>(h);
  if (!ws->ran) return set_error(NWG_ESTATE, "no traversal has run on this workspace");
  DeviceGuard dg(ws->device);
  NWG_CUDA_TRY(cudaMemcpy(ws->ctrl_host, ws->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
  fill_stats(*ws->ctrl_host, stats);
  stats->device_ms = 0.f;
  return NWG_OK;
  NWG_GUARD_END
}

NWG_API int nwg_msbfs_ws_create(nwg_graph h, nwg_msbfs_ws* out) {
  NWG_GUARD_BEGIN
  if (!h || !out) return set_error(NWG_EINVAL, "NULL argument");
  auto*                       g = reinterpret_cast<GraphDev*>(h);
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard                 dg(g->device);
  auto*                       ws = new MsWorkspace();
  int                         rc = ms_ws_init(g, ws);
  if (rc) {
    ms_ws_free(ws);
    return rc;
  }
  g->ms_workspaces.push_back(ws);
  *out = reinterpret_cast<nwg_msbfs_ws>(ws);
  return NWG_OK;
  NWG_GUARD_END
}

NWG_API int nwg_msbfs_ws_destroy(nwg_msbfs_ws h) {
  NWG_GUARD_BEGIN
  if (!h) return set_error(NWG_EINVAL, "NULL workspace");
  auto*                       ws = reinterpret_cast<MsWorkspace*>(h);
  GraphDev*                   g  = ws->g;
  std::lock_guard<std::mutex> lk(g->mu);
  DeviceGuard                 dg(g->device);
  g->ms_workspaces.erase(std::remove(g->ms_workspaces.begin(), g->ms_workspaces.end(), ws), g->ms_workspaces.end());
  ms_ws_free(ws);
  return NWG_OK;
  NWG_GUARD_END
}

namespace {
int msbfs_common(nwg_msbfs_ws h, const uint32_t* roots_host, uint32_t k, void* depths_dev, uint32_t depth_bytes,
                 uint8_t* deep_flags, int alpha, void* stream, nwg_msbfs_stats* stats) {
  if (!h || (!roots_host && k) || (!depths_dev && k)) return set_error(NWG_EINVAL, "NULL argument");
  auto*           ws = reinterpret_cast<MsWorkspace*>(h);
  DeviceGuard     dg(ws->g->device);
  nwg_msbfs_stats st = {};
  cudaStream_t    s  = stream ? reinterpret_cast<cudaStream_t>(stream) : ws->stream;
  NWG_CUDA_TRY(cudaEventRecord(ws->ev0, s));  // re-recorded by ms_run before its first device operation
  NWG_CUDA_TRY(cudaEventRecord(ws->ev1, s));  // re-recorded by ms_run at the end of the device work
  int rc = ms_run(ws, roots_host, k, depths_dev, depth_bytes, deep_flags, alpha, s, &st, ws->ev1, ws->ev0);
  NWG_CUDA_TRY(cudaEventSynchronize(ws->ev1));
  cudaEventElapsedTime(&st.device_ms, ws->ev0, ws->ev1);
  st.status = rc;
  if (stats) *stats = st;
  return rc;
}
}  // namespace

NWG_API int nwg_msbfs(nwg_msbfs_ws h, const uint32_t* roots_host, uint32_t k, uint8_t* depths_dev, int alpha,
                      void* stream, nwg_msbfs_stats* stats) {
  NWG_GUARD_BEGIN
  nwg_msbfs_stats st = {};
  int rc = msbfs_common(h, roots_host, k, depths_dev, 1, nullptr, alpha, stream, &st);
  if (rc == NWG_OK && st.deep_sources) {
    st.status = rc = set_error(NWG_EOVERFLOW, std::to_string(st.deep_sources) +
                                                  " source(s) reach depth 255 or more, beyond uint8: their rows hold "
                                                  "the depths up to 254 (255 beyond); every other row is exact");
  }
  if (stats) *stats = st;
  return rc;
  NWG_GUARD_END
}

NWG_API int nwg_msbfs_ex(nwg_msbfs_ws h, const uint32_t* roots_host, uint32_t k, void* depths_dev,
                         uint32_t depth_bytes, uint8_t* deep_flags_host, int alpha, void* stream,
                         nwg_msbfs_stats* stats) {
  NWG_GUARD_BEGIN
  return msbfs_common(h, roots_host, k, depths_dev, depth_bytes, deep_flags_host, alpha, stream, stats);
  NWG_GUARD_END
}

NWG_API int nwg_selftest_wait_timeout(uint32_t spins, int32_t* status, float* waited_ms) {
  NWG_GUARD_BEGIN
  if (!status || !waited_ms) return set_error(NWG_EINVAL, "NULL argument");
  if (spins == 0 || spins > (1u << 24)) return set_error(NWG_EINVAL, "spins must be 1..2^24");
  return wait_probe(spins, status, waited_ms);
  NWG_GUARD_END
}

NWG_API int nwg_component_edges(nwg_graph h, const uint32_t* parents_dev, uint64_t* edges, uint64_t* vertices) {
  NWG_GUARD_BEGIN
  if (!h || !parents_dev) return set_error(NWG_EINVAL, "NULL argument");
  auto*       g = reinterpret_cast<GraphDev*>(h);
  DeviceGuard dg(g->device);
  return component_edges(g, parents_dev, edges, vertices);
  NWG_GUARD_END
}

NWG_API int nwg_graph_copy_csr(nwg_graph h, uint64_t* out_off, uint32_t* out_col, uint64_t* in_off, uint32_t* in_col) {
  NWG_GUARD_BEGIN
  if (!h) return set_error(NWG_EINVAL, "NULL graph");
  auto*       g = reinterpret_cast<GraphDev*>(h);
  DeviceGuard dg(g->device);
  if (out_off) NWG_CUDA_TRY(cudaMemcpy(out_off, g->off, (g->n + 1) * 8, cudaMemcpyDeviceToHost));
  if (out_col && g->m) NWG_CUDA_TRY(cudaMemcpy(out_col, g->col, g->m * 4, cudaMemcpyDeviceToHost));
  if (in_off) NWG_CUDA_TRY(cudaMemcpy(in_off, g->in_off, (g->n + 1) * 8, cudaMemcpyDeviceToHost));
  if (in_col && g->in_m) NWG_CUDA_TRY(cudaMemcpy(in_col, g->in_col, g->in_m * 4, cudaMemcpyDeviceToHost));
  return NWG_OK;
  NWG_GUARD_END
}

namespace {
template <typename F>
int gen_common(nwg_graph* out, F&& build) {
  if (!out) return set_error(NWG_EINVAL, "out handle pointer is NULL");
  *out    = nullptr;
  auto* g = new (std::nothrow) GraphDev();
  if (!g) return set_error(NWG_ENOMEM, "host allocation failed");
  cudaGetDevice(&g->device);
  g->owns_out  = true;
  g->symmetric = true;
  int rc       = build(g);
  if (!rc) {
    g->in_off = g->off;
    g->in_col = g->col;
    g->in_m   = g->m;
    rc        = finish_register(g);
  }
  if (rc) {
    graph_free(g);
    return rc;
  }
  *out = reinterpret_cast<nwg_graph>(g);
  return NWG_OK;
}
}  // namespace

NWG_API int nwg_gen_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, uint32_t ta, uint32_t tab, uint32_t tabc,
                         nwg_graph* out) {
  NWG_GUARD_BEGIN
  if (scale == 0 || scale > 31 || edge_factor == 0) return set_error(NWG_EINVAL, "scale must be 1..31, edge_factor > 0");
  if (!(ta <= tab && tab <= tabc)) return set_error(NWG_EINVAL, "quadrant thresholds must be non-decreasing");
  return gen_common(out, [&](GraphDev* g) { return gen_rmat(scale, edge_factor, seed, ta, tab, tabc, g); });
  NWG_GUARD_END
}

NWG_API int nwg_gen_uniform(uint64_t n, uint32_t avg_degree, uint64_t seed, nwg_graph* out) {
  NWG_GUARD_BEGIN
  if (n < 2 || n >= 0xFFFFFFFFull) return set_error(NWG_EINVAL, "n must be in [2, 2^32 - 1)");
  return gen_common(out, [&](GraphDev* g) { return gen_uniform(n, avg_degree, seed, g); });
  NWG_GUARD_END
}

NWG_API int nwg_gen_grid(uint32_t width, uint32_t height, uint32_t shortcut_pct, uint64_t seed, nwg_graph* out) {
  NWG_GUARD_BEGIN
  if (width == 0 || height == 0 || (uint64_t)width * height >= 0xFFFFFFFFull)
    return set_error(NWG_EINVAL, "grid size must be positive and below 2^32 - 1 vertices");
  return gen_common(out, [&](GraphDev* g) { return gen_grid(width, height, shortcut_pct, seed, g); });
  NWG_GUARD_END
}

NWG_API int nwg_pick_roots(nwg_graph h, uint64_t seed, uint32_t count, uint32_t* roots_host) {
  NWG_GUARD_BEGIN
  if (!h || (!roots_host && count)) return set_error(NWG_EINVAL, "NULL argument");
  auto*       g = reinterpret_cast<GraphDev*>(h);
  DeviceGuard dg(g->device);
  return pick_roots(g, seed, count, roots_host);
  NWG_GUARD_END
}
