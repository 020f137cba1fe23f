// Device BFSVerifier: the checks of nw::graph::BFSVerifier(g, g_t, source,
// parent) (include/nwgraph/algorithms/bfs.hpp:44-98 in NWGraph) on the GPU.
//
//   1. depth = BFS depths from the source over the out-graph (bfs.hpp:47-63).
//      Computed by a plain level-synchronous top-down BFS written only for
//      this check (a warp per frontier vertex, atomicCAS on depth): it shares
//      no code with the direction-optimizing kernels it is used to verify.
//   2. For every vertex u (bfs.hpp:64-96): when depth[u] and parent[u] are
//      both set, the source must be its own parent at depth 0, and any other
//      u must find parent[u] among its in-neighbours (g_t) with
//      depth[parent[u]] == depth[u] - 1; otherwise depth[u] must equal
//      parent[u] (both unset).
//
// The reference stops at the first failing vertex in vertex order; here
// every vertex is checked in parallel and the lowest failing one is kept
// (a 64-bit atomicMin on vertex << 3 | reason), so the verdict, the vertex
// and the reason are the ones the reference reports.
#include <algorithm>
#include <string>

#include "nwg_internal.cuh"

using namespace nwg;

#define NWG_API extern "C" __attribute__((visibility("default")))

namespace {

constexpr int      kVThreads = 256;
constexpr uint32_t kUnset    = 0xFFFFFFFFu;  // std::numeric_limits<uint32_t>::max()

struct VerifyCounters {
  unsigned long long next;     // vertices appended to the next frontier
  unsigned long long first;    // min over failing vertices of (u << 3 | reason)
  unsigned long long reached;  // vertices with a depth
};

__global__ void k_v_init(uint32_t* depth, uint64_t n, uint32_t source, uint32_t* q0, VerifyCounters* cnt) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    depth[i] = (i == source) ? 0u : kUnset;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    q0[0]        = source;
    cnt->next    = 0;
    cnt->first   = ~0ull;
    cnt->reached = 0;
  }
}

// One level: every out-edge of the frontier claims unvisited targets.
__global__ void __launch_bounds__(kVThreads) k_v_level(const uint64_t* __restrict__ off,
                                                       const uint32_t* __restrict__ col, uint32_t* depth,
                                                       const uint32_t* __restrict__ q, uint64_t qsize, uint32_t* qn,
                                                       uint64_t qcap, uint32_t level, VerifyCounters* cnt) {
  const unsigned lane   = threadIdx.x & 31;
  const uint64_t gwarp  = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = gwarp; i < qsize; i += nwarps) {
    const uint32_t u   = q[i];
    const uint64_t beg = off[u], end = off[u + 1];
    for (uint64_t e0 = beg; e0 < end; e0 += 32) {
      const uint64_t e   = e0 + lane;
      bool           won = false;
      uint32_t       v   = 0;
      if (e < end) {
        v   = col[e];
        won = depth[v] == kUnset && atomicCAS(&depth[v], kUnset, level + 1) == kUnset;
      }
      const unsigned m = __ballot_sync(kFullMask, won);
      if (m) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&cnt->next, (unsigned long long)__popc(m));
        base = __shfl_sync(kFullMask, base, 0);
        if (won) {
          const uint64_t at = base + __popc(m & ((1u << lane) - 1u));
          if (at < qcap) qn[at] = v;
        }
      }
    }
  }
}

// The per-vertex checks.  Lanes take consecutive vertices and scan up to 32
// in-neighbours alone; longer in-lists are scanned by the whole warp.
__global__ void __launch_bounds__(kVThreads) k_v_check(const uint64_t* __restrict__ in_off,
                                                       const uint32_t* __restrict__ in_col,
                                                       const uint32_t* __restrict__ depth,
                                                       const uint32_t* __restrict__ parent, uint64_t n,
                                                       uint32_t source, VerifyCounters* cnt) {
  const unsigned     lane   = threadIdx.x & 31;
  const uint64_t     stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t     n_up   = (n + 31) & ~31ull;
  unsigned long long reached = 0;
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n_up; u += stride) {
    const bool     valid = u < n;
    const uint32_t du    = valid ? depth[u] : kUnset;
    const uint32_t pu    = valid ? parent[u] : kUnset;
    uint32_t       fail  = 0;  // reason: 1 source wrong, 2 wrong depths, 3 no edge from the parent, 4 reachability
    bool           need  = false;  // parent search still open
    uint64_t       e = 0, end = 0;
    if (valid) {
      if (du != kUnset) ++reached;
      if (du != kUnset && pu != kUnset) {
        if (u == source) {
          if (!(pu == u && du == 0)) fail = 1;
        } else {
          e    = in_off[u];
          end  = in_off[u + 1];
          need = true;
        }
      } else if (du != pu) {
        fail = 4;
      }
    }
    // lane scan of the first 32 in-neighbours
    bool found = false;
    if (need) {
      const uint64_t lim = min(end, e + 32);
      for (; e < lim; ++e)
        if (in_col[e] == pu) {
          found = true;
          break;
        }
      if (found) need = false;
    }
    // the rest of long in-lists: the warp scans them together
    unsigned pend = __ballot_sync(kFullMask, need && e < end);
    while (pend) {
      const int      ld = __ffs(pend) - 1;
      pend &= pend - 1;
      const uint64_t b  = __shfl_sync(kFullMask, e, ld);
      const uint64_t en = __shfl_sync(kFullMask, end, ld);
      const uint32_t pp = __shfl_sync(kFullMask, pu, ld);
      bool           hit = false;
      for (uint64_t base = b; base < en && !hit; base += 32) {
        const uint64_t i = base + lane;
        hit              = __any_sync(kFullMask, i < en && in_col[i] == pp);
      }
      if ((int)lane == ld) found = hit;
    }
    if (valid && du != kUnset && pu != kUnset && u != source) {
      if (!found) fail = 3;
      else if (du == 0 || depth[pu] != du - 1) fail = 2;  // the parent's depth (bfs.hpp:79)
    }
    if (fail) atomicMin(&cnt->first, ((unsigned long long)u << 3) | fail);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) reached += __shfl_xor_sync(kFullMask, reached, o);
  if (lane == 0 && reached) atomicAdd(&cnt->reached, reached);
}

int grid_v(const GraphDev* g, uint64_t items, uint64_t per_block) {
  const uint64_t want = (items + per_block - 1) / per_block;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)g->sm_count * 8, want));
}

struct VerifyBuffers {
  uint32_t*       depth = nullptr;
  uint32_t*       q[2]  = {nullptr, nullptr};
  uint32_t*       par   = nullptr;  // device copy of host parents
  VerifyCounters* cnt   = nullptr;
  cudaStream_t    s     = nullptr;
  cudaEvent_t     ev0 = nullptr, ev1 = nullptr;
  ~VerifyBuffers() {
    if (s) cudaStreamSynchronize(s);
    cudaFree(depth);
    cudaFree(q[0]);
    cudaFree(q[1]);
    cudaFree(par);
    cudaFree(cnt);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (s) cudaStreamDestroy(s);
  }
};

int verify(GraphDev* g, uint32_t source, const uint32_t* parents_host, const uint32_t* parents_dev,
           nwg_verify_result* out) {
  const uint64_t n = g->n;
  VerifyBuffers  b;
  if (cudaMalloc(&b.depth, std::max<uint64_t>(n, 1) * 4) != cudaSuccess ||
      cudaMalloc(&b.q[0], std::max<uint64_t>(n, 1) * 4) != cudaSuccess ||
      cudaMalloc(&b.q[1], std::max<uint64_t>(n, 1) * 4) != cudaSuccess ||
      cudaMalloc(&b.cnt, sizeof(VerifyCounters)) != cudaSuccess ||
      (parents_host && cudaMalloc(&b.par, std::max<uint64_t>(n, 1) * 4) != cudaSuccess)) {
    cudaGetLastError();
    return set_error(NWG_ENOMEM, "verifier allocation failed (n=" + std::to_string(n) + ")");
  }
  NWG_CUDA_TRY(cudaStreamCreateWithFlags(&b.s, cudaStreamNonBlocking));
  NWG_CUDA_TRY(cudaEventCreate(&b.ev0));
  NWG_CUDA_TRY(cudaEventCreate(&b.ev1));
  NWG_CUDA_TRY(cudaEventRecord(b.ev0, b.s));
  const uint32_t* par = parents_dev;
  if (parents_host) {
    NWG_CUDA_TRY(cudaMemcpyAsync(b.par, parents_host, n * 4, cudaMemcpyHostToDevice, b.s));
    par = b.par;
  }
  k_v_init<<<grid_v(g, n, kVThreads), kVThreads, 0, b.s>>>(b.depth, n, source, b.q[0], b.cnt);
  NWG_CUDA_TRY(cudaGetLastError());
  uint64_t qsize = 1;
  uint32_t level = 0;
  unsigned long long next = 0;
  while (qsize) {
    NWG_CUDA_TRY(cudaMemsetAsync(&b.cnt->next, 0, sizeof(unsigned long long), b.s));
    k_v_level<<<grid_v(g, qsize, kVThreads / 32), kVThreads, 0, b.s>>>(g->off, g->col, b.depth, b.q[level & 1],
                                                                        qsize, b.q[(level + 1) & 1], n, level, b.cnt);
    NWG_CUDA_TRY(cudaGetLastError());
    NWG_CUDA_TRY(cudaMemcpyAsync(&next, &b.cnt->next, sizeof next, cudaMemcpyDeviceToHost, b.s));
    NWG_CUDA_TRY(cudaStreamSynchronize(b.s));
    qsize = std::min<uint64_t>(next, n);
    ++level;
  }
  k_v_check<<<grid_v(g, n, kVThreads), kVThreads, 0, b.s>>>(g->in_off, g->in_col, b.depth, par, n, source, b.cnt);
  NWG_CUDA_TRY(cudaGetLastError());
  NWG_CUDA_TRY(cudaEventRecord(b.ev1, b.s));
  VerifyCounters hc;
  NWG_CUDA_TRY(cudaMemcpyAsync(&hc, b.cnt, sizeof hc, cudaMemcpyDeviceToHost, b.s));
  NWG_CUDA_TRY(cudaStreamSynchronize(b.s));
  nwg_verify_result r = {};
  r.valid             = hc.first == ~0ull ? 1 : 0;
  r.reason            = r.valid ? 0u : (uint32_t)(hc.first & 7u);
  r.first_bad         = r.valid ? ~0ull : (hc.first >> 3);
  r.reached           = hc.reached;
  r.levels            = level;
  cudaEventElapsedTime(&r.device_ms, b.ev0, b.ev1);
  *out = r;
  return NWG_OK;
}

}  // namespace

NWG_API int nwg_verify(nwg_graph h, uint32_t source, const uint32_t* parents_host, const uint32_t* parents_dev,
                       nwg_verify_result* result) {
  try {
    if (!h || !result || (!parents_host == !parents_dev))
      return set_error(NWG_EINVAL, "NULL graph or result, or not exactly one of parents_host / parents_dev");
    auto* g = reinterpret_cast<GraphDev*>(h);
    if (source >= g->n) return set_error(NWG_EINVAL, "source " + std::to_string(source) + " >= n");
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != g->device) cudaSetDevice(g->device);
    const int rc = verify(g, source, parents_host, parents_dev, result);
    if (prev != g->device) cudaSetDevice(prev);
    return rc;
  } catch (const std::exception& ex) {
    return set_error(NWG_ENOMEM, std::string("verifier failed: ") + ex.what());
  }
}
