// Batched multi-source BFS: 64 sources per 64-bit word, up to 256 sources
// (four words, one 32-byte sector per vertex) per pass.  No reference
// counterpart: NWGraph's bfs is single-source; the oracle is one
// single-source BFS per root, depths compared bit for bit.
//
// State of a pass, vertex-major so one vertex's W words share a sector:
//   VIS[n][W]    sources that have reached the vertex
//   FR[2][n][W]  sources whose BFS has the vertex in its current / next frontier
//   NX[n][W]     top-down accumulator (atomicOr), cleared when consumed
//   depth[k][n]  uint8 output, 255 = unreached
// Each level is either
//   push: the vertices in the frontier list OR their frontier words into
//         NX of their out-neighbours (64-bit atomicOr, only the bits the
//         neighbour has not seen), then a finalize pass turns NX into the
//         next frontier;
//   pull: every vertex some source has not reached ORs the frontier words
//         of its in-neighbours, stopping as soon as every missing source is
//         found (no atomics);
// chosen like the single-source switch: pull when the frontier's out-edges
// exceed the unexplored edges / alpha (nw::graph::bfs, bfs.hpp:186).
#include <algorithm>
#include <vector>

#include "nwg_internal.cuh"

namespace nwg {
namespace {

constexpr int kMsThreads = 256;
constexpr int kMsWarps   = kMsThreads / 32;
constexpr int kMsLaneDeg = 64;  // in-edges a lane scans alone in a pull; longer lists are scanned by the warp
constexpr int kMsProbe   = 4;   // in-neighbours a lane reads per round (independent loads)

struct MsCounters {
  unsigned long long discovered;      // (source, vertex) pairs first reached this level
  unsigned long long frontier_edges;  // out-edges of the next frontier's vertices
  unsigned long long frontier_count;  // chunk entries in the next frontier list
};

constexpr uint32_t kMsChunk      = 256;  // out-edges per frontier chunk entry (one warp's push task)
constexpr uint32_t kMsChunkShift = 8;
constexpr uint64_t kMsLaneChunks = 16;  // a lane writes up to this many chunk entries of one vertex itself

template <int W>
struct MsParams {
  const uint64_t* off;
  const uint32_t* col;
  const uint64_t* in_off;
  const uint32_t* in_col;
  const uint32_t* Z;  // vertices with no in-edges: never reached by a pull
  uint64_t        n;
  uint64_t*       vis;
  uint64_t*       fr_cur;
  uint64_t*       fr_nxt;
  uint64_t*       nx;
  uint64_t*       list_cur;  // frontier chunk entries (vertex << 32 | chunk), push input
  uint64_t*       list_nxt;
  uint64_t        list_cap;
  uint8_t*        depth;     // [k][n], rows of this pass start at depth + src0 * n
  uint64_t        full[W];   // mask of the valid sources of each word
  uint32_t        level;
  MsCounters*     cnt;       // counters of the level being produced
};

template <typename T>
__device__ __forceinline__ T ms_block_sum(T v) {
  __shared__ T red[32];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  T t = 0;
  if (warp == 0) {
    t = (lane < (blockDim.x >> 5)) ? red[lane] : T(0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(kFullMask, t, o);
  }
  return t;  // valid in thread 0
}

// depth[s][v] = level for every source bit s newly set at v.  Lanes hold
// consecutive vertices; the warp walks only the bits some lane has, so each
// store instruction writes one row's bytes for up to 32 adjacent vertices.
template <int W>
__device__ __forceinline__ void write_depths(const MsParams<W>& p, bool has, uint64_t v, const uint64_t (&nw)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) {
    uint64_t any = has ? nw[w] : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) any |= __shfl_xor_sync(kFullMask, any, o);
    while (any) {
      const int s = __ffsll((long long)any) - 1;
      any &= any - 1;
      if (has && ((nw[w] >> s) & 1ull)) p.depth[(uint64_t)(w * 64 + s) * p.n + v] = (uint8_t)p.level;
    }
  }
}

// Roots: VIS, FR[cur] and depth 0 for each source; the frontier list holds
// the distinct roots (deduplicated on the host).
template <int W>
__global__ void k_ms_roots(MsParams<W> p, const uint32_t* roots, uint32_t k) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= k) return;
  const uint64_t v   = roots[s];
  const uint64_t bit = 1ull << (s & 63);
  atomicOr((unsigned long long*)&p.vis[v * W + (s >> 6)], (unsigned long long)bit);
  atomicOr((unsigned long long*)&p.fr_cur[v * W + (s >> 6)], (unsigned long long)bit);
  p.depth[(uint64_t)s * p.n + v] = 0;
}

// Push: one warp per frontier chunk entry (up to kMsChunk out-edges of one
// vertex), so hubs are spread over the grid; lanes stride over the edges.
template <int W>
__global__ void __launch_bounds__(kMsThreads) k_ms_push(MsParams<W> p, uint64_t nlist) {
  const unsigned lane   = threadIdx.x & 31;
  const uint64_t gwarp  = (uint64_t)blockIdx.x * kMsWarps + (threadIdx.x >> 5);
  const uint64_t nwarps = (uint64_t)gridDim.x * kMsWarps;
  for (uint64_t i = gwarp; i < nlist; i += nwarps) {
    const uint64_t ent = p.list_cur[i];
    const uint32_t u   = (uint32_t)(ent >> 32);
    uint64_t       f[W];
#pragma unroll
    for (int w = 0; w < W; ++w) f[w] = p.fr_cur[(uint64_t)u * W + w];
    const uint64_t beg = p.off[u] + ((ent & 0xFFFFFFFFull) << kMsChunkShift);
    const uint64_t end = min(p.off[u + 1], beg + kMsChunk);
    for (uint64_t e = beg + lane; e < end; e += 32) {
      const uint32_t v = __ldg(p.col + e);
#pragma unroll
      for (int w = 0; w < W; ++w) {
        const uint64_t m = f[w] & ~p.vis[(uint64_t)v * W + w];  // VIS is stable during the push
        if (m) atomicOr((unsigned long long*)&p.nx[(uint64_t)v * W + w], (unsigned long long)m);
      }
    }
  }
}

// Appends the warp's new frontier vertices (lane flag `has`, out-degree
// deg) to list_nxt as chunk entries and adds their out-degrees; one atomic
// per warp.  A vertex without out-edges has nothing to push and no entry.
template <int W>
__device__ __forceinline__ void ms_append(const MsParams<W>& p, bool has, uint32_t v, unsigned long long& fedges,
                                          unsigned long long deg) {
  const unsigned           lane = threadIdx.x & 31;
  const unsigned long long nc   = has ? (deg + kMsChunk - 1) >> kMsChunkShift : 0ull;
  if (has) fedges += deg;
  unsigned long long incl = nc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long x = __shfl_up_sync(kFullMask, incl, o);
    if ((int)lane >= o) incl += x;
  }
  const unsigned long long tot = __shfl_sync(kFullMask, incl, 31);
  if (tot == 0) return;
  unsigned long long base = 0;
  if (lane == 31) base = atomicAdd(&p.cnt->frontier_count, tot);
  base                    = __shfl_sync(kFullMask, base, 31);
  const unsigned long long pos = base + incl - nc;
  if (nc && nc <= kMsLaneChunks) {
    for (unsigned long long j = 0; j < nc; ++j)
      if (pos + j < p.list_cap) p.list_nxt[pos + j] = ((uint64_t)v << 32) | j;
  }
  unsigned big = __ballot_sync(kFullMask, nc > kMsLaneChunks);
  while (big) {  // hubs: the whole warp writes their entries
    const int src = __ffs(big) - 1;
    big &= big - 1;
    const uint64_t           vs = __shfl_sync(kFullMask, (uint64_t)v, src);
    const unsigned long long ps = __shfl_sync(kFullMask, pos, src);
    const unsigned long long ns = __shfl_sync(kFullMask, nc, src);
    for (unsigned long long j = lane; j < ns; j += 32)
      if (ps + j < p.list_cap) p.list_nxt[ps + j] = (vs << 32) | j;
  }
}

// Finalize after a push: NX -> new bits, VIS, FR[nxt], depths, next list.
// Every vertex's FR[nxt] words are written (zero when nothing is new).
template <int W>
__global__ void __launch_bounds__(kMsThreads) k_ms_finalize(MsParams<W> p) {
  unsigned long long disc = 0, fedges = 0;
  const uint64_t     stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t     n_up   = (p.n + 31) & ~31ull;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_up; v += stride) {
    const bool valid = v < p.n;
    uint64_t   nw[W];
    bool       has = false;
#pragma unroll
    for (int w = 0; w < W; ++w) {
      nw[w] = 0;
      if (valid) {
        const uint64_t x = p.nx[v * W + w];
        if (x) {
          const uint64_t vis = p.vis[v * W + w];
          nw[w]              = x & ~vis;
          p.nx[v * W + w]    = 0;
          if (nw[w]) p.vis[v * W + w] = vis | nw[w];
        }
        p.fr_nxt[v * W + w] = nw[w];
        has |= nw[w] != 0;
        disc += __popcll(nw[w]);
      }
    }
    write_depths<W>(p, has, v, nw);
    ms_append<W>(p, has, (uint32_t)v, fedges, has ? (unsigned long long)(p.off[v + 1] - p.off[v]) : 0ull);
  }
  const unsigned long long d = ms_block_sum(disc);
  const unsigned long long f = ms_block_sum(fedges);
  if (threadIdx.x == 0) {
    if (d) atomicAdd(&p.cnt->discovered, d);
    if (f) atomicAdd(&p.cnt->frontier_edges, f);
  }
}

// Pull: lane per vertex; a vertex some source has not reached ORs its
// in-neighbours' frontier words until every missing source is found.  Lists
// longer than kMsLaneDeg are scanned by the whole warp afterwards.
template <int W>
__global__ void __launch_bounds__(kMsThreads) k_ms_pull(MsParams<W> p) {
  const unsigned     lane   = threadIdx.x & 31;
  unsigned long long disc = 0, fedges = 0;
  const uint64_t     stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t     n_up   = (p.n + 31) & ~31ull;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_up; v += stride) {
    const bool valid = v < p.n;
    uint64_t   vis[W], acc[W];
    bool       need = false;
    const bool noin = !valid || ((__ldg(p.Z + (v >> 5)) >> (v & 31)) & 1u);
#pragma unroll
    for (int w = 0; w < W; ++w) {
      vis[w] = valid ? p.vis[v * W + w] : p.full[w];
      acc[w] = 0;
      need |= !noin && (vis[w] & p.full[w]) != p.full[w];
    }
    uint64_t beg = 0, end = 0;
    if (need) {
      beg = p.in_off[v];
      end = p.in_off[v + 1];
    }
    const uint64_t lim = min(end, beg + kMsLaneDeg);
    uint64_t       e   = beg;
    bool           sat = !need;
    while (e < lim && !sat) {  // kMsProbe in-neighbours per round, independent loads
      uint32_t u[kMsProbe];
#pragma unroll
      for (int q = 0; q < kMsProbe; ++q) u[q] = (e + q < lim) ? __ldg(p.in_col + e + q) : kNull;
#pragma unroll
      for (int q = 0; q < kMsProbe; ++q)
        if (u[q] != kNull) {
#pragma unroll
          for (int w = 0; w < W; ++w) acc[w] |= p.fr_cur[(uint64_t)u[q] * W + w];
        }
      e   = min(lim, e + kMsProbe);
      sat = true;
#pragma unroll
      for (int w = 0; w < W; ++w) sat &= ((acc[w] | vis[w]) & p.full[w]) == p.full[w];
    }
    // long in-edge lists: the warp scans them together, 32 * kMsProbe in-edges per round
    unsigned pend = __ballot_sync(kFullMask, !sat && e < end);
    while (pend) {
      const int ld = __ffs(pend) - 1;
      pend &= pend - 1;
      const uint64_t b  = __shfl_sync(kFullMask, e, ld);
      const uint64_t en = __shfl_sync(kFullMask, end, ld);
      uint64_t       a[W], vs[W];
#pragma unroll
      for (int w = 0; w < W; ++w) {
        a[w]  = __shfl_sync(kFullMask, acc[w], ld);
        vs[w] = __shfl_sync(kFullMask, vis[w], ld);
      }
      // each lane ORs its own share of a round of 32 * kMsProbe in-edges
      // (independent loads); one warp reduction per round checks saturation
      uint64_t mine[W];
#pragma unroll
      for (int w = 0; w < W; ++w) mine[w] = 0;
      for (uint64_t base = b; base < en; base += 32 * kMsProbe) {
        uint32_t u[kMsProbe];
#pragma unroll
        for (int q = 0; q < kMsProbe; ++q) {
          const uint64_t i = base + q * 32 + lane;
          u[q]             = i < en ? __ldg(p.in_col + i) : kNull;
        }
#pragma unroll
        for (int q = 0; q < kMsProbe; ++q)
          if (u[q] != kNull) {
#pragma unroll
            for (int w = 0; w < W; ++w) mine[w] |= p.fr_cur[(uint64_t)u[q] * W + w];
          }
        bool done = true;
#pragma unroll
        for (int w = 0; w < W; ++w) {
          uint64_t x = mine[w] | a[w];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) x |= __shfl_xor_sync(kFullMask, x, o);
          a[w] = x;
          done &= ((x | vs[w]) & p.full[w]) == p.full[w];
        }
        if (done) break;
      }
      if ((int)lane == ld) {
#pragma unroll
        for (int w = 0; w < W; ++w) acc[w] = a[w];
      }
    }
    uint64_t nw[W];
    bool     has = false;
#pragma unroll
    for (int w = 0; w < W; ++w) {
      nw[w] = acc[w] & ~vis[w] & p.full[w];
      if (valid) {
        if (nw[w]) p.vis[v * W + w] = vis[w] | nw[w];
        p.fr_nxt[v * W + w] = nw[w];
      }
      has |= nw[w] != 0;
      disc += __popcll(nw[w]);
    }
    write_depths<W>(p, has, v, nw);
    ms_append<W>(p, has, (uint32_t)v, fedges, has ? (unsigned long long)(p.off[v + 1] - p.off[v]) : 0ull);
  }
  const unsigned long long d = ms_block_sum(disc);
  const unsigned long long f = ms_block_sum(fedges);
  if (threadIdx.x == 0) {
    if (d) atomicAdd(&p.cnt->discovered, d);
    if (f) atomicAdd(&p.cnt->frontier_edges, f);
  }
}

// The first frontier list (chunk entries of the distinct roots) and its
// out-edge count.  One block; every thread of it calls ms_append.
template <int W>
__global__ void k_ms_root_list(MsParams<W> p, const uint32_t* __restrict__ uniq, uint32_t nuniq) {
  unsigned long long fedges = 0;
  for (uint32_t base = 0; base < nuniq; base += blockDim.x) {
    const uint32_t i   = base + threadIdx.x;
    const bool     has = i < nuniq;
    const uint32_t v   = has ? uniq[i] : 0u;
    ms_append<W>(p, has, v, fedges, has ? (unsigned long long)(p.off[v + 1] - p.off[v]) : 0ull);
  }
  const unsigned long long f = ms_block_sum(fedges);
  if (threadIdx.x == 0 && f) atomicAdd(&p.cnt->frontier_edges, f);
}

// Grid of the grid-stride kernels: 8 blocks per SM, fewer when the graph
// (or the frontier list) has less work than that, so the small graphs of a
// serving mix leave room for other streams' launches.
int grid_ms(const GraphDev* g, int per_sm, uint64_t items, uint64_t per_block) {
  const uint64_t want = (items + per_block - 1) / per_block;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)g->sm_count * per_sm, want));
}

// One pass of up to 64 * W sources.
template <int W>
int ms_pass(GraphDev* g, MsWorkspace* ws, const uint32_t* roots_dev, const uint32_t* roots_host, uint32_t k,
            uint8_t* depth_rows, int alpha, cudaStream_t stream, nwg_msbfs_stats* st) {
  const uint64_t n = g->n;
  MsParams<W>    p = {};
  p.off            = g->off;
  p.col            = g->col;
  p.in_off         = g->in_off;
  p.in_col         = g->in_col;
  p.Z              = g->Z;
  p.n              = n;
  p.vis            = ws->vis;
  p.fr_cur         = ws->fr[0];
  p.fr_nxt         = ws->fr[1];
  p.nx             = ws->nx;
  p.list_cur       = ws->list[0];
  p.list_nxt       = ws->list[1];
  p.list_cap       = ws->list_cap;
  p.depth          = depth_rows;
  for (int w = 0; w < W; ++w) {
    const int64_t bits = std::min<int64_t>(64, (int64_t)k - 64 * w);
    p.full[w]          = bits >= 64 ? ~0ull : bits <= 0 ? 0ull : ((1ull << bits) - 1);
  }
  const size_t words = (size_t)n * W * sizeof(uint64_t);
  NWG_CUDA_TRY(cudaMemsetAsync(ws->vis, 0, words, stream));
  NWG_CUDA_TRY(cudaMemsetAsync(ws->fr[0], 0, words, stream));
  NWG_CUDA_TRY(cudaMemsetAsync(ws->nx, 0, words, stream));
  NWG_CUDA_TRY(cudaMemsetAsync(depth_rows, 0xFF, (size_t)k * n, stream));
  k_ms_roots<W><<<(k + 255) / 256, 256, 0, stream>>>(p, roots_dev, k);
  NWG_CUDA_TRY(cudaGetLastError());

  // distinct roots form the first frontier; their chunk entries the first list
  std::vector<uint32_t> uniq(roots_host, roots_host + k);
  std::sort(uniq.begin(), uniq.end());
  uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
  NWG_CUDA_TRY(cudaMemcpyAsync(ws->roots_uniq, uniq.data(), uniq.size() * 4, cudaMemcpyHostToDevice, stream));
  MsCounters& hc = *static_cast<MsCounters*>(ws->cnt_host);
  NWG_CUDA_TRY(cudaMemsetAsync(ws->cnt, 0, sizeof(MsCounters), stream));
  p.cnt = static_cast<MsCounters*>(ws->cnt);
  k_ms_root_list<W><<<1, kMsThreads, 0, stream>>>(p, ws->roots_uniq, (uint32_t)uniq.size());
  NWG_CUDA_TRY(cudaGetLastError());
  NWG_CUDA_TRY(cudaMemcpyAsync(&hc, ws->cnt, sizeof(hc), cudaMemcpyDeviceToHost, stream));
  NWG_CUDA_TRY(cudaStreamSynchronize(stream));
  uint64_t fedges = hc.frontier_edges;
  std::swap(p.list_cur, p.list_nxt);  // the root list was written as "next"
  uint64_t nlist     = hc.frontier_count;
  uint64_t unchecked = g->m;
  for (uint32_t level = 1;; ++level) {
    if (level >= 255) return set_error(NWG_EOVERFLOW, "a depth reaches 255: does not fit the uint8 encoding");
    p.level = level;
    p.cnt   = static_cast<MsCounters*>(ws->cnt);
    NWG_CUDA_TRY(cudaMemsetAsync(ws->cnt, 0, sizeof(MsCounters), stream));
    const bool pull   = fedges > unchecked / (uint64_t)alpha;
    const bool traced = st->passes == 0 && st->trace_len < NWG_MS_TRACE_CAP;
    if (traced) NWG_CUDA_TRY(cudaEventRecord(ws->ev_lvl[0], stream));
    if (pull) {
      k_ms_pull<W><<<grid_ms(g, 8, n, kMsThreads), kMsThreads, 0, stream>>>(p);
      st->pull_levels++;
    } else {
      unchecked -= std::min(unchecked, fedges);
      const uint64_t nl = std::min<uint64_t>(nlist, ws->list_cap);
      k_ms_push<W><<<grid_ms(g, 8, nl, kMsWarps), kMsThreads, 0, stream>>>(p, nl);
      NWG_CUDA_TRY(cudaGetLastError());
      k_ms_finalize<W><<<grid_ms(g, 8, n, kMsThreads), kMsThreads, 0, stream>>>(p);
      st->push_levels++;
    }
    NWG_CUDA_TRY(cudaGetLastError());
    if (traced) NWG_CUDA_TRY(cudaEventRecord(ws->ev_lvl[1], stream));
    NWG_CUDA_TRY(cudaMemcpyAsync(&hc, ws->cnt, sizeof(hc), cudaMemcpyDeviceToHost, stream));
    NWG_CUDA_TRY(cudaStreamSynchronize(stream));
    if (traced) {
      const uint32_t i = st->trace_len++;
      st->trace_pull[i] = pull ? 1 : 0;
      cudaEventElapsedTime(&st->trace_ms[i], ws->ev_lvl[0], ws->ev_lvl[1]);
      st->trace_frontier_edges[i] = fedges;
      st->trace_discovered[i]     = hc.discovered;
    }
    if (hc.discovered == 0) break;
    st->levels = std::max(st->levels, level + 1);
    fedges     = hc.frontier_edges;
    nlist      = hc.frontier_count;
    std::swap(p.fr_cur, p.fr_nxt);
    std::swap(p.list_cur, p.list_nxt);
  }
  return NWG_OK;
}

}  // namespace

uint64_t ms_ws_bytes(uint64_t n_cap, uint64_t m_cap) {
  const uint64_t n = std::max<uint64_t>(n_cap, 1);
  // VIS, FR[2], NX at four words per vertex, two frontier lists (every
  // frontier vertex has at most deg / kMsChunk + 1 entries), counters, roots
  return 4 * n * 4 * sizeof(uint64_t) + 2 * (n + m_cap / kMsChunk + 1) * 8 + sizeof(MsCounters) + 2 * 256 * 4;
}

int ms_ws_init_cap(GraphDev* g, uint64_t n_cap, uint64_t m_cap, MsWorkspace* ws) {
  const uint64_t n        = std::max<uint64_t>(n_cap, 1);
  const size_t   words    = (size_t)n * 4 * sizeof(uint64_t);  // room for W = 4
  const uint64_t list_cap = n + m_cap / kMsChunk + 1;
  ws->g                   = g;
  ws->n_cap               = n_cap;
  ws->m_cap               = m_cap;
  ws->list_cap            = list_cap;
  if (cudaMalloc(&ws->vis, words) != cudaSuccess || cudaMalloc(&ws->fr[0], words) != cudaSuccess ||
      cudaMalloc(&ws->fr[1], words) != cudaSuccess || cudaMalloc(&ws->nx, words) != cudaSuccess ||
      cudaMalloc(&ws->list[0], list_cap * 8) != cudaSuccess || cudaMalloc(&ws->list[1], list_cap * 8) != cudaSuccess ||
      cudaMalloc(&ws->cnt, sizeof(MsCounters)) != cudaSuccess || cudaMalloc(&ws->roots, 256 * 4) != cudaSuccess ||
      cudaMalloc(&ws->roots_uniq, 256 * 4) != cudaSuccess ||
      cudaMallocHost(&ws->cnt_host, sizeof(MsCounters)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(NWG_ENOMEM, "multi-source workspace allocation failed");
  }
  NWG_CUDA_TRY(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
  NWG_CUDA_TRY(cudaEventCreate(&ws->ev0));
  NWG_CUDA_TRY(cudaEventCreate(&ws->ev1));
  NWG_CUDA_TRY(cudaEventCreate(&ws->ev_lvl[0]));
  NWG_CUDA_TRY(cudaEventCreate(&ws->ev_lvl[1]));
  return NWG_OK;
}

int ms_ws_init(GraphDev* g, MsWorkspace* ws) { return ms_ws_init_cap(g, g->n, g->m, ws); }

void ms_ws_free(MsWorkspace* ws) {
  if (!ws) return;
  if (ws->stream) cudaStreamSynchronize(ws->stream);
  cudaFree(ws->vis);
  cudaFree(ws->fr[0]);
  cudaFree(ws->fr[1]);
  cudaFree(ws->nx);
  cudaFree(ws->list[0]);
  cudaFree(ws->list[1]);
  cudaFree(ws->cnt);
  cudaFree(ws->roots);
  cudaFree(ws->roots_uniq);
  if (ws->cnt_host) cudaFreeHost(ws->cnt_host);
  if (ws->ev0) cudaEventDestroy(ws->ev0);
  if (ws->ev1) cudaEventDestroy(ws->ev1);
  if (ws->ev_lvl[0]) cudaEventDestroy(ws->ev_lvl[0]);
  if (ws->ev_lvl[1]) cudaEventDestroy(ws->ev_lvl[1]);
  if (ws->stream) cudaStreamDestroy(ws->stream);
  delete ws;
}

// Runs ceil(k / 256) passes of up to 256 sources over graph g, which must
// fit the workspace's capacity, on `stream` (or the workspace's own).
int ms_run_on(MsWorkspace* ws, GraphDev* g, const uint32_t* roots_host, uint32_t k, uint8_t* depths_dev, int alpha,
              cudaStream_t stream, nwg_msbfs_stats* st) {
  if (g->n > ws->n_cap || g->m > ws->m_cap)
    return set_error(NWG_EINVAL, "graph larger than the multi-source workspace's capacity");
  for (uint32_t i = 0; i < k; ++i)
    if (roots_host[i] >= g->n) return set_error(NWG_EINVAL, "root " + std::to_string(roots_host[i]) + " >= n");
  if (alpha <= 0) return set_error(NWG_EINVAL, "alpha must be positive");
  cudaStream_t s = stream ? stream : ws->stream;
  for (uint32_t b = 0; b < k; b += 256) {
    const uint32_t kk = std::min<uint32_t>(256, k - b);
    NWG_CUDA_TRY(cudaMemcpyAsync(ws->roots, roots_host + b, kk * 4, cudaMemcpyHostToDevice, s));
    uint8_t* rows = depths_dev + (uint64_t)b * g->n;
    int      rc;
    if (kk <= 64) {
      rc = ms_pass<1>(g, ws, ws->roots, roots_host + b, kk, rows, alpha, s, st);
    } else if (kk <= 128) {
      rc = ms_pass<2>(g, ws, ws->roots, roots_host + b, kk, rows, alpha, s, st);
    } else if (kk <= 192) {
      rc = ms_pass<3>(g, ws, ws->roots, roots_host + b, kk, rows, alpha, s, st);
    } else {
      rc = ms_pass<4>(g, ws, ws->roots, roots_host + b, kk, rows, alpha, s, st);
    }
    if (rc) return rc;
    st->passes++;
  }
  return NWG_OK;
}

int ms_run(MsWorkspace* ws, const uint32_t* roots_host, uint32_t k, uint8_t* depths_dev, int alpha,
           cudaStream_t stream, nwg_msbfs_stats* st) {
  return ms_run_on(ws, ws->g, roots_host, k, depths_dev, alpha, stream, st);
}

}  // namespace nwg
