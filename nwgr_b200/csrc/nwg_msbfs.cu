// Batched multi-source BFS: 64 sources per 64-bit word, up to 256 sources
// (four words, one 32-byte sector per vertex) per pass.  No reference
// counterpart: NWGraph's bfs is single-source; the oracle is one
// single-source BFS per root, depths compared bit for bit.
//
// State of a pass, vertex-major so one vertex's W words share a sector:
//   VIS[n][W]    sources that have reached the vertex
//   FR[2][n][W]  sources whose BFS has the vertex in its current / next frontier
//   NX[n][W]     top-down accumulator (atomicOr), cleared when consumed
//   DP[8][n][W]  level bit-planes: bit s of DP[j][v][w] is bit j of the depth
//                of v from source 64w + s; all zero between passes
//   depth[k][n]  uint8 output, 255 = unreached, written once after the last
//                level from VIS and DP (rows of 64 contiguous bytes per store)
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
#include <new>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "nwg_internal.cuh"

namespace nwg {
namespace {

constexpr int kMsThreads = 256;
constexpr int kMsWarps   = kMsThreads / 32;
// Pull: a lane scans up to kMsLaneDeg in-edges of its vertex alone, kMsProbe
// per round (independent loads); longer lists are scanned by the warp.  On
// RMAT-22, 32 and 8 against 64 and 4: passes of 64 / 256 / 1,024 sources
// 1.48 / 4.27 / 15.3 ms against 1.57 / 4.49 / 16.0 (a warp's lanes wait for
// its longest lane, and RMAT in-degrees vary widely).
constexpr int kMsLaneDeg = 32;
constexpr int kMsProbe   = 8;

struct MsCounters {
  unsigned long long discovered;      // (source, vertex) pairs first reached this level
  unsigned long long frontier_edges;  // out-edges of the next frontier's vertices
  unsigned long long frontier_count;  // chunk entries in the next frontier list
  unsigned long long alive[4];        // sources with a vertex in the next frontier (their BFS goes on)
  unsigned long long touched;         // push: vertices in the touched list (NX made non-zero)
};

constexpr uint32_t kMsChunk      = 256;  // out-edges per frontier chunk entry (one warp's push task)
constexpr uint32_t kMsChunkShift = 8;
constexpr uint64_t kMsLaneChunks = 16;  // a lane writes up to this many chunk entries of one vertex itself
constexpr uint64_t kMsPlanes     = 8;   // level bit-planes: depths up to 254 (255 = unreached)

// Level-loop state of a pass in device memory: the decide kernel advances
// it, the level kernels read the level number and list length from it.
constexpr uint32_t kMsTrace = NWG_MS_TRACE_CAP;
struct MsPassDev {
  uint64_t   list_cap;
  uint32_t   k, nuniq;
  int32_t    alpha;
  uint32_t   level;      // level being run (0 = roots)
  uint64_t   unchecked;  // out-edges not yet pushed (the switch's edges_to_check)
  uint64_t   nlist;      // chunk entries of the current frontier list
  int32_t    status;
  uint32_t   levels;     // max depth + 1
  uint32_t   pull, stopped, push_levels, pull_levels, trace_len;
  uint64_t   sparse_max;  // a push level finalizes only its touched vertices when it pushes at most this many edges
  uint64_t   clear_max;   // ... and the frontier two levels back has at most this many chunk entries
  uint64_t   nclear;      // chunk entries of the frontier two levels back (still in list_nxt)
  uint32_t   sparse_ok;   // this push level finalizes sparsely
  unsigned long long deep[4];  // sources that still discovered vertices at level 255 (their depths exceed uint8)
  MsCounters cnt[2];     // level L's kernels add into cnt[L & 1]
  uint32_t   roots[256], uniq[256];
  uint8_t    tr_pull[kMsTrace];
  uint64_t   tr_fedges[kMsTrace], tr_disc[kMsTrace], tr_t[kMsTrace + 1];
};

// Kernel arguments (constant bank).  Level L reads FR[(L-1)&1] and
// list[(L-1)&1] and writes FR[L&1], list[L&1], cnt[L&1]; the pass graph
// holds one set of level nodes per parity, so these pointers are fixed per
// node.  The roots are level 0 (FR[0], list[0], cnt[0]).
template <int W>
struct MsParams {
  const uint64_t*  off;
  const uint32_t*  col;
  const uint64_t*  in_off;
  const uint32_t*  in_col;
  const uint32_t*  Z;  // vertices with no in-edges: never reached by a pull
  uint64_t         n;
  uint64_t*        vis;
  uint64_t*        fr_cur;
  uint64_t*        fr_nxt;
  uint64_t*        nx;
  uint64_t*        dp;        // level bit-planes, plane j at dp + j * plane
  uint32_t*        tlist;     // vertices a push level touched (NX made non-zero), in touch order
  uint32_t*        T;         // bitmap of those vertices (deduplicates the list); zero between levels
  uint64_t         plane;     // words per plane (n * W)
  uint64_t*        list_cur;  // frontier chunk entries (vertex << 32 | chunk), push input
  uint64_t*        list_nxt;
  uint64_t         list_cap;
  uint8_t*         depth;     // [k][n] rows of depth_bytes each, this pass's first row at `depth`
  uint32_t         depth_bytes;  // 1: uint8 rows (255 = unreached), 2: uint16 rows (0xFFFF = unreached)
  uint64_t         full[W];   // mask of the valid sources of each word
  MsCounters*      cnt;       // counters of the level being produced
  const MsCounters* prev;     // counters of the level before (its alive sources)
  const MsPassDev* d;
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

// The sources in nw first reach v at `level`: OR them into the planes of
// the level's set bits (at most three words for levels below 16).  Only
// v's own thread touches v's plane words in a level, and kernel boundaries
// order the levels, so a plain read-modify-write is enough.  A warp's lanes
// hold consecutive vertices, so each plane access is one coalesced run.
template <int W>
__device__ __forceinline__ void record_level(const MsParams<W>& p, uint32_t level, uint64_t v,
                                             const uint64_t (&nw)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) {
    if (!nw[w]) continue;
    for (uint32_t b = level; b; b &= b - 1) {
      uint64_t* q = p.dp + (uint64_t)(__ffs(b) - 1) * p.plane + v * W + w;
      *q |= nw[w];
    }
  }
}

// The W words of one vertex (read-only during the kernel) with 16-byte
// loads where W is even: a vertex's words start 16-byte aligned then (the
// arrays are 256-byte aligned and each vertex owns W consecutive words), so
// two words come per load instruction instead of one.
template <int W>
__device__ __forceinline__ void ms_words(const uint64_t* __restrict__ src, uint64_t (&x)[W]) {
  if constexpr (W % 2 == 0) {
#pragma unroll
    for (int w = 0; w < W; w += 2) {
      const ulonglong2 t = __ldg(reinterpret_cast<const ulonglong2*>(src + w));
      x[w]               = t.x;
      x[w + 1]           = t.y;
    }
  } else {
#pragma unroll
    for (int w = 0; w < W; ++w) x[w] = __ldg(src + w);
  }
}

// spread4(x), x < 16: bit t of x to bit 0 of byte t.  The four partial
// products x, x << 7, x << 14, x << 21 occupy disjoint bit ranges, so the
// multiply never carries.
__device__ __forceinline__ uint32_t spread4(uint32_t x) { return (x * 0x00204081u) & 0x01010101u; }

// Depth rows, one block tile at a time: kDtTile consecutive vertices of one
// source word (64 sources).  Each thread takes kDtVerts consecutive vertices,
// forms their depth bytes for 4 sources at a time (255 where VIS lacks the
// bit), transposes them with byte permutes and stores, per source, its
// vertices' bytes into a shared-memory row.  The
// block then writes every row of the tile as kDtTile contiguous bytes
// (16-byte stores; widened to uint16 for 2-byte rows).  Writing 64-byte
// pieces of 64 rows 4 MB apart from each warp reached half the HBM
// bandwidth (165 us for 476 MB at 64 sources on RMAT-22); with 512-byte
// runs per row a 64-source pass took 5% less in all.  The planes read are
// cleared.
constexpr int      kDtVerts = 2;                      // 2 or 4 (4: 1 KB runs, 64 KB, 3 blocks per SM, 5% slower)
constexpr uint32_t kDtTile  = kMsThreads * kDtVerts;  // 512 vertices
constexpr uint32_t kDtRowW  = kDtTile / 4;            // 32-bit words per shared row
constexpr size_t   kDtSmem  = 64 * (size_t)kDtTile;   // 32 KB: a byte per (source, vertex)

template <int W, int P>
__device__ __forceinline__ void depth_rows_tile(const MsParams<W>& p, uint32_t* rows, int planes, uint64_t v0, int w,
                                                int nsrc) {
  const uint64_t n  = p.n;
  const uint64_t vb = v0 + (uint64_t)threadIdx.x * kDtVerts;
  uint64_t       vis[kDtVerts], pl[kDtVerts][P];
#pragma unroll
  for (int i = 0; i < kDtVerts; ++i) {
    const uint64_t v  = vb + i;
    const bool     ok = v < n;
    vis[i]            = ok ? p.vis[v * W + w] : 0ull;
#pragma unroll
    for (int j = 0; j < P; ++j) {
      pl[i][j] = 0;
      if (ok && j < planes) {
        uint64_t* q = p.dp + (uint64_t)j * p.plane + v * W + w;
        pl[i][j]    = *q;
        if (pl[i][j]) *q = 0;
      }
    }
  }
  for (int s0 = 0; s0 < nsrc; s0 += 4) {
    uint32_t b[kDtVerts];  // byte t: depth of vertex vb + i from source 64 w + s0 + t
#pragma unroll
    for (int i = 0; i < kDtVerts; ++i) {
      uint32_t d = 0;
#pragma unroll
      for (int j = 0; j < P; ++j) d |= spread4((uint32_t)(pl[i][j] >> s0) & 15u) << j;
      const uint32_t m = spread4((uint32_t)(vis[i] >> s0) & 15u) * 0xFFu;
      b[i]             = d | ~m;
    }
    if constexpr (kDtVerts == 4) {  // 4 x 4 byte transpose: row s0 + t, byte i = b[i] byte t
      const uint32_t lo01 = __byte_perm(b[0], b[1], 0x5140), lo23 = __byte_perm(b[2], b[3], 0x5140);
      const uint32_t hi01 = __byte_perm(b[0], b[1], 0x7362), hi23 = __byte_perm(b[2], b[3], 0x7362);
      uint32_t* const r = rows + (uint32_t)s0 * kDtRowW + threadIdx.x;
      r[0]              = __byte_perm(lo01, lo23, 0x5410);
      r[kDtRowW]        = __byte_perm(lo01, lo23, 0x7632);
      r[2 * kDtRowW]    = __byte_perm(hi01, hi23, 0x5410);
      r[3 * kDtRowW]    = __byte_perm(hi01, hi23, 0x7632);
    } else {  // 4 x 2: row s0 + t holds the 2 bytes b[0] byte t, b[1] byte t
      const uint32_t lo = __byte_perm(b[0], b[1], 0x5140), hi = __byte_perm(b[0], b[1], 0x7362);
      uint16_t* const r = reinterpret_cast<uint16_t*>(rows) + (uint32_t)s0 * (2 * kDtRowW) + threadIdx.x;
      r[0]              = (uint16_t)lo;
      r[2 * kDtRowW]    = (uint16_t)(lo >> 16);
      r[4 * kDtRowW]    = (uint16_t)hi;
      r[6 * kDtRowW]    = (uint16_t)(hi >> 16);
    }
  }
}

// 255 (unreached) -> 0xFFFF, any other depth d -> d, for the 4 bytes of x:
// vertices 0, 1 in the first word, 2, 3 in the second.
__device__ __forceinline__ uint2 widen4(uint32_t x) {
  const uint32_t ff = __vcmpeq4(x, 0xFFFFFFFFu);
  return make_uint2(__byte_perm(x, ff, 0x5140), __byte_perm(x, ff, 0x7362));
}

// After the last level: every depth row of the pass from VIS and the level
// planes (the planes in use are those of the highest level run), and those
// planes cleared for the next pass.  Replaces a 255-fill of the rows and
// the per-level byte stores of each discovery.  Dynamic shared memory:
// kDtSmem bytes.
template <int W>
__global__ void __launch_bounds__(kMsThreads, 5) k_ms_depths(MsParams<W> p) {
  extern __shared__ uint32_t rows[];  // [64][kDtRowW]
  const uint32_t top    = p.d->level;
  const int      planes = top ? 32 - __clz(top) : 0;
  const int      k      = (int)p.d->k;
  const uint64_t n      = p.n;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t tiles  = (n + kDtTile - 1) / kDtTile * W;
  const bool     two    = p.depth_bytes == 2;
  // 16-byte stores when every row start stays 16-byte aligned
  const bool vec = (reinterpret_cast<uintptr_t>(p.depth) & 15u) == 0 && (n & (two ? 7u : 15u)) == 0;
  for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int      w    = (int)(t % W);  // words of the same vertices in adjacent blocks: shared VIS sectors
    const uint64_t v0   = (t / W) * kDtTile;
    const int      nsrc = min(64, k - 64 * w);
    const uint32_t nv   = (uint32_t)min((uint64_t)kDtTile, n - v0);
    if (planes <= 3) depth_rows_tile<W, 3>(p, rows, planes, v0, w, nsrc);
    else if (planes <= 4) depth_rows_tile<W, 4>(p, rows, planes, v0, w, nsrc);
    else depth_rows_tile<W, 8>(p, rows, planes, v0, w, nsrc);
    __syncthreads();
    for (int s = (int)warp; s < nsrc; s += kMsWarps) {
      const uint4*   src = reinterpret_cast<const uint4*>(rows + (uint32_t)s * kDtRowW);  // 16 vertices per uint4
      const uint64_t row = (uint64_t)(64 * w + s) * n + v0;
      if (two) {
        uint16_t* dst = reinterpret_cast<uint16_t*>(p.depth) + row;
        for (uint32_t c = lane; c * 16 < nv; c += 32) {  // 16 vertices: two 16-byte stores
          const uint4 x = src[c];
          const uint2 a = widen4(x.x), b = widen4(x.y), e = widen4(x.z), f = widen4(x.w);
          if (vec && c * 16 + 16 <= nv) {
            reinterpret_cast<uint4*>(dst + c * 16)[0] = make_uint4(a.x, a.y, b.x, b.y);
            reinterpret_cast<uint4*>(dst + c * 16)[1] = make_uint4(e.x, e.y, f.x, f.y);
          } else {
            const uint32_t wd[8] = {a.x, a.y, b.x, b.y, e.x, e.y, f.x, f.y};
            for (uint32_t i = 0; i < 16 && c * 16 + i < nv; ++i)
              dst[c * 16 + i] = (uint16_t)(wd[i >> 1] >> (16 * (i & 1)));
          }
        }
      } else {
        uint8_t* dst = p.depth + row;
        for (uint32_t c = lane; c * 16 < nv; c += 32) {
          const uint4 x = src[c];
          if (vec && c * 16 + 16 <= nv) {
            *reinterpret_cast<uint4*>(dst + c * 16) = x;
          } else {
            const uint32_t wd[4] = {x.x, x.y, x.z, x.w};
            for (uint32_t i = 0; i < 16 && c * 16 + i < nv; ++i) dst[c * 16 + i] = (uint8_t)(wd[i >> 2] >> (8 * (i & 3)));
          }
        }
      }
    }
    __syncthreads();
  }
}

// The depth kernel's shared memory is above the 48 KB default: raised once
// per word count and device, before the first launch or graph node that
// uses it.
template <int W>
int ms_depths_prepare() {
  static std::mutex        mu;
  static std::vector<char> done;  // per device
  int                      dev = 0;
  NWG_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if ((int)done.size() <= dev) done.resize(dev + 1, 0);
  if (!done[dev]) {
    NWG_CUDA_TRY(cudaFuncSetAttribute((const void*)k_ms_depths<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kDtSmem));
    done[dev] = 1;
  }
  return NWG_OK;
}

// Roots: VIS and FR[cur] for each source (depth 0: no plane bits); the
// frontier list holds the distinct roots (deduplicated on the host).
template <int W>
__global__ void k_ms_roots(MsParams<W> p) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= p.d->k) return;
  const uint64_t v   = p.d->roots[s];
  const uint64_t bit = 1ull << (s & 63);
  atomicOr((unsigned long long*)&p.vis[v * W + (s >> 6)], (unsigned long long)bit);
  atomicOr((unsigned long long*)&p.fr_nxt[v * W + (s >> 6)], (unsigned long long)bit);
  atomicOr(&p.cnt->alive[s >> 6], (unsigned long long)bit);
}

// Sources seen in the new frontier, per warp in shared memory (lane 0 ORs
// the warp's hardware OR-reduction of each word after every iteration), and
// published with one atomic per word per block at the end of the kernel.
template <int W>
__device__ __forceinline__ void ms_seen_add(uint64_t (&slot)[4], const uint64_t (&nw)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) {
    const uint32_t lo = __reduce_or_sync(kFullMask, (uint32_t)nw[w]);
    const uint32_t hi = __reduce_or_sync(kFullMask, (uint32_t)(nw[w] >> 32));
    if ((threadIdx.x & 31) == 0 && (lo | hi)) slot[w] |= ((uint64_t)hi << 32) | lo;
  }
}

template <int W>
__device__ __forceinline__ void ms_seen_publish(const MsParams<W>& p, uint64_t (*seen)[4]) {
  __syncthreads();
  if (threadIdx.x < W) {
    uint64_t x = 0;
    for (int wp = 0; wp < kMsWarps; ++wp) x |= seen[wp][threadIdx.x];
    if (x) atomicOr(&p.cnt->alive[threadIdx.x], (unsigned long long)x);
  }
}

// Push: one warp per frontier chunk entry (up to kMsChunk out-edges of one
// vertex), so hubs are spread over the grid; lanes stride over the edges.
// On a level that finalizes sparsely (at most sparse_max edges pushed, at
// most clear_max entries two levels back) it also
//   * clears FR[nxt] of the frontier two levels back, whose chunk entries
//     list_nxt still holds (this kernel reads neither FR[nxt] nor list_nxt);
//     a frontier vertex without out-edges has no entry and keeps its stale
//     word, which no kernel reads: a push reads the frontier words of list
//     entries only, a pull those of in-neighbours, which have out-edges;
//   * lists each vertex whose NX it makes non-zero, once (the T bitmap
//     deduplicates).  The list cannot outgrow sparse_max; should a warp see
//     more, it stops listing and the finalize sweeps every vertex.
template <int W>
__global__ void __launch_bounds__(kMsThreads) k_ms_push(MsParams<W> p) {
  const uint64_t nlist  = p.d->nlist;
  const bool     sparse = p.d->sparse_ok != 0;
  const uint64_t smax   = p.d->sparse_max;
  const unsigned lane   = threadIdx.x & 31;
  const uint64_t gwarp  = (uint64_t)blockIdx.x * kMsWarps + (threadIdx.x >> 5);
  const uint64_t nwarps = (uint64_t)gridDim.x * kMsWarps;
  if (sparse) {
    const uint64_t nclear = p.d->nclear;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nclear; i += stride) {
      const uint64_t u = p.list_nxt[i] >> 32;
#pragma unroll
      for (int w = 0; w < W; ++w) p.fr_nxt[u * W + w] = 0;
    }
  }
  for (uint64_t i = gwarp; i < nlist; i += nwarps) {
    const uint64_t ent = p.list_cur[i];
    const uint32_t u   = (uint32_t)(ent >> 32);
    uint64_t       f[W];
    ms_words<W>(p.fr_cur + (uint64_t)u * W, f);
    const uint64_t beg = p.off[u] + ((ent & 0xFFFFFFFFull) << kMsChunkShift);
    const uint64_t end = min(p.off[u + 1], beg + kMsChunk);
    unsigned long long seen_count = 0;
    if (sparse && lane == 0) seen_count = *(volatile unsigned long long*)&p.cnt->touched;
    const bool track = sparse && __shfl_sync(kFullMask, seen_count, 0) <= smax;  // warp-uniform
    for (uint64_t base = beg; base < end; base += 32) {
      const uint64_t e     = base + lane;
      bool           first = false;  // this lane made one of v's NX words non-zero
      uint32_t       v     = 0;
      if (e < end) {
        v = __ldg(p.col + e);
        uint64_t seen[W];
        ms_words<W>(p.vis + (uint64_t)v * W, seen);  // VIS is stable during the push
#pragma unroll
        for (int w = 0; w < W; ++w) {
          const uint64_t m = f[w] & ~seen[w];
          if (!m) continue;
          if (track) {  // the old value is needed only here: elsewhere the OR stays a fire-and-forget reduction
            if (atomicOr((unsigned long long*)&p.nx[(uint64_t)v * W + w], (unsigned long long)m) == 0ull) first = true;
          } else {
            atomicOr((unsigned long long*)&p.nx[(uint64_t)v * W + w], (unsigned long long)m);
          }
        }
      }
      if (track) {
        const uint32_t bit = 1u << (v & 31);
        const bool     add = first && !(atomicOr(&p.T[v >> 5], bit) & bit);
        const unsigned am  = __ballot_sync(kFullMask, add);
        if (am) {
          unsigned long long b = 0;
          if (lane == 0) b = atomicAdd(&p.cnt->touched, (unsigned long long)__popc(am));
          b = __shfl_sync(kFullMask, b, 0);
          if (add) {
            const unsigned long long pos = b + __popc(am & ((1u << lane) - 1u));
            if (pos < p.n) p.tlist[pos] = v;
          }
        }
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

// One vertex of a finalize: NX -> new bits, VIS, FR[nxt], level planes,
// next list.  All 32 lanes of the warp call it (valid false for padding).
template <int W>
__device__ __forceinline__ void finalize_vertex(const MsParams<W>& p, uint32_t level, bool valid, uint64_t v,
                                                unsigned long long& disc, unsigned long long& fedges,
                                                uint64_t (&seen_slot)[4]) {
  uint64_t nw[W];
  bool     has = false;
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
  if (has) record_level<W>(p, level, v, nw);
  ms_seen_add<W>(seen_slot, nw);
  ms_append<W>(p, has, (uint32_t)v, fedges, has ? (unsigned long long)(p.off[v + 1] - p.off[v]) : 0ull);
}

// Finalize after a push.  Sparse when the push listed every vertex it
// touched and cleared FR[nxt] of the frontier two levels back: only the listed vertices are visited, every other FR[nxt]
// word is already zero (or stale for a vertex no kernel reads).  Otherwise
// every vertex's FR[nxt] words are written (zero when nothing is new).
// Either way the T bits the push set are cleared.
template <int W>
__global__ void __launch_bounds__(kMsThreads) k_ms_finalize(MsParams<W> p) {
  const uint32_t level = p.d->level;
  unsigned long long disc = 0, fedges = 0;
  __shared__ uint64_t s_seen[kMsWarps][4];
  if ((threadIdx.x & 31) < 4) s_seen[threadIdx.x >> 5][threadIdx.x & 31] = 0;
  __syncwarp();
  const uint64_t     stride  = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t     touched = p.cnt->touched;
  const bool         sparse  = p.d->sparse_ok != 0 && touched <= p.d->sparse_max;
  if (sparse) {
    const uint64_t t_up = (touched + 31) & ~31ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < t_up; i += stride) {
      const bool     valid = i < touched;
      const uint64_t v     = valid ? p.tlist[i] : 0;
      if (valid) p.T[v >> 5] = 0;
      finalize_vertex<W>(p, level, valid, v, disc, fedges, s_seen[threadIdx.x >> 5]);
    }
  } else {
    const uint64_t n_up = (p.n + 31) & ~31ull;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_up; v += stride) {
      const bool valid = v < p.n;
      if (valid && (v & 31) == 0) p.T[v >> 5] = 0;
      finalize_vertex<W>(p, level, valid, v, disc, fedges, s_seen[threadIdx.x >> 5]);
    }
  }
  ms_seen_publish<W>(p, s_seen);
  const unsigned long long dsum = ms_block_sum(disc);
  const unsigned long long f    = ms_block_sum(fedges);
  if (threadIdx.x == 0) {
    if (dsum) atomicAdd(&p.cnt->discovered, dsum);
    if (f) atomicAdd(&p.cnt->frontier_edges, f);
  }
}

// Pull: lane per vertex; a vertex some source has not reached ORs its
// in-neighbours' frontier words until every missing source is found.  Lists
// longer than kMsLaneDeg are scanned by the whole warp afterwards.
template <int W>
__global__ void __launch_bounds__(kMsThreads, W == 1 ? 5 : 4) k_ms_pull(MsParams<W> p) {
  const uint32_t level = p.d->level;
  const unsigned     lane   = threadIdx.x & 31;
  unsigned long long disc = 0, fedges = 0;
  __shared__ uint64_t s_seen[kMsWarps][4];
  __shared__ uint64_t s_act[4];  // sources that can still reach a vertex: valid, frontier not empty
  if ((threadIdx.x & 31) < 4) s_seen[threadIdx.x >> 5][threadIdx.x & 31] = 0;
  if (threadIdx.x < W) s_act[threadIdx.x] = p.full[threadIdx.x] & p.prev->alive[threadIdx.x];
  __syncthreads();
  const uint64_t     stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t     n_up   = (p.n + 31) & ~31ull;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_up; v += stride) {
    const bool valid = v < p.n;
    uint64_t   vis[W], acc[W];
    bool       need = false;
    const bool noin = !valid || ((__ldg(p.Z + (v >> 5)) >> (v & 31)) & 1u);
    // only sources whose frontier is not empty can still reach v (s_act): a
    // source in a small component must not keep every vertex scanning all
    // its in-edges at every level
#pragma unroll
    for (int w = 0; w < W; ++w) {
      vis[w] = valid ? p.vis[v * W + w] : p.full[w];
      acc[w] = 0;
      need |= !noin && (vis[w] & s_act[w]) != s_act[w];
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
          uint64_t x[W];
          ms_words<W>(p.fr_cur + (uint64_t)u[q] * W, x);
#pragma unroll
          for (int w = 0; w < W; ++w) acc[w] |= x[w];
        }
      e   = min(lim, e + kMsProbe);
      sat = true;
#pragma unroll
      for (int w = 0; w < W; ++w) sat &= ((acc[w] | vis[w]) & s_act[w]) == s_act[w];
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
            uint64_t x[W];
            ms_words<W>(p.fr_cur + (uint64_t)u[q] * W, x);
#pragma unroll
            for (int w = 0; w < W; ++w) mine[w] |= x[w];
          }
        bool done = true;
#pragma unroll
        for (int w = 0; w < W; ++w) {
          uint64_t x = mine[w] | a[w];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) x |= __shfl_xor_sync(kFullMask, x, o);
          a[w] = x;
          done &= ((x | vs[w]) & s_act[w]) == s_act[w];
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
    if (has) record_level<W>(p, level, v, nw);
    ms_seen_add<W>(s_seen[threadIdx.x >> 5], nw);
    ms_append<W>(p, has, (uint32_t)v, fedges, has ? (unsigned long long)(p.off[v + 1] - p.off[v]) : 0ull);
  }
  ms_seen_publish<W>(p, s_seen);
  const unsigned long long dsum = ms_block_sum(disc);
  const unsigned long long f    = ms_block_sum(fedges);
  if (threadIdx.x == 0) {
    if (dsum) atomicAdd(&p.cnt->discovered, dsum);
    if (f) atomicAdd(&p.cnt->frontier_edges, f);
  }
}

// The first frontier list (chunk entries of the distinct roots) and its
// out-edge count.  One block; every thread of it calls ms_append.
template <int W>
__global__ void k_ms_root_list(MsParams<W> p) {  // level 0: writes list[0] and cnt[0]
  const uint32_t*    uniq   = p.d->uniq;
  const uint32_t     nuniq  = p.d->nuniq;
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

// The level loop's decision, one thread, before every level: stop when the
// level just run discovered nothing, or after level 255 (depths from 255 on
// do not fit the level planes; the sources that still discovered vertices
// at level 255 are recorded as deep, the others' depths are complete), else pull
// when the frontier's out-edges exceed the unpushed edges / alpha
// (nw::graph::bfs, bfs.hpp:186), push otherwise.  Records the per-level
// trace; with set_cond it drives the graph's WHILE node and this parity's
// SWITCH node.  The call that stops the loop selects the depth rows (which
// also clear the level planes, so they must run exactly once); later calls
// only keep the loop stopped.
__global__ void k_ms_decide(MsPassDev* d, cudaGraphConditionalHandle h_loop, cudaGraphConditionalHandle h_sw,
                            int set_cond) {
  if (threadIdx.x != 0) return;
  const bool was_stopped = d->stopped != 0;
  bool       stop        = was_stopped;
  if (!stop) {
    const uint32_t    L    = d->level + 1;
    const MsCounters& prev = d->cnt[(L - 1) & 1];
    uint64_t          now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    if (L - 1 <= kMsTrace) d->tr_t[L - 1] = now;
    if (L > 1) {
      if (L - 2 < kMsTrace) d->tr_disc[L - 2] = prev.discovered;
      if (prev.discovered == 0) stop = true;
      else d->levels = L;
    }
    if (!stop && L >= 256) {
#pragma unroll
      for (int w = 0; w < 4; ++w) d->deep[w] = prev.alive[w];
      d->status = NWG_EOVERFLOW;
      stop      = true;
    }
    if (stop) {
      d->trace_len = min(L - 1, kMsTrace);
      d->stopped   = 1;
    } else {
      const uint64_t fedges = prev.frontier_edges;
      d->nlist              = min((uint64_t)prev.frontier_count, d->list_cap);
      // list[L & 1] still holds the chunk entries of level L - 2's frontier
      const uint64_t old    = min((uint64_t)d->cnt[L & 1].frontier_count, d->list_cap);
      d->cnt[L & 1]         = MsCounters{};
      const bool pull       = fedges > d->unchecked / (uint64_t)d->alpha;
      d->nclear             = old;
      // the push touches at most fedges vertices, so a sparse level's list never overflows
      d->sparse_ok          = (!pull && fedges <= d->sparse_max && old <= d->clear_max) ? 1u : 0u;
      if (!pull) d->unchecked -= min(d->unchecked, fedges);
      if (L - 1 < kMsTrace) {
        d->tr_pull[L - 1]   = pull ? 1 : 0;
        d->tr_fedges[L - 1] = fedges;
      }
      if (pull) d->pull_levels++;
      else d->push_levels++;
      d->pull  = pull ? 1 : 0;
      d->level = L;
    }
  }
  if (set_cond) {  // switch 2: the depth rows, once; 3: no branch
    cudaGraphSetConditional(h_sw, stop ? (was_stopped ? 3u : 2u) : d->pull);
    cudaGraphSetConditional(h_loop, stop ? 0u : 1u);
  }
}

// Grids of the grid-stride kernels: at most 8 blocks per SM and no more
// than are resident at once (the kernels deal their work out statically by
// block index, so a second wave would finish last), fewer when the pass's
// graph has less work than that, so the small graphs of a serving mix leave
// room for other streams' launches.
int ms_occupancy(const void* kernel) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kMsThreads, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return per_sm;
}

int grid_for(const MsWorkspace* ws, int per_sm, uint64_t items, uint64_t per_block) {
  const uint64_t want = (items + per_block - 1) / per_block;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)ws->sm_count * std::min(per_sm, 8), want));
}

int grid_ms(const MsWorkspace* ws, const void* kernel, uint64_t items, uint64_t per_block) {
  return grid_for(ws, ms_occupancy(kernel), items, per_block);
}

template <int W>
int ms_depths_occupancy() {
  int per_sm = 0;
  if (ms_depths_prepare<W>() != NWG_OK ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_ms_depths<W>, kMsThreads, kDtSmem) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return per_sm;
}

// Node slots of a pass graph.
enum { kNRoots, kNList, kNPush0, kNFin0, kNPull0, kNPush1, kNFin1, kNPull1, kNDepths0, kNDepths1, kNNodes };

// Arguments of a pass: the base set (roots, level 0) and the two parities.
template <int W>
struct MsArgs {
  MsParams<W> base;    // level 0: writes FR[0], list[0], cnt[0]
  MsParams<W> par[2];  // par[L & 1] for level L
  uint64_t    m;       // out-edges of the pass's graph (bounds its frontier lists)
};

template <int W>
MsArgs<W> ms_args(GraphDev* g, MsWorkspace* ws, uint8_t* depth_rows, uint32_t depth_bytes, uint32_t k) {
  MsArgs<W> a;
  std::memset(&a, 0, sizeof a);  // padding too: passes compare their arguments bytewise
  MsParams<W>& p = a.base;
  a.m        = g->m;
  p.off      = g->off;
  p.col      = g->col;
  p.in_off   = g->in_off;
  p.in_col   = g->in_col;
  p.Z        = g->Z;
  p.n        = g->n;
  p.vis      = ws->vis;
  p.nx       = ws->nx;
  p.dp       = ws->dp;
  p.tlist    = ws->tlist;
  p.T        = ws->tbits;
  p.plane    = g->n * W;
  p.list_cap = ws->list_cap;
  p.depth    = depth_rows;
  p.depth_bytes = depth_bytes;
  for (int w = 0; w < W; ++w) {
    const int64_t bits = std::min<int64_t>(64, (int64_t)k - 64 * w);
    p.full[w]          = bits >= 64 ? ~0ull : bits <= 0 ? 0ull : ((1ull << bits) - 1);
  }
  MsPassDev* d = static_cast<MsPassDev*>(ws->pass_dev);
  p.d          = d;
  for (int par = 0; par < 2; ++par) {  // level L with L & 1 == par
    MsParams<W>& q = a.par[par];
    q              = p;
    q.fr_cur       = ws->fr[par ^ 1];
    q.fr_nxt       = ws->fr[par];
    q.list_cur     = ws->list[par ^ 1];
    q.list_nxt     = ws->list[par];
    q.cnt          = &d->cnt[par];
    q.prev         = &d->cnt[par ^ 1];
  }
  p.fr_nxt   = ws->fr[0];
  p.list_nxt = ws->list[0];
  p.cnt      = &d->cnt[0];
  p.prev     = &d->cnt[1];  // unused at level 0
  return a;
}

template <int W>
void* ms_node_fn(int slot) {
  switch (slot) {
    case kNRoots: return (void*)k_ms_roots<W>;
    case kNList: return (void*)k_ms_root_list<W>;
    case kNPush0:
    case kNPush1: return (void*)k_ms_push<W>;
    case kNFin0:
    case kNFin1: return (void*)k_ms_finalize<W>;
    case kNDepths0:
    case kNDepths1: return (void*)k_ms_depths<W>;
    default: return (void*)k_ms_pull<W>;
  }
}

template <int W>
MsParams<W>* ms_node_args(MsArgs<W>& a, int slot) {
  if (slot == kNRoots || slot == kNList || slot == kNDepths0 || slot == kNDepths1) return &a.base;
  return slot < kNPush1 ? &a.par[1] : &a.par[0];  // the first half of the body runs odd levels
}

template <int W>
cudaKernelNodeParams ms_node_params(MsWorkspace* ws, MsArgs<W>& a, int slot, void** argv) {
  cudaKernelNodeParams kp = {};
  kp.func                 = ms_node_fn<W>(slot);
  argv[0]                 = ms_node_args(a, slot);
  kp.kernelParams         = argv;
  kp.blockDim             = dim3(kMsThreads);
  if (slot == kNRoots) kp.gridDim = dim3(1);
  else if (slot == kNList) kp.gridDim = dim3(1);
  else {
    // grids fit the pass's own graph (a workspace may be sized for a much
    // larger one, as a serving slot's is); occupancy is queried once
    const bool depths = slot >= kNDepths0;
    int&       per_sm = ws->node_occ[W - 1][slot];
    if (!per_sm) per_sm = depths ? ms_depths_occupancy<W>() : ms_occupancy(kp.func);
    const uint64_t n = a.base.n;
    kp.gridDim = dim3((slot == kNPush0 || slot == kNPush1) ? grid_for(ws, per_sm, n + a.m / kMsChunk + 1, kMsWarps)
                      : depths                             ? grid_for(ws, per_sm, (n + kDtTile - 1) / kDtTile * W, 1)
                                                           : grid_for(ws, per_sm, n, kMsThreads));
    if (depths) kp.sharedMemBytes = (unsigned)kDtSmem;
  }
  return kp;
}

// The pass as a CUDA graph: roots, first frontier list, then
// WHILE(decide -> SWITCH{push + finalize | pull | depth rows} for an odd
// level, the same for the following even level); no host round trip per
// level.  The decide that stops the loop selects the depth-rows branch of
// its own switch, so the WHILE node stays the graph's last node.  The depth
// kernel after the WHILE node, or launched on the stream after the graph,
// made every pass of a 16-slot serving mix markedly slower (p99 at 50k
// queries/s 13-14 ms against 8 ms with the branch).
template <int W>
int ms_build_exec(MsWorkspace* ws, MsArgs<W>& a) {
  MsPassDev*  d = static_cast<MsPassDev*>(ws->pass_dev);
  cudaGraph_t graph;
  NWG_CUDA_TRY(cudaGraphCreate(&graph, 0));
  auto fail = [&](cudaError_t e, const char* what) {
    cudaGraphDestroy(graph);
    return cuda_error(e, what);
  };
  cudaGraphNode_t* nodes = ws->nodes[W - 1];
  void*            argv[kNNodes][1];
  auto add = [&](cudaGraph_t gr, const cudaGraphNode_t* dep, int slot) {
    cudaKernelNodeParams kp = ms_node_params<W>(ws, a, slot, argv[slot]);
    return cudaGraphAddKernelNode(&nodes[slot], gr, dep, dep ? 1 : 0, &kp);
  };
  cudaError_t e;
  if ((e = add(graph, nullptr, kNRoots)) != cudaSuccess || (e = add(graph, &nodes[kNRoots], kNList)) != cudaSuccess)
    return fail(e, "multi-source graph nodes");
  cudaGraphConditionalHandle h_loop, h_sw[2];
  if ((e = cudaGraphConditionalHandleCreate(&h_loop, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess)
    return fail(e, "loop handle");
  cudaGraphNodeParams wp = {};
  wp.type                = cudaGraphNodeTypeConditional;
  wp.conditional.handle  = h_loop;
  wp.conditional.type    = cudaGraphCondTypeWhile;
  wp.conditional.size    = 1;
  cudaGraphNode_t n_while;
  if ((e = cudaGraphAddNode(&n_while, graph, &nodes[kNList], 1, &wp)) != cudaSuccess) return fail(e, "while node");
  cudaGraph_t     body = wp.conditional.phGraph_out[0];
  cudaGraphNode_t prev = nullptr;
  int             set_cond = 1;
  for (int half = 0; half < 2; ++half) {  // half 0: odd level (parity 1), half 1: even level (parity 0)
    if ((e = cudaGraphConditionalHandleCreate(&h_sw[half], body, 2, cudaGraphCondAssignDefault)) != cudaSuccess)
      return fail(e, "switch handle");
    void*                decargs[] = {&d, &h_loop, &h_sw[half], &set_cond};
    cudaKernelNodeParams dp        = {};
    dp.func                        = (void*)k_ms_decide;
    dp.gridDim                     = dim3(1);
    dp.blockDim                    = dim3(32);
    dp.kernelParams                = decargs;
    cudaGraphNode_t n_dec, n_sw;
    if ((e = cudaGraphAddKernelNode(&n_dec, body, prev ? &prev : nullptr, prev ? 1 : 0, &dp)) != cudaSuccess)
      return fail(e, "decide node");
    cudaGraphNodeParams sp = {};
    sp.type                = cudaGraphNodeTypeConditional;
    sp.conditional.handle  = h_sw[half];
    sp.conditional.type    = cudaGraphCondTypeSwitch;
    sp.conditional.size    = 3;
    if ((e = cudaGraphAddNode(&n_sw, body, &n_dec, 1, &sp)) != cudaSuccess) return fail(e, "switch node");
    const int push = half == 0 ? kNPush0 : kNPush1;
    if ((e = add(sp.conditional.phGraph_out[0], nullptr, push)) != cudaSuccess ||
        (e = add(sp.conditional.phGraph_out[0], &nodes[push], push + 1)) != cudaSuccess ||
        (e = add(sp.conditional.phGraph_out[1], nullptr, push + 2)) != cudaSuccess ||
        (e = add(sp.conditional.phGraph_out[2], nullptr, kNDepths0 + half)) != cudaSuccess)
      return fail(e, "level nodes");
    prev = n_sw;
  }
  cudaGraphExec_t exec;
  if ((e = cudaGraphInstantiate(&exec, graph, 0)) != cudaSuccess) return fail(e, "multi-source graph instantiate");
  if (ws->tmpl[W - 1]) cudaGraphDestroy(ws->tmpl[W - 1]);
  ws->tmpl[W - 1] = graph;  // kept: the nodes above belong to it
  ws->exec[W - 1] = exec;
  return NWG_OK;
}

// Points an instantiated pass graph at this pass's graph, depth rows and
// source masks; rebuilds it if the driver refuses the in-place update.  A
// pass with the same arguments as the previous one (same graph, source
// count and rows) skips the ten node updates, which cost more host time
// than a short pass takes on the device.
template <int W>
int ms_update_exec(MsWorkspace* ws, MsArgs<W>& a) {
  std::vector<unsigned char>& last = ws->last_args[W - 1];
  const unsigned char*        now  = reinterpret_cast<const unsigned char*>(&a);
  if (ws->exec[W - 1] && last.size() == sizeof a && std::memcmp(last.data(), now, sizeof a) == 0) return NWG_OK;
  last.clear();
  int rc = NWG_OK;
  if (!ws->exec[W - 1]) {
    rc = ms_build_exec<W>(ws, a);
  } else {
    void* argv[kNNodes][1];
    for (int slot = 0; slot < kNNodes; ++slot) {
      cudaKernelNodeParams kp = ms_node_params<W>(ws, a, slot, argv[slot]);
      if (cudaGraphExecKernelNodeSetParams(ws->exec[W - 1], ws->nodes[W - 1][slot], &kp) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphExecDestroy(ws->exec[W - 1]);
        ws->exec[W - 1] = nullptr;
        rc = ms_build_exec<W>(ws, a);
        break;
      }
    }
  }
  if (rc == NWG_OK) last.assign(now, now + sizeof a);
  return rc;
}

// Instantiates the pass graph of every word count up front (with arguments
// of an empty graph; each pass updates them), so no pass pays for it.
template <int W>
int ms_prepare(MsWorkspace* ws) {
  GraphDev  empty;
  empty.n = 0;
  empty.m = 0;
  MsArgs<W> a = ms_args<W>(&empty, ws, nullptr, 1, 0);
  return ms_build_exec<W>(ws, a);
}

// The same kernels launched one at a time, the decision read back by the
// host after each decide (for profilers that cannot see inside conditional
// graphs).
template <int W>
int ms_run_stepped(MsWorkspace* ws, MsArgs<W>& a, cudaStream_t stream) {
  MsPassDev* d  = static_cast<MsPassDev*>(ws->pass_dev);
  MsPassDev* hd = static_cast<MsPassDev*>(ws->pass_host);
  k_ms_roots<W><<<1, kMsThreads, 0, stream>>>(a.base);
  k_ms_root_list<W><<<1, kMsThreads, 0, stream>>>(a.base);
  const int g_list = grid_ms(ws, (const void*)k_ms_push<W>, ws->list_cap, kMsWarps);
  const int g_fin  = grid_ms(ws, (const void*)k_ms_finalize<W>, ws->n_cap, kMsThreads);
  const int g_pull = grid_ms(ws, (const void*)k_ms_pull<W>, ws->n_cap, kMsThreads);
  for (;;) {
    k_ms_decide<<<1, 32, 0, stream>>>(d, cudaGraphConditionalHandle{}, cudaGraphConditionalHandle{}, 0);
    NWG_CUDA_TRY(cudaGetLastError());
    NWG_CUDA_TRY(cudaMemcpyAsync(&hd->level, &d->level, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    NWG_CUDA_TRY(cudaMemcpyAsync(&hd->pull, &d->pull, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    NWG_CUDA_TRY(cudaStreamSynchronize(stream));
    if (hd->stopped) break;
    MsParams<W>& q = a.par[hd->level & 1];
    if (hd->pull) {
      k_ms_pull<W><<<g_pull, kMsThreads, 0, stream>>>(q);
    } else {
      k_ms_push<W><<<g_list, kMsThreads, 0, stream>>>(q);
      k_ms_finalize<W><<<g_fin, kMsThreads, 0, stream>>>(q);
    }
    NWG_CUDA_TRY(cudaGetLastError());
  }
  {
    const int rc = ms_depths_prepare<W>();
    if (rc) return rc;
  }
  k_ms_depths<W><<<grid_for(ws, ms_depths_occupancy<W>(), (a.base.n + kDtTile - 1) / kDtTile * W, 1), kMsThreads,
                   kDtSmem, stream>>>(a.base);
  NWG_CUDA_TRY(cudaGetLastError());
  return NWG_OK;
}

// One pass of up to 64 * W sources: the host writes the pass record (one
// copy from pinned memory), clears the state, launches the pass graph and
// reads the record back once at the end.  Every byte of the k depth rows is
// written by the pass's last kernel (no fill beforehand).
template <int W>
int ms_pass_launch(GraphDev* g, MsWorkspace* ws, const uint32_t* roots_host, uint32_t k, uint8_t* depth_rows,
                   uint32_t depth_bytes, int alpha, cudaStream_t stream, cudaEvent_t start_ev) {
  const uint64_t n  = g->n;
  MsPassDev&     h  = *static_cast<MsPassDev*>(ws->pass_host);
  MsPassDev*     dd = static_cast<MsPassDev*>(ws->pass_dev);
  std::memset(&h, 0, sizeof h);
  h.list_cap  = ws->list_cap;
  h.k         = k;
  h.alpha     = alpha;
  h.unchecked = g->m;
  h.sparse_max = std::max<uint64_t>(1024, n / 64);
  h.clear_max  = std::max<uint64_t>(1024, n / 8);
  std::memcpy(h.roots, roots_host, k * sizeof(uint32_t));
  // distinct roots form the first frontier; their chunk entries the first list
  std::vector<uint32_t> uniq(roots_host, roots_host + k);
  std::sort(uniq.begin(), uniq.end());
  uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
  h.nuniq = (uint32_t)uniq.size();
  std::memcpy(h.uniq, uniq.data(), uniq.size() * sizeof(uint32_t));

  MsArgs<W>    a     = ms_args<W>(g, ws, depth_rows, depth_bytes, k);
  const size_t words = (size_t)n * W * sizeof(uint64_t);
  if (!ws->stepped) {  // host work first, so the device work below runs back to back
    int rc = ms_update_exec<W>(ws, a);
    if (rc) return rc;
  }
  if (start_ev) NWG_CUDA_TRY(cudaEventRecord(start_ev, stream));
  NWG_CUDA_TRY(cudaMemsetAsync(ws->vis, 0, words, stream));
  NWG_CUDA_TRY(cudaMemsetAsync(ws->fr[0], 0, words, stream));
  NWG_CUDA_TRY(cudaMemsetAsync(ws->fr[1], 0, words, stream));  // a sparse first level writes only what it touches
  NWG_CUDA_TRY(cudaMemsetAsync(ws->nx, 0, words, stream));
  NWG_CUDA_TRY(cudaMemcpyAsync(dd, &h, sizeof h, cudaMemcpyHostToDevice, stream));
  if (ws->stepped) {
    int rc = ms_run_stepped<W>(ws, a, stream);
    if (rc) return rc;
  } else {
    NWG_CUDA_TRY(cudaGraphLaunch(ws->exec[W - 1], stream));
  }
  NWG_CUDA_TRY(cudaMemcpyAsync(&h, dd, sizeof h, cudaMemcpyDeviceToHost, stream));
  return NWG_OK;
}

// Waits for the pass launched on ws (on `stream`) and takes its record: the
// deep sources (indices within the pass) and the statistics.
int ms_pass_finish(MsWorkspace* ws, uint32_t k, std::vector<uint32_t>& deep, cudaStream_t stream,
                   nwg_msbfs_stats* st) {
  const MsPassDev& h = *static_cast<const MsPassDev*>(ws->pass_host);
  NWG_CUDA_TRY(cudaStreamSynchronize(stream));
  if (h.status == NWG_EOVERFLOW) {  // per source: the others' rows are complete
    for (uint32_t i = 0; i < k; ++i)
      if ((h.deep[i >> 6] >> (i & 63)) & 1ull) deep.push_back(i);
  } else if (h.status != NWG_OK) {
    return set_error(h.status, "multi-source pass failed");
  }
  st->levels = std::max(st->levels, h.levels);
  st->push_levels += h.push_levels;
  st->pull_levels += h.pull_levels;
  if (st->passes == 0) {
    st->trace_len = h.trace_len;
    for (uint32_t i = 0; i < h.trace_len; ++i) {
      st->trace_pull[i]           = h.tr_pull[i];
      st->trace_ms[i]             = (float)((double)(h.tr_t[i + 1] - h.tr_t[i]) * 1e-6);
      st->trace_frontier_edges[i] = h.tr_fedges[i];
      st->trace_discovered[i]     = h.tr_disc[i];
    }
  }
  return NWG_OK;
}

}  // namespace

uint64_t ms_ws_bytes(uint64_t n_cap, uint64_t m_cap) {
  const uint64_t n = std::max<uint64_t>(n_cap, 1);
  // VIS, FR[2], NX and the 8 level planes at four words per vertex, two
  // frontier lists (every frontier vertex has at most deg / kMsChunk + 1
  // entries), the pass record
  // plus the touched list and its bitmap
  return (4 + kMsPlanes) * n * 4 * sizeof(uint64_t) + 2 * (n + m_cap / kMsChunk + 1) * 8 + sizeof(MsPassDev) +
         4 * n + 4 * (n / 32 + 1);
}

int ms_ws_init_cap(GraphDev* g, uint64_t n_cap, uint64_t m_cap, MsWorkspace* ws) {
  const uint64_t n        = std::max<uint64_t>(n_cap, 1);
  const size_t   words    = (size_t)n * 4 * sizeof(uint64_t);  // room for W = 4
  const uint64_t list_cap = n + m_cap / kMsChunk + 1;
  ws->g                   = g;
  ws->n_cap               = n_cap;
  ws->m_cap               = m_cap;
  ws->list_cap            = list_cap;
  const char* stepped     = std::getenv("NWG_MS_STEPPED");
  ws->stepped             = stepped && stepped[0] == '1';
  int dev                 = 0;
  NWG_CUDA_TRY(cudaGetDevice(&dev));
  NWG_CUDA_TRY(cudaDeviceGetAttribute(&ws->sm_count, cudaDevAttrMultiProcessorCount, dev));
  if (cudaMalloc(&ws->vis, words) != cudaSuccess || cudaMalloc(&ws->fr[0], words) != cudaSuccess ||
      cudaMalloc(&ws->fr[1], words) != cudaSuccess || cudaMalloc(&ws->nx, words) != cudaSuccess ||
      cudaMalloc(&ws->dp, kMsPlanes * words) != cudaSuccess ||
      cudaMalloc(&ws->tlist, n * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&ws->tbits, (n / 32 + 1) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&ws->list[0], list_cap * 8) != cudaSuccess || cudaMalloc(&ws->list[1], list_cap * 8) != cudaSuccess ||
      cudaMalloc(&ws->pass_dev, sizeof(MsPassDev)) != cudaSuccess ||
      cudaMallocHost(&ws->pass_host, sizeof(MsPassDev)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(NWG_ENOMEM, "multi-source workspace allocation failed");
  }
  NWG_CUDA_TRY(cudaMemset(ws->dp, 0, kMsPlanes * words));  // the planes start (and end every pass) zero
  NWG_CUDA_TRY(cudaMemset(ws->tbits, 0, (n / 32 + 1) * sizeof(uint32_t)));  // so does T (every finalize clears it)
  NWG_CUDA_TRY(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
  NWG_CUDA_TRY(cudaEventCreate(&ws->ev0));
  NWG_CUDA_TRY(cudaEventCreate(&ws->ev1));
  NWG_CUDA_TRY(cudaEventCreateWithFlags(&ws->ev_fork, cudaEventDisableTiming));
  if (!ws->stepped) {
    int rc = ms_prepare<1>(ws);
    if (!rc) rc = ms_prepare<2>(ws);
    if (!rc) rc = ms_prepare<3>(ws);
    if (!rc) rc = ms_prepare<4>(ws);
    if (rc) return rc;
  }
  return NWG_OK;
}

int ms_ws_init(GraphDev* g, MsWorkspace* ws) { return ms_ws_init_cap(g, g->n, g->m, ws); }

void ms_ws_free(MsWorkspace* ws) {
  if (!ws) return;
  for (MsWorkspace* lane : ws->lanes) ms_ws_free(lane);
  ws->lanes.clear();
  if (ws->stream) cudaStreamSynchronize(ws->stream);
  for (cudaGraphExec_t e : ws->exec)
    if (e) cudaGraphExecDestroy(e);
  for (cudaGraph_t t : ws->tmpl)
    if (t) cudaGraphDestroy(t);
  cudaFree(ws->vis);
  cudaFree(ws->fr[0]);
  cudaFree(ws->fr[1]);
  cudaFree(ws->nx);
  cudaFree(ws->dp);
  cudaFree(ws->tlist);
  cudaFree(ws->tbits);
  cudaFree(ws->list[0]);
  cudaFree(ws->list[1]);
  cudaFree(ws->pass_dev);
  if (ws->pass_host) cudaFreeHost(ws->pass_host);
  if (ws->ev0) cudaEventDestroy(ws->ev0);
  if (ws->ev1) cudaEventDestroy(ws->ev1);
  if (ws->ev_fork) cudaEventDestroy(ws->ev_fork);
  if (ws->stream) cudaStreamDestroy(ws->stream);
  delete ws;
}

namespace {

int ms_launch_any(GraphDev* g, MsWorkspace* ws, const uint32_t* roots, uint32_t kk, uint8_t* rows,
                  uint32_t depth_bytes, int alpha, cudaStream_t s, cudaEvent_t start_ev) {
  if (kk <= 64) return ms_pass_launch<1>(g, ws, roots, kk, rows, depth_bytes, alpha, s, start_ev);
  if (kk <= 128) return ms_pass_launch<2>(g, ws, roots, kk, rows, depth_bytes, alpha, s, start_ev);
  if (kk <= 192) return ms_pass_launch<3>(g, ws, roots, kk, rows, depth_bytes, alpha, s, start_ev);
  return ms_pass_launch<4>(g, ws, roots, kk, rows, depth_bytes, alpha, s, start_ev);
}

constexpr uint32_t kMsLanes = 4;  // passes of one call in flight at once

}  // namespace

// Runs ceil(k / 256) passes of up to 256 sources over graph g, which must
// fit the workspace's capacity, into k rows of depth_bytes (1 or 2) per
// vertex.  The first pass runs on `stream` (or the workspace's own); with
// more than one pass, up to kMsLanes passes are in flight at once, each on
// a lane of its own (a second set of pass state and a stream, created on the
// first such call and kept), which overlaps one pass's latency-bound levels
// with the others'.  The lanes start after the work already on `stream`
// and `stream` waits for them, so the call keeps its stream order.
//
// A source whose traversal goes deeper than level 254 does not fail the
// pass: the other sources' rows are complete, and that source is counted in
// st->deep_sources and flagged in deep_flags[i] (k bytes; may be null).
// With uint16 rows its row is then computed exactly by one single-source
// traversal on a workspace made for the purpose and freed again (such
// sources are rare: a graph whose diameter passes 254); with uint8 rows it
// keeps the depths up to 254 and 255 beyond.
//
// start_ev and end_ev (either may be null) bracket the call's device work:
// start_ev is recorded on the stream after the first pass's host
// preparation, just before its first device operation, and end_ev once the
// device work is enqueued, before the host waits for the last passes'
// records (so it marks the end of the device work, not the host's wake-up).
int ms_run_on(MsWorkspace* ws, GraphDev* g, const uint32_t* roots_host, uint32_t k, void* depths_dev,
              uint32_t depth_bytes, uint8_t* deep_flags, int alpha, cudaStream_t stream, nwg_msbfs_stats* st,
              cudaEvent_t end_ev, cudaEvent_t start_ev) {
  if (g->n > ws->n_cap || g->m > ws->m_cap)
    return set_error(NWG_EINVAL, "graph larger than the multi-source workspace's capacity");
  for (uint32_t i = 0; i < k; ++i)
    if (roots_host[i] >= g->n) return set_error(NWG_EINVAL, "root " + std::to_string(roots_host[i]) + " >= n");
  if (alpha <= 0) return set_error(NWG_EINVAL, "alpha must be positive");
  if (depth_bytes != 1 && depth_bytes != 2) return set_error(NWG_EINVAL, "depth rows must have 1 or 2 bytes per vertex");
  if (deep_flags) std::memset(deep_flags, 0, k);
  cudaStream_t   s       = stream ? stream : ws->stream;
  const uint32_t npasses = (k + 255) / 256;
  const uint32_t nlanes  = std::min(npasses, kMsLanes);
  // lane 0 is the workspace itself on `s`; the others wait for `s`'s prior work
  while (ws->lanes.size() + 1 < nlanes) {
    auto* lane = new (std::nothrow) MsWorkspace();
    if (!lane) return set_error(NWG_ENOMEM, "host allocation failed");
    const int rc = ms_ws_init_cap(ws->g, ws->n_cap, ws->m_cap, lane);
    if (rc) {
      ms_ws_free(lane);
      return rc;
    }
    ws->lanes.push_back(lane);
  }
  auto lane_ws     = [&](uint32_t l) { return l == 0 ? ws : ws->lanes[l - 1]; };
  auto lane_stream = [&](uint32_t l) { return l == 0 ? s : ws->lanes[l - 1]->stream; };
  if (nlanes > 1) {
    NWG_CUDA_TRY(cudaEventRecord(ws->ev_fork, s));
    for (uint32_t l = 1; l < nlanes; ++l) NWG_CUDA_TRY(cudaStreamWaitEvent(lane_stream(l), ws->ev_fork, 0));
  }
  std::vector<uint32_t> deep;
  Workspace*            single = nullptr;  // single-source traversals of deep sources (uint16 rows only)
  int                   rc     = NWG_OK;
  auto rows_of = [&](uint32_t p) {
    return static_cast<uint8_t*>(depths_dev) + (uint64_t)p * 256 * g->n * depth_bytes;
  };
  // pass p runs on lane p % nlanes; before a lane takes a pass it finishes
  // its previous one (p - nlanes), so passes finish in order
  auto finish = [&](uint32_t p) -> int {
    const uint32_t l  = p % nlanes;
    const uint32_t kk = std::min<uint32_t>(256, k - 256 * p);
    deep.clear();
    int r = ms_pass_finish(lane_ws(l), kk, deep, lane_stream(l), st);
    if (r) return r;
    st->passes++;
    for (uint32_t i : deep) {
      st->deep_sources++;
      if (deep_flags) deep_flags[256 * p + i] = 1;
      if (depth_bytes != 2) continue;
      if (!single) {
        single = new (std::nothrow) Workspace();
        if (!single) return set_error(NWG_ENOMEM, "host allocation failed");
        if ((r = ws_init(g, single)) != NWG_OK) return r;
      }
      r = depth_row16(single, roots_host[256 * p + i], reinterpret_cast<uint16_t*>(rows_of(p)) + (uint64_t)i * g->n,
                      lane_stream(l));
      if (r) return r;
    }
    return NWG_OK;
  };
  uint32_t done = 0;  // passes finished
  for (uint32_t p = 0; p < npasses && rc == NWG_OK; ++p) {
    if (p >= nlanes && (rc = finish(done++)) != NWG_OK) break;
    const uint32_t l  = p % nlanes;
    const uint32_t kk = std::min<uint32_t>(256, k - 256 * p);
    rc = ms_launch_any(g, lane_ws(l), roots_host + 256 * p, kk, rows_of(p), depth_bytes, alpha, lane_stream(l),
                       p == 0 ? start_ev : nullptr);
  }
  auto join = [&]() {  // `s` continues after every lane's work
    for (uint32_t l = 1; l < nlanes; ++l) {
      cudaEventRecord(ws->lanes[l - 1]->ev0, lane_stream(l));
      cudaStreamWaitEvent(s, ws->lanes[l - 1]->ev0, 0);
    }
    if (end_ev) cudaEventRecord(end_ev, s);
  };
  join();
  while (done < npasses) {  // after an error, what was launched still completes before the call returns
    const int r = finish(done++);
    if (rc == NWG_OK) rc = r;
  }
  if (single) {  // uint16 rows of deep sources were computed after the passes
    join();
    ws_free(single);
  }
  return rc;
}

int ms_run(MsWorkspace* ws, const uint32_t* roots_host, uint32_t k, void* depths_dev, uint32_t depth_bytes,
           uint8_t* deep_flags, int alpha, cudaStream_t stream, nwg_msbfs_stats* st, cudaEvent_t end_ev,
           cudaEvent_t start_ev) {
  return ms_run_on(ws, ws->g, roots_host, k, depths_dev, depth_bytes, deep_flags, alpha, stream, st, end_ev,
                   start_ev);
}

}  // namespace nwg
