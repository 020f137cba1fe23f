// Direction-optimizing BFS on sm_100a: the device level loop.
//
// Restates nw::graph::bfs(out, in, root, num_bins, alpha, beta)
// (include/nwgraph/algorithms/bfs.hpp:160-311 in NWGraph) as one persistent
// cooperative kernel, k_trav: init, then per step a decision and one action
// (top-down step, bottom-up pull, or bitmap -> queue), with a grid barrier
// between steps and no host round trip.
//
// The decision (decide_on) reproduces the reference's integer switch rules
// exactly (scout_count > edges_to_check / alpha selects bottom-up,
// bfs.hpp:186; stay bottom-up while awake >= old_awake or awake > N / beta,
// bfs.hpp:229; scout_count = 1 after a bottom-up phase, bfs.hpp:241; stop
// when the next queue is empty, bfs.hpp:297-303, or a pull finds nothing,
// bfs.hpp:231-233).
//
// The same steps also run as separate kernels driven from the host (k_init,
// k_decide, k_td, k_bu, k_b2q, and k_td_loop / k_td_cluster for runs of
// small top-down levels): the host-stepped traversal that profilers see
// kernel by kernel and that the entry point without allocation uses; and
// per block in k_ragged, one whole traversal per block.
//
// Device state (HBM):
//   parents[n]   output; null = 0xFFFFFFFF
//   V[n/32]      visited bitmap.  The top-down step sets a vertex's bit with
//                atomicOr when it claims it (this is the queue->bitmap
//                conversion of bfs.hpp:199-202, fused into the step that
//                fills the queue), and the claim decides which discoverer
//                writes parents[v] (the CAS of bfs.hpp:283).
//   C0/C1[n/32]  discoveries of the latest bottom-up pulls (bfs.hpp:205-229's
//                front/curr pair).
//   Z[n/32]      vertices with no in-edges, never candidates of a pull.
//   qs[2], qc[2] frontier queues: small-degree vertex ids, and 256-edge
//                chunks of every other vertex (instead of the reference's
//                u % 32 bins).
//
// Bottom-up front: the first pull of a phase uses V itself as the front
// bitmap.  V holds the frontier plus all earlier levels; an earlier-level
// vertex can never be an in-neighbour of a vertex that is still unvisited
// (the top-down step that expanded it would have claimed that vertex), so a
// pull over V finds exactly the in-neighbours a pull over the frontier
// bitmap finds, in the same row order.  The reference's own front bitmap
// also carries such stale bits (curr is not cleared after bitmap->queue,
// bfs.hpp:235-239).  Later pulls of the phase use the previous pull's C.
#include <algorithm>
#include <cooperative_groups.h>

#include "nwg_internal.cuh"

namespace nwg {
namespace {

constexpr int kThreads     = 256;
constexpr int kWarps       = kThreads / 32;
constexpr int kBuProbe     = 4;   // in-edges a lane tests per round (independent loads)
constexpr int kBuLane      = 32;  // in-edges a lane scans alone before the warp helps
constexpr int kTileWords   = 16;  // bitmap words per warp tile of the bitmap->queue pass (512 vertices; <= 32)
constexpr int kBuTileWords = 16;  // bitmap words per pull tile (512 vertices; <= 32)
constexpr int kSmallBlocks = 64;  // grid of the small-frontier top-down branch
constexpr int kClusterCtas = 8;   // the tiny-frontier branch: one cluster of this many blocks
constexpr int kClusterUnits = kClusterCtas * (kThreads / 32);  // its work-unit limit: one per warp
constexpr int kVisit       = 4;   // edges a lane claims per batch
constexpr int kTdPerSm     = 4;   // k_td blocks per SM (64 registers per thread, no spills: 3% faster than 3 on the grid)
// Solo levels of the persistent traversal kernel (block 0 alone): at most
// this many frontier out-edges (so a level's discoveries fit a shared list;
// one SM's loads and claims in flight bound it: a level of 2,000 edges took
// 27 us alone against 15 us on the grid, one of 1,000 8 us), and at most
// kSoloLevels levels per turn (the other blocks' wait).
constexpr uint32_t kSoloCap    = 1024;
constexpr uint32_t kSoloLevels = 256;
constexpr uint32_t kSoloPer    = kSoloCap / kThreads;  // list entries per thread in the prefix pass

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
  const unsigned lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T x = __shfl_up_sync(kFullMask, v, o);
    if ((int)lane >= o) v += x;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T block_sum(T v) {
  __shared__ T red[32];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
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

__host__ __device__ __forceinline__ uint64_t chunks_of(uint64_t deg, const Thresholds& t) {
  return (deg + t.chunk - 1) >> t.chunk_shift;
}

constexpr uint64_t kLaneChunks = 8;  // a lane writes up to this many chunk entries of one vertex itself

// What one step of the traversal reads and where it adds its counts.  The
// level-loop kernels take it from the control header; the persistent
// traversal kernel from its own copy of the decision state and the step's
// counter slot.
struct StepView {
  uint32_t*           parents;
  uint32_t            in;       // queue buffer a top-down step expands
  uint32_t            out;      // queue buffer a step appends to
  uint64_t            nS, nC;   // small and chunk entries of the input queues
  uint32_t            bu_mode;  // pull: 0 = front is V, 1 = front is the previous pull's discoveries
  uint32_t            bm;       // pull: index of the discovery bitmap of the previous pull
  unsigned long long* qpos;     // output queues' entries: small | chunk << 32
  uint32_t*           qbig;     // chunked vertices appended
  uint32_t*           nhub;     // deferred hub records appended
  unsigned long long* scout;    // out-degree sum of the vertices a top-down step discovers
  unsigned long long* awake;    // vertices a pull discovers
  uint32_t*           mark;     // top-down step: NULL = queue the discoveries, else set their bits here
  uint32_t            mark_deg; // marking step: also sum the discoveries' out-degrees into scout
};

// ---------------------------------------------------------------------------
// Appending discovered vertices to the next queue buffer `qi`.
//
// A lane holds K vertices (mask bit k set = v[k] valid) with their
// out-degrees.  Small-degree vertices take one small-queue slot, the others
// chunks_of(d) chunk-queue slots.  Space in both queues is reserved with ONE
// 64-bit atomicAdd on the packed position counter qpos[qi] per warp
// (append_warp, a warp's buffer ran full) or per block (append_block, the
// end-of-kernel flush): same-address atomics serialise in L2, so their
// number, not the bytes written, bounds a step that discovers millions of
// vertices.  The chunk entries of each chunked vertex are written by the
// whole warp, 32 at a time.
template <int K>
__device__ __forceinline__ void count_entries(const DobfsParams& p, const uint64_t (&d)[K], uint32_t mask,
                                              uint32_t& ns, uint32_t& nch, uint32_t& nb) {
  ns = nch = nb = 0;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (mask & (1u << k)) {
      if (d[k] < p.th.warp_min) {
        ++ns;
      } else {
        ++nb;
        nch += (uint32_t)chunks_of(d[k], p.th);
      }
    }
  }
}

// All 32 lanes of the warp must call.  Small entries and the chunk entries
// of vertices with at most kLaneChunks chunks are written by their own lane.
// Hubs (more chunks): with kDefer and hub-record buffers, the warp only
// records (vertex, first slot, chunk count) -- one atomic per warp -- and the
// persistent kernel's whole grid writes their entries after the level
// barrier (expand_hubs); a single SM writing tens of thousands of entries is
// bound by its outstanding-store limit.  Otherwise the whole warp writes them,
// 32 at a time.
template <int K, bool kDefer>
__device__ __forceinline__ void write_entries(const DobfsParams& p, const StepView& sv, const uint32_t (&v)[K],
                                              const uint64_t (&d)[K], uint32_t mask, uint64_t spos, uint64_t cpos) {
  const uint32_t  qi   = sv.out;
  const unsigned  lane = threadIdx.x & 31;
  uint32_t* const qs   = p.qs[qi];
  uint64_t* const qc   = p.qc[qi];
  const uint64_t  scap = p.qs_cap, ccap = p.qc_cap;
  const uint64_t  c0   = cpos;
  bool            over = false;
  bool            hub  = false;
  uint32_t        nh   = 0;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!(mask & (1u << k))) continue;
    if (d[k] < p.th.warp_min) {
      if (spos < scap) {
        qs[spos] = v[k];
      } else {
        over = true;
      }
      ++spos;
    } else {
      const uint64_t nc = chunks_of(d[k], p.th);
      if (nc <= kLaneChunks) {
        for (uint64_t j = 0; j < nc; ++j) {
          if (cpos + j < ccap) {
            qc[cpos + j] = ((uint64_t)v[k] << 32) | j;
          } else {
            over = true;
          }
        }
      } else {
        hub = true;
        ++nh;
      }
      cpos += nc;
    }
  }
  HubRec* const rec = kDefer ? p.hubrec[qi] : nullptr;
  if (kDefer && rec != nullptr) {  // uniform: the buffers exist or not
    uint32_t incl = nh;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t x = __shfl_up_sync(kFullMask, incl, o);
      if ((int)lane >= o) incl += x;
    }
    const uint32_t tot  = __shfl_sync(kFullMask, incl, 31);
    uint32_t       base = 0;
    if (tot && lane == 31) base = atomicAdd(sv.nhub, tot);
    base         = __shfl_sync(kFullMask, base, 31);
    uint64_t idx = base + incl - nh;
    uint64_t pos = c0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!(mask & (1u << k)) || d[k] < p.th.warp_min) continue;
      const uint64_t nc = chunks_of(d[k], p.th);
      if (nc > kLaneChunks) {
        if (idx < p.hub_cap) {
          rec[idx] = HubRec{v[k], (uint32_t)nc, pos};
        } else {
          over = true;
        }
        ++idx;
      }
      pos += nc;
    }
  } else {
    unsigned todo = __ballot_sync(kFullMask, hub);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      uint64_t pos = __shfl_sync(kFullMask, c0, src);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const unsigned valid = __shfl_sync(kFullMask, (mask >> k) & 1u, src);
        const uint64_t dk    = __shfl_sync(kFullMask, d[k], src);
        if (valid && dk >= p.th.warp_min) {
          const uint64_t nc = chunks_of(dk, p.th);
          if (nc > kLaneChunks) {
            const uint32_t vk = __shfl_sync(kFullMask, v[k], src);
            for (uint64_t j = lane; j < nc; j += 32) {
              if (pos + j < ccap) {
                qc[pos + j] = ((uint64_t)vk << 32) | j;
              } else {
                over = true;
              }
            }
          }
          pos += nc;
        }
      }
    }
  }
  if (over) atomicCAS(&p.ctrl->err, 0, NWG_EOVERFLOW);
}

template <int K, bool kDefer>
__device__ __forceinline__ void append_warp(const DobfsParams& p, const StepView& sv, const uint32_t (&v)[K],
                                            const uint64_t (&d)[K], uint32_t mask, uint32_t& nbig) {
  uint32_t ns, nch, nb;
  count_entries<K>(p, d, mask, ns, nch, nb);
  nbig += nb;
  const unsigned long long mine = (unsigned long long)ns | ((unsigned long long)nch << 32);
  const unsigned long long incl = warp_incl_scan(mine);
  const unsigned long long tot  = __shfl_sync(kFullMask, incl, 31);
  if (tot == 0) return;
  unsigned long long base = 0;
  if ((threadIdx.x & 31) == 31) base = atomicAdd(sv.qpos, tot);
  base                          = __shfl_sync(kFullMask, base, 31);
  const unsigned long long excl = incl - mine;
  write_entries<K, kDefer>(p, sv, v, d, mask, (base & 0xFFFFFFFFull) + (excl & 0xFFFFFFFFull),
                           (base >> 32) + (excl >> 32));
}

// Exclusive block-wide scan of a 64-bit value; all threads call.
__device__ __forceinline__ unsigned long long block_excl_scan(unsigned long long x, unsigned long long& total) {
  __shared__ unsigned long long s_w[kWarps];
  __shared__ unsigned long long s_p[kWarps];
  const unsigned                lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const unsigned long long      inc  = warp_incl_scan(x);
  if (lane == 31) s_w[wib] = inc;
  __syncthreads();
  if (wib == 0) {
    const unsigned long long t  = lane < kWarps ? s_w[lane] : 0ull;
    const unsigned long long ti = warp_incl_scan(t);
    if (lane < kWarps) s_p[lane] = ti;
  }
  __syncthreads();
  total                         = s_p[kWarps - 1];
  const unsigned long long excl = (wib ? s_p[wib - 1] : 0ull) + inc - x;
  __syncthreads();
  return excl;
}

template <int K, bool kDefer>
__device__ __forceinline__ void append_block(const DobfsParams& p, const StepView& sv, const uint32_t (&v)[K],
                                             const uint64_t (&d)[K], uint32_t mask, uint32_t& nbig) {
  __shared__ unsigned long long s_base;
  uint32_t                      ns, nch, nb;
  count_entries<K>(p, d, mask, ns, nch, nb);
  nbig += nb;
  const unsigned long long mine = (unsigned long long)ns | ((unsigned long long)nch << 32);
  unsigned long long       tot  = 0;
  const unsigned long long excl = block_excl_scan(mine, tot);
  if (tot == 0) return;  // block-uniform
  if (threadIdx.x == 0) s_base = atomicAdd(sv.qpos, tot);
  __syncthreads();
  const unsigned long long base = s_base;
  write_entries<K, kDefer>(p, sv, v, d, mask, (base & 0xFFFFFFFFull) + (excl & 0xFFFFFFFFull),
                           (base >> 32) + (excl >> 32));
  __syncthreads();
}

// Per-warp shared state of the top-down step: the ranges of the current
// gather group (owner search) and a buffer of claimed vertices whose degree
// lookup and queue append are done in bulk.
constexpr int kWinBuf = 256;
struct TdWarp {
  uint32_t vexcl[33];  // exclusive prefix of the ranges' aligned-body vector counts; [32] = total
  uint32_t sexcl[33];  // exclusive prefix of the ranges' head + tail edge counts; [32] = total
  uint32_t u[32];      // source vertex of each range
  uint32_t nhead[32];  // head length (edges before the first 16-byte boundary)
  uint64_t lo[32];     // first edge of the range
  uint64_t al[32];     // first edge of the aligned body
  uint64_t ah[32];     // end of the aligned body (= start of the tail)
  uint32_t win[kWinBuf];
};

// Shared memory of the step functions in one block.  A top-down step uses
// tw, bitmap -> queue uses tw and list, a pull uses PullSmem; a kernel that
// runs more than one kind of step overlays the two (StepShared), since no
// two steps run at once.
struct TdSmem {
  TdWarp   tw[kWarps];
  uint16_t list[kWarps][kTileWords * 32];  // bitmap -> queue: one tile's set bits (local vertex indices)
};
struct PullSmem {
  uint16_t cand[kWarps][kBuTileWords * 32];  // a tile's candidates (local vertex indices)
  uint32_t fresh[kWarps][kBuTileWords];      // a tile's discoveries
};
// Solo levels (k_trav, block 0 alone): the frontier and the next one as
// vertex lists, and the exclusive prefix of the frontier's out-degrees.
struct SoloSmem {
  uint32_t q[2][kSoloCap];
  uint32_t pre[kSoloCap + 1];
  uint32_t cnt;
  uint32_t nhub;
};
union StepShared {
  TdSmem   td;
  PullSmem pull;
  SoloSmem solo;
};

// Out-degrees of the valid v[k]: the 2-byte saturated copy (a 33 MB array at
// 2^24 vertices, which stays mostly in L2, where the offsets take 134 MB),
// and the offsets only for saturated entries.  All loads are issued first.
template <int K>
__device__ __forceinline__ void out_degrees(const DobfsParams& p, const uint32_t (&v)[K], uint32_t mask,
                                            uint64_t (&d)[K]) {
  uint32_t d16[K];
#pragma unroll
  for (int k = 0; k < K; ++k) d16[k] = ((mask & (1u << k)) && p.deg16) ? (uint32_t)__ldg(p.deg16 + v[k]) : 0xFFFFu;
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (mask & (1u << k)) d[k] = d16[k] != 0xFFFFu ? (uint64_t)d16[k] : p.off[v[k] + 1] - p.off[v[k]];
}

// A warp's winner buffer ran full: degree lookup and append of its entries
// (all 32 lanes call).
template <bool kDefer>
__device__ __forceinline__ void flush_winners(const DobfsParams& p, const StepView& sv, TdWarp& tw, uint32_t& wcnt,
                                              unsigned long long& scout, uint32_t& nbig) {
  const unsigned lane = threadIdx.x & 31;
  __syncwarp();
  for (uint32_t r = 0; r < wcnt; r += 32 * kVisit) {
    uint32_t v[kVisit];
    uint64_t d[kVisit];
    uint32_t mask = 0;
#pragma unroll
    for (int k = 0; k < kVisit; ++k) {
      const uint32_t i = r + k * 32 + lane;
      v[k]             = 0;
      d[k]             = 0;
      if (i < wcnt) {
        v[k] = tw.win[i];
        mask |= 1u << k;
      }
    }
    out_degrees<kVisit>(p, v, mask, d);
#pragma unroll
    for (int k = 0; k < kVisit; ++k) scout += d[k];
    append_warp<kVisit, kDefer>(p, sv, v, d, mask, nbig);
  }
  wcnt = 0;
  __syncwarp();
}

// End of a step: every warp's remaining buffered winners are appended with
// one reservation for the whole block.  All threads of the block call.
template <bool kDefer>
__device__ __forceinline__ void flush_block(const DobfsParams& p, const StepView& sv, TdWarp* tws, uint32_t wcnt,
                                            unsigned long long& scout, uint32_t& nbig, bool count_scout) {
  __shared__ uint32_t s_cnt[kWarps];
  if ((threadIdx.x & 31) == 0) s_cnt[threadIdx.x >> 5] = wcnt;
  __syncthreads();
  uint32_t v[kWarps];
  uint64_t d[kWarps];
  uint32_t mask = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    v[w] = 0;
    d[w] = 0;
    if (threadIdx.x < s_cnt[w]) {
      v[w] = tws[w].win[threadIdx.x];
      mask |= 1u << w;
    }
  }
  out_degrees<kWarps>(p, v, mask, d);
  if (count_scout) {
#pragma unroll
    for (int w = 0; w < kWarps; ++w) scout += d[w];
  }
  append_block<kWarps, kDefer>(p, sv, v, d, mask, nbig);
}

// One batch of top-down edge tests (bfs.hpp:280-289): lane edges u[k] -> v[k]
// for the valid k.  Every V word is read first (independent loads, through L1:
// bits only ever go from 0 to 1, so a stale word can only cost an extra
// atomic, never a wrong claim), then the unvisited ones are claimed with
// atomicOr (all issued before any result is used).  A claim's winner writes parents[v] = u (the reference's CAS
// winner) and is buffered; scout and the next queue are updated when the
// buffer is flushed.  In a marking step (kMark; sv.mark) the winner instead
// sets its bit in sv.mark and counts itself in `nbig`, which such a step
// adds to the awake count; a marking top-down step (sv.mark_deg) adds its
// out-degree to `scout` as well.  All 32 lanes must call.
template <bool kDefer, bool kMark = false>
__device__ __forceinline__ void visit_batch(const DobfsParams& p, const StepView& sv, const uint32_t (&u)[kVisit],
                                            const uint32_t (&v)[kVisit], uint32_t valid, TdWarp& tw, uint32_t& wcnt,
                                            unsigned long long& scout, uint32_t& nbig) {
  uint32_t* __restrict__ parents = sv.parents;
  uint32_t w[kVisit];
#pragma unroll
  for (int k = 0; k < kVisit; ++k) w[k] = (valid & (1u << k)) ? p.V[v[k] >> 5] : ~0u;
  uint32_t old[kVisit];
  uint32_t try_mask = 0;
#pragma unroll
  for (int k = 0; k < kVisit; ++k) {
    const uint32_t bit = 1u << (v[k] & 31);
    old[k]             = ~0u;
    if (!(w[k] & bit)) {
      old[k] = atomicOr(p.V + (v[k] >> 5), bit);
      try_mask |= 1u << k;
    }
  }
  uint32_t win = 0;
#pragma unroll
  for (int k = 0; k < kVisit; ++k)
    if ((try_mask & (1u << k)) && !(old[k] & (1u << (v[k] & 31)))) win |= 1u << k;
  const uint32_t cnt = __popc(win);
  if (kMark) {  // marking step: the bit is the discovery record; no queue entry
#pragma unroll
    for (int k = 0; k < kVisit; ++k) {
      if (win & (1u << k)) {
        parents[v[k]] = u[k];
        atomicOr(sv.mark + (v[k] >> 5), 1u << (v[k] & 31));
      }
    }
    nbig += cnt;  // discoveries
    if (sv.mark_deg) {  // a marking top-down step also sums their out-degrees (bfs.hpp:286)
      uint64_t d[kVisit];
      out_degrees<kVisit>(p, v, win, d);
#pragma unroll
      for (int k = 0; k < kVisit; ++k)
        if (win & (1u << k)) scout += d[k];
    }
    return;
  }
  const uint32_t inc = warp_incl_scan(cnt);
  const uint32_t tot = __shfl_sync(kFullMask, inc, 31);
  if (tot == 0) return;
  uint32_t pos = wcnt + inc - cnt;
#pragma unroll
  for (int k = 0; k < kVisit; ++k) {
    if (win & (1u << k)) {
      parents[v[k]] = u[k];
      tw.win[pos++] = v[k];
    }
  }
  wcnt += tot;
  if (wcnt > kWinBuf - 32 * kVisit) flush_winners<kDefer>(p, sv, tw, wcnt, scout, nbig);
}

// Largest range index whose exclusive prefix (in `excl`) is <= e.
__device__ __forceinline__ int owner_of(const uint32_t* excl, uint32_t e) {
  int lo = 0;
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1)
    if (excl[lo + s] <= e) lo += s;
  return lo;
}

// Expands up to 32 edge ranges at once (lane i holds range i: source u,
// edges [lo, hi); lo == hi = none).  Each range splits into an unaligned head,
// a 16-byte-aligned body and a tail.  The bodies of all ranges are flattened
// by a warp scan and dealt out one 128-bit non-coherent load (4 edges of one
// range) per lane per batch; the heads and tails (< 4 edges each) are dealt
// out as scalar edges, kVisit per lane per batch.  A unit's range is found by
// binary search over the prefix in shared memory.  All 32 lanes must call.
template <bool kDefer, bool kMark = false>
__device__ __forceinline__ void gather_ranges(const DobfsParams& p, const StepView& sv, uint32_t u, uint64_t lo,
                                              uint64_t hi, TdWarp& tw, uint32_t& wcnt, unsigned long long& scout,
                                              uint32_t& nbig) {
  const unsigned lane = threadIdx.x & 31;
  const uint64_t al   = min(hi, (lo + 3) & ~(uint64_t)3);
  const uint64_t ah   = max(al, hi & ~(uint64_t)3);
  const uint32_t nvec = (uint32_t)((ah - al) >> 2);
  const uint32_t nsc  = (uint32_t)((al - lo) + (hi - ah));
  const uint32_t vinc = warp_incl_scan(nvec);
  const uint32_t sinc = warp_incl_scan(nsc);
  const uint32_t vtot = __shfl_sync(kFullMask, vinc, 31);
  const uint32_t stot = __shfl_sync(kFullMask, sinc, 31);
  if (vtot == 0 && stot == 0) return;
  tw.vexcl[lane] = vinc - nvec;
  tw.sexcl[lane] = sinc - nsc;
  tw.u[lane]     = u;
  tw.nhead[lane] = (uint32_t)(al - lo);
  tw.lo[lane]    = lo;
  tw.al[lane]    = al;
  tw.ah[lane]    = ah;
  if (lane == 31) {
    tw.vexcl[32] = vtot;
    tw.sexcl[32] = stot;
  }
  __syncwarp();
  const uint4* col4 = reinterpret_cast<const uint4*>(p.col);
  for (uint32_t j = 0; j < vtot; j += 32) {
    const uint32_t e  = j + lane;
    uint32_t       uu[kVisit] = {0, 0, 0, 0}, vv[kVisit] = {0, 0, 0, 0}, valid = 0;
    if (e < vtot) {
      const int   o = owner_of(tw.vexcl, e);
      const uint4 x = __ldg(col4 + ((tw.al[o] >> 2) + (e - tw.vexcl[o])));
      uu[0] = uu[1] = uu[2] = uu[3] = tw.u[o];
      vv[0] = x.x;
      vv[1] = x.y;
      vv[2] = x.z;
      vv[3] = x.w;
      valid = 0xFu;
    }
    visit_batch<kDefer, kMark>(p, sv, uu, vv, valid, tw, wcnt, scout, nbig);
  }
  for (uint32_t j = 0; j < stot; j += 32 * kVisit) {
    uint32_t uu[kVisit], vv[kVisit], valid = 0;
#pragma unroll
    for (int k = 0; k < kVisit; ++k) {
      const uint32_t e = j + k * 32 + lane;
      uu[k]            = 0;
      vv[k]            = 0;
      if (e < stot) {
        const int      o = owner_of(tw.sexcl, e);
        const uint32_t t = e - tw.sexcl[o];
        const uint64_t i = t < tw.nhead[o] ? tw.lo[o] + t : tw.ah[o] + (t - tw.nhead[o]);
        uu[k]            = tw.u[o];
        vv[k]            = __ldg(p.col + i);
        valid |= 1u << k;
      }
    }
    visit_batch<kDefer, kMark>(p, sv, uu, vv, valid, tw, wcnt, scout, nbig);
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// k_init: parents := null except root (bfs.hpp:175,180), V := {root},
// control block := the reference's initial state (bfs.hpp:166-181).
// reset_barrier: clear the grid barrier's arrival count (not in a kernel
// whose blocks may already be waiting at that barrier).
__device__ __forceinline__ void init_step(const DobfsParams& p, uint32_t root, uint32_t alpha, uint32_t beta,
                                          uint32_t* parents, uint32_t topdown_only, uint32_t block, uint32_t nblocks,
                                          bool reset_barrier = true) {
  const uint64_t n      = p.n;
  const uint64_t tid    = (uint64_t)block * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)nblocks * blockDim.x;
  if ((reinterpret_cast<uintptr_t>(parents) & 15) == 0) {
    const uint64_t n4 = n >> 2;
    uint4*         p4 = reinterpret_cast<uint4*>(parents);
    const uint64_t r4 = root >> 2;
    for (uint64_t i = tid; i < n4; i += stride) {
      uint4 v = make_uint4(kNull, kNull, kNull, kNull);
      if (i == r4) {
        switch (root & 3) {
          case 0: v.x = root; break;
          case 1: v.y = root; break;
          case 2: v.z = root; break;
          default: v.w = root; break;
        }
      }
      p4[i] = v;
    }
    for (uint64_t i = (n4 << 2) + tid; i < n; i += stride) parents[i] = (i == root) ? root : kNull;
  } else {
    for (uint64_t i = tid; i < n; i += stride) parents[i] = (i == root) ? root : kNull;
  }
  const uint32_t rw = root >> 5;
  for (uint64_t w = tid; w < p.nwords; w += stride) p.V[w] = (w == rw) ? (1u << (root & 31)) : 0u;
  {  // a hub root's chunk entries, written by the whole grid
    const uint64_t rdeg = p.off[root + 1] - p.off[root];
    if (rdeg >= p.th.warp_min) {
      const uint64_t nc = chunks_of(rdeg, p.th);
      for (uint64_t j = tid; j < nc && j < p.qc_cap; j += stride) p.qc[0][j] = ((uint64_t)root << 32) | j;
    }
  }

  if (tid == 0) {
    CtrlHdr&       c   = p.ctrl->h;
    const uint64_t deg = p.off[root + 1] - p.off[root];
    c.parents          = parents;
    c.root             = root;
    c.alpha            = alpha;
    c.beta             = beta;
    c.topdown_only     = topdown_only;
    c.edges_to_check   = p.m;
    c.scout_count      = deg;
    c.awake_count      = 0;
    c.old_awake        = 0;
    c.acc_scout        = 0;
    c.acc_awake        = 0;
    c.qpos[0] = c.qpos[1] = 0;
    c.qbig[0] = c.qbig[1] = 0;
    if (deg < p.th.warp_min) {
      p.qs[0][0] = root;
      c.qpos[0]  = 1;
    } else {
      c.qpos[0] = chunks_of(deg, p.th) << 32;  // entries written above
      c.qbig[0] = 1;
    }
    c.nhub[0] = c.nhub[1] = 0;
    c.cur       = 0;
    c.bm        = 1;
    c.bu_mode   = 0;
    c.action    = kActNone;
    c.steps     = 0;
    c.levels    = 1;
    c.td_steps  = 0;
    c.bu_steps  = 0;
    c.b2q_steps = 0;
    c.status      = 0;
    c.pre_decided = 0;
    c.bu_push     = 0;
    if (reset_barrier) p.ctrl->bar.count = 0;
    p.ctrl->err       = 0;
    p.ctrl->decides   = 0;
    p.ctrl->kernels   = 0;
    c.reached     = 1;
    c.t_start     = globaltimer();
    c.trace_len = 0;
    c.scout_exact = 1;  // scout_count = the root's out-degree
    c.prev_small  = 0;
    c.mark_ok     = 0;
    c.b2q_then_td = 0;
    const uint64_t cap = 2 * n + 64;
    c.max_steps = cap > 0xFFFFFF00ull ? 0xFFFFFF00u : (uint32_t)cap;
  }
}

__global__ void __launch_bounds__(kThreads) k_init(DobfsParams p, uint32_t root, uint32_t alpha, uint32_t beta,
                                                   uint32_t* parents, uint32_t topdown_only) {
  init_step(p, root, alpha, beta, parents, topdown_only, blockIdx.x, gridDim.x);
}

__device__ __forceinline__ uint64_t frontier_size(const CtrlHdr& c, uint32_t qi) {
  return (c.qpos[qi] & 0xFFFFFFFFull) + c.qbig[qi];
}

// Appends one trace record.  Only the writer (the one thread that owns the
// trace) stores it; every copy of the state counts it, so copies stay equal.
__device__ __forceinline__ void trace_add(Ctrl* ctrl, CtrlHdr& c, uint8_t dir, uint64_t frontier, uint64_t found,
                                          unsigned long long now, bool writer) {
  if (c.trace_len < NWG_TRACE_CAP) {
    if (writer) {
      ctrl->trace_dir[c.trace_len]      = dir;
      ctrl->trace_frontier[c.trace_len] = frontier;
      ctrl->trace_found[c.trace_len]    = found;
      ctrl->trace_end_ns[c.trace_len]   = now - c.t_start;
    }
    c.trace_len++;
  }
}

// Sets up a step of the top-down kernels over the queue in buffer c.cur
// (writing buffer c.cur ^ 1) and returns the kernel that runs it: one
// cluster for a tiny frontier, the persistent small grid for a small one,
// the full grid otherwise.
__device__ __forceinline__ uint32_t td_kernel_setup(CtrlHdr& c) {
  const uint32_t nxt = c.cur ^ 1u;
  c.qpos[nxt]        = 0;
  c.qbig[nxt]        = 0;
  c.nhub[nxt]        = 0;
  c.acc_scout        = 0;
  // warp work units of the step: chunk entries + groups of 32 small vertices
  const uint64_t units = (c.qpos[c.cur] >> 32) + ((c.qpos[c.cur] & 0xFFFFFFFFull) + 31) / 32;
  return units <= (uint64_t)kClusterUnits            ? kActTDCluster
         : units <= (uint64_t)kSmallBlocks * kWarps ? kActTDSmall
                                                    : kActTD;
}

// A bottom-up pull whose front is held as a queue (the first pull of a
// phase: the frontier queue; or the pull after one run this way: its
// discoveries) may run as a push from that queue with the top-down kernels.
// On a symmetric graph the unvisited vertices with an in-neighbour in the
// front are exactly the unvisited out-neighbours of the front, so the step
// discovers the same set and the same awake count as bfs.hpp:211-228; only
// a parent may name another front vertex, which BFSVerifier's rules allow.
// The push is taken when its estimated time is below the pull's, in tenths
// of a nanosecond, with costs fitted to B200 step times of the RMAT,
// uniform and grid workloads at 2^24 vertices:
//   push: 300 per front vertex (queue entry, offsets), 50 per front
//         out-edge (column, visited test), 500 per discovery (claim,
//         parent, degree, queue entry);
//   pull: 26 per vertex (the bitmap scan) plus, per candidate (unvisited,
//         with in-edges), 30 per in-edge tested, growing with the scan
//         length (x (1 + t / 16)), where an in-edge is in the front with
//         probability about front_edges / m, so t = min(average degree,
//         m / front_edges).
// Discoveries are estimated as the front's out-edges times the unvisited
// share, at most the candidates, and, on graphs of average degree <= 8
// (meshes and roads, whose fronts are bands), at most twice the front.
__device__ __forceinline__ uint64_t active_vertices(const DobfsParams& p) {
  return p.n > p.nzero ? p.n - p.nzero : 1;  // vertices with edges
}
__device__ __forceinline__ uint64_t avg_degree(const DobfsParams& p) {
  return max((uint64_t)1, p.m / active_vertices(p));
}
__device__ __forceinline__ uint64_t pull_candidates(const DobfsParams& p, uint64_t reached) {
  const uint64_t excl = p.nzero + reached;
  return p.n > excl ? p.n - excl : 0;
}
// Estimated discoveries of a step from `front` with `front_edges` out-edges
// when `reached` vertices are visited.
__device__ __forceinline__ uint64_t est_wins(const DobfsParams& p, uint64_t reached, uint64_t front,
                                             uint64_t front_edges) {
  const uint64_t cand = pull_candidates(p, reached);
  uint64_t wins = min(cand, (uint64_t)((double)front_edges * (double)cand / (double)active_vertices(p)));
  if (avg_degree(p) <= 8) wins = min(wins, 2 * front);
  return wins;
}
__device__ __forceinline__ bool push_cheaper(const DobfsParams& p, uint64_t reached, uint64_t front,
                                             uint64_t front_edges) {
  if (!p.symmetric || front_edges == 0) return false;
  const uint64_t cand   = pull_candidates(p, reached);
  const uint64_t wins   = est_wins(p, reached, front, front_edges);
  const uint64_t t      = max((uint64_t)1, min(avg_degree(p), p.m / front_edges));
  const uint64_t push   = 300 * front + 50 * front_edges + 500 * wins;
  const uint64_t pull   = 26 * p.n + cand * (30 * t + 30 * t * t / 16);
  return push < pull;
}
__device__ __forceinline__ bool pull_as_push(const DobfsParams& p, const CtrlHdr& c, uint64_t front,
                                             uint64_t front_edges) {
  return push_cheaper(p, c.reached, front, front_edges);
}

// A pull run as a push (pull_as_push true) whose discoveries will be the
// front of a real pull gains nothing from a queue: the pull reads its front
// from a bitmap.  The push then only marks its discoveries in the pull's
// discovery bitmap (kActBUMark): no out-degree lookup and no queue entry per
// discovery, which on a uniform graph of degree 32 is the bulk of the step
// that discovers most of the graph.  It is chosen when the same estimates
// say, one step ahead, that the bottom-up phase goes on (bfs.hpp:229) and
// its next step is a pull, and the step discovers at least n / 32 vertices.
// When the real counts decide otherwise the results stay the same: a push
// that was wanted runs as a pull; a phase that ends gets its queue from the
// bitmap, as after any pull (bfs.hpp:235-239).
__device__ __forceinline__ bool mark_push(const DobfsParams& p, const CtrlHdr& c, uint64_t front,
                                          uint64_t front_edges) {
  if (!c.mark_ok) return false;
  const uint64_t wins = est_wins(p, c.reached, front, front_edges);
  if (wins < p.n / 32) return false;
  if (!(wins >= front || wins > p.n / c.beta)) return false;
  return !push_cheaper(p, c.reached + wins, wins, wins * avg_degree(p));
}

// A top-down step after which the reference's rule will very likely switch
// to a pull needs no queue either: the first pull reads its front from V.
// Such a step (kActTDMark) marks its discoveries in C0 and sums only their
// count and out-degrees, which the switch rule needs (bfs.hpp:186).  Chosen
// when, by the same estimates, the step discovers at least n / 32 vertices,
// their out-degree sum is at least twice the switch threshold, and the
// pull after it would not run as a push.  If the real sum keeps the
// traversal top-down, bitmap -> queue rebuilds the queue from C0 first.
__device__ __forceinline__ bool mark_td(const DobfsParams& p, const CtrlHdr& c, uint64_t front,
                                        uint64_t front_edges) {
  if (!c.mark_ok || c.topdown_only) return false;
  const uint64_t wins = est_wins(p, c.reached, front, front_edges);
  if (wins < p.n / 32) return false;
  const uint64_t scout = wins * avg_degree(p);
  if (scout / 2 <= c.edges_to_check / c.alpha) return false;
  return !push_cheaper(p, c.reached + wins, wins, scout);
}

// Starts a marking push from the queue in c.cur; it writes C[bm ^ 1] like a
// first pull (bm = 1: C0), and its completion is a pull's.
__device__ __forceinline__ uint32_t mark_setup(CtrlHdr& c) {
  c.bu_push   = 0;
  c.acc_awake = 0;
  c.acc_scout = 0;
  c.bu_mode   = 0;
  c.bm        = 1;
  return kActBUMark;
}

// Starts a marking top-down step from the queue in c.cur (writes C0).
__device__ __forceinline__ uint32_t mark_td_setup(CtrlHdr& c) {
  c.acc_awake = 0;
  c.acc_scout = 0;
  c.bm        = 1;
  return kActTDMark;
}

// ---------------------------------------------------------------------------
// decide_on: one thread; consumes the previous action's counters (already
// in `c`) and picks the next action.  Every branch below cites the reference
// line it reproduces.  Returns the next action (kActNone when the traversal
// is over).  It advances a copy `c` of the decision state; `writer` marks
// the one caller that writes the trace.  It reads nothing else that changes
// during a step except the sticky error word, so equal copies given equal
// counters make equal decisions.
__device__ uint32_t decide_on(const DobfsParams& p, CtrlHdr& c, bool writer, bool read_err = true) {
  const unsigned long long now = globaltimer();
  const uint64_t N    = p.n;
  uint32_t       next = kActNone;
  bool           done = false, queue_decision = false;

  const bool was_exact = c.scout_exact != 0;
  if (c.action != kActNone) c.scout_exact = 0;  // set again below after a top-down step
  c.prev_small = 0;
  switch (c.action) {
    case kActNone:  // first iteration: frontier = {root}
      queue_decision = true;
      if (writer) p.ctrl->t_first_decide = now - c.t_start;
      break;
    case kActTD:
    case kActTDSmall:
    case kActTDCluster: {
      const uint32_t nxt = c.cur ^ 1u;
      const uint64_t nq  = frontier_size(c, nxt);
      if (c.bu_push) {  // a bottom-up pull run as a push: the pull's bookkeeping
        const uint64_t awake = nq;
        trace_add(p.ctrl, c, 1, c.old_awake, awake, now, writer);
        c.bu_steps++;
        c.reached += awake;
        c.cur = nxt;  // the discoveries, held as a queue, are the next front
        if (awake > 0) c.levels++;
        if (awake >= c.old_awake || awake > N / c.beta) {  // bfs.hpp:229
          c.old_awake   = awake;                           // bfs.hpp:206
          c.awake_count = awake;
          if (pull_as_push(p, c, awake, c.acc_scout)) {
            next = mark_push(p, c, awake, c.acc_scout) ? mark_setup(c) : td_kernel_setup(c);
          } else {  // a pull over V, which holds every visited vertex
            c.bu_push   = 0;
            c.acc_awake = 0;
            c.bu_mode   = 0;
            c.bm        = 1;
            next        = kActBU;
          }
        } else if (awake == 0) {
          done = true;  // bfs.hpp:231-233
        } else {
          // the phase ends; the discoveries are already the queue that
          // bitmap->queue would build (bfs.hpp:235-239)
          c.bu_push      = 0;
          c.awake_count  = awake;
          c.scout_count  = 1;  // bfs.hpp:241
          queue_decision = true;
        }
        break;
      }
      c.prev_small = was_exact && c.scout_count <= kSoloCap && frontier_size(c, c.cur) <= kSoloCap;
      trace_add(p.ctrl, c, 0, frontier_size(c, c.cur), nq, now, writer);
      c.td_steps++;
      c.reached += nq;
      c.scout_count = c.acc_scout;  // bfs.hpp:271
      c.scout_exact = 1;
      c.cur         = nxt;          // swap(q1, q2), bfs.hpp:304
      if (nq == 0) {
        done = true;  // all q2 bins empty, bfs.hpp:297-303
      } else {
        c.levels++;
        queue_decision = true;
      }
      break;
    }
    case kActTDMark: {  // a top-down step (bfs.hpp:242-295) whose discoveries are marked in C0
      const uint64_t nq = c.acc_awake;
      trace_add(p.ctrl, c, 0, frontier_size(c, c.cur), nq, now, writer);
      c.td_steps++;
      c.reached += nq;
      c.scout_count = c.acc_scout;  // bfs.hpp:271
      c.scout_exact = 1;
      if (nq == 0) {
        done = true;  // bfs.hpp:297-303
        break;
      }
      c.levels++;
      if (c.scout_count > c.edges_to_check / c.alpha) {  // bfs.hpp:186
        c.awake_count = nq;                                // bfs.hpp:199-202
        c.old_awake   = nq;
        // a pull over V (a push would need the queue; both discover the same set)
        c.acc_awake = 0;
        c.bu_mode   = 0;
        c.bm        = 1;
        next        = kActBU;
      } else {
        c.edges_to_check -= c.scout_count;  // bfs.hpp:243
        c.qpos[c.cur]     = 0;               // the queue is rebuilt from C0 into buffer cur
        c.qbig[c.cur]     = 0;
        c.nhub[c.cur]     = 0;
        c.bm              = 0;
        c.b2q_then_td     = 1;
        next              = kActB2Q;
      }
      break;
    }
    case kActBU:
    case kActBUMark: {  // a marking push ends like a pull: its discoveries are in C[bm ^ 1]
      const uint64_t awake = c.acc_awake;
      trace_add(p.ctrl, c, 1, c.old_awake, awake, now, writer);
      c.bu_steps++;
      c.reached += awake;
      c.bm ^= 1u;  // C[bm] now holds this pull's discoveries (the new "front")
      if (awake > 0) c.levels++;
      if (awake >= c.old_awake || awake > N / c.beta) {  // bfs.hpp:229
        c.old_awake   = awake;                           // bfs.hpp:206
        c.awake_count = awake;
        c.acc_awake   = 0;
        c.bu_mode     = 1;
            next          = kActBU;
      } else if (awake == 0) {
        done = true;  // bfs.hpp:231-233
      } else {
        c.awake_count = awake;
        c.qpos[c.cur] = 0;
        c.qbig[c.cur] = 0;
        next          = kActB2Q;  // bfs.hpp:235-239
      }
      break;
    }
    case kActB2Q:
      c.b2q_steps++;
      if (c.b2q_then_td) {  // the queue of a marking top-down step, whose decision was top-down
        c.b2q_then_td = 0;
        next          = td_kernel_setup(c);
        break;
      }
      c.scout_count  = 1;  // bfs.hpp:241
      queue_decision = true;
      break;
    default:
      c.status = NWG_ESTATE;
      done     = true;
      break;
  }

  if (queue_decision) {
    const uint64_t nq = frontier_size(c, c.cur);
    if (!c.topdown_only && c.scout_count > c.edges_to_check / c.alpha) {  // bfs.hpp:186
      c.awake_count = nq;                                                // bfs.hpp:199-202
      c.old_awake   = nq;
      if (pull_as_push(p, c, nq, c.scout_count)) {  // scout_count: the frontier's out-edges
        if (mark_push(p, c, nq, c.scout_count)) {
          next = mark_setup(c);
        } else {
          c.bu_push = 1;
          next      = td_kernel_setup(c);
        }
      } else {
        c.acc_awake = 0;
        c.bu_mode   = 0;
        c.bm        = 1;  // the first pull writes C0
        next        = kActBU;
      }
    } else {
      c.edges_to_check -= c.scout_count;  // bfs.hpp:243
      next = td_kernel_setup(c);
      if (mark_td(p, c, nq, c.scout_count)) next = mark_td_setup(c);
    }
  }
  if (!done && ++c.steps > c.max_steps) {
    c.status = NWG_ETIMEDOUT;  // loop bound; a BFS needs at most ~2n actions
  }
  const int32_t err = read_err ? *(volatile int32_t*)&p.ctrl->err : 0;
  if (c.status == 0 && err != 0) c.status = err;
  if (c.status != 0) done = true;
  c.action      = done ? kActNone : next;
  c.pre_decided = 0;
  return c.action;
}

// decide_core: the decision on the control header itself (one thread).
// The header is loaded and stored with 16-byte vector accesses so the
// decision costs one memory round trip, not one per field.
__device__ uint32_t decide_core(const DobfsParams& p) {
  constexpr int kV = sizeof(CtrlHdr) / 16;
  CtrlHdr       c;
  {
    const uint4* src = reinterpret_cast<const uint4*>(&p.ctrl->h);
    uint4*       dst = reinterpret_cast<uint4*>(&c);
#pragma unroll
    for (int i = 0; i < kV; ++i) dst[i] = __ldcg(src + i);
  }
  const uint32_t next = decide_on(p, c, true);
  {
    const uint4* src = reinterpret_cast<const uint4*>(&c);
    uint4*       dst = reinterpret_cast<uint4*>(&p.ctrl->h);
#pragma unroll
    for (int i = 0; i < kV; ++i) dst[i] = src[i];
  }
  return next;
}

// k_decide: the host-stepped traversal's decision (one thread).  When the
// previous action (a persistent small-frontier kernel) already decided, it
// only clears that mark; the host reads the action from the header.
__global__ void k_decide(DobfsParams p) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  p.ctrl->decides++;  // only this thread writes it
  if (__ldcg(&p.ctrl->h.pre_decided)) {
    p.ctrl->h.pre_decided = 0;
  } else {
    decide_core(p);
  }
}

// ---------------------------------------------------------------------------
// One top-down step (bfs.hpp:242-295) by blocks [0, nblocks): chunk entries
// first (256-edge pieces of every vertex with out-degree >= warp_min, so
// hubs spread over the grid), then the small-degree queue; both go through
// gather_ranges, a group of entries per warp.  The group size of chunk
// entries shrinks when there are few so every warp gets work.
template <bool kDefer, bool kMark = false>
__device__ __forceinline__ void td_step(const DobfsParams& p, const StepView& sv, TdWarp* tws, uint32_t block,
                                        uint32_t nblocks) {
  const uint32_t     cur     = sv.in;
  const uint64_t     nS      = sv.nS;
  const uint64_t     nC      = sv.nC;
  TdWarp&            tw      = tws[threadIdx.x >> 5];
  uint32_t           nbig    = 0;
  const unsigned     lane    = threadIdx.x & 31;
  const uint64_t     gwarp   = (uint64_t)block * kWarps + (threadIdx.x >> 5);
  const uint64_t     nwarps  = (uint64_t)nblocks * kWarps;
  uint32_t           wcnt    = 0;
  unsigned long long scout   = 0;

  uint64_t gsz = 1;  // chunk entries per warp group: at least ~4 groups per warp
  while (gsz < 32 && nC > nwarps * gsz * 4) gsz <<= 1;
  const uint64_t* qc = p.qc[cur];
  for (uint64_t g0 = gwarp * gsz; g0 < nC; g0 += nwarps * gsz) {
    const uint64_t i  = g0 + lane;
    uint32_t       u  = 0;
    uint64_t       lo = 0, hi = 0;
    if (lane < gsz && i < nC) {
      const uint64_t ent = __ldcg(qc + i);  // L2: written by other SMs earlier in a persistent launch
      u                  = (uint32_t)(ent >> 32);
      const uint64_t ob = p.off[u], oe = p.off[u + 1];
      lo = ob + (ent & 0xFFFFFFFFull) * p.th.chunk;
      hi = min(oe, lo + p.th.chunk);
    }
    gather_ranges<kDefer, kMark>(p, sv, u, lo, hi, tw, wcnt, scout, nbig);
  }

  // small vertices per warp group: fewer when there are few, so that every
  // warp gets work (a frontier of 40k degree-32 vertices in groups of 32
  // left three quarters of a 4-block-per-SM grid idle)
  uint64_t sgs = 32;
  while (sgs > 4 && nS < nwarps * sgs * 2) sgs >>= 1;
  const uint32_t* qs = p.qs[cur];
  for (uint64_t g0 = gwarp * sgs; g0 < nS; g0 += nwarps * sgs) {
    const uint64_t i  = g0 + lane;
    uint32_t       u  = 0;
    uint64_t       lo = 0, hi = 0;
    if (lane < sgs && i < nS) {
      u  = __ldcg(qs + i);
      lo = p.off[u];
      hi = p.off[u + 1];
    }
    gather_ranges<kDefer, kMark>(p, sv, u, lo, hi, tw, wcnt, scout, nbig);
  }
  if (!kMark) flush_block<kDefer>(p, sv, tws, wcnt, scout, nbig, true);

  const unsigned long long tot = block_sum(scout);
  __syncthreads();
  const uint32_t nb = block_sum(nbig);  // a marking step: its discoveries
  if (threadIdx.x == 0) {
    if (tot) atomicAdd(sv.scout, tot);
    if (nb) {
      if (kMark)
        atomicAdd(sv.awake, (unsigned long long)nb);
      else
        atomicAdd(sv.qbig, nb);
    }
  }
}

// Views of the step the control header describes (the level-loop kernels).
// A top-down step expands queue buffer cur into cur ^ 1.
__device__ __forceinline__ StepView td_view(const DobfsParams& p) {
  CtrlHdr*       c = &p.ctrl->h;
  StepView       sv;
  sv.parents       = c->parents;
  sv.in            = __ldcg(&c->cur);
  sv.out           = sv.in ^ 1u;
  const uint64_t q = __ldcg(&c->qpos[sv.in]);
  sv.nS            = min((uint64_t)(q & 0xFFFFFFFFull), p.qs_cap);
  sv.nC            = min((uint64_t)(q >> 32), p.qc_cap);
  sv.bu_mode       = 0;
  sv.bm            = 0;
  sv.qpos          = &c->qpos[sv.out];
  sv.qbig          = &c->qbig[sv.out];
  sv.nhub          = &c->nhub[sv.out];
  sv.scout         = &c->acc_scout;
  sv.awake         = &c->acc_awake;
  sv.mark          = nullptr;
  sv.mark_deg      = 0;
  return sv;
}

// A pull, or the bitmap -> queue pass that refills buffer cur.
__device__ __forceinline__ StepView bu_view(const DobfsParams& p) {
  CtrlHdr* c = &p.ctrl->h;
  StepView sv;
  sv.parents = c->parents;
  sv.in = sv.out = __ldcg(&c->cur);
  sv.nS = sv.nC = 0;
  sv.bu_mode    = __ldcg(&c->bu_mode);
  sv.bm         = __ldcg(&c->bm);
  sv.qpos       = &c->qpos[sv.out];
  sv.qbig       = &c->qbig[sv.out];
  sv.nhub       = &c->nhub[sv.out];
  sv.scout      = &c->acc_scout;
  sv.awake      = &c->acc_awake;
  sv.mark       = nullptr;
  sv.mark_deg   = 0;
  return sv;
}

// k_td: one top-down step over the whole grid.
__global__ void __launch_bounds__(kThreads, kTdPerSm) k_td(DobfsParams p) {
  __shared__ TdWarp s_tw[kWarps];
  td_step<false>(p, td_view(p), s_tw, blockIdx.x, gridDim.x);
}

// Grid-wide barrier of a cooperative launch.  The wait is bounded: after
// kBarrierSpins polls the block records NWG_ETIMEDOUT in ctrl->err and
// returns false, and every later barrier returns false at once, so a
// broken barrier can never hang the GPU.
constexpr unsigned kBarrierSpins = 1u << 22;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* a) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_barrier(const DobfsParams& p, unsigned nblocks, unsigned max_spins = kBarrierSpins) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int      ok  = __ldcg(&p.ctrl->err) == 0;
    GridBar* bar = &p.ctrl->bar;
    if (ok) {
      const unsigned g = ld_acquire(&bar->gen);
      __threadfence();
      if (atomicAdd(&bar->count, 1u) == nblocks - 1) {
        atomicExch(&bar->count, 0u);
        __threadfence();
        atomicAdd(&bar->gen, 1u);
      } else {
        unsigned spins = 0;
        while (ld_acquire(&bar->gen) == g) {
          if (++spins > max_spins) {
            atomicCAS(&p.ctrl->err, 0, NWG_ETIMEDOUT);
            ok = 0;
            break;
          }
          __nanosleep(32);
        }
      }
      __threadfence();
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// k_td_loop: the small-frontier branch.  A persistent cooperative kernel of
// kSmallBlocks blocks runs consecutive top-down steps, each followed by a
// grid barrier and the decision (block 0), while the frontier stays small
// and the direction stays top-down; it then leaves the next decision for
// the graph's decide node (pre_decided).  Long, thin traversals (grids,
// roads) thus pay a barrier per level instead of two kernel launches.
// Writes the chunk entries of the hub records the level deferred (queue
// buffer qi): a warp per record, grid-strided, so the writes come from every
// SM.  Runs after the level's barrier, beside the decision; the next barrier
// (or the kernel's end) orders them before the next level reads the queue.
__device__ __forceinline__ void expand_hubs(const DobfsParams& p, uint32_t qi, uint64_t nhub, uint32_t block,
                                            uint32_t nblocks) {
  const HubRec* rec = p.hubrec[qi];
  if (rec == nullptr) return;
  const uint64_t  nrec   = min(nhub, p.hub_cap);
  const unsigned  lane   = threadIdx.x & 31;
  const uint64_t  gwarp  = (uint64_t)block * kWarps + (threadIdx.x >> 5);
  const uint64_t  nwarps = (uint64_t)nblocks * kWarps;
  uint64_t* const qc     = p.qc[qi];
  static_assert(sizeof(HubRec) == 16, "one 16-byte load per record");
  for (uint64_t r = gwarp; r < nrec; r += nwarps) {
    // L2 loads: the records were written by other SMs during this launch
    const uint4    raw = __ldcg(reinterpret_cast<const uint4*>(rec) + r);
    const uint64_t pos = (uint64_t)raw.z | ((uint64_t)raw.w << 32);
    for (uint64_t j = lane; j < raw.y; j += 32)
      if (pos + j < p.qc_cap) qc[pos + j] = ((uint64_t)raw.x << 32) | j;
  }
}

__global__ void __launch_bounds__(kThreads) k_td_loop(DobfsParams p) {
  __shared__ TdWarp   s_tw[kWarps];
  __shared__ uint32_t s_next;
  for (;;) {
    const StepView sv = td_view(p);
    td_step<true>(p, sv, s_tw, blockIdx.x, gridDim.x);
    if (!grid_barrier(p, gridDim.x)) break;
    expand_hubs(p, sv.out, __ldcg(sv.nhub), blockIdx.x, gridDim.x);
    if (blockIdx.x == 0 && threadIdx.x == 0) s_next = decide_core(p);
    if (!grid_barrier(p, gridDim.x)) break;
    if (threadIdx.x == 0) s_next = __ldcg(&p.ctrl->h.action);
    __syncthreads();
    if (s_next != kActTDSmall) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (__ldcg(&p.ctrl->err) != 0) {
      // a barrier ran out: end the traversal with the error
      p.ctrl->h.status = __ldcg(&p.ctrl->err);
      p.ctrl->h.action = kActNone;
    }
    __threadfence();
    p.ctrl->h.pre_decided = 1;
  }
}

// k_td_cluster: consecutive tiny top-down levels in ONE thread-block cluster
// (kClusterCtas blocks).  The level barriers are the cluster's hardware
// barrier (barrier.cluster arrive/wait: release/acquire at cluster scope, so
// the appends, counters and hub records of every block are visible after
// it) instead of the global-memory grid barrier of k_td_loop, and no block
// polls.  Rank 0 decides; every block reads that one decision from rank 0's
// shared memory (distributed shared memory) after the second barrier, so all
// blocks take the same branch and reach the same barriers.  Queue entries,
// counters and hub records are read with L2 loads, as in k_td_loop.
__global__ void __cluster_dims__(kClusterCtas, 1, 1) __launch_bounds__(kThreads) k_td_cluster(DobfsParams p) {
  __shared__ TdWarp   s_tw[kWarps];
  __shared__ uint32_t s_next;
  namespace cg              = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t    rank    = cluster.block_rank();
  const uint32_t    nblk    = cluster.num_blocks();
  uint32_t* const   rank0_next = cluster.map_shared_rank(&s_next, 0);  // rank 0's copy, read over DSMEM
  for (;;) {
    const StepView sv = td_view(p);
    td_step<true>(p, sv, s_tw, rank, nblk);
    cluster.sync();
    expand_hubs(p, sv.out, __ldcg(sv.nhub), rank, nblk);
    if (rank == 0 && threadIdx.x == 0) s_next = decide_core(p);
    cluster.sync();
    // every block reads the one decision rank 0 made; rank 0 writes it again
    // only after the next level's first barrier, which all reads precede
    const uint32_t next = *rank0_next;
    if (next != kActTDCluster) break;
  }
  cluster.sync();  // rank 0's shared memory stays alive until every block has read it
  if (rank == 0 && threadIdx.x == 0) {
    __threadfence();
    p.ctrl->h.pre_decided = 1;
  }
}


// ---------------------------------------------------------------------------
// Candidate compaction shared by k_bu and k_b2q: lane `lane` holds bitmap
// word `bits` of a 32-word tile; the set bits are written to `list` as local
// vertex indices (word * 32 + bit).  Returns the count (warp-uniform).
__device__ __forceinline__ uint32_t compact_tile(uint32_t bits, uint16_t* list) {
  const unsigned lane  = threadIdx.x & 31;
  const uint32_t cnt   = __popc(bits);
  const uint32_t incl  = warp_incl_scan(cnt);
  const uint32_t total = __shfl_sync(kFullMask, incl, 31);
  uint32_t       pos   = incl - cnt;
  while (bits) {
    const int b = __ffs(bits) - 1;
    bits &= bits - 1;
    list[pos++] = (uint16_t)(lane * 32 + b);
  }
  __syncwarp();
  return total;
}

// ---------------------------------------------------------------------------
// k_bu: one bottom-up pull (bfs.hpp:211-228).
//
// Warps take tiles of kBuTileWords bitmap words (512 vertices), interleaved
// over the grid (about seven tiles per warp at 2^24 vertices, so uneven tiles
// average out; 256-vertex tiles were 2-5% slower on RMAT and the grid).  A lane reads one word of V, of the previous pull's C and of
// Z (loaded while the warp works on its previous tile), folds C into V (the
// owner is the only writer), and the tile's candidates (unvisited, with
// in-edges) are compacted into a per-warp list in shared memory.
//
// The front bitmap is read with plain (coherent) loads: in the persistent
// traversal kernel it was written earlier in the same launch, by other SMs,
// which the non-coherent path does not allow.
//
// The candidates then stream through the lanes.  Each lane holds the
// candidate whose in-edges it is testing and the next one, whose in-CSR
// offsets are already loading.  When a lane's scan ends (a hit, or its list
// is exhausted) it promotes its next candidate, and the lanes that need a
// next one take the following list entries with one ballot.  A round tests
// kBuProbe in-edges of the current candidate with independent loads.  Every
// lane thus keeps a scan in flight until the tile's list runs out (a batch
// of 32 candidates no longer waits for its longest scan), and the offsets'
// latency hides behind the current scan.  A lane that has tested kBuLane
// in-edges without a hit hands the rest of its list to the whole warp, 32
// in-edges per step.  The first hit in row order becomes the parent, exactly
// as the reference's sequential scan with `break`.
__device__ __forceinline__ void bu_step(const DobfsParams& p, const StepView& sv, PullSmem& sm, uint32_t block,
                                        uint32_t nblocks) {
  const uint32_t  mode    = sv.bu_mode;
  const uint32_t  bm      = sv.bm;
  uint32_t* const parents = sv.parents;
  const uint32_t* Cf      = bm ? p.C1 : p.C0;  // previous pull's discoveries
  uint32_t*       Cw      = bm ? p.C0 : p.C1;  // this pull's discoveries
  const uint32_t* front   = mode ? Cf : p.V;
  const unsigned  lane    = threadIdx.x & 31;
  const unsigned  wib     = threadIdx.x >> 5;
  uint16_t* const cand    = sm.cand[wib];
  uint32_t* const fresh   = sm.fresh[wib];
  const uint64_t  ntiles  = (p.nwords + kBuTileWords - 1) / kBuTileWords;
  const unsigned  lt_mask = (1u << lane) - 1u;
  uint32_t        awake   = 0;

  const uint64_t  gwarp   = (uint64_t)block * kWarps + wib;
  const uint64_t  nwarps  = (uint64_t)nblocks * kWarps;
  // V, C and Z words of the warp's next tile, loaded one tile ahead (the
  // tiles are the warp's own, so no other warp writes these words)
  uint32_t nxv = 0, nxf = 0, nxz = 0;
  {
    const uint64_t w = gwarp * kBuTileWords + lane;
    if (gwarp < ntiles && lane < kBuTileWords && w < p.nwords) {
      nxv = p.V[w];
      nxf = mode ? Cf[w] : 0u;
      nxz = p.Z[w];
    }
  }
  for (uint64_t t = gwarp; t < ntiles; t += nwarps) {
    const uint64_t w  = t * kBuTileWords + lane;
    const bool     wv = lane < kBuTileWords && w < p.nwords;
    const uint32_t vw = nxv, fw = nxf, zw = nxz;
    {
      const uint64_t wn = w + nwarps * kBuTileWords;
      if (t + nwarps < ntiles && lane < kBuTileWords && wn < p.nwords) {
        nxv = p.V[wn];
        nxf = mode ? Cf[wn] : 0u;
        nxz = p.Z[wn];
      }
    }
    uint32_t cm = 0;
    if (wv) {
      if (fw) p.V[w] = vw | fw;  // fold the previous pull into V
      cm = ~(vw | fw) & ~zw;
    }
    if (lane < kBuTileWords) fresh[lane] = 0;
    const uint32_t total = compact_tile(cm, cand);
    const uint64_t vbase = t * kBuTileWords * 32;

    // current candidate (cu: local index, ce: next in-edge, cend, cn: edges
    // tested) and next candidate (nu, nb, nend, offsets in flight)
    uint32_t cu = 0, nu = 0, cn = 0;
    uint64_t ce = 0, cend = 0, nb = 0, nend = 0;
    bool     cv = false, nv = false;
    if (lane < total) {
      cu   = cand[lane];
      ce   = p.in_off[vbase + cu];
      cend = p.in_off[vbase + cu + 1];
      cv   = true;
    }
    uint32_t ptr = min(total, 32u);  // next unassigned list entry (warp-uniform)
    if (ptr + lane < total) {
      nu   = cand[ptr + lane];
      nb   = p.in_off[vbase + nu];
      nend = p.in_off[vbase + nu + 1];
      nv   = true;
    }
    ptr = min(total, ptr + 32u);

    while (__any_sync(kFullMask, cv)) {
      bool     found = false, handoff = false;
      uint32_t par   = 0;
      if (cv) {
        uint32_t nbv[kBuProbe];
#pragma unroll
        for (int k = 0; k < kBuProbe; ++k) nbv[k] = (ce + k < cend) ? __ldg(p.in_col + ce + k) : kNull;
        uint32_t hit = 0;
#pragma unroll
        for (int k = 0; k < kBuProbe; ++k)
          if (nbv[k] != kNull && ((front[nbv[k] >> 5] >> (nbv[k] & 31)) & 1u)) hit |= 1u << k;
        if (hit) {
          const int k = __ffs(hit) - 1;
#pragma unroll
          for (int q = 0; q < kBuProbe; ++q)
            if (q == k) par = nbv[q];
          found = true;
        } else {
          ce += kBuProbe;
          cn += kBuProbe;
          if (ce >= cend) {
            cv = false;  // list exhausted: no parent this pull
          } else if (cn >= kBuLane) {
            handoff = true;  // long list: the warp scans the rest
          }
        }
      }
      unsigned pend = __ballot_sync(kFullMask, handoff);
      while (pend) {
        const int leader = __ffs(pend) - 1;
        pend &= pend - 1;
        const uint64_t b  = __shfl_sync(kFullMask, ce, leader);
        const uint64_t en = __shfl_sync(kFullMask, cend, leader);
        bool           lf = false;
        uint32_t       lp = 0;
        for (uint64_t base = b; base < en; base += 32) {
          const uint64_t i = base + lane;
          uint32_t       v = 0;
          bool           h = false;
          if (i < en) {
            v = __ldg(p.in_col + i);
            h = (front[v >> 5] >> (v & 31)) & 1u;
          }
          const unsigned hm = __ballot_sync(kFullMask, h);
          if (hm) {
            lp = __shfl_sync(kFullMask, v, __ffs(hm) - 1);
            lf = true;
            break;
          }
        }
        if ((int)lane == leader) {
          found = lf;
          par   = lp;
          cv    = false;
        }
      }
      if (found) {
        parents[vbase + cu] = par;
        atomicOr(&fresh[cu >> 5], 1u << (cu & 31));
        cv = false;
      }
      if (!cv && nv) {  // promote the next candidate
        cu   = nu;
        ce   = nb;
        cend = nend;
        cn   = 0;
        cv   = true;
        nv   = false;
      }
      if (ptr < total) {  // warp-uniform: hand the next entries to the lanes without a next candidate
        const unsigned need = __ballot_sync(kFullMask, !nv);
        const uint32_t rank = __popc(need & lt_mask);
        if (!nv && ptr + rank < total) {
          nu   = cand[ptr + rank];
          nb   = p.in_off[vbase + nu];
          nend = p.in_off[vbase + nu + 1];
          nv   = true;
        }
        ptr = min(total, ptr + (uint32_t)__popc(need));
      }
    }
    __syncwarp();
    if (wv) {
      const uint32_t nw = fresh[lane];
      Cw[w]             = nw;
      awake += __popc(nw);
    }
    __syncwarp();
  }
  const uint32_t tot = block_sum(awake);
  if (threadIdx.x == 0 && tot) atomicAdd(sv.awake, (unsigned long long)tot);
}

__global__ void __launch_bounds__(kThreads) k_bu(DobfsParams p) {
  __shared__ PullSmem sm;
  bu_step(p, bu_view(p), sm, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// k_b2q: bitmap -> queue (bfs.hpp:235-239) from C[bm], folding C[bm] into V
// on the way.  Each warp compacts tiles of 32 words into its vertex buffer;
// full buffers are appended per warp, the rest once per block at the end.
__device__ __forceinline__ void b2q_step(const DobfsParams& p, const StepView& sv, TdSmem& sm, uint32_t block,
                                         uint32_t nblocks) {
  TdWarp* const      s_tw   = sm.tw;
  const uint32_t*    Cs     = sv.bm ? p.C1 : p.C0;
  const unsigned     lane   = threadIdx.x & 31;
  const unsigned     wib    = threadIdx.x >> 5;
  const uint64_t     gwarp  = (uint64_t)block * kWarps + wib;
  const uint64_t     nwarps = (uint64_t)nblocks * kWarps;
  const uint64_t     ntiles = (p.nwords + kTileWords - 1) / kTileWords;
  uint16_t* const    list   = sm.list[wib];
  TdWarp&            tw     = s_tw[wib];
  uint32_t           wcnt   = 0, nbig = 0;
  unsigned long long scout  = 0;
  for (uint64_t t = gwarp; t < ntiles; t += nwarps) {
    const uint64_t w = t * kTileWords + lane;  // lanes >= kTileWords hold no word
    const uint32_t x = (lane < kTileWords && w < p.nwords) ? Cs[w] : 0u;
    if (x) p.V[w] |= x;
    const uint32_t total = compact_tile(x, list);  // at most kTileWords * 32 entries
    const uint64_t vbase = t * kTileWords * 32;
    for (uint32_t j = 0; j < total; j += 32) {
      const uint32_t k = min(32u, total - j);  // warp-uniform
      if (wcnt + k > kWinBuf) flush_winners<false>(p, sv, tw, wcnt, scout, nbig);
      if (lane < k) tw.win[wcnt + lane] = (uint32_t)(vbase + list[j + lane]);
      wcnt += k;
    }
    __syncwarp();
  }
  flush_block<false>(p, sv, s_tw, wcnt, scout, nbig, false);
  const uint32_t nb = block_sum(nbig);
  if (threadIdx.x == 0 && nb) atomicAdd(sv.qbig, nb);
}

__global__ void __launch_bounds__(kThreads) k_b2q(DobfsParams p) {
  __shared__ TdSmem sm;
  b2q_step(p, bu_view(p), sm, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// k_trav: the whole traversal in one cooperative launch (every block
// resident), one grid barrier between steps instead of the level-loop
// graph's decide kernel and conditional nodes, which cost about 13 us per
// step on a B200 (decide 1.5 us, 5 us from its end to the next kernel's
// first block, 6 us from a kernel's end to the next decide).
//
// Every block keeps its own copy of the decision state in shared memory and
// runs decide_on on it after each barrier; all copies start equal and see
// the same counters, so every block takes the same action and reaches the
// same barriers.  A step adds its counts into StepAcc slot step % 3; block 0
// clears slot (step + 1) % 3 during the step.  That slot was last read in
// the decisions at the start of step - 1, which every block finished before
// the barrier ending step - 1, and it is next written in step + 1, after the
// barrier ending this step.  Deferred hub chunk entries are written by the
// whole grid after the barrier and a second barrier orders them before the
// next step reads the queue.  The steps are the level-loop kernels' own
// (td_step, bu_step, b2q_step); the barrier's arrival count is cleared by
// the host before the launch.
constexpr int kTravPerSm = 4;  // 64 registers: the top-down step does not spill

// Grid barrier of k_trav: every block arrives (even after an error, so the
// others are not left waiting); the wait is bounded like grid_barrier's.
// The arrival count only grows during a launch (the host clears it before
// each one): the block that makes the k-th arrival waits until the count
// reaches the next multiple of nblocks.  Passing costs one atomic per block
// and the polls; there is no reset or generation word to update, so the
// last block to arrive releases the others with its own arrival.  The fence
// before the arrival and the acquire loads of the count order every
// block's writes before the barrier ahead of every read after it.
__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* a) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(a) : "memory");
  return v;
}

__device__ __forceinline__ bool trav_barrier(const DobfsParams& p, unsigned nblocks,
                                             unsigned max_spins = kBarrierSpins, unsigned sleep_ns = 32) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long* cnt = &p.ctrl->bar.arrivals;
    int                 ok  = 1;
    __threadfence();
    const unsigned long long k      = atomicAdd(cnt, 1ull);
    const unsigned long long target = (k / nblocks + 1) * nblocks;
    unsigned                 spins  = 0;
    while (ld_acquire64(cnt) < target) {
      if (++spins > max_spins) {
        atomicCAS(&p.ctrl->err, 0, NWG_ETIMEDOUT);
        ok = 0;
        break;
      }
      __nanosleep(sleep_ns);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---------------------------------------------------------------------------
// Solo levels.  A top-down step whose frontier has at most kSoloCap
// out-edges moves a few thousand bytes; on the whole grid it still costs a
// chain of global round trips (queue, offsets, columns, claims, degree
// lookups, queue append, counters) plus a grid barrier and the decision,
// 10-15 us.  Instead block 0 runs such levels alone, one after another,
// with the frontier lists, the out-degree prefix and the counters in shared
// memory, and the decision (decide_on, the same rules) made by its thread 0
// after each level; the other blocks wait at one grid barrier.  When a
// decision leaves the solo case (a bigger frontier, a pull, the level
// bound, the end), block 0 writes the frontier into the global queue buffer
// in the usual form (small entries, chunk entries of the vertices with
// out-degree >= warp_min) and publishes its decision state, which the
// other blocks adopt after the barrier.

// Out-degree prefix of list[0, cnt) into pre (pre[cnt] = total); returns the
// total.  Thread t takes entries [t * kSoloPer, (t + 1) * kSoloPer).  All
// threads of the block call.
__device__ __forceinline__ uint64_t solo_prefix(const DobfsParams& p, const uint32_t* list, uint32_t cnt,
                                                uint32_t* pre) {
  const uint32_t i0 = threadIdx.x * kSoloPer;
  uint32_t       d[kSoloPer];
  uint64_t       sum = 0;
#pragma unroll
  for (uint32_t k = 0; k < kSoloPer; ++k) {
    d[k] = 0;
    if (i0 + k < cnt) {
      const uint32_t v = list[i0 + k];
      d[k]             = (uint32_t)min(__ldg(p.off + v + 1) - __ldg(p.off + v), (uint64_t)0xFFFFFFFFu);
      sum += d[k];
    }
  }
  unsigned long long total = 0;
  unsigned long long run   = block_excl_scan(sum, total);
#pragma unroll
  for (uint32_t k = 0; k < kSoloPer; ++k) {
    if (i0 + k < cnt) pre[i0 + k] = (uint32_t)run;
    run += d[k];
  }
  if (threadIdx.x == 0) pre[cnt] = (uint32_t)total;
  __syncthreads();
  return total;
}

// Largest index o in [0, cnt) with pre[o] <= e: the list entry whose edge
// range holds flattened edge e (entries without edges share their
// successor's prefix and are skipped).
__device__ __forceinline__ uint32_t solo_owner(const uint32_t* pre, uint32_t cnt, uint32_t e) {
  uint32_t lo = 0, hi = cnt - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= e) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One top-down level over list[0, cnt) (edges flattened, total E <=
// kSoloCap): claims as in visit_batch (atomicOr on V; the winner writes the
// parent), winners appended to out through the shared counter *ocnt.  A
// thread takes kSoloBatch edges at once, phase by phase (owner searches,
// then all offset loads, all column loads, all claims), so its loads are in
// flight together; one chain per edge made a level of 2,000 edges take 25 us.
// All threads of the block call.
constexpr int kSoloBatch = (int)kSoloPer;
__device__ __forceinline__ void solo_expand(const DobfsParams& p, uint32_t* parents, const uint32_t* list, uint32_t cnt,
                                            const uint32_t* pre, uint32_t E, uint32_t* out, uint32_t* ocnt) {
  for (uint32_t base = 0; base < E; base += kThreads * kSoloBatch) {
    uint32_t u[kSoloBatch], v[kSoloBatch], r[kSoloBatch];
    uint32_t valid = 0;
#pragma unroll
    for (int k = 0; k < kSoloBatch; ++k) {
      const uint32_t e = base + k * kThreads + threadIdx.x;
      u[k] = r[k] = 0;
      if (e < E) {
        const uint32_t o = solo_owner(pre, cnt, e);
        u[k]             = list[o];
        r[k]             = e - pre[o];  // the edge's rank in u's row
        valid |= 1u << k;
      }
    }
    uint64_t at[kSoloBatch];
#pragma unroll
    for (int k = 0; k < kSoloBatch; ++k) at[k] = (valid & (1u << k)) ? __ldg(p.off + u[k]) + r[k] : 0ull;
#pragma unroll
    for (int k = 0; k < kSoloBatch; ++k) v[k] = (valid & (1u << k)) ? __ldg(p.col + at[k]) : 0u;
#pragma unroll
    for (int k = 0; k < kSoloBatch; ++k)
      r[k] = (valid & (1u << k)) ? atomicOr(p.V + (v[k] >> 5), 1u << (v[k] & 31)) : ~0u;
#pragma unroll
    for (int k = 0; k < kSoloBatch; ++k) {
      if ((valid & (1u << k)) && !(r[k] & (1u << (v[k] & 31)))) {
        parents[v[k]]       = u[k];
        const uint32_t slot = atomicAdd(ocnt, 1u);  // winners <= E <= kSoloCap
        if (slot < kSoloCap) out[slot] = v[k];
      }
    }
  }
}

// Writes list[0, cnt) into queue buffer qi as the top-down kernels expect it
// and records the buffer's counts in c.  A vertex with more than kLaneChunks
// chunks gets a hub record instead (c.nhub[qi] of them), whose chunk entries
// the whole grid writes before the next step, as after a top-down step; one
// block writing a hub frontier's 10^5 entries took 100+ us.  Without record
// buffers the block writes them: `spare` (kSoloCap words) lists those
// entries' indices, sm.pre their first chunk slots.  All threads of the
// block call.
__device__ __forceinline__ void solo_publish(const DobfsParams& p, CtrlHdr& c, uint32_t qi, const uint32_t* list,
                                             uint32_t cnt, uint32_t* spare, SoloSmem& sm) {
  const uint32_t i0 = threadIdx.x * kSoloPer;
  uint64_t       deg[kSoloPer];
  uint32_t       ns = 0, nb = 0;
  uint64_t       nch = 0;
#pragma unroll
  for (uint32_t k = 0; k < kSoloPer; ++k) {
    deg[k] = 0;
    if (i0 + k < cnt) {
      const uint32_t v = list[i0 + k];
      deg[k]           = __ldg(p.off + v + 1) - __ldg(p.off + v);
      if (deg[k] < p.th.warp_min) {
        ++ns;
      } else {
        nch += chunks_of(deg[k], p.th);
        ++nb;
      }
    }
  }
  if (threadIdx.x == 0) sm.nhub = 0;
  unsigned long long tot  = 0;
  const unsigned long long excl = block_excl_scan((unsigned long long)ns | ((unsigned long long)nch << 32), tot);
  const unsigned long long tb   = block_sum((unsigned long long)nb);
  uint64_t spos = excl & 0xFFFFFFFFull, cpos = excl >> 32;
  bool     over = false;
  uint32_t* const qs = p.qs[qi];
  uint64_t* const qc = p.qc[qi];
#pragma unroll
  for (uint32_t k = 0; k < kSoloPer; ++k) {
    if (i0 + k >= cnt) continue;
    const uint32_t v = list[i0 + k];
    if (deg[k] < p.th.warp_min) {
      if (spos < p.qs_cap) qs[spos] = v;
      else over = true;
      ++spos;
    } else {
      const uint64_t nc = chunks_of(deg[k], p.th);
      if (nc <= kLaneChunks) {
        for (uint64_t j = 0; j < nc; ++j) {
          if (cpos + j < p.qc_cap) qc[cpos + j] = ((uint64_t)v << 32) | j;
          else over = true;
        }
      } else if (p.hubrec[qi] != nullptr) {
        const uint32_t h = atomicAdd(&sm.nhub, 1u);
        if (h < p.hub_cap) p.hubrec[qi][h] = HubRec{v, (uint32_t)nc, cpos};
        else over = true;
      } else {  // the block writes it below
        spare[atomicAdd(&sm.nhub, 1u)] = i0 + k;  // at most cnt <= kSoloCap entries
        sm.pre[i0 + k]                 = (uint32_t)min(cpos, (uint64_t)0xFFFFFFFFu);
      }
      cpos += nc;
    }
  }
  __syncthreads();
  const uint32_t nh    = sm.nhub;
  const bool     defer = p.hubrec[qi] != nullptr;
  for (uint32_t h = 0; h < (defer ? 0u : nh); ++h) {
    const uint32_t i  = spare[h];
    const uint32_t v  = list[i];
    const uint64_t c0 = sm.pre[i];
    const uint64_t nc = chunks_of(__ldg(p.off + v + 1) - __ldg(p.off + v), p.th);
    for (uint64_t j = threadIdx.x; j < nc; j += kThreads) {
      if (c0 + j < p.qc_cap) qc[c0 + j] = ((uint64_t)v << 32) | j;
      else over = true;
    }
  }
  if (over) atomicCAS(&p.ctrl->err, 0, NWG_EOVERFLOW);
  if (threadIdx.x == 0) {
    c.qpos[qi] = tot;  // small entries | chunk entries << 32
    c.qbig[qi] = (uint32_t)tb;
    c.nhub[qi] = defer ? nh : 0u;
  }
  __syncthreads();
}

// Whether the step just decided (a top-down action) runs as solo levels:
// the same answer in every block, from its copy of the decision state.
// Only after a small top-down step: a single small level (an RMAT root
// whose neighbours are hubs) gains less than handing the frontier back
// to the grid costs.
__device__ __forceinline__ bool solo_ok(const CtrlHdr& c, uint32_t next) {
  const bool td = next == kActTD || next == kActTDSmall || next == kActTDCluster;
  return td && !c.bu_push && c.prev_small && c.scout_exact && c.scout_count <= kSoloCap &&
         frontier_size(c, c.cur) <= kSoloCap && (c.qpos[c.cur] >> 32) <= kSoloCap && c.nhub[c.cur] == 0;
}

// Block 0's solo levels, from the frontier in queue buffer c.cur (decided:
// a top-down step, solo_ok).  Leaves the next decision in c (c.action) with
// its frontier in the global queue.  All threads of block 0 call.
__device__ __forceinline__ void solo_run(const DobfsParams& p, CtrlHdr& c, SoloSmem& sm, uint32_t* s_flag) {
  const uint32_t cur = c.cur;
  const uint64_t qp  = c.qpos[cur];
  const uint32_t nS  = (uint32_t)(qp & 0xFFFFFFFFull), nC = (uint32_t)(qp >> 32);
  if (threadIdx.x == 0) sm.cnt = nS;
  for (uint32_t i = threadIdx.x; i < nS; i += kThreads) sm.q[0][i] = __ldcg(p.qs[cur] + i);
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nC; i += kThreads) {  // a chunked vertex once: its chunk 0
    const uint64_t ent = __ldcg(p.qc[cur] + i);
    if ((ent & 0xFFFFFFFFull) == 0) {
      const uint32_t slot = atomicAdd(&sm.cnt, 1u);
      if (slot < kSoloCap) sm.q[0][slot] = (uint32_t)(ent >> 32);
    }
  }
  __syncthreads();
  uint32_t a  = 0;
  uint32_t na = sm.cnt;  // == frontier_size(c, cur) <= kSoloCap
  uint64_t E  = na <= kSoloCap ? solo_prefix(p, sm.q[0], na, sm.pre) : ~0ull;  // == c.scout_count
  if (E > kSoloCap) {  // the queue disagrees with the counts it was decided on
    if (threadIdx.x == 0) {
      atomicCAS(&p.ctrl->err, 0, NWG_ESTATE);
      c.status = NWG_ESTATE;
      c.action = kActNone;
    }
    __syncthreads();
    return;
  }
  for (uint32_t lv = 0;; ++lv) {
    if (threadIdx.x == 0) sm.cnt = 0;
    __syncthreads();
    solo_expand(p, c.parents, sm.q[a], na, sm.pre, (uint32_t)E, sm.q[a ^ 1], &sm.cnt);
    __syncthreads();
    const uint32_t nq = min(sm.cnt, kSoloCap);
    a ^= 1;
    E = solo_prefix(p, sm.q[a], nq, sm.pre);
    na = nq;
    if (threadIdx.x == 0) {
      const uint32_t nxt = c.cur ^ 1u;
      c.qpos[nxt]        = nq;
      c.qbig[nxt]        = 0;
      c.nhub[nxt]        = 0;
      c.acc_scout        = E;
      const uint32_t next = decide_on(p, c, true, false);
      *s_flag = (solo_ok(c, next) && lv + 1 < kSoloLevels) ? 1u : 0u;
    }
    __syncthreads();
    if (!*s_flag) break;
  }
  // a pull reads V, not the queue (bitmap -> queue refills the buffer after it)
  if (c.action != kActNone && c.action != kActBU) solo_publish(p, c, c.cur, sm.q[a], na, sm.q[a ^ 1], sm);
}

__global__ void __launch_bounds__(kThreads, kTravPerSm)
    k_trav(DobfsParams p, uint32_t root, uint32_t alpha, uint32_t beta, uint32_t* parents, uint32_t topdown_only) {
  __shared__ StepShared sm;
  __shared__ CtrlHdr    s_c;  // this block's copy of the decision state
  __shared__ uint32_t   s_next;
  constexpr int       kV = sizeof(CtrlHdr) / 16;
  init_step(p, root, alpha, beta, parents, topdown_only, blockIdx.x, gridDim.x, false);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int i = 0; i < 3; ++i) p.ctrl->acc[i] = StepAcc{};
    p.ctrl->kernels = 1;
  }
  bool ok = trav_barrier(p, gridDim.x);
  if (ok && threadIdx.x == 0) {
    const uint4* src = reinterpret_cast<const uint4*>(&p.ctrl->h);
    uint4*       dst = reinterpret_cast<uint4*>(&s_c);
#pragma unroll
    for (int i = 0; i < kV; ++i) dst[i] = __ldcg(src + i);
    s_c.mark_ok = 1;  // every block's copy: this kernel runs marking pushes
  }
  uint32_t last   = kActNone;
  bool     resume = false;  // block 0 ran solo levels: its decision state is the next one
  for (uint32_t step = 0; ok; ++step) {
    if (threadIdx.x == 0) {
      if (resume) {
        if (blockIdx.x != 0) {
          const uint4* src = reinterpret_cast<const uint4*>(&p.ctrl->h);
          uint4*       dst = reinterpret_cast<uint4*>(&s_c);
#pragma unroll
          for (int i = 0; i < kV; ++i) dst[i] = __ldcg(src + i);
        }
        s_next = s_c.action;
      } else {
        if (step > 0) {  // the previous step's counters, final after the barrier
          const StepAcc* a = &p.ctrl->acc[(step - 1) % 3];
          if (last != kActBU && last != kActBUMark && last != kActTDMark) {
            const uint32_t ob = last == kActB2Q ? s_c.cur : (s_c.cur ^ 1u);  // the queue buffer it wrote
            s_c.qpos[ob]      = __ldcg(&a->qpos);
            s_c.qbig[ob]      = __ldcg(&a->qbig);
            s_c.nhub[ob]      = __ldcg(&a->nhub);
          }
          s_c.acc_scout = __ldcg(&a->scout);
          s_c.acc_awake = __ldcg(&a->awake);
        }
        s_next = decide_on(p, s_c, blockIdx.x == 0);
      }
    }
    __syncthreads();
    const uint32_t next = s_next;
    if (resume && next != kActNone && s_c.nhub[s_c.cur] != 0) {  // hub records of the solo frontier
      expand_hubs(p, s_c.cur, s_c.nhub[s_c.cur], blockIdx.x, gridDim.x);
      ok = trav_barrier(p, gridDim.x);
      if (!ok) break;
      if (threadIdx.x == 0) s_c.nhub[s_c.cur] = 0;
      __syncthreads();
    }
    resume = false;
    if (next == kActNone) break;
    StepAcc* a = &p.ctrl->acc[step % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) p.ctrl->acc[(step + 1) % 3] = StepAcc{};
    if (solo_ok(s_c, next)) {  // the same in every block
      if (blockIdx.x == 0) {
        solo_run(p, s_c, sm.solo, &s_next);
        if (threadIdx.x == 0) {
          const uint4* src = reinterpret_cast<const uint4*>(&s_c);
          uint4*       dst = reinterpret_cast<uint4*>(&p.ctrl->h);
#pragma unroll
          for (int i = 0; i < kV; ++i) dst[i] = src[i];
        }
      }
      ok     = trav_barrier(p, gridDim.x);
      resume = true;
      last   = kActNone;
      continue;
    }
    StepView sv;
    sv.parents = s_c.parents;
    sv.bu_mode = s_c.bu_mode;
    sv.bm      = s_c.bm;
    sv.qpos    = &a->qpos;
    sv.qbig    = &a->qbig;
    sv.nhub    = &a->nhub;
    sv.scout   = &a->scout;
    sv.awake   = &a->awake;
    sv.mark     = nullptr;
    sv.mark_deg = next == kActTDMark ? 1u : 0u;
    if (next == kActBUMark || next == kActTDMark) {
      // the discovery bitmap is cleared by the whole grid before any claim
      uint32_t* const cw = s_c.bm ? p.C0 : p.C1;
      for (uint64_t w = (uint64_t)blockIdx.x * kThreads + threadIdx.x; w < p.nwords; w += (uint64_t)gridDim.x * kThreads)
        cw[w] = 0u;
      ok = trav_barrier(p, gridDim.x);
      if (!ok) break;
      sv.mark = cw;
    }
    if (next == kActBU) {
      sv.in = sv.out = s_c.cur;
      sv.nS = sv.nC = 0;
      bu_step(p, sv, sm.pull, blockIdx.x, gridDim.x);
    } else if (next == kActB2Q) {
      sv.in = sv.out = s_c.cur;
      sv.nS = sv.nC = 0;
      b2q_step(p, sv, sm.td, blockIdx.x, gridDim.x);
    } else {  // a top-down step, or a pull run as a push
      sv.in          = s_c.cur;
      sv.out         = s_c.cur ^ 1u;
      const uint64_t q = s_c.qpos[s_c.cur];
      sv.nS          = min((uint64_t)(q & 0xFFFFFFFFull), p.qs_cap);
      sv.nC          = min((uint64_t)(q >> 32), p.qc_cap);
      if (sv.mark)
        td_step<true, true>(p, sv, sm.td.tw, blockIdx.x, gridDim.x);
      else
        td_step<true>(p, sv, sm.td.tw, blockIdx.x, gridDim.x);
    }
    ok = trav_barrier(p, gridDim.x);
    if (ok && next != kActBU && next != kActB2Q && next != kActBUMark && next != kActTDMark) {
      const uint32_t nh = __ldcg(&a->nhub);  // the same in every block after the barrier
      if (nh) {
        expand_hubs(p, sv.out, nh, blockIdx.x, gridDim.x);
        ok = trav_barrier(p, gridDim.x);
      }
    }
    last = next;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int32_t err = __ldcg(&p.ctrl->err);
    if (s_c.status == 0 && err != 0) s_c.status = err;
    s_c.action = kActNone;
    const uint4* src = reinterpret_cast<const uint4*>(&s_c);
    uint4*       dst = reinterpret_cast<uint4*>(&p.ctrl->h);
#pragma unroll
    for (int i = 0; i < kV; ++i) dst[i] = src[i];
  }
}

// Out-degrees saturated at 0xFFFF (a saturated entry means: read off).
__global__ void k_deg16(const uint64_t* __restrict__ off, uint64_t n, uint16_t* __restrict__ deg16) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    deg16[v] = (uint16_t)min(off[v + 1] - off[v], (uint64_t)0xFFFFu);
}

// In-degree-zero bitmap; bits past n are set so they are never candidates.
__global__ void k_zero_indegree(const uint64_t* __restrict__ in_off, uint64_t n, uint32_t nwords,
                                uint32_t* __restrict__ Z) {
  const unsigned lane   = threadIdx.x & 31;
  const uint64_t wpb    = blockDim.x >> 5;
  const uint64_t gwarp  = blockIdx.x * wpb + (threadIdx.x >> 5);
  const uint64_t nwarps = gridDim.x * wpb;
  for (uint64_t w = gwarp; w < nwords; w += nwarps) {
    const uint64_t u    = w * 32 + lane;
    const bool     zero = (u >= n) || (in_off[u + 1] == in_off[u]);
    const unsigned b    = __ballot_sync(kFullMask, zero);
    if (lane == 0) Z[w] = b;
  }
}

__global__ void k_popc_words(const uint32_t* __restrict__ w, uint64_t nwords, unsigned long long* out) {
  unsigned long long c = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nwords; i += (uint64_t)gridDim.x * blockDim.x)
    c += __popc(w[i]);
  c = block_sum(c);
  if (threadIdx.x == 0 && c) atomicAdd(out, c);
}

__global__ void k_component(const uint64_t* __restrict__ off, const uint32_t* __restrict__ parents, uint64_t n,
                            unsigned long long* out) {
  unsigned long long e = 0, v = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (parents[i] != kNull) {
      e += off[i + 1] - off[i];
      v += 1;
    }
  }
  e = block_sum(e);
  __syncthreads();
  v = block_sum(v);
  if (threadIdx.x == 0) {
    atomicAdd(out, e);
    atomicAdd(out + 1, v);
  }
}

// Depths from a parent array by pointer jumping (Wyllie's list ranking).
// pair[v] = (ancestor << 32) | distance to it, starting at (parent, 1) and
// (root, 0) for the root; unreached vertices hold ~0.  A round replaces
// each pair by (ancestor's ancestor, sum of the two distances).  A pair is
// read and written whole (one aligned 64-bit access), so any pair a thread
// sees, updated this round or not, is a consistent (ancestor, distance) of
// that vertex, and reading a newer one only shortens the remaining path:
// after ceil(log2 n) + 1 rounds every reached vertex's ancestor is the root.
__global__ void k_jump_init(const uint32_t* __restrict__ parents, uint64_t n, uint32_t root,
                            unsigned long long* __restrict__ pair) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t par = parents[v];
    pair[v] = par == kNull ? ~0ull : ((unsigned long long)par << 32) | (v == root ? 0u : 1u);
  }
}

__global__ void k_jump_round(uint64_t n, unsigned long long* pair) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long pv = pair[v];
    if (pv == ~0ull) continue;
    const unsigned long long pa = pair[pv >> 32];
    pair[v] = (pa & 0xFFFFFFFF00000000ull) | ((pv & 0xFFFFFFFFull) + (pa & 0xFFFFFFFFull));
  }
}

// uint16 depth row from the jumped pairs: 0xFFFF = unreached; a depth that
// does not fit below 0xFFFF sets *overflow.
__global__ void k_jump_row16(const unsigned long long* __restrict__ pair, uint64_t n, uint16_t* __restrict__ row,
                             int* overflow) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long pv = pair[v];
    const uint64_t           d  = pv & 0xFFFFFFFFull;
    if (pv == ~0ull) {
      row[v] = 0xFFFF;
    } else {
      if (d >= 0xFFFF) *overflow = 1;
      row[v] = (uint16_t)min(d, (uint64_t)0xFFFE);
    }
  }
}

__global__ void k_widen(const uint32_t* __restrict__ src, uint64_t* __restrict__ dst, uint64_t count) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// ---------------------------------------------------------------------------
// k_ragged: a ragged batch of (graph, root) traversals over many small packed
// graphs in one persistent launch.  Each block takes items from an atomic
// counter and runs the whole level loop of one item by itself: the same
// init / decide / top-down / bottom-up / bitmap->queue steps as the
// single-graph path, with nblocks = 1 and __syncthreads() in place of
// kernel boundaries, in a scratch slot of its own.  No block ever waits on
// another.
constexpr uint64_t kAlign = 256;
__host__ __device__ inline uint64_t al(uint64_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct SlotLayout {
  uint64_t ctrl, bits, qs, qc, bytes, qs_cap, qc_cap, nwords;
};

__host__ __device__ inline SlotLayout slot_layout(uint64_t nmax, uint64_t mmax) {
  SlotLayout L;
  L.nwords  = (nmax + 31) / 32;
  L.qs_cap  = nmax > 0 ? nmax : 1;
  const uint64_t big = (mmax / 32) < nmax ? (mmax / 32) : nmax;  // warp_min >= 32 in the ragged path
  L.qc_cap  = mmax / 256 + big + 1;
  L.ctrl    = 0;
  L.bits    = al(sizeof(Ctrl));
  L.qs      = al(L.bits + 3 * L.nwords * 4);
  L.qc      = al(L.qs + 2 * L.qs_cap * 4);
  L.bytes   = al(L.qc + 2 * L.qc_cap * 8);
  return L;
}

__global__ void __launch_bounds__(kThreads) k_ragged(RaggedParams rp) {
  __shared__ StepShared sm;
  __shared__ uint32_t   s_item, s_next;
  const SlotLayout    L    = slot_layout(rp.nmax, rp.mmax);
  unsigned char*      slot = rp.scratch + (uint64_t)blockIdx.x * rp.slot_bytes;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(rp.next_item, 1u);
    __syncthreads();
    const uint32_t it = s_item;
    __syncthreads();
    if (it >= rp.n_items) break;
    const RaggedItem  item = rp.items[it];
    const RaggedGraph gr   = rp.graphs[item.graph];
    DobfsParams       p    = {};
    p.off                  = rp.off + gr.off_base;
    p.col                  = rp.col + gr.col_base;
    p.in_off               = p.off;
    p.in_col               = p.col;
    p.n                    = gr.n;
    p.m                    = gr.m;
    p.nwords               = (uint32_t)((gr.n + 31) / 32);
    uint32_t* bits         = reinterpret_cast<uint32_t*>(slot + L.bits);
    p.V                    = bits;
    p.C0                   = bits + L.nwords;
    p.C1                   = bits + 2 * L.nwords;
    p.Z                    = rp.Z + gr.z_base;
    uint32_t* qs           = reinterpret_cast<uint32_t*>(slot + L.qs);
    uint64_t* qc           = reinterpret_cast<uint64_t*>(slot + L.qc);
    p.qs[0]                = qs;
    p.qs[1]                = qs + L.qs_cap;
    p.qc[0]                = qc;
    p.qc[1]                = qc + L.qc_cap;
    p.qs_cap               = L.qs_cap;
    p.qc_cap               = L.qc_cap;
    p.th                   = Thresholds{item.warp_min, 256, 8};
    p.nzero                = 0;  // unknown here: the push-or-pull estimate then counts isolated vertices too
    p.symmetric            = 1;  // packed graphs are symmetric
    p.ctrl                 = reinterpret_cast<Ctrl*>(slot + L.ctrl);
    init_step(p, item.root, (uint32_t)item.alpha, (uint32_t)item.beta, rp.parents + item.out_base, 0u, 0, 1);
    __syncthreads();
    for (;;) {
      if (threadIdx.x == 0) s_next = decide_core(p);
      __syncthreads();
      const uint32_t next = s_next;
      if (next == kActNone) break;
      if (next == kActBU) {
        bu_step(p, bu_view(p), sm.pull, 0, 1);
      } else if (next == kActB2Q) {
        b2q_step(p, bu_view(p), sm.td, 0, 1);
      } else {
        td_step<false>(p, td_view(p), sm.td.tw, 0, 1);
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      const CtrlHdr& c = p.ctrl->h;
      RaggedResult   r;
      r.status    = c.status ? c.status : p.ctrl->err;
      r.steps     = c.steps;
      r.levels    = c.levels;
      r.td_steps  = c.td_steps;
      r.bu_steps  = c.bu_steps;
      r.b2q_steps = c.b2q_steps;
      r.reached   = c.reached;
      rp.results[it] = r;
    }
    __syncthreads();
  }
}

// In-degree-zero bitmaps of every packed graph (bits past n set).
__global__ void k_zero_indegree_packed(const uint64_t* __restrict__ off, const RaggedGraph* __restrict__ graphs,
                                       uint32_t ngraphs, uint32_t* __restrict__ Z) {
  const unsigned lane = threadIdx.x & 31;
  for (uint32_t g = blockIdx.x; g < ngraphs; g += gridDim.x) {
    const RaggedGraph gr     = graphs[g];
    const uint64_t    nwords = (gr.n + 31) / 32;
    for (uint64_t w = threadIdx.x >> 5; w < nwords; w += blockDim.x >> 5) {
      const uint64_t u    = w * 32 + lane;
      const bool     zero = (u >= gr.n) || (off[gr.off_base + u + 1] == off[gr.off_base + u]);
      const unsigned b    = __ballot_sync(kFullMask, zero);
      if (lane == 0) Z[gr.z_base + w] = b;
    }
  }
}

int grid_for(const GraphDev* g, int per_sm) { return std::max(1, g->sm_count * per_sm); }

// Blocks of a grid-stride kernel that are resident at once (at most
// per_sm_cap per SM): its work is dealt out statically by block index, so a
// block that has to wait for a second wave would finish last.
template <class K>
int resident_grid(int sm_count, K kernel, int per_sm_cap) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return std::max(1, sm_count * std::min(per_sm, per_sm_cap));
}

}  // namespace

int ws_init(GraphDev* g, Workspace* ws) {
  ws->g      = g;
  ws->device = g->device;
  const uint64_t n      = g->n;
  const uint32_t nwords = (uint32_t)((n + 31) / 32);
  const uint64_t m      = g->m;
  // A vertex enters a queue at most once per level: n small entries.  The
  // chunked vertices have out-degree >= warp_min, so there are at most
  // m / warp_min of them, with at most m / chunk + that many chunk entries.
  const uint64_t qs_cap = std::max<uint64_t>(n, 1);
  const uint64_t big    = std::min<uint64_t>(n, m / g->th.warp_min);
  const uint64_t qc_cap = std::max<uint64_t>(1, m / g->th.chunk + big + 1);
  // deferred hubs have more than kLaneChunks chunks: out-degree > chunk * kLaneChunks
  const uint64_t hub_cap = m / ((uint64_t)g->th.chunk * kLaneChunks) + 1;

  NWG_CUDA_TRY(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
  NWG_CUDA_TRY(cudaEventCreate(&ws->ev0));
  NWG_CUDA_TRY(cudaEventCreate(&ws->ev1));
  if (cudaMalloc(&ws->parents, std::max<uint64_t>(n, 4) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&ws->V, 3ull * std::max<uint32_t>(nwords, 1) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&ws->qbuf, 2ull * qs_cap * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&ws->cbuf, 2ull * qc_cap * sizeof(uint64_t)) != cudaSuccess ||
      cudaMalloc(&ws->hubbuf, 2ull * hub_cap * sizeof(HubRec)) != cudaSuccess ||
      cudaMalloc(&ws->ctrl, sizeof(Ctrl)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(NWG_ENOMEM, "workspace allocation failed (n=" + std::to_string(n) + ")");
  }
  NWG_CUDA_TRY(cudaMallocHost(&ws->ctrl_host, sizeof(Ctrl)));
  NWG_CUDA_TRY(cudaMemset(ws->ctrl, 0, sizeof(Ctrl)));

  DobfsParams& P = ws->params;
  P.off          = g->off;
  P.col          = g->col;
  P.in_off       = g->in_off;
  P.in_col       = g->in_col;
  P.n            = n;
  P.m            = m;
  P.nwords       = nwords;
  P.V            = ws->V;
  P.C0           = ws->V + std::max<uint32_t>(nwords, 1);
  P.C1           = ws->V + 2ull * std::max<uint32_t>(nwords, 1);
  P.Z            = g->Z;
  P.deg16        = g->deg16;
  P.qs[0]        = ws->qbuf;
  P.qs[1]        = ws->qbuf + qs_cap;
  P.qc[0]        = ws->cbuf;
  P.qc[1]        = ws->cbuf + qc_cap;
  P.qs_cap       = qs_cap;
  P.qc_cap       = qc_cap;
  P.hubrec[0]    = ws->hubbuf;
  P.hubrec[1]    = ws->hubbuf + hub_cap;
  P.hub_cap      = hub_cap;
  P.th           = g->th;
  P.nzero        = g->nzero;
  P.symmetric    = g->symmetric ? 1u : 0u;
  P.ctrl         = ws->ctrl;
  // every block of the persistent kernel must be resident (cooperative launch)
  ws->trav_grid = resident_grid(g->sm_count, k_trav, kTravPerSm);
  return NWG_OK;
}

void ws_free(Workspace* ws) {
  if (!ws) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ws->device);
  if (ws->stream) cudaStreamSynchronize(ws->stream);
  if (ws->ev0) cudaEventDestroy(ws->ev0);
  if (ws->ev1) cudaEventDestroy(ws->ev1);
  if (ws->stream) cudaStreamDestroy(ws->stream);
  cudaFree(ws->parents);
  cudaFree(ws->V);
  cudaFree(ws->qbuf);
  cudaFree(ws->cbuf);
  cudaFree(ws->hubbuf);
  cudaFree(ws->ctrl);
  if (ws->ctrl_host) cudaFreeHost(ws->ctrl_host);
  cudaSetDevice(prev);
  delete ws;
}

// Cooperative launches of one device run one at a time, in launch order,
// whatever their streams: each waits (on the device, through an event) for
// the previous one to finish.  Two grids launched together on two streams
// (two server slots, two host threads) can each become only partly
// resident, each waiting at its grid barrier for blocks that only the
// other's exit would make room for; their bounded waits then end in
// NWG_ETIMEDOUT.  Other kernels may still run beside a cooperative grid:
// they wait for nothing, so they only delay its blocks.  A stream being
// captured into a CUDA graph launches directly (the capture cannot wait on
// an event recorded outside it); such graphs must not overlap.
static int coop_launch(const void* fn, dim3 grid, void** args, cudaStream_t stream) {
  struct Chain {
    std::mutex  mu;
    cudaEvent_t last = nullptr;
  };
  static std::mutex                 map_mu;
  static std::vector<Chain*>        chains;  // per device, never freed (process lifetime)
  int                               dev = 0;
  NWG_CUDA_TRY(cudaGetDevice(&dev));
  Chain* c = nullptr;
  {
    std::lock_guard<std::mutex> lk(map_mu);
    if ((int)chains.size() <= dev) chains.resize(dev + 1, nullptr);
    if (!chains[dev]) chains[dev] = new Chain();
    c = chains[dev];
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  NWG_CUDA_TRY(cudaStreamIsCapturing(stream, &cap));
  if (cap != cudaStreamCaptureStatusNone) {
    NWG_CUDA_TRY(cudaLaunchCooperativeKernel(fn, grid, dim3(kThreads), args, 0, stream));
    return NWG_OK;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  if (!c->last) {
    NWG_CUDA_TRY(cudaEventCreateWithFlags(&c->last, cudaEventDisableTiming));
  } else {
    NWG_CUDA_TRY(cudaStreamWaitEvent(stream, c->last, 0));
  }
  NWG_CUDA_TRY(cudaLaunchCooperativeKernel(fn, grid, dim3(kThreads), args, 0, stream));
  NWG_CUDA_TRY(cudaEventRecord(c->last, stream));
  return NWG_OK;
}

// A traversal on `stream`: the persistent traversal kernel, one cooperative
// launch after clearing its barrier's arrival count.
int ws_launch(Workspace* ws, uint32_t root, int alpha, int beta, uint32_t* parents, cudaStream_t stream,
              bool topdown_only) {
  GraphDev* g = ws->g;
  if (root >= g->n) return set_error(NWG_EINVAL, "root " + std::to_string(root) + " >= n " + std::to_string(g->n));
  if (alpha <= 0 || beta <= 0) return set_error(NWG_EINVAL, "alpha and beta must be positive");
  uint32_t  r = root, a = (uint32_t)alpha, b = (uint32_t)beta, td = topdown_only ? 1u : 0u;
  uint32_t* par    = parents ? parents : ws->parents;
  void*     args[] = {&ws->params, &r, &a, &b, &par, &td};
  NWG_CUDA_TRY(cudaMemsetAsync(&ws->ctrl->bar, 0, sizeof(GridBar), stream));
  const int rc = coop_launch((const void*)k_trav, dim3(ws->trav_grid), args, stream);
  if (rc) return rc;
  ws->ran = true;
  return NWG_OK;
}

// The level loop driven from the host: the kernels of the CUDA graph
// launched one at a time on `stream`, the decision read back after every
// step into host stack memory.  Allocates nothing.
int run_stepped(const DobfsParams& params, int sm_count, uint32_t root, int alpha, int beta, uint32_t* parents,
                cudaStream_t stream) {
  DobfsParams P = params;
  const int g_init = resident_grid(sm_count, k_init, 8);
  const int g_bu   = resident_grid(sm_count, k_bu, 8);
  const int g_b2q  = resident_grid(sm_count, k_b2q, 8);
  const int td     = std::max(1, sm_count * kTdPerSm);
  k_init<<<g_init, kThreads, 0, stream>>>(P, root, (uint32_t)alpha, (uint32_t)beta, parents, 0u);
  NWG_CUDA_TRY(cudaGetLastError());
  const uint64_t cap = 2 * P.n + 64;
  for (uint64_t step = 0; step <= cap; ++step) {
    k_decide<<<1, 32, 0, stream>>>(P);
    NWG_CUDA_TRY(cudaGetLastError());
    uint32_t action = kActNone;
    NWG_CUDA_TRY(cudaMemcpyAsync(&action, &P.ctrl->h.action, sizeof(action), cudaMemcpyDeviceToHost, stream));
    NWG_CUDA_TRY(cudaStreamSynchronize(stream));
    if (action == kActTD) {
      k_td<<<td, kThreads, 0, stream>>>(P);
    } else if (action == kActTDSmall) {
      void* args[] = {&P};
      const int rc = coop_launch((const void*)k_td_loop, dim3(kSmallBlocks), args, stream);
      if (rc) return rc;
    } else if (action == kActTDCluster) {
      k_td_cluster<<<kClusterCtas, kThreads, 0, stream>>>(P);  // one cluster (compiled-in cluster size)
    } else if (action == kActBU) {
      k_bu<<<g_bu, kThreads, 0, stream>>>(P);
    } else if (action == kActB2Q) {
      k_b2q<<<g_b2q, kThreads, 0, stream>>>(P);
    } else {
      break;
    }
    NWG_CUDA_TRY(cudaGetLastError());
  }
  return NWG_OK;
}

int ws_launch_stepped(Workspace* ws, uint32_t root, int alpha, int beta, uint32_t* parents, cudaStream_t stream) {
  GraphDev* g = ws->g;
  if (root >= g->n) return set_error(NWG_EINVAL, "root " + std::to_string(root) + " >= n " + std::to_string(g->n));
  if (alpha <= 0 || beta <= 0) return set_error(NWG_EINVAL, "alpha and beta must be positive");
  const int rc = run_stepped(ws->params, g->sm_count, root, alpha, beta, parents ? parents : ws->parents, stream);
  if (rc == NWG_OK) ws->ran = true;
  return rc;
}

int zero_indegree_into(const uint64_t* in_off, uint64_t n, uint32_t* Z, int sm_count, cudaStream_t stream) {
  const uint32_t nwords = (uint32_t)((n + 31) / 32);
  if (nwords) {
    k_zero_indegree<<<std::max(1, sm_count * 4), kThreads, 0, stream>>>(in_off, n, nwords, Z);
    NWG_CUDA_TRY(cudaGetLastError());
  }
  return NWG_OK;
}

void fill_stats(const Ctrl& c, nwg_bfs_stats* s) {
  s->status    = c.h.status ? c.h.status : c.err;
  // the persistent traversal kernel alone; or the init kernel, every decide,
  // and one action after each decide but the last
  s->kernel_launches = c.kernels ? c.kernels : 2 * c.decides;
  s->steps     = c.h.steps;
  s->levels    = c.h.levels;
  s->td_steps  = c.h.td_steps;
  s->bu_steps  = c.h.bu_steps;
  s->b2q_steps = c.h.b2q_steps;
  s->reached   = c.h.reached;
  s->trace_len = std::min<uint32_t>(c.h.trace_len, NWG_TRACE_CAP);
  for (uint32_t i = 0; i < s->trace_len; ++i) {
    s->trace_dir[i]      = c.trace_dir[i];
    s->trace_frontier[i] = c.trace_frontier[i];
    s->trace_found[i]    = c.trace_found[i];
    s->trace_end_ns[i]   = c.trace_end_ns[i];
  }
  s->first_decide_ns = c.t_first_decide;
}

// Builds the in-degree-zero bitmap Z and counts the vertices without
// in-edges (g->nzero; the bits past n are set in Z and not counted).
// Synchronises the stream.
int build_deg16(GraphDev* g, cudaStream_t stream) {
  NWG_CUDA_TRY(cudaMalloc(&g->deg16, std::max<uint64_t>(g->n, 1) * sizeof(uint16_t)));
  if (g->n) {
    k_deg16<<<grid_for(g, 4), kThreads, 0, stream>>>(g->off, g->n, g->deg16);
    NWG_CUDA_TRY(cudaGetLastError());
  }
  return NWG_OK;
}

int build_zero_indegree(GraphDev* g, cudaStream_t stream) {
  const uint32_t nwords = (uint32_t)((g->n + 31) / 32);
  NWG_CUDA_TRY(cudaMalloc(&g->Z, std::max<uint32_t>(nwords, 1) * sizeof(uint32_t)));
  g->nzero = 0;
  if (nwords) {
    k_zero_indegree<<<grid_for(g, 4), kThreads, 0, stream>>>(g->in_off, g->n, nwords, g->Z);
    NWG_CUDA_TRY(cudaGetLastError());
    unsigned long long* d = nullptr;
    NWG_CUDA_TRY(cudaMalloc(&d, sizeof(unsigned long long)));
    unsigned long long h  = 0;
    cudaError_t        e  = cudaMemsetAsync(d, 0, sizeof(h), stream);
    if (e == cudaSuccess) {
      k_popc_words<<<grid_for(g, 4), kThreads, 0, stream>>>(g->Z, nwords, d);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_error(e, "zero in-degree count");
    g->nzero = h - ((uint64_t)nwords * 32 - g->n);
  }
  return NWG_OK;
}

int component_edges(GraphDev* g, const uint32_t* parents, uint64_t* edges, uint64_t* vertices) {
  unsigned long long* d = nullptr;
  NWG_CUDA_TRY(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
  cudaMemset(d, 0, 2 * sizeof(unsigned long long));
  k_component<<<grid_for(g, 4), kThreads>>>(g->off, parents, g->n, d);
  unsigned long long h[2] = {0, 0};
  cudaError_t        e    = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_error(e, "component_edges");
  if (edges) *edges = h[0];
  if (vertices) *vertices = h[1];
  return NWG_OK;
}

int widen_offsets(const uint32_t* src, uint64_t* dst, uint64_t count, cudaStream_t stream) {
  k_widen<<<592, kThreads, 0, stream>>>(src, dst, count);
  NWG_CUDA_TRY(cudaGetLastError());
  return NWG_OK;
}

// One single-source traversal on workspace ws (its graph) and the uint16
// depth row of every vertex from its parents (row[v], 0xFFFF = unreached).
// The pointer-jumping pairs use the workspace's small-queue buffers (2 n
// uint32 entries), which the finished traversal no longer needs.  Returns
// NWG_EOVERFLOW when a depth does not fit uint16.
int depth_row16(Workspace* ws, uint32_t root, uint16_t* row, cudaStream_t stream) {
  GraphDev* g = ws->g;
  int       rc = ws_launch(ws, root, 15, 18, ws->parents, stream, false);
  if (rc) return rc;
  const uint64_t      n    = g->n;
  unsigned long long* pair = reinterpret_cast<unsigned long long*>(ws->qbuf);
  int* flag = reinterpret_cast<int*>(&ws->ctrl->err);  // the traversal's sticky error word, zero after a clean run
  const int grid = grid_for(g, 4);
  k_jump_init<<<grid, kThreads, 0, stream>>>(ws->parents, n, root, pair);
  NWG_CUDA_TRY(cudaGetLastError());
  int rounds = 1;
  while ((1ull << (rounds - 1)) < n) ++rounds;  // ceil(log2 n) + 1
  for (int r = 0; r < rounds; ++r) {
    k_jump_round<<<grid, kThreads, 0, stream>>>(n, pair);
    NWG_CUDA_TRY(cudaGetLastError());
  }
  k_jump_row16<<<grid, kThreads, 0, stream>>>(pair, n, row, flag);
  NWG_CUDA_TRY(cudaGetLastError());
  int32_t status[2] = {0, 0};
  NWG_CUDA_TRY(cudaMemcpyAsync(&status[0], &ws->ctrl->h.status, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
  NWG_CUDA_TRY(cudaMemcpyAsync(&status[1], flag, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
  NWG_CUDA_TRY(cudaStreamSynchronize(stream));
  if (status[0] != 0) return set_error(status[0], "single-source traversal of a deep source failed");
  if (status[1] != 0) return set_error(NWG_EOVERFLOW, "a depth reaches 65535: does not fit the uint16 encoding");
  return NWG_OK;
}

int ragged_slot_bytes(uint64_t nmax, uint64_t mmax, uint64_t* bytes) {
  *bytes = slot_layout(nmax, mmax).bytes;
  return NWG_OK;
}

int zero_indegree_packed(RaggedDev* r) {
  if (r->ngraphs == 0) return NWG_OK;
  k_zero_indegree_packed<<<std::max(1, r->sm_count * 4), kThreads>>>(r->off, r->graphs, r->ngraphs, r->Z);
  NWG_CUDA_TRY(cudaGetLastError());
  return NWG_OK;
}

// One persistent launch over the r->items table (already on the device),
// captured into a CUDA graph with the counter reset and replayed while the
// item count, slot count and output buffer stay the same.
int ragged_launch(RaggedDev* r, uint32_t n_items, uint32_t* parents_dev, uint32_t blocks_per_sm, float* ms) {
  const uint32_t slots = (uint32_t)std::max(1, r->sm_count * (int)blocks_per_sm);
  if (!r->exec || r->exec_items != n_items || r->exec_slots != slots || r->exec_parents != parents_dev) {
    if (r->exec) {
      cudaGraphExecDestroy(r->exec);
      r->exec = nullptr;
    }
    RaggedParams rp = {};
    rp.off          = r->off;
    rp.col          = r->col;
    rp.Z            = r->Z;
    rp.graphs       = r->graphs;
    rp.items        = r->items;
    rp.results      = r->results;
    rp.parents      = parents_dev;
    rp.n_items      = n_items;
    rp.next_item    = r->counter;
    rp.scratch      = r->scratch;
    rp.slot_bytes   = slot_layout(r->nmax, r->mmax).bytes;
    rp.nmax         = r->nmax;
    rp.mmax         = r->mmax;
    cudaGraph_t graph;
    NWG_CUDA_TRY(cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(r->counter, 0, sizeof(unsigned int), r->stream);
    k_ragged<<<slots, kThreads, 0, r->stream>>>(rp);
    const cudaError_t le = cudaGetLastError();
    const cudaError_t ce = cudaStreamEndCapture(r->stream, &graph);
    if (le != cudaSuccess) return cuda_error(le, "k_ragged launch (capture)");
    if (ce != cudaSuccess) return cuda_error(ce, "cudaStreamEndCapture(ragged)");
    const cudaError_t ie = cudaGraphInstantiate(&r->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return cuda_error(ie, "cudaGraphInstantiate(ragged)");
    r->exec_items   = n_items;
    r->exec_slots   = slots;
    r->exec_parents = parents_dev;
  }
  NWG_CUDA_TRY(cudaEventRecord(r->ev0, r->stream));
  NWG_CUDA_TRY(cudaGraphLaunch(r->exec, r->stream));
  NWG_CUDA_TRY(cudaEventRecord(r->ev1, r->stream));
  NWG_CUDA_TRY(cudaEventSynchronize(r->ev1));
  if (ms) cudaEventElapsedTime(ms, r->ev0, r->ev1);
  return NWG_OK;
}

// Failure-detection probe: the persistent traversal kernel's grid barrier,
// waited on for one more block than the grid has, so no one ever releases
// it.  Every block gives up after max_spins polls, records NWG_ETIMEDOUT and
// returns -- the path a real barrier takes when a block never arrives.
__global__ void k_wait_probe(DobfsParams p, unsigned max_spins) {
  const bool ok = trav_barrier(p, gridDim.x + 1, max_spins);
  if (!ok && threadIdx.x == 0 && blockIdx.x == 0) p.ctrl->h.status = __ldcg(&p.ctrl->err);
}

int wait_probe(uint32_t spins, int32_t* status, float* waited_ms) {
  Ctrl* ctrl = nullptr;
  if (cudaMalloc(&ctrl, sizeof(Ctrl)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(NWG_ENOMEM, "probe control block");
  }
  DobfsParams p = {};
  p.ctrl        = ctrl;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e  = cudaMemset(ctrl, 0, sizeof(Ctrl));
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e == cudaSuccess) e = cudaEventRecord(e0, 0);
  if (e == cudaSuccess) {
    k_wait_probe<<<2, kThreads, 0, 0>>>(p, spins);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1, 0);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  int32_t st = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&st, &ctrl->h.status, sizeof st, cudaMemcpyDeviceToHost);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(ctrl);
  if (e != cudaSuccess) return cuda_error(e, "wait probe");
  *status    = st;
  *waited_ms = ms;
  return NWG_OK;
}

}  // namespace nwg
