// Direction-optimizing BFS on sm_100a: the device level loop.
//
// Restates nw::graph::bfs(out, in, root, num_bins, alpha, beta)
// (include/nwgraph/algorithms/bfs.hpp:160-311 in NWGraph) as a CUDA graph:
//
//   k_init ──► WHILE(h_loop) { k_decide ──► SWITCH(h_switch) { k_td | k_bu | k_b2q } }
//
// k_decide is a one-thread kernel that reproduces the reference's integer
// switch rules exactly (scout_count > edges_to_check / alpha selects
// bottom-up, bfs.hpp:186; stay bottom-up while awake >= old_awake or
// awake > N / beta, bfs.hpp:229; scout_count = 1 after a bottom-up phase,
// bfs.hpp:241; stop when the next queue is empty, bfs.hpp:297-303, or a pull
// finds nothing, bfs.hpp:231-233) and sets the graph's conditional handles,
// so no level makes a host round trip.
//
// Device state (HBM, all uint32 words):
//   parents[n]   output; null = 0xFFFFFFFF
//   V[n/32]      visited bitmap.  The top-down step sets a vertex's bit with
//                atomicOr when it claims it (this is the queue->bitmap
//                conversion of bfs.hpp:199-202, fused into the step that
//                fills the queue), and the claim decides which discoverer
//                writes parents[v] (the CAS of bfs.hpp:283).
//   C0/C1[n/32]  discoveries of the latest bottom-up pulls (bfs.hpp:205-229's
//                front/curr pair).
//   Z[n/32]      vertices with no in-edges, never candidates of a pull.
//   q[2][4][..]  frontier queues, binned by out-degree (thread-gather, warp,
//                CTA, grid) instead of the reference's u % 32 bins.
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

#include "nwg_internal.cuh"

namespace nwg {
namespace {

constexpr int kThreads = 256;
constexpr int kBuProbe = 4;  // sequential in-edge probes per lane before the warp helps

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
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

// ---------------------------------------------------------------------------
// k_init: parents := null except root (bfs.hpp:175,180), V := {root},
// control block := the reference's initial state (bfs.hpp:166-181).
__global__ void __launch_bounds__(kThreads) k_init(DobfsParams p, uint32_t root, uint32_t alpha, uint32_t beta,
                                                   uint32_t* parents, uint32_t topdown_only) {
  const uint64_t n      = p.n;
  const uint64_t tid    = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
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

  if (tid == 0) {
    Ctrl&          c   = *p.ctrl;
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
    for (int b = 0; b < kNumBins; ++b) c.qcount[0][b] = c.qcount[1][b] = 0;
    const int b = degree_bin(deg, p.th);
    p.q[0][b][0] = root;
    c.qcount[0][b] = 1;
    c.cur       = 0;
    c.bm        = 1;
    c.bu_mode   = 0;
    c.action    = kActNone;
    c.steps     = 0;
    c.levels    = 1;
    c.td_steps  = 0;
    c.bu_steps  = 0;
    c.b2q_steps = 0;
    c.status    = 0;
    c.reached   = 1;
    c.trace_len = 0;
    const uint64_t cap = 2 * n + 64;
    c.max_steps = cap > 0xFFFFFF00ull ? 0xFFFFFF00u : (uint32_t)cap;
  }
}

__device__ __forceinline__ uint64_t qsum(const Ctrl& c, uint32_t qi) {
  uint64_t s = 0;
#pragma unroll
  for (int b = 0; b < kNumBins; ++b) s += c.qcount[qi][b];
  return s;
}

__device__ __forceinline__ void trace_add(Ctrl& c, uint8_t dir, uint64_t frontier, uint64_t found) {
  if (c.trace_len < NWG_TRACE_CAP) {
    c.trace_dir[c.trace_len]      = dir;
    c.trace_frontier[c.trace_len] = frontier;
    c.trace_found[c.trace_len]    = found;
    c.trace_len++;
  }
}

// ---------------------------------------------------------------------------
// k_decide: one thread; consumes the previous action's counters and picks the
// next action.  Every branch below cites the reference line it reproduces.
__global__ void k_decide(DobfsParams p) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Ctrl&          c    = *p.ctrl;
  const uint64_t N    = p.n;
  uint32_t       next = kActNone;
  bool           done = false, queue_decision = false;

  switch (c.action) {
    case kActNone:  // first iteration: frontier = {root}
      queue_decision = true;
      break;
    case kActTD: {
      const uint32_t nxt = c.cur ^ 1u;
      const uint64_t nq  = qsum(c, nxt);
      trace_add(c, 0, qsum(c, c.cur), nq);
      c.td_steps++;
      c.reached += nq;
      c.scout_count = c.acc_scout;  // bfs.hpp:271
      c.cur         = nxt;          // swap(q1, q2), bfs.hpp:304
      if (nq == 0) {
        done = true;  // all q2 bins empty, bfs.hpp:297-303
      } else {
        c.levels++;
        queue_decision = true;
      }
      break;
    }
    case kActBU: {
      const uint64_t awake = c.acc_awake;
      trace_add(c, 1, c.old_awake, awake);
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
        for (int b = 0; b < kNumBins; ++b) c.qcount[c.cur][b] = 0;
        next = kActB2Q;  // bfs.hpp:235-239
      }
      break;
    }
    case kActB2Q:
      c.b2q_steps++;
      c.scout_count  = 1;  // bfs.hpp:241
      queue_decision = true;
      break;
    default:
      c.status = NWG_ESTATE;
      done     = true;
      break;
  }

  if (queue_decision) {
    const uint64_t nq = qsum(c, c.cur);
    if (!c.topdown_only && c.scout_count > c.edges_to_check / c.alpha) {  // bfs.hpp:186
      c.awake_count = nq;                                                // bfs.hpp:199-202
      c.old_awake   = nq;
      c.acc_awake   = 0;
      c.bu_mode     = 0;
      c.bm          = 1;  // the first pull writes C0
      next          = kActBU;
    } else {
      c.edges_to_check -= c.scout_count;  // bfs.hpp:244
      const uint32_t nxt = c.cur ^ 1u;
      for (int b = 0; b < kNumBins; ++b) c.qcount[nxt][b] = 0;
      c.acc_scout = 0;
      next        = kActTD;
    }
  }
  if (!done && ++c.steps > c.max_steps) {
    c.status = NWG_ETIMEDOUT;  // loop bound; a BFS needs at most ~2n actions
  }
  if (c.status != 0) done = true;
  c.action = done ? kActNone : next;
  cudaGraphSetConditional(p.h_switch, done ? (unsigned)kActNone : next);
  cudaGraphSetConditional(p.h_loop, done ? 0u : 1u);
}

// ---------------------------------------------------------------------------
// Warp-aggregated append of discovered vertices into the degree-binned queue
// `qi`: one atomicAdd per (warp, bin) instead of one per vertex.  All 32
// lanes must call.
__device__ __forceinline__ void append_binned(const DobfsParams& p, uint32_t qi, bool has, uint32_t v, int bin) {
  Ctrl*          c    = p.ctrl;
  const unsigned lane = threadIdx.x & 31;
#pragma unroll
  for (int b = 0; b < kNumBins; ++b) {
    const unsigned m = __ballot_sync(kFullMask, has && bin == b);
    if (m == 0) continue;
    const int leader = __ffs(m) - 1;
    uint32_t  base   = 0;
    if ((int)lane == leader) base = atomicAdd(&c->qcount[qi][b], (uint32_t)__popc(m));
    base = __shfl_sync(kFullMask, base, leader);
    if (has && bin == b) {
      const uint32_t pos = base + __popc(m & lanemask_lt());
      if (pos < p.qcap[b]) {
        p.q[qi][b][pos] = v;
      } else {
        c->status = NWG_EOVERFLOW;
      }
    }
  }
}

// One top-down edge test u -> v (bfs.hpp:280-289): claim v in V; the winner
// writes parents[v] = u, adds out-degree(v) to scout and appends v.
// All 32 lanes must call.
__device__ __forceinline__ void td_visit(const DobfsParams& p, uint32_t* __restrict__ parents, uint32_t nxt,
                                         bool valid, uint32_t u, uint32_t v, unsigned long long& scout) {
  bool win = false;
  if (valid) {
    const uint32_t w   = v >> 5;
    const uint32_t bit = 1u << (v & 31);
    if (!(__ldcg(p.V + w) & bit)) {
      const uint32_t old = atomicOr(p.V + w, bit);
      win                = !(old & bit);
    }
  }
  if (__ballot_sync(kFullMask, win) == 0) return;
  int bin = 0;
  if (win) {
    parents[v]       = u;
    const uint64_t d = p.off[v + 1] - p.off[v];
    scout += d;
    bin = degree_bin(d, p.th);
  }
  append_binned(p, nxt, win, v, bin);
}

// Expand out-edges [beg, end) of u with `nthr` cooperating threads (rank
// `tr`); 128-bit non-coherent loads for the 16-byte-aligned body.  Trip
// counts depend only on (beg, end, nthr), so every warp stays converged.
__device__ __forceinline__ void expand_range(const DobfsParams& p, uint32_t* __restrict__ parents, uint32_t nxt,
                                             uint32_t u, uint64_t beg, uint64_t end, uint32_t tr, uint32_t nthr,
                                             unsigned long long& scout) {
  const uint64_t a = min(end, (beg + 3) & ~(uint64_t)3);
  for (uint64_t base = beg; base < a; base += nthr) {  // unaligned head (< 4 entries)
    const uint64_t i     = base + tr;
    const bool     valid = i < a;
    td_visit(p, parents, nxt, valid, u, valid ? __ldg(p.col + i) : 0u, scout);
  }
  const uint64_t nvec = (end - a) >> 2;
  const uint4*   col4 = reinterpret_cast<const uint4*>(p.col + a);
  for (uint64_t base = 0; base < nvec; base += nthr) {
    const uint64_t i     = base + tr;
    const bool     valid = i < nvec;
    uint4          x     = make_uint4(0, 0, 0, 0);
    if (valid) x = __ldg(col4 + i);
    td_visit(p, parents, nxt, valid, u, x.x, scout);
    td_visit(p, parents, nxt, valid, u, x.y, scout);
    td_visit(p, parents, nxt, valid, u, x.z, scout);
    td_visit(p, parents, nxt, valid, u, x.w, scout);
  }
  const uint64_t t0 = a + (nvec << 2);
  for (uint64_t base = t0; base < end; base += nthr) {  // tail (< 4 entries)
    const uint64_t i     = base + tr;
    const bool     valid = i < end;
    td_visit(p, parents, nxt, valid, u, valid ? __ldg(p.col + i) : 0u, scout);
  }
}

// ---------------------------------------------------------------------------
// k_td: one top-down step (bfs.hpp:242-295) over the four degree bins.
__global__ void __launch_bounds__(kThreads) k_td(DobfsParams p) {
  Ctrl*           c       = p.ctrl;
  const uint32_t  cur     = c->cur;
  const uint32_t  nxt     = cur ^ 1u;
  uint32_t* const parents = c->parents;
  const uint32_t  nS = c->qcount[cur][kBinS], nM = c->qcount[cur][kBinM];
  const uint32_t  nL = c->qcount[cur][kBinL], nH = c->qcount[cur][kBinH];
  const unsigned  lane   = threadIdx.x & 31;
  const uint64_t  wpb    = blockDim.x >> 5;
  const uint64_t  gwarp  = blockIdx.x * wpb + (threadIdx.x >> 5);
  const uint64_t  nwarps = gridDim.x * wpb;
  unsigned long long scout = 0;

  // H: every CTA takes chunks of each huge vertex's edge list.
  const uint64_t chunk = (uint64_t)blockDim.x * 16;
  for (uint32_t i = 0; i < nH; ++i) {
    const uint32_t u   = p.q[cur][kBinH][i];
    const uint64_t beg = p.off[u], end = p.off[u + 1];
    const uint64_t nch = (end - beg + chunk - 1) / chunk;
    for (uint64_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
      const uint64_t cb = beg + ch * chunk;
      expand_range(p, parents, nxt, u, cb, min(end, cb + chunk), threadIdx.x, blockDim.x, scout);
    }
  }
  // L: one CTA per vertex.
  for (uint32_t i = blockIdx.x; i < nL; i += gridDim.x) {
    const uint32_t u = p.q[cur][kBinL][i];
    expand_range(p, parents, nxt, u, p.off[u], p.off[u + 1], threadIdx.x, blockDim.x, scout);
  }
  // M: one warp per vertex.
  for (uint64_t i = gwarp; i < nM; i += nwarps) {
    const uint32_t u = p.q[cur][kBinM][i];
    expand_range(p, parents, nxt, u, p.off[u], p.off[u + 1], lane, 32, scout);
  }
  // S: 32 low-degree vertices per warp, their edge lists flattened by a warp
  // scan and dealt out one edge per lane (scan-based gather).
  for (uint64_t g0 = gwarp * 32; g0 < nS; g0 += nwarps * 32) {
    const uint64_t qi   = g0 + lane;
    const bool     have = qi < nS;
    const uint32_t u    = have ? p.q[cur][kBinS][qi] : 0u;
    const uint64_t beg  = have ? p.off[u] : 0;
    const uint32_t deg  = have ? (uint32_t)(p.off[u + 1] - beg) : 0u;
    uint32_t       incl = deg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(kFullMask, incl, o);
      if ((int)lane >= o) incl += t;
    }
    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
    const uint32_t excl  = incl - deg;
    for (uint32_t j = 0; j < total; j += 32) {
      const uint32_t e     = j + lane;
      const bool     valid = e < total;
      int            lo    = 0;  // largest lane whose exclusive prefix <= e
#pragma unroll
      for (int s = 16; s >= 1; s >>= 1) {
        const uint32_t ex = __shfl_sync(kFullMask, excl, lo + s);
        if (ex <= e) lo += s;
      }
      const uint32_t ex_o  = __shfl_sync(kFullMask, excl, lo);
      const uint64_t beg_o = __shfl_sync(kFullMask, beg, lo);
      const uint32_t u_o   = __shfl_sync(kFullMask, u, lo);
      const uint32_t v     = valid ? __ldg(p.col + beg_o + (e - ex_o)) : 0u;
      td_visit(p, parents, nxt, valid, u_o, v, scout);
    }
  }

  const unsigned long long tot = block_sum(scout);
  if (threadIdx.x == 0 && tot) atomicAdd(&c->acc_scout, tot);
}

// ---------------------------------------------------------------------------
// k_bu: one bottom-up pull (bfs.hpp:211-228).  A warp owns 32 vertices (one
// bitmap word): it skips the word when none is a candidate, each candidate
// lane probes its first in-edges, and the warp then scans the remaining
// in-edges of unresolved lanes 32 at a time, stopping at the first hit.  The
// first hit in row order becomes the parent, exactly as the reference's
// sequential scan with break.
__global__ void __launch_bounds__(kThreads) k_bu(DobfsParams p) {
  Ctrl*           c       = p.ctrl;
  const uint32_t  mode    = c->bu_mode;
  const uint32_t  bm      = c->bm;
  uint32_t* const parents = c->parents;
  const uint32_t* Cf      = bm ? p.C1 : p.C0;  // previous pull's discoveries
  uint32_t*       Cw      = bm ? p.C0 : p.C1;  // this pull's discoveries
  const uint32_t* front   = mode ? Cf : p.V;
  const unsigned  lane    = threadIdx.x & 31;
  const uint64_t  wpb     = blockDim.x >> 5;
  const uint64_t  gwarp   = blockIdx.x * wpb + (threadIdx.x >> 5);
  const uint64_t  nwarps  = gridDim.x * wpb;
  uint32_t        awake   = 0;

  for (uint64_t w = gwarp; w < p.nwords; w += nwarps) {
    const uint32_t vw = p.V[w];
    const uint32_t fw = mode ? Cf[w] : 0u;
    if (fw && lane == 0) p.V[w] = vw | fw;  // fold the previous pull into V
    const uint32_t cand  = ~(vw | fw) & ~p.Z[w];
    bool           found = false;
    uint32_t       par   = 0;
    if (cand) {
      const uint64_t u    = w * 32 + lane;
      const bool     mine = (cand >> lane) & 1u;
      uint64_t       beg = 0, end = 0;
      if (mine) {
        beg = p.in_off[u];
        end = p.in_off[u + 1];
      }
      const uint64_t lim = min(end, beg + kBuProbe);
      uint64_t       e   = beg;
      for (; e < lim; ++e) {
        const uint32_t v = __ldg(p.in_col + e);
        if ((__ldg(front + (v >> 5)) >> (v & 31)) & 1u) {
          found = true;
          par   = v;
          break;
        }
      }
      unsigned pend = __ballot_sync(kFullMask, mine && !found && e < end);
      while (pend) {
        const int leader = __ffs(pend) - 1;
        pend &= pend - 1;
        const uint64_t b  = __shfl_sync(kFullMask, e, leader);
        const uint64_t en = __shfl_sync(kFullMask, end, leader);
        for (uint64_t base = b; base < en; base += 32) {
          const uint64_t i = base + lane;
          uint32_t       v = 0;
          bool           h = false;
          if (i < en) {
            v = __ldg(p.in_col + i);
            h = (__ldg(front + (v >> 5)) >> (v & 31)) & 1u;
          }
          const unsigned hm = __ballot_sync(kFullMask, h);
          if (hm) {
            const uint32_t pv = __shfl_sync(kFullMask, v, __ffs(hm) - 1);
            if ((int)lane == leader) {
              found = true;
              par   = pv;
            }
            break;
          }
        }
      }
    }
    const unsigned nb = __ballot_sync(kFullMask, found);
    if (found) parents[w * 32 + lane] = par;
    if (lane == 0) {
      Cw[w] = nb;
      awake += __popc(nb);
    }
  }
  const uint32_t tot = block_sum(awake);
  if (threadIdx.x == 0 && tot) atomicAdd(&c->acc_awake, (unsigned long long)tot);
}

// ---------------------------------------------------------------------------
// k_b2q: bitmap -> binned queue (bfs.hpp:235-239) from C[bm], folding C[bm]
// into V on the way.  Each warp reads 32 words and expands the non-zero ones
// one at a time, one bit per lane.
__global__ void __launch_bounds__(kThreads) k_b2q(DobfsParams p) {
  Ctrl*           c      = p.ctrl;
  const uint32_t* Cs     = c->bm ? p.C1 : p.C0;
  const uint32_t  qi     = c->cur;
  const unsigned  lane   = threadIdx.x & 31;
  const uint64_t  wpb    = blockDim.x >> 5;
  const uint64_t  gwarp  = blockIdx.x * wpb + (threadIdx.x >> 5);
  const uint64_t  nwarps = gridDim.x * wpb;
  for (uint64_t w0 = gwarp * 32; w0 < p.nwords; w0 += nwarps * 32) {
    const uint64_t w = w0 + lane;
    const uint32_t x = (w < p.nwords) ? Cs[w] : 0u;
    if (x) p.V[w] |= x;
    unsigned nz = __ballot_sync(kFullMask, x != 0);
    while (nz) {
      const int src = __ffs(nz) - 1;
      nz &= nz - 1;
      const uint32_t word = __shfl_sync(kFullMask, x, src);
      const uint32_t v    = (uint32_t)((w0 + src) * 32 + lane);
      const bool     has  = (word >> lane) & 1u;
      int            bin  = 0;
      if (has) bin = degree_bin(p.off[v + 1] - p.off[v], p.th);
      append_binned(p, qi, has, v, bin);
    }
  }
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

__global__ void k_widen(const uint32_t* __restrict__ src, uint64_t* __restrict__ dst, uint64_t count) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

int grid_for(const GraphDev* g, int per_sm) { return std::max(1, g->sm_count * per_sm); }

// Builds the level-loop CUDA graph of a workspace.
int build_exec(Workspace* ws) {
  GraphDev*   g = ws->g;
  cudaGraph_t graph;
  NWG_CUDA_TRY(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle h_loop, h_switch;
  NWG_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_loop, graph, 1, cudaGraphCondAssignDefault));

  DobfsParams& P     = ws->params;
  uint32_t     root0 = 0, alpha0 = 15, beta0 = 18, td0 = 0;
  uint32_t*    par0  = ws->parents;
  void*        init_args[] = {&P, &root0, &alpha0, &beta0, &par0, &td0};

  cudaKernelNodeParams kp = {};
  kp.func                 = (void*)k_init;
  kp.gridDim              = dim3(grid_for(g, 8));
  kp.blockDim             = dim3(kThreads);
  kp.kernelParams         = init_args;
  cudaGraphNode_t init_node;
  NWG_CUDA_TRY(cudaGraphAddKernelNode(&init_node, graph, nullptr, 0, &kp));

  cudaGraphNodeParams wp = {};
  wp.type                = cudaGraphNodeTypeConditional;
  wp.conditional.handle  = h_loop;
  wp.conditional.type    = cudaGraphCondTypeWhile;
  wp.conditional.size    = 1;
  cudaGraphNode_t while_node;
  NWG_CUDA_TRY(cudaGraphAddNode(&while_node, graph, &init_node, 1, &wp));
  cudaGraph_t body = wp.conditional.phGraph_out[0];

  NWG_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_switch, body, kActNone, cudaGraphCondAssignDefault));
  P.h_loop   = h_loop;
  P.h_switch = h_switch;

  void*                decide_args[] = {&P};
  cudaKernelNodeParams dp            = {};
  dp.func                            = (void*)k_decide;
  dp.gridDim                         = dim3(1);
  dp.blockDim                        = dim3(32);
  dp.kernelParams                    = decide_args;
  cudaGraphNode_t decide_node;
  NWG_CUDA_TRY(cudaGraphAddKernelNode(&decide_node, body, nullptr, 0, &dp));

  cudaGraphNodeParams sp = {};
  sp.type                = cudaGraphNodeTypeConditional;
  sp.conditional.handle  = h_switch;
  sp.conditional.type    = cudaGraphCondTypeSwitch;
  sp.conditional.size    = kNumActions;
  cudaGraphNode_t switch_node;
  NWG_CUDA_TRY(cudaGraphAddNode(&switch_node, body, &decide_node, 1, &sp));

  void* (kernels[kNumActions]) = {(void*)k_td, (void*)k_bu, (void*)k_b2q};
  const int per_sm[kNumActions] = {8, 8, 8};
  for (int a = 0; a < kNumActions; ++a) {
    void*                args[] = {&P};
    cudaKernelNodeParams ap     = {};
    ap.func                     = kernels[a];
    ap.gridDim                  = dim3(grid_for(g, per_sm[a]));
    ap.blockDim                 = dim3(kThreads);
    ap.kernelParams             = args;
    cudaGraphNode_t n;
    NWG_CUDA_TRY(cudaGraphAddKernelNode(&n, sp.conditional.phGraph_out[a], nullptr, 0, &ap));
  }

  cudaGraphExec_t exec;
  cudaError_t     e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return cuda_error(e, "cudaGraphInstantiate(level loop)");
  }
  ws->exec[0]      = exec;
  ws->init_node[0] = init_node;
  ws->template_graph = graph;
  return NWG_OK;
}

}  // namespace

int ws_init(GraphDev* g, Workspace* ws) {
  ws->g      = g;
  ws->device = g->device;
  const uint64_t n      = g->n;
  const uint32_t nwords = (uint32_t)((n + 31) / 32);
  const uint64_t m      = g->m;
  uint64_t       cap[kNumBins];
  cap[kBinS] = std::max<uint64_t>(n, 1);
  cap[kBinM] = std::max<uint64_t>(1, std::min<uint64_t>(n, m / g->th.warp_min + 1));
  cap[kBinL] = std::max<uint64_t>(1, std::min<uint64_t>(n, m / g->th.cta_min + 1));
  cap[kBinH] = std::max<uint64_t>(1, std::min<uint64_t>(n, m / g->th.grid_min + 1));
  uint64_t qtot = 0;
  for (int b = 0; b < kNumBins; ++b) qtot += cap[b];

  NWG_CUDA_TRY(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
  NWG_CUDA_TRY(cudaEventCreate(&ws->ev0));
  NWG_CUDA_TRY(cudaEventCreate(&ws->ev1));
  if (cudaMalloc(&ws->parents, std::max<uint64_t>(n, 4) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&ws->V, 3ull * std::max<uint32_t>(nwords, 1) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&ws->qbuf, 2ull * qtot * sizeof(uint32_t)) != cudaSuccess ||
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
  uint32_t* qp   = ws->qbuf;
  for (int q = 0; q < 2; ++q)
    for (int b = 0; b < kNumBins; ++b) {
      P.q[q][b] = qp;
      qp += cap[b];
    }
  for (int b = 0; b < kNumBins; ++b) P.qcap[b] = (uint32_t)std::min<uint64_t>(cap[b], 0xFFFFFFFFull);
  P.th   = g->th;
  P.ctrl = ws->ctrl;
  return build_exec(ws);
}

void ws_free(Workspace* ws) {
  if (!ws) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ws->device);
  if (ws->stream) cudaStreamSynchronize(ws->stream);
  if (ws->exec[0]) cudaGraphExecDestroy(ws->exec[0]);
  if (ws->template_graph) cudaGraphDestroy(ws->template_graph);
  if (ws->ev0) cudaEventDestroy(ws->ev0);
  if (ws->ev1) cudaEventDestroy(ws->ev1);
  if (ws->stream) cudaStreamDestroy(ws->stream);
  cudaFree(ws->parents);
  cudaFree(ws->V);
  cudaFree(ws->qbuf);
  cudaFree(ws->ctrl);
  if (ws->ctrl_host) cudaFreeHost(ws->ctrl_host);
  cudaSetDevice(prev);
  delete ws;
}

int ws_launch(Workspace* ws, uint32_t root, int alpha, int beta, uint32_t* parents, cudaStream_t stream,
              bool topdown_only) {
  GraphDev* g = ws->g;
  if (root >= g->n) return set_error(NWG_EINVAL, "root " + std::to_string(root) + " >= n " + std::to_string(g->n));
  if (alpha <= 0 || beta <= 0) return set_error(NWG_EINVAL, "alpha and beta must be positive");
  uint32_t  r = root, a = (uint32_t)alpha, b = (uint32_t)beta, td = topdown_only ? 1u : 0u;
  uint32_t* par = parents ? parents : ws->parents;
  void*     args[] = {&ws->params, &r, &a, &b, &par, &td};
  cudaKernelNodeParams kp = {};
  kp.func                 = (void*)k_init;
  kp.gridDim              = dim3(grid_for(g, 8));
  kp.blockDim             = dim3(kThreads);
  kp.kernelParams         = args;
  NWG_CUDA_TRY(cudaGraphExecKernelNodeSetParams(ws->exec[0], ws->init_node[0], &kp));
  NWG_CUDA_TRY(cudaGraphLaunch(ws->exec[0], stream));
  ws->ran = true;
  return NWG_OK;
}

void fill_stats(const Ctrl& c, nwg_bfs_stats* s) {
  s->status    = c.status;
  s->steps     = c.steps;
  s->levels    = c.levels;
  s->td_steps  = c.td_steps;
  s->bu_steps  = c.bu_steps;
  s->b2q_steps = c.b2q_steps;
  s->reached   = c.reached;
  s->trace_len = std::min<uint32_t>(c.trace_len, NWG_TRACE_CAP);
  for (uint32_t i = 0; i < s->trace_len; ++i) {
    s->trace_dir[i]      = c.trace_dir[i];
    s->trace_frontier[i] = c.trace_frontier[i];
    s->trace_found[i]    = c.trace_found[i];
  }
}

int build_zero_indegree(GraphDev* g, cudaStream_t stream) {
  const uint32_t nwords = (uint32_t)((g->n + 31) / 32);
  NWG_CUDA_TRY(cudaMalloc(&g->Z, std::max<uint32_t>(nwords, 1) * sizeof(uint32_t)));
  if (nwords) {
    k_zero_indegree<<<grid_for(g, 4), kThreads, 0, stream>>>(g->in_off, g->n, nwords, g->Z);
    NWG_CUDA_TRY(cudaGetLastError());
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

}  // namespace nwg
