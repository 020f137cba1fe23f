// Approximate betweenness centrality over a list of sources (Brandes), the
// computation of NWGraph's brandes_bc<float, double>(graph, sources, threads,
// ..., normalize) (include/nwgraph/algorithms/betweenness_centrality.hpp:
// 218-324 in NWGraph), on the GPU.
//
// Per source, over the out-graph:
//   forward  -- level-synchronous BFS from the source; every edge u -> v with
//               level[v] == level[u] + 1 adds path_counts[u] to
//               path_counts[v] (double; the reference's accum_t).  That edge
//               test is the reference's succ bit (set when v is new or on
//               the level being built, :262-266), recomputed instead of
//               stored.
//   backward -- levels deepest first: delta[u] = sum over those edges of
//               path_counts[u] / path_counts[v] * (1 + delta[v]), and
//               bc[u] += delta[u] for every reached vertex, the source
//               included (:297-307).
// Then bc /= max(bc) when normalizing (:316-319).
//
// Work split: a level's vertices (contiguous in the BFS order array) are
// cut into tasks of at most kBcTask out-edges; a prefix sum over the task
// counts maps a task to its vertex.  A warp runs a task.  The forward phase
// claims levels with atomicCAS and adds path counts with double atomics
// (integers: exact below 2^53, so the order of the adds does not matter);
// the backward phase sums a task's terms with a warp reduction and adds one
// double per task.
// Every vertex's level, dependency and path count (or, once its dependency
// is final, its weight) share one 16-byte record.  Several sources run at once, one host thread and stream
// each.  Scores are float sums across sources, as in the reference.
#include <algorithm>
#include <atomic>
#include <cub/cub.cuh>
#include <string>
#include <thread>
#include <vector>

#include "nwg_internal.cuh"

using namespace nwg;

#define NWG_API extern "C" __attribute__((visibility("default")))

namespace {

constexpr int      kBcThreads = 256;
constexpr uint32_t kBcTask    = 2048;  // out-edges per warp task
constexpr uint32_t kUnset     = 0xFFFFFFFFu;

// Per-vertex state of one source, one 16-byte record so that a backward
// edge reads its target's level, dependency and path count in one sector.
struct alignas(16) BcVertex {
  uint32_t level;  // BFS level (kUnset = unreached)
  float    delta;  // dependency (score_t)
  double   sigma;  // shortest-path count (accum_t)
};

struct BcCounters {
  unsigned long long next;      // vertices appended to the next level
  unsigned int       tasks;     // out-edge tasks of the current level
  unsigned int       pad;
};

// tasks[i] = ceil(deg(order[i]) / kBcTask) for the level's vertices.
__global__ void k_bc_tasks(const uint64_t* __restrict__ off, const uint32_t* __restrict__ order, uint64_t count,
                           uint32_t* __restrict__ tasks) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    const uint32_t u = order[i];
    tasks[i]         = (uint32_t)((off[u + 1] - off[u] + kBcTask - 1) / kBcTask);
  }
}

// total = last exclusive prefix + last count (into *total); the claim pass
// also restarts the next-level counter.
__global__ void k_bc_total(const uint32_t* tpre, const uint32_t* tasks, uint64_t count, unsigned int* total,
                           unsigned long long* next) {
  *total = count ? tpre[count - 1] + tasks[count - 1] : 0u;
  if (next) *next = 0;
}

// Owner of task t: the last i with tpre[i] <= t.
__device__ __forceinline__ uint64_t task_owner(const uint32_t* tpre, uint64_t count, uint32_t t) {
  uint64_t lo = 0, hi = count;  // tpre[lo] <= t < tpre[hi] (tpre[count] = +inf)
  while (hi - lo > 1) {
    const uint64_t mid = (lo + hi) >> 1;
    if (tpre[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kBcThreads) k_bc_forward(const uint64_t* __restrict__ off,
                                                           const uint32_t* __restrict__ col, BcVertex* vx,
                                                           const uint32_t* __restrict__ order,
                                                           const uint32_t* __restrict__ tpre, uint64_t count,
                                                           uint32_t* next, uint64_t next_cap, uint32_t lvl,
                                                           BcCounters* cnt) {
  const unsigned lane   = threadIdx.x & 31;
  const uint64_t gwarp  = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t ntask  = cnt->tasks;
  for (uint64_t t = gwarp; t < ntask; t += nwarps) {
    const uint64_t i   = task_owner(tpre, count, (uint32_t)t);
    const uint32_t u   = order[i];
    const double   su  = vx[u].sigma;
    const uint64_t beg = off[u] + (uint64_t)((uint32_t)t - tpre[i]) * kBcTask;
    const uint64_t end = min(off[u + 1], beg + kBcTask);
    for (uint64_t e0 = beg; e0 < end; e0 += 32) {
      const uint64_t e   = e0 + lane;
      bool           won = false;
      uint32_t       v   = 0;
      if (e < end) {
        v           = col[e];
        uint32_t lv = vx[v].level;
        if (lv == kUnset) {
          lv  = atomicCAS(&vx[v].level, kUnset, lvl + 1);
          won = lv == kUnset;
          if (won) lv = lvl + 1;
        }
        if (lv == lvl + 1) atomicAdd(&vx[v].sigma, su);  // same 16-byte record as the level
      }
      const unsigned m = __ballot_sync(kFullMask, won);
      if (m) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&cnt->next, (unsigned long long)__popc(m));
        base = __shfl_sync(kFullMask, base, 0);
        if (won) {
          const uint64_t at = base + __popc(m & ((1u << lane) - 1u));
          if (at < next_cap) next[at] = v;
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kBcThreads, 4) k_bc_backward(const uint64_t* __restrict__ off,
                                                            const uint32_t* __restrict__ col,
                                                            const BcVertex* __restrict__ vx, double* dsum,
                                                            const uint32_t* __restrict__ order,
                                                            const uint32_t* __restrict__ tpre, uint64_t count,
                                                            uint32_t ntask, uint32_t lvl) {
  const unsigned lane   = threadIdx.x & 31;
  const uint64_t gwarp  = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t t = gwarp; t < ntask; t += nwarps) {
    const uint64_t i   = task_owner(tpre, count, (uint32_t)t);
    const uint32_t u   = order[i];
    const double   su  = vx[u].sigma;
    const uint64_t beg = off[u] + (uint64_t)((uint32_t)t - tpre[i]) * kBcTask;
    const uint64_t end = min(off[u + 1], beg + kBcTask);
    double         acc = 0.0;
    for (uint64_t e = beg + lane; e < end; e += 32) {
      const BcVertex r = vx[col[e]];  // level and weight in one 16-byte load
      if (r.level == lvl + 1) acc += su * r.sigma;  // r.sigma holds (1 + delta[v]) / path_counts[v] by now
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFullMask, acc, o);
    if (lane == 0 && acc != 0.0) atomicAdd(&dsum[u], acc);
  }
}

// delta[u] = the level's sums as float; bc[u] += delta[u].  The path count
// of u is not needed any more (u's own sum is done), so its slot takes the
// weight (1 + delta[u]) / path_counts[u] that the level above multiplies by:
// the reference's path_counts[w] / path_counts[u] * (1.0f + deltas[u])
// (:301) with the division done once per vertex instead of once per edge.
__global__ void k_bc_finish(const uint32_t* __restrict__ order, uint64_t count, double* dsum, BcVertex* vx,
                            float* bc) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    const uint32_t u = order[i];
    const float    d = (float)dsum[u];
    vx[u].delta      = d;
    vx[u].sigma      = (double)(1.0f + d) / vx[u].sigma;
    dsum[u]          = 0.0;
    atomicAdd(&bc[u], d);
  }
}

// Every vertex unreached, no path, no dependency; then the source.
__global__ void k_bc_reset(BcVertex* vx, uint64_t n, uint32_t* order, uint32_t s) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    vx[i] = (i == s) ? BcVertex{0u, 0.0f, 1.0} : BcVertex{kUnset, 0.0f, 0.0};
  if (blockIdx.x == 0 && threadIdx.x == 0) order[0] = s;
}

// Largest score (non-negative floats: their bit patterns order as integers).
__global__ void k_bc_max(const float* bc, uint64_t n, unsigned int* maxbits) {
  unsigned int   m      = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    m = max(m, __float_as_uint(fmaxf(bc[i], 0.0f)));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(kFullMask, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits, m);
}

__global__ void k_bc_divide(float* bc, uint64_t n, const unsigned int* maxbits) {
  const float    big    = __uint_as_float(*maxbits);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) bc[i] = bc[i] / big;
}

// Grid of a grid-stride kernel: no more blocks than fit on the GPU at once
// (the tasks are dealt out statically, so blocks of a second wave would
// start only when the first wave ends), and no more than the work needs.
template <class K>
int grid_bc(const GraphDev* g, K kernel, uint64_t items, uint64_t per_block) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBcThreads, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const uint64_t want = (items + per_block - 1) / per_block;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)g->sm_count * per_sm, want));
}

// One concurrent source lane: its stream and per-vertex state.
struct BcSlot {
  cudaStream_t s     = nullptr;
  BcVertex*    vx    = nullptr;
  double*      dsum  = nullptr;
  uint32_t*    order = nullptr;
  uint32_t*    tasks = nullptr;
  uint32_t*    tpre  = nullptr;
  BcCounters*  cnt   = nullptr;  // device
  BcCounters*  hcnt  = nullptr;  // pinned
  void*        tmp   = nullptr;  // cub scan scratch
  size_t       tmp_bytes = 0;
  uint32_t     max_levels = 0;
  int          rc = NWG_OK;
  std::string  err;
};

void slot_free(BcSlot& b) {
  if (b.s) cudaStreamSynchronize(b.s);
  cudaFree(b.vx);
  cudaFree(b.dsum);
  cudaFree(b.order);
  cudaFree(b.tasks);
  cudaFree(b.tpre);
  cudaFree(b.cnt);
  cudaFree(b.tmp);
  if (b.hcnt) cudaFreeHost(b.hcnt);
  if (b.s) cudaStreamDestroy(b.s);
}

int slot_init(const GraphDev* g, BcSlot& b) {
  const uint64_t n = std::max<uint64_t>(g->n, 1);
  if (cudaMalloc(&b.vx, n * sizeof(BcVertex)) != cudaSuccess || cudaMalloc(&b.dsum, n * 8) != cudaSuccess ||
      cudaMalloc(&b.order, n * 4) != cudaSuccess || cudaMalloc(&b.tasks, n * 4) != cudaSuccess ||
      cudaMalloc(&b.tpre, n * 4) != cudaSuccess || cudaMalloc(&b.cnt, sizeof(BcCounters)) != cudaSuccess ||
      cudaMallocHost(&b.hcnt, sizeof(BcCounters)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(NWG_ENOMEM, "betweenness workspace allocation failed");
  }
  if (cub::DeviceScan::ExclusiveSum(nullptr, b.tmp_bytes, b.tasks, b.tpre, (int64_t)n) != cudaSuccess ||
      cudaMalloc(&b.tmp, std::max<size_t>(b.tmp_bytes, 16)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(NWG_ENOMEM, "betweenness scan scratch allocation failed");
  }
  NWG_CUDA_TRY(cudaStreamCreateWithFlags(&b.s, cudaStreamNonBlocking));
  NWG_CUDA_TRY(cudaMemsetAsync(b.dsum, 0, n * 8, b.s));
  return NWG_OK;
}

// One source: forward levels (one read-back per level for the next level's
// size), then every backward level, then one synchronisation.
int run_source(const GraphDev* g, BcSlot& b, uint32_t s, float* bc) {
  const uint64_t n = g->n;
  cudaStream_t   st = b.s;
  k_bc_reset<<<grid_bc(g, k_bc_reset, n, kBcThreads), kBcThreads, 0, st>>>(b.vx, n, b.order, s);
  std::vector<uint64_t> lo = {0, 1};  // level L = order[lo[L], lo[L + 1])
  std::vector<uint32_t> ntask;         // tasks of each level (kept for the backward pass)
  for (uint32_t L = 0;; ++L) {
    const uint64_t count = lo[L + 1] - lo[L];
    const uint32_t* lv   = b.order + lo[L];
    k_bc_tasks<<<grid_bc(g, k_bc_tasks, count, kBcThreads), kBcThreads, 0, st>>>(g->off, lv, count, b.tasks + lo[L]);
    NWG_CUDA_TRY(cub::DeviceScan::ExclusiveSum(b.tmp, b.tmp_bytes, b.tasks + lo[L], b.tpre + lo[L], (int64_t)count, st));
    k_bc_total<<<1, 1, 0, st>>>(b.tpre + lo[L], b.tasks + lo[L], count, &b.cnt->tasks, &b.cnt->next);
    // claims: a task covers at most kBcTask edges, the grid is sized by the level's edges
    k_bc_forward<<<grid_bc(g, k_bc_forward, g->m / kBcTask + count, kBcThreads / 32), kBcThreads, 0, st>>>(
        g->off, g->col, b.vx, lv, b.tpre + lo[L], count, b.order + lo[L + 1], n - lo[L + 1], L, b.cnt);
    NWG_CUDA_TRY(cudaGetLastError());
    NWG_CUDA_TRY(cudaMemcpyAsync(b.hcnt, b.cnt, sizeof(BcCounters), cudaMemcpyDeviceToHost, st));
    NWG_CUDA_TRY(cudaStreamSynchronize(st));
    const uint64_t nxt = std::min<uint64_t>(b.hcnt->next, n - lo[L + 1]);
    ntask.push_back(b.hcnt->tasks);
    if (nxt == 0) break;
    lo.push_back(lo[L + 1] + nxt);
  }
  const uint32_t nlev = (uint32_t)(lo.size() - 1);
  b.max_levels        = std::max(b.max_levels, nlev);
  for (int64_t L = (int64_t)nlev - 1; L >= 0; --L) {
    const uint64_t count = lo[L + 1] - lo[L];
    const uint32_t nt    = ntask[L];  // the forward pass left the level's tpre in place
    if (nt)
      k_bc_backward<<<grid_bc(g, k_bc_backward, nt, kBcThreads / 32), kBcThreads, 0, st>>>(
          g->off, g->col, b.vx, b.dsum, b.order + lo[L], b.tpre + lo[L], count, nt, (uint32_t)L);
    k_bc_finish<<<grid_bc(g, k_bc_finish, count, kBcThreads), kBcThreads, 0, st>>>(b.order + lo[L], count, b.dsum, b.vx, bc);
    NWG_CUDA_TRY(cudaGetLastError());
  }
  NWG_CUDA_TRY(cudaStreamSynchronize(st));
  return NWG_OK;
}

}  // namespace

NWG_API int nwg_bc(nwg_graph h, const uint32_t* sources, uint32_t k, int normalize, uint32_t lanes, float* scores_host,
                   float* scores_dev, nwg_bc_stats* stats) {
  try {
    if (!h || (!sources && k)) return set_error(NWG_EINVAL, "NULL graph or sources");
    if (!scores_host && !scores_dev) return set_error(NWG_EINVAL, "no output array");
    auto* g = reinterpret_cast<GraphDev*>(h);
    for (uint32_t i = 0; i < k; ++i)
      if (sources[i] >= g->n) return set_error(NWG_EINVAL, "source " + std::to_string(sources[i]) + " >= n");
    if (lanes == 0) lanes = 4;
    lanes = std::min<uint32_t>(std::min<uint32_t>(lanes, 16), std::max<uint32_t>(k, 1));
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    struct Restore {
      int d;
      ~Restore() { cudaSetDevice(d); }
    } restore{prev};
    const uint64_t n  = g->n;
    float*         bc = scores_dev;
    float*         own = nullptr;
    unsigned int*  maxbits = nullptr;
    if (!bc) {
      if (cudaMalloc(&own, std::max<uint64_t>(n, 1) * 4) != cudaSuccess) {
        cudaGetLastError();
        return set_error(NWG_ENOMEM, "betweenness score allocation failed");
      }
      bc = own;
    }
    struct FreeOwn {
      float**        p;
      unsigned int** m;
      ~FreeOwn() {
        cudaFree(*p);
        cudaFree(*m);
      }
    } free_own{&own, &maxbits};
    NWG_CUDA_TRY(cudaMalloc(&maxbits, sizeof(unsigned int)));
    cudaEvent_t ev0, ev1;
    NWG_CUDA_TRY(cudaEventCreate(&ev0));
    NWG_CUDA_TRY(cudaEventCreate(&ev1));
    NWG_CUDA_TRY(cudaMemset(bc, 0, n * 4));
    NWG_CUDA_TRY(cudaMemset(maxbits, 0, sizeof(unsigned int)));
    std::vector<BcSlot> slots(lanes);
    int                 rc = NWG_OK;
    for (auto& b : slots)
      if (!rc) rc = slot_init(g, b);
    NWG_CUDA_TRY(cudaDeviceSynchronize());
    NWG_CUDA_TRY(cudaEventRecord(ev0, 0));
    if (!rc) {
      std::atomic<uint32_t> next{0};
      auto                  lane_loop = [&, dev = g->device](BcSlot* bp) {
        cudaSetDevice(dev);
        for (uint32_t i = next++; i < k && bp->rc == NWG_OK; i = next++) {
          bp->rc = run_source(g, *bp, sources[i], bc);
          if (bp->rc) {
            char buf[512];
            nwg_last_error(buf, sizeof buf);
            bp->err = buf;
          }
        }
      };
      if (slots.size() == 1) {
        lane_loop(&slots[0]);  // one lane: the calling thread (profiler ranges stay on it)
      } else {
        std::vector<std::thread> th;
        for (auto& b : slots) th.emplace_back(lane_loop, &b);
        for (auto& t : th) t.join();
      }
      for (auto& b : slots)
        if (b.rc && !rc) {
          rc = b.rc;
          set_error(b.rc, b.err);
        }
    }
    if (!rc && normalize) {
      k_bc_max<<<grid_bc(g, k_bc_max, n, 256), 256>>>(bc, n, maxbits);
      k_bc_divide<<<grid_bc(g, k_bc_divide, n, 256), 256>>>(bc, n, maxbits);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) rc = cuda_error(e, "betweenness normalisation");
    }
    cudaEventRecord(ev1, 0);
    cudaError_t e = cudaDeviceSynchronize();
    if (!rc && e != cudaSuccess) rc = cuda_error(e, "betweenness");
    if (!rc && scores_host) {
      e = cudaMemcpy(scores_host, bc, n * 4, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) rc = cuda_error(e, "betweenness read-back");
    }
    if (stats) {
      nwg_bc_stats st = {};
      st.sources      = k;
      st.lanes        = lanes;
      for (auto& b : slots) st.max_levels = std::max(st.max_levels, b.max_levels);
      cudaEventElapsedTime(&st.device_ms, ev0, ev1);
      *stats = st;
    }
    for (auto& b : slots) slot_free(b);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    return rc;
  } catch (const std::exception& ex) {
    return set_error(NWG_ENOMEM, std::string("betweenness failed: ") + ex.what());
  }
}
