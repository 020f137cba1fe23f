// Seeded synthetic graphs built directly in HBM: RMAT/Kronecker, uniform
// random and 2D grid with random shortcuts.  NWGraph ships no such
// generator; the clean-up pipeline follows its edge-list path (symmetrize as
// io/mmio.hpp:96-100 does for symmetric files, remove_self_loops
// build.hpp:427-444, lexical sort + uniq build.hpp:58-70,344-355, CSR fill
// with sorted rows build.hpp:210-266), done here as one radix sort of packed
// (source << 32 | target) keys, a unique pass and an offsets scatter.
//
// Randomness is counter-based so each edge is independent of the others:
//   splitmix64(x)             Steele, Lea and Flood's SplitMix64 finaliser
//   draw(seed, stream, idx) = splitmix64(splitmix64(seed) ^ (stream << 56) ^ idx)
//   lemire(h, n)            = ((h >> 32) * n) >> 32
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "nwg_internal.cuh"

namespace nwg {
namespace {

constexpr int      kThreads      = 256;
constexpr uint64_t kStreamRmat   = 1;
constexpr uint64_t kStreamPerm   = 2;
constexpr uint64_t kStreamUnif   = 3;
constexpr uint64_t kStreamGrid   = 4;
constexpr uint64_t kStreamRoots  = 5;
constexpr uint64_t kSentinel     = ~0ull;

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t stream_key(uint64_t seed, uint64_t stream) {
  return splitmix64(seed) ^ (stream << 56);
}

__host__ __device__ __forceinline__ uint64_t lemire(uint64_t h, uint64_t n) { return ((h >> 32) * n) >> 32; }

struct Perm {
  uint64_t k[3], c[3];
  uint64_t mask;
  uint32_t shift;
};

Perm make_perm(uint32_t scale, uint64_t seed) {
  Perm           p;
  const uint64_t key = stream_key(seed, kStreamPerm);
  for (int r = 0; r < 3; ++r) {
    p.k[r] = splitmix64(key ^ (uint64_t)(2 * r)) | 1ull;
    p.c[r] = splitmix64(key ^ (uint64_t)(2 * r + 1));
  }
  p.mask  = (scale >= 64) ? ~0ull : ((1ull << scale) - 1);
  p.shift = (scale + 1) >> 1;
  return p;
}

__device__ __forceinline__ uint64_t permute(uint64_t x, const Perm& p) {
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    x = (x * p.k[r] + p.c[r]) & p.mask;
    x ^= x >> p.shift;
  }
  return x;
}

__device__ __forceinline__ void emit_pair(uint64_t* keys, uint64_t e, uint64_t u, uint64_t v) {
  if (u == v) {
    keys[2 * e]     = kSentinel;
    keys[2 * e + 1] = kSentinel;
  } else {
    keys[2 * e]     = (u << 32) | v;
    keys[2 * e + 1] = (v << 32) | u;
  }
}

__global__ void k_rmat(uint64_t* keys, uint64_t n_edges, uint32_t scale, uint64_t key, uint32_t ta, uint32_t tab,
                       uint32_t tabc, Perm perm) {
  const uint32_t words = (scale + 1) >> 1;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_edges;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t u = 0, v = 0, w = 0;
    for (uint32_t lvl = 0; lvl < scale; ++lvl) {
      if ((lvl & 1) == 0) w = splitmix64((e * words + (lvl >> 1)) ^ key);
      const uint32_t t  = (lvl & 1) ? (uint32_t)(w >> 32) : (uint32_t)w;
      const uint64_t ub = t >= tab;
      const uint64_t vb = (t >= ta && t < tab) || t >= tabc;
      u                 = (u << 1) | ub;
      v                 = (v << 1) | vb;
    }
    emit_pair(keys, e, permute(u, perm), permute(v, perm));
  }
}

__global__ void k_uniform(uint64_t* keys, uint64_t pairs, uint64_t n, uint64_t key) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < pairs;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t u = lemire(splitmix64((2 * e) ^ key), n);
    const uint64_t v = lemire(splitmix64((2 * e + 1) ^ key), n);
    emit_pair(keys, e, u, v);
  }
}

__global__ void k_grid(uint64_t* keys, uint32_t W, uint32_t H, uint64_t shortcuts, uint64_t key) {
  const uint64_t right = (uint64_t)(W - 1) * H;
  const uint64_t down  = (uint64_t)W * (H - 1);
  const uint64_t total = right + down + shortcuts;
  const uint64_t n     = (uint64_t)W * H;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t u, v;
    if (e < right) {
      const uint64_t y = e / (W - 1), x = e % (W - 1);
      u = y * W + x;
      v = u + 1;
    } else if (e < right + down) {
      const uint64_t i = e - right;
      u                = i;  // (y, x) = (i / W, i % W)
      v                = i + W;
    } else {
      const uint64_t i = e - right - down;
      u                = lemire(splitmix64((2 * i) ^ key), n);
      v                = lemire(splitmix64((2 * i + 1) ^ key), n);
    }
    emit_pair(keys, e, u, v);
  }
}

// keys sorted and unique: col[i] = low half; offsets by scattering each row
// start (rows without entries take the next row's start).
__global__ void k_csr(const uint64_t* __restrict__ keys, uint64_t m, uint64_t n, uint64_t* __restrict__ off,
                      uint32_t* __restrict__ col) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t s  = (i < m) ? (keys[i] >> 32) : n;
    const uint64_t sp = (i == 0) ? 0 : (keys[i - 1] >> 32) + 1;
    for (uint64_t t = sp; t <= s && t <= n; ++t) off[t] = i;
    if (i < m) col[i] = (uint32_t)keys[i];
  }
}

__global__ void k_gather_deg(const uint64_t* __restrict__ off, const uint32_t* __restrict__ ids, uint32_t count,
                             uint64_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) out[i] = off[ids[i] + 1] - off[ids[i]];
}

// keys[0, 2*count) -> sorted unique CSR in g (allocates g->off, g->col).
int build_csr(uint64_t* keys, uint64_t nkeys, uint64_t n, GraphDev* g) {
  uint64_t* alt = nullptr;
  NWG_CUDA_TRY(cudaMalloc(&alt, std::max<uint64_t>(nkeys, 1) * sizeof(uint64_t)));
  cub::DoubleBuffer<uint64_t> db(keys, alt);
  size_t                      tmp_bytes = 0;
  // sort on the bits in use: target bits [0, b) and source bits [32, 32 + b);
  // the sentinel (all ones) sorts last.
  const int end_bit = 64;
  if (cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, (int64_t)nkeys, 0, end_bit) != cudaSuccess) {
    cudaFree(alt);
    return cuda_error(cudaGetLastError(), "cub SortKeys (size query)");
  }
  size_t    uniq_bytes = 0;
  uint64_t* nsel       = nullptr;
  cub::DeviceSelect::Unique(nullptr, uniq_bytes, keys, alt, nsel, (int64_t)nkeys);
  void* tmp = nullptr;
  if (cudaMalloc(&tmp, std::max(tmp_bytes, uniq_bytes) + 16) != cudaSuccess ||
      cudaMalloc(&nsel, sizeof(uint64_t)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(alt);
    cudaFree(tmp);
    return set_error(NWG_ENOMEM, "generator sort buffers");
  }
  cudaError_t e = cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, (int64_t)nkeys, 0, end_bit);
  uint64_t*   sorted = db.Current();
  uint64_t*   other  = db.Alternate();
  if (e == cudaSuccess) e = cub::DeviceSelect::Unique(tmp, uniq_bytes, sorted, other, nsel, (int64_t)nkeys);
  uint64_t m_all = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&m_all, nsel, sizeof(uint64_t), cudaMemcpyDeviceToHost);
  uint64_t last = 0;
  if (e == cudaSuccess && m_all) e = cudaMemcpy(&last, other + m_all - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost);
  cudaFree(tmp);
  cudaFree(nsel);
  if (e != cudaSuccess) {
    cudaFree(alt);
    return cuda_error(e, "generator sort/unique");
  }
  const uint64_t m = (m_all && last == kSentinel) ? m_all - 1 : m_all;
  g->n             = n;
  g->m             = m;
  if (cudaMalloc(&g->off, (n + 1) * sizeof(uint64_t)) != cudaSuccess ||
      cudaMalloc(&g->col, std::max<uint64_t>(m, 4) * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(alt);
    return set_error(NWG_ENOMEM, "generator CSR allocation");
  }
  k_csr<<<std::max(1, g->sm_count * 8), kThreads>>>(other, m, n, g->off, g->col);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(alt);
  if (e != cudaSuccess) return cuda_error(e, "generator CSR fill");
  return NWG_OK;
}

int alloc_keys(uint64_t** keys, uint64_t count) {
  if (cudaMalloc(keys, std::max<uint64_t>(count, 1) * sizeof(uint64_t)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(NWG_ENOMEM, "generator key buffer (" + std::to_string(count * 8) + " bytes)");
  }
  return NWG_OK;
}

void set_sm_count(GraphDev* g) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, g->device) == cudaSuccess) g->sm_count = prop.multiProcessorCount;
}

}  // namespace

int gen_rmat(uint32_t scale, uint32_t ef, uint64_t seed, uint32_t ta, uint32_t tab, uint32_t tabc, GraphDev* g) {
  set_sm_count(g);
  const uint64_t n       = 1ull << scale;
  const uint64_t n_edges = (uint64_t)ef << scale;
  uint64_t*      keys    = nullptr;
  int            rc      = alloc_keys(&keys, 2 * n_edges);
  if (rc) return rc;
  k_rmat<<<g->sm_count * 8, kThreads>>>(keys, n_edges, scale, stream_key(seed, kStreamRmat), ta, tab, tabc,
                                         make_perm(scale, seed));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaFree(keys);
    return cuda_error(e, "k_rmat");
  }
  rc = build_csr(keys, 2 * n_edges, n, g);
  cudaFree(keys);
  return rc;
}

int gen_uniform(uint64_t n, uint32_t deg, uint64_t seed, GraphDev* g) {
  set_sm_count(g);
  const uint64_t pairs = (n * deg) / 2;
  uint64_t*      keys  = nullptr;
  int            rc    = alloc_keys(&keys, 2 * pairs);
  if (rc) return rc;
  k_uniform<<<g->sm_count * 8, kThreads>>>(keys, pairs, n, stream_key(seed, kStreamUnif));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaFree(keys);
    return cuda_error(e, "k_uniform");
  }
  rc = build_csr(keys, 2 * pairs, n, g);
  cudaFree(keys);
  return rc;
}

int gen_grid(uint32_t w, uint32_t h, uint32_t pct, uint64_t seed, GraphDev* g) {
  set_sm_count(g);
  const uint64_t grid_edges = (uint64_t)(w - 1) * h + (uint64_t)w * (h - 1);
  const uint64_t shortcuts  = grid_edges * pct / 100;
  const uint64_t total      = grid_edges + shortcuts;
  uint64_t*      keys       = nullptr;
  int            rc         = alloc_keys(&keys, 2 * total);
  if (rc) return rc;
  k_grid<<<g->sm_count * 8, kThreads>>>(keys, w, h, shortcuts, stream_key(seed, kStreamGrid));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaFree(keys);
    return cuda_error(e, "k_grid");
  }
  rc = build_csr(keys, 2 * total, (uint64_t)w * h, g);
  cudaFree(keys);
  return rc;
}

int pick_roots(GraphDev* g, uint64_t seed, uint32_t count, uint32_t* roots_host) {
  if (count == 0) return NWG_OK;
  if (g->m == 0) return set_error(NWG_EINVAL, "graph has no vertex with out-degree > 0");
  const uint64_t key   = stream_key(seed, kStreamRoots);
  const uint32_t batch = 1024;
  uint32_t*      d_ids = nullptr;
  uint64_t*      d_deg = nullptr;
  if (cudaMalloc(&d_ids, batch * 4) != cudaSuccess || cudaMalloc(&d_deg, batch * 8) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(d_ids);
    return set_error(NWG_ENOMEM, "pick_roots buffers");
  }
  std::vector<uint32_t> ids(batch);
  std::vector<uint64_t> deg(batch);
  uint32_t              got = 0;
  int                   rc  = NWG_OK;
  for (uint64_t k = 0; got < count; k += batch) {
    if (k > (1ull << 40)) {
      rc = set_error(NWG_ETIMEDOUT, "pick_roots: no vertex with out-degree > 0 found");
      break;
    }
    for (uint32_t i = 0; i < batch; ++i) ids[i] = (uint32_t)lemire(splitmix64((k + i) ^ key), g->n);
    cudaError_t e = cudaMemcpy(d_ids, ids.data(), batch * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      k_gather_deg<<<(batch + 255) / 256, 256>>>(g->off, d_ids, batch, d_deg);
      e = cudaMemcpy(deg.data(), d_deg, batch * 8, cudaMemcpyDeviceToHost);
    }
    if (e != cudaSuccess) {
      rc = cuda_error(e, "pick_roots");
      break;
    }
    for (uint32_t i = 0; i < batch && got < count; ++i)
      if (deg[i] > 0) roots_host[got++] = ids[i];
  }
  cudaFree(d_ids);
  cudaFree(d_deg);
  return rc;
}

}  // namespace nwg
