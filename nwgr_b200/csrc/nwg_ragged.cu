// C ABI of the ragged batch: many small CSR graphs packed into HBM once, and
// a table of (graph, root) traversals run in one persistent launch replayed
// as a CUDA graph (k_ragged in nwg_dobfs.cu).  No reference counterpart:
// NWGraph runs one bfs call per (graph, root); the results are the same.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "nwg_internal.cuh"

using namespace nwg;

#define NWG_API extern "C" __attribute__((visibility("default")))

namespace {

void ragged_free(RaggedDev* r) {
  if (!r) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(r->device);
  if (r->stream) cudaStreamSynchronize(r->stream);
  if (r->exec) cudaGraphExecDestroy(r->exec);
  cudaFree(r->off);
  cudaFree(r->col);
  cudaFree(r->Z);
  cudaFree(r->graphs);
  cudaFree(r->items);
  cudaFree(r->results);
  cudaFree(r->counter);
  cudaFree(r->scratch);
  if (r->ev0) cudaEventDestroy(r->ev0);
  if (r->ev1) cudaEventDestroy(r->ev1);
  if (r->stream) cudaStreamDestroy(r->stream);
  cudaSetDevice(prev);
  delete r;
}

int ragged_register(uint32_t num_graphs, const uint64_t* graph_n, const uint64_t* off_concat, const uint32_t* col_concat,
                    nwg_ragged* out) {
  if (!out) return set_error(NWG_EINVAL, "out handle pointer is NULL");
  *out = nullptr;
  if (num_graphs == 0 || !graph_n || !off_concat) return set_error(NWG_EINVAL, "empty or NULL ragged graph set");
  auto* r = new (std::nothrow) RaggedDev();
  if (!r) return set_error(NWG_ENOMEM, "host allocation failed");
  auto fail = [&](int rc) {
    ragged_free(r);
    return rc;
  };
  cudaGetDevice(&r->device);
  NWG_CUDA_TRY(cudaDeviceGetAttribute(&r->sm_count, cudaDevAttrMultiProcessorCount, r->device));
  r->ngraphs = num_graphs;
  r->graphs_host.resize(num_graphs);
  uint64_t off_total = 0, col_total = 0, col_packed = 0, z_total = 0;
  for (uint32_t g = 0; g < num_graphs; ++g) {
    const uint64_t n = graph_n[g];
    if (n == 0 || n >= 0xFFFFFFFFull) return fail(set_error(NWG_EINVAL, "graph " + std::to_string(g) + ": bad n"));
    const uint64_t* off = off_concat + off_total;
    if (off[0] != 0) return fail(set_error(NWG_EINVAL, "graph " + std::to_string(g) + ": offsets must start at 0"));
    for (uint64_t i = 0; i < n; ++i)
      if (off[i + 1] < off[i]) return fail(set_error(NWG_EINVAL, "graph " + std::to_string(g) + ": offsets not monotone"));
    const uint64_t m = off[n];
    for (uint64_t e = 0; e < m; ++e)
      if (col_concat[col_total + e] >= n)
        return fail(set_error(NWG_EINVAL, "graph " + std::to_string(g) + ": column id out of range"));
    RaggedGraph& gr = r->graphs_host[g];
    gr.n            = n;
    gr.m            = m;
    gr.off_base     = off_total;
    gr.col_base     = col_packed;
    gr.z_base       = z_total;
    off_total += n + 1;
    col_total += m;
    col_packed += (m + 3) & ~3ull;  // next graph's columns start 16-byte aligned
    z_total += (n + 31) / 32;
    r->nmax    = std::max(r->nmax, n);
    r->mmax    = std::max(r->mmax, m);
    r->total_n += n;
  }
  std::vector<uint32_t> cols(std::max<uint64_t>(col_packed, 4), 0u);
  uint64_t              srcpos = 0;
  for (uint32_t g = 0; g < num_graphs; ++g) {
    const RaggedGraph& gr = r->graphs_host[g];
    std::memcpy(cols.data() + gr.col_base, col_concat + srcpos, gr.m * 4);
    srcpos += gr.m;
  }
  if (cudaMalloc(&r->off, off_total * 8) != cudaSuccess || cudaMalloc(&r->col, cols.size() * 4) != cudaSuccess ||
      cudaMalloc(&r->Z, std::max<uint64_t>(z_total, 1) * 4) != cudaSuccess ||
      cudaMalloc(&r->graphs, num_graphs * sizeof(RaggedGraph)) != cudaSuccess ||
      cudaMalloc(&r->counter, sizeof(unsigned int)) != cudaSuccess) {
    cudaGetLastError();
    return fail(set_error(NWG_ENOMEM, "ragged graph allocation failed"));
  }
  if (cudaMemcpy(r->off, off_concat, off_total * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(r->col, cols.data(), cols.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(r->graphs, r->graphs_host.data(), num_graphs * sizeof(RaggedGraph), cudaMemcpyHostToDevice) !=
          cudaSuccess)
    return fail(cuda_error(cudaGetLastError(), "ragged upload"));
  int rc = zero_indegree_packed(r);
  if (rc) return fail(rc);
  if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&r->ev0) != cudaSuccess || cudaEventCreate(&r->ev1) != cudaSuccess)
    return fail(cuda_error(cudaGetLastError(), "ragged stream"));
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(cuda_error(cudaGetLastError(), "ragged registration"));
  *out = reinterpret_cast<nwg_ragged>(r);
  return NWG_OK;
}

int ragged_bfs(RaggedDev* r, uint32_t num_items, const nwg_ragged_item* items, uint32_t* parents_dev,
               uint64_t* item_offsets_host, nwg_ragged_result* results_host, uint32_t blocks_per_sm, float* device_ms) {
  if (num_items == 0) return NWG_OK;
  if (!items || !parents_dev) return set_error(NWG_EINVAL, "NULL items or parents");
  if (blocks_per_sm == 0) blocks_per_sm = 2;
  if (blocks_per_sm > 8) return set_error(NWG_EINVAL, "blocks_per_sm must be 1..8");
  std::vector<RaggedItem> table(num_items);
  uint64_t                base = 0;
  for (uint32_t i = 0; i < num_items; ++i) {
    const nwg_ragged_item& it = items[i];
    if (it.graph >= r->ngraphs) return set_error(NWG_EINVAL, "item " + std::to_string(i) + ": graph index out of range");
    const RaggedGraph& gr = r->graphs_host[it.graph];
    if (it.root >= gr.n) return set_error(NWG_EINVAL, "item " + std::to_string(i) + ": root >= n");
    if (it.alpha <= 0 || it.beta <= 0) return set_error(NWG_EINVAL, "item " + std::to_string(i) + ": alpha, beta must be positive");
    const uint32_t wm = it.warp_min ? it.warp_min : 32;
    if (wm < 32 || wm > 256) return set_error(NWG_EINVAL, "item " + std::to_string(i) + ": warp_min must be 32..256");
    table[i] = RaggedItem{it.graph, it.root, base, it.alpha, it.beta, wm, 0};
    if (item_offsets_host) item_offsets_host[i] = base;
    base += gr.n;
  }
  uint64_t slot_bytes = 0;
  ragged_slot_bytes(r->nmax, r->mmax, &slot_bytes);
  const uint64_t slots = (uint64_t)std::max(1, r->sm_count * (int)blocks_per_sm);
  if (num_items > r->items_cap) {
    cudaFree(r->items);
    cudaFree(r->results);
    r->items   = nullptr;
    r->results = nullptr;
    if (cudaMalloc(&r->items, num_items * sizeof(RaggedItem)) != cudaSuccess ||
        cudaMalloc(&r->results, num_items * sizeof(RaggedResult)) != cudaSuccess) {
      cudaGetLastError();
      r->items_cap = 0;
      return set_error(NWG_ENOMEM, "ragged item table allocation failed");
    }
    r->items_cap = num_items;
    if (r->exec) {
      cudaGraphExecDestroy(r->exec);
      r->exec = nullptr;
    }
  }
  if (slots * slot_bytes > r->scratch_bytes) {
    cudaFree(r->scratch);
    r->scratch = nullptr;
    if (cudaMalloc(&r->scratch, slots * slot_bytes) != cudaSuccess) {
      cudaGetLastError();
      r->scratch_bytes = 0;
      return set_error(NWG_ENOMEM, "ragged scratch (" + std::to_string(slots * slot_bytes) + " bytes) allocation failed");
    }
    r->scratch_bytes = slots * slot_bytes;
    if (r->exec) {
      cudaGraphExecDestroy(r->exec);
      r->exec = nullptr;
    }
  }
  NWG_CUDA_TRY(cudaMemcpyAsync(r->items, table.data(), num_items * sizeof(RaggedItem), cudaMemcpyHostToDevice, r->stream));
  float ms = 0.f;
  int   rc = ragged_launch(r, num_items, parents_dev, blocks_per_sm, &ms);
  if (rc) return rc;
  if (device_ms) *device_ms = ms;
  std::vector<RaggedResult> res(num_items);
  NWG_CUDA_TRY(cudaMemcpy(res.data(), r->results, num_items * sizeof(RaggedResult), cudaMemcpyDeviceToHost));
  int32_t first_bad = 0;
  for (uint32_t i = 0; i < num_items; ++i) {
    if (results_host) {
      nwg_ragged_result& o = results_host[i];
      o.status             = res[i].status;
      o.steps              = res[i].steps;
      o.levels             = res[i].levels;
      o.td_steps           = res[i].td_steps;
      o.bu_steps           = res[i].bu_steps;
      o.b2q_steps          = res[i].b2q_steps;
      o.reached            = res[i].reached;
    }
    if (res[i].status && !first_bad) first_bad = res[i].status;
  }
  if (first_bad) return set_error(first_bad, "a ragged item reported status " + std::to_string(first_bad));
  return NWG_OK;
}

}  // namespace

NWG_API int nwg_ragged_register(uint32_t num_graphs, const uint64_t* graph_n, const uint64_t* off_concat,
                                const uint32_t* col_concat, nwg_ragged* out) {
  try {
    return ragged_register(num_graphs, graph_n, off_concat, col_concat, out);
  } catch (const std::bad_alloc&) {
    return set_error(NWG_ENOMEM, "host allocation failed");
  } catch (...) {
    return set_error(NWG_ESTATE, "unexpected C++ exception");
  }
}

NWG_API int nwg_ragged_release(nwg_ragged h) {
  if (!h) return set_error(NWG_EINVAL, "NULL ragged handle");
  ragged_free(reinterpret_cast<RaggedDev*>(h));
  return NWG_OK;
}

NWG_API int nwg_ragged_info(nwg_ragged h, uint32_t* num_graphs, uint64_t* total_n, uint64_t* nmax, uint64_t* mmax) {
  if (!h) return set_error(NWG_EINVAL, "NULL ragged handle");
  auto* r = reinterpret_cast<RaggedDev*>(h);
  if (num_graphs) *num_graphs = r->ngraphs;
  if (total_n) *total_n = r->total_n;
  if (nmax) *nmax = r->nmax;
  if (mmax) *mmax = r->mmax;
  return NWG_OK;
}

NWG_API int nwg_ragged_bfs(nwg_ragged h, uint32_t num_items, const nwg_ragged_item* items, uint32_t* parents_dev,
                           uint64_t* item_offsets_host, nwg_ragged_result* results_host, uint32_t blocks_per_sm,
                           float* device_ms) {
  try {
    if (!h) return set_error(NWG_EINVAL, "NULL ragged handle");
    auto*                       r = reinterpret_cast<RaggedDev*>(h);
    std::lock_guard<std::mutex> lk(r->mu);
    int                         prev = 0;
    cudaGetDevice(&prev);
    if (prev != r->device) cudaSetDevice(r->device);
    const int rc = ragged_bfs(r, num_items, items, parents_dev, item_offsets_host, results_host, blocks_per_sm, device_ms);
    if (prev != r->device) cudaSetDevice(prev);
    return rc;
  } catch (const std::bad_alloc&) {
    return set_error(NWG_ENOMEM, "host allocation failed");
  } catch (...) {
    return set_error(NWG_ESTATE, "unexpected C++ exception");
  }
}
