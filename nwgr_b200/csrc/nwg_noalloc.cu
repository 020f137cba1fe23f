// nwg_bfs_noalloc: the direction-optimizing BFS for callers that cannot
// allocate device memory.
//
// Who needs it: cudaMalloc and cudaFree synchronise the whole device and may
// block behind other streams, so latency-bound services often forbid them
// after start-up; processes that hand all device memory to their own pool
// allocator, or that run inside a framework owning the device memory, may
// not call them at all.  nwg_bfs needs a registered graph and a workspace,
// both of which allocate.  This entry point allocates nothing: the caller
// passes the CSR arrays and the parents array in its own device memory, and
// every piece of scratch state (control block, visited and discovery
// bitmaps, the in-degree-zero bitmap, both frontier queues) lives in one
// file-scope static __device__ array of fixed size, which every GPU that
// loads the library holds until the process exits.
//
// Limits: n <= 2^20 vertices and m <= 2^24 CSR entries (about 18 MB of
// static device memory); larger graphs are rejected with NWG_EINVAL before
// anything is launched.  Every call shares the one array, so calls whose
// GPU work overlaps (two host threads, or two streams) race and corrupt each
// other; serialise them.  The first call on a device looks the array's
// device address up (cudaGetSymbolAddress) and keeps it for the life of the
// process, so the entry point must not be used on a device across
// cudaDeviceReset (which unloads the module holding the array).  The level
// loop is driven from the host (one small device-to-host read per step,
// which synchronises the caller's stream), so a call must not be made while
// that stream is being captured into a CUDA graph, and it is slower than the
// CUDA-graph path of nwg_bfs.
#include <algorithm>
#include <mutex>

#include "nwg_internal.cuh"

namespace nwg {
namespace {

constexpr uint64_t kNaMaxN  = 1ull << 20;
constexpr uint64_t kNaMaxM  = 1ull << 24;
constexpr uint64_t kNaWords = kNaMaxN / 32;
constexpr uint64_t kNaQsCap = kNaMaxN;
constexpr uint64_t kNaQcCap = kNaMaxM / 256 + (kNaMaxN < kNaMaxM / 32 ? kNaMaxN : kNaMaxM / 32) + 1;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kNaOffCtrl = 0;
constexpr size_t kNaOffV    = align256(kNaOffCtrl + sizeof(Ctrl));
constexpr size_t kNaOffZ    = align256(kNaOffV + 3 * kNaWords * sizeof(uint32_t));
constexpr size_t kNaOffQs   = align256(kNaOffZ + kNaWords * sizeof(uint32_t));
constexpr size_t kNaOffQc   = align256(kNaOffQs + 2 * kNaQsCap * sizeof(uint32_t));
constexpr size_t kNaBytes   = align256(kNaOffQc + 2 * kNaQcCap * sizeof(uint64_t));

// The scratch.  In host code this name is only a stand-in for the symbol: its
// device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

constexpr int kMaxDevices = 64;
std::mutex    g_setup_mu;
void*         g_scratch_ptr[kMaxDevices] = {};

int scratch_for_device(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return set_error(NWG_EINVAL, "device index out of range");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void*             ptr = nullptr;
    const cudaError_t e   = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_scratch_ptr[dev] = ptr;
  }
  *out = static_cast<unsigned char*>(g_scratch_ptr[dev]);
  return NWG_OK;
}

}  // namespace
}  // namespace nwg

using namespace nwg;

extern "C" __attribute__((visibility("default"))) int nwg_bfs_noalloc(const uint64_t* out_off, const uint32_t* out_col,
                                                                      const uint64_t* in_off, const uint32_t* in_col,
                                                                      uint64_t n, uint32_t root, int alpha, int beta,
                                                                      uint32_t* parents_dev, void* stream_ptr) {
  try {
    if (!out_off || !out_col || !parents_dev) return set_error(NWG_EINVAL, "NULL array");
    if ((in_off == nullptr) != (in_col == nullptr)) return set_error(NWG_EINVAL, "in_off and in_col must both be set or both be NULL");
    if (n == 0 || n > kNaMaxN)
      return set_error(NWG_EINVAL, "nwg_bfs_noalloc: n = " + std::to_string(n) + " is outside [1, " +
                                       std::to_string(kNaMaxN) + "] (the static scratch limit)");
    if (root >= n) return set_error(NWG_EINVAL, "root " + std::to_string(root) + " >= n " + std::to_string(n));
    if (alpha <= 0 || beta <= 0) return set_error(NWG_EINVAL, "alpha and beta must be positive");
    if (reinterpret_cast<uintptr_t>(out_col) & 15)
      return set_error(NWG_EINVAL, "nwg_bfs_noalloc: out_col must be 16-byte aligned (128-bit neighbour loads)");
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_ptr);
    int          dev    = 0;
    NWG_CUDA_TRY(cudaGetDevice(&dev));
    unsigned char* base = nullptr;
    int            rc   = scratch_for_device(dev, &base);
    if (rc) return rc;

    uint64_t m = 0, in_m = 0;
    NWG_CUDA_TRY(cudaMemcpyAsync(&m, out_off + n, sizeof(m), cudaMemcpyDeviceToHost, stream));
    if (in_off) NWG_CUDA_TRY(cudaMemcpyAsync(&in_m, in_off + n, sizeof(in_m), cudaMemcpyDeviceToHost, stream));
    NWG_CUDA_TRY(cudaStreamSynchronize(stream));
    if (m > kNaMaxM)
      return set_error(NWG_EINVAL, "nwg_bfs_noalloc: m = " + std::to_string(m) + " exceeds " + std::to_string(kNaMaxM) +
                                       " (the static scratch limit)");
    if (in_off && in_m != m)
      return set_error(NWG_EINVAL, "in-graph entry count differs from out-graph (not a transpose)");

    int sm = 148;
    NWG_CUDA_TRY(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev));

    DobfsParams P   = {};
    P.off           = out_off;
    P.col           = out_col;
    P.in_off        = in_off ? in_off : out_off;
    P.in_col        = in_col ? in_col : out_col;
    P.n             = n;
    P.m             = m;
    P.nwords        = (uint32_t)((n + 31) / 32);
    uint32_t* bits  = reinterpret_cast<uint32_t*>(base + kNaOffV);
    P.V             = bits;
    P.C0            = bits + kNaWords;
    P.C1            = bits + 2 * kNaWords;
    P.Z             = reinterpret_cast<uint32_t*>(base + kNaOffZ);
    uint32_t* qs    = reinterpret_cast<uint32_t*>(base + kNaOffQs);
    uint64_t* qc    = reinterpret_cast<uint64_t*>(base + kNaOffQc);
    P.qs[0]         = qs;
    P.qs[1]         = qs + kNaQsCap;
    P.qc[0]         = qc;
    P.qc[1]         = qc + kNaQcCap;
    P.qs_cap        = kNaQsCap;
    P.qc_cap        = kNaQcCap;
    // Chunked vertices from out-degree 32 on (registered graphs use 64):
    // kNaQcCap bounds the chunk entries for that threshold, m / 256 + min(n, m / 32) + 1.
    P.th            = Thresholds{32, 256, 8};
    P.symmetric     = in_off ? 0u : 1u;
    P.nzero         = 0;  // not counted here (it would need a reduction and a read-back)
    P.ctrl          = reinterpret_cast<Ctrl*>(base + kNaOffCtrl);

    // Everything the traversal reads before writing is (re)initialised here
    // or by the init kernel: Z below, V and the control block by k_init; the
    // discovery bitmaps and queues are always written before they are read.
    rc = zero_indegree_into(P.in_off, n, const_cast<uint32_t*>(P.Z), sm, stream);
    if (rc) return rc;
    rc = run_stepped(P, sm, root, alpha, beta, parents_dev, stream);
    if (rc) return rc;
    int32_t st[2] = {0, 0};
    NWG_CUDA_TRY(cudaMemcpyAsync(&st[0], &P.ctrl->h.status, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    NWG_CUDA_TRY(cudaMemcpyAsync(&st[1], &P.ctrl->err, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    NWG_CUDA_TRY(cudaStreamSynchronize(stream));
    const int status = st[0] ? st[0] : st[1];
    if (status != 0) return set_error(status, "device traversal reported status " + std::to_string(status));
    return NWG_OK;
  } catch (...) {
    return set_error(NWG_ESTATE, "unexpected C++ exception");
  }
}
