// Serving loop: (graph, root) BFS queries against graphs kept resident in
// HBM, answered as depth rows: uint8 (255 = unreached) or, with
// depth_bytes = 2, uint16 (0xFFFF = unreached).  No reference
// counterpart: NWGraph answers one bfs call at a time; each answer here equals
// the single-source BFS depths of that (graph, root).
//
// Design:
//   * graphs are registered handles (nwg_graph_register / generators), all on
//     one device; the server borrows them and never copies them;
//   * `slots` worker threads, each owning a CUDA stream and a multi-source
//     workspace sized for the largest graph, run batches concurrently, so a
//     batch admitted while others are on the device overlaps with them
//     (continuous batching at batch granularity: a slot that finishes takes
//     the next batch at once);
//   * a free slot takes the graph of the oldest waiting query and coalesces
//     up to max_batch waiting queries on that graph into one multi-source
//     pass (64 sources per 64-bit word, nwg_msbfs.cu);
//   * admission: each query holds per-query state (device depth row, its
//     share of the four bitsets, the pinned host row) from the moment a slot
//     takes it until its answer is in host memory; the sum over taken
//     queries never exceeds budget_bytes -- a query that does not fit waits.
//     The slots' fixed buffers come out of the same budget at creation.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "nwg_internal.cuh"

using namespace nwg;

#define NWG_API extern "C" __attribute__((visibility("default")))

namespace {

using Clock = std::chrono::steady_clock;

constexpr uint32_t kMaxBatch = 256;  // sources of one multi-source pass

struct Query {
  uint32_t          graph = 0, root = 0;
  uint8_t*          out   = nullptr;  // host destination (n * depth_bytes bytes of the graph) or null
  uint64_t          bytes = 0;        // per-query state while taken
  Clock::time_point arrival{}, done_at{};
  uint32_t          batch  = 0;       // size of the batch it ran in
  uint32_t*         group_done = nullptr;  // completion counter of its trace (under the server lock)
  int               status = 0;
  bool              taken = false, done = false, heap = false;
};

struct Slot {
  MsWorkspace* ws        = nullptr;
  uint8_t*     depth_dev = nullptr;  // kMaxBatch * n_cap * depth_bytes
  uint8_t*     staging   = nullptr;  // pinned, the same size
  std::thread  th;
};

struct Server {
  int                     device = 0;
  std::vector<GraphDev*>  graphs;
  uint32_t                max_batch = kMaxBatch;
  uint64_t                budget    = 0;
  int                     alpha     = 4;
  uint32_t                depth_bytes = 1;  // bytes per vertex of an answer row
  uint64_t                n_cap = 0, m_cap = 0, slot_bytes = 0;
  std::vector<Slot>       slots;
  std::mutex              mu;
  std::condition_variable cv_work;  // workers: a query arrived or budget was freed
  std::condition_variable cv_done;  // waiters: a batch completed
  std::deque<Query*>              fifo;       // arrival order; taken entries are dropped lazily
  std::vector<std::deque<Query*>> per_graph;  // waiting queries of each graph, arrival order
  std::unordered_map<uint64_t, Query*> tickets;
  uint64_t    next_ticket = 1;
  uint64_t    in_use = 0, peak_in_use = 0;
  uint32_t    in_flight = 0, peak_in_flight = 0;
  uint64_t    batches = 0, done_count = 0;
  double      batch_time_s = 0;  // summed host time of batches from take to answer
  bool        stop = false;
  std::string first_error;
};

// State a query holds while a slot works on it: its depth row on the device
// and in pinned host memory, and one bit per vertex in each of the pass's
// four bitsets (VIS, FR[2], NX).
uint64_t query_bytes(uint64_t n, uint32_t depth_bytes) { return 2 * n * depth_bytes + (4 * n + 7) / 8; }

Query* oldest_waiting(Server* s) {
  while (!s->fifo.empty() && s->fifo.front()->taken) s->fifo.pop_front();
  return s->fifo.empty() ? nullptr : s->fifo.front();
}

void worker(Server* s, Slot* slot) {
  cudaSetDevice(s->device);
  std::vector<Query*>   batch;
  std::vector<uint32_t> roots;
  std::vector<uint8_t>  deep(kMaxBatch);
  batch.reserve(kMaxBatch);
  roots.reserve(kMaxBatch);
  for (;;) {
    std::unique_lock<std::mutex> lk(s->mu);
    Query*                       head = nullptr;
    s->cv_work.wait(lk, [&] {
      if (s->stop) return true;
      head = oldest_waiting(s);
      return head && s->in_use + head->bytes <= s->budget;
    });
    if (s->stop) return;
    const uint32_t gi = head->graph;
    auto&          dq = s->per_graph[gi];
    batch.clear();
    while (!dq.empty() && batch.size() < s->max_batch) {
      Query* q = dq.front();
      if (s->in_use + q->bytes > s->budget) break;
      dq.pop_front();
      q->taken = true;
      s->in_use += q->bytes;
      batch.push_back(q);
    }
    s->peak_in_use    = std::max(s->peak_in_use, s->in_use);
    s->peak_in_flight = std::max(s->peak_in_flight, ++s->in_flight);
    lk.unlock();

    const auto t_take = Clock::now();
    GraphDev*  g      = s->graphs[gi];
    const auto k      = (uint32_t)batch.size();
    roots.clear();
    for (Query* q : batch) roots.push_back(q->root);
    nwg_msbfs_stats st   = {};
    const size_t    row  = (size_t)g->n * s->depth_bytes;
    int rc = ms_run_on(slot->ws, g, roots.data(), k, slot->depth_dev, s->depth_bytes, deep.data(), s->alpha,
                       slot->ws->stream, &st);
    if (rc == NWG_OK) {
      cudaError_t e = cudaMemcpyAsync(slot->staging, slot->depth_dev, k * row, cudaMemcpyDeviceToHost,
                                      slot->ws->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(slot->ws->stream);
      if (e != cudaSuccess) rc = cuda_error(e, "serving batch read-back");
    }
    if (rc == NWG_OK)
      for (uint32_t i = 0; i < k; ++i)
        if (batch[i]->out) std::memcpy(batch[i]->out, slot->staging + i * row, row);
    std::string err;
    if (rc != NWG_OK) {
      char buf[512];
      nwg_last_error(buf, sizeof buf);
      err = buf;
    } else if (st.deep_sources) {  // only uint8 answers can be deep: those queries alone fail
      err = "a query's traversal goes deeper than 254 levels: its uint8 answer holds the depths up to 254 and "
            "255 beyond (depth_bytes = 2 answers it exactly)";
    }
    const auto t_done = Clock::now();

    lk.lock();
    for (uint32_t i = 0; i < k; ++i) {
      Query* q   = batch[i];
      q->done_at = t_done;
      q->batch   = k;
      q->status  = (rc == NWG_OK && s->depth_bytes == 1 && deep[i]) ? NWG_EOVERFLOW : rc;
      q->done    = true;
      if (q->group_done) ++*q->group_done;
      s->in_use -= q->bytes;
    }
    if (!err.empty() && s->first_error.empty()) s->first_error = err;
    s->in_flight--;
    s->batches++;
    s->done_count += k;
    s->batch_time_s += std::chrono::duration<double>(t_done - t_take).count();
    lk.unlock();
    s->cv_done.notify_all();
    s->cv_work.notify_all();  // budget was freed
  }
}

void server_free(Server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (Slot& sl : s->slots)
    if (sl.th.joinable()) sl.th.join();
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  for (Slot& sl : s->slots) {
    if (sl.ws) ms_ws_free(sl.ws);
    cudaFree(sl.depth_dev);
    if (sl.staging) cudaFreeHost(sl.staging);
  }
  // queries nobody will answer: submitted ones are freed, none is left waiting
  for (auto& kv : s->tickets)
    if (kv.second->heap) delete kv.second;
  cudaSetDevice(prev);
  delete s;
}

int check_query(const Server* s, uint32_t graph, uint32_t root, uint32_t i) {
  if (graph >= s->graphs.size())
    return set_error(NWG_EINVAL, "query " + std::to_string(i) + ": graph index out of range");
  if (root >= s->graphs[graph]->n) return set_error(NWG_EINVAL, "query " + std::to_string(i) + ": root >= n");
  if (query_bytes(s->graphs[graph]->n, s->depth_bytes) > s->budget)
    return set_error(NWG_EINVAL, "query " + std::to_string(i) + ": its state alone exceeds the budget");
  return NWG_OK;
}

// Caller holds s->mu.
void enqueue(Server* s, Query* q) {
  s->fifo.push_back(q);
  s->per_graph[q->graph].push_back(q);
}

double percentile(std::vector<double>& v, double p) {
  if (v.empty()) return 0.0;
  const size_t i = std::min(v.size() - 1, (size_t)(p * (double)(v.size() - 1) + 0.5));
  std::nth_element(v.begin(), v.begin() + i, v.end());
  return v[i];
}

}  // namespace

NWG_API int nwg_server_create(const nwg_graph* graphs, uint32_t num_graphs, const nwg_server_config* cfg,
                              nwg_server* out) {
  try {
    if (!out) return set_error(NWG_EINVAL, "out handle pointer is NULL");
    *out = nullptr;
    if (!graphs || num_graphs == 0) return set_error(NWG_EINVAL, "no graphs");
    nwg_server_config c = {};
    if (cfg) c = *cfg;
    const uint32_t want_slots = c.slots ? c.slots : 8;
    const uint32_t max_batch  = c.max_batch ? c.max_batch : kMaxBatch;
    if (want_slots > 64) return set_error(NWG_EINVAL, "slots must be 1..64");
    if (max_batch > kMaxBatch) return set_error(NWG_EINVAL, "max_batch must be 1..256");
    if (c.alpha < 0) return set_error(NWG_EINVAL, "alpha must be positive");
    if (c.depth_bytes > 2) return set_error(NWG_EINVAL, "depth_bytes must be 1 or 2");
    auto* s      = new Server();
    s->depth_bytes = c.depth_bytes ? c.depth_bytes : 1;
    s->max_batch = max_batch;
    s->budget    = c.budget_bytes ? c.budget_bytes : (16ull << 30);
    s->alpha     = c.alpha ? c.alpha : 4;
    for (uint32_t i = 0; i < num_graphs; ++i) {
      if (!graphs[i]) {
        delete s;
        return set_error(NWG_EINVAL, "graph " + std::to_string(i) + " is NULL");
      }
      auto* g = reinterpret_cast<GraphDev*>(graphs[i]);
      if (i == 0) s->device = g->device;
      if (g->device != s->device) {
        delete s;
        return set_error(NWG_EINVAL, "all graphs of a server must live on one device");
      }
      s->graphs.push_back(g);
      s->n_cap = std::max(s->n_cap, g->n);
      s->m_cap = std::max(s->m_cap, g->m);
    }
    s->per_graph.resize(num_graphs);
    const uint64_t rows_bytes = (uint64_t)kMaxBatch * std::max<uint64_t>(s->n_cap, 1) * s->depth_bytes;
    s->slot_bytes = ms_ws_bytes(s->n_cap, s->m_cap) + 2ull * rows_bytes;
    // the slots' fixed buffers count against the budget; keep room for at
    // least one largest query beside them
    const uint64_t biggest = query_bytes(s->n_cap, s->depth_bytes);
    const uint64_t room    = s->budget > biggest ? s->budget - biggest : 0;
    const uint64_t fit  = room / s->slot_bytes;
    if (fit == 0) {
      delete s;
      return set_error(NWG_EINVAL, "budget of " + std::to_string(c.budget_bytes) +
                                       " bytes holds no slot (one slot needs " + std::to_string(s->slot_bytes) + ")");
    }
    const uint32_t nslots = (uint32_t)std::min<uint64_t>(want_slots, fit);
    s->budget -= nslots * s->slot_bytes;  // what is left is for per-query state
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    s->slots.resize(nslots);
    for (Slot& sl : s->slots) {
      sl.ws  = new MsWorkspace();
      int rc = ms_ws_init_cap(nullptr, s->n_cap, s->m_cap, sl.ws);
      if (rc == NWG_OK && (cudaMalloc(&sl.depth_dev, (size_t)rows_bytes) != cudaSuccess ||
                           cudaMallocHost(&sl.staging, (size_t)rows_bytes) != cudaSuccess)) {
        cudaGetLastError();
        rc = set_error(NWG_ENOMEM, "serving slot allocation failed");
      }
      if (rc != NWG_OK) {
        cudaSetDevice(prev);
        server_free(s);
        return rc;
      }
    }
    cudaSetDevice(prev);
    for (Slot& sl : s->slots) sl.th = std::thread(worker, s, &sl);
    *out = reinterpret_cast<nwg_server>(s);
    return NWG_OK;
  } catch (const std::exception& ex) {
    return set_error(NWG_ENOMEM, std::string("server creation failed: ") + ex.what());
  }
}

NWG_API int nwg_server_destroy(nwg_server h) {
  if (!h) return set_error(NWG_EINVAL, "NULL server");
  server_free(reinterpret_cast<Server*>(h));
  return NWG_OK;
}

NWG_API int nwg_server_submit(nwg_server h, uint32_t graph, uint32_t root, uint8_t* depths_host, uint64_t* ticket) {
  if (!h || !ticket) return set_error(NWG_EINVAL, "NULL argument");
  auto* s  = reinterpret_cast<Server*>(h);
  int   rc = check_query(s, graph, root, 0);
  if (rc) return rc;
  auto* q    = new (std::nothrow) Query();
  if (!q) return set_error(NWG_ENOMEM, "host allocation failed");
  q->graph   = graph;
  q->root    = root;
  q->out     = depths_host;
  q->bytes   = query_bytes(s->graphs[graph]->n, s->depth_bytes);
  q->heap    = true;
  q->arrival = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    *ticket = s->next_ticket++;
    s->tickets.emplace(*ticket, q);
    enqueue(s, q);
  }
  s->cv_work.notify_one();
  return NWG_OK;
}

NWG_API int nwg_server_wait(nwg_server h, uint64_t ticket, double* latency_us) {
  if (!h) return set_error(NWG_EINVAL, "NULL server");
  auto*                        s = reinterpret_cast<Server*>(h);
  std::unique_lock<std::mutex> lk(s->mu);
  auto                         it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return set_error(NWG_EINVAL, "unknown ticket");
  Query* q = it->second;
  s->cv_done.wait(lk, [&] { return q->done; });
  s->tickets.erase(it);
  const int rc = q->status;
  if (latency_us) *latency_us = std::chrono::duration<double, std::micro>(q->done_at - q->arrival).count();
  const std::string err = s->first_error;
  lk.unlock();
  delete q;
  if (rc != NWG_OK) return set_error(rc, "query failed: " + err);
  return NWG_OK;
}

NWG_API int nwg_server_run_trace(nwg_server h, uint32_t count, const uint32_t* graph, const uint32_t* root,
                                 const double* arrival_us, uint8_t* const* depths_host, double* latency_us,
                                 uint32_t* batch_size, nwg_server_stats* stats) {
  try {
    if (!h || (count && (!graph || !root || !arrival_us))) return set_error(NWG_EINVAL, "NULL argument");
    auto* s = reinterpret_cast<Server*>(h);
    for (uint32_t i = 0; i < count; ++i) {
      int rc = check_query(s, graph[i], root[i], i);
      if (rc) return rc;
      if (i && arrival_us[i] < arrival_us[i - 1]) return set_error(NWG_EINVAL, "arrival times must not decrease");
    }
    std::vector<Query> qs(count);
    uint32_t           finished = 0;
    for (uint32_t i = 0; i < count; ++i) {
      qs[i].group_done = &finished;
      qs[i].graph = graph[i];
      qs[i].root  = root[i];
      qs[i].out   = depths_host ? depths_host[i] : nullptr;
      qs[i].bytes = query_bytes(s->graphs[graph[i]]->n, s->depth_bytes);
    }
    uint64_t b0;
    double   bt0;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      b0               = s->batches;
      bt0              = s->batch_time_s;
      s->peak_in_use    = s->in_use;
      s->peak_in_flight = s->in_flight;
      s->first_error.clear();
    }
    // open loop: query i is released at t0 + arrival_us[i] whatever the
    // server's progress; its latency runs from that scheduled time
    const auto t0 = Clock::now() + std::chrono::microseconds(1000);
    uint32_t   i  = 0;
    while (i < count) {
      const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(arrival_us[i]));
      auto       now = Clock::now();
      if (now < due) {
        const auto ahead = due - now;
        if (ahead > std::chrono::microseconds(200)) std::this_thread::sleep_for(ahead - std::chrono::microseconds(100));
        else std::this_thread::yield();
        continue;
      }
      uint32_t released = 0;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        while (i < count) {
          const auto d =
              t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(arrival_us[i]));
          if (d > now) break;
          qs[i].arrival = d;
          enqueue(s, &qs[i]);
          ++i;
          ++released;
        }
      }
      if (released > 1) s->cv_work.notify_all();
      else s->cv_work.notify_one();
    }
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return finished == count; });
    const uint64_t    nb      = s->batches - b0;
    const double      btime   = s->batch_time_s - bt0;
    const uint64_t    peak    = s->peak_in_use;
    const uint32_t    peak_fl = s->peak_in_flight;
    const std::string err     = s->first_error;
    lk.unlock();

    std::vector<double> lat(count);
    uint64_t            failed = 0;
    auto                last   = t0;
    for (uint32_t j = 0; j < count; ++j) {
      lat[j] = std::chrono::duration<double, std::micro>(qs[j].done_at - qs[j].arrival).count();
      if (latency_us) latency_us[j] = lat[j];
      if (batch_size) batch_size[j] = qs[j].batch;
      if (qs[j].status != NWG_OK) failed++;
      last = std::max(last, qs[j].done_at);
    }
    if (stats) {
      nwg_server_stats st = {};
      st.queries          = count;
      st.batches          = nb;
      st.failed           = failed;
      const auto first    = count ? qs[0].arrival : t0;
      st.wall_s           = std::chrono::duration<double>(last - first).count();
      st.qps              = st.wall_s > 0 ? (double)count / st.wall_s : 0.0;
      st.mean_batch       = nb ? (double)count / (double)nb : 0.0;
      double sum          = 0;
      for (double x : lat) sum += x;
      st.mean_ms          = count ? sum / count / 1e3 : 0.0;
      std::vector<double> tmp(lat);
      st.p50_ms           = percentile(tmp, 0.50) / 1e3;
      st.p99_ms           = percentile(tmp, 0.99) / 1e3;
      st.max_ms           = tmp.empty() ? 0.0 : *std::max_element(tmp.begin(), tmp.end()) / 1e3;
      st.peak_state_bytes = peak;
      st.budget_bytes     = s->budget;
      st.slot_bytes       = s->slot_bytes;
      st.slots            = (uint32_t)s->slots.size();
      st.peak_in_flight   = peak_fl;
      st.batch_time_s     = btime;
      *stats              = st;
    }
    if (failed) return set_error(NWG_ESTATE, std::to_string(failed) + " queries failed: " + err);
    return NWG_OK;
  } catch (const std::exception& ex) {
    return set_error(NWG_ENOMEM, std::string("trace replay failed: ") + ex.what());
  }
}
