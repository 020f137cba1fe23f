// TBB-compatible scheduling shim used ONLY to compile the reference NWGraph
// headers (include/nwgraph/algorithms/bfs.hpp and what it includes) as the
// test oracle and the timed CPU baseline.  oneTBB is not installed on these
// machines; the reference's BFS arithmetic lives entirely in its own headers,
// TBB only schedules loops and stores queues.  This file is project-written:
// it provides the subset of the TBB API those headers name
// (blocked_range, split, parallel_for, parallel_reduce, parallel_for_each,
// parallel_sort, concurrent_vector, concurrent_queue, global_control,
// this_task_arena) with TBB's documented semantics.
//
// Threading: a fork-join pool whose waiting callers help execute queued
// tasks, so nested parallel loops (the reference's top-down step nests
// parallel_reduce over bins and over queue entries) make progress without
// deadlock.  Ranges are split recursively while `is_divisible()` and while
// the number of pieces is below 8 x threads (TBB's auto_partitioner also
// stops splitting once there is enough parallel slack).  The thread count is
// `global_control(max_allowed_parallelism)` if set, else the environment
// variable NWG_COMPAT_THREADS, else std::thread::hardware_concurrency().
// With one thread every call runs inline and serially.
//
// Deliberately NOT provided: <tbb/tbb.h>.  libstdc++ switches its parallel
// STL backend to TBB when that header exists.
#ifndef NWG_TBB_COMPAT_H
#define NWG_TBB_COMPAT_H

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <deque>
#include <functional>
#include <iterator>
#include <memory>
#include <mutex>
#include <thread>
#include <utility>
#include <vector>

namespace tbb {

struct split {};

namespace detail_compat {

inline std::atomic<long>& threads_override() {
  static std::atomic<long> v{0};
  return v;
}

inline long default_threads() {
  if (const char* e = std::getenv("NWG_COMPAT_THREADS")) {
    long v = std::atol(e);
    if (v > 0) return v;
  }
  long hc = (long)std::thread::hardware_concurrency();
  return hc > 0 ? hc : 1;
}

inline long active_threads() {
  long o = threads_override().load(std::memory_order_relaxed);
  return o > 0 ? o : default_threads();
}

// Fork-join pool.  Tasks are std::function<void()>; a group counts its
// outstanding tasks.  `run_and_wait` enqueues a group's tasks and the caller
// executes queued tasks (its own or others') until its group is done.
class pool {
 public:
  static pool& get() {
    static pool p;
    return p;
  }

  struct group {
    std::atomic<long> pending{0};
  };

  void run_and_wait(std::vector<std::function<void()>>& tasks) {
    if (tasks.empty()) return;
    ensure_workers(active_threads() - 1);
    group g;
    g.pending.store((long)tasks.size(), std::memory_order_relaxed);
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (auto& t : tasks) {
        auto fn = std::move(t);
        q_.push_back([fn = std::move(fn), &g]() {
          fn();
          g.pending.fetch_sub(1, std::memory_order_acq_rel);
        });
      }
    }
    cv_.notify_all();
    while (g.pending.load(std::memory_order_acquire) > 0) {
      std::function<void()> job;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (!q_.empty()) {
          job = std::move(q_.back());
          q_.pop_back();
        }
      }
      if (job) {
        tl_depth()++;
        job();
        tl_depth()--;
      } else {
        std::this_thread::yield();
      }
    }
  }

  static int& tl_depth() {
    thread_local int d = 0;
    return d;
  }

  ~pool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }

 private:
  void ensure_workers(long want) {
    std::lock_guard<std::mutex> lk(start_mu_);
    while ((long)workers_.size() < want) {
      workers_.emplace_back([this] { worker_loop(); });
    }
  }

  void worker_loop() {
    tl_depth() = 1;
    for (;;) {
      std::function<void()> job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return stop_ || !q_.empty(); });
        if (stop_ && q_.empty()) return;
        job = std::move(q_.front());
        q_.pop_front();
      }
      job();
    }
  }

  std::mutex                         mu_, start_mu_;
  std::condition_variable            cv_;
  std::deque<std::function<void()>>  q_;
  std::vector<std::thread>           workers_;
  bool                               stop_ = false;
};

// Split `r` breadth-first into at most `limit` pieces, stopping at
// non-divisible pieces.
template <class Range>
std::vector<Range> split_range(const Range& r, std::size_t limit) {
  std::vector<Range> pieces;
  pieces.push_back(r);
  bool progress = true;
  while (progress && pieces.size() < limit) {
    progress = false;
    std::size_t n = pieces.size();
    for (std::size_t i = 0; i < n && pieces.size() < limit; ++i) {
      if (pieces[i].is_divisible()) {
        Range right(pieces[i], split{});
        pieces.push_back(right);
        progress = true;
      }
    }
  }
  return pieces;
}

inline std::size_t piece_limit() { return (std::size_t)(8 * active_threads()); }

}  // namespace detail_compat

template <class Value>
class blocked_range {
 public:
  using const_iterator = Value;
  using size_type      = std::size_t;
  blocked_range() = default;
  blocked_range(Value b, Value e, size_type grain = 1) : begin_(b), end_(e), grain_(grain ? grain : 1) {}
  blocked_range(blocked_range& r, split) : begin_(r.begin_ + (r.end_ - r.begin_) / 2), end_(r.end_), grain_(r.grain_) {
    r.end_ = begin_;
  }
  Value     begin() const { return begin_; }
  Value     end() const { return end_; }
  size_type size() const { return size_type(end_ - begin_); }
  size_type grainsize() const { return grain_; }
  bool      empty() const { return !(begin_ < end_); }
  bool      is_divisible() const { return grain_ < size(); }

 private:
  Value     begin_{}, end_{};
  size_type grain_ = 1;
};

template <class Range, class Body>
void parallel_for(const Range& range, const Body& body) {
  if (detail_compat::active_threads() <= 1 || !range.is_divisible()) {
    Range r(range);
    body(r);
    return;
  }
  auto pieces = detail_compat::split_range(range, detail_compat::piece_limit());
  std::vector<std::function<void()>> tasks;
  tasks.reserve(pieces.size());
  for (auto& p : pieces) {
    tasks.emplace_back([&body, p]() mutable { body(p); });
  }
  detail_compat::pool::get().run_and_wait(tasks);
}

template <class Index, class Function>
void parallel_for(Index first, Index last, const Function& f) {
  parallel_for(blocked_range<Index>(first, last), [&](const blocked_range<Index>& r) {
    for (Index i = r.begin(); i < r.end(); ++i) f(i);
  });
}

// Functional form: real_body(range, running_value) -> value;
// reduction(a, b) -> value.  Pieces are combined left to right.
template <class Range, class Value, class RealBody, class Reduction>
Value parallel_reduce(const Range& range, const Value& identity, const RealBody& real_body, const Reduction& reduction) {
  if (detail_compat::active_threads() <= 1 || !range.is_divisible()) {
    Range r(range);
    return real_body(r, identity);
  }
  auto pieces = detail_compat::split_range(range, detail_compat::piece_limit());
  std::vector<Value> partial(pieces.size(), identity);
  std::vector<std::function<void()>> tasks;
  tasks.reserve(pieces.size());
  for (std::size_t i = 0; i < pieces.size(); ++i) {
    tasks.emplace_back([&, i]() { partial[i] = real_body(pieces[i], identity); });
  }
  detail_compat::pool::get().run_and_wait(tasks);
  Value acc = identity;
  for (auto& v : partial) acc = reduction(acc, v);
  return acc;
}

template <class Iterator, class Body>
void parallel_for_each(Iterator first, Iterator last, const Body& body) {
  for (; first != last; ++first) body(*first);
}

template <class Container, class Body>
void parallel_for_each(Container& c, const Body& body) {
  parallel_for_each(std::begin(c), std::end(c), body);
}

template <class RandomIt>
void parallel_sort(RandomIt first, RandomIt last) {
  std::sort(first, last);
}

template <class RandomIt, class Compare>
void parallel_sort(RandomIt first, RandomIt last, const Compare& comp) {
  std::sort(first, last, comp);
}

// Segmented vector: element i lives in segment s = floor(log2(i / B + 1)),
// segments are allocated once by CAS and never move, so concurrent
// push_back is safe and references stay valid (TBB's guarantee).
template <class T>
class concurrent_vector {
  static constexpr std::size_t kBase = 64;
  static constexpr int         kSegs = 48;

 public:
  using value_type      = T;
  using size_type       = std::size_t;
  using reference       = T&;
  using const_reference = const T&;

  concurrent_vector() {
    for (auto& s : segs_) s.store(nullptr, std::memory_order_relaxed);
  }
  concurrent_vector(const concurrent_vector& o) : concurrent_vector() {
    for (size_type i = 0; i < o.size(); ++i) push_back(o[i]);
  }
  concurrent_vector(concurrent_vector&& o) noexcept : concurrent_vector() { swap(o); }
  concurrent_vector& operator=(const concurrent_vector& o) {
    if (this != &o) {
      clear();
      for (size_type i = 0; i < o.size(); ++i) push_back(o[i]);
    }
    return *this;
  }
  concurrent_vector& operator=(concurrent_vector&& o) noexcept {
    swap(o);
    return *this;
  }
  ~concurrent_vector() { release(); }

  void swap(concurrent_vector& o) noexcept {
    for (int s = 0; s < kSegs; ++s) {
      T* a = segs_[s].load(std::memory_order_relaxed);
      segs_[s].store(o.segs_[s].load(std::memory_order_relaxed), std::memory_order_relaxed);
      o.segs_[s].store(a, std::memory_order_relaxed);
    }
    size_type a = size_.load(std::memory_order_relaxed);
    size_.store(o.size_.load(std::memory_order_relaxed), std::memory_order_relaxed);
    o.size_.store(a, std::memory_order_relaxed);
  }

  size_type push_back(const T& v) {
    size_type i = size_.fetch_add(1, std::memory_order_acq_rel);
    slot(i) = v;
    return i;
  }

  size_type size() const { return size_.load(std::memory_order_acquire); }
  bool      empty() const { return size() == 0; }
  void      clear() { size_.store(0, std::memory_order_release); }  // keeps segments for reuse

  T&       operator[](size_type i) { return const_cast<T&>(static_cast<const concurrent_vector&>(*this)[i]); }
  const T& operator[](size_type i) const {
    auto [s, off] = locate(i);
    return segs_[s].load(std::memory_order_acquire)[off];
  }

  template <bool Const>
  class iter {
    using vec_t = std::conditional_t<Const, const concurrent_vector, concurrent_vector>;
    vec_t*    v_ = nullptr;
    size_type i_ = 0;

   public:
    using iterator_category = std::random_access_iterator_tag;
    using value_type        = T;
    using difference_type   = std::ptrdiff_t;
    using pointer           = std::conditional_t<Const, const T*, T*>;
    using reference         = std::conditional_t<Const, const T&, T&>;
    iter() = default;
    iter(vec_t* v, size_type i) : v_(v), i_(i) {}
    reference operator*() const { return (*v_)[i_]; }
    pointer   operator->() const { return &(*v_)[i_]; }
    reference operator[](difference_type n) const { return (*v_)[i_ + n]; }
    iter&     operator++() { ++i_; return *this; }
    iter      operator++(int) { iter t = *this; ++i_; return t; }
    iter&     operator--() { --i_; return *this; }
    iter      operator--(int) { iter t = *this; --i_; return t; }
    iter&     operator+=(difference_type n) { i_ += n; return *this; }
    iter&     operator-=(difference_type n) { i_ -= n; return *this; }
    iter      operator+(difference_type n) const { return iter(v_, i_ + n); }
    friend iter operator+(difference_type n, const iter& it) { return it + n; }
    iter      operator-(difference_type n) const { return iter(v_, i_ - n); }
    difference_type operator-(const iter& o) const { return difference_type(i_) - difference_type(o.i_); }
    bool operator==(const iter& o) const { return i_ == o.i_; }
    bool operator!=(const iter& o) const { return i_ != o.i_; }
    bool operator<(const iter& o) const { return i_ < o.i_; }
    bool operator>(const iter& o) const { return i_ > o.i_; }
    bool operator<=(const iter& o) const { return i_ <= o.i_; }
    bool operator>=(const iter& o) const { return i_ >= o.i_; }
  };
  using iterator       = iter<false>;
  using const_iterator = iter<true>;

  iterator       begin() { return iterator(this, 0); }
  iterator       end() { return iterator(this, size()); }
  const_iterator begin() const { return const_iterator(this, 0); }
  const_iterator end() const { return const_iterator(this, size()); }

 private:
  static std::pair<int, size_type> locate(size_type i) {
    size_type q = i / kBase + 1;
    int       s = 63 - __builtin_clzll((unsigned long long)q);
    size_type first = kBase * ((size_type(1) << s) - 1);
    return {s, i - first};
  }
  T& slot(size_type i) {
    auto [s, off] = locate(i);
    T* seg = segs_[s].load(std::memory_order_acquire);
    if (!seg) {
      T* fresh    = new T[kBase << s];
      T* expected = nullptr;
      if (segs_[s].compare_exchange_strong(expected, fresh, std::memory_order_acq_rel)) {
        seg = fresh;
      } else {
        delete[] fresh;
        seg = expected;
      }
    }
    return seg[off];
  }
  void release() {
    for (auto& s : segs_) {
      delete[] s.load(std::memory_order_relaxed);
      s.store(nullptr, std::memory_order_relaxed);
    }
  }

  std::atomic<T*>        segs_[kSegs];
  std::atomic<size_type> size_{0};
};

template <class T>
class concurrent_queue {
 public:
  void push(const T& v) {
    std::lock_guard<std::mutex> lk(mu_);
    q_.push_back(v);
  }
  bool try_pop(T& out) {
    std::lock_guard<std::mutex> lk(mu_);
    if (q_.empty()) return false;
    out = q_.front();
    q_.pop_front();
    return true;
  }
  bool empty() const {
    std::lock_guard<std::mutex> lk(mu_);
    return q_.empty();
  }
  std::size_t unsafe_size() const { return q_.size(); }
  void        clear() {
    std::lock_guard<std::mutex> lk(mu_);
    q_.clear();
  }

 private:
  mutable std::mutex mu_;
  std::deque<T>      q_;
};

class global_control {
 public:
  enum parameter { max_allowed_parallelism, thread_stack_size };
  global_control(parameter p, std::size_t value) : p_(p) {
    if (p_ == max_allowed_parallelism) {
      prev_ = detail_compat::threads_override().exchange((long)value);
    }
  }
  ~global_control() {
    if (p_ == max_allowed_parallelism) detail_compat::threads_override().store(prev_);
  }
  global_control(global_control&& o) noexcept : p_(o.p_), prev_(o.prev_) { o.p_ = thread_stack_size; }
  global_control(const global_control&) = delete;
  static std::size_t active_value(parameter p) {
    return p == max_allowed_parallelism ? (std::size_t)detail_compat::active_threads() : 0;
  }

 private:
  parameter p_;
  long      prev_ = 0;
};

// A priority queue behind one mutex (top = greatest under Compare).
template <class T, class Compare = std::less<T>>
class concurrent_priority_queue {
 public:
  void push(const T& v) {
    std::lock_guard<std::mutex> lk(mu_);
    h_.push_back(v);
    std::push_heap(h_.begin(), h_.end(), cmp_);
  }
  bool try_pop(T& out) {
    std::lock_guard<std::mutex> lk(mu_);
    if (h_.empty()) return false;
    std::pop_heap(h_.begin(), h_.end(), cmp_);
    out = h_.back();
    h_.pop_back();
    return true;
  }
  bool empty() const {
    std::lock_guard<std::mutex> lk(mu_);
    return h_.empty();
  }
  std::size_t size() const {
    std::lock_guard<std::mutex> lk(mu_);
    return h_.size();
  }
  void clear() {
    std::lock_guard<std::mutex> lk(mu_);
    h_.clear();
  }

 private:
  mutable std::mutex mu_;
  std::vector<T>     h_;
  Compare            cmp_;
};

namespace this_task_arena {
inline int max_concurrency() { return (int)detail_compat::active_threads(); }
}  // namespace this_task_arena

class queuing_mutex {
 public:
  class scoped_lock {
   public:
    scoped_lock() = default;
    explicit scoped_lock(queuing_mutex& m) { acquire(m); }
    ~scoped_lock() { release(); }
    void acquire(queuing_mutex& m) {
      m_ = &m;
      m_->mu_.lock();
    }
    void release() {
      if (m_) m_->mu_.unlock();
      m_ = nullptr;
    }

   private:
    queuing_mutex* m_ = nullptr;
  };

 private:
  std::mutex mu_;
};

}  // namespace tbb

#endif  // NWG_TBB_COMPAT_H
