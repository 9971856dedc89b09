// TBB-API shim: test infrastructure for the oracle, not part of the product.
//
// oneTBB is not installed in this image, so the NWGraph reference headers
// (include/nwgraph/util/backend.hpp:41-56 includes <oneapi/tbb.h> and
// <tbb/parallel_*.h>) are compiled against this std::thread-backed subset of
// the TBB interface. It covers exactly what the PageRank path and the CSR
// builder touch: blocked_range + split, parallel_for (range and index forms),
// parallel_reduce (functional form), parallel_for_each, parallel_sort,
// concurrent_vector, concurrent_queue, global_control, queuing_mutex,
// this_task_arena::current_thread_index and auto_partitioner.
//
// Scheduling: a range is split recursively (largest leaf first, TBB's Range
// concept: is_divisible() + splitting constructor) into at most 4x the thread
// count leaves; threads take leaves in order from an atomic counter and
// parallel_reduce combines the leaf results in leaf order, so a reduction is
// deterministic for a given thread count.
//
// Deliberately no <tbb/tbb.h>: libstdc++ switches its PSTL backend to TBB when
// that header exists and would then need parts of TBB this shim lacks.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

namespace tbb {

struct split {};
struct auto_partitioner {};
struct simple_partitioner {};
struct static_partitioner {};

namespace detail {
inline std::atomic<int>& thread_cap() {
  static std::atomic<int> cap{0};
  return cap;
}
inline int num_threads() {
  int c = thread_cap().load();
  if (c > 0) return c;
  unsigned h = std::thread::hardware_concurrency();
  return h ? static_cast<int>(h) : 1;
}
inline int& tls_index() {
  thread_local int idx = 0;
  return idx;
}

// Split `whole` into leaves; leaves keep the left-to-right order of the range.
template <class Range>
std::vector<Range> make_leaves(const Range& whole, int nthreads) {
  std::vector<Range> leaves;
  leaves.push_back(whole);
  const std::size_t target = static_cast<std::size_t>(nthreads) * 4;
  if (nthreads <= 1) return leaves;
  bool progress = true;
  while (leaves.size() < target && progress) {
    progress = false;
    std::vector<Range> next;
    next.reserve(leaves.size() * 2);
    for (auto& r : leaves) {
      if (next.size() + 1 < target * 2 && r.is_divisible()) {
        Range left(r);
        Range right(left, split{});
        next.push_back(left);
        next.push_back(right);
        progress = true;
      } else {
        next.push_back(r);
      }
    }
    leaves.swap(next);
  }
  return leaves;
}

template <class F>
void run_indexed(std::size_t count, int nthreads, F&& f) {
  if (count == 0) return;
  int nt = std::max(1, std::min<int>(nthreads, static_cast<int>(count)));
  if (nt == 1) {
    for (std::size_t i = 0; i < count; ++i) f(i);
    return;
  }
  std::atomic<std::size_t> next{0};
  auto worker = [&](int tid) {
    tls_index() = tid;
    for (std::size_t i = next.fetch_add(1); i < count; i = next.fetch_add(1)) f(i);
  };
  std::vector<std::thread> pool;
  pool.reserve(nt - 1);
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker, t);
  worker(0);
  for (auto& th : pool) th.join();
  tls_index() = 0;
}
}  // namespace detail

template <class Value>
class blocked_range {
  Value       begin_{}, end_{};
  std::size_t grain_ = 1;

public:
  using value_type = Value;
  using const_iterator = Value;
  using size_type = std::size_t;

  blocked_range() = default;
  blocked_range(Value b, Value e, std::size_t grain = 1) : begin_(b), end_(e), grain_(grain ? grain : 1) {}
  blocked_range(blocked_range& r, split) : begin_(r.begin_ + (r.end_ - r.begin_) / 2), end_(r.end_), grain_(r.grain_) {
    r.end_ = begin_;
  }
  Value       begin() const { return begin_; }
  Value       end() const { return end_; }
  std::size_t size() const { return static_cast<std::size_t>(end_ - begin_); }
  std::size_t grainsize() const { return grain_; }
  bool        empty() const { return !(begin_ < end_); }
  bool        is_divisible() const { return grain_ < size(); }
};

template <class Range, class Body>
void parallel_for(const Range& range, const Body& body) {
  auto leaves = detail::make_leaves(range, detail::num_threads());
  detail::run_indexed(leaves.size(), detail::num_threads(), [&](std::size_t i) {
    if (!leaves[i].empty()) body(leaves[i]);
  });
}
template <class Range, class Body, class Partitioner>
  requires(!std::is_integral_v<Range>)
void parallel_for(const Range& range, const Body& body, Partitioner&&) {
  parallel_for(range, body);
}

template <class Index, class F>
  requires std::is_integral_v<Index>
void parallel_for(Index first, Index last, const F& f) {
  parallel_for(blocked_range<Index>(first, last), [&](const blocked_range<Index>& r) {
    for (Index i = r.begin(); i != r.end(); ++i) f(i);
  });
}
template <class Index, class F>
  requires std::is_integral_v<Index>
void parallel_for(Index first, Index last, Index step, const F& f) {
  if (step <= 0 || !(first < last)) return;
  Index n = (last - first + step - 1) / step;
  parallel_for(Index(0), n, [&](Index k) { f(first + k * step); });
}

template <class Range, class Value, class RealBody, class Reduction>
Value parallel_reduce(const Range& range, const Value& identity, const RealBody& real_body, const Reduction& reduction) {
  auto               leaves = detail::make_leaves(range, detail::num_threads());
  std::vector<Value> partial(leaves.size(), identity);
  detail::run_indexed(leaves.size(), detail::num_threads(), [&](std::size_t i) {
    if (!leaves[i].empty()) partial[i] = real_body(leaves[i], identity);
  });
  Value acc = identity;
  for (auto& p : partial) acc = reduction(acc, p);
  return acc;
}
template <class Range, class Value, class RealBody, class Reduction, class Partitioner>
Value parallel_reduce(const Range& range, const Value& identity, const RealBody& real_body, const Reduction& reduction,
                      Partitioner&&) {
  return parallel_reduce(range, identity, real_body, reduction);
}

template <class It, class F>
void parallel_for_each(It first, It last, const F& f) {
  std::vector<It> items;
  for (It it = first; it != last; ++it) items.push_back(it);
  detail::run_indexed(items.size(), detail::num_threads(), [&](std::size_t i) { f(*items[i]); });
}
template <class Container, class F>
void parallel_for_each(Container& c, const F& f) {
  parallel_for_each(std::begin(c), std::end(c), f);
}

template <class It>
void parallel_sort(It first, It last) {
  std::sort(first, last);
}
template <class It, class Cmp>
void parallel_sort(It first, It last, const Cmp& cmp) {
  std::sort(first, last, cmp);
}

class global_control {
public:
  enum parameter { max_allowed_parallelism, thread_stack_size };
  global_control(parameter p, std::size_t value) : param_(p), saved_(detail::thread_cap().load()) {
    if (p == max_allowed_parallelism) detail::thread_cap().store(static_cast<int>(value));
  }
  ~global_control() {
    if (param_ == max_allowed_parallelism) detail::thread_cap().store(saved_);
  }
  global_control(const global_control&) = delete;
  global_control& operator=(const global_control&) = delete;
  static std::size_t active_value(parameter p) {
    return p == max_allowed_parallelism ? static_cast<std::size_t>(detail::num_threads()) : 0;
  }

private:
  parameter param_;
  int       saved_;
};

namespace this_task_arena {
inline int current_thread_index() { return detail::tls_index(); }
inline int max_concurrency() { return detail::num_threads(); }
}  // namespace this_task_arena

class queuing_mutex {
  std::mutex m_;

public:
  class scoped_lock {
    queuing_mutex* owner_ = nullptr;

  public:
    scoped_lock() = default;
    explicit scoped_lock(queuing_mutex& m) { acquire(m); }
    ~scoped_lock() { release(); }
    void acquire(queuing_mutex& m) {
      m.m_.lock();
      owner_ = &m;
    }
    void release() {
      if (owner_) owner_->m_.unlock();
      owner_ = nullptr;
    }
  };
};

template <class T, class Alloc = std::allocator<T>>
class concurrent_vector {
  std::deque<T>      data_;
  mutable std::mutex m_;

public:
  using value_type = T;
  using iterator = typename std::deque<T>::iterator;
  using const_iterator = typename std::deque<T>::const_iterator;
  using size_type = std::size_t;
  using reference = T&;
  using const_reference = const T&;

  concurrent_vector() = default;
  explicit concurrent_vector(std::size_t n) : data_(n) {}
  concurrent_vector(const concurrent_vector& o) : data_(o.data_) {}
  concurrent_vector& operator=(const concurrent_vector& o) {
    data_ = o.data_;
    return *this;
  }
  iterator push_back(const T& v) {
    std::lock_guard<std::mutex> g(m_);
    data_.push_back(v);
    return std::prev(data_.end());
  }
  iterator push_back(T&& v) {
    std::lock_guard<std::mutex> g(m_);
    data_.push_back(std::move(v));
    return std::prev(data_.end());
  }
  template <class... A>
  iterator emplace_back(A&&... a) {
    std::lock_guard<std::mutex> g(m_);
    data_.emplace_back(std::forward<A>(a)...);
    return std::prev(data_.end());
  }
  iterator       grow_by(std::size_t n) {
    std::lock_guard<std::mutex> g(m_);
    std::size_t                 old = data_.size();
    data_.resize(old + n);
    return data_.begin() + old;
  }
  void           reserve(std::size_t) {}
  void           resize(std::size_t n) { data_.resize(n); }
  void           clear() { data_.clear(); }
  std::size_t    size() const { return data_.size(); }
  bool           empty() const { return data_.empty(); }
  T&             operator[](std::size_t i) { return data_[i]; }
  const T&       operator[](std::size_t i) const { return data_[i]; }
  iterator       begin() { return data_.begin(); }
  iterator       end() { return data_.end(); }
  const_iterator begin() const { return data_.begin(); }
  const_iterator end() const { return data_.end(); }
};

template <class T, class Alloc = std::allocator<T>>
class concurrent_queue {
  std::deque<T>      q_;
  mutable std::mutex m_;

public:
  void push(const T& v) {
    std::lock_guard<std::mutex> g(m_);
    q_.push_back(v);
  }
  bool try_pop(T& out) {
    std::lock_guard<std::mutex> g(m_);
    if (q_.empty()) return false;
    out = std::move(q_.front());
    q_.pop_front();
    return true;
  }
  bool empty() const {
    std::lock_guard<std::mutex> g(m_);
    return q_.empty();
  }
  std::size_t unsafe_size() const { return q_.size(); }
  void        clear() {
    std::lock_guard<std::mutex> g(m_);
    q_.clear();
  }
};

}  // namespace tbb

namespace oneapi {
namespace tbb = ::tbb;
}
