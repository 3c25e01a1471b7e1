// Minimal ParlayLib-API shim, written for this project from the call sites
// of ParlayANN's hot-path headers (algorithms/utils/*.h, algorithms/vamana/*.h).
// ParlayLib itself is not vendored with the reference (empty submodule), so the
// reference's own search/build code is compiled in place against this shim.
//
// This is TEST INFRASTRUCTURE: it exists only so that the oracle can run the
// reference's code on the CPU. Nothing in the product links it.
//
// Semantics that matter for determinism (and that the GPU build reproduces):
//   * random_permutation(n): indices ordered by splitmix64(seed + i); a
//     bijective mix, so the order is total and identical on CPU and GPU.
//   * group_by_key: stable by key; values keep their input order.
//   * parallel_for: a persistent std::thread pool, dynamic chunking; nested
//     calls run sequentially on the calling worker.
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <initializer_list>
#include <iostream>
#include <iterator>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <optional>
#include <random>
#include <string>
#include <thread>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace parlay {

// ---------------------------------------------------------------- sequence
template <typename T>
class sequence {
 public:
  using value_type = T;
  using size_type = size_t;
  using iterator = T*;
  using const_iterator = const T*;
  using reference = T&;
  using const_reference = const T&;

  sequence() = default;
  explicit sequence(size_t n) { grow_to(n); for (size_t i = 0; i < n; i++) new (d_ + i) T(); n_ = n; }
  sequence(size_t n, const T& v) { grow_to(n); for (size_t i = 0; i < n; i++) new (d_ + i) T(v); n_ = n; }
  sequence(std::initializer_list<T> l) { grow_to(l.size()); for (auto& x : l) new (d_ + n_++) T(x); }
  template <typename It, typename = decltype(*std::declval<It>()),
            typename = std::enable_if_t<!std::is_integral_v<It>>>
  sequence(It first, It last) {
    size_t n = (size_t)std::distance(first, last);
    grow_to(n);
    for (; first != last; ++first) new (d_ + n_++) T(*first);
  }
  sequence(const sequence& o) { grow_to(o.n_); for (size_t i = 0; i < o.n_; i++) new (d_ + i) T(o.d_[i]); n_ = o.n_; }
  sequence(sequence&& o) noexcept : d_(o.d_), n_(o.n_), cap_(o.cap_) { o.d_ = nullptr; o.n_ = o.cap_ = 0; }
  sequence& operator=(const sequence& o) { if (this != &o) { sequence t(o); swap(t); } return *this; }
  sequence& operator=(sequence&& o) noexcept { if (this != &o) { destroy(); d_ = o.d_; n_ = o.n_; cap_ = o.cap_; o.d_ = nullptr; o.n_ = o.cap_ = 0; } return *this; }
  ~sequence() { destroy(); }

  void swap(sequence& o) noexcept { std::swap(d_, o.d_); std::swap(n_, o.n_); std::swap(cap_, o.cap_); }

  T* begin() { return d_; }
  T* end() { return d_ + n_; }
  const T* begin() const { return d_; }
  const T* end() const { return d_ + n_; }
  T* data() { return d_; }
  const T* data() const { return d_; }
  size_t size() const { return n_; }
  bool empty() const { return n_ == 0; }
  T& operator[](size_t i) { return d_[i]; }
  const T& operator[](size_t i) const { return d_[i]; }
  T& at(size_t i) { return d_[i]; }
  const T& at(size_t i) const { return d_[i]; }
  T& front() { return d_[0]; }
  T& back() { return d_[n_ - 1]; }
  const T& front() const { return d_[0]; }
  const T& back() const { return d_[n_ - 1]; }

  void reserve(size_t c) { if (c > cap_) realloc_to(c); }
  void push_back(const T& v) { if (n_ == cap_) realloc_to(cap_ ? 2 * cap_ : 4); new (d_ + n_++) T(v); }
  void push_back(T&& v) { if (n_ == cap_) realloc_to(cap_ ? 2 * cap_ : 4); new (d_ + n_++) T(std::move(v)); }
  template <typename... A> T& emplace_back(A&&... a) { if (n_ == cap_) realloc_to(cap_ ? 2 * cap_ : 4); new (d_ + n_) T(std::forward<A>(a)...); return d_[n_++]; }
  void pop_back() { d_[--n_].~T(); }
  void clear() { for (size_t i = 0; i < n_; i++) d_[i].~T(); n_ = 0; }
  void resize(size_t n) { if (n < n_) { for (size_t i = n; i < n_; i++) d_[i].~T(); n_ = n; } else { reserve(n); for (size_t i = n_; i < n; i++) new (d_ + i) T(); n_ = n; } }
  void resize(size_t n, const T& v) { if (n < n_) { resize(n); } else { reserve(n); for (size_t i = n_; i < n; i++) new (d_ + i) T(v); n_ = n; } }
  template <typename It> void append(It first, It last) { for (; first != last; ++first) push_back(*first); }
  template <typename R> void append(const R& r) { for (auto& x : r) push_back(x); }
  T* erase(T* pos) { std::move(pos + 1, end(), pos); pop_back(); return pos; }
  T* insert(T* pos, const T& v) { size_t k = pos - d_; push_back(v); std::rotate(d_ + k, d_ + n_ - 1, d_ + n_); return d_ + k; }

  bool operator==(const sequence& o) const { return n_ == o.n_ && std::equal(begin(), end(), o.begin()); }
  bool operator!=(const sequence& o) const { return !(*this == o); }
  bool operator<(const sequence& o) const { return std::lexicographical_compare(begin(), end(), o.begin(), o.end()); }

  // sub-range views
  auto cut(size_t s, size_t e) const;
  auto head(size_t k) const;
  auto tail(size_t k) const;

  static sequence uninitialized(size_t n) { return sequence(n); }
  // construct element i as f(i), in parallel, without default construction
  template <typename F> static sequence build(size_t n, F&& f);
  template <typename F> static sequence from_function(size_t n, F f) { sequence s; s.reserve(n); for (size_t i = 0; i < n; i++) s.push_back(f(i)); return s; }

 private:
  void grow_to(size_t n) { if (n > cap_) realloc_to(n); }
  void realloc_to(size_t c) {
    T* nd = static_cast<T*>(::operator new(sizeof(T) * (c ? c : 1), std::align_val_t(alignof(T) > 16 ? alignof(T) : 16)));
    if constexpr (std::is_move_constructible_v<T>) {
      for (size_t i = 0; i < n_; i++) { new (nd + i) T(std::move(d_[i])); d_[i].~T(); }
    } else {
      if (n_ != 0) std::abort();  // non-movable elements cannot be relocated
    }
    if (d_) ::operator delete(d_, std::align_val_t(alignof(T) > 16 ? alignof(T) : 16));
    d_ = nd; cap_ = c;
  }
  void destroy() {
    if (d_) { clear(); ::operator delete(d_, std::align_val_t(alignof(T) > 16 ? alignof(T) : 16)); }
    d_ = nullptr; n_ = cap_ = 0;
  }
  T* d_ = nullptr;
  size_t n_ = 0;
  size_t cap_ = 0;
};

// ---------------------------------------------------------------- slice
template <typename It, typename S = It>
struct slice {
  It b, e;
  slice(It b_, S e_) : b(b_), e(e_) {}
  slice() : b(), e() {}
  It begin() const { return b; }
  It end() const { return e; }
  size_t size() const { return (size_t)(e - b); }
  bool empty() const { return b == e; }
  decltype(auto) operator[](size_t i) const { return b[i]; }
  slice cut(size_t s, size_t t) const { return slice(b + s, b + t); }
};
template <typename It, typename S> slice<It, S> make_slice(It b, S e) { return slice<It, S>(b, e); }
template <typename R> auto make_slice(R&& r) { return make_slice(std::begin(r), std::end(r)); }

template <typename T> auto sequence<T>::cut(size_t s, size_t e) const { return make_slice(d_ + s, d_ + e); }
template <typename T> auto sequence<T>::head(size_t k) const { return make_slice(d_, d_ + k); }
template <typename T> auto sequence<T>::tail(size_t k) const { return make_slice(d_ + n_ - k, d_ + n_); }

template <typename R> using range_value_type_t = std::remove_cv_t<std::remove_reference_t<decltype(*std::begin(std::declval<R&>()))>>;

// ---------------------------------------------------------------- scheduler
namespace internal {
class pool {
 public:
  static pool& get() { static pool p; return p; }
  size_t workers() const { return nthreads_ + 1; }
  // run body(i) for i in [0, nblocks) across the pool; the caller participates
  void run(size_t nblocks, const std::function<void(size_t)>& body) {
    if (nthreads_ == 0 || nblocks <= 1 || in_worker()) { for (size_t i = 0; i < nblocks; i++) body(i); return; }
    std::unique_lock<std::mutex> job_lock(job_mu_);  // one parallel region at a time
    {
      std::lock_guard<std::mutex> g(mu_);
      body_ = &body; nblocks_ = nblocks; next_.store(0); active_ = nthreads_; epoch_++;
    }
    cv_.notify_all();
    tl_in_worker() = true;
    work();
    tl_in_worker() = false;
    std::unique_lock<std::mutex> g(mu_);
    done_cv_.wait(g, [&] { return active_ == 0; });
    body_ = nullptr;
  }
  static bool& tl_in_worker() { thread_local bool b = false; return b; }
  static size_t& tl_worker_id() { thread_local size_t id = 0; return id; }
  bool in_worker() const { return tl_in_worker(); }

 private:
  pool() {
    size_t n = std::thread::hardware_concurrency();
    if (const char* e = std::getenv("PARLAY_NUM_THREADS")) { long v = std::atol(e); if (v > 0) n = (size_t)v; }
    if (n == 0) n = 1;
    nthreads_ = n - 1;
    for (size_t t = 0; t < nthreads_; t++) threads_.emplace_back([this, t] { loop(t + 1); });
  }
  ~pool() {
    { std::lock_guard<std::mutex> g(mu_); stop_ = true; epoch_++; }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }
  void work() {
    for (;;) {
      size_t i = next_.fetch_add(1);
      if (i >= nblocks_) break;
      (*body_)(i);
    }
  }
  void loop(size_t id) {
    tl_worker_id() = id;
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return stop_ || epoch_ != seen; });
        if (stop_) return;
        seen = epoch_;
      }
      tl_in_worker() = true;
      work();
      tl_in_worker() = false;
      std::lock_guard<std::mutex> g(mu_);
      if (--active_ == 0) done_cv_.notify_all();
    }
  }
  size_t nthreads_ = 0;
  std::vector<std::thread> threads_;
  std::mutex mu_, job_mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(size_t)>* body_ = nullptr;
  size_t nblocks_ = 0;
  std::atomic<size_t> next_{0};
  size_t active_ = 0;
  uint64_t epoch_ = 0;
  bool stop_ = false;
};
}  // namespace internal

inline size_t num_workers() { return internal::pool::get().workers(); }
inline size_t worker_id() { return internal::pool::tl_worker_id(); }

template <typename F>
void parallel_for(long start, long end, F&& f, long granularity = 0, bool = false) {
  if (end <= start) return;
  long n = end - start;
  long nw = (long)num_workers();
  long g = granularity > 0 ? granularity : std::max<long>(1, n / (8 * nw));
  if (n <= g || nw == 1 || internal::pool::get().in_worker()) { for (long i = start; i < end; i++) f(i); return; }
  size_t nblocks = (size_t)((n + g - 1) / g);
  std::function<void(size_t)> body = [&](size_t b) {
    long s = start + (long)b * g, e = std::min(end, s + g);
    for (long i = s; i < e; i++) f(i);
  };
  internal::pool::get().run(nblocks, body);
}

template <typename L, typename R>
void par_do(L&& l, R&& r, bool = false) { l(); r(); }

// ---------------------------------------------------------------- delayed
template <typename T, typename F>
struct delayed_sequence {
  using value_type = T;
  struct iterator {
    using iterator_category = std::random_access_iterator_tag;
    using value_type = T;
    using difference_type = std::ptrdiff_t;
    using pointer = void;
    using reference = T;
    const F* f; long i;
    T operator*() const { return (*f)(i); }
    T operator[](long k) const { return (*f)(i + k); }
    iterator& operator++() { ++i; return *this; }
    iterator operator++(int) { auto t = *this; ++i; return t; }
    iterator& operator--() { --i; return *this; }
    iterator& operator+=(long k) { i += k; return *this; }
    iterator& operator-=(long k) { i -= k; return *this; }
    iterator operator+(long k) const { return iterator{f, i + k}; }
    iterator operator-(long k) const { return iterator{f, i - k}; }
    long operator-(const iterator& o) const { return i - o.i; }
    bool operator==(const iterator& o) const { return i == o.i; }
    bool operator!=(const iterator& o) const { return i != o.i; }
    bool operator<(const iterator& o) const { return i < o.i; }
  };
  long n; F f;
  delayed_sequence(long n_, F f_) : n(n_), f(std::move(f_)) {}
  iterator begin() const { return iterator{&f, 0}; }
  iterator end() const { return iterator{&f, n}; }
  size_t size() const { return (size_t)n; }
  T operator[](size_t i) const { return f((long)i); }
};
template <typename T, typename F> auto delayed_seq(size_t n, F f) { return delayed_sequence<T, F>((long)n, std::move(f)); }
template <typename F> auto delayed_tabulate(size_t n, F f) {
  using T = std::remove_cv_t<std::remove_reference_t<decltype(f((size_t)0))>>;
  auto g = [f](long i) { return f((size_t)i); };
  return delayed_sequence<T, decltype(g)>((long)n, g);
}

// ---------------------------------------------------------------- primitives
template <typename T> template <typename F> sequence<T> sequence<T>::build(size_t n, F&& f) {
  sequence<T> s;
  s.grow_to(n);
  parallel_for(0, (long)n, [&](long i) { new (s.d_ + i) T(f((size_t)i)); });
  s.n_ = n;
  return s;
}
template <typename F> auto tabulate(size_t n, F&& f, size_t = 0) {
  using T = std::remove_cv_t<std::remove_reference_t<decltype(f((size_t)0))>>;
  return sequence<T>::build(n, f);
}
template <typename R, typename F> auto map(R&& r, F&& f, size_t = 0) {
  size_t n = r.size();
  auto b = std::begin(r);
  using T = std::remove_cv_t<std::remove_reference_t<decltype(f(*b))>>;
  return sequence<T>::build(n, [&](size_t i) { return f(b[i]); });
}
template <typename R> auto to_sequence(R&& r) {
  using T = range_value_type_t<R>;
  sequence<T> s; s.reserve(r.size());
  for (auto it = std::begin(r); it != std::end(r); ++it) s.push_back(*it);
  return s;
}
template <typename T> sequence<T> to_sequence(const sequence<T>& r) { return r; }
template <typename T = size_t> sequence<T> iota(size_t n) { sequence<T> s(n); for (size_t i = 0; i < n; i++) s[i] = (T)i; return s; }

template <typename T> struct addm { using value_type = T; T identity = T(0); T f(T a, T b) const { return a + b; } T operator()(T a, T b) const { return a + b; } };
template <typename T> struct minm { using value_type = T; T identity = std::numeric_limits<T>::max(); T f(T a, T b) const { return std::min(a, b); } T operator()(T a, T b) const { return std::min(a, b); } };
template <typename T> struct maxm { using value_type = T; T identity = std::numeric_limits<T>::lowest(); T f(T a, T b) const { return std::max(a, b); } T operator()(T a, T b) const { return std::max(a, b); } };

template <typename R> auto reduce(R&& r) {
  using T = range_value_type_t<R>;
  T acc = T(0);
  for (auto it = std::begin(r); it != std::end(r); ++it) acc = acc + *it;
  return acc;
}
template <typename R, typename M> auto reduce(R&& r, M m) {
  auto acc = m.identity;
  for (auto it = std::begin(r); it != std::end(r); ++it) acc = m(acc, *it);
  return acc;
}
// exclusive prefix sum; returns (offsets, total)
template <typename R> auto scan(R&& r) {
  using T = range_value_type_t<R>;
  sequence<T> s(r.size());
  T acc = T(0); size_t i = 0;
  for (auto it = std::begin(r); it != std::end(r); ++it, ++i) { s[i] = acc; acc = acc + *it; }
  return std::make_pair(std::move(s), acc);
}
template <typename R> auto scan_inclusive(R&& r) {
  using T = range_value_type_t<R>;
  sequence<T> s(r.size()); T acc = T(0); size_t i = 0;
  for (auto it = std::begin(r); it != std::end(r); ++it, ++i) { acc = acc + *it; s[i] = acc; }
  return s;
}
template <typename R, typename P> auto filter(R&& r, P&& p) {
  using T = range_value_type_t<R>;
  sequence<T> s;
  for (auto it = std::begin(r); it != std::end(r); ++it) if (p(*it)) s.push_back(*it);
  return s;
}
template <typename R, typename F> auto map_maybe(R&& r, F&& f) {
  using O = decltype(f(*std::begin(r)));
  using T = typename O::value_type;
  sequence<T> s;
  for (auto it = std::begin(r); it != std::end(r); ++it) { auto o = f(*it); if (o) s.push_back(*o); }
  return s;
}
template <typename R> auto flatten(R&& r) {
  using Inner = range_value_type_t<R>;
  using T = range_value_type_t<Inner>;
  sequence<T> s;
  for (auto it = std::begin(r); it != std::end(r); ++it) for (auto jt = std::begin(*it); jt != std::end(*it); ++jt) s.push_back(*jt);
  return s;
}
template <typename R> auto sort(R&& r) { auto s = to_sequence(r); std::sort(s.begin(), s.end()); return s; }
template <typename R, typename C> auto sort(R&& r, C&& c) { auto s = to_sequence(r); std::sort(s.begin(), s.end(), c); return s; }
template <typename R> void sort_inplace(R&& r) { std::sort(std::begin(r), std::end(r)); }
template <typename R, typename C> void sort_inplace(R&& r, C&& c) { std::sort(std::begin(r), std::end(r), c); }
template <typename R> auto stable_sort(R&& r) { auto s = to_sequence(r); std::stable_sort(s.begin(), s.end()); return s; }
template <typename R> auto max_element(R&& r) { return std::max_element(std::begin(r), std::end(r)); }
template <typename R, typename C> auto max_element(R&& r, C&& c) { return std::max_element(std::begin(r), std::end(r), c); }
template <typename R> auto min_element(R&& r) { return std::min_element(std::begin(r), std::end(r)); }
template <typename R, typename C> auto min_element(R&& r, C&& c) { return std::min_element(std::begin(r), std::end(r), c); }
template <typename R, typename F> void for_each(R&& r, F&& f) { for (auto it = std::begin(r); it != std::end(r); ++it) f(*it); }
template <typename R> auto kth_smallest_copy(R&& r, size_t k) { auto s = to_sequence(r); std::nth_element(s.begin(), s.begin() + k, s.end()); return s[k]; }
template <typename R, typename I> auto histogram_by_index(R&& r, I m) {
  sequence<I> h((size_t)m, (I)0);
  for (auto it = std::begin(r); it != std::end(r); ++it) h[(size_t)*it]++;
  return h;
}
template <typename R> auto remove_duplicates(R&& r) {
  auto s = to_sequence(r); std::sort(s.begin(), s.end());
  auto e = std::unique(s.begin(), s.end());
  return sequence<range_value_type_t<R>>(s.begin(), e);
}
// stable semisort: keys in ascending order, values in input order
template <typename R> auto group_by_key(R&& r) {
  using P = range_value_type_t<R>;
  using K = std::remove_cv_t<typename P::first_type>;
  using V = std::remove_cv_t<typename P::second_type>;
  auto s = to_sequence(r);
  std::stable_sort(s.begin(), s.end(), [](const P& a, const P& b) { return a.first < b.first; });
  sequence<std::pair<K, sequence<V>>> out;
  size_t i = 0;
  while (i < s.size()) {
    size_t j = i;
    sequence<V> vals;
    while (j < s.size() && !(s[i].first < s[j].first) && !(s[j].first < s[i].first)) vals.push_back(s[j++].second);
    out.push_back(std::make_pair(s[i].first, std::move(vals)));
    i = j;
  }
  return out;
}
template <typename R> auto reduce_by_key(R&& r) {
  using P = range_value_type_t<R>;
  using K = std::remove_cv_t<typename P::first_type>;
  using V = std::remove_cv_t<typename P::second_type>;
  auto g = group_by_key(r);
  sequence<std::pair<K, V>> out;
  for (auto& kv : g) { V acc = V(0); for (auto& v : kv.second) acc = acc + v; out.push_back(std::make_pair(kv.first, acc)); }
  return out;
}
struct size_of { template <typename T> size_t operator()(const T& x) const { return x.size(); } };

template <typename T, typename C> bool write_min(std::atomic<T>* a, T b, C less) {
  T c = a->load();
  while (less(b, c)) { if (a->compare_exchange_strong(c, b)) return true; }
  return false;
}
template <typename T, typename C> bool write_min(T* a, T b, C less) {
  T c = *a;
  while (less(b, c)) { if (__atomic_compare_exchange(a, &c, &b, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) return true; }
  return false;
}

// ---------------------------------------------------------------- random
inline uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
struct random_generator {
  using result_type = uint64_t;
  uint64_t state;
  explicit random_generator(uint64_t seed = 0) : state(seed) {}
  static constexpr result_type min() { return 0; }
  static constexpr result_type max() { return std::numeric_limits<uint64_t>::max(); }
  result_type operator()() { state = splitmix64(state); return state; }
  random_generator operator[](size_t i) const { return random_generator(splitmix64(state ^ (0x632be59bd9b4e019ULL * (i + 1)))); }
};
// Permutation of [0,n): indices ordered by splitmix64(seed + i). The GPU
// build regenerates exactly this order (same mix, same sort key).
constexpr uint64_t kPermSeed = 0x5eed5eed5eedULL;
template <typename T = size_t> sequence<T> random_permutation(size_t n, uint64_t seed = kPermSeed) {
  sequence<std::pair<uint64_t, T>> k(n);
  for (size_t i = 0; i < n; i++) k[i] = std::make_pair(splitmix64(seed + i), (T)i);
  std::sort(k.begin(), k.end());
  sequence<T> s(n);
  for (size_t i = 0; i < n; i++) s[i] = k[i].second;
  return s;
}
template <typename R> auto random_shuffle(R&& r) {
  auto p = random_permutation<size_t>(r.size());
  using T = range_value_type_t<R>;
  sequence<T> s(r.size());
  auto b = std::begin(r);
  for (size_t i = 0; i < r.size(); i++) s[i] = b[p[i]];
  return s;
}

// ---------------------------------------------------------------- misc
template <typename T> sequence<char> to_chars(const T& x) {
  std::string s;
  if constexpr (std::is_arithmetic_v<T>) s = std::to_string(x);
  else { s = "["; bool first = true; for (auto& v : x) { if (!first) s += ", "; s += std::to_string(v); first = false; } s += "]"; }
  return sequence<char>(s.begin(), s.end());
}
inline std::ostream& operator<<(std::ostream& os, const sequence<char>& s) { os.write(s.begin(), (std::streamsize)s.size()); return os; }

template <typename T> struct WorkerSpecific {
  std::vector<T> v;
  WorkerSpecific() : v(num_workers() + 1) {}
  T& operator*() { return v[worker_id()]; }
  T* operator->() { return &v[worker_id()]; }
  T& get() { return v[worker_id()]; }
  auto begin() { return v.begin(); }
  auto end() { return v.end(); }
};

namespace internal {
struct timer {
  using clk = std::chrono::steady_clock;
  std::string name; double total_ = 0; bool on = false; clk::time_point last;
  explicit timer(std::string n = "", bool start_now = true) : name(std::move(n)) { if (start_now) start(); }
  static double secs(clk::duration d) { return std::chrono::duration<double>(d).count(); }
  void start() { on = true; last = clk::now(); }
  double stop() { if (on) { auto t = clk::now(); total_ += secs(t - last); on = false; } return total_; }
  void reset() { total_ = 0; on = false; }
  double get_total() { if (on) { auto t = clk::now(); return total_ + secs(t - last); } return total_; }
  double next_time() { auto t = clk::now(); double d = secs(t - last); last = t; total_ += d; return d; }
  void next(const std::string& s) { double d = next_time(); std::cout << name << ": " << s << ": " << d << std::endl; }
  void total() { std::cout << name << ": " << get_total() << std::endl; }
  double total_time() { return get_total(); }
};
}  // namespace internal

namespace delayed {
template <typename R, typename F> auto map(R&& r, F f) {
  auto b = std::begin(r);
  using T = std::remove_cv_t<std::remove_reference_t<decltype(f(*b))>>;
  auto g = [b, f](long i) { return f(b[i]); };
  return delayed_sequence<T, decltype(g)>((long)r.size(), g);
}
template <typename R> auto flatten(R&& r) {
  using Inner = range_value_type_t<R>;
  using T = std::remove_cv_t<std::remove_reference_t<decltype(*std::begin(std::declval<Inner&>()))>>;
  sequence<T> s;
  for (auto it = std::begin(r); it != std::end(r); ++it) for (auto jt = std::begin(*it); jt != std::end(*it); ++jt) s.push_back(*jt);
  return s;
}
template <typename R> auto to_sequence(R&& r) { return parlay::to_sequence(r); }
}  // namespace delayed

}  // namespace parlay
