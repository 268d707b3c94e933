/*
 * Kokkos_Core.hpp — project-written stand-in for the subset of the Kokkos 4.5 API that CLEO's
 * hot-path sources use (TEST INFRASTRUCTURE ONLY: it exists so that the reference's own
 * translation units compile unmodified into the oracle's reference build).
 *
 * Semantics: host memory only. Team policies run one league rank after another on one thread
 * (team size 1), or, when kokkos_shim::set_num_threads(n > 1), spread league ranks over OpenMP
 * threads. Nested TeamThreadRange loops run sequentially in index order. Random pools hand out
 * the injected counter-based stream of include/cleo_b200_rng.h keyed by (pool seed, the SDM step
 * set with kokkos_shim::set_rng_time, the league rank of the enclosing team policy, the draw
 * number inside that league rank). Kokkos::abort throws kokkos_shim::Abort.
 */
#ifndef CLEO_KOKKOS_SHIM_CORE_HPP_
#define CLEO_KOKKOS_SHIM_CORE_HPP_

#include <algorithm>
#include <atomic>
#include <tuple>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <numbers>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../../include/cleo_b200_rng.h"

#define KOKKOS_FUNCTION
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [ =, *this ]

namespace kokkos_shim {

struct Abort : std::runtime_error {
  explicit Abort(const char* m) : std::runtime_error(m) {}
};

inline int& num_threads() {
  static int n = 1;
  return n;
}
inline void set_num_threads(int n) { num_threads() = n < 1 ? 1 : n; }

/* injected random stream context */
inline uint32_t& rng_time() {
  static uint32_t t = 0;
  return t;
}
inline void set_rng_time(uint32_t t) { rng_time() = t; }
struct RngCtx {
  uint64_t league = 0;
  uint64_t slot = 0;
};
inline RngCtx& rng_ctx() {
  static thread_local RngCtx c;
  return c;
}

}  // namespace kokkos_shim

namespace Kokkos {

/* ---------------------------------------------------------------- spaces, pair, misc */
struct HostSpace {};
struct LayoutRight {};
struct LayoutLeft {};
struct Serial {
  using memory_space = HostSpace;
  using execution_space = Serial;
  using array_layout = LayoutRight;
};
using DefaultExecutionSpace = Serial;
using DefaultHostExecutionSpace = Serial;

struct InitializationSettings {
  template <class T>
  InitializationSettings& set_num_threads(T) { return *this; }
  template <class T>
  InitializationSettings& set_device_id(T) { return *this; }
};
inline void initialize(...) {}
inline void finalize() {}
inline bool is_initialized() { return true; }
inline void fence(...) {}

template <class T1, class T2>
struct pair {
  using first_type = T1;
  using second_type = T2;
  T1 first;
  T2 second;
  constexpr pair() = default;
  constexpr pair(const T1& a, const T2& b) : first(a), second(b) {}
  template <class U1, class U2>
  constexpr pair(const pair<U1, U2>& o) : first(o.first), second(o.second) {}
  template <class U1, class U2>
  constexpr pair(const std::pair<U1, U2>& o) : first(o.first), second(o.second) {}
};
template <class T1, class T2>
constexpr pair<T1, T2> make_pair(T1 a, T2 b) {
  return pair<T1, T2>(a, b);
}

[[noreturn]] inline void abort(const char* msg) { throw kokkos_shim::Abort(msg); }

namespace numbers {
inline constexpr double pi = std::numbers::pi;
}

/* ---------------------------------------------------------------- math */
inline double pow(double a, double b) { return std::pow(a, b); }
inline double exp(double a) { return std::exp(a); }
inline double sqrt(double a) { return std::sqrt(a); }
inline double floor(double a) { return std::floor(a); }
inline double round(double a) { return std::round(a); }
inline double log(double a) { return std::log(a); }
inline double tanh(double a) { return std::tanh(a); }
inline double abs(double a) { return std::fabs(a); }
template <class A, class B>
inline double fmin(A a, B b) {
  return std::fmin(static_cast<double>(a), static_cast<double>(b));
}
template <class A, class B>
inline double fmax(A a, B b) {
  return std::fmax(static_cast<double>(a), static_cast<double>(b));
}
template <class T>
constexpr const T& min(const T& a, const T& b) {
  return (b < a) ? b : a;
}
template <class T>
constexpr const T& max(const T& a, const T& b) {
  return (a < b) ? b : a;
}

template <class T>
inline T atomic_fetch_add(T* p, T v) {
  return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}
template <class T, class U>
inline T atomic_fetch_add(T* p, U v) {
  return __atomic_fetch_add(p, static_cast<T>(v), __ATOMIC_RELAXED);
}
template <class T, class U>
inline void atomic_add(T* p, U v) {  // integer or floating point
  std::atomic_ref<T>(*p).fetch_add(static_cast<T>(v), std::memory_order_relaxed);
}

/* ---------------------------------------------------------------- views */
template <class DataType>
struct ViewTraits;
template <class T>
struct ViewTraits<T*> {
  using value_type = T;
  using non_const_data_type = std::remove_const_t<T>*;
  static constexpr size_t static_extent = 0;
};
template <class T, size_t N>
struct ViewTraits<T[N]> {
  using value_type = T;
  using non_const_data_type = std::remove_const_t<T>[N];
  static constexpr size_t static_extent = N;
};

template <class DataType, class... Props>
class View {
 public:
  using traits = ViewTraits<DataType>;
  using value_type = typename traits::value_type;
  using non_const_value_type = std::remove_const_t<value_type>;
  using pointer_type = value_type*;
  using reference_type = value_type&;
  /* as in Kokkos, a host mirror holds non-const data (here: the same memory) */
  using HostMirror = View<typename traits::non_const_data_type>;
  using memory_space = HostSpace;
  using execution_space = Serial;

  View() = default;
  explicit View(const std::string& /*label*/, size_t n = traits::static_extent) { allocate(n); }
  View(const char* label, size_t n = traits::static_extent) : View(std::string(label), n) {}
  View(value_type* p, size_t n) : ptr_(p), n_(n) {}
  /* const conversion View<T*> -> View<const T*> */
  template <class D2, class... P2,
            class = std::enable_if_t<std::is_convertible_v<typename View<D2, P2...>::pointer_type,
                                                           pointer_type> &&
                                     !std::is_same_v<View<D2, P2...>, View>>>
  View(const View<D2, P2...>& o) : own_(o.owner()), ptr_(o.data()), n_(o.extent(0)) {}

  reference_type operator()(size_t i) const { return ptr_[i]; }
  reference_type operator[](size_t i) const { return ptr_[i]; }
  pointer_type data() const { return ptr_; }
  size_t extent(size_t d) const { return d == 0 ? n_ : 1; }
  size_t size() const { return n_; }
  size_t span() const { return n_; }
  bool is_allocated() const { return ptr_ != nullptr; }
  const std::shared_ptr<void>& owner() const { return own_; }
  std::string label() const { return ""; }
  void reallocate(size_t n) { allocate(n); }  // contents not kept (Kokkos::realloc)
  HostMirror mirror_alias() const {
    HostMirror m;
    m.own_ = own_;
    m.ptr_ = const_cast<non_const_value_type*>(ptr_);
    m.n_ = n_;
    return m;
  }

 private:
  void allocate(size_t n) {
    auto buf = std::shared_ptr<non_const_value_type[]>(new non_const_value_type[n ? n : 1]());
    own_ = std::shared_ptr<void>(buf, buf.get());
    ptr_ = buf.get();
    n_ = n;
  }
  std::shared_ptr<void> own_;
  pointer_type ptr_ = nullptr;
  size_t n_ = 0;

  template <class D, class... P>
  friend class View;
};

template <class D, class... P>
void realloc(View<D, P...>& v, size_t n) {
  v.reallocate(n);
}

/* Subview of a 1-D view by an index range is a 1-D view of the same type. */
template <class V, class... Args>
using Subview = V;

template <class D, class... P, class I>
View<D, P...> subview(const View<D, P...>& v, const pair<I, I>& r) {
  View<D, P...> s(v.data() + r.first, static_cast<size_t>(r.second - r.first));
  return s;
}
template <class D, class... P, class I>
View<D, P...> subview(const View<D, P...>& v, const std::pair<I, I>& r) {
  return subview(v, pair<I, I>(r.first, r.second));
}

/* host mirrors: host memory is the only memory, so a mirror aliases the view's data */
template <class V>
typename V::HostMirror create_mirror_view(const V& v) {
  return v.mirror_alias();
}
template <class S, class V>
typename V::HostMirror create_mirror_view(const S&, const V& v) {
  return v.mirror_alias();
}
template <class S, class V>
typename V::HostMirror create_mirror_view_and_copy(const S&, const V& v) {
  return v.mirror_alias();
}
template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  if (dst.data() == src.data()) return;
  for (size_t i = 0; i < src.extent(0); ++i) dst(i) = src(i);
}
template <class D1, class... P1>
void deep_copy(const View<D1, P1...>& dst, const typename View<D1, P1...>::non_const_value_type& v) {
  for (size_t i = 0; i < dst.extent(0); ++i) dst(i) = v;
}

template <class DataType, class... Props>
class DualView {
 public:
  using t_dev = View<DataType>;
  using t_host = View<DataType>;
  DualView() = default;
  DualView(const std::string& label, size_t n) : v_(label, n) {}
  t_dev view_device() const { return v_; }
  t_host view_host() const { return v_; }
  template <class S>
  View<DataType> view() const {
    return v_;
  }
  void modify_host() const {}
  void modify_device() const {}
  void sync_host() const {}
  void sync_device() const {}
  template <class S>
  void sync() const {}
  template <class S>
  void modify() const {}
  size_t extent(size_t d) const { return v_.extent(d); }
  t_dev h_view_() const { return v_; }

 private:
  View<DataType> v_;
};

/* ---------------------------------------------------------------- execution policies */
struct AUTO_t {
  constexpr const AUTO_t& operator()() const { return *this; }
};
inline constexpr AUTO_t AUTO = AUTO_t();

template <class ExecSpace = Serial>
struct RangePolicy {
  size_t begin_, end_;
  RangePolicy(size_t b, size_t e) : begin_(b), end_(e) {}
};

struct TeamMemberImpl {
  size_t league_rank_ = 0;
  size_t league_size_ = 0;
  size_t league_rank() const { return league_rank_; }
  size_t league_size() const { return league_size_; }
  int team_rank() const { return 0; }
  int team_size() const { return 1; }
  void team_barrier() const {}
};

template <class ExecSpace = Serial>
struct TeamPolicy {
  using member_type = TeamMemberImpl;
  size_t league_size;
  TeamPolicy(size_t n, AUTO_t) : league_size(n) {}
  TeamPolicy(size_t n, int) : league_size(n) {}
};

template <class M>
struct TeamThreadRangeBoundaries {
  const M& member;
  size_t begin_, end_;
};
template <class M, class I>
TeamThreadRangeBoundaries<M> TeamThreadRange(const M& m, I n) {
  return {m, 0, static_cast<size_t>(n)};
}
template <class M, class I>
TeamThreadRangeBoundaries<M> TeamThreadRange(const M& m, I b, I e) {
  return {m, static_cast<size_t>(b), static_cast<size_t>(e)};
}
template <class M>
struct ThreadVectorRangeBoundaries {
  const M& member;
  size_t begin_, end_;
};
template <class M, class I>
ThreadVectorRangeBoundaries<M> ThreadVectorRange(const M& m, I n) {
  return {m, 0, static_cast<size_t>(n)};
}

template <class M>
struct PerTeamTag {
  const M& member;
};
template <class M>
PerTeamTag<M> PerTeam(const M& m) {
  return {m};
}
template <class M, class F>
void single(const PerTeamTag<M>&, const F& f) {
  f();
}
template <class M, class F, class T>
void single(const PerTeamTag<M>&, const F& f, T& v) {
  f(v);
}

/* logical-or reducer */
template <class T>
struct LOr {
  T& ref;
  explicit LOr(T& r) : ref(r) {}
};

namespace detail {
template <class Body>
void league_loop(size_t n, const Body& body) {
  auto run = [&](size_t ii) {
    auto& ctx = kokkos_shim::rng_ctx();
    ctx.league = ii;
    ctx.slot = 0;
    TeamMemberImpl tm{ii, n};
    body(tm);
  };
#ifdef _OPENMP
  if (kokkos_shim::num_threads() > 1) {
    std::exception_ptr err = nullptr;
#pragma omp parallel for schedule(dynamic, 64) num_threads(kokkos_shim::num_threads())
    for (long long ii = 0; ii < (long long)n; ++ii) {
      try {
        run((size_t)ii);
      } catch (...) {
#pragma omp critical
        if (!err) err = std::current_exception();
      }
    }
    if (err) std::rethrow_exception(err);
    return;
  }
#endif
  for (size_t ii = 0; ii < n; ++ii) run(ii);
}
template <class Body>
void range_loop(size_t b, size_t e, const Body& body) {
#ifdef _OPENMP
  if (kokkos_shim::num_threads() > 1) {
    std::exception_ptr err = nullptr;
#pragma omp parallel for schedule(static) num_threads(kokkos_shim::num_threads())
    for (long long i = (long long)b; i < (long long)e; ++i) {
      try {
        body((size_t)i);
      } catch (...) {
#pragma omp critical
        if (!err) err = std::current_exception();
      }
    }
    if (err) std::rethrow_exception(err);
    return;
  }
#endif
  for (size_t i = b; i < e; ++i) body(i);
}
}  // namespace detail

/* parallel_for */
template <class E, class F>
void parallel_for(const std::string&, const RangePolicy<E>& p, const F& f) {
  detail::range_loop(p.begin_, p.end_, [&](size_t i) { f(i); });
}
template <class E, class F>
void parallel_for(const RangePolicy<E>& p, const F& f) {
  parallel_for(std::string(), p, f);
}
template <class E, class F>
void parallel_for(const std::string&, const TeamPolicy<E>& p, const F& f) {
  detail::league_loop(p.league_size, [&](const TeamMemberImpl& tm) { f(tm); });
}
template <class E, class F>
void parallel_for(const TeamPolicy<E>& p, const F& f) {
  parallel_for(std::string(), p, f);
}
template <class F, class I, class = std::enable_if_t<std::is_integral_v<I>>>
void parallel_for(const std::string&, I n, const F& f) {
  for (I i = 0; i < n; ++i) f(i);
}
template <class M, class F>
void parallel_for(const TeamThreadRangeBoundaries<M>& r, const F& f) {
  for (size_t i = r.begin_; i < r.end_; ++i) f(i);
}
template <class M, class F>
void parallel_for(const ThreadVectorRangeBoundaries<M>& r, const F& f) {
  for (size_t i = r.begin_; i < r.end_; ++i) f(i);
}

/* parallel_reduce */
template <class M, class F, class T>
void parallel_reduce(const TeamThreadRangeBoundaries<M>& r, const F& f, T& result) {
  T acc = T{};
  for (size_t i = r.begin_; i < r.end_; ++i) f(i, acc);
  result = acc;
}
/* several sum reductions at once, accumulated in index order */
template <class M, class F, class T1, class T2, class... Ts>
void parallel_reduce(const TeamThreadRangeBoundaries<M>& r, const F& f, T1& r1, T2& r2,
                     Ts&... rs) {
  T1 a1{};
  T2 a2{};
  std::tuple<Ts...> as{};
  for (size_t i = r.begin_; i < r.end_; ++i)
    std::apply([&](auto&... a) { f(i, a1, a2, a...); }, as);
  r1 = a1;
  r2 = a2;
  std::apply([&](auto&... a) { ((rs = a), ...); }, as);
}
template <class E, class F>
void parallel_reduce(const std::string&, const TeamPolicy<E>& p, const F& f, const LOr<bool>& red) {
  std::atomic<bool> any{false};
  detail::league_loop(p.league_size, [&](const TeamMemberImpl& tm) {
    bool upd = false;
    f(tm, upd);
    if (upd) any.store(true);
  });
  red.ref = any.load();
}

/* ---------------------------------------------------------------- random */
template <class DeviceType>
struct Random_XorShift64 {
  uint64_t seed = 0;
  uint64_t next_u64() {
    auto& ctx = kokkos_shim::rng_ctx();
    const uint64_t key = cleo_rng_key(seed, kokkos_shim::rng_time(), (uint32_t)ctx.league);
    return cleo_rng_u64(key, ctx.slot++);
  }
  uint64_t urand(uint64_t start, uint64_t end) {
    return cleo_rng_range(next_u64(), start, end);
  }
  uint64_t urand64(uint64_t start, uint64_t end) { return urand(start, end); }
  double drand(double start, double end) {
    return start + (end - start) * cleo_rng_to_unit(next_u64());
  }
  double drand() { return cleo_rng_to_unit(next_u64()); }
};
template <class DeviceType>
struct Random_XorShift64_Pool {
  uint64_t seed = 0;
  Random_XorShift64_Pool() = default;
  explicit Random_XorShift64_Pool(uint64_t s) : seed(s) {}
  Random_XorShift64<DeviceType> get_state() const { return Random_XorShift64<DeviceType>{seed}; }
  void free_state(const Random_XorShift64<DeviceType>&) const {}
};

/* ---------------------------------------------------------------- unordered map */
template <class K, class V>
struct UnorderedMapStore {
  std::vector<K> keys;
  std::vector<V> vals;
  std::vector<unsigned char> used;
  size_t mask = 0;
  size_t count = 0;
};

template <class K, class V, class Space = Serial>
class UnorderedMap {
  using Store = UnorderedMapStore<K, V>;

 public:
  using HostMirror = UnorderedMap<K, V, HostSpace>;
  static constexpr uint32_t invalid_index = ~0u;
  UnorderedMap() : UnorderedMap(0) {}
  explicit UnorderedMap(size_t capacity) : s_(std::make_shared<Store>()) {
    size_t cap = 16;
    while (cap < 2 * capacity + 2) cap <<= 1;
    s_->keys.resize(cap);
    s_->vals.resize(cap);
    s_->used.assign(cap, 0);
    s_->mask = cap - 1;
  }
  template <class S2>
  UnorderedMap(const UnorderedMap<K, V, S2>& o) : s_(o.store()) {}

  static size_t hash(const K& k) {
    uint64_t z = (uint64_t)k;
    return (size_t)cleo_mix64(z + 0x9E3779B97F4A7C15ull);
  }
  struct insert_result {
    bool ok;
    bool success() const { return ok; }
    bool failed() const { return !ok; }
    bool existing() const { return false; }
  };
  insert_result insert(const K& k, const V& v) const {
    size_t i = hash(k) & s_->mask;
    for (size_t probe = 0; probe <= s_->mask; ++probe) {
      if (!s_->used[i]) {
        s_->used[i] = 1;
        s_->keys[i] = k;
        s_->vals[i] = v;
        s_->count++;
        return {true};
      }
      if (s_->keys[i] == k) {
        s_->vals[i] = v;
        return {true};
      }
      i = (i + 1) & s_->mask;
    }
    return {false};
  }
  uint32_t find(const K& k) const {
    size_t i = hash(k) & s_->mask;
    for (size_t probe = 0; probe <= s_->mask; ++probe) {
      if (!s_->used[i]) return invalid_index;
      if (s_->keys[i] == k) return (uint32_t)i;
      i = (i + 1) & s_->mask;
    }
    return invalid_index;
  }
  bool exists(const K& k) const { return find(k) != invalid_index; }
  bool valid_at(uint32_t i) const { return i != invalid_index && s_->used[i]; }
  const V& value_at(uint32_t i) const { return s_->vals[i]; }
  const K& key_at(uint32_t i) const { return s_->keys[i]; }
  size_t size() const { return s_->count; }
  size_t capacity() const { return s_->mask + 1; }
  template <class S2>
  void create_copy_view(const UnorderedMap<K, V, S2>& src) {
    s_ = std::make_shared<Store>(*src.store());
  }
  const std::shared_ptr<Store>& store() const { return s_; }

 private:
  std::shared_ptr<Store> s_;
  template <class, class, class>
  friend class UnorderedMap;
};

/* ---------------------------------------------------------------- std-algorithms, sort, scatter */
namespace Experimental {
template <class D, class... P>
auto begin(const View<D, P...>& v) {
  return v.data();
}
template <class D, class... P>
auto end(const View<D, P...>& v) {
  return v.data() + v.extent(0);
}
template <class It>
auto distance(It a, It b) {
  return b - a;
}
template <class M, class D, class... P, class Pred>
bool all_of(const M&, const View<D, P...>& v, Pred pred) {
  return std::all_of(v.data(), v.data() + v.extent(0), pred);
}
template <class M, class D, class... P, class Pred>
bool none_of(const M&, const View<D, P...>& v, Pred pred) {
  return std::none_of(v.data(), v.data() + v.extent(0), pred);
}
template <class E, class D, class... P, class Comp>
bool is_sorted(const std::string&, const E&, const View<D, P...>& v, Comp comp) {
  return std::is_sorted(v.data(), v.data() + v.extent(0), comp);
}
template <class E, class D1, class... P1, class D2, class... P2, class T>
void exclusive_scan(const std::string&, const E&, const View<D1, P1...>& in,
                    const View<D2, P2...>& out, T init) {
  auto acc = static_cast<typename View<D2, P2...>::non_const_value_type>(init);
  for (size_t i = 0; i < in.extent(0); ++i) {
    const auto v = in(i);
    out(i) = acc;
    acc += v;
  }
}
template <class E, class D, class... P, class T>
void fill(const E&, const View<D, P...>& v, T val) {
  for (size_t i = 0; i < v.extent(0); ++i) v(i) = val;
}
/* sort_team: stable sort (Kokkos' bitonic team sort leaves equal keys in unspecified order) */
template <class M, class D, class... P, class Comp>
void sort_team(const M&, const View<D, P...>& v, Comp comp) {
  std::stable_sort(v.data(), v.data() + v.extent(0), comp);
}

template <class T>
struct AtomicIncRef {
  T* p;
  AtomicIncRef& operator++() {
    __atomic_fetch_add(p, (T)1, __ATOMIC_RELAXED);
    return *this;
  }
  AtomicIncRef& operator+=(T v) {
    __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
    return *this;
  }
};
template <class DataType, class... Props>
class ScatterView {
 public:
  using value_type = typename View<DataType>::non_const_value_type;
  ScatterView() = default;
  explicit ScatterView(const View<DataType>& v) : v_(v) {}
  struct Access {
    View<DataType> v;
    AtomicIncRef<value_type> operator()(size_t i) const { return {&v(i)}; }
  };
  Access access() const { return Access{v_}; }
  void reset() {}
  void reset_except(const View<DataType>&) {}
  const View<DataType>& subview() const { return v_; }

 private:
  View<DataType> v_;
};
template <class D, class... P, class S>
void contribute(const View<D, P...>&, const S&) {}
}  // namespace Experimental

/* ---------------------------------------------------------------- profiling */
namespace Profiling {
inline void pushRegion(const std::string&) {}
inline void popRegion() {}
struct ScopedRegion {
  explicit ScopedRegion(const std::string&) {}
};
}  // namespace Profiling

struct Timer {
  double seconds() const { return 0.0; }
  void reset() {}
};

}  // namespace Kokkos

#endif  // CLEO_KOKKOS_SHIM_CORE_HPP_
