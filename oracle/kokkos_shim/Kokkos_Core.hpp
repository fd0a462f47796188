// Project-written stand-in for the subset of the Kokkos API that the Chasqui reference uses,
// so that the reference's unmodified headers compile with plain g++ + OpenMP into a CPU
// oracle. This is NOT Kokkos: it implements only what the reference calls
//   View<T*|T***|T****, LayoutRight> (ref-counted, zero-initialised host buffers),
//   create_mirror / create_mirror_view / create_mirror_view_and_copy / deep_copy,
//   MDRangePolicy<ExecSpace, Rank<3, Right, Right>> over {lo}..{hi},
//   parallel_for, parallel_reduce with plain sums, Min<T>, Max<T> and the variadic
//   multi-reducer form, fence, ScopeGuard, DefaultExecutionSpace::name().
// Schedules are static so that results are reproducible run to run; min/max reductions are
// order independent, floating-point sums are combined in thread order.
//
// Test infrastructure only: nothing in the product links this file.
#pragma once
#include <omp.h>
#include <array>
#include <cfloat>
#include <climits>
#include <cstddef>
#include <cstring>
#include <initializer_list>
#include <limits>
#include <memory>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]

namespace Kokkos {

struct LayoutRight {};
struct HostSpace {};
struct OpenMP {
  static const char *name() { return "OpenMP (project Kokkos-API shim)"; }
};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;

inline void fence() {}

struct ScopeGuard {
  template <class... A>
  explicit ScopeGuard(A &&...) {}
};

// ---------------------------------------------------------------------------------------
// View: rank deduced from the number of '*' in T; storage is contiguous LayoutRight.
template <class T> struct ViewTraits;
template <class T> struct ViewTraits<T *> { using value = T; static constexpr int rank = 1; };
template <class T> struct ViewTraits<T **> { using value = T; static constexpr int rank = 2; };
template <class T> struct ViewTraits<T ***> { using value = T; static constexpr int rank = 3; };
template <class T> struct ViewTraits<T ****> { using value = T; static constexpr int rank = 4; };

template <class DataType, class Layout = LayoutRight>
class View {
 public:
  using value_type = typename ViewTraits<DataType>::value;
  static constexpr int rank = ViewTraits<DataType>::rank;
  using HostMirror = View<DataType, Layout>;

  View() = default;
  template <class... N>
  explicit View(const std::string &label, N... n) : label_(label) {
    static_assert(sizeof...(N) == rank, "wrong number of extents");
    const size_t e[] = {static_cast<size_t>(n)...};
    size_t total = 1;
    for (int r = 0; r < rank; ++r) { ext_[r] = e[r]; total *= e[r]; }
    for (int r = rank - 1, s = 1; r >= 0; --r) { str_[r] = s; s *= static_cast<int>(ext_[r]); }
    size_ = total;
    buf_ = std::shared_ptr<value_type[]>(new value_type[total]());   // zero-initialised
    ptr_ = buf_.get();
  }

  inline value_type &operator()(int i0) const { return ptr_[i0]; }
  inline value_type &operator()(int i0, int i1) const { return ptr_[(size_t)i0 * str_[0] + i1]; }
  inline value_type &operator()(int i0, int i1, int i2) const {
    return ptr_[((size_t)i0 * ext_[1] + i1) * ext_[2] + i2];
  }
  inline value_type &operator()(int i0, int i1, int i2, int i3) const {
    return ptr_[(((size_t)i0 * ext_[1] + i1) * ext_[2] + i2) * ext_[3] + i3];
  }
  value_type *data() const { return ptr_; }
  size_t size() const { return size_; }
  size_t span() const { return size_; }
  size_t extent(int r) const { return ext_[r]; }
  const std::string &label() const { return label_; }

 private:
  std::shared_ptr<value_type[]> buf_;
  value_type *ptr_ = nullptr;
  size_t ext_[4] = {0, 0, 0, 0};
  int str_[4] = {0, 0, 0, 0};
  size_t size_ = 0;
  std::string label_;
};

template <class V> V create_mirror(const HostSpace &, const V &v) {
  V m = v;
  // a mirror made by create_mirror always owns fresh storage of the same shape
  if constexpr (V::rank == 1) m = V(v.label() + "_mirror", v.extent(0));
  else if constexpr (V::rank == 2) m = V(v.label() + "_mirror", v.extent(0), v.extent(1));
  else if constexpr (V::rank == 3) m = V(v.label() + "_mirror", v.extent(0), v.extent(1), v.extent(2));
  else m = V(v.label() + "_mirror", v.extent(0), v.extent(1), v.extent(2), v.extent(3));
  return m;
}
template <class V> V create_mirror(const V &v) { return create_mirror(HostSpace(), v); }
// host execution space: the mirror view aliases the original
template <class V> V create_mirror_view(const V &v) { return v; }
template <class V> V create_mirror_view(const HostSpace &, const V &v) { return v; }
template <class V> V create_mirror_view_and_copy(const HostSpace &, const V &v) { return v; }

template <class V>
void deep_copy(const V &dst, const V &src) {
  if (dst.data() == src.data()) return;
  std::memcpy(dst.data(), src.data(), dst.size() * sizeof(typename V::value_type));
}

// ---------------------------------------------------------------------------------------
namespace Iterate { struct Right {}; struct Left {}; }
template <int N, class Outer = Iterate::Right, class Inner = Iterate::Right> struct Rank {};

template <class Exec, class RankT>
struct MDRangePolicy {
  std::array<long, 3> lo{}, hi{};
  MDRangePolicy(std::initializer_list<long> l, std::initializer_list<long> h) {
    std::copy(l.begin(), l.end(), lo.begin());
    std::copy(h.begin(), h.end(), hi.begin());
  }
};

template <class Exec, class RankT, class F>
void parallel_for(const std::string &, const MDRangePolicy<Exec, RankT> &p, const F &f) {
  const long k0 = p.lo[0], k1 = p.hi[0], j0 = p.lo[1], j1 = p.hi[1], i0 = p.lo[2], i1 = p.hi[2];
  if (k1 <= k0 || j1 <= j0 || i1 <= i0) return;
#pragma omp parallel for collapse(2) schedule(static)
  for (long k = k0; k < k1; ++k)
    for (long j = j0; j < j1; ++j)
      for (long i = i0; i < i1; ++i) f(static_cast<int>(k), static_cast<int>(j), static_cast<int>(i));
}

// ---------------------------------------------------------------------------------------
// Reducers. A plain scalar argument means a sum into that scalar.
template <class T> struct Min {
  T &ref;
  explicit Min(T &r) : ref(r) {}
  static T identity() { return std::numeric_limits<T>::max(); }
  static void join(T &a, const T &b) { if (b < a) a = b; }
};
template <class T> struct Max {
  T &ref;
  explicit Max(T &r) : ref(r) {}
  static T identity() { return std::numeric_limits<T>::lowest(); }
  static void join(T &a, const T &b) { if (b > a) a = b; }
};
template <class T> struct SumRef {
  T &ref;
  static T identity() { return T(0); }
  static void join(T &a, const T &b) { a += b; }
};

namespace detail {
template <class R> struct AsReducer { using type = SumRef<R>; static type make(R &r) { return type{r}; } };
template <class T> struct AsReducer<Min<T>> { using type = Min<T>; static type make(Min<T> &r) { return r; } };
template <class T> struct AsReducer<Max<T>> { using type = Max<T>; static type make(Max<T> &r) { return r; } };
template <class R> struct ValueOf { using type = R; };
template <class T> struct ValueOf<Min<T>> { using type = T; };
template <class T> struct ValueOf<Max<T>> { using type = T; };
}  // namespace detail

template <class Exec, class RankT, class F, class... R>
void parallel_reduce(const std::string &, const MDRangePolicy<Exec, RankT> &p, const F &f, R &&...rs) {
  using Tup = std::tuple<typename detail::ValueOf<std::remove_reference_t<R>>::type...>;
  auto reducers = std::make_tuple(detail::AsReducer<std::remove_reference_t<R>>::make(rs)...);
  constexpr size_t NR = sizeof...(R);
  const long k0 = p.lo[0], k1 = p.hi[0], j0 = p.lo[1], j1 = p.hi[1], i0 = p.lo[2], i1 = p.hi[2];
  const int nth = omp_get_max_threads();
  std::vector<Tup> part(nth);
  auto init = [&](Tup &t) {
    [&]<size_t... I>(std::index_sequence<I...>) {
      ((std::get<I>(t) = std::tuple_element_t<I, decltype(reducers)>::identity()), ...);
    }(std::make_index_sequence<NR>{});
  };
  for (auto &t : part) init(t);
#pragma omp parallel num_threads(nth)
  {
    Tup &loc = part[omp_get_thread_num()];
#pragma omp for collapse(2) schedule(static)
    for (long k = k0; k < k1; ++k)
      for (long j = j0; j < j1; ++j)
        for (long i = i0; i < i1; ++i)
          std::apply([&](auto &...v) { f(static_cast<int>(k), static_cast<int>(j), static_cast<int>(i), v...); }, loc);
  }
  Tup tot;
  init(tot);
  for (int t = 0; t < nth; ++t) {
    [&]<size_t... I>(std::index_sequence<I...>) {
      (std::tuple_element_t<I, decltype(reducers)>::join(std::get<I>(tot), std::get<I>(part[t])), ...);
    }(std::make_index_sequence<NR>{});
  }
  [&]<size_t... I>(std::index_sequence<I...>) {
    ((std::get<I>(reducers).ref = std::get<I>(tot)), ...);
  }(std::make_index_sequence<NR>{});
}

}  // namespace Kokkos
