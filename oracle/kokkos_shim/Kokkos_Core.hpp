// Kokkos-compatible host shim used ONLY by the oracle (test infrastructure).
//
// It provides the small subset of the Kokkos 4.x API that the reference DGSEM
// headers use (View up to rank 7 with LayoutRight indexing, realloc,
// deep_copy, create_mirror_view, parallel_for over Range/MDRange policies,
// parallel_reduce, Array, initialize/finalize) so that the reference's own
// header-only solver can be compiled unmodified for the CPU, with optional
// OpenMP threading of the element loops.  None of the reference's numerics
// live here: every flux, integral and indicator is the reference's own code.
//
// This file is written for this project; it is not Kokkos source.
#pragma once

#include <Kokkos_Macros.hpp>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

namespace Kokkos {

struct HostSpace {};
struct OpenMP {
  using memory_space = HostSpace;
};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;

template <class ExecSpace, class MemSpace>
struct Device {
  using execution_space = ExecSpace;
  using memory_space = MemSpace;
};

struct LayoutRight {};

namespace impl_shim {
template <class T>
struct value_and_rank {
  using type = T;
  static constexpr std::size_t rank = 0;
};
template <class T>
struct value_and_rank<T*> {
  using type = typename value_and_rank<T>::type;
  static constexpr std::size_t rank = value_and_rank<T>::rank + 1;
};
}  // namespace impl_shim

// Reference-counted, LayoutRight (row-major) multidimensional array.
template <class DataType, class... Props>
class View {
 public:
  using value_type = typename impl_shim::value_and_rank<DataType>::type;
  using non_const_value_type = std::remove_const_t<value_type>;
  static constexpr std::size_t rank = impl_shim::value_and_rank<DataType>::rank;
  using HostMirror = View<DataType, Props...>;
  using memory_space = HostSpace;

  View() { ext_.fill(0); }

  template <class... Ints>
    requires(sizeof...(Ints) <= rank && (std::is_integral_v<Ints> && ...))
  explicit View(const std::string& label, Ints... n) : label_(label) {
    allocate(static_cast<std::size_t>(n)...);
  }

  template <class... Ints>
  void allocate(Ints... n) {
    ext_.fill(1);
    std::size_t dims[] = {static_cast<std::size_t>(n)..., 0};
    constexpr std::size_t given = sizeof...(Ints);
    for (std::size_t i = 0; i < rank; ++i) ext_[i] = (i < given) ? dims[i] : 1;
    std::size_t total = 1;
    for (std::size_t i = 0; i < rank; ++i) total *= ext_[i];
    data_ = std::shared_ptr<std::vector<non_const_value_type>>(
        new std::vector<non_const_value_type>(total, non_const_value_type{}));
    compute_strides();
  }

  std::size_t extent(std::size_t i) const { return i < rank ? ext_[i] : 1; }
  int extent_int(std::size_t i) const { return static_cast<int>(extent(i)); }
  std::size_t size() const {
    std::size_t total = 1;
    for (std::size_t i = 0; i < rank; ++i) total *= ext_[i];
    return total;
  }
  std::size_t span() const { return size(); }
  bool is_allocated() const { return static_cast<bool>(data_); }
  value_type* data() const { return data_ ? data_->data() : nullptr; }
  const std::string& label() const { return label_; }

  template <class... Idx>
    requires(sizeof...(Idx) == rank)
  KOKKOS_INLINE_FUNCTION value_type& operator()(Idx... idx) const {
    std::size_t ids[] = {static_cast<std::size_t>(idx)...};
    std::size_t off = 0;
    for (std::size_t i = 0; i < rank; ++i) off += ids[i] * stride_[i];
    return (*data_)[off];
  }

  value_type& operator[](std::size_t i) const
    requires(rank == 1)
  {
    return (*data_)[i];
  }

 private:
  void compute_strides() {
    std::size_t s = 1;
    for (std::size_t i = rank; i-- > 0;) {
      stride_[i] = s;
      s *= ext_[i];
    }
  }

  std::shared_ptr<std::vector<non_const_value_type>> data_;
  std::array<std::size_t, rank == 0 ? 1 : rank> ext_{};
  std::array<std::size_t, rank == 0 ? 1 : rank> stride_{};
  std::string label_;
};

template <class V, class... Ints>
void realloc(V& v, Ints... n) {
  V fresh(v.label().empty() ? std::string("realloc") : v.label(), n...);
  v = fresh;
}

template <class V>
  requires requires(V v) { V::rank; }
void deep_copy(const V& dst, const typename V::value_type& value) {
  auto* p = dst.data();
  const std::size_t n = dst.size();
  for (std::size_t i = 0; i < n; ++i) p[i] = value;
}

template <class VD, class VS>
  requires requires(VD d, VS s) {
    VD::rank;
    VS::rank;
  }
void deep_copy(const VD& dst, const VS& src) {
  if (dst.data() == src.data()) return;
  const std::size_t n = std::min(dst.size(), src.size());
  std::memmove(dst.data(), src.data(), n * sizeof(typename VD::value_type));
}

template <class V>
typename V::HostMirror create_mirror_view(const V& v) {
  return v;
}

template <class V>
typename V::HostMirror create_mirror_view_and_copy(const HostSpace&,
                                                   const V& v) {
  return v;
}

template <class T, std::size_t N>
struct Array {
  T m_internal_implementation_private_member_data[N > 0 ? N : 1];
  KOKKOS_INLINE_FUNCTION T& operator[](std::size_t i) {
    return m_internal_implementation_private_member_data[i];
  }
  KOKKOS_INLINE_FUNCTION const T& operator[](std::size_t i) const {
    return m_internal_implementation_private_member_data[i];
  }
  KOKKOS_INLINE_FUNCTION static constexpr std::size_t size() { return N; }
  T* data() { return m_internal_implementation_private_member_data; }
  const T* data() const { return m_internal_implementation_private_member_data; }
};

template <class... Args>
struct RangePolicy {
  std::int64_t begin = 0;
  std::int64_t end = 0;
  RangePolicy(std::int64_t b, std::int64_t e) : begin(b), end(e) {}
};

template <unsigned R>
struct Rank {
  static constexpr unsigned value = R;
};

template <class RankT, class... Args>
struct MDRangePolicy {
  static constexpr unsigned R = RankT::value;
  std::array<std::int64_t, R> lo{};
  std::array<std::int64_t, R> hi{};
  template <class A, class B>
  MDRangePolicy(std::initializer_list<A> l, std::initializer_list<B> h) {
    std::size_t i = 0;
    for (auto v : l) lo[i++] = static_cast<std::int64_t>(v);
    i = 0;
    for (auto v : h) hi[i++] = static_cast<std::int64_t>(v);
  }
};

template <class F>
void parallel_for(const std::string&, std::int64_t n, const F& f) {
#pragma omp parallel for schedule(static)
  for (std::int64_t i = 0; i < n; ++i) f(static_cast<std::size_t>(i));
}

template <class F, class... A>
void parallel_for(const std::string&, const RangePolicy<A...>& p, const F& f) {
#pragma omp parallel for schedule(static)
  for (std::int64_t i = p.begin; i < p.end; ++i) f(static_cast<std::size_t>(i));
}

template <class F, class... A>
void parallel_for(const std::string&, const MDRangePolicy<Rank<2>, A...>& p,
                  const F& f) {
  const std::int64_t n0 = p.hi[0] - p.lo[0];
  const std::int64_t n1 = p.hi[1] - p.lo[1];
#pragma omp parallel for schedule(static)
  for (std::int64_t t = 0; t < n0 * n1; ++t) {
    const std::size_t i = static_cast<std::size_t>(p.lo[0] + t / n1);
    const std::size_t j = static_cast<std::size_t>(p.lo[1] + t % n1);
    f(i, j);
  }
}

template <class F, class... A>
void parallel_for(const std::string&, const MDRangePolicy<Rank<3>, A...>& p,
                  const F& f) {
  const std::int64_t n0 = p.hi[0] - p.lo[0];
  const std::int64_t n1 = p.hi[1] - p.lo[1];
  const std::int64_t n2 = p.hi[2] - p.lo[2];
#pragma omp parallel for schedule(static)
  for (std::int64_t t = 0; t < n0 * n1 * n2; ++t) {
    const std::size_t i = static_cast<std::size_t>(p.lo[0] + t / (n1 * n2));
    const std::size_t j = static_cast<std::size_t>(p.lo[1] + (t / n2) % n1);
    const std::size_t k = static_cast<std::size_t>(p.lo[2] + t % n2);
    f(i, j, k);
  }
}

// Serial reductions (only the analyzers use these; they are not on the RHS).
template <class F, class Reducer>
void parallel_reduce(const std::string&, std::int64_t n, const F& f,
                     Reducer& r) {
  for (std::int64_t i = 0; i < n; ++i) f(static_cast<std::size_t>(i), r);
}

inline bool& shim_initialized_flag() {
  static bool flag = false;
  return flag;
}
inline void initialize() { shim_initialized_flag() = true; }
inline void initialize(int&, char**) { shim_initialized_flag() = true; }
inline void finalize() { shim_initialized_flag() = false; }
inline bool is_initialized() { return shim_initialized_flag(); }
inline void fence() {}

template <class T>
KOKKOS_INLINE_FUNCTION T abs(T x) {
  return std::abs(x);
}
template <class T>
KOKKOS_INLINE_FUNCTION T log(T x) {
  return std::log(x);
}
template <class T>
KOKKOS_INLINE_FUNCTION bool isnan(T x) {
  return std::isnan(x);
}

}  // namespace Kokkos
