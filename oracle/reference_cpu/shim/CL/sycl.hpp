// TEST INFRASTRUCTURE ONLY.
//
// A host-only stand-in for the subset of SYCL 2020 that the reference's
// time-step modules use, so that their unmodified sources compile with g++
// and run on the CPU: queue::submit / parallel_for / memcpy / memset,
// handler::parallel_for (with and without a sum reduction), range, id, item,
// event, and the USM allocators.  Semantics follow the SYCL 2020
// specification for a device that executes synchronously:
//  * parallel_for(range<N>(d0, .., d{N-1}), f) calls f once per work item,
//    with item[0] the slowest index and get_linear_id() = row-major index;
//    the work items are spread over OpenMP threads (SYCL kernels carry no
//    ordering between items, so the reference's kernels are race-free under
//    any schedule);
//  * a reduction with sycl::plus combines each thread's partial sum in
//    thread order and adds it to the value the pointer held (SYCL 2020
//    reductions combine with the initial value); the reference leaves the
//    order of the terms to the implementation;
//  * every operation completes before it returns, so events are empty;
//  * malloc_shared / malloc_host / malloc_device are host allocations.
#pragma once

#include <omp.h>

#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <initializer_list>
#include <tuple>
#include <type_traits>
#include <vector>

namespace sycl {

template <int N>
struct range {
  size_t v[N];
  template <class... I,
            std::enable_if_t<sizeof...(I) == N && (std::is_integral_v<I> && ...), int> = 0>
  range(I... d) : v{static_cast<size_t>(d)...} {}
  size_t operator[](int d) const { return v[d]; }
  size_t size() const {
    size_t n = 1;
    for (int d = 0; d < N; ++d) n *= v[d];
    return n;
  }
};
template <class A>
range(A)->range<1>;
template <class A, class B>
range(A, B)->range<2>;
template <class A, class B, class C>
range(A, B, C)->range<3>;

template <int N>
struct id {
  size_t v[N];
  size_t operator[](int d) const { return v[d]; }
};

template <int N>
struct item {
  size_t v[N];
  range<N> r;
  size_t operator[](int d) const { return v[d]; }
  range<N> get_range() const { return r; }
  size_t get_range(int d) const { return r[d]; }
  id<N> get_id() const {
    id<N> i;
    for (int d = 0; d < N; ++d) i.v[d] = v[d];
    return i;
  }
  operator id<N>() const { return get_id(); }
  size_t get_linear_id() const {
    size_t l = 0;
    for (int d = 0; d < N; ++d) l = l * r[d] + v[d];
    return l;
  }
};

class event {
 public:
  void wait() {}
  static void wait(const std::vector<event> &) {}
};

template <class T = void>
struct plus {
  T operator()(const T &a, const T &b) const { return a + b; }
};
template <>
struct plus<void> {
  template <class T>
  T operator()(const T &a, const T &b) const {
    return a + b;
  }
};

template <class T, class Op>
struct reduction_spec {
  T *target;
  Op op;
};
template <class T, class Op>
reduction_spec<T, Op> reduction(T *target, Op op) {
  return reduction_spec<T, Op>{target, op};
}

template <class T, class Op>
struct reducer {
  T value;
  Op op;
  reducer &operator+=(const T &x) {
    value = op(value, x);
    return *this;
  }
  void combine(const T &x) { value = op(value, x); }
};

namespace detail {

// Calls f(item) for every work item of r; rows of the slowest one (1-D, 2-D)
// or two (3-D) dimensions are distributed over the OpenMP threads.
template <int N, class F>
void run(const range<N> &r, F &f) {
  if constexpr (N == 1) {
    const long long n0 = (long long)r[0];
#pragma omp parallel for schedule(static)
    for (long long a = 0; a < n0; ++a) f(item<1>{{(size_t)a}, r});
  } else if constexpr (N == 2) {
    const long long n0 = (long long)r[0], n1 = (long long)r[1];
#pragma omp parallel for schedule(static)
    for (long long a = 0; a < n0; ++a)
      for (long long b = 0; b < n1; ++b) f(item<2>{{(size_t)a, (size_t)b}, r});
  } else {
    const long long n0 = (long long)r[0], n1 = (long long)r[1], n2 = (long long)r[2];
#pragma omp parallel for schedule(static)
    for (long long ab = 0; ab < n0 * n1; ++ab) {
      const long long a = ab / n1, b = ab - a * n1;
      for (long long c = 0; c < n2; ++c) f(item<3>{{(size_t)a, (size_t)b, (size_t)c}, r});
    }
  }
}

template <int N, class T, class Op, class F>
void run_reduce(const range<N> &r, reduction_spec<T, Op> spec, F &f) {
  const int nth = omp_get_max_threads();
  std::vector<T> part((size_t)nth, T(0));
  const long long rows = N == 1 ? 1 : (long long)r[0] * (N == 3 ? (long long)r[1] : 1);
#pragma omp parallel num_threads(nth)
  {
    const int t = omp_get_thread_num();
    reducer<T, Op> red{T(0), spec.op};
#pragma omp for schedule(static)
    for (long long row = 0; row < rows; ++row) {
      if constexpr (N == 1) {
        for (size_t a = 0; a < r[0]; ++a) f(id<1>{{a}}, red);
      } else if constexpr (N == 2) {
        for (size_t b = 0; b < r[1]; ++b) f(id<2>{{(size_t)row, b}}, red);
      } else {
        const size_t a = (size_t)(row / (long long)r[1]), b = (size_t)(row % (long long)r[1]);
        for (size_t c = 0; c < r[2]; ++c) f(id<3>{{a, b, c}}, red);
      }
    }
    part[(size_t)t] = red.value;
  }
  T acc = *spec.target;
  for (int t = 0; t < nth; ++t) acc = spec.op(acc, part[(size_t)t]);
  *spec.target = acc;
}

}  // namespace detail

class handler {
 public:
  template <int N, class F>
  void parallel_for(range<N> r, F f) {
    detail::run(r, f);
  }
  template <int N, class T, class Op, class F>
  void parallel_for(range<N> r, reduction_spec<T, Op> red, F f) {
    detail::run_reduce(r, red, f);
  }
};

class queue {
 public:
  template <class F>
  event submit(F f) {
    handler h;
    f(h);
    return event{};
  }
  template <int N, class F>
  event parallel_for(range<N> r, F f) {
    detail::run(r, f);
    return event{};
  }
  template <int N, class F>
  event parallel_for(range<N> r, event, F f) {
    detail::run(r, f);
    return event{};
  }
  template <int N, class F>
  event parallel_for(range<N> r, const std::vector<event> &, F f) {
    detail::run(r, f);
    return event{};
  }
  event memcpy(void *dst, const void *src, size_t bytes, event = event{}) {
    if (bytes) std::memcpy(dst, src, bytes);
    return event{};
  }
  event memset(void *dst, int value, size_t bytes, event = event{}) {
    if (bytes) std::memset(dst, value, bytes);
    return event{};
  }
  void wait() {}
};

template <class T>
T *malloc_shared(size_t n, const queue &) {
  return static_cast<T *>(std::malloc(sizeof(T) * (n ? n : 1)));
}
template <class T>
T *malloc_host(size_t n, const queue &) {
  return static_cast<T *>(std::malloc(sizeof(T) * (n ? n : 1)));
}
template <class T>
T *malloc_device(size_t n, const queue &) {
  return static_cast<T *>(std::malloc(sizeof(T) * (n ? n : 1)));
}
template <class T>
T *aligned_alloc_shared(size_t alignment, size_t n, const queue &) {
  size_t bytes = sizeof(T) * (n ? n : 1);
  bytes = (bytes + alignment - 1) / alignment * alignment;
  return static_cast<T *>(std::aligned_alloc(alignment, bytes));
}
inline void *aligned_alloc_shared(size_t alignment, size_t bytes, const queue &) {
  bytes = (bytes ? bytes : 1);
  bytes = (bytes + alignment - 1) / alignment * alignment;
  return std::aligned_alloc(alignment, bytes);
}
inline void free(void *p, const queue &) { std::free(p); }

}  // namespace sycl
