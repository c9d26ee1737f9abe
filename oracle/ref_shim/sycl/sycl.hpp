// Host-only subset of the SYCL 2020 interface, written for this project so
// that the reference renderer's kernel sources (Pale/Renderer/Kernels/
// PrimalKernels.cpp, AdjointKernels.cpp, PostprocessKernel.cpp and the
// headers they include) compile unmodified with g++ and run on the CPU.
//
// TEST INFRASTRUCTURE ONLY: the build in oracle/build_ref.py links these
// sources into oracle/_ref/libpale_ref.so, which the tests use to pin the C
// oracle to the reference's own kernel code and which the CPU baseline of
// the benchmark times.  Nothing of the product includes this header.
//
// Execution model.  A queue runs every command group to completion when it
// is submitted (an in-order queue whose wait() is a no-op).
//   * parallel_for over a range runs its work items in index order on one
//     thread (the default: the result equals a sequential run of the
//     reference, which is what the oracle restates), or on an OpenMP team
//     when sycl_shim_set_threads(n > 1) asked for it (timing only; the
//     atomic appends then interleave as on a real device).
//   * parallel_for over an nd_range runs each work group's items as fibers
//     that yield at item.barrier(), so group barriers have their SYCL
//     meaning; groups run one after another on each thread of the team.
// Device memory is host memory; atomic_ref wraps std::atomic_ref.
#pragma once

// The reference's kernels call abs() unqualified on floats
// (KernelHelpers.h: safeInvDir, intersectTriangle, the cosine-hemisphere
// frame); a SYCL implementation resolves that to the floating-point abs.
// libstdc++'s <math.h> and <stdlib.h> wrappers put std::abs's overloads
// into the global namespace, which gives the same meaning here.
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#ifndef SYCL_EXTERNAL
#define SYCL_EXTERNAL
#endif

// Threads used by parallel_for (1 = sequential, index order).
void sycl_shim_set_threads(int n);
int sycl_shim_threads();

namespace sycl {

// ------------------------------------------------------------------ vec
template <typename T, int N>
struct vec {
  static_assert(N >= 1 && N <= 16, "vec size");
  static constexpr int kStorage = (N == 3) ? 4 : N;   // a 3-vector occupies 4 elements
  T s[kStorage];

  constexpr vec() : s{} {}
  constexpr explicit vec(const T& a) : s{} {
    for (int i = 0; i < N; ++i) s[i] = a;
  }
  template <typename... A, typename = std::enable_if_t<(sizeof...(A) == N) && (N > 1) &&
                                                       (std::is_arithmetic_v<std::decay_t<A>> && ...)>>
  constexpr vec(A... a) : s{static_cast<T>(a)...} {}
  constexpr vec(const vec&) = default;
  constexpr vec& operator=(const vec&) = default;
  vec& operator=(const T& a) {
    for (int i = 0; i < N; ++i) s[i] = a;
    return *this;
  }

  static constexpr int size() { return N; }
  T& operator[](int i) { return s[i]; }
  const T& operator[](int i) const { return s[i]; }
  T& x() { return s[0]; }
  const T& x() const { return s[0]; }
  T& y() { static_assert(N >= 2, "y"); return s[1]; }
  const T& y() const { static_assert(N >= 2, "y"); return s[1]; }
  T& z() { static_assert(N >= 3, "z"); return s[2]; }
  const T& z() const { static_assert(N >= 3, "z"); return s[2]; }
  T& w() { static_assert(N >= 4, "w"); return s[3]; }
  const T& w() const { static_assert(N >= 4, "w"); return s[3]; }

  vec operator-() const {
    vec r;
    for (int i = 0; i < N; ++i) r.s[i] = -s[i];
    return r;
  }
  vec operator+() const { return *this; }
#define SHIM_VEC_COMPOUND(OP)                          \
  vec& operator OP##=(const vec & b) {                 \
    for (int i = 0; i < N; ++i) s[i] = s[i] OP b.s[i]; \
    return *this;                                      \
  }                                                    \
  vec& operator OP##=(const T & b) {                   \
    for (int i = 0; i < N; ++i) s[i] = s[i] OP b;      \
    return *this;                                      \
  }
  SHIM_VEC_COMPOUND(+)
  SHIM_VEC_COMPOUND(-)
  SHIM_VEC_COMPOUND(*)
  SHIM_VEC_COMPOUND(/)
#undef SHIM_VEC_COMPOUND
};

#define SHIM_VEC_BINARY(OP)                                   \
  template <typename T, int N>                               \
  vec<T, N> operator OP(const vec<T, N>& a, const vec<T, N>& b) { \
    vec<T, N> r;                                             \
    for (int i = 0; i < N; ++i) r.s[i] = a.s[i] OP b.s[i];   \
    return r;                                                \
  }                                                          \
  template <typename T, int N>                               \
  vec<T, N> operator OP(const vec<T, N>& a, const std::type_identity_t<T>& b) { \
    vec<T, N> r;                                             \
    for (int i = 0; i < N; ++i) r.s[i] = a.s[i] OP b;        \
    return r;                                                \
  }                                                          \
  template <typename T, int N>                               \
  vec<T, N> operator OP(const std::type_identity_t<T>& a, const vec<T, N>& b) { \
    vec<T, N> r;                                             \
    for (int i = 0; i < N; ++i) r.s[i] = a OP b.s[i];        \
    return r;                                                \
  }
SHIM_VEC_BINARY(+)
SHIM_VEC_BINARY(-)
SHIM_VEC_BINARY(*)
SHIM_VEC_BINARY(/)
#undef SHIM_VEC_BINARY

using float2 = vec<float, 2>;
using float3 = vec<float, 3>;
using float4 = vec<float, 4>;
using int2 = vec<int, 2>;
using int3 = vec<int, 3>;
using int4 = vec<int, 4>;
using uint2 = vec<uint32_t, 2>;
using uint3 = vec<uint32_t, 3>;
using uint4 = vec<uint32_t, 4>;
using uchar4 = vec<unsigned char, 4>;

static_assert(sizeof(float3) == 16, "a SYCL 3-vector is 16 bytes");

// --------------------------------------------------------------- math
// Scalar functions are the C library's float functions; the geometric
// functions (dot, cross, length) sum their products left to right.
inline float fmax(float a, float b) { return std::fmax(a, b); }
inline float fmin(float a, float b) { return std::fmin(a, b); }
inline float fabs(float a) { return std::fabs(a); }
inline float sqrt(float a) { return std::sqrt(a); }
inline float rsqrt(float a) { return 1.0f / std::sqrt(a); }
inline float floor(float a) { return std::floor(a); }
inline float ceil(float a) { return std::ceil(a); }
inline float exp(float a) { return std::exp(a); }
inline float log(float a) { return std::log(a); }
inline float pow(float a, float b) { return std::pow(a, b); }
inline float sin(float a) { return std::sin(a); }
inline float cos(float a) { return std::cos(a); }
inline float tan(float a) { return std::tan(a); }
inline float acos(float a) { return std::acos(a); }
inline float atan2(float a, float b) { return std::atan2(a, b); }
inline float copysign(float a, float b) { return std::copysign(a, b); }
inline bool isfinite(float a) { return std::isfinite(a); }
inline bool isnan(float a) { return std::isnan(a); }
inline bool isinf(float a) { return std::isinf(a); }
inline double sqrt(double a) { return std::sqrt(a); }
inline double fabs(double a) { return std::fabs(a); }

// min / max: y if y < x (resp. x < y), else x
template <typename T>
inline std::enable_if_t<std::is_arithmetic_v<T>, T> min(T a, T b) { return b < a ? b : a; }
template <typename T>
inline std::enable_if_t<std::is_arithmetic_v<T>, T> max(T a, T b) { return a < b ? b : a; }
template <typename T, int N>
vec<T, N> min(const vec<T, N>& a, const vec<T, N>& b) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = b.s[i] < a.s[i] ? b.s[i] : a.s[i];
  return r;
}
template <typename T, int N>
vec<T, N> min(const vec<T, N>& a, std::type_identity_t<T> b) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = b < a.s[i] ? b : a.s[i];
  return r;
}
template <typename T, int N>
vec<T, N> max(const vec<T, N>& a, const vec<T, N>& b) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = a.s[i] < b.s[i] ? b.s[i] : a.s[i];
  return r;
}
template <typename T, int N>
vec<T, N> max(const vec<T, N>& a, std::type_identity_t<T> b) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = a.s[i] < b ? b : a.s[i];
  return r;
}
// clamp(x, lo, hi) = min(max(x, lo), hi); floats use fmin/fmax
inline float clamp(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }
template <typename T>
inline std::enable_if_t<std::is_integral_v<T>, T> clamp(T x, T lo, T hi) {
  return sycl::min(sycl::max(x, lo), hi);
}
template <typename T, int N>
vec<T, N> clamp(const vec<T, N>& x, std::type_identity_t<T> lo, std::type_identity_t<T> hi) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = clamp(x.s[i], lo, hi);
  return r;
}
template <typename T, int N>
vec<T, N> fmax(const vec<T, N>& a, const vec<T, N>& b) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = std::fmax(a.s[i], b.s[i]);
  return r;
}
template <typename T, int N>
vec<T, N> fmax(const vec<T, N>& a, std::type_identity_t<T> b) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = std::fmax(a.s[i], b);
  return r;
}
template <typename T, int N>
vec<T, N> fmin(const vec<T, N>& a, const vec<T, N>& b) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = std::fmin(a.s[i], b.s[i]);
  return r;
}
template <typename T, int N>
vec<T, N> fmin(const vec<T, N>& a, std::type_identity_t<T> b) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = std::fmin(a.s[i], b);
  return r;
}
template <typename T, int N>
vec<T, N> fabs(const vec<T, N>& a) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r.s[i] = std::fabs(a.s[i]);
  return r;
}
template <typename T, int N>
T dot(const vec<T, N>& a, const vec<T, N>& b) {
  T r = a.s[0] * b.s[0];
  for (int i = 1; i < N; ++i) r = r + a.s[i] * b.s[i];
  return r;
}
template <typename T>
vec<T, 3> cross(const vec<T, 3>& a, const vec<T, 3>& b) {
  return vec<T, 3>(a.s[1] * b.s[2] - a.s[2] * b.s[1], a.s[2] * b.s[0] - a.s[0] * b.s[2],
                   a.s[0] * b.s[1] - a.s[1] * b.s[0]);
}
template <typename T, int N>
T length(const vec<T, N>& a) { return std::sqrt(dot(a, a)); }
template <typename T, int N>
vec<T, N> normalize(const vec<T, N>& a) {
  const T inv = T(1) / std::sqrt(dot(a, a));
  return a * inv;
}

// ------------------------------------------------------- enums, traits
enum class memory_order { relaxed, acquire, release, acq_rel, seq_cst };
enum class memory_scope { work_item, sub_group, work_group, device, system };
namespace access {
enum class address_space { global_space, local_space, constant_space, private_space, generic_space };
enum class fence_space { local_space, global_space, global_and_local };
enum class mode { read, write, read_write };
}  // namespace access
template <typename T>
struct is_device_copyable : std::is_trivially_copyable<T> {};

// --------------------------------------------------------------- atomics
template <typename T, memory_order O = memory_order::relaxed, memory_scope S = memory_scope::device,
          access::address_space A = access::address_space::global_space>
class atomic_ref {
 public:
  explicit atomic_ref(T& r) : ref_(r) {}
  T load() const { return ref_.load(std::memory_order_relaxed); }
  void store(T v) const { ref_.store(v, std::memory_order_relaxed); }
  T exchange(T v) const { return ref_.exchange(v, std::memory_order_relaxed); }
  T fetch_add(T v) const { return ref_.fetch_add(v, std::memory_order_relaxed); }
  T fetch_sub(T v) const { return ref_.fetch_sub(v, std::memory_order_relaxed); }
  T fetch_min(T v) const {
    T cur = load();
    while (v < cur && !ref_.compare_exchange_weak(cur, v, std::memory_order_relaxed)) {
    }
    return cur;
  }
  T fetch_max(T v) const {
    T cur = load();
    while (cur < v && !ref_.compare_exchange_weak(cur, v, std::memory_order_relaxed)) {
    }
    return cur;
  }
  bool compare_exchange_strong(T& expected, T desired) const {
    return ref_.compare_exchange_strong(expected, desired, std::memory_order_relaxed);
  }
  bool compare_exchange_weak(T& expected, T desired) const {
    return ref_.compare_exchange_weak(expected, desired, std::memory_order_relaxed);
  }
  T operator+=(T v) const { return fetch_add(v) + v; }
  T operator-=(T v) const { return fetch_sub(v) - v; }
  T operator++(int) const { return fetch_add(T(1)); }
  operator T() const { return load(); }

 private:
  mutable std::atomic_ref<T> ref_;
};

// ------------------------------------------------------ index spaces
template <int D = 1>
struct range {
  size_t v[D];
  range(size_t a) : v{a} { static_assert(D == 1, "1-d ranges only"); }
  size_t operator[](int i) const { return v[i]; }
  size_t size() const { return v[0]; }
  size_t get(int i) const { return v[i]; }
};
template <int D = 1>
struct id {
  size_t v[D];
  id() : v{} {}
  id(size_t a) : v{a} {}
  size_t operator[](int i) const { return v[i]; }
  size_t& operator[](int i) { return v[i]; }
  size_t get(int i) const { return v[i]; }
  operator size_t() const { return v[0]; }
};
template <int D = 1>
struct item {
  size_t idx, rng;
  size_t get_id(int = 0) const { return idx; }
  size_t operator[](int) const { return idx; }
  size_t get_linear_id() const { return idx; }
  size_t get_range(int = 0) const { return rng; }
  operator id<D>() const { return id<D>(idx); }
};
template <int D = 1>
struct nd_range {
  range<D> global, local;
  nd_range(range<D> g, range<D> l) : global(g), local(l) {}
  range<D> get_global_range() const { return global; }
  range<D> get_local_range() const { return local; }
};

}  // namespace sycl

// fiber runtime of the nd_range executor (oracle/ref_shim/sycl_shim.cpp)
namespace sycl_shim {
void group_barrier();
int current_thread();
void run_nd_range(size_t groups, size_t local, const std::function<void(size_t, size_t)>& body);
void run_range(size_t n, const std::function<void(size_t)>& body);
}  // namespace sycl_shim

namespace sycl {

template <int D = 1>
struct nd_item {
  size_t global_id, local_id, group_id, local_range, group_range;
  size_t get_global_id(int = 0) const { return global_id; }
  size_t get_local_id(int = 0) const { return local_id; }
  size_t get_group(int = 0) const { return group_id; }
  size_t get_group_linear_id() const { return group_id; }
  size_t get_local_range(int = 0) const { return local_range; }
  size_t get_global_range(int = 0) const { return local_range * group_range; }
  size_t get_global_linear_id() const { return global_id; }
  size_t get_local_linear_id() const { return local_id; }
  void barrier(access::fence_space = access::fence_space::global_and_local) const { sycl_shim::group_barrier(); }
};

class handler;

// Work-group local memory: one array per thread of the team (groups run
// one after another on each thread); copies of the accessor (the kernel
// lambda captures it by value) share them.
template <typename T, int D = 1>
class local_accessor {
 public:
  local_accessor(range<D> r, handler&)
      : buf_(std::make_shared<std::vector<std::vector<T>>>(static_cast<size_t>(sycl_shim_threads()),
                                                           std::vector<T>(r[0]))) {}
  T& operator[](size_t i) const { return (*buf_)[static_cast<size_t>(sycl_shim::current_thread())][i]; }

 private:
  std::shared_ptr<std::vector<std::vector<T>>> buf_;
};

class event {
 public:
  void wait() {}
  static void wait(const std::vector<event>&) {}
};

class handler {
 public:
  template <typename Name = void, typename F>
  void parallel_for(range<1> r, F f) {
    const size_t n = r[0];
    if constexpr (std::is_invocable_v<F, id<1>>) {
      sycl_shim::run_range(n, [&](size_t i) { f(id<1>(i)); });
    } else {
      sycl_shim::run_range(n, [&](size_t i) { f(item<1>{i, n}); });
    }
  }
  template <typename Name = void, typename F>
  void parallel_for(nd_range<1> r, F f) {
    const size_t local = r.local[0];
    const size_t groups = (r.global[0] + local - 1) / local;
    sycl_shim::run_nd_range(groups, local, [&](size_t g, size_t l) {
      f(nd_item<1>{g * local + l, l, g, local, groups});
    });
  }
  template <typename Name = void, typename F>
  void single_task(F f) {
    f();
  }
};

class queue {
 public:
  queue() = default;
  template <typename F>
  event submit(F f) {
    handler h;
    f(h);
    return event{};
  }
  void wait() {}
  void wait_and_throw() {}
  template <typename T>
  event fill(T* p, const T& v, size_t n) {
    for (size_t i = 0; i < n; ++i) p[i] = v;
    return event{};
  }
  event memcpy(void* dst, const void* src, size_t bytes) {
    if (bytes) std::memmove(dst, src, bytes);
    return event{};
  }
  event memset(void* p, int v, size_t bytes) {
    if (bytes) std::memset(p, v, bytes);
    return event{};
  }
  template <typename T>
  event copy(const T* src, T* dst, size_t n) {
    return memcpy(dst, src, n * sizeof(T));
  }
};

template <typename T>
T* malloc_device(size_t n, const queue&) {
  return static_cast<T*>(std::calloc(n ? n : 1, sizeof(T)));
}
template <typename T>
T* malloc_shared(size_t n, const queue&) {
  return malloc_device<T>(n, queue{});
}
template <typename T>
T* malloc_host(size_t n, const queue&) {
  return malloc_device<T>(n, queue{});
}
inline void free(void* p, const queue&) { std::free(p); }

}  // namespace sycl
