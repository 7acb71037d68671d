// Minimal host-only stand-in for <Kokkos_Core.hpp>, used ONLY to compile the
// reference's header-only hot-path templates (src/common, src/geometry,
// src/camera, src/geodesic, src/radiation, src/frame, src/model, and the
// image drivers of src/image and src/diagnostics) on the CPU as the parity
// oracle.  It provides what those headers use: KOKKOS_INLINE_FUNCTION, the
// Kokkos:: math forwards, reference-counted host Views of rank 1 and 2, and a
// serial stand-in for the execution API (parallel_for and parallel_reduce over
// a RangePolicy in index order, fence, deep_copy, mirrors, Timer).  Test infrastructure; never linked
// into the product.
#pragma once

#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <type_traits>

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]

#ifdef KPREF_PERTURB_LIBM
// Conditioning probe (the _ref/libkpref_ulp.so build): every transcendental
// result below is moved by a pseudo-random whole number of ulps in [-2, 2],
// a fixed sequence per pixel and seed (kpref_perturb_pixel).  sqrt, floor
// and ceil are correctly rounded everywhere and stay exact.
namespace kpref_ulp {
inline unsigned long long g_seed = 0;
inline thread_local unsigned long long t_rng = 1;
inline void seed_pixel(int pixel) {
    t_rng = 0x9E3779B97F4A7C15ull * static_cast<unsigned long long>(pixel + 1) +
            0xD1B54A32D192ED03ull * (g_seed + 1);
    if (!t_rng) t_rng = 1;
}
template<class T> inline T perturb(T r) {
    if (!(r == r) || r == T(0) || r - r != T(0)) return r;
    t_rng ^= t_rng << 13;
    t_rng ^= t_rng >> 7;
    t_rng ^= t_rng << 17;
    const int k = static_cast<int>(t_rng % 5ull) - 2;
    for (int i = 0; i < k; ++i) r = std::nextafter(r, T(INFINITY));
    for (int i = 0; i > k; --i) r = std::nextafter(r, -T(INFINITY));
    return r;
}
}  // namespace kpref_ulp
#define KPREF_P(expr) kpref_ulp::perturb(expr)
#else
#define KPREF_P(expr) (expr)
#endif

namespace Kokkos {

template<class T> inline T sqrt(T x) { return std::sqrt(x); }
template<class T> inline T cbrt(T x) { return KPREF_P(std::cbrt(x)); }
template<class T> inline T exp(T x) { return KPREF_P(std::exp(x)); }
template<class T> inline T log(T x) { return KPREF_P(std::log(x)); }
template<class T> inline T sin(T x) { return KPREF_P(std::sin(x)); }
template<class T> inline T cos(T x) { return KPREF_P(std::cos(x)); }
template<class T> inline T tan(T x) { return KPREF_P(std::tan(x)); }
template<class T> inline T tanh(T x) { return KPREF_P(std::tanh(x)); }
template<class T> inline T acos(T x) { return KPREF_P(std::acos(x)); }
template<class T> inline T atan(T x) { return KPREF_P(std::atan(x)); }
template<class T> inline T atan2(T y, T x) { return KPREF_P(std::atan2(y, x)); }
template<class T> inline T floor(T x) { return std::floor(x); }
template<class T> inline T ceil(T x) { return std::ceil(x); }
template<class T, class U> inline auto pow(T x, U y) { return KPREF_P(std::pow(x, y)); }
template<class T> inline bool isfinite(T x) { return std::isfinite(x); }
template<class T> inline bool isnan(T x) { return std::isnan(x); }

inline void abort(const char* msg) {
    std::fprintf(stderr, "Kokkos::abort: %s\n", msg);
    std::abort();
}

struct RandomAccess {};
template<class... T> struct MemoryTraits {};
struct HostSpace {};

// Host View of rank 1 only (all the hot-path headers need).
template<class DataType, class... Props>
class View;

template<class T, class... Props>
class View<T*, Props...> {
public:
    using value_type = T;
    using non_const_value_type = std::remove_const_t<T>;
    using array_layout = void;
    using device_type = void;

    View() = default;
    View(const std::string&, std::size_t n)
        : storage_(std::shared_ptr<non_const_value_type[]>(new non_const_value_type[n]())),
          ptr_(storage_.get()), n_(n) {}
    View(T* ptr, std::size_t n) : ptr_(ptr), n_(n) {}
    template<class U, class... P2,
             class = std::enable_if_t<std::is_convertible_v<U*, T*>>>
    View(const View<U*, P2...>& other)
        : storage_(other.storage()), ptr_(other.data()), n_(other.extent(0)) {}

    T& operator()(std::size_t i) const { return ptr_[i]; }
    T& operator[](std::size_t i) const { return ptr_[i]; }
    std::size_t extent(int) const { return n_; }
    std::size_t span() const { return n_; }
    std::size_t size() const { return n_; }
    T* data() const { return ptr_; }
    const std::shared_ptr<non_const_value_type[]>& storage() const { return storage_; }

private:
    std::shared_ptr<non_const_value_type[]> storage_;
    T* ptr_ = nullptr;
    std::size_t n_ = 0;
};

// Runtime lifetime: the host shim has nothing to start or stop.
inline bool is_initialized() { return true; }
inline void finalize() {}

// Host View of rank 2 (the image drivers' [nfreq][npix] arrays).
template<class T, class... Props>
class View<T**, Props...> {
public:
    using value_type = T;
    using non_const_value_type = std::remove_const_t<T>;
    View() = default;
    View(const std::string&, std::size_t n0, std::size_t n1)
        : storage_(std::shared_ptr<non_const_value_type[]>(new non_const_value_type[n0 * n1]())),
          ptr_(storage_.get()), n0_(n0), n1_(n1) {}
    T& operator()(std::size_t i, std::size_t j) const { return ptr_[i * n1_ + j]; }
    std::size_t extent(int d) const { return d == 0 ? n0_ : n1_; }
    std::size_t span() const { return n0_ * n1_; }
    std::size_t size() const { return n0_ * n1_; }
    T* data() const { return ptr_; }

private:
    std::shared_ptr<non_const_value_type[]> storage_;
    T* ptr_ = nullptr;
    std::size_t n0_ = 0, n1_ = 0;
};

// Execution: one serial host space.  The image drivers' parallel_for loops
// run in index order on the calling thread.
struct OpenMP {};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;
struct Unmanaged {};
struct Dynamic {};
struct Static {};
template<class T> struct Schedule {};
template<class T> struct IndexType {};

template<class... Args>
struct RangePolicy {
    long long begin = 0, end = 0;
    RangePolicy(long long b, long long e) : begin(b), end(e) {}
    template<class Space>
    RangePolicy(const Space&, long long b, long long e) : begin(b), end(e) {}
};

template<class... Args, class F>
inline void parallel_for(const RangePolicy<Args...>& policy, const F& f) {
    for (long long i = policy.begin; i < policy.end; ++i) f(static_cast<int>(i));
}
template<class... Args, class F>
inline void parallel_for(const std::string&, const RangePolicy<Args...>& policy, const F& f) {
    parallel_for(policy, f);
}
template<class F>
inline void parallel_for(const std::string&, long long n, const F& f) {
    for (long long i = 0; i < n; ++i) f(static_cast<int>(i));
}
template<class F>
inline void parallel_for(long long n, const F& f) {
    for (long long i = 0; i < n; ++i) f(static_cast<int>(i));
}

inline void fence() {}
inline void fence(const std::string&) {}

template<class A, class B>
inline void deep_copy(const A& dst, const B& src) {
    for (std::size_t i = 0; i < src.span(); ++i) dst.data()[i] = src.data()[i];
}

struct Timer {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double seconds() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    void reset() { t0 = std::chrono::steady_clock::now(); }
};

// Host views already live in host memory: the mirror is the view itself.
template<class Space, class V>
inline V create_mirror_view_and_copy(const Space&, const V& v) {
    return v;
}
template<class V>
inline V create_mirror_view(const V& v) {
    return v;
}

// Serial sum reduction (the slow-light driver's active-ray count).
template<class... Args, class F, class T>
inline void parallel_reduce(const std::string&, const RangePolicy<Args...>& policy, const F& f, T& result) {
    T acc = T();
    for (long long i = policy.begin; i < policy.end; ++i) f(static_cast<int>(i), acc);
    result = acc;
}
template<class... Args, class F, class T>
inline void parallel_reduce(const RangePolicy<Args...>& policy, const F& f, T& result) {
    parallel_reduce(std::string(), policy, f, result);
}
template<class F, class T>
inline void parallel_reduce(const std::string& name, long long n, const F& f, T& result) {
    parallel_reduce(name, RangePolicy<>(0, n), f, result);
}

} // namespace Kokkos
