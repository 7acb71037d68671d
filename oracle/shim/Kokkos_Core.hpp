// Minimal host-only stand-in for <Kokkos_Core.hpp>, used ONLY to compile the
// reference's header-only hot-path templates (src/common, src/geometry,
// src/camera, src/geodesic, src/radiation, src/frame, src/model) on the CPU
// as the parity oracle.  It provides exactly what those headers use:
// KOKKOS_INLINE_FUNCTION, the Kokkos:: math forwards and a reference-counted
// host View<T*>.  Test infrastructure; never linked into the product.
#pragma once

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

namespace Kokkos {

template<class T> inline T sqrt(T x) { return std::sqrt(x); }
template<class T> inline T cbrt(T x) { return std::cbrt(x); }
template<class T> inline T exp(T x) { return std::exp(x); }
template<class T> inline T log(T x) { return std::log(x); }
template<class T> inline T sin(T x) { return std::sin(x); }
template<class T> inline T cos(T x) { return std::cos(x); }
template<class T> inline T tan(T x) { return std::tan(x); }
template<class T> inline T tanh(T x) { return std::tanh(x); }
template<class T> inline T acos(T x) { return std::acos(x); }
template<class T> inline T atan(T x) { return std::atan(x); }
template<class T> inline T atan2(T y, T x) { return std::atan2(y, x); }
template<class T> inline T floor(T x) { return std::floor(x); }
template<class T> inline T ceil(T x) { return std::ceil(x); }
template<class T, class U> inline auto pow(T x, U y) { return std::pow(x, y); }

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

} // namespace Kokkos
