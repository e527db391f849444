// Host-only stand-in for the subset of Kokkos that the QuantKos reference headers use.
//
// TEST INFRASTRUCTURE (oracle). This is not Kokkos: it is a small project-written
// runtime that lets the reference's own C++ headers (schemes, payoffs, solver,
// pricer, LSM engine, runners, dispatcher) compile with g++ and run on the host
// cores through OpenMP, so that the reference code itself can serve as the CPU
// oracle and the CPU baseline.  Only what the reference headers touch is provided:
//   * KOKKOS_* function/lambda macros and the host/device branch macros
//     (the host branch is always taken, as in a Kokkos OpenMP/Serial build);
//   * math forwarding (sqrt, exp, log, erf, fmax, fmin, abs, pow);
//   * View<T*> / View<T**> with LayoutLeft / LayoutRight / LayoutStride, subview,
//     deep_copy, create_mirror_view (host mirrors alias their source, as for
//     HostSpace views in Kokkos);
//   * parallel_for / parallel_reduce over an int range (OpenMP, static schedule,
//     per-thread partials combined in thread order so results are reproducible
//     for a fixed thread count);
//   * fence, initialize/finalize, DefaultExecutionSpace::name().
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [=, *this]
#define QKSHIM_STRIP(...) __VA_ARGS__
#define KOKKOS_IF_ON_HOST(CODE) { QKSHIM_STRIP CODE }
#define KOKKOS_IF_ON_DEVICE(CODE) {}

namespace Kokkos {

// ---------------------------------------------------------------- math
using std::abs;
using std::erf;
using std::exp;
using std::fmax;
using std::fmin;
using std::log;
using std::pow;
using std::sqrt;

// ---------------------------------------------------------------- layouts / spaces
struct LayoutLeft {};
struct LayoutRight {};
struct LayoutStride {};
struct HostSpace {};

struct DefaultExecutionSpace {
    static const char *name() { return "OpenMP (host shim)"; }
};
using DefaultHostExecutionSpace = DefaultExecutionSpace;

inline void fence() {}
inline void fence(const std::string &) {}
inline void initialize(int &, char **) {}
inline void initialize() {}
inline void finalize() {}
inline bool is_initialized() { return true; }

struct ALL_t {};
inline ALL_t ALL() { return {}; }

namespace shim_detail {
template <class T> struct rank_of { static constexpr int value = 0; using elem = T; };
template <class T> struct rank_of<T *> { static constexpr int value = 1 + rank_of<T>::value; using elem = typename rank_of<T>::elem; };

template <class... Props> struct pick_layout { using type = LayoutRight; };
template <class P, class... Rest> struct pick_layout<P, Rest...> {
    using type = std::conditional_t<std::is_same_v<P, LayoutLeft> || std::is_same_v<P, LayoutRight> ||
                                        std::is_same_v<P, LayoutStride>,
                                    P, typename pick_layout<Rest...>::type>;
};
}  // namespace shim_detail

// ---------------------------------------------------------------- View
template <class DataType, class... Props>
class View {
public:
    using value_type = typename shim_detail::rank_of<DataType>::elem;
    using non_const_value_type = std::remove_const_t<value_type>;
    static constexpr int rank = shim_detail::rank_of<DataType>::value;
    using array_layout = typename shim_detail::pick_layout<Props...>::type;
    using host_mirror_type = View<DataType, Props...>;
    using HostMirror = host_mirror_type;

    View() = default;

    explicit View(const std::string &label, size_t n0 = 0, size_t n1 = 0) : label_(label) {
        ext_[0] = n0;
        ext_[1] = (rank >= 2) ? n1 : 1;
        const size_t total = ext_[0] * ext_[1];
        store_ = std::shared_ptr<non_const_value_type[]>(new non_const_value_type[total > 0 ? total : 1]());
        ptr_ = store_.get();
        if constexpr (std::is_same_v<array_layout, LayoutLeft>) {
            str_[0] = 1;
            str_[1] = ext_[0];
        } else {
            str_[0] = (rank >= 2) ? ext_[1] : 1;
            str_[1] = 1;
        }
    }

    // Conversion between views of the same element type and rank (what Kokkos
    // allows for compatible layouts, e.g. any 1-D layout to any other).
    template <class D2, class... P2,
              std::enable_if_t<!std::is_same_v<View<D2, P2...>, View<DataType, Props...>> &&
                                   View<D2, P2...>::rank == rank,
                               int> = 0>
    View(const View<D2, P2...> &o) : store_(o.store_), ptr_(o.ptr_), label_(o.label_) {
        ext_[0] = o.ext_[0];
        ext_[1] = o.ext_[1];
        str_[0] = o.str_[0];
        str_[1] = o.str_[1];
    }

    // Raw construction used by subview().
    View(std::shared_ptr<non_const_value_type[]> store, value_type *ptr, size_t e0, size_t e1, size_t s0, size_t s1)
        : store_(std::move(store)), ptr_(ptr) {
        ext_[0] = e0;
        ext_[1] = e1;
        str_[0] = s0;
        str_[1] = s1;
    }

    template <class I>
    value_type &operator()(I i) const { return ptr_[static_cast<size_t>(i) * str_[0]]; }
    template <class I, class J>
    value_type &operator()(I i, J j) const {
        return ptr_[static_cast<size_t>(i) * str_[0] + static_cast<size_t>(j) * str_[1]];
    }

    size_t extent(int r) const { return (r < 2) ? ext_[r] : 1; }
    int extent_int(int r) const { return static_cast<int>(extent(r)); }
    size_t stride(int r) const { return str_[r]; }
    size_t size() const { return (rank >= 2) ? ext_[0] * ext_[1] : ext_[0]; }
    size_t span() const { return size(); }
    value_type *data() const { return ptr_; }
    const std::string &label() const { return label_; }
    bool span_is_contiguous() const {
        if (rank < 2) return str_[0] == 1 || ext_[0] <= 1;
        return (str_[1] == 1 && str_[0] == ext_[1]) || (str_[0] == 1 && str_[1] == ext_[0]);
    }
    bool is_allocated() const { return ptr_ != nullptr; }

    std::shared_ptr<non_const_value_type[]> store_{};
    value_type *ptr_ = nullptr;
    size_t ext_[2] = {0, 1};
    size_t str_[2] = {1, 1};
    std::string label_{};
};

template <class V>
inline V create_mirror_view(const V &v) { return v; }
template <class Space, class V>
inline V create_mirror_view(const Space &, const V &v) { return v; }

// 1-D range of a 1-D view
template <class D, class... P, class A, class B>
inline View<D, LayoutStride> subview(const View<D, P...> &v, const std::pair<A, B> &r) {
    static_assert(View<D, P...>::rank == 1, "shim: 1-D subview expects a 1-D view");
    const size_t b = static_cast<size_t>(r.first), e = static_cast<size_t>(r.second);
    return View<D, LayoutStride>(v.store_, v.ptr_ + b * v.str_[0], e - b, 1, v.str_[0], 1);
}
// rows [b,e) of a 2-D view
template <class D, class... P, class A, class B>
inline View<D, LayoutStride> subview(const View<D, P...> &v, const std::pair<A, B> &r, ALL_t) {
    const size_t b = static_cast<size_t>(r.first), e = static_cast<size_t>(r.second);
    return View<D, LayoutStride>(v.store_, v.ptr_ + b * v.str_[0], e - b, v.ext_[1], v.str_[0], v.str_[1]);
}
// column j of a 2-D view
template <class D, class... P, class J, std::enable_if_t<std::is_integral_v<J>, int> = 0>
inline View<typename View<D, P...>::value_type *, LayoutStride> subview(const View<D, P...> &v, ALL_t, J j) {
    using V1 = View<typename View<D, P...>::value_type *, LayoutStride>;
    return V1(v.store_, v.ptr_ + static_cast<size_t>(j) * v.str_[1], v.ext_[0], 1, v.str_[0], 1);
}
// row i of a 2-D view
template <class D, class... P, class I, std::enable_if_t<std::is_integral_v<I>, int> = 0>
inline View<typename View<D, P...>::value_type *, LayoutStride> subview(const View<D, P...> &v, I i, ALL_t) {
    using V1 = View<typename View<D, P...>::value_type *, LayoutStride>;
    return V1(v.store_, v.ptr_ + static_cast<size_t>(i) * v.str_[0], v.ext_[1], 1, v.str_[1], 1);
}

template <class D1, class... P1, class D2, class... P2>
inline void deep_copy(const View<D1, P1...> &dst, const View<D2, P2...> &src) {
    if (dst.extent(0) != src.extent(0) || dst.extent(1) != src.extent(1))
        throw std::runtime_error("Kokkos shim: deep_copy extents mismatch");
    if (dst.data() == src.data()) return;
    if constexpr (View<D1, P1...>::rank == 1) {
        for (size_t i = 0; i < dst.extent(0); ++i) dst(i) = src(i);
    } else {
        for (size_t i = 0; i < dst.extent(0); ++i)
            for (size_t j = 0; j < dst.extent(1); ++j) dst(i, j) = src(i, j);
    }
}
template <class D1, class... P1, class S, std::enable_if_t<std::is_arithmetic_v<S>, int> = 0>
inline void deep_copy(const View<D1, P1...> &dst, const S &val) {
    for (size_t i = 0; i < dst.extent(0); ++i)
        for (size_t j = 0; j < dst.extent(1); ++j) {
            if constexpr (View<D1, P1...>::rank == 1) dst(i) = val; else dst(i, j) = val;
        }
}

// ---------------------------------------------------------------- parallel patterns
inline int shim_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
inline int shim_thread_id() {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

template <class Idx>
struct RangePolicy {
    Idx begin, end;
    RangePolicy(Idx b, Idx e) : begin(b), end(e) {}
};

template <class F>
inline void parallel_for(const std::string &, const int n, const F &f) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) f(i);
}
template <class F>
inline void parallel_for(const int n, const F &f) { parallel_for(std::string(), n, f); }

template <class F, class T>
inline void parallel_reduce(const std::string &, const int n, const F &f, T &result) {
    const int nt = shim_num_threads();
    std::vector<T> part(static_cast<size_t>(nt));
    for (auto &p : part) p = T{};
#pragma omp parallel
    {
        T local{};
        const int tid = shim_thread_id();
#pragma omp for schedule(static)
        for (int i = 0; i < n; ++i) f(i, local);
        part[static_cast<size_t>(tid)] = local;
    }
    T total{};
    for (auto &p : part) total += p;
    result = total;
}
template <class F, class T>
inline void parallel_reduce(const int n, const F &f, T &result) { parallel_reduce(std::string(), n, f, result); }

}  // namespace Kokkos
