// Host-only stand-in for Kokkos::sort on a 1-D view (TEST INFRASTRUCTURE, oracle).
#pragma once

#include <algorithm>

#include "Kokkos_Core.hpp"

namespace Kokkos {
template <class D, class... P>
inline void sort(const View<D, P...> &v) {
    static_assert(View<D, P...>::rank == 1, "shim: sort expects a 1-D view");
    if (v.span_is_contiguous()) {
        std::sort(v.data(), v.data() + v.extent(0));
        return;
    }
    std::vector<typename View<D, P...>::non_const_value_type> tmp(v.extent(0));
    for (size_t i = 0; i < tmp.size(); ++i) tmp[i] = v(i);
    std::sort(tmp.begin(), tmp.end());
    for (size_t i = 0; i < tmp.size(); ++i) v(i) = tmp[i];
}
}  // namespace Kokkos
