// Minimal stand-in for the KArray.h of RapidSFM's missing cuda-utils submodule, written for this
// project so that the reference's matcher sources compile as a test oracle. A fixed-size
// multi-dimensional array: KArray<T, d0, d1, ...> holds d0 elements of KArray<T, d1, ...>,
// aligned to the largest power of two (<= 16) dividing its size.
#pragma once
#include <cstddef>
#include <cstdint>
#include <type_traits>
#include <algorithm>
#include <array>
#include <limits>
#include <vector>
#include <stdexcept>
#ifdef __CUDACC__
#define RSFM_SHIM_HD __host__ __device__ __forceinline__
#else
#define RSFM_SHIM_HD inline
#endif

namespace cudapp {
template <typename T, size_t... dims>
struct KArray;

namespace detail {
template <typename T, size_t... dims>
struct KArrayElem;
template <typename T, size_t d0>
struct KArrayElem<T, d0> { using type = T; };
template <typename T, size_t d0, size_t d1, size_t... rest>
struct KArrayElem<T, d0, d1, rest...> { using type = KArray<T, d1, rest...>; };

constexpr size_t align_for(size_t bytes, size_t natural) {
    size_t a = 16;
    while (a > natural && bytes % a != 0) a /= 2;
    return a > natural ? a : natural;
}
}  // namespace detail

template <typename T, size_t d0, size_t... rest>
struct alignas(detail::align_for(sizeof(typename detail::KArrayElem<T, d0, rest...>::type) * d0,
                                 alignof(typename detail::KArrayElem<T, d0, rest...>::type))) KArray<T, d0, rest...> {
    using Elem = typename detail::KArrayElem<T, d0, rest...>::type;
    static constexpr size_t dimension = d0;
    Elem data[d0];
    RSFM_SHIM_HD Elem& operator[](size_t i) { return data[i]; }
    RSFM_SHIM_HD const Elem& operator[](size_t i) const { return data[i]; }
    RSFM_SHIM_HD Elem* begin() { return data; }
    RSFM_SHIM_HD const Elem* begin() const { return data; }
    RSFM_SHIM_HD Elem* end() { return data + d0; }
    RSFM_SHIM_HD const Elem* end() const { return data + d0; }
    RSFM_SHIM_HD static constexpr size_t size() { return d0; }
};
}  // namespace cudapp
