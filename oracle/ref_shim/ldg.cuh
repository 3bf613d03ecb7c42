// Minimal stand-in for cuda-utils' ldg.cuh (written for this project): read-only-path loads of
// small trivially-copyable values, also through a cudapp::Ptr.
#pragma once
#include <cstring>
#include <type_traits>
#include <cuda_runtime.h>
#include "ptr.h"

namespace cudapp {
template <typename T>
__device__ __forceinline__ std::remove_const_t<T> ldg(const T* p) {
    using R = std::remove_const_t<T>;
    R r;
    if constexpr (sizeof(R) == 16 && alignof(R) >= 16) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
        memcpy(&r, &v, 16);
    } else if constexpr (sizeof(R) == 8 && alignof(R) >= 8) {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
        memcpy(&r, &v, 8);
    } else if constexpr (sizeof(R) == 4 && alignof(R) >= 4) {
        const unsigned v = __ldg(reinterpret_cast<const unsigned*>(p));
        memcpy(&r, &v, 4);
    } else {
        r = *p;
    }
    return r;
}
template <typename T, typename O>
__device__ __forceinline__ std::remove_const_t<T> ldg(const Ptr<T, O>& p) {
    return ldg(p.get());
}
}  // namespace cudapp
