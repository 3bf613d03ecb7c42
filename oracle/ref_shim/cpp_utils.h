// Minimal stand-in for cuda-utils' cpp_utils.h (written for this project): the helpers
// RapidSFM's RANSAC match filter kernels use. Test infrastructure only.
#pragma once
template <typename T>
__host__ __device__ constexpr T square(T x) {
    return x * x;
}
