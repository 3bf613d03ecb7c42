// Minimal stand-in for cuda-utils' kmat.h (written for this project; the submodule is absent):
// small fixed-size row-major matrices with the operations RapidSFM's RANSAC match filter uses
// (RansacMatchFilter.cu), and the 3x3 solver it calls. Test infrastructure only.
//
// Two arithmetic modes, for two builds of the reference kernels:
//  - default: plain C++ operators in the natural order (a matrix-vector product is a sum over k,
//    then the shift is added), for the build with the reference's own flags (--use_fast_math);
//  - RSFM_SHIM_KMAT_MATCH: the B200 kernel's explicit round-to-nearest order (A l + t as
//    fma(a0, lx, fma(a1, ly, t)), |d|^2 as fma(dx, dx, dy * dy), the same Gaussian elimination),
//    for a build with -fmad=false that can be compared with the B200 kernel bit for bit.
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

template <typename T, int R, int C = 1>
struct kmat {
    T d[R * C];
    kmat() = default;
    __host__ __device__ kmat(const T (&init)[R * C]) {
        for (int i = 0; i < R * C; ++i) d[i] = init[i];
    }
    __host__ __device__ T& operator()(int i, int j = 0) { return d[i * C + j]; }
    __host__ __device__ const T& operator()(int i, int j = 0) const { return d[i * C + j]; }
    template <int r, int c>
    __host__ __device__ kmat<T, r, c> block(int i, int j) const {
        kmat<T, r, c> m;
        for (int a = 0; a < r; ++a)
            for (int b = 0; b < c; ++b) m(a, b) = (*this)(i + a, j + b);
        return m;
    }
    __host__ __device__ kmat<T, R, 1> col(int j) const {
        kmat<T, R, 1> m;
        for (int a = 0; a < R; ++a) m(a, 0) = (*this)(a, j);
        return m;
    }
    __host__ __device__ kmat<T, C, R> transpose() const {
        kmat<T, C, R> m;
        for (int a = 0; a < R; ++a)
            for (int b = 0; b < C; ++b) m(b, a) = (*this)(a, b);
        return m;
    }
    template <int r, int c>
    __host__ __device__ void assignBlock(int i, int j, const kmat<T, r, c>& m) {
        for (int a = 0; a < r; ++a)
            for (int b = 0; b < c; ++b) (*this)(i + a, j + b) = m(a, b);
    }
    __host__ __device__ T sqrNorm() const {
        static_assert(C == 1 && R == 2, "2-vectors only");
#ifdef RSFM_SHIM_KMAT_MATCH
        return __fmaf_rn(d[0], d[0], __fmul_rn(d[1], d[1]));
#else
        return d[0] * d[0] + d[1] * d[1];
#endif
    }
};

// A 2x2 matrix times a 2-vector, kept unevaluated so that "A * l + t" is evaluated as one
// expression (in the B200 kernel's order in the matching mode).
template <typename T>
struct kmat_mv2 {
    kmat<T, 2, 2> a;
    kmat<T, 2, 1> v;
    __host__ __device__ operator kmat<T, 2, 1>() const {
        kmat<T, 2, 1> r;
        for (int i = 0; i < 2; ++i) r(i) = a(i, 0) * v(0) + a(i, 1) * v(1);
        return r;
    }
};
template <typename T>
__host__ __device__ kmat_mv2<T> operator*(const kmat<T, 2, 2>& a, const kmat<T, 2, 1>& v) {
    return kmat_mv2<T>{a, v};
}
template <typename T>
__host__ __device__ kmat<T, 2, 1> operator+(const kmat_mv2<T>& e, const kmat<T, 2, 1>& t) {
    kmat<T, 2, 1> r;
    for (int i = 0; i < 2; ++i) {
#ifdef RSFM_SHIM_KMAT_MATCH
        r(i) = __fmaf_rn(e.a(i, 0), e.v(0), __fmaf_rn(e.a(i, 1), e.v(1), t(i)));
#else
        r(i) = (e.a(i, 0) * e.v(0) + e.a(i, 1) * e.v(1)) + t(i);
#endif
    }
    return r;
}
template <typename T, int R, int C>
__host__ __device__ kmat<T, R, C> operator-(const kmat<T, R, C>& x, const kmat<T, R, C>& y) {
    kmat<T, R, C> r;
    for (int i = 0; i < R * C; ++i) {
#ifdef RSFM_SHIM_KMAT_MATCH
        r.d[i] = __fsub_rn(x.d[i], y.d[i]);
#else
        r.d[i] = x.d[i] - y.d[i];
#endif
    }
    return r;
}

// A X = B for a 3x3 A and 3x2 B by Gaussian elimination with partial pivoting (rows swapped when a
// later row's pivot column entry is strictly larger in magnitude), then back substitution.
#ifdef RSFM_SHIM_KMAT_MATCH
__device__ inline kmat<float, 3, 2> solveGaussElim(
#else
__host__ __device__ inline kmat<float, 3, 2> solveGaussElim(
#endif
    const kmat<float, 3, 3>& A, const kmat<float, 3, 2>& B) {
    float m[3][5];
    for (int i = 0; i < 3; ++i) {
        for (int k = 0; k < 3; ++k) m[i][k] = A(i, k);
        m[i][3] = B(i, 0);
        m[i][4] = B(i, 1);
    }
    for (int c = 0; c < 3; ++c) {
        int piv = c;
        for (int r = c + 1; r < 3; ++r)
            if (fabsf(m[r][c]) > fabsf(m[piv][c])) piv = r;
        if (piv != c)
            for (int k = 0; k < 5; ++k) {
                const float x = m[c][k];
                m[c][k] = m[piv][k];
                m[piv][k] = x;
            }
        for (int r = c + 1; r < 3; ++r) {
#ifdef RSFM_SHIM_KMAT_MATCH
            const float f = __fdiv_rn(m[r][c], m[c][c]);
            for (int k = c; k < 5; ++k) m[r][k] = __fsub_rn(m[r][k], __fmul_rn(f, m[c][k]));
#else
            const float f = m[r][c] / m[c][c];
            for (int k = c; k < 5; ++k) m[r][k] = m[r][k] - f * m[c][k];
#endif
        }
    }
    kmat<float, 3, 2> X;
    for (int r = 2; r >= 0; --r)
        for (int h = 0; h < 2; ++h) {
            float v = m[r][3 + h];
            for (int k = r + 1; k < 3; ++k) {
#ifdef RSFM_SHIM_KMAT_MATCH
                v = __fsub_rn(v, __fmul_rn(m[r][k], X(k, h)));
#else
                v = v - m[r][k] * X(k, h);
#endif
            }
#ifdef RSFM_SHIM_KMAT_MATCH
            X(r, h) = __fdiv_rn(v, m[r][r]);
#else
            X(r, h) = v / m[r][r];
#endif
        }
    return X;
}
