// Forward-mode dual numbers (value + N directional derivatives) for the adjoint kernels.
//
// The return map's principal-space function sigma -> (exp(eps_c), tau_c) is a chain of a few dozen
// scalar operations plus one implicit scalar solve; carrying N tangents through it gives its
// Jacobian with respect to the three singular values and the material parameters in one pass.
#pragma once

#include <cuda_runtime.h>

namespace bk {

template <int N>
struct Dual {
    float v;
    float d[N];
    __device__ __forceinline__ Dual() : v(0.f) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.f;
    }
    __device__ __forceinline__ Dual(float value) : v(value) {  // NOLINT: constants promote implicitly
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.f;
    }
    __device__ __forceinline__ static Dual seed(float value, int direction) {
        Dual r(value);
        r.d[direction] = 1.f;
        return r;
    }
};

#define BK_DUAL_BINARY(op, value_expr, deriv_expr)                                        \
    template <int N>                                                                       \
    __device__ __forceinline__ Dual<N> operator op(const Dual<N>& a, const Dual<N>& b) {   \
        Dual<N> r;                                                                         \
        r.v = value_expr;                                                                  \
        _Pragma("unroll") for (int k = 0; k < N; ++k) r.d[k] = deriv_expr;                 \
        return r;                                                                          \
    }

BK_DUAL_BINARY(+, a.v + b.v, a.d[k] + b.d[k])
BK_DUAL_BINARY(-, a.v - b.v, a.d[k] - b.d[k])
BK_DUAL_BINARY(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
#undef BK_DUAL_BINARY

template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    float inv = 1.f / b.v;
    r.v = a.v * inv;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> scale(const Dual<N>& a, float s) {
    Dual<N> r;
    r.v = a.v * s;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * s;
    return r;
}

// Apply a scalar function with value f and derivative df at a.v.
template <int N>
__device__ __forceinline__ Dual<N> chain(const Dual<N>& a, float f, float df) {
    Dual<N> r;
    r.v = f;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = df * a.d[k];
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> dlog(const Dual<N>& a) { return chain(a, logf(a.v), 1.f / a.v); }

template <int N>
__device__ __forceinline__ Dual<N> dexp(const Dual<N>& a) {
    float e = expf(a.v);
    return chain(a, e, e);
}

template <int N>
__device__ __forceinline__ Dual<N> dcbrt(const Dual<N>& a) {
    float c = cbrtf(a.v);
    return chain(a, c, c / (3.f * a.v));
}

}  // namespace bk
