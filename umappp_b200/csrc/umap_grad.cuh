// Derivatives of the UMAP fuzzy cross-entropy along one edge, shared by the
// adjoint (adjoint.cu) and the SGD epochs (sgd.cu).
//
// For an edge with squared embedding distance d2 and q = 1 / (1 + a d2^b):
//   dA/dd2 =  a b d2^(b-1) / (1 + a d2^b)          A = -log q          (attractive term)
//   dR/dd2 = -b / ((d2 + eps) (1 + a d2^b))        R = -log(1 - q)     (repulsive term, with
//                                                  d2 -> d2 + eps in its 1/d2 factor)
// The reference's SGD step on an edge (include/umappp/optimize_layout.hpp)
// moves the head by alpha clamp(coef (y_i - y_j)) with
//   attractive coef = -2 a b d2^b / (d2 (a d2^b + 1))          (:147-149)  = -2 dA/dd2
//   repulsive  coef = 2 gamma b / ((0.001 + d2) (a d2^b + 1))  (:170-171)  = -2 gamma dR/dd2 (eps = 0.001)
// Both are written here once, with the factor in front folded into the
// numerator: attract_dd2(d2, a, b, s a b) = s dA/dd2, repulse_dd2(d2, a, b, -s b,
// eps) = s dR/dd2.  FAST selects __powf, __fdividef and a fused a d2^b + 1 (FP32
// layouts, where the step is stochastic and clamped) over pow, IEEE division
// and separately rounded operations.
#pragma once

namespace umapb {

__device__ __forceinline__ float grad_pow(float x, float b, bool fast) { return fast ? __powf(x, b) : powf(x, b); }
__device__ __forceinline__ double grad_pow(double x, double b, bool) { return pow(x, b); }
__device__ __forceinline__ float grad_div(float x, float y, bool fast) { return fast ? __fdividef(x, y) : x / y; }
__device__ __forceinline__ double grad_div(double x, double y, bool) { return x / y; }
// a x + 1: one fused multiply-add on the FAST path, separately rounded otherwise
__device__ __forceinline__ float grad_ax1(float a, float x, bool fast) { return fast ? __fmaf_rn(a, x, 1.0f) : a * x + 1.0f; }
__device__ __forceinline__ double grad_ax1(double a, double x, bool) { return a * x + 1.0; }

// s dA/dd2, with sab = s a b.
template <bool FAST, typename T>
__device__ __forceinline__ T attract_dd2(T d2, T a, T b, T sab) {
    const T pd2b = grad_pow(d2, b, FAST);
    return grad_div(sab * pd2b, d2 * grad_ax1(a, pd2b, FAST), FAST);
}

// s dR/dd2, with msb = -s b.
template <bool FAST, typename T>
__device__ __forceinline__ T repulse_dd2(T d2, T a, T b, T msb, T eps) {
    return grad_div(msb, (eps + d2) * grad_ax1(a, grad_pow(d2, b, FAST), FAST), FAST);
}

}  // namespace umapb
