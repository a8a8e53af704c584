// Correctly rounded FP64 exp for the device, so that weights computed on the
// GPU equal those of a host libm whose exp rounds correctly (the reference
// computes them with std::exp, include/umappp/neighbor_similarities.hpp:139,198).
//
// Method (Tang-style table-free reduction evaluated in double-double
// arithmetic; Dekker 1971 / Shewchuk 1997 error-free transformations):
//   x = k ln2 + r,   k = nearest integer to x / ln2,   |r| <= ln2 / 2,
//   with ln2 held as a triple of doubles (the first two with trailing zero
//   bits, so k * ln2_hi and k * ln2_mid are exact for |k| < 2^11);
//   r is scaled by 2^-10, exp of the scaled value is a degree-9 Taylor
//   polynomial in double-double (truncation < 2^-110), then squared 10 times
//   in double-double; finally exp(x) = 2^k * (hi + lo), with hi + lo rounded
//   once to double.  The double-double result carries ~100 correct bits, so
//   the final rounding is correct except for inputs whose exp lies within
//   ~2^-100 relative of a rounding midpoint.
// Domain: results that are normal doubles; below that the result goes through
// ldexp (rounded twice), and overflow / underflow give inf / 0.
#pragma once

#include <math_constants.h>

namespace umapb {

struct DD {
    double hi, lo;
};

__device__ __forceinline__ DD dd_two_sum(double a, double b) {
    const double s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    const double e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
    return DD{s, e};
}

__device__ __forceinline__ DD dd_fast_two_sum(double a, double b) {
    const double s = __dadd_rn(a, b);
    return DD{s, __dsub_rn(b, __dsub_rn(s, a))};
}

__device__ __forceinline__ DD dd_add(DD a, DD b) {
    DD s = dd_two_sum(a.hi, b.hi);
    const double t = __dadd_rn(__dadd_rn(a.lo, b.lo), s.lo);
    return dd_fast_two_sum(s.hi, t);
}

__device__ __forceinline__ DD dd_mul(DD a, DD b) {
    const double p = __dmul_rn(a.hi, b.hi);
    const double e = fma(a.hi, b.hi, -p);               // exact low part of the product
    const double t = fma(a.hi, b.lo, fma(a.lo, b.hi, e));
    return dd_fast_two_sum(p, t);
}

__device__ __forceinline__ DD dd_mul_d(DD a, double b) {
    const double p = __dmul_rn(a.hi, b);
    const double e = fma(a.hi, b, -p);
    return dd_fast_two_sum(p, fma(a.lo, b, e));
}

__device__ __forceinline__ double exp_cr(double x) {
    if (!(x == x)) return x;                              // NaN
    if (x > 709.782712893384) return CUDART_INF;
    if (x < -745.2) return 0.0;
    // ln 2 = L1 + L2 + L3 (to 2^-143); L1 and L2 carry 42 significant bits, so
    // k L1 and k L2 are exact for |k| < 2^11
    const double L1 = 0x1.62e42fefa3800p-1;
    const double L2 = 0x1.ef35793c76800p-45;
    const double L3 = -0x1.9ff0342542fc3p-90;
    const double inv_ln2 = 0x1.71547652b82fep+0;
    const double kd = rint(__dmul_rn(x, inv_ln2));
    const int k = static_cast<int>(kd);
    // r = x - k L1 - k L2 - k L3 in double-double
    DD r = dd_two_sum(x, -__dmul_rn(kd, L1));
    r = dd_add(r, DD{-__dmul_rn(kd, L2), 0.0});
    {
        const double p3 = __dmul_rn(kd, L3);
        r = dd_add(r, DD{-p3, -fma(kd, L3, -p3)});
    }
    // scale by 2^-10 (exact)
    r.hi = ldexp(r.hi, -10);
    r.lo = ldexp(r.lo, -10);
    // Taylor polynomial sum_{n=0..9} r^n / n!, Horner in double-double with the
    // coefficients 1/n! as double-double pairs (hi = fl(1/n!), lo = fl(1/n! - hi))
    const double c_hi[10] = {1.0, 1.0, 0.5, 0x1.5555555555555p-3, 0x1.5555555555555p-5, 0x1.1111111111111p-7,
                             0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-16,
                             0x1.71de3a556c734p-19};
    const double c_lo[10] = {0.0, 0.0, 0.0, 0x1.5555555555555p-57, 0x1.5555555555555p-59, 0x1.1111111111111p-63,
                             -0x1.f49f49f49f49fp-65, 0x1.a01a01a01a01ap-73, 0x1.a01a01a01a01ap-76,
                             -0x1.c154f8ddc6c00p-73};
    DD p = DD{c_hi[9], c_lo[9]};
    for (int nn = 8; nn >= 0; --nn) p = dd_add(dd_mul(p, r), DD{c_hi[nn], c_lo[nn]});
    for (int i = 0; i < 10; ++i) p = dd_mul(p, p);
    // round hi + lo once, then scale by 2^k
    const double y = __dadd_rn(p.hi, p.lo);
    if (k > -1022) return ldexp(y, k);
    return ldexp(ldexp(y, 54), k - 54);
}

}  // namespace umapb
