// Project-written stand-in for the aarand library (random distributions over a
// C++ engine), which the reference fetches at configure time and is not vendored.  The distributions are written from
// their textbook definitions; the streams therefore differ from upstream
// aarand, which is why layouts are compared by quality metrics rather than
// bit-for-bit against upstream umappp.  oracle/oracle.c draws from the same
// definitions so that the C restatement and the compiled reference agree
// exactly.
//
// Test infrastructure only.
#ifndef ORACLE_SHIM_AARAND_HPP
#define ORACLE_SHIM_AARAND_HPP

#include <cmath>
#include <cstdint>
#include <utility>

namespace aarand {

// Uniform on [0, 1): the top 53 bits of one 64-bit draw, scaled by 2^-53.
// For float, the double is rounded and a result of exactly 1 is redrawn.
template<typename Float_ = double, class Engine_>
Float_ standard_uniform(Engine_& eng) {
    while (true) {
        const uint64_t raw = static_cast<uint64_t>(eng() - Engine_::min());
        const double u = static_cast<double>(raw >> 11) * 0x1.0p-53;
        const Float_ out = static_cast<Float_>(u);
        if (out < static_cast<Float_>(1)) {
            return out;
        }
    }
}

// Exactly uniform integer in [0, bound) by rejection: draws r from the 64-bit
// engine and accepts r < limit, the largest multiple of 'bound' not above
// 2^64; the result is r % bound.
template<class Engine_, typename Int_>
Int_ discrete_uniform(Engine_& eng, Int_ bound) {
    const uint64_t b = static_cast<uint64_t>(bound);
    const uint64_t limit = UINT64_MAX - (UINT64_MAX % b + 1) % b; // accept r <= limit
    while (true) {
        const uint64_t r = static_cast<uint64_t>(eng() - Engine_::min());
        if (r <= limit) {
            return static_cast<Int_>(r % b);
        }
    }
}

// A pair of independent standard normals by the Box-Muller transform on two
// uniforms, the first of which is redrawn while it is zero.
template<typename Float_ = double, class Engine_>
std::pair<Float_, Float_> standard_normal(Engine_& eng) {
    constexpr double two_pi = 6.283185307179586476925286766559;
    double u1;
    do {
        u1 = standard_uniform<double>(eng);
    } while (u1 == 0);
    const double u2 = standard_uniform<double>(eng);
    const double r = std::sqrt(-2.0 * std::log(u1));
    const double theta = two_pi * u2;
    return std::make_pair(static_cast<Float_>(r * std::cos(theta)), static_cast<Float_>(r * std::sin(theta)));
}

}

#endif
