// Project-written stand-in for the sanisizer library (overflow-checked size
// arithmetic), which the reference fetches at configure time and which is
// absent here.  Only the calls made by the reference headers are provided,
// written from their call sites: each checks for overflow and throws
// std::overflow_error, the "_unsafe" variants skip the check.
//
// Test infrastructure only: used to compile the reference headers into
// oracle/_ref for parity pinning and the CPU baseline.
#ifndef ORACLE_SHIM_SANISIZER_HPP
#define ORACLE_SHIM_SANISIZER_HPP

#include <cmath>
#include <cstddef>
#include <limits>
#include <stdexcept>
#include <type_traits>

namespace sanisizer {

template<typename Out_, typename In_>
constexpr Out_ cap(In_ x) {
    if (static_cast<unsigned long long>(x) > static_cast<unsigned long long>(std::numeric_limits<Out_>::max())) {
        return std::numeric_limits<Out_>::max();
    }
    return static_cast<Out_>(x);
}

template<typename Out_, typename In_>
Out_ checked_cast(In_ x) {
    if constexpr (std::is_signed<In_>::value) {
        if (x < 0) {
            throw std::overflow_error("negative size");
        }
    }
    if (static_cast<unsigned long long>(x) > static_cast<unsigned long long>(std::numeric_limits<Out_>::max())) {
        throw std::overflow_error("size does not fit in the target type");
    }
    return static_cast<Out_>(x);
}

template<typename Out_, typename A_, typename B_>
Out_ sum(A_ a, B_ b) {
    Out_ x = checked_cast<Out_>(a);
    Out_ y = checked_cast<Out_>(b);
    if (x > std::numeric_limits<Out_>::max() - y) {
        throw std::overflow_error("overflow in size sum");
    }
    return x + y;
}

template<typename Out_, typename A_, typename B_>
Out_ sum_unsafe(A_ a, B_ b) {
    return static_cast<Out_>(a) + static_cast<Out_>(b);
}

template<typename Out_, typename A_, typename B_>
Out_ product(A_ a, B_ b) {
    Out_ x = checked_cast<Out_>(a);
    Out_ y = checked_cast<Out_>(b);
    if (y != 0 && x > std::numeric_limits<Out_>::max() / y) {
        throw std::overflow_error("overflow in size product");
    }
    return x * y;
}

template<typename Out_, typename A_, typename B_>
Out_ product_unsafe(A_ a, B_ b) {
    return static_cast<Out_>(a) * static_cast<Out_>(b);
}

// Offset of element (d, c) in a column-major array with 'num_dim' rows.
template<typename Out_, typename D_, typename N_, typename C_>
Out_ nd_offset(D_ d, N_ num_dim, C_ c) {
    return static_cast<Out_>(d) + static_cast<Out_>(num_dim) * static_cast<Out_>(c);
}

template<class Container_, typename N_>
Container_ create(N_ n) {
    return Container_(checked_cast<typename Container_::size_type>(n));
}

template<typename Out_, typename Float_>
Out_ from_float(Float_ x) {
    if (!std::isfinite(x)) {
        throw std::overflow_error("non-finite value cannot be cast to an integer");
    }
    const Float_ t = std::trunc(x);
    if (t < static_cast<Float_>(std::numeric_limits<Out_>::min()) || t > static_cast<Float_>(std::numeric_limits<Out_>::max())) {
        throw std::overflow_error("floating-point value does not fit in the integer type");
    }
    return static_cast<Out_>(t);
}

template<typename A_, typename B_>
bool is_less_than_or_equal(A_ a, B_ b) {
    if constexpr (std::is_signed<A_>::value) {
        if (a < 0) {
            return true;
        }
    }
    if constexpr (std::is_signed<B_>::value) {
        if (b < 0) {
            return false;
        }
    }
    return static_cast<unsigned long long>(a) <= static_cast<unsigned long long>(b);
}

}

#endif
