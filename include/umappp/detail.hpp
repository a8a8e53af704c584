#ifndef UMAPPP_DETAIL_HPP
#define UMAPPP_DETAIL_HPP

/**
 * @file detail.hpp
 * @brief Marshalling between the C++ drop-in headers and the C ABI (umapb.h).
 */

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../umapb.h"
#include "NeighborList.hpp"
#include "Options.hpp"

namespace umappp {
namespace detail {

template <typename Float_>
constexpr int dtype() {
    static_assert(std::is_same<Float_, float>::value || std::is_same<Float_, double>::value,
                  "Float_ must be float or double");
    return std::is_same<Float_, double>::value ? UMAPB_F64 : UMAPB_F32;
}

/** Throws the reference's exception types for a failing C-ABI call. */
inline void check(int rc) {
    if (rc == UMAPB_OK) return;
    const std::string msg = umapb_last_error();
    if (rc == UMAPB_ERR_OVERFLOW) throw std::overflow_error(msg);
    throw std::runtime_error(msg);
}

inline umapb_options to_c(const Options& o) {
    umapb_options c;
    umapb_options_init(&c);
    c.local_connectivity = o.local_connectivity;
    c.bandwidth = o.bandwidth;
    c.mix_ratio = o.mix_ratio;
    c.spread = o.spread;
    c.min_dist = o.min_dist;
    c.has_a = o.a.has_value();
    c.a = o.a.value_or(0);
    c.has_b = o.b.has_value();
    c.b = o.b.value_or(0);
    c.repulsion_strength = o.repulsion_strength;
    c.initialize_method = static_cast<int>(o.initialize_method);
    c.initialize_random_on_spectral_fail = o.initialize_random_on_spectral_fail;
    c.irlba_extra_work = o.initialize_spectral_irlba_options.extra_work;
    c.irlba_max_iterations = o.initialize_spectral_irlba_options.max_iterations;
    c.irlba_convergence_tolerance = o.initialize_spectral_irlba_options.convergence_tolerance;
    c.initialize_spectral_scale = o.initialize_spectral_scale;
    c.initialize_spectral_jitter = o.initialize_spectral_jitter;
    c.initialize_spectral_jitter_sd = o.initialize_spectral_jitter_sd;
    c.initialize_random_scale = o.initialize_random_scale;
    c.initialize_seed = o.initialize_seed;
    c.has_num_epochs = o.num_epochs.has_value();
    c.num_epochs = o.num_epochs.value_or(0);
    c.learning_rate = o.learning_rate;
    c.negative_sample_rate = o.negative_sample_rate;
    c.num_neighbors = o.num_neighbors;
    c.optimize_seed = o.optimize_seed;
    c.num_threads = o.num_threads;
    c.num_threads_spectral = o.num_threads_spectral;
    c.num_threads_optimize = o.num_threads_optimize;
    return c;
}

/** A NeighborList flattened to CSR (int64 row pointers, int32 indices). */
template <typename Float_>
struct Csr {
    std::vector<int64_t> ptr;
    std::vector<int32_t> idx;
    std::vector<Float_> val;
};

template <typename Index_, typename Float_>
Csr<Float_> to_csr(const NeighborList<Index_, Float_>& x) {
    Csr<Float_> out;
    out.ptr.resize(x.size() + 1);
    out.ptr[0] = 0;
    for (size_t i = 0; i < x.size(); ++i) out.ptr[i + 1] = out.ptr[i] + static_cast<int64_t>(x[i].size());
    out.idx.reserve(out.ptr.back());
    out.val.reserve(out.ptr.back());
    for (const auto& row : x) {
        for (const auto& e : row) {
            if (static_cast<long long>(e.first) > INT32_MAX || static_cast<long long>(e.first) < 0) {
                throw std::overflow_error("neighbour index does not fit the 32-bit device index");
            }
            out.idx.push_back(static_cast<int32_t>(e.first));
            out.val.push_back(e.second);
        }
    }
    return out;
}

template <typename Index_, typename Float_>
NeighborList<Index_, Float_> from_csr(const std::vector<int64_t>& ptr, const std::vector<int32_t>& idx,
                                      const std::vector<Float_>& val) {
    NeighborList<Index_, Float_> out(ptr.empty() ? 0 : ptr.size() - 1);
    for (size_t i = 0; i + 1 < ptr.size(); ++i) {
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) out[i].emplace_back(static_cast<Index_>(idx[p]), val[p]);
    }
    return out;
}

}  // namespace detail
}  // namespace umappp

#endif
