#ifndef UMAPPP_EXTENSIONS_HPP
#define UMAPPP_EXTENSIONS_HPP

/**
 * @file extensions.hpp
 * @brief C++ forms of two entry points without a counterpart in the
 * reference: many independent runs in one call (umapb_batch_run), and the
 * loss and gradient of the UMAP fuzzy cross-entropy (umapb_loss_grad), whose
 * per-edge derivatives are the reference's step coefficients
 * (include/umappp/optimize_layout.hpp:148-149,171).  Pointers may be host or
 * device memory; arrays are row-major, one observation per row.
 */

#include <array>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "Options.hpp"
#include "detail.hpp"

namespace umappp {

/**
 * Many independent UMAP runs in one call: instance i is the next sizes[i]
 * observations of 'data' (data_dim values each) and of 'embedding' (num_dim
 * values each, overwritten with its final layout).  Each instance gets what
 * initialize(data, builder, ...) + Status::run() with 'options' gives it,
 * except that its negative samples come from another generator stream.  All
 * instances must resolve to the same epoch count (set Options::num_epochs
 * when their sizes straddle 10,000).  Returns the device milliseconds of the
 * stages: knn, similarities, union, init, epochs, schedule, sgd.
 */
template <typename Float_>
std::array<double, 7> batch_run(const std::vector<int32_t>& sizes, const std::size_t data_dim, const Float_* const data,
                                const std::size_t num_dim, Float_* const embedding, const Options& options) {
    const auto copt = detail::to_c(options);
    std::array<double, 7> ms{};
    detail::check(umapb_batch_run(detail::dtype<Float_>(), static_cast<int32_t>(sizes.size()), sizes.data(), data_dim,
                                  data, num_dim, embedding, &copt, ms.data()));
    return ms;
}

/** Loss and gradient of loss_grad(). */
template <typename Float_>
struct LossGrad {
    double loss = 0;
    std::vector<Float_> grad_embedding;   ///< num_obs x num_dim
    double grad_a = 0;                    ///< dL/da
    double grad_b = 0;                    ///< dL/db
};

/**
 * The fuzzy cross-entropy of a layout over a symmetric graph in CSR form
 * (row_ptr[num_obs + 1], indices and weights of the stored edges, as
 * combine_neighbor_sets returns them) and its gradient with respect to the
 * embedding, a and b:
 *   L = sum over stored edges (i -> j, w) of w (-log q) + (1 - w) (-log(1 - q))
 *       [+ w log w + (1 - w) log(1 - w) with with_constant],
 *   q = 1 / (1 + a d^(2b)), d = |y_i - y_j|,
 * accumulated in FP64.  eps_rep > 0 puts d^2 + eps_rep in the repulsive
 * derivative's denominator, as the reference's step does with 0.001.
 * Host arrays here; the result is returned on the host.
 */
template <typename Float_>
LossGrad<Float_> loss_grad(const std::size_t num_dim, const Float_* const embedding, const int32_t num_obs,
                           const int64_t* const row_ptr, const int32_t* const indices, const Float_* const weights,
                           const double a, const double b, const double eps_rep = 0.0,
                           const bool with_constant = false) {
    LossGrad<Float_> out;
    out.grad_embedding.resize(static_cast<std::size_t>(num_obs) * num_dim);
    double ab[2] = {0, 0};
    detail::check(umapb_loss_grad(detail::dtype<Float_>(), num_dim, embedding, num_obs, row_ptr, indices, weights, a, b,
                                  eps_rep, with_constant ? 1 : 0, &out.loss, out.grad_embedding.data(), ab));
    out.grad_a = ab[0];
    out.grad_b = ab[1];
    return out;
}

}  // namespace umappp

#endif
