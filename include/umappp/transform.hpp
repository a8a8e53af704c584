#ifndef UMAPPP_TRANSFORM_HPP
#define UMAPPP_TRANSFORM_HPP

/**
 * @file transform.hpp
 * @brief Out-of-sample embedding: an extension, the reference has no transform.
 *
 * transform() places new points in a finished layout of reference points
 * (umapb_transform): each new point's nearest reference points and their
 * similarities (neighbor_similarities.hpp), a start at the
 * similarity-weighted mean of those points' positions, then the per-row steps
 * of optimize_layout (optimize_layout.hpp:136-180) with only the new points
 * moving and negative samples drawn among the reference points, at a quarter
 * of Options::learning_rate.  Options::num_neighbors, local_connectivity,
 * bandwidth, a/b (or spread/min_dist), repulsion_strength,
 * negative_sample_rate and optimize_seed apply.  Pointers may be host or
 * device memory; all arrays are row-major (one observation per row).
 */

#include <cstddef>
#include <optional>

#include "Options.hpp"
#include "detail.hpp"

namespace umappp {

/**
 * @param data_dim     columns of the data
 * @param num_ref      reference points
 * @param ref_data     num_ref x data_dim
 * @param num_dim      columns of the embedding
 * @param ref_embedding num_ref x num_dim, the finished layout (not changed)
 * @param num_new      new points
 * @param new_data     num_new x data_dim
 * @param new_embedding receives num_new x num_dim
 * @param num_epochs   epochs (unset: a third of Options::num_epochs when that
 *                     is set, else 100 up to 10,000 new points and 30 above)
 */
template <typename Index_, typename Float_>
void transform(const std::size_t data_dim, const Index_ num_ref, const Float_* const ref_data,
               const std::size_t num_dim, const Float_* const ref_embedding, const Index_ num_new,
               const Float_* const new_data, Float_* const new_embedding, const Options& options,
               const std::optional<int> num_epochs = std::nullopt) {
    const auto copt = detail::to_c(options);
    detail::check(umapb_transform(detail::dtype<Float_>(), data_dim, static_cast<int32_t>(num_ref), ref_data,
                                  ref_embedding, static_cast<int32_t>(num_new), new_data, num_dim, &copt,
                                  num_epochs.value_or(0), new_embedding));
}

}  // namespace umappp

#endif
