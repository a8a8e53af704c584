#ifndef UMAPPP_STAGES_HPP
#define UMAPPP_STAGES_HPP

/**
 * @file stages.hpp
 * @brief The reference's stage functions, run on the GPU (drop-ins for
 * libscran/umappp include/umappp/{neighbor_similarities,combine_neighbor_sets,
 * spectral_init,find_ab,optimize_layout}.hpp).  Each takes and returns host
 * containers like the reference's.
 */

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <utility>
#include <vector>

#include "Status.hpp"
#include "detail.hpp"

namespace umappp {

/** neighbor_similarities options (neighbor_similarities.hpp:38-44). */
template <typename Float_>
struct NeighborSimilaritiesOptions {
    Float_ local_connectivity = 1.0;
    Float_ bandwidth = 1.0;
    Float_ min_k_dist_scale = 1e-3;
    int num_threads = 1;
};

/** neighbor_similarities (neighbor_similarities.hpp:46-207): distances -> weights in place. */
template <bool use_newton_ = true, typename Index_, typename Float_>
void neighbor_similarities(NeighborList<Index_, Float_>& x, const NeighborSimilaritiesOptions<Float_>& options) {
    auto csr = detail::to_csr(x);
    detail::check(umapb_neighbor_similarities(detail::dtype<Float_>(), static_cast<int32_t>(x.size()), csr.ptr.data(),
                                              csr.val.data(), options.local_connectivity, options.bandwidth,
                                              options.min_k_dist_scale, use_newton_ ? 1 : 0, nullptr, nullptr));
    size_t t = 0;
    for (auto& row : x)
        for (auto& e : row) e.second = csr.val[t++];
}

/** combine_neighbor_sets (combine_neighbor_sets.hpp:16-99). */
template <typename Index_, typename Float_>
void combine_neighbor_sets(NeighborList<Index_, Float_>& x, const Float_ mix_ratio) {
    const auto csr = detail::to_csr(x);
    const int64_t cap = 2 * static_cast<int64_t>(csr.idx.size()) + 1;
    std::vector<int64_t> ptr(x.size() + 1);
    std::vector<int32_t> idx(cap);
    std::vector<Float_> val(cap);
    int64_t nnz = 0;
    detail::check(umapb_combine_neighbor_sets(detail::dtype<Float_>(), static_cast<int32_t>(x.size()), csr.ptr.data(),
                                              csr.idx.data(), csr.val.data(), mix_ratio, ptr.data(), idx.data(),
                                              val.data(), cap, &nnz));
    x = detail::from_csr<Index_, Float_>(ptr, idx, val);
}

/** has_multiple_components (spectral_init.hpp:142-168). */
template <typename Index_, typename Float_>
bool has_multiple_components(const NeighborList<Index_, Float_>& edges) {
    const auto csr = detail::to_csr(edges);
    int out = 0;
    detail::check(umapb_has_multiple_components(static_cast<int32_t>(edges.size()), csr.ptr.data(), csr.idx.data(), &out));
    return out != 0;
}

/** spectral_init (spectral_init.hpp:170-207). */
template <typename Index_, typename Float_>
bool spectral_init(const NeighborList<Index_, Float_>& edges, const std::size_t num_dim, Float_* const vals,
                   const IrlbaOptions& irlba_opt, int /*nthreads*/, double scale, bool jitter, double jitter_sd,
                   RngEngine::result_type seed) {
    const auto csr = detail::to_csr(edges);
    int ok = 0;
    detail::check(umapb_spectral_init(detail::dtype<Float_>(), static_cast<int32_t>(edges.size()), csr.ptr.data(),
                                      csr.idx.data(), csr.val.data(), num_dim, vals, irlba_opt.extra_work,
                                      irlba_opt.max_iterations, irlba_opt.convergence_tolerance, scale, jitter ? 1 : 0,
                                      jitter_sd, seed, &ok, nullptr));
    return ok != 0;
}

/** random_init (spectral_init.hpp:209-225). */
template <typename Index_, typename Float_>
void random_init(const Index_ num_obs, const std::size_t num_dim, Float_* const vals, RngEngine::result_type seed,
                 double scale) {
    detail::check(umapb_random_init(detail::dtype<Float_>(), static_cast<int32_t>(num_obs), num_dim, vals, seed, scale));
}

/** find_ab (find_ab.hpp:44-168). */
template <typename Float_>
std::pair<Float_, Float_> find_ab(const Float_ spread, const Float_ min_dist) {
    double a = 0, b = 0;
    detail::check(umapb_find_ab(spread, min_dist, &a, &b));
    return std::make_pair(static_cast<Float_>(a), static_cast<Float_>(b));
}

/** similarities_to_epochs (optimize_layout.hpp:47-92). */
template <typename Index_, typename Float_>
EpochData<Index_, Float_> similarities_to_epochs(const NeighborList<Index_, Float_>& p, const int num_epochs,
                                                 const Float_ negative_sample_rate) {
    const auto csr = detail::to_csr(p);
    const size_t cap = csr.idx.size() + 1;
    std::vector<int64_t> ptr(p.size() + 1);
    std::vector<int32_t> targets(cap);
    EpochData<Index_, Float_> out;
    out.epochs_per_sample.resize(cap);
    out.epoch_of_next_sample.resize(cap);
    out.epoch_of_next_negative_sample.resize(cap);
    int64_t nnz = 0;
    detail::check(umapb_similarities_to_epochs(detail::dtype<Float_>(), static_cast<int32_t>(p.size()), csr.ptr.data(),
                                               csr.idx.data(), csr.val.data(), num_epochs, negative_sample_rate,
                                               ptr.data(), targets.data(), out.epochs_per_sample.data(),
                                               out.epoch_of_next_sample.data(), out.epoch_of_next_negative_sample.data(),
                                               &nnz));
    out.cumulative_num_edges.assign(ptr.begin(), ptr.end());
    out.edge_targets.assign(targets.begin(), targets.begin() + nnz);
    out.epochs_per_sample.resize(nnz);
    out.epoch_of_next_sample.resize(nnz);
    out.epoch_of_next_negative_sample.resize(nnz);
    out.total_epochs = num_epochs;
    out.negative_sample_rate = negative_sample_rate;
    return out;
}

/**
 * optimize_layout (optimize_layout.hpp:116-185) on the GPU.  The reference's
 * engine argument is replaced by a seed: negative samples come from a
 * counter-based generator keyed by (seed, epoch, edge).
 */
template <typename Index_, typename Float_>
void optimize_layout(std::size_t num_dim, Float_* embedding, EpochData<Index_, Float_>& setup, Float_ a, Float_ b,
                     Float_ gamma, Float_ initial_alpha, uint64_t seed, int epoch_limit) {
    std::vector<int64_t> ptr(setup.cumulative_num_edges.begin(), setup.cumulative_num_edges.end());
    std::vector<int32_t> targets(setup.edge_targets.begin(), setup.edge_targets.end());
    const int32_t n = static_cast<int32_t>(ptr.size()) - 1;
    detail::check(umapb_optimize_layout(detail::dtype<Float_>(), num_dim, embedding, n, ptr.data(), targets.data(),
                                        setup.epochs_per_sample.data(), setup.epoch_of_next_sample.data(),
                                        setup.epoch_of_next_negative_sample.data(), setup.negative_sample_rate,
                                        setup.total_epochs, &setup.current_epoch, a, b, gamma, initial_alpha, seed,
                                        epoch_limit));
}

}  // namespace umappp

#endif
