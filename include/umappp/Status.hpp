#ifndef UMAPPP_STATUS_HPP
#define UMAPPP_STATUS_HPP

/**
 * @file Status.hpp
 * @brief Status of the UMAP optimisation (drop-in for libscran/umappp
 * include/umappp/Status.hpp:25-141).  The optimisation state lives on the GPU;
 * run() reads the caller's embedding, advances the epochs on the device and
 * writes the embedding back, so the caller's array stays the state as in the
 * reference.
 */

#include <cstddef>
#include <memory>
#include <vector>

#include "detail.hpp"

namespace umappp {

/** The reference's EpochData (include/umappp/optimize_layout.hpp:27-45), by value. */
template <typename Index_, typename Float_>
struct EpochData {
    int total_epochs = 0;
    int current_epoch = 0;
    std::vector<std::size_t> cumulative_num_edges;
    std::vector<Index_> edge_targets;
    std::vector<Float_> epochs_per_sample;
    std::vector<Float_> epoch_of_next_sample;
    std::vector<Float_> epoch_of_next_negative_sample;
    Float_ negative_sample_rate = 0;
};

template <typename Index_, typename Float_>
class Status {
public:
    /** @cond */
    Status(umapb_status* handle, double negative_sample_rate)
        : my_handle(handle, &umapb_status_free), my_rate(negative_sample_rate) {}
    /** @endcond */

    /** Status::num_dimensions() (Status.hpp:63-65). */
    std::size_t num_dimensions() const { return umapb_status_num_dimensions(my_handle.get()); }
    /** Status::epoch() (Status.hpp:70-72): epochs completed so far. */
    int epoch() const { return umapb_status_epoch(my_handle.get()); }
    /** Status::num_epochs() (Status.hpp:78-80). */
    int num_epochs() const { return umapb_status_num_epochs(my_handle.get()); }
    /** Status::num_observations() (Status.hpp:85-87). */
    Index_ num_observations() const { return static_cast<Index_>(umapb_status_num_observations(my_handle.get())); }

    /** Status::run(embedding, epoch_limit) (Status.hpp:101-128): advances to epoch_limit. */
    void run(Float_* const embedding, int epoch_limit) {
        detail::check(umapb_status_run(my_handle.get(), embedding, epoch_limit));
    }

    /** Status::run(embedding) (Status.hpp:138-140): advances to num_epochs(). */
    void run(Float_* const embedding) { run(embedding, num_epochs()); }

    /** The schedule at the current epoch (a copy; the reference returns a reference). */
    EpochData<Index_, Float_> get_epoch_data() const {
        EpochData<Index_, Float_> out;
        const auto n = static_cast<std::size_t>(num_observations());
        const auto nnz = static_cast<std::size_t>(umapb_status_num_edges(my_handle.get()));
        std::vector<int64_t> ptr(n + 1);
        std::vector<int32_t> targets(nnz);
        out.epochs_per_sample.resize(nnz);
        out.epoch_of_next_sample.resize(nnz);
        out.epoch_of_next_negative_sample.resize(nnz);
        detail::check(umapb_status_get_epoch_data(my_handle.get(), ptr.data(), targets.data(), out.epochs_per_sample.data(),
                                                  out.epoch_of_next_sample.data(),
                                                  out.epoch_of_next_negative_sample.data()));
        out.cumulative_num_edges.assign(ptr.begin(), ptr.end());
        out.edge_targets.assign(targets.begin(), targets.end());
        out.total_epochs = num_epochs();
        out.current_epoch = epoch();
        out.negative_sample_rate = static_cast<Float_>(my_rate);
        return out;
    }

    /** The a and b of the attraction curve in use. */
    double a() const { return umapb_status_a(my_handle.get()); }
    double b() const { return umapb_status_b(my_handle.get()); }

private:
    std::shared_ptr<umapb_status> my_handle;
    double my_rate;
};

}  // namespace umappp

#endif
