#ifndef UMAPPP_INITIALIZE_HPP
#define UMAPPP_INITIALIZE_HPP

/**
 * @file initialize.hpp
 * @brief Initialize the UMAP algorithm (drop-in for libscran/umappp
 * include/umappp/initialize.hpp:27-177).
 *
 * Overloads:
 *  - initialize(NeighborList x, num_dim, embedding, options)   (:69-119)
 *  - initialize(DevicePrebuilt, num_dim, embedding, options) and, with
 *    knncolle, initialize(knncolle::Prebuilt, ...)            (:138-142)
 *  - initialize(data_dim, num_obs, data, DeviceBuilder, num_dim, embedding, options)
 *    with the exact Euclidean neighbour search running on the GPU (:165-177);
 *  - initialize(data_dim, num_obs, data, builder, ...) for any knncolle-style
 *    builder (build_unique + find_nearest_neighbors on the host, as the
 *    reference does), then the GPU for everything after the neighbour search.
 * Pointers may be host or device memory.
 */

#include <cmath>
#include <cstddef>
#include <optional>
#include <utility>

#include "Options.hpp"
#include "Status.hpp"
#include "detail.hpp"

namespace umappp {

/** choose_num_epochs (include/umappp/initialize.hpp:27-47). */
template <typename Index_>
int choose_num_epochs(const std::optional<int> num_epochs, const Index_ size) {
    return umapb_choose_num_epochs(num_epochs.has_value(), num_epochs.value_or(0), static_cast<int64_t>(size));
}

/** The exact Euclidean kNN of the GPU as the neighbour-search "builder". */
struct DeviceBuilder {};

/**
 * A neighbour-search index resident on the device (the role of
 * knncolle::Prebuilt): the data copied to the current device once and searched
 * by every initialize() on it (include/umappp/initialize.hpp:138-142).
 */
template <typename Float_>
class DevicePrebuilt {
public:
    DevicePrebuilt(const std::size_t data_dim, const int num_obs, const Float_* const data) {
        detail::check(umapb_prebuilt_create(detail::dtype<Float_>(), data_dim, num_obs, data, &pb_));
    }
    DevicePrebuilt(const DevicePrebuilt&) = delete;
    DevicePrebuilt& operator=(const DevicePrebuilt&) = delete;
    ~DevicePrebuilt() { umapb_prebuilt_free(pb_); }
    const umapb_prebuilt* handle() const { return pb_; }

private:
    umapb_prebuilt* pb_ = nullptr;
};

/**
 * initialize(NeighborList x, num_dim, embedding, Options)
 * (include/umappp/initialize.hpp:69-119): similarities, union, initial layout
 * and epoch schedule on the device; the initial layout is written to
 * 'embedding' (n x num_dim, row-major) as in the reference.
 */
template <typename Index_, typename Float_>
Status<Index_, Float_> initialize(const NeighborList<Index_, Float_>& x, const std::size_t num_dim, Float_* const embedding,
                                  Options options) {
    const auto csr = detail::to_csr(x);
    const auto copt = detail::to_c(options);
    umapb_status* st = nullptr;
    detail::check(umapb_initialize_neighbors(detail::dtype<Float_>(), static_cast<int32_t>(x.size()), csr.ptr.data(),
                                             csr.idx.data(), csr.val.data(), num_dim, embedding, &copt, &st));
    return Status<Index_, Float_>(st, options.negative_sample_rate);
}

/**
 * initialize(data_dim, num_obs, data, builder, num_dim, embedding, Options)
 * (include/umappp/initialize.hpp:165-177) with the device's exact Euclidean
 * neighbour search as the builder (data: observation i at
 * [i * data_dim, (i + 1) * data_dim)).
 */
template <typename Index_, typename Float_>
Status<Index_, Float_> initialize(const std::size_t data_dim, const Index_ num_obs, const Float_* const data,
                                  const DeviceBuilder&, const std::size_t num_dim, Float_* const embedding,
                                  Options options) {
    const auto copt = detail::to_c(options);
    umapb_status* st = nullptr;
    detail::check(umapb_initialize_data(detail::dtype<Float_>(), data_dim, static_cast<int32_t>(num_obs), data, num_dim,
                                        embedding, &copt, &st));
    return Status<Index_, Float_>(st, options.negative_sample_rate);
}

/** initialize(const Prebuilt&, num_dim, embedding, Options) (:138-142) on a device-resident index. */
template <typename Index_, typename Float_>
Status<Index_, Float_> initialize(const DevicePrebuilt<Float_>& prebuilt, const std::size_t num_dim,
                                  Float_* const embedding, Options options) {
    const auto copt = detail::to_c(options);
    umapb_status* st = nullptr;
    detail::check(umapb_initialize_prebuilt(prebuilt.handle(), num_dim, embedding, &copt, &st));
    return Status<Index_, Float_>(st, options.negative_sample_rate);
}

#if __has_include("knncolle/knncolle.hpp")
}  // namespace umappp
#include "knncolle/knncolle.hpp"
namespace umappp {

/** A knncolle builder: the neighbour search runs on the host as in the reference (:138-142, 165-177). */
template <typename Index_, typename Float_, class Matrix_ = knncolle::Matrix<Index_, Float_> >
Status<Index_, Float_> initialize(const std::size_t data_dim, const Index_ num_obs, const Float_* const data,
                                  const knncolle::Builder<Index_, Float_, Float_, Matrix_>& builder,
                                  const std::size_t num_dim, Float_* const embedding, Options options) {
    const auto prebuilt = builder.build_unique(knncolle::SimpleMatrix<Index_, Float_>(data_dim, num_obs, data));
    auto x = knncolle::find_nearest_neighbors(*prebuilt, options.num_neighbors, options.num_threads);
    return initialize(x, num_dim, embedding, std::move(options));
}

/** A knncolle prebuilt index: searched on the host as in the reference (:138-142). */
template <typename Index_, typename Input_, typename Float_>
Status<Index_, Float_> initialize(const knncolle::Prebuilt<Index_, Input_, Float_>& prebuilt, const std::size_t num_dim,
                                  Float_* const embedding, Options options) {
    auto x = knncolle::find_nearest_neighbors(prebuilt, options.num_neighbors, options.num_threads);
    return initialize(x, num_dim, embedding, std::move(options));
}
#endif

}  // namespace umappp

#endif
