// Drop-in check: the reference's quick-start usage (README "Quick start")
// written against the GPU headers: 2000 observations x 10 dims of N(0, 1)
// data, exact neighbours on the device, initialize() then run(), plus a
// partial run, the NeighborList overload, a device-resident prebuilt index
// and the transform of new points into the finished layout.  Prints one line
// of results.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "umappp/umappp.hpp"

int main() {
    const int ndim = 10, nobs = 2000;
    std::vector<double> data(static_cast<size_t>(ndim) * nobs);
    std::mt19937_64 rng(1000);
    std::normal_distribution<double> ndist;
    for (auto& x : data) x = ndist(rng);

    const size_t out_dim = 2;
    std::vector<double> embedding(nobs * out_dim);
    umappp::Options opt;
    auto status = umappp::initialize(ndim, nobs, data.data(), umappp::DeviceBuilder(), out_dim, embedding.data(), opt);
    if (status.epoch() != 0 || status.num_epochs() != 500 || status.num_observations() != nobs) return 2;
    status.run(embedding.data(), 200);
    if (status.epoch() != 200) return 3;
    status.run(embedding.data());
    if (status.epoch() != 500) return 4;
    for (double v : embedding)
        if (!std::isfinite(v)) return 5;

    // the NeighborList overload with float data
    umappp::NeighborList<int, float> nl(nobs);
    for (int i = 0; i < nobs; ++i)
        for (int j = 1; j <= 5; ++j) nl[i].emplace_back((i + j) % nobs, 0.1f * j);
    std::vector<float> emb2(nobs * out_dim);
    opt.num_epochs = 50;
    auto st2 = umappp::initialize(nl, out_dim, emb2.data(), opt);
    st2.run(emb2.data());
    const auto ep = st2.get_epoch_data();

    // a device-resident prebuilt index (initialize.hpp:138-142) gives the same
    // initial state as the data overload
    umappp::DevicePrebuilt<double> prebuilt(ndim, nobs, data.data());
    std::vector<double> e_a(nobs * out_dim), e_b(nobs * out_dim);
    umappp::Options o2;
    auto sa = umappp::initialize<int, double>(prebuilt, out_dim, e_a.data(), o2);
    auto sb = umappp::initialize(ndim, nobs, data.data(), umappp::DeviceBuilder(), out_dim, e_b.data(), o2);
    if (e_a != e_b || sa.get_epoch_data().edge_targets != sb.get_epoch_data().edge_targets) return 6;
    // the transform extension: 100 new points into the finished layout
    const int nnew = 100;
    std::vector<double> fresh(static_cast<size_t>(ndim) * nnew), placed(nnew * out_dim);
    for (auto& x : fresh) x = ndist(rng);
    umappp::transform(ndim, nobs, data.data(), out_dim, embedding.data(), nnew, fresh.data(), placed.data(), opt, 20);
    for (double v : placed)
        if (!std::isfinite(v)) return 7;
    const auto ab = umappp::find_ab<double>(1.0, 0.1);
    std::printf("quickstart ok: epochs=%d edges=%zu a=%.6f b=%.6f y0=%.4f\n", status.epoch(), ep.edge_targets.size(),
                ab.first, ab.second, embedding[0]);
    return 0;
}
