// Project-written stand-in for the knncolle types named by the reference
// (include/umappp/NeighborList.hpp:28-29, initialize.hpp:138-177): the
// NeighborList alias, Matrix/SimpleMatrix, Prebuilt, Builder and
// find_nearest_neighbors.  knncolle (and its VP-tree) is absent here, so the
// only builder is an exact multithreaded brute-force Euclidean search:
// neighbours of each observation, self excluded, sorted by increasing
// distance with ties broken by index.  Squared distances are accumulated in
// the data type from coordinate differences.
//
// Test infrastructure only (the CPU baseline's kNN stage and the builder path).
#ifndef ORACLE_SHIM_KNNCOLLE_HPP
#define ORACLE_SHIM_KNNCOLLE_HPP

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <memory>
#include <thread>
#include <utility>
#include <vector>

namespace knncolle {

template<typename Index_, typename Distance_>
using NeighborList = std::vector<std::vector<std::pair<Index_, Distance_> > >;

template<typename Index_, typename Data_>
class Matrix {
public:
    virtual ~Matrix() = default;
    virtual Index_ num_observations() const = 0;
    virtual std::size_t num_dimensions() const = 0;
    virtual const Data_* data() const = 0;
};

template<typename Index_, typename Data_>
class SimpleMatrix final : public Matrix<Index_, Data_> {
public:
    SimpleMatrix(std::size_t num_dim, Index_ num_obs, const Data_* data) : my_dim(num_dim), my_obs(num_obs), my_data(data) {}
    Index_ num_observations() const override { return my_obs; }
    std::size_t num_dimensions() const override { return my_dim; }
    const Data_* data() const override { return my_data; }

private:
    std::size_t my_dim;
    Index_ my_obs;
    const Data_* my_data;
};

template<typename Index_, typename Data_, typename Distance_>
class Prebuilt {
public:
    virtual ~Prebuilt() = default;
    virtual Index_ num_observations() const = 0;
    // Neighbours of observations [start, start + count) among all observations.
    virtual void search_range(Index_ start, Index_ count, int k, int num_threads, NeighborList<Index_, Distance_>& out) const = 0;
};

template<typename Index_, typename Data_, typename Distance_, class Matrix_ = Matrix<Index_, Data_> >
class Builder {
public:
    virtual ~Builder() = default;
    virtual Prebuilt<Index_, Data_, Distance_>* build_raw(const Matrix_& mat) const = 0;
    std::unique_ptr<Prebuilt<Index_, Data_, Distance_> > build_unique(const Matrix_& mat) const {
        return std::unique_ptr<Prebuilt<Index_, Data_, Distance_> >(build_raw(mat));
    }
};

template<typename Index_, typename Data_, typename Distance_>
NeighborList<Index_, Distance_> find_nearest_neighbors(const Prebuilt<Index_, Data_, Distance_>& index, int k, int num_threads) {
    NeighborList<Index_, Distance_> out(index.num_observations());
    index.search_range(0, index.num_observations(), k, num_threads, out);
    return out;
}

template<typename Index_, typename Data_, typename Distance_>
class BruteforcePrebuilt final : public Prebuilt<Index_, Data_, Distance_> {
public:
    BruteforcePrebuilt(std::size_t dim, Index_ nobs, const Data_* data) : my_dim(dim), my_obs(nobs), my_data(data, data + dim * static_cast<std::size_t>(nobs)) {}
    Index_ num_observations() const override { return my_obs; }

    void search_range(Index_ start, Index_ count, int k, int num_threads, NeighborList<Index_, Distance_>& out) const override {
        const Index_ kk = std::min<Index_>(k, my_obs > 0 ? my_obs - 1 : 0);
        if (static_cast<Index_>(out.size()) < count) {
            out.resize(count);
        }
        auto work = [&](Index_ qs, Index_ qe) {
            std::vector<std::pair<Data_, Index_> > heap;
            heap.reserve(kk + 1);
            for (Index_ q = qs; q < qe; ++q) {
                const Data_* xq = my_data.data() + my_dim * static_cast<std::size_t>(q);
                heap.clear();
                for (Index_ j = 0; j < my_obs; ++j) {
                    if (j == q) {
                        continue;
                    }
                    const Data_* xj = my_data.data() + my_dim * static_cast<std::size_t>(j);
                    Data_ d2 = 0;
                    for (std::size_t d = 0; d < my_dim; ++d) {
                        const Data_ diff = xq[d] - xj[d];
                        d2 += diff * diff;
                    }
                    if (static_cast<Index_>(heap.size()) < kk) {
                        heap.emplace_back(d2, j);
                        std::push_heap(heap.begin(), heap.end());
                    } else if (kk > 0 && std::make_pair(d2, j) < heap.front()) {
                        std::pop_heap(heap.begin(), heap.end());
                        heap.back() = std::make_pair(d2, j);
                        std::push_heap(heap.begin(), heap.end());
                    }
                }
                std::sort_heap(heap.begin(), heap.end());
                auto& row = out[q - start];
                row.clear();
                for (const auto& h : heap) {
                    row.emplace_back(h.second, static_cast<Distance_>(std::sqrt(h.first)));
                }
            }
        };
        const int nt = std::max(1, num_threads);
        std::vector<std::thread> threads;
        const Index_ per = (count + nt - 1) / nt;
        for (int t = 0; t < nt; ++t) {
            const Index_ s = start + per * t;
            const Index_ e = std::min<Index_>(start + count, s + per);
            if (s < e) {
                threads.emplace_back(work, s, e);
            }
        }
        for (auto& t : threads) {
            t.join();
        }
    }

private:
    std::size_t my_dim;
    Index_ my_obs;
    std::vector<Data_> my_data;
};

template<typename Index_, typename Data_, typename Distance_, class Matrix_ = Matrix<Index_, Data_> >
class BruteforceBuilder final : public Builder<Index_, Data_, Distance_, Matrix_> {
public:
    Prebuilt<Index_, Data_, Distance_>* build_raw(const Matrix_& mat) const override {
        return new BruteforcePrebuilt<Index_, Data_, Distance_>(mat.num_dimensions(), mat.num_observations(), mat.data());
    }
};

}

#endif
