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

// Vectorised exact search (oracle/ref_knn.cpp): squared distances, sorted by
// (distance, index), self excluded, k per query.
void oracle_bruteforce_knn(const float* data, std::size_t dim, int nobs, int qstart, int qcount, int k, int nthreads,
                           int* out_idx, float* out_d2);
void oracle_bruteforce_knn(const double* data, std::size_t dim, int nobs, int qstart, int qcount, int k, int nthreads,
                           int* out_idx, double* out_d2);

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
        const int kk = std::min<int>(k, my_obs > 0 ? static_cast<int>(my_obs) - 1 : 0);
        if (static_cast<Index_>(out.size()) < count) {
            out.resize(count);
        }
        std::vector<int> idx(static_cast<std::size_t>(count) * kk);
        std::vector<Data_> d2(static_cast<std::size_t>(count) * kk);
        if (kk > 0) {
            oracle_bruteforce_knn(my_data.data(), my_dim, static_cast<int>(my_obs), static_cast<int>(start),
                                  static_cast<int>(count), kk, num_threads, idx.data(), d2.data());
        }
        for (Index_ q = 0; q < count; ++q) {
            auto& row = out[q];
            row.clear();
            for (int t = 0; t < kk; ++t) {
                const std::size_t o = static_cast<std::size_t>(q) * kk + t;
                row.emplace_back(static_cast<Index_>(idx[o]), static_cast<Distance_>(std::sqrt(d2[o])));
            }
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
