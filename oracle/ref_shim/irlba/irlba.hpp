// Project-written stand-in for the parts of the irlba library named by the
// reference (include/umappp/Options.hpp:110, spectral_init.hpp:105-126):
// irlba::Options, irlba::ParallelSparseMatrix (compressed sparse columns),
// irlba::EigenThreadScope and irlba::compute returning .U and
// .metrics.converged.  irlba is absent here; compute() solves the symmetric
// case the reference uses it for (the shifted normalised Laplacian) with the
// FP64 thick-restart Lanczos of oracle/lanczos.h, so the singular vectors are
// eigenvectors in decreasing order of eigenvalue.
//
// Test infrastructure only.
#ifndef ORACLE_SHIM_IRLBA_HPP
#define ORACLE_SHIM_IRLBA_HPP

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <thread>
#include <vector>

#include "Eigen/Dense"
#include "../../lanczos.h"

namespace irlba {

template<class Vector_ = Eigen::VectorXd>
struct Options {
    int extra_work = 7;
    int max_iterations = 1000;
    double convergence_tolerance = 1e-6;
    std::uint64_t seed = 5489u;
};

template<class Vector_, class Matrix_, class Values_, class Indices_, class Pointers_>
class ParallelSparseMatrix {
public:
    ParallelSparseMatrix(std::size_t nrow, std::size_t ncol, Values_ values, Indices_ indices, Pointers_ pointers,
                         bool column_major, int nthreads)
        : my_nrow(nrow), my_ncol(ncol), my_values(std::move(values)), my_indices(std::move(indices)),
          my_pointers(std::move(pointers)), my_column_major(column_major), my_nthreads(nthreads) {}

    std::size_t rows() const { return my_nrow; }
    std::size_t cols() const { return my_ncol; }

    // y = A x for the symmetric matrices used here: a compressed-column
    // symmetric matrix equals its compressed-row transpose, so each output
    // element is a dot product over one stored column.
    void multiply(const double* x, double* y) const {
        const std::size_t n = my_ncol;
        auto work = [&](std::size_t start, std::size_t end) {
            for (std::size_t c = start; c < end; ++c) {
                double sum = 0;
                for (auto p = my_pointers[c]; p < my_pointers[c + 1]; ++p) {
                    sum += my_values[p] * x[my_indices[p]];
                }
                y[c] = sum;
            }
        };
        const int nt = std::max(1, my_nthreads);
        if (nt == 1 || n < 10000) {
            work(0, n);
            return;
        }
        std::vector<std::thread> threads;
        const std::size_t per = (n + nt - 1) / nt;
        for (int t = 0; t < nt; ++t) {
            const std::size_t s = per * t, e = std::min(n, s + per);
            if (s < e) {
                threads.emplace_back(work, s, e);
            }
        }
        for (auto& t : threads) {
            t.join();
        }
    }

private:
    std::size_t my_nrow, my_ncol;
    Values_ my_values;
    Indices_ my_indices;
    Pointers_ my_pointers;
    bool my_column_major;
    int my_nthreads;
};

struct EigenThreadScope {
    explicit EigenThreadScope(int) {}
};

struct Metrics {
    bool converged = false;
    int iterations = 0;
};

struct Results {
    Eigen::MatrixXd U;
    Eigen::VectorXd D;
    Metrics metrics;
};

template<class Matrix_>
void shim_matvec(void* ctx, const double* x, double* y) {
    static_cast<const Matrix_*>(ctx)->multiply(x, y);
}

template<class Matrix_, class Vector_>
Results compute(const Matrix_& mat, int number, const Options<Vector_>& opt) {
    if (mat.rows() != mat.cols()) {
        throw std::runtime_error("the irlba stand-in only handles the square symmetric case");
    }
    const std::int64_t n = static_cast<std::int64_t>(mat.rows());
    Results out;
    out.U = Eigen::MatrixXd(n, number);
    out.D = Eigen::VectorXd(number);
    const int ncv = number + std::max(opt.extra_work, number) + 8;
    int restarts = 0;
    const int ok = oracle_lanczos(n, number, ncv, opt.max_iterations, opt.convergence_tolerance, opt.seed,
                                  &shim_matvec<Matrix_>, const_cast<Matrix_*>(&mat), out.D.data(), out.U.data(), &restarts);
    out.metrics.converged = (ok != 0);
    out.metrics.iterations = restarts;
    return out;
}

}

#endif
