#ifndef UMAPPP_OPTIONS_HPP
#define UMAPPP_OPTIONS_HPP

/**
 * @file Options.hpp
 * @brief Options for the UMAP algorithm (drop-in for libscran/umappp
 * include/umappp/Options.hpp:27-218): same enum, same fields, same defaults.
 * The irlba::Options member becomes IrlbaOptions (the device eigensolver's
 * knobs); num_threads* are accepted and ignored (the GPU replaces the CPU
 * thread pools).
 */

#include <cstdint>
#include <optional>
#include <random>

namespace umappp {

enum InitializeMethod : char { SPECTRAL, RANDOM, NONE };

typedef std::mt19937_64 RngEngine;

/** Knobs of the spectral eigensolver (stands in for irlba::Options). */
struct IrlbaOptions {
    /** Extra Krylov basis vectors beyond the requested eigenvectors. */
    int extra_work = 7;
    /** Maximum number of restarts. */
    int max_iterations = 1000;
    /** A Ritz pair is converged when its residual is below this times the largest eigenvalue. */
    double convergence_tolerance = 1e-6;
};

struct Options {
    double local_connectivity = 1;
    double bandwidth = 1;
    double mix_ratio = 1;
    double spread = 1;
    double min_dist = 0.1;
    std::optional<double> a;
    std::optional<double> b;
    double repulsion_strength = 1;
    InitializeMethod initialize_method = InitializeMethod::SPECTRAL;
    bool initialize_random_on_spectral_fail = true;
    IrlbaOptions initialize_spectral_irlba_options;
    double initialize_spectral_scale = 10;
    bool initialize_spectral_jitter = false;
    double initialize_spectral_jitter_sd = 0.0001;
    double initialize_random_scale = 10;
    typename RngEngine::result_type initialize_seed = 9876543210ULL;
    std::optional<int> num_epochs;
    double learning_rate = 1;
    double negative_sample_rate = 5;
    int num_neighbors = 15;
    typename RngEngine::result_type optimize_seed = 1234567890ULL;
    int num_threads = 1;
    int num_threads_spectral = 1;
    int num_threads_optimize = 1;
};

}  // namespace umappp

#endif
