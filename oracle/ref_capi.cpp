// C entry points over the reference's own headers (include/umappp/*.hpp),
// compiled unmodified against the project-written stand-ins in ref_shim/ for
// its absent dependencies.  Built by oracle/Makefile into
// oracle/_ref/libumappp_ref.so.  Test infrastructure: used only to pin the C
// restatement and the CUDA path to the reference, and as the timed CPU
// baseline.
//
// Layout conventions of every entry point: neighbour lists are CSR
// (row_ptr[n + 1] as int64, indices as int32, values as the float type);
// embeddings and data are column-major with observations as columns, i.e.
// observation i at [i * dim, (i + 1) * dim).
#include "umappp/umappp.hpp"
#include "umappp/neighbor_similarities.hpp"
#include "umappp/combine_neighbor_sets.hpp"
#include "umappp/spectral_init.hpp"
#include "umappp/optimize_layout.hpp"
#include "umappp/find_ab.hpp"
#include "umappp/initialize.hpp"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>

namespace {

thread_local std::string last_error;

template<typename Float_>
umappp::NeighborList<int, Float_> to_list(int n, const int64_t* ptr, const int32_t* idx, const Float_* val) {
    umappp::NeighborList<int, Float_> out(n);
    for (int i = 0; i < n; ++i) {
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            out[i].emplace_back(idx[p], val[p]);
        }
    }
    return out;
}

template<typename Float_>
int64_t from_list(const umappp::NeighborList<int, Float_>& x, int64_t* ptr, int32_t* idx, Float_* val, int64_t capacity) {
    int64_t total = 0;
    ptr[0] = 0;
    for (size_t i = 0; i < x.size(); ++i) {
        for (const auto& e : x[i]) {
            if (total >= capacity) {
                return -1;
            }
            idx[total] = e.first;
            val[total] = e.second;
            ++total;
        }
        ptr[i + 1] = total;
    }
    return total;
}

struct RefOptions {
    double local_connectivity, bandwidth, mix_ratio, spread, min_dist;
    double a, b;
    int has_a, has_b;
    double repulsion_strength;
    int initialize_method;
    int initialize_random_on_spectral_fail;
    int irlba_extra_work, irlba_max_iterations;
    double irlba_convergence_tolerance;
    double initialize_spectral_scale;
    int initialize_spectral_jitter;
    double initialize_spectral_jitter_sd;
    double initialize_random_scale;
    uint64_t initialize_seed;
    int num_epochs, has_num_epochs;
    double learning_rate, negative_sample_rate;
    int num_neighbors;
    uint64_t optimize_seed;
    int num_threads, num_threads_spectral, num_threads_optimize;
};

umappp::Options to_options(const RefOptions& r) {
    umappp::Options o;
    o.local_connectivity = r.local_connectivity;
    o.bandwidth = r.bandwidth;
    o.mix_ratio = r.mix_ratio;
    o.spread = r.spread;
    o.min_dist = r.min_dist;
    if (r.has_a) o.a = r.a;
    if (r.has_b) o.b = r.b;
    o.repulsion_strength = r.repulsion_strength;
    o.initialize_method = static_cast<umappp::InitializeMethod>(r.initialize_method);
    o.initialize_random_on_spectral_fail = r.initialize_random_on_spectral_fail != 0;
    o.initialize_spectral_irlba_options.extra_work = r.irlba_extra_work;
    o.initialize_spectral_irlba_options.max_iterations = r.irlba_max_iterations;
    o.initialize_spectral_irlba_options.convergence_tolerance = r.irlba_convergence_tolerance;
    o.initialize_spectral_scale = r.initialize_spectral_scale;
    o.initialize_spectral_jitter = r.initialize_spectral_jitter != 0;
    o.initialize_spectral_jitter_sd = r.initialize_spectral_jitter_sd;
    o.initialize_random_scale = r.initialize_random_scale;
    o.initialize_seed = r.initialize_seed;
    if (r.has_num_epochs) o.num_epochs = r.num_epochs;
    o.learning_rate = r.learning_rate;
    o.negative_sample_rate = r.negative_sample_rate;
    o.num_neighbors = r.num_neighbors;
    o.optimize_seed = r.optimize_seed;
    o.num_threads = r.num_threads;
    o.num_threads_spectral = r.num_threads_spectral;
    o.num_threads_optimize = r.num_threads_optimize;
    return o;
}

template<typename Float_>
struct RefStatus {
    umappp::Status<int, Float_> status;
    double a, b;
};

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

template<typename Float_>
void* status_from_neighbors(int n, const int64_t* ptr, const int32_t* idx, const Float_* dist, int num_dim, Float_* emb, const RefOptions* ro) {
    auto opt = to_options(*ro);
    auto st = umappp::initialize(to_list(n, ptr, idx, dist), static_cast<std::size_t>(num_dim), emb, opt);
    return new RefStatus<Float_>{std::move(st), 0, 0};
}

template<typename Float_>
void* status_from_data(int dim, int n, const Float_* data, int num_dim, Float_* emb, const RefOptions* ro) {
    auto opt = to_options(*ro);
    knncolle::BruteforceBuilder<int, Float_, Float_> builder;
    auto st = umappp::initialize(static_cast<std::size_t>(dim), n, data, builder, static_cast<std::size_t>(num_dim), emb, opt);
    return new RefStatus<Float_>{std::move(st), 0, 0};
}

} // namespace

#define REF_TRY(...) \
    try { __VA_ARGS__ } catch (const std::exception& e) { last_error = e.what(); return -1; } catch (...) { last_error = "unknown error"; return -1; }

extern "C" {

const char* ref_last_error() { return last_error.c_str(); }

int ref_choose_num_epochs(int has_value, int value, int n) {
    std::optional<int> v;
    if (has_value) v = value;
    return umappp::choose_num_epochs<int>(v, n);
}

int ref_find_ab(double spread, double min_dist, double* a, double* b) {
    REF_TRY({
        auto out = umappp::find_ab<double>(spread, min_dist);
        *a = out.first;
        *b = out.second;
        return 0;
    })
}

#define REF_FLOAT_FUNCS(SUFFIX, Float_) \
int ref_neighbor_similarities_##SUFFIX(int n, const int64_t* ptr, const int32_t* idx, Float_* dist, double local_connectivity, double bandwidth, double min_k_dist_scale, int use_newton, int num_threads) { \
    REF_TRY({ \
        auto x = to_list<Float_>(n, ptr, idx, dist); \
        umappp::NeighborSimilaritiesOptions<Float_> o; \
        o.local_connectivity = local_connectivity; \
        o.bandwidth = bandwidth; \
        o.min_k_dist_scale = min_k_dist_scale; \
        o.num_threads = num_threads; \
        if (use_newton) { umappp::neighbor_similarities<true>(x, o); } else { umappp::neighbor_similarities<false>(x, o); } \
        int64_t t = 0; \
        for (int i = 0; i < n; ++i) for (auto& e : x[i]) dist[t++] = e.second; \
        return 0; \
    }) \
} \
int64_t ref_combine_neighbor_sets_##SUFFIX(int n, const int64_t* ptr, const int32_t* idx, const Float_* w, double mix_ratio, int64_t* out_ptr, int32_t* out_idx, Float_* out_w, int64_t capacity) { \
    REF_TRY({ \
        auto x = to_list<Float_>(n, ptr, idx, w); \
        umappp::combine_neighbor_sets(x, static_cast<Float_>(mix_ratio)); \
        return from_list<Float_>(x, out_ptr, out_idx, out_w, capacity); \
    }) \
} \
int64_t ref_similarities_to_epochs_##SUFFIX(int n, const int64_t* ptr, const int32_t* idx, const Float_* w, int num_epochs, double rate, int64_t* out_ptr, int32_t* targets, Float_* eps, Float_* enext, Float_* enneg) { \
    REF_TRY({ \
        auto x = to_list<Float_>(n, ptr, idx, w); \
        auto ep = umappp::similarities_to_epochs<int, Float_>(x, num_epochs, static_cast<Float_>(rate)); \
        for (size_t i = 0; i < ep.cumulative_num_edges.size(); ++i) out_ptr[i] = static_cast<int64_t>(ep.cumulative_num_edges[i]); \
        for (size_t j = 0; j < ep.edge_targets.size(); ++j) { \
            targets[j] = ep.edge_targets[j]; eps[j] = ep.epochs_per_sample[j]; \
            enext[j] = ep.epoch_of_next_sample[j]; enneg[j] = ep.epoch_of_next_negative_sample[j]; \
        } \
        return static_cast<int64_t>(ep.edge_targets.size()); \
    }) \
} \
int ref_spectral_init_##SUFFIX(int n, const int64_t* ptr, const int32_t* idx, const Float_* w, int num_dim, Float_* out, double tol, int max_iter, double scale, int jitter, double jitter_sd, uint64_t seed, int nthreads) { \
    REF_TRY({ \
        auto x = to_list<Float_>(n, ptr, idx, w); \
        irlba::Options<Eigen::VectorXd> io; \
        io.convergence_tolerance = tol; \
        io.max_iterations = max_iter; \
        return umappp::spectral_init(x, static_cast<std::size_t>(num_dim), out, io, nthreads, scale, jitter != 0, jitter_sd, seed) ? 1 : 0; \
    }) \
} \
int ref_random_init_##SUFFIX(int n, int num_dim, Float_* out, uint64_t seed, double scale) { \
    REF_TRY({ umappp::random_init<int, Float_>(n, static_cast<std::size_t>(num_dim), out, seed, scale); return 0; }) \
} \
int ref_has_multiple_components_##SUFFIX(int n, const int64_t* ptr, const int32_t* idx, const Float_* w) { \
    REF_TRY({ auto x = to_list<Float_>(n, ptr, idx, w); return umappp::has_multiple_components(x) ? 1 : 0; }) \
} \
int ref_optimize_layout_##SUFFIX(int num_dim, Float_* emb, int n, const int64_t* ptr, const int32_t* targets, const Float_* eps, Float_* enext, Float_* enneg, double rate, int total_epochs, int* current_epoch, double a, double b, double gamma, double alpha, uint64_t seed, int epoch_limit, int nthreads) { \
    REF_TRY({ \
        umappp::EpochData<int, Float_> ep(n); \
        ep.total_epochs = total_epochs; \
        ep.current_epoch = *current_epoch; \
        const int64_t nnz = ptr[n]; \
        for (int i = 0; i <= n; ++i) ep.cumulative_num_edges[i] = static_cast<std::size_t>(ptr[i]); \
        ep.edge_targets.assign(targets, targets + nnz); \
        ep.epochs_per_sample.assign(eps, eps + nnz); \
        ep.epoch_of_next_sample.assign(enext, enext + nnz); \
        ep.epoch_of_next_negative_sample.assign(enneg, enneg + nnz); \
        ep.negative_sample_rate = static_cast<Float_>(rate); \
        std::mt19937_64 rng(seed); \
        if (nthreads <= 1) { \
            umappp::optimize_layout<int, Float_>(num_dim, emb, ep, a, b, gamma, alpha, rng, epoch_limit); \
        } else { \
            umappp::optimize_layout_parallel<int, Float_>(num_dim, emb, ep, a, b, gamma, alpha, rng, epoch_limit, nthreads); \
        } \
        std::copy(ep.epoch_of_next_sample.begin(), ep.epoch_of_next_sample.end(), enext); \
        std::copy(ep.epoch_of_next_negative_sample.begin(), ep.epoch_of_next_negative_sample.end(), enneg); \
        *current_epoch = ep.current_epoch; \
        return 0; \
    }) \
} \
int ref_knn_##SUFFIX(int dim, int n, const Float_* data, int k, int qstart, int qcount, int nthreads, int32_t* out_idx, Float_* out_dist) { \
    REF_TRY({ \
        knncolle::BruteforcePrebuilt<int, Float_, Float_> index(static_cast<std::size_t>(dim), n, data); \
        knncolle::NeighborList<int, Float_> out; \
        index.search_range(qstart, qcount, k, nthreads, out); \
        int64_t t = 0; \
        for (int q = 0; q < qcount; ++q) { \
            for (const auto& e : out[q]) { out_idx[t] = e.first; out_dist[t] = e.second; ++t; } \
        } \
        return static_cast<int>(out.empty() ? 0 : out[0].size()); \
    }) \
} \
void* ref_status_from_neighbors_##SUFFIX(int n, const int64_t* ptr, const int32_t* idx, const Float_* dist, int num_dim, Float_* emb, const void* opts) { \
    try { return status_from_neighbors<Float_>(n, ptr, idx, dist, num_dim, emb, static_cast<const RefOptions*>(opts)); } \
    catch (const std::exception& e) { last_error = e.what(); return nullptr; } \
} \
void* ref_status_from_data_##SUFFIX(int dim, int n, const Float_* data, int num_dim, Float_* emb, const void* opts) { \
    try { return status_from_data<Float_>(dim, n, data, num_dim, emb, static_cast<const RefOptions*>(opts)); } \
    catch (const std::exception& e) { last_error = e.what(); return nullptr; } \
} \
int ref_status_run_##SUFFIX(void* h, Float_* emb, int epoch_limit) { \
    REF_TRY({ static_cast<RefStatus<Float_>*>(h)->status.run(emb, epoch_limit); return 0; }) \
} \
int ref_status_epoch_##SUFFIX(void* h) { return static_cast<RefStatus<Float_>*>(h)->status.epoch(); } \
int ref_status_num_epochs_##SUFFIX(void* h) { return static_cast<RefStatus<Float_>*>(h)->status.num_epochs(); } \
int64_t ref_status_num_edges_##SUFFIX(void* h) { return static_cast<int64_t>(static_cast<RefStatus<Float_>*>(h)->status.get_epoch_data().edge_targets.size()); } \
int ref_status_epoch_data_##SUFFIX(void* h, int64_t* ptr, int32_t* targets, Float_* eps, Float_* enext, Float_* enneg) { \
    const auto& ep = static_cast<RefStatus<Float_>*>(h)->status.get_epoch_data(); \
    for (size_t i = 0; i < ep.cumulative_num_edges.size(); ++i) ptr[i] = static_cast<int64_t>(ep.cumulative_num_edges[i]); \
    for (size_t j = 0; j < ep.edge_targets.size(); ++j) { \
        targets[j] = ep.edge_targets[j]; eps[j] = ep.epochs_per_sample[j]; \
        enext[j] = ep.epoch_of_next_sample[j]; enneg[j] = ep.epoch_of_next_negative_sample[j]; \
    } \
    return 0; \
} \
void ref_status_destroy_##SUFFIX(void* h) { delete static_cast<RefStatus<Float_>*>(h); }

REF_FLOAT_FUNCS(f64, double)
REF_FLOAT_FUNCS(f32, float)

// Size of the options struct, so the Python side can check its mirror.
int ref_options_size() { return static_cast<int>(sizeof(RefOptions)); }

// The stages of initialize(data, builder, ...) and Status::run
// (include/umappp/initialize.hpp:69-119,165-177; Status.hpp:101-128) called
// one by one through the reference's own functions, timed in seconds:
// secs[0] kNN, [1] similarities, [2] union, [3] initial layout, [4] a/b +
// epochs, [5] the first 'sgd_epochs' epochs of optimize_layout(_parallel).
// The data is float, n x dim; the embedding n x 2.
int ref_pipeline_timed_f32(int dim, int n, const float* data, int k, int num_epochs, int sgd_epochs, int nthreads,
                           float* embedding, double* secs) {
    REF_TRY({
        using clock = std::chrono::steady_clock;
        umappp::Options opt;
        opt.num_neighbors = k;
        opt.num_epochs = num_epochs;
        opt.num_threads = nthreads;
        opt.num_threads_spectral = nthreads;
        opt.num_threads_optimize = nthreads;
        auto t0 = clock::now();
        knncolle::BruteforcePrebuilt<int, float, float> index(static_cast<std::size_t>(dim), n, data);
        auto x = knncolle::find_nearest_neighbors(index, k, nthreads);
        secs[0] = seconds_since(t0);

        t0 = clock::now();
        umappp::NeighborSimilaritiesOptions<float> nsopt;
        nsopt.num_threads = nthreads;
        umappp::neighbor_similarities(x, nsopt);
        secs[1] = seconds_since(t0);

        t0 = clock::now();
        umappp::combine_neighbor_sets(x, 1.0f);
        secs[2] = seconds_since(t0);

        t0 = clock::now();
        const bool ok = umappp::spectral_init(x, 2, embedding, opt.initialize_spectral_irlba_options, nthreads,
                                              opt.initialize_spectral_scale, false, 0.0, opt.initialize_seed);
        if (!ok) umappp::random_init<int, float>(n, 2, embedding, opt.initialize_seed, opt.initialize_random_scale);
        secs[3] = seconds_since(t0);

        t0 = clock::now();
        const auto ab = umappp::find_ab(opt.spread, opt.min_dist);
        auto ep = umappp::similarities_to_epochs<int, float>(x, num_epochs, static_cast<float>(opt.negative_sample_rate));
        secs[4] = seconds_since(t0);

        t0 = clock::now();
        std::mt19937_64 rng(opt.optimize_seed);
        if (nthreads <= 1) {
            umappp::optimize_layout<int, float>(2, embedding, ep, ab.first, ab.second, 1.0f, 1.0f, rng, sgd_epochs);
        } else {
            umappp::optimize_layout_parallel<int, float>(2, embedding, ep, ab.first, ab.second, 1.0f, 1.0f, rng,
                                                         sgd_epochs, nthreads);
        }
        secs[5] = seconds_since(t0);
        return ok ? 1 : 0;
    })
}

}
