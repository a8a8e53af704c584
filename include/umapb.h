/*
 * umapb.h -- C ABI of the B200 (sm_100a) UMAP library libumappp_b200.so.
 *
 * Every entry point is plain C: pointers, sizes and an int status.  Pointer
 * arguments may be host memory (pageable or pinned) or device memory on the
 * current CUDA device; the library detects which and copies as needed.  Device
 * memory of another GPU is rejected with UMAPB_ERR_INVALID.
 * Layouts follow the reference (libscran/umappp v3.3.2):
 *   - data and embeddings are column-major with observations as columns,
 *     i.e. observation i occupies [i * dim, (i + 1) * dim)
 *     (include/umappp/initialize.hpp:58-63,150-152);
 *   - neighbour lists and graphs are CSR: row i holds
 *     indices/values[row_ptr[i] .. row_ptr[i + 1]) with int64 row pointers and
 *     int32 indices; neighbour rows are sorted by increasing distance
 *     (include/umappp/NeighborList.hpp:24-29).
 * dtype selects the reference's Float_ template argument (UMAPB_F32 = float,
 * UMAPB_F64 = double); value arrays then hold that type.
 *
 * Errors: every function returns UMAPB_OK or an error code and leaves a
 * message for umapb_last_error() (per calling thread).  Nothing throws and no
 * call falls back to the CPU: without a usable sm_100 device the calls fail
 * with UMAPB_ERR_NO_DEVICE.
 */
#ifndef UMAPB_H
#define UMAPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UMAPB_VERSION 100

enum umapb_code {
    UMAPB_OK = 0,
    UMAPB_ERR_INVALID = 1,        /* bad argument (sizes, layout, options) */
    UMAPB_ERR_OOM = 2,            /* device allocation failed */
    UMAPB_ERR_CUDA = 3,           /* CUDA runtime error */
    UMAPB_ERR_DEVICE_TIMEOUT = 4, /* a bounded device-side wait gave up */
    UMAPB_ERR_OVERFLOW = 5,       /* a size or cast would overflow (sanisizer's role) */
    UMAPB_ERR_NO_DEVICE = 6       /* no usable CUDA device */
};

enum umapb_dtype { UMAPB_F32 = 0, UMAPB_F64 = 1 };

/* Mirrors umappp::InitializeMethod (include/umappp/Options.hpp:27). */
enum umapb_init_method { UMAPB_INIT_SPECTRAL = 0, UMAPB_INIT_RANDOM = 1, UMAPB_INIT_NONE = 2 };

/*
 * Mirrors umappp::Options (include/umappp/Options.hpp:37-218) field for field.
 * std::optional fields carry a has_* flag.  irlba_* replace the
 * irlba::Options member (Options.hpp:110); num_threads* are accepted and
 * ignored (the device replaces the CPU thread pools).
 */
typedef struct umapb_options {
    double local_connectivity;               /* Options.hpp:43  default 1 */
    double bandwidth;                        /* :49  default 1 */
    double mix_ratio;                        /* :57  default 1 */
    double spread;                           /* :63  default 1 */
    double min_dist;                         /* :71  default 0.1 */
    double a;                                /* :79  optional */
    double b;                                /* :87  optional */
    int has_a;
    int has_b;
    double repulsion_strength;               /* :93  default 1 */
    int initialize_method;                   /* :98  default SPECTRAL */
    int initialize_random_on_spectral_fail;  /* :105 default 1 */
    int irlba_extra_work;                    /* Krylov basis size = num_dim + 1 + max(extra, num_dim + 1) + 8; default 7 */
    int irlba_max_iterations;                /* restart cap, default 1000 */
    double irlba_convergence_tolerance;      /* residual <= tol * largest eigenvalue, default 1e-6 */
    double initialize_spectral_scale;        /* :118 default 10 */
    int initialize_spectral_jitter;          /* :125 default 0 */
    double initialize_spectral_jitter_sd;    /* :131 default 1e-4 */
    double initialize_random_scale;          /* :139 default 10 */
    uint64_t initialize_seed;                /* :147 default 9876543210 */
    int num_epochs;                          /* :159 optional */
    int has_num_epochs;
    double learning_rate;                    /* :165 default 1 */
    double negative_sample_rate;             /* :171 default 5 */
    int num_neighbors;                       /* :178 default 15 */
    uint64_t optimize_seed;                  /* :183 default 1234567890 */
    int num_threads;                         /* :192 ignored */
    int num_threads_spectral;                /* :201 ignored */
    int num_threads_optimize;                /* :217 ignored */
} umapb_options;

/* Fills the reference's defaults (Options.hpp:37-218). */
void umapb_options_init(umapb_options* opt);

/* Message of the last failing call on this thread ("" if none).  The reference
 * throws C++ exceptions instead (e.g. include/umappp/optimize_layout.hpp:29,89);
 * here every call returns a status code and leaves its message here. */
const char* umapb_last_error(void);

/* Version of this library.  No reference counterpart (a header-only library). */
int umapb_version(void);

/* sizeof(umapb_options), for bindings that mirror the struct.  No reference
 * counterpart: a binding check. */
size_t umapb_options_size(void);

/* Number of kernels this library has launched in this process (all threads).
 * No reference counterpart: a measurement hook. */
int64_t umapb_launch_count(void);

/*
 * Poll limit of the bounded device-side waits of the tensor-core kNN kernels
 * (an extension; the reference has no device code).  A role of the kernel
 * that waits longer than this for another role gives up: the kernel stops
 * all roles, waits for its copies and MMAs in flight, frees its tensor memory
 * and the call returns UMAPB_ERR_DEVICE_TIMEOUT, leaving the device usable.
 * polls <= 0 restores the default (2^26 polls, seconds).  Process-wide; read
 * at each launch.  Returns the previous limit.  Meant for failure testing.
 */
int64_t umapb_set_device_wait_limit(int64_t polls);

/*
 * Roofline probe (an extension): the rate of uniformly random float2 accesses
 * to an array of num_points float2 values in device memory, with nothing else
 * to do -- mode 0: loads through L2 (ld.global.cg), mode 1: atomic adds
 * (red.global.add.v2.f32) -- measured with CUDA events over 'reps' launches of
 * about 'accesses' accesses each.  At 10^6 points the array (8 MB) stays in
 * L2, which is where the SGD epochs' gathers and atomics land.
 */
int umapb_measure_random_access(int64_t num_points, int64_t accesses, int mode, int reps, double* per_second);

/*
 * Caps the device memory the library has in use at once (process-wide, all
 * devices): an allocation beyond the cap fails with UMAPB_ERR_OOM, as a real
 * out-of-memory does, and the library's cache of freed blocks is returned to
 * the device before in-use plus cached bytes would exceed it.  0 removes the cap (the default).  Returns the
 * previous cap.  An extension (the reference allocates host memory only): for
 * callers that share a GPU, and for testing the out-of-memory path.
 */
size_t umapb_set_workspace_limit(size_t bytes);

/* ------------------------------------------------------------------ Status */

typedef struct umapb_status umapb_status;

/*
 * umappp::initialize(NeighborList, num_dim, embedding, Options)
 * (include/umappp/initialize.hpp:69-119): similarities, fuzzy union,
 * initial layout (spectral / random / none, written into 'embedding'),
 * a/b fit, epoch count and per-edge schedule.  'embedding' holds
 * num_obs * num_dim values of dtype.  On success *out owns the state.
 */
int umapb_initialize_neighbors(int dtype, int32_t num_obs, const int64_t* row_ptr, const int32_t* indices,
                               const void* distances, size_t num_dim, void* embedding, const umapb_options* opt,
                               umapb_status** out);

/*
 * umappp::initialize(data_dim, num_obs, data, builder, num_dim, embedding,
 * Options) (include/umappp/initialize.hpp:165-177) with an exact Euclidean
 * neighbour search on the device as the builder: opt->num_neighbors
 * neighbours per observation (self excluded), then as above.
 */
int umapb_initialize_data(int dtype, size_t data_dim, int32_t num_obs, const void* data, size_t num_dim,
                          void* embedding, const umapb_options* opt, umapb_status** out);

/*
 * umappp::initialize(NeighborList, ...) (include/umappp/initialize.hpp:69-119)
 * with the neighbours given as two k x num_obs column-major matrices, one
 * column per observation -- indices[i * k + j] and distances[i * k + j] are
 * observation i's j-th neighbour, sorted by increasing distance -- the layout
 * the reference's R harness builds its NeighborList from
 * (tests/R/package/src/test.cpp:9-19) and knncolle's dense outputs use.
 * Device arrays are used in place and host arrays copied as they are: no
 * CSR is built on the host.  index_base is 0, or 1 for R's 1-based indices.
 */
int umapb_initialize_knn_matrix(int dtype, int32_t num_obs, int32_t k, const int32_t* indices, const void* distances,
                                int index_base, size_t num_dim, void* embedding, const umapb_options* opt,
                                umapb_status** out);

/*
 * A neighbour-search index resident on the device, the role of
 * knncolle::Prebuilt that include/umappp/initialize.hpp:138-142 takes: the data
 * (num_obs x data_dim of dtype, observation i at
 * [i * data_dim, (i + 1) * data_dim)) copied to the current device once and
 * searched by every umapb_initialize_prebuilt, without copying it again.
 */
typedef struct umapb_prebuilt umapb_prebuilt;
int umapb_prebuilt_create(int dtype, size_t data_dim, int32_t num_obs, const void* data, umapb_prebuilt** out);
void umapb_prebuilt_free(umapb_prebuilt* prebuilt);

/*
 * umappp::initialize(const knncolle::Prebuilt&, num_dim, embedding, Options)
 * (include/umappp/initialize.hpp:138-142): the exact Euclidean neighbour search
 * of opt->num_neighbors on the prebuilt index's device data, then as
 * umapb_initialize_neighbors.  Call with the index's device current.
 */
int umapb_initialize_prebuilt(const umapb_prebuilt* prebuilt, size_t num_dim, void* embedding, const umapb_options* opt,
                              umapb_status** out);

/*
 * Status::run(embedding, epoch_limit) (include/umappp/Status.hpp:101-128):
 * advances the layout in 'embedding' (read on entry, written on exit) from
 * epoch() to epoch_limit.  epoch_limit < 0 means num_epochs()
 * (Status::run(embedding), Status.hpp:138-140).
 */
int umapb_status_run(umapb_status* st, void* embedding, int epoch_limit);

int umapb_status_epoch(const umapb_status* st);                 /* Status.hpp:70-72 */
int umapb_status_num_epochs(const umapb_status* st);            /* Status.hpp:78-80 */
int32_t umapb_status_num_observations(const umapb_status* st);  /* Status.hpp:85-87 */
size_t umapb_status_num_dimensions(const umapb_status* st);     /* Status.hpp:63-65 */
/* The a and b in use: Options::a / Options::b (Options.hpp:79,87) or the fit of
 * find_ab.hpp:44-168 made by initialize (initialize.hpp:105-110). */
double umapb_status_a(const umapb_status* st);
double umapb_status_b(const umapb_status* st);
/* Edges of the status' EpochData, the last entry of cumulative_num_edges
 * (optimize_layout.hpp:27-45). */
int64_t umapb_status_num_edges(const umapb_status* st);

/*
 * Status::get_epoch_data() (Status.hpp:52-54, EpochData optimize_layout.hpp:27-45)
 * at the current epoch: row_ptr[n + 1], targets[nnz] and the dtype arrays
 * epochs_per_sample, epoch_of_next_sample, epoch_of_next_negative_sample
 * (any of them may be NULL).
 */
int umapb_status_get_epoch_data(const umapb_status* st, int64_t* row_ptr, int32_t* targets, void* epochs_per_sample,
                                void* epoch_of_next_sample, void* epoch_of_next_negative_sample);

/*
 * Exact per-epoch counts of the deterministic schedule over [first, last):
 * counts[2 * e] = firing edges, counts[2 * e + 1] = negative samples drawn
 * (self-samples included, as the reference draws and then skips them).
 * No reference counterpart: the counts of the schedule that
 * optimize_layout.hpp:136-180 walks, for measurement and checks.
 */
int umapb_status_schedule_counts(const umapb_status* st, int first, int last, int64_t* counts);

/*
 * Device milliseconds of the stages of the last initialize / run on this
 * status, in the order: knn, similarities, union, init, epochs, schedule,
 * sgd.  'count' entries are written (at most 7).  No reference counterpart:
 * a measurement hook.
 */
int umapb_status_stage_ms(const umapb_status* st, double* ms, int count);

/* Releases the status and its device state (the end of a umappp::Status,
 * Status.hpp:25-141). */
void umapb_status_free(umapb_status* st);

/* ----------------------------------------------------------- stage entries */

/*
 * Exact Euclidean k-nearest neighbours of every observation among all
 * others (the knncolle search called at include/umappp/initialize.hpp:140):
 * out_indices and out_distances are num_obs x k, sorted by increasing
 * distance, ties by index.  For F32 data the candidates are found with
 * split-precision tensor-core distances and the k-th boundary is rescored in
 * FP64; for F64 data distances are computed in FP64.  k must be below num_obs.
 */
int umapb_knn(int dtype, size_t data_dim, int32_t num_obs, const void* data, int k, int32_t* out_indices,
              void* out_distances);

/*
 * One shard of umapb_knn, for a neighbour search split across GPUs (every
 * rank holds the whole data and computes its shard; an all-gather of the
 * shards' rows gives every rank the full lists -- umappp_b200.distributed).
 * Shard 'shard' of 'num_shards' takes, for F32 data on the tensor-core path, a
 * contiguous range of the search's tree-ordered query tiles carrying an equal
 * share of the computed tile pairs, else a contiguous range of observations;
 * the shards partition the observations.  Writes *out_count rows, ascending:
 * out_rows[r] is an observation and out_indices / out_distances[r * k ..) its
 * neighbours as umapb_knn gives them.  The output arrays need room for
 * num_obs rows (host or device memory).  An extension: the reference's
 * search runs on one machine.
 */
int umapb_knn_shard(int dtype, size_t data_dim, int32_t num_obs, const void* data, int k, int32_t shard,
                    int32_t num_shards, int32_t* out_rows, int32_t* out_indices, void* out_distances,
                    int32_t* out_count);

/* Exact Euclidean neighbours of num_query query points among num_ref reference
 * points (row-major data_dim columns each): out_indices / out_distances are
 * num_query x k, reference indices sorted by (distance, index).  The
 * knncolle search of initialize.hpp:138-142 with the query and reference sets
 * apart (the search the transform below makes). */
int umapb_knn_query(int dtype, size_t data_dim, int32_t num_ref, const void* ref_data, int32_t num_query,
                    const void* query_data, int k, int32_t* out_indices, void* out_distances);

/* Out-of-sample embedding (an extension: the reference has no transform).
 * new_embedding (num_new x num_dim) receives the positions of new points in a
 * finished layout of num_ref reference points (ref_data: num_ref x data_dim,
 * ref_embedding: num_ref x num_dim, neither changed):
 *   1. each new point's options->num_neighbors nearest reference points
 *      (umapb_knn_query) and their similarities (neighbor_similarities.hpp with
 *      the options' local_connectivity and bandwidth);
 *   2. start at the similarity-weighted mean of those neighbours' positions;
 *   3. the schedule of similarities_to_epochs over these edges and
 *      optimize_layout's per-row steps (optimize_layout.hpp:136-180) in which
 *      only the new point moves and the negative samples are reference points
 *      (seeded by optimize_seed), at a quarter of learning_rate.
 * num_epochs <= 0 picks the count: a third of options->num_epochs when that is
 * set, else 100 for up to 10,000 new points and 30 above
 * (umapb_transform_epochs).  The result does not depend on launch shapes. */
int umapb_transform(int dtype, size_t data_dim, int32_t num_ref, const void* ref_data, const void* ref_embedding,
                    int32_t num_new, const void* new_data, size_t num_dim, const umapb_options* options,
                    int num_epochs, void* new_embedding);
/* The epoch count umapb_transform uses for these arguments (an extension, as
 * umapb_transform). */
int umapb_transform_epochs(const umapb_options* options, int num_epochs, int32_t num_new);

/* Queries of the last F32 neighbour search in this process whose candidate
 * set could not be certified by the error bound and were recomputed in FP64.
 * No reference counterpart: a diagnostic of the search. */
int umapb_knn_last_fp64_recomputed(void);

/* Largest error of the tensor-core squared distances of the last float kNN
 * on this process, relative to |q|^2 + max |r|^2 (the scale of the bound that
 * decides which queries are recomputed in FP64); 0 if the last search did not
 * use tensor cores.  No reference counterpart: a precision diagnostic. */
double umapb_knn_last_tc_error(void);

/* Query-tile x reference-tile pairs (128 x 128 squared distances each) that
 * the last tensor-core kNN of this process computed: with tile pruning, the
 * work left of the (n / 128)^2 of a brute-force search.  No reference
 * counterpart: a diagnostic of the search. */
int64_t umapb_knn_last_tile_pairs(void);

/* Device time in milliseconds of the last tensor-core candidate kernel
 * (FP16 search) of this process, from CUDA events around its launch.  No
 * reference counterpart: a measurement hook. */
double umapb_knn_last_kernel_ms(void);

/*
 * neighbor_similarities (include/umappp/neighbor_similarities.hpp:53-207):
 * replaces the distances of each CSR row by membership weights in place.
 * rho_out / sigma_out (may be NULL) receive per-row rho and sigma as double
 * (NaN for rows the reference returns early).  use_newton selects the
 * Newton-with-bisection search (the default) or bisection only.
 */
int umapb_neighbor_similarities(int dtype, int32_t num_obs, const int64_t* row_ptr, void* distances,
                                double local_connectivity, double bandwidth, double min_k_dist_scale, int use_newton,
                                double* rho_out, double* sigma_out);

/*
 * combine_neighbor_sets (include/umappp/combine_neighbor_sets.hpp:16-99):
 * symmetrises a weighted CSR neighbour list into out_* (rows sorted by
 * index).  out_indices/out_weights must hold 'capacity' entries
 * (2 * row_ptr[num_obs] always suffices); *out_nnz receives the count.
 */
int umapb_combine_neighbor_sets(int dtype, int32_t num_obs, const int64_t* row_ptr, const int32_t* indices,
                                const void* weights, double mix_ratio, int64_t* out_row_ptr, int32_t* out_indices,
                                void* out_weights, int64_t capacity, int64_t* out_nnz);

/*
 * similarities_to_epochs (include/umappp/optimize_layout.hpp:47-92): keeps
 * edges with weight >= max / num_epochs and writes the per-edge schedule.
 * Output arrays must hold row_ptr[num_obs] entries; *out_nnz receives the
 * kept count.
 */
int umapb_similarities_to_epochs(int dtype, int32_t num_obs, const int64_t* row_ptr, const int32_t* indices,
                                 const void* weights, int num_epochs, double negative_sample_rate,
                                 int64_t* out_row_ptr, int32_t* out_targets, void* epochs_per_sample,
                                 void* epoch_of_next_sample, void* epoch_of_next_negative_sample, int64_t* out_nnz);

/* has_multiple_components (include/umappp/spectral_init.hpp:142-168); *out = 0 or 1. */
int umapb_has_multiple_components(int32_t num_obs, const int64_t* row_ptr, const int32_t* indices, int* out);

/*
 * spectral_init (include/umappp/spectral_init.hpp:171-207): *ok = 1 and the
 * scaled eigenvectors of the normalised Laplacian in 'embedding'
 * (num_obs x num_dim), or *ok = 0 (several components / no convergence,
 * embedding untouched).  evals_out (may be NULL) receives num_dim + 1
 * eigenvalues of I + D^-1/2 W D^-1/2 in decreasing order.
 */
int umapb_spectral_init(int dtype, int32_t num_obs, const int64_t* row_ptr, const int32_t* indices,
                        const void* weights, size_t num_dim, void* embedding, int extra_work, int max_iterations,
                        double tolerance, double scale, int jitter, double jitter_sd, uint64_t seed, int* ok,
                        double* evals_out);

/* random_init (include/umappp/spectral_init.hpp:209-225): uniform on (-scale, scale). */
int umapb_random_init(int dtype, int32_t num_obs, size_t num_dim, void* embedding, uint64_t seed, double scale);

/* find_ab (include/umappp/find_ab.hpp:44-168). */
int umapb_find_ab(double spread, double min_dist, double* a, double* b);

/* choose_num_epochs (include/umappp/initialize.hpp:27-47). */
int umapb_choose_num_epochs(int has_value, int value, int64_t num_obs);

/*
 * optimize_layout (include/umappp/optimize_layout.hpp:116-185) on the device
 * from the given schedule state: advances epochs [*current_epoch,
 * epoch_limit), updating the embedding and epoch_of_next_* in place and
 * *current_epoch.  Negative samples come from a counter-based generator keyed
 * by (seed, epoch, edge), so the result does not depend on how the epochs
 * are split across calls.
 */
int umapb_optimize_layout(int dtype, size_t num_dim, void* embedding, int32_t num_obs, const int64_t* row_ptr,
                          const int32_t* targets, const void* epochs_per_sample, void* epoch_of_next_sample,
                          void* epoch_of_next_negative_sample, double negative_sample_rate, int total_epochs,
                          int* current_epoch, double a, double b, double gamma, double learning_rate, uint64_t seed,
                          int epoch_limit);

/* ----------------------------------------------------------------- batched */

/*
 * Many independent UMAP instances in one call (no counterpart in the
 * reference, where each would be its own initialize() + run()).  Instance i is
 * the next sizes[i] observations of 'data' (num_instances blocks one after
 * another, data_dim values per observation); its embedding is written to the
 * matching rows of 'embedding'.  Every instance uses 'opt' as one
 * initialize(data, builder, ...) + Status::run() would, with these shared
 * steps: one tensor-core kNN launch over all instances (each query searches
 * its own instance only), one similarity / union / schedule pass over the
 * block-diagonal graph (each instance keeps its own maximum weight), and one
 * SGD launch per epoch over all instances (negative samples drawn inside the
 * head's instance), the epochs recorded as one CUDA graph, with the launch
 * shape chosen by the autotuner.  All instances must resolve to the same
 * epoch count (set opt->num_epochs when their sizes differ across 10000).
 * stage_ms (may be NULL) receives the 7 stage times of umapb_status_stage_ms.
 */
int umapb_batch_run(int dtype, int32_t num_instances, const int32_t* sizes, size_t data_dim, const void* data,
                    size_t num_dim, void* embedding, const umapb_options* opt, double* stage_ms);

/* ----------------------------------------------------------------- adjoint */

/*
 * Loss and gradient of the UMAP fuzzy cross-entropy (no counterpart in the
 * reference, which only applies its per-edge derivatives,
 * include/umappp/optimize_layout.hpp:148-149,171):
 *   L = sum over stored edges (i -> j, w) of
 *       w * (-log q) + (1 - w) * (-log(1 - q)) [+ w log w + (1 - w) log(1 - w) if with_constant]
 *   q = 1 / (1 + a d^(2b)),  d = |y_i - y_j|.
 * With eps_rep > 0 the repulsive derivative uses 1 / (d^2 + eps_rep) in place
 * of 1 / d^2, as the reference's step does (eps 0.001).  Outputs: *loss,
 * grad_embedding (num_obs x num_dim, may be NULL), grad_ab[2] = dL/da, dL/db
 * (may be NULL).  Accumulation is FP64 for both dtypes.  A row_ptr that does
 * not run upwards within [0, row_ptr[num_obs]], or an index outside
 * [0, num_obs), is reported as UMAPB_ERR_INVALID (detected on the device; the
 * bad edges are not read).
 */
int umapb_loss_grad(int dtype, size_t num_dim, const void* embedding, int32_t num_obs, const int64_t* row_ptr,
                    const int32_t* indices, const void* weights, double a, double b, double eps_rep,
                    int with_constant, double* loss, void* grad_embedding, double* grad_ab);

/*
 * umapb_loss_grad without any device allocation.  It has no counterpart in
 * the reference.
 *
 * For callers that cannot call cudaMalloc: a framework that owns all device
 * memory through its own pool (where a stray allocation fails or fragments
 * it), or a serving loop whose per-request path must not block on the
 * allocator, which also synchronises the device.  Same arguments and results as
 * umapb_loss_grad, with these differences:
 *   - embedding, row_ptr, indices, weights and grad_embedding must be device
 *     memory of the current device (host pointers and other devices' memory
 *     are rejected with UMAPB_ERR_INVALID); loss and grad_ab are host memory;
 *     with num_obs == 0 no pointer is read (NULL is accepted) and the results
 *     are zero;
 *   - the work runs on the calling thread's per-thread default stream;
 *   - its scratch is a fixed array in the library's device memory (32 MB on
 *     every device that loads the library, held until exit); for UMAPB_F32 a
 *     gradient of more than 4,194,304 elements (num_obs * num_dim) is rejected
 *     with UMAPB_ERR_INVALID;
 *   - the first call on a device looks up the scratch's device address
 *     (cudaGetSymbolAddress) and keeps it for the life of the process; make
 *     that first call before any stream capture, and make no call after a
 *     cudaDeviceReset of that device;
 *   - every call shares the one scratch array, so calls that overlap on the
 *     GPU (other threads, other streams) race; serialise them.
 */
int umapb_loss_grad_noalloc(int dtype, size_t num_dim, const void* embedding, int32_t num_obs, const int64_t* row_ptr,
                            const int32_t* indices, const void* weights, double a, double b, double eps_rep,
                            int with_constant, double* loss, void* grad_embedding, double* grad_ab);

#ifdef __cplusplus
}
#endif

#endif
