// Device-side stage functions of the UMAP pipeline.  All pointers are device
// pointers; all work is enqueued on the given stream.  Float_ is the storage
// type of distances, weights, schedules and embeddings (float or double).
#pragma once

#include <vector>

#include "common.cuh"

namespace umapb {

// Weighted graph / neighbour list in CSR form, owned on the device.
template <typename T>
struct DeviceCsr {
    int32_t n = 0;
    int64_t nnz = 0;
    DevArray<int64_t> ptr;
    DevArray<int32_t> idx;
    DevArray<T> val;
};

// The reference's EpochData (include/umappp/optimize_layout.hpp:27-45) on the
// device, plus the head (row) of every edge.
template <typename T>
struct DeviceEpochs {
    int32_t n = 0;
    int64_t nnz = 0;
    int total_epochs = 0;
    T negative_sample_rate = 0;
    DevArray<int64_t> ptr;
    DevArray<int32_t> heads;
    DevArray<int32_t> targets;
    DevArray<T> eps;     // epochs_per_sample
    DevArray<T> enext0;  // epoch_of_next_sample at epoch 0
    DevArray<T> enneg0;  // epoch_of_next_negative_sample at epoch 0
};

// ---- kNN (knn.cu) ----------------------------------------------------------
// The shard of a neighbour search split across ranks: shard 'index' of
// 'count' takes a contiguous range of the query tiles in tree order with an
// equal share of the tile pairs (count 1: everything).
struct KnnShard {
    int32_t index = 0, count = 1;
};
// Exact Euclidean neighbours: out_idx/out_dist are n x k row-major, sorted by
// (distance, index), self excluded.  Float data: FP32 candidate search then
// FP64 rescoring of the candidate set; double data: FP64 throughout.
template <typename T>
void knn_exact(const T* data, int32_t n, int32_t dim, int32_t k, int32_t* out_idx, T* out_dist, cudaStream_t s,
               double* out_dist_f64 = nullptr);
// The shard's part of knn_exact: its queries' data rows in rows[0, nrows)
// (ascending), their neighbours at those rows of out_idx / out_dist.
template <typename T>
void knn_exact_shard(const T* data, int32_t n, int32_t dim, int32_t k, KnnShard shard, int32_t* out_idx, T* out_dist,
                     DevArray<int32_t>& rows, int32_t& nrows, cudaStream_t s);

// Tensor-core candidate search (knn_tc.cu): KCAP candidates per query with
// FP32 squared distances; norms_out receives |x|^2 (n rounded up to 128 entries).
bool knn_tc_supported(int32_t dim, int kcap);
// With a shard (count > 1): only the shard's queries (their data rows in
// *shard_rows, *shard_count of them); returns false, computing nothing, when
// the search in use cannot be sharded.
bool knn_tc_candidates(const float* data, int32_t n, int32_t dim, int kcap, int32_t* cand_idx, float* cand_d2,
                       float* norms_out, int* d_err, cudaStream_t s, KnnShard shard = KnnShard(),
                       DevArray<int32_t>* shard_rows = nullptr, int32_t* shard_count = nullptr,
                       DevArray<int32_t>* tree_rows = nullptr);
// Batched: instance i is data rows [inst[i], inst[i + 1]) (host vector).
void knn_tc_candidates_batched(const float* data, const std::vector<int32_t>& inst, int32_t dim, int kcap,
                               int32_t* cand_idx, float* cand_d2, int* d_err, cudaStream_t s);
// Tile pruning (knn_tree.cu).  KnnTiles: operand row -> data row map of the
// padded, tree-ordered operands (-1 for padding), each instance starting at
// pad_start[i] (a multiple of 128).  KnnTasks: per query block of the search
// {first operand row, offset and length of its reference-tile list, end of
// its instance's rows}, and the concatenated lists.
struct KnnTiles {
    DevArray<int32_t> row_map;
    std::vector<int32_t> pad_start;
    int32_t n_pad = 0;
};
struct KnnTasks {
    DevArray<int4> tasks;          // per CTA: {first operand row, first query tile, query tiles, 0}
    DevArray<int64_t> qlist_off;   // per query tile: its reference tiles are
    DevArray<int32_t> qlist_len;   //   tile_list[qlist_off .. + qlist_len)
    DevArray<int32_t> tile_list;
    int32_t count = 0;
    int64_t total_tiles = 0;       // sum of the query tiles' list lengths
    std::vector<int4> host_tasks;  // the tasks, in launch order
};
// Data rows of the query tiles of a task list (ascending): the rows a sharded
// search computes.
// The data rows in tree order (the operand rows without padding): n entries.
void knn_tree_rows(const KnnTiles& t, int32_t n, DevArray<int32_t>& rows, cudaStream_t s);
void knn_task_rows(const KnnTiles& t, const KnnTasks& tk, int32_t n, DevArray<int32_t>& rows, int32_t& count,
                   cudaStream_t s);
// tree == false keeps each instance in data order.
void knn_tree_order(const float* data, int32_t dim, const std::vector<int32_t>& inst, bool tree, KnnTiles& out,
                    cudaStream_t s);
// Every query tile lists the reference tiles of its instance that may hold one
// of its rows' k nearest neighbours (all of them when prune is false); CTAs
// take qt consecutive query tiles of one instance.
void knn_tile_tasks(const float* data, int32_t dim, const KnnTiles& t, const std::vector<int32_t>& inst, int qt,
                    int32_t k, bool prune, KnnTasks& out, cudaStream_t s, KnnShard shard = KnnShard());
// Candidate search over tree-ordered operands and task lists; candidate and
// norm outputs are indexed by data row.
void knn_tc16_run_tasks(const float* data, int32_t dim, int kcap, float scale, const KnnTiles& tiles,
                        const KnnTasks& tasks, int32_t* cand_idx, float* cand_d2, float* norms_by_row, int* d_err,
                        cudaStream_t s, float* kernel_ms = nullptr, int shape = 0);
// Launch shapes of the FP16 search for 'dim', coded 10 * query tiles per CTA +
// reference-ring stages (the first is the default; the tasks must be built
// with the shape's query tiles, shape / 10).
std::vector<int> knn_tc16_shapes(int32_t dim);

// FP16-operand variant (knn_tc16.cu): power-of-two scale of the data (0 when
// unusable), support test, query tiles per CTA, and the search itself.
float knn_tc16_scale(const float* data, size_t count, cudaStream_t s);
bool knn_tc16_supported(int32_t dim, int kcap);
int knn_tc16_query_tiles(int32_t dim);
// Number of queries the last float kNN recomputed in FP64 (certainty check).
int& last_knn_redo_count();
// Query-tile x reference-tile pairs (128 x 128 distances each) computed by the
// last tensor-core candidate search: the work left after pruning.
int64_t& last_knn_tiles_scanned();
// Device time (ms) of the last tensor-core candidate kernel (FP16 search).
float& last_knn_kernel_ms();
// Largest |tensor-core FP32 squared distance - FP64 squared distance| /
// (|q|^2 + max |r|^2) over the candidates of the last float kNN (0 without
// the tensor-core search).
double& last_knn_tc_error();

// Exact kNN of every observation within its own instance (instance i is data
// rows [inst[i], inst[i + 1]), host vector); indices are data rows.
// Exact Euclidean neighbours of nq query points among nref reference points:
// 'data' holds the reference rows [0, nref) followed by the query rows
// [nref, nref + nq); out_idx/out_dist are nq x k in query order, reference
// indices sorted by (distance, index).  Float data: FP32 candidates, FP64
// rescoring and certification; double data: FP64 throughout.
template <typename T>
void knn_query(const T* data, int32_t nref, int32_t nq, int32_t dim, int32_t k, int32_t* out_idx, T* out_dist,
               cudaStream_t s);

template <typename T>
void knn_exact_batched(const T* data, const std::vector<int32_t>& inst, int32_t dim, int32_t k, int32_t* out_idx,
                       T* out_dist, cudaStream_t s);

// ---- similarities (similarities.cu) -----------------------------------------
template <typename T>
void neighbor_similarities(int32_t n, const int64_t* ptr, T* val, double local_connectivity, double bandwidth,
                           double min_k_dist_scale, bool use_newton, double* rho_out, double* sigma_out,
                           cudaStream_t s);

// ---- graph (graph.cu) -------------------------------------------------------
template <typename T>
void combine_neighbor_sets(int32_t n, const int64_t* ptr, const int32_t* idx, const T* w, int64_t nnz_in,
                           double mix_ratio, DeviceCsr<T>& out, cudaStream_t s);

// inst_start (device, num_inst + 1 entries) splits the rows into independent
// instances, each with its own maximum weight (batched runs); NULL: one instance.
template <typename T>
void similarities_to_epochs(int32_t n, const int64_t* ptr, const int32_t* idx, const T* w, int64_t nnz,
                            int num_epochs, double negative_sample_rate, DeviceEpochs<T>& out, cudaStream_t s,
                            const int32_t* inst_start = nullptr, int32_t num_inst = 1);

// Number of connected components (undirected union-find); status word set on timeout.
int64_t count_components(int32_t n, const int64_t* ptr, const int32_t* idx, int* d_status, cudaStream_t s);

// ---- initial layouts (spectral.cu) -------------------------------------------
struct SpectralResult {
    bool ok = false;
    int restarts = 0;
    double evals[64] = {0};
};

template <typename T>
SpectralResult spectral_init(int32_t n, const int64_t* ptr, const int32_t* idx, const T* w, int num_dim, T* Y,
                             int extra_work, int max_iterations, double tol, double scale, bool jitter,
                             double jitter_sd, uint64_t seed, int* d_status, cudaStream_t s);

template <typename T>
void random_init(int32_t n, int num_dim, T* Y, uint64_t seed, double scale, cudaStream_t s);

// ---- SGD (sgd.cu) -----------------------------------------------------------
// Epochs of the reference's SGD: one thread per head row, the schedule
// advanced in place in the reference's Float_ arithmetic (see sgd.cu).
template <typename T>
class SgdEngine {
public:
    // ep->enext0 / enneg0 describe the schedule at epoch 'base_epoch'.
    void setup(const DeviceEpochs<T>* ep, cudaStream_t s, int base_epoch = 0);
    // Runs epochs [first, last) on Y (n x num_dim, device).  ms_schedule is
    // always 0 (no schedule stage); ms_sgd is the epochs' device time.
    void run(T* Y, int num_dim, int first, int last, double a, double b, double gamma, double learning_rate,
             uint64_t seed, cudaStream_t s, float* ms_schedule, float* ms_sgd);
    // Exact per-epoch [firing, negatives] counts over [first, last) (host output).
    void counts(int first, int last, int64_t* out, cudaStream_t s);
    // Schedule state (enext, enneg) at 'epoch' into device arrays.
    void state_at(int epoch, T* enext, T* enneg, cudaStream_t s);
    // Batched runs: instance i owns observations [inst_start[i], inst_start[i+1])
    // (device array of num_inst + 1 entries); negative samples stay inside it.
    void set_instances(const int32_t* inst_start, int32_t num_inst) {
        inst_start_ = inst_start;
        num_inst_ = num_inst;
    }
    // Record the epochs of each run() call as one CUDA graph and launch that.
    bool use_graphs = false;
    // Pick the 2-d epoch kernel's block size and variant by timing the
    // candidates on scratch copies (sgd.cu, tune()).
    bool autotune = false;
    // Firing edges between publications of a row's head (sgd.cu).
    int publish_every = default_publish_every();
    // Rows in flight at most n / window_div (sgd.cu, run(); 0: no cap).
    int window_div = default_window_div();
    // 2-d kernel: each epoch after the first of a run() call claims its rows
    // sorted by this epoch's firing edges within chunks of the run's order
    // (sgd.cu, epoch_bulk_order_kernel).
    bool epoch_order = default_epoch_order();
    int block_size() const { return block_; }
    int variant() const { return variant_; }   // 2-d kernel variant (sgd.cu, SGD_2D_VARIANTS)

private:
    template <class Launch>
    void tune(T* Y, int num_dim, int epoch, Launch& launch, cudaStream_t s);
    static int default_variant();
    static int default_publish_every();
    static int default_window_div();
    static bool default_epoch_order();
    int block_ = 256, variant_ = default_variant();
    const DeviceEpochs<T>* ep_ = nullptr;
    DevArray<uint16_t> next_count_;   // per row: firing edges in the next epoch
    DevArray<int32_t> bulk_;          // this epoch's claim order of the non-hub rows
    const int32_t* inst_start_ = nullptr;
    int32_t num_inst_ = 1;
    int base_epoch_ = 0;
    DevArray<T> enext_, enneg_;    // schedule state at state_epoch_
    DevArray<int32_t> order_;      // rows by descending firing rate
    int nhub_ = 0;                 // leading rows of order_ taken by a whole warp (2-d kernel)
    int state_epoch_ = 0;          // epoch the state arrays describe
};

// ---- adjoint (adjoint.cu) ----------------------------------------------------
// ---- transform (sgd.cu) -------------------------------------------------------
// Out-of-sample embedding of nq new points against a fixed reference layout
// Yref (nref points): transform_init puts every new point at the
// similarity-weighted mean of its neighbours' positions (CSR ptr/idx/w over
// the new points, reference indices); transform_layout then runs the
// schedule 'ep' (rows = new points, targets = reference points) with only the
// new points moving and negative samples drawn among the reference points.
template <typename T>
void transform_init(int32_t nq, int num_dim, const int64_t* ptr, const int32_t* idx, const T* w, const T* Yref,
                    T* Ynew, cudaStream_t s);
template <typename T>
void transform_layout(const DeviceEpochs<T>& ep, int num_dim, const T* Yref, int32_t nref, T* Ynew, int32_t head0,
                      double a, double b, double gamma, double learning_rate, uint64_t seed, cudaStream_t s);

template <typename T>
void loss_grad(int32_t n, int num_dim, const T* Y, const int64_t* ptr, const int32_t* idx, const T* w, double a,
               double b, double eps_rep, bool with_constant, double* loss_out, T* grad_Y, double* grad_ab,
               cudaStream_t s);

// ---- roofline probes (probe.cu) ----------------------------------------------
// Random float2 accesses per second over an n-point array (mode 0: L2 gathers,
// 1: atomic adds).
double measure_random_access(int64_t n, int64_t accesses, int mode, int reps, cudaStream_t s);

// ---- host (find_ab.cpp) -------------------------------------------------------
void find_ab(double spread, double min_dist, double* a, double* b);
int choose_num_epochs(bool has_value, int value, int64_t n);

}  // namespace umapb
