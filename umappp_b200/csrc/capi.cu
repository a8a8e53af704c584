// The C ABI (include/umapb.h) and the host orchestration behind it: the
// reference's initialize() / Status::run() pipeline
// (include/umappp/initialize.hpp:69-177, include/umappp/Status.hpp:25-141)
// driven as a sequence of device stages on one CUDA stream per status.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "stages.cuh"
#include "umapb.h"

namespace umapb {

std::atomic<long long> g_launches{0};
std::atomic<long long> g_wait_limit{1ll << 26};

namespace {

thread_local std::string g_last_error;

void set_error(const std::string& m) { g_last_error = m; }

// Fails unless a compute capability 10.x device is current (the library
// carries sm_100a code only; there is no CPU path).
void require_device() {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        fail(UMAPB_ERR_NO_DEVICE, "no CUDA device is available (libumappp_b200 runs on sm_100 GPUs only)");
    }
    int dev = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    int major = 0;
    UMAPB_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) fail(UMAPB_ERR_NO_DEVICE, "the current CUDA device is not sm_100 (B200/GB200)");
    // Keep freed stream-ordered allocations in the device pool instead of
    // unmapping them at every synchronisation: the schedule windows are tens of
    // GB and are re-created on every run.
    thread_local int pooled_device = -1;
    if (pooled_device != dev) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
        pooled_device = dev;
    }
}

}  // namespace

void set_last_error(const std::string& m) { set_error(m); }

Context& thread_context() {
    thread_local Context ctx;
    int dev = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    if (ctx.device != dev) {
        UMAPB_CUDA(cudaStreamCreateWithFlags(&ctx.stream, cudaStreamNonBlocking));
        UMAPB_CUDA(cudaMalloc(reinterpret_cast<void**>(&ctx.d_status), sizeof(int)));
        UMAPB_CUDA(cudaMemset(ctx.d_status, 0, sizeof(int)));
        ctx.device = dev;
    }
    return ctx;
}

// ------------------------------------------------------------- status ---

struct StatusBase {
    virtual ~StatusBase() = default;
    virtual void run(void* embedding, int epoch_limit) = 0;
    virtual int64_t num_edges() const = 0;
    virtual void epoch_data(int64_t* ptr, int32_t* targets, void* eps, void* enext, void* enneg) = 0;
    virtual void counts(int first, int last, int64_t* out) = 0;
};

}  // namespace umapb

// A search index resident on the device (the role of knncolle::Prebuilt): the
// data, kept for repeated neighbour searches without copying it again.
struct umapb_prebuilt {
    int dtype = UMAPB_F32;
    int device = 0;
    size_t dim = 0;
    int32_t n = 0;
    size_t bytes = 0;
    void* data = nullptr;
    ~umapb_prebuilt() {
        if (data) cudaFree(data);
    }
};

struct umapb_status {
    int dtype = UMAPB_F32;
    int device = 0;
    cudaStream_t stream = nullptr;
    int* d_status = nullptr;
    int32_t n = 0;
    size_t num_dim = 0;
    umapb_options opt{};
    double a = 0, b = 0;
    int num_epochs = 0;
    int current_epoch = 0;
    float stage_ms[7] = {0, 0, 0, 0, 0, 0, 0};
    std::unique_ptr<umapb::StatusBase> impl;

    ~umapb_status() {
        impl.reset();
        if (stream) {
            if (d_status) umapb::ws_free(d_status, stream);
            cudaStreamSynchronize(stream);
            umapb::stream_put(stream);   // streams are pooled: creating one is a resource-manager call
        }
    }
};

namespace umapb {

namespace {

enum Stage { ST_KNN = 0, ST_SIM, ST_UNION, ST_INIT, ST_EPOCHS, ST_SCHEDULE, ST_SGD };
const char* const STAGE_RANGE[] = {"umapb knn", "umapb similarities", "umapb union", "umapb init",
                                   "umapb epochs", "umapb schedule", "umapb sgd"};

// An NVTX range on the calling host thread for the life of the object: the
// stages and calls show by name on a profiler's timeline (and ncu can filter
// on them with --nvtx); without a tool attached the calls return at once.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Event pair per stage, resolved at the end of a call; each stage is also an
// NVTX range (closed by end(), or by the destructor when a stage throws).
struct StageTimer {
    cudaStream_t s;
    float* out;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
    int open = 0;
    explicit StageTimer(cudaStream_t st, float* o) : s(st), out(o) {}
    void begin(int stage) {
        cudaEvent_t a = event_get(), b = event_get();
        UMAPB_CUDA(cudaEventRecord(a, s));
        marks.push_back({stage, {a, b}});
        nvtxRangePushA(STAGE_RANGE[stage]);
        ++open;
    }
    void end() {
        if (open > 0) {
            nvtxRangePop();
            --open;
        }
        UMAPB_CUDA(cudaEventRecord(marks.back().second.second, s));
    }
    void resolve() {
        UMAPB_SYNC(s);
        for (auto& m : marks) {
            float t = 0;
            cudaEventElapsedTime(&t, m.second.first, m.second.second);
            out[m.first] = t;
        }
    }
    ~StageTimer() {
        for (; open > 0; --open) nvtxRangePop();
        for (auto& m : marks) {
            event_put(m.second.first);
            event_put(m.second.second);
        }
    }
};

__global__ void dense_row_ptr_kernel(int32_t n, int32_t k, int64_t* ptr) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i <= n; i += int64_t(gridDim.x) * blockDim.x)
        ptr[i] = i * k;
}

template <typename T>
struct StatusImpl final : StatusBase {
    umapb_status* st;
    DeviceEpochs<T> epochs;
    SgdEngine<T> engine;

    explicit StatusImpl(umapb_status* s) : st(s) {}

    // Stages after the neighbour search (initialize.hpp:69-119).  ptr/idx/dist
    // are device arrays; dist is consumed (turned into weights).
    void initialize(const int64_t* ptr, const int32_t* idx, T* dist, int64_t nnz, void* embedding, StageTimer& tm) {
        cudaStream_t s = st->stream;
        const umapb_options& o = st->opt;
        const int32_t n = st->n;

        tm.begin(ST_SIM);
        neighbor_similarities<T>(n, ptr, dist, o.local_connectivity, o.bandwidth, 1e-3, true, nullptr, nullptr, s);
        tm.end();

        tm.begin(ST_UNION);
        DeviceCsr<T> g;
        combine_neighbor_sets<T>(n, ptr, idx, dist, nnz, o.mix_ratio, g, s);
        tm.end();

        // initial layout (initialize.hpp:79-103)
        tm.begin(ST_INIT);
        const size_t total = static_cast<size_t>(n) * st->num_dim;
        DeviceInOut<T> Y(static_cast<T*>(embedding), total, s, /*load=*/false);
        bool wrote = false;
        bool use_random = (o.initialize_method == UMAPB_INIT_RANDOM);
        if (o.initialize_method == UMAPB_INIT_SPECTRAL) {
            const SpectralResult r = spectral_init<T>(
                n, g.ptr.get(), g.idx.get(), g.val.get(), static_cast<int>(st->num_dim), Y.get(), o.irlba_extra_work,
                o.irlba_max_iterations, o.irlba_convergence_tolerance, o.initialize_spectral_scale,
                o.initialize_spectral_jitter != 0, o.initialize_spectral_jitter_sd, o.initialize_seed, st->d_status, s);
            wrote = r.ok;
            use_random = (o.initialize_random_on_spectral_fail != 0 && !r.ok);
        }
        if (use_random) {
            random_init<T>(n, static_cast<int>(st->num_dim), Y.get(), o.initialize_seed, o.initialize_random_scale, s);
            wrote = true;
        }
        if (wrote) Y.finish();
        tm.end();

        // a, b (initialize.hpp:105-110) and the epoch count (:112)
        if (!o.has_a || !o.has_b) {
            find_ab(o.spread, o.min_dist, &st->a, &st->b);
        } else {
            st->a = o.a;
            st->b = o.b;
        }
        st->num_epochs = choose_num_epochs(o.has_num_epochs != 0, o.num_epochs, n);

        tm.begin(ST_EPOCHS);
        similarities_to_epochs<T>(n, g.ptr.get(), g.idx.get(), g.val.get(), g.nnz, st->num_epochs,
                                  o.negative_sample_rate, epochs, s);
        engine.setup(&epochs, s);
        tm.end();
        st->current_epoch = 0;
    }

    void run(void* embedding, int epoch_limit) override {
        cudaStream_t s = st->stream;
        if (epoch_limit <= st->current_epoch) return;
        const size_t total = static_cast<size_t>(st->n) * st->num_dim;
        DeviceInOut<T> Y(static_cast<T*>(embedding), total, s, /*load=*/true);
        float ms_sched = 0, ms_sgd = 0;
        engine.run(Y.get(), static_cast<int>(st->num_dim), st->current_epoch, epoch_limit, st->a, st->b,
                   st->opt.repulsion_strength, st->opt.learning_rate, st->opt.optimize_seed, s, &ms_sched, &ms_sgd);
        Y.finish();
        UMAPB_SYNC(s);
        st->stage_ms[ST_SCHEDULE] = ms_sched;
        st->stage_ms[ST_SGD] = ms_sgd;
        st->current_epoch = epoch_limit;
    }

    int64_t num_edges() const override { return epochs.nnz; }

    void epoch_data(int64_t* ptr, int32_t* targets, void* eps, void* enext, void* enneg) override {
        cudaStream_t s = st->stream;
        const int64_t nnz = epochs.nnz;
        copy_out(ptr, epochs.ptr.get(), sizeof(int64_t) * (static_cast<size_t>(st->n) + 1), s);
        copy_out(targets, epochs.targets.get(), sizeof(int32_t) * nnz, s);
        copy_out(eps, epochs.eps.get(), sizeof(T) * nnz, s);
        if (enext || enneg) {
            DevArray<T> a(nnz, s), b(nnz, s);
            engine.state_at(st->current_epoch, a.get(), b.get(), s);
            copy_out(enext, a.get(), sizeof(T) * nnz, s);
            copy_out(enneg, b.get(), sizeof(T) * nnz, s);
            UMAPB_SYNC(s);
        }
        UMAPB_SYNC(s);
    }

    void counts(int first, int last, int64_t* out) override { engine.counts(first, last, out, st->stream); }
};

std::unique_ptr<umapb_status> new_status(int dtype, int32_t n, size_t num_dim, const umapb_options* opt) {
    require_device();
    require(dtype == UMAPB_F32 || dtype == UMAPB_F64, "dtype must be UMAPB_F32 or UMAPB_F64");
    require(opt != nullptr, "options must not be NULL");
    require(n >= 0, "num_obs must be non-negative");
    require(num_dim >= 1 && num_dim <= 64, "num_dim must be between 1 and 64");
    auto st = std::make_unique<umapb_status>();
    st->dtype = dtype;
    UMAPB_CUDA(cudaGetDevice(&st->device));
    st->stream = stream_get();
    st->d_status = static_cast<int*>(ws_alloc(sizeof(int), st->stream));
    UMAPB_CUDA(cudaMemsetAsync(st->d_status, 0, sizeof(int), st->stream));
    st->n = n;
    st->num_dim = num_dim;
    st->opt = *opt;
    return st;
}

template <typename T>
void init_from_neighbors(umapb_status* st, const int64_t* row_ptr, const int32_t* indices, const void* distances,
                         void* embedding) {
    cudaStream_t s = st->stream;
    const int32_t n = st->n;
    require(row_ptr != nullptr, "row_ptr must not be NULL");
    // the row pointers are needed on the host for the edge count
    int64_t nnz = 0;
    if (is_device_pointer(row_ptr)) {
        UMAPB_CUDA(cudaMemcpyAsync(&nnz, row_ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);
    } else {
        nnz = row_ptr[n];
    }
    require(nnz >= 0, "row_ptr must be non-decreasing from 0");
    DeviceIn<int64_t> dptr(row_ptr, static_cast<size_t>(n) + 1, s);
    DeviceIn<int32_t> didx(indices, nnz, s);
    DevArray<T> w(nnz, s);
    if (nnz) UMAPB_CUDA(cudaMemcpyAsync(w.get(), distances, sizeof(T) * nnz, cudaMemcpyDefault, s));
    auto impl = std::make_unique<StatusImpl<T>>(st);
    StageTimer tm(s, st->stage_ms);
    impl->initialize(dptr.get(), didx.get(), w.get(), nnz, embedding, tm);
    tm.resolve();
    st->impl = std::move(impl);
}

template <typename T>
void init_from_data(umapb_status* st, size_t data_dim, const void* data, void* embedding) {
    cudaStream_t s = st->stream;
    const int32_t n = st->n;
    require(data_dim >= 1 && data_dim <= INT32_MAX, "data_dim must be positive");
    const int k = std::min<int>(st->opt.num_neighbors, n - 1);   // knncolle returns at most n - 1 neighbours
    require(st->opt.num_neighbors >= 1, "num_neighbors must be positive");
    StageTimer tm(s, st->stage_ms);
    // resident data (a prebuilt index of this device) is used in place, host data staged
    DeviceIn<T> d(static_cast<const T*>(data), static_cast<size_t>(n) * data_dim, s);
    const int64_t nnz = static_cast<int64_t>(n) * k;
    DevArray<int32_t> idx(nnz, s);
    DevArray<T> dist(nnz, s);
    DevArray<int64_t> ptr(static_cast<size_t>(n) + 1, s);
    tm.begin(ST_KNN);
    if (k >= 1) knn_exact<T>(d.get(), n, static_cast<int32_t>(data_dim), k, idx.get(), dist.get(), s);
    dense_row_ptr_kernel<<<grid_for(static_cast<size_t>(n) + 1, 256), 256, 0, s>>>(n, k, ptr.get());
    UMAPB_LAUNCH_CHECK();
    tm.end();
    auto impl = std::make_unique<StatusImpl<T>>(st);
    impl->initialize(ptr.get(), idx.get(), dist.get(), nnz, embedding, tm);
    tm.resolve();
    st->impl = std::move(impl);
}

// out[r * k + c] = in[rows[r] * k + c]
template <typename V>
__global__ void gather_rows_kernel(int32_t nrows, int32_t k, const int32_t* __restrict__ rows, const V* __restrict__ in,
                                   V* __restrict__ out) {
    const int64_t total = static_cast<int64_t>(nrows) * k;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = t / k, c = t % k;
        out[t] = in[static_cast<int64_t>(rows[r]) * k + c];
    }
}

__global__ void rebase_indices_kernel(int64_t total, const int32_t* __restrict__ in, int32_t base,
                                      int32_t* __restrict__ out) {
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x)
        out[t] = in[t] - base;
}

// Neighbour matrices with one column per observation (k x n, column-major:
// observation i's neighbours at [i k, (i + 1) k), sorted by distance) -- the
// layout of the reference's R harness (tests/R/package/src/test.cpp:9-19) and
// of knncolle's dense outputs.  Device arrays are used in place (no CSR is
// built on the host: the row pointers are i k); index_base 1 takes R's
// 1-based indices.
template <typename T>
void init_from_knn_matrix(umapb_status* st, int32_t k, const int32_t* indices, const void* distances,
                          int index_base, void* embedding) {
    cudaStream_t s = st->stream;
    const int32_t n = st->n;
    require(k >= 0 && k < n, "k must be in [0, num_obs)");
    require(index_base == 0 || index_base == 1, "index_base must be 0 or 1");
    const int64_t nnz = static_cast<int64_t>(n) * k;
    DeviceIn<int32_t> din(indices, nnz, s);
    DevArray<int32_t> rebased;
    const int32_t* idx = din.get();
    if (index_base != 0 && nnz) {
        rebased.allocate(nnz, s);
        rebase_indices_kernel<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, din.get(), index_base, rebased.get());
        UMAPB_LAUNCH_CHECK();
        idx = rebased.get();
    }
    DevArray<T> w(nnz, s);   // consumed (turned into weights)
    if (nnz) UMAPB_CUDA(cudaMemcpyAsync(w.get(), distances, sizeof(T) * nnz, cudaMemcpyDefault, s));
    DevArray<int64_t> ptr(static_cast<size_t>(n) + 1, s);
    dense_row_ptr_kernel<<<grid_for(static_cast<size_t>(n) + 1, 256), 256, 0, s>>>(n, k, ptr.get());
    UMAPB_LAUNCH_CHECK();
    auto impl = std::make_unique<StatusImpl<T>>(st);
    StageTimer tm(s, st->stage_ms);
    impl->initialize(ptr.get(), idx, w.get(), nnz, embedding, tm);
    tm.resolve();
    st->impl = std::move(impl);
}

// Rows [start, start + len) of a CSR graph as a graph of their own (indices shifted by -start).
__global__ void sub_csr_kernel(int32_t start, int32_t len, const int64_t* __restrict__ ptr,
                               const int32_t* __restrict__ idx, int64_t* __restrict__ sub_ptr,
                               int32_t* __restrict__ sub_idx) {
    const int64_t base = ptr[start];
    const int64_t nnz = ptr[start + len] - base;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t <= len; t += int64_t(gridDim.x) * blockDim.x)
        sub_ptr[t] = ptr[start + t] - base;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < nnz; t += int64_t(gridDim.x) * blockDim.x)
        sub_idx[t] = idx[base + t] - start;
}

// Batched pipeline (umapb_batch_run): the stages of init_from_data + run over
// all instances at once, instance boundaries carried by 'inst'.
template <typename T>
void batch_pipeline(const std::vector<int32_t>& inst, size_t data_dim, const void* data, size_t num_dim,
                    void* embedding, const umapb_options& o, float* stage_ms) {
    Context& ctx = thread_context();
    cudaStream_t s = ctx.stream;
    const int ninst = static_cast<int>(inst.size()) - 1;
    const int32_t n = inst[ninst];
    const int k = o.num_neighbors;
    require(k >= 1, "num_neighbors must be positive");
    require(data_dim >= 1 && data_dim <= INT32_MAX, "data_dim must be positive");
    int epochs = -1;
    for (int i = 0; i < ninst; ++i) {
        require(inst[i + 1] - inst[i] > k, "every instance needs more than num_neighbors observations");
        const int e = choose_num_epochs(o.has_num_epochs != 0, o.num_epochs, inst[i + 1] - inst[i]);
        require(epochs < 0 || e == epochs, "batched instances resolve to different epoch counts: set num_epochs");
        epochs = e;
    }
    StageTimer tm(s, stage_ms);
    DeviceIn<T> d(static_cast<const T*>(data), static_cast<size_t>(n) * data_dim, s);
    DevArray<int32_t> d_inst(inst.size(), s);
    UMAPB_CUDA(cudaMemcpyAsync(d_inst.get(), inst.data(), inst.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    const int64_t nnz = static_cast<int64_t>(n) * k;
    DevArray<int32_t> idx(nnz, s);
    DevArray<T> dist(nnz, s);
    DevArray<int64_t> ptr(static_cast<size_t>(n) + 1, s);
    tm.begin(ST_KNN);
    knn_exact_batched<T>(d.get(), inst, static_cast<int32_t>(data_dim), k, idx.get(), dist.get(), s);
    dense_row_ptr_kernel<<<grid_for(static_cast<size_t>(n) + 1, 256), 256, 0, s>>>(n, k, ptr.get());
    UMAPB_LAUNCH_CHECK();
    tm.end();

    tm.begin(ST_SIM);
    neighbor_similarities<T>(n, ptr.get(), dist.get(), o.local_connectivity, o.bandwidth, 1e-3, true, nullptr, nullptr, s);
    tm.end();
    tm.begin(ST_UNION);
    DeviceCsr<T> g;
    combine_neighbor_sets<T>(n, ptr.get(), idx.get(), dist.get(), nnz, o.mix_ratio, g, s);
    tm.end();

    // initial layouts, instance by instance (initialize.hpp:79-103)
    tm.begin(ST_INIT);
    DeviceInOut<T> Y(static_cast<T*>(embedding), static_cast<size_t>(n) * num_dim, s, /*load=*/true);
    std::vector<int64_t> hptr(inst.size());
    for (int i = 0; i <= ninst; ++i) {
        UMAPB_CUDA(cudaMemcpyAsync(&hptr[i], g.ptr.get() + inst[i], sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    }
    UMAPB_SYNC(s);
    for (int i = 0; i < ninst; ++i) {
        const int32_t start = inst[i], len = inst[i + 1] - inst[i];
        T* Yi = Y.get() + static_cast<size_t>(start) * num_dim;
        bool use_random = (o.initialize_method == UMAPB_INIT_RANDOM);
        if (o.initialize_method == UMAPB_INIT_SPECTRAL) {
            const int64_t sub_nnz = hptr[i + 1] - hptr[i];
            DevArray<int64_t> sp(static_cast<size_t>(len) + 1, s);
            DevArray<int32_t> si(std::max<int64_t>(sub_nnz, 1), s);
            sub_csr_kernel<<<grid_for(std::max<int64_t>(sub_nnz, len + 1), 256), 256, 0, s>>>(start, len, g.ptr.get(),
                                                                                            g.idx.get(), sp.get(),
                                                                                            si.get());
            UMAPB_LAUNCH_CHECK();
            const SpectralResult r = spectral_init<T>(
                len, sp.get(), si.get(), g.val.get() + hptr[i], static_cast<int>(num_dim), Yi, o.irlba_extra_work,
                o.irlba_max_iterations, o.irlba_convergence_tolerance, o.initialize_spectral_scale,
                o.initialize_spectral_jitter != 0, o.initialize_spectral_jitter_sd, o.initialize_seed, ctx.d_status, s);
            use_random = (o.initialize_random_on_spectral_fail != 0 && !r.ok);
        }
        if (use_random) {
            random_init<T>(len, static_cast<int>(num_dim), Yi, o.initialize_seed, o.initialize_random_scale, s);
        }
    }
    tm.end();

    double a = o.a, b = o.b;
    if (!o.has_a || !o.has_b) find_ab(o.spread, o.min_dist, &a, &b);
    tm.begin(ST_EPOCHS);
    DeviceEpochs<T> ep;
    similarities_to_epochs<T>(n, g.ptr.get(), g.idx.get(), g.val.get(), g.nnz, epochs, o.negative_sample_rate, ep, s,
                              d_inst.get(), ninst);
    SgdEngine<T> engine;
    engine.setup(&ep, s);
    engine.set_instances(d_inst.get(), ninst);
    engine.use_graphs = true;
    engine.autotune = true;
    tm.end();
    float ms_sched = 0, ms_sgd = 0;
    engine.run(Y.get(), static_cast<int>(num_dim), 0, epochs, a, b, o.repulsion_strength, o.learning_rate,
               o.optimize_seed, s, &ms_sched, &ms_sgd);
    Y.finish();
    tm.resolve();
    stage_ms[ST_SCHEDULE] = ms_sched;
    stage_ms[ST_SGD] = ms_sgd;
}

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return UMAPB_OK;
    } catch (const Error& e) {
        set_error(e.what());
        cudaGetLastError();
        return e.code;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return UMAPB_ERR_OOM;
    } catch (const std::exception& e) {
        set_error(e.what());
        return UMAPB_ERR_INVALID;
    } catch (...) {
        set_error("unknown error");
        return UMAPB_ERR_INVALID;
    }
}


int64_t host_nnz(const int64_t* row_ptr, int32_t n, cudaStream_t s) {
    require(row_ptr != nullptr, "row_ptr must not be NULL");
    int64_t nnz = 0;
    if (is_device_pointer(row_ptr)) {
        UMAPB_CUDA(cudaMemcpyAsync(&nnz, row_ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);
    } else {
        nnz = row_ptr[n];
    }
    require(nnz >= 0, "row_ptr must be non-decreasing from 0");
    return nnz;
}

}  // namespace

void check_device_status(Context& ctx) {
    int st = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&st, ctx.d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    UMAPB_SYNC(ctx.stream);
    if (st != DEV_OK) {
        UMAPB_CUDA(cudaMemsetAsync(ctx.d_status, 0, sizeof(int), ctx.stream));
        if (st == DEV_TIMEOUT) fail(UMAPB_ERR_DEVICE_TIMEOUT, "a bounded device wait gave up");
        fail(UMAPB_ERR_INVALID, "invalid input detected on the device");
    }
}

}  // namespace umapb

using namespace umapb;

namespace {

// Epochs of a transform when the caller passes none: a third of the layout's
// epoch count when the options set one, else 100 for up to 10,000 new points
// and 30 above (umap-learn's rule for its transform).
int transform_epochs(const umapb_options& o, int requested, int32_t nq) {
    if (requested > 0) return requested;
    if (o.has_num_epochs && o.num_epochs > 0) return std::max(1, o.num_epochs / 3);
    return nq <= 10000 ? 100 : 30;
}

template <typename T>
void transform_impl(size_t data_dim, int32_t nref, const void* ref_data, const void* ref_embedding, int32_t nq,
                    const void* new_data, size_t num_dim, const umapb_options& o, int num_epochs, void* new_embedding,
                    cudaStream_t s) {
    require(data_dim >= 1 && data_dim <= static_cast<size_t>(INT32_MAX), "data_dim must be positive");
    require(num_dim >= 1 && num_dim <= 64, "num_dim must be between 1 and 64");
    require(nref >= 1, "the transform needs at least one reference point");
    require(nq >= 0, "num_new must not be negative");
    const int k = o.num_neighbors;
    require(k >= 1 && k <= nref, "num_neighbors must be in [1, num_ref]");
    require(o.learning_rate > 0 && std::isfinite(o.learning_rate), "learning_rate must be positive");
    require(o.negative_sample_rate >= 0 && std::isfinite(o.negative_sample_rate),
            "negative_sample_rate must not be negative");
    if (nq == 0) return;
    const size_t D = data_dim, nr = static_cast<size_t>(nref), nn = static_cast<size_t>(nq);
    DeviceIn<T> rd(static_cast<const T*>(ref_data), nr * D, s);
    DeviceIn<T> nd(static_cast<const T*>(new_data), nn * D, s);
    DeviceIn<T> ry(static_cast<const T*>(ref_embedding), nr * num_dim, s);
    DeviceInOut<T> ny(static_cast<T*>(new_embedding), nn * num_dim, s, false);
    // the reference rows, then the new rows, in one array
    DevArray<T> data((nr + nn) * D, s);
    UMAPB_CUDA(cudaMemcpyAsync(data.get(), rd.get(), nr * D * sizeof(T), cudaMemcpyDeviceToDevice, s));
    UMAPB_CUDA(cudaMemcpyAsync(data.get() + nr * D, nd.get(), nn * D * sizeof(T), cudaMemcpyDeviceToDevice, s));
    DevArray<int32_t> idx(nn * k, s);
    DevArray<T> w(nn * k, s);
    knn_query<T>(data.get(), nref, nq, static_cast<int32_t>(D), k, idx.get(), w.get(), s);
    data.release();
    DevArray<int64_t> ptr(nn + 1, s);
    dense_row_ptr_kernel<<<grid_for(nn + 1, 256), 256, 0, s>>>(nq, k, ptr.get());
    UMAPB_LAUNCH_CHECK();
    // the new points' similarities to their neighbours (neighbor_similarities.hpp), in place
    neighbor_similarities<T>(nq, ptr.get(), w.get(), o.local_connectivity, o.bandwidth, 1e-3, true, nullptr, nullptr, s);
    transform_init<T>(nq, static_cast<int>(num_dim), ptr.get(), idx.get(), w.get(), ry.get(), ny.get(), s);
    double a = o.a, b = o.b;
    if (!o.has_a || !o.has_b) find_ab(o.spread, o.min_dist, &a, &b);
    DeviceEpochs<T> ep;
    similarities_to_epochs<T>(nq, ptr.get(), idx.get(), w.get(), static_cast<int64_t>(nn * k),
                              transform_epochs(o, num_epochs, nq), o.negative_sample_rate, ep, s);
    // a quarter of the layout's learning rate, as umap-learn's transform uses
    transform_layout<T>(ep, static_cast<int>(num_dim), ry.get(), nref, ny.get(), nref, a, b, o.repulsion_strength,
                        o.learning_rate / 4.0, o.optimize_seed, s);
    ny.finish();
    UMAPB_SYNC(s);
}

}  // namespace

extern "C" {

void umapb_options_init(umapb_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->local_connectivity = 1;
    o->bandwidth = 1;
    o->mix_ratio = 1;
    o->spread = 1;
    o->min_dist = 0.1;
    o->repulsion_strength = 1;
    o->initialize_method = UMAPB_INIT_SPECTRAL;
    o->initialize_random_on_spectral_fail = 1;
    o->irlba_extra_work = 7;
    o->irlba_max_iterations = 1000;
    o->irlba_convergence_tolerance = 1e-6;
    o->initialize_spectral_scale = 10;
    o->initialize_spectral_jitter = 0;
    o->initialize_spectral_jitter_sd = 1e-4;
    o->initialize_random_scale = 10;
    o->initialize_seed = 9876543210ULL;
    o->learning_rate = 1;
    o->negative_sample_rate = 5;
    o->num_neighbors = 15;
    o->optimize_seed = 1234567890ULL;
    o->num_threads = 1;
    o->num_threads_spectral = 1;
    o->num_threads_optimize = 1;
}

const char* umapb_last_error(void) { return g_last_error.c_str(); }

int umapb_version(void) { return UMAPB_VERSION; }

size_t umapb_options_size(void) { return sizeof(umapb_options); }

int64_t umapb_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

size_t umapb_set_workspace_limit(size_t bytes) { return umapb::ws_set_limit(bytes); }

int64_t umapb_set_device_wait_limit(int64_t polls) {
    return g_wait_limit.exchange(polls > 0 ? polls : (1ll << 26), std::memory_order_relaxed);
}

int umapb_initialize_neighbors(int dtype, int32_t num_obs, const int64_t* row_ptr, const int32_t* indices,
                               const void* distances, size_t num_dim, void* embedding, const umapb_options* opt,
                               umapb_status** out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        *out = nullptr;
        auto st = new_status(dtype, num_obs, num_dim, opt);
        if (dtype == UMAPB_F64) {
            init_from_neighbors<double>(st.get(), row_ptr, indices, distances, embedding);
        } else {
            init_from_neighbors<float>(st.get(), row_ptr, indices, distances, embedding);
        }
        *out = st.release();
    });
}

int umapb_initialize_knn_matrix(int dtype, int32_t num_obs, int32_t k, const int32_t* indices, const void* distances,
                                int index_base, size_t num_dim, void* embedding, const umapb_options* opt,
                                umapb_status** out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        *out = nullptr;
        auto st = new_status(dtype, num_obs, num_dim, opt);
        if (dtype == UMAPB_F64) {
            init_from_knn_matrix<double>(st.get(), k, indices, distances, index_base, embedding);
        } else {
            init_from_knn_matrix<float>(st.get(), k, indices, distances, index_base, embedding);
        }
        *out = st.release();
    });
}

int umapb_prebuilt_create(int dtype, size_t data_dim, int32_t num_obs, const void* data, umapb_prebuilt** out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        *out = nullptr;
        require_device();
        require(dtype == UMAPB_F32 || dtype == UMAPB_F64, "dtype must be UMAPB_F32 or UMAPB_F64");
        require(num_obs >= 2, "the neighbour search needs at least two observations");
        require(data_dim >= 1 && data_dim <= INT32_MAX, "data_dim must be positive");
        require(data != nullptr, "data must not be NULL");
        auto pb = std::make_unique<umapb_prebuilt>();
        pb->dtype = dtype;
        pb->dim = data_dim;
        pb->n = num_obs;
        UMAPB_CUDA(cudaGetDevice(&pb->device));
        pb->bytes = static_cast<size_t>(num_obs) * data_dim * (dtype == UMAPB_F64 ? 8 : 4);
        UMAPB_CUDA(cudaMalloc(&pb->data, pb->bytes));
        UMAPB_CUDA(cudaMemcpy(pb->data, data, pb->bytes, cudaMemcpyDefault));
        *out = pb.release();
    });
}

void umapb_prebuilt_free(umapb_prebuilt* pb) { delete pb; }

int umapb_initialize_prebuilt(const umapb_prebuilt* pb, size_t num_dim, void* embedding, const umapb_options* opt,
                              umapb_status** out) {
    return guarded([&] {
        require(pb != nullptr && pb->data != nullptr, "invalid prebuilt index");
        int dev = -1;
        UMAPB_CUDA(cudaGetDevice(&dev));
        require(dev == pb->device, "the prebuilt index belongs to another device");
        require(out != nullptr, "out must not be NULL");
        *out = nullptr;
        auto st = new_status(pb->dtype, pb->n, num_dim, opt);
        if (pb->dtype == UMAPB_F64) {
            init_from_data<double>(st.get(), pb->dim, pb->data, embedding);
        } else {
            init_from_data<float>(st.get(), pb->dim, pb->data, embedding);
        }
        *out = st.release();
    });
}

int umapb_initialize_data(int dtype, size_t data_dim, int32_t num_obs, const void* data, size_t num_dim,
                          void* embedding, const umapb_options* opt, umapb_status** out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        *out = nullptr;
        auto st = new_status(dtype, num_obs, num_dim, opt);
        require(num_obs >= 2, "the neighbour search needs at least two observations");
        if (dtype == UMAPB_F64) {
            init_from_data<double>(st.get(), data_dim, data, embedding);
        } else {
            init_from_data<float>(st.get(), data_dim, data, embedding);
        }
        *out = st.release();
    });
}

int umapb_status_run(umapb_status* st, void* embedding, int epoch_limit) {
    return guarded([&] {
        require(st != nullptr && st->impl, "invalid status");
        UMAPB_CUDA(cudaSetDevice(st->device));
        NvtxRange range("umapb run");
        st->impl->run(embedding, epoch_limit < 0 ? st->num_epochs : epoch_limit);
    });
}

int umapb_status_epoch(const umapb_status* st) { return st ? st->current_epoch : -1; }
int umapb_status_num_epochs(const umapb_status* st) { return st ? st->num_epochs : -1; }
int32_t umapb_status_num_observations(const umapb_status* st) { return st ? st->n : -1; }
size_t umapb_status_num_dimensions(const umapb_status* st) { return st ? st->num_dim : 0; }
double umapb_status_a(const umapb_status* st) { return st ? st->a : 0; }
double umapb_status_b(const umapb_status* st) { return st ? st->b : 0; }
int64_t umapb_status_num_edges(const umapb_status* st) { return (st && st->impl) ? st->impl->num_edges() : -1; }

int umapb_status_get_epoch_data(const umapb_status* st, int64_t* row_ptr, int32_t* targets, void* eps, void* enext,
                                void* enneg) {
    return guarded([&] {
        require(st != nullptr && st->impl, "invalid status");
        UMAPB_CUDA(cudaSetDevice(st->device));
        st->impl->epoch_data(row_ptr, targets, eps, enext, enneg);
    });
}

int umapb_status_schedule_counts(const umapb_status* st, int first, int last, int64_t* counts) {
    return guarded([&] {
        require(st != nullptr && st->impl, "invalid status");
        require(first >= 0 && last >= first, "bad epoch range");
        UMAPB_CUDA(cudaSetDevice(st->device));
        st->impl->counts(first, last, counts);
    });
}

int umapb_status_stage_ms(const umapb_status* st, double* ms, int count) {
    return guarded([&] {
        require(st != nullptr && ms != nullptr, "invalid arguments");
        for (int i = 0; i < count && i < 7; ++i) ms[i] = st->stage_ms[i];
    });
}

void umapb_status_free(umapb_status* st) { delete st; }

int umapb_knn(int dtype, size_t data_dim, int32_t num_obs, const void* data, int k, int32_t* out_indices,
              void* out_distances) {
    return guarded([&] {
        require_device();
        Context& c = thread_context();
        const size_t total = static_cast<size_t>(num_obs) * data_dim;
        const size_t nk = static_cast<size_t>(num_obs) * (k > 0 ? k : 0);
        DeviceInOut<int32_t> oi(out_indices, nk, c.stream, false);
        if (dtype == UMAPB_F64) {
            DeviceIn<double> d(static_cast<const double*>(data), total, c.stream);
            DeviceInOut<double> od(static_cast<double*>(out_distances), nk, c.stream, false);
            knn_exact<double>(d.get(), num_obs, static_cast<int32_t>(data_dim), k, oi.get(), od.get(), c.stream);
            od.finish();
        } else {
            DeviceIn<float> d(static_cast<const float*>(data), total, c.stream);
            DeviceInOut<float> od(static_cast<float*>(out_distances), nk, c.stream, false);
            knn_exact<float>(d.get(), num_obs, static_cast<int32_t>(data_dim), k, oi.get(), od.get(), c.stream);
            od.finish();
        }
        oi.finish();
        UMAPB_SYNC(c.stream);
    });
}

int umapb_knn_shard(int dtype, size_t data_dim, int32_t num_obs, const void* data, int k, int32_t shard,
                    int32_t num_shards, int32_t* out_rows, int32_t* out_indices, void* out_distances,
                    int32_t* out_count) {
    return guarded([&] {
        require_device();
        require(out_count != nullptr, "out_count must not be NULL");
        require(num_shards >= 1 && shard >= 0 && shard < num_shards, "shard must be in [0, num_shards)");
        Context& c = thread_context();
        cudaStream_t s = c.stream;
        const size_t total = static_cast<size_t>(num_obs) * data_dim;
        const size_t nk = static_cast<size_t>(num_obs) * (k > 0 ? k : 0);
        auto body = [&](auto tag) {
            using T = decltype(tag);
            DeviceIn<T> d(static_cast<const T*>(data), total, s);
            DevArray<int32_t> idx(nk, s), rows;
            DevArray<T> dist(nk, s);
            int32_t nrows = 0;
            knn_exact_shard<T>(d.get(), num_obs, static_cast<int32_t>(data_dim), k, KnnShard{shard, num_shards},
                               idx.get(), dist.get(), rows, nrows, s);
            // the shard's rows, compacted in row order
            DevArray<int32_t> cidx(static_cast<size_t>(nrows) * k, s);
            DevArray<T> cdist(static_cast<size_t>(nrows) * k, s);
            if (nrows > 0) {
                gather_rows_kernel<int32_t><<<grid_for(static_cast<size_t>(nrows) * k, 256), 256, 0, s>>>(
                    nrows, k, rows.get(), idx.get(), cidx.get());
                gather_rows_kernel<T><<<grid_for(static_cast<size_t>(nrows) * k, 256), 256, 0, s>>>(
                    nrows, k, rows.get(), dist.get(), cdist.get());
                UMAPB_LAUNCH_CHECK();
                require(out_rows && out_indices && out_distances, "output arrays must not be NULL");
                UMAPB_CUDA(cudaMemcpyAsync(out_rows, rows.get(), sizeof(int32_t) * nrows, cudaMemcpyDefault, s));
                UMAPB_CUDA(cudaMemcpyAsync(out_indices, cidx.get(), sizeof(int32_t) * nrows * k, cudaMemcpyDefault, s));
                UMAPB_CUDA(cudaMemcpyAsync(out_distances, cdist.get(), sizeof(T) * nrows * k, cudaMemcpyDefault, s));
            }
            UMAPB_SYNC(s);
            *out_count = nrows;
        };
        if (dtype == UMAPB_F64) body(double{}); else body(float{});
    });
}

int umapb_transform(int dtype, size_t data_dim, int32_t num_ref, const void* ref_data, const void* ref_embedding,
                    int32_t num_new, const void* new_data, size_t num_dim, const umapb_options* opt, int num_epochs,
                    void* new_embedding) {
    return guarded([&] {
        require_device();
        require(opt != nullptr, "options must not be NULL");
        Context& c = thread_context();
        if (dtype == UMAPB_F64)
            transform_impl<double>(data_dim, num_ref, ref_data, ref_embedding, num_new, new_data, num_dim, *opt,
                                   num_epochs, new_embedding, c.stream);
        else
            transform_impl<float>(data_dim, num_ref, ref_data, ref_embedding, num_new, new_data, num_dim, *opt,
                                  num_epochs, new_embedding, c.stream);
    });
}

int umapb_transform_epochs(const umapb_options* opt, int num_epochs, int32_t num_new) {
    if (!opt) return -1;
    return transform_epochs(*opt, num_epochs, num_new);
}

int umapb_knn_query(int dtype, size_t data_dim, int32_t num_ref, const void* ref_data, int32_t num_query,
                    const void* query_data, int k, int32_t* out_indices, void* out_distances) {
    return guarded([&] {
        require_device();
        require(data_dim >= 1 && data_dim <= static_cast<size_t>(INT32_MAX), "data_dim must be positive");
        require(num_ref >= 1 && num_query >= 0, "bad point counts");
        Context& c = thread_context();
        cudaStream_t s = c.stream;
        const size_t D = data_dim, nr = static_cast<size_t>(num_ref), nq = static_cast<size_t>(num_query);
        const size_t nk = nq * static_cast<size_t>(k > 0 ? k : 0);
        auto body = [&](auto tag) {
            using T = decltype(tag);
            DeviceIn<T> rd(static_cast<const T*>(ref_data), nr * D, s);
            DeviceIn<T> qd(static_cast<const T*>(query_data), nq * D, s);
            DevArray<T> data((nr + nq) * D, s);
            UMAPB_CUDA(cudaMemcpyAsync(data.get(), rd.get(), nr * D * sizeof(T), cudaMemcpyDeviceToDevice, s));
            if (nq) UMAPB_CUDA(cudaMemcpyAsync(data.get() + nr * D, qd.get(), nq * D * sizeof(T), cudaMemcpyDeviceToDevice, s));
            DeviceInOut<int32_t> oi(out_indices, nk, s, false);
            DeviceInOut<T> od(static_cast<T*>(out_distances), nk, s, false);
            knn_query<T>(data.get(), num_ref, num_query, static_cast<int32_t>(D), k, oi.get(), od.get(), s);
            oi.finish();
            od.finish();
            UMAPB_SYNC(s);
        };
        if (dtype == UMAPB_F64) body(double{}); else body(float{});
    });
}

int umapb_knn_last_fp64_recomputed(void) { return last_knn_redo_count(); }

double umapb_knn_last_tc_error(void) { return last_knn_tc_error(); }

int64_t umapb_knn_last_tile_pairs(void) { return last_knn_tiles_scanned(); }

double umapb_knn_last_kernel_ms(void) { return last_knn_kernel_ms(); }

int umapb_measure_random_access(int64_t num_points, int64_t accesses, int mode, int reps, double* per_second) {
    return guarded([&] {
        require_device();
        require(per_second != nullptr, "per_second must not be NULL");
        Context& c = thread_context();
        *per_second = measure_random_access(num_points, accesses, mode, reps, c.stream);
    });
}

int umapb_neighbor_similarities(int dtype, int32_t num_obs, const int64_t* row_ptr, void* distances,
                                double local_connectivity, double bandwidth, double min_k_dist_scale, int use_newton,
                                double* rho_out, double* sigma_out) {
    return guarded([&] {
        require_device();
        Context& c = thread_context();
        const int64_t nnz = host_nnz(row_ptr, num_obs, c.stream);
        DeviceIn<int64_t> p(row_ptr, static_cast<size_t>(num_obs) + 1, c.stream);
        DeviceInOut<double> rho(rho_out, rho_out ? num_obs : 0, c.stream, false);
        DeviceInOut<double> sig(sigma_out, sigma_out ? num_obs : 0, c.stream, false);
        if (dtype == UMAPB_F64) {
            DeviceInOut<double> v(static_cast<double*>(distances), nnz, c.stream, true);
            neighbor_similarities<double>(num_obs, p.get(), v.get(), local_connectivity, bandwidth, min_k_dist_scale,
                                          use_newton != 0, rho.get(), sig.get(), c.stream);
            v.finish();
        } else {
            DeviceInOut<float> v(static_cast<float*>(distances), nnz, c.stream, true);
            neighbor_similarities<float>(num_obs, p.get(), v.get(), local_connectivity, bandwidth, min_k_dist_scale,
                                         use_newton != 0, rho.get(), sig.get(), c.stream);
            v.finish();
        }
        rho.finish();
        sig.finish();
        UMAPB_SYNC(c.stream);
    });
}

int umapb_combine_neighbor_sets(int dtype, int32_t num_obs, const int64_t* row_ptr, const int32_t* indices,
                                const void* weights, double mix_ratio, int64_t* out_row_ptr, int32_t* out_indices,
                                void* out_weights, int64_t capacity, int64_t* out_nnz) {
    return guarded([&] {
        require_device();
        Context& c = thread_context();
        const int64_t nnz = host_nnz(row_ptr, num_obs, c.stream);
        DeviceIn<int64_t> p(row_ptr, static_cast<size_t>(num_obs) + 1, c.stream);
        DeviceIn<int32_t> ix(indices, nnz, c.stream);
        auto body = [&](auto tag) {
            using T = decltype(tag);
            DeviceIn<T> w(static_cast<const T*>(weights), nnz, c.stream);
            DeviceCsr<T> g;
            combine_neighbor_sets<T>(num_obs, p.get(), ix.get(), w.get(), nnz, mix_ratio, g, c.stream);
            require(g.nnz <= capacity, "output capacity is too small for the combined graph");
            copy_out(out_row_ptr, g.ptr.get(), sizeof(int64_t) * (static_cast<size_t>(num_obs) + 1), c.stream);
            copy_out(out_indices, g.idx.get(), sizeof(int32_t) * g.nnz, c.stream);
            copy_out(out_weights, g.val.get(), sizeof(T) * g.nnz, c.stream);
            UMAPB_SYNC(c.stream);
            if (out_nnz) *out_nnz = g.nnz;
        };
        if (dtype == UMAPB_F64) body(double{}); else body(float{});
    });
}

int umapb_similarities_to_epochs(int dtype, int32_t num_obs, const int64_t* row_ptr, const int32_t* indices,
                                 const void* weights, int num_epochs, double negative_sample_rate,
                                 int64_t* out_row_ptr, int32_t* out_targets, void* eps, void* enext, void* enneg,
                                 int64_t* out_nnz) {
    return guarded([&] {
        require_device();
        Context& c = thread_context();
        const int64_t nnz = host_nnz(row_ptr, num_obs, c.stream);
        DeviceIn<int64_t> p(row_ptr, static_cast<size_t>(num_obs) + 1, c.stream);
        DeviceIn<int32_t> ix(indices, nnz, c.stream);
        auto body = [&](auto tag) {
            using T = decltype(tag);
            DeviceIn<T> w(static_cast<const T*>(weights), nnz, c.stream);
            DeviceEpochs<T> ep;
            similarities_to_epochs<T>(num_obs, p.get(), ix.get(), w.get(), nnz, num_epochs, negative_sample_rate, ep,
                                      c.stream);
            copy_out(out_row_ptr, ep.ptr.get(), sizeof(int64_t) * (static_cast<size_t>(num_obs) + 1), c.stream);
            copy_out(out_targets, ep.targets.get(), sizeof(int32_t) * ep.nnz, c.stream);
            copy_out(eps, ep.eps.get(), sizeof(T) * ep.nnz, c.stream);
            copy_out(enext, ep.enext0.get(), sizeof(T) * ep.nnz, c.stream);
            copy_out(enneg, ep.enneg0.get(), sizeof(T) * ep.nnz, c.stream);
            UMAPB_SYNC(c.stream);
            if (out_nnz) *out_nnz = ep.nnz;
        };
        if (dtype == UMAPB_F64) body(double{}); else body(float{});
    });
}

int umapb_has_multiple_components(int32_t num_obs, const int64_t* row_ptr, const int32_t* indices, int* out) {
    return guarded([&] {
        require_device();
        require(out != nullptr, "out must not be NULL");
        Context& c = thread_context();
        const int64_t nnz = host_nnz(row_ptr, num_obs, c.stream);
        DeviceIn<int64_t> p(row_ptr, static_cast<size_t>(num_obs) + 1, c.stream);
        DeviceIn<int32_t> ix(indices, nnz, c.stream);
        // include/umappp/spectral_init.hpp:144-146: an empty graph is not "multiple"
        *out = (num_obs > 0 && count_components(num_obs, p.get(), ix.get(), c.d_status, c.stream) > 1) ? 1 : 0;
    });
}

int umapb_spectral_init(int dtype, int32_t num_obs, const int64_t* row_ptr, const int32_t* indices,
                        const void* weights, size_t num_dim, void* embedding, int extra_work, int max_iterations,
                        double tolerance, double scale, int jitter, double jitter_sd, uint64_t seed, int* ok,
                        double* evals_out) {
    return guarded([&] {
        require_device();
        Context& c = thread_context();
        const int64_t nnz = host_nnz(row_ptr, num_obs, c.stream);
        DeviceIn<int64_t> p(row_ptr, static_cast<size_t>(num_obs) + 1, c.stream);
        DeviceIn<int32_t> ix(indices, nnz, c.stream);
        auto body = [&](auto tag) {
            using T = decltype(tag);
            DeviceIn<T> w(static_cast<const T*>(weights), nnz, c.stream);
            DeviceInOut<T> Y(static_cast<T*>(embedding), static_cast<size_t>(num_obs) * num_dim, c.stream, true);
            const SpectralResult r = spectral_init<T>(num_obs, p.get(), ix.get(), w.get(), static_cast<int>(num_dim),
                                                      Y.get(), extra_work, max_iterations, tolerance, scale,
                                                      jitter != 0, jitter_sd, seed, c.d_status, c.stream);
            if (r.ok) Y.finish();
            UMAPB_SYNC(c.stream);
            if (ok) *ok = r.ok ? 1 : 0;
            if (evals_out) for (size_t d = 0; d <= num_dim && d < 64; ++d) evals_out[d] = r.evals[d];
        };
        if (dtype == UMAPB_F64) body(double{}); else body(float{});
    });
}

int umapb_random_init(int dtype, int32_t num_obs, size_t num_dim, void* embedding, uint64_t seed, double scale) {
    return guarded([&] {
        require_device();
        Context& c = thread_context();
        auto body = [&](auto tag) {
            using T = decltype(tag);
            DeviceInOut<T> Y(static_cast<T*>(embedding), static_cast<size_t>(num_obs) * num_dim, c.stream, false);
            random_init<T>(num_obs, static_cast<int>(num_dim), Y.get(), seed, scale, c.stream);
            Y.finish();
            UMAPB_SYNC(c.stream);
        };
        if (dtype == UMAPB_F64) body(double{}); else body(float{});
    });
}

int umapb_find_ab(double spread, double min_dist, double* a, double* b) {
    return guarded([&] {
        require(a != nullptr && b != nullptr, "outputs must not be NULL");
        find_ab(spread, min_dist, a, b);
    });
}

int umapb_choose_num_epochs(int has_value, int value, int64_t num_obs) {
    return choose_num_epochs(has_value != 0, value, num_obs);
}

int umapb_optimize_layout(int dtype, size_t num_dim, void* embedding, int32_t num_obs, const int64_t* row_ptr,
                          const int32_t* targets, const void* epochs_per_sample, void* epoch_of_next_sample,
                          void* epoch_of_next_negative_sample, double negative_sample_rate, int total_epochs,
                          int* current_epoch, double a, double b, double gamma, double learning_rate, uint64_t seed,
                          int epoch_limit) {
    return guarded([&] {
        require_device();
        require(current_epoch != nullptr, "current_epoch must not be NULL");
        Context& c = thread_context();
        const int64_t nnz = host_nnz(row_ptr, num_obs, c.stream);
        auto body = [&](auto tag) {
            using T = decltype(tag);
            DeviceEpochs<T> ep;
            ep.n = num_obs;
            ep.nnz = nnz;
            ep.total_epochs = total_epochs;
            ep.negative_sample_rate = static_cast<T>(negative_sample_rate);
            ep.ptr.allocate(static_cast<size_t>(num_obs) + 1, c.stream);
            ep.heads.allocate(nnz, c.stream);
            ep.targets.allocate(nnz, c.stream);
            ep.eps.allocate(nnz, c.stream);
            ep.enext0.allocate(nnz, c.stream);
            ep.enneg0.allocate(nnz, c.stream);
            UMAPB_CUDA(cudaMemcpyAsync(ep.ptr.get(), row_ptr, sizeof(int64_t) * (num_obs + 1), cudaMemcpyDefault, c.stream));
            if (nnz) {
                UMAPB_CUDA(cudaMemcpyAsync(ep.targets.get(), targets, sizeof(int32_t) * nnz, cudaMemcpyDefault, c.stream));
                UMAPB_CUDA(cudaMemcpyAsync(ep.eps.get(), epochs_per_sample, sizeof(T) * nnz, cudaMemcpyDefault, c.stream));
                UMAPB_CUDA(cudaMemcpyAsync(ep.enext0.get(), epoch_of_next_sample, sizeof(T) * nnz, cudaMemcpyDefault, c.stream));
                UMAPB_CUDA(cudaMemcpyAsync(ep.enneg0.get(), epoch_of_next_negative_sample, sizeof(T) * nnz, cudaMemcpyDefault, c.stream));
            }
            // heads from the row pointers
            std::vector<int64_t> hp(static_cast<size_t>(num_obs) + 1);
            UMAPB_CUDA(cudaMemcpyAsync(hp.data(), ep.ptr.get(), sizeof(int64_t) * (num_obs + 1), cudaMemcpyDeviceToHost, c.stream));
            UMAPB_SYNC(c.stream);
            std::vector<int32_t> heads(nnz);
            for (int32_t i = 0; i < num_obs; ++i)
                for (int64_t q = hp[i]; q < hp[i + 1]; ++q) heads[q] = i;
            if (nnz) UMAPB_CUDA(cudaMemcpyAsync(ep.heads.get(), heads.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, c.stream));
            // the given state describes the schedule at *current_epoch
            SgdEngine<T> eng;
            const int first = *current_epoch;
            eng.setup(&ep, c.stream, first);
            DeviceInOut<T> Y(static_cast<T*>(embedding), static_cast<size_t>(num_obs) * num_dim, c.stream, true);
            eng.run(Y.get(), static_cast<int>(num_dim), first, epoch_limit, a, b, gamma, learning_rate, seed, c.stream,
                    nullptr, nullptr);
            Y.finish();
            if (epoch_limit > first) {
                DevArray<T> en(nnz, c.stream), enn(nnz, c.stream);
                eng.state_at(epoch_limit, en.get(), enn.get(), c.stream);
                copy_out(epoch_of_next_sample, en.get(), sizeof(T) * nnz, c.stream);
                copy_out(epoch_of_next_negative_sample, enn.get(), sizeof(T) * nnz, c.stream);
                *current_epoch = epoch_limit;
            }
            UMAPB_SYNC(c.stream);
        };
        if (dtype == UMAPB_F64) body(double{}); else body(float{});
    });
}

int umapb_batch_run(int dtype, int32_t num_instances, const int32_t* sizes, size_t data_dim, const void* data,
                    size_t num_dim, void* embedding, const umapb_options* opt, double* stage_ms) {
    return guarded([&] {
        require_device();
        require(dtype == UMAPB_F32 || dtype == UMAPB_F64, "dtype must be UMAPB_F32 or UMAPB_F64");
        require(opt != nullptr && sizes != nullptr, "options and sizes must not be NULL");
        require(num_instances >= 1, "at least one instance is needed");
        require(num_dim >= 1 && num_dim <= 64, "num_dim must be between 1 and 64");
        std::vector<int32_t> inst(static_cast<size_t>(num_instances) + 1, 0);
        for (int i = 0; i < num_instances; ++i) {
            require(sizes[i] >= 2, "every instance needs at least two observations");
            require(static_cast<int64_t>(inst[i]) + sizes[i] <= INT32_MAX, "too many observations", UMAPB_ERR_OVERFLOW);
            inst[i + 1] = inst[i] + sizes[i];
        }
        float ms[7] = {0, 0, 0, 0, 0, 0, 0};
        if (dtype == UMAPB_F64) {
            batch_pipeline<double>(inst, data_dim, data, num_dim, embedding, *opt, ms);
        } else {
            batch_pipeline<float>(inst, data_dim, data, num_dim, embedding, *opt, ms);
        }
        if (stage_ms) for (int i = 0; i < 7; ++i) stage_ms[i] = ms[i];
    });
}

int umapb_loss_grad(int dtype, size_t num_dim, const void* embedding, int32_t num_obs, const int64_t* row_ptr,
                    const int32_t* indices, const void* weights, double a, double b, double eps_rep, int with_constant,
                    double* loss, void* grad_embedding, double* grad_ab) {
    return guarded([&] {
        require_device();
        Context& c = thread_context();
        const int64_t nnz = host_nnz(row_ptr, num_obs, c.stream);
        DeviceIn<int64_t> p(row_ptr, static_cast<size_t>(num_obs) + 1, c.stream);
        DeviceIn<int32_t> ix(indices, nnz, c.stream);
        auto body = [&](auto tag) {
            using T = decltype(tag);
            const size_t total = static_cast<size_t>(num_obs) * num_dim;
            DeviceIn<T> Y(static_cast<const T*>(embedding), total, c.stream);
            DeviceIn<T> w(static_cast<const T*>(weights), nnz, c.stream);
            DeviceInOut<T> g(static_cast<T*>(grad_embedding), grad_embedding ? total : 0, c.stream, false);
            loss_grad<T>(num_obs, static_cast<int>(num_dim), Y.get(), p.get(), ix.get(), w.get(), a, b, eps_rep,
                         with_constant != 0, loss, grad_embedding ? g.get() : nullptr, grad_ab, c.stream);
            g.finish();
            UMAPB_SYNC(c.stream);
        };
        if (dtype == UMAPB_F64) body(double{}); else body(float{});
    });
}

}  // extern "C"
