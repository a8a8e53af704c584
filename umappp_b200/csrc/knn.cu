// Exact Euclidean k-nearest neighbours on the device (the role of the
// knncolle search called at include/umappp/initialize.hpp:140).
//
// Candidate search (CUDA cores): one thread per query; tiles of 32 reference
// points and 32 dimensions are staged in shared memory (queries transposed so
// each thread reads its own column without bank conflicts, points broadcast),
// squared distances are accumulated from coordinate differences, and each
// thread keeps a sorted register list of its KCAP best (distance, index)
// candidates (ties keep the smaller index, as points arrive in index order).
//
// Float data: the list holds k + 8 candidates in FP32; a second kernel rescores
// them in FP64 from the original coordinates and keeps the best k by
// (distance, index).  A query whose (k+8)-th FP32 candidate is not clear of
// its k-th FP64 distance by more than the FP32 error bound is recomputed by
// the FP64 kernel, so the result equals an FP64 brute force except for ties.
// Double data: the FP64 kernel directly, with multiply and add kept separate
// so the sums round exactly as a sequential FP64 loop.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "stages.cuh"

namespace umapb {

int& last_knn_redo_count() {
    static int count = 0;
    return count;
}

static float bits_to_float(unsigned int b) {
    float f;
    std::memcpy(&f, &b, sizeof(f));
    return f;
}

int64_t& last_knn_tiles_scanned() {
    static int64_t tiles = 0;
    return tiles;
}

float& last_knn_kernel_ms() {
    static float ms = 0.0f;
    return ms;
}

double& last_knn_tc_error() {
    static double worst = 0.0;
    return worst;
}

namespace {

constexpr int KNN_BLOCK = 128;  // queries per block

// The tensor-core candidate search is the default; UMAPB_KNN_TENSOR_CORES=0
// selects the CUDA-core search instead (used by the precision comparison).
bool use_tensor_cores() {
    const char* v = std::getenv("UMAPB_KNN_TENSOR_CORES");
    return !(v && v[0] == '0');
}
constexpr int PT = 32;          // points per tile
constexpr int CH = 32;          // dimensions per chunk

__device__ __forceinline__ void add_sq(float& acc, float d) { acc = fmaf(d, d, acc); }
__device__ __forceinline__ void add_sq(double& acc, double d) { acc = __dadd_rn(acc, __dmul_rn(d, d)); }

template <typename A>
struct Inf;
template <>
struct Inf<float> {
    static __device__ __forceinline__ float v() { return CUDART_INF_F; }
};
template <>
struct Inf<double> {
    static __device__ __forceinline__ double v() { return CUDART_INF; }
};

// Sorted insertion into a register list (bd ascending); entries equal to an
// existing distance go after it, so earlier (smaller) indices win ties.
template <typename A, int KCAP>
__device__ __forceinline__ void insert_sorted(A (&bd)[KCAP], int (&bi)[KCAP], A cd, int ci) {
#pragma unroll
    for (int i = KCAP - 1; i > 0; --i) {
        if (cd < bd[i - 1]) {
            bd[i] = bd[i - 1];
            bi[i] = bi[i - 1];
        } else if (cd < bd[i]) {
            bd[i] = cd;
            bi[i] = ci;
        }
    }
    if (cd < bd[0]) {
        bd[0] = cd;
        bi[0] = ci;
    }
}

// Brute-force candidate kernel.  T = storage type, A = accumulation type.
// If 'queries' is non-null the block's threads take their query ids from it
// (nq entries), else queries are 0..nq-1.  The candidates are the data rows
// [0, n) other than the query itself.
template <typename T, typename A, int KCAP>
__global__ void __launch_bounds__(KNN_BLOCK) knn_bruteforce_kernel(const T* __restrict__ data, int32_t n, int32_t dim,
                                                                   const int32_t* __restrict__ queries, int32_t nq,
                                                                   int32_t* __restrict__ cand_idx,
                                                                   A* __restrict__ cand_d2) {
    __shared__ A qs[CH][KNN_BLOCK];
    __shared__ A ps[PT][CH + 1];
    const int tid = threadIdx.x;
    const int32_t slot = blockIdx.x * KNN_BLOCK + tid;
    const bool active = slot < nq;
    const int32_t q = active ? (queries ? queries[slot] : slot) : 0;

    A bd[KCAP];
    int bi[KCAP];
#pragma unroll
    for (int i = 0; i < KCAP; ++i) {
        bd[i] = Inf<A>::v();
        bi[i] = -1;
    }

    for (int32_t base = 0; base < n; base += PT) {
        A acc[PT];
#pragma unroll
        for (int p = 0; p < PT; ++p) acc[p] = 0;
        for (int c0 = 0; c0 < dim; c0 += CH) {
            const int cw = min(CH, dim - c0);
            __syncthreads();
            // stage this block's queries (transposed) and the point tile
            for (int c = 0; c < cw; ++c) qs[c][tid] = active ? static_cast<A>(data[static_cast<size_t>(q) * dim + c0 + c]) : A(0);
            for (int e = tid; e < PT * CH; e += KNN_BLOCK) {
                const int p = e / CH, c = e % CH;
                const int32_t j = base + p;
                ps[p][c] = (j < n && c < cw) ? static_cast<A>(data[static_cast<size_t>(j) * dim + c0 + c]) : A(0);
            }
            __syncthreads();
            for (int c = 0; c < cw; ++c) {
                const A qv = qs[c][tid];
#pragma unroll
                for (int p = 0; p < PT; ++p) add_sq(acc[p], qv - ps[p][c]);
            }
        }
        if (active) {
#pragma unroll
            for (int p = 0; p < PT; ++p) {
                const int32_t j = base + p;
                if (j < n && j != q && acc[p] < bd[KCAP - 1]) insert_sorted<A, KCAP>(bd, bi, acc[p], j);
            }
        }
    }
    if (active) {
#pragma unroll
        for (int i = 0; i < KCAP; ++i) {
            cand_idx[static_cast<size_t>(slot) * KCAP + i] = bi[i];
            cand_d2[static_cast<size_t>(slot) * KCAP + i] = bd[i];
        }
    }
}

// FP64 rescoring of the FP32 candidates of every query: keeps the best k by
// (FP64 distance, index) and flags queries whose candidate set may miss a
// true neighbour.
template <int KCAP>
__global__ void knn_rescore_kernel(const float* __restrict__ data, int32_t others, int32_t dim, int32_t k,
                                   const int32_t* __restrict__ queries, int32_t nq, int cand_by_slot, int out_by_slot,
                                   const int32_t* __restrict__ cand_idx, const float* __restrict__ cand_d2,
                                   int32_t* __restrict__ out_idx, float* __restrict__ out_dist,
                                   double* __restrict__ out_dist64, int32_t* __restrict__ redo,
                                   int32_t* __restrict__ redo_count, const float* __restrict__ norms,
                                   const unsigned int* __restrict__ norm_max_bits, double tc_rel,
                                   unsigned int* __restrict__ tc_err_bits) {
    const int32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nq) return;
    const int32_t q = queries ? queries[slot] : slot;     // the query's data row (output row)
    const size_t crow = static_cast<size_t>(cand_by_slot ? slot : q);   // its candidate list
    double d64[KCAP];
    int id[KCAP];
    const int32_t* ci = cand_idx + crow * KCAP;
    const float* xq = data + static_cast<size_t>(q) * dim;
    int m = 0;
    float worst = 0.0f;   // largest |FP32 candidate distance - FP64 distance| / (|q|^2 + max |r|^2)
    const double err_scale = (norms && tc_err_bits)
                                 ? 1.0 / (static_cast<double>(norms[q]) + static_cast<double>(__uint_as_float(*norm_max_bits)) + 1e-300)
                                 : 0.0;
    for (int c = 0; c < KCAP; ++c) {
        const int32_t j = ci[c];
        double s = 0;
        if (j >= 0) {
            const float* xj = data + static_cast<size_t>(j) * dim;
            for (int d = 0; d < dim; ++d) {
                const double diff = static_cast<double>(xq[d]) - static_cast<double>(xj[d]);
                s = __dadd_rn(s, __dmul_rn(diff, diff));
            }
            if (err_scale > 0.0) {
                const double e = fabs(static_cast<double>(cand_d2[crow * KCAP + c]) - s) * err_scale;
                worst = fmaxf(worst, static_cast<float>(e));
            }
        } else {
            s = CUDART_INF;
        }
        // insertion by (distance, index); empty slots (j < 0) carry +inf and sort last
        const uint32_t jkey = static_cast<uint32_t>(j);   // -1 maps above every index
        int pos = m++;
        while (pos > 0 && (s < d64[pos - 1] || (s == d64[pos - 1] && jkey < static_cast<uint32_t>(id[pos - 1])))) {
            d64[pos] = d64[pos - 1];
            id[pos] = id[pos - 1];
            --pos;
        }
        d64[pos] = s;
        id[pos] = j;
    }
    // Certainty check: every point outside the candidate list has FP32 distance
    // >= the list's last FP32 value.  FP32 squared distances from differences
    // carry relative error below (dim + 2) * 2^-24 (plus the rounding of the
    // inputs, which is exact here); if the k-th FP64 distance could exceed the
    // true distance of such a point, the query is recomputed in FP64.
    // For tensor-core candidates (norms given) the FP32 values are
    // |q|^2 + |r|^2 - 2 q.r with an absolute error below tc_rel * (|q|^2 + max |r|^2).
    const float last32 = cand_d2[crow * KCAP + KCAP - 1];
    const double rel = (dim + 2) * 1.2e-7 * 2.0;
    const double kth = d64[k - 1];
    const bool full_list = others <= KCAP;   // every candidate point is in the list
    bool certain;
    if (norms) {
        const double bound = tc_rel * (static_cast<double>(norms[q]) + static_cast<double>(__uint_as_float(*norm_max_bits)));
        certain = static_cast<double>(last32) - bound > kth * (1.0 + 1e-12) + 1e-300;
    } else {
        certain = static_cast<double>(last32) * (1.0 - rel) > kth * (1.0 + rel);
    }
    if (!full_list && !certain) {
        const int32_t r = atomicAdd(redo_count, 1);
        redo[r] = out_by_slot ? slot : q;   // a slot when the output is by slot, else the data row
    }
    if (err_scale > 0.0 && worst > 0.0f) atomicMax(tc_err_bits, __float_as_uint(worst));
    const size_t orow = static_cast<size_t>(out_by_slot ? slot : q);
    for (int c = 0; c < k; ++c) {
        out_idx[orow * k + c] = id[c];
        const double dd = sqrt(d64[c]);
        out_dist[orow * k + c] = static_cast<float>(dd);
        if (out_dist64) out_dist64[orow * k + c] = dd;
    }
}

// Writes the first k entries of FP64 candidate lists (sqrt of squared distance).
// Output row of entry 'slot': out_rows[slot] if given, else the query's data row.
template <typename T, int KCAP>
__global__ void knn_emit_f64_kernel(int32_t nq, const int32_t* __restrict__ queries, const int32_t* __restrict__ out_rows,
                                    int32_t k, const int32_t* __restrict__ cand_idx, const double* __restrict__ cand_d2,
                                    int32_t* __restrict__ out_idx, T* __restrict__ out_dist,
                                    double* __restrict__ out_dist64) {
    const int32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nq) return;
    const int32_t q = out_rows ? out_rows[slot] : queries ? queries[slot] : slot;
    for (int c = 0; c < k; ++c) {
        out_idx[static_cast<size_t>(q) * k + c] = cand_idx[static_cast<size_t>(slot) * KCAP + c];
        const double dd = sqrt(cand_d2[static_cast<size_t>(slot) * KCAP + c]);
        out_dist[static_cast<size_t>(q) * k + c] = static_cast<T>(dd);
        if (out_dist64) out_dist64[static_cast<size_t>(q) * k + c] = dd;
    }
}

// FP64 search of the queries (data rows 'queries') among the data rows [0, n);
// results go to the queries' own rows, or to rows out_rows[slot] if given.
template <typename T, int KCAP>
void run_f64(const T* data, int32_t n, int32_t dim, int32_t k, const int32_t* queries, int32_t nq, int32_t* out_idx,
             T* out_dist, double* out_dist64, cudaStream_t s, const int32_t* out_rows = nullptr) {
    if (nq <= 0) return;
    DevArray<int32_t> ci(static_cast<size_t>(nq) * KCAP, s);
    DevArray<double> cd(static_cast<size_t>(nq) * KCAP, s);
    knn_bruteforce_kernel<T, double, KCAP><<<(nq + KNN_BLOCK - 1) / KNN_BLOCK, KNN_BLOCK, 0, s>>>(
        data, n, dim, queries, nq, ci.get(), cd.get());
    UMAPB_LAUNCH_CHECK();
    knn_emit_f64_kernel<T, KCAP><<<(nq + 127) / 128, 128, 0, s>>>(nq, queries, out_rows, k, ci.get(), cd.get(), out_idx,
                                                                  out_dist, out_dist64);
    UMAPB_LAUNCH_CHECK();
}

__global__ void norm_max_kernel(int32_t n, const float* __restrict__ norms, unsigned int* __restrict__ out) {
    unsigned int m = 0;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = max(m, __float_as_uint(norms[i]));    // non-negative floats order like their bits
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Tolerance of the tensor-core squared distances, relative to |q|^2 + |r|^2:
// 3xTF32 products (about 3 * 2^-22), FP32 accumulation over up to 64 terms and
// the final FP32 additions stay below 2^-17.
constexpr double TC_REL_BOUND = 1.0 / 131072.0;

__global__ void iota_kernel(int32_t count, int32_t first, int32_t* __restrict__ out) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) out[i] = first + i;
}

// The rows [lo, hi) of shard 'index' of 'count' equal contiguous ranges of the data rows.
void shard_row_range(int32_t n, KnnShard shard, int32_t& lo, int32_t& hi) {
    lo = static_cast<int32_t>(static_cast<int64_t>(n) * shard.index / shard.count);
    hi = static_cast<int32_t>(static_cast<int64_t>(n) * (shard.index + 1) / shard.count);
}

// With a shard (count > 1) the search covers only the shard's queries, whose
// data rows go to *rows (*nrows of them); out_idx / out_dist are written at
// those rows only.
template <int KCAP>
void run_f32(const float* data, int32_t n, int32_t dim, int32_t k, int32_t* out_idx, float* out_dist,
             double* out_dist64, cudaStream_t s, KnnShard shard = KnnShard(), DevArray<int32_t>* rows = nullptr,
             int32_t* nrows = nullptr) {
    const bool sharded = shard.count > 1;
    DevArray<float> norms;
    DevArray<unsigned int> norm_max(1, s);
    bool tc = use_tensor_cores() && knn_tc_supported(dim, KCAP);
    // candidates: by data row (tensor-core search, unsharded brute force) or by
    // slot of the shard's row list (sharded brute force)
    DevArray<int32_t> ci;
    DevArray<float> cd;
    DevArray<int32_t> tree_rows;
    int32_t nq = n;
    const int32_t* queries = nullptr;
    bool by_slot = false;
    if (tc) {
        ci.allocate(static_cast<size_t>(n) * KCAP, s);
        cd.allocate(static_cast<size_t>(n) * KCAP, s);
        const int32_t n_pad = ((n + 127) / 128) * 128;
        norms.allocate(n_pad, s);
        DevArray<int> err(1, s);
        err.zero(s);
        // unsharded: the rows in tree order, so that the rescoring walks the
        // queries with nearby ones together (their candidates share L2 lines)
        tc = knn_tc_candidates(data, n, dim, KCAP, ci.get(), cd.get(), norms.get(), err.get(), s, shard, rows, nrows,
                               sharded ? nullptr : &tree_rows);
        int h_err = 0;
        UMAPB_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);
        if (h_err != DEV_OK) fail(UMAPB_ERR_DEVICE_TIMEOUT, "tensor-core kNN: a pipeline wait gave up");
        if (tc) {
            norm_max.zero(s);
            norm_max_kernel<<<grid_for(n, 256, 1024), 256, 0, s>>>(n, norms.get(), norm_max.get());
            UMAPB_LAUNCH_CHECK();
            if (sharded) {
                nq = *nrows;
                queries = rows->get();
            } else if (tree_rows.get()) {
                queries = tree_rows.get();   // nq = n; candidates and output by data row
            }
        }
    }
    if (!tc) {
        if (sharded) {   // contiguous data rows, CUDA-core candidates by slot
            int32_t lo, hi;
            shard_row_range(n, shard, lo, hi);
            *nrows = hi - lo;
            rows->allocate(std::max<int32_t>(hi - lo, 1), s);
            if (hi > lo) {
                iota_kernel<<<grid_for(hi - lo, 256), 256, 0, s>>>(hi - lo, lo, rows->get());
                UMAPB_LAUNCH_CHECK();
            }
            nq = hi - lo;
            queries = rows->get();
            by_slot = true;
        }
        ci.allocate(static_cast<size_t>(std::max(nq, 1)) * KCAP, s);
        cd.allocate(static_cast<size_t>(std::max(nq, 1)) * KCAP, s);
        if (nq > 0) {
            knn_bruteforce_kernel<float, float, KCAP><<<(nq + KNN_BLOCK - 1) / KNN_BLOCK, KNN_BLOCK, 0, s>>>(
                data, n, dim, queries, nq, ci.get(), cd.get());
            UMAPB_LAUNCH_CHECK();
        }
    }
    DevArray<int32_t> redo(std::max(nq, 1), s), redo_count(1, s);
    redo_count.zero(s);
    DevArray<unsigned int> tc_err(1, s);
    tc_err.zero(s);
    if (nq > 0) {
        knn_rescore_kernel<KCAP><<<(nq + 127) / 128, 128, 0, s>>>(data, n - 1, dim, k, queries, nq, by_slot ? 1 : 0, 0, ci.get(),
                                                                  cd.get(), out_idx, out_dist, out_dist64, redo.get(),
                                                                  redo_count.get(), tc ? norms.get() : nullptr,
                                                                  norm_max.get(), TC_REL_BOUND, tc_err.get());
    }
    UMAPB_LAUNCH_CHECK();
    int32_t nredo = 0;
    unsigned int err_bits = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&nredo, redo_count.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(&err_bits, tc_err.get(), sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    last_knn_redo_count() = nredo;
    last_knn_tc_error() = tc ? static_cast<double>(bits_to_float(err_bits)) : 0.0;
    if (nredo > 0) {
        // exact FP64 search for the uncertain queries (same output rows)
        if (k + 8 <= 32) {
            run_f64<float, 32>(data, n, dim, k, redo.get(), nredo, out_idx, out_dist, out_dist64, s);
        } else if (k + 8 <= 64) {
            run_f64<float, 64>(data, n, dim, k, redo.get(), nredo, out_idx, out_dist, out_dist64, s);
        } else {
            run_f64<float, 128>(data, n, dim, k, redo.get(), nredo, out_idx, out_dist, out_dist64, s);
        }
    }
}

__global__ void row_norms_kernel(const float* __restrict__ data, int32_t n, int32_t dim, float* __restrict__ norms) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int d = 0; d < dim; ++d) {
            const double v = data[static_cast<size_t>(i) * dim + d];
            s += v * v;
        }
        norms[i] = static_cast<float>(s);
    }
}

__global__ void shift_indices_kernel(int32_t* __restrict__ idx, size_t count, int32_t delta) {
    for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < count; t += size_t(gridDim.x) * blockDim.x)
        idx[t] += delta;
}

// Batched tensor-core search with FP64 rescoring; instances holding uncertain
// queries are recomputed whole by the per-instance search.
template <int KCAP>
void run_f32_batched(const float* data, const std::vector<int32_t>& inst, int32_t dim, int32_t k, int32_t* out_idx,
                     float* out_dist, cudaStream_t s) {
    const int ninst = static_cast<int>(inst.size()) - 1;
    const int32_t n = inst[ninst];
    DevArray<int32_t> ci(static_cast<size_t>(n) * KCAP, s);
    DevArray<float> cd(static_cast<size_t>(n) * KCAP, s);
    DevArray<int> err(1, s);
    err.zero(s);
    knn_tc_candidates_batched(data, inst, dim, KCAP, ci.get(), cd.get(), err.get(), s);
    int h_err = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    if (h_err != DEV_OK) fail(UMAPB_ERR_DEVICE_TIMEOUT, "tensor-core kNN: a pipeline wait gave up");
    DevArray<float> norms(n, s);
    DevArray<unsigned int> norm_max(1, s);
    norm_max.zero(s);
    row_norms_kernel<<<grid_for(n, 256), 256, 0, s>>>(data, n, dim, norms.get());
    UMAPB_LAUNCH_CHECK();
    norm_max_kernel<<<grid_for(n, 256, 1024), 256, 0, s>>>(n, norms.get(), norm_max.get());
    UMAPB_LAUNCH_CHECK();
    DevArray<int32_t> redo(n, s), redo_count(1, s);
    redo_count.zero(s);
    DevArray<unsigned int> tc_err(1, s);
    tc_err.zero(s);
    knn_rescore_kernel<KCAP><<<(n + 127) / 128, 128, 0, s>>>(data, n - 1, dim, k, nullptr, n, 0, 0, ci.get(), cd.get(),
                                                             out_idx,
                                                             out_dist,
                                                             nullptr, redo.get(), redo_count.get(), norms.get(),
                                                             norm_max.get(), TC_REL_BOUND, tc_err.get());
    UMAPB_LAUNCH_CHECK();
    int32_t nredo = 0;
    unsigned int err_bits = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&nredo, redo_count.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(&err_bits, tc_err.get(), sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    last_knn_redo_count() = nredo;
    last_knn_tc_error() = static_cast<double>(bits_to_float(err_bits));
    if (nredo > 0) {
        std::vector<int32_t> rq(nredo);
        UMAPB_CUDA(cudaMemcpyAsync(rq.data(), redo.get(), nredo * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);
        std::vector<char> mark(ninst, 0);
        for (int32_t q : rq) mark[std::upper_bound(inst.begin(), inst.end(), q) - inst.begin() - 1] = 1;
        for (int i = 0; i < ninst; ++i) {
            if (!mark[i]) continue;
            const int32_t start = inst[i], len = inst[i + 1] - inst[i];
            run_f64<float, KCAP>(data + static_cast<size_t>(start) * dim, len, dim, k, nullptr, len,
                                 out_idx + static_cast<size_t>(start) * k, out_dist + static_cast<size_t>(start) * k,
                                 nullptr, s);
            shift_indices_kernel<<<grid_for(static_cast<size_t>(len) * k, 256), 256, 0, s>>>(
                out_idx + static_cast<size_t>(start) * k, static_cast<size_t>(len) * k, start);
            UMAPB_LAUNCH_CHECK();
        }
    }
}

}  // namespace

template <typename T>
void knn_exact_batched(const T* data, const std::vector<int32_t>& inst, int32_t dim, int32_t k, int32_t* out_idx,
                       T* out_dist, cudaStream_t s) {
    const int ninst = static_cast<int>(inst.size()) - 1;
    require(ninst >= 1, "at least one instance is needed");
    require(k >= 1 && k <= 120, "num_neighbors must be in [1, 120] for the device search");
    for (int i = 0; i < ninst; ++i) {
        require(inst[i + 1] - inst[i] > k, "every instance needs more observations than num_neighbors");
    }
    if constexpr (std::is_same<T, float>::value) {
        const int kcap = (k + 8 <= 16) ? 16 : (k + 8 <= 24) ? 24 : 32;
        if (k + 8 <= 32 && use_tensor_cores() && knn_tc_supported(dim, kcap)) {
            if (kcap == 16) run_f32_batched<16>(data, inst, dim, k, out_idx, out_dist, s);
            else if (kcap == 24) run_f32_batched<24>(data, inst, dim, k, out_idx, out_dist, s);
            else run_f32_batched<32>(data, inst, dim, k, out_idx, out_dist, s);
            return;
        }
    }
    for (int i = 0; i < ninst; ++i) {
        const int32_t start = inst[i], len = inst[i + 1] - inst[i];
        knn_exact<T>(data + static_cast<size_t>(start) * dim, len, dim, k, out_idx + static_cast<size_t>(start) * k,
                     out_dist + static_cast<size_t>(start) * k, s);
        shift_indices_kernel<<<grid_for(static_cast<size_t>(len) * k, 256), 256, 0, s>>>(
            out_idx + static_cast<size_t>(start) * k, static_cast<size_t>(len) * k, start);
        UMAPB_LAUNCH_CHECK();
    }
}

template void knn_exact_batched<float>(const float*, const std::vector<int32_t>&, int32_t, int32_t, int32_t*, float*,
                                       cudaStream_t);
template void knn_exact_batched<double>(const double*, const std::vector<int32_t>&, int32_t, int32_t, int32_t*,
                                        double*, cudaStream_t);

template <typename T>
void knn_exact_shard(const T* data, int32_t n, int32_t dim, int32_t k, KnnShard shard, int32_t* out_idx, T* out_dist,
                     DevArray<int32_t>& rows, int32_t& nrows, cudaStream_t s) {
    require(n >= 2, "the neighbour search needs at least two observations");
    require(dim >= 1, "data_dim must be positive");
    require(k >= 1 && k < n, "num_neighbors must be in [1, num_obs)");
    require(k <= 120, "num_neighbors above 120 is not supported by the device search");
    require(shard.count >= 1 && shard.index >= 0 && shard.index < shard.count, "shard must be in [0, num_shards)");
    if (shard.count == 1) {
        knn_exact<T>(data, n, dim, k, out_idx, out_dist, s);
        rows.allocate(n, s);
        iota_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, 0, rows.get());
        UMAPB_LAUNCH_CHECK();
        nrows = n;
        return;
    }
    if constexpr (std::is_same<T, float>::value) {
        if (k + 8 <= 16) run_f32<16>(data, n, dim, k, out_idx, out_dist, nullptr, s, shard, &rows, &nrows);
        else if (k + 8 <= 24) run_f32<24>(data, n, dim, k, out_idx, out_dist, nullptr, s, shard, &rows, &nrows);
        else if (k + 8 <= 32) run_f32<32>(data, n, dim, k, out_idx, out_dist, nullptr, s, shard, &rows, &nrows);
        else if (k + 8 <= 64) run_f32<64>(data, n, dim, k, out_idx, out_dist, nullptr, s, shard, &rows, &nrows);
        else run_f32<128>(data, n, dim, k, out_idx, out_dist, nullptr, s, shard, &rows, &nrows);
    } else {
        int32_t lo, hi;
        shard_row_range(n, shard, lo, hi);
        nrows = hi - lo;
        rows.allocate(std::max<int32_t>(nrows, 1), s);
        if (nrows > 0) {
            iota_kernel<<<grid_for(nrows, 256), 256, 0, s>>>(nrows, lo, rows.get());
            UMAPB_LAUNCH_CHECK();
            if (k <= 16) run_f64<double, 16>(data, n, dim, k, rows.get(), nrows, out_idx, out_dist, nullptr, s);
            else if (k <= 32) run_f64<double, 32>(data, n, dim, k, rows.get(), nrows, out_idx, out_dist, nullptr, s);
            else if (k <= 64) run_f64<double, 64>(data, n, dim, k, rows.get(), nrows, out_idx, out_dist, nullptr, s);
            else run_f64<double, 128>(data, n, dim, k, rows.get(), nrows, out_idx, out_dist, nullptr, s);
        }
    }
}

template void knn_exact_shard<float>(const float*, int32_t, int32_t, int32_t, KnnShard, int32_t*, float*,
                                     DevArray<int32_t>&, int32_t&, cudaStream_t);
template void knn_exact_shard<double>(const double*, int32_t, int32_t, int32_t, KnnShard, int32_t*, double*,
                                      DevArray<int32_t>&, int32_t&, cudaStream_t);

__global__ void add_offset_kernel(int32_t count, const int32_t* __restrict__ src, int32_t add,
                                  int32_t* __restrict__ dst) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) dst[i] = src[i] + add;
}

// Float queries against reference rows: FP32 brute-force candidates (from
// differences), FP64 rescoring and certification, FP64 search of the
// uncertain queries.  rows[slot] = nref + slot are the queries' data rows;
// results are written by slot.
template <int KCAP>
void run_query_f32(const float* data, int32_t nref, int32_t nq, int32_t dim, int32_t k, const int32_t* rows,
                   int32_t* out_idx, float* out_dist, cudaStream_t s) {
    DevArray<int32_t> ci(static_cast<size_t>(nq) * KCAP, s);
    DevArray<float> cd(static_cast<size_t>(nq) * KCAP, s);
    knn_bruteforce_kernel<float, float, KCAP><<<(nq + KNN_BLOCK - 1) / KNN_BLOCK, KNN_BLOCK, 0, s>>>(
        data, nref, dim, rows, nq, ci.get(), cd.get());
    UMAPB_LAUNCH_CHECK();
    DevArray<int32_t> redo(nq, s), redo_count(1, s);
    redo_count.zero(s);
    knn_rescore_kernel<KCAP><<<(nq + 127) / 128, 128, 0, s>>>(data, nref, dim, k, rows, nq, 1, 1, ci.get(), cd.get(),
                                                              out_idx, out_dist, nullptr, redo.get(), redo_count.get(),
                                                              nullptr, nullptr, TC_REL_BOUND, nullptr);
    UMAPB_LAUNCH_CHECK();
    int32_t nredo = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&nredo, redo_count.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    last_knn_redo_count() = nredo;
    if (nredo > 0) {   // redo holds slots: their data rows are nref + slot
        DevArray<int32_t> redo_rows(nredo, s);
        add_offset_kernel<<<grid_for(nredo, 256), 256, 0, s>>>(nredo, redo.get(), nref, redo_rows.get());
        UMAPB_LAUNCH_CHECK();
        if (k + 8 <= 32) run_f64<float, 32>(data, nref, dim, k, redo_rows.get(), nredo, out_idx, out_dist, nullptr, s, redo.get());
        else if (k + 8 <= 64) run_f64<float, 64>(data, nref, dim, k, redo_rows.get(), nredo, out_idx, out_dist, nullptr, s, redo.get());
        else run_f64<float, 128>(data, nref, dim, k, redo_rows.get(), nredo, out_idx, out_dist, nullptr, s, redo.get());
    }
}

template <typename T>
void knn_query(const T* data, int32_t nref, int32_t nq, int32_t dim, int32_t k, int32_t* out_idx, T* out_dist,
               cudaStream_t s) {
    require(nref >= 1, "the search needs at least one reference point");
    require(dim >= 1, "data_dim must be positive");
    require(nq >= 0, "the number of query points must not be negative");
    require(k >= 1 && k <= nref, "num_neighbors must be in [1, number of reference points]");
    require(k <= 120, "num_neighbors above 120 is not supported by the device search");
    require(static_cast<int64_t>(nref) + nq <= INT32_MAX, "too many points for 32-bit indices");
    if (nq == 0) return;
    DevArray<int32_t> rows(nq, s);
    iota_kernel<<<grid_for(nq, 256), 256, 0, s>>>(nq, nref, rows.get());
    UMAPB_LAUNCH_CHECK();
    if constexpr (std::is_same<T, float>::value) {
        if (k + 8 <= 16) run_query_f32<16>(data, nref, nq, dim, k, rows.get(), out_idx, out_dist, s);
        else if (k + 8 <= 24) run_query_f32<24>(data, nref, nq, dim, k, rows.get(), out_idx, out_dist, s);
        else if (k + 8 <= 32) run_query_f32<32>(data, nref, nq, dim, k, rows.get(), out_idx, out_dist, s);
        else if (k + 8 <= 64) run_query_f32<64>(data, nref, nq, dim, k, rows.get(), out_idx, out_dist, s);
        else run_query_f32<128>(data, nref, nq, dim, k, rows.get(), out_idx, out_dist, s);
    } else {
        DevArray<int32_t> slots(nq, s);
        iota_kernel<<<grid_for(nq, 256), 256, 0, s>>>(nq, 0, slots.get());
        UMAPB_LAUNCH_CHECK();
        if (k <= 16) run_f64<double, 16>(data, nref, dim, k, rows.get(), nq, out_idx, out_dist, nullptr, s, slots.get());
        else if (k <= 32) run_f64<double, 32>(data, nref, dim, k, rows.get(), nq, out_idx, out_dist, nullptr, s, slots.get());
        else if (k <= 64) run_f64<double, 64>(data, nref, dim, k, rows.get(), nq, out_idx, out_dist, nullptr, s, slots.get());
        else run_f64<double, 128>(data, nref, dim, k, rows.get(), nq, out_idx, out_dist, nullptr, s, slots.get());
    }
}

template void knn_query<float>(const float*, int32_t, int32_t, int32_t, int32_t, int32_t*, float*, cudaStream_t);
template void knn_query<double>(const double*, int32_t, int32_t, int32_t, int32_t, int32_t*, double*, cudaStream_t);

template <typename T>
void knn_exact(const T* data, int32_t n, int32_t dim, int32_t k, int32_t* out_idx, T* out_dist, cudaStream_t s,
               double* out_dist_f64) {
    require(n >= 2, "the neighbour search needs at least two observations");
    require(dim >= 1, "data_dim must be positive");
    require(k >= 1 && k < n, "num_neighbors must be in [1, num_obs)");
    require(k <= 120, "num_neighbors above 120 is not supported by the device search");
    if constexpr (std::is_same<T, float>::value) {
        if (k + 8 <= 16) {
            run_f32<16>(data, n, dim, k, out_idx, out_dist, out_dist_f64, s);
        } else if (k + 8 <= 24) {
            run_f32<24>(data, n, dim, k, out_idx, out_dist, out_dist_f64, s);
        } else if (k + 8 <= 32) {
            run_f32<32>(data, n, dim, k, out_idx, out_dist, out_dist_f64, s);
        } else if (k + 8 <= 64) {
            run_f32<64>(data, n, dim, k, out_idx, out_dist, out_dist_f64, s);
        } else {
            run_f32<128>(data, n, dim, k, out_idx, out_dist, out_dist_f64, s);
        }
    } else {
        if (k <= 16) {
            run_f64<double, 16>(data, n, dim, k, nullptr, n, out_idx, out_dist, out_dist_f64, s);
        } else if (k <= 32) {
            run_f64<double, 32>(data, n, dim, k, nullptr, n, out_idx, out_dist, out_dist_f64, s);
        } else if (k <= 64) {
            run_f64<double, 64>(data, n, dim, k, nullptr, n, out_idx, out_dist, out_dist_f64, s);
        } else {
            run_f64<double, 128>(data, n, dim, k, nullptr, n, out_idx, out_dist, out_dist_f64, s);
        }
    }
}

template void knn_exact<float>(const float*, int32_t, int32_t, int32_t, int32_t*, float*, cudaStream_t, double*);
template void knn_exact<double>(const double*, int32_t, int32_t, int32_t, int32_t*, double*, cudaStream_t, double*);

}  // namespace umapb
