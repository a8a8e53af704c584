// Graph stages on the device:
//  - combine_neighbor_sets (include/umappp/combine_neighbor_sets.hpp:16-99) as
//    a sort-and-reduce: every directed entry i -> j is emitted under both keys
//    (i, j) and (j, i); one radix sort groups the at most two records of each
//    ordered pair, and a segmented pass applies the reference's union /
//    intersection / mixture rule and emits rows already sorted by index (CSR).
//  - similarities_to_epochs (include/umappp/optimize_layout.hpp:47-92): max
//    reduction, per-row compaction of edges with w >= max / num_epochs and the
//    per-edge schedule.
//  - connected components by lock-free union-find (for
//    has_multiple_components, include/umappp/spectral_init.hpp:142-168).
// Compiled with -fmad=false: the union's w + w' - w w' and the schedule's
// divisions must round exactly as in the reference.
#include <cub/cub.cuh>

#include <vector>

#include "stages.cuh"

namespace umapb {

static int bits_for(int64_t n) {
    int b = 1;
    while ((int64_t(1) << b) < n) ++b;
    return b;
}

// ------------------------------------------------------------ union ---

template <typename T>
__global__ void union_emit_kernel(int32_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                  const T* __restrict__ w, int bits, uint64_t* __restrict__ keys, T* __restrict__ vals,
                                  int* __restrict__ status) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            const int32_t j = idx[p];
            if (j < 0 || j >= n || j == i) {
                atomicExch(status, DEV_BAD_INPUT);
                keys[2 * p] = keys[2 * p + 1] = ~uint64_t(0);
                vals[2 * p] = vals[2 * p + 1] = T(0);
                continue;
            }
            keys[2 * p] = (static_cast<uint64_t>(i) << bits) | static_cast<uint64_t>(j);
            keys[2 * p + 1] = (static_cast<uint64_t>(j) << bits) | static_cast<uint64_t>(i);
            vals[2 * p] = w[p];
            vals[2 * p + 1] = w[p];
        }
    }
}

// For each sorted position that starts a key group: the combined value and
// whether it is kept (combine_neighbor_sets.hpp:47-90).
template <typename T>
__global__ void union_reduce_kernel(int64_t m, const uint64_t* __restrict__ keys, const T* __restrict__ vals, T mix,
                                    int* __restrict__ keep, T* __restrict__ value, int* __restrict__ status) {
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < m; p += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t key = keys[p];
        const bool head = (p == 0 || keys[p - 1] != key) && key != ~uint64_t(0);
        int k = 0;
        T v = T(0);
        if (head) {
            const bool pair = (p + 1 < m && keys[p + 1] == key);
            if (pair && p + 2 < m && keys[p + 2] == key) atomicExch(status, DEV_BAD_INPUT);  // duplicate neighbour
            const T x = vals[p];
            if (pair) {
                const T y = vals[p + 1];
                const T product = x * y;
                if (mix == T(1)) {
                    v = x + y - product;
                } else if (mix == T(0)) {
                    v = product;
                } else {
                    v = mix * (x + y - product) + (T(1) - mix) * product;
                }
                k = (mix == T(0)) ? (v != T(0)) : 1;
            } else {
                if (mix == T(1)) {
                    v = x;
                    k = 1;
                } else if (mix == T(0)) {
                    k = 0;
                } else {
                    v = x * mix;
                    k = 1;
                }
            }
        }
        keep[p] = k;
        value[p] = v;
    }
}

template <typename T>
__global__ void union_scatter_kernel(int64_t m, const uint64_t* __restrict__ keys, const int* __restrict__ keep,
                                     const int64_t* __restrict__ pos, const T* __restrict__ value, int bits,
                                     int32_t* __restrict__ out_idx, T* __restrict__ out_val,
                                     int32_t* __restrict__ out_row) {
    const uint64_t mask = (uint64_t(1) << bits) - 1;
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < m; p += int64_t(gridDim.x) * blockDim.x) {
        if (keep[p]) {
            const int64_t q = pos[p];
            out_idx[q] = static_cast<int32_t>(keys[p] & mask);
            out_row[q] = static_cast<int32_t>(keys[p] >> bits);
            out_val[q] = value[p];
        }
    }
}

// row_ptr from the (sorted) row of every output entry.
__global__ void rows_to_ptr_kernel(int32_t n, int64_t nnz, const int32_t* __restrict__ row, int64_t* __restrict__ ptr) {
    for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q <= nnz; q += int64_t(gridDim.x) * blockDim.x) {
        const int64_t lo = (q == 0) ? -1 : row[q - 1];
        const int64_t hi = (q == nnz) ? n : row[q];
        for (int64_t r = lo + 1; r <= hi; ++r) ptr[r] = q;
    }
}

template <typename T>
void combine_neighbor_sets(int32_t n, const int64_t* ptr, const int32_t* idx, const T* w, int64_t nnz_in,
                           double mix_ratio, DeviceCsr<T>& out, cudaStream_t s) {
    out.n = n;
    out.ptr.allocate(static_cast<size_t>(n) + 1, s);
    if (nnz_in == 0) {
        out.ptr.zero(s);
        out.nnz = 0;
        return;
    }
    const int bits = bits_for(n);
    require(2 * bits <= 64, "too many observations for the union keys", UMAPB_ERR_OVERFLOW);
    const int64_t m = 2 * nnz_in;
    DevArray<int> status(1, s);
    status.zero(s);
    DevArray<uint64_t> keys_a(m, s), keys_b(m, s);
    DevArray<T> vals_a(m, s), vals_b(m, s);
    union_emit_kernel<T><<<grid_for(n, 256), 256, 0, s>>>(n, ptr, idx, w, bits, keys_a.get(), vals_a.get(), status.get());
    UMAPB_LAUNCH_CHECK();

    cub::DoubleBuffer<uint64_t> dk(keys_a.get(), keys_b.get());
    cub::DoubleBuffer<T> dv(vals_a.get(), vals_b.get());
    size_t temp_bytes = 0;
    UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, dk, dv, m, 0, 2 * bits, s));
    {
        DevArray<unsigned char> temp(temp_bytes, s);
        UMAPB_CUDA(cub::DeviceRadixSort::SortPairs(temp.get(), temp_bytes, dk, dv, m, 0, 2 * bits, s));
    }
    // keys equal to ~0 (bad entries) sort last only if they exceed 2*bits; they are never heads anyway.
    const uint64_t* skeys = dk.Current();
    const T* svals = dv.Current();

    DevArray<int> keep(m, s);
    DevArray<T> value(m, s);
    union_reduce_kernel<T><<<grid_for(m, 256), 256, 0, s>>>(m, skeys, svals, static_cast<T>(mix_ratio), keep.get(),
                                                            value.get(), status.get());
    UMAPB_LAUNCH_CHECK();

    // exclusive positions of the kept groups; the total is the last position plus the last flag
    DevArray<int64_t> pos(m, s);
    {
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, keep.get(), pos.get(), m, s));
        DevArray<unsigned char> temp(tb, s);
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(temp.get(), tb, keep.get(), pos.get(), m, s));
    }
    int64_t last_pos = 0;
    int last_keep = 0, st = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&last_pos, pos.get() + (m - 1), sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(&last_keep, keep.get() + (m - 1), sizeof(int), cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(&st, status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    require(st == DEV_OK,
            "neighbour list has an out-of-range index, a self edge or a duplicate neighbour (when the list comes from "
            "a neighbour search of the data: a NaN or infinite coordinate leaves rows without neighbours, index -1)");
    const int64_t nnz = last_pos + last_keep;

    out.nnz = nnz;
    out.idx.allocate(nnz, s);
    out.val.allocate(nnz, s);
    DevArray<int32_t> rows(nnz, s);
    union_scatter_kernel<T><<<grid_for(m, 256), 256, 0, s>>>(m, skeys, keep.get(), pos.get(), value.get(), bits,
                                                             out.idx.get(), out.val.get(), rows.get());
    UMAPB_LAUNCH_CHECK();
    rows_to_ptr_kernel<<<grid_for(nnz + 1, 256), 256, 0, s>>>(n, nnz, rows.get(), out.ptr.get());
    UMAPB_LAUNCH_CHECK();
}

// ----------------------------------------------------------- epochs ---

template <typename T>
struct MaxOp {
    __device__ __forceinline__ T operator()(const T& a, const T& b) const { return (a < b) ? b : a; }   // std::max
};

// The maximum weight that applies to row i: one value, or (batched runs) the
// maximum of row i's instance, instance j owning rows [inst[j], inst[j + 1]).
template <typename T>
__device__ __forceinline__ T row_max(int32_t i, const T* __restrict__ maxed, const int32_t* __restrict__ inst,
                                     int num_inst) {
    if (num_inst <= 1) return maxed[0];
    int lo = 0, hi = num_inst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (inst[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return maxed[lo];
}

template <typename T>
__global__ void epochs_count_kernel(int32_t n, const int64_t* __restrict__ ptr, const T* __restrict__ w,
                                    const T* __restrict__ maxed, const int32_t* __restrict__ inst, int num_inst,
                                    int num_epochs, int64_t* __restrict__ counts) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const T limit = row_max(i, maxed, inst, num_inst) / static_cast<T>(num_epochs);      // :63
        int64_t c = 0;
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) c += (w[p] >= limit);
        counts[i] = c;
    }
}

template <typename T>
__global__ void epochs_fill_kernel(int32_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                   const T* __restrict__ w, const T* __restrict__ maxed,
                                   const int32_t* __restrict__ inst, int num_inst, int num_epochs, T rate,
                                   const int64_t* __restrict__ out_ptr, int32_t* __restrict__ heads,
                                   int32_t* __restrict__ targets, T* __restrict__ eps, T* __restrict__ enext,
                                   T* __restrict__ enneg) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const T mx = row_max(i, maxed, inst, num_inst);
        const T limit = mx / static_cast<T>(num_epochs);
        int64_t q = out_ptr[i];
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            if (w[p] >= limit) {                                   // :68-71
                const T e = mx / w[p];
                heads[q] = i;
                targets[q] = idx[p];
                eps[q] = e;
                enext[q] = e;                                      // :77
                enneg[q] = e / rate;                               // :78-81
                ++q;
            }
        }
    }
}

// Per-instance maxima (weights are non-negative, so their bit patterns order like the values).
template <typename T>
struct Bits;
template <>
struct Bits<float> {
    typedef unsigned int type;
    static __device__ __forceinline__ unsigned int of(float v) { return __float_as_uint(v); }
};
template <>
struct Bits<double> {
    typedef unsigned long long type;
    static __device__ __forceinline__ unsigned long long of(double v) {
        return static_cast<unsigned long long>(__double_as_longlong(v));
    }
};

template <typename T>
__global__ void instance_max_kernel(int32_t n, const int64_t* __restrict__ ptr, const T* __restrict__ w,
                                    const int32_t* __restrict__ inst, int num_inst,
                                    typename Bits<T>::type* __restrict__ maxed_bits) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int lo = 0, hi = num_inst - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (inst[mid] <= i) lo = mid; else hi = mid - 1;
        }
        typename Bits<T>::type m = 0;
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            const typename Bits<T>::type b = Bits<T>::of(w[p]);
            m = (m < b) ? b : m;
        }
        if (m) atomicMax(&maxed_bits[lo], m);
    }
}

template <typename T>
void similarities_to_epochs(int32_t n, const int64_t* ptr, const int32_t* idx, const T* w, int64_t nnz, int num_epochs,
                            double negative_sample_rate, DeviceEpochs<T>& out, cudaStream_t s,
                            const int32_t* inst_start, int32_t num_inst) {
    require(num_epochs > 0, "num_epochs must be positive");
    // the reference checks that num_epochs * rate fits an int (optimize_layout.hpp:89)
    const double cap = static_cast<double>(static_cast<T>(num_epochs) * static_cast<T>(negative_sample_rate));
    require(std::isfinite(cap) && std::trunc(cap) <= 2147483647.0 && std::trunc(cap) >= -2147483648.0,
            "num_epochs * negative_sample_rate does not fit an int", UMAPB_ERR_OVERFLOW);
    out.n = n;
    out.total_epochs = num_epochs;
    out.negative_sample_rate = static_cast<T>(negative_sample_rate);
    out.ptr.allocate(static_cast<size_t>(n) + 1, s);

    const int ni = (inst_start && num_inst > 1) ? num_inst : 1;
    DevArray<T> maxed(ni, s);
    if (ni > 1) {
        maxed.zero(s);
        if (n > 0) {
            instance_max_kernel<T><<<grid_for(n, 256), 256, 0, s>>>(
                n, ptr, w, inst_start, ni, reinterpret_cast<typename Bits<T>::type*>(maxed.get()));
            UMAPB_LAUNCH_CHECK();
        }
    } else if (nnz > 0) {
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceReduce::Reduce(nullptr, tb, w, maxed.get(), nnz, MaxOp<T>(), T(0), s));
        DevArray<unsigned char> temp(tb, s);
        UMAPB_CUDA(cub::DeviceReduce::Reduce(temp.get(), tb, w, maxed.get(), nnz, MaxOp<T>(), T(0), s));
    } else {
        maxed.zero(s);
    }
    DevArray<int64_t> counts(static_cast<size_t>(n) + 1, s);
    counts.zero(s);
    if (n > 0) {
        epochs_count_kernel<T><<<grid_for(n, 256), 256, 0, s>>>(n, ptr, w, maxed.get(), inst_start, ni, num_epochs,
                                                                counts.get());
        UMAPB_LAUNCH_CHECK();
    }
    {
        size_t tb = 0;
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, counts.get(), out.ptr.get(), n + 1, s));
        DevArray<unsigned char> temp(tb, s);
        UMAPB_CUDA(cub::DeviceScan::ExclusiveSum(temp.get(), tb, counts.get(), out.ptr.get(), n + 1, s));
    }
    int64_t kept = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&kept, out.ptr.get() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    out.nnz = kept;
    out.heads.allocate(kept, s);
    out.targets.allocate(kept, s);
    out.eps.allocate(kept, s);
    out.enext0.allocate(kept, s);
    out.enneg0.allocate(kept, s);
    if (n > 0 && kept > 0) {
        epochs_fill_kernel<T><<<grid_for(n, 256), 256, 0, s>>>(n, ptr, idx, w, maxed.get(), inst_start, ni, num_epochs,
                                                               static_cast<T>(negative_sample_rate), out.ptr.get(),
                                                               out.heads.get(), out.targets.get(), out.eps.get(),
                                                               out.enext0.get(), out.enneg0.get());
        UMAPB_LAUNCH_CHECK();
    }
}

// ------------------------------------------------------- components ---

__device__ __forceinline__ int32_t uf_find(int32_t* parent, int32_t x) {
    // path halving; every step moves strictly toward a smaller index, so it ends
    int32_t p = parent[x];
    while (p != x) {
        const int32_t gp = parent[p];
        if (gp != p) atomicMin(&parent[x], gp);
        x = p;
        p = parent[x];
    }
    return x;
}

__global__ void uf_init_kernel(int32_t n, int32_t* parent) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) parent[i] = i;
}

// Hooks the larger root under the smaller one.  Roots only ever point to
// smaller indices, so the loop makes progress; it is still capped, and a cap
// hit is reported through the status word.
__global__ void uf_hook_kernel(int32_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                               int32_t* parent, int* status) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            const int32_t j = idx[p];
            if (j < 0 || j >= n) {
                atomicExch(status, DEV_BAD_INPUT);
                continue;
            }
            int32_t a = i, b = j;
            bool done = false;
            for (int iter = 0; iter < (1 << 20) && !done; ++iter) {
                a = uf_find(parent, a);
                b = uf_find(parent, b);
                if (a == b) {
                    done = true;
                } else {
                    if (a < b) {
                        const int32_t t = a;
                        a = b;
                        b = t;
                    }
                    // a > b: try to make b the parent of root a
                    if (atomicCAS(&parent[a], a, b) == a) done = true;
                }
            }
            if (!done) atomicExch(status, DEV_TIMEOUT);
        }
    }
}

__global__ void uf_count_roots_kernel(int32_t n, const int32_t* parent, unsigned long long* count) {
    unsigned long long local = 0;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) local += (parent[i] == i);
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

int64_t count_components(int32_t n, const int64_t* ptr, const int32_t* idx, int* d_status, cudaStream_t s) {
    if (n <= 0) return 0;
    DevArray<int32_t> parent(n, s);
    DevArray<unsigned long long> count(1, s);
    count.zero(s);
    UMAPB_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), s));
    uf_init_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, parent.get());
    UMAPB_LAUNCH_CHECK();
    uf_hook_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, ptr, idx, parent.get(), d_status);
    UMAPB_LAUNCH_CHECK();
    uf_count_roots_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, parent.get(), count.get());
    UMAPB_LAUNCH_CHECK();
    unsigned long long h = 0;
    int st = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&h, count.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    UMAPB_CUDA(cudaMemcpyAsync(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    if (st == DEV_TIMEOUT) fail(UMAPB_ERR_DEVICE_TIMEOUT, "union-find hook loop hit its iteration cap");
    if (st == DEV_BAD_INPUT) fail(UMAPB_ERR_INVALID, "graph has an out-of-range neighbour index");
    return static_cast<int64_t>(h);
}

template void combine_neighbor_sets<float>(int32_t, const int64_t*, const int32_t*, const float*, int64_t, double,
                                           DeviceCsr<float>&, cudaStream_t);
template void combine_neighbor_sets<double>(int32_t, const int64_t*, const int32_t*, const double*, int64_t, double,
                                            DeviceCsr<double>&, cudaStream_t);
template void similarities_to_epochs<float>(int32_t, const int64_t*, const int32_t*, const float*, int64_t, int, double,
                                            DeviceEpochs<float>&, cudaStream_t, const int32_t*, int32_t);
template void similarities_to_epochs<double>(int32_t, const int64_t*, const int32_t*, const double*, int64_t, int,
                                             double, DeviceEpochs<double>&, cudaStream_t, const int32_t*, int32_t);

}  // namespace umapb
