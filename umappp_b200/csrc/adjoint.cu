// Adjoint of the UMAP fuzzy cross-entropy (no counterpart in the reference,
// whose SGD applies the per-edge derivatives directly,
// include/umappp/optimize_layout.hpp:147-149 attractive, :170-171 repulsive).
//
// For every stored directed edge (i -> j, weight w), with d2 = |y_i - y_j|^2
// and q = 1 / (1 + a d2^b):
//   loss  += w * (-log q) + (1 - w) * (-log(1 - q))
//          = w log(1 + a d2^b) + (1 - w) (log(1 + a d2^b) - log a - b log d2)
//   dL/dd2 = w * a b d2^(b-1) / (1 + a d2^b) - (1 - w) * b / ((d2 + eps_rep) (1 + a d2^b))
//   dL/dy_i = 2 dL/dd2 (y_i - y_j) = -dL/dy_j
//   dL/da  = w d2^b / (1 + a d2^b) - (1 - w) / (a (1 + a d2^b))
//   dL/db  = w a d2^b log d2 / (1 + a d2^b) - (1 - w) log d2 / (1 + a d2^b)
// The reference's SGD step on an edge is y_i -= alpha clamp(dL/dy_i) for the
// w = 1 term (attractive) and for a w = 0 term with eps_rep = 0.001 and the
// factor gamma (repulsive), which is what the tests check.
// One thread per observation walks its row (coalesced CSR reads); FP64
// accumulation; the loss and dL/da, dL/db are block-reduced then added once
// per block; per-coordinate gradients use FP64 atomics.
#include <cub/cub.cuh>

#include <mutex>
#include <type_traits>

#include "stages.cuh"
#include "umap_grad.cuh"

namespace umapb {

namespace {

constexpr int ADJ_BLOCK = 256;

template <typename T>
__global__ void __launch_bounds__(ADJ_BLOCK) loss_grad_kernel(int32_t n, int dim, const T* __restrict__ Y,
                                                              const int64_t* __restrict__ ptr,
                                                              const int32_t* __restrict__ idx, const T* __restrict__ w,
                                                              double a, double b, double eps_rep, int with_constant,
                                                              double* __restrict__ gY, double* __restrict__ acc) {
    typedef cub::BlockReduce<double, ADJ_BLOCK> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    double loss = 0, ga = 0, gb = 0;
    const double log_a = log(a);
    const int32_t i = blockIdx.x * ADJ_BLOCK + threadIdx.x;
    bool bad = false;
    if (i < n) {
        const T* yi = Y + static_cast<size_t>(i) * dim;
        // a row outside [0, ptr[n]] or running backwards is skipped and flagged
        const int64_t p0 = ptr[i], p1 = ptr[i + 1], nnz = ptr[n];
        if (p0 < 0 || p1 < p0 || p1 > nnz) bad = true;
        for (int64_t p = p0; !bad && p < p1; ++p) {
            const int32_t j = idx[p];
            if (j < 0 || j >= n) {   // out-of-range neighbour: skipped and flagged
                bad = true;
                continue;
            }
            const T* yj = Y + static_cast<size_t>(j) * dim;
            double d2 = 0;
            for (int d = 0; d < dim; ++d) {
                const double diff = static_cast<double>(yi[d]) - static_cast<double>(yj[d]);
                d2 += diff * diff;
            }
            const double wij = static_cast<double>(w[p]);
            const double pd2b = pow(d2, b);
            const double denom = 1 + a * pd2b;
            const double lq = log(denom);
            const double ld2 = log(d2);
            loss += wij * lq + (1 - wij) * (lq - log_a - b * ld2);
            if (with_constant) {
                if (wij > 0) loss += wij * log(wij);
                if (wij < 1) loss += (1 - wij) * log(1 - wij);
            }
            const double att = attract_dd2<false>(d2, a, b, a * b);    // dA/dd2 (umap_grad.cuh)
            const double rep = repulse_dd2<false>(d2, a, b, -b, eps_rep);   // dR/dd2
            const double dd2 = wij * att + (1 - wij) * rep;
            if (gY) {
                for (int d = 0; d < dim; ++d) {
                    const double g = 2 * dd2 * (static_cast<double>(yi[d]) - static_cast<double>(yj[d]));
                    atomicAdd(gY + static_cast<size_t>(i) * dim + d, g);
                    atomicAdd(gY + static_cast<size_t>(j) * dim + d, -g);
                }
            }
            ga += wij * (pd2b / denom) + (1 - wij) * (-1.0 / (a * denom));
            gb += wij * (a * pd2b * ld2 / denom) + (1 - wij) * (-ld2 / denom);
        }
    }
    loss = Reduce(tmp).Sum(loss);
    __syncthreads();
    ga = Reduce(tmp).Sum(ga);
    __syncthreads();
    gb = Reduce(tmp).Sum(gb);
    if (threadIdx.x == 0) {
        atomicAdd(acc + 0, loss);
        atomicAdd(acc + 1, ga);
        atomicAdd(acc + 2, gb);
    }
    if (bad) acc[3] = 1.0;   // invalid row_ptr or indices
}

template <typename T>
__global__ void cast_grad_kernel(size_t total, const double* __restrict__ src, T* __restrict__ dst) {
    for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x)
        dst[t] = static_cast<T>(src[t]);
}

}  // namespace

template <typename T>
void loss_grad(int32_t n, int num_dim, const T* Y, const int64_t* ptr, const int32_t* idx, const T* w, double a,
               double b, double eps_rep, bool with_constant, double* loss_out, T* grad_Y, double* grad_ab,
               cudaStream_t s) {
    require(a > 0 && b > 0, "a and b must be positive");
    DevArray<double> acc(4, s);
    acc.zero(s);
    const size_t total = static_cast<size_t>(n) * num_dim;
    DevArray<double> g64;
    double* gptr = nullptr;
    if (grad_Y) {
        if constexpr (std::is_same<T, double>::value) {
            gptr = grad_Y;
        } else {
            g64.allocate(total, s);
            gptr = g64.get();
        }
        UMAPB_CUDA(cudaMemsetAsync(gptr, 0, total * sizeof(double), s));
    }
    if (n > 0) {
        loss_grad_kernel<T><<<(n + ADJ_BLOCK - 1) / ADJ_BLOCK, ADJ_BLOCK, 0, s>>>(
            n, num_dim, Y, ptr, idx, w, a, b, eps_rep, with_constant ? 1 : 0, gptr, acc.get());
        UMAPB_LAUNCH_CHECK();
    }
    if (grad_Y && !std::is_same<T, double>::value) {
        cast_grad_kernel<T><<<grid_for(total, 256), 256, 0, s>>>(total, gptr, grad_Y);
        UMAPB_LAUNCH_CHECK();
    }
    double h[4];
    UMAPB_CUDA(cudaMemcpyAsync(h, acc.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    require(h[3] == 0, "row_ptr or indices out of range (row_ptr must run from 0 upwards, indices in [0, num_obs))");
    if (loss_out) *loss_out = h[0];
    if (grad_ab) {
        grad_ab[0] = h[1];
        grad_ab[1] = h[2];
    }
}

template void loss_grad<float>(int32_t, int, const float*, const int64_t*, const int32_t*, const float*, double, double,
                               double, bool, double*, float*, double*, cudaStream_t);
template void loss_grad<double>(int32_t, int, const double*, const int64_t*, const int32_t*, const double*, double,
                                double, double, bool, double*, double*, double*, cudaStream_t);

// ------------------------------------------------- allocation-free variant --
//
// Scratch for umapb_loss_grad_noalloc, resident on every device that loads the
// library: [0, 3) the loss and dL/da, dL/db accumulators, [3] the invalid-input
// flag, [4, 4 + max) the FP64 accumulation of a float gradient.  Its host-side
// name is only a stand-in; kernels get the device address from
// cudaGetSymbolAddress.
constexpr size_t NOALLOC_GRAD_MAX = size_t(1) << 22;   // gradient elements (n * num_dim) for float data
constexpr size_t NOALLOC_ACC_OFFSET = 0;
constexpr size_t NOALLOC_GRAD_OFFSET = 4;
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_GRAD_OFFSET + NOALLOC_GRAD_MAX];

namespace {

constexpr int MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[MAX_DEVICES] = {nullptr};

// Device address of the scratch on the current device, looked up on the first
// call on that device and cached for the life of the process (a
// cudaDeviceReset of that device invalidates it; the library does not support
// calls after a reset).
double* noalloc_scratch(int dev) {
    require(dev >= 0 && dev < MAX_DEVICES, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        UMAPB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    return g_noalloc_ptr[dev];
}

template <typename T>
void loss_grad_noalloc(int32_t n, int num_dim, const T* Y, const int64_t* ptr, const int32_t* idx, const T* w, double a,
                       double b, double eps_rep, bool with_constant, double* loss_out, T* grad_Y, double* grad_ab) {
    require(a > 0 && b > 0, "a and b must be positive");
    require(n >= 0 && num_dim >= 1, "num_obs must be non-negative and num_dim positive");
    const size_t total = static_cast<size_t>(n) * num_dim;
    if (grad_Y && std::is_same<T, float>::value) {
        require(total <= NOALLOC_GRAD_MAX,
                "num_obs * num_dim exceeds the allocation-free scratch (4194304 gradient elements for float data)");
    }
    if (n == 0) {   // nothing to read: no pointer is looked at, the results are zero
        if (loss_out) *loss_out = 0;
        if (grad_ab) grad_ab[0] = grad_ab[1] = 0;
        return;
    }
    // pointers of another device are rejected inside is_device_pointer
    require(is_device_pointer(Y) && is_device_pointer(ptr) && is_device_pointer(idx) && is_device_pointer(w),
            "the allocation-free entry point takes device pointers for embedding, row_ptr, indices and weights");
    require(!grad_Y || is_device_pointer(grad_Y), "grad_embedding must be a device pointer (or NULL)");
    int dev = 0;
    UMAPB_CUDA(cudaGetDevice(&dev));
    double* scratch = noalloc_scratch(dev);
    double* acc = scratch + NOALLOC_ACC_OFFSET;
    const cudaStream_t s = cudaStreamPerThread;
    UMAPB_CUDA(cudaMemsetAsync(acc, 0, 4 * sizeof(double), s));
    double* gptr = nullptr;
    if (grad_Y) {
        if constexpr (std::is_same<T, double>::value) {
            gptr = grad_Y;
        } else {
            gptr = scratch + NOALLOC_GRAD_OFFSET;
        }
        UMAPB_CUDA(cudaMemsetAsync(gptr, 0, total * sizeof(double), s));
    }
    loss_grad_kernel<T><<<(n + ADJ_BLOCK - 1) / ADJ_BLOCK, ADJ_BLOCK, 0, s>>>(
        n, num_dim, Y, ptr, idx, w, a, b, eps_rep, with_constant ? 1 : 0, gptr, acc);
    UMAPB_LAUNCH_CHECK();
    if (grad_Y && !std::is_same<T, double>::value) {
        cast_grad_kernel<T><<<grid_for(total, 256), 256, 0, s>>>(total, gptr, grad_Y);
        UMAPB_LAUNCH_CHECK();
    }
    double h[4];
    UMAPB_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    require(h[3] == 0, "row_ptr or indices out of range (row_ptr must run from 0 upwards, indices in [0, num_obs))");
    if (loss_out) *loss_out = h[0];
    if (grad_ab) {
        grad_ab[0] = h[1];
        grad_ab[1] = h[2];
    }
}

}  // namespace

}  // namespace umapb

extern "C" int umapb_loss_grad_noalloc(int dtype, size_t num_dim, const void* embedding, int32_t num_obs,
                                       const int64_t* row_ptr, const int32_t* indices, const void* weights, double a,
                                       double b, double eps_rep, int with_constant, double* loss,
                                       void* grad_embedding, double* grad_ab) {
    using namespace umapb;
    try {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            cudaGetLastError();
            fail(UMAPB_ERR_NO_DEVICE, "no CUDA device is available (libumappp_b200 runs on sm_100 GPUs only)");
        }
        require(dtype == UMAPB_F32 || dtype == UMAPB_F64, "dtype must be UMAPB_F32 or UMAPB_F64");
        if (dtype == UMAPB_F64) {
            loss_grad_noalloc<double>(num_obs, static_cast<int>(num_dim), static_cast<const double*>(embedding), row_ptr,
                                      indices, static_cast<const double*>(weights), a, b, eps_rep, with_constant != 0,
                                      loss, static_cast<double*>(grad_embedding), grad_ab);
        } else {
            loss_grad_noalloc<float>(num_obs, static_cast<int>(num_dim), static_cast<const float*>(embedding), row_ptr,
                                     indices, static_cast<const float*>(weights), a, b, eps_rep, with_constant != 0,
                                     loss, static_cast<float*>(grad_embedding), grad_ab);
        }
        return UMAPB_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        cudaGetLastError();
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return UMAPB_ERR_INVALID;
    }
}
