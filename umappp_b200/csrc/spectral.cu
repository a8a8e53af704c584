// Initial layouts on the device.
//
// spectral_init (include/umappp/spectral_init.hpp:171-207): connectivity
// check, then the top num_dim + 1 eigenvectors of the shifted normalised
// Laplacian I + D^-1/2 W D^-1/2 (built in FP64 exactly as :38-78), of which
// the last num_dim are scaled to a maximum magnitude of 'scale' (:126-137).
// The reference obtains them with irlba; here a thick-restart Lanczos
// iteration (Wu and Simon, SIAM J. Matrix Anal. Appl. 22(2), 2000) runs its
// sparse products, Gram-Schmidt reorthogonalisation (two passes, FP64) and
// Ritz-vector updates on the device; only the small projected eigenproblem
// (ncv x ncv, ncv <= 64) is solved on the host by cyclic Jacobi.  Eigenvectors
// are signed so that their largest-magnitude entry is positive.
//
// random_init (:209-225): uniform on (-scale, scale) from Philox4x32-10.
// Jitter (:190-204): Box-Muller normals from Philox4x32-10.
#include <algorithm>
#include <cmath>
#include <vector>

#include "stages.cuh"

namespace umapb {

namespace {

template <typename T>
__global__ void degree_sqrt_kernel(int32_t n, const int64_t* __restrict__ ptr, const T* __restrict__ w,
                                   double* __restrict__ sums) {
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        double s = 0;
        for (int64_t p = ptr[c]; p < ptr[c + 1]; ++p) s += static_cast<double>(w[p]);
        sums[c] = sqrt(s);
    }
}

template <typename T>
__global__ void laplacian_values_kernel(int32_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                        const T* __restrict__ w, const double* __restrict__ sums,
                                        double* __restrict__ lap) {
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        for (int64_t p = ptr[c]; p < ptr[c + 1]; ++p) {
            lap[p] = __dmul_rn(__ddiv_rn(__ddiv_rn(-static_cast<double>(w[p]), sums[idx[p]]), sums[c]), -1.0);
        }
    }
}

// y = (I + D^-1/2 W D^-1/2) x, each row summed in stored order with the unit
// diagonal at its sorted position (the compressed layout of :60-78).
__global__ void lap_spmv_kernel(int32_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                const double* __restrict__ lap, const double* __restrict__ x, double* __restrict__ y) {
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        int64_t p = ptr[c];
        const int64_t e = ptr[c + 1];
        double s = 0;
        for (; p < e && idx[p] < c; ++p) s = __dadd_rn(s, __dmul_rn(lap[p], x[idx[p]]));
        s = __dadd_rn(s, x[c]);
        for (; p < e; ++p) s = __dadd_rn(s, __dmul_rn(lap[p], x[idx[p]]));
        y[c] = s;
    }
}

constexpr int DOT_BLOCK = 256;

// partial[b * ncol + c] = sum over the rows of block b of V[:, c] * w
__global__ void __launch_bounds__(DOT_BLOCK) multi_dot_kernel(int32_t n, const double* __restrict__ V, int ncol,
                                                              const double* __restrict__ w,
                                                              double* __restrict__ partial) {
    __shared__ double red[DOT_BLOCK / 32];
    const int c = blockIdx.y;
    const double* v = V + static_cast<size_t>(c) * n;
    double s = 0;
    for (int32_t i = blockIdx.x * DOT_BLOCK + threadIdx.x; i < n; i += gridDim.x * DOT_BLOCK) s += v[i] * w[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int q = 0; q < DOT_BLOCK / 32; ++q) t += red[q];
        partial[static_cast<size_t>(blockIdx.x) * ncol + c] = t;
    }
}

__global__ void reduce_partials_kernel(int nblk, int ncol, const double* __restrict__ partial, double* __restrict__ h,
                                       double* __restrict__ h_accum) {
    const int c = threadIdx.x;
    if (c >= ncol) return;
    double t = 0;
    for (int b = 0; b < nblk; ++b) t += partial[static_cast<size_t>(b) * ncol + c];
    h[c] = t;
    if (h_accum) h_accum[c] += t;
}

// w -= V[:, :ncol] h
__global__ void subtract_projection_kernel(int32_t n, const double* __restrict__ V, int ncol,
                                           const double* __restrict__ h, double* __restrict__ w) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = w[i];
        for (int c = 0; c < ncol; ++c) s -= h[c] * V[static_cast<size_t>(c) * n + i];
        w[i] = s;
    }
}

__global__ void scale_vector_kernel(int32_t n, const double* __restrict__ x, double f, double* __restrict__ y) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i] * f;
}

// out[:, c] = V[:, :nrow] S[:, c] for c < ncol (S row-major nrow x ldS)
__global__ void ritz_vectors_kernel(int32_t n, const double* __restrict__ V, int nrow, const double* __restrict__ S,
                                    int ldS, int ncol, double* __restrict__ out) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int c = 0; c < ncol; ++c) {
            double s = 0;
            for (int r = 0; r < nrow; ++r) s += V[static_cast<size_t>(r) * n + i] * S[r * ldS + c];
            out[static_cast<size_t>(c) * n + i] = s;
        }
    }
}

// Deterministic start vector: splitmix64 of (seed + (i + 1) * golden) mapped to [-0.5, 0.5).
__global__ void start_vector_kernel(int32_t n, uint64_t seed, double* __restrict__ v) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint64_t z = seed + 0x9E3779B97F4A7C15ULL * static_cast<uint64_t>(i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        v[i] = static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
    }
}

// Per column: largest magnitude (as ordered bits; non-negative doubles order
// like their bit patterns), then the first index attaining it.
__global__ void col_max_abs_kernel(int32_t n, const double* __restrict__ V, unsigned long long* __restrict__ best) {
    const int c = blockIdx.y;
    const double* v = V + static_cast<size_t>(c) * n;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        atomicMax(&best[c], static_cast<unsigned long long>(__double_as_longlong(fabs(v[i]))));
    }
}

__global__ void col_first_at_kernel(int32_t n, const double* __restrict__ V, const unsigned long long* __restrict__ best,
                                    int* __restrict__ where) {
    const int c = blockIdx.y;
    const double* v = V + static_cast<size_t>(c) * n;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (static_cast<unsigned long long>(__double_as_longlong(fabs(v[i]))) == best[c]) atomicMin(&where[c], i);
    }
}

__global__ void max_abs_kernel(int32_t n, const double* __restrict__ V, int first_col, int ncol,
                               unsigned long long* __restrict__ out) {
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < int64_t(n) * ncol; t += int64_t(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(t / n);
        const int32_t i = static_cast<int32_t>(t % n);
        const double a = fabs(V[static_cast<size_t>(first_col + c) * n + i]);
        atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(a)));
    }
}

template <typename T>
__global__ void write_embedding_kernel(int32_t n, int num_dim, const double* __restrict__ U, const double* __restrict__ sign,
                                       double expansion, T* __restrict__ Y) {
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < int64_t(n) * num_dim; t += int64_t(gridDim.x) * blockDim.x) {
        const int32_t c = static_cast<int32_t>(t / num_dim);
        const int d = static_cast<int>(t % num_dim);
        Y[t] = static_cast<T>(U[static_cast<size_t>(d + 1) * n + c] * sign[d + 1] * expansion);
    }
}

template <typename T>
__global__ void jitter_kernel(size_t ntotal, T* __restrict__ Y, double sd, uint32_t k0, uint32_t k1) {
    const size_t npairs = (ntotal + 1) / 2;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < npairs; i += size_t(gridDim.x) * blockDim.x) {
        const Philox4 r = philox4x32_10(static_cast<uint32_t>(i), static_cast<uint32_t>(i >> 32), 0, 0, k0, k1);
        double u1 = u64_to_unit_double(r.v[0], r.v[1]);
        const double u2 = u64_to_unit_double(r.v[2], r.v[3]);
        if (u1 <= 0) u1 = 1.0 / 9007199254740992.0;
        const double rad = sqrt(-2.0 * log(u1));
        const double th = 6.283185307179586476925286766559 * u2;
        Y[2 * i] = static_cast<T>(static_cast<double>(Y[2 * i]) + rad * cos(th) * sd);
        if (2 * i + 1 < ntotal) Y[2 * i + 1] = static_cast<T>(static_cast<double>(Y[2 * i + 1]) + rad * sin(th) * sd);
    }
}

template <typename T>
__global__ void random_init_kernel(size_t ntotal, T* __restrict__ Y, T mult, T shift, uint32_t k0, uint32_t k1) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < ntotal; i += size_t(gridDim.x) * blockDim.x) {
        const Philox4 r = philox4x32_10(static_cast<uint32_t>(i), static_cast<uint32_t>(i >> 32), 0, 0, k0, k1);
        T u;
        if constexpr (std::is_same<T, float>::value) {
            u = u32_to_unit_float(r.v[0]);
        } else {
            u = u64_to_unit_double(r.v[0], r.v[1]);
        }
        Y[i] = u * mult - shift;   // (-scale, scale), spectral_init.hpp:217-223
    }
}

// Cyclic Jacobi for a symmetric m x m matrix (row-major, destroyed): evals in
// decreasing order, evecs row-major with column i = eigenvector i.
void jacobi_eigen(int m, std::vector<double>& A, std::vector<double>& evals, std::vector<double>& evecs) {
    std::vector<double> V(static_cast<size_t>(m) * m, 0.0);
    for (int i = 0; i < m; ++i) V[i * m + i] = 1;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0, total = 0;
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                const double a = A[i * m + j] * A[i * m + j];
                total += a;
                if (i != j) off += a;
            }
        if (off == 0 || off <= 1e-30 * total) break;
        for (int p = 0; p < m; ++p) {
            for (int q = p + 1; q < m; ++q) {
                const double apq = A[p * m + q];
                if (apq == 0) continue;
                const double theta = (A[q * m + q] - A[p * m + p]) / (2 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                const double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < m; ++k) {
                    const double akp = A[k * m + p], akq = A[k * m + q];
                    A[k * m + p] = c * akp - s * akq;
                    A[k * m + q] = s * akp + c * akq;
                }
                for (int k = 0; k < m; ++k) {
                    const double apk = A[p * m + k], aqk = A[q * m + k];
                    A[p * m + k] = c * apk - s * aqk;
                    A[q * m + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < m; ++k) {
                    const double vkp = V[k * m + p], vkq = V[k * m + q];
                    V[k * m + p] = c * vkp - s * vkq;
                    V[k * m + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    std::vector<int> order(m);
    for (int i = 0; i < m; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return A[x * m + x] > A[y * m + y]; });
    evals.assign(m, 0);
    evecs.assign(static_cast<size_t>(m) * m, 0);
    for (int i = 0; i < m; ++i) {
        evals[i] = A[order[i] * m + order[i]];
        for (int k = 0; k < m; ++k) evecs[k * m + i] = V[k * m + order[i]];
    }
}

// Lanczos workspace and primitive steps on the device.
struct LanczosDevice {
    int32_t n;
    int ncv;
    cudaStream_t s;
    const int64_t* ptr;
    const int32_t* idx;
    const double* lap;
    DevArray<double> V, h, hsum, partial, tmp;
    int nblk;

    LanczosDevice(int32_t n_, int ncv_, const int64_t* p, const int32_t* i, const double* l, cudaStream_t st)
        : n(n_), ncv(ncv_), s(st), ptr(p), idx(i), lap(l) {
        V.allocate(static_cast<size_t>(n) * (ncv + 1), s);
        h.allocate(ncv + 2, s);
        hsum.allocate(ncv + 2, s);
        nblk = static_cast<int>(std::min<int64_t>((n + 1023) / 1024, 256));
        partial.allocate(static_cast<size_t>(nblk) * (ncv + 2), s);
        tmp.allocate(static_cast<size_t>(n) * (ncv + 1), s);
    }
    double* col(int c) const { return V.get() + static_cast<size_t>(c) * n; }

    void matvec(const double* x, double* y) {
        lap_spmv_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, ptr, idx, lap, x, y);
        UMAPB_LAUNCH_CHECK();
    }
    // two-pass classical Gram-Schmidt of w against columns [0, ncol); hsum gets the coefficients
    void reorth(double* w, int ncol) {
        UMAPB_CUDA(cudaMemsetAsync(hsum.get(), 0, sizeof(double) * (ncv + 2), s));
        for (int pass = 0; pass < 2; ++pass) {
            multi_dot_kernel<<<dim3(nblk, ncol), DOT_BLOCK, 0, s>>>(n, V.get(), ncol, w, partial.get());
            UMAPB_LAUNCH_CHECK();
            reduce_partials_kernel<<<1, 128, 0, s>>>(nblk, ncol, partial.get(), h.get(), hsum.get());
            UMAPB_LAUNCH_CHECK();
            subtract_projection_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, V.get(), ncol, h.get(), w);
            UMAPB_LAUNCH_CHECK();
        }
    }
    double norm(const double* w) {
        multi_dot_kernel<<<dim3(nblk, 1), DOT_BLOCK, 0, s>>>(n, w, 1, w, partial.get());
        UMAPB_LAUNCH_CHECK();
        reduce_partials_kernel<<<1, 32, 0, s>>>(nblk, 1, partial.get(), h.get(), nullptr);
        UMAPB_LAUNCH_CHECK();
        double v = 0;
        UMAPB_CUDA(cudaMemcpyAsync(&v, h.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);
        return std::sqrt(v);
    }
    void scale(const double* x, double f, double* y) {
        scale_vector_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, x, f, y);
        UMAPB_LAUNCH_CHECK();
    }
    double hsum_at(int c) {
        double v = 0;
        UMAPB_CUDA(cudaMemcpyAsync(&v, hsum.get() + c, sizeof(double), cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);
        return v;
    }
};

}  // namespace

template <typename T>
SpectralResult spectral_init(int32_t n, const int64_t* ptr, const int32_t* idx, const T* w, int num_dim, T* Y,
                             int extra_work, int max_iterations, double tol, double scale, bool jitter,
                             double jitter_sd, uint64_t seed, int* d_status, cudaStream_t s) {
    SpectralResult res;
    const int nev = num_dim + 1;
    require(num_dim >= 1 && nev <= 63, "num_dim must be between 1 and 62 for spectral initialisation");
    if (n <= 0 || nev > n) return res;
    if (count_components(n, ptr, idx, d_status, s) > 1) return res;     // :182-184

    int64_t nnz = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&nnz, ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    DevArray<double> sums(n, s), lap(std::max<int64_t>(nnz, 1), s);
    degree_sqrt_kernel<T><<<grid_for(n, 256), 256, 0, s>>>(n, ptr, w, sums.get());
    UMAPB_LAUNCH_CHECK();
    laplacian_values_kernel<T><<<grid_for(n, 256), 256, 0, s>>>(n, ptr, idx, w, sums.get(), lap.get());
    UMAPB_LAUNCH_CHECK();

    int ncv = nev + std::max(extra_work, nev) + 8;
    if (ncv > n) ncv = n;
    if (ncv > 64) ncv = 64;
    LanczosDevice L(n, ncv, ptr, idx, lap.get(), s);
    const uint64_t start_seed = 5489u;
    start_vector_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, start_seed, L.col(0));
    UMAPB_LAUNCH_CHECK();
    {
        const double nrm = L.norm(L.col(0));
        L.scale(L.col(0), 1.0 / nrm, L.col(0));
    }

    std::vector<double> T_(static_cast<size_t>(ncv) * ncv, 0.0), Tc, theta, S;
    int k = 0;
    double beta_last = 0;
    bool converged = false;
    std::vector<double> Sdev_host;
    DevArray<double> Sdev(static_cast<size_t>(ncv) * ncv, s);
    const int restarts = std::max(max_iterations, 1);
    for (int restart = 0; restart < restarts; ++restart) {
        for (int j = k; j < ncv; ++j) {
            double* vj = L.col(j);
            double* wv = L.col(j + 1);
            L.matvec(vj, wv);
            L.reorth(wv, j + 1);
            T_[j * ncv + j] = L.hsum_at(j);
            double beta = L.norm(wv);
            if (!(beta > 1e-12 * (std::fabs(T_[j * ncv + j]) + 1e-300))) {
                // invariant subspace: continue from a fresh direction orthogonal to the basis
                start_vector_kernel<<<grid_for(n, 256), 256, 0, s>>>(
                    n, start_seed + 7919u * static_cast<uint64_t>(j + 1) + 104729u * static_cast<uint64_t>(restart), wv);
                UMAPB_LAUNCH_CHECK();
                L.reorth(wv, j + 1);
                const double nrm = L.norm(wv);
                L.scale(wv, nrm > 0 ? 1.0 / nrm : 0.0, wv);   // a full basis leaves nothing to add
                beta = 0;
            } else {
                L.scale(wv, 1.0 / beta, wv);
            }
            if (j + 1 < ncv) {
                T_[j * ncv + j + 1] = beta;
                T_[(j + 1) * ncv + j] = beta;
            }
            beta_last = beta;
        }
        Tc = T_;
        jacobi_eigen(ncv, Tc, theta, S);
        const double tscale = std::fabs(theta[0]) > 0 ? std::fabs(theta[0]) : 1;
        bool ok = true;
        for (int i = 0; i < nev; ++i) {
            if (std::fabs(beta_last * S[(ncv - 1) * ncv + i]) > tol * tscale) ok = false;
        }
        // with a full basis (ncv == n) the projection is exact
        if (ncv == n) ok = true;
        res.restarts = restart + 1;
        const bool last = ok || restart == restarts - 1;
        int keep = last ? nev : nev + (ncv - nev) / 2;
        keep = std::min(keep, ncv - 1);
        if (keep < nev) keep = nev;
        UMAPB_CUDA(cudaMemcpyAsync(Sdev.get(), S.data(), sizeof(double) * S.size(), cudaMemcpyHostToDevice, s));
        ritz_vectors_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, L.V.get(), ncv, Sdev.get(), ncv, keep, L.tmp.get());
        UMAPB_LAUNCH_CHECK();
        if (last) {
            converged = ok;
            for (int c = 0; c < nev && c < 64; ++c) res.evals[c] = theta[c];
            break;
        }
        // thick restart: Ritz vectors first, then the residual direction
        UMAPB_CUDA(cudaMemcpyAsync(L.col(keep), L.col(ncv), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        UMAPB_CUDA(cudaMemcpyAsync(L.V.get(), L.tmp.get(), sizeof(double) * n * keep, cudaMemcpyDeviceToDevice, s));
        std::fill(T_.begin(), T_.end(), 0.0);
        for (int c = 0; c < keep; ++c) {
            T_[c * ncv + c] = theta[c];
            const double coupling = beta_last * S[(ncv - 1) * ncv + c];
            T_[c * ncv + keep] = coupling;
            T_[keep * ncv + c] = coupling;
        }
        k = keep;
    }
    if (!converged) return res;   // :123-125

    // normalise and sign the nev Ritz vectors (in L.tmp)
    std::vector<double> sign(nev, 1.0);
    {
        DevArray<unsigned long long> best(nev, s);
        DevArray<int> where(nev, s);
        best.zero(s);
        UMAPB_CUDA(cudaMemsetAsync(where.get(), 0x7f, sizeof(int) * nev, s));
        for (int c = 0; c < nev; ++c) {
            const double nrm = L.norm(L.tmp.get() + static_cast<size_t>(c) * n);
            L.scale(L.tmp.get() + static_cast<size_t>(c) * n, 1.0 / nrm, L.tmp.get() + static_cast<size_t>(c) * n);
        }
        col_max_abs_kernel<<<dim3(grid_for(n, 256, 1024), nev), 256, 0, s>>>(n, L.tmp.get(), best.get());
        UMAPB_LAUNCH_CHECK();
        col_first_at_kernel<<<dim3(grid_for(n, 256, 1024), nev), 256, 0, s>>>(n, L.tmp.get(), best.get(), where.get());
        UMAPB_LAUNCH_CHECK();
        std::vector<int> hw(nev);
        UMAPB_CUDA(cudaMemcpyAsync(hw.data(), where.get(), sizeof(int) * nev, cudaMemcpyDeviceToHost, s));
        UMAPB_SYNC(s);
        for (int c = 0; c < nev; ++c) {
            const int32_t i = (hw[c] >= 0 && hw[c] < n) ? hw[c] : 0;
            double v = 0;
            UMAPB_CUDA(cudaMemcpyAsync(&v, L.tmp.get() + static_cast<size_t>(c) * n + i, sizeof(double),
                                       cudaMemcpyDeviceToHost, s));
            UMAPB_SYNC(s);
            sign[c] = (v < 0) ? -1.0 : 1.0;
        }
    }
    // scale to max |value| = scale over the kept columns (:128-131)
    DevArray<unsigned long long> mx(1, s);
    mx.zero(s);
    max_abs_kernel<<<grid_for(static_cast<size_t>(n) * num_dim, 256), 256, 0, s>>>(n, L.tmp.get(), 1, num_dim, mx.get());
    UMAPB_LAUNCH_CHECK();
    unsigned long long mbits = 0;
    UMAPB_CUDA(cudaMemcpyAsync(&mbits, mx.get(), sizeof(mbits), cudaMemcpyDeviceToHost, s));
    UMAPB_SYNC(s);
    double max_val;
    std::memcpy(&max_val, &mbits, sizeof(double));
    const double expansion = (max_val > 0 ? scale / max_val : 1);
    DevArray<double> dsign(nev, s);
    UMAPB_CUDA(cudaMemcpyAsync(dsign.get(), sign.data(), sizeof(double) * nev, cudaMemcpyHostToDevice, s));
    write_embedding_kernel<T><<<grid_for(static_cast<size_t>(n) * num_dim, 256), 256, 0, s>>>(
        n, num_dim, L.tmp.get(), dsign.get(), expansion, Y);
    UMAPB_LAUNCH_CHECK();
    if (jitter) {
        const size_t ntotal = static_cast<size_t>(n) * num_dim;
        jitter_kernel<T><<<grid_for((ntotal + 1) / 2, 256), 256, 0, s>>>(
            ntotal, Y, jitter_sd, static_cast<uint32_t>(seed) ^ RNG_JITTER, static_cast<uint32_t>(seed >> 32));
        UMAPB_LAUNCH_CHECK();
    }
    UMAPB_SYNC(s);
    res.ok = true;
    return res;
}

template <typename T>
void random_init(int32_t n, int num_dim, T* Y, uint64_t seed, double scale, cudaStream_t s) {
    const size_t ntotal = static_cast<size_t>(n) * num_dim;
    if (ntotal == 0) return;
    random_init_kernel<T><<<grid_for(ntotal, 256), 256, 0, s>>>(ntotal, Y, static_cast<T>(scale * 2),
                                                                static_cast<T>(scale),
                                                                static_cast<uint32_t>(seed) ^ RNG_RANDOM_INIT,
                                                                static_cast<uint32_t>(seed >> 32));
    UMAPB_LAUNCH_CHECK();
}

template SpectralResult spectral_init<float>(int32_t, const int64_t*, const int32_t*, const float*, int, float*, int, int,
                                             double, double, bool, double, uint64_t, int*, cudaStream_t);
template SpectralResult spectral_init<double>(int32_t, const int64_t*, const int32_t*, const double*, int, double*, int,
                                              int, double, double, bool, double, uint64_t, int*, cudaStream_t);
template void random_init<float>(int32_t, int, float*, uint64_t, double, cudaStream_t);
template void random_init<double>(int32_t, int, double*, uint64_t, double, cudaStream_t);

}  // namespace umapb
