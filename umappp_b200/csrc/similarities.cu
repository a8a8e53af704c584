// neighbor_similarities on the device: one thread per observation runs the
// reference's Newton-with-bisection search for sigma in FP64
// (include/umappp/neighbor_similarities.hpp:53-207), following its iterate
// sequence exactly (same start, same bracketing and Newton acceptance rules,
// same tolerance and 64-iteration cap), so that sigma and the weights agree
// with an FP64 evaluation of the reference to rounding.  Compiled with
// -fmad=false so no multiply-add is contracted, as in the reference's
// -ffp-contract=off build.  exp is the correctly rounded exp_cr (exp_cr.cuh),
// and log2(k + 1) comes from the host's libm, so the values track a host
// evaluation to the last bit except where the host's exp itself misrounds.
#include <cfloat>
#include <cmath>

#include "exp_cr.cuh"
#include "stages.cuh"

namespace umapb {

constexpr int LOG2_TABLE = 256;

struct Log2Table {
    double v[LOG2_TABLE];   // v[m] = log2(m + 1)
};

template <typename T>
__global__ void __launch_bounds__(128) similarities_kernel(int32_t n, const int64_t* __restrict__ ptr, T* __restrict__ val,
                                                           int raw_connect_index, double interpolation,
                                                           double bandwidth, double min_k_dist_scale, int use_newton,
                                                           double* __restrict__ rho_out, double* __restrict__ sigma_out,
                                                           const Log2Table log2_tab) {
    const double* log2_table = log2_tab.v;
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t start = ptr[i];
    const int nnb = static_cast<int>(ptr[i + 1] - start);
    T* d = val + start;
    double rho_report = CUDART_NAN, sigma_report = CUDART_NAN;

    if (nnb > 0) {
        int num_zero = 0;                                          // :72-78
        for (int k = 0; k < nnb; ++k) {
            if (d[k] != T(0)) break;
            ++num_zero;
        }
        if (nnb - num_zero <= raw_connect_index) {                 // :80-88
            for (int k = 0; k < nnb; ++k) d[k] = T(1);
        } else {
            const int connect_index = num_zero + raw_connect_index;   // :89-92
            const double lower = connect_index > 0 ? static_cast<double>(d[connect_index - 1]) : 0.0;
            const double upper = static_cast<double>(d[connect_index]);
            const double rho = lower + interpolation * (upper - lower);
            rho_report = rho;

            double num_le_rho = num_zero;                             // :95-104
            int nactive = 0;
            double largest = 0;
            for (int k = num_zero; k < nnb; ++k) {
                const double cur = static_cast<double>(d[k]);
                if (cur > rho) {
                    ++nactive;
                    largest = cur - rho;      // last active delta (rows are sorted)
                } else {
                    num_le_rho += 1;
                }
            }
            if (nactive == 0) {                                       // :106-112
                for (int k = 0; k < nnb; ++k) d[k] = T(1);
            } else {
                double sigma = largest;                               // :115-121
                double lo = 0;
                const double max_val = DBL_MAX;
                double hi = max_val;
                // :127, log2(k + 1) from the host's libm for row lengths up to the table size
                const double target = (nnb < LOG2_TABLE ? log2_table[nnb] : log2(static_cast<double>(nnb + 1))) * bandwidth;

                for (int iter = 0; iter < 64; ++iter) {               // :129-184
                    double observed = num_le_rho;
                    double deriv = 0;
                    const double invsigma = 1.0 / sigma;
                    const double invsigma2 = invsigma * invsigma;
                    for (int k = num_zero; k < nnb; ++k) {
                        const double cur = static_cast<double>(d[k]);
                        if (cur > rho) {
                            const double dd = cur - rho;
                            const double current = exp_cr(-dd * invsigma);
                            observed += current;
                            deriv += dd * current * invsigma2;
                        }
                    }
                    const double diff = observed - target;
                    if (fabs(diff) < 1e-5) break;
                    if (diff > 0) {
                        hi = sigma;
                    } else {
                        lo = sigma;
                    }
                    bool nr_ok = false;
                    if (use_newton && deriv != 0) {
                        const double alt = sigma - (diff / deriv);
                        if (alt > lo && alt < hi) {
                            sigma = alt;
                            nr_ok = true;
                        }
                    }
                    if (!nr_ok) {
                        if (diff > 0) {
                            sigma += (lo - sigma) / 2;
                        } else if (hi == max_val) {
                            sigma *= 2;
                        } else {
                            sigma += (hi - sigma) / 2;
                        }
                    }
                }

                double mean_dist = 0;                                 // :187-192
                for (int k = 0; k < nnb; ++k) mean_dist += static_cast<double>(d[k]);
                mean_dist /= nnb;
                const double floor_sigma = min_k_dist_scale * mean_dist;
                sigma = (floor_sigma < sigma) ? sigma : floor_sigma;
                sigma_report = sigma;

                const double invsigma = 1.0 / sigma;                  // :194-202
                for (int k = 0; k < nnb; ++k) {
                    const double cur = static_cast<double>(d[k]);
                    d[k] = (cur > rho) ? static_cast<T>(exp_cr(-(cur - rho) * invsigma)) : T(1);
                }
            }
        }
    }
    if (rho_out) rho_out[i] = rho_report;
    if (sigma_out) sigma_out[i] = sigma_report;
}

template <typename T>
void neighbor_similarities(int32_t n, const int64_t* ptr, T* val, double local_connectivity, double bandwidth,
                           double min_k_dist_scale, bool use_newton, double* rho_out, double* sigma_out,
                           cudaStream_t s) {
    if (n <= 0) return;
    require(std::isfinite(local_connectivity) && local_connectivity >= 0 && local_connectivity < 2147483647.0,
            "local_connectivity must be a finite non-negative value", UMAPB_ERR_OVERFLOW);
    const int raw = static_cast<int>(std::trunc(local_connectivity));       // :56
    const double interpolation = local_connectivity - raw;                  // :57
    Log2Table tab;
    for (int m = 0; m < LOG2_TABLE; ++m) tab.v[m] = std::log2(static_cast<double>(m + 1));
    const unsigned block = 128;
    similarities_kernel<T><<<(n + block - 1) / block, block, 0, s>>>(n, ptr, val, raw, interpolation, bandwidth,
                                                                      min_k_dist_scale, use_newton ? 1 : 0, rho_out,
                                                                      sigma_out, tab);
    UMAPB_LAUNCH_CHECK();
}

template void neighbor_similarities<float>(int32_t, const int64_t*, float*, double, double, double, bool, double*,
                                           double*, cudaStream_t);
template void neighbor_similarities<double>(int32_t, const int64_t*, double*, double, double, double, bool, double*,
                                            double*, cudaStream_t);

}  // namespace umapb
