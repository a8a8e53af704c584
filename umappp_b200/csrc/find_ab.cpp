// Host-side scalar stages (FP64, microseconds; no device work is worth a launch):
//  - find_ab (include/umappp/find_ab.hpp:44-168): least-squares fit of
//    1 / (1 + a x^(2b)) to min(1, exp(-(x - min_dist) / spread)) on 300 grid
//    points by Gauss-Newton with Levenberg-Marquardt damping, in the
//    reference's operation order (compiled with -ffp-contract=off) so a and b
//    come out bit-identical;
//  - choose_num_epochs (include/umappp/initialize.hpp:27-47).
#include <cfloat>
#include <cmath>
#include <vector>

#include "stages.cuh"

namespace umapb {

void find_ab(double spread, double min_dist, double* a_out, double* b_out) {
    constexpr int grid = 300;
    std::vector<double> gx(grid), gy(grid), lx(grid), fit(grid), xpow(grid), resid(grid);
    const double delta = spread * 3 / grid;
    for (int g = 0; g < grid; ++g) {
        gx[g] = (g + 1) * delta;
        lx[g] = std::log(gx[g]);
        gy[g] = (gx[g] <= min_dist ? 1 : std::exp(-(gx[g] - min_dist) / spread));
    }
    constexpr double limit = 0.5;
    const double x_half = std::log(limit) * -spread + min_dist;
    const double d_half = limit / -spread;
    double b = -d_half * x_half / (1 / limit - 1) / (2 * limit * limit);
    double a = (1 / limit - 1) / std::pow(x_half, 2 * b);

    auto sum_squares = [&](double A, double B) {
        double ss = 0;
        for (int g = 0; g < grid; ++g) {
            xpow[g] = std::pow(gx[g], 2 * B);
            fit[g] = 1 / (1 + A * xpow[g]);
            resid[g] = gy[g] - fit[g];
            ss += resid[g] * resid[g];
        }
        return ss;
    };
    double ss = sum_squares(a, b);
    double damp = 0;
    for (int it = 0; it < 50; ++it) {
        double da2 = 0, db2 = 0, dadb = 0, da_r = 0, db_r = 0;
        for (int g = 0; g < grid; ++g) {
            const double da = xpow[g] * fit[g] * fit[g];
            const double db = a * (lx[g] * 2) * da;
            da2 += da * da;
            db2 += db * db;
            dadb += da * db;
            da_r += da * resid[g];
            db_r += db * resid[g];
        }
        bool okay = false;
        double ca = 0, cb = 0, ss_next = 0;
        while (damp < 1024) {
            const double mult = 1 + damp;
            const double dda2 = da2 * mult, ddb2 = db2 * mult;
            const double det = dda2 * ddb2 - dadb * dadb;
            const double delta_a = -(da_r * ddb2 - dadb * db_r) / det;
            const double delta_b = -(-da_r * dadb + dda2 * db_r) / det;
            ca = a + delta_a;
            cb = b + delta_b;
            ss_next = sum_squares(ca, cb);
            if (ss_next < ss) {
                okay = true;
                damp /= 2;
                break;
            }
            damp = (damp == 0) ? DBL_EPSILON : damp * 2;
        }
        if (!okay) break;
        if (ss - ss_next <= ss * 1e-6) break;
        a = ca;
        b = cb;
        ss = ss_next;
    }
    *a_out = a;
    *b_out = b;
}

int choose_num_epochs(bool has_value, int value, int64_t n) {
    if (has_value) return value;
    constexpr int64_t limit = 10000;
    if (n <= limit) return 500;
    return 200 + static_cast<int>(std::ceil(300 * static_cast<double>(limit) / static_cast<double>(n)));
}

}  // namespace umapb
