/*
 * Oracle (test infrastructure, never part of the product): a plain-C
 * restatement of the reference UMAP pipeline (libscran/umappp v3.3.2,
 * include/umappp/*.hpp) for checking the CUDA path.  Built by oracle/Makefile
 * into oracle/liboracle.so with -O2 -ffp-contract=off.  Only tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py may load it.
 *
 * Contents:
 *  - mt19937_64 (Matsumoto and Nishimura's published 64-bit Mersenne
 *    Twister, the engine the reference names at include/umappp/Options.hpp:32)
 *    and the distributions of the aarand stand-in in ref_shim/aarand;
 *  - the stages of the pipeline, per float type (oracle_impl.h);
 *  - an exact FP64 brute-force kNN (the knncolle search the reference calls
 *    at include/umappp/initialize.hpp:140), trustworthiness, the fuzzy
 *    cross-entropy and its gradient with respect to Y, a and b.
 *
 * Parity pinning: the stage functions are checked against the reference
 * headers compiled in oracle/_ref (same stand-ins) and against the known
 * answers of the reference's tests (tests/src/*.cpp); see tests/test_oracle.py.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "lanczos.h"

/* ---------------------------------------------------------------- RNG --- */

typedef struct {
    uint64_t mt[312];
    int mti;
} oracle_mt64;

void oracle_mt64_seed(oracle_mt64* s, uint64_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 312; ++i) {
        s->mt[i] = 6364136223846793005ULL * (s->mt[i - 1] ^ (s->mt[i - 1] >> 62)) + (uint64_t)i;
    }
    s->mti = 312;
}

uint64_t oracle_mt64_next(oracle_mt64* s) {
    static const uint64_t mag01[2] = {0ULL, 0xB5026F5AA96619E9ULL};
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
    if (s->mti >= 312) {
        int i;
        for (i = 0; i < 312 - 156; ++i) {
            const uint64_t x = (s->mt[i] & UM) | (s->mt[i + 1] & LM);
            s->mt[i] = s->mt[i + 156] ^ (x >> 1) ^ mag01[(int)(x & 1ULL)];
        }
        for (; i < 311; ++i) {
            const uint64_t x = (s->mt[i] & UM) | (s->mt[i + 1] & LM);
            s->mt[i] = s->mt[i + (156 - 312)] ^ (x >> 1) ^ mag01[(int)(x & 1ULL)];
        }
        const uint64_t x = (s->mt[311] & UM) | (s->mt[0] & LM);
        s->mt[311] = s->mt[155] ^ (x >> 1) ^ mag01[(int)(x & 1ULL)];
        s->mti = 0;
    }
    uint64_t x = s->mt[s->mti++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= (x >> 43);
    return x;
}

/* Same rules as ref_shim/aarand/aarand.hpp. */
double oracle_standard_uniform_f64(oracle_mt64* s) {
    while (1) {
        const double u = (double)(oracle_mt64_next(s) >> 11) * 0x1.0p-53;
        if (u < 1.0) return u;
    }
}

float oracle_standard_uniform_f32(oracle_mt64* s) {
    while (1) {
        const double u = (double)(oracle_mt64_next(s) >> 11) * 0x1.0p-53;
        const float out = (float)u;
        if (out < 1.0f) return out;
    }
}

uint64_t oracle_discrete_uniform(oracle_mt64* s, uint64_t bound) {
    const uint64_t limit = UINT64_MAX - (UINT64_MAX % bound + 1) % bound;
    while (1) {
        const uint64_t r = oracle_mt64_next(s);
        if (r <= limit) return r % bound;
    }
}

void oracle_standard_normal(oracle_mt64* s, double* z1, double* z2) {
    const double two_pi = 6.283185307179586476925286766559;
    double u1;
    do {
        u1 = oracle_standard_uniform_f64(s);
    } while (u1 == 0);
    const double u2 = oracle_standard_uniform_f64(s);
    const double r = sqrt(-2.0 * log(u1));
    const double theta = two_pi * u2;
    *z1 = r * cos(theta);
    *z2 = r * sin(theta);
}

/* Draws 'count' values of the engine seeded with 'seed' (for pinning the engine). */
void oracle_mt64_stream(uint64_t seed, int64_t count, uint64_t* out) {
    oracle_mt64 s;
    oracle_mt64_seed(&s, seed);
    for (int64_t i = 0; i < count; ++i) out[i] = oracle_mt64_next(&s);
}

/*
 * The device's negative-sample stream (restated for the transform oracle):
 * Philox4x32 with 7 rounds (Salmon, Moraes, Dror and Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC 2011; multipliers 0xD2511F53 and
 * 0xCD9E8D57, key increments 0x9E3779B9 and 0xBB67AE85), counter (head,
 * tail, epoch, block), key (seed low word ^ stream tag, seed high word);
 * bounded integers by Lemire's multiply-shift with rejection ("Fast random
 * integer generation in an interval", ACM TOMACS 2019).
 */
#define ORACLE_RNG_NEGATIVE 0x4E454731u

typedef struct {
    uint32_t c0, c1, c2, c3, k0, k1;
    uint32_t buf[4];
    int used;
} oracle_negstream;

static void oracle_philox4x32_7(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                                uint32_t out[4]) {
    for (int r = 0; r < 7; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = (uint32_t)p1;
        c2 = n2;
        c3 = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

static void oracle_negstream_init(oracle_negstream* s, uint32_t head, uint32_t tail, uint32_t epoch, uint32_t k0,
                                  uint32_t k1) {
    s->c0 = head;
    s->c1 = tail;
    s->c2 = epoch;
    s->c3 = 0;
    s->k0 = k0;
    s->k1 = k1;
    s->used = 4;
}

static uint32_t oracle_negstream_next(oracle_negstream* s) {
    if (s->used == 4) {
        oracle_philox4x32_7(s->c0, s->c1, s->c2, s->c3++, s->k0, s->k1, s->buf);
        s->used = 0;
    }
    return s->buf[s->used++];
}

static int32_t oracle_negstream_bounded(oracle_negstream* s, uint32_t n) {
    uint64_t m = (uint64_t)oracle_negstream_next(s) * n;
    uint32_t l = (uint32_t)m;
    if (l < n) {
        const uint32_t thr = (0u - n) % n;
        while (l < thr) {
            m = (uint64_t)oracle_negstream_next(s) * n;
            l = (uint32_t)m;
        }
    }
    return (int32_t)(m >> 32);
}

/* 'count' bounded draws of one stream (for pinning the stream). */
void oracle_negstream_draws(uint32_t head, uint32_t tail, uint32_t epoch, uint64_t seed, uint32_t n, int count,
                            int32_t* out) {
    oracle_negstream s;
    oracle_negstream_init(&s, head, tail, epoch, (uint32_t)seed ^ ORACLE_RNG_NEGATIVE, (uint32_t)(seed >> 32));
    for (int i = 0; i < count; ++i) out[i] = oracle_negstream_bounded(&s, n);
}

/* ------------------------------------------------------------- stages --- */

#define FLOAT double
#define SUF f64
#define EXP exp
#define POW pow
#define FABS fabs
#define FLOAT_MAX DBL_MAX
#define FLOAT_EPSILON DBL_EPSILON
#include "oracle_impl.h"
#undef FLOAT
#undef SUF
#undef EXP
#undef POW
#undef FABS
#undef FLOAT_MAX
#undef FLOAT_EPSILON

#define FLOAT float
#define SUF f32
#define EXP expf
#define POW powf
#define FABS fabsf
#define FLOAT_MAX FLT_MAX
#define FLOAT_EPSILON FLT_EPSILON
#include "oracle_impl.h"
#undef FLOAT
#undef SUF
#undef EXP
#undef POW
#undef FABS
#undef FLOAT_MAX
#undef FLOAT_EPSILON

/*
 * find_ab: include/umappp/find_ab.hpp:44-168 (Float_ = double), a 300-point
 * Gauss-Newton fit with Levenberg-Marquardt damping.
 */
void oracle_find_ab(double spread, double min_dist, double* a_out, double* b_out) {
    enum { grid = 300 };
    double grid_x[grid], grid_y[grid], log_x[grid], fit_y[grid], xpow[grid], resid[grid];
    const double delta = spread * 3 / grid;
    for (int g = 0; g < grid; ++g) {
        grid_x[g] = (double)(g + 1) * delta;
        log_x[g] = log(grid_x[g]);
        grid_y[g] = (grid_x[g] <= min_dist ? 1 : exp(-(grid_x[g] - min_dist) / spread));
    }
    const double limit = 0.5;
    const double x_half = log(limit) * -spread + min_dist;
    const double d_half = limit / -spread;
    double b = -d_half * x_half / (1 / limit - 1) / (2 * limit * limit);
    double a = (1 / limit - 1) / pow(x_half, 2 * b);

#define ORACLE_SS(A, B, OUT)                                   \
    do {                                                       \
        double ss_ = 0;                                        \
        for (int g = 0; g < grid; ++g) {                       \
            xpow[g] = pow(grid_x[g], 2 * (B));                 \
            fit_y[g] = 1 / (1 + (A) * xpow[g]);                \
            resid[g] = grid_y[g] - fit_y[g];                   \
            ss_ += resid[g] * resid[g];                        \
        }                                                      \
        (OUT) = ss_;                                           \
    } while (0)

    double ss;
    ORACLE_SS(a, b, ss);
    double lm = 0;
    for (int it = 0; it < 50; ++it) {
        double da2 = 0, db2 = 0, dadb = 0, da_resid = 0, db_resid = 0;
        for (int g = 0; g < grid; ++g) {
            const double x2b = xpow[g];
            const double oy = fit_y[g];
            const double r = resid[g];
            const double da = x2b * oy * oy;
            const double db = a * (log_x[g] * 2) * da;
            da2 += da * da;
            db2 += db * db;
            dadb += da * db;
            da_resid += da * r;
            db_resid += db * r;
        }
        int okay = 0;
        double ca = 0, cb = 0, ss_next = 0;
        const double max_dampener = 1024;
        while (lm < max_dampener) {
            const double mult = 1 + lm;
            const double dda2 = da2 * mult;
            const double ddb2 = db2 * mult;
            const double det = dda2 * ddb2 - dadb * dadb;
            const double delta_a = -(da_resid * ddb2 - dadb * db_resid) / det;
            const double delta_b = -(-da_resid * dadb + dda2 * db_resid) / det;
            ca = a + delta_a;
            cb = b + delta_b;
            ORACLE_SS(ca, cb, ss_next);
            if (ss_next < ss) {
                okay = 1;
                lm /= 2;
                break;
            }
            lm = (lm == 0) ? DBL_EPSILON : lm * 2;
        }
        if (!okay) break;
        if (ss - ss_next <= ss * 1e-6) break;
        a = ca;
        b = cb;
        ss = ss_next;
    }
#undef ORACLE_SS
    *a_out = a;
    *b_out = b;
}

/* choose_num_epochs: include/umappp/initialize.hpp:27-47. */
int oracle_choose_num_epochs(int has_value, int value, int64_t size) {
    if (has_value) return value;
    if (size <= 10000) return 500;
    return 200 + (int)ceil(300 * 10000.0 / (double)size);
}

/* ----------------------------------------------------------------- kNN --- */

typedef struct {
    double d2;
    int32_t j;
} oracle_cand;

static int oracle_cand_less(const oracle_cand* x, const oracle_cand* y) {
    return x->d2 < y->d2 || (x->d2 == y->d2 && x->j < y->j);
}

/*
 * Exact Euclidean kNN in FP64 from coordinate differences, self excluded,
 * sorted by (distance, index).  data: observation i at data[i*dim .. +dim)
 * (column-major with observations as columns, include/umappp/initialize.hpp:150-152).
 * Queries [qstart, qstart + qcount); outputs qcount x k indices and FP64 distances.
 */
void oracle_knn_f64(int n, int dim, const double* data, int k, int qstart, int qcount, int32_t* out_idx, double* out_dist) {
    oracle_cand* best = (oracle_cand*)malloc(sizeof(oracle_cand) * (size_t)(k + 1));
    for (int q = qstart; q < qstart + qcount; ++q) {
        int count = 0;
        const double* xq = data + (size_t)q * dim;
        for (int j = 0; j < n; ++j) {
            if (j == q) continue;
            const double* xj = data + (size_t)j * dim;
            double d2 = 0;
            for (int d = 0; d < dim; ++d) {
                const double diff = xq[d] - xj[d];
                d2 += diff * diff;
            }
            oracle_cand c = {d2, j};
            if (count < k) {
                int pos = count++;
                while (pos > 0 && oracle_cand_less(&c, &best[pos - 1])) {
                    best[pos] = best[pos - 1];
                    --pos;
                }
                best[pos] = c;
            } else if (k > 0 && oracle_cand_less(&c, &best[k - 1])) {
                int pos = k - 1;
                while (pos > 0 && oracle_cand_less(&c, &best[pos - 1])) {
                    best[pos] = best[pos - 1];
                    --pos;
                }
                best[pos] = c;
            }
        }
        for (int t = 0; t < count; ++t) {
            out_idx[(size_t)(q - qstart) * k + t] = best[t].j;
            out_dist[(size_t)(q - qstart) * k + t] = sqrt(best[t].d2);
        }
        for (int t = count; t < k; ++t) {
            out_idx[(size_t)(q - qstart) * k + t] = -1;
            out_dist[(size_t)(q - qstart) * k + t] = INFINITY;
        }
    }
    free(best);
}

/* Queries against a separate reference set: the k nearest of the nref rows of
 * 'ref' to each of the nq rows of 'qd' (FP64 sums in dimension order, ties by
 * index); outputs nq x k. */
void oracle_knn_query_f64(int nref, int nq, int dim, const double* ref, const double* qd, int k, int32_t* out_idx,
                          double* out_dist) {
    oracle_cand* best = (oracle_cand*)malloc(sizeof(oracle_cand) * (size_t)(k + 1));
    for (int q = 0; q < nq; ++q) {
        int count = 0;
        const double* xq = qd + (size_t)q * dim;
        for (int j = 0; j < nref; ++j) {
            const double* xj = ref + (size_t)j * dim;
            double d2 = 0;
            for (int d = 0; d < dim; ++d) {
                const double diff = xq[d] - xj[d];
                d2 += diff * diff;
            }
            oracle_cand c = {d2, j};
            int pos;
            if (count < k) {
                pos = count++;
            } else if (k > 0 && oracle_cand_less(&c, &best[k - 1])) {
                pos = k - 1;
            } else {
                continue;
            }
            while (pos > 0 && oracle_cand_less(&c, &best[pos - 1])) {
                best[pos] = best[pos - 1];
                --pos;
            }
            best[pos] = c;
        }
        for (int t = 0; t < k; ++t) {
            out_idx[(size_t)q * k + t] = t < count ? best[t].j : -1;
            out_dist[(size_t)q * k + t] = t < count ? sqrt(best[t].d2) : INFINITY;
        }
    }
    free(best);
}

/* Same search over float data (the distances are still accumulated in FP64). */
void oracle_knn_f32(int n, int dim, const float* data, int k, int qstart, int qcount, int32_t* out_idx, double* out_dist) {
    double* tmp = (double*)malloc(sizeof(double) * (size_t)n * dim);
    for (size_t i = 0; i < (size_t)n * dim; ++i) tmp[i] = (double)data[i];
    oracle_knn_f64(n, dim, tmp, k, qstart, qcount, out_idx, out_dist);
    free(tmp);
}

/* ----------------------------------------------------- layout quality --- */

static int oracle_dbl_cmp(const void* a, const void* b) {
    const double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

/*
 * Trustworthiness (Venna and Kaski, 2001) of embedding Y (n x dy) against
 * data X (n x dx), evaluated over 'nq' query observations 'queries' with the
 * full data set as candidates:
 *   T = 1 - 2 / (nq k (2n - 3k - 1)) * sum_i sum_{j in N_k^Y(i)} max(0, r(i, j) - k)
 * where r(i, j) is the rank of j among i's neighbours in X (1-based, ties by
 * index).  With nq == n this is the usual definition.
 */
double oracle_trustworthiness(int n, int dx, const double* X, int dy, const double* Y, int k, int nq, const int32_t* queries) {
    double* dX = (double*)malloc(sizeof(double) * (size_t)n);
    oracle_cand* cY = (oracle_cand*)malloc(sizeof(oracle_cand) * (size_t)n);
    double total = 0;
    for (int t = 0; t < nq; ++t) {
        const int i = queries[t];
        for (int j = 0; j < n; ++j) {
            double s = 0;
            for (int d = 0; d < dx; ++d) {
                const double diff = X[(size_t)i * dx + d] - X[(size_t)j * dx + d];
                s += diff * diff;
            }
            dX[j] = s;
            double sy = 0;
            for (int d = 0; d < dy; ++d) {
                const double diff = Y[(size_t)i * dy + d] - Y[(size_t)j * dy + d];
                sy += diff * diff;
            }
            cY[j].d2 = (j == i) ? -1 : sy;
            cY[j].j = j;
        }
        /* k nearest in Y (excluding self, which has d2 = -1 and sorts first) */
        oracle_cand* best = (oracle_cand*)malloc(sizeof(oracle_cand) * (size_t)(k + 1));
        int count = 0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            oracle_cand c = cY[j];
            if (count < k) {
                int pos = count++;
                while (pos > 0 && oracle_cand_less(&c, &best[pos - 1])) { best[pos] = best[pos - 1]; --pos; }
                best[pos] = c;
            } else if (oracle_cand_less(&c, &best[k - 1])) {
                int pos = k - 1;
                while (pos > 0 && oracle_cand_less(&c, &best[pos - 1])) { best[pos] = best[pos - 1]; --pos; }
                best[pos] = c;
            }
        }
        for (int t2 = 0; t2 < count; ++t2) {
            const int j = best[t2].j;
            /* rank of j in X among all points except i: number of points closer, ties by index, plus one */
            int64_t rank = 1;
            const double dj = dX[j];
            for (int m = 0; m < n; ++m) {
                if (m == i || m == j) continue;
                if (dX[m] < dj || (dX[m] == dj && m < j)) ++rank;
            }
            if (rank > k) total += (double)(rank - k);
        }
        free(best);
    }
    free(dX);
    free(cY);
    (void)oracle_dbl_cmp;
    return 1.0 - 2.0 / ((double)nq * k * (2.0 * n - 3.0 * k - 1.0)) * total;
}

/*
 * Fuzzy-set cross-entropy of a layout over the stored (directed) edges of a
 * weighted graph, FP64:
 *   CE = sum_e  w log(w / q) + (1 - w) log((1 - w) / (1 - q)),
 *   q = 1 / (1 + a d2^b),  d2 = |y_i - y_j|^2,
 * with 0 log 0 = 0 and q clipped to [1e-300, 1 - 1e-16] inside the logs.
 * This is the objective whose per-edge derivatives the reference's SGD
 * follows (include/umappp/optimize_layout.hpp:148-149, 171).
 */
double oracle_cross_entropy(int n, const int64_t* ptr, const int32_t* idx, const double* w, int dim, const double* Y, double a, double b) {
    double total = 0;
    for (int i = 0; i < n; ++i) {
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            const int j = idx[p];
            double d2 = 0;
            for (int d = 0; d < dim; ++d) {
                const double diff = Y[(size_t)i * dim + d] - Y[(size_t)j * dim + d];
                d2 += diff * diff;
            }
            double q = 1.0 / (1.0 + a * pow(d2, b));
            if (q < 1e-300) q = 1e-300;
            if (q > 1 - 1e-16) q = 1 - 1e-16;
            const double wij = w[p];
            if (wij > 0) total += wij * log(wij / q);
            if (wij < 1) total += (1 - wij) * log((1 - wij) / (1 - q));
        }
    }
    return total;
}

/*
 * Loss and gradient of the fuzzy cross-entropy (without its w-only constant)
 *   L = sum_e  w * (-log q) + (1 - w) * (-log(1 - q)),  q = 1 / (1 + a d2^b),
 * over the stored edges, FP64, and with eps_rep > 0 the repulsive factor
 * 1/d2 replaced by 1/(d2 + eps_rep) as in the reference's repulsive step
 * (optimize_layout.hpp:171) (then only the gradient is defined, and the loss
 * returned is the exact one).  grad_Y: n x dim; grad_ab: [dL/da, dL/db].
 */
double oracle_loss_grad(int n, const int64_t* ptr, const int32_t* idx, const double* w, int dim, const double* Y,
                        double a, double b, double eps_rep, double* grad_Y, double* grad_ab) {
    double loss = 0, ga = 0, gb = 0;
    memset(grad_Y, 0, sizeof(double) * (size_t)n * dim);
    for (int i = 0; i < n; ++i) {
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            const int j = idx[p];
            double d2 = 0;
            for (int d = 0; d < dim; ++d) {
                const double diff = Y[(size_t)i * dim + d] - Y[(size_t)j * dim + d];
                d2 += diff * diff;
            }
            const double wij = w[p];
            const double pd2b = pow(d2, b);
            const double denom = 1 + a * pd2b;
            /* -log q = log(1 + a d2^b);  -log(1 - q) = log(1 + a d2^b) - log(a) - b log(d2) */
            const double lq = log(denom);
            const double ld2 = log(d2);
            loss += wij * lq + (1 - wij) * (lq - log(a) - b * ld2);
            /* dL/dd2 */
            const double att = a * b * pd2b / (d2 * denom);
            const double rep = -b / ((d2 + eps_rep) * denom);
            const double dd2 = wij * att + (1 - wij) * rep;
            for (int d = 0; d < dim; ++d) {
                const double diff = Y[(size_t)i * dim + d] - Y[(size_t)j * dim + d];
                grad_Y[(size_t)i * dim + d] += 2 * dd2 * diff;
                grad_Y[(size_t)j * dim + d] -= 2 * dd2 * diff;
            }
            /* dL/da, dL/db */
            ga += wij * (pd2b / denom) + (1 - wij) * (-1.0 / (a * denom));
            gb += wij * (a * pd2b * ld2 / denom) + (1 - wij) * (-ld2 / denom);
        }
    }
    grad_ab[0] = ga;
    grad_ab[1] = gb;
    return loss;
}
