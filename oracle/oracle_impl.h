/*
 * Oracle (test infrastructure): C restatement of the reference's UMAP stages,
 * instantiated once per floating-point type by oracle.c (FLOAT = double with
 * SUF = f64, FLOAT = float with SUF = f32).  The arithmetic follows the
 * reference's operation order and types, including its mixed float/double
 * expressions, so that with -ffp-contract=off the results equal the
 * reference compiled the same way.  Only tests, smoke() and the CPU baseline
 * of bench.py may use this code; the product never links it.
 */
#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUF)

/*
 * neighbor_similarities: include/umappp/neighbor_similarities.hpp:53-207.
 * Row i holds ptr[i+1]-ptr[i] distances sorted increasingly; they are replaced
 * in place by membership weights.  rho_out/sigma_out (may be NULL) receive the
 * per-row rho and final sigma (NAN where the reference returns early).
 */
void FN(oracle_neighbor_similarities)(int n, const int64_t* ptr, FLOAT* dist, double local_connectivity, double bandwidth,
                                      double min_k_dist_scale, int use_newton, FLOAT* rho_out, FLOAT* sigma_out) {
    const FLOAT lc = (FLOAT)local_connectivity;
    const FLOAT bw = (FLOAT)bandwidth;
    const FLOAT mkds = (FLOAT)min_k_dist_scale;
    const int raw_connect_index = (int)trunc(lc);                      /* :56 */
    const FLOAT interpolation = lc - (FLOAT)raw_connect_index;         /* :57 */
    int64_t maxk = 0;
    for (int i = 0; i < n; ++i) {
        if (ptr[i + 1] - ptr[i] > maxk) maxk = ptr[i + 1] - ptr[i];
    }
    FLOAT* active = (FLOAT*)malloc(sizeof(FLOAT) * (size_t)(maxk > 0 ? maxk : 1));

    for (int i = 0; i < n; ++i) {
        FLOAT* d = dist + ptr[i];
        const int nnb = (int)(ptr[i + 1] - ptr[i]);
        if (rho_out) rho_out[i] = (FLOAT)NAN;
        if (sigma_out) sigma_out[i] = (FLOAT)NAN;
        if (nnb == 0) {                                                 /* :66-68 */
            continue;
        }
        int num_zero = 0;                                               /* :72-78 */
        for (int k = 0; k < nnb; ++k) {
            if (d[k] != 0) break;
            ++num_zero;
        }
        if (nnb - num_zero <= raw_connect_index) {                      /* :80-88 */
            for (int k = 0; k < nnb; ++k) d[k] = 1;
            continue;
        }
        const int connect_index = num_zero + raw_connect_index;        /* :89-92 */
        const FLOAT lower = connect_index > 0 ? d[connect_index - 1] : (FLOAT)0;
        const FLOAT upper = d[connect_index];
        const FLOAT rho = lower + interpolation * (upper - lower);

        int nactive = 0;                                                /* :95-104 */
        FLOAT num_le_rho = (FLOAT)num_zero;
        for (int k = num_zero; k < nnb; ++k) {
            const FLOAT cur = d[k];
            if (cur > rho) {
                active[nactive++] = cur - rho;
            } else {
                num_le_rho += 1;
            }
        }
        if (rho_out) rho_out[i] = rho;
        if (nactive == 0) {                                             /* :106-112 */
            for (int k = 0; k < nnb; ++k) d[k] = 1;
            continue;
        }

        FLOAT sigma = active[nactive - 1];                              /* :115-121 */
        FLOAT lo = 0;
        const FLOAT max_val = FLOAT_MAX;
        FLOAT hi = max_val;
        const FLOAT target = (FLOAT)(log2((double)(nnb + 1)) * (double)bw); /* :127, std::log2(int) is the double overload */

        for (int iter = 0; iter < 64; ++iter) {                         /* :129-184 */
            FLOAT observed = num_le_rho;
            FLOAT deriv = 0;
            const FLOAT invsigma = (FLOAT)1 / sigma;
            const FLOAT invsigma2 = invsigma * invsigma;
            for (int a = 0; a < nactive; ++a) {
                const FLOAT dd = active[a];
                const FLOAT current = EXP(-dd * invsigma);
                observed += current;
                deriv += dd * current * invsigma2;
            }
            const FLOAT diff = observed - target;
            const FLOAT tol = (FLOAT)1e-5;
            if (FABS(diff) < tol) break;
            if (diff > 0) {
                hi = sigma;
            } else {
                lo = sigma;
            }
            int nr_ok = 0;
            if (use_newton && deriv != 0) {
                const FLOAT alt_sigma = sigma - (diff / deriv);
                if (alt_sigma > lo && alt_sigma < hi) {
                    sigma = alt_sigma;
                    nr_ok = 1;
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

        FLOAT mean_dist = 0;                                            /* :187-192 */
        for (int k = 0; k < nnb; ++k) mean_dist += d[k];
        mean_dist /= (FLOAT)nnb;
        const FLOAT floor_sigma = mkds * mean_dist;
        sigma = (floor_sigma < sigma) ? sigma : floor_sigma;             /* std::max(a, b) == (a < b ? b : a) */
        if (sigma_out) sigma_out[i] = sigma;

        const FLOAT invsigma = (FLOAT)1 / sigma;                        /* :194-202 */
        for (int k = 0; k < nnb; ++k) {
            if (d[k] > rho) {
                d[k] = EXP(-(d[k] - rho) * invsigma);
            } else {
                d[k] = 1;
            }
        }
    }
    free(active);
}

typedef struct {
    int32_t idx;
    FLOAT val;
} FN(oracle_pair);

static int FN(oracle_pair_cmp)(const void* a, const void* b) {
    const FN(oracle_pair)* x = (const FN(oracle_pair)*)a;
    const FN(oracle_pair)* y = (const FN(oracle_pair)*)b;
    if (x->idx != y->idx) return x->idx < y->idx ? -1 : 1;
    if (x->val != y->val) return x->val < y->val ? -1 : 1;
    return 0;
}

/*
 * combine_neighbor_sets: include/umappp/combine_neighbor_sets.hpp:16-99.
 * Input CSR (in_ptr, in_idx, in_w); output CSR with rows sorted by index.
 * The output arrays must hold 2 * in_ptr[n] entries.  Returns the output nnz.
 */
int64_t FN(oracle_combine_neighbor_sets)(int n, const int64_t* in_ptr, const int32_t* in_idx, const FLOAT* in_w, double mix,
                                          int64_t* out_ptr, int32_t* out_idx, FLOAT* out_w) {
    const FLOAT mix_ratio = (FLOAT)mix;
    /* growable rows */
    FN(oracle_pair)** rows = (FN(oracle_pair)**)malloc(sizeof(void*) * (size_t)(n > 0 ? n : 1));
    int64_t* size = (int64_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(int64_t));
    int64_t* cap = (int64_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(int64_t));
    int64_t* last = (int64_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(int64_t));
    int64_t* original = (int64_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(int64_t));
    for (int i = 0; i < n; ++i) {
        const int64_t len = in_ptr[i + 1] - in_ptr[i];
        cap[i] = len * 2 + 4;
        rows[i] = (FN(oracle_pair)*)malloc(sizeof(FN(oracle_pair)) * (size_t)cap[i]);
        for (int64_t p = 0; p < len; ++p) {
            rows[i][p].idx = in_idx[in_ptr[i] + p];
            rows[i][p].val = in_w[in_ptr[i] + p];
        }
        size[i] = len;
        qsort(rows[i], (size_t)len, sizeof(FN(oracle_pair)), FN(oracle_pair_cmp));  /* :21-25 */
        original[i] = len;
    }

    for (int i = 0; i < n; ++i) {                                        /* :27-72 */
        for (int64_t yi = 0; yi < size[i]; ++yi) {   /* size[i] may grow while iterating, as the range-for does */
            FN(oracle_pair)* y = &rows[i][yi];
            const int32_t t = y->idx;
            FN(oracle_pair)* target = rows[t];
            int64_t* curlast = &last[t];
            const int64_t limits = original[t];
            while (*curlast < limits && target[*curlast].idx < i) ++(*curlast);
            if (*curlast < limits && target[*curlast].idx == i) {
                if (i < t) {
                    const FLOAT product = y->val * target[*curlast].val;
                    FLOAT prob_final;
                    if (mix_ratio == 1) {
                        prob_final = y->val + target[*curlast].val - product;
                    } else if (mix_ratio == 0) {
                        prob_final = product;
                    } else {
                        prob_final = mix_ratio * (y->val + target[*curlast].val - product) + (1 - mix_ratio) * product;
                    }
                    y->val = prob_final;
                    target[*curlast].val = prob_final;
                }
            } else {
                if (mix_ratio == 1) {
                    /* append (i, y) to row t */
                    if (size[t] == cap[t]) {
                        cap[t] = cap[t] * 2 + 4;
                        rows[t] = (FN(oracle_pair)*)realloc(rows[t], sizeof(FN(oracle_pair)) * (size_t)cap[t]);
                        if (t == i) y = &rows[i][yi];
                    }
                    rows[t][size[t]].idx = i;
                    rows[t][size[t]].val = y->val;
                    ++size[t];
                } else if (mix_ratio == 0) {
                    y->val = 0;
                } else {
                    y->val *= mix_ratio;
                    if (size[t] == cap[t]) {
                        cap[t] = cap[t] * 2 + 4;
                        rows[t] = (FN(oracle_pair)*)realloc(rows[t], sizeof(FN(oracle_pair)) * (size_t)cap[t]);
                        if (t == i) y = &rows[i][yi];
                    }
                    rows[t][size[t]].idx = i;
                    rows[t][size[t]].val = y->val;
                    ++size[t];
                }
            }
        }
    }

    if (mix_ratio == 0) {                                                /* :75-90 */
        for (int i = 0; i < n; ++i) {
            int64_t counter = 0;
            for (int64_t j = 0; j < size[i]; ++j) {
                if (rows[i][j].val != 0) {
                    rows[i][counter++] = rows[i][j];
                }
            }
            size[i] = counter;
        }
    }

    int64_t total = 0;
    out_ptr[0] = 0;
    for (int i = 0; i < n; ++i) {                                        /* :94-96 */
        qsort(rows[i], (size_t)size[i], sizeof(FN(oracle_pair)), FN(oracle_pair_cmp));
        for (int64_t j = 0; j < size[i]; ++j) {
            out_idx[total] = rows[i][j].idx;
            out_w[total] = rows[i][j].val;
            ++total;
        }
        out_ptr[i + 1] = total;
        free(rows[i]);
    }
    free(rows); free(size); free(cap); free(last); free(original);
    return total;
}

/*
 * similarities_to_epochs: include/umappp/optimize_layout.hpp:47-92.
 * Output arrays must hold ptr[n] entries; returns the kept edge count.
 */
int64_t FN(oracle_similarities_to_epochs)(int n, const int64_t* ptr, const int32_t* idx, const FLOAT* w, int num_epochs, double rate,
                                           int64_t* out_ptr, int32_t* targets, FLOAT* eps, FLOAT* enext, FLOAT* enneg) {
    FLOAT maxed = 0;
    for (int64_t p = 0; p < ptr[n]; ++p) {
        maxed = (maxed < w[p]) ? w[p] : maxed;                           /* std::max */
    }
    const FLOAT limit = maxed / (FLOAT)num_epochs;                       /* :63, Float_ / int */
    int64_t count = 0;
    out_ptr[0] = 0;
    for (int i = 0; i < n; ++i) {
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
            if (w[p] >= limit) {
                targets[count] = idx[p];
                eps[count] = maxed / w[p];                               /* :70 */
                ++count;
            }
        }
        out_ptr[i + 1] = count;
    }
    const FLOAT r = (FLOAT)rate;
    for (int64_t j = 0; j < count; ++j) {                                /* :77-82 */
        enext[j] = eps[j];
        enneg[j] = eps[j] / r;
    }
    return count;
}

/* random_init: include/umappp/spectral_init.hpp:209-225 (engine: mt19937_64(seed)). */
void FN(oracle_random_init)(int n, int num_dim, FLOAT* vals, uint64_t seed, double scale) {
    oracle_mt64 rng;
    oracle_mt64_seed(&rng, seed);
    const FLOAT mult = (FLOAT)(scale * 2);
    const FLOAT shift = (FLOAT)scale;
    const size_t ntotal = (size_t)num_dim * (size_t)n;
    for (size_t i = 0; i < ntotal; ++i) {
        vals[i] = FN(oracle_standard_uniform)(&rng) * mult - shift;
    }
}

/*
 * Serial SGD: include/umappp/optimize_layout.hpp:116-185, with the negative
 * samples drawn from mt19937_64(seed) through the bounded-integer rule of the
 * aarand stand-in.  Advances *current_epoch to epoch_limit and updates
 * enext/enneg and the embedding in place.  counts (may be NULL) receives, per
 * epoch in [*current_epoch, epoch_limit), the number of firing edges and of
 * negative samples drawn (including skipped self-samples) as pairs.
 */
void FN(oracle_optimize_layout)(int num_dim, FLOAT* embedding, int n, const int64_t* ptr, const int32_t* targets, const FLOAT* eps,
                                FLOAT* enext, FLOAT* enneg, double rate, int total_epochs, int* current_epoch,
                                double a_in, double b_in, double gamma_in, double alpha_in, uint64_t seed, int epoch_limit,
                                int64_t* counts) {
    const FLOAT a = (FLOAT)a_in, b = (FLOAT)b_in, gamma = (FLOAT)gamma_in, initial_alpha = (FLOAT)alpha_in;
    const FLOAT negative_sample_rate = (FLOAT)rate;
    const FLOAT dist_eps = FLOAT_EPSILON;
    oracle_mt64 rng;
    oracle_mt64_seed(&rng, seed);
    int e0 = *current_epoch;
    for (int ep = *current_epoch; ep < epoch_limit; ++ep) {
        const FLOAT epoch = (FLOAT)ep;
        const FLOAT alpha = (FLOAT)((double)initial_alpha * (1.0 - (double)(epoch / (FLOAT)total_epochs)));   /* :133 */
        int64_t nfire = 0, nneg_total = 0;
        for (int i = 0; i < n; ++i) {
            FLOAT* left = embedding + (size_t)i * num_dim;
            for (int64_t j = ptr[i]; j < ptr[i + 1]; ++j) {
                if (enext[j] > epoch) continue;                               /* :141-143 */
                ++nfire;
                {
                    FLOAT* right = embedding + (size_t)targets[j] * num_dim;
                    FLOAT dist2 = 0;                                          /* :94-103 */
                    for (int d = 0; d < num_dim; ++d) {
                        const FLOAT delta = left[d] - right[d];
                        dist2 += delta * delta;
                    }
                    dist2 = (dist_eps < dist2) ? dist2 : dist_eps;
                    const FLOAT pd2b = POW(dist2, b);
                    const FLOAT grad_coef = (FLOAT)((double)(-2 * a * b * pd2b) / ((double)dist2 * ((double)(a * pd2b) + 1.0)));  /* :149 */
                    for (int d = 0; d < num_dim; ++d) {
                        FLOAT g = grad_coef * (left[d] - right[d]);
                        g = (g < (FLOAT)-4) ? (FLOAT)-4 : g;                  /* clamp :105-110 */
                        g = ((FLOAT)4 < g) ? (FLOAT)4 : g;
                        const FLOAT gradient = alpha * g;
                        left[d] += gradient;
                        right[d] -= gradient;
                    }
                }
                const FLOAT epns = eps[j] / negative_sample_rate;               /* :160 */
                const int num_neg = (int)((epoch - enneg[j]) / epns);           /* :161 */
                for (int p = 0; p < num_neg; ++p) {
                    const int sampled = (int)oracle_discrete_uniform(&rng, (uint64_t)n);
                    ++nneg_total;
                    if (sampled == i) continue;
                    const FLOAT* right = embedding + (size_t)sampled * num_dim;
                    FLOAT dist2 = 0;
                    for (int d = 0; d < num_dim; ++d) {
                        const FLOAT delta = left[d] - right[d];
                        dist2 += delta * delta;
                    }
                    dist2 = (dist_eps < dist2) ? dist2 : dist_eps;
                    const FLOAT grad_coef = (FLOAT)((double)(2 * gamma * b) / ((0.001 + (double)dist2) * ((double)(a * POW(dist2, b)) + 1.0)));  /* :171 */
                    for (int d = 0; d < num_dim; ++d) {
                        FLOAT g = grad_coef * (left[d] - right[d]);
                        g = (g < (FLOAT)-4) ? (FLOAT)-4 : g;
                        g = ((FLOAT)4 < g) ? (FLOAT)4 : g;
                        left[d] += alpha * g;
                    }
                }
                enext[j] += eps[j];                                              /* :178-179 */
                enneg[j] += (FLOAT)num_neg * epns;
            }
        }
        if (counts) {
            counts[2 * (ep - e0)] = nfire;
            counts[2 * (ep - e0) + 1] = nneg_total;
        }
    }
    if (epoch_limit > *current_epoch) *current_epoch = epoch_limit;
}

/*
 * Transform (no counterpart in the reference: restates the device's
 * umapb_transform): the rows of the transform graph -- new point i's edges to
 * reference points -- are optimised one after another through all epochs
 * with the steps of FN(oracle_optimize_layout) above (optimize_layout.hpp:
 * 141-179), the coefficients written as the device writes them
 * (neg2ab pd2b / (d2 (a pd2b + 1)) and gamma2b / ((0.001 + d2) (a d2^b + 1))),
 * except that only the new point moves and the negative samples are
 * reference points drawn from the device's stream (oracle_negstream, counter
 * (head0 + i, tail, epoch)).  Ynew (nq x num_dim) holds the starting positions
 * and receives the result; enext/enneg are advanced in place.
 */
void FN(oracle_transform_layout)(int num_dim, FLOAT* Ynew, int nq, const int64_t* ptr, const int32_t* targets,
                                 const FLOAT* eps, FLOAT* enext, FLOAT* enneg, double rate, int total_epochs,
                                 const FLOAT* Yref, int nref, int head0, double a_in, double b_in, double gamma_in,
                                 double lr_in, uint64_t seed) {
    const FLOAT a = (FLOAT)a_in, b = (FLOAT)b_in, gamma = (FLOAT)gamma_in, lr = (FLOAT)lr_in;
    const FLOAT negative_sample_rate = (FLOAT)rate;
    const FLOAT dist_eps = FLOAT_EPSILON;
    const FLOAT neg2ab = (FLOAT)-2 * a * b, gamma2b = (FLOAT)2 * gamma * b;
    const uint32_t k0 = (uint32_t)seed ^ ORACLE_RNG_NEGATIVE, k1 = (uint32_t)(seed >> 32);
    for (int i = 0; i < nq; ++i) {
        FLOAT* head = Ynew + (size_t)i * num_dim;
        for (int ep = 0; ep < total_epochs; ++ep) {
            const FLOAT epoch = (FLOAT)ep;
            const FLOAT alpha = (FLOAT)((double)lr * (1.0 - (double)(epoch / (FLOAT)total_epochs)));
            for (int64_t j = ptr[i]; j < ptr[i + 1]; ++j) {
                if (!(enext[j] <= epoch)) continue;
                const FLOAT e_p = eps[j];
                const FLOAT epns = e_p / negative_sample_rate;
                const FLOAT enn = enneg[j];
                const int nn = (int)((epoch - enn) / epns);
                enext[j] = enext[j] + e_p;
                enneg[j] = enn + (FLOAT)nn * epns;
                const FLOAT* yt = Yref + (size_t)targets[j] * num_dim;
                FLOAT d2 = 0;
                for (int d = 0; d < num_dim; ++d) {
                    const FLOAT diff = head[d] - yt[d];
                    d2 += diff * diff;
                }
                d2 = (dist_eps < d2) ? d2 : dist_eps;
                {
                    const FLOAT pd2b = POW(d2, b);
                    const FLOAT c = (neg2ab * pd2b) / (d2 * (a * pd2b + (FLOAT)1));
                    for (int d = 0; d < num_dim; ++d) {
                        FLOAT g = c * (head[d] - yt[d]);
                        g = (g < (FLOAT)-4) ? (FLOAT)-4 : g;
                        g = ((FLOAT)4 < g) ? (FLOAT)4 : g;
                        head[d] += alpha * g;
                    }
                }
                if (nn > 0) {
                    oracle_negstream rs;
                    oracle_negstream_init(&rs, (uint32_t)(head0 + i), (uint32_t)targets[j], (uint32_t)ep, k0, k1);
                    for (int q = 0; q < nn; ++q) {
                        const FLOAT* yk = Yref + (size_t)oracle_negstream_bounded(&rs, (uint32_t)nref) * num_dim;
                        FLOAT dd2 = 0;
                        for (int d = 0; d < num_dim; ++d) {
                            const FLOAT diff = head[d] - yk[d];
                            dd2 += diff * diff;
                        }
                        dd2 = (dist_eps < dd2) ? dd2 : dist_eps;
                        const FLOAT c = gamma2b / (((FLOAT)0.001 + dd2) * (a * POW(dd2, b) + (FLOAT)1));
                        for (int d = 0; d < num_dim; ++d) {
                            FLOAT g = c * (head[d] - yk[d]);
                            g = (g < (FLOAT)-4) ? (FLOAT)-4 : g;
                            g = ((FLOAT)4 < g) ? (FLOAT)4 : g;
                            head[d] += alpha * g;
                        }
                    }
                }
            }
        }
    }
}

/* Matrix-vector product with I + D^-1/2 W D^-1/2, values built as in
 * include/umappp/spectral_init.hpp:38-78 (FP64). */
typedef struct {
    int n;
    const int64_t* ptr;
    const int32_t* idx;
    double* val;   /* off-diagonal values in row order, diagonal implicit (1) */
} FN(oracle_lap);

static void FN(oracle_lap_matvec)(void* ctx, const double* x, double* y) {
    const FN(oracle_lap)* L = (const FN(oracle_lap)*)ctx;
    for (int c = 0; c < L->n; ++c) {
        /* summed in stored order, with the unit diagonal (1 * (-1) + 2) at its
         * sorted position as in the compressed matrix of :60-78 */
        double s = 0;
        int64_t p = L->ptr[c];
        const int64_t e = L->ptr[c + 1];
        for (; p < e && L->idx[p] < c; ++p) s += L->val[p] * x[L->idx[p]];
        s += 1.0 * x[c];
        for (; p < e; ++p) s += L->val[p] * x[L->idx[p]];
        y[c] = s;
    }
}

/* has_multiple_components: include/umappp/spectral_init.hpp:142-168. */
int FN(oracle_has_multiple_components)(int n, const int64_t* ptr, const int32_t* idx) {
    if (n == 0) return 0;
    unsigned char* seen = (unsigned char*)calloc((size_t)n, 1);
    int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int64_t top = 0, in_component = 1;
    stack[top++] = 0;
    seen[0] = 1;
    while (top > 0) {
        const int32_t cur = stack[--top];
        for (int64_t p = ptr[cur]; p < ptr[cur + 1]; ++p) {
            const int32_t f = idx[p];
            if (!seen[f]) {
                seen[f] = 1;
                stack[top++] = f;
                ++in_component;
            }
        }
    }
    free(seen);
    free(stack);
    return in_component != n;
}

/*
 * spectral_init: include/umappp/spectral_init.hpp:171-207 with
 * normalized_laplacian :25-140.  Eigenvectors come from oracle_lanczos (the
 * reference's irlba call, :122).  Returns 1 on success, 0 when the graph has
 * several components or the eigensolver did not converge.  evals_out (may be
 * NULL) receives the num_dim + 1 eigenvalues.
 */
int FN(oracle_spectral_init)(int n, const int64_t* ptr, const int32_t* idx, const FLOAT* w, int num_dim, FLOAT* Y,
                             int ncv, int max_restarts, double tol, double scale, int jitter, double jitter_sd,
                             uint64_t seed, double* evals_out) {
    if (FN(oracle_has_multiple_components)(n, ptr, idx)) return 0;
    double* sums = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int c = 0; c < n; ++c) {                                         /* :38-50 */
        double s = 0;
        for (int64_t p = ptr[c]; p < ptr[c + 1]; ++p) s += (double)w[p];
        sums[c] = sqrt(s);
    }
    double* val = (double*)malloc(sizeof(double) * (size_t)(ptr[n] > 0 ? ptr[n] : 1));
    for (int c = 0; c < n; ++c) {                                         /* :60-78 */
        for (int64_t p = ptr[c]; p < ptr[c + 1]; ++p) {
            val[p] = -(double)w[p] / sums[idx[p]] / sums[c] * (-1);
        }
    }
    FN(oracle_lap) L = {n, ptr, idx, val};
    const int nev = num_dim + 1;
    double* ev = (double*)malloc(sizeof(double) * nev);
    double* U = (double*)malloc(sizeof(double) * (size_t)n * nev);
    int restarts = 0;
    if (ncv <= 0) ncv = nev + (7 > nev ? 7 : nev) + 8;
    const int ok = oracle_lanczos(n, nev, ncv, max_restarts, tol, 5489u, FN(oracle_lap_matvec), &L, ev, U, &restarts);
    if (evals_out) {
        for (int c = 0; c < nev; ++c) evals_out[c] = ev[c];
    }
    if (ok) {
        double mn = INFINITY, mx = -INFINITY;                             /* :126-131 */
        for (int d = 0; d < num_dim; ++d) {
            for (int c = 0; c < n; ++c) {
                const double v = U[(size_t)(d + 1) * n + c];
                mn = v < mn ? v : mn;
                mx = v > mx ? v : mx;
            }
        }
        const double max_val = fabs(mn) > fabs(mx) ? fabs(mn) : fabs(mx);
        const double expansion = max_val > 0 ? scale / max_val : 1;
        for (int c = 0; c < n; ++c) {                                     /* :133-137 */
            for (int d = 0; d < num_dim; ++d) {
                Y[(size_t)c * num_dim + d] = (FLOAT)(U[(size_t)(d + 1) * n + c] * expansion);
            }
        }
        if (jitter) {                                                     /* :190-204 */
            oracle_mt64 rng;
            oracle_mt64_seed(&rng, seed);
            const size_t ntotal = (size_t)num_dim * (size_t)n;
            const size_t half = ntotal / 2;
            for (size_t i = 0; i < half; ++i) {
                double z1, z2;
                oracle_standard_normal(&rng, &z1, &z2);
                Y[2 * i] = (FLOAT)((double)Y[2 * i] + z1 * jitter_sd);
                Y[2 * i + 1] = (FLOAT)((double)Y[2 * i + 1] + z2 * jitter_sd);
            }
            if (ntotal % 2 == 1) {
                double z1, z2;
                oracle_standard_normal(&rng, &z1, &z2);
                Y[ntotal - 1] = (FLOAT)((double)Y[ntotal - 1] + z1 * jitter_sd);
            }
        }
    }
    free(sums); free(val); free(ev); free(U);
    return ok;
}

#undef FN
#undef CAT
#undef CAT2
