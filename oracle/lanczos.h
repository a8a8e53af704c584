/*
 * Oracle (test infrastructure): FP64 thick-restart Lanczos for the largest
 * eigenpairs of a symmetric operator, plus a cyclic Jacobi eigensolver.
 *
 * The reference computes its spectral initialisation with irlba::compute on
 * the shifted normalised Laplacian (include/umappp/spectral_init.hpp:105-126).
 * irlba and Eigen are dependencies the reference fetches at configure time
 * (not vendored with it), so this file restates the
 * published thick-restart Lanczos method (Wu and Simon, SIAM J. Matrix Anal.
 * Appl. 22(2), 2000) for the symmetric positive semi-definite case, where the
 * top singular vectors are the top eigenvectors.  It is shared by the C
 * restatement (oracle.c) and by the irlba stand-in used to compile the
 * reference headers (ref_shim/irlba/irlba.hpp), so both produce the same
 * vectors.  Only tests, smoke() and the CPU baseline of bench.py may use it.
 *
 * Conventions: eigenvalues in decreasing order; each eigenvector has unit
 * norm and is signed so that its entry of largest magnitude (first such
 * entry on ties) is positive.
 */
#ifndef ORACLE_LANCZOS_H
#define ORACLE_LANCZOS_H

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef void (*oracle_matvec_fn)(void* ctx, const double* x, double* y);

/* Cyclic Jacobi on a symmetric m x m matrix A (row-major, destroyed).
 * On return evals[i] (decreasing) and evecs column i (row-major m x m, column
 * i holds eigenvector i). */
static void oracle_jacobi_eigen(int m, double* A, double* evals, double* evecs) {
    double* V = (double*)malloc(sizeof(double) * (size_t)m * m);
    for (int i = 0; i < m; ++i) {
        for (int j = 0; j < m; ++j) {
            V[i * m + j] = (i == j);
        }
    }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0, total = 0;
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < m; ++j) {
                const double a = A[i * m + j] * A[i * m + j];
                total += a;
                if (i != j) {
                    off += a;
                }
            }
        }
        if (off <= 1e-30 * total || off == 0) {
            break;
        }
        for (int p = 0; p < m; ++p) {
            for (int q = p + 1; q < m; ++q) {
                const double apq = A[p * m + q];
                if (apq == 0) {
                    continue;
                }
                const double app = A[p * m + p], aqq = A[q * m + q];
                const double theta = (aqq - app) / (2 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
                const double c = 1 / sqrt(t * t + 1), s = t * c;
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
    /* sort decreasing (selection sort, m is small) */
    int* order = (int*)malloc(sizeof(int) * m);
    for (int i = 0; i < m; ++i) {
        order[i] = i;
    }
    for (int i = 0; i < m; ++i) {
        int best = i;
        for (int j = i + 1; j < m; ++j) {
            if (A[order[j] * m + order[j]] > A[order[best] * m + order[best]]) {
                best = j;
            }
        }
        const int tmp = order[i];
        order[i] = order[best];
        order[best] = tmp;
    }
    for (int i = 0; i < m; ++i) {
        evals[i] = A[order[i] * m + order[i]];
        for (int k = 0; k < m; ++k) {
            evecs[k * m + i] = V[k * m + order[i]];
        }
    }
    free(order);
    free(V);
}

static void oracle_fix_sign(int64_t n, double* v) {
    int64_t best = 0;
    for (int64_t i = 1; i < n; ++i) {
        if (fabs(v[i]) > fabs(v[best])) {
            best = i;
        }
    }
    if (v[best] < 0) {
        for (int64_t i = 0; i < n; ++i) {
            v[i] = -v[i];
        }
    }
}

/* Deterministic start vector: splitmix64 stream mapped to [-0.5, 0.5). */
static void oracle_start_vector(int64_t n, uint64_t seed, double* v) {
    uint64_t state = seed;
    for (int64_t i = 0; i < n; ++i) {
        state += 0x9E3779B97F4A7C15ULL;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        v[i] = (double)(z >> 11) * 0x1.0p-53 - 0.5;
    }
}

/* Gram-Schmidt of w against columns 0..ncol-1 of V (column-major, leading
 * dimension n), two classical passes.  Adds the coefficients into h. */
static void oracle_reorth(int64_t n, int ncol, const double* V, double* w, double* h) {
    double* hh = (double*)malloc(sizeof(double) * (size_t)(ncol > 0 ? ncol : 1));
    for (int pass = 0; pass < 2; ++pass) {
        /* all projections of this pass first, then the subtraction (classical GS) */
        for (int c = 0; c < ncol; ++c) {
            const double* vc = V + (size_t)c * n;
            double dot = 0;
            for (int64_t i = 0; i < n; ++i) {
                dot += vc[i] * w[i];
            }
            hh[c] = dot;
        }
        for (int c = 0; c < ncol; ++c) {
            h[c] += hh[c];
            const double* vc = V + (size_t)c * n;
            for (int64_t i = 0; i < n; ++i) {
                w[i] -= hh[c] * vc[i];
            }
        }
    }
    free(hh);
}

static double oracle_norm(int64_t n, const double* w) {
    double s = 0;
    for (int64_t i = 0; i < n; ++i) {
        s += w[i] * w[i];
    }
    return sqrt(s);
}

/*
 * Largest 'nev' eigenpairs of the symmetric operator 'mv' of order n.
 * ncv: Krylov basis size (clamped to [nev + 2, n]); max_restarts: restart
 * cap; tol: a Ritz pair is converged when its residual norm is at most
 * tol * |largest Ritz value|.  Writes evals[nev] and evecs (n x nev,
 * column-major).  Returns 1 when converged, 0 otherwise.
 * For n <= ncv the operator is materialised and solved densely (exact).
 */
static int oracle_lanczos(int64_t n, int nev, int ncv, int max_restarts, double tol, uint64_t seed,
                          oracle_matvec_fn mv, void* ctx, double* evals, double* evecs, int* restarts_out) {
    if (restarts_out) {
        *restarts_out = 0;
    }
    if (nev <= 0 || n <= 0 || nev > n) {
        return 0;
    }
    if (ncv < nev + 2) {
        ncv = nev + 2;
    }
    if (n <= ncv) {
        const int m = (int)n;
        double* A = (double*)malloc(sizeof(double) * (size_t)m * m);
        double* e = (double*)calloc((size_t)m, sizeof(double));
        double* col = (double*)malloc(sizeof(double) * (size_t)m);
        for (int j = 0; j < m; ++j) {
            memset(e, 0, sizeof(double) * m);
            e[j] = 1;
            mv(ctx, e, col);
            for (int i = 0; i < m; ++i) {
                A[i * m + j] = col[i];
            }
        }
        for (int i = 0; i < m; ++i) {
            for (int j = i + 1; j < m; ++j) {
                const double avg = 0.5 * (A[i * m + j] + A[j * m + i]);
                A[i * m + j] = avg;
                A[j * m + i] = avg;
            }
        }
        double* w = (double*)malloc(sizeof(double) * m);
        double* S = (double*)malloc(sizeof(double) * (size_t)m * m);
        oracle_jacobi_eigen(m, A, w, S);
        for (int c = 0; c < nev; ++c) {
            evals[c] = w[c];
            for (int i = 0; i < m; ++i) {
                evecs[(size_t)c * n + i] = S[i * m + c];
            }
            oracle_fix_sign(n, evecs + (size_t)c * n);
        }
        free(A); free(e); free(col); free(w); free(S);
        return 1;
    }

    double* V = (double*)calloc((size_t)n * (ncv + 1), sizeof(double));
    double* T = (double*)calloc((size_t)ncv * ncv, sizeof(double));
    double* Tcopy = (double*)malloc(sizeof(double) * (size_t)ncv * ncv);
    double* theta = (double*)malloc(sizeof(double) * ncv);
    double* S = (double*)malloc(sizeof(double) * (size_t)ncv * ncv);
    double* h = (double*)malloc(sizeof(double) * (ncv + 1));
    double* tmp = (double*)malloc(sizeof(double) * (size_t)n * ncv);
    int converged = 0;

    oracle_start_vector(n, seed, V);
    {
        const double nrm = oracle_norm(n, V);
        for (int64_t i = 0; i < n; ++i) {
            V[i] /= nrm;
        }
    }

    int k = 0;           /* number of kept Ritz vectors at the start of a cycle */
    double beta_last = 0;
    for (int restart = 0; restart < max_restarts; ++restart) {
        for (int j = k; j < ncv; ++j) {
            double* vj = V + (size_t)j * n;
            double* w = V + (size_t)(j + 1) * n;
            mv(ctx, vj, w);
            memset(h, 0, sizeof(double) * (ncv + 1));
            oracle_reorth(n, j + 1, V, w, h);
            T[j * ncv + j] = h[j];
            if (j > k) {
                /* T[j-1][j] was set when v_j was normalised */
            }
            double beta = oracle_norm(n, w);
            if (beta < 1e-12 * (fabs(h[j]) + 1e-300)) {
                /* invariant subspace: continue with a fresh orthogonal direction */
                oracle_start_vector(n, seed + 7919u * (uint64_t)(j + 1) + 104729u * (uint64_t)restart, w);
                memset(h, 0, sizeof(double) * (ncv + 1));
                oracle_reorth(n, j + 1, V, w, h);
                const double nrm = oracle_norm(n, w);
                for (int64_t i = 0; i < n; ++i) {
                    w[i] /= nrm;
                }
                beta = 0;
            } else {
                for (int64_t i = 0; i < n; ++i) {
                    w[i] /= beta;
                }
            }
            if (j + 1 < ncv) {
                T[j * ncv + j + 1] = beta;
                T[(j + 1) * ncv + j] = beta;
            }
            beta_last = beta;
        }

        memcpy(Tcopy, T, sizeof(double) * (size_t)ncv * ncv);
        oracle_jacobi_eigen(ncv, Tcopy, theta, S);
        const double scale = fabs(theta[0]) > 0 ? fabs(theta[0]) : 1;
        int ok = 1;
        for (int i = 0; i < nev; ++i) {
            const double res = fabs(beta_last * S[(ncv - 1) * ncv + i]);
            if (res > tol * scale) {
                ok = 0;
            }
        }
        if (restarts_out) {
            *restarts_out = restart + 1;
        }

        const int last = (ok || restart == max_restarts - 1);
        int keep = last ? nev : nev + (ncv - nev) / 2;
        if (keep > ncv - 1) {
            keep = ncv - 1;
        }
        /* tmp = V[:, :ncv] * S[:, :keep] */
        for (int c = 0; c < keep; ++c) {
            double* out = tmp + (size_t)c * n;
            memset(out, 0, sizeof(double) * n);
            for (int r = 0; r < ncv; ++r) {
                const double s = S[r * ncv + c];
                const double* vr = V + (size_t)r * n;
                for (int64_t i = 0; i < n; ++i) {
                    out[i] += s * vr[i];
                }
            }
        }
        if (last) {
            for (int c = 0; c < nev; ++c) {
                evals[c] = theta[c];
                memcpy(evecs + (size_t)c * n, tmp + (size_t)c * n, sizeof(double) * n);
                const double nrm = oracle_norm(n, evecs + (size_t)c * n);
                for (int64_t i = 0; i < n; ++i) {
                    evecs[(size_t)c * n + i] /= nrm;
                }
                oracle_fix_sign(n, evecs + (size_t)c * n);
            }
            converged = ok;
            break;
        }
        /* thick restart: keep Ritz vectors, continue from the residual direction */
        memcpy(V + (size_t)keep * n, V + (size_t)ncv * n, sizeof(double) * n);
        memcpy(V, tmp, sizeof(double) * (size_t)n * keep);
        memset(T, 0, sizeof(double) * (size_t)ncv * ncv);
        for (int c = 0; c < keep; ++c) {
            T[c * ncv + c] = theta[c];
            const double coupling = beta_last * S[(ncv - 1) * ncv + c];
            T[c * ncv + keep] = coupling;
            T[keep * ncv + c] = coupling;
        }
        k = keep;
    }

    free(V); free(T); free(Tcopy); free(theta); free(S); free(h); free(tmp);
    return converged;
}

#endif
