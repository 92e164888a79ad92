/*
 * ORACLE -- test infrastructure only. Not part of the product path.
 *
 * A plain-C restatement of oneDAL's dense k-means Lloyd algorithm (the DAAL
 * CPU kernel that oneapi::dal::train/infer(kmeans::descriptor) reaches on the
 * host), written from the reference's behaviour, used by tests/, the smoke
 * check and bench.py's CPU-baseline leg as the checker. Parity is pinned
 * against the reference test suite's golden vectors (tests/golden/) and
 * against the reference kernel itself compiled from source
 * (oracle/ref/Makefile -> oracle/_ref/libkmeans_daal_ref.so).
 *
 * Semantics restated (file:line in the reference project):
 *  - half squared centroid norms  clSq_j = 0.5 * sum_t c_jt^2 in F
 *      cpp/daal/src/algorithms/kmeans/kmeans_lloyd_impl.i:66-76
 *  - per-row score  clSq_j - x.c_j ; argmin with strict '<' scanning j upward,
 *    so ties go to the lowest cluster index
 *      kmeans_lloyd_impl.i:185-216
 *  - squared distance of a row to its centroid  2*min + sum_t x_t^2  (F)
 *      kmeans_lloyd_impl.i:212, 220-229
 *  - per-cluster sums S1 (F partials) and counts S0; the dense path reduces the
 *    partials in double and stores F  kmeans_lloyd_impl.i:220-229, 384-411
 *  - empty-cluster candidates: the rows with the largest squared distance,
 *    descending; an equal value does not displace an earlier row
 *      kmeans_lloyd_impl.i:413-436
 *  - merge: c_i = S1_i * F(1/S0_i) when S0_i > 0, else the next candidate row
 *    (clusters in ascending index); shift l2 = sum ||c_old - c_new||^2 in F;
 *    fail with "too many empty clusters" when candidates run out
 *      cpp/daal/src/algorithms/kmeans/kmeans_lloyd_batch_impl.i:153-188
 *  - convergence: l2 <= eps -> count the iteration and stop
 *      kmeans_lloyd_batch_impl.i:189-212
 *  - responses recomputed against the final centroids (strict '>' update, so
 *    lowest index on ties)  cpp/daal/src/algorithms/kmeans/kmeans_lloyd_postprocessing.h:64-136
 *  - exact objective  sum_i sum_t (x_it - c_{a_i,t})^2, per-block partials in F
 *      kmeans_lloyd_postprocessing.h:138-183
 *  - max_iteration_count == 0: responses/objective against the initial
 *    centroids  kmeans_lloyd_batch_impl.i:215-218
 *
 * The restatement runs as one logical DAAL thread (one partial-sum set, one
 * candidate list); DAAL's own FP32 results additionally depend on its thread
 * count and on BLAS summation order, so FP32 parity is a tolerance, while the
 * double instantiation is the oracle every tolerance is measured against.
 * Row scoring is parallelised with OpenMP; each row's result does not depend on
 * the thread count.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KMO_OK 0
#define KMO_EINVAL 1
#define KMO_ENOMEM 2
#define KMO_ETOO_MANY_EMPTY 3

/* Block size used for the objective partials, as BSHelper computes it
 * (cpp/daal/src/algorithms/kmeans/kmeans_lloyd_helper.h:119-146) with the L1/L2
 * sizes pinned to 48 KiB / 2 MiB. */
static int64_t kmo_block_size(int64_t d, int64_t k, size_t fsize)
{
    /* size_t arithmetic as in the reference: the subtraction wraps when the
     * centroids do not fit, which then selects the 512-row maximum. */
    const double fullness = 0.8;
    const size_t kk = (size_t)k, dd = (size_t)d;
    const size_t fit1 = (size_t)((double)((48 * 1024 / fsize - kk * dd) / (kk + dd)) * fullness);
    const size_t fit2 = (size_t)((double)((2 * 1024 * 1024 / fsize - kk * dd) / (kk + dd)) * fullness);
    size_t bs = 96;
    if (fit1 >= 256 && fit1 <= 512)
        bs = fit1;
    else if (fit2 >= 8 && fit2 <= 512)
        bs = fit2;
    else if (fit2 >= 512)
        bs = 512;
    return (int64_t)bs;
}

#define KMO_DEFINE(F, SFX)                                                                                                         \
    /* clSq_j = 0.5 * ||c_j||^2 in F */                                                                                            \
    static void kmo_half_norms_##SFX(const F *C, int64_t k, int64_t d, F *h)                                                       \
    {                                                                                                                              \
        for (int64_t j = 0; j < k; ++j) {                                                                                          \
            F s = 0;                                                                                                               \
            for (int64_t t = 0; t < d; ++t) s += C[j * d + t] * C[j * d + t];                                                      \
            h[j] = s * (F)0.5;                                                                                                     \
        }                                                                                                                          \
    }                                                                                                                              \
                                                                                                                                   \
    /* Scores one row: label (lowest index on ties), best and second-best score. */                                              \
    static void kmo_score_row_##SFX(const F *x, const F *C, const F *h, int64_t k, int64_t d, int32_t *lab, F *best, F *second)  \
    {                                                                                                                              \
        F b = 0, s2 = (F)INFINITY;                                                                                                 \
        int32_t bi = 0;                                                                                                            \
        for (int64_t j = 0; j < k; ++j) {                                                                                          \
            F dot = 0;                                                                                                             \
            const F *c = C + j * d;                                                                                                \
            for (int64_t t = 0; t < d; ++t) dot += x[t] * c[t];                                                                    \
            const F v = h[j] - dot;                                                                                                \
            if (j == 0) {                                                                                                          \
                b = v;                                                                                                             \
            } else if (v < b) {                                                                                                    \
                s2 = b;                                                                                                            \
                b  = v;                                                                                                            \
                bi = (int32_t)j;                                                                                                   \
            } else if (v < s2) {                                                                                                   \
                s2 = v;                                                                                                            \
            }                                                                                                                      \
        }                                                                                                                          \
        *lab = bi;                                                                                                                 \
        if (best) *best = b;                                                                                                       \
        if (second) *second = s2;                                                                                                  \
    }                                                                                                                              \
                                                                                                                                   \
    /* Labels plus best/second scores for every row (scores are clSq - x.c). */                                                  \
    int kmo_assign_##SFX(const F *X, int64_t n, int64_t d, const F *C, int64_t k, int32_t *labels, F *best, F *second)          \
    {                                                                                                                              \
        if (n < 0 || d <= 0 || k <= 0) return KMO_EINVAL;                                                                          \
        F *h = (F *)malloc(sizeof(F) * (size_t)k);                                                                                 \
        if (!h) return KMO_ENOMEM;                                                                                                 \
        kmo_half_norms_##SFX(C, k, d, h);                                                                                          \
        _Pragma("omp parallel for schedule(static)") for (int64_t i = 0; i < n; ++i)                                               \
            kmo_score_row_##SFX(X + i * d, C, h, k, d, labels + i, best ? best + i : NULL, second ? second + i : NULL);            \
        free(h);                                                                                                                   \
        return KMO_OK;                                                                                                             \
    }                                                                                                                              \
                                                                                                                                   \
    /* Exact objective sum_i ||x_i - c_{a_i}||^2 with per-block partials in F. */                                                 \
    F kmo_objective_##SFX(const F *X, int64_t n, int64_t d, const F *C, int64_t k, const int32_t *labels)                       \
    {                                                                                                                              \
        const int64_t bs = kmo_block_size(d, k, sizeof(F));                                                                        \
        F total = 0;                                                                                                               \
        for (int64_t b0 = 0; b0 < n; b0 += bs) {                                                                                   \
            const int64_t b1 = b0 + bs < n ? b0 + bs : n;                                                                          \
            F g = 0;                                                                                                               \
            for (int64_t i = b0; i < b1; ++i) {                                                                                    \
                const F *x = X + i * d, *c = C + (int64_t)labels[i] * d;                                                           \
                for (int64_t t = 0; t < d; ++t) g += (x[t] - c[t]) * (x[t] - c[t]);                                                \
            }                                                                                                                      \
            total += g;                                                                                                            \
        }                                                                                                                          \
        return total;                                                                                                              \
    }                                                                                                                              \
                                                                                                                                   \
    /* Candidate insert: keeps the k largest values, descending; ties keep the earlier row first. */                              \
    static void kmo_insert_##SFX(F *cv, int64_t *ci, int64_t *cnum, int64_t cap, F value, int64_t row)                           \
    {                                                                                                                              \
        int64_t pos = *cnum;                                                                                                       \
        while (pos > 0 && cv[pos - 1] < value) {                                                                                   \
            if (pos < cap) {                                                                                                       \
                cv[pos] = cv[pos - 1];                                                                                             \
                ci[pos] = ci[pos - 1];                                                                                             \
            }                                                                                                                      \
            --pos;                                                                                                                 \
        }                                                                                                                          \
        if (pos < cap) {                                                                                                           \
            cv[pos] = value;                                                                                                       \
            ci[pos] = row;                                                                                                         \
            if (*cnum < cap) ++*cnum;                                                                                              \
        }                                                                                                                          \
    }                                                                                                                              \
                                                                                                                                   \
    /* One Lloyd update from C_in (k x d) -> C_out. labels receive the assignment                                                \
     * under C_in. Reports the centroid shift (F), the number of empty clusters and                                              \
     * the within-cluster sum under C_in (F). Returns KMO_ETOO_MANY_EMPTY when the                                               \
     * candidates run out. */                                                                                                    \
    int kmo_step_##SFX(const F *X, int64_t n, int64_t d, const F *C_in, int64_t k, F *C_out, int32_t *labels, F *shift,         \
                       int64_t *n_empty, F *goal)                                                                                  \
    {                                                                                                                              \
        if (n <= 0 || d <= 0 || k <= 0) return KMO_EINVAL;                                                                         \
        int rc       = KMO_OK;                                                                                                     \
        F *h         = (F *)malloc(sizeof(F) * (size_t)k);                                                                         \
        F *best      = (F *)malloc(sizeof(F) * (size_t)n);                                                                         \
        F *S1        = (F *)calloc((size_t)(k * d), sizeof(F));                                                                    \
        int64_t *S0  = (int64_t *)calloc((size_t)k, sizeof(int64_t));                                                             \
        F *cv        = (F *)malloc(sizeof(F) * (size_t)k);                                                                         \
        int64_t *ci  = (int64_t *)malloc(sizeof(int64_t) * (size_t)k);                                                             \
        double *aux  = (double *)malloc(sizeof(double) * (size_t)d);                                                               \
        if (!h || !best || !S1 || !S0 || !cv || !ci || !aux) {                                                                     \
            rc = KMO_ENOMEM;                                                                                                       \
            goto done;                                                                                                             \
        }                                                                                                                          \
        kmo_half_norms_##SFX(C_in, k, d, h);                                                                                       \
        _Pragma("omp parallel for schedule(static)") for (int64_t i = 0; i < n; ++i)                                               \
            kmo_score_row_##SFX(X + i * d, C_in, h, k, d, labels + i, best + i, NULL);                                             \
        {                                                                                                                          \
            int64_t cnum = 0;                                                                                                      \
            F g          = 0;                                                                                                      \
            for (int64_t i = 0; i < n; ++i) {                                                                                      \
                const F *x = X + i * d;                                                                                            \
                const int32_t a = labels[i];                                                                                       \
                F v = best[i] * (F)2.0;                                                                                            \
                for (int64_t t = 0; t < d; ++t) {                                                                                  \
                    S1[(int64_t)a * d + t] += x[t];                                                                                \
                    v += x[t] * x[t];                                                                                              \
                }                                                                                                                  \
                kmo_insert_##SFX(cv, ci, &cnum, k, v, i);                                                                          \
                S0[a]++;                                                                                                           \
                g += v;                                                                                                            \
            }                                                                                                                      \
            F l2 = 0;                                                                                                              \
            int64_t cpos = 0, empt = 0;                                                                                            \
            for (int64_t j = 0; j < k; ++j) {                                                                                      \
                if (S0[j] > 0) {                                                                                                   \
                    for (int64_t t = 0; t < d; ++t) aux[t] = (double)S1[j * d + t];                                                \
                    const F coeff = (F)(1.0 / (double)S0[j]);                                                                      \
                    for (int64_t t = 0; t < d; ++t) {                                                                              \
                        const F nc = (F)aux[t] * coeff;                                                                            \
                        const F df = C_in[j * d + t] - nc;                                                                         \
                        l2 += df * df;                                                                                             \
                        C_out[j * d + t] = nc;                                                                                     \
                    }                                                                                                              \
                } else {                                                                                                           \
                    ++empt;                                                                                                        \
                    if (cpos >= cnum) {                                                                                            \
                        rc = KMO_ETOO_MANY_EMPTY;                                                                                  \
                        goto done;                                                                                                 \
                    }                                                                                                              \
                    const F *row = X + ci[cpos] * d;                                                                               \
                    for (int64_t t = 0; t < d; ++t) {                                                                              \
                        const F df = C_in[j * d + t] - row[t];                                                                     \
                        l2 += df * df;                                                                                             \
                        C_out[j * d + t] = row[t];                                                                                 \
                    }                                                                                                              \
                    ++cpos;                                                                                                        \
                }                                                                                                                  \
            }                                                                                                                      \
            if (shift) *shift = l2;                                                                                                \
            if (n_empty) *n_empty = empt;                                                                                          \
            if (goal) *goal = g;                                                                                                   \
        }                                                                                                                          \
    done:                                                                                                                          \
        free(h);                                                                                                                   \
        free(best);                                                                                                                \
        free(S1);                                                                                                                  \
        free(S0);                                                                                                                  \
        free(cv);                                                                                                                  \
        free(ci);                                                                                                                  \
        free(aux);                                                                                                                 \
        return rc;                                                                                                                 \
    }                                                                                                                              \
                                                                                                                                   \
    /* Full train: T Lloyd updates (stopping when shift <= eps), then responses and                                              \
     * the exact objective against the final centroids. */                                                                       \
    int kmo_train_##SFX(const F *X, int64_t n, int64_t d, const F *C0, int64_t k, int64_t max_iter, double eps, F *C_out,       \
                        int32_t *labels, F *objective, int64_t *iterations)                                                        \
    {                                                                                                                              \
        if (n <= 0 || d <= 0 || k <= 0 || max_iter < 0 || eps < 0) return KMO_EINVAL;                                              \
        F *cur = (F *)malloc(sizeof(F) * (size_t)(k * d));                                                                         \
        F *nxt = (F *)malloc(sizeof(F) * (size_t)(k * d));                                                                         \
        if (!cur || !nxt) {                                                                                                        \
            free(cur);                                                                                                             \
            free(nxt);                                                                                                             \
            return KMO_ENOMEM;                                                                                                     \
        }                                                                                                                          \
        memcpy(cur, C0, sizeof(F) * (size_t)(k * d));                                                                              \
        int64_t it = 0;                                                                                                            \
        int rc     = KMO_OK;                                                                                                       \
        for (it = 0; it < max_iter;) {                                                                                             \
            F shift = 0;                                                                                                           \
            rc      = kmo_step_##SFX(X, n, d, cur, k, nxt, labels, &shift, NULL, NULL);                                            \
            if (rc != KMO_OK) break;                                                                                               \
            F *tmp = cur;                                                                                                          \
            cur    = nxt;                                                                                                          \
            nxt    = tmp;                                                                                                          \
            ++it;                                                                                                                  \
            if ((double)shift <= eps) break;                                                                                       \
        }                                                                                                                          \
        if (rc == KMO_OK) {                                                                                                        \
            kmo_assign_##SFX(X, n, d, cur, k, labels, NULL, NULL);                                                                 \
            if (objective) *objective = kmo_objective_##SFX(X, n, d, cur, k, labels);                                              \
            memcpy(C_out, cur, sizeof(F) * (size_t)(k * d));                                                                       \
            if (iterations) *iterations = it;                                                                                      \
        }                                                                                                                          \
        free(cur);                                                                                                                 \
        free(nxt);                                                                                                                 \
        return rc;                                                                                                                 \
    }                                                                                                                              \
                                                                                                                                   \
    /* Infer: responses, and the exact objective when want_objective != 0. */                                                    \
    int kmo_infer_##SFX(const F *X, int64_t n, int64_t d, const F *C, int64_t k, int want_objective, int32_t *labels,           \
                        F *objective)                                                                                              \
    {                                                                                                                              \
        if (n <= 0 || d <= 0 || k <= 0) return KMO_EINVAL;                                                                         \
        int rc = kmo_assign_##SFX(X, n, d, C, k, labels, NULL, NULL);                                                              \
        if (rc == KMO_OK && want_objective && objective) *objective = kmo_objective_##SFX(X, n, d, C, k, labels);                  \
        return rc;                                                                                                                 \
    }

KMO_DEFINE(double, f64)
KMO_DEFINE(float, f32)

/* Exact FP64 score for a float32 row against float32 centroids, used by tests
 * to classify near-ties: returns best/second of 0.5||c||^2 - x.c computed in
 * double from the float inputs (the FP64 oracle applied to FP32 data). */
int kmo_assign_f32_in_f64(const float *X, int64_t n, int64_t d, const float *C, int64_t k, int32_t *labels, double *best,
                          double *second)
{
    if (n < 0 || d <= 0 || k <= 0) return KMO_EINVAL;
    double *Cd = (double *)malloc(sizeof(double) * (size_t)(k * d));
    double *h  = (double *)malloc(sizeof(double) * (size_t)k);
    if (!Cd || !h) {
        free(Cd);
        free(h);
        return KMO_ENOMEM;
    }
    for (int64_t i = 0; i < k * d; ++i) Cd[i] = (double)C[i];
    kmo_half_norms_f64(Cd, k, d, h);
#pragma omp parallel
    {
        double *xd = (double *)malloc(sizeof(double) * (size_t)d);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            for (int64_t t = 0; t < d; ++t) xd[t] = (double)X[i * d + t];
            kmo_score_row_f64(xd, Cd, h, k, d, labels + i, best ? best + i : NULL, second ? second + i : NULL);
        }
        free(xd);
    }
    free(Cd);
    free(h);
    return KMO_OK;
}

/* Checker for full-size runs: per-cluster sums and counts of float32 rows under
 * given labels, and (when C and objective are given) the objective
 * sum_i ||x_i - c_{a_i}||^2 against C, all accumulated in double. These are the
 * quantities of one Lloyd update (cluster sums kmeans_lloyd_impl.i:220-229,
 * merged and divided in kmeans_lloyd_batch_impl.i:153-166) and of the exact
 * objective (kmeans_lloyd_postprocessing.h:138-183), evaluated in FP64 so that
 * a GPU result can be compared with them at the stated tolerances. Threads take
 * contiguous row ranges; their partials are added in thread order. */
int kmo_cluster_stats_f32(const float *X, int64_t n, int64_t d, const int32_t *labels, int64_t k, const float *C,
                          double *sums, int64_t *counts, double *objective)
{
    if (n < 0 || d <= 0 || k <= 0) return KMO_EINVAL;
    for (int64_t i = 0; i < n; ++i)
        if (labels[i] < 0 || labels[i] >= k) return KMO_EINVAL;
    int nt = 1;
#pragma omp parallel
    {
#pragma omp single
        nt = omp_get_num_threads();
    }
    double *ps = (double *)calloc((size_t)nt * (size_t)(k * d), sizeof(double));
    int64_t *pc = (int64_t *)calloc((size_t)nt * (size_t)k, sizeof(int64_t));
    double *po = (double *)calloc((size_t)nt, sizeof(double));
    if (!ps || !pc || !po) {
        free(ps);
        free(pc);
        free(po);
        return KMO_ENOMEM;
    }
#pragma omp parallel num_threads(nt)
    {
        const int t = omp_get_thread_num();
        const int64_t r0 = n * t / nt, r1 = n * (t + 1) / nt;
        double *s = ps + (size_t)t * (size_t)(k * d);
        int64_t *c = pc + (size_t)t * (size_t)k;
        double o = 0.0;
        for (int64_t i = r0; i < r1; ++i) {
            const float *x = X + i * d;
            const int64_t a = labels[i];
            double *sa = s + a * d;
            for (int64_t j = 0; j < d; ++j) sa[j] += (double)x[j];
            c[a]++;
            if (C) {
                const float *ca = C + a * d;
                for (int64_t j = 0; j < d; ++j) {
                    const double df = (double)x[j] - (double)ca[j];
                    o += df * df;
                }
            }
        }
        po[t] = o;
    }
    memset(sums, 0, sizeof(double) * (size_t)(k * d));
    memset(counts, 0, sizeof(int64_t) * (size_t)k);
    double obj = 0.0;
    for (int t = 0; t < nt; ++t) {
        const double *s = ps + (size_t)t * (size_t)(k * d);
        for (int64_t j = 0; j < k * d; ++j) sums[j] += s[j];
        for (int64_t j = 0; j < k; ++j) counts[j] += pc[(size_t)t * (size_t)k + j];
        obj += po[t];
    }
    if (objective) *objective = obj;
    free(ps);
    free(pc);
    free(po);
    return KMO_OK;
}
