/*
 * ORACLE -- test infrastructure only. Not part of the product path.
 *
 * A plain-C restatement of oneDAL's CSR k-means Lloyd algorithm
 * (kmeans::method::lloyd_csr: the DAAL CPU kernel KMeansBatchKernel<lloydCSR>),
 * used by tests/ as the checker of the CUDA CSR path. Rows are given as
 * zero-based CSR arrays (values, column indices, row offsets of n + 1 entries);
 * DAAL itself reads one-based indices (ReadRowsCSR), which only shifts them.
 * Parity is pinned against the reference kernel compiled from source
 * (oracle/ref/daal_ref_entry.cpp, daalref_train_csr_*).
 *
 * Semantics restated (file:line in the reference project):
 *  - half squared centroid norms clSq_j = 0.5 * sum_t c_jt^2 in F
 *      cpp/daal/src/algorithms/kmeans/kmeans_lloyd_impl.i:66-76
 *  - x.c_j = sum of v * c_j[col] over the row's stored entries in their order
 *    (the sparse product of kmeans_lloyd_impl.i:300-301; with sorted column
 *    indices this is the ascending-column order of the reference's sparse BLAS,
 *    cpp/daal/src/externals/service_spblas_ref.h:178-214)
 *  - argmin of clSq_j - x.c_j with strict '>' replacement scanning j upward
 *    (lowest index on ties); squared distance 2*min + sum of v^2 over the stored
 *    entries; the row's values are scattered into the cluster's F sum
 *      kmeans_lloyd_impl.i:304-336
 *  - per-cluster sums are reduced in F (kmeans_lloyd_impl.i:403-409; only the
 *    dense method widens to double); candidates, merge, reseed (the candidate row
 *    expanded to dense), shift and stop as the dense method
 *      cpp/daal/src/algorithms/kmeans/kmeans_lloyd_batch_impl.i:153-212
 *  - final responses against the final centroids and the exact objective per
 *    512-row block: row term = sum over stored entries of (x*x - 2*x*c) +
 *    ||c||^2 (full norm), clipped at zero; block partials added in order
 *      cpp/daal/src/algorithms/kmeans/kmeans_lloyd_postprocessing.h:186-350,
 *      kmeans_lloyd_helper.h:150-154 (CSR block size 512)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KMO_OK 0
#define KMO_EINVAL 1
#define KMO_ENOMEM 2
#define KMO_ETOO_MANY_EMPTY 3

#define KMO_CSR_DEFINE(F, SFX)                                                                                           \
    static void kmoc_half_norms_##SFX(const F *C, int64_t k, int64_t d, F *h, F scale)                                   \
    {                                                                                                                    \
        for (int64_t j = 0; j < k; ++j) {                                                                                \
            F s = 0;                                                                                                     \
            for (int64_t t = 0; t < d; ++t) s += C[j * d + t] * C[j * d + t];                                            \
            h[j] = s * scale;                                                                                            \
        }                                                                                                                \
    }                                                                                                                    \
                                                                                                                         \
    /* label (lowest index on ties) and best score clSq - x.c of one sparse row */                                      \
    static void kmoc_score_row_##SFX(const F *v, const int64_t *col, int64_t nz, const F *C, const F *h, int64_t k,     \
                                     int64_t d, int32_t *lab, F *best)                                                   \
    {                                                                                                                    \
        F b = 0;                                                                                                         \
        int32_t bi = 0;                                                                                                  \
        for (int64_t j = 0; j < k; ++j) {                                                                                \
            F dot = 0;                                                                                                   \
            for (int64_t e = 0; e < nz; ++e) dot += v[e] * C[j * d + col[e]];                                            \
            const F s = h[j] - dot;                                                                                      \
            if (j == 0 || b > s) {                                                                                       \
                b = s;                                                                                                   \
                bi = (int32_t)j;                                                                                         \
            }                                                                                                            \
        }                                                                                                                \
        *lab = bi;                                                                                                       \
        if (best) *best = b;                                                                                             \
    }                                                                                                                    \
                                                                                                                         \
    static int kmoc_check_##SFX(const int64_t *rowptr, const int64_t *cols, int64_t n, int64_t d)                        \
    {                                                                                                                    \
        if (!rowptr || n <= 0 || d <= 0 || rowptr[0] != 0) return 0;                                                     \
        for (int64_t i = 0; i < n; ++i)                                                                                  \
            if (rowptr[i + 1] < rowptr[i]) return 0;                                                                     \
        for (int64_t e = 0; e < rowptr[n]; ++e)                                                                          \
            if (cols[e] < 0 || cols[e] >= d) return 0;                                                                   \
        return 1;                                                                                                        \
    }                                                                                                                    \
                                                                                                                         \
    int kmoc_assign_##SFX(const F *vals, const int64_t *cols, const int64_t *rowptr, int64_t n, int64_t d, const F *C,  \
                          int64_t k, int32_t *labels, F *best)                                                           \
    {                                                                                                                    \
        if (k <= 0 || !kmoc_check_##SFX(rowptr, cols, n, d)) return KMO_EINVAL;                                          \
        F *h = (F *)malloc(sizeof(F) * (size_t)k);                                                                       \
        if (!h) return KMO_ENOMEM;                                                                                       \
        kmoc_half_norms_##SFX(C, k, d, h, (F)0.5);                                                                       \
        _Pragma("omp parallel for schedule(static)") for (int64_t i = 0; i < n; ++i)                                     \
            kmoc_score_row_##SFX(vals + rowptr[i], cols + rowptr[i], rowptr[i + 1] - rowptr[i], C, h, k, d, labels + i,  \
                                 best ? best + i : NULL);                                                                \
        free(h);                                                                                                         \
        return KMO_OK;                                                                                                   \
    }                                                                                                                    \
                                                                                                                         \
    /* exact objective (postprocessing.h:276-347): 512-row block partials in F */                                       \
    F kmoc_objective_##SFX(const F *vals, const int64_t *cols, const int64_t *rowptr, int64_t n, int64_t d, const F *C,  \
                           int64_t k, const int32_t *labels)                                                             \
    {                                                                                                                    \
        F *sq = (F *)malloc(sizeof(F) * (size_t)k);                                                                      \
        if (!sq) return (F)NAN;                                                                                          \
        kmoc_half_norms_##SFX(C, k, d, sq, (F)1.0);                                                                      \
        F total = 0;                                                                                                     \
        for (int64_t b0 = 0; b0 < n; b0 += 512) {                                                                        \
            const int64_t b1 = b0 + 512 < n ? b0 + 512 : n;                                                              \
            F g = 0;                                                                                                     \
            for (int64_t i = b0; i < b1; ++i) {                                                                          \
                const int64_t a = labels[i];                                                                             \
                F r = 0;                                                                                                 \
                for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) {                                                    \
                    const F x = vals[e], c = C[a * d + cols[e]];                                                         \
                    r += x * x - (F)2 * x * c;                                                                           \
                }                                                                                                        \
                F rs = r + sq[a];                                                                                        \
                if (rs < (F)0) rs = 0;                                                                                   \
                g += rs;                                                                                                 \
            }                                                                                                            \
            total += g;                                                                                                  \
        }                                                                                                                \
        free(sq);                                                                                                        \
        return total;                                                                                                    \
    }                                                                                                                    \
                                                                                                                         \
    static void kmoc_insert_##SFX(F *cv, int64_t *ci, int64_t *cnum, int64_t cap, F value, int64_t row)                  \
    {                                                                                                                    \
        int64_t pos = *cnum;                                                                                             \
        while (pos > 0 && cv[pos - 1] < value) {                                                                         \
            if (pos < cap) {                                                                                             \
                cv[pos] = cv[pos - 1];                                                                                   \
                ci[pos] = ci[pos - 1];                                                                                   \
            }                                                                                                            \
            --pos;                                                                                                       \
        }                                                                                                                \
        if (pos < cap) {                                                                                                 \
            cv[pos] = value;                                                                                             \
            ci[pos] = row;                                                                                               \
            if (*cnum < cap) ++*cnum;                                                                                    \
        }                                                                                                                \
    }                                                                                                                    \
                                                                                                                         \
    /* One Lloyd update from C_in -> C_out (labels under C_in). */                                                      \
    int kmoc_step_##SFX(const F *vals, const int64_t *cols, const int64_t *rowptr, int64_t n, int64_t d,                 \
                        const F *C_in, int64_t k, F *C_out, int32_t *labels, F *shift, int64_t *n_empty)                 \
    {                                                                                                                    \
        if (k <= 0 || !kmoc_check_##SFX(rowptr, cols, n, d)) return KMO_EINVAL;                                          \
        int rc = KMO_OK;                                                                                                 \
        F *h = (F *)malloc(sizeof(F) * (size_t)k);                                                                       \
        F *best = (F *)malloc(sizeof(F) * (size_t)n);                                                                    \
        F *S1 = (F *)calloc((size_t)(k * d), sizeof(F));                                                                 \
        int64_t *S0 = (int64_t *)calloc((size_t)k, sizeof(int64_t));                                                    \
        F *cv = (F *)malloc(sizeof(F) * (size_t)k);                                                                      \
        int64_t *ci = (int64_t *)malloc(sizeof(int64_t) * (size_t)k);                                                    \
        if (!h || !best || !S1 || !S0 || !cv || !ci) {                                                                   \
            rc = KMO_ENOMEM;                                                                                             \
            goto done;                                                                                                   \
        }                                                                                                                \
        kmoc_half_norms_##SFX(C_in, k, d, h, (F)0.5);                                                                    \
        _Pragma("omp parallel for schedule(static)") for (int64_t i = 0; i < n; ++i)                                     \
            kmoc_score_row_##SFX(vals + rowptr[i], cols + rowptr[i], rowptr[i + 1] - rowptr[i], C_in, h, k, d,           \
                                 labels + i, best + i);                                                                  \
        {                                                                                                                \
            int64_t cnum = 0;                                                                                            \
            for (int64_t i = 0; i < n; ++i) {                                                                            \
                const int32_t a = labels[i];                                                                             \
                F v = best[i] * (F)2.0;                                                                                  \
                for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) {                                                    \
                    S1[(int64_t)a * d + cols[e]] += vals[e];                                                             \
                    v += vals[e] * vals[e];                                                                              \
                }                                                                                                        \
                kmoc_insert_##SFX(cv, ci, &cnum, k, v, i);                                                               \
                S0[a]++;                                                                                                 \
            }                                                                                                            \
            F l2 = 0;                                                                                                    \
            int64_t cpos = 0, empt = 0;                                                                                  \
            for (int64_t j = 0; j < k; ++j) {                                                                            \
                if (S0[j] > 0) {                                                                                         \
                    const F coeff = (F)(1.0 / (double)S0[j]);                                                            \
                    for (int64_t t = 0; t < d; ++t) {                                                                    \
                        const F nc = S1[j * d + t] * coeff;                                                              \
                        const F df = C_in[j * d + t] - nc;                                                               \
                        l2 += df * df;                                                                                   \
                        C_out[j * d + t] = nc;                                                                           \
                    }                                                                                                    \
                } else {                                                                                                 \
                    ++empt;                                                                                              \
                    if (cpos >= cnum) {                                                                                  \
                        rc = KMO_ETOO_MANY_EMPTY;                                                                        \
                        goto done;                                                                                       \
                    }                                                                                                    \
                    const int64_t r = ci[cpos];                                                                          \
                    for (int64_t t = 0; t < d; ++t) C_out[j * d + t] = 0;                                                \
                    for (int64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) C_out[j * d + cols[e]] = vals[e];                \
                    for (int64_t t = 0; t < d; ++t) {                                                                    \
                        const F df = C_in[j * d + t] - C_out[j * d + t];                                                 \
                        l2 += df * df;                                                                                   \
                    }                                                                                                    \
                    ++cpos;                                                                                              \
                }                                                                                                        \
            }                                                                                                            \
            if (shift) *shift = l2;                                                                                      \
            if (n_empty) *n_empty = empt;                                                                                \
        }                                                                                                                \
    done:                                                                                                                \
        free(h);                                                                                                         \
        free(best);                                                                                                      \
        free(S1);                                                                                                        \
        free(S0);                                                                                                        \
        free(cv);                                                                                                        \
        free(ci);                                                                                                        \
        return rc;                                                                                                       \
    }                                                                                                                    \
                                                                                                                         \
    int kmoc_train_##SFX(const F *vals, const int64_t *cols, const int64_t *rowptr, int64_t n, int64_t d, const F *C0,  \
                         int64_t k, int64_t max_iter, double eps, F *C_out, int32_t *labels, F *objective,               \
                         int64_t *iterations)                                                                            \
    {                                                                                                                    \
        if (k <= 0 || max_iter < 0 || eps < 0 || !kmoc_check_##SFX(rowptr, cols, n, d)) return KMO_EINVAL;             \
        F *cur = (F *)malloc(sizeof(F) * (size_t)(k * d));                                                               \
        F *nxt = (F *)malloc(sizeof(F) * (size_t)(k * d));                                                               \
        if (!cur || !nxt) {                                                                                              \
            free(cur);                                                                                                   \
            free(nxt);                                                                                                   \
            return KMO_ENOMEM;                                                                                           \
        }                                                                                                                \
        memcpy(cur, C0, sizeof(F) * (size_t)(k * d));                                                                    \
        int64_t it = 0;                                                                                                  \
        int rc = KMO_OK;                                                                                                 \
        for (it = 0; it < max_iter;) {                                                                                   \
            F shift = 0;                                                                                                 \
            rc = kmoc_step_##SFX(vals, cols, rowptr, n, d, cur, k, nxt, labels, &shift, NULL);                           \
            if (rc != KMO_OK) break;                                                                                     \
            F *tmp = cur;                                                                                                \
            cur = nxt;                                                                                                   \
            nxt = tmp;                                                                                                   \
            ++it;                                                                                                        \
            if ((double)shift <= eps) break;                                                                             \
        }                                                                                                                \
        if (rc == KMO_OK) {                                                                                              \
            kmoc_assign_##SFX(vals, cols, rowptr, n, d, cur, k, labels, NULL);                                           \
            if (objective) *objective = kmoc_objective_##SFX(vals, cols, rowptr, n, d, cur, k, labels);                  \
            memcpy(C_out, cur, sizeof(F) * (size_t)(k * d));                                                             \
            if (iterations) *iterations = it;                                                                            \
        }                                                                                                                \
        free(cur);                                                                                                       \
        free(nxt);                                                                                                       \
        return rc;                                                                                                       \
    }                                                                                                                    \
                                                                                                                         \
    int kmoc_infer_##SFX(const F *vals, const int64_t *cols, const int64_t *rowptr, int64_t n, int64_t d, const F *C,   \
                         int64_t k, int want_objective, int32_t *labels, F *objective)                                   \
    {                                                                                                                    \
        int rc = kmoc_assign_##SFX(vals, cols, rowptr, n, d, C, k, labels, NULL);                                        \
        if (rc == KMO_OK && want_objective && objective)                                                                 \
            *objective = kmoc_objective_##SFX(vals, cols, rowptr, n, d, C, k, labels);                                   \
        return rc;                                                                                                       \
    }

KMO_CSR_DEFINE(double, f64)
KMO_CSR_DEFINE(float, f32)
