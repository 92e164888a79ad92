/*
 * ORACLE -- test infrastructure only (tests/, the smoke check and bench.py's
 * CPU-baseline leg use it; the product never does). CPU restatement of DAAL's
 * dense k-means++ initialisation with one trial, the path oneDAL's train()
 * takes without initial centroids
 * (cpp/oneapi/dal/algo/kmeans/detail/train_init_centroids.hpp:47-74):
 *
 *   engine         std::mt19937 seeded with 777777, uniform draws from
 *                  std::uniform_real_distribution<F>(0, 1) -- the reference's
 *                  own RNG backend (cpp/daal/src/externals/service_rng_ref.h:
 *                  109-117, 190-199) and default seed
 *                  (cpp/daal/src/algorithms/kmeans/kmeans_init_parameter_types.cpp:41-48)
 *   probabilities  k draws up front (kmeans_plusplus_init_impl.i:551, 403-407)
 *   first center   row = size_t(p0 * F(n)), n - 1 on round-off (:573-585)
 *   min distances  per 512-row block: d2 = sum_i (x_i - c_i)^2 in F in
 *                  coordinate order, each step an FMA, min(best, d2) keeping
 *                  best on ties, block sum in row order, overall = block sums
 *                  in block order (:191-216, 637-656). The reference marks the
 *                  d2 loop `omp simd reduction(+)` (:201), so its own order is
 *                  the compiler's vector-lane split; that changes d2 by a few
 *                  ulps and the chosen row only when a sample lands within
 *                  rounding of a boundary. The reference built with its GNU
 *                  flags (-fopenmp-simd, avx2) picks the same rows as this
 *                  restatement on every recorded fixture.
 *   next centers   sample = overall * p; walk block sums, then the block's rows,
 *                  subtracting while sample >= value (:588-611); a row whose
 *                  distance is <= eps = 0.1 * overall / n is resampled with a
 *                  fresh draw, the chosen row's distance is zeroed (:613-635);
 *                  no update after the last center (:669-673).
 *   CSR rows       plusPlusCSR (the default init of method::lloyd_csr) differs only
 *                  in the distance (DataHelperCSR, :244-316): d2 = ||c||^2 (the
 *                  sum of c_i^2 over all columns in order, i.e. over the center
 *                  row's stored entries) then, per stored entry in order,
 *                  d2 += x*x - 2*x*c_col, every operation rounded; the first and
 *                  the chosen centers are their rows expanded to dense.
 *   no candidate   when the overall distance is zero (fewer than k distinct rows)
 *                  or not finite, no draw can succeed and the reference's loop
 *                  never ends; this restatement returns 4 instead.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

namespace {

// Dense rows: d2 = sum_i (x_i - c_i)^2 in coordinate order.
template <typename F>
struct DenseRows {
    const F *X;
    int64_t d;
    int fused;
    F dist(int64_t r, const F *c, F) const {
        const F *x = X + r * d;
        F d2 = F(0);
        for (int64_t i = 0; i < d; ++i) {
            const F t = x[i] - c[i];
            d2 = fused ? std::fma(t, t, d2) : d2 + t * t;
        }
        return d2;
    }
    F center_norm(const F *) const { return F(0); }
    void copy_row(int64_t r, F *dst) const { std::memcpy(dst, X + r * d, sizeof(F) * (size_t)d); }
};

// CSR rows (zero-based): d2 = ||c||^2, then d2 += x*x - 2*x*c per stored entry.
template <typename F>
struct CsrRowsOracle {
    const F *v;
    const int64_t *col, *rowptr;
    int64_t d;
    F dist(int64_t r, const F *c, F cnorm) const {
        F d2 = cnorm;
        for (int64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) {
            const F x = v[e];
            const F a = x * x;
            const F b = (F(2) * x) * c[col[e]];
            d2 = d2 + (a - b);
        }
        return d2;
    }
    F center_norm(const F *c) const {
        F s = F(0);
        for (int64_t i = 0; i < d; ++i) s = s + c[i] * c[i];
        return s;
    }
    void copy_row(int64_t r, F *dst) const {
        for (int64_t i = 0; i < d; ++i) dst[i] = F(0);
        for (int64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) dst[col[e]] = v[e];
    }
};

template <typename F, typename Rows>
int init_plusplus_rows(const Rows &rows, int64_t n, int64_t d, int64_t k, uint32_t seed, F *C, int64_t *rows_out) {
    if (!C || n <= 0 || d <= 0 || k <= 0 || k > n) return 2;
    std::mt19937 gen(seed);
    std::uniform_real_distribution<F> uni(F(0), F(1));
    std::vector<F> prob((size_t)k);
    for (int64_t i = 0; i < k; ++i) prob[(size_t)i] = uni(gen);
    const int64_t B = 512, nb = (n + B - 1) / B;
    std::vector<F> md((size_t)n, std::numeric_limits<F>::max()), acc((size_t)nb);
    F overall = F(0);
    auto update = [&](const F *c) {
        const F cnorm = rows.center_norm(c);
        for (int64_t b = 0; b < nb; ++b) {
            const int64_t r0 = b * B, r1 = std::min(n, r0 + B);
            F sum = F(0);
            for (int64_t r = r0; r < r1; ++r) {
                const F d2 = rows.dist(r, c, cnorm);
                md[(size_t)r] = !(d2 < md[(size_t)r]) ? md[(size_t)r] : d2;
                sum += md[(size_t)r];
            }
            acc[(size_t)b] = sum;
        }
        overall = acc[0];
        for (int64_t b = 1; b < nb; ++b) overall += acc[(size_t)b];
    };
    auto find = [&](F sample) -> int64_t {
        int64_t b = 0;
        for (; b + 1 < nb && sample >= acc[(size_t)b]; ++b) sample -= acc[(size_t)b];
        const int64_t r0 = b * B, cnt = (b == nb - 1) ? n - r0 : B;
        int64_t r = 0;
        for (; r + 1 < cnt && sample >= md[(size_t)(r0 + r)]; ++r) sample -= md[(size_t)(r0 + r)];
        return r0 + r;
    };
    int64_t row = (int64_t)(size_t)(prob[0] * F(n));
    if (row == n) --row;
    rows.copy_row(row, C);
    if (rows_out) rows_out[0] = row;
    update(C);
    for (int64_t c = 1; c < k; ++c) {
        F p = prob[(size_t)c];
        if (!(overall > F(0)) || !(overall <= std::numeric_limits<F>::max())) return 4;
        const F eps = F(0.1) * overall / F(n);
        int64_t tries = 0;
        for (;;) {
            row = find(overall * p);
            if (md[(size_t)row] > eps) {
                md[(size_t)row] = F(0);
                break;
            }
            if (++tries > 10000000) return 3;  // the reference would retry forever
            p = uni(gen);
        }
        rows.copy_row(row, C + c * d);
        if (rows_out) rows_out[c] = row;
        if (c == k - 1) break;
        update(C + c * d);
    }
    return 0;
}

template <typename F>
int init_plusplus(const F *X, int64_t n, int64_t d, int64_t k, uint32_t seed, int fused, F *C, int64_t *rows_out) {
    if (!X) return 2;
    return init_plusplus_rows<F>(DenseRows<F>{X, d, fused}, n, d, k, seed, C, rows_out);
}

template <typename F>
int init_plusplus_csr(const F *v, const int64_t *col, const int64_t *rowptr, int64_t n, int64_t d, int64_t k,
                      uint32_t seed, F *C, int64_t *rows_out) {
    if (!v || !col || !rowptr || n <= 0 || rowptr[0] != 0) return 2;
    return init_plusplus_rows<F>(CsrRowsOracle<F>{v, col, rowptr, d}, n, d, k, seed, C, rows_out);
}

}  // namespace

extern "C" {
int kmo_init_plusplus_f64(const double *X, int64_t n, int64_t d, int64_t k, uint32_t seed, int fused, double *C,
                          int64_t *rows) {
    return init_plusplus<double>(X, n, d, k, seed, fused, C, rows);
}
int kmo_init_plusplus_f32(const float *X, int64_t n, int64_t d, int64_t k, uint32_t seed, int fused, float *C,
                          int64_t *rows) {
    return init_plusplus<float>(X, n, d, k, seed, fused, C, rows);
}
int kmo_init_plusplus_csr_f64(const double *v, const int64_t *col, const int64_t *rowptr, int64_t n, int64_t d,
                              int64_t k, uint32_t seed, double *C, int64_t *rows) {
    return init_plusplus_csr<double>(v, col, rowptr, n, d, k, seed, C, rows);
}
int kmo_init_plusplus_csr_f32(const float *v, const int64_t *col, const int64_t *rowptr, int64_t n, int64_t d,
                              int64_t k, uint32_t seed, float *C, int64_t *rows) {
    return init_plusplus_csr<float>(v, col, rowptr, n, d, k, seed, C, rows);
}
}
