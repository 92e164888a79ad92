/*
 * Test infrastructure only: a C entry point over the reference's own DAAL
 * k-means++ initialisation (KMeansInitKernel<plusPlusDense, F, avx2>,
 * cpp/daal/src/algorithms/kmeans/kmeans_plusplus_init_impl.i:538-569), compiled
 * from the read-only reference tree by oracle/ref/Makefile into
 * oracle/_ref/libkmeans_daal_ref.so.
 *
 * It is called as oneDAL's host path calls it when train() gets no initial
 * centroids (cpp/oneapi/dal/algo/kmeans/detail/train_init_centroids.hpp:47-74):
 * init::Parameter(k) -- nTrials = 1, seed 777777
 * (cpp/daal/src/algorithms/kmeans/kmeans_init_parameter_types.cpp:41-48,89) --
 * and an mt19937 engine with that seed; here the engine is the reference's own
 * mt19937 BatchImpl for avx2, built directly instead of through the CPU
 * dispatch of engines::mt19937::Batch<>::create.
 */
#include "src/algorithms/kmeans/kmeans_init_kernel.h"
#include "src/algorithms/kmeans/kmeans_plusplus_init_impl.i"
#include "src/algorithms/engines/mt19937/mt19937_batch_impl.h"
#include "src/algorithms/distributions/uniform/uniform_kernel.h"
#include "src/algorithms/distributions/uniform/uniform_impl.i"
#include "data_management/data/homogen_numeric_table.h"
#include "data_management/data/csr_numeric_table.h"

#include <cstdint>
#include <vector>

namespace daal { namespace algorithms { namespace kmeans { namespace init { namespace internal {
template class KMeansInitKernel<plusPlusDense, double, daal::internal::avx2>;
template class KMeansInitKernel<plusPlusDense, float, daal::internal::avx2>;
template class KMeansInitKernel<plusPlusCSR, double, daal::internal::avx2>;
template class KMeansInitKernel<plusPlusCSR, float, daal::internal::avx2>;
}}}}}

namespace daal { namespace algorithms { namespace distributions { namespace uniform { namespace internal {
template class UniformKernel<double, defaultDense, daal::internal::avx2>;
template class UniformKernel<float, defaultDense, daal::internal::avx2>;
}}}}}

namespace {
using namespace daal;
using namespace daal::data_management;
namespace kinit = daal::algorithms::kmeans::init;

template <typename F>
int run_init(const F * X, int64_t n, int64_t d, int64_t k, uint32_t seed, F * C_out)
{
    if (n <= 0 || d <= 0 || k <= 0 || k > n) return 2;
    services::Status st;
    auto tX = HomogenNumericTable<F>::create(const_cast<F *>(X), (size_t)d, (size_t)n, &st);
    auto tC = HomogenNumericTable<F>::create(C_out, (size_t)d, (size_t)k, &st);
    kinit::Parameter par((size_t)k, 0, seed);
    daal::algorithms::engines::mt19937::internal::BatchImpl<daal::internal::avx2, F> engine(seed);
    const NumericTable * in[1] = { tX.get() };
    const NumericTable * out[1] = { tC.get() };
    kinit::internal::KMeansInitKernel<kinit::plusPlusDense, F, daal::internal::avx2> kernel;
    services::Status s = kernel.compute(1, in, 1, out, &par, engine);
    return s.ok() ? 0 : 1;
}
// plusPlusCSR (the default init of train() with method::lloyd_csr,
// cpp/oneapi/dal/algo/kmeans/detail/train_init_centroids.hpp:39-42) on zero-based
// CSR arrays, given to DAAL one-based.
template <typename F>
int run_init_csr(const F * vals, const int64_t * cols, const int64_t * rowptr, int64_t n, int64_t d, int64_t k, uint32_t seed,
                 F * C_out)
{
    if (n <= 0 || d <= 0 || k <= 0 || k > n || rowptr[0] != 0) return 2;
    const int64_t nnz = rowptr[n];
    std::vector<F> v(vals, vals + nnz);
    std::vector<size_t> c((size_t)nnz), r((size_t)n + 1);
    for (int64_t e = 0; e < nnz; ++e) c[(size_t)e] = (size_t)cols[e] + 1;
    for (int64_t i = 0; i <= n; ++i) r[(size_t)i] = (size_t)rowptr[i] + 1;
    services::Status st;
    auto tX = CSRNumericTable::create<F>(v.data(), c.data(), r.data(), (size_t)d, (size_t)n, CSRNumericTableIface::oneBased, &st);
    auto tC = HomogenNumericTable<F>::create(C_out, (size_t)d, (size_t)k, &st);
    kinit::Parameter par((size_t)k, 0, seed);
    daal::algorithms::engines::mt19937::internal::BatchImpl<daal::internal::avx2, F> engine(seed);
    const NumericTable * in[1] = { tX.get() };
    const NumericTable * out[1] = { tC.get() };
    kinit::internal::KMeansInitKernel<kinit::plusPlusCSR, F, daal::internal::avx2> kernel;
    services::Status s = kernel.compute(1, in, 1, out, &par, engine);
    return s.ok() ? 0 : 1;
}
} // namespace

extern "C" {
int daalref_init_plusplus_csr_f64(const double * v, const int64_t * c, const int64_t * r, int64_t n, int64_t d, int64_t k, uint32_t seed,
                                  double * C_out)
{
    return run_init_csr<double>(v, c, r, n, d, k, seed, C_out);
}
int daalref_init_plusplus_csr_f32(const float * v, const int64_t * c, const int64_t * r, int64_t n, int64_t d, int64_t k, uint32_t seed,
                                  float * C_out)
{
    return run_init_csr<float>(v, c, r, n, d, k, seed, C_out);
}
int daalref_init_plusplus_f64(const double * X, int64_t n, int64_t d, int64_t k, uint32_t seed, double * C_out)
{
    return run_init<double>(X, n, d, k, seed, C_out);
}
int daalref_init_plusplus_f32(const float * X, int64_t n, int64_t d, int64_t k, uint32_t seed, float * C_out)
{
    return run_init<float>(X, n, d, k, seed, C_out);
}
} // extern "C"
