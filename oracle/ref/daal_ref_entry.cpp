/*
 * Test infrastructure only: a C entry point over the reference's own DAAL
 * k-means Lloyd batch kernel, compiled from the read-only reference tree by
 * oracle/ref/Makefile into oracle/_ref/libkmeans_daal_ref.so.
 *
 * The kernel is instantiated exactly as the oneAPI CPU backend uses it:
 *   train: cpp/oneapi/dal/algo/kmeans/backend/cpu/train_kernel_lloyd.cpp:71-144
 *          (Parameter(k, T), accuracyThreshold = eps, default resultsToEvaluate =
 *           centroids | assignments | exact objective,
 *           cpp/daal/src/algorithms/kmeans/kmeans_parameter_types.cpp:44-52)
 *   infer: cpp/oneapi/dal/algo/kmeans/backend/cpu/infer_kernel.cpp:52-116
 *          (Parameter(k, 0), assignments [| exact objective]; output[0] = null)
 * Kernel: KMeansBatchKernel<lloydDense, F, avx2>
 *          (cpp/daal/src/algorithms/kmeans/kmeans_lloyd_batch_impl.i:48-242),
 *         and KMeansBatchKernel<lloydCSR, F, avx2> on a one-based CSRNumericTable
 *          for kmeans::method::lloyd_csr (the *_csr_* entry points; zero-based
 *          input indices are shifted to DAAL's one-based convention here).
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg load this library.
 */
#include "src/algorithms/kmeans/kmeans_lloyd_kernel.h"
#include "src/algorithms/kmeans/kmeans_lloyd_batch_impl.i"
#include "data_management/data/homogen_numeric_table.h"
#include "data_management/data/csr_numeric_table.h"

#include <vector>

#include <cstdint>

namespace daal { namespace algorithms { namespace kmeans { namespace internal {
template class KMeansBatchKernel<lloydDense, double, daal::internal::avx2>;
template class KMeansBatchKernel<lloydDense, float, daal::internal::avx2>;
template class KMeansBatchKernel<lloydCSR, double, daal::internal::avx2>;
template class KMeansBatchKernel<lloydCSR, float, daal::internal::avx2>;
}}}}

extern "C" void daalref_shim_set_threads(int t);
extern "C" int daalref_shim_get_threads();

namespace {

using namespace daal;
using namespace daal::data_management;
namespace km = daal::algorithms::kmeans;

/* Returns 0 on success, 1 on a DAAL error status, 2 on a bad argument.
 * status_code receives the DAAL ErrorID (0 when ok) so that callers can see
 * ErrorKMeansNumberOfClustersIsTooLarge. */
template <typename F, km::Method M = km::lloydDense>
int run(const F * X, int64_t n, int64_t d, const F * C0, int64_t k, int64_t max_iter, double eps, int want_obj, int is_train, F * C_out,
        int * labels, F * obj, int64_t * iters, int * status_code, NumericTablePtr tX = NumericTablePtr())
{
    if (n <= 0 || d <= 0 || k <= 0 || max_iter < 0) return 2;
    services::Status st;
    if (!tX) tX = HomogenNumericTable<F>::create(const_cast<F *>(X), (size_t)d, (size_t)n, &st);
    auto tC = HomogenNumericTable<F>::create(const_cast<F *>(C0), (size_t)d, (size_t)k, &st);
    NumericTablePtr oC, oA, oO, oI;
    int iter_buf = 0;
    F obj_buf    = 0;
    if (is_train) oC = HomogenNumericTable<F>::create(C_out, (size_t)d, (size_t)k, &st);
    oA = HomogenNumericTable<int>::create(labels, 1, (size_t)n, &st);
    oO = HomogenNumericTable<F>::create(&obj_buf, 1, 1, &st);
    if (is_train) oI = HomogenNumericTable<int>::create(&iter_buf, 1, 1, &st);

    km::Parameter par((size_t)k, is_train ? (size_t)max_iter : 0);
    if (is_train) {
        par.accuracyThreshold = eps;
    } else {
        par.resultsToEvaluate = want_obj ? (DAAL_UINT64)(km::computeAssignments | km::computeExactObjectiveFunction)
                                         : (DAAL_UINT64)km::computeAssignments;
    }
    const NumericTable * in[2]  = { tX.get(), tC.get() };
    const NumericTable * out[4] = { oC.get(), oA.get(), oO.get(), oI.get() };
    km::internal::KMeansBatchKernel<M, F, daal::internal::avx2> kernel;
    services::Status s = kernel.compute(in, out, &par);
    if (obj) *obj = obj_buf;
    if (iters) *iters = iter_buf;
    if (!s.ok()) {
        if (status_code) *status_code = (int)(*s.getCollection()->getErrors())[0]->id();
        return 1;
    }
    if (status_code) *status_code = 0;
    return 0;
}

// One-based CSR copy of zero-based (values, columns, row offsets) for DAAL.
template <typename F>
struct CsrInput
{
    std::vector<F> v;
    std::vector<size_t> c, r;
    NumericTablePtr table;
    CsrInput(const F * vals, const int64_t * cols, const int64_t * rowptr, int64_t n, int64_t d)
    {
        const int64_t nnz = rowptr[n];
        v.assign(vals, vals + nnz);
        c.resize((size_t)nnz);
        r.resize((size_t)n + 1);
        for (int64_t e = 0; e < nnz; ++e) c[(size_t)e] = (size_t)cols[e] + 1;
        for (int64_t i = 0; i <= n; ++i) r[(size_t)i] = (size_t)rowptr[i] + 1;
        services::Status st;
        table = CSRNumericTable::create<F>(v.data(), c.data(), r.data(), (size_t)d, (size_t)n, CSRNumericTableIface::oneBased, &st);
    }
};

template <typename F>
int run_csr(const F * vals, const int64_t * cols, const int64_t * rowptr, int64_t n, int64_t d, const F * C0, int64_t k, int64_t max_iter,
            double eps, int want_obj, int is_train, F * C_out, int * labels, F * obj, int64_t * iters, int * status_code)
{
    if (n <= 0 || d <= 0 || !rowptr || rowptr[0] != 0) return 2;
    CsrInput<F> in(vals, cols, rowptr, n, d);
    return run<F, km::lloydCSR>(nullptr, n, d, C0, k, max_iter, eps, want_obj, is_train, C_out, labels, obj, iters, status_code,
                                in.table);
}

} // namespace

extern "C" {

int daalref_train_csr_f64(const double * v, const int64_t * c, const int64_t * r, int64_t n, int64_t d, const double * C0, int64_t k,
                          int64_t max_iter, double eps, double * C_out, int * labels, double * obj, int64_t * iters, int * status_code)
{
    return run_csr<double>(v, c, r, n, d, C0, k, max_iter, eps, 1, 1, C_out, labels, obj, iters, status_code);
}

int daalref_train_csr_f32(const float * v, const int64_t * c, const int64_t * r, int64_t n, int64_t d, const float * C0, int64_t k,
                          int64_t max_iter, double eps, float * C_out, int * labels, float * obj, int64_t * iters, int * status_code)
{
    return run_csr<float>(v, c, r, n, d, C0, k, max_iter, eps, 1, 1, C_out, labels, obj, iters, status_code);
}

int daalref_infer_csr_f64(const double * v, const int64_t * c, const int64_t * r, int64_t n, int64_t d, const double * C, int64_t k,
                          int want_obj, int * labels, double * obj, int * status_code)
{
    return run_csr<double>(v, c, r, n, d, C, k, 0, 0.0, want_obj, 0, nullptr, labels, obj, nullptr, status_code);
}

int daalref_infer_csr_f32(const float * v, const int64_t * c, const int64_t * r, int64_t n, int64_t d, const float * C, int64_t k,
                          int want_obj, int * labels, float * obj, int * status_code)
{
    return run_csr<float>(v, c, r, n, d, C, k, 0, 0.0, want_obj, 0, nullptr, labels, obj, nullptr, status_code);
}

int daalref_set_threads(int t)
{
    daalref_shim_set_threads(t);
    return daalref_shim_get_threads();
}

int daalref_train_f64(const double * X, int64_t n, int64_t d, const double * C0, int64_t k, int64_t max_iter, double eps, double * C_out,
                      int * labels, double * obj, int64_t * iters, int * status_code)
{
    return run<double>(X, n, d, C0, k, max_iter, eps, 1, 1, C_out, labels, obj, iters, status_code);
}

int daalref_train_f32(const float * X, int64_t n, int64_t d, const float * C0, int64_t k, int64_t max_iter, double eps, float * C_out,
                      int * labels, float * obj, int64_t * iters, int * status_code)
{
    return run<float>(X, n, d, C0, k, max_iter, eps, 1, 1, C_out, labels, obj, iters, status_code);
}

int daalref_infer_f64(const double * X, int64_t n, int64_t d, const double * C, int64_t k, int want_obj, int * labels, double * obj,
                      int * status_code)
{
    return run<double>(X, n, d, C, k, 0, 0.0, want_obj, 0, nullptr, labels, obj, nullptr, status_code);
}

int daalref_infer_f32(const float * X, int64_t n, int64_t d, const float * C, int64_t k, int want_obj, int * labels, float * obj,
                      int * status_code)
{
    return run<float>(X, n, d, C, k, 0, 0.0, want_obj, 0, nullptr, labels, obj, nullptr, status_code);
}

} // extern "C"
