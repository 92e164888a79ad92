/*
 * Test infrastructure only: the runtime services DAAL's k-means Lloyd kernel
 * needs, supplied without TBB or MKL so that the reference kernel can be
 * compiled here from its own sources (oracle/ref/Makefile).
 *
 * - Threading ABI (cpp/daal/src/threading/threading.h:88-140) over a plain
 *   std::thread fork/join. static_threader_for keeps the documented static
 *   split (threading.h:340-360: thread t runs iterations [t*nI, (t+1)*nI)),
 *   so per-thread partial sums -- and therefore FP32 results -- depend only on
 *   the thread count, which daalref_shim_set_threads pins.
 * - BLAS: sgemm_/dgemm_ forward to the OpenBLAS that SciPy bundles
 *   (scipy_sgemm_/scipy_dgemm_), the "ref" backend DAAL uses without MKL
 *   (cpp/daal/src/externals/service_blas_ref.h). OpenBLAS runs single-threaded
 *   inside each DAAL worker.
 * - Cache sizes are pinned (48 KiB L1, 2 MiB L2) so BSHelper's block size
 *   (cpp/daal/src/algorithms/kmeans/kmeans_lloyd_helper.h:119-146) is the same
 *   on every host.
 * - Serialization / factory / CPU-detection entry points that the Lloyd path
 *   never calls are stubbed.
 */
#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <thread>
#include <vector>

namespace daal {
typedef void (*functype)(int i, const void * a);
typedef void (*functype_static)(size_t i, size_t tid, const void * a);
typedef void (*functype_blocked_size)(size_t first, size_t last, const void * a);
typedef void * (*tls_functype)(const void * a);
typedef void (*tls_reduce_functype)(void * p, const void * a);
} // namespace daal

namespace {

constexpr int kMaxThreads = 512;
int g_threads             = 1;
thread_local int t_index  = 0;

template <typename Body>
void fork_join(int nthreads, const Body & body)
{
    if (nthreads <= 1) {
        body(0);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(nthreads - 1);
    for (int t = 1; t < nthreads; ++t) {
        pool.emplace_back([t, &body]() {
            t_index = t;
            body(t);
        });
    }
    const int saved = t_index;
    t_index         = 0;
    body(0);
    t_index = saved;
    for (auto & th : pool) th.join();
}

struct TlsSlots
{
    daal::tls_functype make;
    const void * arg;
    void * slot[kMaxThreads];
};

} // namespace

extern "C" {

void daalref_shim_set_threads(int t)
{
    g_threads = std::max(1, std::min(t, kMaxThreads));
}
int daalref_shim_get_threads()
{
    return g_threads;
}

int _daal_threader_get_max_threads()
{
    return g_threads;
}
int _daal_threader_get_current_thread_index()
{
    return t_index;
}

void _daal_static_threader_for(size_t n, const void * a, daal::functype_static f)
{
    const size_t T  = (size_t)g_threads;
    const size_t nI = (n + T - 1) / T;
    const int used  = (int)std::min(T, nI ? (n + nI - 1) / nI : (size_t)1);
    fork_join(used, [&](int tid) {
        const size_t b = (size_t)tid * nI;
        const size_t e = std::min(n, b + nI);
        for (size_t i = b; i < e; ++i) f(i, (size_t)tid, a);
    });
}

void _daal_threader_for(int n, int, const void * a, daal::functype f)
{
    std::atomic<int> next(0);
    const int used = std::max(1, std::min(g_threads, n));
    fork_join(used, [&](int) {
        for (int i = next.fetch_add(1); i < n; i = next.fetch_add(1)) f(i, a);
    });
}

void _daal_threader_for_simple(int n, int req, const void * a, daal::functype f)
{
    _daal_threader_for(n, req, a, f);
}

void _daal_threader_for_blocked_size(size_t n, size_t block, const void * a, daal::functype_blocked_size f)
{
    if (block == 0) block = 1;
    const size_t nb = (n + block - 1) / block;
    std::atomic<size_t> next(0);
    const int used = (int)std::max<size_t>(1, std::min<size_t>((size_t)g_threads, nb));
    fork_join(used, [&](int) {
        for (size_t i = next.fetch_add(1); i < nb; i = next.fetch_add(1)) f(i * block, std::min(n, (i + 1) * block), a);
    });
}

void * _daal_get_tls_ptr(void * a, daal::tls_functype f)
{
    TlsSlots * t = new TlsSlots;
    t->make      = f;
    t->arg       = a;
    std::fill(t->slot, t->slot + kMaxThreads, nullptr);
    return t;
}
void * _daal_get_tls_local(void * p)
{
    TlsSlots * t = static_cast<TlsSlots *>(p);
    void *& v    = t->slot[t_index];
    if (!v) v = t->make(t->arg);
    return v;
}
void _daal_reduce_tls(void * p, void * a, daal::tls_reduce_functype f)
{
    TlsSlots * t = static_cast<TlsSlots *>(p);
    for (int i = 0; i < kMaxThreads; ++i)
        if (t->slot[i]) f(t->slot[i], a);
}
void _daal_parallel_reduce_tls(void * p, void * a, daal::tls_reduce_functype f)
{
    _daal_reduce_tls(p, a, f);
}
void _daal_del_tls_ptr(void * p)
{
    delete static_cast<TlsSlots *>(p);
}

void * _daal_new_mutex()
{
    return new std::mutex;
}
void _daal_del_mutex(void * m)
{
    delete static_cast<std::mutex *>(m);
}
void _daal_lock_mutex(void * m)
{
    static_cast<std::mutex *>(m)->lock();
}
void _daal_unlock_mutex(void * m)
{
    static_cast<std::mutex *>(m)->unlock();
}
bool _daal_is_in_parallel()
{
    return t_index != 0;
}

void * _threaded_scalable_malloc(const size_t size, const size_t alignment)
{
    const size_t al = alignment < 64 ? 64 : alignment;
    return aligned_alloc(al, (size + al - 1) / al * al);
}
void _threaded_scalable_free(void * p)
{
    free(p);
}

/* BLAS forwarding to SciPy's bundled OpenBLAS (exported entry points only). */
void scipy_openblas_set_num_threads(int);
void scipy_dgemm_(const char *, const char *, const int *, const int *, const int *, const double *, const double *, const int *, const double *,
                  const int *, const double *, double *, const int *);
void scipy_sgemm_(const char *, const char *, const int *, const int *, const int *, const float *, const float *, const int *, const float *,
                  const int *, const float *, float *, const int *);

int openblas_get_num_threads()
{
    return 1;
}
void openblas_set_num_threads(int) {}

void dgemm_(const char * ta, const char * tb, const int * m, const int * n, const int * k, const double * al, const double * A, const int * lda,
            const double * B, const int * ldb, const double * be, double * C, const int * ldc)
{
    static std::once_flag once;
    std::call_once(once, []() { scipy_openblas_set_num_threads(1); });
    scipy_dgemm_(ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc);
}
void sgemm_(const char * ta, const char * tb, const int * m, const int * n, const int * k, const float * al, const float * A, const int * lda,
            const float * B, const int * ldb, const float * be, float * C, const int * ldc)
{
    static std::once_flag once;
    std::call_once(once, []() { scipy_openblas_set_num_threads(1); });
    scipy_sgemm_(ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc);
}

} // extern "C"

bool daal_check_is_intel_cpu()
{
    return false;
}

namespace daal { namespace services { namespace internal {
size_t getL1CacheSize()
{
    return 48 * 1024;
}
size_t getL2CacheSize()
{
    return 2 * 1024 * 1024;
}
}}} // namespace daal::services::internal
