// kmb_infer_noalloc: k-means responses (and optionally the exact objective) for
// callers that cannot allocate device memory.
//
// Some callers of this library do not own the device allocator: a plugin that
// runs inside a host framework which hands out all device memory itself and
// forbids allocations behind its back, or a latency-critical request loop that
// cannot afford cudaMalloc/cudaFree (both can synchronise the whole device and
// take milliseconds). kmb_infer allocates its scratch (row norms, transposed
// centroids, per-row distances, objective partials) in a context workspace;
// this variant computes the same result with the same kernels, but its scratch
// lives in one file-scope device array that the CUDA loader reserves when the
// library is loaded on a device, so the call itself allocates nothing.
//
// Limits and sharing rules:
//  * The array is kNoAllocScratchBytes (24 MiB) per device, held by every GPU
//    that loads the library until the process exits. A call needs
//    2*n*sizeof(F) + kpad*dpad*sizeof(F) + kpad*sizeof(F) + 9728 bytes
//    (kpad = k rounded up to 128, dpad = d rounded up to 8, each part rounded
//    up to 256 bytes; 9728 = the objective's kObjectivePartials = 1184 FP64
//    partials and one scalar);
//    larger problems are rejected with KMB_EINVAL and a message on stderr.
//  * All calls on a device share the array and it keeps the last call's
//    contents. Calls whose work overlaps on the GPU (different streams, or
//    different host threads) race on it: serialise them on one stream.
//  * A `__device__` array has one address per CUDA context (the primary context
//    of a device, or a context the caller created with the driver API and made
//    current). The first call in each context resolves the address with
//    cudaGetSymbolAddress while that context is current and caches it under the
//    context's unique id (cuCtxGetId); make that first call before any stream
//    capture in the context. A context created after cudaDeviceReset has a new
//    id, so a cached address never outlives the context it belongs to.
#include "kmb_internal.cuh"

#include <cuda.h>

#include <cstdio>
#include <mutex>

namespace kmb {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(24) << 20;
constexpr int kCacheSlots = 64;
// The fixed part of a call's scratch: the objective partials plus one scalar.
static_assert((sizeof(double) * kObjectivePartials + 255) / 256 * 256 + 256 == 9728,
              "the documented fixed scratch of kmb_infer_noalloc");

// The scratch. Device code may name it directly; host code must use the
// address obtained from cudaGetSymbolAddress (the symbol itself is a host-side
// stand-in, not a device address).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The current context and its process-unique id, through the runtime's driver
// entry points (the library does not link libcuda directly).
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

template <typename Fn>
Fn driver_fn(const char *name) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
        return nullptr;
    return (Fn)p;
}

struct CacheSlot {
    unsigned long long ctx_id;
    void *addr;
};

std::mutex g_mu;
CacheSlot g_cache[kCacheSlots] = {};
int g_cache_next = 0;

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

int current_context_id(unsigned long long *id) {
    static const CtxGetCurrentFn get_current = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
    static const CtxGetIdFn get_id = driver_fn<CtxGetIdFn>("cuCtxGetId");
    if (!get_current || !get_id) return KMB_EUNSUPPORTED;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) return KMB_ECUDA;
    if (!ctx) return KMB_EINVAL;  // no context current yet
    return get_id(ctx, id) == CUDA_SUCCESS ? KMB_OK : KMB_ECUDA;
}

// The scratch address in the calling thread's current context, resolved with
// that context current the first time the context is seen.
int scratch_for_current_context(void **out) {
    unsigned long long id = 0;
    int rc = current_context_id(&id);
    if (rc == KMB_EINVAL) {
        // No context is current on this thread yet: the runtime call below makes
        // the current device's primary context current, which is the one to use.
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) {
            cudaGetLastError();
            return KMB_ECUDA;
        }
        rc = current_context_id(&id);
    }
    if (rc != KMB_OK) return rc;
    std::lock_guard<std::mutex> lock(g_mu);
    for (int i = 0; i < kCacheSlots; ++i)
        if (g_cache[i].addr && g_cache[i].ctx_id == id) {
            *out = g_cache[i].addr;
            return KMB_OK;
        }
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        return KMB_ECUDA;
    }
    g_cache[g_cache_next] = CacheSlot{id, p};
    g_cache_next = (g_cache_next + 1) % kCacheSlots;
    *out = p;
    return KMB_OK;
}

template <typename F>
int infer_noalloc(const F *X, int64_t n, int64_t d, const F *C, int64_t k, int32_t *labels, double *objective,
                  cudaStream_t s) {
    const int64_t kpad = (k + 127) / 128 * 128, dpad = (d + 7) / 8 * 8;
    const size_t need = 2 * align256(sizeof(F) * n) + align256(sizeof(F) * kpad * dpad) + align256(sizeof(F) * kpad) +
                        align256(sizeof(double) * kObjectivePartials) + align256(sizeof(double) * 2);
    if (need > kNoAllocScratchBytes) {
        fprintf(stderr,
                "kmb_infer_noalloc: n=%lld d=%lld k=%lld needs %zu bytes of scratch; the fixed scratch array holds "
                "%zu bytes (24 MiB). Use kmb_infer for this size.\n",
                (long long)n, (long long)d, (long long)k, need, kNoAllocScratchBytes);
        return KMB_EINVAL;
    }
    void *base = nullptr;
    int rc = scratch_for_current_context(&base);
    if (rc != KMB_OK) return rc;
    unsigned char *p = (unsigned char *)base;
    F *xnorm = (F *)p;
    p += align256(sizeof(F) * n);
    F *d2 = (F *)p;
    p += align256(sizeof(F) * n);
    F *Ct = (F *)p;
    p += align256(sizeof(F) * kpad * dpad);
    F *h = (F *)p;
    p += align256(sizeof(F) * kpad);
    double *partials = (double *)p;
    p += align256(sizeof(double) * kObjectivePartials);
    double *cnorm_max = (double *)p;  // zeroed by the centroid preparation on every call

    launch_row_norms<F>(X, n, d, xnorm, s);
    launch_prep_centroids<F>(C, k, d, kpad, Ct, h, cnorm_max, nullptr, s);
    launch_assign_plain<F>(X, n, d, Ct, h, k, kpad, xnorm, cnorm_max, labels, d2, nullptr, nullptr, s);
    if (objective) launch_objective<F>(X, n, d, C, labels, partials, objective, s);
    return cudaGetLastError() == cudaSuccess ? KMB_OK : KMB_ECUDA;
}

}  // namespace
}  // namespace kmb

extern "C" int kmb_infer_noalloc(int dtype, const void *X, int64_t n, int64_t d, const void *C, int64_t k,
                                 int32_t *responses, double *objective, void *cuda_stream) {
    if (dtype != KMB_F32 && dtype != KMB_F64) return KMB_EINVAL;
    if (!X || !C || !responses || n <= 0 || n > INT32_MAX || d <= 0 || k <= 0 || k > INT32_MAX) return KMB_EINVAL;
    cudaStream_t s = (cudaStream_t)cuda_stream;
    if (dtype == KMB_F32)
        return kmb::infer_noalloc<float>((const float *)X, n, d, (const float *)C, k, responses, objective, s);
    return kmb::infer_noalloc<double>((const double *)X, n, d, (const double *)C, k, responses, objective, s);
}
