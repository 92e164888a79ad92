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
//    up to 256 bytes; 9728 = the objective's 1184 FP64 partials and one scalar);
//    larger problems are rejected with KMB_EINVAL and a message on stderr.
//  * All calls on a device share the array and it keeps the last call's
//    contents. Calls whose work overlaps on the GPU (different streams, or
//    different host threads) race on it: serialise them on one stream.
//  * The first call on each device resolves the array's device address with
//    cudaGetSymbolAddress while that device is current; make that first call
//    before any stream capture on the device.
#include "kmb_internal.cuh"

#include <cstdio>
#include <mutex>

namespace kmb {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(24) << 20;
constexpr int kMaxDevices = 64;
constexpr int kObjectivePartials = 148 * 8;  // partial sums of the objective kernel

// The scratch. Device code may name it directly; host code must use the
// address obtained from cudaGetSymbolAddress (the symbol itself is a host-side
// stand-in, not a device address).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {nullptr};

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// Resolves (once per device, with that device current) the scratch address.
int scratch_for_current_device(void **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return KMB_ECUDA;
    if (dev < 0 || dev >= kMaxDevices) return KMB_EUNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return KMB_ECUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
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
    int rc = scratch_for_current_device(&base);
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
