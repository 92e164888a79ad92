// kmb_measure_fma_peak: the device's sustained fused multiply-add rate in FP32 or
// FP64, measured (not derived from a datasheet) so that the plain form's
// assignment kernel can be reported against the peak of the units it runs on.
//
// Every thread runs kChains independent dependent-FMA chains (enough to cover
// the FMA pipeline latency with several warps per scheduler), the grid is a
// multiple of the SM count, and the loop body is unrolled so that the issue
// slots go to FMAs. The chain values stay in a bounded range (a fixed point of
// x -> x * a + b with |a| < 1), so no denormals or infinities slow the pipe.
// The result is 2 flops per FMA over the whole grid divided by the CUDA-event
// time of the best of a few launches. KMB_FMA_PEAK_F32X2 measures the packed
// FP32 pair instruction (fma.rn.f32x2) the resident plain kernel issues.
#include "kmb_internal.cuh"

#include <algorithm>

namespace kmb {
namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;
constexpr int kBlocksPerSm = 8;

template <typename T>
__global__ void __launch_bounds__(kThreads) fma_peak_kernel(int iters, T a, T b, T *sink) {
    T x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == (T)-12345) *sink = s;  // keeps the chains live; never true for these inputs
}

// Packed FP32 pairs (fma.rn.f32x2, two FMAs per instruction): kChains pairs.
__global__ void __launch_bounds__(kThreads) fma2_peak_kernel(int iters, float a, float b, float *sink) {
    float2 x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = make_float2((float)(threadIdx.x + c) * 1e-3f, (float)(threadIdx.x - c) * 1e-3f);
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = __ffma2_rn(x[c], a2, b2);
    }
    float s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c].x + x[c].y;
    if (s == -12345.f) *sink = s;  // keeps the chains live; never true for these inputs
}

template <typename T, bool PACKED = false>
int measure(int device, double *gflops) {
    if (cudaSetDevice(device) != cudaSuccess) return KMB_ECUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * kBlocksPerSm;
    const int iters = sizeof(T) == 4 ? 4096 : 512;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    T *sink = nullptr;
    int rc = KMB_OK;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess || cudaMallocAsync((void **)&sink, sizeof(T), s) != cudaSuccess) {
        rc = KMB_ECUDA;
    } else {
        float best = 0.f;
        for (int rep = 0; rep < 5 && rc == KMB_OK; ++rep) {
            cudaEventRecord(e0, s);
            if (PACKED)
                fma2_peak_kernel<<<blocks, kThreads, 0, s>>>(iters, 0.999f, 1e-4f, (float *)sink);
            else
                fma_peak_kernel<T><<<blocks, kThreads, 0, s>>>(iters, (T)0.999, (T)1e-4, sink);
            KMB_LAUNCHED();
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                rc = KMB_ECUDA;
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0 && (best == 0.f || ms < best)) best = ms;  // the first launch is a warm-up
        }
        if (rc == KMB_OK) {
            const double fmas = (double)blocks * kThreads * kChains * 16.0 * iters * (PACKED ? 2 : 1);
            *gflops = 2.0 * fmas / (best * 1e-3) / 1e9;
        }
    }
    if (sink) cudaFreeAsync(sink, s);
    if (s) cudaStreamSynchronize(s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (rc != KMB_OK) cudaGetLastError();
    return rc;
}

}  // namespace
}  // namespace kmb

extern "C" int kmb_measure_fma_peak(int device, int dtype, double *gflops) {
    if (!gflops || (dtype != KMB_F32 && dtype != KMB_F64 && dtype != KMB_FMA_PEAK_F32X2)) return KMB_EINVAL;
    *gflops = 0.0;
    if (dtype == KMB_FMA_PEAK_F32X2) return kmb::measure<float, true>(device, gflops);
    return dtype == KMB_F32 ? kmb::measure<float>(device, gflops) : kmb::measure<double>(device, gflops);
}
