// FP64 recheck of near-tie rows.
//
// The assignment kernels queue every row whose best/second score gap lies
// inside their derived rounding bound, with its two best clusters and a flag
// when a third cluster is also inside the band. This kernel re-scores those
// candidates (or, when flagged, all k clusters) exactly in double from the
// F inputs, with the reference's score 0.5||c||^2 - x.c and its lowest-index
// tie rule (cpp/daal/src/algorithms/kmeans/kmeans_lloyd_impl.i:197-216), so the
// final labels equal the FP64 oracle's.
#include "kmb_internal.cuh"

namespace kmb {
namespace {

template <typename F>
__device__ __forceinline__ double warp_score(const F *__restrict__ x, const F *__restrict__ c, int d, int lane) {
    double cc = 0.0, xc = 0.0;
    for (int t = lane; t < d; t += 32) {
        const double cv = (double)c[t];
        cc = fma(cv, cv, cc);
        xc = fma((double)x[t], cv, xc);
    }
    for (int m = 16; m >= 1; m >>= 1) {
        cc += __shfl_xor_sync(0xffffffffu, cc, m);
        xc += __shfl_xor_sync(0xffffffffu, xc, m);
    }
    return 0.5 * cc - xc;
}

template <typename F>
__global__ void recheck_kernel(const F *__restrict__ X, int d, const F *__restrict__ C, int k,
                               const RecheckEntry *__restrict__ queue, int32_t *__restrict__ labels,
                               F *__restrict__ d2, const F *__restrict__ xnorm, LoopState *st) {
    if (st->done) return;
    const int count = st->n_recheck;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    int changed = 0;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < count; w += warps) {
        const RecheckEntry q = queue[w];
        const F *x = X + (int64_t)q.row * d;
        double best;
        int bi;
        if (q.full) {
            best = warp_score(x, C, d, lane);
            bi = 0;
            for (int j = 1; j < k; ++j) {
                const double v = warp_score(x, C + (int64_t)j * d, d, lane);
                if (v < best) {
                    best = v;
                    bi = j;
                }
            }
        } else {
            const int a = min(q.c1, q.c2), b = max(q.c1, q.c2);
            const double va = warp_score(x, C + (int64_t)a * d, d, lane);
            const double vb = warp_score(x, C + (int64_t)b * d, d, lane);
            best = va;
            bi = a;
            if (vb < va) {
                best = vb;
                bi = b;
            }
        }
        if (lane == 0) {
            if (labels[q.row] != bi) ++changed;
            labels[q.row] = bi;
            d2[q.row] = F(2.0 * best + (double)xnorm[q.row]);
        }
    }
    if (lane == 0 && changed) atomicAdd(&st->n_changed, changed);
}

}  // namespace

template <typename F>
void launch_recheck(const F *X, int64_t n, int64_t d, const F *C, int64_t k, const RecheckEntry *queue,
                    int32_t *labels, F *d2, const F *xnorm, LoopState *st, cudaStream_t s) {
    (void)n;
    recheck_kernel<F><<<148 * 8, 256, 0, s>>>(X, (int)d, C, (int)k, queue, labels, d2, xnorm, st);
    KMB_LAUNCHED();
}

template void launch_recheck<float>(const float *, int64_t, int64_t, const float *, int64_t, const RecheckEntry *,
                                    int32_t *, float *, const float *, LoopState *, cudaStream_t);
template void launch_recheck<double>(const double *, int64_t, int64_t, const double *, int64_t, const RecheckEntry *,
                                     int32_t *, double *, const double *, LoopState *, cudaStream_t);

}  // namespace kmb
