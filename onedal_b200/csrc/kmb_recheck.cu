// FP64 recheck of near-tie rows.
//
// The assignment kernels queue every row whose best/second score gap lies
// inside their derived rounding bound, with its two best clusters and a flag
// when a third cluster is also inside the band. This kernel re-scores those
// candidates (or, when flagged, all k clusters) exactly in double from the
// F inputs, with the reference's score 0.5||c||^2 - x.c and its lowest-index
// tie rule (cpp/daal/src/algorithms/kmeans/kmeans_lloyd_impl.i:197-216), so the
// final labels equal the FP64 oracle's. Two-candidate entries (nearly all of
// them) take two threads each; entries flagged for a full scan take a warp.
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

// Two-candidate entries: two threads per entry (one candidate each, a
// sequential FP64 dot product over d), decided with one shuffle.
template <typename F>
__global__ void recheck_pairs_kernel(const F *__restrict__ X, int d, const F *__restrict__ C,
                                     const RecheckEntry *__restrict__ queue, int32_t *__restrict__ labels,
                                     F *__restrict__ d2, const F *__restrict__ xnorm, LoopState *st) {
    if (st->done) return;
    const int count = st->n_recheck;
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    int changed = 0;
    // each warp takes 16 entries per step; the loop bound is uniform across the warp
    for (long long base = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 16; base < count;
         base += warps * 16) {
        const long long e = base + (lane >> 1);
        const bool valid = e < count;
        RecheckEntry q;
        q.row = 0;
        q.c1 = q.c2 = 0;
        q.full = 1;
        if (valid) q = queue[e];
        const bool active = valid && !q.full;
        const int a = min(q.c1, q.c2), b = max(q.c1, q.c2);
        const int cand = (lane & 1) ? b : a;
        double score = 0.0;
        if (active) {
            const F *x = X + (int64_t)q.row * d;
            const F *c = C + (int64_t)cand * d;
            double cc = 0.0, xc = 0.0;
            for (int t = 0; t < d; ++t) {
                const double cv = (double)c[t];
                cc = fma(cv, cv, cc);
                xc = fma((double)x[t], cv, xc);
            }
            score = 0.5 * cc - xc;
        }
        const double other = __shfl_xor_sync(0xffffffffu, score, 1);
        if (active && (lane & 1) == 0) {
            // lane holds the lower index a; b wins only when strictly better
            const bool take_b = other < score;
            const int bi = take_b ? b : a;
            const double best = take_b ? other : score;
            if (labels[q.row] != bi) ++changed;
            labels[q.row] = bi;
            d2[q.row] = F(2.0 * best + (double)xnorm[q.row]);
        }
    }
    for (int m = 16; m >= 1; m >>= 1) changed += __shfl_xor_sync(0xffffffffu, changed, m);
    if (lane == 0 && changed) atomicAdd(&st->n_changed, changed);
}

// Entries with a third cluster inside the band: a warp scans all k clusters.
template <typename F>
__global__ void recheck_full_kernel(const F *__restrict__ X, int d, const F *__restrict__ C, int k,
                                    const RecheckEntry *__restrict__ queue, int32_t *__restrict__ labels,
                                    F *__restrict__ d2, const F *__restrict__ xnorm, LoopState *st) {
    if (st->done) return;
    const int count = st->n_recheck;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    int changed = 0;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < count; w += warps) {
        const RecheckEntry q = queue[w];
        if (!q.full) continue;
        const F *x = X + (int64_t)q.row * d;
        double best = warp_score(x, C, d, lane);
        int bi = 0;
        for (int j = 1; j < k; ++j) {
            const double v = warp_score(x, C + (int64_t)j * d, d, lane);
            if (v < best) {  // ascending j: lowest index on ties
                best = v;
                bi = j;
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
    recheck_pairs_kernel<F><<<148 * 8, 256, 0, s>>>(X, (int)d, C, queue, labels, d2, xnorm, st);
    KMB_LAUNCHED();
    recheck_full_kernel<F><<<148 * 4, 256, 0, s>>>(X, (int)d, C, (int)k, queue, labels, d2, xnorm, st);
    KMB_LAUNCHED();
}

template void launch_recheck<float>(const float *, int64_t, int64_t, const float *, int64_t, const RecheckEntry *,
                                    int32_t *, float *, const float *, LoopState *, cudaStream_t);
template void launch_recheck<double>(const double *, int64_t, int64_t, const double *, int64_t, const RecheckEntry *,
                                     int32_t *, double *, const double *, LoopState *, cudaStream_t);

}  // namespace kmb
