// FP64 recheck of near-tie rows.
//
// The assignment kernels queue every row whose best/second score gap lies
// inside their derived rounding bound, with its two best clusters and a flag
// when a third cluster is also inside the band. This kernel re-scores those
// candidates (or, when flagged, all k clusters) exactly in double from the
// F inputs, with the reference's score 0.5||c||^2 - x.c and its lowest-index
// tie rule (cpp/daal/src/algorithms/kmeans/kmeans_lloyd_impl.i:197-216), so the
// final labels equal the FP64 oracle's. Two-candidate entries (nearly all of
// them) take two threads each; entries flagged for a full scan take a warp (32 clusters per step).
#include "kmb_internal.cuh"

namespace kmb {
namespace {

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

// Butterfly reduce-scatter over the warp: on entry lane L holds 32 partial sums
// a[0..31] (one per cluster of a group of 32); on exit a[0] on lane L is the
// total for cluster L. Every cluster's total has the same association, so equal
// inputs give equal sums.
template <int H>
__device__ __forceinline__ void reduce_scatter_step(double (&a)[32], int lane) {
    const bool upper = (lane & H) != 0;
#pragma unroll
    for (int i = 0; i < H; ++i) {
        const double send = upper ? a[i] : a[i + H];
        const double keep = upper ? a[i + H] : a[i];
        a[i] = keep + __shfl_xor_sync(0xffffffffu, send, H);
    }
}
__device__ __forceinline__ void reduce_scatter32(double (&a)[32], int lane) {
    reduce_scatter_step<16>(a, lane);
    reduce_scatter_step<8>(a, lane);
    reduce_scatter_step<4>(a, lane);
    reduce_scatter_step<2>(a, lane);
    reduce_scatter_step<1>(a, lane);
}

// Entries with a third cluster inside the band: a warp re-scores all k
// clusters, 32 at a time. Lane L accumulates its coordinates' (t = L, L+32,
// ...) contributions to ||c||^2 and x.c for the 32 clusters (coalesced loads of
// each centroid row), then one reduce-scatter per quantity leaves cluster
// j0 + L's sums on lane L. Lanes keep a running best in ascending cluster
// order; the warp argmin breaks ties to the lowest index.
template <typename F>
__global__ void __launch_bounds__(256) recheck_full_kernel(const F *__restrict__ X, int d, const F *__restrict__ C,
                                                           int k, const RecheckEntry *__restrict__ queue,
                                                           int32_t *__restrict__ labels, F *__restrict__ d2,
                                                           const F *__restrict__ xnorm, LoopState *st) {
    if (st->done) return;
    const int count = st->n_recheck;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    int changed = 0, fulls = 0;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < count; w += warps) {
        const RecheckEntry q = queue[w];
        if (!q.full) continue;
        ++fulls;
        const F *x = X + (int64_t)q.row * d;
        double best = 0.0;
        int bi = 0x7fffffff;
        for (int j0 = 0; j0 < k; j0 += 32) {
            double xc[32], cc[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) xc[i] = cc[i] = 0.0;
            for (int t = lane; t < d; t += 32) {
                const double xv = (double)x[t];
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const int j = min(j0 + i, k - 1);  // rows past k are read but not used
                    const double cv = (double)C[(int64_t)j * d + t];
                    cc[i] = fma(cv, cv, cc[i]);
                    xc[i] = fma(xv, cv, xc[i]);
                }
            }
            reduce_scatter32(cc, lane);
            reduce_scatter32(xc, lane);
            const int j = j0 + lane;
            if (j < k) {
                const double sc = 0.5 * cc[0] - xc[0];
                if (bi == 0x7fffffff || sc < best) {  // ascending j per lane: lowest index on ties
                    best = sc;
                    bi = j;
                }
            }
        }
        for (int m = 16; m >= 1; m >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, m);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, m);
            if (oi != 0x7fffffff && (bi == 0x7fffffff || ob < best || (ob == best && oi < bi))) {
                best = ob;
                bi = oi;
            }
        }
        if (lane == 0) {
            if (labels[q.row] != bi) ++changed;
            labels[q.row] = bi;
            d2[q.row] = F(2.0 * best + (double)xnorm[q.row]);
        }
    }
    if (lane == 0 && changed) atomicAdd(&st->n_changed, changed);
    if (lane == 0 && fulls) atomicAdd(&st->n_full, fulls);
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
