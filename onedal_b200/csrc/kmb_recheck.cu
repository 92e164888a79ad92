// FP64 recheck of near-tie rows.
//
// The assignment kernels queue every row whose best/second score gap lies
// inside their derived rounding bound, with its two best clusters and a flag
// when a third cluster is also inside the band. This kernel re-scores those
// candidates (or, when flagged, all k clusters) exactly in double from the
// F inputs, with the reference's score 0.5||c||^2 - x.c and its lowest-index
// tie rule (cpp/daal/src/algorithms/kmeans/kmeans_lloyd_impl.i:197-216), so the
// final labels equal the FP64 oracle's. Two-candidate entries (nearly all of
// them; the front of the queue) take eight lanes each; entries flagged for a
// full scan (the back of the queue) take a block, 8 warps x 32 clusters per step.
#include "kmb_internal.cuh"

namespace kmb {
namespace {

// Two-candidate entries (the front of the queue): eight lanes per entry, four
// entries per warp. Lane l of a group accumulates coordinates t = l, l+8, ...
// of ||c||^2 and x.c for both candidates in double (consecutive lanes read
// consecutive floats of the row and of each centroid), then three butterfly
// steps give the group's totals; both candidates' sums have the same
// association, so equal centroids give equal scores. With VEC (float rows, d a
// multiple of 4, 16-byte aligned bases) lane l reads 16 bytes at a time
// (t = 4l .. 4l+3, then 32 further), a quarter of the loads in flight per row.
template <typename F>
__device__ __forceinline__ void pair_sums(const F *x, const F *ca, const F *cb, int d, int sub, double &cca,
                                          double &xca, double &ccb, double &xcb) {
    for (int t = sub; t < d; t += 8) {
        const double xv = (double)x[t], va = (double)ca[t], vb = (double)cb[t];
        cca = fma(va, va, cca);
        xca = fma(xv, va, xca);
        ccb = fma(vb, vb, ccb);
        xcb = fma(xv, vb, xcb);
    }
}
__device__ __forceinline__ void pair_sums_vec(const float *x, const float *ca, const float *cb, int d, int sub,
                                              double &cca, double &xca, double &ccb, double &xcb) {
    const float4 *x4 = reinterpret_cast<const float4 *>(x), *a4 = reinterpret_cast<const float4 *>(ca),
                 *b4 = reinterpret_cast<const float4 *>(cb);
#pragma unroll 4
    for (int t = sub; t < (d >> 2); t += 8) {
        const float4 xq = x4[t], aq = a4[t], bq = b4[t];
        const double xv[4] = {xq.x, xq.y, xq.z, xq.w}, va[4] = {aq.x, aq.y, aq.z, aq.w},
                     vb[4] = {bq.x, bq.y, bq.z, bq.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            cca = fma(va[i], va[i], cca);
            xca = fma(xv[i], va[i], xca);
            ccb = fma(vb[i], vb[i], ccb);
            xcb = fma(xv[i], vb[i], xcb);
        }
    }
}

template <typename F, bool VEC>
__global__ void __launch_bounds__(256) recheck_pairs_kernel(const F *__restrict__ X, int d, const F *__restrict__ C,
                                                            const RecheckEntry *__restrict__ queue,
                                                            int32_t *__restrict__ labels, F *__restrict__ d2,
                                                            const F *__restrict__ xnorm, LoopState *st) {
    if (st->done) return;
    const int count = st->n_recheck;
    const int lane = threadIdx.x & 31;
    const int sub = lane & 7;
    const long long groups = ((long long)gridDim.x * blockDim.x) >> 3;
    int changed = 0;
    // the loop bound is uniform across the warp (four groups step together)
    for (long long base = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < count;
         base += groups) {
        const long long e = base + (lane >> 3);
        const bool valid = e < count;
        RecheckEntry q;
        q.row = 0;
        q.c1 = q.c2 = 0;
        if (valid) q = queue[e];
        const int a = min(q.c1, q.c2), b = max(q.c1, q.c2);
        double cca = 0.0, xca = 0.0, ccb = 0.0, xcb = 0.0;
        if (valid) {
            const F *x = X + (int64_t)q.row * d;
            const F *ca = C + (int64_t)a * d;
            const F *cb = C + (int64_t)b * d;
            if constexpr (VEC)
                pair_sums_vec(x, ca, cb, d, sub, cca, xca, ccb, xcb);
            else
                pair_sums(x, ca, cb, d, sub, cca, xca, ccb, xcb);
        }
#pragma unroll
        for (int m = 4; m >= 1; m >>= 1) {
            cca += __shfl_xor_sync(0xffffffffu, cca, m);
            xca += __shfl_xor_sync(0xffffffffu, xca, m);
            ccb += __shfl_xor_sync(0xffffffffu, ccb, m);
            xcb += __shfl_xor_sync(0xffffffffu, xcb, m);
        }
        if (valid && sub == 0) {
            const double sa = 0.5 * cca - xca, sb = 0.5 * ccb - xcb;
            const bool take_b = sb < sa;  // the lower index a wins ties
            const int bi = take_b ? b : a;
            const double best = take_b ? sb : sa;
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

// Entries with a third cluster inside the band (the back of the queue): a block
// re-scores all k clusters of one row. Its 8 warps take interleaved groups of
// 32 clusters; lane L accumulates its coordinates' (t = L, L+32, ...)
// contributions to ||c||^2 and x.c for the group's 32 clusters (coalesced loads
// of each centroid row), then one reduce-scatter per quantity leaves cluster
// j0 + L's sums on lane L. Every lane keeps a running best in ascending cluster
// order; the warp and then the block reduce with ties to the lowest index.
template <typename F>
__global__ void __launch_bounds__(256) recheck_full_kernel(const F *__restrict__ X, int d, const F *__restrict__ C,
                                                           int k, const RecheckEntry *__restrict__ queue, int64_t cap,
                                                           int32_t *__restrict__ labels, F *__restrict__ d2,
                                                           const F *__restrict__ xnorm, LoopState *st) {
    if (st->done) return;
    __shared__ double s_best[8];
    __shared__ int s_idx[8];
    const int count = st->n_full;  // entries queue[cap - 1], queue[cap - 2], ...
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int changed = 0;
    for (int e = blockIdx.x; e < count; e += gridDim.x) {
        const RecheckEntry q = queue[cap - 1 - e];
        const F *x = X + (int64_t)q.row * d;
        double best = 0.0;
        int bi = 0x7fffffff;
        for (int j0 = 32 * warp; j0 < k; j0 += 256) {
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
            s_best[warp] = best;
            s_idx[warp] = bi;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < 8; ++w) {
                const double ob = s_best[w];
                const int oi = s_idx[w];
                if (oi != 0x7fffffff && (bi == 0x7fffffff || ob < best || (ob == best && oi < bi))) {
                    best = ob;
                    bi = oi;
                }
            }
            if (labels[q.row] != bi) ++changed;
            labels[q.row] = bi;
            d2[q.row] = F(2.0 * best + (double)xnorm[q.row]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && changed) atomicAdd(&st->n_changed, changed);
}

// Entries flagged for a full scan, R rows per block: the rows go to shared
// memory, thread i scores clusters i, i + 256, ... against all R rows, so each
// centroid row is read once per R entries instead of once per entry. A
// cluster's ||c||^2 and x.c are summed in ascending coordinate order (one
// association for every cluster); every thread keeps, per row, a running best
// in ascending cluster order, then the warps and the block reduce with ties to
// the lowest index.
template <typename F, int R, bool VEC>
__global__ void __launch_bounds__(256) recheck_full_rows_kernel(const F *__restrict__ X, int d,
                                                                const F *__restrict__ C, int k,
                                                                const RecheckEntry *__restrict__ queue, int64_t cap,
                                                                int32_t *__restrict__ labels, F *__restrict__ d2,
                                                                const F *__restrict__ xnorm, LoopState *st) {
    if (st->done) return;
    extern __shared__ __align__(16) unsigned char recheck_smem[];
    F *xs = reinterpret_cast<F *>(recheck_smem);  // R x d
    __shared__ double s_best[8][R];
    __shared__ int s_idx[8][R];
    __shared__ int s_row[R];
    const int count = st->n_full;  // entries queue[cap - 1], queue[cap - 2], ...
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int changed = 0;
    for (int e0 = blockIdx.x * R; e0 < count; e0 += gridDim.x * R) {
        const int nr = min(R, count - e0);
        if (threadIdx.x < R) s_row[threadIdx.x] = (int)threadIdx.x < nr ? queue[cap - 1 - (e0 + threadIdx.x)].row : 0;
        __syncthreads();
        for (int i = threadIdx.x; i < R * d; i += blockDim.x) {
            const int r = i / d, t = i - r * d;
            xs[i] = r < nr ? X[(int64_t)s_row[r] * d + t] : F(0);
        }
        __syncthreads();
        double best[R];
        int bi[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            best[r] = 0.0;
            bi[r] = 0x7fffffff;
        }
        for (int j = threadIdx.x; j < k; j += blockDim.x) {
            const F *c = C + (int64_t)j * d;
            double cc = 0.0, acc[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = 0.0;
            if constexpr (VEC && sizeof(F) == 4) {  // float, d % 4 == 0, 16-byte aligned: 16 bytes at a time
                const float4 *c4 = reinterpret_cast<const float4 *>(c);
#pragma unroll 2
                for (int t4 = 0; t4 < (d >> 2); ++t4) {
                    const float4 q = c4[t4];
                    const double cv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        cc = fma(cv[u], cv[u], cc);
#pragma unroll
                        for (int r = 0; r < R; ++r) acc[r] = fma((double)xs[r * d + 4 * t4 + u], cv[u], acc[r]);
                    }
                }
            } else {
#pragma unroll 4
                for (int t = 0; t < d; ++t) {
                    const double cv = (double)c[t];
                    cc = fma(cv, cv, cc);
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[r] = fma((double)xs[r * d + t], cv, acc[r]);
                }
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const double sc = 0.5 * cc - acc[r];
                if (bi[r] == 0x7fffffff || sc < best[r]) {  // ascending j per thread: lowest index on ties
                    best[r] = sc;
                    bi[r] = j;
                }
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            for (int m = 16; m >= 1; m >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best[r], m);
                const int oi = __shfl_xor_sync(0xffffffffu, bi[r], m);
                if (oi != 0x7fffffff && (bi[r] == 0x7fffffff || ob < best[r] || (ob == best[r] && oi < bi[r]))) {
                    best[r] = ob;
                    bi[r] = oi;
                }
            }
            if (lane == 0) {
                s_best[warp][r] = best[r];
                s_idx[warp][r] = bi[r];
            }
        }
        __syncthreads();
        if ((int)threadIdx.x < nr) {
            const int r = threadIdx.x;
            double b = s_best[0][r];
            int ii = s_idx[0][r];
            for (int w = 1; w < 8; ++w) {
                const double ob = s_best[w][r];
                const int oi = s_idx[w][r];
                if (oi != 0x7fffffff && (ii == 0x7fffffff || ob < b || (ob == b && oi < ii))) {
                    b = ob;
                    ii = oi;
                }
            }
            const int row = s_row[r];
            if (labels[row] != ii) ++changed;
            labels[row] = ii;
            d2[row] = F(2.0 * b + (double)xnorm[row]);
        }
        __syncthreads();
    }
    if (changed) atomicAdd(&st->n_changed, changed);
}

constexpr int kFullRows = 8;

}  // namespace

template <typename F>
void launch_recheck(const F *X, int64_t n, int64_t d, const F *C, int64_t k, const RecheckEntry *queue,
                    int32_t *labels, F *d2, const F *xnorm, LoopState *st, int num_sms, cudaStream_t s) {
    bool vec = false;
    const bool vec_c = sizeof(F) == 4 && d % 4 == 0 && (uintptr_t)C % 16 == 0;
    if constexpr (sizeof(F) == 4) {
        vec = d % 4 == 0 && (uintptr_t)X % 16 == 0 && (uintptr_t)C % 16 == 0;
        if (vec)
            recheck_pairs_kernel<float, true><<<num_sms * 8, 256, 0, s>>>(X, (int)d, C, queue, labels, d2, xnorm, st);
    }
    if (!vec)
        recheck_pairs_kernel<F, false><<<num_sms * 8, 256, 0, s>>>(X, (int)d, C, queue, labels, d2, xnorm, st);
    KMB_LAUNCHED();
    const size_t rows_smem = (size_t)kFullRows * d * sizeof(F);
    if (rows_smem <= 48 * 1024) {
        if (vec_c)
            recheck_full_rows_kernel<F, kFullRows, true><<<num_sms * 2, 256, rows_smem, s>>>(X, (int)d, C, (int)k,
                                                                                            queue, n, labels, d2,
                                                                                            xnorm, st);
        else
            recheck_full_rows_kernel<F, kFullRows, false><<<num_sms * 2, 256, rows_smem, s>>>(X, (int)d, C, (int)k,
                                                                                             queue, n, labels, d2,
                                                                                             xnorm, st);
    } else {
        // wide rows: one wave (254 registers per thread: one 256-thread block per SM), a block per entry
        recheck_full_kernel<F><<<num_sms, 256, 0, s>>>(X, (int)d, C, (int)k, queue, n, labels, d2, xnorm, st);
    }
    KMB_LAUNCHED();
}

template void launch_recheck<float>(const float *, int64_t, int64_t, const float *, int64_t, const RecheckEntry *,
                                    int32_t *, float *, const float *, LoopState *, int, cudaStream_t);
template void launch_recheck<double>(const double *, int64_t, int64_t, const double *, int64_t, const RecheckEntry *,
                                     int32_t *, double *, const double *, LoopState *, int, cudaStream_t);

}  // namespace kmb
