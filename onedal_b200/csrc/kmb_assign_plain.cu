// Plain-form assignment: fused x.c contraction + per-row argmin (FP32 / FP64 FMA).
//
// Replaces, for every row block, DAAL's
//   buf = clSq - X_b * C^T  (xxgemm, α = -1, β = 1) followed by a strict-'<'
//   argmin scan over clusters
// (cpp/daal/src/algorithms/kmeans/kmeans_lloyd_impl.i:174-216 in the update loop and
//  cpp/daal/src/algorithms/kmeans/kmeans_lloyd_postprocessing.h:95-130 for the final
//  responses). The n x k score matrix is never materialised: each CTA owns a
// 128-row tile, streams 128-cluster tiles of C^T through shared memory and keeps
// a running (best, index, second, index2, third) per row in registers.
//
// Scores are h_j - x.c_j with h_j = 0.5 ||c_j||^2 (the DAAL form); ties resolve to
// the lowest cluster index. Rows whose best/second gap lies inside the derived
// rounding bound are queued for an FP64 recheck when a queue is given.
#include "kmb_internal.cuh"

#include <float.h>

#include <algorithm>
#include <cstdlib>

namespace kmb {
namespace {

constexpr int BM = 128;  // rows per CTA
constexpr int BN = 128;  // clusters per N-tile
constexpr int BK = 8;    // contraction chunk
constexpr int NT = 256;  // threads
constexpr int PAD = 4;   // smem row padding (keeps 16-byte alignment, breaks bank conflicts)

template <typename F> struct Vec4;
template <> struct Vec4<float> { using T = float4; };
template <> struct Vec4<double> { using T = double4; };

template <typename F> __device__ __forceinline__ F f_inf();
template <> __device__ __forceinline__ float f_inf<float>() { return __int_as_float(0x7f800000); }
template <> __device__ __forceinline__ double f_inf<double>() { return __longlong_as_double(0x7ff0000000000000LL); }

template <typename F> __device__ __forceinline__ double unit_roundoff();
template <> __device__ __forceinline__ double unit_roundoff<float>() { return 5.9604644775390625e-8; }   // 2^-24
template <> __device__ __forceinline__ double unit_roundoff<double>() { return 1.1102230246251565e-16; } // 2^-53

// (value, index) lexicographic "less".
template <typename F>
__device__ __forceinline__ bool lex_less(F a, int ia, F b, int ib) {
    return a < b || (a == b && ia < ib);
}

// acc[i][j] += a[i] * b[j] for the thread's 8 x 8 tile; for float as packed
// pairs (fma.rn.f32x2: two correctly rounded FMAs, the same results as fmaf).
template <typename F>
__device__ __forceinline__ void fma_tile(F (&acc)[8][8], const F (&a)[8], const F (&b)[8]) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
}
template <>
__device__ __forceinline__ void fma_tile<float>(float (&acc)[8][8], const float (&a)[8], const float (&b)[8]) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float2 ai = make_float2(a[i], a[i]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float2 t = __ffma2_rn(ai, make_float2(b[2 * q], b[2 * q + 1]), make_float2(acc[i][2 * q], acc[i][2 * q + 1]));
            acc[i][2 * q] = t.x;
            acc[i][2 * q + 1] = t.y;
        }
    }
}

template <typename F>
struct RowTop {
    F b, s, t;   // best, second, third score
    int ib, is;  // best / second cluster index
};

template <typename F>
__device__ __forceinline__ void top_push(RowTop<F> &r, F v, int c) {
    // Columns arrive in increasing order within a thread, so strict '<' keeps
    // the lowest index on ties.
    if (v < r.b) {
        r.t = r.s;
        r.s = r.b;
        r.is = r.ib;
        r.b = v;
        r.ib = c;
    } else if (v < r.s) {
        r.t = r.s;
        r.s = v;
        r.is = c;
    } else if (v < r.t) {
        r.t = v;
    }
}

// top_push with selects instead of branches (the same result).
template <typename F>
__device__ __forceinline__ void top_push_sel(RowTop<F> &r, F v, int c) {
    const bool lb = v < r.b, ls = v < r.s, lt = v < r.t;
    r.t = ls ? r.s : (lt ? v : r.t);
    r.s = lb ? r.b : (ls ? v : r.s);
    r.is = lb ? r.ib : (ls ? c : r.is);
    r.b = lb ? v : r.b;
    r.ib = lb ? c : r.ib;
}

template <typename F>
__device__ __forceinline__ RowTop<F> top_merge(const RowTop<F> &x, const RowTop<F> &y) {
    // Merge two sorted triples ((value, index) order); indices are kept for the
    // first two places only. After o outputs a + b == o <= 2, so a, b < 3.
    const F xv[3] = {x.b, x.s, x.t}, yv[3] = {y.b, y.s, y.t};
    const int xi[3] = {x.ib, x.is, 0x7fffffff}, yi[3] = {y.ib, y.is, 0x7fffffff};
    F ov[3];
    int oi[3];
    int a = 0, b = 0;
#pragma unroll
    for (int o = 0; o < 3; ++o) {
        if (lex_less(xv[a], xi[a], yv[b], yi[b])) {
            ov[o] = xv[a];
            oi[o] = xi[a];
            ++a;
        } else {
            ov[o] = yv[b];
            oi[o] = yi[b];
            ++b;
        }
    }
    RowTop<F> r;
    r.b = ov[0];
    r.ib = oi[0];
    r.s = ov[1];
    r.is = oi[1];
    r.t = ov[2];
    return r;
}

// top_merge with selects instead of indexed arrays (the same result, the same
// comparisons in the same argument order).
template <typename F>
__device__ __forceinline__ RowTop<F> top_merge_sel(const RowTop<F> &x, const RowTop<F> &y) {
    constexpr int kNone = 0x7fffffff;  // index of a third place
    const bool c0 = lex_less(x.b, x.ib, y.b, y.ib);
    // second place: the heads of both lists after the first output
    const F xa = c0 ? x.s : x.b, ya = c0 ? y.b : y.s;
    const int xai = c0 ? x.is : x.ib, yai = c0 ? y.ib : y.is;
    const bool c1 = lex_less(xa, xai, ya, yai);
    // third place: x took both (x.t vs y.b), y took both (x.b vs y.t), or one each (x.s vs y.s)
    const bool xx = c0 && c1, yy = !c0 && !c1;
    const F xh = xx ? x.t : (yy ? x.b : x.s), yh = xx ? y.b : (yy ? y.t : y.s);
    const int xhi = xx ? kNone : (yy ? x.ib : x.is), yhi = xx ? y.ib : (yy ? kNone : y.is);
    const bool c2 = lex_less(xh, xhi, yh, yhi);
    RowTop<F> r;
    r.b = c0 ? x.b : y.b;
    r.ib = c0 ? x.ib : y.ib;
    r.s = c1 ? xa : ya;
    r.is = c1 ? xai : yai;
    r.t = c2 ? xh : yh;
    return r;
}

template <typename F>
__device__ __forceinline__ RowTop<F> shfl_top(const RowTop<F> &x, int mask) {
    RowTop<F> y;
    y.b = __shfl_xor_sync(0xffffffffu, x.b, mask);
    y.s = __shfl_xor_sync(0xffffffffu, x.s, mask);
    y.t = __shfl_xor_sync(0xffffffffu, x.t, mask);
    y.ib = __shfl_xor_sync(0xffffffffu, x.ib, mask);
    y.is = __shfl_xor_sync(0xffffffffu, x.is, mask);
    return y;
}

// float: two CTAs per SM (16 warps): the register cap of 128 costs a few spilled
// epilogue values but doubles the warps that hide the FMA and shared-memory
// latencies (10 % faster at d=128, k=1024 and 32 % at d=64, k=256).
// double: one CTA per SM. The 8 x 8 FP64 accumulators alone take 128 registers;
// under the 128 cap they spilled 3.5 KB per thread and ran at 2.9 TFLOP/s, with
// 254 registers the same launch runs at 15.4 TFLOP/s (d=128, k=1024).
template <typename F, bool VEC>
__global__ void __launch_bounds__(NT, sizeof(F) == 4 ? 2 : 1)
assign_plain_kernel(const F *__restrict__ X, int64_t n, int d, const F *__restrict__ Ct, const F *__restrict__ h,
                    int k, int kpad, const F *__restrict__ xnorm, const double *__restrict__ cnorm_max,
                    int32_t *__restrict__ labels, F *__restrict__ d2, RecheckEntry *__restrict__ queue,
                    LoopState *__restrict__ st) {
    if (st && st->done) return;
    using V4 = typename Vec4<F>::T;
    __shared__ __align__(16) F Xs[2][BK][BM + PAD];
    __shared__ __align__(16) F Cs[2][BK][BN + PAD];

    const int tid = threadIdx.x;
    const int ty = tid >> 4, tx = tid & 15;
    const int64_t row0 = (int64_t)blockIdx.x * BM;

    // Global-load mapping. X tile: 128 rows x 8 dims; thread -> row tid/2, dims (tid&1)*4..+3.
    const int lr = tid >> 1, lk = (tid & 1) * 4;
    const int64_t grow = row0 + lr;
    const bool row_ok = grow < n;
    const F *xrow = X + (row_ok ? grow : 0) * (int64_t)d;
    // C tile: 8 dims x 128 clusters; thread -> dim tid/32, clusters (tid&31)*4..+3.
    const int ck = tid >> 5, cn = (tid & 31) * 4;

    const int nk = (d + BK - 1) / BK;
    const int ntiles = kpad / BN;
    const int steps = nk * ntiles;

    F xr[4];
    V4 cr;
    auto gload = [&](int step) {
        const int nt = step / nk, kc = step - nt * nk;
        const int kb = kc * BK;
        if (VEC) {
            if (row_ok && kb + lk < d) {
                V4 v = *reinterpret_cast<const V4 *>(xrow + kb + lk);
                xr[0] = v.x; xr[1] = v.y; xr[2] = v.z; xr[3] = v.w;
            } else {
                xr[0] = xr[1] = xr[2] = xr[3] = F(0);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) xr[q] = (row_ok && kb + lk + q < d) ? xrow[kb + lk + q] : F(0);
        }
        // Ct has nk*BK rows (zero padded) and kpad columns.
        cr = *reinterpret_cast<const V4 *>(Ct + (int64_t)(kb + ck) * kpad + nt * BN + cn);
    };
    auto sstore = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 4; ++q) Xs[buf][lk + q][lr] = xr[q];
        *reinterpret_cast<V4 *>(&Cs[buf][ck][cn]) = cr;
    };

    RowTop<F> top[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        top[i].b = top[i].s = top[i].t = f_inf<F>();
        top[i].ib = 0;
        top[i].is = 0;
    }
    F acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = F(0);

    gload(0);
    sstore(0);
    __syncthreads();

    for (int step = 0; step < steps; ++step) {
        const int buf = step & 1;
        if (step + 1 < steps) gload(step + 1);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            F a[8], b[8];
            V4 a0 = *reinterpret_cast<const V4 *>(&Xs[buf][kk][ty * 4]);
            V4 a1 = *reinterpret_cast<const V4 *>(&Xs[buf][kk][64 + ty * 4]);
            V4 b0 = *reinterpret_cast<const V4 *>(&Cs[buf][kk][tx * 4]);
            V4 b1 = *reinterpret_cast<const V4 *>(&Cs[buf][kk][64 + tx * 4]);
            a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w;
            a[4] = a1.x; a[5] = a1.y; a[6] = a1.z; a[7] = a1.w;
            b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w;
            b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
            fma_tile(acc, a, b);
        }
        const int nt = step / nk;
        if (step - nt * nk == nk - 1) {
            // Epilogue of one N-tile: scores h_j - x.c_j into the running top-3.
            const int cbase = nt * BN;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int col = cbase + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
                const F hj = h[col];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    top_push_sel(top[i], hj - acc[i][j], col);
                    acc[i][j] = F(0);
                }
            }
        }
        if (step + 1 < steps) sstore(buf ^ 1);
        __syncthreads();
    }

    // Reduce across the 16 lanes (tx) that share the same rows.
#pragma unroll
    for (int i = 0; i < 8; ++i) {
#pragma unroll
        for (int m = 8; m >= 1; m >>= 1) top[i] = top_merge_sel(top[i], shfl_top(top[i], m));
    }
    if (tx == 0) {
        const double u = unit_roundoff<F>();
        const double cmax = cnorm_max ? *cnorm_max : 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int64_t r = row0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
            if (r >= n) continue;
            const RowTop<F> &t = top[i];
            labels[r] = t.ib;
            const F xn = xnorm[r];
            d2[r] = F(2) * t.b + xn;
            if (queue) {
                // |computed - exact| per score <= u*cmax^2 + (d+2)*u*||x||*cmax (+ slack);
                // the order of two scores is certain when their gap exceeds twice that.
                const double xl = sqrt(fmax((double)xn, 0.0));
                const double e = 1.0625 * u * (cmax * cmax + (double)(d + 2) * xl * cmax);
                const double band = 2.0 * e;
                if ((double)t.s - (double)t.b <= band)
                    enqueue_recheck(queue, n, st, (int)r, t.ib, t.is, (double)t.t - (double)t.b <= band);
            }
        }
    }
}

// Per-iteration centroid preparation: Ct (dpad x kpad, zero padded), h (kpad,
// +inf padding), max ||c|| (double).
template <typename F>
__global__ void prep_centroids_kernel(const F *__restrict__ C, int k, int d, int dpad, int kpad, F *__restrict__ Ct,
                                      F *__restrict__ h, double *__restrict__ cnorm_max, const LoopState *st) {
    if (st && st->done) return;
    __shared__ double red[32];
    const int j = blockIdx.x;  // one block per (padded) cluster
    double s = 0.0;
    for (int t = threadIdx.x; t < dpad; t += blockDim.x) {
        F v = (j < k && t < d) ? C[(int64_t)j * d + t] : F(0);
        Ct[(int64_t)t * kpad + j] = v;
        s += (double)v * (double)v;
    }
    for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        h[j] = (j < k) ? F(0.5 * tot) : f_inf<F>();
        if (j < k) {
            // max of non-negative doubles via the ordered integer view
            atomicMax(reinterpret_cast<unsigned long long *>(cnorm_max),
                      (unsigned long long)__double_as_longlong(sqrt(tot)));
        }
    }
}

// ||x||^2 per row: FP64 sum of squares (lane t, t+32, ...; then a butterfly),
// rounded to F. One warp per row, grid-stride over rows.
template <typename F>
__global__ void row_norms_kernel(const F *__restrict__ X, int64_t n, int d, F *__restrict__ xnorm) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += warps) {
        const F *x = X + row * d;
        double s = 0.0;
        for (int t = lane; t < d; t += 32) s += (double)x[t] * (double)x[t];
        for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
        if (lane == 0) xnorm[row] = F(s);
    }
}

__global__ void reset_double_kernel(double *p, const LoopState *st) {
    if (st && st->done) return;
    *p = 0.0;
}

constexpr int kSmallK = 32;        // clusters handled by assign_small_kernel
constexpr int kSmallThreads = 128;

// Few clusters (k <= 32, d <= 64): one row per thread, its d values in registers,
// all centroids in shared memory (read as broadcasts). The contraction of row and
// cluster accumulates x_t * c_t in ascending t, as the tiled kernel does, so the
// scores -- and the labels, distances and recheck entries -- are the same; only
// the 128-cluster tile padding and the tile epilogue are gone.
template <typename F, int DMAX>
__global__ void __launch_bounds__(kSmallThreads)
assign_small_kernel(const F *__restrict__ X, int64_t n, int d, const F *__restrict__ Ct, const F *__restrict__ h,
                    int k, int kpad, const F *__restrict__ xnorm, const double *__restrict__ cnorm_max,
                    int32_t *__restrict__ labels, F *__restrict__ d2, RecheckEntry *__restrict__ queue,
                    LoopState *__restrict__ st) {
    if (st && st->done) return;
    __shared__ __align__(16) F Cs[kSmallK][DMAX];
    __shared__ F hs[kSmallK];
    for (int i = threadIdx.x; i < kSmallK * DMAX; i += blockDim.x) {
        const int j = i / DMAX, t = i % DMAX;
        Cs[j][t] = (j < k && t < d) ? Ct[(int64_t)t * kpad + j] : F(0);
    }
    for (int j = threadIdx.x; j < kSmallK; j += blockDim.x) hs[j] = j < k ? h[j] : f_inf<F>();
    __syncthreads();
    const double u = unit_roundoff<F>();
    const double cmax = cnorm_max ? *cnorm_max : 0.0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        F x[DMAX];
        const F *xr = X + r * (int64_t)d;
#pragma unroll
        for (int t = 0; t < DMAX; ++t) x[t] = t < d ? xr[t] : F(0);
        RowTop<F> top;
        top.b = top.s = top.t = f_inf<F>();
        top.ib = top.is = 0;
        for (int j = 0; j < k; ++j) {
            F dot = F(0);
#pragma unroll
            for (int t = 0; t < DMAX; t += 4) {
                const typename Vec4<F>::T c = *reinterpret_cast<const typename Vec4<F>::T *>(&Cs[j][t]);
                dot = fma(x[t], c.x, dot);
                dot = fma(x[t + 1], c.y, dot);
                dot = fma(x[t + 2], c.z, dot);
                dot = fma(x[t + 3], c.w, dot);
            }
            top_push(top, hs[j] - dot, j);
        }
        labels[r] = top.ib;
        const F xn = xnorm[r];
        d2[r] = F(2) * top.b + xn;
        if (queue) {
            const double xl = sqrt(fmax((double)xn, 0.0));
            const double e = 1.0625 * u * (cmax * cmax + (double)(d + 2) * xl * cmax);
            const double band = 2.0 * e;
            if ((double)top.s - (double)top.b <= band)
                enqueue_recheck(queue, n, st, (int)r, top.ib, top.is, (double)top.t - (double)top.b <= band);
        }
    }
}

// ---- FP32, centroids resident in shared memory ------------------------------
// When the (padded) centroids -- all of them, or a chunk of them -- fit in shared
// memory next to the row stages, one persistent CTA per SM keeps C^T and the half
// norms resident and streams 64-row tiles of X through TMA, so no centroid byte is
// re-read per row tile. 16 warps in two groups of 8; each group owns every other
// 64-row tile (group g of CTA b takes tiles 2(b + i·grid) + g) and one or two TMA
// stages. In a group, warp w owns rows 8w..8w+7 of the tile, lane l the clusters
// 4l..4l+3 and 128+4l..128+4l+3 of each 256-cluster pass: the row values are
// shared-memory broadcasts and the centroid reads are conflict-free 16-byte
// loads. Per (row, cluster) the contraction accumulates x_t * c_t in ascending
// t with FMAs from zero, as assign_plain_kernel does, so the scores -- and the
// labels, distances and recheck entries -- are the same. After each pass a
// lane holds the top-3 of its 8 clusters for its warp's 8 rows; five exchange
// rounds halve the rows a lane keeps while merging in the partner's (value,
// index) triples, leaving each row's top-3 in four lanes; with more than one
// pass the row's owner lane merges it into the running top-3 in shared memory.
//
// Chunks: when all clusters do not fit, they are taken kchunk at a time (a
// multiple of 256). A CTA walks blocks of bt row tiles per group; for each chunk it
// loads the chunk's C^T and half norms (every warp past a CTA barrier before and
// after), then runs the block's tiles against it; the running top-3 of the block's
// rows stays in shared memory across chunks and passes (merged in ascending cluster
// order, as one long pass would), and the block's rows come back from L2 for every
// chunk (bt = 8: 1024 rows per CTA, 76 MB over the grid at d = 128).
//
// Ping-pong: the two groups take turns at the FMA pipe. A group runs a pass's
// contraction only in its turn and hands the turn over (named barriers 1 and 2)
// before its top-3 epilogue, so one group's epilogue (compares, selects,
// shuffles) issues beside the other group's FMAs instead of every warp of the SM
// reaching its epilogue at once and leaving the FMA pipe idle. Both groups take
// the same number of turns (a group without a tile left takes empty turns), so
// every barrier completes. With two stages per group the next tile's load is
// issued at the start of a tile's first turn (the turn barriers order the
// stage's last reads before it); with one stage, after the tile's last
// contraction, once the group's warps have met at named barrier 3 + g.
constexpr int kResThreads = 512;
constexpr int kResGroupThreads = 256;
constexpr int kResRows = 64;    // rows per tile (one group's)
constexpr int kResCtaRows = 128;  // rows per CTA step (both groups)
constexpr int kResPass = 256;
constexpr long long kResTimeout = 4000000000ll;  // ~2 s of SM clocks per wait

struct ResBarriers {
    uint64_t full[4];  // [group][stage]
    int abort;
    int issued[4];  // loads issued into each stage (the group's thread 0)
};

__device__ __forceinline__ uint32_t res_su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool res_try_wait(uint64_t *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(res_su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false after ~2 s (recorded in abort) or when another thread aborted.
__device__ __forceinline__ bool res_wait(uint64_t *b, uint32_t parity, volatile int *abort) {
    if (res_try_wait(b, parity)) return true;
    const long long t0 = clock64();
    while (!res_try_wait(b, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > kResTimeout) {
            *abort = 1;
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void res_load_tile(float *dst, const CUtensorMap *tm, uint64_t *bar, int row0,
                                              uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(res_su32(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            res_su32(dst)),
        "l"(tm), "r"(res_su32(bar)), "r"(0), "r"(row0)
        : "memory");
}

// Named barriers of the turn protocol: the waiting group's 256 threads sync, the
// other group's 256 arrive.
__device__ __forceinline__ void res_turn_wait(int id) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(kResThreads) : "memory");
}
__device__ __forceinline__ void res_turn_give(int id) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(kResThreads) : "memory");
}

// Keeps the rows of one half of `t` (hi: the upper half) and merges in the
// partner lane's triples of the same rows.
template <int R>
__device__ __forceinline__ void res_exchange(RowTop<float> (&t)[8], int mask, bool hi) {
#pragma unroll
    for (int q = 0; q < R / 2; ++q) {
        const RowTop<float> keep = hi ? t[R / 2 + q] : t[q];
        const RowTop<float> send = hi ? t[q] : t[R / 2 + q];
        t[q] = top_merge_sel(keep, shfl_top(send, mask));
    }
}

// DPADT > 0 fixes the padded row width at compile time (row and centroid offsets
// become immediates); 0 reads it from dpad. STAGES: TMA stages per group (1 or 2).
// kres: all clusters, padded to 256; kchunk: clusters resident at a time (kres when
// n_chunks == 1); bt: row tiles per block and group (the running top-3 rows).
// CHUNK false: all clusters resident (n_chunks = bt = 1 at compile time).
template <int DPADT, int STAGES, bool CHUNK>
__global__ void __launch_bounds__(kResThreads, 1)
assign_resident_kernel(const __grid_constant__ CUtensorMap tmX, int64_t n, int d, int dpad_rt, const float *__restrict__ Ct,
                       const float *__restrict__ h, int k, int kpad, int kres, int kchunk, int n_chunks_rt, int bt_rt,
                       const float *__restrict__ xnorm, const double *__restrict__ cnorm_max,
                       int32_t *__restrict__ labels, float *__restrict__ d2, RecheckEntry *__restrict__ queue,
                       LoopState *__restrict__ st) {
    __shared__ int s_skip;
    if (threadIdx.x == 0) s_skip = st ? st->done : 0;
    __syncthreads();
    if (s_skip) return;
    const int dpad = DPADT > 0 ? DPADT : dpad_rt;
    const int n_chunks = CHUNK ? n_chunks_rt : 1, bt = CHUNK ? bt_rt : 1;
    extern __shared__ uint8_t res_smem_raw[];
    uint8_t *sm = (uint8_t *)(((uintptr_t)res_smem_raw + 127) & ~(uintptr_t)127);
    const int tile_floats = kResRows * dpad;
    float *Xs = (float *)sm;                        // [group][stage][64][dpad]
    float *Cs = Xs + 2 * STAGES * tile_floats;      // [kchunk / 256][dpad][256]: pass-major blocks
    float *hs = Cs + (size_t)dpad * kchunk;         // [kchunk]
    RowTop<float> *run = (RowTop<float> *)(hs + kchunk);  // [group][bt][64] running top-3
    ResBarriers *bar = (ResBarriers *)(run + 2 * bt * kResRows);
    volatile int *abort = &bar->abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = warp >> 3, gw = warp & 7, gtid = tid & (kResGroupThreads - 1);
    // tiles of group g: 2 (b + i·grid) + g for i = 0 .. my_tiles - 1
    const int64_t n_tiles = (n + kResRows - 1) / kResRows;
    const int64_t par_tiles = (n_tiles - g + 1) / 2;     // tiles of parity g
    const int64_t par_tiles0 = (n_tiles + 1) / 2;        // of parity 0 (the most)
    const int grid = (int)gridDim.x, b = (int)blockIdx.x;
    const int my_tiles = par_tiles > b ? (int)((par_tiles - b + grid - 1) / grid) : 0;
    const int steps = par_tiles0 > b ? (int)((par_tiles0 - b + grid - 1) / grid) : 0;  // group 0's count
    const uint32_t tile_bytes = (uint32_t)tile_floats * 4u;
    float *Xg = Xs + STAGES * g * tile_floats;  // this group's stages
    uint64_t *full = &bar->full[2 * g];
    int *issued = &bar->issued[2 * g];
    if (tid == 0) {
        for (int i = 0; i < 4; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(res_su32(&bar->full[i])) : "memory");
            bar->issued[i] = 0;
        }
        bar->abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int m_issue = 0, m_wait = 0;  // this group's loads issued (its thread 0) and waited for
    if (gtid == 0 && my_tiles > 0) {
        res_load_tile(Xg, &tmX, &full[0], (int)((2 * (int64_t)b + g) * kResRows), tile_bytes);
        issued[0] = 1;
        m_issue = 1;
    }
    // Resident centroids of chunk q: C^T in 256-column blocks, one per pass, so a pass
    // reads rows 256 floats apart (zero columns past kpad), and the half norms (+inf
    // past kpad).
    auto load_chunk = [&](int q) {
        const int c0 = q * kchunk, kc = min(kchunk, kres - c0), kq = kc / 4;
        for (int i = tid; i < dpad * kq; i += kResThreads) {
            const int t = i / kq, c = 4 * (i - t * kq);
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (c0 + c < kpad) v = *reinterpret_cast<const float4 *>(Ct + (size_t)t * kpad + c0 + c);
            *reinterpret_cast<float4 *>(Cs + ((size_t)(c / kResPass) * dpad + t) * kResPass + (c % kResPass)) = v;
        }
        for (int j = tid; j < kc; j += kResThreads) hs[j] = c0 + j < kpad ? h[c0 + j] : f_inf<float>();
    };
    load_chunk(0);
    __syncthreads();

    const double u = 5.9604644775390625e-8;  // 2^-24
    const double cmax = cnorm_max ? *cnorm_max : 0.0;
    const int total_turns = steps * (kres / kResPass);  // the same for both groups
    // the row of the tile whose final top-3 this lane holds after the exchange
    const int own = 8 * gw + ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
    bool ok = true;
    int turn = 0;
    const int n_blocks = (steps + bt - 1) / bt;
    for (int blk = 0; blk < n_blocks; ++blk) {
        const int u_n = min(bt, steps - blk * bt);
        for (int q = 0; q < n_chunks; ++q) {
            if (n_chunks > 1 && (blk > 0 || q > 0)) {
                __syncthreads();  // every warp is done with the previous chunk's centroids
                load_chunk(q);
                __syncthreads();
            }
            const int c0 = q * kchunk;
            const int ppc = min(kchunk, kres - c0) / kResPass;
            for (int ut = 0; ut < u_n; ++ut) {
                const int lt = blk * bt + ut;
                const bool has = lt < my_tiles;
                const int64_t row0 = (2 * ((int64_t)b + (int64_t)lt * grid) + g) * kResRows;
                // the next tile this group loads: the next of the block, else the block's
                // first (next chunk), else the next block's first
                int nxt;
                if (ut + 1 < u_n && lt + 1 < my_tiles) nxt = lt + 1;
                else if (q + 1 < n_chunks) nxt = blk * bt;
                else nxt = (blk + 1) * bt;
                const bool nxt_has = has && nxt < my_tiles;
                RowTop<float> *grun = run + (g * bt + ut) * kResRows;
                // this tile's stage and load parity (all clusters resident: the group's
                // tiles are loaded in order, so its load count is lt)
                const int mw = CHUNK ? m_wait : lt;
                const int stage = mw % STAGES;
                const uint32_t parity = (uint32_t)(mw / STAGES) & 1u;
                if (has) ++m_wait;
                for (int pass = 0; pass < ppc; ++pass, ++turn) {
                    // wait for this group's turn at the FMA pipe: group 0 goes first
                    if (g == 0) {
                        if (turn > 0) res_turn_wait(1);
                    } else {
                        res_turn_wait(2);
                    }
                    if (pass == 0 && has) {
                        // Two stages: the next tile goes into the other stage, whose last
                        // reads (the previous tile's contractions) came before this group
                        // handed over its previous turn.
                        if (STAGES == 2 && gtid == 0 && ok && nxt_has) {
                            const int s2 = (CHUNK ? m_issue : lt + 1) % STAGES;
                            res_load_tile(Xg + s2 * tile_floats, &tmX, &full[s2],
                                          (int)((2 * ((int64_t)b + (int64_t)nxt * grid) + g) * kResRows), tile_bytes);
                            issued[s2] += 1;
                            ++m_issue;
                        }
                        if (ok && !__all_sync(0xffffffffu, res_wait(&full[stage], parity, abort))) ok = false;
                    }
                    const bool work = has && ok;
                    // Packed FP32 FMAs (fma.rn.f32x2: two correctly rounded FMAs, the same
                    // results as fmaf): each pair holds two of this lane's clusters for one
                    // row, with the row's value duplicated; one issue slot per two FMAs.
                    float2 acc2[8][4];  // acc2[i][q] = clusters 2q, 2q + 1 of this lane's eight
#pragma unroll
                    for (int i = 0; i < 8; ++i)
#pragma unroll
                        for (int q2 = 0; q2 < 4; ++q2) acc2[i][q2] = make_float2(0.f, 0.f);
                    if (work) {
                        const float *xa = Xg + stage * tile_floats + (8 * gw) * dpad;
                        const float *cb = Cs + (size_t)pass * dpad * kResPass + 4 * lane;
#pragma unroll 1
                        for (int t = 0; t < dpad; t += 2) {
                            float2 a[8];
#pragma unroll
                            for (int i = 0; i < 8; ++i) a[i] = *reinterpret_cast<const float2 *>(xa + i * dpad + t);
                            const float4 b00 = *reinterpret_cast<const float4 *>(cb + t * kResPass);
                            const float4 b01 = *reinterpret_cast<const float4 *>(cb + t * kResPass + 128);
                            const float4 b10 = *reinterpret_cast<const float4 *>(cb + (t + 1) * kResPass);
                            const float4 b11 = *reinterpret_cast<const float4 *>(cb + (t + 1) * kResPass + 128);
                            const float2 bx[4] = {make_float2(b00.x, b00.y), make_float2(b00.z, b00.w),
                                                  make_float2(b01.x, b01.y), make_float2(b01.z, b01.w)};
                            const float2 by[4] = {make_float2(b10.x, b10.y), make_float2(b10.z, b10.w),
                                                  make_float2(b11.x, b11.y), make_float2(b11.z, b11.w)};
#pragma unroll
                            for (int i = 0; i < 8; ++i) {
                                const float2 ax = make_float2(a[i].x, a[i].x);
#pragma unroll
                                for (int q2 = 0; q2 < 4; ++q2) acc2[i][q2] = __ffma2_rn(ax, bx[q2], acc2[i][q2]);
                            }
#pragma unroll
                            for (int i = 0; i < 8; ++i) {
                                const float2 ay = make_float2(a[i].y, a[i].y);
#pragma unroll
                                for (int q2 = 0; q2 < 4; ++q2) acc2[i][q2] = __ffma2_rn(ay, by[q2], acc2[i][q2]);
                            }
                        }
                    }
                    const bool last_pass = pass + 1 == ppc;
                    // One stage: the group's warps meet once the tile's last contraction is
                    // done (warp 0 waits, the others arrive), before the turn goes over.
                    if (STAGES == 1 && last_pass) {
                        if (gw == 0) asm volatile("bar.sync %0, %1;" ::"r"(3 + g), "r"(kResGroupThreads) : "memory");
                        else asm volatile("bar.arrive %0, %1;" ::"r"(3 + g), "r"(kResGroupThreads) : "memory");
                    }
                    // hand the FMA pipe to the other group (group 1's last turn has no taker)
                    if (g == 0) {
                        res_turn_give(2);
                    } else if (turn + 1 < total_turns) {
                        res_turn_give(1);
                    }
                    if (STAGES == 1 && last_pass && gtid == 0 && ok && nxt_has) {
                        res_load_tile(Xg, &tmX, &full[0], (int)((2 * ((int64_t)b + (int64_t)nxt * grid) + g) * kResRows),
                                      tile_bytes);
                        issued[0] += 1;
                        ++m_issue;
                    }
                    if (!work) continue;
                    float acc[8][8];
#pragma unroll
                    for (int i = 0; i < 8; ++i)
#pragma unroll
                        for (int q2 = 0; q2 < 4; ++q2) {
                            acc[i][2 * q2] = acc2[i][q2].x;
                            acc[i][2 * q2 + 1] = acc2[i][q2].y;
                        }
                    // this lane's clusters in ascending order: strict '<' keeps the lowest index
                    // on ties; row by row, so a row's scores are dead once its top-3 is built
                    float hv[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) hv[j] = hs[pass * kResPass + (j < 4 ? 4 * lane + j : 128 + 4 * lane + (j - 4))];
                    const int col0 = c0 + pass * kResPass + 4 * lane;
                    RowTop<float> top[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const float v0 = hv[0] - acc[i][0];
                        const bool l0 = v0 < f_inf<float>();  // a push into an empty triple
                        top[i].b = l0 ? v0 : f_inf<float>();
                        top[i].ib = l0 ? col0 : 0;
                        top[i].s = top[i].t = f_inf<float>();
                        top[i].is = 0;
#pragma unroll
                        for (int j = 1; j < 8; ++j) top_push_sel(top[i], hv[j] - acc[i][j], col0 + (j < 4 ? j : 124 + j));
                    }
                    res_exchange<8>(top, 16, (lane >> 4) & 1);
                    res_exchange<4>(top, 8, (lane >> 3) & 1);
                    res_exchange<2>(top, 4, (lane >> 2) & 1);
                    top[0] = top_merge_sel(top[0], shfl_top(top[0], 2));
                    top[0] = top_merge_sel(top[0], shfl_top(top[0], 1));
                    if ((lane & 3) == 0) {
                        RowTop<float> r = top[0];
                        if (q > 0 || pass > 0) r = top_merge_sel(grun[own], r);
                        if (q + 1 < n_chunks || !last_pass) {
                            grun[own] = r;
                        } else {
                            const int64_t row = row0 + own;
                            if (row < n) {
                                labels[row] = r.ib;
                                const float xn = xnorm[row];
                                d2[row] = 2.0f * r.b + xn;
                                if (queue) {
                                    const double xl = sqrt(fmax((double)xn, 0.0));
                                    const double e = 1.0625 * u * (cmax * cmax + (double)(d + 2) * xl * cmax);
                                    const double band = 2.0 * e;
                                    if ((double)r.s - (double)r.b <= band)
                                        enqueue_recheck(queue, n, st, (int)row, r.ib, r.is,
                                                        (double)r.t - (double)r.b <= band);
                                }
                            }
                        }
                    }
                }
            }
        }
    }
    __syncthreads();  // every wait of both groups has ended before abort is read
    if (gtid == 0) {
        if (*abort) {
            // leave no bulk copy landing in shared memory behind: wait (bounded) for
            // the last load this group issued into each of its stages
            for (int s2 = 0; s2 < STAGES; ++s2) {
                const int iss = issued[s2];
                if (!iss) continue;
                const long long t0 = clock64();
                while (!res_try_wait(&full[s2], (uint32_t)((iss - 1) & 1)) && clock64() - t0 < kResTimeout) {
                }
            }
            if (st) {
                st->error = KMB_ETIMEDOUT;
                st->done = 1;
            }
        }
    }
}

// Shared memory of assign_resident_kernel for dpad features, kchunk resident
// clusters, STAGES stages per group and bt running-top-3 tiles per group.
size_t resident_smem_bytes(int dpad, int kchunk, int stages, int bt) {
    return 128 + (size_t)2 * stages * kResRows * dpad * 4 + (size_t)dpad * kchunk * 4 + (size_t)kchunk * 4 +
           (size_t)2 * bt * kResRows * sizeof(RowTop<float>) + sizeof(ResBarriers);
}

}  // namespace

template <typename F>
void launch_prep_centroids(const F *C, int64_t k, int64_t d, int64_t kpad, F *Ct, F *h, double *cnorm_max,
                           const LoopState *st, cudaStream_t s) {
    const int dpad = (int)((d + BK - 1) / BK * BK);
    reset_double_kernel<<<1, 1, 0, s>>>(cnorm_max, st);
    KMB_LAUNCHED();
    prep_centroids_kernel<F><<<(unsigned)kpad, 128, 0, s>>>(C, (int)k, (int)d, dpad, (int)kpad, Ct, h, cnorm_max, st);
    KMB_LAUNCHED();
}

template <typename F>
void launch_row_norms(const F *X, int64_t n, int64_t d, F *xnorm, cudaStream_t s) {
    if (n == 0) return;
    const int64_t blocks = std::min<int64_t>((n * 32 + 255) / 256, 148 * 16);
    row_norms_kernel<F><<<(unsigned)blocks, 256, 0, s>>>(X, n, (int)d, xnorm);
    KMB_LAUNCHED();
}

template <typename F, int DMAX>
void launch_small(const F *X, int64_t n, int64_t d, const F *Ct, const F *h, int64_t k, int64_t kpad, const F *xnorm,
                  const double *cnorm_max, int32_t *labels, F *d2, RecheckEntry *queue, LoopState *st,
                  cudaStream_t s) {
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((n + kSmallThreads - 1) / kSmallThreads, 148 * 16));
    assign_small_kernel<F, DMAX><<<(unsigned)blocks, kSmallThreads, 0, s>>>(X, n, (int)d, Ct, h, (int)k, (int)kpad,
                                                                           xnorm, cnorm_max, labels, d2, queue, st);
    KMB_LAUNCHED();
}

// FP32 rows whose centroids -- all of them, or 256-cluster multiples at a time --
// fit in shared memory (d a multiple of 4 and at most 256, 16-byte aligned rows):
// the resident kernel. False when it does not apply.
template <typename F>
bool launch_resident(const F *, int64_t, int64_t, const F *, const F *, int64_t, int64_t, const F *, const double *,
                     int32_t *, F *, RecheckEntry *, LoopState *, cudaStream_t) {
    return false;
}
template <>
bool launch_resident<float>(const float *X, int64_t n, int64_t d, const float *Ct, const float *h, int64_t k,
                            int64_t kpad, const float *xnorm, const double *cnorm_max, int32_t *labels, float *d2,
                            RecheckEntry *queue, LoopState *st, cudaStream_t s) {
    if (d % 4 != 0 || d > 256 || (reinterpret_cast<uintptr_t>(X) % 16) != 0 || n > INT32_MAX - 2 * kResCtaRows)
        return false;
    const char *e = getenv("KMB_PLAIN_RESIDENT");
    if (e && e[0] == '0') return false;
    const int dpad = (int)((d + BK - 1) / BK * BK);  // the rows of Ct
    const int kres = (int)((kpad + kResPass - 1) / kResPass * kResPass);
    int dev = 0, optin = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // All clusters resident with two stages per group; else chunks of clusters, the
    // first of (stages, bt) = (2, 8), (2, 4), (1, 8), (1, 4) that holds 256 of them,
    // with the chunks evened out.
    int stages = 2, bt = 1, kchunk = kres;
    if (resident_smem_bytes(dpad, kres, 2, 1) > (size_t)optin) {
        const int opts[4][2] = {{2, 8}, {2, 4}, {1, 8}, {1, 4}};
        kchunk = 0;
        for (const auto &o : opts) {
            const size_t base = resident_smem_bytes(dpad, 0, o[0], o[1]);
            if (base >= (size_t)optin) continue;
            const int fit = (int)(((size_t)optin - base) / ((size_t)dpad * 4 + 4)) / kResPass * kResPass;
            if (fit >= kResPass) {
                stages = o[0];
                bt = o[1];
                kchunk = std::min(fit, kres);
                break;
            }
        }
        if (kchunk == 0) return false;
        const int nc = (kres + kchunk - 1) / kchunk;
        kchunk = (kres / kResPass + nc - 1) / nc * kResPass;
    }
    const int n_chunks = (kres + kchunk - 1) / kchunk;
    const size_t smem = resident_smem_bytes(dpad, kchunk, stages, bt);
    if (smem > (size_t)optin) return false;
    CUtensorMap tm;
    // box: 64 rows x dpad columns (columns past d read as zeros)
    if (!encode_tensor_map_2d(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, X, (uint64_t)d, (uint64_t)n, (uint64_t)d * 4,
                              (uint32_t)dpad, (uint32_t)kResRows, CU_TENSOR_MAP_SWIZZLE_NONE))
        return false;
    auto pick = [&](auto k32, auto k64, auto k128, auto k0) { return dpad == 32 ? k32 : dpad == 64 ? k64 : dpad == 128 ? k128 : k0; };
    auto kern = n_chunks == 1 && bt == 1
                    ? pick(assign_resident_kernel<32, 2, false>, assign_resident_kernel<64, 2, false>,
                           assign_resident_kernel<128, 2, false>, assign_resident_kernel<0, 2, false>)
                : stages == 2 ? pick(assign_resident_kernel<32, 2, true>, assign_resident_kernel<64, 2, true>,
                                     assign_resident_kernel<128, 2, true>, assign_resident_kernel<0, 2, true>)
                              : pick(assign_resident_kernel<32, 1, true>, assign_resident_kernel<64, 1, true>,
                                     assign_resident_kernel<128, 1, true>, assign_resident_kernel<0, 1, true>);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const int64_t n_steps = (n + kResCtaRows - 1) / kResCtaRows;  // 128-row steps: two tiles, one per group
    const int grid = (int)std::min<int64_t>(n_steps, sms);
    kern<<<grid, kResThreads, smem, s>>>(tm, n, (int)d, dpad, Ct, h, (int)k, (int)kpad, kres, kchunk, n_chunks, bt,
                                         xnorm, cnorm_max, labels, d2, queue, st);
    KMB_LAUNCHED();
    return true;
}

template <typename F>
void launch_assign_plain(const F *X, int64_t n, int64_t d, const F *Ct, const F *h, int64_t k, int64_t kpad,
                         const F *xnorm, const double *cnorm_max, int32_t *labels, F *d2, RecheckEntry *queue,
                         LoopState *st, cudaStream_t s) {
    if (n == 0) return;
    if (k <= kSmallK && d <= 64) {  // few clusters: row per thread, centroids in shared memory
        if (d <= 16) launch_small<F, 16>(X, n, d, Ct, h, k, kpad, xnorm, cnorm_max, labels, d2, queue, st, s);
        else if (d <= 32) launch_small<F, 32>(X, n, d, Ct, h, k, kpad, xnorm, cnorm_max, labels, d2, queue, st, s);
        else launch_small<F, 64>(X, n, d, Ct, h, k, kpad, xnorm, cnorm_max, labels, d2, queue, st, s);
        return;
    }
    if (launch_resident(X, n, d, Ct, h, k, kpad, xnorm, cnorm_max, labels, d2, queue, st, s)) return;
    const unsigned blocks = (unsigned)((n + BM - 1) / BM);
    const bool vec = (d % 4 == 0) && ((reinterpret_cast<uintptr_t>(X) % (4 * sizeof(F))) == 0);
    if (vec) {
        assign_plain_kernel<F, true><<<blocks, NT, 0, s>>>(X, n, (int)d, Ct, h, (int)k, (int)kpad, xnorm, cnorm_max,
            labels, d2, queue, st);
        KMB_LAUNCHED();
    } else {
        assign_plain_kernel<F, false><<<blocks, NT, 0, s>>>(X, n, (int)d, Ct, h, (int)k, (int)kpad, xnorm, cnorm_max,
            labels, d2, queue, st);
        KMB_LAUNCHED();
    }
}

#define KMB_INST(F)                                                                                                \
    template void launch_prep_centroids<F>(const F *, int64_t, int64_t, int64_t, F *, F *, double *,            \
                                           const LoopState *, cudaStream_t);                                     \
    template void launch_row_norms<F>(const F *, int64_t, int64_t, F *, cudaStream_t);                                            \
    template void launch_assign_plain<F>(const F *, int64_t, int64_t, const F *, const F *, int64_t, int64_t,    \
                                         const F *, const double *, int32_t *, F *, RecheckEntry *, LoopState *, \
                                         cudaStream_t);
KMB_INST(float)
KMB_INST(double)
#undef KMB_INST

}  // namespace kmb
