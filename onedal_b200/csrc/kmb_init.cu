// k-means++ initialisation on the GPU with the reference's exact semantics:
// DAAL's dense plusPlus init with one trial, as oneDAL's train() runs it when
// no initial centroids are given (cpp/oneapi/dal/algo/kmeans/detail/
// train_init_centroids.hpp:47-74; cpp/daal/src/algorithms/kmeans/
// kmeans_plusplus_init_impl.i:538-673).
//
// Everything that decides which row becomes a center is computed in F with
// the reference's order of operations, so the chosen rows are the same:
//   * per row, d2 = sum_i (x_i - c_i)^2 in coordinate order, each step an FMA
//     (the reference's loop is an `omp simd` reduction whose lane split is the
//     compiler's; it moves d2 by ulps, and a chosen row only when the sample
//     falls within rounding of a boundary); the running minimum keeps the old
//     value on ties;
//   * per 512-row block, the sum of the minima in row order; the overall sum
//     in block order;
//   * the sample overall * p walks the block sums, then the block's rows;
//     a row whose minimum is <= 0.1 * overall / n is resampled with the next
//     uniform draw.
// The host draws the uniforms with the reference's generator (std::mt19937,
// std::uniform_real_distribution<F>(0, 1)); the device consumes them in the
// same order. Parallel work is per row (the distance update, coalesced through
// shared memory) and per block (one thread sums a block's 512 minima); the
// sequential folds (overall sum, sampling walk) run in one thread of a CTA whose
// other warps stage the block sums into shared memory, so a round needs no host
// round trip.
#include "kmb_internal.cuh"

#include <algorithm>
#include <cfloat>

namespace kmb {
namespace {

constexpr int kPPBlock = 512;  // DAAL's rows per block (kmeans_plusplus_init_impl.i:52)

template <typename F> __device__ __forceinline__ F f_max();
template <> __device__ __forceinline__ float f_max<float>() { return FLT_MAX; }
template <> __device__ __forceinline__ double f_max<double>() { return DBL_MAX; }

template <typename F>
__global__ void pp_fill_kernel(F *__restrict__ md, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        md[i] = f_max<F>();
}

// One CTA per 512-row block, 16 warps x 32 rows, each lane owning one row's
// distance. Rows are staged through shared memory one 128-byte segment per row
// at a time (W columns; a warp load instruction covers 32/W rows, fully
// coalesced), and the next segment's loads are in flight while the current one
// is folded, so each warp keeps 4 KB of loads outstanding. Each lane folds its
// row's columns in coordinate order; thread 0 then sums the block's minima in
// row order. Rows narrower than one segment are read directly (the warp's 32
// rows are one contiguous range, so the lanes' reads share cache lines).
template <typename F>
__global__ void __launch_bounds__(kPPBlock, 2) pp_update_kernel(const F *__restrict__ X, int64_t n, int d,
                                                                const F *__restrict__ center, F *__restrict__ md,
                                                                F *__restrict__ acc, const PPState *st) {
    constexpr int W = 128 / (int)sizeof(F);  // columns per segment
    constexpr int RPI = 32 / W;              // rows per warp load instruction
    constexpr int NLD = 32 / RPI;            // load instructions per 32-row segment
    if (st->stopped) return;
    extern __shared__ __align__(16) unsigned char pp_smem[];
    F(*tile)[32][W + 1] = reinterpret_cast<F(*)[32][W + 1]>(pp_smem);  // [16 warps][32 rows][W + pad]
    F *s_md = reinterpret_cast<F *>(pp_smem) + 16 * 32 * (W + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r0 = (int64_t)blockIdx.x * kPPBlock + warp * 32;
    const int64_t row = r0 + lane;
    F d2 = F(0);
    if (d < W) {
        if (row < n) {
            const F *x = X + row * d;
            for (int i = 0; i < d; ++i) {
                const F t = x[i] - center[i];
                d2 = fma(t, t, d2);
            }
        }
    } else {
        const int sub = lane / W, col = lane % W;
        F v[NLD];
        auto load_segment = [&](int c0) {
            const int c = c0 + col;
#pragma unroll
            for (int j = 0; j < NLD; ++j) {
                const int64_t r = r0 + j * RPI + sub;
                v[j] = (r < n && c < d) ? X[r * d + c] : F(0);
            }
        };
        load_segment(0);
        for (int c0 = 0; c0 < d; c0 += W) {
#pragma unroll
            for (int j = 0; j < NLD; ++j) tile[warp][j * RPI + sub][col] = v[j];
            __syncwarp();
            if (c0 + W < d) load_segment(c0 + W);
            const F cv = c0 + col < d ? center[c0 + col] : F(0);
            const int cols = min(W, d - c0);
            for (int i = 0; i < cols; ++i) {
                const F t = tile[warp][lane][i] - __shfl_sync(0xffffffffu, cv, i);
                d2 = fma(t, t, d2);
            }
            __syncwarp();
        }
    }
    F m = F(0);
    if (row < n) {
        const F old = md[row];
        m = !(d2 < old) ? old : d2;  // the reference's min(best, d2)
        md[row] = m;
    }
    s_md[threadIdx.x] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        const int64_t b0 = (int64_t)blockIdx.x * kPPBlock;
        const int cnt = (int)((n - b0) < (int64_t)kPPBlock ? (n - b0) : (int64_t)kPPBlock);
        F sum = F(0);
        for (int i = 0; i < cnt; ++i) sum += s_md[i];
        acc[blockIdx.x] = sum;
    }
}

constexpr int kSelThreads = 1024;

// Sequential walk of the block sums for thread 0 over a[lo, hi): advances while
// s >= a[j], subtracting, exactly as the scalar loop would; eight steps at a
// time are computed speculatively and kept when all eight pass.
template <typename F>
__device__ __forceinline__ int64_t walk_span(const F *a, int64_t lo, int64_t hi, F &s) {
    int64_t j = lo;
    F t = s;
    while (j + 8 <= hi) {
        F u[9];
        u[0] = t;
        bool all = true;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            all = all & (u[q] >= a[j + q]);
            u[q + 1] = u[q] - a[j + q];
        }
        if (!all) break;
        t = u[8];
        j += 8;
    }
    while (j < hi && t >= a[j]) {
        t -= a[j];
        ++j;
    }
    s = t;
    return j;
}

// Round c's sequential part in one CTA: the overall sum of the block sums, the
// sampling walk (block sums, then the chosen block's rows) with resampling,
// and the new center. The block sums stream through two shared-memory chunks:
// warps 1.. load chunk q + 1 while thread 0 folds chunk q.
template <typename F>
__global__ void __launch_bounds__(kSelThreads) pp_select_kernel(const F *__restrict__ X, int64_t n, int d, int64_t nb,
                                                                const F *__restrict__ acc, F *__restrict__ md,
                                                                const F *__restrict__ probs,
                                                                const F *__restrict__ pool, int pool_n, int64_t c,
                                                                F *__restrict__ C, PPState *st) {
    constexpr int CH = 16384 / (int)sizeof(F);  // elements per chunk
    __shared__ __align__(16) F buf[2][CH];
    __shared__ __align__(16) F rows[kPPBlock];
    __shared__ F s_val;          // overall sum, then the walk's remainder
    __shared__ long long s_pos;  // chosen block, then chosen row (-1: give up)
    __shared__ int s_flag;
    const int tid = threadIdx.x;
    if (st->stopped) return;
    const int64_t nchunks = (nb + CH - 1) / CH;
    auto load_chunk = [&](int64_t q, int t0, int nt) {
        const int64_t lo = q * CH, cnt = min((int64_t)CH, nb - lo);
        for (int64_t i = t0; i < cnt; i += nt) buf[q & 1][i] = acc[lo + i];
    };
    // overall = acc[0] + acc[1] + ... in block order
    load_chunk(0, tid, kSelThreads);
    __syncthreads();
    F overall = F(0);
    for (int64_t q = 0; q < nchunks; ++q) {
        if (tid >= 32 && q + 1 < nchunks) load_chunk(q + 1, tid - 32, kSelThreads - 32);
        if (tid == 0) {
            const int64_t cnt = min((int64_t)CH, nb - q * CH);
            const F *a = buf[q & 1];
            int64_t i = 0;
            for (; i + 8 <= cnt; i += 8) {
#pragma unroll
                for (int u = 0; u < 8; ++u) overall += a[i + u];
            }
            for (; i < cnt; ++i) overall += a[i];
        }
        __syncthreads();
    }
    if (tid == 0) {
        s_val = overall;
        s_flag = 0;
    }
    __syncthreads();
    overall = s_val;
    if (!(overall > F(0)) || !(overall <= f_max<F>())) {
        // every remaining distance is zero (fewer than k distinct rows) or the sum is not
        // finite: no draw can ever succeed, the reference would sample forever
        if (tid == 0) {
            st->stopped = 2;
            st->stop_round = c;
        }
        return;
    }
    const F eps = F(0.1) * overall / F(n);
    F p = probs[c];
    int used = st->pool_used;
    __syncthreads();  // every thread has read pool_used before thread 0 may change it
    for (;;) {
        // walk the block sums: advance while b + 1 < nb and sample >= acc[b]
        F s = overall * p;
        if (tid == 0) s_flag = 0;
        load_chunk(0, tid, kSelThreads);
        __syncthreads();
        for (int64_t q = 0; q < nchunks; ++q) {
            if (tid >= 32 && q + 1 < nchunks) load_chunk(q + 1, tid - 32, kSelThreads - 32);
            if (tid == 0) {
                const int64_t lo = q * CH, hi = min(lo + CH, nb - 1);
                const int64_t j = lo < hi ? lo + walk_span(buf[q & 1], 0, hi - lo, s) : lo;
                if (j < hi || hi == nb - 1) {
                    s_pos = j;
                    s_val = s;
                    s_flag = 1;
                }
            }
            __syncthreads();
            if (s_flag) break;
        }
        const int64_t b = s_pos;
        const int64_t s0 = b * kPPBlock, cnt = (b == nb - 1) ? n - s0 : kPPBlock;
        for (int64_t i = tid; i < cnt; i += kSelThreads) rows[i] = md[s0 + i];
        __syncthreads();
        if (tid == 0) {
            F r_s = s_val;
            const int64_t r = walk_span(rows, 0, cnt - 1, r_s);
            if (rows[r] > eps) {
                s_pos = s0 + r;
                s_flag = 2;
            } else if (used >= pool_n) {  // out of uniforms: the host refills and resumes at round c
                st->stopped = 1;
                st->stop_round = c;
                st->pool_used = used;
                s_flag = 3;
            } else {
                s_val = pool[used];
                s_flag = 4;
            }
        }
        __syncthreads();
        const int flag = s_flag;
        if (flag == 3) return;
        if (flag == 2) break;
        p = s_val;
        ++used;
        __syncthreads();  // s_val / s_flag are rewritten by the next attempt
    }
    const int64_t row = s_pos;
    for (int i = tid; i < d; i += kSelThreads) C[c * d + i] = X[row * d + i];
    if (tid == 0) {
        md[row] = F(0);
        st->pool_used = used;
        st->rows_chosen += 1;
    }
}

template <typename F>
__global__ void pp_first_kernel(const F *__restrict__ X, int d, int64_t row, F *__restrict__ C) {
    for (int i = threadIdx.x; i < d; i += blockDim.x) C[i] = X[row * d + i];
}

}  // namespace

template <typename F>
void launch_pp_fill(F *md, int64_t n, cudaStream_t s) {
    pp_fill_kernel<F><<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 8), 256, 0, s>>>(md, n);
    KMB_LAUNCHED();
}

template <typename F>
void launch_pp_first(const F *X, int64_t d, int64_t row, F *C, cudaStream_t s) {
    pp_first_kernel<F><<<1, 128, 0, s>>>(X, (int)d, row, C);
    KMB_LAUNCHED();
}

// Rounds c_begin .. k-1; `update_first` = false when the distances already
// include center c_begin - 1 (a resumed round).
template <typename F>
void launch_pp_rounds(const F *X, int64_t n, int64_t d, int64_t k, int64_t c_begin, bool update_first, F *md, F *acc,
                      const F *probs, const F *pool, int pool_n, F *C, PPState *st, cudaStream_t s) {
    const int64_t nb = (n + kPPBlock - 1) / kPPBlock;
    const size_t smem = sizeof(F) * (16 * 32 * (128 / sizeof(F) + 1) + kPPBlock);
    cudaFuncSetAttribute(pp_update_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    for (int64_t c = c_begin; c < k; ++c) {
        if (c > c_begin || update_first) {
            pp_update_kernel<F><<<(unsigned)nb, kPPBlock, smem, s>>>(X, n, (int)d, C + (c - 1) * d, md, acc, st);
            KMB_LAUNCHED();
        }
        pp_select_kernel<F><<<1, kSelThreads, 0, s>>>(X, n, (int)d, nb, acc, md, probs, pool, pool_n, c, C, st);
        KMB_LAUNCHED();
    }
}

#define KMB_PP_INST(F)                                                                                               \
    template void launch_pp_fill<F>(F *, int64_t, cudaStream_t);                                                    \
    template void launch_pp_first<F>(const F *, int64_t, int64_t, F *, cudaStream_t);                               \
    template void launch_pp_rounds<F>(const F *, int64_t, int64_t, int64_t, int64_t, bool, F *, F *, const F *,     \
                                      const F *, int, F *, PPState *, cudaStream_t);
KMB_PP_INST(float)
KMB_PP_INST(double)
#undef KMB_PP_INST

}  // namespace kmb
