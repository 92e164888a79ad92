// k-means++ initialisation on the GPU with the reference's exact semantics:
// DAAL's dense plusPlus init with one trial, as oneDAL's train() runs it when
// no initial centroids are given (cpp/oneapi/dal/algo/kmeans/detail/
// train_init_centroids.hpp:47-74; cpp/daal/src/algorithms/kmeans/
// kmeans_plusplus_init_impl.i:538-673).
//
// Everything that decides which row becomes a center is computed in F with
// the reference's order of operations, so the chosen rows are the same:
//   * per row, d2 = sum_i (x_i - c_i)^2 in coordinate order, each step an FMA;
//     the running minimum keeps the old value on ties;
//   * per 512-row block, the sum of the minima in row order; the overall sum
//     in block order;
//   * the sample overall * p walks the block sums, then the block's rows;
//     a row whose minimum is <= 0.1 * overall / n is resampled with the next
//     uniform draw.
// The host draws the uniforms with the reference's generator (std::mt19937,
// std::uniform_real_distribution<F>(0, 1)); the device consumes them in the
// same order. Parallel work is per row (the distance update, coalesced through
// shared memory) and per block (one thread sums a block's 512 minima); the
// sequential steps run in one thread, so a round needs no host round trip.
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

// One CTA per 512-row block, 16 warps x 32 rows. Rows are staged through
// shared memory 32 columns at a time (coalesced loads), then each lane folds
// its row's columns in order.
template <typename F>
__global__ void __launch_bounds__(kPPBlock) pp_update_kernel(const F *__restrict__ X, int64_t n, int d,
                                                             const F *__restrict__ center, F *__restrict__ md,
                                                             F *__restrict__ acc, const PPState *st) {
    if (st->stopped) return;
    extern __shared__ __align__(16) unsigned char pp_smem[];
    F(*tile)[32][33] = reinterpret_cast<F(*)[32][33]>(pp_smem);  // [16 warps][32 rows][32 columns + pad]
    F *s_md = reinterpret_cast<F *>(pp_smem) + 16 * 32 * 33;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r0 = (int64_t)blockIdx.x * kPPBlock + warp * 32;
    const int64_t row = r0 + lane;
    F d2 = F(0);
    for (int c0 = 0; c0 < d; c0 += 32) {
        const int c = c0 + lane;
        const F cv = c < d ? center[c] : F(0);
#pragma unroll 4
        for (int j = 0; j < 32; ++j) {
            const int64_t r = r0 + j;
            tile[warp][j][lane] = (r < n && c < d) ? X[r * d + c] : F(0);
        }
        __syncwarp();
        const int cols = min(32, d - c0);
        for (int i = 0; i < cols; ++i) {
            const F t = tile[warp][lane][i] - __shfl_sync(0xffffffffu, cv, i);
            d2 = fma(t, t, d2);
        }
        __syncwarp();
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

// Round c's sequential part (one thread): overall error, sampling with
// resampling, and the new center.
template <typename F>
__global__ void pp_select_kernel(const F *__restrict__ X, int64_t n, int d, int64_t nb, const F *__restrict__ acc,
                                 F *__restrict__ md, const F *__restrict__ probs, const F *__restrict__ pool,
                                 int pool_n, int64_t c, F *__restrict__ C, PPState *st) {
    if (st->stopped) return;
    F overall = acc[0];
    for (int64_t b = 1; b < nb; ++b) overall += acc[b];
    const F big = sizeof(F) == 4 ? F(FLT_MAX) : F(DBL_MAX);
    if (!(overall > F(0)) || !(overall <= big)) {
        // every remaining distance is zero (fewer than k distinct rows) or the sum is not
        // finite: no draw can ever succeed, the reference would sample forever
        st->stopped = 2;
        st->stop_round = c;
        return;
    }
    const F eps = F(0.1) * overall / F(n);
    F p = probs[c];
    int64_t row;
    for (;;) {
        F sample = overall * p;
        int64_t b = 0;
        for (; b + 1 < nb && sample >= acc[b]; ++b) sample -= acc[b];
        const int64_t s0 = b * kPPBlock, cnt = (b == nb - 1) ? n - s0 : kPPBlock;
        int64_t r = 0;
        for (; r + 1 < cnt && sample >= md[s0 + r]; ++r) sample -= md[s0 + r];
        row = s0 + r;
        if (md[row] > eps) break;
        if (st->pool_used >= pool_n) {  // out of uniforms: the host refills and resumes at round c
            st->stopped = 1;
            st->stop_round = c;
            return;
        }
        p = pool[st->pool_used++];
    }
    md[row] = F(0);
    for (int i = 0; i < d; ++i) C[c * d + i] = X[row * d + i];
    st->rows_chosen += 1;
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
    const size_t smem = sizeof(F) * (16 * 32 * 33 + kPPBlock);
    cudaFuncSetAttribute(pp_update_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    for (int64_t c = c_begin; c < k; ++c) {
        if (c > c_begin || update_first) {
            pp_update_kernel<F><<<(unsigned)nb, kPPBlock, smem, s>>>(X, n, (int)d, C + (c - 1) * d, md, acc, st);
            KMB_LAUNCHED();
        }
        pp_select_kernel<F><<<1, 1, 0, s>>>(X, n, (int)d, nb, acc, md, probs, pool, pool_n, c, C, st);
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
