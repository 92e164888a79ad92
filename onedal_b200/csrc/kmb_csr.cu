// CSR rows for kmeans::method::lloyd_csr: index preparation, the assignment
// pass and the exact objective. The update (counting sort, FP64 piece sums,
// reseeding, shift) is kmb_update.cu's with its CSR row source.
//
// Reference semantics (DAAL CSR Lloyd, cpp/daal/src/algorithms/kmeans/):
//  - x.c_j over the row's stored entries (sparse product, kmeans_lloyd_impl.i:300-301)
//  - argmin of 0.5||c_j||^2 - x.c_j, lowest index on ties (:304-318)
//  - squared distance 2*min + sum of the row's v^2 in entry order (:320-328)
//  - exact objective: per row sum over stored entries of (x^2 - 2xc) + ||c||^2,
//    clipped at zero (kmeans_lloyd_postprocessing.h:276-347)
//
// B200 design. One warp per row: the row's entries are read 32 at a time and
// broadcast by shuffles; lane l owns clusters c0 + l + 32t (t < T) of a chunk of
// 32T clusters (T <= 16; wider k takes several passes over the row's entries),
// so each entry costs T coalesced 128-byte reads of the
// transposed centroids (d x kpad, L2-resident for moderate d*k) and T FMAs per
// lane. The running minimum is lane-local in ascending cluster order, then a
// warp reduction breaks ties by the lower index. The objective is FP64 with a
// fixed reduction order (deterministic).
#include "kmb_internal.cuh"

#include <algorithm>

namespace kmb {
namespace {

constexpr int kCsrObjectiveBlocks = 148 * 4;

__global__ void csr_prepare_kernel(const int64_t *__restrict__ cols_in, const int64_t *__restrict__ rowptr_in,
                                   int64_t n, int64_t d, int64_t nnz, int base, int32_t *__restrict__ cols_out,
                                   int64_t *__restrict__ rowptr_out, int *bad) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r0 = rowptr_in[i] - base, r1 = rowptr_in[i + 1] - base;
        if ((i == 0 && r0 != 0) || r0 < 0 || r1 < r0 || r1 > nnz) {
            atomicOr(bad, 1);
            continue;
        }
        rowptr_out[i] = r0;
        if (i == n - 1) rowptr_out[n] = r1;
        int64_t prev = -1;
        for (int64_t e = r0; e < r1; ++e) {
            const int64_t c = cols_in[e] - base;
            if (c < 0 || c >= d || c <= prev) {
                atomicOr(bad, 2);
                break;
            }
            cols_out[e] = (int32_t)c;
            prev = c;
        }
    }
}

// G entries are gathered before any of them is folded, so G * T loads per lane
// are in flight (the folds stay in entry order per accumulator).
template <typename F, int T, int G>
__global__ void __launch_bounds__(256) csr_assign_kernel(const F *__restrict__ vals, const int32_t *__restrict__ cols,
                                                         const int64_t *__restrict__ rowptr, int64_t n,
                                                         const F *__restrict__ Ct, const F *__restrict__ h, int kpad,
                                                         int32_t *__restrict__ labels, F *__restrict__ d2,
                                                         const LoopState *st) {
    if (st && st->done) return;
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += nwarps) {
        const int64_t rs = rowptr[i], re = rowptr[i + 1];
        F best = F(INFINITY);
        int bidx = 0;
        for (int c0 = 0; c0 < kpad; c0 += 32 * T) {
            F acc[T];
#pragma unroll
            for (int t = 0; t < T; ++t) acc[t] = F(0);
            for (int64_t e0 = rs; e0 < re; e0 += 32) {
                const int64_t e = e0 + lane;
                const F v = e < re ? vals[e] : F(0);
                const int col = e < re ? cols[e] : 0;
                const int cnt = (int)min((int64_t)32, re - e0);
                for (int q = 0; q < cnt; q += G) {
                    F vq[G], x[G][T];
#pragma unroll
                    for (int g = 0; g < G; ++g) {
                        // entries past the row's end fold 0 * (a valid centroid value): no change
                        const int qq = (q + g) & 31;
                        const F vg = __shfl_sync(0xffffffffu, v, qq);
                        const int cg = __shfl_sync(0xffffffffu, col, qq);
                        vq[g] = q + g < cnt ? vg : F(0);
                        const F *crow = Ct + (int64_t)(q + g < cnt ? cg : 0) * kpad + c0 + lane;
#pragma unroll
                        for (int t = 0; t < T; ++t) x[g][t] = c0 + 32 * t < kpad ? crow[32 * t] : F(0);
                    }
#pragma unroll
                    for (int g = 0; g < G; ++g)
#pragma unroll
                        for (int t = 0; t < T; ++t) acc[t] = fma(vq[g], x[g][t], acc[t]);
                }
            }
#pragma unroll
            for (int t = 0; t < T; ++t) {
                const int j = c0 + 32 * t + lane;
                if (c0 + 32 * t < kpad) {
                    const F s = h[j] - acc[t];
                    if (s < best) {
                        best = s;
                        bidx = j;
                    }
                }
            }
        }
        for (int m = 16; m >= 1; m >>= 1) {
            const F ob = __shfl_xor_sync(0xffffffffu, best, m);
            const int oi = __shfl_xor_sync(0xffffffffu, bidx, m);
            if (ob < best || (ob == best && oi < bidx)) {
                best = ob;
                bidx = oi;
            }
        }
        if (lane == 0) {
            labels[i] = bidx;
            F g = best * F(2);
            for (int64_t e = rs; e < re; ++e) g += vals[e] * vals[e];
            d2[i] = g;
        }
    }
}

__global__ void cnorm2_kernel(const void *Cv, int fsize, int d, double *__restrict__ out) {
    __shared__ double red[32];
    const int j = blockIdx.x;
    double s = 0.0;
    for (int t = threadIdx.x; t < d; t += blockDim.x) {
        const double c = fsize == 4 ? (double)((const float *)Cv)[(int64_t)j * d + t]
                                    : ((const double *)Cv)[(int64_t)j * d + t];
        s += c * c;
    }
    for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        out[j] = tot;
    }
}

// Block b owns a contiguous range of rows; warp w takes every 8th row of it.
template <typename F>
__global__ void __launch_bounds__(256) csr_objective_kernel(const F *__restrict__ vals, const int32_t *__restrict__ cols,
                                                            const int64_t *__restrict__ rowptr, int64_t n, int d,
                                                            const F *__restrict__ C, const int32_t *__restrict__ labels,
                                                            const double *__restrict__ cnorm2,
                                                            double *__restrict__ partials) {
    __shared__ double wsum[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t b = (int64_t)blockIdx.x * per, e = min(n, b + per);
    double mine = 0.0;
    for (int64_t i = b + warp; i < e; i += 8) {
        const int64_t a = labels[i];
        double r = 0.0;
        for (int64_t x = rowptr[i] + lane; x < rowptr[i + 1]; x += 32) {
            const double v = (double)vals[x], c = (double)C[a * d + cols[x]];
            r += v * v - 2.0 * v * c;
        }
        for (int m = 16; m >= 1; m >>= 1) r += __shfl_xor_sync(0xffffffffu, r, m);
        double rs = r + cnorm2[a];
        if (rs < 0.0) rs = 0.0;
        mine += rs;
    }
    if (lane == 0) wsum[warp] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < 8; ++w) tot += wsum[w];
        partials[blockIdx.x] = tot;
    }
}

__global__ void csr_sum_partials_kernel(const double *__restrict__ partials, int count, double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < count; ++i) s += partials[i];
        *out = s;
    }
}

template <typename F, int T>
void assign_t(const CsrRows &X, const F *Ct, const F *h, int64_t kpad, int32_t *labels, F *d2, const LoopState *st,
              cudaStream_t s) {
    constexpr int G = T <= 8 ? 4 : (T <= 16 ? 2 : 1);
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((X.n + 7) / 8, 148 * 8));
    csr_assign_kernel<F, T, G><<<(unsigned)blocks, 256, 0, s>>>((const F *)X.vals, X.cols, X.rowptr, X.n, Ct, h,
                                                             (int)kpad, labels, d2, st);
    KMB_LAUNCHED();
}

}  // namespace

void launch_csr_prepare(const int64_t *cols_in, const int64_t *rowptr_in, int64_t n, int64_t d, int64_t nnz, int base,
                        int32_t *cols_out, int64_t *rowptr_out, int *bad, cudaStream_t s) {
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8));
    csr_prepare_kernel<<<(unsigned)blocks, 256, 0, s>>>(cols_in, rowptr_in, n, d, nnz, base, cols_out, rowptr_out,
                                                        bad);
    KMB_LAUNCHED();
}

template <typename F>
void launch_csr_assign(const CsrRows &X, const F *Ct, const F *h, int64_t k, int64_t kpad, int32_t *labels, F *d2,
                       const LoopState *st, cudaStream_t s) {
    if (X.n == 0) return;
    const int64_t per_lane = (kpad + 31) / 32;
    if (per_lane <= 1) assign_t<F, 1>(X, Ct, h, kpad, labels, d2, st, s);
    else if (per_lane <= 2) assign_t<F, 2>(X, Ct, h, kpad, labels, d2, st, s);
    else if (per_lane <= 4) assign_t<F, 4>(X, Ct, h, kpad, labels, d2, st, s);
    else if (per_lane <= 8) assign_t<F, 8>(X, Ct, h, kpad, labels, d2, st, s);
    else assign_t<F, 16>(X, Ct, h, kpad, labels, d2, st, s);  // wider k: 512-cluster passes (two CTAs per SM fit)
}

template <typename F>
void launch_csr_objective(const CsrRows &X, const F *C, int64_t k, const int32_t *labels, double *cnorm2,
                          double *partials, double *out, cudaStream_t s) {
    cnorm2_kernel<<<(unsigned)k, 128, 0, s>>>(C, (int)sizeof(F), (int)X.d, cnorm2);
    KMB_LAUNCHED();
    csr_objective_kernel<F><<<kCsrObjectiveBlocks, 256, 0, s>>>((const F *)X.vals, X.cols, X.rowptr, X.n, (int)X.d, C,
                                                                labels, cnorm2, partials);
    KMB_LAUNCHED();
    csr_sum_partials_kernel<<<1, 32, 0, s>>>(partials, kCsrObjectiveBlocks, out);
    KMB_LAUNCHED();
}

#define KMB_CSR_INST(F)                                                                                              \
    template void launch_csr_assign<F>(const CsrRows &, const F *, const F *, int64_t, int64_t, int32_t *, F *,     \
                                       const LoopState *, cudaStream_t);                                             \
    template void launch_csr_objective<F>(const CsrRows &, const F *, int64_t, const int32_t *, double *, double *, \
                                          double *, cudaStream_t);
KMB_CSR_INST(float)
KMB_CSR_INST(double)
#undef KMB_CSR_INST

}  // namespace kmb
