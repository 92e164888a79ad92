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
#include <type_traits>

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

constexpr int kUpdWarps = 4;  // warps per CTA of the distance update

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned load_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void store_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// A block's sum is published: acc[b] first, then flags[b] = epoch (release).
template <typename F>
__device__ __forceinline__ void publish_block_sum(F *acc, unsigned *flags, int64_t b, F sum, unsigned epoch) {
    acc[b] = sum;
    store_release(flags + b, epoch);
}

// The overall sum acc[0] + acc[1] + ... in block order, folded by the update
// grid's leading CTA while the other CTAs still produce block sums: each lane
// waits for eight consecutive blocks' flags (acquire loads issued together),
// reads their sums past L1, and every lane folds the 256 values in order
// through shuffles. Blocks are produced in
// roughly increasing order, so the fold trails the update by about one wave of
// warps and the round's sequential part shrinks to the sampling walk. Producers
// never wait, so the wait always ends; it is still bounded (10 s), after which
// the round is marked timed out. Result: st->overall.
template <typename F>
__device__ void fold_overall(const F *acc, const unsigned *flags, int64_t nb, unsigned epoch, PPState *st) {
    const int lane = threadIdx.x & 31;
    const unsigned long long deadline = global_ns() + 10000000000ull;
    F overall = F(0);
    bool ok = true;
    constexpr int PER = 8;  // blocks per lane per batch
    for (int64_t b0 = 0; b0 < nb && ok; b0 += 32 * PER) {
        const int64_t mine = b0 + lane * PER;  // this lane's first block
        const int have = (int)max((int64_t)0, min((int64_t)PER, nb - mine));
        for (;;) {  // wait until all of this lane's flags carry the epoch
            bool ready = true;
#pragma unroll
            for (int i = 0; i < PER; ++i)
                if (i < have && load_acquire(flags + mine + i) != epoch) ready = false;
            if (ready) break;
            if (global_ns() > deadline) {
                ok = false;
                break;
            }
            __nanosleep(200);
        }
        F v[PER];
#pragma unroll
        for (int i = 0; i < PER; ++i) v[i] = (ok && i < have) ? __ldcg(acc + mine + i) : F(0);
        ok = __all_sync(0xffffffffu, ok);
        const int64_t cnt = min((int64_t)32 * PER, nb - b0);
#pragma unroll 2
        for (int src = 0; src < 32; ++src) {
#pragma unroll
            for (int i = 0; i < PER; ++i) {
                const F x = __shfl_sync(0xffffffffu, v[i], src);
                if (src * PER + i < cnt) overall += x;
            }
        }
    }
    if (lane == 0) {
        if (ok) {
            st->overall = (double)overall;
        } else {
            st->stopped = 3;
            st->stop_round = (long long)epoch;
        }
    }
}

// One warp per 512-row block: the block's rows go 32 at a time (a group), one
// row per lane. A group's rows are staged through shared memory one 128-byte
// segment per row at a time (W columns; one warp load instruction covers 32/W
// rows, fully coalesced), and the next segment's loads are in flight while the
// current one is folded (4 KB outstanding per warp). Each lane folds its row's
// columns in coordinate order, reading the row and the center 16 bytes at a
// time (row pitch W + 16/sizeof(F): conflict-free for 16-byte reads). After
// the last group, lane 0 sums the block's 512 new minima in row order. Rows
// narrower than one segment are read directly (the group's 32 rows are one
// contiguous range, so the lanes' reads share cache lines). Warps never wait
// for one another.
template <typename F>
__global__ void __launch_bounds__(kUpdWarps * 32, 8)
    pp_update_kernel(const F *__restrict__ X, int64_t n, int d, int64_t nb, const F *__restrict__ center,
                     F *__restrict__ md, F *__restrict__ acc, unsigned *__restrict__ flags, unsigned epoch,
                     PPState *st) {
    constexpr int W = 128 / (int)sizeof(F);  // columns per segment
    constexpr int V = 16 / (int)sizeof(F);   // elements per 16-byte read
    constexpr int P = W + V;                 // tile row pitch
    constexpr int RPI = 32 / W;              // rows per warp load instruction
    constexpr int NLD = 32 / RPI;            // load instructions per segment
    using Vec = typename std::conditional<sizeof(F) == 4, float4, double2>::type;
    __shared__ __align__(16) F tile[kUpdWarps][32][P];
    __shared__ __align__(16) F cseg[kUpdWarps][W];
    __shared__ __align__(16) F s_md[kUpdWarps][kPPBlock];
    if (st->stopped) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (blockIdx.x == 0) {  // the leading CTA folds the overall sum
        if (warp == 0) fold_overall(acc, flags, nb, epoch, st);
        return;
    }
    const int64_t b = (int64_t)(blockIdx.x - 1) * kUpdWarps + warp;
    if (b >= nb) return;  // warp-uniform; no CTA-wide barrier below
    const int64_t base = b * kPPBlock;
    const int cnt = (int)min((int64_t)kPPBlock, n - base);
    const int ngroups = (cnt + 31) / 32;
    if (d < W) {
        for (int g = 0; g < ngroups; ++g) {
            const int r = g * 32 + lane;
            if (r < cnt) {
                const F *x = X + (base + r) * d;
                F d2 = F(0);
                for (int i = 0; i < d; ++i) {
                    const F t = x[i] - center[i];
                    d2 = fma(t, t, d2);
                }
                const F old = md[base + r];
                const F m = !(d2 < old) ? old : d2;  // the reference's min(best, d2)
                md[base + r] = m;
                s_md[warp][r] = m;
            }
        }
    } else {
        const int sub = lane / W, col = lane % W;
        const int nseg = (d + W - 1) / W;
        F v[NLD];
        auto load_segment = [&](int g, int c0) {
            const int c = c0 + col;
#pragma unroll
            for (int j = 0; j < NLD; ++j) {
                const int r = g * 32 + j * RPI + sub;
                v[j] = (r < cnt && c < d) ? X[(base + r) * d + c] : F(0);
            }
        };
        load_segment(0, 0);
        F d2 = F(0), old = F(0);
        int g = 0, sg = 0;
        for (;;) {
            const int c0 = sg * W;
            if (sg == 0 && g * 32 + lane < cnt) old = md[base + g * 32 + lane];
#pragma unroll
            for (int j = 0; j < NLD; ++j) tile[warp][j * RPI + sub][col] = v[j];
            if (sub == 0) cseg[warp][col] = c0 + col < d ? center[c0 + col] : F(0);
            __syncwarp();
            // next segment (of this group, else the next group's first)
            int ng = g, nsg = sg + 1;
            if (nsg == nseg) {
                nsg = 0;
                ++ng;
            }
            if (ng < ngroups) load_segment(ng, nsg * W);
            const F *xr = &tile[warp][lane][0];
            const F *cr = &cseg[warp][0];
            if (c0 + W <= d) {
#pragma unroll
                for (int i = 0; i < W; i += V) {
                    const Vec xv = *reinterpret_cast<const Vec *>(xr + i);
                    const Vec cv = *reinterpret_cast<const Vec *>(cr + i);
                    const F *xe = reinterpret_cast<const F *>(&xv), *ce = reinterpret_cast<const F *>(&cv);
#pragma unroll
                    for (int u = 0; u < V; ++u) {
                        const F t = xe[u] - ce[u];
                        d2 = fma(t, t, d2);
                    }
                }
            } else {
                for (int i = 0; i < d - c0; ++i) {
                    const F t = xr[i] - cr[i];
                    d2 = fma(t, t, d2);
                }
            }
            __syncwarp();
            if (nsg == 0) {  // the group's rows are complete
                const int r = g * 32 + lane;
                if (r < cnt) {
                    const F m = !(d2 < old) ? old : d2;  // the reference's min(best, d2)
                    md[base + r] = m;
                    s_md[warp][r] = m;
                }
                d2 = F(0);
            }
            if (ng >= ngroups) break;
            g = ng;
            sg = nsg;
        }
    }
    __syncwarp();
    if (lane == 0) {
        const F *m = s_md[warp];
        F sum = F(0);
        int i = 0;
        for (; i + V <= cnt; i += V) {
            const Vec x = *reinterpret_cast<const Vec *>(m + i);
            const F *e = reinterpret_cast<const F *>(&x);
#pragma unroll
            for (int u = 0; u < V; ++u) sum += e[u];
        }
        for (; i < cnt; ++i) sum += m[i];
        publish_block_sum(acc, flags, b, sum, epoch);
    }
}

// 16-byte global -> shared copies that bypass registers (zero-filled past
// `src_bytes`), grouped per pipeline stage.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

constexpr int kAsyncStages = 4;

template <typename F>
__host__ __device__ constexpr int async_warp_smem() {  // bytes per warp: stages of (32 row segments + center segment) + minima
    return kAsyncStages * (32 * (128 + 16) + 128) + kPPBlock * (int)sizeof(F);
}

// The distance update for rows of 16-byte multiple length at a 16-byte aligned
// base: the same one-warp-per-block fold as pp_update_kernel, but each 4 KB
// group segment (32 row pieces of 128 bytes, plus the center's piece) goes
// global -> shared with cp.async in a 4-stage ring per warp, so three segments
// stay in flight while one is folded, no registers hold loads and a lane issues
// eight 16-byte copies per segment. Columns past d and rows past the block are
// zero-filled; they add (0 - 0)^2 = +0 to a non-negative sum, which leaves it
// unchanged, so every segment is folded whole.
template <typename F>
__global__ void __launch_bounds__(kUpdWarps * 32)
    pp_update_async_kernel(const F *__restrict__ X, int64_t n, int d, int64_t nb, const F *__restrict__ center,
                           F *__restrict__ md, F *__restrict__ acc, unsigned *__restrict__ flags, unsigned epoch,
                           PPState *st) {
    constexpr int W = 128 / (int)sizeof(F);  // columns per segment
    constexpr int V = 16 / (int)sizeof(F);   // columns per 16-byte piece
    constexpr int P = W + V;                 // tile row pitch (144 bytes)
    using Vec = typename std::conditional<sizeof(F) == 4, float4, double2>::type;
    extern __shared__ __align__(16) unsigned char pp_async_smem[];
    if (st->stopped) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (blockIdx.x == 0) {  // the leading CTA folds the overall sum
        if (warp == 0) fold_overall(acc, flags, nb, epoch, st);
        return;
    }
    const int64_t b = (int64_t)(blockIdx.x - 1) * kUpdWarps + warp;
    if (b >= nb) return;  // warp-uniform; no CTA-wide barrier below
    unsigned char *ws = pp_async_smem + (size_t)warp * async_warp_smem<F>();
    F(*tile)[32][P] = reinterpret_cast<F(*)[32][P]>(ws);                            // [stage][row][P]
    F(*cst)[W] = reinterpret_cast<F(*)[W]>(ws + kAsyncStages * 32 * P * sizeof(F));  // [stage][W]
    F *s_md = reinterpret_cast<F *>(ws + kAsyncStages * (32 * P + W) * sizeof(F));
    const int64_t base = b * kPPBlock;
    const int cnt = (int)min((int64_t)kPPBlock, n - base);
    const int ngroups = (cnt + 31) / 32;
    const int nseg = (d + W - 1) / W;
    const int total = ngroups * nseg;
    // this lane's copies: piece q of rows (lane >> 3) + 4 k, k = 0..7
    const int q = lane & 7, rl = lane >> 3;
    const F *src0 = X + (base + rl) * (int64_t)d + q * V;
    int ig = 0, isg = 0;  // next (group, segment) to issue
    auto issue = [&](int stage) {
        const int c = isg * W + q * V;
        const bool col_ok = c < d;
        const F *p = src0 + (int64_t)ig * 32 * d + isg * W;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int r = ig * 32 + rl + 4 * k;
            const bool ok = col_ok && r < cnt;
            cp_async16(&tile[stage][rl + 4 * k][q * V], ok ? (const void *)(p + (int64_t)4 * k * d) : (const void *)X,
                       ok ? 16 : 0);
        }
        if (lane < 8) cp_async16(&cst[stage][q * V], col_ok ? (const void *)(center + c) : (const void *)center,
                                 col_ok ? 16 : 0);
        if (++isg == nseg) {
            isg = 0;
            ++ig;
        }
    };
#pragma unroll
    for (int t = 0; t < kAsyncStages - 1; ++t) {
        if (t < total) issue(t);
        cp_async_commit();
    }
    F d2 = F(0), old = F(0);
    int g = 0, sg = 0;
    for (int t = 0; t < total; ++t) {
        if (t + kAsyncStages - 1 < total) issue((t + kAsyncStages - 1) % kAsyncStages);
        cp_async_commit();
        if (sg == 0 && g * 32 + lane < cnt) old = md[base + g * 32 + lane];
        cp_async_wait<kAsyncStages - 1>();
        __syncwarp();
        const int stage = t % kAsyncStages;
        const F *xr = &tile[stage][lane][0];
        const F *cr = &cst[stage][0];
#pragma unroll
        for (int i = 0; i < W; i += V) {
            const Vec xv = *reinterpret_cast<const Vec *>(xr + i);
            const Vec cv = *reinterpret_cast<const Vec *>(cr + i);
            const F *xe = reinterpret_cast<const F *>(&xv), *ce = reinterpret_cast<const F *>(&cv);
#pragma unroll
            for (int u = 0; u < V; ++u) {
                const F e = xe[u] - ce[u];
                d2 = fma(e, e, d2);
            }
        }
        __syncwarp();
        if (++sg == nseg) {  // the group's rows are complete
            const int r = g * 32 + lane;
            if (r < cnt) {
                const F m = !(d2 < old) ? old : d2;  // the reference's min(best, d2)
                md[base + r] = m;
                s_md[r] = m;
            }
            d2 = F(0);
            sg = 0;
            ++g;
        }
    }
    cp_async_wait<0>();
    __syncwarp();
    if (lane == 0) {
        F sum = F(0);
        int i = 0;
        for (; i + V <= cnt; i += V) {
            const Vec x = *reinterpret_cast<const Vec *>(s_md + i);
            const F *e = reinterpret_cast<const F *>(&x);
#pragma unroll
            for (int u = 0; u < V; ++u) sum += e[u];
        }
        for (; i < cnt; ++i) sum += s_md[i];
        publish_block_sum(acc, flags, b, sum, epoch);
    }
}

constexpr int kSelThreads = 256;

// Eight consecutive values from 16-byte aligned shared memory in 16-byte loads.
__device__ __forceinline__ void load8(const float *p, float (&o)[8]) {
    const float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
    o[0] = a.x, o[1] = a.y, o[2] = a.z, o[3] = a.w, o[4] = b.x, o[5] = b.y, o[6] = b.z, o[7] = b.w;
}
__device__ __forceinline__ void load8(const double *p, double (&o)[8]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double2 a = reinterpret_cast<const double2 *>(p)[q];
        o[2 * q] = a.x, o[2 * q + 1] = a.y;
    }
}

// Sequential walk of the block sums for thread 0 over a[lo, hi): advances while
// s >= a[j], subtracting, exactly as the scalar loop would; eight steps at a
// time are computed speculatively and kept when all eight pass.
// `a` is 16-byte aligned; the next eight values load while the current eight
// are folded.
template <typename F>
__device__ __forceinline__ int walk_span(const F *a, int hi, F &s) {
    int j = 0;
    F t = s;
    if (hi >= 8) {
        F v[8];
        load8(a, v);
        for (;;) {
            F w[8];
            const bool more = j + 16 <= hi;
            if (more) load8(a + j + 8, w);
            F u[9];
            u[0] = t;
            bool all = true;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                all = all & (u[q] >= v[q]);
                u[q + 1] = u[q] - v[q];
            }
            if (!all) break;
            t = u[8];
            j += 8;
            if (!more) break;
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = w[q];
        }
    }
    while (j < hi && t >= a[j]) {
        t -= a[j];
        ++j;
    }
    s = t;
    return j;
}

// Round c's sequential part in one CTA: the sampling walk (block sums, then the
// chosen block's rows) with resampling, and the new center. The block sums
// stream through two shared-memory chunks: warps 1.. load chunk q + 1 while
// thread 0 walks chunk q.
template <typename F>
__global__ void __launch_bounds__(kSelThreads) pp_select_kernel(const F *__restrict__ X, int64_t n, int d, int64_t nb,
                                                                const F *__restrict__ acc, F *__restrict__ md,
                                                                const F *__restrict__ probs,
                                                                const F *__restrict__ pool, int pool_n, int64_t c,
                                                                F *__restrict__ C, PPState *st) {
    constexpr int CH = 16384 / (int)sizeof(F);  // elements per chunk
    __shared__ __align__(16) F buf[2][CH];
    __shared__ __align__(16) F rows[kPPBlock];
    __shared__ F s_val;          // the walk's remainder, then a resample draw
    __shared__ long long s_pos;  // chosen block, then chosen row (-1: give up)
    __shared__ int s_flag;
    const int tid = threadIdx.x;
    if (st->stopped) return;
    const int64_t nchunks = (nb + CH - 1) / CH;
    auto load_chunk = [&](int64_t q, int t0, int nt) {
        const int64_t lo = q * CH, cnt = min((int64_t)CH, nb - lo);
        for (int64_t i = t0; i < cnt; i += nt) buf[q & 1][i] = acc[lo + i];
    };
    // the overall sum, folded in block order by the update grid's leading CTA
    const F overall = (F)st->overall;
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
    if (tid == 0) s_flag = 0;
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
                const int64_t j = lo < hi ? lo + walk_span(buf[q & 1], (int)(hi - lo), s) : lo;
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
            const int64_t r = walk_span(rows, (int)cnt - 1, r_s);
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
    if (X)  // dense rows; CSR rows are expanded by pp_csr_emit_kernel
        for (int i = tid; i < d; i += kSelThreads) C[c * d + i] = X[row * d + i];
    if (tid == 0) {
        md[row] = F(0);
        st->pool_used = used;
        st->rows_chosen += 1;
        st->last_row = row;
    }
}

// ---- CSR rows (plusPlusCSR, DataHelperCSR of kmeans_plusplus_init_impl.i:244-316) ----

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// Center c = row (st->last_row, or `row` when >= 0) expanded to dense, and its
// squared norm in F summed in column order (the unstored zeros add nothing).
template <typename F>
__global__ void pp_csr_emit_kernel(const F *__restrict__ vals, const int32_t *__restrict__ cols,
                                   const int64_t *__restrict__ rowptr, int d, int64_t c, int64_t row, F *__restrict__ C,
                                   PPState *st) {
    if (st->stopped) return;
    const int64_t r = row >= 0 ? row : st->last_row;
    F *out = C + c * d;
    for (int i = threadIdx.x; i < d; i += blockDim.x) out[i] = F(0);
    __syncthreads();
    for (int64_t e = rowptr[r] + threadIdx.x; e < rowptr[r + 1]; e += blockDim.x) out[cols[e]] = vals[e];
    if (threadIdx.x == 0) {
        F s = F(0);
        for (int64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) s = add_rn(s, mul_rn(vals[e], vals[e]));
        st->cnorm = (double)s;
    }
}

// d2 = ||c||^2, then per stored entry in order d2 += x*x - (2x)*c_col, every
// operation rounded as written (no contraction). One warp per 512-row block, one
// lane per row; lane 0 sums the block's minima in row order and publishes them
// for the leading CTA's overall-sum fold.
template <typename F>
__global__ void __launch_bounds__(kUpdWarps * 32)
    pp_update_csr_kernel(const F *__restrict__ vals, const int32_t *__restrict__ cols,
                         const int64_t *__restrict__ rowptr, int64_t n, int64_t nb, const F *__restrict__ center,
                         F *__restrict__ md, F *__restrict__ acc, unsigned *__restrict__ flags, unsigned epoch,
                         PPState *st) {
    __shared__ F s_md[kUpdWarps][kPPBlock];
    if (st->stopped) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (blockIdx.x == 0) {
        if (warp == 0) fold_overall(acc, flags, nb, epoch, st);
        return;
    }
    const int64_t b = (int64_t)(blockIdx.x - 1) * kUpdWarps + warp;
    if (b >= nb) return;
    const int64_t base = b * kPPBlock;
    const int cnt = (int)min((int64_t)kPPBlock, n - base);
    const F cn = (F)st->cnorm;
    for (int r = lane; r < cnt; r += 32) {
        const int64_t row = base + r;
        F d2 = cn;
        for (int64_t e = rowptr[row]; e < rowptr[row + 1]; ++e) {
            const F x = vals[e];
            d2 = add_rn(d2, sub_rn(mul_rn(x, x), mul_rn(mul_rn(F(2), x), center[cols[e]])));
        }
        const F old = md[row];
        const F m = !(d2 < old) ? old : d2;  // the reference's min(best, d2)
        md[row] = m;
        s_md[warp][r] = m;
    }
    __syncwarp();
    if (lane == 0) {
        F sum = F(0);
        for (int i = 0; i < cnt; ++i) sum += s_md[warp][i];
        publish_block_sum(acc, flags, b, sum, epoch);
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
                      unsigned *flags, const F *probs, const F *pool, int pool_n, F *C, PPState *st, cudaStream_t s) {
    const int64_t nb = (n + kPPBlock - 1) / kPPBlock;
    const unsigned grid = 1 + (unsigned)((nb + kUpdWarps - 1) / kUpdWarps);  // + the overall-sum CTA
    // 16-byte copies need 16-byte aligned rows; narrower rows take the register path
    const bool async = ((uintptr_t)X % 16) == 0 && ((uintptr_t)C % 16) == 0 && (d * sizeof(F)) % 16 == 0 &&
                       d >= 128 / (int64_t)sizeof(F);
    const int async_smem = kUpdWarps * async_warp_smem<F>();
    if (async) cudaFuncSetAttribute(pp_update_async_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, async_smem);
    for (int64_t c = c_begin; c < k; ++c) {
        if (c > c_begin || update_first) {
            if (async)
                pp_update_async_kernel<F><<<grid, kUpdWarps * 32, async_smem, s>>>(
                    X, n, (int)d, nb, C + (c - 1) * d, md, acc, flags, (unsigned)c, st);
            else
                pp_update_kernel<F><<<grid, kUpdWarps * 32, 0, s>>>(X, n, (int)d, nb, C + (c - 1) * d, md, acc, flags,
                                                                    (unsigned)c, st);
            KMB_LAUNCHED();
        }
        pp_select_kernel<F><<<1, kSelThreads, 0, s>>>(X, n, (int)d, nb, acc, md, probs, pool, pool_n, c, C, st);
        KMB_LAUNCHED();
    }
}

template <typename F>
void launch_pp_first_csr(const CsrRows &X, int64_t row, F *C, PPState *st, cudaStream_t s) {
    pp_csr_emit_kernel<F><<<1, 256, 0, s>>>((const F *)X.vals, X.cols, X.rowptr, (int)X.d, 0, row, C, st);
    KMB_LAUNCHED();
}

template <typename F>
void launch_pp_rounds_csr(const CsrRows &X, int64_t k, int64_t c_begin, bool update_first, F *md, F *acc,
                          unsigned *flags, const F *probs, const F *pool, int pool_n, F *C, PPState *st, cudaStream_t s) {
    const int64_t n = X.n, d = X.d;
    const int64_t nb = (n + kPPBlock - 1) / kPPBlock;
    const unsigned grid = 1 + (unsigned)((nb + kUpdWarps - 1) / kUpdWarps);  // + the overall-sum CTA
    for (int64_t c = c_begin; c < k; ++c) {
        if (c > c_begin || update_first) {
            pp_update_csr_kernel<F><<<grid, kUpdWarps * 32, 0, s>>>((const F *)X.vals, X.cols, X.rowptr, n, nb,
                                                                    C + (c - 1) * d, md, acc, flags, (unsigned)c, st);
            KMB_LAUNCHED();
        }
        pp_select_kernel<F><<<1, kSelThreads, 0, s>>>(nullptr, n, (int)d, nb, acc, md, probs, pool, pool_n, c, C, st);
        KMB_LAUNCHED();
        pp_csr_emit_kernel<F><<<1, 256, 0, s>>>((const F *)X.vals, X.cols, X.rowptr, (int)d, c, -1, C, st);
        KMB_LAUNCHED();
    }
}

#define KMB_PP_INST(F)                                                                                               \
    template void launch_pp_first_csr<F>(const CsrRows &, int64_t, F *, PPState *, cudaStream_t);                  \
    template void launch_pp_rounds_csr<F>(const CsrRows &, int64_t, int64_t, bool, F *, F *, unsigned *, const F *, \
                                          const F *, int, F *, PPState *, cudaStream_t);                           \
    template void launch_pp_fill<F>(F *, int64_t, cudaStream_t);                                                    \
    template void launch_pp_first<F>(const F *, int64_t, int64_t, F *, cudaStream_t);                               \
    template void launch_pp_rounds<F>(const F *, int64_t, int64_t, int64_t, int64_t, bool, F *, F *, unsigned *,    \
                                      const F *, const F *, int, F *, PPState *, cudaStream_t);
KMB_PP_INST(float)
KMB_PP_INST(double)
#undef KMB_PP_INST

}  // namespace kmb
