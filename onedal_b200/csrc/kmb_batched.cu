// Batched form: thousands of independent k-means problems (uneven n, k, d) train
// together in ONE persistent grouped kernel. A cooperative grid walks, for every
// Lloyd iteration, four phases over flat work lists of all problems, separated
// by grid-wide barriers (bounded waits: a barrier that does not complete within
// ~2 s sets an error flag, every CTA leaves, and the call returns KMB_ETIMEDOUT).
// The launch can be captured into a CUDA graph and replayed.
//
// Per iteration (the semantics of one pass of cpp/daal/src/algorithms/kmeans/
// kmeans_lloyd_batch_impl.i:117-212, for every problem not yet converged):
//   prep        (problem, cluster)   C -> transposed Ct, h = 0.5||c||^2
//   work        (problem, block of 4096 rows)
//                 assign:     FP32 FMA scores h_j - x.c_j over all of the problem's
//                             clusters (k <= 256), lowest index on ties; labels and
//                             squared distances, tile by tile
//                 accumulate: exact fixed-point cluster sums of the same block (the
//                             rows are still in L2): every value as three 32-bit
//                             limbs (the Lloyd loop's exact update,
//                             kmb_internal.cuh), summed per label-sorted row list,
//                             then added to the problem's int64 limb sums -- or,
//                             once at most n/4 rows moved in the previous
//                             iteration, only the moved rows, taken out of their
//                             old cluster's sums and added to the new one's
//                             (integer atomics: the same sums in any order)
//   finalize    (problem, cluster)   c = F(S / count) from the 128-bit sum, shift
//                                    part (the sums are kept, normalised)
//   decide      (problem)            empty clusters reseeded with the farthest rows
//                                    (squared distance descending, row ascending;
//                                    empty clusters ascending), shift, stop test
// Each step computes what the single-problem path (kmb_lloyd_iterate, plain form)
// computes, in the same floating-point order -- row norms, half norms, scores,
// exact sums, centroids -- so a problem trained here equals the same problem
// trained alone bit for bit.
//
// Work items of a phase are found on the device from per-problem prefix counts
// and taken round-robin; the work list is ordered by cost (rows x padded clusters
// x padded features) so the largest blocks start first. The assignment tile of
// each (d, k) class comes from a built-in autotuner that times the candidates on
// synthetic rows of that shape the first time the class is seen on a device
// (cached under a lock).
#include "kmb_internal.cuh"

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

namespace kmb {
namespace batched {

constexpr int NT = 256;            // threads per CTA
constexpr int BK = 8;              // contraction chunk of the assignment tile
constexpr int kMaxK = 256;         // clusters per problem (one assignment tile covers all)
constexpr int kAccRows = 4096;     // rows per accumulate / setup work item
constexpr long long kBarrierTimeout = 4000000000ll;  // ~2 s of SM clocks

struct Problem {
    const float *X;
    float *C;
    float *Ct;          // dpad x kpad
    float *h;           // kpad (+inf padding)
    int32_t *labels;
    float *d2;
    float *xnorm;
    long long *acc;     // 3 limb planes of k x d (kept across iterations)
    int *counts;        // k (kept across iterations)
    int32_t *prev;      // n: the labels the sums describe (-1 before the first pass)
    double *shift_part; // k
    int *colexp;        // d (column maxima as float bits during setup, then E_t)
    long long n;
    int d, dpad, k, kpad, tm;
    int done, iters, max_iters, empty_events;
    int inc;            // this iteration's accumulation: 0 every row, 1 the moved rows only
    long long moved;    // rows whose label changed in this iteration's work phase
    double eps, shift;
};

// Work of a phase as per-problem item counts: prefix[q] = items of the problems
// before position q of the phase's problem order; item i belongs to the last q
// with prefix[q] <= i (binary search on the device), so the host builds O(problems)
// data, not O(tiles).
struct Phase {
    const long long *prefix;  // count + 1 entries
    const int *order;         // problem at each position (null: identity)
    long long items;
};

struct Lists {
    Phase blocks;  // (problem, row block of kAccRows): setup
    Phase work;    // its order: every problem, costliest blocks first
    int n_problems;
    int iterations;
    // The problems not yet converged, rebuilt on the device before every iteration
    // (in the work order), so converged problems cost no walking: their count and,
    // per phase, prefix counts over them (prep: padded clusters; work: row blocks;
    // finalize: clusters) -- count + 1 entries each.
    int *act_order;
    long long *act_prep, *act_work, *act_fin;
    int *act_count;
};

// Rebuilds the active lists (one CTA): per thread a contiguous run of the work
// order, its active problems counted, an exclusive scan over the threads, then
// written in order.
__device__ void compact_active(const Problem *P, const Lists &L, unsigned char *smem) {
    long long *s_prep = reinterpret_cast<long long *>(smem), *s_work = s_prep + NT, *s_fin = s_work + NT;
    int *s_cnt = reinterpret_cast<int *>(s_fin + NT);
    const int per = (L.n_problems + NT - 1) / NT;
    const int q0 = min(L.n_problems, (int)threadIdx.x * per), q1 = min(L.n_problems, q0 + per);
    int c = 0;
    long long wp = 0, ww = 0, wf = 0;
    for (int q = q0; q < q1; ++q) {
        const Problem &p = P[L.work.order[q]];
        if (p.done) continue;
        ++c;
        wp += p.kpad;
        ww += (p.n + kAccRows - 1) / kAccRows;
        wf += p.k;
    }
    s_cnt[threadIdx.x] = c;
    s_prep[threadIdx.x] = wp;
    s_work[threadIdx.x] = ww;
    s_fin[threadIdx.x] = wf;
    __syncthreads();
    if (threadIdx.x == 0) {  // exclusive scan over the threads (NT entries)
        int ac = 0;
        long long ap = 0, aw = 0, af = 0;
        for (int t = 0; t < NT; ++t) {
            const int c2 = s_cnt[t];
            const long long p2 = s_prep[t], w2 = s_work[t], f2 = s_fin[t];
            s_cnt[t] = ac;
            s_prep[t] = ap;
            s_work[t] = aw;
            s_fin[t] = af;
            ac += c2;
            ap += p2;
            aw += w2;
            af += f2;
        }
        *L.act_count = ac;
        L.act_prep[ac] = ap;
        L.act_work[ac] = aw;
        L.act_fin[ac] = af;
    }
    __syncthreads();
    int o = s_cnt[threadIdx.x];
    long long ap = s_prep[threadIdx.x], aw = s_work[threadIdx.x], af = s_fin[threadIdx.x];
    for (int q = q0; q < q1; ++q) {
        const int pid = L.work.order[q];
        const Problem &p = P[pid];
        if (p.done) continue;
        L.act_order[o] = pid;
        L.act_prep[o] = ap;
        L.act_work[o] = aw;
        L.act_fin[o] = af;
        ++o;
        ap += p.kpad;
        aw += (p.n + kAccRows - 1) / kAccRows;
        af += p.k;
    }
}

struct GridBarrier {
    unsigned count;
    unsigned gen;
    int error;   // 1: a barrier wait ran out; 2: an invalid label reached the accumulation
    int active;  // problems not yet converged
};

__device__ __forceinline__ int2 item_of(const Phase &ph, int count, long long i) {
    int lo = 0, hi = count;  // prefix[lo] <= i < prefix[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (ph.prefix[mid] <= i) lo = mid;
        else hi = mid;
    }
    return make_int2(ph.order ? ph.order[lo] : lo, (int)(i - ph.prefix[lo]));
}

// Grid-wide barrier of a cooperative launch; false once any CTA gave up waiting
// (or flagged an error). Thread 0 decides and the CTA follows its decision, so
// every thread of a CTA takes the same path.
__device__ __forceinline__ bool grid_sync(GridBarrier *gb) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = &gb->gen;
        const unsigned g = *vgen;
        __threadfence();
        if (atomicAdd(&gb->count, 1u) == gridDim.x - 1) {
            gb->count = 0;
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            const long long t0 = clock64();
            while (*vgen == g) {
                if (*(volatile int *)&gb->error) break;
                if (clock64() - t0 > kBarrierTimeout) {
                    atomicExch(&gb->error, 1);
                    break;
                }
            }
        }
        __threadfence();
        s_ok = *(volatile int *)&gb->error == 0;
    }
    __syncthreads();
    return s_ok != 0;
}

// ---- setup: row norms (the values launch_row_norms gives) and column maxima ----
__device__ void setup_item(Problem &p, int blk, float *smax) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = threadIdx.x; t < p.d; t += NT) smax[t] = 0.f;
    __syncthreads();
    const long long b = (long long)blk * kAccRows, e = min(p.n, b + kAccRows);
    for (long long r = b + warp; r < e; r += NT / 32) {
        const float *x = p.X + r * p.d;
        double s = 0.0;
        for (int t = lane; t < p.d; t += 32) {
            const float v = x[t];
            s += (double)v * (double)v;
            const float a = fabsf(v);
            if (a > 0.f) atomicMax(reinterpret_cast<unsigned *>(&smax[t]), __float_as_uint(a));
        }
        for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
        if (lane == 0) {
            p.xnorm[r] = (float)s;
            p.prev[r] = -1;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < p.d; t += NT) {
        const unsigned v = __float_as_uint(smax[t]);
        if (v) atomicMax(reinterpret_cast<unsigned *>(&p.colexp[t]), v);
    }
    __syncthreads();
}

// E_t from the column maximum (as the Lloyd loop's exact update), sums cleared.
__device__ void scales_item(Problem &p) {
    for (int t = threadIdx.x; t < p.d; t += NT) {
        const unsigned b = (unsigned)p.colexp[t];
        const float m = __uint_as_float(b);
        int e = 0;
        if (b != 0u && isfinite(m)) {
            int ex;
            frexpf(m, &ex);
            e = kExactMaxBits - ex;
        }
        p.colexp[t] = e;
    }
    const long long kd = (long long)p.k * p.d;
    for (long long i = threadIdx.x; i < 3 * kd; i += NT) p.acc[i] = 0;
    for (int j = threadIdx.x; j < p.k; j += NT) p.counts[j] = 0;
}

// ---- prep: one warp per (problem, padded cluster) ------------------------------
// h is summed in the order of prep_centroids_kernel's 128-thread blocks (thread
// v takes features v, v + 128, ...; four warp butterflies; warps added in order),
// so it equals the single-problem path's half norm bit for bit.
__device__ void prep_item(Problem &p, int j, int lane) {
    if (!p.inc && j < p.k) {  // a full accumulation follows: cluster j's sums and count start at zero
        const long long plane = (long long)p.k * p.d;
        for (int t = lane; t < p.d; t += 32) {
            const long long g = (long long)j * p.d + t;
            p.acc[g] = 0;
            p.acc[plane + g] = 0;
            p.acc[2 * plane + g] = 0;
        }
        if (lane == 0) p.counts[j] = 0;
    }
    for (int t = lane; t < p.dpad; t += 32) {
        const float v = (j < p.k && t < p.d) ? p.C[(long long)j * p.d + t] : 0.f;
        p.Ct[(long long)t * p.kpad + j] = v;
    }
    double tot = 0.0;
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        double s = 0.0;
        for (int t = 32 * w + lane; t < p.dpad; t += 128) {
            const float v = (j < p.k && t < p.d) ? p.C[(long long)j * p.d + t] : 0.f;
            s += (double)v * (double)v;
        }
        for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
        tot += s;
    }
    if (lane == 0) p.h[j] = j < p.k ? (float)(0.5 * tot) : __int_as_float(0x7f800000);
}

// ---- assign: BM = 16 * TM rows x BN clusters, thread micro-tile TM x BN/16 -----
template <int BN, int TM>
__device__ void assign_tile(const Problem &p, int tile, float *smem) {
    constexpr int TN = BN / 16, BM = 16 * TM;
    float(*Xs)[BM + 4] = reinterpret_cast<float(*)[BM + 4]>(smem);
    float(*Cs)[BN + 4] = reinterpret_cast<float(*)[BN + 4]>(smem + BK * (BM + 4));
    const long long row0 = (long long)tile * BM;
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    float acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = 0.f;
    for (int kb = 0; kb < p.dpad; kb += BK) {
        for (int e = tid; e < BM * BK; e += NT) {
            const int r = e / BK, c = e - r * BK;
            const long long gr = row0 + r;
            Xs[c][r] = (gr < p.n && kb + c < p.d) ? p.X[gr * p.d + kb + c] : 0.f;
        }
        for (int e = tid; e < BK * BN; e += NT) {
            const int c = e / BN, j = e - c * BN;
            Cs[c][j] = p.Ct[(long long)(kb + c) * p.kpad + j];
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < BK; ++c) {
            float a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = Xs[c][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = Cs[c][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        float best = __int_as_float(0x7f800000);
        int bi = 0;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int col = tx + 16 * j;
            const float v = p.h[col] - acc[i][j];
            if (v < best) {  // columns increase with j: lowest index on ties
                best = v;
                bi = col;
            }
        }
#pragma unroll
        for (int m = 8; m >= 1; m >>= 1) {
            const float ob = __shfl_xor_sync(0xffffffffu, best, m);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, m);
            if (ob < best || (ob == best && oi < bi)) {
                best = ob;
                bi = oi;
            }
        }
        const long long r = row0 + ty + 16 * i;
        if (tx == 0 && r < p.n) {
            p.labels[r] = bi;
            p.d2[r] = 2.f * best + p.xnorm[r];
        }
    }
}

// Row-per-thread tile (the rows-per-thread choice 0): NT rows, each thread holds
// its row (DP = dpad <= 64 values) in registers and walks the problem's clusters
// from shared memory (16-byte broadcast reads), accumulating x_t * c_t in
// ascending t with FMAs -- the order of every single-problem kernel -- and keeping
// the lowest index among equal minimum scores.
// The centroids stay in shared memory across consecutive tiles of one problem
// (cached: the CTA-uniform id of the problem whose centroids are there).
template <int DP>
__device__ void assign_rows(const Problem &p, int pid, int tile, float *smem, int &cached) {
    float *Cs = smem;                  // kpad x DP
    float *hs = smem + p.kpad * DP;    // k
    if (cached != pid) {
        for (int e = threadIdx.x; e < p.k * DP; e += NT) {
            const int j = e / DP, t = e - j * DP;
            Cs[e] = t < p.d ? p.C[(long long)j * p.d + t] : 0.f;
        }
        for (int j = threadIdx.x; j < p.k; j += NT) hs[j] = p.h[j];
        cached = pid;
        __syncthreads();
    }
    const long long r = (long long)tile * NT + threadIdx.x;
    if (r < p.n) {
        float x[DP];
        if (p.d == DP && (p.d & 3) == 0 && (reinterpret_cast<uintptr_t>(p.X) & 15) == 0) {
#pragma unroll
            for (int q = 0; q < DP / 4; ++q) {
                const float4 v = reinterpret_cast<const float4 *>(p.X + r * DP)[q];
                x[4 * q] = v.x;
                x[4 * q + 1] = v.y;
                x[4 * q + 2] = v.z;
                x[4 * q + 3] = v.w;
            }
        } else {
#pragma unroll
            for (int t = 0; t < DP; ++t) x[t] = t < p.d ? p.X[r * p.d + t] : 0.f;
        }
        float best = __int_as_float(0x7f800000);
        int bi = 0;
        // four clusters at a time: four independent FMA chains
        const int k4 = p.k & ~3;
#pragma unroll 1
        for (int j = 0; j < k4; j += 4) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int q = 0; q < DP / 4; ++q) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float4 c = reinterpret_cast<const float4 *>(Cs + (j + u) * DP)[q];
                    acc[u] = fmaf(x[4 * q], c.x, acc[u]);
                    acc[u] = fmaf(x[4 * q + 1], c.y, acc[u]);
                    acc[u] = fmaf(x[4 * q + 2], c.z, acc[u]);
                    acc[u] = fmaf(x[4 * q + 3], c.w, acc[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float v = hs[j + u] - acc[u];
                if (v < best) {  // ascending clusters: the lowest index among equal minima
                    best = v;
                    bi = j + u;
                }
            }
        }
#pragma unroll 1
        for (int j = k4; j < p.k; ++j) {
            const float4 *c4 = reinterpret_cast<const float4 *>(Cs + j * DP);
            float acc = 0.f;
#pragma unroll
            for (int q = 0; q < DP / 4; ++q) {
                const float4 c = c4[q];
                acc = fmaf(x[4 * q], c.x, acc);
                acc = fmaf(x[4 * q + 1], c.y, acc);
                acc = fmaf(x[4 * q + 2], c.z, acc);
                acc = fmaf(x[4 * q + 3], c.w, acc);
            }
            const float v = hs[j] - acc;
            if (v < best) {
                best = v;
                bi = j;
            }
        }
        p.labels[r] = bi;
        p.d2[r] = 2.f * best + p.xnorm[r];
    }
}

__host__ __device__ constexpr int rows_per_item(int tm) { return tm ? 16 * tm : NT; }

// The tile variants the autotuner chooses from: rows per thread 2, 4, 8 of the
// (rows x clusters) tile -- its micro-tile stays at most 32 accumulators so every
// variant fits the 80 registers of three CTAs per SM (the kernel is bound by
// memory latency, so the third CTA's warps pay more than larger tiles would) --
// or 0, the row-per-thread tile (dpad <= 64, kpad <= 128).
// cached: the problem whose centroids the row-per-thread tile holds in shared
// memory (-1: none); a change of problem first waits for every thread of the
// CTA to be done with the previous tile.
__device__ __forceinline__ void assign_dispatch(const Problem &p, int pid, int tile, float *smem, int &cached) {
    if (p.tm == 0) {
        if (cached != pid) __syncthreads();
        switch (p.dpad) {
            case 8: assign_rows<8>(p, pid, tile, smem, cached); break;
            case 16: assign_rows<16>(p, pid, tile, smem, cached); break;
            case 24: assign_rows<24>(p, pid, tile, smem, cached); break;
            case 32: assign_rows<32>(p, pid, tile, smem, cached); break;
            case 40: assign_rows<40>(p, pid, tile, smem, cached); break;
            case 48: assign_rows<48>(p, pid, tile, smem, cached); break;
            case 56: assign_rows<56>(p, pid, tile, smem, cached); break;
            case 64: assign_rows<64>(p, pid, tile, smem, cached); break;
            default: break;
        }
        return;
    }
    if (cached >= 0) {  // the tiled variants overwrite the shared centroids
        __syncthreads();
        cached = -1;
    }
    switch (p.kpad * 16 + p.tm) {
        case 16 * 16 + 2: assign_tile<16, 2>(p, tile, smem); break;
        case 16 * 16 + 4: assign_tile<16, 4>(p, tile, smem); break;
        case 16 * 16 + 8: assign_tile<16, 8>(p, tile, smem); break;
        case 32 * 16 + 2: assign_tile<32, 2>(p, tile, smem); break;
        case 32 * 16 + 4: assign_tile<32, 4>(p, tile, smem); break;
        case 32 * 16 + 8: assign_tile<32, 8>(p, tile, smem); break;
        case 64 * 16 + 2: assign_tile<64, 2>(p, tile, smem); break;
        case 64 * 16 + 4: assign_tile<64, 4>(p, tile, smem); break;
        case 64 * 16 + 8: assign_tile<64, 8>(p, tile, smem); break;
        case 128 * 16 + 2: assign_tile<128, 2>(p, tile, smem); break;
        case 128 * 16 + 4: assign_tile<128, 4>(p, tile, smem); break;
        case 256 * 16 + 2: assign_tile<256, 2>(p, tile, smem); break;
        default: break;
    }
}

// ---- accumulate: exact limb sums of a row block ------------------------------
// The block's rows are listed by label in shared memory (warp-aggregated
// histogram, warp scan, warp-ranked scatter). Then each warp takes (cluster,
// column chunk, slice) tasks: its lanes cover CW = min(32, 2^ceil(log2 d))
// consecutive columns of 32 / CW rows at a time (coalesced row reads, eight rows
// per lane in flight), sum the fixed-point limbs of the slice's rows -- every S-th
// group of rows of the cluster's list -- in registers, fold the lanes of equal
// column with shuffles and add the totals to the problem's limb sums with one
// global atomic per limb. Integer sums: the result depends on neither the order
// of the rows nor the slicing.
__device__ void accumulate_item(Problem &p, int blk, int *sm, GridBarrier *gb) {
    int *s_cnt = sm, *s_off = sm + kMaxK, *s_fill = sm + 2 * kMaxK, *s_rows = sm + 3 * kMaxK;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long b = (long long)blk * kAccRows, e = min(p.n, b + kAccRows);
    const int rows = (int)(e - b);
    const int k = p.k, d = p.d;
    for (int j = threadIdx.x; j < k; j += NT) {
        s_cnt[j] = 0;
        s_fill[j] = 0;
    }
    __syncthreads();
    for (int r0 = 0; r0 < rows; r0 += NT) {  // warp-uniform trip count
        const int r = r0 + threadIdx.x;
        int lab = r < rows ? p.labels[b + r] : -1;
        if (r < rows && (unsigned)lab >= (unsigned)k) {  // cannot happen: the assignment writes every row
            atomicExch(&gb->error, 2);
            lab = -1;
        }
        const unsigned peers = __match_any_sync(0xffffffffu, lab);
        if (lab >= 0 && lane == __ffs(peers) - 1) atomicAdd(&s_cnt[lab], __popc(peers));
    }
    __syncthreads();
    if (warp == 0) {  // exclusive scan of the k <= 256 counts, 8 per lane
        int loc[8], sum = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = lane * 8 + q;
            loc[q] = sum;
            sum += idx < k ? s_cnt[idx] : 0;
        }
        int inc = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = lane * 8 + q;
            if (idx < k) s_off[idx] = inc - sum + loc[q];
        }
    }
    __syncthreads();
    for (int r0 = 0; r0 < rows; r0 += NT) {
        const int r = r0 + threadIdx.x;
        int lab = r < rows ? p.labels[b + r] : -1;
        if ((unsigned)lab >= (unsigned)k) lab = -1;
        const unsigned peers = __match_any_sync(0xffffffffu, lab);
        const int leader = __ffs(peers) - 1;
        int base = 0;
        if (lab >= 0 && lane == leader) base = atomicAdd(&s_fill[lab], __popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (lab >= 0) s_rows[s_off[lab] + base + __popc(peers & ((1u << lane) - 1))] = r;
    }
    __syncthreads();
    int cw = 1;
    while (cw < d && cw < 32) cw <<= 1;
    const int rps = 32 / cw;               // rows per warp step
    const int cl = lane & (cw - 1), rl = lane / cw;
    const int nch = (d + cw - 1) / cw;     // column chunks
    const int kc = k * nch;
    const int S = min(8, max(1, (2 * (NT / 32) + kc - 1) / kc));  // slices: at least two tasks per warp
    const long long plane = (long long)k * d;
    const float *Xb = p.X + b * d;
    for (int task = warp; task < kc * S; task += NT / 32) {
        const int j = task / (nch * S), rest = task - j * nch * S;
        const int ch = rest / S, sl = rest - ch * S;
        const int c = ch * cw + cl;
        const bool active = c < d;
        const int cnt = s_cnt[j], base = s_off[j];
        const int ec = active ? p.colexp[c] : 0;
        long long a0 = 0, a1 = 0, a2 = 0;
        const int step = S * rps;
        for (int i = sl * rps + rl; i < cnt; i += 8 * step) {  // eight gathered loads in flight
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int ii = i + u * step;
                v[u] = (active && ii < cnt) ? Xb[(long long)s_rows[base + ii] * d + c] : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const Limbs L = fixed_of(v[u], ec);
                a0 += L.l0;
                a1 += L.l1;
                a2 += L.l2;
            }
        }
        for (int o = 16; o >= cw; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (rl == 0 && active) {
            const long long g = (long long)j * d + c;
            if (a0) atomicAdd(reinterpret_cast<unsigned long long *>(&p.acc[g]), (unsigned long long)a0);
            if (a1) atomicAdd(reinterpret_cast<unsigned long long *>(&p.acc[plane + g]), (unsigned long long)a1);
            if (a2) atomicAdd(reinterpret_cast<unsigned long long *>(&p.acc[2 * plane + g]), (unsigned long long)a2);
        }
    }
    for (int j = threadIdx.x; j < k; j += NT)
        if (s_cnt[j]) atomicAdd(&p.counts[j], s_cnt[j]);
    __syncthreads();
}

// Full accumulation's bookkeeping: the block's rows that changed label, and prev.
__device__ void track_item(Problem &p, int blk) {
    const long long b = (long long)blk * kAccRows, e = min(p.n, b + kAccRows);
    int c = 0;
    for (long long r = b + threadIdx.x; r < e; r += NT) {
        const int lab = p.labels[r];
        c += lab != p.prev[r];
        p.prev[r] = lab;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(reinterpret_cast<unsigned long long *>(&p.moved), (unsigned long long)c);
}

// Moved-rows accumulation of a block: a warp walks 32 rows; each moved row's values
// leave the old cluster's limb sums and join the new one's (integer atomics, exact
// in any order), counts follow, prev follows the labels.
__device__ void moves_item(Problem &p, int blk, GridBarrier *gb) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long b = (long long)blk * kAccRows, e = min(p.n, b + kAccRows);
    const int k = p.k, d = p.d;
    const long long plane = (long long)k * d;
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(p.acc);
    int moved = 0;
    for (long long base = b + 32 * warp; base < e; base += NT) {  // warp-uniform trip count
        const long long r = base + lane;
        int lab = -1, old = -1;
        if (r < e) {
            lab = p.labels[r];
            old = p.prev[r];
            if ((unsigned)lab >= (unsigned)k || (unsigned)old >= (unsigned)k) {  // cannot happen
                atomicExch(&gb->error, 2);
                lab = old;
            }
        }
        unsigned mv = __ballot_sync(0xffffffffu, r < e && lab != old);
        moved += __popc(mv);
        while (mv) {
            const int src = __ffs(mv) - 1;
            mv &= mv - 1;
            const long long row = base + src;
            const int nl = __shfl_sync(0xffffffffu, lab, src), ol = __shfl_sync(0xffffffffu, old, src);
            const float *x = p.X + row * d;
            for (int t = lane; t < d; t += 32) {
                const Limbs L = fixed_of(x[t], p.colexp[t]);
                const long long in = (long long)nl * d + t, out = (long long)ol * d + t;
                if (L.l0) {
                    atomicAdd(&acc[in], (unsigned long long)L.l0);
                    atomicAdd(&acc[out], (unsigned long long)-L.l0);
                }
                if (L.l1) {
                    atomicAdd(&acc[plane + in], (unsigned long long)L.l1);
                    atomicAdd(&acc[plane + out], (unsigned long long)-L.l1);
                }
                if (L.l2) {
                    atomicAdd(&acc[2 * plane + in], (unsigned long long)L.l2);
                    atomicAdd(&acc[2 * plane + out], (unsigned long long)-L.l2);
                }
            }
            if (lane == 0) {
                atomicAdd(&p.counts[nl], 1);
                atomicSub(&p.counts[ol], 1);
            }
        }
        if (r < e && lab != old) p.prev[r] = lab;
    }
    if (lane == 0 && moved) atomicAdd(reinterpret_cast<unsigned long long *>(&p.moved), (unsigned long long)moved);
}

// ---- finalize: one warp per (problem, cluster) ---------------------------------
// c = F(nearest double of the 128-bit sum * 2^-E_t / count), as the Lloyd loop's
// exact update; empty clusters keep their centroid for decide to reseed.
__device__ void finalize_item(Problem &p, int j, int lane) {
    const int cnt = p.counts[j];
    const long long plane = (long long)p.k * p.d;
    double a = 0.0;
    for (int t = lane; t < p.d; t += 32) {
        const long long g = (long long)j * p.d + t;
        const __int128 S = ((__int128)p.acc[2 * plane + g] << 64) + ((__int128)p.acc[plane + g] << 32) +
                           (__int128)p.acc[g];
        // kept for the next iteration's moved rows, normalised (l0, l1 in [0, 2^32))
        p.acc[g] = (long long)(S & 0xffffffffll);
        p.acc[plane + g] = (long long)((S >> 32) & 0xffffffffll);
        p.acc[2 * plane + g] = (long long)(S >> 64);
        if (cnt > 0) {
            const double Sd = S < 0 ? -u128_to_double((unsigned __int128)(-S)) : u128_to_double((unsigned __int128)S);
            const float c = (float)(ldexp(Sd, -p.colexp[t]) / (double)cnt);
            const double df = (double)p.C[g] - (double)c;
            a += df * df;
            p.C[g] = c;
        }
    }
    for (int m = 16; m >= 1; m >>= 1) a += __shfl_xor_sync(0xffffffffu, a, m);
    if (lane == 0) p.shift_part[j] = cnt > 0 ? a : 0.0;
}

// ---- decide: one CTA per problem ------------------------------------------------
// Empty cluster e (ascending id) takes the e-th row in (squared distance
// descending, row ascending) order: each pick is the block argmax over the rows
// that come after the previous pick in that order.
__device__ void decide_item(Problem &p, double *sred, float *sv, long long *sr, GridBarrier *gb) {
    int n_empty = 0;
    for (int j = 0; j < p.k; ++j) n_empty += p.counts[j] == 0;  // uniform loop (k <= 256)
    float pv = __int_as_float(0x7f800000);
    long long pr = -1;
    for (int j = 0; n_empty > 0 && j < p.k; ++j) {
        if (p.counts[j] != 0) continue;
        float bv = -__int_as_float(0x7f800000);
        long long br = -1;
        for (long long r = threadIdx.x; r < p.n; r += NT) {
            const float v = p.d2[r];
            const bool after = v < pv || (v == pv && r > pr);
            if (after && (br < 0 || v > bv)) {  // rows ascend per thread: first of equals kept
                bv = v;
                br = r;
            }
        }
        sv[threadIdx.x] = bv;
        sr[threadIdx.x] = br;
        __syncthreads();
        if (threadIdx.x == 0) {
            float v0 = sv[0];
            long long r0 = sr[0];
            for (int t = 1; t < NT; ++t) {
                if (sr[t] < 0) continue;
                if (r0 < 0 || sv[t] > v0 || (sv[t] == v0 && sr[t] < r0)) {
                    v0 = sv[t];
                    r0 = sr[t];
                }
            }
            sv[0] = v0;
            sr[0] = r0;
        }
        __syncthreads();
        const long long row = sr[0];
        pv = sv[0];
        pr = row;
        __syncthreads();
        if (row < 0 || row >= p.n) break;  // no ordered row left (non-finite distances): keep the centroid
        double a = 0.0;
        for (int t = threadIdx.x; t < p.d; t += NT) {
            const float x = p.X[row * p.d + t];
            const double df = (double)p.C[(long long)j * p.d + t] - (double)x;
            a += df * df;
            p.C[(long long)j * p.d + t] = x;
        }
        sred[threadIdx.x] = a;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int t = 0; t < NT; ++t) tot += sred[t];
            p.shift_part[j] = tot;
        }
        __syncthreads();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double shift = 0.0;
        for (int j = 0; j < p.k; ++j) shift += p.shift_part[j];
        p.shift = shift;
        p.empty_events += n_empty;
        p.iters += 1;
        // the next iteration's accumulation: the moved rows only when at most a quarter
        // moved in this one (the first iteration's rows all count as moved); measured on
        // the 4096-problem workload: a quarter 0.604 s, a sixteenth 0.617 s, 1/64 0.628 s
        p.inc = p.moved * 4 <= p.n ? 1 : 0;
        p.moved = 0;
        if (shift <= p.eps || p.iters >= p.max_iters) {
            p.done = 1;
            atomicSub(&gb->active, 1);
        }
    }
    __syncthreads();
}

// Dynamic shared memory: the largest phase's needs (assignment tiles, the
// accumulate limb planes of the largest k, decide's scratch).
// Shared memory of the fused assign + accumulate phase: the assignment tiles' region
// (kept across a problem's blocks by the row-per-thread tile), then the accumulation's.
constexpr size_t kAssignSmem = sizeof(float) * (128 * 64 + kMaxK) > sizeof(float) * BK * (16 * 8 + 4 + 256 + 4)
                                   ? sizeof(float) * (128 * 64 + kMaxK)
                                   : sizeof(float) * BK * (16 * 8 + 4 + 256 + 4);
constexpr size_t kAccSmem = sizeof(int) * (3 * kMaxK + kAccRows);

size_t smem_bytes(int kmax, int dmax) {
    (void)kmax;
    const size_t work = kAssignSmem + kAccSmem;
    const size_t setup = sizeof(float) * (size_t)dmax;
    const size_t decide = (sizeof(double) + sizeof(float) + sizeof(long long)) * NT;
    return std::max(std::max(work, setup), decide);
}

__global__ void __launch_bounds__(NT, 3) persistent_kernel(Problem *P, Lists L, GridBarrier *gb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *fsm = reinterpret_cast<float *>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int warps = gridDim.x * (NT / 32);
    // setup (once): column maxima accumulate in colexp, so it starts at zero
    for (int i = blockIdx.x; i < L.n_problems; i += gridDim.x)
        for (int t = threadIdx.x; t < P[i].d; t += NT) P[i].colexp[t] = 0;
    if (!grid_sync(gb)) return;
    for (long long i = blockIdx.x; i < L.blocks.items; i += gridDim.x) {
        const int2 w = item_of(L.blocks, L.n_problems, i);
        setup_item(P[w.x], w.y, fsm);
    }
    if (!grid_sync(gb)) return;
    for (int i = blockIdx.x; i < L.n_problems; i += gridDim.x) scales_item(P[i]);
    if (!grid_sync(gb)) return;
    for (int it = 0; it < L.iterations; ++it) {
        if (blockIdx.x == 0) compact_active(P, L, smem_raw);
        if (!grid_sync(gb)) return;
        const int na = *(volatile int *)L.act_count;  // the same for every CTA until the next compaction
        const Phase prep{L.act_prep, L.act_order, *(volatile long long *)&L.act_prep[na]};
        const Phase work{L.act_work, L.act_order, *(volatile long long *)&L.act_work[na]};
        const Phase fin{L.act_fin, L.act_order, *(volatile long long *)&L.act_fin[na]};
        for (long long i = blockIdx.x * (NT / 32) + warp; i < prep.items; i += warps) {
            const int2 w = item_of(prep, na, i);
            prep_item(P[w.x], w.y, lane);
        }
        if (!grid_sync(gb)) return;
        {
            // (problem, block of kAccRows rows), round-robin, costliest problems first:
            // the block's assignment tiles, then its accumulation, which finds the rows
            // this CTA has just read in L2. A problem with more blocks than the grid has
            // CTAs gives a CTA consecutive blocks of itself, whose centroids then stay in
            // shared memory.
            int cached = -1;
            int *acc_smem = reinterpret_cast<int *>(smem_raw + kAssignSmem);
            for (long long i = blockIdx.x; i < work.items; i += gridDim.x) {
                const int2 w = item_of(work, na, i);
                Problem &p = P[w.x];
                const int bm = rows_per_item(p.tm);
                const long long t0 = (long long)w.y * (kAccRows / bm);
                const long long t1 = min((p.n + bm - 1) / bm, t0 + kAccRows / bm);
                for (long long t = t0; t < t1; ++t) assign_dispatch(p, w.x, (int)t, fsm, cached);
                __syncthreads();  // the block's labels, written by every thread, before they are read
                if (p.inc) {
                    moves_item(p, w.y, gb);
                } else {
                    accumulate_item(p, w.y, acc_smem, gb);
                    track_item(p, w.y);
                }
            }
        }
        if (!grid_sync(gb)) return;
        for (long long i = blockIdx.x * (NT / 32) + warp; i < fin.items; i += warps) {
            const int2 w = item_of(fin, na, i);
            finalize_item(P[w.x], w.y, lane);
        }
        if (!grid_sync(gb)) return;
        for (int q = blockIdx.x; q < na; q += gridDim.x) {
            const int i = L.act_order[q];
            double *sred = reinterpret_cast<double *>(smem_raw);
            long long *sr = reinterpret_cast<long long *>(sred + NT);
            float *sv = reinterpret_cast<float *>(sr + NT);
            decide_item(P[i], sred, sv, sr, gb);
        }
        if (!grid_sync(gb)) return;
        if (*(volatile int *)&gb->active == 0) break;  // read by every CTA between the same two barriers
    }
}

// ---- one shard of a sharded float training (kmb_train_spmd) -----------------------
// The batched accumulation and finalize over one problem: the same exact limb sums
// and the same centroid formula as the single-problem Lloyd loop.
__global__ void __launch_bounds__(NT, 3) shard_sums_kernel(Problem p, int nblocks, GridBarrier *gb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for (int blk = blockIdx.x; blk < nblocks; blk += gridDim.x) accumulate_item(p, blk, reinterpret_cast<int *>(smem_raw), gb);
}

__global__ void shard_finalize_kernel(Problem p) {
    const int lane = threadIdx.x & 31;
    for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < p.k; j += (gridDim.x * blockDim.x) >> 5)
        finalize_item(p, j, lane);
}

// ---- autotuner ------------------------------------------------------------------
// Times the assignment tile of one (dpad, kpad) class for each rows-per-thread
// candidate on synthetic rows of that shape (uniform values, so the scores and
// their ties are those of real data, not all equal), enough of them to fill the
// grid with every candidate: timed on 32768 rows the 256-row tile left most CTAs
// idle and lost to the small tiles it beats by 18 % in the batched runs.
__global__ void tune_fill_kernel(float *p, long long count, unsigned seed) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x) {
        unsigned x = (unsigned)i * 2654435761u ^ seed;
        x ^= x >> 15;
        x *= 2246822519u;
        x ^= x >> 13;
        p[i] = (float)(x & 0xffffff) * (1.0f / 16777216.0f) * 4.0f - 2.0f;
    }
}

__global__ void __launch_bounds__(NT, 3) tune_assign_kernel(const Problem *pp, int tiles) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int cached = -1;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x)
        assign_dispatch(*pp, 0, t, reinterpret_cast<float *>(smem_raw), cached);
}

}  // namespace batched

namespace {

int batched_kpad(int k) {
    int b = 16;
    while (b < k) b <<= 1;
    return b;
}

std::mutex g_tune_mu;
std::map<long long, int> g_tuned;  // (device, dpad, kpad) -> rows per thread

int tuned_tm(int dev, int dpad, int kpad, cudaStream_t s) {
    using namespace batched;
    const long long key = ((long long)dev << 40) | ((long long)dpad << 16) | kpad;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto found = g_tuned.find(key);
    if (found != g_tuned.end()) return found->second;
    std::vector<int> cands = kpad >= 256 ? std::vector<int>{2} : kpad >= 128 ? std::vector<int>{2, 4} : std::vector<int>{2, 4, 8};
    if (dpad <= 64 && kpad <= 128) cands.push_back(0);
    // enough rows that every candidate fills the grid (the batched kernel runs with
    // thousands of problems in flight): four 256-row tiles per CTA of three per SM
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid_ctas = 3 * sms;
    const long long n = (long long)grid_ctas * NT * 4;
    float *X = nullptr, *Ct = nullptr, *h = nullptr, *d2 = nullptr, *xn = nullptr;
    int32_t *lab = nullptr;
    Problem *dp = nullptr;
    int best_tm = 4;
    cudaEvent_t a = nullptr, b = nullptr;
    bool ok = cudaMallocAsync(&X, sizeof(float) * n * dpad, s) == cudaSuccess &&
              cudaMallocAsync(&Ct, sizeof(float) * dpad * kpad, s) == cudaSuccess &&
              cudaMallocAsync(&h, sizeof(float) * kpad, s) == cudaSuccess &&
              cudaMallocAsync(&d2, sizeof(float) * n, s) == cudaSuccess &&
              cudaMallocAsync(&xn, sizeof(float) * n, s) == cudaSuccess &&
              cudaMallocAsync(&lab, sizeof(int32_t) * n, s) == cudaSuccess &&
              cudaMallocAsync(&dp, sizeof(Problem), s) == cudaSuccess && cudaEventCreate(&a) == cudaSuccess &&
              cudaEventCreate(&b) == cudaSuccess;
    if (ok) {
        tune_fill_kernel<<<256, 256, 0, s>>>(X, n * dpad, 1u);
        tune_fill_kernel<<<64, 256, 0, s>>>(Ct, (long long)dpad * kpad, 2u);
        tune_fill_kernel<<<1, 256, 0, s>>>(h, kpad, 3u);
        tune_fill_kernel<<<64, 256, 0, s>>>(xn, n, 4u);
        launch_count() += 4;
        const size_t smem = smem_bytes(kpad, 1);
        cudaFuncSetAttribute(tune_assign_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        float best_ms = 1e30f;
        for (int tm : cands) {
            Problem p;
            std::memset(&p, 0, sizeof(p));
            p.X = X;
            p.C = Ct;  // the row-per-thread tile reads C (k x d); any values of the right size do
            p.Ct = Ct;
            p.h = h;
            p.labels = lab;
            p.d2 = d2;
            p.xnorm = xn;
            p.n = n;
            p.d = dpad;
            p.dpad = dpad;
            p.k = kpad;
            p.kpad = kpad;
            p.tm = tm;
            cudaMemcpyAsync(dp, &p, sizeof(p), cudaMemcpyHostToDevice, s);
            const int tiles = (int)((n + rows_per_item(tm) - 1) / rows_per_item(tm));
            tune_assign_kernel<<<std::min(tiles, grid_ctas), NT, smem, s>>>(dp, tiles);  // warm-up
            cudaEventRecord(a, s);
            for (int r = 0; r < 3; ++r) tune_assign_kernel<<<std::min(tiles, grid_ctas), NT, smem, s>>>(dp, tiles);
            cudaEventRecord(b, s);
            launch_count() += 4;
            float ms = 0.f;
            if (cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess &&
                ms < best_ms) {
                best_ms = ms;
                best_tm = tm;
            }
        }
    }
    for (void *q : {(void *)X, (void *)Ct, (void *)h, (void *)d2, (void *)xn, (void *)lab, (void *)dp})
        if (q) cudaFreeAsync(q, s);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaGetLastError();
    g_tuned[key] = best_tm;
    return best_tm;
}

}  // namespace
}  // namespace kmb

namespace kmb {
void launch_shard_exact_sums(const float *X, int64_t n, int d, int k, const int32_t *labels, const int *colexp,
                             long long *acc, int *counts, int *bad, cudaStream_t s) {
    using namespace batched;
    cudaMemsetAsync(acc, 0, sizeof(long long) * 3 * (size_t)k * d, s);
    cudaMemsetAsync(counts, 0, sizeof(int) * k, s);
    Problem p;
    std::memset(&p, 0, sizeof(p));
    p.X = X;
    p.labels = const_cast<int32_t *>(labels);
    p.n = n;
    p.d = d;
    p.k = k;
    p.colexp = const_cast<int *>(colexp);
    p.acc = acc;
    p.counts = counts;
    const int nblocks = (int)((n + kAccRows - 1) / kAccRows);
    // the accumulation reports an out-of-range label in the error word of a grid barrier
    GridBarrier *gb = reinterpret_cast<GridBarrier *>(reinterpret_cast<char *>(bad) - offsetof(GridBarrier, error));
    cudaFuncSetAttribute(shard_sums_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAccSmem);
    shard_sums_kernel<<<(unsigned)std::max(1, std::min(nblocks, 148 * 3)), NT, kAccSmem, s>>>(p, nblocks, gb);
    KMB_LAUNCHED();
}

void launch_shard_exact_finalize(long long *acc, const int *counts, const int *colexp, float *C, int k, int d,
                                 double *shift_part, cudaStream_t s) {
    using namespace batched;
    Problem p;
    std::memset(&p, 0, sizeof(p));
    p.C = C;
    p.k = k;
    p.d = d;
    p.acc = acc;
    p.counts = const_cast<int *>(counts);
    p.colexp = const_cast<int *>(colexp);
    p.shift_part = shift_part;
    shard_finalize_kernel<<<(unsigned)std::max(1, std::min((k + 7) / 8, 148 * 8)), 256, 0, s>>>(p);
    KMB_LAUNCHED();
}
}  // namespace kmb

extern "C" int kmb_batched_train(int dtype, kmb_batched_problem *problems, int64_t count, int64_t max_iteration_count,
                                 double accuracy_threshold, int32_t use_graph, void *cuda_stream,
                                 kmb_batched_info *info) {
    using namespace kmb;
    using namespace kmb::batched;
    if (dtype != KMB_F32 || !problems || count <= 0 || count > INT32_MAX || max_iteration_count < 0 ||
        max_iteration_count > INT32_MAX || !(accuracy_threshold >= 0))
        return KMB_EINVAL;
    int kmax = 1, dmax = 1;
    for (int64_t i = 0; i < count; ++i) {
        const kmb_batched_problem &q = problems[i];
        if (!q.X || !q.C || !q.labels || q.n <= 0 || q.n > INT32_MAX || q.d <= 0 || q.d > INT32_MAX / 4 || q.k <= 0 ||
            q.k > kMaxK || q.k > q.n || (q.k * q.d + q.k) * 8 > 200 * 1024)
            return KMB_EINVAL;
        kmax = std::max(kmax, (int)q.k);
        dmax = std::max(dmax, (int)q.d);
    }
    cudaStream_t s = (cudaStream_t)cuda_stream;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // Per-problem scratch in one stream-ordered arena (no device-wide synchronisation).
    size_t arena = 0;
    auto take = [&](size_t bytes) {
        const size_t o = arena;
        arena += (bytes + 255) / 256 * 256;
        return o;
    };
    std::vector<Problem> H(count);
    std::vector<size_t> off((size_t)count * 9);
    for (int64_t i = 0; i < count; ++i) {
        const kmb_batched_problem &q = problems[i];
        const int kpad = batched_kpad((int)q.k), dpad = (int)((q.d + 7) / 8 * 8);
        off[i * 9 + 0] = take(sizeof(float) * dpad * kpad);
        off[i * 9 + 1] = take(sizeof(float) * kpad);
        off[i * 9 + 2] = take(sizeof(float) * q.n);
        off[i * 9 + 3] = take(sizeof(float) * q.n);
        off[i * 9 + 4] = take(sizeof(long long) * 3 * q.k * q.d);
        off[i * 9 + 5] = take(sizeof(int) * q.k);
        off[i * 9 + 6] = take(sizeof(double) * q.k);
        off[i * 9 + 7] = take(sizeof(int) * q.d);
        off[i * 9 + 8] = take(sizeof(int32_t) * q.n);
    }
    const size_t bar_off = take(sizeof(GridBarrier));
    unsigned char *base = nullptr;
    if (pool_alloc((void **)&base, arena, dev, s) != cudaSuccess) {
        cudaGetLastError();
        return KMB_ENOMEM;
    }
    std::map<long long, int> classes;  // (kpad, tm) variants in use
    // per-problem item counts of each phase, as prefix sums (see Phase)
    const size_t P1 = (size_t)count + 1;
    std::vector<long long> pre(4 * P1, 0);
    std::vector<int> order((size_t)count);
    std::vector<long long> nblocks((size_t)count);
    std::vector<double> block_cost((size_t)count);
    for (int64_t i = 0; i < count; ++i) {
        const kmb_batched_problem &q = problems[i];
        Problem &p = H[i];
        std::memset(&p, 0, sizeof(p));
        p.X = (const float *)q.X;
        p.C = (float *)q.C;
        p.labels = q.labels;
        p.n = q.n;
        p.d = (int)q.d;
        p.dpad = (int)((q.d + 7) / 8 * 8);
        p.k = (int)q.k;
        p.kpad = batched_kpad(p.k);
        p.tm = tuned_tm(dev, p.dpad, p.kpad, s);
        p.Ct = (float *)(base + off[i * 9 + 0]);
        p.h = (float *)(base + off[i * 9 + 1]);
        p.d2 = (float *)(base + off[i * 9 + 2]);
        p.xnorm = (float *)(base + off[i * 9 + 3]);
        p.acc = (long long *)(base + off[i * 9 + 4]);
        p.counts = (int *)(base + off[i * 9 + 5]);
        p.shift_part = (double *)(base + off[i * 9 + 6]);
        p.colexp = (int *)(base + off[i * 9 + 7]);
        p.prev = (int32_t *)(base + off[i * 9 + 8]);
        p.max_iters = (int)max_iteration_count;
        p.eps = accuracy_threshold;
        p.done = max_iteration_count == 0 ? 1 : 0;
        classes[(long long)p.kpad * 16 + p.tm] = 1;
        pre[0 * P1 + i + 1] = pre[0 * P1 + i] + (p.n + kAccRows - 1) / kAccRows;
        pre[1 * P1 + i + 1] = pre[1 * P1 + i] + p.kpad;
        pre[3 * P1 + i + 1] = pre[3 * P1 + i] + p.k;
        nblocks[i] = (p.n + kAccRows - 1) / kAccRows;
        block_cost[i] = (double)std::min<long long>(p.n, kAccRows) * p.kpad * p.dpad;
        order[i] = (int)i;
    }
    // work: problems with the costliest blocks first (round-robin over the grid then balances well)
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return block_cost[a] > block_cost[b]; });
    for (int64_t q = 0; q < count; ++q) pre[2 * P1 + q + 1] = pre[2 * P1 + q] + nblocks[order[q]];
    Problem *dP = nullptr;
    long long *dPre = nullptr;
    int *dOrder = nullptr;
    if (pool_alloc((void **)&dP, sizeof(Problem) * count, dev, s) != cudaSuccess ||
        pool_alloc((void **)&dPre, sizeof(long long) * (8 * P1), dev, s) != cudaSuccess ||
        pool_alloc((void **)&dOrder, sizeof(int) * 2 * order.size(), dev, s) != cudaSuccess) {
        cudaGetLastError();
        if (dP) cudaFreeAsync(dP, s);
        if (dPre) cudaFreeAsync(dPre, s);
        cudaFreeAsync(base, s);
        return KMB_ENOMEM;
    }
    GridBarrier *gb = (GridBarrier *)(base + bar_off);
    GridBarrier gb_init;
    std::memset(&gb_init, 0, sizeof(gb_init));
    for (int64_t i = 0; i < count; ++i) gb_init.active += H[i].done ? 0 : 1;
    int rc = KMB_OK;
    if (cudaMemcpyAsync(dP, H.data(), sizeof(Problem) * count, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dPre, pre.data(), sizeof(long long) * pre.size(), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dOrder, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(gb, &gb_init, sizeof(GridBarrier), cudaMemcpyHostToDevice, s) != cudaSuccess)
        rc = KMB_ECUDA;

    Lists L;
    L.blocks = Phase{dPre + 0 * P1, nullptr, pre[0 * P1 + count]};
    L.work = Phase{dPre + 2 * P1, dOrder, pre[2 * P1 + count]};
    L.act_order = dOrder + count;
    L.act_prep = dPre + 4 * P1;
    L.act_work = dPre + 5 * P1;
    L.act_fin = dPre + 6 * P1;
    L.act_count = (int *)(dPre + 7 * P1);
    L.n_problems = (int)count;
    L.iterations = (int)max_iteration_count;
    const size_t smem = smem_bytes(kmax, dmax);
    int per_sm = 0;
    if (rc == KMB_OK &&
        (cudaFuncSetAttribute(persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
         cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_kernel, NT, smem) != cudaSuccess ||
         per_sm < 1))
        rc = KMB_EUNSUPPORTED;
    const int grid = std::max(1, per_sm) * sms;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    bool graphed = false;
    // device time of the kernel alone (host set-up excluded)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    const bool timed = cudaEventCreate(&ev0) == cudaSuccess && cudaEventCreate(&ev1) == cudaSuccess;
    if (timed) cudaEventRecord(ev0, s);
    if (rc == KMB_OK && use_graph) {
        // one cooperative kernel node, captured on a private stream (the caller's
        // may be the legacy default stream) and launched on the caller's
        cudaStream_t cap = nullptr;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            cfg.stream = cap;
            const cudaError_t le = cudaLaunchKernelEx(&cfg, persistent_kernel, dP, L, gb);
            const cudaError_t ce = cudaStreamEndCapture(cap, &graph);
            if (le == cudaSuccess && ce == cudaSuccess && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess &&
                cudaGraphLaunch(exec, s) == cudaSuccess)
                graphed = true;
        }
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (cap) cudaStreamDestroy(cap);
    }
    if (rc == KMB_OK && !graphed) {
        cfg.stream = s;
        if (cudaLaunchKernelEx(&cfg, persistent_kernel, dP, L, gb) != cudaSuccess) rc = KMB_ECUDA;
    }
    if (rc == KMB_OK) KMB_LAUNCHED();
    if (timed) cudaEventRecord(ev1, s);
    GridBarrier hb;
    std::memset(&hb, 0, sizeof(hb));
    if (rc == KMB_OK && (cudaMemcpyAsync(H.data(), dP, sizeof(Problem) * count, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                         cudaMemcpyAsync(&hb, gb, sizeof(hb), cudaMemcpyDeviceToHost, s) != cudaSuccess))
        rc = KMB_ECUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = KMB_ECUDA;
    if (rc == KMB_OK && hb.error) rc = hb.error == 1 ? KMB_ETIMEDOUT : KMB_ECUDA;
    if (rc == KMB_OK) {
        long long total_iters = 0;
        for (int64_t i = 0; i < count; ++i) {
            problems[i].iterations = H[i].iters;
            problems[i].last_shift = H[i].shift;
            total_iters += H[i].iters;
        }
        if (info) {
            info->problems = count;
            info->variants = (int32_t)classes.size();
            info->total_iterations = total_iters;
            info->graph_launches = graphed ? 1 : 0;
            float ms = 0.f;
            info->kernel_ms = (timed && cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) ? (double)ms : -1.0;
        }
    }
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    cudaFreeAsync(dP, s);
    cudaFreeAsync(dPre, s);
    cudaFreeAsync(dOrder, s);
    cudaFreeAsync(base, s);
    return rc;
}
