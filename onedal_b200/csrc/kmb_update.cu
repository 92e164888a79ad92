// Lloyd update on the GPU: centroid sums, counts, empty-cluster reseeding,
// centroid shift and the convergence test.
//
// Reference semantics (DAAL dense Lloyd):
//  - per-cluster sums S1 and counts S0 over the rows' labels, reduced in double
//      cpp/daal/src/algorithms/kmeans/kmeans_lloyd_impl.i:220-229, 363-411
//  - c_j = S1_j / S0_j for non-empty clusters; empty clusters take, in ascending
//    cluster order, the rows with the largest squared distance (descending)
//      cpp/daal/src/algorithms/kmeans/kmeans_lloyd_batch_impl.i:153-188,
//      kmeans_lloyd_impl.i:413-480
//  - shift = sum_j ||c_old - c_new||^2 ; stop when shift <= eps
//      kmeans_lloyd_batch_impl.i:189-212
//
// B200 design. The sums are FP64 and deterministic: rows are counting-sorted
// by label with a stable scatter (per-chunk histograms, label-major scan,
// warp-ranked scatter), then each cluster's rows are summed in row order in
// fixed pieces of `piece_rows` rows and the pieces are added in order. Equal
// labels therefore give bit-identical centroids run to run, which is what
// makes the eps == 0 fixed-point stop (DAAL's "centroids unchanged") exact.
// Every kernel returns at once when the device loop state says `done`.
#include "kmb_internal.cuh"

#include <algorithm>

namespace kmb {
namespace {

constexpr int kSmemKMax = 8192;      // labels counted in shared memory up to this k
constexpr int64_t kGroupChunks = 64; // chunks per scan group
constexpr int64_t kPieceRows = 512;  // rows per FP64 partial sum

__device__ __forceinline__ bool is_done(const LoopState *st) { return st && st->done; }
// The counting sort is skipped when the exact update applies the moved rows only.
__device__ __forceinline__ bool sort_skipped(const LoopState *st) { return st && (st->done || st->upd_mode == 1); }

// ---- counting sort ---------------------------------------------------------

__global__ void hist_smem_kernel(const int32_t *__restrict__ labels, int64_t n, int k, int64_t R,
                                 int32_t *__restrict__ H, const LoopState *st) {
    if (sort_skipped(st)) return;
    extern __shared__ int sh[];
    for (int j = threadIdx.x; j < k; j += blockDim.x) sh[j] = 0;
    __syncthreads();
    const int64_t c = blockIdx.x;
    const int64_t b = c * R, e = min(n, b + R);
    for (int64_t r = b + threadIdx.x; r < e; r += blockDim.x) atomicAdd(&sh[labels[r]], 1);
    __syncthreads();
    int32_t *Hc = H + c * (int64_t)k;
    for (int j = threadIdx.x; j < k; j += blockDim.x) Hc[j] = sh[j];
}

__global__ void zero_i32_kernel(int32_t *__restrict__ p, int64_t count, const LoopState *st) {
    if (sort_skipped(st)) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = 0;
}

__global__ void hist_global_kernel(const int32_t *__restrict__ labels, int64_t n, int k, int64_t R,
                                   int32_t *__restrict__ H, const LoopState *st) {
    if (sort_skipped(st)) return;
    const int64_t c = blockIdx.x;
    const int64_t b = c * R, e = min(n, b + R);
    int32_t *Hc = H + c * (int64_t)k;
    for (int64_t r = b + threadIdx.x; r < e; r += blockDim.x) atomicAdd(&Hc[labels[r]], 1);
}

// Gs[g][j] = sum of H[c][j] over the chunks c of group g.
__global__ void scan_group_sum_kernel(const int32_t *__restrict__ H, int64_t n_chunks, int k,
                                      int64_t *__restrict__ Gs, const LoopState *st) {
    if (sort_skipped(st)) return;
    const int j = blockIdx.y * blockDim.x + threadIdx.x;
    if (j >= k) return;
    const int64_t g = blockIdx.x;
    const int64_t c0 = g * kGroupChunks, c1 = min(n_chunks, c0 + kGroupChunks);
    int64_t s = 0;
#pragma unroll 8
    for (int64_t c = c0; c < c1; ++c) s += H[c * k + j];
    Gs[g * k + j] = s;
}

// Exclusive scan of Gs over groups, per label; counts[j] = total rows of label j.
__global__ void scan_groups_kernel(int64_t *__restrict__ Gs, int64_t n_groups, int k, int64_t *__restrict__ counts,
                                   const LoopState *st) {
    if (sort_skipped(st)) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    int64_t run = 0;
    for (int64_t g = 0; g < n_groups; ++g) {
        const int64_t v = Gs[g * k + j];
        Gs[g * k + j] = run;
        run += v;
    }
    counts[j] = run;
}

// Single block: offsets = exclusive scan of counts (k+1 entries) and
// piece_base = exclusive scan of ceil(counts / piece_rows) (k+1 entries).
__global__ void offsets_kernel(const int64_t *__restrict__ counts, int k, int64_t piece_rows,
                               int64_t *__restrict__ offsets, int64_t *__restrict__ piece_base, const LoopState *st) {
    if (sort_skipped(st)) return;
    __shared__ int64_t s_rows[1024], s_pcs[1024];
    const int T = blockDim.x;
    const int per = (k + T - 1) / T;
    const int j0 = threadIdx.x * per, j1 = min(k, j0 + per);
    int64_t rows = 0, pcs = 0;
    for (int j = j0; j < j1; ++j) {
        rows += counts[j];
        pcs += (counts[j] + piece_rows - 1) / piece_rows;
    }
    s_rows[threadIdx.x] = rows;
    s_pcs[threadIdx.x] = pcs;
    __syncthreads();
    // Inclusive Hillis-Steele scan over the per-thread totals.
    for (int off = 1; off < T; off <<= 1) {
        int64_t a = 0, b = 0;
        if ((int)threadIdx.x >= off) {
            a = s_rows[threadIdx.x - off];
            b = s_pcs[threadIdx.x - off];
        }
        __syncthreads();
        s_rows[threadIdx.x] += a;
        s_pcs[threadIdx.x] += b;
        __syncthreads();
    }
    int64_t r = s_rows[threadIdx.x] - rows, p = s_pcs[threadIdx.x] - pcs;
    for (int j = j0; j < j1; ++j) {
        offsets[j] = r;
        piece_base[j] = p;
        r += counts[j];
        p += (counts[j] + piece_rows - 1) / piece_rows;
    }
    if (threadIdx.x == T - 1) {
        offsets[k] = s_rows[T - 1];
        piece_base[k] = s_pcs[T - 1];
    }
}

// H[c][j] <- first output position of chunk c's rows with label j.
__global__ void scan_chunks_kernel(int32_t *__restrict__ H, int64_t n_chunks, int k, const int64_t *__restrict__ Gs,
                                   const int64_t *__restrict__ offsets, const LoopState *st) {
    if (sort_skipped(st)) return;
    const int j = blockIdx.y * blockDim.x + threadIdx.x;
    if (j >= k) return;
    const int64_t g = blockIdx.x;
    const int64_t c0 = g * kGroupChunks, c1 = min(n_chunks, c0 + kGroupChunks);
    int64_t run = offsets[j] + Gs[g * k + j];
    for (int64_t c = c0; c < c1; ++c) {
        const int32_t v = H[c * k + j];
        H[c * k + j] = (int32_t)run;
        run += v;
    }
}

// One warp per chunk: rows are visited in order 32 at a time; equal labels in a
// group are ranked by lane, so the scatter is stable.
template <bool SMEM>
__global__ void scatter_kernel(const int32_t *__restrict__ labels, int64_t n, int k, int64_t R,
                               int32_t *__restrict__ H, int32_t *__restrict__ perm, const LoopState *st) {
    if (sort_skipped(st)) return;
    extern __shared__ int sh[];
    const int lane = threadIdx.x;
    const int64_t c = blockIdx.x;
    int32_t *Hc = H + c * (int64_t)k;
    int *cnt = SMEM ? sh : Hc;
    if (SMEM) {
        for (int j = lane; j < k; j += 32) sh[j] = Hc[j];
        __syncwarp();
    }
    const int64_t b = c * R, e = min(n, b + R);
    const unsigned lt = (1u << lane) - 1u;
    for (int64_t base = b; base < e; base += 32) {
        const int64_t r = base + lane;
        const bool valid = r < e;
        const unsigned mask = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const int lab = labels[r];
            const unsigned peers = __match_any_sync(mask, lab);
            const int rank = __popc(peers & lt);
            const int pos = cnt[lab] + rank;
            perm[pos] = (int32_t)r;
            __syncwarp(mask);
            if (lane == __ffs(peers) - 1) cnt[lab] = pos - rank + __popc(peers);
        }
        __syncwarp();
    }
}

// ---- FP64 sums ---------------------------------------------------------------

// Thread layout for row-sum style kernels over d columns with NT threads:
// dl columns lanes (power of two >= min(d, NT)), rp = NT / dl rows in parallel.
__device__ __forceinline__ void row_layout(int d, int nt, int &dl, int &rp) {
    dl = 32;
    while (dl < d && dl < nt) dl <<= 1;
    rp = nt / dl;
}

// Block p sums the rows of piece p (part of one cluster's segment of `perm`)
// into records[p * d + t], in row order.
template <typename F>
__global__ void __launch_bounds__(128)
segsum_kernel(const F *__restrict__ X, int d, int k, const int32_t *__restrict__ perm,
              const int64_t *__restrict__ offsets, const int64_t *__restrict__ piece_base, int64_t piece_rows,
              double *__restrict__ records, const LoopState *st) {
    if (is_done(st)) return;
    constexpr int NT = 128;
    __shared__ int32_t rows[kPieceRows];
    __shared__ double part[NT];
    const int64_t p = blockIdx.x;
    if (p >= piece_base[k]) return;
    // cluster j: piece_base[j] <= p < piece_base[j + 1]
    int lo = 0, hi = k;  // invariant: piece_base[lo] <= p < piece_base[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (piece_base[mid] <= p) lo = mid; else hi = mid;
    }
    const int j = lo;
    const int64_t q = p - piece_base[j];
    const int64_t s = offsets[j] + q * piece_rows;
    const int64_t e = min(s + piece_rows, offsets[j + 1]);
    const int cnt = (int)(e - s);
    for (int i = threadIdx.x; i < cnt; i += NT) rows[i] = perm[s + i];
    __syncthreads();

    int dl, rp;
    row_layout(d, NT, dl, rp);
    const int t = threadIdx.x % dl, rr = threadIdx.x / dl;
    for (int t0 = 0; t0 < d; t0 += dl) {
        const int col = t0 + t;
        double acc = 0.0;
        if (col < d) {
            int i = rr;
            for (; i + 3 * rp < cnt; i += 4 * rp) {
                const F v0 = X[(int64_t)rows[i] * d + col];
                const F v1 = X[(int64_t)rows[i + rp] * d + col];
                const F v2 = X[(int64_t)rows[i + 2 * rp] * d + col];
                const F v3 = X[(int64_t)rows[i + 3 * rp] * d + col];
                acc += (double)v0;
                acc += (double)v1;
                acc += (double)v2;
                acc += (double)v3;
            }
            for (; i < cnt; i += rp) acc += (double)X[(int64_t)rows[i] * d + col];
        }
        part[threadIdx.x] = acc;
        __syncthreads();
        if (rr == 0 && col < d) {
            double tot = part[t];
            for (int r2 = 1; r2 < rp; ++r2) tot += part[r2 * dl + t];
            records[p * d + col] = tot;
        }
        __syncthreads();
    }
}

// CSR form of segsum_kernel: one warp per piece. The piece's record is zeroed,
// then its rows' stored entries are added in row order (a row's columns are
// distinct, so its lanes never collide; __syncwarp orders consecutive rows).
template <typename F>
__global__ void __launch_bounds__(128)
csr_segsum_kernel(const F *__restrict__ vals, const int32_t *__restrict__ cols, const int64_t *__restrict__ rowptr,
                  int d, int k, const int32_t *__restrict__ perm, const int64_t *__restrict__ offsets,
                  const int64_t *__restrict__ piece_base, int64_t piece_rows, int64_t max_pieces,
                  double *__restrict__ records, const LoopState *st) {
    if (is_done(st)) return;
    const int lane = threadIdx.x & 31;
    const int64_t p = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    if (p >= max_pieces || p >= piece_base[k]) return;
    int lo = 0, hi = k;  // invariant: piece_base[lo] <= p < piece_base[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (piece_base[mid] <= p) lo = mid; else hi = mid;
    }
    const int j = lo;
    const int64_t q = p - piece_base[j];
    const int64_t s = offsets[j] + q * piece_rows;
    const int64_t e = min(s + piece_rows, offsets[j + 1]);
    double *rec = records + p * (int64_t)d;
    for (int t = lane; t < d; t += 32) rec[t] = 0.0;
    __syncwarp();
    for (int64_t i = s; i < e; ++i) {
        const int64_t r = perm[i];
        for (int64_t x = rowptr[r] + lane; x < rowptr[r + 1]; x += 32) rec[cols[x]] += (double)vals[x];
        __syncwarp();
    }
}

// S[t] = sum over pieces p0..p1-1 of records[p * d + t], added in piece order
// (four loads in flight per step; the additions stay sequential).
__device__ __forceinline__ double piece_sum(const double *__restrict__ records, int64_t p0, int64_t p1, int64_t d,
                                            int t) {
    double S = 0.0;
    int64_t p = p0;
    for (; p + 4 <= p1; p += 4) {
        const double a = records[p * d + t], b = records[(p + 1) * d + t];
        const double c = records[(p + 2) * d + t], e = records[(p + 3) * d + t];
        S += a;
        S += b;
        S += c;
        S += e;
    }
    for (; p < p1; ++p) S += records[p * d + t];
    return S;
}

constexpr int kFinalizeCols = 128;  // columns per finalize block (one per thread)

// Block (j, tile): S = sum of cluster j's pieces (in order) for the tile's
// columns; c = F(S / count); the tile's shift part. One large cluster thus
// spreads over d / 128 blocks instead of serialising on one.
template <typename F>
__global__ void __launch_bounds__(kFinalizeCols)
finalize_kernel(const double *__restrict__ records, const int64_t *__restrict__ counts,
                const int64_t *__restrict__ piece_base, const F *__restrict__ C_old, F *__restrict__ C_new, int d,
                double *__restrict__ shift_tiles, int32_t *__restrict__ empty_flag, const LoopState *st) {
    if (is_done(st)) return;
    __shared__ double red[kFinalizeCols / 32];
    const int j = blockIdx.x;
    const int t = blockIdx.y * kFinalizeCols + threadIdx.x;
    const int64_t cnt = counts[j];
    double acc = 0.0;
    if (t < d) {
        const F old = C_old[(int64_t)j * d + t];
        if (cnt > 0) {
            const F c = F(piece_sum(records, piece_base[j], piece_base[j + 1], d, t) / (double)cnt);
            const double df = (double)old - (double)c;
            acc = df * df;
            C_new[(int64_t)j * d + t] = c;
        } else {
            C_new[(int64_t)j * d + t] = old;
        }
    }
    for (int m = 16; m >= 1; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < kFinalizeCols / 32; ++w) tot += red[w];
        shift_tiles[(int64_t)j * gridDim.y + blockIdx.y] = tot;
        if (blockIdx.y == 0) empty_flag[j] = cnt > 0 ? 0 : 1;
    }
}

// shift_part[j] = the tiles' parts of cluster j, in tile order.
__global__ void shift_tiles_kernel(const double *__restrict__ shift_tiles, int k, int tiles,
                                   double *__restrict__ shift_part, const LoopState *st) {
    if (is_done(st)) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int y = 0; y < tiles; ++y) s += shift_tiles[(int64_t)j * tiles + y];
        shift_part[j] = s;
    }
}

// Sums of the pieces without the division (sharded training); block (j, tile).
__global__ void sums_kernel(const double *__restrict__ records, const int64_t *__restrict__ counts_in,
                            const int64_t *__restrict__ piece_base, int d, double *__restrict__ sums,
                            int64_t *__restrict__ counts_out) {
    const int j = blockIdx.x;
    const int t = blockIdx.y * kFinalizeCols + threadIdx.x;
    if (t < d) sums[(int64_t)j * d + t] = piece_sum(records, piece_base[j], piece_base[j + 1], d, t);
    if (threadIdx.x == 0 && blockIdx.y == 0) counts_out[j] = counts_in[j];
}

// Single block: lists empty clusters in ascending order; when none, reduces the
// shift in a fixed order.
__global__ void empties_kernel(const int32_t *__restrict__ empty_flag, int k, int32_t *__restrict__ empty_ids,
                               const double *__restrict__ shift_part, LoopState *st) {
    if (is_done(st)) return;
    __shared__ int s_cnt[1024];
    __shared__ double s_sh[1024];
    const int T = blockDim.x;
    const int per = (k + T - 1) / T;
    const int j0 = threadIdx.x * per, j1 = min(k, j0 + per);
    int c = 0;
    double sh = 0.0;
    for (int j = j0; j < j1; ++j) {
        c += empty_flag[j];
        sh += shift_part[j];
    }
    s_cnt[threadIdx.x] = c;
    s_sh[threadIdx.x] = sh;
    __syncthreads();
    for (int off = 1; off < T; off <<= 1) {
        int a = 0;
        if ((int)threadIdx.x >= off) a = s_cnt[threadIdx.x - off];
        __syncthreads();
        s_cnt[threadIdx.x] += a;
        __syncthreads();
    }
    int pos = s_cnt[threadIdx.x] - c;
    for (int j = j0; j < j1; ++j)
        if (empty_flag[j]) empty_ids[pos++] = j;
    if (threadIdx.x == 0) {
        const int ne = s_cnt[T - 1];
        st->n_empty = ne;
        if (ne == 0) {
            double tot = 0.0;
            for (int w = 0; w < T; ++w) tot += s_sh[w];
            st->shift = tot;
        }
    }
}

// ---- empty-cluster reseeding: top-m rows by squared distance ---------------

template <typename F> struct KeyOf;
template <> struct KeyOf<float> {
    using U = unsigned int;
    static constexpr int BITS = 32;
    __device__ static U key(float v) {
        const U u = __float_as_uint(v);
        return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    }
};
template <> struct KeyOf<double> {
    using U = unsigned long long;
    static constexpr int BITS = 64;
    __device__ static U key(double v) {
        const U u = (U)__double_as_longlong(v);
        return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
    }
};

struct SelState {
    unsigned long long prefix;
    unsigned long long mask;
    long long need;       // rows still to take at or below the current prefix
    long long above;      // rows strictly above the threshold
    int active;
};

// Exact squared distances for the empty-cluster candidates: when some cluster is
// empty, d2 of every row becomes ||x - c_label||^2 summed in FP64 (rounded to F),
// so the candidate order does not depend on the assignment form's rounding (the
// tensor-core forms' distances carry their contraction error outside the recheck
// band). One warp per row; nothing runs when no cluster is empty.
template <typename F>
__global__ void refresh_d2_kernel(const F *__restrict__ X, int64_t n, int d, const F *__restrict__ C,
                                  const int32_t *__restrict__ labels, F *__restrict__ d2, const LoopState *st) {
    if (is_done(st) || st->n_empty == 0) return;
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
        const F *x = X + r * d, *c = C + (int64_t)labels[r] * d;
        double acc = 0.0;
        for (int t = lane; t < d; t += 32) {
            const double df = (double)x[t] - (double)c[t];
            acc += df * df;
        }
        for (int m = 16; m >= 1; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
        if (lane == 0) d2[r] = F(acc);
    }
}

__global__ void sel_init_kernel(SelState *ss, unsigned int *hist, const LoopState *st) {
    if (is_done(st) || st->n_empty == 0) return;
    if (threadIdx.x == 0) {
        ss->prefix = 0;
        ss->mask = 0;
        ss->need = st->n_empty;
        ss->above = 0;
        ss->active = 1;
    }
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
}

template <typename F>
__global__ void sel_hist_kernel(const F *__restrict__ d2, int64_t n, int shift, const SelState *ss,
                                unsigned int *__restrict__ hist, const LoopState *st) {
    if (is_done(st) || st->n_empty == 0) return;
    using K = KeyOf<F>;
    __shared__ unsigned int sh[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const unsigned long long prefix = ss->prefix, mask = ss->mask;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long key = (unsigned long long)K::key(d2[i]);
        if ((key & mask) == prefix) atomicAdd(&sh[(key >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

__global__ void sel_pick_kernel(SelState *ss, unsigned int *hist, int shift, const LoopState *st) {
    if (is_done(st) || st->n_empty == 0) return;
    if (threadIdx.x == 0) {
        long long cum = 0;
        int b = 255;
        for (; b >= 0; --b) {
            if (cum + (long long)hist[b] >= ss->need) break;
            cum += hist[b];
        }
        if (b < 0) b = 0;  // not reachable when need <= rows matching the prefix
        ss->need -= cum;
        ss->above += cum;
        ss->prefix |= ((unsigned long long)b) << shift;
        ss->mask |= 0xFFull << shift;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
}

struct Cand {
    unsigned long long key;
    long long row;
};

// Single block: rows with key > T in row order, then the lowest rows with key == T.
template <typename F>
__global__ void sel_collect_kernel(const F *__restrict__ d2, int64_t n, const SelState *ss, Cand *__restrict__ cand,
                                   int cap, const LoopState *st) {
    if (is_done(st) || st->n_empty == 0) return;
    using K = KeyOf<F>;
    __shared__ int s_hi[1024], s_eq[1024];
    __shared__ long long base_hi, base_eq;
    const unsigned long long T = ss->prefix;
    const long long n_hi = ss->above, n_eq = ss->need;
    if (threadIdx.x == 0) {
        base_hi = 0;
        base_eq = 0;
    }
    __syncthreads();
    for (int64_t b0 = 0; b0 < n; b0 += blockDim.x) {
        if (base_hi >= n_hi && base_eq >= n_eq) break;
        const int64_t i = b0 + threadIdx.x;
        unsigned long long key = 0;
        int is_hi = 0, is_eq = 0;
        if (i < n) {
            key = (unsigned long long)K::key(d2[i]);
            is_hi = key > T;
            is_eq = key == T;
        }
        s_hi[threadIdx.x] = is_hi;
        s_eq[threadIdx.x] = is_eq;
        __syncthreads();
        for (int off = 1; off < (int)blockDim.x; off <<= 1) {
            int a = 0, c = 0;
            if ((int)threadIdx.x >= off) {
                a = s_hi[threadIdx.x - off];
                c = s_eq[threadIdx.x - off];
            }
            __syncthreads();
            s_hi[threadIdx.x] += a;
            s_eq[threadIdx.x] += c;
            __syncthreads();
        }
        const long long ph = base_hi + s_hi[threadIdx.x] - is_hi;
        const long long pe = base_eq + s_eq[threadIdx.x] - is_eq;
        if (is_hi && ph < n_hi && ph < cap) {
            cand[ph].key = key;
            cand[ph].row = i;
        }
        if (is_eq && pe < n_eq && n_hi + pe < cap) {
            cand[n_hi + pe].key = key;
            cand[n_hi + pe].row = i;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) {
            base_hi += s_hi[threadIdx.x];
            base_eq += s_eq[threadIdx.x];
        }
        __syncthreads();
    }
}

// Single block bitonic sort of the m = n_empty candidates by (key desc, row asc);
// positions [m, P) hold sentinels that order last. The buffer holds
// next_pow2(k) entries.
__device__ __forceinline__ bool cand_before(const Cand &a, const Cand &b) {
    return a.key > b.key || (a.key == b.key && a.row < b.row);
}

__global__ void sel_sort_kernel(Cand *__restrict__ cand, const LoopState *st) {
    if (is_done(st) || st->n_empty == 0) return;
    const long long m = st->n_empty;
    if (m <= 1) return;
    long long P = 1;
    while (P < m) P <<= 1;
    for (long long i = m + threadIdx.x; i < P; i += blockDim.x) {
        cand[i].key = 0ull;
        cand[i].row = 0x7fffffffffffffffll;
    }
    __syncthreads();
    for (long long size = 2; size <= P; size <<= 1) {
        for (long long stride = size >> 1; stride > 0; stride >>= 1) {
            for (long long i = threadIdx.x; i < P; i += blockDim.x) {
                const long long j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const Cand a = cand[i], b = cand[j];
                    const bool swap = up ? cand_before(b, a) : cand_before(a, b);
                    if (swap) {
                        cand[i] = b;
                        cand[j] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

__global__ void select_state_kernel(LoopState *st, int m) {
    LoopState z = {};
    z.n_empty = m;
    *st = z;
}

__global__ void cand_rows_kernel(const Cand *__restrict__ cand, int m, long long *__restrict__ rows) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) rows[e] = cand[e].row;
}

// Empty cluster e (ascending id) takes candidate e; shift part = ||c_old - x||^2.
template <typename F>
__global__ void reseed_apply_kernel(const F *__restrict__ X, int d, const Cand *__restrict__ cand,
                                    const int32_t *__restrict__ empty_ids, const F *__restrict__ C_old,
                                    F *__restrict__ C_new, double *__restrict__ shift_part, LoopState *st) {
    if (is_done(st)) return;
    const int ne = st->n_empty;
    __shared__ double red[32];
    for (int e = blockIdx.x; e < ne; e += gridDim.x) {
        const int id = empty_ids[e];
        const long long row = cand[e].row;
        double acc = 0.0;
        for (int t = threadIdx.x; t < d; t += blockDim.x) {
            const F x = X[row * d + t];
            const double df = (double)C_old[(int64_t)id * d + t] - (double)x;
            acc += df * df;
            C_new[(int64_t)id * d + t] = x;
        }
        for (int m = 16; m >= 1; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
            shift_part[id] = tot;
        }
        __syncthreads();
    }
}

// CSR form of reseed_apply_kernel: the candidate row expanded to dense.
template <typename F>
__global__ void csr_reseed_apply_kernel(const F *__restrict__ vals, const int32_t *__restrict__ cols,
                                        const int64_t *__restrict__ rowptr, int d, const Cand *__restrict__ cand,
                                        const int32_t *__restrict__ empty_ids, const F *__restrict__ C_old,
                                        F *__restrict__ C_new, double *__restrict__ shift_part, LoopState *st) {
    if (is_done(st)) return;
    const int ne = st->n_empty;
    __shared__ double red[32];
    for (int e = blockIdx.x; e < ne; e += gridDim.x) {
        const int id = empty_ids[e];
        const long long row = cand[e].row;
        F *c = C_new + (int64_t)id * d;
        for (int t = threadIdx.x; t < d; t += blockDim.x) c[t] = F(0);
        __syncthreads();
        for (int64_t x = rowptr[row] + threadIdx.x; x < rowptr[row + 1]; x += blockDim.x) c[cols[x]] = vals[x];
        __syncthreads();
        double acc = 0.0;
        for (int t = threadIdx.x; t < d; t += blockDim.x) {
            const double df = (double)C_old[(int64_t)id * d + t] - (double)c[t];
            acc += df * df;
        }
        for (int m = 16; m >= 1; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
            shift_part[id] = tot;
        }
        __syncthreads();
    }
}

// After reseeding: shift = sum of all parts in a fixed order (single block).
__global__ void shift_total_kernel(const double *__restrict__ shift_part, int k, LoopState *st) {
    if (is_done(st) || st->n_empty == 0) return;
    __shared__ double s[1024];
    const int T = blockDim.x;
    const int per = (k + T - 1) / T;
    const int j0 = threadIdx.x * per, j1 = min(k, j0 + per);
    double a = 0.0;
    for (int j = j0; j < j1; ++j) a += shift_part[j];
    s[threadIdx.x] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < T; ++w) tot += s[w];
        st->shift = tot;
        st->empty_events += st->n_empty;
    }
}

template <typename F>
__global__ void commit_copy_kernel(const F *__restrict__ src, F *__restrict__ dst, int64_t count, const LoopState *st) {
    if (is_done(st)) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

__global__ void decide_kernel(LoopState *st) {
    if (st->done) return;
    st->iterations += 1;
    if (st->shift <= st->eps) st->done = 1;
}

// ---- objective -------------------------------------------------------------

template <typename F>
__global__ void __launch_bounds__(256)
objective_kernel(const F *__restrict__ X, int64_t n, int d, const F *__restrict__ C, const int32_t *__restrict__ labels,
                 double *__restrict__ partials) {
    constexpr int NT = 256;
    __shared__ double part[NT];
    int dl, rp;
    row_layout(d, NT, dl, rp);
    const int t = threadIdx.x % dl, rr = threadIdx.x / dl;
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t b = (int64_t)blockIdx.x * per, e = min(n, b + per);
    double acc = 0.0;
    for (int t0 = 0; t0 < d; t0 += dl) {
        const int col = t0 + t;
        if (col >= d) continue;
        for (int64_t i = b + rr; i < e; i += rp) {
            const double df = (double)X[i * d + col] - (double)C[(int64_t)labels[i] * d + col];
            acc += df * df;
        }
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = part[0];
}

__global__ void sum_partials_kernel(const double *__restrict__ partials, int count, double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < count; ++i) s += partials[i];
        *out = s;
    }
}

// ---- sharded (SPMD) helpers ---------------------------------------------------

// Centroids from all-reduced FP64 sums and counts: c = F(S / count); empty
// clusters keep C_in (the caller reseeds them) and are flagged.
template <typename F>
__global__ void finalize_from_sums_kernel(const double *__restrict__ sums, const int64_t *__restrict__ counts,
                                          const F *__restrict__ C_old, F *__restrict__ C_new, int d,
                                          double *__restrict__ shift_part, int32_t *__restrict__ empty_flag) {
    __shared__ double red[32];
    const int j = blockIdx.x;
    const int64_t cnt = counts[j];
    double acc = 0.0;
    for (int t = threadIdx.x; t < d; t += blockDim.x) {
        const F old = C_old[(int64_t)j * d + t];
        if (cnt > 0) {
            const F c = F(sums[(int64_t)j * d + t] / (double)cnt);
            const double df = (double)old - (double)c;
            acc += df * df;
            C_new[(int64_t)j * d + t] = c;
        } else {
            C_new[(int64_t)j * d + t] = old;
        }
    }
    for (int m = 16; m >= 1; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        shift_part[j] = tot;
        empty_flag[j] = cnt > 0 ? 0 : 1;
    }
}

// Fixed-order sum of k doubles (single block).
__global__ void sum_doubles_kernel(const double *__restrict__ v, int k, double *__restrict__ out) {
    __shared__ double s[1024];
    const int T = blockDim.x;
    const int per = (k + T - 1) / T;
    const int j0 = threadIdx.x * per, j1 = min(k, j0 + per);
    double a = 0.0;
    for (int j = j0; j < j1; ++j) a += v[j];
    s[threadIdx.x] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < T; ++w) tot += s[w];
        *out = tot;
    }
}

// Deterministic FP64 sum of n values of F (per-block partials, then one block).
template <typename F>
__global__ void sum_values_kernel(const F *__restrict__ v, int64_t n, double *__restrict__ partials) {
    __shared__ double s[256];
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t b = (int64_t)blockIdx.x * per, e = min(n, b + per);
    double a = 0.0;
    for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) a += (double)v[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = s[0];
}

__global__ void list_empties_kernel(const int32_t *__restrict__ empty_flag, int k, int32_t *__restrict__ empty_ids,
                                    long long *__restrict__ n_empty) {
    __shared__ int s_cnt[1024];
    const int T = blockDim.x;
    const int per = (k + T - 1) / T;
    const int j0 = threadIdx.x * per, j1 = min(k, j0 + per);
    int c = 0;
    for (int j = j0; j < j1; ++j) c += empty_flag[j];
    s_cnt[threadIdx.x] = c;
    __syncthreads();
    for (int off = 1; off < T; off <<= 1) {
        int a = 0;
        if ((int)threadIdx.x >= off) a = s_cnt[threadIdx.x - off];
        __syncthreads();
        s_cnt[threadIdx.x] += a;
        __syncthreads();
    }
    int pos = s_cnt[threadIdx.x] - c;
    for (int j = j0; j < j1; ++j)
        if (empty_flag[j]) empty_ids[pos++] = j;
    if (threadIdx.x == 0) *n_empty = s_cnt[T - 1];
}

// ---- exact update (FP32 rows) -------------------------------------------------
// A value x of column t is the integer v = round(x * 2^E_t), |v| < 2^94, with E_t
// chosen once per call from the column's largest |x|: every float within 2^70 of
// that maximum is represented exactly (a 24-bit significand), smaller ones to
// 2^-94 of the maximum. v is kept as three signed 32-bit limbs, v = l2 * 2^64 +
// l1 * 2^32 + l0 (fixed_of), and a cluster-column sum as three int64 limb sums,
// so additions and subtractions of rows in any order give the same integer. The
// finalize folds the limb sums into one 128-bit integer, stores it back
// normalised, and converts it to the nearest double.

// colexp[t] <- max |x| of column t, as float bits (non-negative floats order as ints).
__global__ void colmax_kernel(const float *__restrict__ X, int64_t n, int d, unsigned *__restrict__ colbits,
                              const LoopState *st) {
    if (is_done(st)) return;
    extern __shared__ unsigned smax[];
    for (int t = threadIdx.x; t < d; t += blockDim.x) smax[t] = 0u;
    __syncthreads();
    const int64_t total = n * (int64_t)d;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = fabsf(X[i]);
        if (v > 0.0f) atomicMax(&smax[(int)(i % d)], __float_as_uint(v));
    }
    __syncthreads();
    for (int t = threadIdx.x; t < d; t += blockDim.x)
        if (smax[t]) atomicMax(&colbits[t], smax[t]);
}

// The same maxima for d <= 1024 with one register maximum per (thread, column):
// thread t covers column t % d of every (256 / d)-th row when d <= 256, else
// columns t, t + 256, ... of every row; reads are coalesced along the rows and
// each thread issues one atomic per column at the end (NaN never compares greater
// and is skipped, as above).
__global__ void __launch_bounds__(256) colmax_rows_kernel(const float *__restrict__ X, int64_t n, int d,
                                                          unsigned *__restrict__ colbits, const LoopState *st) {
    if (is_done(st)) return;
    if (d <= 256) {
        const int rpb = 256 / d;
        if ((int)threadIdx.x >= rpb * d) return;
        const int c = threadIdx.x % d;
        float m = 0.0f;
        for (int64_t r = (int64_t)blockIdx.x * rpb + threadIdx.x / d; r < n; r += (int64_t)gridDim.x * rpb) {
            const float v = fabsf(X[r * d + c]);
            if (v > m) m = v;
        }
        if (m > 0.0f) atomicMax(&colbits[c], __float_as_uint(m));
    } else {
        float m[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int64_t r = blockIdx.x; r < n; r += gridDim.x) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int c = threadIdx.x + 256 * q;
                if (c < d) {
                    const float v = fabsf(X[r * d + c]);
                    if (v > m[q]) m[q] = v;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (m[q] > 0.0f) atomicMax(&colbits[threadIdx.x + 256 * q], __float_as_uint(m[q]));
    }
}

__global__ void colmax_global_kernel(const float *__restrict__ X, int64_t n, int d, unsigned *__restrict__ colbits,
                                     const LoopState *st) {
    if (is_done(st)) return;
    const int64_t total = n * (int64_t)d;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = fabsf(X[i]);
        if (v > 0.0f) atomicMax(&colbits[(int)(i % d)], __float_as_uint(v));
    }
}

// E_t such that max |x_t| * 2^E_t < 2^94 (E_t = 0 for an all-zero column); the
// non-finite maximum of a column holding inf/NaN gives E_t = 0 too.
__global__ void colexp_kernel(int *__restrict__ colexp, int d, const LoopState *st) {
    if (is_done(st)) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < d; t += gridDim.x * blockDim.x) {
        const unsigned b = (unsigned)colexp[t];
        const float m = __uint_as_float(b);
        int e = 0;
        if (b != 0u && isfinite(m)) {
            int ex;
            frexpf(m, &ex);  // m < 2^ex
            e = kExactMaxBits - ex;
        }
        colexp[t] = e;
    }
}

// Rows whose label changed since the previous pass (block sums added atomically:
// an integer, so the order does not matter); then the update mode.
__global__ void count_moved_kernel(const int32_t *__restrict__ labels, const int32_t *__restrict__ prev, int64_t n,
                                   LoopState *st) {
    if (is_done(st) || !st->upd_valid) return;
    __shared__ int s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    int c = 0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        c += labels[r] != prev[r];
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&s_cnt, c);
    __syncthreads();
    if (threadIdx.x == 0 && s_cnt)
        atomicAdd(reinterpret_cast<unsigned long long *>(&st->n_moved), (unsigned long long)s_cnt);
}

__global__ void choose_mode_kernel(int64_t n, LoopState *st) {
    if (is_done(st)) return;
    // moved rows only when at most an eighth moved (20M x 128, BF16x3, 20 iterations:
    // update 1.85-1.93 ms per iteration at n/8, 1.95 at n/4, 2.04 at n/2, 2.08-2.11 at n/16)
    st->upd_mode = (st->upd_valid && st->n_moved * 8 <= n) ? 1 : 0;
}

// Block p sums piece p's rows (one cluster's rows in row order) as integers.
// records: three limb planes of (pieces x d) int64.
__global__ void __launch_bounds__(128)
segsum_fixed_kernel(const float *__restrict__ X, int d, int k, const int32_t *__restrict__ perm,
                    const int64_t *__restrict__ offsets, const int64_t *__restrict__ piece_base, int64_t piece_rows,
                    int64_t max_pieces, const int *__restrict__ colexp, long long *__restrict__ records,
                    const LoopState *st) {
    if (sort_skipped(st)) return;
    constexpr int NT = 128;
    __shared__ int32_t rows[kPieceRows];
    __shared__ long long part[3][NT];
    const int64_t p = blockIdx.x;
    if (p >= piece_base[k]) return;
    int lo = 0, hi = k;  // invariant: piece_base[lo] <= p < piece_base[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (piece_base[mid] <= p) lo = mid; else hi = mid;
    }
    const int j = lo;
    const int64_t q = p - piece_base[j];
    const int64_t s = offsets[j] + q * piece_rows;
    const int64_t e = min(s + piece_rows, offsets[j + 1]);
    const int cnt = (int)(e - s);
    for (int i = threadIdx.x; i < cnt; i += NT) rows[i] = perm[s + i];
    __syncthreads();
    int dl, rp;
    row_layout(d, NT, dl, rp);
    const int t = threadIdx.x % dl, rr = threadIdx.x / dl;
    const int64_t plane = max_pieces * (int64_t)d;
    for (int t0 = 0; t0 < d; t0 += dl) {
        const int col = t0 + t;
        long long a0 = 0, a1 = 0, a2 = 0;
        if (col < d) {
            const int ex = colexp[col];
            int i = rr;
            for (; i + 7 * rp < cnt; i += 8 * rp) {  // eight gathered loads in flight per thread
                float v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = X[(int64_t)rows[i + u * rp] * d + col];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const Limbs L = fixed_of(v[u], ex);
                    a0 += L.l0;
                    a1 += L.l1;
                    a2 += L.l2;
                }
            }
            for (; i < cnt; i += rp) {
                const Limbs L = fixed_of(X[(int64_t)rows[i] * d + col], ex);
                a0 += L.l0;
                a1 += L.l1;
                a2 += L.l2;
            }
        }
        part[0][threadIdx.x] = a0;
        part[1][threadIdx.x] = a1;
        part[2][threadIdx.x] = a2;
        __syncthreads();
        if (rr == 0 && col < d) {
            long long t0s = part[0][t], t1s = part[1][t], t2s = part[2][t];
            for (int r2 = 1; r2 < rp; ++r2) {
                t0s += part[0][r2 * dl + t];
                t1s += part[1][r2 * dl + t];
                t2s += part[2][r2 * dl + t];
            }
            records[p * d + col] = t0s;
            records[plane + p * d + col] = t1s;
            records[2 * plane + p * d + col] = t2s;
        }
        __syncthreads();
    }
}

// Moved rows (incremental mode): each leaves its old cluster's sums and joins the
// new one's (integer atomics, exact in any order); prev follows the labels.
// acc: three limb planes of (k x d) int64.
__global__ void apply_moves_kernel(const float *__restrict__ X, int64_t n, int d, int k,
                                   const int32_t *__restrict__ labels, int32_t *__restrict__ prev,
                                   const int *__restrict__ colexp, unsigned long long *__restrict__ acc,
                                   unsigned long long *__restrict__ cnt, const LoopState *st) {
    if (is_done(st) || st->upd_mode != 1) return;
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~(int64_t)31; base < n; base += stride) {
        const int64_t r = base + lane;
        int lab = -1, old = -1;
        if (r < n) {
            lab = labels[r];
            old = prev[r];
        }
        unsigned moved = __ballot_sync(0xffffffffu, r < n && lab != old);
        while (moved) {
            const int src = __ffs(moved) - 1;
            moved &= moved - 1;
            const int64_t row = base + src;
            const int nl = __shfl_sync(0xffffffffu, lab, src), ol = __shfl_sync(0xffffffffu, old, src);
            const float *x = X + row * d;
            const int64_t plane = (int64_t)k * d;
            for (int t = lane; t < d; t += 32) {
                const Limbs L = fixed_of(x[t], colexp[t]);
                const int64_t in = (int64_t)nl * d + t, out = (int64_t)ol * d + t;
                atomicAdd(&acc[in], (unsigned long long)L.l0);
                atomicAdd(&acc[plane + in], (unsigned long long)L.l1);
                atomicAdd(&acc[2 * plane + in], (unsigned long long)L.l2);
                atomicAdd(&acc[out], (unsigned long long)-L.l0);
                atomicAdd(&acc[plane + out], (unsigned long long)-L.l1);
                atomicAdd(&acc[2 * plane + out], (unsigned long long)-L.l2);
            }
            if (lane == 0) {
                atomicAdd(&cnt[nl], 1ull);
                atomicAdd(&cnt[ol], (unsigned long long)-1ll);
            }
        }
        if (r < n && lab != old) prev[r] = lab;
    }
}

// Full mode: prev <- labels.
__global__ void copy_prev_kernel(const int32_t *__restrict__ labels, int32_t *__restrict__ prev, int64_t n,
                                 const LoopState *st) {
    if (is_done(st) || st->upd_mode == 1) return;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        prev[r] = labels[r];
}

// Block (j, tile): cluster j's limb sums (full mode: from its pieces; incremental, or
// from_acc:
// the maintained ones), normalised and kept; c = F(S * 2^-E / count) in FP64; the
// tile's shift part and the empty flag, as finalize_kernel.
__global__ void __launch_bounds__(kFinalizeCols)
finalize_exact_kernel(const long long *__restrict__ records, int64_t max_pieces, const int64_t *__restrict__ counts_sort,
                      const int64_t *__restrict__ piece_base, const int *__restrict__ colexp, int k,
                      long long *__restrict__ lacc, long long *__restrict__ cnt, const float *__restrict__ C_old,
                      float *__restrict__ C_new, int d, double *__restrict__ shift_tiles,
                      int32_t *__restrict__ empty_flag, const LoopState *st, bool from_acc = false) {
    if (is_done(st)) return;
    __shared__ double red[kFinalizeCols / 32];
    const int j = blockIdx.x;
    const int t = blockIdx.y * kFinalizeCols + threadIdx.x;
    // from_acc: the maintained limb sums and counts hold this pass's sums in both
    // modes (the CSR form accumulates full passes there too)
    const bool full = !from_acc && st->upd_mode == 0;
    const long long c_j = full ? (long long)counts_sort[j] : cnt[j];
    double acc = 0.0;
    if (t < d) {
        const int64_t idx = (int64_t)j * d + t, plane = (int64_t)k * d, rplane = max_pieces * (int64_t)d;
        long long s0 = 0, s1 = 0, s2 = 0;
        if (full) {
            for (int64_t p = piece_base[j]; p < piece_base[j + 1]; ++p) {
                s0 += records[p * d + t];
                s1 += records[rplane + p * d + t];
                s2 += records[2 * rplane + p * d + t];
            }
        } else {
            s0 = lacc[idx];
            s1 = lacc[plane + idx];
            s2 = lacc[2 * plane + idx];
        }
        // one 128-bit integer, stored back normalised (l0, l1 in [0, 2^32))
        const __int128 S = ((__int128)s2 << 64) + ((__int128)s1 << 32) + (__int128)s0;
        lacc[idx] = (long long)(S & 0xffffffffll);
        lacc[plane + idx] = (long long)((S >> 32) & 0xffffffffll);
        lacc[2 * plane + idx] = (long long)(S >> 64);
        const float old = C_old[idx];
        if (c_j > 0) {
            const double Sd = S < 0 ? -u128_to_double((unsigned __int128)(-S)) : u128_to_double((unsigned __int128)S);
            const float c = (float)(ldexp(Sd, -colexp[t]) / (double)c_j);
            const double df = (double)old - (double)c;
            acc = df * df;
            C_new[idx] = c;
        } else {
            C_new[idx] = old;
        }
    }
    for (int m = 16; m >= 1; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < kFinalizeCols / 32; ++w) tot += red[w];
        shift_tiles[(int64_t)j * gridDim.y + blockIdx.y] = tot;
        if (blockIdx.y == 0) {
            empty_flag[j] = c_j > 0 ? 0 : 1;
            if (full) cnt[j] = c_j;
        }
    }
}

// ---- exact update of CSR rows with float values ------------------------------
// The same integers as the dense rows' exact update, from the stored entries (an
// unstored entry is a zero and adds nothing): the column scales come from the
// columns' largest stored |x|, which is the column's largest |x|. The sums are kept
// in the maintained limb planes and counts in both modes: a full pass clears them
// and adds every row's entries by integer atomics (exact in any order), an
// incremental pass moves the moved rows' entries from the old cluster to the new.

// colbits[t] <- max |x| over the stored entries of column t, as float bits.
__global__ void csr_colmax_kernel(const float *__restrict__ vals, const int32_t *__restrict__ cols, int64_t nnz,
                                  int d, bool in_smem, unsigned *__restrict__ colbits) {
    extern __shared__ unsigned smax[];
    if (in_smem) {
        for (int t = threadIdx.x; t < d; t += blockDim.x) smax[t] = 0u;
        __syncthreads();
    }
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < nnz; x += (int64_t)gridDim.x * blockDim.x) {
        const float v = fabsf(vals[x]);
        if (v > 0.0f) atomicMax(in_smem ? &smax[cols[x]] : &colbits[cols[x]], __float_as_uint(v));
    }
    if (in_smem) {
        __syncthreads();
        for (int t = threadIdx.x; t < d; t += blockDim.x)
            if (smax[t]) atomicMax(&colbits[t], smax[t]);
    }
}

// Full mode: limb planes and counts cleared.
__global__ void csr_exact_clear_kernel(long long *__restrict__ acc, int64_t words, long long *__restrict__ cnt, int k,
                                       const LoopState *st) {
    if (is_done(st) || st->upd_mode != 0) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (int64_t)gridDim.x * blockDim.x)
        acc[i] = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x)
        cnt[i] = 0;
}

// Full mode: one warp per row adds the row's stored entries to its cluster's limb
// sums; the CTA counts its rows per cluster in shared memory (k <= kCsrCountSmem)
// before one atomic per cluster.
constexpr int kCsrCountSmem = 8192;
__global__ void __launch_bounds__(256) csr_sums_fixed_kernel(const float *__restrict__ vals,
                                                             const int32_t *__restrict__ cols,
                                                             const int64_t *__restrict__ rowptr, int64_t n, int d,
                                                             int k, const int32_t *__restrict__ labels,
                                                             const int *__restrict__ colexp,
                                                             unsigned long long *__restrict__ acc,
                                                             unsigned long long *__restrict__ cnt, const LoopState *st) {
    if (is_done(st) || st->upd_mode != 0) return;
    extern __shared__ unsigned scnt[];
    const bool shared_counts = k <= kCsrCountSmem;
    if (shared_counts) {
        for (int j = threadIdx.x; j < k; j += blockDim.x) scnt[j] = 0u;
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
    const int64_t plane = (int64_t)k * d;
    for (int64_t r = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); r < n; r += warps) {
        const int lab = labels[r];
        if ((unsigned)lab >= (unsigned)k) continue;  // cannot happen: the assignment writes every row
        const int64_t base = (int64_t)lab * d;
        for (int64_t x = rowptr[r] + lane; x < rowptr[r + 1]; x += 32) {
            const int c = cols[x];
            const Limbs L = fixed_of(vals[x], colexp[c]);
            if (L.l0 | L.l1 | L.l2) {
                atomicAdd(&acc[base + c], (unsigned long long)L.l0);
                atomicAdd(&acc[plane + base + c], (unsigned long long)L.l1);
                atomicAdd(&acc[2 * plane + base + c], (unsigned long long)L.l2);
            }
        }
        if (lane == 0) {
            if (shared_counts) atomicAdd(&scnt[lab], 1u);
            else atomicAdd(&cnt[lab], 1ull);
        }
    }
    if (shared_counts) {
        __syncthreads();
        for (int j = threadIdx.x; j < k; j += blockDim.x)
            if (scnt[j]) atomicAdd(&cnt[j], (unsigned long long)scnt[j]);
    }
}

// Incremental mode: the moved rows' entries leave the old cluster's sums and join
// the new one's (a warp walks 32 rows, then each moved row's entries); prev follows
// the labels.
__global__ void csr_apply_moves_kernel(const float *__restrict__ vals, const int32_t *__restrict__ cols,
                                       const int64_t *__restrict__ rowptr, int64_t n, int d, int k,
                                       const int32_t *__restrict__ labels, int32_t *__restrict__ prev,
                                       const int *__restrict__ colexp, unsigned long long *__restrict__ acc,
                                       unsigned long long *__restrict__ cnt, const LoopState *st) {
    if (is_done(st) || st->upd_mode != 1) return;
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t plane = (int64_t)k * d;
    for (int64_t base = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~(int64_t)31; base < n; base += stride) {
        const int64_t r = base + lane;
        int lab = -1, old = -1;
        if (r < n) {
            lab = labels[r];
            old = prev[r];
        }
        unsigned moved = __ballot_sync(0xffffffffu, r < n && lab != old);
        while (moved) {
            const int src = __ffs(moved) - 1;
            moved &= moved - 1;
            const int64_t row = base + src;
            const int nl = __shfl_sync(0xffffffffu, lab, src), ol = __shfl_sync(0xffffffffu, old, src);
            for (int64_t x = rowptr[row] + lane; x < rowptr[row + 1]; x += 32) {
                const int c = cols[x];
                const Limbs L = fixed_of(vals[x], colexp[c]);
                if (L.l0 | L.l1 | L.l2) {
                    const int64_t in = (int64_t)nl * d + c, out = (int64_t)ol * d + c;
                    atomicAdd(&acc[in], (unsigned long long)L.l0);
                    atomicAdd(&acc[plane + in], (unsigned long long)L.l1);
                    atomicAdd(&acc[2 * plane + in], (unsigned long long)L.l2);
                    atomicAdd(&acc[out], (unsigned long long)-L.l0);
                    atomicAdd(&acc[plane + out], (unsigned long long)-L.l1);
                    atomicAdd(&acc[2 * plane + out], (unsigned long long)-L.l2);
                }
            }
            if (lane == 0) {
                atomicAdd(&cnt[nl], 1ull);
                atomicAdd(&cnt[ol], (unsigned long long)-1ll);
            }
        }
        if (r < n && lab != old) prev[r] = lab;
    }
}

// After the update: the maintained state describes this pass's labels.
__global__ void exact_valid_kernel(LoopState *st) {
    if (is_done(st)) return;
    st->upd_valid = 1;
    st->n_moved = 0;
}

}  // namespace

UpdatePlan make_update_plan(int64_t n, int64_t k, int64_t d) {
    UpdatePlan p;
    p.n = n;
    p.k = k;
    p.d = d;
    // Chunk histograms are n_chunks x k int32: keep them under 2^25 entries.
    int64_t R = 2048;
    const double need = (double)n * (double)k / (double)(1ll << 25);
    while ((double)R < need) R <<= 1;
    p.chunk_rows = R;
    p.n_chunks = n > 0 ? (n + R - 1) / R : 0;
    p.piece_rows = kPieceRows;
    p.max_pieces = (n + kPieceRows - 1) / kPieceRows + k;
    return p;
}

bool ensure_update_buffers(Workspace &ws, const UpdatePlan &p, size_t fsize, bool fp64_records) {
    const int64_t n_groups = (p.n_chunks + kGroupChunks - 1) / kGroupChunks;
    bool ok = true;
    ok &= ws.ensure(ws.H, sizeof(int32_t) * std::max<int64_t>(1, p.n_chunks * p.k));
    ok &= ws.ensure(ws.Gs, sizeof(int64_t) * std::max<int64_t>(1, n_groups * p.k));
    ok &= ws.ensure(ws.counts, sizeof(int64_t) * (p.k + 1));
    ok &= ws.ensure(ws.offsets, sizeof(int64_t) * (p.k + 1));
    ok &= ws.ensure(ws.piece_base, sizeof(int64_t) * (p.k + 1));
    ok &= ws.ensure(ws.perm, sizeof(int32_t) * std::max<int64_t>(1, p.n));
    if (fp64_records) ok &= ws.ensure(ws.records, sizeof(double) * p.max_pieces * p.d);
    ok &= ws.ensure(ws.shift_part, sizeof(double) * p.k);
    ok &= ws.ensure(ws.shift_tiles, sizeof(double) * p.k * ((p.d + kFinalizeCols - 1) / kFinalizeCols));
    ok &= ws.ensure(ws.empty_flag, sizeof(int32_t) * p.k);
    ok &= ws.ensure(ws.empty_ids, sizeof(int32_t) * p.k);
    ok &= ws.ensure(ws.sel_hist, sizeof(unsigned int) * 256);
    ok &= ws.ensure(ws.sel_state, sizeof(SelState));
    int64_t pk = 1;
    while (pk < p.k) pk <<= 1;
    ok &= ws.ensure(ws.cand, sizeof(Cand) * pk);
    ok &= ws.ensure(ws.obj_part, sizeof(double) * kObjectivePartials);
    (void)fsize;
    return ok;
}

// Stable counting sort of rows by label + FP64 piece sums (records).
static void sort_and_sum_pieces(const void *Xv, size_t fsize, const UpdatePlan &p, const int32_t *labels,
                                Workspace &ws, const LoopState *st, cudaStream_t s, const CsrRows *csr = nullptr,
                                bool sort_only = false) {
    const int k = (int)p.k;
    const int64_t n_groups = (p.n_chunks + kGroupChunks - 1) / kGroupChunks;
    int32_t *H = (int32_t *)ws.H.ptr;
    int64_t *Gs = (int64_t *)ws.Gs.ptr;
    int64_t *counts = (int64_t *)ws.counts.ptr;
    int64_t *offsets = (int64_t *)ws.offsets.ptr;
    int64_t *piece_base = (int64_t *)ws.piece_base.ptr;
    int32_t *perm = (int32_t *)ws.perm.ptr;
    const bool smem = k <= kSmemKMax;
    if (smem) {
        hist_smem_kernel<<<(unsigned)p.n_chunks, 256, sizeof(int) * k, s>>>(labels, p.n, k, p.chunk_rows, H, st);
        KMB_LAUNCHED();
    } else {
        zero_i32_kernel<<<1184, 256, 0, s>>>(H, p.n_chunks * p.k, st);
        KMB_LAUNCHED();
        hist_global_kernel<<<(unsigned)p.n_chunks, 256, 0, s>>>(labels, p.n, k, p.chunk_rows, H, st);
        KMB_LAUNCHED();
    }
    const dim3 g2((unsigned)n_groups, (unsigned)((k + 255) / 256));
    scan_group_sum_kernel<<<g2, 256, 0, s>>>(H, p.n_chunks, k, Gs, st);
    KMB_LAUNCHED();
    scan_groups_kernel<<<(unsigned)((k + 255) / 256), 256, 0, s>>>(Gs, n_groups, k, counts, st);
    KMB_LAUNCHED();
    offsets_kernel<<<1, 1024, 0, s>>>(counts, k, p.piece_rows, offsets, piece_base, st);
    KMB_LAUNCHED();
    scan_chunks_kernel<<<g2, 256, 0, s>>>(H, p.n_chunks, k, Gs, offsets, st);
    KMB_LAUNCHED();
    if (smem) {
        scatter_kernel<true><<<(unsigned)p.n_chunks, 32, sizeof(int) * k, s>>>(labels, p.n, k, p.chunk_rows, H, perm, st);
        KMB_LAUNCHED();
    } else {
        scatter_kernel<false><<<(unsigned)p.n_chunks, 32, 0, s>>>(labels, p.n, k, p.chunk_rows, H, perm, st);
        KMB_LAUNCHED();
    }
    if (sort_only) return;
    double *records = (double *)ws.records.ptr;
    if (csr) {
        const unsigned grid = (unsigned)((p.max_pieces + 3) / 4);
        if (fsize == sizeof(float))
            csr_segsum_kernel<float><<<grid, 128, 0, s>>>((const float *)csr->vals, csr->cols, csr->rowptr, (int)p.d,
                                                          k, perm, offsets, piece_base, p.piece_rows, p.max_pieces,
                                                          records, st);
        else
            csr_segsum_kernel<double><<<grid, 128, 0, s>>>((const double *)csr->vals, csr->cols, csr->rowptr,
                                                           (int)p.d, k, perm, offsets, piece_base, p.piece_rows,
                                                           p.max_pieces, records, st);
        KMB_LAUNCHED();
    } else if (fsize == sizeof(float)) {
        segsum_kernel<float><<<(unsigned)p.max_pieces, 128, 0, s>>>((const float *)Xv, (int)p.d, k, perm, offsets,
            piece_base, p.piece_rows, records, st);
        KMB_LAUNCHED();
    } else {
        segsum_kernel<double><<<(unsigned)p.max_pieces, 128, 0, s>>>((const double *)Xv, (int)p.d, k, perm, offsets,
            piece_base, p.piece_rows, records, st);
        KMB_LAUNCHED();
    }
}

template <typename F>
static void reseed_and_commit(const F *X, const UpdatePlan &p, const int32_t *labels, const F *d2, F *exact_d2,
                              F *C_old, F *C_new, Workspace &ws, LoopState *st, bool commit, cudaStream_t s,
                              const CsrRows *csr = nullptr) {
    const int k = (int)p.k, d = (int)p.d;
    double *shift_part = (double *)ws.shift_part.ptr;
    int32_t *empty_ids = (int32_t *)ws.empty_ids.ptr;
    // Reseeding: every kernel below returns at once unless some cluster is empty.
    if (exact_d2 && !csr) {
        refresh_d2_kernel<F><<<(unsigned)std::min<int64_t>((p.n * 32 + 255) / 256, 148 * 16), 256, 0, s>>>(
            X, p.n, d, C_old, labels, exact_d2, st);
        KMB_LAUNCHED();
        d2 = exact_d2;
    }
    SelState *ss = (SelState *)ws.sel_state.ptr;
    unsigned int *hist = (unsigned int *)ws.sel_hist.ptr;
    Cand *cand = (Cand *)ws.cand.ptr;
    sel_init_kernel<<<1, 256, 0, s>>>(ss, hist, st);
    KMB_LAUNCHED();
    for (int shift = KeyOf<F>::BITS - 8; shift >= 0; shift -= 8) {
        sel_hist_kernel<F><<<592, 256, 0, s>>>(d2, p.n, shift, ss, hist, st);
        KMB_LAUNCHED();
        sel_pick_kernel<<<1, 256, 0, s>>>(ss, hist, shift, st);
        KMB_LAUNCHED();
    }
    sel_collect_kernel<F><<<1, 1024, 0, s>>>(d2, p.n, ss, cand, k, st);
    KMB_LAUNCHED();
    sel_sort_kernel<<<1, 1024, 0, s>>>(cand, st);
    KMB_LAUNCHED();
    if (csr)
        csr_reseed_apply_kernel<F><<<std::min(k, 1024), 128, 0, s>>>((const F *)csr->vals, csr->cols, csr->rowptr, d,
                                                                     cand, empty_ids, C_old, C_new, shift_part, st);
    else
        reseed_apply_kernel<F><<<std::min(k, 1024), 128, 0, s>>>(X, d, cand, empty_ids, C_old, C_new, shift_part, st);
    KMB_LAUNCHED();
    shift_total_kernel<<<1, 1024, 0, s>>>(shift_part, k, st);
    KMB_LAUNCHED();
    if (commit) {
        commit_copy_kernel<F><<<std::max<int64_t>(1, std::min<int64_t>(1184, (p.k * p.d + 255) / 256)), 256, 0, s>>>(
            C_new, C_old, p.k * p.d, st);
        KMB_LAUNCHED();
        decide_kernel<<<1, 1, 0, s>>>(st);
        KMB_LAUNCHED();
    }
}

template <typename F>
void launch_update(const F *X, const UpdatePlan &p, const int32_t *labels, const F *d2, F *C_old, F *C_new,
                   Workspace &ws, LoopState *st, bool commit, cudaStream_t s, const CsrRows *csr, F *exact_d2) {
    const int k = (int)p.k, d = (int)p.d;
    sort_and_sum_pieces(X, sizeof(F), p, labels, ws, st, s, csr);
    double *shift_part = (double *)ws.shift_part.ptr;
    int32_t *empty_flag = (int32_t *)ws.empty_flag.ptr;
    int32_t *empty_ids = (int32_t *)ws.empty_ids.ptr;
    const int tiles = (d + kFinalizeCols - 1) / kFinalizeCols;
    finalize_kernel<F><<<dim3((unsigned)k, (unsigned)tiles), kFinalizeCols, 0, s>>>(
        (const double *)ws.records.ptr, (const int64_t *)ws.counts.ptr, (const int64_t *)ws.piece_base.ptr, C_old,
        C_new, d, (double *)ws.shift_tiles.ptr, empty_flag, st);
    KMB_LAUNCHED();
    shift_tiles_kernel<<<(unsigned)std::min(148, (k + 255) / 256), 256, 0, s>>>((const double *)ws.shift_tiles.ptr, k,
                                                                              tiles, shift_part, st);
    KMB_LAUNCHED();
    empties_kernel<<<1, 1024, 0, s>>>(empty_flag, k, empty_ids, shift_part, st);
    KMB_LAUNCHED();
    reseed_and_commit<F>(X, p, labels, d2, exact_d2, C_old, C_new, ws, st, commit, s, csr);
}

bool ensure_exact_buffers(Workspace &ws, int64_t n, int64_t k, int64_t d, bool piece_records) {
    bool ok = true;
    ok &= ws.ensure(ws.ex_acc, sizeof(long long) * 3 * k * d);
    if (piece_records) ok &= ws.ensure(ws.ex_records, sizeof(long long) * 3 * (n / kPieceRows + k + 1) * d);
    ok &= ws.ensure(ws.ex_cnt, sizeof(long long) * k);
    ok &= ws.ensure(ws.ex_prev, sizeof(int32_t) * std::max<int64_t>(1, n));
    ok &= ws.ensure(ws.ex_colexp, sizeof(int) * d);
    return ok;
}

void launch_column_max_bits(const float *X, int64_t n, int64_t d, unsigned *bits, cudaStream_t s) {
    cudaMemsetAsync(bits, 0, sizeof(unsigned) * d, s);
    const int64_t total = n * d;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 8));
    if (d <= 1024)
        colmax_rows_kernel<<<148 * 8, 256, 0, s>>>(X, n, (int)d, bits, nullptr);
    else if (d <= 8192)
        colmax_kernel<<<blocks, 256, sizeof(unsigned) * d, s>>>(X, n, (int)d, bits, nullptr);
    else
        colmax_global_kernel<<<blocks, 256, 0, s>>>(X, n, (int)d, bits, nullptr);
    KMB_LAUNCHED();
}

void prepare_exact_update(const float *X, int64_t n, int64_t d, Workspace &ws, LoopState *st, cudaStream_t s) {
    int *colexp = (int *)ws.ex_colexp.ptr;
    cudaMemsetAsync(colexp, 0, sizeof(int) * d, s);
    const int64_t total = n * d;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 8));
    if (d <= 1024) {
        colmax_rows_kernel<<<148 * 8, 256, 0, s>>>(X, n, (int)d, (unsigned *)colexp, st);
    } else if (d <= 8192) {
        colmax_kernel<<<blocks, 256, sizeof(unsigned) * d, s>>>(X, n, (int)d, (unsigned *)colexp, st);
    } else {
        colmax_global_kernel<<<blocks, 256, 0, s>>>(X, n, (int)d, (unsigned *)colexp, st);
    }
    KMB_LAUNCHED();
    colexp_kernel<<<(unsigned)((d + 255) / 256), 256, 0, s>>>(colexp, (int)d, st);
    KMB_LAUNCHED();
}

template <typename F>
bool launch_top_rows(const F *d2, int64_t n, int m, Workspace &ws, LoopState *st, long long *rows_out, cudaStream_t s) {
    if (m <= 0 || m > n) return m == 0;
    int64_t pm = 1;
    while (pm < m) pm <<= 1;
    if (!ws.ensure(ws.sel_hist, sizeof(unsigned int) * 256) || !ws.ensure(ws.sel_state, sizeof(SelState)) ||
        !ws.ensure(ws.cand, sizeof(Cand) * pm))
        return false;
    SelState *ss = (SelState *)ws.sel_state.ptr;
    unsigned int *hist = (unsigned int *)ws.sel_hist.ptr;
    Cand *cand = (Cand *)ws.cand.ptr;
    select_state_kernel<<<1, 1, 0, s>>>(st, m);
    KMB_LAUNCHED();
    sel_init_kernel<<<1, 256, 0, s>>>(ss, hist, st);
    KMB_LAUNCHED();
    for (int shift = KeyOf<F>::BITS - 8; shift >= 0; shift -= 8) {
        sel_hist_kernel<F><<<592, 256, 0, s>>>(d2, n, shift, ss, hist, st);
        KMB_LAUNCHED();
        sel_pick_kernel<<<1, 256, 0, s>>>(ss, hist, shift, st);
        KMB_LAUNCHED();
    }
    sel_collect_kernel<F><<<1, 1024, 0, s>>>(d2, n, ss, cand, m, st);
    KMB_LAUNCHED();
    sel_sort_kernel<<<1, 1024, 0, s>>>(cand, st);
    KMB_LAUNCHED();
    cand_rows_kernel<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(cand, m, rows_out);
    KMB_LAUNCHED();
    return true;
}
template bool launch_top_rows<float>(const float *, int64_t, int, Workspace &, LoopState *, long long *, cudaStream_t);
template bool launch_top_rows<double>(const double *, int64_t, int, Workspace &, LoopState *, long long *, cudaStream_t);

void launch_update_exact(const float *X, const UpdatePlan &p, int32_t *labels, const float *d2, float *C_old,
                         float *C_new, Workspace &ws, LoopState *st, bool commit, cudaStream_t s, float *exact_d2) {
    const int k = (int)p.k, d = (int)p.d;
    int32_t *prev = (int32_t *)ws.ex_prev.ptr;
    const int *colexp = (const int *)ws.ex_colexp.ptr;
    long long *acc = (long long *)ws.ex_acc.ptr;
    long long *cnt = (long long *)ws.ex_cnt.ptr;
    long long *records = (long long *)ws.ex_records.ptr;
    const unsigned rb = (unsigned)std::max<int64_t>(1, std::min<int64_t>((p.n + 255) / 256, 148 * 8));
    count_moved_kernel<<<rb, 256, 0, s>>>(labels, prev, p.n, st);
    KMB_LAUNCHED();
    choose_mode_kernel<<<1, 1, 0, s>>>(p.n, st);
    KMB_LAUNCHED();
    // full mode: counting sort + integer piece sums (every kernel returns at once otherwise)
    sort_and_sum_pieces(nullptr, 0, p, labels, ws, st, s, nullptr, /*sort_only=*/true);
    segsum_fixed_kernel<<<(unsigned)p.max_pieces, 128, 0, s>>>(X, d, k, (const int32_t *)ws.perm.ptr,
                                                                (const int64_t *)ws.offsets.ptr,
                                                                (const int64_t *)ws.piece_base.ptr, p.piece_rows,
                                                                p.max_pieces, colexp, records, st);
    KMB_LAUNCHED();
    // incremental mode: the moved rows
    apply_moves_kernel<<<rb, 256, 0, s>>>(X, p.n, d, k, labels, prev, colexp, (unsigned long long *)acc,
                                          (unsigned long long *)cnt, st);
    KMB_LAUNCHED();
    double *shift_part = (double *)ws.shift_part.ptr;
    int32_t *empty_flag = (int32_t *)ws.empty_flag.ptr;
    int32_t *empty_ids = (int32_t *)ws.empty_ids.ptr;
    const int tiles = (d + kFinalizeCols - 1) / kFinalizeCols;
    finalize_exact_kernel<<<dim3((unsigned)k, (unsigned)tiles), kFinalizeCols, 0, s>>>(
        records, p.max_pieces, (const int64_t *)ws.counts.ptr, (const int64_t *)ws.piece_base.ptr, colexp, k, acc,
        cnt, C_old, C_new, d, (double *)ws.shift_tiles.ptr, empty_flag, st);
    KMB_LAUNCHED();
    copy_prev_kernel<<<rb, 256, 0, s>>>(labels, prev, p.n, st);
    KMB_LAUNCHED();
    exact_valid_kernel<<<1, 1, 0, s>>>(st);
    KMB_LAUNCHED();
    shift_tiles_kernel<<<(unsigned)std::min(148, (k + 255) / 256), 256, 0, s>>>((const double *)ws.shift_tiles.ptr, k,
                                                                              tiles, shift_part, st);
    KMB_LAUNCHED();
    empties_kernel<<<1, 1024, 0, s>>>(empty_flag, k, empty_ids, shift_part, st);
    KMB_LAUNCHED();
    reseed_and_commit<float>(X, p, labels, exact_d2 ? exact_d2 : d2, exact_d2, C_old, C_new, ws, st, commit, s);
}

void prepare_exact_update_csr(const CsrRows &X, Workspace &ws, LoopState *st, cudaStream_t s) {
    int *colexp = (int *)ws.ex_colexp.ptr;
    const int d = (int)X.d;
    cudaMemsetAsync(colexp, 0, sizeof(int) * d, s);
    const bool in_smem = (size_t)d * sizeof(unsigned) <= (size_t)96 * 1024;
    const size_t smem = in_smem ? sizeof(unsigned) * d : 0;
    if (in_smem) cudaFuncSetAttribute(csr_colmax_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const unsigned blocks =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>((X.nnz + 255) / 256, in_smem ? 148 * 2 : 148 * 8));
    csr_colmax_kernel<<<blocks, 256, smem, s>>>((const float *)X.vals, X.cols, X.nnz, d, in_smem, (unsigned *)colexp);
    KMB_LAUNCHED();
    colexp_kernel<<<(unsigned)((d + 255) / 256), 256, 0, s>>>(colexp, d, st);
    KMB_LAUNCHED();
}

void launch_update_exact_csr(const CsrRows &X, const UpdatePlan &p, int32_t *labels, const float *d2, float *C_old,
                             float *C_new, Workspace &ws, LoopState *st, bool commit, cudaStream_t s) {
    const int k = (int)p.k, d = (int)p.d;
    int32_t *prev = (int32_t *)ws.ex_prev.ptr;
    const int *colexp = (const int *)ws.ex_colexp.ptr;
    long long *acc = (long long *)ws.ex_acc.ptr;
    long long *cnt = (long long *)ws.ex_cnt.ptr;
    const unsigned rb = (unsigned)std::max<int64_t>(1, std::min<int64_t>((p.n + 255) / 256, 148 * 8));
    count_moved_kernel<<<rb, 256, 0, s>>>(labels, prev, p.n, st);
    KMB_LAUNCHED();
    choose_mode_kernel<<<1, 1, 0, s>>>(p.n, st);
    KMB_LAUNCHED();
    // full mode: clear, then every row's entries (each kernel returns at once otherwise)
    csr_exact_clear_kernel<<<148 * 8, 256, 0, s>>>(acc, 3 * (int64_t)k * d, cnt, k, st);
    KMB_LAUNCHED();
    const size_t cs = k <= kCsrCountSmem ? sizeof(unsigned) * k : 0;
    csr_sums_fixed_kernel<<<148 * 8, 256, cs, s>>>((const float *)X.vals, X.cols, X.rowptr, p.n, d, k, labels, colexp,
                                                   (unsigned long long *)acc, (unsigned long long *)cnt, st);
    KMB_LAUNCHED();
    // incremental mode: the moved rows
    csr_apply_moves_kernel<<<rb, 256, 0, s>>>((const float *)X.vals, X.cols, X.rowptr, p.n, d, k, labels, prev, colexp,
                                              (unsigned long long *)acc, (unsigned long long *)cnt, st);
    KMB_LAUNCHED();
    int32_t *empty_flag = (int32_t *)ws.empty_flag.ptr;
    int32_t *empty_ids = (int32_t *)ws.empty_ids.ptr;
    double *shift_part = (double *)ws.shift_part.ptr;
    const int tiles = (d + kFinalizeCols - 1) / kFinalizeCols;
    finalize_exact_kernel<<<dim3((unsigned)k, (unsigned)tiles), kFinalizeCols, 0, s>>>(
        nullptr, 0, nullptr, nullptr, colexp, k, acc, cnt, C_old, C_new, d, (double *)ws.shift_tiles.ptr, empty_flag,
        st, /*from_acc=*/true);
    KMB_LAUNCHED();
    copy_prev_kernel<<<rb, 256, 0, s>>>(labels, prev, p.n, st);
    KMB_LAUNCHED();
    exact_valid_kernel<<<1, 1, 0, s>>>(st);
    KMB_LAUNCHED();
    shift_tiles_kernel<<<(unsigned)std::min(148, (k + 255) / 256), 256, 0, s>>>((const double *)ws.shift_tiles.ptr, k,
                                                                              tiles, shift_part, st);
    KMB_LAUNCHED();
    empties_kernel<<<1, 1024, 0, s>>>(empty_flag, k, empty_ids, shift_part, st);
    KMB_LAUNCHED();
    reseed_and_commit<float>(nullptr, p, labels, d2, nullptr, C_old, C_new, ws, st, commit, s, &X);
}

template <typename F>
void launch_partial_sums(const F *X, const UpdatePlan &p, const int32_t *labels, double *sums, int64_t *counts,
                         Workspace &ws, cudaStream_t s) {
    sort_and_sum_pieces(X, sizeof(F), p, labels, ws, nullptr, s);
    sums_kernel<<<dim3((unsigned)p.k, (unsigned)((p.d + kFinalizeCols - 1) / kFinalizeCols)), kFinalizeCols, 0, s>>>(
        (const double *)ws.records.ptr, (const int64_t *)ws.counts.ptr,
                                             (const int64_t *)ws.piece_base.ptr, (int)p.d, sums, counts);
    KMB_LAUNCHED();
}

template <typename F>
void launch_objective(const F *X, int64_t n, int64_t d, const F *C, const int32_t *labels, double *partials,
                      double *out, cudaStream_t s) {
    objective_kernel<F><<<kObjectivePartials, 256, 0, s>>>(X, n, (int)d, C, labels, partials);
    KMB_LAUNCHED();
    sum_partials_kernel<<<1, 32, 0, s>>>(partials, kObjectivePartials, out);
    KMB_LAUNCHED();
}

template <typename F>
void launch_finalize_from_sums(const double *sums, const int64_t *counts, const F *C_old, F *C_new, int64_t k,
                               int64_t d, Workspace &ws, double *shift_out, int32_t *empty_ids, long long *n_empty,
                               cudaStream_t s) {
    double *shift_part = (double *)ws.shift_part.ptr;
    int32_t *empty_flag = (int32_t *)ws.empty_flag.ptr;
    finalize_from_sums_kernel<F><<<(unsigned)k, 128, 0, s>>>(sums, counts, C_old, C_new, (int)d, shift_part,
                                                             empty_flag);
    KMB_LAUNCHED();
    sum_doubles_kernel<<<1, 1024, 0, s>>>(shift_part, (int)k, shift_out);
    KMB_LAUNCHED();
    list_empties_kernel<<<1, 1024, 0, s>>>(empty_flag, (int)k, empty_ids, n_empty);
    KMB_LAUNCHED();
}

template <typename F>
void launch_sum_values(const F *v, int64_t n, double *partials, double *out, cudaStream_t s) {
    sum_values_kernel<F><<<kObjectivePartials, 256, 0, s>>>(v, n, partials);
    KMB_LAUNCHED();
    sum_partials_kernel<<<1, 32, 0, s>>>(partials, kObjectivePartials, out);
    KMB_LAUNCHED();
}

template void launch_finalize_from_sums<float>(const double *, const int64_t *, const float *, float *, int64_t,
                                               int64_t, Workspace &, double *, int32_t *, long long *, cudaStream_t);
template void launch_finalize_from_sums<double>(const double *, const int64_t *, const double *, double *, int64_t,
                                                int64_t, Workspace &, double *, int32_t *, long long *,
                                                cudaStream_t);
template void launch_sum_values<float>(const float *, int64_t, double *, double *, cudaStream_t);
template void launch_sum_values<double>(const double *, int64_t, double *, double *, cudaStream_t);

#define KMB_INST(F)                                                                                                 \
    template void launch_update<F>(const F *, const UpdatePlan &, const int32_t *, const F *, F *, F *, Workspace &, \
                                   LoopState *, bool, cudaStream_t, const CsrRows *, F *);                         \
    template void launch_partial_sums<F>(const F *, const UpdatePlan &, const int32_t *, double *, int64_t *,       \
                                         Workspace &, cudaStream_t);                                               \
    template void launch_objective<F>(const F *, int64_t, int64_t, const F *, const int32_t *, double *, double *, \
                                      cudaStream_t);
KMB_INST(float)
KMB_INST(double)
#undef KMB_INST

}  // namespace kmb
