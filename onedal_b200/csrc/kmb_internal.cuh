// Internal declarations shared by the k-means Lloyd kernels (sm_100a).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/onedal_b200_kmeans.h"

namespace kmb {

// Number of kernels this host thread has launched through the library (read by
// kmb_context_kernel_time(ctx, 3, ...) for the launch count of a timed region).
int64_t &launch_count();
#define KMB_LAUNCHED() (++::kmb::launch_count())

// Device-resident loop state. Every per-iteration kernel reads `done` first and
// returns at once when it is set, so the whole Lloyd loop is enqueued without a
// host round trip per iteration (the reference's GPU loop synchronises on the
// objective every iteration, cpp/oneapi/dal/algo/kmeans/backend/gpu/cluster_updater.hpp:135-136).
struct LoopState {
    int done;             // converged (shift <= eps) or failed
    int error;            // kmb_status of a device-detected failure
    int iterations;       // completed Lloyd updates
    int n_empty;          // empty clusters in the current update
    int n_recheck;        // rows queued for the FP64 recheck
    int n_changed;        // rows whose label the recheck changed
    long long empty_events;
    long long rechecked_total;
    double shift;         // sum ||c_old - c_new||^2 of the current update
    double eps;
    int n_full;           // queued rows that needed the full k rescan (this pass)
    int pad_;
    long long full_total;
    // Exact update (FP32 rows): the integer cluster sums are a function of the
    // labels, so a pass that moved few rows updates them by those rows only.
    int upd_mode;         // 0: recompute from all rows (counting sort), 1: apply the moved rows
    int upd_valid;        // sums, counts and previous labels describe the previous pass
    long long n_moved;    // rows whose label changed in this pass
};

// Recheck queue entry written by the assignment kernels for near-tie rows.
struct RecheckEntry {
    int row;
    int c1;    // approximate best cluster
    int c2;    // approximate second-best cluster
    int full;  // 1: more than two clusters lie inside the error band -> scan all k
};

// Device state of the k-means++ initialisation (kmb_init.cu).
struct PPState {
    int stopped;          // 1: out of uniforms (stop_round is to be redone); 2: no row can be drawn;
                          // 3: the overall-sum fold timed out waiting for a block sum
    int pool_used;        // resample draws consumed from the current pool
    long long stop_round;
    long long rows_chosen;
    double overall;       // the current round's overall distance sum (computed in F)
    long long last_row;   // the row chosen by the last selection
    double cnorm;         // CSR rows: ||c||^2 of the last center (computed in F)
};

template <typename F>
void launch_pp_fill(F *md, int64_t n, cudaStream_t s);
template <typename F>
void launch_pp_first(const F *X, int64_t d, int64_t row, F *C, cudaStream_t s);
template <typename F>
void launch_pp_rounds(const F *X, int64_t n, int64_t d, int64_t k, int64_t c_begin, bool update_first, F *md, F *acc,
                      unsigned *flags, const F *probs, const F *pool, int pool_n, F *C, PPState *st, cudaStream_t s);
// The same for CSR rows (plusPlusCSR): center c = row `row` expanded to dense,
// with ||c||^2 in st->cnorm; launch_pp_first_csr places center 0.
struct CsrRows;
template <typename F>
void launch_pp_first_csr(const CsrRows &X, int64_t row, F *C, PPState *st, cudaStream_t s);
template <typename F>
void launch_pp_rounds_csr(const CsrRows &X, int64_t k, int64_t c_begin, bool update_first, F *md, F *acc,
                          unsigned *flags, const F *probs, const F *pool, int pool_n, F *C, PPState *st, cudaStream_t s);

// Queues a near-tie row for the FP64 recheck. Two-candidate entries fill the
// queue from the front (count st->n_recheck), full-rescan entries from the back
// (count st->n_full); the capacity is the row count, and a row is queued once.
__device__ __forceinline__ void enqueue_recheck(RecheckEntry *queue, int64_t cap, LoopState *st, int row, int c1,
                                                int c2, bool full) {
    RecheckEntry q;
    q.row = row;
    q.c1 = c1;
    q.c2 = c2;
    q.full = full ? 1 : 0;
    if (full)
        queue[cap - 1 - atomicAdd(&st->n_full, 1)] = q;
    else
        queue[atomicAdd(&st->n_recheck, 1)] = q;
}

// Per-call sizing of the update (counting sort + segmented FP64 sums).
struct UpdatePlan {
    int64_t n, k, d;
    int64_t chunk_rows;   // rows per stable-scatter chunk
    int64_t n_chunks;
    int64_t piece_rows;   // rows per FP64 partial-sum piece
    int64_t max_pieces;   // n / piece_rows + k (upper bound)
};

// Device scratch of one context. Buffers grow on demand and are reused across
// calls; `bytes_*` track capacities.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

struct Workspace {
    int device = 0;
    // Buffers are stream-ordered allocations on the context's stream: growing
    // one never synchronises the device (a plain cudaFree would stall every
    // other stream's host thread, e.g. a serving loop's lanes, until the device
    // drains).
    cudaStream_t stream = nullptr;
    DevBuf X, C0, Cout, labels, d2, xnorm, Ccur, Cnew, Ct, h, queue;
    DevBuf H, Gs, counts, offsets, piece_base, perm, records, shift_part, shift_tiles, empty_flag, empty_ids;
    DevBuf sel_hist, sel_state, cand, obj_part, scalars, state;
    DevBuf Xhi, Xlo, Chi, Clo, tcx, rowb, pp_acc, pp_rand, pp_state, pp_flags;
    DevBuf csr_vals, csr_cols64, csr_rowptr64, csr_cols, csr_rowptr, csr_bad, csr_cnorm;
    DevBuf ex_acc, ex_cnt, ex_prev, ex_colexp, ex_records;  // exact update: limb sums, counts, previous
    DevBuf sp_sums, sp_counts, sp_sq, sp_rowsq, sp_Ca, sp_Cb, sp_ids, sp_rows, sp_state, sp_gather;  // kmb_train_spmd
    DevBuf sp_acc, sp_colexp, sp_shift;                                                                // (exact sums)
                                                             // labels, scales, per-piece limb sums
    // Grows `b` to at least `bytes`; returns false on allocation failure.
    bool ensure(DevBuf &b, size_t bytes);
    void release();
};

// Scalars kept in device memory (one DevBuf "scalars").
struct DevScalars {
    double cnorm_max;
    double xnorm_max;
    double objective;
    double pad;
    double cnorm_max_prev;  // max ||c|| of the previous tensor-core pass's centroids
};

// ---- assignment (plain FMA form) ------------------------------------------
// Prepares per-iteration centroid data: transposed copy Ct (d x kpad), half
// squared norms h (kpad, +inf padding) and max ||c|| for the error bound.
template <typename F>
void launch_prep_centroids(const F *C, int64_t k, int64_t d, int64_t kpad, F *Ct, F *h, double *cnorm_max,
                           const LoopState *st, cudaStream_t s);

// Row squared norms (once per call; X is constant across iterations).
template <typename F>
void launch_row_norms(const F *X, int64_t n, int64_t d, F *xnorm, cudaStream_t s);

// Fused distance + argmin over all clusters for every row.
// Writes labels, d2 (squared distance to the winner, 2*best + ||x||^2, in F)
// and, when `queue` is non-null, appends near-tie rows to the recheck queue.
template <typename F>
void launch_assign_plain(const F *X, int64_t n, int64_t d, const F *Ct, const F *h, int64_t k, int64_t kpad,
                         const F *xnorm, const double *cnorm_max, int32_t *labels, F *d2, RecheckEntry *queue,
                         LoopState *st, cudaStream_t s);

// FP64 recheck of queued rows (exact expanded score in double, lowest index on ties).
template <typename F>
void launch_recheck(const F *X, int64_t n, int64_t d, const F *C, int64_t k, const RecheckEntry *queue,
                    int32_t *labels, F *d2, const F *xnorm, LoopState *st, int num_sms, cudaStream_t s);

// ---- assignment (tensor-core BF16x3 form, float32 data) ----------------------
int64_t tc_dpad(int64_t d);   // d rounded up to the 64-wide K panel
// Stream-ordered allocation from the library's memory pool of device `dev` (freed
// memory is kept for reuse instead of going back to the driver at synchronisations).
cudaError_t pool_alloc(void **p, size_t bytes, int dev, cudaStream_t s);
int tc_tile_n(int64_t k);      // cluster tile of the tensor-core kernel: 128 or 256
int64_t tc_kpad(int64_t k);   // k rounded up to a multiple of tc_tile_n(k)
bool tc_supported(int64_t d); // dpad <= 256
// x -> BF16 hi/lo panels [rows][dpad] (lo may be null: hi only) and ||x||^2 (the
// same value launch_row_norms gives).
void launch_split_rows(const float *X, int64_t rows, int64_t d, void *hi, void *lo, float *xnorm, int num_sms,
                       cudaStream_t s);
// C -> Chi/Clo [kpad][dpad], -h = -0.5||c||^2 (kpad, -inf padding), max ||c||.
// Also moves the previous max ||c|| into *cnorm_max_prev before recomputing it.
void launch_prep_centroids_tc(const float *C, int64_t k, int64_t d, void *Chi, void *Clo, float *h,
                              double *cnorm_max, double *cnorm_max_prev, const LoopState *st, cudaStream_t s);
// xchg: tc_xchg_bytes(num_sms) bytes of device scratch (epilogue hand-off).
// prior: labels/d2 hold the previous pass's results under the centroids that
// the update in between moved by sqrt(shift_part[j]); they seed a lower bound
// on each row's best score that lets the epilogue skip hopeless clusters.
// products: 3 = split BF16 (xh.ch + xh.cl + xl.ch), 1 = one BF16 product (xh.ch;
// Xlo / Clo unused). The recheck band follows the form's error bound.
int launch_assign_tc(const void *Xhi, const void *Xlo, int64_t n, int64_t d, const void *Chi, const void *Clo,
                     const float *h, int64_t k, const float *xnorm, const double *cnorm_max, int32_t *labels,
                     float *d2, RecheckEntry *queue, LoopState *st, int num_sms, void *xchg, bool prior,
                     const double *shift_part, const double *cnorm_max_prev, void *rowb, int products,
                     cudaStream_t s);
size_t tc_xchg_bytes();

// Encodes a 2-D tiled tensor map (inner x outer elements, rows row_bytes apart,
// box_inner x box_outer boxes) through the runtime's driver entry point, so the
// library does not link libcuda directly. False when the driver rejects it.
bool encode_tensor_map_2d(CUtensorMap *m, CUtensorMapDataType type, const void *base, uint64_t inner, uint64_t outer,
                          uint64_t row_bytes, uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle swizzle);

// ---- CSR rows (kmeans::method::lloyd_csr) ------------------------------------
// Zero-based, device-resident CSR rows: values (nnz, F), column indices (int32,
// strictly increasing within a row, in [0, d)) and row offsets (n + 1, int64,
// rowptr[0] == 0).
struct CsrRows {
    const void *vals;
    const int32_t *cols;
    const int64_t *rowptr;
    int64_t n, d, nnz;
};

// Converts caller indices (int64, `base` 0 or 1) into CsrRows' form and checks
// them; *bad (device int) becomes nonzero when an offset is out of order or a
// column index is out of range or not strictly increasing within its row.
void launch_csr_prepare(const int64_t *cols_in, const int64_t *rowptr_in, int64_t n, int64_t d, int64_t nnz, int base,
                        int32_t *cols_out, int64_t *rowptr_out, int *bad, cudaStream_t s);

// Labels and squared distances (2*best + sum of the row's v^2, in F) of CSR rows
// against centroids prepared by launch_prep_centroids (Ct d x kpad, h kpad).
template <typename F>
void launch_csr_assign(const CsrRows &X, const F *Ct, const F *h, int64_t k, int64_t kpad, int32_t *labels, F *d2,
                       const LoopState *st, cudaStream_t s);

// Exact objective of CSR rows: per row sum over stored entries of (x^2 - 2xc) +
// ||c||^2, clipped at zero, in FP64, deterministic. cnorm2: k doubles of scratch.
template <typename F>
void launch_csr_objective(const CsrRows &X, const F *C, int64_t k, const int32_t *labels, double *cnorm2,
                          double *partials, double *out, cudaStream_t s);

// ---- update ----------------------------------------------------------------
UpdatePlan make_update_plan(int64_t n, int64_t k, int64_t d);
// Sizes the update buffers of `ws` for plan `p` (false on allocation failure).
// fp64_records false: no FP64 piece records (an update that never sums pieces in FP64).
bool ensure_update_buffers(Workspace &ws, const UpdatePlan &p, size_t fsize, bool fp64_records = true);

// One Lloyd update: counting-sort the rows by label (stable, so each cluster's
// rows are summed in row order), FP64 sums per fixed piece of rows, centroid =
// sum / count rounded to F, empty clusters reseeded with the farthest rows,
// centroid shift, convergence flag. C_old is overwritten by the new centroids
// when `commit` (the loop path); otherwise they are left in C_new.
// With `csr`, the rows are CSR (X is unused): piece sums scatter the stored
// entries and a reseeded cluster takes its candidate row expanded to dense.
// With exact_d2 (the d2 buffer itself), an iteration with empty clusters first
// recomputes every row's squared distance in FP64 so the candidates follow the
// exact distances (the tensor-core forms' d2 is exact only for rechecked rows).
template <typename F>
void launch_update(const F *X, const UpdatePlan &p, const int32_t *labels, const F *d2, F *C_old, F *C_new,
                   Workspace &ws, LoopState *st, bool commit, cudaStream_t s, const CsrRows *csr = nullptr,
                   F *exact_d2 = nullptr);

// ---- exact fixed-point sums (shared by the Lloyd update and the batched form) ----
// A value x of column t is the integer v = round(x * 2^E_t), |v| < 2^94, E_t =
// 94 - (exponent of the column's largest |x|); v is handled as three 32-bit
// limbs, v = l2 * 2^64 + l1 * 2^32 + l0 (l0, l1 in [0, 2^32), l2 signed), so limb
// sums in int64 add and subtract rows exactly in any order.
constexpr int kExactMaxBits = 94;  // |round(x * 2^E_t)| < 2^94

struct Limbs {
    long long l0, l1, l2;
};

// round(x * 2^e) (round half to even) as three signed 32-bit limbs,
// v = l2 * 2^64 + l1 * 2^32 + l0 with |l_i| < 2^32 (each limb carries the sign of
// x), computed in 64-bit integer arithmetic. Requires |x| * 2^e < 2^94. Limb sums
// of fewer than 2^31 values stay below 2^63, and any order of additions and
// subtractions gives the same integer l2 * 2^64 + l1 * 2^32 + l0.
__device__ __forceinline__ Limbs fixed_of(float x, int e) {
    // x = mant * 2^((be ? be : 1) - 150) exactly, so x * 2^e = mant * 2^sh with the
    // exponent added as an integer (no float scaling; the same integer as scaling
    // first whenever |x| * 2^e < 2^94). Non-finite x keeps its raw pattern (sh 105).
    const unsigned bits = __float_as_uint(x);
    const int be = (int)((bits >> 23) & 0xffu);
    unsigned long long mant = bits & 0x7fffffu;
    if (be) mant |= 0x800000u;
    const int sh = be == 255 ? 105 : (be ? be : 1) - 150 + e;  // mant * 2^sh < 2^94
    long long l0 = 0, l1 = 0, l2 = 0;
    if (sh >= 0) {
        const int q = sh >> 5;
        const unsigned long long w = mant << (sh & 31);  // < 2^55, limbs q and q + 1
        const long long lo = (long long)(w & 0xffffffffull), hi = (long long)(w >> 32);
        if (q == 0) {
            l0 = lo;
            l1 = hi;
        } else if (q == 1) {
            l1 = lo;
            l2 = hi;
        } else {
            l2 = lo;  // sh >= 64: w < 2^31 because |f| < 2^94
        }
    } else if (sh > -26) {
        const int r = -sh;  // round half to even
        const unsigned long long q = mant >> r, rem = mant & ((1ull << r) - 1), half = 1ull << (r - 1);
        l0 = (long long)(q + ((rem > half || (rem == half && (q & 1ull))) ? 1ull : 0ull));
    }
    if (bits >> 31) {
        l0 = -l0;
        l1 = -l1;
        l2 = -l2;
    }
    Limbs L;
    L.l0 = l0;
    L.l1 = l1;
    L.l2 = l2;
    return L;
}

// The nearest double to |m| (round half to even), m < 2^127.
__device__ __forceinline__ double u128_to_double(unsigned __int128 m) {
    const unsigned long long hi = (unsigned long long)(m >> 64), lo = (unsigned long long)m;
    if (hi == 0 && lo < (1ull << 53)) return (double)lo;
    const int top = hi ? 127 - __clzll((long long)hi) : 63 - __clzll((long long)lo);
    const int sh = top - 52;
    unsigned long long q = (unsigned long long)(m >> sh);
    const unsigned __int128 rem = m & (((unsigned __int128)1 << sh) - 1);
    const unsigned __int128 half = (unsigned __int128)1 << (sh - 1);
    if (rem > half || (rem == half && (q & 1ull))) ++q;
    return ldexp((double)q, sh);
}


// The exact update of FP32 rows (the Lloyd loop's update for float data). Every
// value x of column t is taken as the integer round(x * 2^E_t), E_t chosen once
// per call so that the column's largest |x| stays below 2^94 (every float within
// 2^70 of it exact); a cluster's sum is then an exact integer (three 32-bit
// limbs summed in int64), independent of the order in which rows are added, and
// the centroid is that integer rounded to the nearest double, scaled back,
// divided by the count in FP64 and rounded to float. Because the sums are a function of the
// labels alone, a pass that moved at most n/8 rows is applied as those rows'
// moves (subtract from the old cluster, add to the new one, exact) instead of a
// full counting-sort pass over X; the result is bit for bit the same.
// prepare_exact_update: once per call (the scales; the next update recomputes).
void prepare_exact_update(const float *X, int64_t n, int64_t d, Workspace &ws, LoopState *st, cudaStream_t s);
// piece_records: the dense rows' full passes sum per-piece records (the CSR form
// accumulates into the maintained sums instead and needs none).
bool ensure_exact_buffers(Workspace &ws, int64_t n, int64_t k, int64_t d, bool piece_records = true);
// CSR rows with float values: column scales from the stored entries, and the
// exact update (the dense rows' integers, accumulated by atomics).
void prepare_exact_update_csr(const CsrRows &X, Workspace &ws, LoopState *st, cudaStream_t s);
void launch_update_exact_csr(const CsrRows &X, const UpdatePlan &p, int32_t *labels, const float *d2, float *C_old,
                             float *C_new, Workspace &ws, LoopState *st, bool commit, cudaStream_t s);
void launch_update_exact(const float *X, const UpdatePlan &p, int32_t *labels, const float *d2, float *C_old,
                         float *C_new, Workspace &ws, LoopState *st, bool commit, cudaStream_t s, float *exact_d2);

// The m rows with the largest d2, in (d2 descending, row ascending) order, into
// rows_out (device, m int64); m <= n. st is scratch device state (its n_empty is set
// to m). The sharded training's reseed candidates. False when a buffer cannot grow.
template <typename F>
bool launch_top_rows(const F *d2, int64_t n, int m, Workspace &ws, LoopState *st, long long *rows_out, cudaStream_t s);

// Sharded float training with exact sums (kmb_train_spmd): the column maxima of a
// shard as float bits (|x| of non-NaN values; 0 for an all-zero column), the
// exact limb sums of a shard's rows by label (acc: 3 x k x d int64, counts: k int32,
// both cleared first; *bad set to 2 on a label out of range), and the centroids
// from summed limbs (non-empty clusters; C updated in place, shift_part[j] =
// ||c_old - c_new||^2, acc cleared). The formulas are the Lloyd loop's exact update.
void launch_column_max_bits(const float *X, int64_t n, int64_t d, unsigned *bits, cudaStream_t s);
void launch_shard_exact_sums(const float *X, int64_t n, int d, int k, const int32_t *labels, const int *colexp,
                             long long *acc, int *counts, int *bad, cudaStream_t s);
void launch_shard_exact_finalize(long long *acc, const int *counts, const int *colexp, float *C, int k, int d,
                                 double *shift_part, cudaStream_t s);

// Just the sums/counts half of the update (sharded training).
template <typename F>
void launch_partial_sums(const F *X, const UpdatePlan &p, const int32_t *labels, double *sums, int64_t *counts,
                         Workspace &ws, cudaStream_t s);

// Sharded helpers: centroids from all-reduced sums/counts (shift over the
// non-empty clusters, ascending list of empty clusters), and a deterministic
// FP64 sum of n values.
template <typename F>
void launch_finalize_from_sums(const double *sums, const int64_t *counts, const F *C_old, F *C_new, int64_t k,
                               int64_t d, Workspace &ws, double *shift_out, int32_t *empty_ids, long long *n_empty,
                               cudaStream_t s);
template <typename F>
void launch_sum_values(const F *v, int64_t n, double *partials, double *out, cudaStream_t s);

// Blocks of the objective / value-sum kernels, hence the number of FP64
// partials their `partials` scratch holds (launch_objective, launch_sum_values).
constexpr int kObjectivePartials = 148 * 8;

// Exact objective sum ||x - c_label||^2 in FP64, deterministic.
// partials: kObjectivePartials doubles of scratch.
template <typename F>
void launch_objective(const F *X, int64_t n, int64_t d, const F *C, const int32_t *labels, double *partials,
                      double *out, cudaStream_t s);

}  // namespace kmb
