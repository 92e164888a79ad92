// Batched form: thousands of independent k-means problems (uneven n, k, d) run
// their Lloyd iterations together. Every iteration is a fixed sequence of
// grouped launches over all problems, captured once into a CUDA graph and
// replayed; converged problems are skipped on the device through per-problem
// flags, so the host does not synchronise between iterations.
//
// Per iteration (semantics of one pass of cpp/daal/src/algorithms/kmeans/
// kmeans_lloyd_batch_impl.i:117-212 for every problem):
//   prep        C -> transposed Ct, h = 0.5||c||^2 (FP32 from a double sum)
//   assign      one work item = (problem, row tile); FP32 FMA scores
//               h_j - x.c_j over all of the problem's clusters (k <= 256),
//               lowest index on ties; labels + squared distances
//   accumulate  one work item = (problem, row block): the rows' values are
//               converted to 64-bit fixed point with a per-problem scale and
//               summed with integer atomics in shared memory, then in global
//               memory. Integer addition is associative, so the sums are exact
//               on the fixed-point grid and independent of scheduling.
//   finalize    one work item = (problem, cluster): c = F(S / count), shift part
//   decide      one block per problem: shift, empty-cluster reseed with the
//               farthest rows (descending squared distance, ascending row; empty
//               clusters in ascending order), iteration count, stop test.
// The assignment tile (rows per thread) is chosen per (d, k-tile) class by a
// small autotuner that times both candidates on synthetic rows once per context.
#include "kmb_internal.cuh"

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

namespace kmb {
namespace batched {

constexpr int NT = 256;
constexpr int BK = 8;
constexpr int kMaxK = 256;       // clusters per problem handled by one tile
constexpr int kAccRows = 2048;   // rows per accumulate work item

struct Problem {
    const float *X;
    float *C;
    float *Ct;        // dpad x kpad
    float *h;         // kpad (+inf padding)
    int32_t *labels;
    float *d2;
    float *xnorm;
    unsigned long long *acc;  // k*d fixed-point sums (two's complement)
    int *counts;              // k
    double *shift_part;       // k
    long long n;
    int d, dpad, k, kpad;
    double scale;             // fixed-point scale
    int amax_bits;            // max |x| of the problem (float bits, non-negative)
    int done, iters, max_iters, empty_events;
    double eps, shift;
};

// ---- prep --------------------------------------------------------------------
__global__ void prep_kernel(Problem *P, const int2 *items, int n_items) {
    const int it = blockIdx.x;  // one warp per (problem, padded cluster)
    if (it >= n_items) return;
    const int2 w = items[it];
    Problem &p = P[w.x];
    if (p.done) return;
    const int j = w.y;
    double s = 0.0;
    for (int t = threadIdx.x; t < p.dpad; t += 32) {
        const float v = (j < p.k && t < p.d) ? p.C[(long long)j * p.d + t] : 0.f;
        p.Ct[(long long)t * p.kpad + j] = v;
        s += (double)v * (double)v;
    }
    for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
    if (threadIdx.x == 0) p.h[j] = j < p.k ? (float)(0.5 * s) : __int_as_float(0x7f800000);
}

// ---- assign -------------------------------------------------------------------
// Tile: BM = 16*TM rows x BN clusters, thread micro-tile TM x BN/16.
template <int BN, int TM>
__global__ void __launch_bounds__(NT)
assign_kernel(Problem *P, const int2 *items, int n_items) {
    constexpr int TN = BN / 16, BM = 16 * TM;
    __shared__ __align__(16) float Xs[BK][BM + 4];
    __shared__ __align__(16) float Cs[BK][BN + 4];
    const int it = blockIdx.x;
    if (it >= n_items) return;
    const int2 w = items[it];  // (problem, row tile)
    const Problem &p = P[w.x];
    if (p.done) return;
    const long long row0 = (long long)w.y * BM;
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

// ---- accumulate -----------------------------------------------------------------
__global__ void zero_kernel(Problem *P, const int2 *items, int n_items) {
    const int it = blockIdx.x;
    if (it >= n_items) return;
    Problem &p = P[items[it].x];
    if (p.done) return;
    const int j = items[it].y;  // cluster
    for (int t = threadIdx.x; t < p.d; t += blockDim.x) p.acc[(long long)j * p.d + t] = 0ull;
    if (threadIdx.x == 0) p.counts[j] = 0;
}

__global__ void accumulate_kernel(Problem *P, const int2 *items, int n_items) {
    extern __shared__ unsigned long long sacc[];  // k*d sums, then k counts
    const int it = blockIdx.x;
    if (it >= n_items) return;
    const int2 w = items[it];  // (problem, row block)
    Problem &p = P[w.x];
    if (p.done) return;
    const int kd = p.k * p.d;
    for (int i = threadIdx.x; i < kd + p.k; i += blockDim.x) sacc[i] = 0ull;
    __syncthreads();
    const long long b = (long long)w.y * kAccRows, e = min(p.n, b + kAccRows);
    const long long total = (e - b) * p.d;
    const float *X = p.X + b * p.d;
    for (long long q = threadIdx.x; q < total; q += blockDim.x) {
        const long long r = q / p.d;
        const int t = (int)(q - r * p.d);
        const int lab = p.labels[b + r];
        const long long v = llrint((double)X[q] * p.scale);
        atomicAdd(&sacc[lab * p.d + t], (unsigned long long)v);
        if (t == 0) atomicAdd(&sacc[kd + lab], 1ull);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kd; i += blockDim.x)
        if (sacc[i]) atomicAdd(&p.acc[i], sacc[i]);
    for (int j = threadIdx.x; j < p.k; j += blockDim.x)
        if (sacc[kd + j]) atomicAdd(&p.counts[j], (int)sacc[kd + j]);
}

// ---- finalize / decide -------------------------------------------------------------
__global__ void finalize_kernel(Problem *P, const int2 *items, int n_items) {
    __shared__ double red[32];
    const int it = blockIdx.x;
    if (it >= n_items) return;
    Problem &p = P[items[it].x];
    if (p.done) return;
    const int j = items[it].y;
    const int cnt = p.counts[j];
    double a = 0.0;
    for (int t = threadIdx.x; t < p.d; t += blockDim.x) {
        if (cnt > 0) {
            const double S = (double)(long long)p.acc[(long long)j * p.d + t] / p.scale;
            const float c = (float)(S / (double)cnt);
            const double df = (double)p.C[(long long)j * p.d + t] - (double)c;
            a += df * df;
            p.C[(long long)j * p.d + t] = c;
        }
    }
    for (int m = 16; m >= 1; m >>= 1) a += __shfl_xor_sync(0xffffffffu, a, m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        p.shift_part[j] = cnt > 0 ? tot : 0.0;
    }
}

// One block per problem: shift, empty-cluster reseed, stop test.
__global__ void decide_kernel(Problem *P, int n_problems) {
    __shared__ double sred[NT];
    __shared__ float sv[NT];
    __shared__ long long sr[NT];
    __shared__ long long chosen[kMaxK];
    const int pi = blockIdx.x;
    if (pi >= n_problems) return;
    Problem &p = P[pi];
    if (p.done) return;
    // empty clusters, ascending
    int n_empty = 0;
    for (int j = 0; j < p.k; ++j) n_empty += p.counts[j] == 0;  // uniform loop (k <= 256)
    double shift = 0.0;
    if (n_empty > 0) {
        // m = n_empty farthest rows: repeated block argmax of d2 excluding chosen rows
        int e = 0;
        for (int j = 0; j < p.k; ++j) {
            if (p.counts[j] != 0) continue;
            float bv = -__int_as_float(0x7f800000);
            long long br = 0x7fffffffffffffffll;
            for (long long r = threadIdx.x; r < p.n; r += blockDim.x) {
                bool taken = false;
                for (int q = 0; q < e; ++q) taken |= chosen[q] == r;
                const float v = p.d2[r];
                if (!taken && (v > bv || (v == bv && r < br))) {
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
                for (int t = 1; t < (int)blockDim.x; ++t)
                    if (sv[t] > v0 || (sv[t] == v0 && sr[t] < r0)) {
                        v0 = sv[t];
                        r0 = sr[t];
                    }
                chosen[e] = r0;
            }
            __syncthreads();
            const long long row = chosen[e];
            double a = 0.0;
            for (int t = threadIdx.x; t < p.d; t += blockDim.x) {
                const float x = p.X[row * p.d + t];
                const double df = (double)p.C[(long long)j * p.d + t] - (double)x;
                a += df * df;
                p.C[(long long)j * p.d + t] = x;
            }
            sred[threadIdx.x] = a;
            __syncthreads();
            if (threadIdx.x == 0) {
                double tot = 0.0;
                for (int t = 0; t < (int)blockDim.x; ++t) tot += sred[t];
                p.shift_part[j] = tot;
            }
            __syncthreads();
            ++e;
        }
    }
    if (threadIdx.x == 0) {
        for (int j = 0; j < p.k; ++j) shift += p.shift_part[j];
        p.shift = shift;
        p.empty_events += n_empty;
        p.iters += 1;
        if (shift <= p.eps || p.iters >= p.max_iters) p.done = 1;
    }
}

// Row norms (once per call) and the per-problem fixed-point scale.
__global__ void setup_kernel(Problem *P, const int2 *items, int n_items) {
    const int it = blockIdx.x;
    if (it >= n_items) return;
    Problem &p = P[items[it].x];
    const long long b = (long long)items[it].y * kAccRows, e = min(p.n, b + kAccRows);
    float amax = 0.f;
    for (long long r = b + threadIdx.x; r < e; r += blockDim.x) {
        double s = 0.0;
        for (int t = 0; t < p.d; ++t) {
            const float x = p.X[r * p.d + t];
            s += (double)x * (double)x;
            amax = fmaxf(amax, fabsf(x));
        }
        p.xnorm[r] = (float)s;
    }
    for (int m = 16; m >= 1; m >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, m));
    if ((threadIdx.x & 31) == 0) atomicMax(&p.amax_bits, __float_as_int(amax));  // non-negative floats order as ints
}

__global__ void scale_kernel(Problem *P, int n_problems) {
    const int pi = blockIdx.x * blockDim.x + threadIdx.x;
    if (pi >= n_problems) return;
    Problem &p = P[pi];
    const float amax = __int_as_float(p.amax_bits);
    // sums stay below 2^62: |sum| <= n * amax * scale
    const double bound = (double)p.n * (double)fmaxf(amax, 1e-30f);
    const int e = (int)floor(62.0 - log2(bound));
    p.scale = ldexp(1.0, min(e, 1000));
}

}  // namespace batched

// ---- host side ------------------------------------------------------------------------

struct BatchedPlan {
    std::vector<batched::Problem> host;
    batched::Problem *dev = nullptr;
    std::vector<std::vector<int2>> assign_items;  // per variant
    std::vector<int> variant_bn, variant_tm;
    int2 *d_items = nullptr;
    std::vector<size_t> assign_off;  // offsets into d_items per variant
    size_t prep_off = 0, zero_off = 0, acc_off = 0;
    int n_prep = 0, n_zero = 0, n_acc = 0;
    size_t acc_smem = 0;
};

typedef void (*AssignFn)(batched::Problem *, const int2 *, int);

static AssignFn assign_fn(int bn, int tm) {
    using namespace batched;
    switch (bn * 10 + tm) {
        case 164: return assign_kernel<16, 4>;
        case 168: return assign_kernel<16, 8>;
        case 324: return assign_kernel<32, 4>;
        case 328: return assign_kernel<32, 8>;
        case 644: return assign_kernel<64, 4>;
        case 648: return assign_kernel<64, 8>;
        case 1284: return assign_kernel<128, 4>;
        case 1288: return assign_kernel<128, 8>;
        case 2564: return assign_kernel<256, 4>;
        case 2568: return assign_kernel<256, 8>;
    }
    return nullptr;
}

int batched_kpad(int k) {
    int b = 16;
    while (b < k) b <<= 1;
    return b;
}

}  // namespace kmb

#include <cstring>

namespace kmb {

// Autotuner cache: (d, kpad) -> rows per thread (4 or 8), per device.
static std::map<long long, int> g_tuned;

static int tuned_tm(int dev, int d, int kpad, cudaStream_t s) {
    const long long key = ((long long)dev << 40) | ((long long)d << 16) | kpad;
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) return it->second;
    // Time both candidates on 64K synthetic rows of this shape.
    using namespace batched;
    const long long n = 65536;
    const int dpad = (d + 7) / 8 * 8;
    float *X = nullptr, *Ct = nullptr, *h = nullptr, *d2 = nullptr, *xn = nullptr;
    int32_t *lab = nullptr;
    Problem *dp = nullptr;
    int2 *items = nullptr;
    int best_tm = 8;
    if (cudaMalloc(&X, sizeof(float) * n * d) == cudaSuccess && cudaMalloc(&Ct, sizeof(float) * dpad * kpad) == cudaSuccess &&
        cudaMalloc(&h, sizeof(float) * kpad) == cudaSuccess && cudaMalloc(&d2, sizeof(float) * n) == cudaSuccess &&
        cudaMalloc(&xn, sizeof(float) * n) == cudaSuccess && cudaMalloc(&lab, sizeof(int32_t) * n) == cudaSuccess &&
        cudaMalloc(&dp, sizeof(Problem)) == cudaSuccess && cudaMalloc(&items, sizeof(int2) * (n / 64)) == cudaSuccess) {
        cudaMemsetAsync(X, 0, sizeof(float) * n * d, s);
        cudaMemsetAsync(Ct, 0, sizeof(float) * dpad * kpad, s);
        cudaMemsetAsync(h, 0, sizeof(float) * kpad, s);
        cudaMemsetAsync(xn, 0, sizeof(float) * n, s);
        Problem p;
        std::memset(&p, 0, sizeof(p));
        p.X = X; p.Ct = Ct; p.h = h; p.labels = lab; p.d2 = d2; p.xnorm = xn;
        p.n = n; p.d = d; p.dpad = dpad; p.k = kpad; p.kpad = kpad;
        cudaMemcpyAsync(dp, &p, sizeof(p), cudaMemcpyHostToDevice, s);
        float best_ms = 1e30f;
        for (int tm : {4, 8}) {
            const int bm = 16 * tm;
            const int nit = (int)((n + bm - 1) / bm);
            std::vector<int2> hv(nit);
            for (int i = 0; i < nit; ++i) hv[i] = make_int2(0, i);
            cudaMemcpyAsync(items, hv.data(), sizeof(int2) * nit, cudaMemcpyHostToDevice, s);
            AssignFn f = assign_fn(kpad, tm);
            cudaEvent_t a, b;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            f<<<nit, NT, 0, s>>>(dp, items, nit);  // warm-up
            KMB_LAUNCHED();
            cudaEventRecord(a, s);
            for (int r = 0; r < 5; ++r) {
                f<<<nit, NT, 0, s>>>(dp, items, nit);
                KMB_LAUNCHED();
            }
            cudaEventRecord(b, s);
            cudaEventSynchronize(b);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            cudaEventDestroy(a);
            cudaEventDestroy(b);
            if (ms < best_ms) {
                best_ms = ms;
                best_tm = tm;
            }
        }
    }
    cudaGetLastError();
    cudaFree(X); cudaFree(Ct); cudaFree(h); cudaFree(d2); cudaFree(xn); cudaFree(lab); cudaFree(dp); cudaFree(items);
    g_tuned[key] = best_tm;
    return best_tm;
}

}  // namespace kmb

extern "C" int kmb_batched_train(int dtype, kmb_batched_problem *problems, int64_t count, int64_t max_iteration_count,
                                 double accuracy_threshold, int32_t use_graph, void *cuda_stream,
                                 kmb_batched_info *info) {
    using namespace kmb;
    using namespace kmb::batched;
    if (dtype != KMB_F32 || !problems || count <= 0 || max_iteration_count < 0 || !(accuracy_threshold >= 0))
        return KMB_EINVAL;
    for (int64_t i = 0; i < count; ++i) {
        const kmb_batched_problem &q = problems[i];
        if (!q.X || !q.C || !q.labels || q.n <= 0 || q.n > INT32_MAX || q.d <= 0 || q.k <= 0 || q.k > kMaxK ||
            q.k > q.n || (q.k * q.d + q.k) * 8 > 200 * 1024)
            return KMB_EINVAL;
    }
    cudaStream_t s = (cudaStream_t)cuda_stream;
    int dev = 0;
    cudaGetDevice(&dev);
    // Device allocations: per-problem scratch in one arena.
    size_t arena = 0;
    std::vector<size_t> off(count * 8);
    auto take = [&](size_t bytes) {
        const size_t o = arena;
        arena += (bytes + 255) / 256 * 256;
        return o;
    };
    std::vector<Problem> H(count);
    for (int64_t i = 0; i < count; ++i) {
        const kmb_batched_problem &q = problems[i];
        const int kpad = batched_kpad((int)q.k), dpad = (int)((q.d + 7) / 8 * 8);
        off[i * 8 + 0] = take(sizeof(float) * dpad * kpad);
        off[i * 8 + 1] = take(sizeof(float) * kpad);
        off[i * 8 + 2] = take(sizeof(float) * q.n);       // d2
        off[i * 8 + 3] = take(sizeof(float) * q.n);       // xnorm
        off[i * 8 + 4] = take(sizeof(unsigned long long) * q.k * q.d);
        off[i * 8 + 5] = take(sizeof(int) * q.k);
        off[i * 8 + 6] = take(sizeof(double) * q.k);
    }
    unsigned char *base = nullptr;
    if (cudaMalloc(&base, arena) != cudaSuccess) {
        cudaGetLastError();
        return KMB_ENOMEM;
    }
    std::vector<int2> prep_items, zero_items, acc_items;
    std::map<long long, std::vector<int2>> assign_by_variant;  // key bn*10+tm
    size_t acc_smem = 0;
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
        p.Ct = (float *)(base + off[i * 8 + 0]);
        p.h = (float *)(base + off[i * 8 + 1]);
        p.d2 = (float *)(base + off[i * 8 + 2]);
        p.xnorm = (float *)(base + off[i * 8 + 3]);
        p.acc = (unsigned long long *)(base + off[i * 8 + 4]);
        p.counts = (int *)(base + off[i * 8 + 5]);
        p.shift_part = (double *)(base + off[i * 8 + 6]);
        p.scale = 0.0;
        p.max_iters = (int)max_iteration_count;
        p.eps = accuracy_threshold;
        p.done = max_iteration_count == 0 ? 1 : 0;
        for (int j = 0; j < p.kpad; ++j) prep_items.push_back(make_int2((int)i, j));
        for (int j = 0; j < p.k; ++j) zero_items.push_back(make_int2((int)i, j));
        const int tm = tuned_tm(dev, p.d, p.kpad, s);
        const int bm = 16 * tm;
        auto &v = assign_by_variant[(long long)p.kpad * 10 + tm];
        for (long long t = 0; t < (p.n + bm - 1) / bm; ++t) v.push_back(make_int2((int)i, (int)t));
        for (long long b = 0; b < (p.n + kAccRows - 1) / kAccRows; ++b) acc_items.push_back(make_int2((int)i, (int)b));
        acc_smem = std::max(acc_smem, sizeof(unsigned long long) * (size_t)(p.k * p.d + p.k));
    }
    // one items array: prep | zero | acc | assign variants
    std::vector<int2> all;
    const size_t prep_off = all.size();
    all.insert(all.end(), prep_items.begin(), prep_items.end());
    const size_t zero_off = all.size();
    all.insert(all.end(), zero_items.begin(), zero_items.end());
    const size_t acc_off = all.size();
    all.insert(all.end(), acc_items.begin(), acc_items.end());
    std::vector<std::pair<long long, std::pair<size_t, int>>> variants;
    for (auto &kv : assign_by_variant) {
        variants.push_back({kv.first, {all.size(), (int)kv.second.size()}});
        all.insert(all.end(), kv.second.begin(), kv.second.end());
    }
    Problem *dP = nullptr;
    int2 *dI = nullptr;
    if (cudaMalloc(&dP, sizeof(Problem) * count) != cudaSuccess || cudaMalloc(&dI, sizeof(int2) * all.size()) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(base);
        cudaFree(dP);
        return KMB_ENOMEM;
    }
    cudaMemcpyAsync(dP, H.data(), sizeof(Problem) * count, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dI, all.data(), sizeof(int2) * all.size(), cudaMemcpyHostToDevice, s);
    if (acc_smem > 48 * 1024)
        cudaFuncSetAttribute(accumulate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)acc_smem);
    setup_kernel<<<(unsigned)acc_items.size(), NT, 0, s>>>(dP, dI + acc_off, (int)acc_items.size());
    KMB_LAUNCHED();
    scale_kernel<<<(unsigned)((count + 127) / 128), 128, 0, s>>>(dP, (int)count);
    KMB_LAUNCHED();

    auto enqueue_iteration = [&](cudaStream_t st) {
        prep_kernel<<<(unsigned)prep_items.size(), 32, 0, st>>>(dP, dI + prep_off, (int)prep_items.size());
        for (auto &v : variants) {
            const int bn = (int)(v.first / 10), tm = (int)(v.first % 10);
            assign_fn(bn, tm)<<<(unsigned)v.second.second, NT, 0, st>>>(dP, dI + v.second.first, v.second.second);
        }
        zero_kernel<<<(unsigned)zero_items.size(), 64, 0, st>>>(dP, dI + zero_off, (int)zero_items.size());
        accumulate_kernel<<<(unsigned)acc_items.size(), NT, acc_smem, st>>>(dP, dI + acc_off, (int)acc_items.size());
        finalize_kernel<<<(unsigned)zero_items.size(), 64, 0, st>>>(dP, dI + zero_off, (int)zero_items.size());
        decide_kernel<<<(unsigned)count, NT, 0, st>>>(dP, (int)count);
    };
    const int per_iter = 5 + (int)variants.size();
    int rc = KMB_OK;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    if (use_graph && max_iteration_count > 0) {
        // Capture on a private stream (the caller's may be the legacy default
        // stream, which cannot be captured); the graph is then launched on the
        // caller's stream, after the setup work above.
        cudaStream_t cap = nullptr;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            rc = KMB_ECUDA;
        if (rc == KMB_OK) {
            enqueue_iteration(cap);
            if (cudaStreamEndCapture(cap, &graph) != cudaSuccess ||
                cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
                rc = KMB_ECUDA;
        }
        if (cap) cudaStreamDestroy(cap);
        if (rc != KMB_OK) cudaGetLastError();
        for (int64_t it = 0; rc == KMB_OK && it < max_iteration_count; ++it) {
            if (cudaGraphLaunch(exec, s) != cudaSuccess) rc = KMB_ECUDA;
            launch_count() += per_iter;
        }
    } else {
        for (int64_t it = 0; it < max_iteration_count; ++it) {
            enqueue_iteration(s);
            launch_count() += per_iter;
        }
    }
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = KMB_ECUDA;
    if (rc == KMB_OK) {
        cudaMemcpy(H.data(), dP, sizeof(Problem) * count, cudaMemcpyDeviceToHost);
        long long total_iters = 0;
        for (int64_t i = 0; i < count; ++i) {
            problems[i].iterations = H[i].iters;
            problems[i].last_shift = H[i].shift;
            total_iters += H[i].iters;
        }
        if (info) {
            info->problems = count;
            info->variants = (int32_t)variants.size();
            info->total_iterations = total_iters;
            info->graph_launches = use_graph ? max_iteration_count : 0;
        }
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaFree(dP);
    cudaFree(dI);
    cudaFree(base);
    return rc;
}
