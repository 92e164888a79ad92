// Grouped assignment for the serving loop: many infer requests (each with its
// own rows, model, k and d) in one launch.
//
// A work item is (request, 128-row tile, chunk of up to 512 clusters). Each CTA
// computes h_j - x.c_j with the same register-tiled FP32 FMA scheme as the
// plain assignment kernel (scores of cpp/daal/src/algorithms/kmeans/
// kmeans_lloyd_postprocessing.h:95-130) and folds its rows' best (score, index)
// into a 64-bit key per row with atomicMin: the key is the order-preserving
// bit pattern of the FP32 score in the high word and the cluster index in the
// low word, so the minimum key is the best score with the lowest index on ties,
// whatever order the chunks finish in. A second pass unpacks the labels.
#include "kmb_internal.cuh"

namespace kmb {
namespace serve {

struct ReqDesc {
    const float *X;        // n x d rows (device)
    const float *Ct;       // model: dpad x kpad transposed centroids
    const float *h;        // model: kpad half squared norms (+inf padding)
    unsigned long long *key;  // n packed (score, index) keys
    int32_t *labels;       // n labels
    long long n;
    int d, k, kpad, chunks;  // chunks = ceil(kpad / kChunk)
    long long item_begin;    // first work item of this request
    long long row_begin;     // first row of this request in the batch's row space
};

constexpr int BM = 128, BN = 128, BK = 8, NT = 256, PAD = 4;
constexpr int kChunk = 512;  // clusters per work item

__device__ __forceinline__ unsigned int ordered_bits(float v) {
    const unsigned int u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ int find_req(const ReqDesc *__restrict__ reqs, int nreq, long long item) {
    int lo = 0, hi = nreq;  // reqs[lo].item_begin <= item < reqs[hi].item_begin
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (reqs[mid].item_begin <= item) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(NT, 1)
grouped_assign_kernel(const ReqDesc *__restrict__ reqs, int nreq, long long n_items) {
    __shared__ __align__(16) float Xs[2][BK][BM + PAD];
    __shared__ __align__(16) float Cs[2][BK][BN + PAD];
    const long long item = blockIdx.x;
    if (item >= n_items) return;
    const ReqDesc R = reqs[find_req(reqs, nreq, item)];
    const long long local = item - R.item_begin;
    const long long tile = local / R.chunks;
    const int chunk = (int)(local - tile * R.chunks);
    const long long row0 = tile * BM;
    const int col_begin = chunk * kChunk;
    const int col_end = min(R.kpad, col_begin + kChunk);
    const int d = R.d;

    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    const int lr = tid >> 1, lk = (tid & 1) * 4;
    const long long grow = row0 + lr;
    const bool row_ok = grow < R.n;
    const float *xrow = R.X + (row_ok ? grow : 0) * (long long)d;
    const bool vec = (d % 4 == 0) && ((reinterpret_cast<uintptr_t>(R.X) & 15) == 0);
    const int ck = tid >> 5, cn = (tid & 31) * 4;
    const int nk = (d + BK - 1) / BK;
    const int ntl = (col_end - col_begin) / BN;
    const int steps = nk * ntl;

    float xr[4];
    float4 cr;
    auto gload = [&](int step) {
        const int nt = step / nk, kc = step - nt * nk;
        const int kb = kc * BK;
        if (vec) {
            if (row_ok && kb + lk < d) {
                const float4 v = *reinterpret_cast<const float4 *>(xrow + kb + lk);
                xr[0] = v.x; xr[1] = v.y; xr[2] = v.z; xr[3] = v.w;
            } else {
                xr[0] = xr[1] = xr[2] = xr[3] = 0.f;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) xr[q] = (row_ok && kb + lk + q < d) ? xrow[kb + lk + q] : 0.f;
        }
        cr = *reinterpret_cast<const float4 *>(R.Ct + (long long)(kb + ck) * R.kpad + col_begin + nt * BN + cn);
    };
    auto sstore = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 4; ++q) Xs[buf][lk + q][lr] = xr[q];
        *reinterpret_cast<float4 *>(&Cs[buf][ck][cn]) = cr;
    };

    float best[8];
    int bidx[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        best[i] = __int_as_float(0x7f800000);
        bidx[i] = 0;
    }
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

    gload(0);
    sstore(0);
    __syncthreads();
    for (int step = 0; step < steps; ++step) {
        const int buf = step & 1;
        if (step + 1 < steps) gload(step + 1);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&Xs[buf][kk][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&Xs[buf][kk][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4 *>(&Cs[buf][kk][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&Cs[buf][kk][64 + tx * 4]);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        const int nt = step / nk;
        if (step - nt * nk == nk - 1) {
            const int cbase = col_begin + nt * BN;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int col = cbase + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
                const float hj = R.h[col];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float v = hj - acc[i][j];
                    if (v < best[i]) {  // columns increase within a thread: lowest index on ties
                        best[i] = v;
                        bidx[i] = col;
                    }
                    acc[i][j] = 0.f;
                }
            }
        }
        if (step + 1 < steps) sstore(buf ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const long long r = row0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        unsigned long long key = ((unsigned long long)ordered_bits(best[i]) << 32) | (unsigned int)bidx[i];
#pragma unroll
        for (int m = 8; m >= 1; m >>= 1) {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, m);
            key = o < key ? o : key;
        }
        if (tx == 0 && r < R.n) atomicMin(&R.key[r], key);
    }
}

__global__ void init_keys_kernel(const ReqDesc *__restrict__ reqs, int nreq, long long total_rows) {
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total_rows;
         g += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nreq;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (reqs[mid].row_begin <= g) lo = mid; else hi = mid;
        }
        reqs[lo].key[g - reqs[lo].row_begin] = ~0ull;
    }
}

__global__ void unpack_labels_kernel(const ReqDesc *__restrict__ reqs, int nreq, long long total_rows) {
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total_rows;
         g += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nreq;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (reqs[mid].row_begin <= g) lo = mid; else hi = mid;
        }
        const long long r = g - reqs[lo].row_begin;
        reqs[lo].labels[r] = (int32_t)(reqs[lo].key[r] & 0xffffffffull);
    }
}

}  // namespace serve

// Host entry used by the serving engine: reqs_dev holds nreq descriptors (with
// item_begin / row_begin filled); total items / rows are their sums.
void launch_grouped_infer(const void *reqs_dev, int nreq, long long n_items, long long total_rows, cudaStream_t s) {
    if (nreq == 0) return;
    const serve::ReqDesc *r = (const serve::ReqDesc *)reqs_dev;
    const int eb = (int)std::min<long long>((total_rows + 255) / 256, 148 * 8);
    serve::init_keys_kernel<<<eb, 256, 0, s>>>(r, nreq, total_rows);
    KMB_LAUNCHED();
    serve::grouped_assign_kernel<<<(unsigned)n_items, serve::NT, 0, s>>>(r, nreq, n_items);
    KMB_LAUNCHED();
    serve::unpack_labels_kernel<<<eb, 256, 0, s>>>(r, nreq, total_rows);
    KMB_LAUNCHED();
}

size_t grouped_desc_bytes() { return sizeof(serve::ReqDesc); }
int grouped_chunk_clusters() { return serve::kChunk; }

}  // namespace kmb
