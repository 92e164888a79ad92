// Tensor-core assignment (KMB_FORM_BF16X3): split-BF16 x.c on tcgen05 with FP32
// accumulation in TMEM, fused per-row argmin, near-tie queue for the FP64 recheck.
//
// Same contract as the plain kernel (scores h_j - x.c_j, lowest index on ties,
// DAAL's kmeans_lloyd_impl.i:185-216 / kmeans_lloyd_postprocessing.h:95-130),
// different arithmetic: x = xh + xl and c = ch + cl with xh = bf16(x),
// xl = bf16(x - xh) (same for c), and
//     x.c ~= xh.ch + xh.cl + xl.ch
// as three tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulate) per 16-wide
// k-step into one TMEM accumulator.
//
// Per-score error bound (u_b = 2^-8 bf16 unit roundoff, u = 2^-24 FP32):
//   |dropped terms| <= 3.03 u_b^2 sum_t |x_t c_t|                (split)
//   |accumulation|  <= 2 * 3 dpad * 2u * sum_t |x_t c_t|         (FP32 adds in the
//                      tensor core, truncation allowed, factor 2 margin)
//   |h rounding + final subtraction| <= 2u (h + ||x|| ||c||)
// with sum_t |x_t c_t| <= ||x|| ||c|| <= ||x|| cmax. Two scores whose computed
// gap exceeds twice the bound are ordered as the exact ones; every other row
// is queued with its two best clusters (or flagged for a full rescan when a
// third cluster is inside the band) and re-scored in FP64 by the recheck kernel.
//
// Kernel structure (one CTA per SM, persistent over 128-row tiles, 10 warps):
//   warp 0   TMA producer: A = the tile's Xhi/Xlo panels (128 rows x 64 bf16,
//            SWIZZLE_128B), B = Chi/Clo panels of BN clusters (BN = 256: 32 bf16,
//            SWIZZLE_64B; BN = 128 where padding k to 256 would cost more than
//            the wider tile gains: 64 bf16, SWIZZLE_128B), ring of 32 KB stages
//   warp 1   TMEM allocation + single-thread tcgen05.mma issue (M=128, N=BN,
//            K=16); commits free B stages, publish accumulators and release A tiles
//   warps 2-9 epilogue, two groups of 4 warps (one per TMEM lane quarter):
//            group g drains the 32-column chunks g, g+2, g+4, ... of every
//            accumulator. Before the MMAs of a tile start, the drain of the
//            accumulator's previous tile writes -h_j into every lane of it
//            (tcgen05.st), so the MMAs leave
//            y = x.c - h = -score there and no per-score subtraction is needed.
//            A group reads y with tcgen05.ld (one TMEM lane = one row per
//            thread) and keeps a running top-3 per row: each 32-column chunk
//            is first reduced to its maximum (branch-free, 3-input max); only
//            chunks holding a value at or above the row's threshold take the
//            exact insertion path. At the end of a row tile group 1 hands
//            its top-3 to group 0 through a small global scratch (per SM, by
//            row-tile parity) and a named barrier; group 0 merges and writes
//            the row's outputs.
// 512 / BN accumulators of BN columns (all 512 TMEM columns): while the groups
// drain one, the MMAs fill the others. The 256-wide tile halves the shared-memory reads
// of the A panels per MMA; at N=128 the operand reads plus the B panel writes
// exceeded the shared-memory bandwidth at full tensor rate. Every mbarrier
// wait is bounded; on timeout the
// CTA records KMB_ETIMEDOUT in the loop state, drains its own TMA loads and
// MMAs with bounded waits, frees TMEM and returns.
#include "kmb_internal.cuh"

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>

namespace kmb {
namespace tc {

constexpr int BM = 128;                 // rows per tile (UMMA M)
// Clusters per tile (UMMA N) is the kernel's template parameter BN: 256 when
// the padded cluster count (a multiple of 128) divides by 256, else 128.
constexpr int KP = 64;                  // bf16 per A panel row (128 bytes, SWIZZLE_128B)
// bf16 per B panel row: 32 (64 B, SWIZZLE_64B) for 256-cluster tiles, 64 (128 B,
// SWIZZLE_128B) for 128-cluster tiles, so a B stage (hi + lo panels) is 32 KB
// either way; 16-wide panels in six stages measured 11 % slower.
__host__ __device__ constexpr int kpb_of(int bn, bool pair = false) { return (bn == 256 && !pair) ? 32 : 64; }
// Clusters of one B panel in a CTA's shared memory: the whole cluster tile, or,
// for a CTA pair, its half (each CTA of the pair holds BN/2 clusters).
__host__ __device__ constexpr int b_rows_of(int bn, bool pair) { return pair ? bn / 2 : bn; }
constexpr int PANEL = 128 * 128;        // bytes per A panel (128 rows x 128 B)
constexpr int TMEM_COLS = 512;          // all of TMEM: 512 / BN accumulators of BN columns
constexpr int kMaxAcc = 4;
__host__ __device__ constexpr int panel_b_bytes(int bn, bool pair = false) {
    return b_rows_of(bn, pair) * kpb_of(bn, pair) * 2;  // one B panel (16 KB; 8 KB for a pair's half of BN = 128)
}
constexpr int NGROUPS = 2;              // epilogue groups of 4 warps (one warp per TMEM lane quarter)
constexpr int NTHREADS = 64 + NGROUPS * 128;  // warp 0 TMA, warp 1 MMA, warps 2.. epilogue
constexpr int MAX_B_STAGES = 8;
constexpr int kMaxSmid = 1024;
constexpr long long kTimeoutCycles = 4000000000ll;  // ~2 s at 1.9 GHz

// One row's running top-3 (score space) as handed between the epilogue groups.
struct Top3x {
    float b, s, t;
    int ib, is;
    int pad[3];
};

struct Params {
    int64_t n;
    int d, dpad, k, kpad;
    int n_tiles, kpanels, ntiles_n;
    int a_stages, b_stages;
    const float *h;  // -0.5||c_j||^2 per cluster, -inf padding
    const float *xnorm;
    const float2 *rowb;  // per row: {prior threshold, band}, from row_bounds_kernel
    int32_t *labels;
    float *d2;
    RecheckEntry *queue;
    LoopState *st;
    Top3x *xchg;  // per SM (one CTA fits an SM): 2 (row-tile parity) x (NGROUPS-1) x 128 rows of top-3
    long long wait_cycles;  // limit of every pipeline wait (the abort-path drains keep kTimeoutCycles)
};

struct Barriers {
    uint64_t a_full[2], a_empty[2];
    uint64_t b_full[MAX_B_STAGES], b_empty[MAX_B_STAGES];
    uint64_t acc_full[kMaxAcc], acc_empty[kMaxAcc];
    uint64_t mma_done;
    uint32_t tmem_base;
    int abort;
};

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false on abort (set by any role) or after `limit` cycles (which
// sets abort).
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, volatile int *abort,
                                          long long limit = kTimeoutCycles) {
    if (mbar_test(b, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test(b, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > limit) {
            *abort = 1;
            return false;
        }
    }
    return true;
}
// Drain wait used on the abort path: ignores the abort flag, still bounded.
__device__ __forceinline__ void mbar_drain(uint64_t *b, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_test(b, parity)) {
        if (clock64() - t0 > kTimeoutCycles) return;
    }
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, uint64_t *bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            su32(dst)),
        "l"(tm), "r"(su32(bar)), "r"(x), "r"(y)
        : "memory");
}

// ---- CTA-pair (cta_group::2) helpers --------------------------------------
__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// Address of the same shared-memory variable in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t peer_addr(const void *p, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(su32(p)), "r"(rank));
    return r;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Arrive on an mbarrier given by its shared::cluster address (this CTA's or the peer's).
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
// Tile load of a CTA pair: lands in this CTA's shared memory, completes on the
// pair's (leader CTA's) mbarrier, given by its shared::cluster address.
__device__ __forceinline__ void tma_load_2d_pair(void *dst, const CUtensorMap *tm, uint32_t bar_cluster, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
        "[%2];" ::"r"(su32(dst)),
        "l"(tm), "r"(bar_cluster), "r"(x), "r"(y)
        : "memory");
}

// K-major SWIZZLE_128B operand descriptor (sm100 format: version 1, LBO 16 B
// (unused for swizzled K-major), SBO 1024 B between 8-row groups, layout 2).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)1 << 16;          // LBO
    d |= (uint64_t)(1024 >> 4) << 32; // SBO
    d |= (uint64_t)1 << 46;          // version
    d |= (uint64_t)2 << 61;          // SWIZZLE_128B
    return d;
}

// K-major B panel descriptor: rows of KPB bf16 (128 B: SWIZZLE_128B, layout 2;
// 64 B: SWIZZLE_64B, layout 4), SBO = 8 rows between 8-row groups.
template <int KPB>
__device__ __forceinline__ uint64_t swb_desc(uint32_t saddr) {
    static_assert(KPB == 32 || KPB == 64, "B panel width");
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)1 << 16;                       // LBO
    d |= (uint64_t)((8 * KPB * 2) >> 4) << 32;    // SBO
    d |= (uint64_t)1 << 46;                       // version
    d |= (uint64_t)(KPB == 32 ? 4 : 2) << 61;     // SWIZZLE_64B / SWIZZLE_128B
    return d;
}

// kind::f16 instruction descriptor: D f32, A/B bf16, both K-major, M = 128 (one
// CTA) or 256 (a CTA pair), N = bn.
__host__ __device__ constexpr uint32_t make_idesc(int bn, int m = BM) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// The three split-BF16 products of one k-step (xh.ch, xh.cl, xl.ch) into one
// accumulator; descriptors are passed precomputed.
__device__ __forceinline__ void mma_bf16x3(uint32_t tmem_d, uint64_t ah, uint64_t al, uint64_t bh, uint64_t bl,
                                           uint32_t idesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, 1, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %3, %5, p;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %4, %5, p;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %2, %3, %5, p;\n\t}" ::"r"(tmem_d),
        "l"(ah), "l"(al), "l"(bh), "l"(bl), "r"(idesc)
        : "memory");
}
// One BF16 product per k-step (xh.ch): the single-product form.
__device__ __forceinline__ void mma_bf16x1(uint32_t tmem_d, uint64_t ah, uint64_t bh, uint32_t idesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, 1, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(ah), "l"(bh), "r"(idesc)
        : "memory");
}
__device__ __forceinline__ void mma_bf16x1_pair(uint32_t tmem_d, uint64_t ah, uint64_t bh, uint32_t idesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, 1, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(ah), "l"(bh), "r"(idesc)
        : "memory");
}

// The same for a CTA pair (issued by the leader CTA): M = 256 rows, 128 from
// each CTA's A panels; the B tile's two halves come from the two CTAs.
__device__ __forceinline__ void mma_bf16x3_pair(uint32_t tmem_d, uint64_t ah, uint64_t al, uint64_t bh, uint64_t bl,
                                                uint32_t idesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, 1, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %3, %5, p;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %4, %5, p;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %2, %3, %5, p;\n\t}" ::"r"(tmem_d),
        "l"(ah), "l"(al), "l"(bh), "l"(bl), "r"(idesc)
        : "memory");
}
// Completion of the pair's MMAs issued so far, signalled on the mbarrier at the
// same offset in both CTAs of the pair.
__device__ __forceinline__ void mma_commit_pair(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            su32(bar)),
        "h"((uint16_t)3)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// tcgen05.ld of 32 columns without the wait (the caller issues wait::ld).
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

struct Top3 {
    float b, s, t;
    int ib, is;
};

__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Stores 32 consecutive floats of global memory (the same for every lane) into
// this warp's 32 TMEM lanes, 32 columns starting at taddr.
__device__ __forceinline__ void tmem_st32_from(uint32_t taddr, const float *src) {
    uint32_t r[32];
#pragma unroll
    for (int i = 0; i < 32; i += 4) {
        const float4 q = __ldg(reinterpret_cast<const float4 *>(src + i));
        r[i] = __float_as_uint(q.x);
        r[i + 1] = __float_as_uint(q.y);
        r[i + 2] = __float_as_uint(q.z);
        r[i + 3] = __float_as_uint(q.w);
    }
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]),
        "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]),
        "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void named_bar_sync(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Waits for this thread's tcgen05.ld; v is tied to the wait, so no use of v can
// be scheduled above it.
__device__ __forceinline__ void tmem_wait_ld_regs(float (&v)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7]),
                   "+f"(v[8]), "+f"(v[9]), "+f"(v[10]), "+f"(v[11]), "+f"(v[12]), "+f"(v[13]), "+f"(v[14]),
                   "+f"(v[15]), "+f"(v[16]), "+f"(v[17]), "+f"(v[18]), "+f"(v[19]), "+f"(v[20]), "+f"(v[21]),
                   "+f"(v[22]), "+f"(v[23]), "+f"(v[24]), "+f"(v[25]), "+f"(v[26]), "+f"(v[27]), "+f"(v[28]),
                   "+f"(v[29]), "+f"(v[30]), "+f"(v[31])
                 :
                 : "memory");
}

// 32 consecutive floats of global memory (the same for every lane) into registers.
__device__ __forceinline__ void load_h32(const float *src, uint32_t (&r)[32]) {
#pragma unroll
    for (int i = 0; i < 32; i += 4) {
        const float4 q = __ldg(reinterpret_cast<const float4 *>(src + i));
        r[i] = __float_as_uint(q.x);
        r[i + 1] = __float_as_uint(q.y);
        r[i + 2] = __float_as_uint(q.z);
        r[i + 3] = __float_as_uint(q.w);
    }
}

// Stores 32 registers into this warp's 32 TMEM lanes, 32 columns starting at taddr.
__device__ __forceinline__ void tmem_st32_regs(uint32_t taddr, const uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]),
        "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]),
        "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}

// Inserts value x of column col (columns arrive in ascending order) into the
// row's running top-3 in y = -score space when x >= thr and x beats the third:
// strict '>' keeps the lowest index on ties. Branch-free; thr is raised to
// max(thr0, third, best - band) after an insertion.
__device__ __forceinline__ void top3_insert(Top3 &r, float &thr, float thr0, float band_up, float x, int col) {
    const bool ins = x >= thr && x > r.t;
    const bool gb = ins && x > r.b;
    const bool gs = ins && x > r.s;  // implied by gb (b >= s)
    const float t = gs ? r.s : (ins ? x : r.t);
    const float s2 = gb ? r.b : (gs ? x : r.s);
    const int is2 = gb ? r.ib : (gs ? col : r.is);
    r.b = gb ? x : r.b;
    r.ib = gb ? col : r.ib;
    r.s = s2;
    r.is = is2;
    r.t = t;
    thr = ins ? fmaxf(fmaxf(thr0, r.t), __fsub_rd(r.b, band_up)) : thr;
}

// One 32-column chunk of a row into its running top-3. The chunk is reduced to
// its maximum (3-input max.f32); only when a lane of the warp holds a value at or
// above its threshold are the column triples walked, group by group, a triple
// being visited (warp-uniformly, static register indices) when some lane's
// triple maximum reaches that lane's threshold.
__device__ __forceinline__ void scan_chunk(const float (&w)[32], int colbase, float thr0, float band_up, float &thr,
                                           Top3 &r) {
    float m[11];
#pragma unroll
    for (int i = 0; i < 10; ++i) m[i] = max3f(w[3 * i], w[3 * i + 1], w[3 * i + 2]);
    m[10] = fmaxf(w[30], w[31]);
    // four groups of triples (columns 0-8, 9-17, 18-26, 27-31): a group is walked
    // only when some lane's group maximum reaches that lane's threshold
    const float gm[4] = {max3f(m[0], m[1], m[2]), max3f(m[3], m[4], m[5]), max3f(m[6], m[7], m[8]), fmaxf(m[9], m[10])};
    const float m1 = max3f(gm[0], gm[1], fmaxf(gm[2], gm[3]));
    if (__any_sync(0xffffffffu, m1 >= thr)) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (__any_sync(0xffffffffu, gm[q] >= thr)) {
#pragma unroll
                for (int g = 3 * q; g < 3 * q + 3 && g < 11; ++g) {
                    if (__any_sync(0xffffffffu, m[g] >= thr)) {
#pragma unroll
                        for (int i = 0; i < 3; ++i)
                            if (3 * g + i < 32) top3_insert(r, thr, thr0, band_up, w[3 * g + i], colbase + 3 * g + i);
                    }
                }
            }
        }
    }
}

// (value, index) order; indices kept for the first two places.
__device__ __forceinline__ bool lex_lt(float a, int ia, float b, int ib) { return a < b || (a == b && ia < ib); }

// Merge of two sorted triples by selects (no indexed arrays, so no local memory):
// the same comparisons, in the same argument order, as a two-list merge of three
// outputs; a third place carries no index.
__device__ __forceinline__ Top3 top3_merge(const Top3 &x, const Top3 &y) {
    constexpr int kNone = 0x7fffffff;
    const bool c0 = lex_lt(x.b, x.ib, y.b, y.ib);
    const float xa = c0 ? x.s : x.b, ya = c0 ? y.b : y.s;
    const int xai = c0 ? x.is : x.ib, yai = c0 ? y.ib : y.is;
    const bool c1 = lex_lt(xa, xai, ya, yai);
    const bool xx = c0 && c1, yy = !c0 && !c1;
    const float xh = xx ? x.t : (yy ? x.b : x.s), yh = xx ? y.b : (yy ? y.t : y.s);
    const int xhi = xx ? kNone : (yy ? x.ib : x.is), yhi = xx ? y.ib : (yy ? kNone : y.is);
    const bool c2 = lex_lt(xh, xhi, yh, yhi);
    Top3 r;
    r.b = c0 ? x.b : y.b;
    r.ib = c0 ? x.ib : y.ib;
    r.s = c1 ? xa : ya;
    r.is = c1 ? xai : yai;
    r.t = c2 ? xh : yh;
    return r;
}


template <int BN, bool PAIR, int NPROD>
__global__ void __launch_bounds__(NTHREADS, 1)
assign_tc_kernel(const __grid_constant__ CUtensorMap tmXh, const __grid_constant__ CUtensorMap tmXl,
                 const __grid_constant__ CUtensorMap tmCh, const __grid_constant__ CUtensorMap tmCl, Params p) {
    constexpr int NACC = TMEM_COLS / BN;  // TMEM accumulators (double-buffered or more)
    constexpr int PANEL_B = panel_b_bytes(BN, PAIR);
    constexpr int KPB = kpb_of(BN, PAIR);
    constexpr int BROWS = b_rows_of(BN, PAIR);  // clusters of a B panel in this CTA
    constexpr int NCTA = PAIR ? 2 : 1;          // CTAs sharing one MMA (a pair: M = 256)
    constexpr uint32_t kIdesc = make_idesc(BN, NCTA * BM);
    static_assert(NACC >= 2 && NACC <= kMaxAcc, "accumulator count");
    static_assert(NPROD == 1 || NPROD == 3, "products per k-step");
    constexpr int NSPLIT = NPROD == 3 ? 2 : 1;  // panels per operand: hi (+ lo for the split form)
    constexpr int BSTAGE = NSPLIT * PANEL_B;    // bytes of one B stage in this CTA
    const uint32_t rank = PAIR ? cluster_rank() : 0u;  // 0: the pair's leader (issues the MMAs)
    // One read of the loop flag for the whole CTA (for a pair: the leader's read,
    // for both CTAs), so every thread of the pair takes the same path.
    __shared__ int s_skip;
    if (threadIdx.x == 0) s_skip = p.st->done;
    if (PAIR) {
        cluster_sync_all();
        if (threadIdx.x == 0 && rank != 0) {
            uint32_t v;
            asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(peer_addr(&s_skip, 0)) : "memory");
            s_skip = (int)v;
        }
        cluster_sync_all();
    } else {
        __syncthreads();
    }
    if (s_skip) return;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int a_stage_bytes = NSPLIT * p.kpanels * PANEL;  // hi (+ lo) panels
    uint8_t *A = smem;
    uint8_t *B = A + (size_t)p.a_stages * a_stage_bytes;
    Barriers *bar = (Barriers *)(B + (size_t)p.b_stages * BSTAGE);
    volatile int *abort = &bar->abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(&bar->a_full[i], 1);
            mbar_init(&bar->a_empty[i], 1);
        }
        for (int i = 0; i < p.b_stages; ++i) {
            mbar_init(&bar->b_full[i], 1);
            mbar_init(&bar->b_empty[i], 1);
        }
        for (int i = 0; i < NACC; ++i) {
            mbar_init(&bar->acc_full[i], 1);
            mbar_init(&bar->acc_empty[i], 4 * NGROUPS * NCTA);  // every epilogue warp of the pair
        }
        mbar_init(&bar->mma_done, 1);
        bar->abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        if (PAIR) {
            // both CTAs of the pair allocate together; the same columns in each
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             su32(&bar->tmem_base)),
                         "r"(TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             su32(&bar->tmem_base)),
                         "r"(TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
    }
    tc_fence_before();
    if (PAIR)
        cluster_sync_all();  // barriers initialised and TMEM allocated in both CTAs
    else
        __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = bar->tmem_base;

    // Work units: 128-row tiles, or for a pair 256-row tiles (the leader's 128 rows
    // first). A CTA's row tile of unit u is u (one CTA) or 2u + rank (a pair).
    int unit0 = (int)blockIdx.x, unit_stride = (int)gridDim.x;
    if (PAIR) {
        asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(unit0));
        asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(unit_stride));
    }
    const int n_units = PAIR ? (p.n_tiles + 1) / 2 : p.n_tiles;
    const int my_tiles = (n_units - unit0 + unit_stride - 1) / unit_stride;
    auto tile_of = [&](int lt_) { return PAIR ? (unit0 + lt_ * unit_stride) * 2 + (int)rank : unit0 + lt_ * unit_stride; };
    uint32_t smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    if (smid >= (uint32_t)kMaxSmid) smid = 0;  // (cannot happen on sm_100: ids stay below the SM count)

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            int a_issued[2] = {0, 0};
            int b_issued[MAX_B_STAGES];
            for (int i = 0; i < MAX_B_STAGES; ++i) b_issued[i] = 0;
            int bs = 0;
            uint32_t bphase = 0;  // B ring position and the parity of its current lap
            bool ok = true;
            // A pair's loads complete on the leader's full barriers, whose expected
            // byte counts (set by the leader) cover both CTAs' loads.
            auto load = [&](void *dst, const CUtensorMap *tm, uint64_t *full, int x, int y) {
                if (PAIR)
                    tma_load_2d_pair(dst, tm, peer_addr(full, 0), x, y);
                else
                    tma_load_2d(dst, tm, full, x, y);
            };
            for (int lt = 0; lt < my_tiles && ok; ++lt) {
                const int tile = tile_of(lt);
                const int as = p.a_stages == 2 ? (lt & 1) : 0;
                const int ause = p.a_stages == 2 ? (lt >> 1) : lt;
                if (!mbar_wait(&bar->a_empty[as], (ause & 1) ^ 1, abort, p.wait_cycles)) { ok = false; break; }
                if (rank == 0) mbar_expect_tx(&bar->a_full[as], (uint32_t)(NCTA * a_stage_bytes));
                uint8_t *Ab = A + (size_t)as * a_stage_bytes;
                for (int kp = 0; kp < p.kpanels; ++kp) {
                    load(Ab + (size_t)kp * PANEL, &tmXh, &bar->a_full[as], kp * KP, tile * BM);
                    if (NPROD == 3)
                        load(Ab + (size_t)(p.kpanels + kp) * PANEL, &tmXl, &bar->a_full[as], kp * KP, tile * BM);
                }
                a_issued[as]++;
                for (int j = 0; j < p.ntiles_n && ok; ++j) {
                    for (int kb = 0; kb < p.kpanels * (KP / KPB); ++kb) {
                        if (!mbar_wait(&bar->b_empty[bs], bphase ^ 1, abort, p.wait_cycles)) { ok = false; break; }
                        if (rank == 0) mbar_expect_tx(&bar->b_full[bs], NCTA * BSTAGE);
                        uint8_t *Bb = B + (size_t)bs * BSTAGE;
                        const int brow = j * BN + (int)rank * BROWS;
                        load(Bb, &tmCh, &bar->b_full[bs], kb * KPB, brow);
                        if (NPROD == 3) load(Bb + PANEL_B, &tmCl, &bar->b_full[bs], kb * KPB, brow);
                        b_issued[bs]++;
                        if (++bs == p.b_stages) {
                            bs = 0;
                            bphase ^= 1;
                        }
                    }
                }
            }
            if (!ok && rank == 0) {
                // Do not leave while bulk copies may still land in shared memory (a
                // pair's copies all complete on the leader's barriers; the peer stays
                // until the final cluster barrier, after this drain).
                for (int i = 0; i < 2; ++i)
                    if (a_issued[i]) mbar_drain(&bar->a_full[i], (a_issued[i] - 1) & 1);
                for (int i = 0; i < p.b_stages; ++i)
                    if (b_issued[i]) mbar_drain(&bar->b_full[i], (b_issued[i] - 1) & 1);
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && PAIR && rank != 0) {
            // the peer of a pair issues no MMAs; the leader's final commit reaches it
            mbar_drain(&bar->mma_done, 0);
        } else if (lane == 0) {
            // ---------------- MMA issuer ----------------
            auto commit = [](uint64_t *b) {
                if (PAIR)
                    mma_commit_pair(b);
                else
                    mma_commit(b);
            };
            long long acount = 0;
            int bs = 0;
            uint32_t bphase = 0;  // B ring position and the parity of its current lap
            bool ok = true;
            for (int lt = 0; lt < my_tiles && ok; ++lt) {
                const int as = p.a_stages == 2 ? (lt & 1) : 0;
                const int ause = p.a_stages == 2 ? (lt >> 1) : lt;
                if (!mbar_wait(&bar->a_full[as], ause & 1, abort, p.wait_cycles)) { ok = false; break; }
                tc_fence_after();
                const uint32_t a_base = su32(A + (size_t)as * a_stage_bytes);
                for (int j = 0; j < p.ntiles_n && ok; ++j, ++acount) {
                    const int slot = (int)(acount % NACC);
                    const int use = (int)(acount / NACC);
                    // the epilogue has written -h into this accumulator (first use included)
                    if (!mbar_wait(&bar->acc_empty[slot], use & 1, abort, p.wait_cycles)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t tmem_d = tmem_base + (uint32_t)(slot * BN);
                    for (int kb = 0; kb < p.kpanels * (KP / KPB); ++kb) {
                        if (!mbar_wait(&bar->b_full[bs], bphase, abort, p.wait_cycles)) { ok = false; break; }
                        tc_fence_after();
                        // A: the 64-wide panel holding this 32-wide slice, advanced to the slice
                        const int kp = kb / (KP / KPB), ka = (kb % (KP / KPB)) * (KPB * 2 / 16);
                        const uint64_t ah = sw128_desc(a_base + kp * PANEL) + ka;
                        const uint64_t al = sw128_desc(a_base + (p.kpanels + kp) * PANEL) + ka;
                        const uint64_t bh = swb_desc<KPB>(su32(B + (size_t)bs * BSTAGE));
                        const uint64_t bl = swb_desc<KPB>(su32(B + (size_t)bs * BSTAGE + PANEL_B));
                        // 16 bf16 = 32 bytes along the swizzled row = 2 in the descriptor's address field
#pragma unroll
                        for (int ks = 0; ks < KPB / 16; ++ks) {
                            if (NPROD == 1) {
                                if (PAIR)
                                    mma_bf16x1_pair(tmem_d, ah + 2 * ks, bh + 2 * ks, kIdesc);
                                else
                                    mma_bf16x1(tmem_d, ah + 2 * ks, bh + 2 * ks, kIdesc);
                            } else if (PAIR) {
                                mma_bf16x3_pair(tmem_d, ah + 2 * ks, al + 2 * ks, bh + 2 * ks, bl + 2 * ks, kIdesc);
                            } else {
                                mma_bf16x3(tmem_d, ah + 2 * ks, al + 2 * ks, bh + 2 * ks, bl + 2 * ks, kIdesc);
                            }
                        }
                        commit(&bar->b_empty[bs]);  // frees the B stage (both CTAs' halves) once these MMAs finish
                        if (++bs == p.b_stages) {
                            bs = 0;
                            bphase ^= 1;
                        }
                    }
                    if (ok) commit(&bar->acc_full[slot]);
                }
                if (ok) commit(&bar->a_empty[as]);
            }
            // All issued MMAs complete before TMEM is released (in both CTAs of a pair).
            commit(&bar->mma_done);
            mbar_drain(&bar->mma_done, 0);
        }
    } else {
        // ---------------- epilogue (warps 2.., NGROUPS groups of 4) ----------------
        const int quarter = warp & 3;          // TMEM lanes 32*quarter .. +31
        const int group = (warp - 2) >> 2;     // 0: warps 2-5, 1: warps 6-9, ...
        const int row_in_tile = quarter * 32 + lane;
        const uint32_t lane_base = tmem_base + ((uint32_t)(quarter * 32) << 16);
        long long acount = 0;
        bool ok = true;
        // An accumulator is free for the next MMAs once every epilogue warp (of both
        // CTAs of a pair: the barrier is the leader's) has drained it and refilled -h.
        auto release_acc = [&](int slot_) {
            if (PAIR)
                mbar_arrive_remote(peer_addr(&bar->acc_empty[slot_], 0));
            else
                mbar_arrive(&bar->acc_empty[slot_]);
        };
        // Accumulators start from -h (written here, one row per lane), so after the
        // MMAs they hold y = x.c - h = -score and the argmin becomes a max over y.
        // Every group drains the 32-column chunks group, group + NGROUPS, ... of each
        // accumulator (ascending columns within a group).
        for (int a0 = 0; a0 < NACC; ++a0) {  // first uses of the accumulators
            const float *hn = p.h + (size_t)(a0 % p.ntiles_n) * BN;
#pragma unroll 1
            for (int c0 = 32 * group; c0 < BN; c0 += 32 * NGROUPS) {
                __syncwarp();
                tmem_st32_from(lane_base + (uint32_t)(a0 * BN + c0), hn + c0);
            }
            tmem_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) release_acc(a0);
        }
        // Both groups pass the same number of named barriers (one per row tile),
        // also after an abort, so neither can be left waiting on the other.
        // Per-row inputs (band, prior threshold, ||x||^2) come from the row-bounds
        // pass and are loaded one row tile ahead, so no latency sits between two
        // accumulator drains.
        auto row_of = [&](int lt_) { return (int64_t)tile_of(lt_) * BM + row_in_tile; };
        float2 nb = make_float2(__int_as_float(0xff800000), 0.0f);
        float nxn = 0.0f;
        if (my_tiles > 0 && row_of(0) < p.n) {
            nb = p.rowb[row_of(0)];
            nxn = p.xnorm[row_of(0)];
        }
        for (int lt = 0; lt < my_tiles; ++lt) {
            const int64_t row = row_of(lt);
            const float thr0 = nb.x;     // prior lower bound minus the band (-inf without a prior)
            const float band_up = nb.y;  // 2e rounded up
            const double band = (double)band_up;
            const float xn = nxn;
            if (lt + 1 < my_tiles && row_of(lt + 1) < p.n) {
                nb = p.rowb[row_of(lt + 1)];
                nxn = p.xnorm[row_of(lt + 1)];
            }
            Top3 r;  // in y = -score space: b >= s >= t
            r.b = r.s = r.t = __int_as_float(0xff800000);
            r.ib = r.is = 0;
            float thr = thr0;  // values below thr cannot change the outputs
            for (int j = 0; j < p.ntiles_n; ++j, ++acount) {
                if (!ok) continue;
                const int slot = (int)(acount % NACC);
                const int use = (int)(acount / NACC);
                // every lane waits; the warp proceeds only if all lanes saw completion
                if (!__all_sync(0xffffffffu, mbar_wait(&bar->acc_full[slot], use & 1, abort, p.wait_cycles))) {
                    ok = false;
                    continue;
                }
                tc_fence_after();
                // -h of the cluster tile this accumulator holds next
                const float *hn = p.h + (size_t)((acount + NACC) % p.ntiles_n) * BN;
#pragma unroll 1
                for (int c0 = 32 * group; c0 < BN; c0 += 32 * NGROUPS) {
                    float v[32];
                    uint32_t hr[32];
                    __syncwarp();  // tcgen05.ld/st are warp-collective: reconverge after the scan
                    const uint32_t taddr = lane_base + (uint32_t)(slot * BN + c0);
                    tmem_ld32_nowait(taddr, v);
                    tmem_wait_ld_regs(v);
                    load_h32(hn + c0, hr);  // the refill's -h, in flight during the scan
                    scan_chunk(v, j * BN + c0, thr0, band_up, thr, r);
                    __syncwarp();
                    tmem_st32_regs(taddr, hr);
                }
                tmem_wait_st();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) release_acc(slot);
            }
            // back to score space (score = -y) for the merge and the outputs
            r.b = -r.b;
            r.s = -r.s;
            r.t = -r.t;
            // Groups 1.. hand their top-3 to group 0 (same rows) through the SM's
            // scratch slots for this row-tile parity, then group 0 merges.
            Top3x *xs = p.xchg + ((size_t)smid * 2 + (lt & 1)) * (NGROUPS - 1) * BM + row_in_tile;
            if (group > 0) {
                Top3x q;
                q.b = r.b;
                q.s = r.s;
                q.t = r.t;
                q.ib = r.ib;
                q.is = r.is;
                xs[(group - 1) * BM] = q;
                __threadfence_block();
            }
            named_bar_sync(1 + quarter, 32 * NGROUPS);
            if (group > 0 || !ok) continue;
#pragma unroll
            for (int g = 1; g < NGROUPS; ++g) {
                const Top3x q = xs[(g - 1) * BM];
                Top3 o;
                o.b = q.b;
                o.s = q.s;
                o.t = q.t;
                o.ib = q.ib;
                o.is = q.is;
                r = top3_merge(r, o);
            }
            if (row < p.n) {
                p.labels[row] = r.ib;
                p.d2[row] = 2.0f * r.b + xn;
                if (p.queue) {
                    // (a row for which no cluster passed the filters -- impossible while
                    // the prior bound holds -- goes to the full FP64 rescan)
                    const bool none = !(r.b < __int_as_float(0x7f800000));
                    if ((double)r.s - (double)r.b <= band || none)
                        enqueue_recheck(p.queue, p.n, p.st, (int)row, r.ib, r.is,
                                        (double)r.t - (double)r.b <= band || none);
                }
            }
        }
    }

    __syncwarp();
    tc_fence_before();
    if (PAIR)
        cluster_sync_all();  // neither CTA leaves (or frees TMEM) while the pair still works on it
    else
        __syncthreads();
    if (bar->abort && threadIdx.x == 0) {
        p.st->error = KMB_ETIMEDOUT;
        p.st->done = 1;
    }
    if (warp == 1) {
        tc_fence_after();
        if (PAIR)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS)
                         : "memory");
        else
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS)
                         : "memory");
    }
}

// Per row, ahead of the tensor-core pass (after the centroid prep has computed
// max ||c||): the recheck band 2e rounded up, and the prior threshold.
//   e = 1.0625 ((3.03 u_b^2 + 2 * 3 dpad * 2u) ||x|| cmax + 2u (cmax^2 / 2 + ||x|| cmax))
// (the per-score bound of the kernel header). The prior: with l the previous
// label and D_old^2 <= d2_prev + (its rounding bound, e of the previous
// centroids), the triangle inequality gives ||x - c_new[l]|| <= D_old +
// ||c_new[l] - c_old[l]||, hence the row's computed best y (= -score) is at
// least 0.5 (||x||^2 - (D_old + delta_l)^2) - e. Any cluster that can be the
// best or lie inside the band of the best has y >= that bound - 2e, so the
// epilogue skips values below thr0 = bound - 2e (rounded down). Without a prior,
// or for a row without a valid previous label, thr0 = -inf.
__global__ void row_bounds_kernel(int64_t n, const float *__restrict__ xnorm, const int32_t *__restrict__ labels,
                                  const float *__restrict__ d2, const double *__restrict__ shift_part,
                                  const double *__restrict__ cnorm_max, const double *__restrict__ cnorm_max_prev,
                                  int dpad, int k, int prior, int products, float2 *__restrict__ out,
                                  const LoopState *st) {
    if (st && st->done) return;
    const double u = 5.9604644775390625e-8;  // 2^-24
    const double ub = 3.90625e-3;             // 2^-8
    const double ub2 = 1.52587890625e-5;      // 2^-16
    const double cmax = *cnorm_max;
    const double cmax_prev = prior ? *cnorm_max_prev : 0.0;
    // split form: the dropped xl.cl term and the bf16 rounding of the lo parts;
    // single product: |x.c - bf16(x).bf16(c)| <= (2 u_b + u_b^2) sum |x_t c_t|
    const double split = products == 3 ? 3.03 * ub2 : 2.0 * ub + ub2;
    const double acc = split + 2.0 * products * dpad * 2.0 * u;
    for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < n;
         row += (int64_t)gridDim.x * blockDim.x) {
        const float xn = xnorm[row];
        const double xl = sqrt(fmax((double)xn, 0.0));
        const double xc = xl * cmax;
        const double e = 1.0625 * (acc * xc + 2.0 * u * (0.5 * cmax * cmax + xc));
        float thr0 = __int_as_float(0xff800000);
        const int l = prior ? labels[row] : -1;
        if (l >= 0 && l < k) {
            const double d2p = (double)d2[row];
            const double xcp = xl * cmax_prev;
            const double e_prev = 1.0625 * (acc * xcp + 2.0 * u * (0.5 * cmax_prev * cmax_prev + xcp));
            const double dsq = fmax(d2p, 0.0) + 2.0 * e_prev + 2.0 * u * (fabs(d2p) + (double)xn);
            const double rad = sqrt(dsq) + sqrt(shift_part[l]) * (1.0 + 1e-12);
            const double r2 = rad * rad;
            const double lb = 0.5 * ((double)xn * (1.0 - 2.0 * u) - r2) - 3.0 * e -
                              9.5367431640625e-7 * ((double)xn + r2);  // 2^-20 slack for this arithmetic
            if (lb >= -3.0e38) thr0 = __double2float_rd(lb);          // also rejects NaN
        }
        out[row] = make_float2(thr0, __double2float_ru(2.0 * e));
    }
}

// x -> (bf16(x), bf16(x - bf16(x))) into [rows][dpad] panels, zero padding,
// and ||x||^2 with the summation order of row_norms_kernel. One warp per row,
// grid-stride over rows; every element of X is read once.
__global__ void split_rows_kernel(const float *__restrict__ src, int64_t rows, int d, int dpad,
                                  __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                                  float *__restrict__ xnorm) {
    // lo == nullptr: the single-product form reads the hi panels only
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += warps) {
        const float *x = src + r * d;
        double s = 0.0;
        for (int t = lane; t < dpad; t += 32) {
            const float v = t < d ? x[t] : 0.0f;
            if (t < d) s += (double)v * (double)v;
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            hi[r * dpad + t] = h;
            if (lo) lo[r * dpad + t] = __float2bfloat16_rn(v - __bfloat162float(h));
        }
        for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
        if (lane == 0) xnorm[r] = (float)s;
    }
}

// Per-iteration centroid prep for the tensor-core form: Chi/Clo [kpad][dpad],
// -h = -0.5||c||^2 (FP32 from a double sum, -inf padding), max ||c||.
__global__ void prep_centroids_tc_kernel(const float *__restrict__ C, int k, int d, int dpad, int kpad,
                                         __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                                         float *__restrict__ h, double *__restrict__ cnorm_max, const LoopState *st) {
    if (st && st->done) return;
    __shared__ double red[32];
    const int j = blockIdx.x;
    double s = 0.0;
    for (int t = threadIdx.x; t < dpad; t += blockDim.x) {
        const float x = (j < k && t < d) ? C[(int64_t)j * d + t] : 0.0f;
        const __nv_bfloat16 b = __float2bfloat16_rn(x);
        hi[(int64_t)j * dpad + t] = b;
        lo[(int64_t)j * dpad + t] = __float2bfloat16_rn(x - __bfloat162float(b));
        s += (double)x * (double)x;
    }
    for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        h[j] = (j < k) ? (float)(-0.5 * tot) : __int_as_float(0xff800000);  // -h, -inf padding
        if (j < k)
            atomicMax(reinterpret_cast<unsigned long long *>(cnorm_max),
                      (unsigned long long)__double_as_longlong(sqrt(tot)));
    }
}

__global__ void reset_cmax_kernel(double *p, double *prev, const LoopState *st) {
    if (st && st->done) return;
    *prev = *p;
    *p = 0.0;
}

}  // namespace tc

// Hand-off slots are indexed by %smid (a CTA needs a whole SM's shared memory,
// so no two CTAs of this kernel share an SM at a time); ids are below kMaxSmid.
size_t tc_xchg_bytes() { return (size_t)tc::kMaxSmid * 2 * (tc::NGROUPS - 1) * tc::BM * sizeof(tc::Top3x); }

int64_t tc_dpad(int64_t d) { return (d + tc::KP - 1) / tc::KP * tc::KP; }
// Cluster tile (UMMA N) for k clusters: 256 unless its padding costs more than
// the wider tile gains. Per padded column the 256-wide tile ran 1.16x faster than
// the 128-wide one (20M x 128, k = 1152: 17.25 ms padded to 1280 against 17.86 ms
// at 1152), so 128 is kept where padding to 256 adds more than 16 %.
int tc_tile_n(int64_t k) {
    const int64_t k128 = (k + 127) / 128 * 128, k256 = (k + 255) / 256 * 256;
    return k256 * 100 <= k128 * 116 ? 256 : 128;
}
int64_t tc_kpad(int64_t k) {
    const int64_t bn = tc_tile_n(k);
    return (k + bn - 1) / bn * bn;
}
bool tc_supported(int64_t d) { return tc_dpad(d) <= 256; }

void launch_split_rows(const float *X, int64_t rows, int64_t d, void *hi, void *lo, float *xnorm, int num_sms,
                       cudaStream_t s) {
    if (rows == 0) return;
    const int64_t dpad = tc_dpad(d);
    const int blocks = (int)std::min<int64_t>((rows * 32 + 255) / 256, (int64_t)num_sms * 16);
    tc::split_rows_kernel<<<blocks, 256, 0, s>>>(X, rows, (int)d, (int)dpad, (__nv_bfloat16 *)hi, (__nv_bfloat16 *)lo,
                                                 xnorm);
    KMB_LAUNCHED();
}

void launch_prep_centroids_tc(const float *C, int64_t k, int64_t d, void *Chi, void *Clo, float *h, double *cnorm_max,
                              double *cnorm_max_prev, const LoopState *st, cudaStream_t s) {
    const int64_t dpad = tc_dpad(d), kpad = tc_kpad(k);
    tc::reset_cmax_kernel<<<1, 1, 0, s>>>(cnorm_max, cnorm_max_prev, st);
    KMB_LAUNCHED();
    tc::prep_centroids_tc_kernel<<<(unsigned)kpad, 128, 0, s>>>(C, (int)k, (int)d, (int)dpad, (int)kpad,
                                                                 (__nv_bfloat16 *)Chi, (__nv_bfloat16 *)Clo, h,
                                                                 cnorm_max, st);
    KMB_LAUNCHED();
}

// cuTensorMapEncodeTiled through the runtime's driver entry point, so the library
// does not link libcuda directly (it loads on hosts without a driver).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

bool encode_tensor_map_2d(CUtensorMap *m, CUtensorMapDataType type, const void *base, uint64_t inner, uint64_t outer,
                          uint64_t row_bytes, uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle swizzle) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
    const cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
    const cuuint32_t box[2] = {box_inner, box_outer};
    const cuuint32_t estr[2] = {1u, 1u};
    return enc(m, type, 2, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Row panels: the split rows (128 rows x 64 bf16, SWIZZLE_128B) or the split
// centroids (256 clusters x 32 bf16, SWIZZLE_64B).
// (A CTA pair's centroid box is half the cluster tile: each CTA loads its half.)
static bool encode_map(CUtensorMap *m, const void *base, int64_t rows, int64_t dpad, bool centroids, int bn = 0,
                       bool pair = false) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)dpad, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)dpad * 2};
    const int kpb = tc::kpb_of(bn, pair);
    const cuuint32_t box[2] = {centroids ? (cuuint32_t)kpb : (cuuint32_t)tc::KP,
                               centroids ? (cuuint32_t)tc::b_rows_of(bn, pair) : (cuuint32_t)tc::BM};
    const cuuint32_t estr[2] = {1u, 1u};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE,
               (centroids && kpb == 32) ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Single CTAs (M = 128) unless the environment variable KMB_TC_PAIR=1 asks for
// CTA pairs (tcgen05 cta_group::2, M = 256); read at every launch. With the three
// split products per k-step the pairs measured slower (14.9 against 14.1 ms per
// 20M-row launch at d = 128, k = 1024): halving each CTA's centroid-panel bytes
// did not pay for the pair's cross-CTA barrier traffic.
static bool use_cta_pairs() {
    const char *e = getenv("KMB_TC_PAIR");
    return e && e[0] == '1';
}

// Launches the tensor-core assignment. Returns KMB_OK, or an error status when
// the shape is outside the kernel's limits or tensor maps cannot be encoded.
int launch_assign_tc(const void *Xhi, const void *Xlo, int64_t n, int64_t d, const void *Chi, const void *Clo,
                     const float *h, int64_t k, const float *xnorm, const double *cnorm_max, int32_t *labels,
                     float *d2, RecheckEntry *queue, LoopState *st, int num_sms, void *xchg, bool prior,
                     const double *shift_part, const double *cnorm_max_prev, void *rowb, int products,
                     cudaStream_t s) {
    if (products != 1 && products != 3) return KMB_EINVAL;
    const int nsplit = products == 3 ? 2 : 1;
    const int64_t dpad = tc_dpad(d), kpad = tc_kpad(k);
    if ((prior && (!shift_part || !cnorm_max_prev)) || !rowb) return KMB_EINVAL;
    if (dpad > 256) return KMB_EUNSUPPORTED;
    if (n == 0) return KMB_OK;
    // Shared memory plan: A stages (hi+lo panels of the row tile), B ring.
    int optin = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int kpanels = (int)(dpad / tc::KP);
    const int a_stage = nsplit * kpanels * tc::PANEL;
    const int fixed = 1024 + (int)sizeof(tc::Barriers) + 64;
    const int bn = tc_tile_n(k);  // cluster tile (UMMA N); kpad is a multiple of it
    const bool pair = use_cta_pairs();
    const int panel_b = tc::panel_b_bytes(bn, pair);
    int a_stages = (2 * a_stage + 3 * nsplit * panel_b + fixed <= optin) ? 2 : 1;
    int b_stages = (optin - fixed - a_stages * a_stage) / (nsplit * panel_b);
    b_stages = std::min(b_stages, tc::MAX_B_STAGES);
    if (b_stages < 2) return KMB_EUNSUPPORTED;
    // More than half of an SM's shared memory: one CTA per SM, which the
    // %smid-indexed hand-off slots rely on.
    const size_t smem = std::max<size_t>((size_t)a_stages * a_stage + (size_t)b_stages * nsplit * panel_b + fixed,
                                         (size_t)optin / 2 + 4096);

    CUtensorMap mXh, mXl, mCh, mCl;
    // (the single-product form never loads the lo panels: their maps alias the hi ones)
    if (products == 1) {
        Xlo = Xhi;
        Clo = Chi;
    }
    if (!encode_map(&mXh, Xhi, n, dpad, false) || !encode_map(&mXl, Xlo, n, dpad, false) ||
        !encode_map(&mCh, Chi, kpad, dpad, true, bn, pair) || !encode_map(&mCl, Clo, kpad, dpad, true, bn, pair))
        return KMB_ECUDA;
    tc::Params p;
    p.n = n;
    p.d = (int)d;
    p.dpad = (int)dpad;
    p.k = (int)k;
    p.kpad = (int)kpad;
    p.n_tiles = (int)((n + tc::BM - 1) / tc::BM);
    p.kpanels = kpanels;
    p.ntiles_n = (int)(kpad / bn);
    p.a_stages = a_stages;
    p.b_stages = b_stages;
    p.h = h;
    p.xnorm = xnorm;
    p.rowb = (const float2 *)rowb;
    p.labels = labels;
    p.d2 = d2;
    p.queue = queue;
    p.st = st;
    p.xchg = (tc::Top3x *)xchg;
    // KMB_TC_WAIT_LIMIT_CYCLES shortens the pipeline waits' limit: a test makes them
    // run out and checks that the launch reports KMB_ETIMEDOUT and leaves the
    // context usable.
    p.wait_cycles = tc::kTimeoutCycles;
    if (const char *e = getenv("KMB_TC_WAIT_LIMIT_CYCLES")) {
        const long long v = atoll(e);
        if (v > 0 && v < tc::kTimeoutCycles) p.wait_cycles = v;
    }
    {
        const int bs = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
        tc::row_bounds_kernel<<<bs, 256, 0, s>>>(n, xnorm, labels, d2, shift_part, cnorm_max, cnorm_max_prev, (int)dpad,
                                                 (int)k, prior ? 1 : 0, products, (float2 *)rowb, st);
        KMB_LAUNCHED();
    }
    if (!pair) {
        auto kern = products == 1 ? (bn == 256 ? tc::assign_tc_kernel<256, false, 1> : tc::assign_tc_kernel<128, false, 1>)
                                  : (bn == 256 ? tc::assign_tc_kernel<256, false, 3> : tc::assign_tc_kernel<128, false, 3>);
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return KMB_ECUDA;
        // num_sms < 0: one CTA per 128-row tile (no persistence), so that other
        // streams' launches interleave with this one at tile granularity
        const int grid = num_sms < 0 ? p.n_tiles : (int)std::min<int64_t>(num_sms, p.n_tiles);
        kern<<<grid, tc::NTHREADS, smem, s>>>(mXh, mXl, mCh, mCl, p);
        KMB_LAUNCHED();
        return cudaGetLastError() == cudaSuccess ? KMB_OK : KMB_ECUDA;
    }
    // CTA pairs: clusters of two CTAs, one 256-row unit per cluster at a time.
    auto kern = products == 1 ? (bn == 256 ? tc::assign_tc_kernel<256, true, 1> : tc::assign_tc_kernel<128, true, 1>)
                              : (bn == 256 ? tc::assign_tc_kernel<256, true, 3> : tc::assign_tc_kernel<128, true, 3>);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return KMB_ECUDA;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(tc::NTHREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int64_t n_units = (p.n_tiles + 1) / 2;
    int64_t clusters = n_units;
    if (num_sms >= 0) {
        // persistent: as many pairs as fit on the device at once (and within the SM cap)
        static int cached_dev = -1, cached_bn = 0, cached_active = 0;
        static size_t cached_smem = 0;
        if (cached_dev != dev || cached_bn != bn || cached_smem != smem) {
            int active = 0;
            cfg.gridDim = dim3(2 * 74, 1, 1);
            if (cudaOccupancyMaxActiveClusters(&active, kern, &cfg) != cudaSuccess || active <= 0) {
                cudaGetLastError();
                active = num_sms > 0 ? num_sms / 2 : 74;
            }
            cached_dev = dev;
            cached_bn = bn;
            cached_smem = smem;
            cached_active = active;
        }
        clusters = std::min<int64_t>(clusters, cached_active);
        if (num_sms > 0) clusters = std::min<int64_t>(clusters, std::max(1, num_sms / 2));
    }
    cfg.gridDim = dim3((unsigned)(2 * clusters), 1, 1);
    if (cudaLaunchKernelEx(&cfg, kern, mXh, mXl, mCh, mCl, p) != cudaSuccess) return KMB_ECUDA;
    KMB_LAUNCHED();
    return cudaGetLastError() == cudaSuccess ? KMB_OK : KMB_ECUDA;
}

}  // namespace kmb
