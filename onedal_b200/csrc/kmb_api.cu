// C ABI of the B200 k-means Lloyd path: context, workspace and the host driver
// of the Lloyd loop (declared in include/onedal_b200_kmeans.h).
//
// Host driver semantics follow DAAL's KMeansBatchKernel::compute
// (cpp/daal/src/algorithms/kmeans/kmeans_lloyd_batch_impl.i:48-242):
//   for it < T: assign under C, update (sums, reseed, shift), stop if shift <= eps
//   then responses against the final centroids + exact objective.
// The whole loop is enqueued on one stream; a device-side LoopState carries the
// convergence flag so later iterations become no-ops, and the host only reads
// it back every few iterations.
#include "kmb_internal.cuh"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <vector>

struct kmb_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    kmb::Workspace ws;
    std::string last_error;
    kmb::LoopState *h_state = nullptr;  // pinned mirror of the device states
    int num_sms = 148;
    bool tc_per_tile = false;  // tensor-core assignment: one CTA per row tile instead of persistent CTAs
    // The last assignment pass that queued near-tie rows (kmb_context_recheck_rows):
    // its row count (the queue's capacity) and its loop state.
    int64_t queue_rows = 0;
    const kmb::LoopState *queue_state = nullptr;
    // BF16 products per k-step of the current call's tensor-core form (3: split, 1: single)
    int tc_products = 3;
    // kernel timing (kmb_context_set_kernel_timing)
    bool timing = false;
    int64_t launches_at_enable = 0;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_used[5];

    cudaEvent_t take_event() {
        if (!ev_pool.empty()) {
            cudaEvent_t e = ev_pool.back();
            ev_pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void recycle_events() {
        for (auto &v : ev_used) {
            for (auto &pr : v) {
                ev_pool.push_back(pr.first);
                ev_pool.push_back(pr.second);
            }
            v.clear();
        }
    }
};

// RAII: records a start/stop event pair around one kernel launch when timing is on.
struct KernelTimer {
    kmb_context *ctx;
    int which;
    cudaEvent_t a = nullptr, b = nullptr;
    KernelTimer(kmb_context *c, int w) : ctx(c), which(w) {
        if (ctx->timing) {
            a = ctx->take_event();
            b = ctx->take_event();
            cudaEventRecord(a, ctx->stream);
        }
    }
    ~KernelTimer() {
        if (ctx->timing) {
            cudaEventRecord(b, ctx->stream);
            ctx->ev_used[which].emplace_back(a, b);
        }
    }
};

namespace kmb {

int64_t &launch_count() {
    static thread_local int64_t count = 0;
    return count;
}

// Host-side fault injection: with KMB_FAIL_ALLOC=1 in the environment every
// workspace growth reports an allocation failure (without calling the
// allocator), so a test can check that the failure surfaces as KMB_ENOMEM and,
// through a dispatcher, as the reference's host_bad_alloc.
static bool alloc_failure_injected() {
    const char *e = getenv("KMB_FAIL_ALLOC");
    return e && e[0] == '1';
}

// The library's stream-ordered allocations (context workspaces, the batched
// form's arenas, the serving loop's arenas) come from a memory pool of the library
// (one per device, created on first use) that keeps freed memory for the next
// allocation instead of returning it to the driver at every synchronisation, as
// the device's default pool does unless told otherwise: a fresh mapping of a large
// block stalled the device for tens of milliseconds. The pool holds at most the
// largest set of buffers in use at one time until the process exits.
static std::mutex g_pool_mu;
static std::map<int, cudaMemPool_t> g_pools;

cudaMemPool_t library_pool(int dev) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) return it->second;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        pool = nullptr;
    } else {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    g_pools[dev] = pool;
    return pool;
}

// From the library's pool when it exists, else the device's default pool.
cudaError_t pool_alloc(void **p, size_t bytes, int dev, cudaStream_t s) {
    cudaMemPool_t pool = library_pool(dev);
    return pool ? cudaMallocFromPoolAsync(p, bytes, pool, s) : cudaMallocAsync(p, bytes, s);
}

bool Workspace::ensure(DevBuf &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return true;
    if (alloc_failure_injected()) return false;
    if (b.ptr) cudaFreeAsync(b.ptr, stream);
    b.ptr = nullptr;
    b.bytes = 0;
    // round up to 2 MiB to limit reallocations
    const size_t rounded = (bytes + (size_t(2) << 20) - 1) / (size_t(2) << 20) * (size_t(2) << 20);
    if (pool_alloc(&b.ptr, rounded, device, stream) != cudaSuccess) {
        cudaGetLastError();
        b.ptr = nullptr;
        return false;
    }
    b.bytes = rounded;
    return true;
}

void Workspace::release() {
    DevBuf *all[] = {&X, &C0, &Cout, &labels, &d2, &xnorm, &Ccur, &Cnew, &Ct, &h, &queue, &H, &Gs,
                     &counts, &offsets, &piece_base, &perm, &records, &shift_part, &shift_tiles, &empty_flag,
                     &empty_ids,
                     &sel_hist, &sel_state, &cand, &obj_part, &scalars, &state, &Xhi, &Xlo, &Chi, &Clo, &tcx, &rowb, &pp_acc, &pp_rand,
                     &pp_state, &pp_flags, &csr_vals, &csr_cols64, &csr_rowptr64, &csr_cols, &csr_rowptr,
                     &csr_bad, &csr_cnorm, &ex_acc, &ex_cnt, &ex_prev, &ex_colexp, &ex_records};
    for (DevBuf *b : all) {
        if (b->ptr) cudaFreeAsync(b->ptr, stream);
        b->ptr = nullptr;
        b->bytes = 0;
    }
}

}  // namespace kmb

namespace {

using kmb::LoopState;
using kmb::RecheckEntry;

int fail(kmb_context *ctx, int status, const char *fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return status;
}

int cuda_fail(kmb_context *ctx, cudaError_t e, const char *where) {
    return fail(ctx, KMB_ECUDA, "%s: %s", where, cudaGetErrorString(e));
}

#define KMB_CUDA(call)                                                    \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);          \
    } while (0)

constexpr int64_t kBN = 128;  // cluster tile of the plain kernel
constexpr int64_t kBK = 8;

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Profiling, gated like the reference's profiler on ONEDAL_VERBOSE
// (cpp/daal/src/services/service_profiler.h:141-151): at level >= 1 the hot-path
// phases are NVTX ranges named after the reference's profiler tasks
// (kmeans_lloyd_batch_impl.i:122,134,145,190) and every train / infer call logs
// one line (shape, form, iterations, status, wall time) to stderr. Read once.
int verbose_level() {
    static const int level = [] {
        const char *e = getenv("ONEDAL_VERBOSE");
        return e ? atoi(e) : 0;
    }();
    return level;
}

struct ProfRange {
    bool on;
    explicit ProfRange(const char *name) : on(verbose_level() >= 1) {
        if (on) nvtxRangePushA(name);
    }
    ~ProfRange() {
        if (on) nvtxRangePop();
    }
};

struct CallLog {
    const char *what;
    int64_t n, d, k;
    int form;
    const int64_t *iterations;
    const int *rc;
    std::chrono::steady_clock::time_point t0;
    CallLog(const char *w, int64_t n_, int64_t d_, int64_t k_, int f, const int64_t *it, const int *rc_)
        : what(w), n(n_), d(d_), k(k_), form(f), iterations(it), rc(rc_), t0(std::chrono::steady_clock::now()) {}
    ~CallLog() {
        if (verbose_level() < 1) return;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        fprintf(stderr, "onedal_b200: %s n=%lld d=%lld k=%lld form=%d iterations=%lld status=%d wall=%.3f ms\n", what,
                (long long)n, (long long)d, (long long)k, form, iterations ? (long long)*iterations : 0LL, *rc, ms);
    }
};

// Buffers shared by train/infer/step. Returns KMB_OK or KMB_ENOMEM.
template <typename F>
int ensure_common(kmb_context *ctx, int64_t n, int64_t d, int64_t k, bool recheck, bool tc = false) {
    kmb::Workspace &ws = ctx->ws;
    const int64_t kpad = round_up(k, kBN), dpad = round_up(d, kBK);
    bool ok = true;
    if (tc) {
        const int64_t tdp = kmb::tc_dpad(d), tkp = kmb::tc_kpad(k);
        ok &= ws.ensure(ws.Xhi, sizeof(uint16_t) * n * tdp);
        if (ctx->tc_products == 3) ok &= ws.ensure(ws.Xlo, sizeof(uint16_t) * n * tdp);
        ok &= ws.ensure(ws.Chi, sizeof(uint16_t) * tkp * tdp);
        ok &= ws.ensure(ws.Clo, sizeof(uint16_t) * tkp * tdp);
        ok &= ws.ensure(ws.h, sizeof(float) * tkp);
        ok &= ws.ensure(ws.tcx, kmb::tc_xchg_bytes());
        ok &= ws.ensure(ws.rowb, sizeof(float) * 2 * n);
    }
    ok &= ws.ensure(ws.labels, sizeof(int32_t) * n);
    ok &= ws.ensure(ws.d2, sizeof(F) * n);
    ok &= ws.ensure(ws.xnorm, sizeof(F) * n);
    ok &= ws.ensure(ws.Ccur, sizeof(F) * k * d);
    ok &= ws.ensure(ws.Cnew, sizeof(F) * k * d);
    ok &= ws.ensure(ws.Ct, sizeof(F) * kpad * dpad);
    ok &= ws.ensure(ws.h, sizeof(F) * kpad);
    ok &= ws.ensure(ws.scalars, sizeof(kmb::DevScalars));
    ok &= ws.ensure(ws.state, sizeof(LoopState) * 2);
    if (recheck) ok &= ws.ensure(ws.queue, sizeof(RecheckEntry) * n);
    if (!ok) return fail(ctx, KMB_ENOMEM, "device allocation failed (n=%lld d=%lld k=%lld)", (long long)n,
                         (long long)d, (long long)k);
    return KMB_OK;
}

__global__ void reset_iteration_kernel(LoopState *st) {
    if (st->done) return;
    st->n_recheck = 0;
    st->n_changed = 0;
    st->n_full = 0;
}

__global__ void account_recheck_kernel(LoopState *st) {
    if (st->done) return;
    st->rechecked_total += st->n_recheck + st->n_full;
    st->full_total += st->n_full;
}

// One assignment pass of the plain form (+ optional FP64 recheck) under C.
template <typename F>
int assign_pass_tc(kmb_context *ctx, const F *X, int64_t n, int64_t d, const F *C, int64_t k, int32_t *labels,
                   F *d2, LoopState *st, bool prior) {
    return KMB_EUNSUPPORTED;  // float64 data has no tensor-core form
}

template <>
int assign_pass_tc<float>(kmb_context *ctx, const float *X, int64_t n, int64_t d, const float *C, int64_t k,
                          int32_t *labels, float *d2, LoopState *st, bool prior) {
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;
    reset_iteration_kernel<<<1, 1, 0, s>>>(st);
    KMB_LAUNCHED();
    kmb::launch_prep_centroids_tc(C, k, d, ws.Chi.ptr, ws.Clo.ptr, (float *)ws.h.ptr, &sc->cnorm_max,
                                  &sc->cnorm_max_prev, st, s);
    int rc;
    {
        KernelTimer timer(ctx, 1);
        rc = kmb::launch_assign_tc(ws.Xhi.ptr, ctx->tc_products == 3 ? ws.Xlo.ptr : ws.Xhi.ptr, n, d, ws.Chi.ptr,
                                   ws.Clo.ptr, (const float *)ws.h.ptr, k,
                                   (const float *)ws.xnorm.ptr, &sc->cnorm_max, labels, d2,
                                   (RecheckEntry *)ws.queue.ptr, st, ctx->tc_per_tile ? -1 : ctx->num_sms,
                                   ws.tcx.ptr, prior,
                                   (const double *)ws.shift_part.ptr, &sc->cnorm_max_prev, ws.rowb.ptr,
                                   ctx->tc_products, s);
    }
    if (rc != KMB_OK) return fail(ctx, rc, "tensor-core assignment launch failed (d=%lld)", (long long)d);
    {
        KernelTimer timer(ctx, 4);
        kmb::launch_recheck<float>(X, n, d, C, k, (const RecheckEntry *)ws.queue.ptr, labels, d2,
                                   (const float *)ws.xnorm.ptr, st, ctx->num_sms, s);
    }
    account_recheck_kernel<<<1, 1, 0, s>>>(st);
    KMB_LAUNCHED();
    ctx->queue_rows = n;
    ctx->queue_state = st;
    return KMB_OK;
}

template <typename F>
int assign_pass(kmb_context *ctx, const F *X, int64_t n, int64_t d, const F *C, int64_t k, bool recheck,
                int32_t *labels, F *d2, LoopState *st, bool tc = false, bool prior = false) {
    ProfRange range("addNTToTaskThreaded");
    if (tc) return assign_pass_tc<F>(ctx, X, n, d, C, k, labels, d2, st, prior);
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    const int64_t kpad = round_up(k, kBN);
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;
    reset_iteration_kernel<<<1, 1, 0, s>>>(st);
    KMB_LAUNCHED();
    kmb::launch_prep_centroids<F>(C, k, d, kpad, (F *)ws.Ct.ptr, (F *)ws.h.ptr, &sc->cnorm_max, st, s);
    {
        KernelTimer timer(ctx, 0);
        kmb::launch_assign_plain<F>(X, n, d, (const F *)ws.Ct.ptr, (const F *)ws.h.ptr, k, kpad,
                                    (const F *)ws.xnorm.ptr, &sc->cnorm_max, labels, d2,
                                    recheck ? (RecheckEntry *)ws.queue.ptr : nullptr, st, s);
    }
    if (recheck) {
        KernelTimer timer(ctx, 4);
        kmb::launch_recheck<F>(X, n, d, C, k, (const RecheckEntry *)ws.queue.ptr, labels, d2,
                               (const F *)ws.xnorm.ptr, st, ctx->num_sms, s);
        account_recheck_kernel<<<1, 1, 0, s>>>(st);
        KMB_LAUNCHED();
        ctx->queue_rows = n;
        ctx->queue_state = st;
    }
    return KMB_OK;
}

// Row ids of the recheck queue (front: two-candidate entries, back: full rescans)
// into out[0 .. min(total, cap)).
__global__ void gather_queue_rows_kernel(const RecheckEntry *queue, int64_t qcap, const LoopState *st, int32_t *out,
                                         int64_t cap) {
    const int64_t front = st->n_recheck, back = st->n_full;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < front + back && i < cap;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = i < front ? queue[i].row : queue[qcap - 1 - (i - front)].row;
}

// Row norms for the pass, plus -- for the tensor-core form -- the BF16 hi/lo
// panels it reads, both from one read of X (once per call).
template <typename F>
void prepare_rows(kmb_context *ctx, const F *X, int64_t n, int64_t d, bool tc) {
    kmb::launch_row_norms<F>(X, n, d, (F *)ctx->ws.xnorm.ptr, ctx->stream);
}
template <>
void prepare_rows<float>(kmb_context *ctx, const float *X, int64_t n, int64_t d, bool tc) {
    if (tc)
        kmb::launch_split_rows(X, n, d, ctx->ws.Xhi.ptr, ctx->tc_products == 3 ? ctx->ws.Xlo.ptr : nullptr,
                               (float *)ctx->ws.xnorm.ptr, ctx->num_sms,
                               ctx->stream);
    else
        kmb::launch_row_norms<float>(X, n, d, (float *)ctx->ws.xnorm.ptr, ctx->stream);
}

template <typename F>
int upload(kmb_context *ctx, kmb::DevBuf &buf, const void *src, size_t bytes, const F **out) {
    if (!ctx->ws.ensure(buf, bytes)) return fail(ctx, KMB_ENOMEM, "device allocation of %zu bytes failed", bytes);
    // in pieces, so that other streams' small copies interleave with a large upload
    const size_t piece = (size_t)8 << 20;
    for (size_t off = 0; off < bytes; off += piece)
        KMB_CUDA(cudaMemcpyAsync((char *)buf.ptr + off, (const char *)src + off, std::min(piece, bytes - off),
                                 cudaMemcpyHostToDevice, ctx->stream));
    *out = (const F *)buf.ptr;
    return KMB_OK;
}

// The tensor-core forms and their BF16 products per k-step.
bool is_tc_form(int form) { return form == KMB_FORM_BF16X3 || form == KMB_FORM_BF16; }
int form_products(int form) { return form == KMB_FORM_BF16 ? 1 : 3; }

int check_form(kmb_context *ctx, int dtype, int form) {
    if (form != KMB_FORM_PLAIN && form != KMB_FORM_BF16X3 && form != KMB_FORM_BF16 && form != KMB_FORM_AUTO)
        return fail(ctx, KMB_EINVAL, "unknown form %d", form);
    if (is_tc_form(form) && dtype != KMB_F32)
        return fail(ctx, KMB_EINVAL, "the BF16 tensor-core forms take float32 data");
    return KMB_OK;
}

// KMB_FORM_AUTO -> the concrete form for this shape.
int resolve_form(int dtype, int form, int64_t n, int64_t k, int64_t d) {
    if (form != KMB_FORM_AUTO) return form;
    if (dtype != KMB_F32 || !kmb::tc_supported(d)) return KMB_FORM_PLAIN;
    // kpad: k rounded up to 128 clusters, dpad: d rounded up to 64 features
    const double macs = (double)n * (double)round_up(k, 128) * (double)kmb::tc_dpad(d);
    return macs >= (double)KMB_AUTO_TC_MACS ? KMB_FORM_BF16X3 : KMB_FORM_PLAIN;
}

void init_state(LoopState &h, double eps) {
    std::memset(&h, 0, sizeof(h));
    h.eps = eps;
}

// The update of one Lloyd iteration: float rows take the exact update (integer
// cluster sums, moved rows only once few rows move), double rows the FP64 one.
template <typename F>
int prepare_update(kmb_context *ctx, const F *X, int64_t n, int64_t d, int64_t k, LoopState *st) {
    return KMB_OK;
}
template <>
int prepare_update<float>(kmb_context *ctx, const float *X, int64_t n, int64_t d, int64_t k, LoopState *st) {
    if (!kmb::ensure_exact_buffers(ctx->ws, n, k, d)) return fail(ctx, KMB_ENOMEM, "exact update buffers");
    kmb::prepare_exact_update(X, n, d, ctx->ws, st, ctx->stream);
    return KMB_OK;
}
template <typename F>
void update_pass(const F *X, const kmb::UpdatePlan &plan, int32_t *labels, F *d2, F *C_old, F *C_new,
                 kmb::Workspace &ws, LoopState *st, bool commit, cudaStream_t s, bool tc) {
    kmb::launch_update<F>(X, plan, labels, d2, C_old, C_new, ws, st, commit, s, nullptr, tc ? d2 : nullptr);
}
template <>
void update_pass<float>(const float *X, const kmb::UpdatePlan &plan, int32_t *labels, float *d2, float *C_old,
                        float *C_new, kmb::Workspace &ws, LoopState *st, bool commit, cudaStream_t s, bool tc) {
    kmb::launch_update_exact(X, plan, labels, d2, C_old, C_new, ws, st, commit, s, tc ? d2 : nullptr);
}

// The Lloyd loop on device-resident X and centroids C (updated in place).
// The host peeks at the device convergence flag every few iterations.
template <typename F>
int run_loop(kmb_context *ctx, const F *X, int64_t n, int64_t d, F *C, const kmb_params *p,
             const kmb::UpdatePlan &plan, int32_t *labels, bool recheck) {
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    const int64_t k = p->cluster_count;
    F *Cnew = (F *)ws.Cnew.ptr;
    F *d2 = (F *)ws.d2.ptr;
    LoopState *st = (LoopState *)ws.state.ptr;
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;
    init_state(ctx->h_state[0], p->accuracy_threshold);
    KMB_CUDA(cudaMemcpyAsync(st, ctx->h_state, sizeof(LoopState), cudaMemcpyHostToDevice, s));
    KMB_CUDA(cudaMemsetAsync(sc, 0, sizeof(kmb::DevScalars), s));
    const bool tc = is_tc_form(p->form);
    ctx->tc_products = form_products(p->form);
    prepare_rows<F>(ctx, X, n, d, tc);
    if (int rc = prepare_update<F>(ctx, X, n, d, k, st)) return rc;
    const int64_t T = p->max_iteration_count;
    int64_t enq = 0;
    int64_t batch = 2;
    while (enq < T) {
        const int64_t upto = std::min(T, enq + batch);
        for (; enq < upto; ++enq) {
            // from the second iteration on, labels/d2/shift_part describe the previous pass
            int rc = assign_pass<F>(ctx, X, n, d, C, k, recheck, labels, d2, st, tc, /*prior=*/enq > 0);
            if (rc) return rc;
            KernelTimer timer(ctx, 2);
            ProfRange range("kmeansMergeReduceCentroids");
            update_pass<F>(X, plan, labels, d2, C, Cnew, ws, st, /*commit=*/true, s, tc);
        }
        KMB_CUDA(cudaGetLastError());
        if (enq < T) {
            KMB_CUDA(cudaMemcpyAsync(ctx->h_state, st, sizeof(LoopState), cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaStreamSynchronize(s));
            if (ctx->h_state[0].done) break;
            batch = std::min<int64_t>(batch * 2, 8);
        }
    }
    return KMB_OK;
}

template <typename F>
int iterate_impl(kmb_context *ctx, const void *Xv, int64_t n, int64_t d, void *Cv, const kmb_params *p,
                 int32_t *labels, int64_t *iteration_count, kmb_stats *stats) {
    const int64_t k = p->cluster_count;
    const bool tc = is_tc_form(p->form);
    ctx->tc_products = form_products(p->form);
    if (tc && !kmb::tc_supported(d)) return fail(ctx, KMB_EUNSUPPORTED, "tensor-core form needs d <= 256");
    const bool recheck = p->recheck != 0 || tc;
    int rc = ensure_common<F>(ctx, n, d, k, recheck, tc);
    if (rc) return rc;
    kmb::UpdatePlan plan = kmb::make_update_plan(n, k, d);
    if (!kmb::ensure_update_buffers(ctx->ws, plan, sizeof(F))) return fail(ctx, KMB_ENOMEM, "update buffers");
    int32_t *lab = labels ? labels : (int32_t *)ctx->ws.labels.ptr;
    if ((rc = run_loop<F>(ctx, (const F *)Xv, n, d, (F *)Cv, p, plan, lab, recheck))) return rc;
    KMB_CUDA(cudaMemcpyAsync(ctx->h_state, ctx->ws.state.ptr, sizeof(LoopState), cudaMemcpyDeviceToHost, ctx->stream));
    KMB_CUDA(cudaStreamSynchronize(ctx->stream));
    const LoopState &hs = ctx->h_state[0];
    if (hs.error) return fail(ctx, hs.error, "device loop failed (status %d)", hs.error);
    if (iteration_count) *iteration_count = hs.iterations;
    if (stats) {
        stats->rechecked_rows = hs.rechecked_total;
        stats->full_rescans = hs.full_total;
        stats->changed_by_recheck = hs.n_changed;
        stats->empty_cluster_events = hs.empty_events;
        stats->last_shift = hs.shift;
    }
    return KMB_OK;
}

template <typename F>
int train_impl(kmb_context *ctx, int memory, const void *Xv, int64_t n, int64_t d, const void *C0v,
               const kmb_params *p, void *C_out, int32_t *responses, double *objective, int64_t *iteration_count,
               kmb_stats *stats) {
    const int64_t k = p->cluster_count;
    const bool tc = is_tc_form(p->form);
    ctx->tc_products = form_products(p->form);
    if (tc && !kmb::tc_supported(d)) return fail(ctx, KMB_EUNSUPPORTED, "tensor-core form needs d <= 256");
    const bool recheck = p->recheck != 0 || tc;
    int rc = ensure_common<F>(ctx, n, d, k, recheck, tc);
    if (rc) return rc;
    kmb::UpdatePlan plan = kmb::make_update_plan(n, k, d);
    if (!kmb::ensure_update_buffers(ctx->ws, plan, sizeof(F))) return fail(ctx, KMB_ENOMEM, "update buffers");
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;

    const F *X = (const F *)Xv;
    const F *C0 = (const F *)C0v;
    if (memory == KMB_MEM_HOST) {
        if ((rc = upload<F>(ctx, ws.X, Xv, sizeof(F) * n * d, &X))) return rc;
        if ((rc = upload<F>(ctx, ws.C0, C0v, sizeof(F) * k * d, &C0))) return rc;
    }
    int32_t *labels = (memory == KMB_MEM_DEVICE && responses) ? responses : (int32_t *)ws.labels.ptr;
    F *Ccur = (F *)ws.Ccur.ptr;
    F *d2 = (F *)ws.d2.ptr;
    LoopState *st = (LoopState *)ws.state.ptr;
    LoopState *st_final = st + 1;
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;

    init_state(ctx->h_state[1], 0.0);
    KMB_CUDA(cudaMemcpyAsync(st + 1, &ctx->h_state[1], sizeof(LoopState), cudaMemcpyHostToDevice, s));
    KMB_CUDA(cudaMemcpyAsync(Ccur, C0, sizeof(F) * k * d, cudaMemcpyDeviceToDevice, s));
    if ((rc = run_loop<F>(ctx, X, n, d, Ccur, p, plan, labels, recheck))) return rc;
    // Responses against the final centroids, then the exact objective.
    // (after at least one iteration, the last assignment + update seed the prior bound)
    if ((rc = assign_pass<F>(ctx, X, n, d, Ccur, k, recheck, labels, d2, st_final, tc,
                             /*prior=*/p->max_iteration_count > 0)))
        return rc;
    double *obj_dev = &sc->objective;
    {
        ProfRange range("kmeansUpdateObjectiveFunction");
        kmb::launch_objective<F>(X, n, d, Ccur, labels, (double *)ws.obj_part.ptr, obj_dev, s);
    }
    KMB_CUDA(cudaGetLastError());

    const cudaMemcpyKind out_kind = memory == KMB_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (C_out) KMB_CUDA(cudaMemcpyAsync(C_out, Ccur, sizeof(F) * k * d, out_kind, s));
    if (responses && labels != responses)
        KMB_CUDA(cudaMemcpyAsync(responses, labels, sizeof(int32_t) * n, out_kind, s));
    double obj_h = 0.0;
    KMB_CUDA(cudaMemcpyAsync(&obj_h, obj_dev, sizeof(double), cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaMemcpyAsync(ctx->h_state, st, sizeof(LoopState) * 2, cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaStreamSynchronize(s));
    const LoopState &hs = ctx->h_state[0];
    if (hs.error) return fail(ctx, hs.error, "device loop failed (status %d)", hs.error);
    if (ctx->h_state[1].error)
        return fail(ctx, ctx->h_state[1].error, "final assignment pass failed (status %d)", ctx->h_state[1].error);
    if (objective) *objective = obj_h;
    if (iteration_count) *iteration_count = hs.iterations;
    if (stats) {
        stats->rechecked_rows = ctx->h_state[1].n_recheck + ctx->h_state[1].n_full;
        stats->full_rescans = ctx->h_state[1].n_full;
        stats->changed_by_recheck = ctx->h_state[1].n_changed;
        stats->empty_cluster_events = hs.empty_events;
        stats->last_shift = hs.shift;
    }
    return KMB_OK;
}

template <typename F>
int infer_impl(kmb_context *ctx, int memory, const void *Xv, int64_t n, int64_t d, const void *Cv, int64_t k,
               int32_t form, int32_t compute_objective, int32_t *responses, double *objective, kmb_stats *stats) {
    const bool tc = is_tc_form(form);
    ctx->tc_products = form_products(form);
    if (tc && !kmb::tc_supported(d)) return fail(ctx, KMB_EUNSUPPORTED, "tensor-core form needs d <= 256");
    const bool recheck = tc;
    int rc = ensure_common<F>(ctx, n, d, k, recheck, tc);
    if (rc) return rc;
    if (!ctx->ws.ensure(ctx->ws.obj_part, sizeof(double) * kmb::kObjectivePartials)) return fail(ctx, KMB_ENOMEM, "objective");
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    const F *X = (const F *)Xv;
    const F *C = (const F *)Cv;
    if (memory == KMB_MEM_HOST) {
        if ((rc = upload<F>(ctx, ws.X, Xv, sizeof(F) * n * d, &X))) return rc;
        if ((rc = upload<F>(ctx, ws.C0, Cv, sizeof(F) * k * d, &C))) return rc;
    }
    int32_t *labels = (memory == KMB_MEM_DEVICE && responses) ? responses : (int32_t *)ws.labels.ptr;
    LoopState *st = (LoopState *)ws.state.ptr + 1;
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;
    init_state(ctx->h_state[1], 0.0);
    KMB_CUDA(cudaMemcpyAsync(st, &ctx->h_state[1], sizeof(LoopState), cudaMemcpyHostToDevice, s));
    KMB_CUDA(cudaMemsetAsync(sc, 0, sizeof(kmb::DevScalars), s));
    prepare_rows<F>(ctx, X, n, d, tc);
    if ((rc = assign_pass<F>(ctx, X, n, d, C, k, recheck, labels, (F *)ws.d2.ptr, st, tc))) return rc;
    if (compute_objective)
        kmb::launch_objective<F>(X, n, d, C, labels, (double *)ws.obj_part.ptr, &sc->objective, s);
    KMB_CUDA(cudaGetLastError());
    const cudaMemcpyKind out_kind = memory == KMB_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (responses && labels != responses)
        KMB_CUDA(cudaMemcpyAsync(responses, labels, sizeof(int32_t) * n, out_kind, s));
    double obj_h = 0.0;
    KMB_CUDA(cudaMemcpyAsync(&obj_h, &sc->objective, sizeof(double), cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaMemcpyAsync(&ctx->h_state[1], st, sizeof(LoopState), cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaStreamSynchronize(s));
    if (ctx->h_state[1].error)
        return fail(ctx, ctx->h_state[1].error, "assignment pass failed (status %d)", ctx->h_state[1].error);
    if (compute_objective && objective) *objective = obj_h;
    if (stats) {
        stats->rechecked_rows = ctx->h_state[1].n_recheck + ctx->h_state[1].n_full;
        stats->full_rescans = ctx->h_state[1].n_full;
        stats->changed_by_recheck = ctx->h_state[1].n_changed;
        stats->empty_cluster_events = 0;
        stats->last_shift = 0.0;
    }
    return KMB_OK;
}

template <typename F>
int step_impl(kmb_context *ctx, const void *Xv, int64_t n, int64_t d, const void *Cin, int64_t k, int32_t form,
              int32_t recheck_flag, void *C_out, int32_t *labels, double *shift, int64_t *n_empty) {
    const bool tc = is_tc_form(form);
    ctx->tc_products = form_products(form);
    if (tc && !kmb::tc_supported(d)) return fail(ctx, KMB_EUNSUPPORTED, "tensor-core form needs d <= 256");
    const bool recheck = recheck_flag != 0 || tc;
    int rc = ensure_common<F>(ctx, n, d, k, recheck, tc);
    if (rc) return rc;
    kmb::UpdatePlan plan = kmb::make_update_plan(n, k, d);
    if (!kmb::ensure_update_buffers(ctx->ws, plan, sizeof(F))) return fail(ctx, KMB_ENOMEM, "update buffers");
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    const F *X = (const F *)Xv;
    F *Ccur = (F *)ws.Ccur.ptr;
    LoopState *st = (LoopState *)ws.state.ptr;
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;
    init_state(ctx->h_state[0], 0.0);
    KMB_CUDA(cudaMemcpyAsync(st, ctx->h_state, sizeof(LoopState), cudaMemcpyHostToDevice, s));
    KMB_CUDA(cudaMemcpyAsync(Ccur, Cin, sizeof(F) * k * d, cudaMemcpyDeviceToDevice, s));
    KMB_CUDA(cudaMemsetAsync(sc, 0, sizeof(kmb::DevScalars), s));
    prepare_rows<F>(ctx, X, n, d, tc);
    if ((rc = prepare_update<F>(ctx, X, n, d, k, st))) return rc;
    if ((rc = assign_pass<F>(ctx, X, n, d, Ccur, k, recheck, labels, (F *)ws.d2.ptr, st, tc))) return rc;
    update_pass<F>(X, plan, labels, (F *)ws.d2.ptr, Ccur, (F *)C_out, ws, st, /*commit=*/false, s, tc);
    KMB_CUDA(cudaGetLastError());
    KMB_CUDA(cudaMemcpyAsync(ctx->h_state, st, sizeof(LoopState), cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaStreamSynchronize(s));
    if (ctx->h_state[0].error) return fail(ctx, ctx->h_state[0].error, "device step failed");
    if (shift) *shift = ctx->h_state[0].shift;
    if (n_empty) *n_empty = ctx->h_state[0].n_empty;
    return KMB_OK;
}

// One shard's statistics under C: labels, FP64 sums/counts, sum of squared
// distances, optional per-row squared distances (for candidate selection).
template <typename F>
int partial_impl(kmb_context *ctx, const F *X, int64_t n, int64_t d, const F *C, int64_t k, int32_t form,
                 int32_t *labels, double *sums, int64_t *counts, double *sq_distances, F *row_sq) {
    const bool tc = is_tc_form(form);
    ctx->tc_products = form_products(form);
    if (tc && !kmb::tc_supported(d)) return fail(ctx, KMB_EUNSUPPORTED, "tensor-core form needs d <= 256");
    int rc = ensure_common<F>(ctx, n, d, k, tc, tc);
    if (rc) return rc;
    kmb::UpdatePlan plan = kmb::make_update_plan(n, k, d);
    if (!kmb::ensure_update_buffers(ctx->ws, plan, sizeof(F))) return fail(ctx, KMB_ENOMEM, "update buffers");
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    LoopState *st = (LoopState *)ws.state.ptr + 1;
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;
    init_state(ctx->h_state[1], 0.0);
    KMB_CUDA(cudaMemcpyAsync(st, &ctx->h_state[1], sizeof(LoopState), cudaMemcpyHostToDevice, s));
    KMB_CUDA(cudaMemsetAsync(sc, 0, sizeof(kmb::DevScalars), s));
    prepare_rows<F>(ctx, X, n, d, tc);
    if ((rc = assign_pass<F>(ctx, X, n, d, C, k, tc, labels, (F *)ws.d2.ptr, st, tc))) return rc;
    if (sums) kmb::launch_partial_sums<F>(X, plan, labels, sums, counts, ws, s);  // (null: labels and distances only)
    if (sq_distances)
        kmb::launch_sum_values<F>((const F *)ws.d2.ptr, n, (double *)ws.obj_part.ptr, sq_distances, s);
    if (row_sq) KMB_CUDA(cudaMemcpyAsync(row_sq, ws.d2.ptr, sizeof(F) * n, cudaMemcpyDeviceToDevice, s));
    KMB_CUDA(cudaGetLastError());
    KMB_CUDA(cudaMemcpyAsync(&ctx->h_state[1], st, sizeof(LoopState), cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaStreamSynchronize(s));
    if (ctx->h_state[1].error)
        return fail(ctx, ctx->h_state[1].error, "assignment pass failed (status %d)", ctx->h_state[1].error);
    return KMB_OK;
}

int validate_shapes(kmb_context *ctx, int dtype, int64_t n, int64_t d, int64_t k) {
    if (!ctx) return KMB_EINVAL;
    if (dtype != KMB_F32 && dtype != KMB_F64) return fail(ctx, KMB_EINVAL, "unknown dtype %d", dtype);
    if (n <= 0) return fail(ctx, KMB_EINVAL, "input data is empty");
    if (n > INT32_MAX) return fail(ctx, KMB_EINVAL, "row count exceeds INT32_MAX");
    if (d <= 0) return fail(ctx, KMB_EINVAL, "column count must be positive");
    if (k <= 0 || k > INT32_MAX) return fail(ctx, KMB_EINVAL, "cluster count must be in (0, INT32_MAX]");
    if (k > n) return fail(ctx, KMB_EINVAL, "cluster count exceeds data row count");
    return KMB_OK;
}

// ---- CSR rows (kmeans::method::lloyd_csr) ----------------------------------

// Brings caller CSR arrays (host or device; indices int64 with base 0 or 1) into
// the device form of kmb::CsrRows and checks them.
template <typename F>
int prepare_csr(kmb_context *ctx, int memory, const void *vals, const int64_t *cols, const int64_t *rowptr, int64_t n,
                int64_t d, int base, kmb::CsrRows *out) {
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    int64_t ends[2];
    if (memory == KMB_MEM_HOST) {
        ends[0] = rowptr[0];
        ends[1] = rowptr[n];
    } else {
        KMB_CUDA(cudaMemcpyAsync(&ends[0], rowptr, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        KMB_CUDA(cudaMemcpyAsync(&ends[1], rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        KMB_CUDA(cudaStreamSynchronize(s));
    }
    if (ends[0] != base) return fail(ctx, KMB_EINVAL, "CSR row offsets must start at the index base (%d)", base);
    const int64_t nnz = ends[1] - base;
    if (nnz < 0) return fail(ctx, KMB_EINVAL, "CSR row offsets are decreasing");
    bool ok = ws.ensure(ws.csr_cols, sizeof(int32_t) * std::max<int64_t>(1, nnz)) &&
              ws.ensure(ws.csr_rowptr, sizeof(int64_t) * (n + 1)) && ws.ensure(ws.csr_bad, sizeof(int));
    const F *v = (const F *)vals;
    const int64_t *c64 = cols, *r64 = rowptr;
    if (ok && memory == KMB_MEM_HOST) {
        ok = ws.ensure(ws.csr_cols64, sizeof(int64_t) * std::max<int64_t>(1, nnz)) &&
             ws.ensure(ws.csr_rowptr64, sizeof(int64_t) * (n + 1));
        if (ok) {
            int rc = upload<F>(ctx, ws.csr_vals, vals, sizeof(F) * std::max<int64_t>(1, nnz), &v);
            if (rc) return rc;
            KMB_CUDA(cudaMemcpyAsync(ws.csr_cols64.ptr, cols, sizeof(int64_t) * nnz, cudaMemcpyHostToDevice, s));
            KMB_CUDA(cudaMemcpyAsync(ws.csr_rowptr64.ptr, rowptr, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, s));
            c64 = (const int64_t *)ws.csr_cols64.ptr;
            r64 = (const int64_t *)ws.csr_rowptr64.ptr;
        }
    }
    if (!ok) return fail(ctx, KMB_ENOMEM, "device allocation failed (CSR rows, nnz=%lld)", (long long)nnz);
    KMB_CUDA(cudaMemsetAsync(ws.csr_bad.ptr, 0, sizeof(int), s));
    kmb::launch_csr_prepare(c64, r64, n, d, nnz, base, (int32_t *)ws.csr_cols.ptr, (int64_t *)ws.csr_rowptr.ptr,
                            (int *)ws.csr_bad.ptr, s);
    int bad = 0;
    KMB_CUDA(cudaMemcpyAsync(&bad, ws.csr_bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaStreamSynchronize(s));
    if (bad & 1) return fail(ctx, KMB_EINVAL, "CSR row offsets are out of order or out of range");
    if (bad & 2)
        return fail(ctx, KMB_EINVAL,
                    "CSR column indices must lie in [0, column_count) and increase strictly within each row");
    *out = kmb::CsrRows{v, (const int32_t *)ws.csr_cols.ptr, (const int64_t *)ws.csr_rowptr.ptr, n, d, nnz};
    return KMB_OK;
}

template <typename F>
void csr_assign_pass(kmb_context *ctx, const kmb::CsrRows &X, const F *C, int64_t k, int32_t *labels, F *d2,
                     LoopState *st) {
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    const int64_t kpad = round_up(k, kBN);
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;
    reset_iteration_kernel<<<1, 1, 0, s>>>(st);
    KMB_LAUNCHED();
    kmb::launch_prep_centroids<F>(C, k, X.d, kpad, (F *)ws.Ct.ptr, (F *)ws.h.ptr, &sc->cnorm_max, st, s);
    KernelTimer timer(ctx, 0);
    kmb::launch_csr_assign<F>(X, (const F *)ws.Ct.ptr, (const F *)ws.h.ptr, k, kpad, labels, d2, st, s);
}

// The CSR update: float values take the exact update (integer cluster sums from the
// stored entries, moved rows only once few rows move), double values the FP64 one.
template <typename F>
bool csr_update_buffers(kmb::Workspace &ws, const kmb::UpdatePlan &plan, int64_t n, int64_t k, int64_t d) {
    return kmb::ensure_update_buffers(ws, plan, sizeof(F));
}
template <>
bool csr_update_buffers<float>(kmb::Workspace &ws, const kmb::UpdatePlan &plan, int64_t n, int64_t k, int64_t d) {
    return kmb::ensure_update_buffers(ws, plan, sizeof(float), /*fp64_records=*/false) &&
           kmb::ensure_exact_buffers(ws, n, k, d, /*piece_records=*/false);
}
template <typename F>
void csr_prepare_update(const kmb::CsrRows &, kmb::Workspace &, LoopState *, cudaStream_t) {}
template <>
void csr_prepare_update<float>(const kmb::CsrRows &X, kmb::Workspace &ws, LoopState *st, cudaStream_t s) {
    kmb::prepare_exact_update_csr(X, ws, st, s);
}
template <typename F>
void csr_update_pass(const kmb::CsrRows &X, const kmb::UpdatePlan &plan, int32_t *labels, F *d2, F *C_old, F *C_new,
                     kmb::Workspace &ws, LoopState *st, cudaStream_t s) {
    kmb::launch_update<F>(nullptr, plan, labels, d2, C_old, C_new, ws, st, /*commit=*/true, s, &X);
}
template <>
void csr_update_pass<float>(const kmb::CsrRows &X, const kmb::UpdatePlan &plan, int32_t *labels, float *d2,
                            float *C_old, float *C_new, kmb::Workspace &ws, LoopState *st, cudaStream_t s) {
    kmb::launch_update_exact_csr(X, plan, labels, d2, C_old, C_new, ws, st, /*commit=*/true, s);
}

template <typename F>
int train_csr_impl(kmb_context *ctx, int memory, const void *vals, const int64_t *cols, const int64_t *rowptr,
                   int64_t n, int64_t d, int base, const void *C0v, const kmb_params *p, void *C_out,
                   int32_t *responses, double *objective, int64_t *iteration_count, kmb_stats *stats) {
    const int64_t k = p->cluster_count;
    int rc = ensure_common<F>(ctx, n, d, k, false, false);
    if (rc) return rc;
    kmb::UpdatePlan plan = kmb::make_update_plan(n, k, d);
    if (!csr_update_buffers<F>(ctx->ws, plan, n, k, d) || !ctx->ws.ensure(ctx->ws.csr_cnorm, sizeof(double) * k))
        return fail(ctx, KMB_ENOMEM, "update buffers");
    kmb::CsrRows X;
    if ((rc = prepare_csr<F>(ctx, memory, vals, cols, rowptr, n, d, base, &X))) return rc;
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    const F *C0 = (const F *)C0v;
    if (memory == KMB_MEM_HOST && (rc = upload<F>(ctx, ws.C0, C0v, sizeof(F) * k * d, &C0))) return rc;
    int32_t *labels = (memory == KMB_MEM_DEVICE && responses) ? responses : (int32_t *)ws.labels.ptr;
    F *Ccur = (F *)ws.Ccur.ptr, *Cnew = (F *)ws.Cnew.ptr, *d2 = (F *)ws.d2.ptr;
    LoopState *st = (LoopState *)ws.state.ptr;
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;
    init_state(ctx->h_state[0], p->accuracy_threshold);
    init_state(ctx->h_state[1], 0.0);
    KMB_CUDA(cudaMemcpyAsync(st, ctx->h_state, sizeof(LoopState) * 2, cudaMemcpyHostToDevice, s));
    KMB_CUDA(cudaMemsetAsync(sc, 0, sizeof(kmb::DevScalars), s));
    KMB_CUDA(cudaMemcpyAsync(Ccur, C0, sizeof(F) * k * d, cudaMemcpyDeviceToDevice, s));
    const int64_t T = p->max_iteration_count;
    if (T > 0) csr_prepare_update<F>(X, ws, st, s);
    int64_t enq = 0, batch = 2;
    while (enq < T) {
        const int64_t upto = std::min(T, enq + batch);
        for (; enq < upto; ++enq) {
            csr_assign_pass<F>(ctx, X, Ccur, k, labels, d2, st);
            KernelTimer timer(ctx, 2);
            csr_update_pass<F>(X, plan, labels, d2, Ccur, Cnew, ws, st, s);
        }
        KMB_CUDA(cudaGetLastError());
        if (enq < T) {
            KMB_CUDA(cudaMemcpyAsync(ctx->h_state, st, sizeof(LoopState), cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaStreamSynchronize(s));
            if (ctx->h_state[0].done) break;
            batch = std::min<int64_t>(batch * 2, 8);
        }
    }
    // responses against the final centroids, then the exact objective
    csr_assign_pass<F>(ctx, X, Ccur, k, labels, d2, st + 1);
    kmb::launch_csr_objective<F>(X, Ccur, k, labels, (double *)ws.csr_cnorm.ptr, (double *)ws.obj_part.ptr,
                                 &sc->objective, s);
    KMB_CUDA(cudaGetLastError());
    const cudaMemcpyKind out_kind = memory == KMB_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (C_out) KMB_CUDA(cudaMemcpyAsync(C_out, Ccur, sizeof(F) * k * d, out_kind, s));
    if (responses && labels != responses)
        KMB_CUDA(cudaMemcpyAsync(responses, labels, sizeof(int32_t) * n, out_kind, s));
    double obj_h = 0.0;
    KMB_CUDA(cudaMemcpyAsync(&obj_h, &sc->objective, sizeof(double), cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaMemcpyAsync(ctx->h_state, st, sizeof(LoopState) * 2, cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaStreamSynchronize(s));
    const LoopState &hs = ctx->h_state[0];
    if (hs.error) return fail(ctx, hs.error, "device loop failed (status %d)", hs.error);
    if (ctx->h_state[1].error)
        return fail(ctx, ctx->h_state[1].error, "final assignment pass failed (status %d)", ctx->h_state[1].error);
    if (objective) *objective = obj_h;
    if (iteration_count) *iteration_count = hs.iterations;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->empty_cluster_events = hs.empty_events;
        stats->last_shift = hs.shift;
    }
    return KMB_OK;
}

template <typename F>
int infer_csr_impl(kmb_context *ctx, int memory, const void *vals, const int64_t *cols, const int64_t *rowptr,
                   int64_t n, int64_t d, int base, const void *Cv, int64_t k, int32_t compute_objective,
                   int32_t *responses, double *objective) {
    int rc = ensure_common<F>(ctx, n, d, k, false, false);
    if (rc) return rc;
    kmb::Workspace &ws = ctx->ws;
    if (!ws.ensure(ws.obj_part, sizeof(double) * kmb::kObjectivePartials) || !ws.ensure(ws.csr_cnorm, sizeof(double) * k))
        return fail(ctx, KMB_ENOMEM, "objective");
    kmb::CsrRows X;
    if ((rc = prepare_csr<F>(ctx, memory, vals, cols, rowptr, n, d, base, &X))) return rc;
    cudaStream_t s = ctx->stream;
    const F *C = (const F *)Cv;
    if (memory == KMB_MEM_HOST && (rc = upload<F>(ctx, ws.C0, Cv, sizeof(F) * k * d, &C))) return rc;
    int32_t *labels = (memory == KMB_MEM_DEVICE && responses) ? responses : (int32_t *)ws.labels.ptr;
    LoopState *st = (LoopState *)ws.state.ptr + 1;
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;
    init_state(ctx->h_state[1], 0.0);
    KMB_CUDA(cudaMemcpyAsync(st, &ctx->h_state[1], sizeof(LoopState), cudaMemcpyHostToDevice, s));
    KMB_CUDA(cudaMemsetAsync(sc, 0, sizeof(kmb::DevScalars), s));
    csr_assign_pass<F>(ctx, X, C, k, labels, (F *)ws.d2.ptr, st);
    if (compute_objective)
        kmb::launch_csr_objective<F>(X, C, k, labels, (double *)ws.csr_cnorm.ptr, (double *)ws.obj_part.ptr,
                                     &sc->objective, s);
    KMB_CUDA(cudaGetLastError());
    const cudaMemcpyKind out_kind = memory == KMB_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (responses && labels != responses)
        KMB_CUDA(cudaMemcpyAsync(responses, labels, sizeof(int32_t) * n, out_kind, s));
    double obj_h = 0.0;
    KMB_CUDA(cudaMemcpyAsync(&obj_h, &sc->objective, sizeof(double), cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaStreamSynchronize(s));
    if (compute_objective && objective) *objective = obj_h;
    return KMB_OK;
}

int validate_csr_call(kmb_context *ctx, int dtype, int memory, const void *vals, const int64_t *cols,
                      const int64_t *rowptr, int32_t indexing) {
    if (dtype != KMB_F32 && dtype != KMB_F64) return fail(ctx, KMB_EINVAL, "unknown dtype %d", dtype);
    if (memory != KMB_MEM_HOST && memory != KMB_MEM_DEVICE) return fail(ctx, KMB_EINVAL, "unknown memory kind");
    if (indexing != 0 && indexing != 1) return fail(ctx, KMB_EINVAL, "indexing must be 0 (zero-based) or 1 (one-based)");
    if (!vals || !cols || !rowptr) return fail(ctx, KMB_EINVAL, "CSR values, column indices and row offsets are required");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, KMB_ECUDA, "cudaSetDevice failed");
    return KMB_OK;
}


// ---- sharded training through a caller's communicator (kmb_train_spmd) --------

// Candidate rows for the sharded reseed: their squared distances and row vectors.
template <typename F>
__global__ void spmd_gather_kernel(const F *__restrict__ X, int d, const long long *__restrict__ rows,
                                   const F *__restrict__ row_sq, int m, double *__restrict__ vals,
                                   F *__restrict__ vecs) {
    for (int e = blockIdx.x; e < m; e += gridDim.x) {
        const long long r = rows[e];
        if (threadIdx.x == 0) vals[e] = (double)row_sq[r];
        for (int t = threadIdx.x; t < d; t += blockDim.x) vecs[(int64_t)e * d + t] = X[r * d + t];
    }
}

template <typename F>
int train_spmd_impl(kmb_context *ctx, int dtype, const F *X, int64_t n, int64_t d, const F *C0, kmb_params p,
                    const kmb_communicator *comm, F *C_out, int32_t *labels, double *objective, int64_t *iters) {
    const int64_t k = p.cluster_count, kd = k * d;
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    // every rank's row count: this rank's first global row and the total
    std::vector<int64_t> ns((size_t)comm->size, 0);
    if (comm->allgather(comm->user, &n, (int64_t)sizeof(int64_t), ns.data()))
        return fail(ctx, KMB_ECOMM, "allgather of the row counts failed");
    int64_t row0 = 0, total = 0;
    for (int r = 0; r < comm->size; ++r) {
        if (r < comm->rank) row0 += ns[r];
        total += ns[r];
    }
    if (k > total) return fail(ctx, KMB_EINVAL, "cluster count exceeds data row count");
    // float rows: the exact fixed-point sums of the single-GPU update, exchanged as
    // exact 32-bit halves, so every rank's centroids are those of a one-GPU train
    const bool exact = sizeof(F) == 4 && total <= INT32_MAX;
    if (!ws.ensure(ws.sp_sums, sizeof(double) * kd) || !ws.ensure(ws.sp_counts, sizeof(int64_t) * k) ||
        !ws.ensure(ws.sp_sq, sizeof(double) * 2) || !ws.ensure(ws.sp_rowsq, sizeof(F) * n) ||
        !ws.ensure(ws.sp_Ca, sizeof(F) * kd) || !ws.ensure(ws.sp_Cb, sizeof(F) * kd) ||
        !ws.ensure(ws.sp_ids, sizeof(int32_t) * k) || !ws.ensure(ws.sp_rows, sizeof(long long) * k) ||
        !ws.ensure(ws.sp_state, sizeof(LoopState)) || !ws.ensure(ws.sp_gather, (sizeof(double) + sizeof(F) * d) * k) ||
        (exact && (!ws.ensure(ws.sp_acc, sizeof(long long) * 3 * kd) || !ws.ensure(ws.sp_colexp, sizeof(int) * d) ||
                   !ws.ensure(ws.sp_shift, sizeof(double) * k))))
        return fail(ctx, KMB_ENOMEM, "sharded training buffers");
    double *sums = (double *)ws.sp_sums.ptr, *sq = (double *)ws.sp_sq.ptr;
    int64_t *counts = (int64_t *)ws.sp_counts.ptr;
    F *row_sq = (F *)ws.sp_rowsq.ptr;
    F *Ccur = (F *)ws.sp_Ca.ptr, *Cnew = (F *)ws.sp_Cb.ptr;
    int32_t *ids = (int32_t *)ws.sp_ids.ptr;
    long long *rows = (long long *)ws.sp_rows.ptr;
    double *gvals = (double *)ws.sp_gather.ptr;
    F *gvecs = (F *)(gvals + k);
    long long *acc = (long long *)ws.sp_acc.ptr;
    int *colexp = (int *)ws.sp_colexp.ptr;
    int *cnt32 = (int *)ws.sp_counts.ptr;  // the exact path's counts (int32) share the buffer
    int *bad = (int *)(sq + 1);
    double *shift_part = (double *)ws.sp_shift.ptr;
    std::vector<double> packed((size_t)(exact ? 6 * kd + k + 1 : kd + k + 1));
    std::vector<int64_t> hcounts((size_t)k);
    std::vector<long long> hacc(exact ? (size_t)(3 * kd) : 0);
    std::vector<int> hcnt(exact ? (size_t)k : 0);
    std::vector<double> hshift(exact ? (size_t)k : 0);
    KMB_CUDA(cudaMemcpyAsync(Ccur, C0, sizeof(F) * kd, cudaMemcpyDeviceToDevice, s));
    if (exact) {
        // column exponents from the column maxima over all ranks (the single-GPU rule:
        // the column's largest |x| maps below 2^94)
        std::vector<unsigned> bits((size_t)d), all((size_t)d * comm->size);
        kmb::launch_column_max_bits((const float *)X, n, d, (unsigned *)colexp, s);
        KMB_CUDA(cudaMemcpyAsync(bits.data(), colexp, sizeof(unsigned) * d, cudaMemcpyDeviceToHost, s));
        KMB_CUDA(cudaStreamSynchronize(s));
        if (comm->allgather(comm->user, bits.data(), (int64_t)(sizeof(unsigned) * d), all.data()))
            return fail(ctx, KMB_ECOMM, "allgather of the column maxima failed");
        std::vector<int> hexp((size_t)d);
        for (int64_t t = 0; t < d; ++t) {
            unsigned b = 0;
            for (int r = 0; r < comm->size; ++r) b = std::max(b, all[(size_t)r * d + t]);
            float m;
            std::memcpy(&m, &b, sizeof(m));
            int e = 0;
            if (b != 0u && std::isfinite(m)) {
                int ex;
                std::frexp(m, &ex);
                e = kmb::kExactMaxBits - ex;
            }
            hexp[(size_t)t] = e;
        }
        KMB_CUDA(cudaMemcpyAsync(colexp, hexp.data(), sizeof(int) * d, cudaMemcpyHostToDevice, s));
    }
    int64_t it = 0;
    int rc;
    while (it < p.max_iteration_count) {
        double shift = 0.0;
        std::vector<int32_t> hids;
        if (exact) {
            if ((rc = partial_impl<F>(ctx, X, n, d, Ccur, k, p.form, labels, nullptr, nullptr, sq, row_sq))) return rc;
            KMB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
            kmb::launch_shard_exact_sums((const float *)X, n, (int)d, (int)k, labels, colexp, acc, cnt32, bad, s);
            int hbad = 0;
            KMB_CUDA(cudaMemcpyAsync(hacc.data(), acc, sizeof(long long) * 3 * kd, cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaMemcpyAsync(hcnt.data(), cnt32, sizeof(int) * k, cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaMemcpyAsync(&packed[6 * kd + k], sq, sizeof(double), cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaStreamSynchronize(s));
            if (hbad) return fail(ctx, KMB_ECUDA, "label out of range in the exact sums");
            // each int64 limb sum as two exact doubles: its low 32 bits and the rest
            for (int64_t i = 0; i < 3 * kd; ++i) {
                packed[(size_t)i] = (double)(hacc[(size_t)i] & 0xffffffffll);
                packed[(size_t)(3 * kd + i)] = (double)(hacc[(size_t)i] >> 32);
            }
            for (int64_t j = 0; j < k; ++j) packed[(size_t)(6 * kd + j)] = (double)hcnt[(size_t)j];
            if (comm->allreduce_sum_f64(comm->user, packed.data(), 6 * kd + k + 1))
                return fail(ctx, KMB_ECOMM, "allreduce of the cluster sums failed");
            for (int64_t i = 0; i < 3 * kd; ++i)
                hacc[(size_t)i] = (long long)std::llround(packed[(size_t)(3 * kd + i)]) * 4294967296ll +
                                  (long long)std::llround(packed[(size_t)i]);
            for (int64_t j = 0; j < k; ++j) {
                hcnt[(size_t)j] = (int)std::llround(packed[(size_t)(6 * kd + j)]);
                if (hcnt[(size_t)j] == 0) hids.push_back((int32_t)j);
            }
            KMB_CUDA(cudaMemcpyAsync(acc, hacc.data(), sizeof(long long) * 3 * kd, cudaMemcpyHostToDevice, s));
            KMB_CUDA(cudaMemcpyAsync(cnt32, hcnt.data(), sizeof(int) * k, cudaMemcpyHostToDevice, s));
            KMB_CUDA(cudaMemcpyAsync(Cnew, Ccur, sizeof(F) * kd, cudaMemcpyDeviceToDevice, s));
            kmb::launch_shard_exact_finalize(acc, cnt32, colexp, (float *)Cnew, (int)k, (int)d, shift_part, s);
            KMB_CUDA(cudaMemcpyAsync(hshift.data(), shift_part, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaStreamSynchronize(s));
            for (int64_t j = 0; j < k; ++j) shift += hshift[(size_t)j];
        } else {
            if ((rc = partial_impl<F>(ctx, X, n, d, Ccur, k, p.form, labels, sums, counts, sq, row_sq))) return rc;
            // one exchange: [sums | counts | squared distances] summed over the ranks
            KMB_CUDA(cudaMemcpyAsync(packed.data(), sums, sizeof(double) * kd, cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaMemcpyAsync(hcounts.data(), counts, sizeof(int64_t) * k, cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaMemcpyAsync(&packed[kd + k], sq, sizeof(double), cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaStreamSynchronize(s));
            for (int64_t j = 0; j < k; ++j) packed[kd + j] = (double)hcounts[j];  // exact below 2^53
            if (comm->allreduce_sum_f64(comm->user, packed.data(), kd + k + 1))
                return fail(ctx, KMB_ECOMM, "allreduce of the cluster sums failed");
            for (int64_t j = 0; j < k; ++j) hcounts[j] = (int64_t)std::llround(packed[kd + j]);
            KMB_CUDA(cudaMemcpyAsync(sums, packed.data(), sizeof(double) * kd, cudaMemcpyHostToDevice, s));
            KMB_CUDA(cudaMemcpyAsync(counts, hcounts.data(), sizeof(int64_t) * k, cudaMemcpyHostToDevice, s));
            int64_t ne = 0;
            if ((rc = kmb_finalize_centroids(ctx, dtype, sums, counts, Ccur, k, d, Cnew, &shift, ids, &ne))) return rc;
            hids.resize((size_t)ne);
            if (ne > 0) {
                KMB_CUDA(cudaMemcpyAsync(hids.data(), ids, sizeof(int32_t) * ne, cudaMemcpyDeviceToHost, s));
                KMB_CUDA(cudaStreamSynchronize(s));
            }
        }
        if (!hids.empty()) {
            // every rank offers its m farthest rows; the global m farthest by (distance
            // descending, global row ascending) reseed the empty clusters, ascending
            const int m = (int)hids.size(), take = (int)std::min<int64_t>(m, n);
            if (!kmb::launch_top_rows<F>(row_sq, n, take, ws, (LoopState *)ws.sp_state.ptr, rows, s))
                return fail(ctx, KMB_ENOMEM, "candidate selection buffers");
            if (take > 0) {
                spmd_gather_kernel<F><<<(unsigned)std::min(take, 1024), 128, 0, s>>>(X, (int)d, rows, row_sq, take,
                                                                                      gvals, gvecs);
                KMB_LAUNCHED();
            }
            const size_t rec = (16 + sizeof(F) * (size_t)d + 7) / 8 * 8;  // value, global row, row vector
            std::vector<unsigned char> send(rec * (size_t)m, 0), recv(rec * (size_t)m * (size_t)comm->size);
            std::vector<long long> hrows((size_t)std::max(take, 1));
            std::vector<double> hvals((size_t)std::max(take, 1));
            std::vector<F> hvecs((size_t)std::max(take, 1) * (size_t)d);
            std::vector<F> hC((size_t)kd);
            if (take > 0) {
                KMB_CUDA(cudaMemcpyAsync(hrows.data(), rows, sizeof(long long) * take, cudaMemcpyDeviceToHost, s));
                KMB_CUDA(cudaMemcpyAsync(hvals.data(), gvals, sizeof(double) * take, cudaMemcpyDeviceToHost, s));
                KMB_CUDA(cudaMemcpyAsync(hvecs.data(), gvecs, sizeof(F) * take * d, cudaMemcpyDeviceToHost, s));
            }
            KMB_CUDA(cudaMemcpyAsync(hC.data(), Ccur, sizeof(F) * kd, cudaMemcpyDeviceToHost, s));
            KMB_CUDA(cudaStreamSynchronize(s));
            for (int e = 0; e < m; ++e) {
                unsigned char *r = send.data() + rec * e;
                const double v = e < take ? (std::isnan(hvals[e]) ? -INFINITY : hvals[e]) : -INFINITY;
                const long long g = e < take ? row0 + hrows[e] : INT64_MAX;
                std::memcpy(r, &v, 8);
                std::memcpy(r + 8, &g, 8);
                if (e < take) std::memcpy(r + 16, hvecs.data() + (size_t)e * d, sizeof(F) * d);
            }
            if (comm->allgather(comm->user, send.data(), (int64_t)send.size(), recv.data()))
                return fail(ctx, KMB_ECOMM, "allgather of the reseed candidates failed");
            const size_t total_recs = (size_t)m * (size_t)comm->size;
            std::vector<size_t> order(total_recs);
            std::vector<double> av(total_recs);
            std::vector<long long> ar(total_recs);
            for (size_t i = 0; i < total_recs; ++i) {
                order[i] = i;
                std::memcpy(&av[i], recv.data() + rec * i, 8);
                std::memcpy(&ar[i], recv.data() + rec * i + 8, 8);
            }
            std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
                return av[a] > av[b] || (av[a] == av[b] && ar[a] < ar[b]);
            });
            for (int e = 0; e < m; ++e) {
                const size_t i = order[e];
                if (!std::isfinite(av[i]))
                    return fail(ctx, KMB_ETOO_MANY_EMPTY, "fewer candidate rows than empty clusters");
                const F *vec = reinterpret_cast<const F *>(recv.data() + rec * i + 16);
                const int cid = hids[e];
                double a = 0.0;
                for (int64_t t = 0; t < d; ++t) {
                    const double df = (double)hC[(size_t)cid * d + t] - (double)vec[t];
                    a += df * df;
                }
                shift += a;
                KMB_CUDA(cudaMemcpyAsync(Cnew + (int64_t)cid * d, vec, sizeof(F) * d, cudaMemcpyHostToDevice, s));
            }
            KMB_CUDA(cudaStreamSynchronize(s));  // the host rows above are copied before they go out of scope
        }
        std::swap(Ccur, Cnew);
        ++it;
        if (shift <= p.accuracy_threshold) break;
    }
    // responses of this rank's rows and the objective under the final centroids
    if ((rc = partial_impl<F>(ctx, X, n, d, Ccur, k, p.form, labels, nullptr, nullptr, sq, nullptr))) return rc;
    double obj = 0.0;
    KMB_CUDA(cudaMemcpyAsync(&obj, sq, sizeof(double), cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaMemcpyAsync(C_out, Ccur, sizeof(F) * kd, cudaMemcpyDeviceToDevice, s));
    KMB_CUDA(cudaStreamSynchronize(s));
    if (comm->allreduce_sum_f64(comm->user, &obj, 1)) return fail(ctx, KMB_ECOMM, "allreduce of the objective failed");
    if (objective) *objective = obj;
    if (iters) *iters = it;
    return KMB_OK;
}

}  // namespace

// k-means++ initialisation (kmb_init.cu has the device side). The host draws
// the uniforms exactly as the reference's generator does and hands them to
// the device in order: k center probabilities, then a pool of resample draws
// (refilled, continuing the same sequence, when a round runs out of them).
template <typename F>
int init_plusplus_core(kmb_context *ctx, int memory, const F *X, const kmb::CsrRows *csr, int64_t n, int64_t d,
                       int64_t k, uint32_t seed, void *C_out) {
    kmb::Workspace &ws = ctx->ws;
    cudaStream_t s = ctx->stream;
    // KMB_PLUSPLUS_POOL (1..2^20) shrinks the resample pool so tests can drive the refill path
    int pool_n = 4096;
    if (const char *e = getenv("KMB_PLUSPLUS_POOL")) pool_n = (int)std::min(std::max(atol(e), 1L), 1L << 20);
    const int64_t nb = (n + 511) / 512;
    bool ok = ws.ensure(ws.d2, sizeof(F) * n) && ws.ensure(ws.pp_acc, sizeof(F) * nb) &&
              ws.ensure(ws.pp_rand, sizeof(F) * (k + pool_n)) && ws.ensure(ws.pp_state, sizeof(kmb::PPState)) &&
              ws.ensure(ws.pp_flags, sizeof(unsigned) * nb) &&
              ws.ensure(ws.Cout, sizeof(F) * k * d);
    if (!ok) return fail(ctx, KMB_ENOMEM, "device allocation failed (k-means++ init, n=%lld)", (long long)n);
    F *md = (F *)ws.d2.ptr, *acc = (F *)ws.pp_acc.ptr, *rnd = (F *)ws.pp_rand.ptr;
    kmb::PPState *st = (kmb::PPState *)ws.pp_state.ptr;
    F *C = memory == KMB_MEM_DEVICE ? (F *)C_out : (F *)ws.Cout.ptr;

    std::mt19937 gen(seed);
    std::uniform_real_distribution<F> uni(F(0), F(1));
    std::vector<F> host((size_t)(k + pool_n));
    for (int64_t i = 0; i < k; ++i) host[(size_t)i] = uni(gen);
    for (int i = 0; i < pool_n; ++i) host[(size_t)(k + i)] = uni(gen);
    KMB_CUDA(cudaMemcpyAsync(rnd, host.data(), sizeof(F) * (k + pool_n), cudaMemcpyHostToDevice, s));
    kmb::PPState hs{};
    KMB_CUDA(cudaMemcpyAsync(st, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
    // block-sum publication flags: round c publishes c, so zero means "none yet"
    KMB_CUDA(cudaMemsetAsync(ws.pp_flags.ptr, 0, sizeof(unsigned) * nb, s));
    int64_t row0 = (int64_t)(size_t)(host[0] * F(n));
    if (row0 == n) --row0;
    kmb::launch_pp_fill<F>(md, n, s);
    if (csr)
        kmb::launch_pp_first_csr<F>(*csr, row0, C, st, s);
    else
        kmb::launch_pp_first<F>(X, d, row0, C, s);
    int64_t c_begin = 1;
    bool update_first = true;
    int64_t round_draws = 0;  // resample draws spent on the round that stopped
    for (;;) {
        if (csr)
            kmb::launch_pp_rounds_csr<F>(*csr, k, c_begin, update_first, md, acc, (unsigned *)ws.pp_flags.ptr, rnd,
                                         rnd + k, pool_n, C, st, s);
        else
            kmb::launch_pp_rounds<F>(X, n, d, k, c_begin, update_first, md, acc, (unsigned *)ws.pp_flags.ptr, rnd,
                                     rnd + k, pool_n, C, st, s);
        KMB_CUDA(cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s));
        KMB_CUDA(cudaStreamSynchronize(s));
        if (!hs.stopped) break;
        if (hs.stopped == 3)
            return fail(ctx, KMB_ETIMEDOUT, "k-means++ init: overall-sum fold timed out in round %lld",
                        (long long)hs.stop_round);
        if (hs.stopped == 2)
            return fail(ctx, KMB_EINVAL,
                        "k-means++ init: no row left to sample for center %lld (fewer than k distinct rows, or "
                        "non-finite distances)",
                        (long long)hs.stop_round);
        // the reference keeps drawing until a row with a positive distance is hit; with a
        // positive finite total at least 90% of the mass lies on such rows, so this bound
        // is only reached on broken arithmetic
        round_draws = hs.stop_round == c_begin && !update_first ? round_draws + hs.pool_used : hs.pool_used;
        if (round_draws > (int64_t)1 << 24)
            return fail(ctx, KMB_EINVAL, "k-means++ init: no row with a positive distance found for center %lld",
                        (long long)hs.stop_round);
        for (int i = 0; i < pool_n; ++i) host[(size_t)(k + i)] = uni(gen);
        KMB_CUDA(cudaMemcpyAsync(rnd + k, host.data() + k, sizeof(F) * pool_n, cudaMemcpyHostToDevice, s));
        c_begin = hs.stop_round;
        update_first = false;
        hs.stopped = 0;
        hs.pool_used = 0;
        KMB_CUDA(cudaMemcpyAsync(st, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
    }
    if (memory == KMB_MEM_HOST) {
        KMB_CUDA(cudaMemcpyAsync(C_out, C, sizeof(F) * k * d, cudaMemcpyDeviceToHost, s));
        KMB_CUDA(cudaStreamSynchronize(s));
    }
    return KMB_OK;
}

template <typename F>
int init_plusplus_impl(kmb_context *ctx, int memory, const void *Xv, int64_t n, int64_t d, int64_t k, uint32_t seed,
                       void *C_out) {
    const F *X = (const F *)Xv;
    if (memory == KMB_MEM_HOST) {
        int rc = upload<F>(ctx, ctx->ws.X, Xv, sizeof(F) * n * d, &X);
        if (rc) return rc;
    }
    return init_plusplus_core<F>(ctx, memory, X, nullptr, n, d, k, seed, C_out);
}

template <typename F>
int init_plusplus_csr_impl(kmb_context *ctx, int memory, const void *vals, const int64_t *cols, const int64_t *rowptr,
                           int64_t n, int64_t d, int base, int64_t k, uint32_t seed, void *C_out) {
    kmb::CsrRows X;
    int rc = prepare_csr<F>(ctx, memory, vals, cols, rowptr, n, d, base, &X);
    if (rc) return rc;
    return init_plusplus_core<F>(ctx, memory, nullptr, &X, n, d, k, seed, C_out);
}

extern "C" {

const char *kmb_version(void) { return "onedal_b200 kmeans 0.1 (sm_100a)"; }

int kmb_train_spmd(kmb_context *ctx, int dtype, const void *X, int64_t n, int64_t d, const void *C0,
                   const kmb_params *params, const kmb_communicator *comm, void *C_out, int32_t *labels,
                   double *objective, int64_t *iteration_count) {
    if (!ctx) return KMB_EINVAL;
    ctx->last_error.clear();
    if (!params || !comm || !comm->allreduce_sum_f64 || !comm->allgather || comm->size <= 0 || comm->rank < 0 ||
        comm->rank >= comm->size)
        return fail(ctx, KMB_EINVAL, "bad params or communicator");
    if (dtype != KMB_F32 && dtype != KMB_F64) return fail(ctx, KMB_EINVAL, "unknown dtype %d", dtype);
    if (n <= 0 || n > INT32_MAX || d <= 0) return fail(ctx, KMB_EINVAL, "bad shape");
    kmb_params p = *params;
    if (p.cluster_count <= 0 || p.cluster_count > INT32_MAX || p.max_iteration_count < 0 || !(p.accuracy_threshold >= 0))
        return fail(ctx, KMB_EINVAL, "bad params");
    int rc = check_form(ctx, dtype, p.form);
    if (rc) return rc;
    if (!X || !C0 || !C_out || !labels) return fail(ctx, KMB_EINVAL, "null device pointer");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, KMB_ECUDA, "cudaSetDevice failed");
    p.form = resolve_form(dtype, p.form, n, p.cluster_count, d);
    if (dtype == KMB_F32)
        return train_spmd_impl<float>(ctx, dtype, (const float *)X, n, d, (const float *)C0, p, comm, (float *)C_out,
                                      labels, objective, iteration_count);
    return train_spmd_impl<double>(ctx, dtype, (const double *)X, n, d, (const double *)C0, p, comm,
                                   (double *)C_out, labels, objective, iteration_count);
}

const char *kmb_status_string(int status) {
    switch (status) {
        case KMB_OK: return "ok";
        case KMB_EINVAL: return "invalid argument";
        case KMB_ENOMEM: return "out of device memory";
        case KMB_ECUDA: return "CUDA error";
        case KMB_ETIMEDOUT: return "timed out";
        case KMB_ETOO_MANY_EMPTY: return "number of clusters is too large (too many empty clusters)";
        case KMB_EUNSUPPORTED: return "unsupported";
        case KMB_ECOMM: return "communicator failure";
        default: return "unknown status";
    }
}

int kmb_context_create(int device, kmb_context **out) {
    if (!out) return KMB_EINVAL;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return KMB_ECUDA;
    }
    kmb_context *ctx = new (std::nothrow) kmb_context;
    if (!ctx) return KMB_ENOMEM;
    ctx->device = device;
    ctx->ws.device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost(&ctx->h_state, sizeof(LoopState) * 2) != cudaSuccess) {
        cudaGetLastError();
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return KMB_ECUDA;
    }
    ctx->own_stream = true;
    ctx->ws.stream = ctx->stream;
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    *out = ctx;
    return KMB_OK;
}

int kmb_context_destroy(kmb_context *ctx) {
    if (!ctx) return KMB_EINVAL;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->ws.release();
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->recycle_events();
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->h_state) cudaFreeHost(ctx->h_state);
    delete ctx;
    return KMB_OK;
}

int kmb_context_set_stream(kmb_context *ctx, void *cuda_stream) {
    if (!ctx) return KMB_EINVAL;
    // workspace buffers were allocated in the old stream's order
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = (cudaStream_t)cuda_stream;
    ctx->ws.stream = ctx->stream;
    ctx->own_stream = false;
    return KMB_OK;
}

const char *kmb_context_last_error(const kmb_context *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int kmb_context_release_workspace(kmb_context *ctx) {
    if (!ctx) return KMB_EINVAL;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->ws.release();
    cudaStreamSynchronize(ctx->stream);
    return KMB_OK;
}

int kmb_train(kmb_context *ctx, int dtype, int memory, const void *X, int64_t n, int64_t d, const void *C0,
              const kmb_params *params, void *C_out, int32_t *responses, double *objective, int64_t *iteration_count,
              kmb_stats *stats) {
    if (!ctx || !params) return KMB_EINVAL;
    ctx->last_error.clear();
    int rc = validate_shapes(ctx, dtype, n, d, params->cluster_count);
    if (rc) return rc;
    if (params->max_iteration_count < 0) return fail(ctx, KMB_EINVAL, "max_iteration_count must be >= 0");
    if (!(params->accuracy_threshold >= 0.0)) return fail(ctx, KMB_EINVAL, "accuracy_threshold must be >= 0");
    if ((rc = check_form(ctx, dtype, params->form))) return rc;
    if (!X || !C0) return fail(ctx, KMB_EINVAL, "data and initial centroids are required");
    if (memory != KMB_MEM_HOST && memory != KMB_MEM_DEVICE) return fail(ctx, KMB_EINVAL, "unknown memory kind");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, KMB_ECUDA, "cudaSetDevice failed");
    kmb_params p = *params;
    p.form = resolve_form(dtype, p.form, n, p.cluster_count, d);
    int64_t it_local = 0;
    int64_t *it_out = iteration_count ? iteration_count : &it_local;
    ProfRange range("kmb_train");
    CallLog log("train", n, d, p.cluster_count, p.form, it_out, &rc);
    if (dtype == KMB_F32)
        rc = train_impl<float>(ctx, memory, X, n, d, C0, &p, C_out, responses, objective, it_out, stats);
    else
        rc = train_impl<double>(ctx, memory, X, n, d, C0, &p, C_out, responses, objective, it_out, stats);
    return rc;
}

int kmb_train_csr(kmb_context *ctx, int dtype, int memory, const void *values, const int64_t *col_indices,
                  const int64_t *row_offsets, int64_t n, int64_t d, int32_t indexing, const void *C0,
                  const kmb_params *params, void *C_out, int32_t *responses, double *objective,
                  int64_t *iteration_count, kmb_stats *stats) {
    if (!ctx || !params) return KMB_EINVAL;
    ctx->last_error.clear();
    int rc = validate_shapes(ctx, dtype, n, d, params->cluster_count);
    if (rc) return rc;
    if (params->max_iteration_count < 0) return fail(ctx, KMB_EINVAL, "max_iteration_count must be >= 0");
    if (!(params->accuracy_threshold >= 0.0)) return fail(ctx, KMB_EINVAL, "accuracy_threshold must be >= 0");
    if (params->form != KMB_FORM_PLAIN) return fail(ctx, KMB_EINVAL, "CSR rows take the plain form");
    if (!C0) return fail(ctx, KMB_EINVAL, "initial centroids are required");
    if ((rc = validate_csr_call(ctx, dtype, memory, values, col_indices, row_offsets, indexing))) return rc;
    if (dtype == KMB_F32)
        return train_csr_impl<float>(ctx, memory, values, col_indices, row_offsets, n, d, indexing, C0, params, C_out,
                                     responses, objective, iteration_count, stats);
    return train_csr_impl<double>(ctx, memory, values, col_indices, row_offsets, n, d, indexing, C0, params, C_out,
                                  responses, objective, iteration_count, stats);
}

int kmb_infer_csr(kmb_context *ctx, int dtype, int memory, const void *values, const int64_t *col_indices,
                  const int64_t *row_offsets, int64_t n, int64_t d, int32_t indexing, const void *C, int64_t k,
                  int32_t compute_objective, int32_t *responses, double *objective) {
    if (!ctx) return KMB_EINVAL;
    ctx->last_error.clear();
    if (n <= 0) return fail(ctx, KMB_EINVAL, "input data is empty");
    if (n > INT32_MAX) return fail(ctx, KMB_EINVAL, "row count exceeds INT32_MAX");
    if (d <= 0 || k <= 0 || k > INT32_MAX) return fail(ctx, KMB_EINVAL, "bad centroid shape");
    if (!C) return fail(ctx, KMB_EINVAL, "centroids are required");
    int rc = validate_csr_call(ctx, dtype, memory, values, col_indices, row_offsets, indexing);
    if (rc) return rc;
    if (dtype == KMB_F32)
        return infer_csr_impl<float>(ctx, memory, values, col_indices, row_offsets, n, d, indexing, C, k,
                                     compute_objective, responses, objective);
    return infer_csr_impl<double>(ctx, memory, values, col_indices, row_offsets, n, d, indexing, C, k,
                                  compute_objective, responses, objective);
}

int kmb_init_plusplus(kmb_context *ctx, int dtype, int memory, const void *X, int64_t n, int64_t d, int64_t k,
                      uint32_t seed, void *C_out) {
    if (!ctx) return KMB_EINVAL;
    ctx->last_error.clear();
    cudaSetDevice(ctx->device);
    if (!X || !C_out || n <= 0 || d <= 0 || k <= 0) return fail(ctx, KMB_EINVAL, "bad argument");
    if (k > n) return fail(ctx, KMB_EINVAL, "cluster_count %lld exceeds the row count %lld", (long long)k, (long long)n);
    if (memory != KMB_MEM_HOST && memory != KMB_MEM_DEVICE) return fail(ctx, KMB_EINVAL, "unknown memory kind");
    if (dtype == KMB_F32) return init_plusplus_impl<float>(ctx, memory, X, n, d, k, seed, C_out);
    if (dtype == KMB_F64) return init_plusplus_impl<double>(ctx, memory, X, n, d, k, seed, C_out);
    return fail(ctx, KMB_EINVAL, "unknown dtype");
}

int kmb_init_plusplus_csr(kmb_context *ctx, int dtype, int memory, const void *values, const int64_t *col_indices,
                          const int64_t *row_offsets, int64_t n, int64_t d, int32_t indexing, int64_t k, uint32_t seed,
                          void *C_out) {
    if (!ctx) return KMB_EINVAL;
    ctx->last_error.clear();
    if (!C_out || n <= 0 || d <= 0 || k <= 0) return fail(ctx, KMB_EINVAL, "bad argument");
    if (k > n) return fail(ctx, KMB_EINVAL, "cluster_count %lld exceeds the row count %lld", (long long)k, (long long)n);
    int rc = validate_csr_call(ctx, dtype, memory, values, col_indices, row_offsets, indexing);
    if (rc) return rc;
    if (dtype == KMB_F32)
        return init_plusplus_csr_impl<float>(ctx, memory, values, col_indices, row_offsets, n, d, indexing, k, seed,
                                             C_out);
    return init_plusplus_csr_impl<double>(ctx, memory, values, col_indices, row_offsets, n, d, indexing, k, seed, C_out);
}

int kmb_infer(kmb_context *ctx, int dtype, int memory, const void *X, int64_t n, int64_t d, const void *C, int64_t k,
              int32_t form, int32_t compute_objective, int32_t *responses, double *objective, kmb_stats *stats) {
    if (!ctx) return KMB_EINVAL;
    ctx->last_error.clear();
    if (dtype != KMB_F32 && dtype != KMB_F64) return fail(ctx, KMB_EINVAL, "unknown dtype %d", dtype);
    if (n <= 0) return fail(ctx, KMB_EINVAL, "input data is empty");
    if (n > INT32_MAX) return fail(ctx, KMB_EINVAL, "row count exceeds INT32_MAX");
    if (d <= 0 || k <= 0 || k > INT32_MAX) return fail(ctx, KMB_EINVAL, "bad centroid shape");
    int rc = check_form(ctx, dtype, form);
    if (rc) return rc;
    if (!X || !C) return fail(ctx, KMB_EINVAL, "data and centroids are required");
    if (memory != KMB_MEM_HOST && memory != KMB_MEM_DEVICE) return fail(ctx, KMB_EINVAL, "unknown memory kind");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, KMB_ECUDA, "cudaSetDevice failed");
    form = resolve_form(dtype, form, n, k, d);
    ProfRange range("kmb_infer");
    CallLog log("infer", n, d, k, form, nullptr, &rc);
    if (dtype == KMB_F32)
        rc = infer_impl<float>(ctx, memory, X, n, d, C, k, form, compute_objective, responses, objective, stats);
    else
        rc = infer_impl<double>(ctx, memory, X, n, d, C, k, form, compute_objective, responses, objective, stats);
    return rc;
}

int kmb_lloyd_step(kmb_context *ctx, int dtype, const void *X, int64_t n, int64_t d, const void *C_in, int64_t k,
                   int32_t form, int32_t recheck, void *C_out, int32_t *labels, double *shift, int64_t *n_empty) {
    if (!ctx) return KMB_EINVAL;
    ctx->last_error.clear();
    int rc = validate_shapes(ctx, dtype, n, d, k);
    if (rc) return rc;
    if ((rc = check_form(ctx, dtype, form))) return rc;
    if (!X || !C_in || !C_out || !labels) return fail(ctx, KMB_EINVAL, "null device pointer");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, KMB_ECUDA, "cudaSetDevice failed");
    form = resolve_form(dtype, form, n, k, d);
    if (dtype == KMB_F32) return step_impl<float>(ctx, X, n, d, C_in, k, form, recheck, C_out, labels, shift, n_empty);
    return step_impl<double>(ctx, X, n, d, C_in, k, form, recheck, C_out, labels, shift, n_empty);
}

int kmb_lloyd_iterate(kmb_context *ctx, int dtype, const void *X, int64_t n, int64_t d, void *C,
                      const kmb_params *params, int32_t *labels, int64_t *iteration_count, kmb_stats *stats) {
    if (!ctx || !params) return KMB_EINVAL;
    ctx->last_error.clear();
    int rc = validate_shapes(ctx, dtype, n, d, params->cluster_count);
    if (rc) return rc;
    if (params->max_iteration_count < 0) return fail(ctx, KMB_EINVAL, "max_iteration_count must be >= 0");
    if (!(params->accuracy_threshold >= 0.0)) return fail(ctx, KMB_EINVAL, "accuracy_threshold must be >= 0");
    if ((rc = check_form(ctx, dtype, params->form))) return rc;
    if (!X || !C) return fail(ctx, KMB_EINVAL, "null device pointer");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, KMB_ECUDA, "cudaSetDevice failed");
    kmb_params p = *params;
    p.form = resolve_form(dtype, p.form, n, p.cluster_count, d);
    if (dtype == KMB_F32) return iterate_impl<float>(ctx, X, n, d, C, &p, labels, iteration_count, stats);
    return iterate_impl<double>(ctx, X, n, d, C, &p, labels, iteration_count, stats);
}

int kmb_context_set_max_sms(kmb_context *ctx, int max_sms) {
    if (!ctx || max_sms < -1) return KMB_EINVAL;
    int all = 148;
    cudaDeviceGetAttribute(&all, cudaDevAttrMultiProcessorCount, ctx->device);
    ctx->tc_per_tile = max_sms == -1;
    ctx->num_sms = (max_sms <= 0 || max_sms > all) ? all : max_sms;
    return KMB_OK;
}

int kmb_context_set_kernel_timing(kmb_context *ctx, int enabled) {
    if (!ctx) return KMB_EINVAL;
    cudaStreamSynchronize(ctx->stream);
    ctx->recycle_events();
    ctx->timing = enabled != 0;
    ctx->launches_at_enable = kmb::launch_count();
    return KMB_OK;
}

int kmb_context_kernel_time(kmb_context *ctx, int kernel, double *total_ms, int64_t *launches) {
    if (!ctx || kernel < 0 || kernel > 4) return KMB_EINVAL;
    if (kernel == 3) {
        // every kernel launched by this thread since timing was enabled
        if (total_ms) *total_ms = 0.0;
        if (launches) *launches = kmb::launch_count() - ctx->launches_at_enable;
        return KMB_OK;
    }
    double tot = 0.0;
    for (auto &pr : ctx->ev_used[kernel]) {
        if (cudaEventSynchronize(pr.second) != cudaSuccess) return cuda_fail(ctx, cudaGetLastError(), "event");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, pr.first, pr.second);
        tot += ms;
    }
    if (total_ms) *total_ms = tot;
    if (launches) *launches = (int64_t)ctx->ev_used[kernel].size();
    return KMB_OK;
}

int kmb_context_recheck_rows(kmb_context *ctx, int32_t *rows_out, int64_t capacity, int64_t *count) {
    if (!ctx || !count || capacity < 0 || (capacity > 0 && !rows_out)) return KMB_EINVAL;
    ctx->last_error.clear();
    *count = 0;
    if (!ctx->queue_state || !ctx->ws.queue.ptr) return KMB_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, KMB_ECUDA, "cudaSetDevice failed");
    cudaStream_t s = ctx->stream;
    LoopState hs;
    KMB_CUDA(cudaMemcpyAsync(&hs, ctx->queue_state, sizeof(LoopState), cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaStreamSynchronize(s));
    *count = (int64_t)hs.n_recheck + hs.n_full;
    if (capacity > 0 && *count > 0) {
        const int64_t m = std::min(*count, capacity);
        gather_queue_rows_kernel<<<(unsigned)std::min<int64_t>((m + 255) / 256, 1024), 256, 0, s>>>(
            (const RecheckEntry *)ctx->ws.queue.ptr, ctx->queue_rows, ctx->queue_state, rows_out, capacity);
        KMB_LAUNCHED();
        KMB_CUDA(cudaGetLastError());
        KMB_CUDA(cudaStreamSynchronize(s));
    }
    return KMB_OK;
}

int kmb_partial_sums(kmb_context *ctx, int dtype, const void *X, int64_t n, int64_t d, const void *C, int64_t k,
                     int32_t form, int32_t *labels, double *sums, int64_t *counts, double *sq_distances,
                     void *row_sq_distance) {
    if (!ctx) return KMB_EINVAL;
    ctx->last_error.clear();
    if (dtype != KMB_F32 && dtype != KMB_F64) return fail(ctx, KMB_EINVAL, "unknown dtype %d", dtype);
    if (n <= 0 || n > INT32_MAX || d <= 0 || k <= 0 || k > INT32_MAX) return fail(ctx, KMB_EINVAL, "bad shape");
    int rc = check_form(ctx, dtype, form);
    if (rc) return rc;
    if (!X || !C || !labels || !sums || !counts) return fail(ctx, KMB_EINVAL, "null device pointer");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, KMB_ECUDA, "cudaSetDevice failed");
    form = resolve_form(dtype, form, n, k, d);
    if (dtype == KMB_F32)
        return partial_impl<float>(ctx, (const float *)X, n, d, (const float *)C, k, form, labels, sums, counts,
                                   sq_distances, (float *)row_sq_distance);
    return partial_impl<double>(ctx, (const double *)X, n, d, (const double *)C, k, form, labels, sums, counts,
                                sq_distances, (double *)row_sq_distance);
}

int kmb_finalize_centroids(kmb_context *ctx, int dtype, const double *sums, const int64_t *counts, const void *C_in,
                           int64_t k, int64_t d, void *C_out, double *shift, int32_t *empty_ids, int64_t *n_empty) {
    if (!ctx) return KMB_EINVAL;
    ctx->last_error.clear();
    if (dtype != KMB_F32 && dtype != KMB_F64) return fail(ctx, KMB_EINVAL, "unknown dtype %d", dtype);
    if (k <= 0 || d <= 0 || !sums || !counts || !C_in || !C_out || !empty_ids)
        return fail(ctx, KMB_EINVAL, "bad arguments");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, KMB_ECUDA, "cudaSetDevice failed");
    kmb::Workspace &ws = ctx->ws;
    if (!ws.ensure(ws.shift_part, sizeof(double) * k) || !ws.ensure(ws.empty_flag, sizeof(int32_t) * k) ||
        !ws.ensure(ws.scalars, sizeof(kmb::DevScalars)))
        return fail(ctx, KMB_ENOMEM, "finalize buffers");
    cudaStream_t s = ctx->stream;
    kmb::DevScalars *sc = (kmb::DevScalars *)ws.scalars.ptr;
    double *shift_dev = &sc->objective;
    long long *ne_dev = (long long *)&sc->pad;
    if (dtype == KMB_F32)
        kmb::launch_finalize_from_sums<float>(sums, counts, (const float *)C_in, (float *)C_out, k, d, ws, shift_dev,
                                              empty_ids, ne_dev, s);
    else
        kmb::launch_finalize_from_sums<double>(sums, counts, (const double *)C_in, (double *)C_out, k, d, ws,
                                               shift_dev, empty_ids, ne_dev, s);
    double hv[2];
    KMB_CUDA(cudaMemcpyAsync(hv, shift_dev, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
    KMB_CUDA(cudaStreamSynchronize(s));
    if (shift) *shift = hv[0];
    long long ne = 0;
    std::memcpy(&ne, &hv[1], sizeof(ne));
    if (n_empty) *n_empty = ne;
    return KMB_OK;
}

}  // extern "C"
