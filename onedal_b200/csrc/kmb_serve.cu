// Serving loop: fitted centroid sets stay resident in HBM; infer and small
// train requests of different n, k and d are admitted under an HBM budget and
// batched, as they arrive, into shared launches on several streams.
//
// Structure (host, C++):
//  * models   -- centroids plus their prepared transposed copy and half norms,
//                kept on the device for the server's lifetime;
//  * admission -- a request is admitted when its device bytes fit in the budget
//                next to everything in flight; otherwise it waits, in FIFO
//                order, until completions free memory;
//  * lanes    -- L CUDA streams. The scheduler thread fills a free lane with
//                every admissible pending infer request (continuous batching:
//                requests that arrived while earlier batches run are picked up
//                by the next free lane), uploads their rows, runs one grouped
//                assignment launch over all of them (kmb_serve_kernels.cu) and
//                copies the labels back, then records an event; the lane's
//                completion thread sleeps on that event (blocking sync), marks
//                the batch complete and returns its memory to the budget.
//                Batches on different lanes overlap on the device;
//  * tensor-core worker -- infer requests large enough for the tensor cores
//                (d <= 256, n * kpad * dpad >= KMB_SERVER_TC_MACS) skip the
//                grouped lanes and run on kTcWorkers worker threads, each with its own
//                context: BF16x3 form with the FP64 recheck, in row chunks of at
//                most kTcChunkRows, its assignment launched as one short CTA
//                per 128-row tile (kmb_context_set_max_sms(-1)). A large
//                request therefore never holds a batch of small ones, and lane
//                launches interleave with it at tile granularity. The workers'
//                workspaces are reserved in the budget once, at creation;
//  * trainers -- small train requests run on worker threads, each with its own
//                kmb_context (workspace) on a low-priority stream, concurrently
//                with the lanes.
// Latency is measured on the host from submit to completion (steady_clock).
// With KMB_SERVE_TRACE=<file> in the environment, the server appends one line
// per finished request (R ...) and per lane batch (B ...) to that file, times
// in microseconds since the server was created.
#include "kmb_internal.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

namespace kmb {
void launch_grouped_infer(const void *reqs_dev, int nreq, long long n_items, long long total_rows, cudaStream_t s);
size_t grouped_desc_bytes();
int grouped_chunk_clusters();
namespace serve {
struct ReqDesc {
    const float *X;
    const float *Ct;
    const float *h;
    unsigned long long *key;
    int32_t *labels;
    long long n;
    int d, k, kpad, chunks;
    long long item_begin;
    long long row_begin;
};
}  // namespace serve
}  // namespace kmb

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { PENDING = 0, RUNNING = 1, DONE = 2, FAILED = 3 };
enum ReqKind { INFER = 0, TRAIN = 1 };

struct Model {
    int64_t k, d, kpad, dpad;
    float *C = nullptr, *Ct = nullptr, *h = nullptr;
};

constexpr int64_t kTcChunkRows = 1 << 18;
constexpr size_t kTcReserveBytes = (size_t)448 << 20;  // one worker's workspace at kTcChunkRows rows, d <= 256
constexpr int kTcWorkers = 2;  // default; KMB_SERVER_TC_WORKERS (1 .. 8) overrides
constexpr double kBatchMacs = 4294967296.0;      // cap on a lane batch's n * kpad * dpad (one large request may exceed it alone)

struct Request {
    int64_t id;
    int kind;
    int form = KMB_FORM_PLAIN;
    bool srv_trace = false;  // the server traces: time the tensor-core phases
    int model;
    int64_t n, d, k, iters;
    const float *X;
    const float *C0;
    int32_t *labels_out;
    float *C_out;
    size_t bytes;
    int state = PENDING;
    int rc = KMB_OK;
    Clock::time_point t_submit, t_start, t_done;  // t_start: admitted and dispatched
    // device buffers while running (infer)
    float *dX = nullptr;
    unsigned long long *dkey = nullptr;
    int32_t *dlab = nullptr;
    int64_t lab_off = 0;  // offset in the lane's pinned label staging
    double us_h2d = 0, us_compute = 0, us_d2h = 0;  // tensor-core worker phases (trace)
    double ms_tc = 0, ms_recheck = 0;                // device time of the assignment / recheck kernels (trace)
};

struct Lane;

struct Server {
    int device = 0;
    int64_t tc_chunk_rows = kTcChunkRows;  // KMB_SERVER_TC_CHUNK_ROWS (4096 .. kTcChunkRows)
    int tc_sms = -1;                       // KMB_SERVER_TC_SMS: the workers' kmb_context_set_max_sms
    int tc_workers = kTcWorkers;
    size_t budget = 0;
    size_t in_use = 0, peak_in_use = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request *> pending;      // infer, FIFO
    std::deque<Request *> train_queue;  // train, FIFO
    std::deque<Request *> tc_queue;     // large infer, FIFO (tensor-core worker)
    bool tc_enabled = false;
    int tc_busy = 0;                    // tensor-core workers running a request
    size_t base_use = 0;                // permanent reservation (tensor-core worker workspaces)
    int prio_low = 0, prio_high = 0;
    int64_t tc_requests = 0;
    std::unordered_map<int64_t, Request *> all;
    std::vector<Model> models;
    std::vector<Lane *> lanes;
    std::vector<std::thread> threads;
    bool stop = false;
    int64_t next_id = 1;
    int64_t batches = 0, batched_requests = 0, completed = 0, failed = 0;
    int64_t max_batch_rows = 1 << 22;
    Clock::time_point t0 = Clock::now();
    FILE *trace = nullptr;  // KMB_SERVE_TRACE
    double us(Clock::time_point t) const { return std::chrono::duration<double, std::micro>(t - t0).count(); }
};

struct Lane {
    Server *srv;
    cudaStream_t stream = nullptr;
    bool busy = false;
    std::vector<Request *> batch;
    kmb::serve::ReqDesc *h_desc = nullptr;  // pinned
    void *d_desc = nullptr;
    int cap = 0;
    // Pinned staging for the batch's labels: the device->host copy stays
    // asynchronous (a copy into pageable memory would block the scheduler
    // thread until the batch finished), and the completion callback moves
    // each request's labels into the caller's buffer.
    int32_t *h_lab = nullptr;
    int64_t h_lab_cap = 0;
    // Pinned buffers replaced by larger ones: freed when the server is destroyed,
    // because cudaFreeHost (like cudaFree) waits for the whole device, which here
    // would stall every stream's work behind the scheduler thread.
    std::vector<void *> retired_host;
    // Device arena for a batch's rows, keys and labels, reused batch after batch
    // and grown (stream-ordered, geometrically) only when a batch needs more: a
    // stream-ordered allocation per request stalled the scheduler thread for up to
    // 54 ms when the shared pool had to grow while other threads allocated.
    void *arena = nullptr;
    size_t arena_bytes = 0;
    int index = 0;
    cudaEvent_t done_ev = nullptr;  // recorded after the batch's last copy
    bool in_flight = false;         // a launched batch awaits its completion thread
    std::thread completer;
    Clock::time_point t_launch, t_launched;  // host time around launch_batch
    double us_alloc = 0, us_h2d = 0, us_kernel = 0, us_tail = 0, us_d2h = 0, us_free = 0;  // host time inside launch_batch
};

int serve_form(const Server *srv, const Model &m, int64_t n) {
    if (!srv->tc_enabled || m.d > 256) return KMB_FORM_PLAIN;
    const int64_t kpad = (m.k + 127) / 128 * 128, dpad = (m.d + 63) / 64 * 64;
    return (double)n * (double)kpad * (double)dpad >= (double)KMB_SERVER_TC_MACS ? KMB_FORM_BF16X3 : KMB_FORM_PLAIN;
}

size_t infer_bytes(int64_t n, int64_t d) { return (size_t)n * d * 4 + (size_t)n * 8 + (size_t)n * 4 + 4096; }
size_t train_bytes(int64_t n, int64_t d, int64_t k) {
    // rows + the context workspace of a small train (labels, sort buffers, records)
    return (size_t)n * d * 4 + (size_t)n * 40 + (size_t)k * d * 64 + (size_t)(n / 512 + k) * d * 8 + (8u << 20);
}

void batch_done(Lane *lane) {
    Server *srv = lane->srv;
    for (Request *r : lane->batch)
        if (r->rc == KMB_OK) std::memcpy(r->labels_out, lane->h_lab + r->lab_off, sizeof(int32_t) * r->n);
    std::lock_guard<std::mutex> lock(srv->mu);
    const auto now = Clock::now();
    for (Request *r : lane->batch) {
        r->t_done = now;
        r->state = r->rc == KMB_OK ? DONE : FAILED;
        srv->in_use -= r->bytes;
        srv->completed += 1;
        if (r->rc != KMB_OK) srv->failed += 1;
    }
    if (srv->trace) {
        int64_t rows = 0;
        for (Request *r : lane->batch) rows += r->n;
        std::fprintf(srv->trace,
                     "B lane=%d nreq=%zu rows=%lld launch=%.1f launched=%.1f done=%.1f alloc=%.1f h2d=%.1f kern=%.1f "
                     "tail=%.1f d2h=%.1f free=%.1f\n",
                     lane->index, lane->batch.size(), (long long)rows, srv->us(lane->t_launch),
                     srv->us(lane->t_launched), srv->us(now), lane->us_alloc, lane->us_h2d, lane->us_kernel,
                     lane->us_tail, lane->us_d2h, lane->us_free);
    }
    lane->batch.clear();
    lane->busy = false;
    lane->in_flight = false;
    srv->cv.notify_all();
}

// One per lane: waits (sleeping, not spinning) for the lane's batch event.
void completer_loop(Lane *lane) {
    Server *srv = lane->srv;
    cudaSetDevice(srv->device);
    std::unique_lock<std::mutex> lock(srv->mu);
    while (true) {
        srv->cv.wait(lock, [&] { return srv->stop || lane->in_flight; });
        if (!lane->in_flight) break;  // stop with nothing in flight
        lock.unlock();
        cudaEventSynchronize(lane->done_ev);
        batch_done(lane);
        lock.lock();
    }
}

// Runs on the scheduler thread with the server lock released.
int launch_batch(Server *srv, Lane *lane) {
    cudaStream_t s = lane->stream;
    const int nreq = (int)lane->batch.size();
    if (nreq > lane->cap) {
        // grow without any device-wide synchronisation: a new pinned block (the old
        // one is retired), the device copy in stream order
        const int cap = std::max(nreq, 2 * lane->cap);
        void *h = nullptr, *dv = nullptr;
        if (cudaMallocHost(&h, sizeof(kmb::serve::ReqDesc) * cap) != cudaSuccess ||
            kmb::pool_alloc(&dv, sizeof(kmb::serve::ReqDesc) * cap, srv->device, s) != cudaSuccess) {
            cudaGetLastError();
            if (h) lane->retired_host.push_back(h);
            return KMB_ENOMEM;
        }
        if (lane->h_desc) lane->retired_host.push_back(lane->h_desc);
        if (lane->d_desc) cudaFreeAsync(lane->d_desc, s);
        lane->h_desc = (kmb::serve::ReqDesc *)h;
        lane->d_desc = dv;
        lane->cap = cap;
    }
    int64_t batch_rows = 0;
    for (Request *r : lane->batch) batch_rows += r->n;
    if (batch_rows > lane->h_lab_cap) {
        const int64_t cap = std::max<int64_t>(batch_rows, 2 * lane->h_lab_cap);
        int32_t *h = nullptr;
        if (cudaMallocHost(&h, sizeof(int32_t) * cap) != cudaSuccess) {
            cudaGetLastError();
            return KMB_ENOMEM;
        }
        if (lane->h_lab) lane->retired_host.push_back(lane->h_lab);
        lane->h_lab = h;
        lane->h_lab_cap = cap;
    }
    const int chunk = kmb::grouped_chunk_clusters();
    auto a256 = [](size_t b) { return (b + 255) / 256 * 256; };
    size_t need = 0;
    for (Request *r : lane->batch)
        need += a256(sizeof(float) * r->n * r->d) + a256(sizeof(unsigned long long) * r->n) +
                a256(sizeof(int32_t) * r->n);
    const auto ta0 = Clock::now();
    if (need > lane->arena_bytes) {
        const size_t bytes = std::max(need, 2 * lane->arena_bytes);
        void *a = nullptr;
        if (kmb::pool_alloc(&a, bytes, srv->device, s) != cudaSuccess) {
            cudaGetLastError();
            return KMB_ENOMEM;
        }
        if (lane->arena) cudaFreeAsync(lane->arena, s);  // after the lane's previous batches
        lane->arena = a;
        lane->arena_bytes = bytes;
    }
    lane->us_alloc += std::chrono::duration<double, std::micro>(Clock::now() - ta0).count();
    char *cursor = (char *)lane->arena;
    long long items = 0, rows = 0;
    for (int i = 0; i < nreq; ++i) {
        Request *r = lane->batch[i];
        const Model &m = srv->models[r->model];
        const auto ta = Clock::now();
        r->dX = (float *)cursor;
        cursor += a256(sizeof(float) * r->n * r->d);
        r->dkey = (unsigned long long *)cursor;
        cursor += a256(sizeof(unsigned long long) * r->n);
        r->dlab = (int32_t *)cursor;
        cursor += a256(sizeof(int32_t) * r->n);
        const auto tb = Clock::now();
        cudaMemcpyAsync(r->dX, r->X, sizeof(float) * r->n * r->d, cudaMemcpyHostToDevice, s);
        const auto tc = Clock::now();
        lane->us_alloc += std::chrono::duration<double, std::micro>(tb - ta).count();
        lane->us_h2d += std::chrono::duration<double, std::micro>(tc - tb).count();
        kmb::serve::ReqDesc &q = lane->h_desc[i];
        q.X = r->dX;
        q.Ct = m.Ct;
        q.h = m.h;
        q.key = r->dkey;
        q.labels = r->dlab;
        q.n = r->n;
        q.d = (int)r->d;
        q.k = (int)m.k;
        q.kpad = (int)m.kpad;
        q.chunks = (int)((m.kpad + chunk - 1) / chunk);
        q.item_begin = items;
        q.row_begin = rows;
        r->lab_off = rows;
        items += ((r->n + 127) / 128) * q.chunks;
        rows += r->n;
    }
    const auto tk0 = Clock::now();
    cudaMemcpyAsync(lane->d_desc, lane->h_desc, sizeof(kmb::serve::ReqDesc) * nreq, cudaMemcpyHostToDevice, s);
    kmb::launch_grouped_infer(lane->d_desc, nreq, items, rows, s);
    const auto tk1 = Clock::now();
    lane->us_kernel += std::chrono::duration<double, std::micro>(tk1 - tk0).count();
    for (Request *r : lane->batch) {
        const auto t0 = Clock::now();
        cudaMemcpyAsync(lane->h_lab + r->lab_off, r->dlab, sizeof(int32_t) * r->n, cudaMemcpyDeviceToHost, s);
        const auto t1 = Clock::now();
        lane->us_d2h += std::chrono::duration<double, std::micro>(t1 - t0).count();
        lane->us_free += std::chrono::duration<double, std::micro>(Clock::now() - t1).count();
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        for (Request *r : lane->batch) r->rc = KMB_ECUDA;
    }
    cudaEventRecord(lane->done_ev, s);
    lane->us_tail += std::chrono::duration<double, std::micro>(Clock::now() - tk1).count();
    return KMB_OK;
}

void scheduler_loop(Server *srv) {
    cudaSetDevice(srv->device);
    std::unique_lock<std::mutex> lock(srv->mu);
    while (true) {
        Lane *lane = nullptr;
        srv->cv.wait(lock, [&] {
            if (srv->stop) return true;
            if (srv->pending.empty()) return false;
            for (Lane *l : srv->lanes)
                if (!l->busy) {
                    lane = l;
                    break;
                }
            if (!lane) return false;
            // admission of at least the head request
            return srv->in_use + srv->pending.front()->bytes <= srv->budget || srv->in_use == srv->base_use;
        });
        if (srv->stop) break;
        // Continuous batching: take every admissible pending request (FIFO).
        int64_t rows = 0;
        double macs = 0.0;
        while (!srv->pending.empty()) {
            Request *r = srv->pending.front();
            if (srv->in_use + r->bytes > srv->budget && !(srv->in_use == srv->base_use && lane->batch.empty())) break;
            const Model &m = srv->models[r->model];
            const double w = (double)r->n * (double)((m.k + 127) / 128 * 128) * (double)((m.d + 7) / 8 * 8);
            // a batch ends when it is large enough: small requests behind it go to the next free lane
            if (!lane->batch.empty() && (rows + r->n > srv->max_batch_rows || macs + w > kBatchMacs)) break;
            macs += w;
            srv->pending.pop_front();
            r->state = RUNNING;
            r->t_start = Clock::now();
        r->t_start = Clock::now();
            srv->in_use += r->bytes;
            srv->peak_in_use = std::max(srv->peak_in_use, srv->in_use);
            rows += r->n;
            lane->batch.push_back(r);
        }
        if (lane->batch.empty()) continue;
        lane->busy = true;
        srv->batches += 1;
        srv->batched_requests += (int64_t)lane->batch.size();
        lock.unlock();
        lane->us_alloc = lane->us_h2d = lane->us_kernel = lane->us_tail = lane->us_d2h = lane->us_free = 0;
        lane->t_launch = Clock::now();
        const int rc = launch_batch(srv, lane);
        lane->t_launched = Clock::now();
        if (rc != KMB_OK) {
            // Release what was allocated and complete the batch as failed, in stream order.
            for (Request *r : lane->batch) r->rc = rc;  // (rows live in the lane's arena)
            cudaEventRecord(lane->done_ev, lane->stream);
        }
        lock.lock();
        lane->in_flight = true;
        srv->cv.notify_all();
    }
}

// Host<->device copy in pieces of at most 8 MiB: a copy engine works through a
// stream's copies in order, so a 300 MB upload in one piece held a small
// request's 100 KB upload on another stream for milliseconds.
cudaError_t copy_in_pieces(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
    const size_t piece = (size_t)8 << 20;
    for (size_t off = 0; off < bytes; off += piece) {
        const cudaError_t e = cudaMemcpyAsync((char *)dst + off, (const char *)src + off, std::min(piece, bytes - off),
                                              kind, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Large infer request on the tensor-core worker: rows uploaded once, then
// kmb_infer (BF16x3, FP64 recheck) over row chunks on the worker's stream.
// The request's rows and labels live in the worker's arena, grown (stream-ordered,
// geometrically) only when a request needs more.
int run_tc_request(kmb_context *ctx, int dev, cudaStream_t s, const Model &m, Request *r, int64_t chunk_rows,
                   void *&arena, size_t &arena_bytes) {
    const size_t xbytes = (sizeof(float) * r->n * r->d + 255) / 256 * 256;
    const size_t need = xbytes + sizeof(int32_t) * r->n;
    if (need > arena_bytes) {
        void *a = nullptr;
        const size_t bytes = std::max(need, 2 * arena_bytes);
        if (kmb::pool_alloc(&a, bytes, dev, s) != cudaSuccess) {
            cudaGetLastError();
            return KMB_ENOMEM;
        }
        if (arena) cudaFreeAsync(arena, s);
        arena = a;
        arena_bytes = bytes;
    }
    float *dX = (float *)arena;
    int32_t *dlab = (int32_t *)((char *)arena + xbytes);
    int rc = KMB_OK;
    const auto t0 = Clock::now();
    if (copy_in_pieces(dX, r->X, sizeof(float) * r->n * r->d, cudaMemcpyHostToDevice, s) != cudaSuccess)
        rc = KMB_ECUDA;
    const bool timed = r->srv_trace;
    if (timed) {
        cudaStreamSynchronize(s);
        kmb_context_set_kernel_timing(ctx, 1);
    }
    const auto t1 = Clock::now();
    for (int64_t off = 0; rc == KMB_OK && off < r->n; off += chunk_rows) {
        const int64_t rows = std::min<int64_t>(chunk_rows, r->n - off);
        rc = kmb_infer(ctx, KMB_F32, KMB_MEM_DEVICE, dX + off * r->d, rows, r->d, m.C, m.k, KMB_FORM_BF16X3, 0,
                       dlab + off, nullptr, nullptr);
    }
    const auto t2 = Clock::now();
    if (rc == KMB_OK &&
        cudaMemcpyAsync(r->labels_out, dlab, sizeof(int32_t) * r->n, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        rc = KMB_ECUDA;
    if (timed) {
        cudaStreamSynchronize(s);
        const auto t3 = Clock::now();
        r->us_h2d = std::chrono::duration<double, std::micro>(t1 - t0).count();
        r->us_compute = std::chrono::duration<double, std::micro>(t2 - t1).count();
        r->us_d2h = std::chrono::duration<double, std::micro>(t3 - t2).count();
        int64_t nl = 0;
        kmb_context_kernel_time(ctx, 1, &r->ms_tc, &nl);
        kmb_context_kernel_time(ctx, 4, &r->ms_recheck, &nl);
        kmb_context_set_kernel_timing(ctx, 0);
    }
    if (cudaStreamSynchronize(s) != cudaSuccess && rc == KMB_OK) rc = KMB_ECUDA;
    return rc;
}

void tc_worker_loop(Server *srv) {
    cudaSetDevice(srv->device);
    kmb_context *ctx = nullptr;
    cudaStream_t ts = nullptr;
    if (kmb_context_create(srv->device, &ctx) != KMB_OK) ctx = nullptr;
    void *arena = nullptr;
    size_t arena_bytes = 0;
    // Same priority as the lanes: a lower one let a stream of small launches
    // starve the persistent CTAs (which need whole SMs) for tens of ms.
    if (ctx && cudaStreamCreateWithPriority(&ts, cudaStreamNonBlocking, srv->prio_high) == cudaSuccess) {
        kmb_context_set_stream(ctx, ts);
        kmb_context_set_max_sms(ctx, srv->tc_sms);
    } else if (ctx) {
        kmb_context_destroy(ctx);
        ctx = nullptr;
    }
    std::unique_lock<std::mutex> lock(srv->mu);
    while (true) {
        srv->cv.wait(lock, [&] {
            if (srv->stop) return true;
            if (srv->tc_queue.empty()) return false;
            return srv->in_use + srv->tc_queue.front()->bytes <= srv->budget || srv->in_use == srv->base_use;
        });
        if (srv->stop) break;
        Request *r = srv->tc_queue.front();
        srv->tc_queue.pop_front();
        r->state = RUNNING;
        r->t_start = Clock::now();
        srv->in_use += r->bytes;
        srv->peak_in_use = std::max(srv->peak_in_use, srv->in_use);
        srv->tc_busy += 1;
        const Model m = srv->models[r->model];
        lock.unlock();
        const int rc = ctx ? run_tc_request(ctx, srv->device, ts, m, r, srv->tc_chunk_rows, arena, arena_bytes) : KMB_ECUDA;
        lock.lock();
        r->rc = rc;
        r->t_done = Clock::now();
        r->state = rc == KMB_OK ? DONE : FAILED;
        srv->in_use -= r->bytes;
        srv->completed += 1;
        srv->tc_requests += 1;
        if (rc != KMB_OK) srv->failed += 1;
        srv->tc_busy -= 1;
        srv->cv.notify_all();
    }
    lock.unlock();
    if (arena) {
        cudaFreeAsync(arena, ts);
        cudaStreamSynchronize(ts);
    }
    if (ctx) kmb_context_destroy(ctx);
    if (ts) cudaStreamDestroy(ts);
}

void trainer_loop(Server *srv) {
    cudaSetDevice(srv->device);
    kmb_context *ctx = nullptr;
    cudaStream_t ts = nullptr;
    if (kmb_context_create(srv->device, &ctx) != KMB_OK) ctx = nullptr;
    if (ctx && cudaStreamCreateWithPriority(&ts, cudaStreamNonBlocking, srv->prio_low) == cudaSuccess)
        kmb_context_set_stream(ctx, ts);
    // Pinned staging of a train's inputs and outputs: the caller's buffers may
    // be pageable, and a pageable copy goes through the driver's own staging,
    // holding a copy engine far longer than the DMA of a pinned buffer.
    float *stage = nullptr;
    size_t stage_bytes = 0;
    auto stage_for = [&](size_t bytes) -> bool {
        if (bytes <= stage_bytes) return true;
        if (stage) cudaFreeHost(stage);
        stage = nullptr;
        stage_bytes = 0;
        if (cudaMallocHost(&stage, bytes) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        stage_bytes = bytes;
        return true;
    };
    stage_for((size_t)96 << 20);
    std::unique_lock<std::mutex> lock(srv->mu);
    while (true) {
        srv->cv.wait(lock, [&] {
            if (srv->stop) return true;
            if (srv->train_queue.empty()) return false;
            return srv->in_use + srv->train_queue.front()->bytes <= srv->budget || srv->in_use == srv->base_use;
        });
        if (srv->stop) break;
        Request *r = srv->train_queue.front();
        srv->train_queue.pop_front();
        r->state = RUNNING;
        r->t_start = Clock::now();
        srv->in_use += r->bytes;
        srv->peak_in_use = std::max(srv->peak_in_use, srv->in_use);
        lock.unlock();
        int rc = KMB_ECUDA;
        if (ctx) {
            kmb_params p{r->k, r->iters, 0.0, KMB_FORM_PLAIN, 0};
            double obj = 0.0;
            int64_t it = 0;
            const size_t nx = (size_t)r->n * r->d, nc = (size_t)r->k * r->d;
            if (stage_for(sizeof(float) * (nx + 2 * nc + r->n))) {
                float *sX = stage, *sC0 = stage + nx, *sC = sC0 + nc;
                int32_t *slab = (int32_t *)(sC + nc);
                std::memcpy(sX, r->X, sizeof(float) * nx);
                std::memcpy(sC0, r->C0, sizeof(float) * nc);
                rc = kmb_train(ctx, KMB_F32, KMB_MEM_HOST, sX, r->n, r->d, sC0, &p, sC, slab, &obj, &it, nullptr);
                if (rc == KMB_OK) {
                    std::memcpy(r->C_out, sC, sizeof(float) * nc);
                    std::memcpy(r->labels_out, slab, sizeof(int32_t) * r->n);
                }
            } else {
                rc = kmb_train(ctx, KMB_F32, KMB_MEM_HOST, r->X, r->n, r->d, r->C0, &p, r->C_out, r->labels_out,
                               &obj, &it, nullptr);
            }
        }
        lock.lock();
        r->rc = rc;
        r->t_done = Clock::now();
        r->state = rc == KMB_OK ? DONE : FAILED;
        srv->in_use -= r->bytes;
        srv->completed += 1;
        if (rc != KMB_OK) srv->failed += 1;
        srv->cv.notify_all();
    }
    lock.unlock();
    if (ctx) kmb_context_destroy(ctx);
    if (ts) cudaStreamDestroy(ts);
    if (stage) cudaFreeHost(stage);
}

__global__ void prep_model_kernel(const float *__restrict__ C, int k, int d, int dpad, int kpad, float *__restrict__ Ct,
                                  float *__restrict__ h) {
    const int j = blockIdx.x;
    double s = 0.0;
    for (int t = 0; t < dpad; ++t) {
        const float v = (j < k && t < d) ? C[(int64_t)j * d + t] : 0.f;
        Ct[(int64_t)t * kpad + j] = v;
        s += (double)v * (double)v;
    }
    h[j] = j < k ? (float)(0.5 * s) : __int_as_float(0x7f800000);
}

}  // namespace

extern "C" {

int kmb_server_create(int device, int64_t hbm_budget_bytes, int32_t lanes, int32_t trainers, void **out) {
    if (!out || hbm_budget_bytes <= 0 || lanes <= 0 || trainers < 0) return KMB_EINVAL;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return KMB_ECUDA;
    Server *srv = new (std::nothrow) Server;
    if (!srv) return KMB_ENOMEM;
    srv->device = device;
    srv->budget = (size_t)hbm_budget_bytes;
    if (const char *path = std::getenv("KMB_SERVE_TRACE")) srv->trace = std::fopen(path, "a");
    // smaller assignment launches let lane kernels queued behind a large request's
    // CTAs start sooner (at a per-launch cost)
    if (const char *e = std::getenv("KMB_SERVER_TC_CHUNK_ROWS"))
        srv->tc_chunk_rows = std::min<int64_t>(std::max<int64_t>(atoll(e), 4096), kTcChunkRows);
    if (const char *e = std::getenv("KMB_SERVER_TC_WORKERS")) srv->tc_workers = std::min(std::max(atoi(e), 1), 8);
    if (const char *e = std::getenv("KMB_SERVER_TC_SMS")) srv->tc_sms = std::max(atoi(e), -1);
    // Request memory (lane and worker arenas, worker and trainer workspaces) comes
    // from the library's stream-ordered pool, which keeps what is freed. Growing that
    // pool maps fresh device memory, which stalled every stream of the device for
    // 70-250 ms when a large request first needed it mid-stream; so the pool is
    // grown here, once, by min(budget, 16 GiB) (KMB_SERVER_RESERVE_BYTES overrides),
    // allocated and freed before any request runs.
    {
        size_t reserve = std::min<size_t>(srv->budget, (size_t)16 << 30);
        if (const char *e = std::getenv("KMB_SERVER_RESERVE_BYTES")) reserve = std::min<size_t>(srv->budget, (size_t)atoll(e));
        cudaStream_t rs = nullptr;
        void *block = nullptr;
        if (reserve > 0 && cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking) == cudaSuccess) {
            if (kmb::pool_alloc(&block, reserve, device, rs) == cudaSuccess) cudaFreeAsync(block, rs);
            cudaGetLastError();  // a failed reservation only means later growth
            cudaStreamSynchronize(rs);
            cudaStreamDestroy(rs);
        }
    }
    cudaDeviceGetStreamPriorityRange(&srv->prio_low, &srv->prio_high);
    for (int i = 0; i < lanes; ++i) {
        Lane *l = new Lane;
        l->srv = srv;
        l->index = i;
        // descriptor and label staging sized up front: growing them later
        // (cudaFree / cudaFreeHost) would synchronise the device mid-stream
        l->cap = 2048;
        l->h_lab_cap = srv->max_batch_rows;
        if (cudaMallocHost(&l->h_desc, sizeof(kmb::serve::ReqDesc) * l->cap) != cudaSuccess ||
            cudaMalloc(&l->d_desc, sizeof(kmb::serve::ReqDesc) * l->cap) != cudaSuccess ||
            cudaMallocHost(&l->h_lab, sizeof(int32_t) * l->h_lab_cap) != cudaSuccess ||
            cudaEventCreateWithFlags(&l->done_ev, cudaEventBlockingSync | cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            if (l->h_desc) cudaFreeHost(l->h_desc);
            if (l->d_desc) cudaFree(l->d_desc);
            delete l;
            return KMB_ENOMEM;
        }
        if (cudaStreamCreateWithPriority(&l->stream, cudaStreamNonBlocking, srv->prio_high) != cudaSuccess) {
            delete l;
            return KMB_ECUDA;
        }
        srv->lanes.push_back(l);
    }
    // The tensor-core worker needs its workspace reserved; small budgets serve everything on the lanes.
    if (srv->budget >= 4 * (size_t)srv->tc_workers * kTcReserveBytes) {
        srv->tc_enabled = true;
        srv->base_use = (size_t)srv->tc_workers * kTcReserveBytes;
        srv->in_use = srv->peak_in_use = srv->base_use;
    }
    srv->threads.emplace_back(scheduler_loop, srv);
    for (Lane *l : srv->lanes) l->completer = std::thread(completer_loop, l);
    if (srv->tc_enabled)
        for (int i = 0; i < srv->tc_workers; ++i) srv->threads.emplace_back(tc_worker_loop, srv);
    for (int i = 0; i < trainers; ++i) srv->threads.emplace_back(trainer_loop, srv);
    *out = srv;
    return KMB_OK;
}

int kmb_server_destroy(void *handle) {
    Server *srv = (Server *)handle;
    if (!srv) return KMB_EINVAL;
    {
        std::unique_lock<std::mutex> lock(srv->mu);
        // wait for in-flight work
        srv->cv.wait(lock, [&] {
            for (Lane *l : srv->lanes)
                if (l->busy) return false;
            return srv->pending.empty() && srv->train_queue.empty() && srv->tc_queue.empty() && srv->tc_busy == 0 &&
                   srv->in_use == srv->base_use;
        });
        srv->stop = true;
    }
    srv->cv.notify_all();
    for (auto &t : srv->threads) t.join();
    for (Lane *l : srv->lanes)
        if (l->completer.joinable()) l->completer.join();
    cudaSetDevice(srv->device);
    for (Lane *l : srv->lanes) {
        cudaStreamSynchronize(l->stream);
        cudaStreamDestroy(l->stream);
        if (l->h_desc) cudaFreeHost(l->h_desc);
        if (l->h_lab) cudaFreeHost(l->h_lab);
        for (void *h : l->retired_host) cudaFreeHost(h);
        if (l->done_ev) cudaEventDestroy(l->done_ev);
        if (l->d_desc) cudaFree(l->d_desc);
        if (l->arena) cudaFree(l->arena);
        delete l;
    }
    for (Model &m : srv->models) {
        cudaFree(m.C);
        cudaFree(m.Ct);
        cudaFree(m.h);
    }
    for (auto &kv : srv->all) delete kv.second;
    if (srv->trace) std::fclose(srv->trace);
    delete srv;
    return KMB_OK;
}

int kmb_server_add_model(void *handle, const float *C_host, int64_t k, int64_t d, int32_t *model_id) {
    Server *srv = (Server *)handle;
    if (!srv || !C_host || k <= 0 || d <= 0 || k > INT32_MAX || !model_id) return KMB_EINVAL;
    cudaSetDevice(srv->device);
    Model m;
    m.k = k;
    m.d = d;
    m.kpad = (k + 127) / 128 * 128;
    m.dpad = (d + 7) / 8 * 8;
    if (cudaMalloc(&m.C, sizeof(float) * k * d) != cudaSuccess ||
        cudaMalloc(&m.Ct, sizeof(float) * m.kpad * m.dpad) != cudaSuccess ||
        cudaMalloc(&m.h, sizeof(float) * m.kpad) != cudaSuccess)
        return KMB_ENOMEM;
    cudaMemcpy(m.C, C_host, sizeof(float) * k * d, cudaMemcpyHostToDevice);
    prep_model_kernel<<<(unsigned)m.kpad, 1>>>(m.C, (int)k, (int)d, (int)m.dpad, (int)m.kpad, m.Ct, m.h);
    KMB_LAUNCHED();
    if (cudaDeviceSynchronize() != cudaSuccess) return KMB_ECUDA;
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->models.push_back(m);
    *model_id = (int32_t)srv->models.size() - 1;
    return KMB_OK;
}

int kmb_server_submit_infer(void *handle, int32_t model_id, const float *X_host, int64_t n, int64_t d,
                            int32_t *labels_host, int64_t *request_id) {
    Server *srv = (Server *)handle;
    if (!srv || !X_host || !labels_host || n <= 0 || !request_id) return KMB_EINVAL;
    Request *r = new (std::nothrow) Request;
    if (!r) return KMB_ENOMEM;
    {
        std::lock_guard<std::mutex> lock(srv->mu);
        if (model_id < 0 || model_id >= (int32_t)srv->models.size() || srv->models[model_id].d != d) {
            delete r;
            return KMB_EINVAL;
        }
        r->id = srv->next_id++;
        r->kind = INFER;
        r->model = model_id;
        r->n = n;
        r->d = d;
        r->k = srv->models[model_id].k;
        r->iters = 0;
        r->X = X_host;
        r->C0 = nullptr;
        r->labels_out = labels_host;
        r->C_out = nullptr;
        r->form = serve_form(srv, srv->models[model_id], n);
        r->srv_trace = srv->trace != nullptr;
        r->bytes = r->form == KMB_FORM_BF16X3 ? (size_t)n * d * 4 + (size_t)n * 4 + 4096 : infer_bytes(n, d);
        r->t_submit = Clock::now();
        srv->all[r->id] = r;
        if (r->form == KMB_FORM_BF16X3)
            srv->tc_queue.push_back(r);
        else
            srv->pending.push_back(r);
        *request_id = r->id;
    }
    srv->cv.notify_all();
    return KMB_OK;
}

int kmb_server_submit_train(void *handle, const float *X_host, int64_t n, int64_t d, const float *C0_host, int64_t k,
                            int64_t iterations, float *C_out_host, int32_t *labels_host, int64_t *request_id) {
    Server *srv = (Server *)handle;
    if (!srv || !X_host || !C0_host || !C_out_host || !labels_host || n <= 0 || d <= 0 || k <= 0 || k > n ||
        iterations < 0 || !request_id)
        return KMB_EINVAL;
    Request *r = new (std::nothrow) Request;
    if (!r) return KMB_ENOMEM;
    {
        std::lock_guard<std::mutex> lock(srv->mu);
        r->id = srv->next_id++;
        r->kind = TRAIN;
        r->model = -1;
        r->n = n;
        r->d = d;
        r->k = k;
        r->iters = iterations;
        r->X = X_host;
        r->C0 = C0_host;
        r->labels_out = labels_host;
        r->C_out = C_out_host;
        r->bytes = train_bytes(n, d, k);
        r->t_submit = Clock::now();
        srv->all[r->id] = r;
        srv->train_queue.push_back(r);
        *request_id = r->id;
    }
    srv->cv.notify_all();
    return KMB_OK;
}

// Waits (up to timeout_s; < 0 = no limit) for a request; returns its status
// (KMB_OK when done) or KMB_ETIMEDOUT. latency_s receives submit -> done,
// queued_s submit -> dispatch. A finished request is forgotten after a
// successful wait.
int kmb_server_wait_detail(void *handle, int64_t request_id, double timeout_s, double *latency_s, double *queued_s) {
    Server *srv = (Server *)handle;
    if (!srv) return KMB_EINVAL;
    std::unique_lock<std::mutex> lock(srv->mu);
    auto it = srv->all.find(request_id);
    if (it == srv->all.end()) return KMB_EINVAL;
    Request *r = it->second;
    auto done = [&] { return r->state == DONE || r->state == FAILED; };
    if (timeout_s < 0) {
        srv->cv.wait(lock, done);
    } else if (!srv->cv.wait_for(lock, std::chrono::duration<double>(timeout_s), done)) {
        return KMB_ETIMEDOUT;
    }
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (queued_s) *queued_s = std::chrono::duration<double>(r->t_start - r->t_submit).count();
    if (srv->trace)
        std::fprintf(srv->trace,
                     "R id=%lld kind=%d form=%d n=%lld k=%lld d=%lld submit=%.1f start=%.1f done=%.1f h2d=%.1f "
                     "compute=%.1f d2h=%.1f tc_ms=%.3f recheck_ms=%.3f\n",
                     (long long)r->id, r->kind, r->form, (long long)r->n, (long long)r->k, (long long)r->d,
                     srv->us(r->t_submit), srv->us(r->t_start), srv->us(r->t_done), r->us_h2d, r->us_compute,
                     r->us_d2h, r->ms_tc, r->ms_recheck);
    const int rc = r->rc;
    srv->all.erase(it);
    delete r;
    return rc;
}

int kmb_server_wait(void *handle, int64_t request_id, double timeout_s, double *latency_s) {
    return kmb_server_wait_detail(handle, request_id, timeout_s, latency_s, nullptr);
}

int kmb_server_infer_form(void *handle, int32_t model_id, int64_t n, int32_t *form) {
    Server *srv = (Server *)handle;
    if (!srv || !form || n <= 0) return KMB_EINVAL;
    std::lock_guard<std::mutex> lock(srv->mu);
    if (model_id < 0 || model_id >= (int32_t)srv->models.size()) return KMB_EINVAL;
    *form = serve_form(srv, srv->models[model_id], n);
    return KMB_OK;
}

int kmb_server_get_stats(void *handle, kmb_server_stats *out) {
    Server *srv = (Server *)handle;
    if (!srv || !out) return KMB_EINVAL;
    std::lock_guard<std::mutex> lock(srv->mu);
    out->completed = srv->completed;
    out->failed = srv->failed;
    out->batches = srv->batches;
    out->batched_requests = srv->batched_requests;
    out->pending = (int64_t)(srv->pending.size() + srv->train_queue.size() + srv->tc_queue.size());
    out->tensor_core_requests = srv->tc_requests;
    out->in_use_bytes = (int64_t)srv->in_use;
    out->peak_in_use_bytes = (int64_t)srv->peak_in_use;
    out->budget_bytes = (int64_t)srv->budget;
    return KMB_OK;
}

}  // extern "C"
