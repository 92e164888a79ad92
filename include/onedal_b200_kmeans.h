/*
 * onedal_b200_kmeans.h -- C ABI of the B200-native k-means Lloyd (dense) path.
 *
 * This library is the compute engine behind oneDAL's unchanged
 *   oneapi::dal::train(kmeans::descriptor<F, method::lloyd_dense>, data[, init])
 *   oneapi::dal::infer(kmeans::descriptor<F, method::lloyd_dense>, model, data)
 * for F in {float, double}. In the reference those calls end in the
 * host-policy dispatcher specialisations
 *   kmeans::detail::v1::train_ops_dispatcher<host_policy, F, lloyd_dense, clustering>
 *     (declared cpp/oneapi/dal/algo/kmeans/detail/train_ops.hpp:25-30,
 *      defined   cpp/oneapi/dal/algo/kmeans/detail/train_ops.cpp:24-42)
 *   kmeans::detail::v1::infer_ops_dispatcher<host_policy, F, lloyd_dense, clustering>
 *     (declared cpp/oneapi/dal/algo/kmeans/detail/infer_ops.hpp:25-30,
 *      defined   cpp/oneapi/dal/algo/kmeans/detail/infer_ops.cpp:26-43)
 * which run DAAL's KMeansBatchKernel<lloydDense, F, cpu>
 * (cpp/daal/src/algorithms/kmeans/kmeans_lloyd_batch_impl.i:48-242).
 * A replacement dispatcher calls kmb_train / kmb_infer below, with the
 * same arguments the DAAL kernel received. All entry points are synchronous with respect to the
 * host unless stated otherwise, take plain pointers and sizes, and return a
 * kmb_status. Matrices are dense row-major (rows x columns).
 */
#ifndef ONEDAL_B200_KMEANS_H
#define ONEDAL_B200_KMEANS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define KMB_API __attribute__((visibility("default")))
#else
#define KMB_API
#endif

/* Status codes. The dispatcher maps them onto the reference's exception types
 * (cpp/oneapi/dal/backend/interop/error_converter.cpp:136-254):
 * KMB_EINVAL -> invalid_argument / domain_error, KMB_ENOMEM -> bad_alloc,
 * KMB_ETOO_MANY_EMPTY -> domain_error (DAAL ErrorKMeansNumberOfClustersIsTooLarge,
 * kmeans_lloyd_batch_impl.i:171), others -> internal_error. */
typedef enum kmb_status {
    KMB_OK = 0,
    KMB_EINVAL = 1,
    KMB_ENOMEM = 2,
    KMB_ECUDA = 3,
    KMB_ETIMEDOUT = 4,
    KMB_ETOO_MANY_EMPTY = 5,
    KMB_EUNSUPPORTED = 6,
    KMB_ECOMM = 7 /* a communicator callback of kmb_train_spmd reported failure */
} kmb_status;

/* Element type of data and centroids: the descriptor's float_t. */
typedef enum kmb_dtype { KMB_F32 = 0, KMB_F64 = 1 } kmb_dtype;

/* Where the caller's buffers live. */
typedef enum kmb_memory { KMB_MEM_HOST = 0, KMB_MEM_DEVICE = 1 } kmb_memory;

/* How the x.c contraction is computed.
 * KMB_FORM_PLAIN : the drop-in. F-precision FMA (FP32 or FP64) distance with a
 *                  fused per-row argmin; lowest index wins ties.
 * KMB_FORM_BF16X3: FP32 data only. Split-BF16 (hi+lo, three products) tcgen05
 *                  tensor-core contraction with FP32 accumulation in TMEM; every
 *                  row whose top-2 gap is inside the derived error bound is
 *                  rechecked exactly in FP64, so responses equal the FP64
 *                  oracle's.
 * KMB_FORM_BF16  : FP32 data only. One BF16 tcgen05 product (bf16(x).bf16(c))
 *                  with FP32 accumulation; its wider error bound sends more
 *                  near-tie rows to the same exact FP64 recheck, so responses
 *                  again equal the FP64 oracle's. A third of the tensor work of
 *                  BF16X3; the faster of the two unless a large share of the rows
 *                  lies near a tie.
 * KMB_FORM_AUTO  : a tensor-core form for FP32 data with d <= 256 once the
 *                  contraction is dense enough to pay for the tensor cores
 *                  (n * kpad * dpad >= KMB_AUTO_TC_MACS), the plain form
 *                  otherwise. */
typedef enum kmb_form { KMB_FORM_PLAIN = 0, KMB_FORM_BF16X3 = 1, KMB_FORM_AUTO = 2, KMB_FORM_BF16 = 3 } kmb_form;
#define KMB_AUTO_TC_MACS (1LL << 30)

typedef struct kmb_context kmb_context;

/* Lloyd parameters: the descriptor fields of
 * cpp/oneapi/dal/algo/kmeans/common.hpp:175-240 (defaults common.cpp:36-42). */
typedef struct kmb_params {
    int64_t cluster_count;       /* k > 0                                   */
    int64_t max_iteration_count; /* >= 0                                    */
    double accuracy_threshold;   /* >= 0; stop when sum ||c_old-c_new||^2 <= it */
    int32_t form;                /* kmb_form                                */
    int32_t recheck;             /* PLAIN form: 1 = FP64 recheck of near-ties */
} kmb_params;

/* Per-call diagnostics (optional output of the train/infer calls). */
typedef struct kmb_stats {
    int64_t rechecked_rows;   /* rows re-scored in FP64 in the last assignment
                                 (kmb_lloyd_iterate: summed over its assignments) */
    int64_t changed_by_recheck;
    int64_t empty_cluster_events; /* clusters reseeded over the whole train  */
    double last_shift;        /* sum ||c_old - c_new||^2 of the last update     */
    int64_t full_rescans;     /* of those, rows re-scored against all k clusters */
} kmb_stats;

/* Context: one CUDA device, one stream, a workspace that grows on demand.
 * A context is not thread-safe; use one per host thread. */
KMB_API int kmb_context_create(int device, kmb_context **out);
KMB_API int kmb_context_destroy(kmb_context *ctx);
/* Use the caller's cudaStream_t (passed as void*) instead of the context's own. */
KMB_API int kmb_context_set_stream(kmb_context *ctx, void *cuda_stream);
KMB_API const char *kmb_context_last_error(const kmb_context *ctx);
KMB_API const char *kmb_status_string(int status);
/* Frees the cached workspace. */
KMB_API int kmb_context_release_workspace(kmb_context *ctx);

/* Train: replaces train_ops_dispatcher<host_policy, F, lloyd_dense, clustering>
 * (cpp/oneapi/dal/algo/kmeans/detail/train_ops.cpp:24-42 ->
 *  backend/cpu/train_kernel_lloyd.cpp:84-144).
 * X: n x d, C0: k x d initial centroids (required here; a dispatcher given
 * none first calls kmb_init_plusplus, as oneDAL's train() does). Outputs: C_out k x d, responses n (int32, against the final
 * centroids), objective = exact sum ||x - c_label||^2 (FP64 accumulation),
 * iteration_count. Pointers are host or device memory per `memory`.
 * stats may be NULL. */
KMB_API int kmb_train(kmb_context *ctx, int dtype, int memory, const void *X, int64_t n, int64_t d, const void *C0,
                      const kmb_params *params, void *C_out, int32_t *responses, double *objective,
                      int64_t *iteration_count, kmb_stats *stats);

/* k-means++ initial centroids: replaces the default initialisation that
 * oneDAL's train() runs when no initial centroids are given
 * (cpp/oneapi/dal/algo/kmeans/detail/train_init_centroids.hpp:47-74 ->
 *  DAAL KMeansInitKernel<plusPlusDense>, kmeans_plusplus_init_impl.i:538-673,
 *  one trial). With seed = 777777 (the reference's default,
 * kmeans_init_parameter_types.cpp:41-48) the chosen rows equal the
 * reference's: the same generator, draw order, block sums and sampling walk.
 * C_out: k x d, host or device per `memory`. KMB_EINVAL for k > n, and when
 * every remaining distance is zero (fewer distinct rows than k) or the total
 * is not finite: the reference's resampling would never end there. */
KMB_API int kmb_init_plusplus(kmb_context *ctx, int dtype, int memory, const void *X, int64_t n, int64_t d, int64_t k,
                              uint32_t seed, void *C_out);
#define KMB_PLUSPLUS_DEFAULT_SEED 777777u

/* CSR rows (kmeans::method::lloyd_csr): replaces the lloyd_csr instantiations of
 * the same dispatchers (detail/train_ops.cpp:41-42, detail/infer_ops.cpp:42-43 ->
 * DAAL KMeansBatchKernel<lloydCSR>, kmeans_lloyd_impl.i:248-344,
 * kmeans_lloyd_postprocessing.h:186-350). Rows are given as csr_table holds them
 * (csr_table::wrap(values, column_indices, row_offsets, row_count, column_count,
 * indexing)): values (nnz, dtype), column_indices (nnz int64), row_offsets
 * (n + 1 int64), indexing 0 = zero_based, 1 = one_based; column indices must
 * increase strictly within each row. Centroids are dense (k x d). Scores are the
 * sparse product over the stored entries; the objective is the reference's CSR
 * form (per row: sum over stored entries of x^2 - 2xc, plus ||c||^2, clipped at
 * zero). Train takes the plain form only and requires initial centroids (a caller
 * without them first runs kmb_init_plusplus_csr, as oneDAL's train() does). */
KMB_API int kmb_train_csr(kmb_context *ctx, int dtype, int memory, const void *values, const int64_t *col_indices,
                          const int64_t *row_offsets, int64_t n, int64_t d, int32_t indexing, const void *C0,
                          const kmb_params *params, void *C_out, int32_t *responses, double *objective,
                          int64_t *iteration_count, kmb_stats *stats);
KMB_API int kmb_infer_csr(kmb_context *ctx, int dtype, int memory, const void *values, const int64_t *col_indices,
                          const int64_t *row_offsets, int64_t n, int64_t d, int32_t indexing, const void *C, int64_t k,
                          int32_t compute_objective, int32_t *responses, double *objective);
/* The default initialisation of train() with method::lloyd_csr and no initial
 * centroids: DAAL plusPlusCSR, one trial (detail/train_init_centroids.hpp:39-74,
 * kmeans_plusplus_init_impl.i:244-316): the sampling of kmb_init_plusplus with the
 * CSR distance ||c||^2 + sum over stored entries of (x*x - 2*x*c), each operation
 * rounded as written. C_out: k x d dense centers, host or device per `memory`. */
KMB_API int kmb_init_plusplus_csr(kmb_context *ctx, int dtype, int memory, const void *values,
                                  const int64_t *col_indices, const int64_t *row_offsets, int64_t n, int64_t d,
                                  int32_t indexing, int64_t k, uint32_t seed, void *C_out);

/* Model serialisation in oneDAL's binary archive format: the bytes of
 * detail::serialize(kmeans::model<task::clustering>, binary_output_archive)
 * (cpp/oneapi/dal/algo/kmeans/common.cpp:44-56,144-156 with
 * cpp/oneapi/dal/detail/archives.hpp:24-78), so archives move between oneDAL
 * and this library in both directions. Context-free; no GPU is needed for host
 * memory.
 * kmb_model_serialize: C is k x d (row-major, host or device per `memory`; k = 0
 *   writes a model without centroids). buf = NULL only reports *size; otherwise
 *   capacity must be >= *size.
 * kmb_model_deserialize: reports the stored dtype (KMB_F32 / KMB_F64) and shape;
 *   with C_out != NULL also copies the centroids (row-major, host or device) when
 *   capacity_bytes suffices. Malformed or mismatched archives (bad magic, ids,
 *   element types, sizes, truncation) return KMB_EINVAL, where oneDAL throws
 *   invalid_argument("Archive content does not match requested type"). */
KMB_API int kmb_model_serialize(int dtype, int memory, const void *C, int64_t k, int64_t d, void *buf,
                                int64_t capacity, int64_t *size);
KMB_API int kmb_model_deserialize(const void *buf, int64_t size, int *dtype, int64_t *k, int64_t *d, int memory,
                                  void *C_out, int64_t capacity_bytes);

/* Infer: replaces infer_ops_dispatcher<host_policy, F, lloyd_dense, clustering>
 * (cpp/oneapi/dal/algo/kmeans/detail/infer_ops.cpp:26-43 ->
 *  backend/cpu/infer_kernel.cpp:52-116). responses against C (k x d);
 * objective only when compute_objective != 0 (may be NULL otherwise). */
KMB_API int kmb_infer(kmb_context *ctx, int dtype, int memory, const void *X, int64_t n, int64_t d, const void *C,
                      int64_t k, int32_t form, int32_t compute_objective, int32_t *responses, double *objective,
                      kmb_stats *stats);

/* One Lloyd update from C_in, device memory only (lock-step parity checks and
 * the sharded multi-GPU driver): labels under C_in, C_out, the centroid shift
 * and the number of empty clusters reseeded. Mirrors one pass of the loop body
 * kmeans_lloyd_batch_impl.i:117-212. */
KMB_API int kmb_lloyd_step(kmb_context *ctx, int dtype, const void *X, int64_t n, int64_t d, const void *C_in,
                           int64_t k, int32_t form, int32_t recheck, void *C_out, int32_t *labels, double *shift,
                           int64_t *n_empty);

/* Partial statistics for row-sharded (SPMD) training, device memory only:
 * labels of this shard's rows under C (k x d), FP64 per-cluster sums
 * sums (k x d), counts (k, int64), the shard's sum of squared distances
 * (*sq_distances, one device double; may be NULL) and, when row_sq_distance
 * is not NULL, each row's squared distance to its centroid (n values of the
 * data type; used to pick empty-cluster candidates). Sums are added in row
 * order, so equal labels give bit-identical sums. The caller all-reduces
 * sums/counts across shards, then calls kmb_finalize_centroids. The
 * reference's SPMD path performs the same exchange
 * (cpp/oneapi/dal/algo/kmeans/backend/gpu/cluster_updater.hpp:117-153). */
KMB_API int kmb_partial_sums(kmb_context *ctx, int dtype, const void *X, int64_t n, int64_t d, const void *C,
                             int64_t k, int32_t form, int32_t *labels, double *sums, int64_t *counts,
                             double *sq_distances, void *row_sq_distance);

/* Centroids from all-reduced sums/counts (device memory): c_j = sums_j / counts_j
 * rounded to F; clusters with count 0 keep C_in and are listed (ascending) in
 * empty_ids (k int32, device) with *n_empty (host) set; *shift (host) = sum over
 * non-empty clusters of ||c_old - c_new||^2. The caller reseeds the listed
 * clusters (kmeans_lloyd_batch_impl.i:167-186) and adds their shift. */
KMB_API int kmb_finalize_centroids(kmb_context *ctx, int dtype, const double *sums, const int64_t *counts,
                                   const void *C_in, int64_t k, int64_t d, void *C_out, double *shift,
                                   int32_t *empty_ids, int64_t *n_empty);

/* ---- Sharded training through the caller's communicator ------------------
 * One call per rank (one process per GPU), each with its own block of rows; every
 * rank returns the same centroids. The loop is the one the reference's SPMD path
 * runs (cpp/oneapi/dal/algo/kmeans/backend/gpu/cluster_updater.hpp:117-153,
 * backend/gpu/empty_cluster_handling_dpc.cpp:273-300): per iteration each rank
 * computes its rows' labels and FP64 per-cluster sums/counts (kmb_partial_sums),
 * the ranks sum [sums | counts | squared distances] with ONE allreduce_sum_f64
 * call, every rank finalizes identically (kmb_finalize_centroids); when clusters
 * are empty, every rank offers its m farthest rows (m = number of empty clusters)
 * through ONE allgather call and the global m farthest by (distance descending,
 * global row ascending) reseed the empty clusters in ascending order; stop when
 * the shift <= accuracy_threshold. After the loop: labels of this rank's rows under
 * the final centroids and the objective summed over ranks. Every rank must call
 * with the same C0, params, k and d. The callbacks work on host memory and return
 * 0 on success (anything else ends the call with KMB_ECOMM on that rank):
 *   allreduce_sum_f64(user, buf, count): in-place elementwise sum over ranks;
 *   allgather(user, send, bytes, recv): recv receives size * bytes, rank order.
 * Device pointers: X (n x d, this rank's rows), C0 and C_out (k x d), labels (n).
 * The oneDAL host-policy SPMD dispatchers stay `unimplemented`, as the reference's
 * host backend's are; this entry serves a caller that brings its own
 * communicator (NCCL, MPI, gloo) around the library. */
typedef struct kmb_communicator {
    void *user;
    int32_t rank, size;
    int (*allreduce_sum_f64)(void *user, double *buf, int64_t count);
    int (*allgather)(void *user, const void *send, int64_t bytes, void *recv);
} kmb_communicator;

KMB_API int kmb_train_spmd(kmb_context *ctx, int dtype, const void *X, int64_t n, int64_t d, const void *C0,
                           const kmb_params *params, const kmb_communicator *comm, void *C_out, int32_t *labels,
                           double *objective, int64_t *iteration_count);

/* Lloyd iterations only, in place, device memory: C (k x d) holds the initial
 * centroids on entry and the updated ones on return; labels (n) receive the
 * assignment of the last completed update. Runs up to max_iteration_count
 * updates, stopping early on the accuracy threshold exactly as kmb_train's
 * loop (kmeans_lloyd_batch_impl.i:117-213), without the final responses /
 * objective pass. Used by the benchmark and the serving loop's small trains. */
KMB_API int kmb_lloyd_iterate(kmb_context *ctx, int dtype, const void *X, int64_t n, int64_t d, void *C,
                              const kmb_params *params, int32_t *labels, int64_t *iteration_count, kmb_stats *stats);

/* Kernel timing: when enabled, CUDA events are recorded on the launching
 * stream around every launch of the dominant assignment kernel; the totals are
 * read (synchronising) with kmb_context_kernel_time and cleared by enabling
 * again. kernel: 0 = plain assignment, 1 = tensor-core assignment, 2 = update,
 * 4 = FP64 near-tie recheck; kernel 3 returns in *launches every kernel this
 * host thread launched since timing was enabled (total_ms = 0). */
KMB_API int kmb_context_set_kernel_timing(kmb_context *ctx, int enabled);
/* Grid of the persistent launches (tensor-core assignment, row splitting,
 * recheck): at most max_sms SMs (0: all), leaving the rest to other streams'
 * work. max_sms = -1 instead launches the tensor-core assignment as one short
 * CTA per 128-row tile, which other streams' launches interleave with at tile
 * granularity -- the serving loop uses it so that neither side waits for a
 * whole launch of the other. */
KMB_API int kmb_context_set_max_sms(kmb_context *ctx, int max_sms);
KMB_API int kmb_context_kernel_time(kmb_context *ctx, int kernel, double *total_ms, int64_t *launches);
/* Diagnostics: the rows the context's last assignment pass re-scored in FP64
 * (the near-tie rows of the tensor-core form, or of the plain form with
 * recheck). *count = how many were queued; the first min(*count, capacity)
 * row indices go to rows_out (device memory, int32). Synchronises the
 * context's stream. No counterpart in the reference (its GEMM-based scoring
 * has no near-tie queue). */
KMB_API int kmb_context_recheck_rows(kmb_context *ctx, int32_t *rows_out, int64_t capacity, int64_t *count);

/* Responses (and, when objective != NULL, the exact objective) of n rows X
 * against k centroids C, like kmb_infer with the plain form, for callers that
 * cannot allocate device memory -- e.g. a plugin inside a framework that owns
 * every device allocation, or a latency-bound loop that cannot pay for
 * cudaMalloc/cudaFree. This entry point has no counterpart in the reference.
 * Everything is device memory: X (n x d), C (k x d), responses (n int32),
 * objective (one double). Kernels are enqueued on cuda_stream (a cudaStream_t,
 * NULL = legacy default stream) and the call returns without waiting.
 * It allocates nothing: its scratch is one fixed 24 MiB device array that the
 * library holds on every GPU that loads it until the process exits. A call
 * needs 2*n*sizeof(F) + kpad*dpad*sizeof(F) + kpad*sizeof(F) + 9728 bytes
 * (kpad = k rounded up to 128, dpad = d rounded up to 8, each part rounded up
 * to 256 bytes); bigger problems return KMB_EINVAL with a message on stderr.
 * All calls on a device share the array, which keeps the last call's
 * contents; calls that overlap on the GPU (other streams or host threads)
 * race, so issue them on one stream. The array's device address belongs to a
 * CUDA context: the first call in each context (the device's primary context,
 * or a driver-API context the caller made current) looks it up with
 * cudaGetSymbolAddress while that context is current and caches it by the
 * context's id; make that first call before any stream capture in the context. */
KMB_API int kmb_infer_noalloc(int dtype, const void *X, int64_t n, int64_t d, const void *C, int64_t k,
                              int32_t *responses, double *objective, void *cuda_stream);

/* ---- Batched form ---------------------------------------------------------
 * Many independent float32 problems (each its own X, n, d, k) train together in
 * one persistent cooperative kernel: per Lloyd iteration it walks prep, assign,
 * accumulate, finalize and decide phases over flat work lists of all problems,
 * separated by grid-wide barriers; converged problems are skipped and the kernel
 * ends when every problem has converged. Per problem the result is that of
 * kmb_lloyd_iterate (plain form) bit for bit -- the same FP32 scores, the same
 * exact fixed-point cluster sums, the same reseeding -- up to max_iteration_count
 * updates, stopping when the shift <= accuracy_threshold (the shift is the same
 * sum in another order, so a threshold that equals it to the last bit may stop
 * one path an iteration before the other; with threshold 0 the two agree). C
 * (k x d) is updated in place; labels hold the assignment of the last completed
 * update. Limits: k <= 256 and k <= n and (k*d + k) * 8 <= 200 KiB per problem.
 * The assignment tile per (d, k) class is chosen by a built-in autotuner the
 * first time the class is seen on a device. use_graph launches the kernel from a
 * CUDA graph (one cooperative kernel node). A grid barrier that does not complete
 * within about two seconds makes every CTA leave and the call return
 * KMB_ETIMEDOUT. No counterpart in the reference. */
typedef struct kmb_batched_problem {
    const void *X;      /* device, n x d */
    int64_t n, d;
    void *C;            /* device, k x d, in/out */
    int64_t k;
    int32_t *labels;    /* device, n */
    int64_t iterations; /* out */
    double last_shift;  /* out */
} kmb_batched_problem;

typedef struct kmb_batched_info {
    int64_t problems;
    int32_t variants;         /* assignment tile variants (rows per thread x cluster tile) in use */
    int64_t total_iterations; /* summed over problems */
    int64_t graph_launches;
    double kernel_ms;         /* device time of the persistent kernel (CUDA events), host set-up excluded */
} kmb_batched_info;

KMB_API int kmb_batched_train(int dtype, kmb_batched_problem *problems, int64_t count, int64_t max_iteration_count,
                              double accuracy_threshold, int32_t use_graph, void *cuda_stream,
                              kmb_batched_info *info);

/* ---- Serving loop ---------------------------------------------------------
 * No counterpart in the reference (its API is one synchronous call per
 * train/infer). A server keeps fitted centroid sets resident on one GPU, admits
 * requests under an HBM byte budget, and batches every admissible pending
 * infer request into one grouped launch per free lane (CUDA stream), so
 * requests that arrive while others run are picked up by the next free lane and
 * their work overlaps on the device. Small train requests run on trainer
 * threads, each with its own context. Large infer requests (d <= 256 and
 * n * kpad * dpad >= KMB_SERVER_TC_MACS, kpad = k rounded up to 128, dpad = d
 * rounded up to 64) run on tensor-core workers instead (BF16x3 form with the
 * FP64 recheck, in row chunks, launched as one short CTA per row tile, so that
 * small batches interleave with them). Every response equals kmb_infer's on the same inputs in
 * the form kmb_server_infer_form reports (plain form: bit-identical to the
 * grouped launch; BF16x3: the FP64 oracle's labels), and kmb_train's (plain
 * form) for trains. Host buffers passed to submit_* must stay valid until the
 * request is waited for; pinned host memory gives the lowest latency.
 * Thread-safe. */
#define KMB_SERVER_TC_MACS (1LL << 33)
typedef struct kmb_server_stats {
    int64_t completed;
    int64_t failed;
    int64_t batches;          /* grouped infer launches */
    int64_t batched_requests; /* infer requests over all batches */
    int64_t pending;
    int64_t in_use_bytes;
    int64_t peak_in_use_bytes;
    int64_t budget_bytes;
    int64_t tensor_core_requests; /* infer requests served by the tensor-core worker */
} kmb_server_stats;

KMB_API int kmb_server_create(int device, int64_t hbm_budget_bytes, int32_t lanes, int32_t trainers, void **server);
/* Waits for all admitted work, then releases everything. */
KMB_API int kmb_server_destroy(void *server);
/* Makes a fitted centroid set (k x d float32, host) resident; returns its id. */
KMB_API int kmb_server_add_model(void *server, const float *C, int64_t k, int64_t d, int32_t *model_id);
/* The same from a oneDAL model archive (kmb_model_deserialize's format); double
 * centroids are rounded to float, the serving engine's working type. */
KMB_API int kmb_server_add_model_serialized(void *server, const void *buf, int64_t size, int32_t *model_id);
/* Responses of n rows (n x d float32, host) against a resident model. */
KMB_API int kmb_server_submit_infer(void *server, int32_t model_id, const float *X, int64_t n, int64_t d,
                                    int32_t *responses, int64_t *request_id);
/* A small train (plain form, eps 0, exactly up to `iterations` Lloyd updates). */
KMB_API int kmb_server_submit_train(void *server, const float *X, int64_t n, int64_t d, const float *C0, int64_t k,
                                    int64_t iterations, float *C_out, int32_t *responses, int64_t *request_id);
/* Waits up to timeout_s (< 0: no limit) for a request; returns its status or
 * KMB_ETIMEDOUT; latency_s = submit -> completion on the host clock. */
KMB_API int kmb_server_wait(void *server, int64_t request_id, double timeout_s, double *latency_s);
/* kmb_server_wait plus queued_s = submit -> dispatch (admitted onto a lane or worker). */
KMB_API int kmb_server_wait_detail(void *server, int64_t request_id, double timeout_s, double *latency_s,
                                   double *queued_s);
/* The form (KMB_FORM_PLAIN or KMB_FORM_BF16X3) an infer of n rows against
 * model_id is served in. */
KMB_API int kmb_server_infer_form(void *server, int32_t model_id, int64_t n, int32_t *form);
KMB_API int kmb_server_get_stats(void *server, kmb_server_stats *stats);

/* Measured fused multiply-add peak of `device` in dtype's precision (GFLOP/s,
 * 2 flops per FMA): a short grid of dependent FMA chains timed with CUDA
 * events, best of four launches. dtype KMB_F32, KMB_F64, or
 * KMB_FMA_PEAK_F32X2 for the packed FP32 pair instruction (fma.rn.f32x2). The
 * plain form's assignment is reported against the larger FP32 figure. No
 * counterpart in the reference. */
#define KMB_FMA_PEAK_F32X2 2
KMB_API int kmb_measure_fma_peak(int device, int dtype, double *gflops);

/* Library version string. */
KMB_API const char *kmb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* ONEDAL_B200_KMEANS_H */
