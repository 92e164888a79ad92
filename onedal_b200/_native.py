"""ctypes binding of libonedal_b200_kmeans.so (C ABI in include/onedal_b200_kmeans.h).

The library is the only compute path: if it is missing or no CUDA device is
visible, loading raises -- there is no CPU fallback.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libonedal_b200_kmeans.so")

KMB_OK, KMB_EINVAL, KMB_ENOMEM, KMB_ECUDA, KMB_ETIMEDOUT, KMB_ETOO_MANY_EMPTY, KMB_EUNSUPPORTED, KMB_ECOMM = range(8)
KMB_F32, KMB_F64 = 0, 1
KMB_FMA_PEAK_F32X2 = 2  # kmb_measure_fma_peak: packed FP32 pair FMA
KMB_MEM_HOST, KMB_MEM_DEVICE = 0, 1
KMB_FORM_PLAIN, KMB_FORM_BF16X3, KMB_FORM_AUTO, KMB_FORM_BF16 = 0, 1, 2, 3

# Every symbol the public header declares; tests check the library exports them all.
EXPORTED = (
    "kmb_context_create", "kmb_context_destroy", "kmb_context_set_stream", "kmb_context_last_error",
    "kmb_status_string", "kmb_context_release_workspace", "kmb_train", "kmb_infer", "kmb_lloyd_step",
    "kmb_partial_sums", "kmb_finalize_centroids", "kmb_version", "kmb_lloyd_iterate",
    "kmb_context_set_kernel_timing", "kmb_context_kernel_time", "kmb_infer_noalloc",
    "kmb_server_create", "kmb_server_destroy", "kmb_server_add_model", "kmb_server_submit_infer",
    "kmb_server_submit_train", "kmb_server_wait", "kmb_server_get_stats", "kmb_server_infer_form", "kmb_server_wait_detail", "kmb_context_set_max_sms", "kmb_init_plusplus", "kmb_batched_train",
    "kmb_model_serialize", "kmb_model_deserialize", "kmb_server_add_model_serialized",
    "kmb_train_csr", "kmb_infer_csr", "kmb_init_plusplus_csr", "kmb_context_recheck_rows",
    "kmb_measure_fma_peak", "kmb_train_spmd",
)


# kmb_communicator callbacks: int allreduce_sum_f64(void *user, double *buf, int64_t count) and
# int allgather(void *user, const void *send, int64_t bytes, void *recv)
ALLREDUCE_F64_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int64)
ALLGATHER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p)


class kmb_communicator(ctypes.Structure):
    _fields_ = [("user", ctypes.c_void_p), ("rank", ctypes.c_int32), ("size", ctypes.c_int32),
                ("allreduce_sum_f64", ALLREDUCE_F64_FN), ("allgather", ALLGATHER_FN)]


class kmb_batched_problem(ctypes.Structure):
    _fields_ = [("X", ctypes.c_void_p), ("n", ctypes.c_int64), ("d", ctypes.c_int64), ("C", ctypes.c_void_p),
                ("k", ctypes.c_int64), ("labels", ctypes.c_void_p), ("iterations", ctypes.c_int64),
                ("last_shift", ctypes.c_double)]


class kmb_batched_info(ctypes.Structure):
    _fields_ = [("problems", ctypes.c_int64), ("variants", ctypes.c_int32), ("total_iterations", ctypes.c_int64),
                ("graph_launches", ctypes.c_int64), ("kernel_ms", ctypes.c_double)]


class kmb_server_stats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int64), ("failed", ctypes.c_int64), ("batches", ctypes.c_int64),
                ("batched_requests", ctypes.c_int64), ("pending", ctypes.c_int64), ("in_use_bytes", ctypes.c_int64),
                ("peak_in_use_bytes", ctypes.c_int64), ("budget_bytes", ctypes.c_int64),
                ("tensor_core_requests", ctypes.c_int64)]


class kmb_params(ctypes.Structure):
    _fields_ = [("cluster_count", ctypes.c_int64), ("max_iteration_count", ctypes.c_int64),
                ("accuracy_threshold", ctypes.c_double), ("form", ctypes.c_int32), ("recheck", ctypes.c_int32)]


class kmb_stats(ctypes.Structure):
    _fields_ = [("rechecked_rows", ctypes.c_int64), ("changed_by_recheck", ctypes.c_int64),
                ("empty_cluster_events", ctypes.c_int64), ("last_shift", ctypes.c_double),
                ("full_rescans", ctypes.c_int64)]


class NativeError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


_lib = None
_lock = threading.Lock()
_contexts = {}


def load_library(path: str = LIB_PATH):
    """Loads the shared library without touching the GPU (symbol checks on CPU hosts)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(path):
                raise ImportError(f"{path} is missing: build it with `python -m onedal_b200.build`")
            lib = ctypes.CDLL(path)
            P, I32, I64, D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
            lib.kmb_context_create.argtypes = [ctypes.c_int, ctypes.POINTER(P)]
            lib.kmb_context_destroy.argtypes = [P]
            lib.kmb_context_set_stream.argtypes = [P, P]
            lib.kmb_context_last_error.argtypes = [P]
            lib.kmb_context_last_error.restype = ctypes.c_char_p
            lib.kmb_status_string.argtypes = [ctypes.c_int]
            lib.kmb_status_string.restype = ctypes.c_char_p
            lib.kmb_context_release_workspace.argtypes = [P]
            lib.kmb_version.restype = ctypes.c_char_p
            lib.kmb_init_plusplus.argtypes = [P, ctypes.c_int, ctypes.c_int, P, I64, I64, I64, ctypes.c_uint32, P]
            lib.kmb_context_set_max_sms.argtypes = [P, ctypes.c_int]
            lib.kmb_train.argtypes = [P, ctypes.c_int, ctypes.c_int, P, I64, I64, P, ctypes.POINTER(kmb_params), P, P,
                                      ctypes.POINTER(D), ctypes.POINTER(I64), ctypes.POINTER(kmb_stats)]
            lib.kmb_infer.argtypes = [P, ctypes.c_int, ctypes.c_int, P, I64, I64, P, I64, I32, I32, P,
                                      ctypes.POINTER(D), ctypes.POINTER(kmb_stats)]
            lib.kmb_lloyd_step.argtypes = [P, ctypes.c_int, P, I64, I64, P, I64, I32, I32, P, P, ctypes.POINTER(D),
                                           ctypes.POINTER(I64)]
            lib.kmb_partial_sums.argtypes = [P, ctypes.c_int, P, I64, I64, P, I64, I32, P, P, P, P, P]
            lib.kmb_train_spmd.argtypes = [P, ctypes.c_int, P, I64, I64, P, P, ctypes.POINTER(kmb_communicator), P, P,
                                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
            lib.kmb_finalize_centroids.argtypes = [P, ctypes.c_int, P, P, P, I64, I64, P, ctypes.POINTER(D), P,
                                                   ctypes.POINTER(I64)]
            lib.kmb_lloyd_iterate.argtypes = [P, ctypes.c_int, P, I64, I64, P, ctypes.POINTER(kmb_params), P,
                                              ctypes.POINTER(I64), ctypes.POINTER(kmb_stats)]
            lib.kmb_context_set_kernel_timing.argtypes = [P, ctypes.c_int]
            lib.kmb_context_kernel_time.argtypes = [P, ctypes.c_int, ctypes.POINTER(D), ctypes.POINTER(I64)]
            lib.kmb_context_recheck_rows.argtypes = [P, P, I64, ctypes.POINTER(I64)]
            lib.kmb_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(D)]
            lib.kmb_infer_noalloc.argtypes = [ctypes.c_int, P, I64, I64, P, I64, P, P, P]
            lib.kmb_server_create.argtypes = [ctypes.c_int, I64, I32, I32, ctypes.POINTER(P)]
            lib.kmb_server_destroy.argtypes = [P]
            lib.kmb_server_add_model.argtypes = [P, P, I64, I64, ctypes.POINTER(I32)]
            lib.kmb_server_submit_infer.argtypes = [P, I32, P, I64, I64, P, ctypes.POINTER(I64)]
            lib.kmb_server_submit_train.argtypes = [P, P, I64, I64, P, I64, I64, P, P, ctypes.POINTER(I64)]
            lib.kmb_server_wait.argtypes = [P, I64, D, ctypes.POINTER(D)]
            lib.kmb_server_wait_detail.argtypes = [P, I64, D, ctypes.POINTER(D), ctypes.POINTER(D)]
            lib.kmb_server_get_stats.argtypes = [P, ctypes.c_void_p]
            lib.kmb_server_infer_form.argtypes = [P, I32, I64, ctypes.POINTER(I32)]
            lib.kmb_batched_train.argtypes = [ctypes.c_int, P, I64, I64, D, I32, P, P]
            lib.kmb_model_serialize.argtypes = [ctypes.c_int, ctypes.c_int, P, I64, I64, P, I64, ctypes.POINTER(I64)]
            lib.kmb_model_deserialize.argtypes = [P, I64, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(I64),
                                                  ctypes.POINTER(I64), ctypes.c_int, P, I64]
            lib.kmb_server_add_model_serialized.argtypes = [P, P, I64, ctypes.POINTER(I32)]
            lib.kmb_train_csr.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, I64, I64, I32, P,
                                          ctypes.POINTER(kmb_params), P, P, ctypes.POINTER(D), ctypes.POINTER(I64),
                                          ctypes.POINTER(kmb_stats)]
            lib.kmb_init_plusplus_csr.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, I64, I64, I32, I64,
                                                  ctypes.c_uint32, P]
            lib.kmb_infer_csr.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, I64, I64, I32, P, I64, I32, P,
                                          ctypes.POINTER(D)]
            _lib = lib
    return _lib


class Context:
    """One CUDA device + stream + cached workspace (kmb_context)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.kmb_context_create(int(device), ctypes.byref(h))
        if rc != KMB_OK:
            raise NativeError(rc, f"kmb_context_create(device={device}) failed: "
                                  f"{self.lib.kmb_status_string(rc).decode()} -- a CUDA device is required")
        self.handle = h
        self.device = device

    def check(self, rc):
        if rc != KMB_OK:
            msg = self.lib.kmb_context_last_error(self.handle).decode() or self.lib.kmb_status_string(rc).decode()
            raise NativeError(rc, msg)

    def set_stream(self, stream_ptr: int):
        self.check(self.lib.kmb_context_set_stream(self.handle, ctypes.c_void_p(stream_ptr)))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.kmb_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def context(device: int = 0) -> Context:
    """Per-thread cached context for `device`."""
    key = (threading.get_ident(), device)
    with _lock:
        ctx = _contexts.get(key)
    if ctx is None:
        ctx = Context(device)
        with _lock:
            _contexts[key] = ctx
    return ctx
