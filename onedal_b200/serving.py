"""k-means serving loop on one B200 (Python front end of the kmb_server_* C ABI).

Fitted centroid sets stay resident in HBM; infer and small-train requests of
different n, k and d are admitted under an HBM byte budget and batched, as they
arrive, into shared grouped launches on several CUDA streams (continuous
batching). Infer requests large enough for the tensor cores (d <= 256 and
n * kpad * dpad >= 2^33) run on a tensor-core worker in the BF16x3 form with the
FP64 recheck; ``infer_form`` tells which form a request gets. Responses equal
those of ``kmeans.infer`` in that form (and of ``kmeans.train``, plain form, for
trains) on the same inputs.

    srv = KMeansServer(hbm_budget_bytes=60 << 30)
    mid = srv.add_model(centroids)              # float32 (k, d)
    req = srv.submit_infer(mid, rows)           # float32 (n, d), kept alive by req
    labels, latency_s = srv.wait(req)
"""
import ctypes

import numpy as np

from . import _native


class ServingError(RuntimeError):
    pass


class Request:
    __slots__ = ("id", "kind", "keep", "labels", "centroids")

    def __init__(self, rid, kind, keep, labels, centroids=None):
        self.id = rid
        self.kind = kind
        self.keep = keep          # input arrays the server reads until completion
        self.labels = labels
        self.centroids = centroids


class KMeansServer:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 60 << 30, lanes: int = 3, trainers: int = 4):
        self.lib = _native.load_library()
        h = ctypes.c_void_p()
        rc = self.lib.kmb_server_create(int(device), int(hbm_budget_bytes), int(lanes), int(trainers), ctypes.byref(h))
        if rc != _native.KMB_OK:
            raise ServingError(f"kmb_server_create failed: {self.lib.kmb_status_string(rc).decode()}")
        self.handle = h

    @staticmethod
    def _f32(a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        if a.ndim != 2:
            raise ValueError("expected a 2-D array")
        return a

    def add_model(self, centroids) -> int:
        C = self._f32(centroids)
        mid = ctypes.c_int32()
        rc = self.lib.kmb_server_add_model(self.handle, C.ctypes.data, C.shape[0], C.shape[1], ctypes.byref(mid))
        if rc != _native.KMB_OK:
            raise ServingError(f"add_model failed ({rc})")
        return mid.value

    def add_model_serialized(self, archive: bytes) -> int:
        """Makes a model resident from oneDAL's binary model archive
        (kmeans.model.serialize(), or oneDAL's own detail::serialize)."""
        raw = bytes(archive)
        mid = ctypes.c_int32()
        rc = self.lib.kmb_server_add_model_serialized(self.handle, raw, len(raw), ctypes.byref(mid))
        if rc != _native.KMB_OK:
            raise ServingError(f"add_model_serialized failed ({rc})")
        return mid.value

    def submit_infer(self, model_id: int, rows) -> Request:
        X = self._f32(rows)
        labels = np.empty(X.shape[0], np.int32)
        rid = ctypes.c_int64()
        rc = self.lib.kmb_server_submit_infer(self.handle, int(model_id), X.ctypes.data, X.shape[0], X.shape[1],
                                              labels.ctypes.data, ctypes.byref(rid))
        if rc != _native.KMB_OK:
            raise ServingError(f"submit_infer failed ({rc})")
        return Request(rid.value, "infer", (X,), labels)

    def submit_train(self, rows, initial_centroids, iterations: int) -> Request:
        X = self._f32(rows)
        C0 = self._f32(initial_centroids)
        labels = np.empty(X.shape[0], np.int32)
        C = np.empty_like(C0)
        rid = ctypes.c_int64()
        rc = self.lib.kmb_server_submit_train(self.handle, X.ctypes.data, X.shape[0], X.shape[1], C0.ctypes.data,
                                              C0.shape[0], int(iterations), C.ctypes.data, labels.ctypes.data,
                                              ctypes.byref(rid))
        if rc != _native.KMB_OK:
            raise ServingError(f"submit_train failed ({rc})")
        return Request(rid.value, "train", (X, C0), labels, C)

    def wait(self, req: Request, timeout: float = -1.0, detail: bool = False):
        """Returns (labels, latency_s) for infer, ((centroids, labels), latency_s) for train;
        with detail=True the latency is a (latency_s, queued_s) pair, queued_s being the
        time from submit to dispatch."""
        lat = ctypes.c_double()
        q = ctypes.c_double()
        rc = self.lib.kmb_server_wait_detail(self.handle, req.id, float(timeout), ctypes.byref(lat), ctypes.byref(q))
        if rc == _native.KMB_ETIMEDOUT:
            raise TimeoutError(f"request {req.id} not done after {timeout} s")
        if rc != _native.KMB_OK:
            raise ServingError(f"request {req.id} failed: {self.lib.kmb_status_string(rc).decode()}")
        req.keep = None
        t = (lat.value, q.value) if detail else lat.value
        if req.kind == "train":
            return (req.centroids, req.labels), t
        return req.labels, t

    def infer_form(self, model_id: int, n: int) -> int:
        """_native.KMB_FORM_PLAIN or KMB_FORM_BF16X3: the form an infer of n rows against
        model_id is served in."""
        f = ctypes.c_int32()
        rc = self.lib.kmb_server_infer_form(self.handle, int(model_id), int(n), ctypes.byref(f))
        if rc != _native.KMB_OK:
            raise ServingError(f"infer_form failed ({rc})")
        return f.value

    def stats(self) -> dict:
        s = _native.kmb_server_stats()
        self.lib.kmb_server_get_stats(self.handle, ctypes.byref(s))
        return {f: getattr(s, f) for f, _ in s._fields_}

    def close(self):
        if getattr(self, "handle", None):
            self.lib.kmb_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
