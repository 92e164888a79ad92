"""ORACLE -- test infrastructure only. ctypes binding of the reference's own DAAL
k-means Lloyd kernel (KMeansBatchKernel<lloydDense, F, avx2>,
cpp/daal/src/algorithms/kmeans/kmeans_lloyd_batch_impl.i:48-242), compiled from
the reference sources by oracle/ref/Makefile into oracle/_ref/.

It is called exactly as the oneAPI CPU backend calls it
(cpp/oneapi/dal/algo/kmeans/backend/cpu/train_kernel_lloyd.cpp:71-144 for
train, backend/cpu/infer_kernel.cpp:52-116 for infer). Threading comes from a
std::thread shim with DAAL's static split, so FP32 results depend only on the
thread count passed here.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None

# services::ErrorKMeansNumberOfClustersIsTooLarge, from DAAL's error-id enum
# (cpp/daal/include/services/error_indexes.h); reported through status_code.


class ReferenceUnavailable(RuntimeError):
    pass


class ReferenceError_(RuntimeError):
    def __init__(self, code):
        super().__init__(f"DAAL kernel returned error id {code}")
        self.code = code


def available() -> bool:
    return os.path.exists(_build.REF_LIB)


def _load():
    global _lib
    if _lib is None:
        if not available():
            raise ReferenceUnavailable(f"{_build.REF_LIB} is not built (make -C oracle/ref)")
        _lib = ctypes.CDLL(_build.REF_LIB)
        P, I64, D = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double
        for sfx in ("f64", "f32"):
            getattr(_lib, f"daalref_train_{sfx}").argtypes = [P, I64, I64, P, I64, I64, D, P, P, P, P, P]
            getattr(_lib, f"daalref_infer_{sfx}").argtypes = [P, I64, I64, P, I64, ctypes.c_int, P, P, P]
        _lib.daalref_set_threads.argtypes = [ctypes.c_int]
        for sfx in ("f64", "f32"):
            getattr(_lib, f"daalref_init_plusplus_{sfx}").argtypes = [P, I64, I64, I64, ctypes.c_uint32, P]
            getattr(_lib, f"daalref_init_plusplus_csr_{sfx}").argtypes = [P, P, P, I64, I64, I64, ctypes.c_uint32, P]
            getattr(_lib, f"daalref_train_csr_{sfx}").argtypes = [P, P, P, I64, I64, P, I64, I64, D, P, P, P, P, P]
            getattr(_lib, f"daalref_infer_csr_{sfx}").argtypes = [P, P, P, I64, I64, P, I64, ctypes.c_int, P, P, P]
    return _lib


def set_threads(t: int) -> int:
    return _load().daalref_set_threads(int(t))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _sfx(dtype):
    return {np.dtype(np.float64): "f64", np.dtype(np.float32): "f32"}[np.dtype(dtype)]


def train(X, C0, max_iteration_count=100, accuracy_threshold=0.0):
    """Returns (centroids, responses int32, objective, iteration_count)."""
    lib = _load()
    X = np.ascontiguousarray(X)
    C0 = np.ascontiguousarray(C0, dtype=X.dtype)
    n, d = X.shape
    k = C0.shape[0]
    C = np.empty_like(C0)
    lab = np.empty(n, np.int32)
    obj = np.zeros(1, X.dtype)
    it = np.zeros(1, np.int64)
    code = np.zeros(1, np.int32)
    rc = getattr(lib, f"daalref_train_{_sfx(X.dtype)}")(_p(X), n, d, _p(C0), k, int(max_iteration_count),
                                                         float(accuracy_threshold), _p(C), _p(lab), _p(obj), _p(it),
                                                         _p(code))
    if rc != 0:
        raise ReferenceError_(int(code[0]))
    return C, lab, float(obj[0]), int(it[0])


def infer(X, C, compute_objective=True):
    """Returns (responses int32, objective or None)."""
    lib = _load()
    X = np.ascontiguousarray(X)
    C = np.ascontiguousarray(C, dtype=X.dtype)
    n, d = X.shape
    lab = np.empty(n, np.int32)
    obj = np.zeros(1, X.dtype)
    code = np.zeros(1, np.int32)
    rc = getattr(lib, f"daalref_infer_{_sfx(X.dtype)}")(_p(X), n, d, _p(C), C.shape[0],
                                                         int(bool(compute_objective)), _p(lab), _p(obj), _p(code))
    if rc != 0:
        raise ReferenceError_(int(code[0]))
    return lab, (float(obj[0]) if compute_objective else None)


def init_plusplus(X, k, seed=777777):
    """The reference's KMeansInitKernel<plusPlusDense, F, avx2> with one trial and an
    mt19937 engine seeded with `seed`, as oneDAL's train() uses it without initial
    centroids (cpp/oneapi/dal/algo/kmeans/detail/train_init_centroids.hpp:47-74)."""
    X = np.ascontiguousarray(X)
    lib = _load()
    n, d = X.shape
    C = np.empty((k, d), X.dtype)
    sfx = "f64" if X.dtype == np.float64 else "f32"
    rc = getattr(lib, f"daalref_init_plusplus_{sfx}")(_p(X), n, d, int(k), int(seed), _p(C))
    if rc != 0:
        raise ReferenceError_(rc)
    return C


def _csr(vals, cols, rowptr, dtype):
    return (np.ascontiguousarray(vals, dtype=dtype), np.ascontiguousarray(cols, dtype=np.int64),
            np.ascontiguousarray(rowptr, dtype=np.int64))


def train_csr(vals, cols, rowptr, d, C0, max_iteration_count=100, accuracy_threshold=0.0):
    """The reference's KMeansBatchKernel<lloydCSR> on zero-based CSR rows.
    Returns (centroids, responses int32, objective, iteration_count)."""
    lib = _load()
    C0 = np.ascontiguousarray(C0)
    v, c, r = _csr(vals, cols, rowptr, C0.dtype)
    n, k = len(r) - 1, C0.shape[0]
    C = np.empty_like(C0)
    lab = np.empty(n, np.int32)
    obj = np.zeros(1, C0.dtype)
    it = np.zeros(1, np.int64)
    code = np.zeros(1, np.int32)
    rc = getattr(lib, f"daalref_train_csr_{_sfx(C0.dtype)}")(_p(v), _p(c), _p(r), n, int(d), _p(C0), k,
                                                             int(max_iteration_count), float(accuracy_threshold), _p(C),
                                                             _p(lab), _p(obj), _p(it), _p(code))
    if rc != 0:
        raise ReferenceError_(int(code[0]))
    return C, lab, float(obj[0]), int(it[0])


def infer_csr(vals, cols, rowptr, d, C, compute_objective=True):
    """Returns (responses int32, objective or None) from the reference CSR kernel."""
    lib = _load()
    C = np.ascontiguousarray(C)
    v, c, r = _csr(vals, cols, rowptr, C.dtype)
    n = len(r) - 1
    lab = np.empty(n, np.int32)
    obj = np.zeros(1, C.dtype)
    code = np.zeros(1, np.int32)
    rc = getattr(lib, f"daalref_infer_csr_{_sfx(C.dtype)}")(_p(v), _p(c), _p(r), n, int(d), _p(C), C.shape[0],
                                                             int(bool(compute_objective)), _p(lab), _p(obj), _p(code))
    if rc != 0:
        raise ReferenceError_(int(code[0]))
    return lab, (float(obj[0]) if compute_objective else None)


def init_plusplus_csr(vals, cols, rowptr, d, k, seed=777777, dtype=None):
    """The reference's KMeansInitKernel<plusPlusCSR> (one trial, mt19937 seeded `seed`)
    on zero-based CSR rows; returns the dense centers."""
    lib = _load()
    dtype = np.asarray(vals).dtype if dtype is None else dtype
    v, c, r = _csr(vals, cols, rowptr, dtype)
    n = len(r) - 1
    C = np.empty((k, d), v.dtype)
    rc = getattr(lib, f"daalref_init_plusplus_csr_{_sfx(v.dtype)}")(_p(v), _p(c), _p(r), n, int(d), int(k), int(seed),
                                                                    _p(C))
    if rc != 0:
        raise ReferenceError_(rc)
    return C
