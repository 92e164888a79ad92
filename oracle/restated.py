"""ORACLE -- test infrastructure only. ctypes binding of the plain-C restatement
of oneDAL's dense k-means Lloyd kernel (oracle/kmeans_oracle.c).

The algorithm follows cpp/daal/src/algorithms/kmeans/kmeans_lloyd_batch_impl.i:48-242
(loop, merge, reseed, convergence), kmeans_lloyd_impl.i:54-496 (scoring, sums,
candidates) and kmeans_lloyd_postprocessing.h:64-183 (final responses, exact
objective); the C file cites each step.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None

OK, EINVAL, ENOMEM, ETOO_MANY_EMPTY = 0, 1, 2, 3


class OracleError(RuntimeError):
    pass


class NoCandidateRows(OracleError):
    """k-means++ found no row with a positive distance to the chosen centers."""


class TooManyEmptyClusters(OracleError):
    """DAAL's ErrorKMeansNumberOfClustersIsTooLarge (kmeans_lloyd_batch_impl.i:171)."""


def _load():
    global _lib
    if _lib is None:
        path = _build.RESTATED_LIB
        if not os.path.exists(path):
            path = _build.build_restated()
        _lib = ctypes.CDLL(path)
        P, I64, D = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double
        for sfx in ("f64", "f32"):
            getattr(_lib, f"kmo_train_{sfx}").argtypes = [P, I64, I64, P, I64, I64, D, P, P, P, P]
            getattr(_lib, f"kmo_infer_{sfx}").argtypes = [P, I64, I64, P, I64, ctypes.c_int, P, P]
            getattr(_lib, f"kmo_step_{sfx}").argtypes = [P, I64, I64, P, I64, P, P, P, P, P]
            getattr(_lib, f"kmo_assign_{sfx}").argtypes = [P, I64, I64, P, I64, P, P, P]
            getattr(_lib, f"kmo_objective_{sfx}").argtypes = [P, I64, I64, P, I64, P]
        _lib.kmo_objective_f64.restype = ctypes.c_double
        _lib.kmo_objective_f32.restype = ctypes.c_float
        _lib.kmo_assign_f32_in_f64.argtypes = [P, I64, I64, P, I64, P, P, P]
        _lib.kmo_cluster_stats_f32.argtypes = [P, I64, I64, P, I64, P, P, P, P]
        for sfx in ("f64", "f32"):
            getattr(_lib, f"kmo_init_plusplus_{sfx}").argtypes = [P, I64, I64, I64, ctypes.c_uint32, ctypes.c_int, P, P]
            getattr(_lib, f"kmo_init_plusplus_csr_{sfx}").argtypes = [P, P, P, I64, I64, I64, ctypes.c_uint32, P, P]
            getattr(_lib, f"kmoc_train_{sfx}").argtypes = [P, P, P, I64, I64, P, I64, I64, D, P, P, P, P]
            getattr(_lib, f"kmoc_infer_{sfx}").argtypes = [P, P, P, I64, I64, P, I64, ctypes.c_int, P, P]
            getattr(_lib, f"kmoc_step_{sfx}").argtypes = [P, P, P, I64, I64, P, I64, P, P, P, P]
            getattr(_lib, f"kmoc_assign_{sfx}").argtypes = [P, P, P, I64, I64, P, I64, P, P]
    return _lib


def _sfx(dtype):
    dtype = np.dtype(dtype)
    if dtype == np.float64:
        return "f64"
    if dtype == np.float32:
        return "f32"
    raise TypeError(f"oracle supports float32/float64, got {dtype}")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _check(rc):
    if rc == ETOO_MANY_EMPTY:
        raise TooManyEmptyClusters("number of clusters is too large (candidates ran out)")
    if rc != OK:
        raise OracleError(f"oracle error {rc}")


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
    sfx = _sfx(X.dtype)
    _check(getattr(lib, f"kmo_train_{sfx}")(_p(X), n, d, _p(C0), k, int(max_iteration_count),
                                            float(accuracy_threshold), _p(C), _p(lab), _p(obj), _p(it)))
    return C, lab, float(obj[0]), int(it[0])


def infer(X, C, compute_objective=True):
    """Returns (responses int32, objective or None)."""
    lib = _load()
    X = np.ascontiguousarray(X)
    C = np.ascontiguousarray(C, dtype=X.dtype)
    n, d = X.shape
    lab = np.empty(n, np.int32)
    obj = np.zeros(1, X.dtype)
    _check(getattr(lib, f"kmo_infer_{_sfx(X.dtype)}")(_p(X), n, d, _p(C), C.shape[0], int(bool(compute_objective)),
                                                      _p(lab), _p(obj)))
    return lab, (float(obj[0]) if compute_objective else None)


def step(X, C_in):
    """One Lloyd update from C_in. Returns (C_out, labels under C_in, shift, n_empty, goal)."""
    lib = _load()
    X = np.ascontiguousarray(X)
    C_in = np.ascontiguousarray(C_in, dtype=X.dtype)
    n, d = X.shape
    k = C_in.shape[0]
    C = np.empty_like(C_in)
    lab = np.empty(n, np.int32)
    shift = np.zeros(1, X.dtype)
    ne = np.zeros(1, np.int64)
    goal = np.zeros(1, X.dtype)
    _check(getattr(lib, f"kmo_step_{_sfx(X.dtype)}")(_p(X), n, d, _p(C_in), k, _p(C), _p(lab), _p(shift), _p(ne),
                                                     _p(goal)))
    return C, lab, float(shift[0]), int(ne[0]), float(goal[0])


def assign(X, C):
    """Labels plus best / second-best score (0.5||c||^2 - x.c) per row, in X's precision."""
    lib = _load()
    X = np.ascontiguousarray(X)
    C = np.ascontiguousarray(C, dtype=X.dtype)
    n, d = X.shape
    lab = np.empty(n, np.int32)
    best = np.empty(n, X.dtype)
    second = np.empty(n, X.dtype)
    _check(getattr(lib, f"kmo_assign_{_sfx(X.dtype)}")(_p(X), n, d, _p(C), C.shape[0], _p(lab), _p(best), _p(second)))
    return lab, best, second


def assign_f32_in_f64(X, C):
    """The FP64 oracle's labels / best / second scores for float32 inputs."""
    lib = _load()
    X = np.ascontiguousarray(X, dtype=np.float32)
    C = np.ascontiguousarray(C, dtype=np.float32)
    n, d = X.shape
    lab = np.empty(n, np.int32)
    best = np.empty(n, np.float64)
    second = np.empty(n, np.float64)
    _check(lib.kmo_assign_f32_in_f64(_p(X), n, d, _p(C), C.shape[0], _p(lab), _p(best), _p(second)))
    return lab, best, second


def cluster_stats_f32(X, labels, k, C=None):
    """FP64 per-cluster sums (k x d), int64 counts and, with C, the FP64 objective
    sum ||x - c_label||^2 of float32 rows under the given labels (a checker for
    full-size GPU runs). Returns (sums, counts, objective or None)."""
    lib = _load()
    X = np.ascontiguousarray(X, dtype=np.float32)
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    n, d = X.shape
    sums = np.empty((k, d), np.float64)
    counts = np.empty(k, np.int64)
    obj = np.zeros(1, np.float64)
    Cc = None if C is None else np.ascontiguousarray(C, dtype=np.float32)
    _check(lib.kmo_cluster_stats_f32(_p(X), n, d, _p(labels), int(k), _p(Cc), _p(sums), _p(counts),
                                     _p(obj) if C is not None else None))
    return sums, counts, (float(obj[0]) if C is not None else None)


def objective(X, C, labels):
    lib = _load()
    X = np.ascontiguousarray(X)
    C = np.ascontiguousarray(C, dtype=X.dtype)
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    n, d = X.shape
    return float(getattr(lib, f"kmo_objective_{_sfx(X.dtype)}")(_p(X), n, d, _p(C), C.shape[0], _p(labels)))


def init_plusplus(X, k, seed=777777, fused=True):
    """DAAL's dense k-means++ initialisation with one trial (kmeans_init_oracle.cpp).
    `fused` computes the squared distances with fused multiply-adds (as the reference's
    vectorised loop and the CUDA kernel do); False rounds every product.
    Returns (centroids k x d, chosen row indices)."""
    X = np.ascontiguousarray(X)
    lib = _load()
    n, d = X.shape
    C = np.empty((k, d), X.dtype)
    rows = np.empty(k, np.int64)
    rc = getattr(lib, f"kmo_init_plusplus_{_sfx(X.dtype)}")(_p(X), n, d, int(k), int(seed), int(bool(fused)), _p(C), _p(rows))
    if rc == 4:
        raise NoCandidateRows("fewer than k distinct rows (no row left to sample)")
    _check(rc)
    return C, rows


def _csr(vals, cols, rowptr, dtype):
    return (np.ascontiguousarray(vals, dtype=dtype), np.ascontiguousarray(cols, dtype=np.int64),
            np.ascontiguousarray(rowptr, dtype=np.int64))


def train_csr(vals, cols, rowptr, d, C0, max_iteration_count, accuracy_threshold):
    """CSR Lloyd (kmeans_csr_oracle.c): zero-based CSR rows (values, column indices,
    n + 1 row offsets) with d columns. Returns (centroids, responses, objective, iterations)."""
    C0 = np.ascontiguousarray(C0)
    v, c, r = _csr(vals, cols, rowptr, C0.dtype)
    n, k = len(r) - 1, C0.shape[0]
    C = np.empty_like(C0)
    lab = np.empty(n, np.int32)
    obj = np.zeros(1, C0.dtype)
    it = np.zeros(1, np.int64)
    lib = _load()
    _check(getattr(lib, f"kmoc_train_{_sfx(C0.dtype)}")(_p(v), _p(c), _p(r), n, int(d), _p(C0), k,
                                                       int(max_iteration_count), float(accuracy_threshold), _p(C),
                                                       _p(lab), _p(obj), _p(it)))
    return C, lab, float(obj[0]), int(it[0])


def infer_csr(vals, cols, rowptr, d, C, compute_objective=True):
    """Returns (responses int32, objective or None) for CSR rows."""
    C = np.ascontiguousarray(C)
    v, c, r = _csr(vals, cols, rowptr, C.dtype)
    n = len(r) - 1
    lab = np.empty(n, np.int32)
    obj = np.zeros(1, C.dtype)
    _check(getattr(_load(), f"kmoc_infer_{_sfx(C.dtype)}")(_p(v), _p(c), _p(r), n, int(d), _p(C), C.shape[0],
                                                          int(bool(compute_objective)), _p(lab), _p(obj)))
    return lab, (float(obj[0]) if compute_objective else None)


def step_csr(vals, cols, rowptr, d, C_in):
    """One CSR Lloyd update: (C_out, labels under C_in, shift, empty count)."""
    C_in = np.ascontiguousarray(C_in)
    v, c, r = _csr(vals, cols, rowptr, C_in.dtype)
    n = len(r) - 1
    C = np.empty_like(C_in)
    lab = np.empty(n, np.int32)
    shift = np.zeros(1, C_in.dtype)
    ne = np.zeros(1, np.int64)
    _check(getattr(_load(), f"kmoc_step_{_sfx(C_in.dtype)}")(_p(v), _p(c), _p(r), n, int(d), _p(C_in), C_in.shape[0],
                                                            _p(C), _p(lab), _p(shift), _p(ne)))
    return C, lab, float(shift[0]), int(ne[0])


def init_plusplus_csr(vals, cols, rowptr, d, k, seed=777777, dtype=None):
    """DAAL's plusPlusCSR with one trial (kmeans_init_oracle.cpp) on zero-based CSR rows.
    Returns (centroids k x d dense, chosen row indices)."""
    dtype = np.asarray(vals).dtype if dtype is None else dtype
    v, c, r = _csr(vals, cols, rowptr, dtype)
    n = len(r) - 1
    C = np.empty((k, d), v.dtype)
    rows = np.empty(k, np.int64)
    rc = getattr(_load(), f"kmo_init_plusplus_csr_{_sfx(v.dtype)}")(_p(v), _p(c), _p(r), n, int(d), int(k), int(seed),
                                                                    _p(C), _p(rows))
    if rc == 4:
        raise NoCandidateRows("fewer than k distinct rows (no row left to sample)")
    _check(rc)
    return C, rows
