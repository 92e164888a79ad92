"""k-means (Lloyd, dense) with oneDAL's train/infer surface, computed on a B200.

Mirrors ``oneapi::dal::kmeans`` (cpp/oneapi/dal/algo/kmeans/common.hpp:175-278,
train_types.hpp:200-320, infer_types.hpp:41-137) and the checks of
``kmeans::detail::train_ops`` / ``infer_ops`` (detail/train_ops.hpp:40-75,
detail/infer_ops.hpp:40-68), so code and tests written against the reference
read the same::

    desc = kmeans.descriptor(np.float32).set_cluster_count(20) \\
                 .set_max_iteration_count(5).set_accuracy_threshold(0.001)
    result = kmeans.train(desc, data, initial_centroids)
    result.get_model().get_centroids(), result.get_responses(),
    result.get_iteration_count(), result.get_objective_function_value()
    kmeans.infer(desc, result.get_model(), data).get_responses()

Tables are 2-D numpy arrays (host memory, like a homogen_table under the host
policy) or CUDA torch tensors (device memory; results stay on the device).
The compute runs in libonedal_b200_kmeans.so through its C ABI; there is no CPU
path -- without the library or a GPU the calls raise.
"""
import ctypes
import os

import numpy as np

from . import _native

__all__ = [
    "descriptor", "train", "infer", "model", "train_result", "infer_result", "result_options", "method",
    "domain_error", "invalid_argument", "internal_error", "bad_alloc",
]

INT32_MAX = 2**31 - 1


# Exception types of oneapi/dal/exceptions.hpp:37-106 (Python analogues).
class domain_error(ValueError):
    pass


class invalid_argument(ValueError):
    pass


class internal_error(RuntimeError):
    pass


class bad_alloc(MemoryError):
    pass


# Error texts of cpp/oneapi/dal/detail/error_messages.cpp.
class _msg:
    cluster_count_leq_zero = "Cluster count is lower than or equal to zero"
    cluster_count_gt_max_int32 = "Cluster count is greater than max int32 value"
    max_iteration_count_lt_zero = "Max iteration count lower than zero"
    accuracy_threshold_lt_zero = "Accuracy_threshold is lower than zero"
    empty_set_of_result_options = "Empty set of result options"
    result_not_enabled = "This result is not enabled via result options"
    input_data_is_empty = "Input data is empty"
    row_count_gt_max_int32 = "Row count is greater than max int32 value"
    cluster_count_exceeds_data_row_count = "Cluster count exceeds data row count"
    init_rc_neq_cluster_count = "Input initial centroids row count is not equal to descriptor cluster count"
    init_cc_neq_data_cc = "Input initial centroids column count is not equal to input data column count"
    model_centroids_are_empty = "Input model centroids are empty"
    model_rc_neq_cluster_count = "Input model centroids row count is not equal to descriptor cluster count"
    model_cc_neq_data_cc = "Input model centroids column count is not equal to input data column count"
    objective_lt_zero = "Objective function value is lower than zero"
    too_many_empty = "Number of clusters exceeds the number of points"
    archive_content_does_not_match_type = "Archive content does not match requested type"


class method:
    """kmeans::method (common.hpp:52-60). Only lloyd_dense is on this path."""
    lloyd_dense = "lloyd_dense"
    lloyd_csr = "lloyd_csr"
    by_default = lloyd_dense


class result_option_id(frozenset):
    def test(self, other: "result_option_id") -> bool:
        return other <= self and bool(other)

    def __or__(self, other):
        return result_option_id(frozenset(self) | frozenset(other))


class result_options:
    """kmeans::result_options (common.hpp:78-84)."""
    compute_exact_objective_function = result_option_id({"compute_exact_objective_function"})
    compute_assignments = result_option_id({"compute_assignments"})


class compute_form:
    """How x.c is contracted on the GPU (the kmb_form of the C ABI). `bf16x3` is the
    split-BF16 tensor-core form (three products per k-step), `bf16` the single-product
    one; both recheck every row inside their error band in FP64, so their responses
    are the FP64 oracle's. `auto` (the default) takes a tensor-core form for float32
    data with d <= 256 once n * k * d is large enough, and the plain FMA form otherwise."""
    plain = _native.KMB_FORM_PLAIN
    bf16x3 = _native.KMB_FORM_BF16X3
    bf16 = _native.KMB_FORM_BF16
    auto = _native.KMB_FORM_AUTO


def _default_form():
    v = os.environ.get("ONEDAL_B200_KMEANS_FORM", "auto").lower()
    if v in ("bf16x3", "tc"):
        return compute_form.bf16x3
    if v == "bf16":
        return compute_form.bf16
    return compute_form.plain if v == "plain" else compute_form.auto


class descriptor:
    """kmeans::descriptor<Float, Method, Task> (common.hpp:175-240; defaults common.cpp:36-42)."""

    def __init__(self, float_type=np.float32, method_=method.lloyd_dense, cluster_count=None):
        self.float_type = np.dtype(float_type)
        if self.float_type not in (np.float32, np.float64):
            raise domain_error("float type must be float32 or float64")
        self.method = method_
        self._cluster_count = 2
        self._max_iteration_count = 100
        self._accuracy_threshold = 0.0
        self._result_options = result_option_id()
        self._form = _default_form()
        self._recheck = False
        if cluster_count is not None:
            self.set_cluster_count(cluster_count)

    def get_cluster_count(self):
        return self._cluster_count

    def get_max_iteration_count(self):
        return self._max_iteration_count

    def get_accuracy_threshold(self):
        return self._accuracy_threshold

    def get_result_options(self):
        return self._result_options

    def set_cluster_count(self, value):
        value = int(value)
        if value <= 0:
            raise domain_error(_msg.cluster_count_leq_zero)
        if value > INT32_MAX:
            raise domain_error(_msg.cluster_count_gt_max_int32)
        self._cluster_count = value
        return self

    def set_max_iteration_count(self, value):
        value = int(value)
        if value < 0:
            raise domain_error(_msg.max_iteration_count_lt_zero)
        self._max_iteration_count = value
        return self

    def set_accuracy_threshold(self, value):
        value = float(value)
        if value < 0.0:
            raise domain_error(_msg.accuracy_threshold_lt_zero)
        self._accuracy_threshold = value
        return self

    def set_result_options(self, value):
        if not value:
            raise domain_error(_msg.empty_set_of_result_options)
        self._result_options = result_option_id(value)
        return self

    # B200-specific knobs (not part of the reference descriptor).
    def set_compute_form(self, form):
        if form not in (compute_form.plain, compute_form.bf16x3, compute_form.bf16, compute_form.auto):
            raise domain_error("unknown compute form")
        self._form = form
        return self

    def get_compute_form(self):
        return self._form

    def set_recheck(self, value: bool):
        """Plain form only: FP64 recheck of rows whose top-2 gap is inside the rounding bound."""
        self._recheck = bool(value)
        return self


class sparse_indexing:
    """oneapi::dal::sparse_indexing (table/common.hpp:37)."""
    zero_based = 0
    one_based = 1


class csr_table:
    """oneapi::dal::csr_table (table/csr.hpp:55-70): values, column_indices, row_offsets
    (row_count + 1 entries), row_count, column_count and the index base (one_based by
    default, as csr_table::wrap). Arrays are numpy (host) or torch CUDA tensors
    (device); indices are int64. Column indices must increase strictly within a row."""

    def __init__(self, data, column_indices, row_offsets, row_count, column_count,
                 indexing=sparse_indexing.one_based):
        self.data = data
        self.column_indices = column_indices
        self.row_offsets = row_offsets
        self.row_count = int(row_count)
        self.column_count = int(column_count)
        self.indexing = int(indexing)
        if self.indexing not in (sparse_indexing.zero_based, sparse_indexing.one_based):
            raise invalid_argument("unknown sparse indexing")

    @classmethod
    def from_scipy(cls, m):
        """From a scipy.sparse matrix (canonical CSR: sorted, no duplicates), zero-based."""
        m = m.tocsr()
        m.sum_duplicates()
        m.sort_indices()
        return cls(m.data, m.indices.astype(np.int64), m.indptr.astype(np.int64), m.shape[0], m.shape[1],
                   sparse_indexing.zero_based)

    @property
    def shape(self):
        return (self.row_count, self.column_count)

    def to_dense(self):
        """Dense row-major copy (host numpy)."""
        base = self.indexing
        v = _to_numpy(self.data)
        c = _to_numpy(self.column_indices).astype(np.int64) - base
        r = _to_numpy(self.row_offsets).astype(np.int64) - base
        out = np.zeros((self.row_count, self.column_count), v.dtype)
        for i in range(self.row_count):
            out[i, c[r[i]:r[i + 1]]] = v[r[i]:r[i + 1]]
        return out


def _to_numpy(a):
    if _is_torch_cuda(a):
        return a.cpu().numpy()
    return np.asarray(a)


def _as_csr(t, dtype):
    """(values, column_indices, row_offsets, on_device) of a csr_table in the descriptor's type."""
    if not isinstance(t, csr_table):
        try:
            import scipy.sparse as sp
            if sp.issparse(t):
                t = csr_table.from_scipy(t)
        except ImportError:
            pass
    if not isinstance(t, csr_table):
        raise invalid_argument("method::lloyd_csr takes a csr_table")
    if _is_torch_cuda(t.data):
        import torch
        tdt = torch.float32 if dtype == np.float32 else torch.float64
        vals = t.data.to(tdt).contiguous()
        cols = t.column_indices.to(torch.int64).contiguous()
        offs = t.row_offsets.to(torch.int64).contiguous()
        return t, vals, cols, offs, True
    vals = np.ascontiguousarray(t.data, dtype=dtype)
    cols = np.ascontiguousarray(t.column_indices, dtype=np.int64)
    offs = np.ascontiguousarray(t.row_offsets, dtype=np.int64)
    if len(offs) != t.row_count + 1:
        raise invalid_argument("row_offsets must hold row_count + 1 entries")
    return t, vals, cols, offs, False


class model:
    """kmeans::model (common.hpp:244-278)."""

    def __init__(self, centroids=None):
        self._centroids = centroids

    def get_centroids(self):
        return self._centroids

    def set_centroids(self, value):
        self._centroids = value
        return self

    def get_cluster_count(self):
        return 0 if self._centroids is None else int(self._centroids.shape[0])

    def has_centroids(self):
        return _has_data(self._centroids)

    def serialize(self) -> bytes:
        """oneDAL's binary archive of this model (the bytes detail::serialize writes into
        binary_output_archive; algo/kmeans/common.cpp:44-56,144-156), via
        kmb_model_serialize. Device-resident centroids are read back by the library."""
        lib = _native.load_library()
        C = self._centroids
        k = 0 if C is None else int(C.shape[0])
        d = 0 if C is None else int(C.shape[1])
        dev = _is_torch_cuda(C) if C is not None else False
        if C is not None:
            if dev:
                C = C.contiguous()
                dtype = _native.KMB_F64 if str(C.dtype) == "torch.float64" else _native.KMB_F32
            else:
                C = np.ascontiguousarray(C)
                if C.dtype not in (np.float32, np.float64):
                    C = C.astype(np.float64)
                dtype = _native.KMB_F64 if C.dtype == np.float64 else _native.KMB_F32
        else:
            dtype = _native.KMB_F32
        size = ctypes.c_int64()
        mem = _native.KMB_MEM_DEVICE if dev else _native.KMB_MEM_HOST
        ptr = None if C is None else _ptr(C, dev)
        rc = lib.kmb_model_serialize(dtype, mem, ptr, k, d, None, 0, ctypes.byref(size))
        if rc != _native.KMB_OK:
            raise invalid_argument(lib.kmb_status_string(rc).decode())
        buf = ctypes.create_string_buffer(size.value)
        rc = lib.kmb_model_serialize(dtype, mem, ptr, k, d, buf, size.value, ctypes.byref(size))
        if rc != _native.KMB_OK:
            raise internal_error(lib.kmb_status_string(rc).decode())
        return buf.raw[:size.value]

    @classmethod
    def deserialize(cls, data: bytes, device=None) -> "model":
        """A model from oneDAL's binary archive (detail::deserialize from
        binary_input_archive). Centroids keep the archive's float type; with `device`
        (a torch device) they are copied straight into device memory. Malformed archives
        raise invalid_argument with oneDAL's message."""
        lib = _native.load_library()
        raw = bytes(data)
        dt, k, d = ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64()
        rc = lib.kmb_model_deserialize(raw, len(raw), ctypes.byref(dt), ctypes.byref(k), ctypes.byref(d),
                                       _native.KMB_MEM_HOST, None, 0)
        if rc != _native.KMB_OK:
            raise invalid_argument(_msg.archive_content_does_not_match_type)
        if k.value == 0:
            return cls()
        npdt = np.float64 if dt.value == _native.KMB_F64 else np.float32
        if device is not None:
            import torch
            C = torch.empty((k.value, d.value), dtype=torch.float64 if npdt == np.float64 else torch.float32,
                            device=device)
            mem, ptr, nbytes = _native.KMB_MEM_DEVICE, C.data_ptr(), C.numel() * C.element_size()
        else:
            C = np.empty((k.value, d.value), npdt)
            mem, ptr, nbytes = _native.KMB_MEM_HOST, C.ctypes.data, C.nbytes
        rc = lib.kmb_model_deserialize(raw, len(raw), ctypes.byref(dt), ctypes.byref(k), ctypes.byref(d), mem,
                                       ptr, nbytes)
        if rc != _native.KMB_OK:
            raise invalid_argument(_msg.archive_content_does_not_match_type)
        return cls(C)

    def __getstate__(self):
        return {"archive": self.serialize()}

    def __setstate__(self, state):
        self._centroids = model.deserialize(state["archive"])._centroids


class train_result:
    """kmeans::train_result (train_types.hpp:227-320)."""

    def __init__(self):
        self._model = model()
        self._responses = None
        self._iteration_count = 0
        self._objective = 0.0
        self.stats = None

    def get_model(self):
        return self._model

    def get_responses(self):
        return self._responses

    def get_iteration_count(self):
        return self._iteration_count

    def get_objective_function_value(self):
        return self._objective

    model = property(get_model)
    responses = property(get_responses)
    iteration_count = property(get_iteration_count)
    objective_function_value = property(get_objective_function_value)


class infer_result:
    """kmeans::infer_result (infer_types.hpp:82-137; getter guard infer_types.cpp:89-95)."""

    def __init__(self, options):
        self._options = result_option_id(options)
        self._responses = None
        self._objective = None
        self.stats = None

    def get_result_options(self):
        return self._options

    def get_responses(self):
        return self._responses

    def get_objective_function_value(self):
        if not self._options.test(result_options.compute_exact_objective_function):
            raise domain_error(_msg.result_not_enabled)
        return self._objective

    def _set_objective(self, value):
        if not self._options.test(result_options.compute_exact_objective_function):
            raise domain_error(_msg.result_not_enabled)
        if value < 0.0:
            raise domain_error(_msg.objective_lt_zero)
        self._objective = value

    responses = property(get_responses)


def _is_torch_cuda(x):
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _has_data(t):
    return t is not None and len(getattr(t, "shape", ())) == 2 and t.shape[0] > 0 and t.shape[1] > 0


def _as_table(t, dtype):
    """Row-major contiguous view in the descriptor's float type (row_accessor<const F>::pull analogue)."""
    if _is_torch_cuda(t):
        import torch
        tdt = torch.float32 if dtype == np.float32 else torch.float64
        return t.to(tdt).contiguous(), True
    return np.ascontiguousarray(t, dtype=dtype), False


def _raise_native(err: _native.NativeError):
    s = err.status
    if s == _native.KMB_EINVAL:
        raise invalid_argument(str(err)) from None
    if s == _native.KMB_ENOMEM:
        raise bad_alloc(str(err)) from None
    if s == _native.KMB_ETOO_MANY_EMPTY:
        raise domain_error(_msg.too_many_empty) from None
    raise internal_error(str(err)) from None


def _ptr(a, on_device):
    return ctypes.c_void_p(a.data_ptr() if on_device else a.ctypes.data)


def _check_train_preconditions(desc, data, initial_centroids):
    """train_ops::check_preconditions (detail/train_ops.hpp:40-61)."""
    if not _has_data(data):
        raise domain_error(_msg.input_data_is_empty)
    if data.shape[0] > INT32_MAX:
        raise domain_error(_msg.row_count_gt_max_int32)
    if desc.get_cluster_count() > data.shape[0]:
        raise invalid_argument(_msg.cluster_count_exceeds_data_row_count)
    if _has_data(initial_centroids):
        if initial_centroids.shape[0] != desc.get_cluster_count():
            raise invalid_argument(_msg.init_rc_neq_cluster_count)
        if initial_centroids.shape[1] != data.shape[1]:
            raise invalid_argument(_msg.init_cc_neq_data_cc)


def _check_infer_preconditions(desc, mdl, data):
    """infer_ops::check_preconditions (detail/infer_ops.hpp:40-56)."""
    if not _has_data(data):
        raise domain_error(_msg.input_data_is_empty)
    if not mdl.has_centroids():
        raise domain_error(_msg.model_centroids_are_empty)
    c = mdl.get_centroids()
    if c.shape[0] != desc.get_cluster_count():
        raise invalid_argument(_msg.model_rc_neq_cluster_count)
    if c.shape[1] != data.shape[1]:
        raise invalid_argument(_msg.model_cc_neq_data_cc)


def _device_of(t):
    return t.device.index if t.device.index is not None else 0


def init_plusplus(data, cluster_count: int, float_type=np.float32, seed: int = 777777, ctx=None):
    """k-means++ initial centroids (k x d) as oneDAL's train() computes them when no
    initial centroids are given: DAAL's dense plusPlus init with one trial
    (kmeans_plusplus_init_impl.i:538-673), seed 777777 by default. Same memory
    space as `data` (numpy array or CUDA tensor)."""
    X, dev = _as_table(data, float_type)
    n, d = X.shape
    k = int(cluster_count)
    if ctx is None:
        ctx = _native.context(_device_of(X) if dev else 0)
    if dev:
        import torch
        C = torch.empty((k, d), dtype=X.dtype, device=X.device)
        ctx.set_stream(torch.cuda.current_stream(X.device).cuda_stream)
    else:
        C = np.empty((k, d), dtype=float_type)
    dtype = _native.KMB_F32 if float_type == np.float32 else _native.KMB_F64
    mem = _native.KMB_MEM_DEVICE if dev else _native.KMB_MEM_HOST
    try:
        ctx.check(ctx.lib.kmb_init_plusplus(ctx.handle, dtype, mem, _ptr(X, dev), n, d, k, ctypes.c_uint32(seed),
                                            _ptr(C, dev)))
    except _native.NativeError as e:
        _raise_native(e)
    return C


def _train_csr(desc, data, initial_centroids):
    """method::lloyd_csr (kmb_train_csr): CSR rows, dense centroids."""
    t, vals, cols, offs, dev = _as_csr(data, desc.float_type)
    n, d = t.shape
    k = desc.get_cluster_count()
    if n <= 0 or d <= 0:
        raise invalid_argument(_msg.input_data_is_empty)
    if k > n:
        raise invalid_argument(_msg.cluster_count_exceeds_data_row_count)
    if _has_data(initial_centroids):
        C0, dev_c = _as_table(initial_centroids, desc.float_type)
        if dev != dev_c:
            raise invalid_argument("data and initial centroids must live in the same memory space")
    else:
        # the reference's default for lloyd_csr: plusPlusCSR, one trial, seed 777777
        C0 = init_plusplus_csr(t, k, desc.float_type)
    if C0.shape[0] != k:
        raise invalid_argument(_msg.init_rc_neq_cluster_count)
    if C0.shape[1] != d:
        raise invalid_argument(_msg.init_cc_neq_data_cc)
    ctx = _native.context(_device_of(vals) if dev else 0)
    if dev:
        import torch
        C = torch.empty_like(C0)
        labels = torch.empty(n, dtype=torch.int32, device=vals.device)
        ctx.set_stream(torch.cuda.current_stream(vals.device).cuda_stream)
    else:
        C = np.empty_like(C0)
        labels = np.empty(n, np.int32)
    params = _native.kmb_params(k, desc.get_max_iteration_count(), desc.get_accuracy_threshold(),
                                _native.KMB_FORM_PLAIN, 0)
    obj, it, stats = ctypes.c_double(0.0), ctypes.c_int64(0), _native.kmb_stats()
    dtype = _native.KMB_F32 if desc.float_type == np.float32 else _native.KMB_F64
    mem = _native.KMB_MEM_DEVICE if dev else _native.KMB_MEM_HOST
    try:
        ctx.check(ctx.lib.kmb_train_csr(ctx.handle, dtype, mem, _ptr(vals, dev), _ptr(cols, dev), _ptr(offs, dev),
                                        n, d, t.indexing, _ptr(C0, dev), ctypes.byref(params), _ptr(C, dev),
                                        _ptr(labels, dev), ctypes.byref(obj), ctypes.byref(it), ctypes.byref(stats)))
    except _native.NativeError as e:
        _raise_native(e)
    r = train_result()
    r._model = model(C)
    r._responses = labels.reshape(n, 1)
    r._iteration_count = int(it.value)
    r._objective = float(obj.value)
    r.stats = stats
    return r


def _infer_csr(desc, mdl, data):
    t, vals, cols, offs, dev = _as_csr(data, desc.float_type)
    n, d = t.shape
    if not mdl.has_centroids():
        raise invalid_argument(_msg.model_centroids_are_empty)
    C, dev_c = _as_table(mdl.get_centroids(), desc.float_type)
    if dev != dev_c:
        raise invalid_argument("data and model centroids must live in the same memory space")
    if C.shape[0] != desc.get_cluster_count():
        raise invalid_argument(_msg.model_rc_neq_cluster_count)
    if C.shape[1] != d:
        raise invalid_argument(_msg.model_cc_neq_data_cc)
    k = C.shape[0]
    want_obj = desc.get_result_options().test(result_options.compute_exact_objective_function)
    ctx = _native.context(_device_of(vals) if dev else 0)
    if dev:
        import torch
        labels = torch.empty(n, dtype=torch.int32, device=vals.device)
        ctx.set_stream(torch.cuda.current_stream(vals.device).cuda_stream)
    else:
        labels = np.empty(n, np.int32)
    obj = ctypes.c_double(0.0)
    dtype = _native.KMB_F32 if desc.float_type == np.float32 else _native.KMB_F64
    mem = _native.KMB_MEM_DEVICE if dev else _native.KMB_MEM_HOST
    try:
        ctx.check(ctx.lib.kmb_infer_csr(ctx.handle, dtype, mem, _ptr(vals, dev), _ptr(cols, dev), _ptr(offs, dev), n,
                                        d, t.indexing, _ptr(C, dev), k, int(want_obj), _ptr(labels, dev),
                                        ctypes.byref(obj)))
    except _native.NativeError as e:
        _raise_native(e)
    r = infer_result(desc.get_result_options())
    r._responses = labels.reshape(n, 1)
    if want_obj:
        r._set_objective(float(obj.value))
    return r


def init_plusplus_csr(data, cluster_count: int, float_type=np.float32, seed: int = 777777, ctx=None):
    """k-means++ centers of CSR rows as oneDAL's train() computes them for method::lloyd_csr
    without initial centroids (DAAL plusPlusCSR, one trial; kmb_init_plusplus_csr). Dense
    k x d centers in the rows' memory space."""
    t, vals, cols, offs, dev = _as_csr(data, float_type)
    n, d = t.shape
    k = int(cluster_count)
    if ctx is None:
        ctx = _native.context(_device_of(vals) if dev else 0)
    if dev:
        import torch
        C = torch.empty((k, d), dtype=vals.dtype, device=vals.device)
        ctx.set_stream(torch.cuda.current_stream(vals.device).cuda_stream)
    else:
        C = np.empty((k, d), dtype=float_type)
    dtype = _native.KMB_F32 if np.dtype(float_type) == np.float32 else _native.KMB_F64
    mem = _native.KMB_MEM_DEVICE if dev else _native.KMB_MEM_HOST
    try:
        ctx.check(ctx.lib.kmb_init_plusplus_csr(ctx.handle, dtype, mem, _ptr(vals, dev), _ptr(cols, dev),
                                                _ptr(offs, dev), n, d, t.indexing, k, ctypes.c_uint32(seed),
                                                _ptr(C, dev)))
    except _native.NativeError as e:
        _raise_native(e)
    return C


def train(desc: descriptor, data, initial_centroids=None) -> train_result:
    """dal::train(desc, data, initial_centroids) for method lloyd_dense and lloyd_csr (train.hpp:26-29)."""
    if desc.method == method.lloyd_csr:
        return _train_csr(desc, data, initial_centroids)
    if desc.method != method.lloyd_dense:
        raise invalid_argument("unknown method")
    _check_train_preconditions(desc, data, initial_centroids)
    X, dev = _as_table(data, desc.float_type)
    n, d = X.shape
    k = desc.get_cluster_count()
    ctx = _native.context(_device_of(X) if dev else 0)
    if _has_data(initial_centroids):
        C0, dev_c = _as_table(initial_centroids, desc.float_type)
        if dev != dev_c:
            raise invalid_argument("data and initial centroids must live in the same memory space")
    else:
        # the reference's default: k-means++ with one trial and seed 777777
        # (detail/train_init_centroids.hpp:47-74), computed on the GPU
        C0 = init_plusplus(X, k, desc.float_type, ctx=ctx)
    if dev:
        import torch
        C = torch.empty_like(C0)
        labels = torch.empty(n, dtype=torch.int32, device=X.device)
        ctx.set_stream(torch.cuda.current_stream(X.device).cuda_stream)
    else:
        C = np.empty_like(C0)
        labels = np.empty(n, np.int32)
    params = _native.kmb_params(k, desc.get_max_iteration_count(), desc.get_accuracy_threshold(),
                                desc.get_compute_form(), int(desc._recheck))
    obj = ctypes.c_double(0.0)
    it = ctypes.c_int64(0)
    stats = _native.kmb_stats()
    dtype = _native.KMB_F32 if desc.float_type == np.float32 else _native.KMB_F64
    mem = _native.KMB_MEM_DEVICE if dev else _native.KMB_MEM_HOST
    try:
        ctx.check(ctx.lib.kmb_train(ctx.handle, dtype, mem, _ptr(X, dev), n, d, _ptr(C0, dev), ctypes.byref(params),
                                    _ptr(C, dev), _ptr(labels, dev), ctypes.byref(obj), ctypes.byref(it),
                                    ctypes.byref(stats)))
    except _native.NativeError as e:
        _raise_native(e)
    r = train_result()
    r._model = model(C)
    r._responses = labels.reshape(n, 1)
    r._iteration_count = int(it.value)
    r._objective = float(obj.value)
    r.stats = stats
    # train_ops::check_postconditions (detail/train_ops.hpp:63-75)
    assert r._iteration_count <= desc.get_max_iteration_count()
    return r


def infer(desc: descriptor, mdl: model, data) -> infer_result:
    """dal::infer(desc, model, data) for method lloyd_dense and lloyd_csr (infer.hpp)."""
    if desc.method == method.lloyd_csr:
        return _infer_csr(desc, mdl, data)
    if desc.method != method.lloyd_dense:
        raise invalid_argument("unknown method")
    _check_infer_preconditions(desc, mdl, data)
    X, dev = _as_table(data, desc.float_type)
    C, dev_c = _as_table(mdl.get_centroids(), desc.float_type)
    if dev != dev_c:
        raise invalid_argument("data and model centroids must live in the same memory space")
    n, d = X.shape
    k = C.shape[0]
    want_obj = desc.get_result_options().test(result_options.compute_exact_objective_function)
    ctx = _native.context(_device_of(X) if dev else 0)
    if dev:
        import torch
        labels = torch.empty(n, dtype=torch.int32, device=X.device)
        ctx.set_stream(torch.cuda.current_stream(X.device).cuda_stream)
    else:
        labels = np.empty(n, np.int32)
    obj = ctypes.c_double(0.0)
    stats = _native.kmb_stats()
    dtype = _native.KMB_F32 if desc.float_type == np.float32 else _native.KMB_F64
    mem = _native.KMB_MEM_DEVICE if dev else _native.KMB_MEM_HOST
    try:
        ctx.check(ctx.lib.kmb_infer(ctx.handle, dtype, mem, _ptr(X, dev), n, d, _ptr(C, dev), k,
                                    desc.get_compute_form(), int(want_obj), _ptr(labels, dev), ctypes.byref(obj),
                                    ctypes.byref(stats)))
    except _native.NativeError as e:
        _raise_native(e)
    r = infer_result(desc.get_result_options())
    r._responses = labels.reshape(n, 1)
    if want_obj:
        r._set_objective(float(obj.value))
    r.stats = stats
    return r
