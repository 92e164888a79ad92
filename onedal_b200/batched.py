"""Batched k-means: many independent float32 problems trained together on one
GPU (front end of kmb_batched_train). One persistent cooperative kernel runs
every Lloyd iteration of every problem (prep, assign, accumulate, finalize and
decide phases over flat work lists, grid-wide barriers between them); converged
problems are skipped on the device and the kernel ends when all have converged.

    results, info = batched_train([(X0, C0), (X1, C1), ...], max_iteration_count=30)
    for C, labels, iterations in results: ...

Inputs are CUDA torch tensors (X: n x d, C0: k x d, float32; k <= 256). Per
problem the result equals ``kmb_lloyd_iterate`` (plain form) bit for bit:
centroids, responses and iteration count.
"""
import ctypes

import torch

from . import _native


class BatchedError(RuntimeError):
    pass


def batched_train(problems, max_iteration_count: int = 30, accuracy_threshold: float = 0.0, use_graph: bool = True,
                  stream=None):
    """problems: list of (X, C0) CUDA float32 tensors. Returns (list of (C, labels, iterations), info dict)."""
    lib = _native.load_library()
    count = len(problems)
    arr = (_native.kmb_batched_problem * count)()
    xs = []
    for X, C0 in problems:
        if not (X.is_cuda and C0.is_cuda) or X.dtype != torch.float32 or C0.dtype != torch.float32:
            raise BatchedError("problems must be CUDA float32 tensors")
        xs.append(X.contiguous())
    # every problem's centroids in one buffer (one copy) and every label array in another,
    # instead of a copy and an allocation per problem
    dev = xs[0].device if count else torch.device("cuda")
    C_all = torch.cat([C0.reshape(-1) for _, C0 in problems]) if count else torch.empty(0, device=dev)
    lab_all = torch.empty(sum(X.shape[0] for X in xs), dtype=torch.int32, device=dev)
    c_ptr, l_ptr = C_all.data_ptr(), lab_all.data_ptr()
    keep = []
    co = lo = 0
    for i, (X, (_, C0)) in enumerate(zip(xs, problems)):
        n, d = X.shape
        k = C0.shape[0]
        arr[i].X = X.data_ptr()
        arr[i].n = n
        arr[i].d = d
        arr[i].C = c_ptr + 4 * co
        arr[i].k = k
        arr[i].labels = l_ptr + 4 * lo
        keep.append((C_all[co:co + k * d].view(k, d), lab_all[lo:lo + n]))
        co += k * d
        lo += n
    info = _native.kmb_batched_info()
    s = stream or torch.cuda.current_stream()
    rc = lib.kmb_batched_train(_native.KMB_F32, ctypes.cast(arr, ctypes.c_void_p), len(problems),
                               int(max_iteration_count), float(accuracy_threshold), int(bool(use_graph)),
                               ctypes.c_void_p(s.cuda_stream), ctypes.byref(info))
    if rc != _native.KMB_OK:
        raise BatchedError(f"kmb_batched_train failed: {lib.kmb_status_string(rc).decode()}")
    out = [(C, lab, int(arr[i].iterations)) for i, (C, lab) in enumerate(keep)]
    return out, {f: getattr(info, f) for f, _ in info._fields_}
