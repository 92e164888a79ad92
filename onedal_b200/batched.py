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
    arr = (_native.kmb_batched_problem * len(problems))()
    keep = []
    for i, (X, C0) in enumerate(problems):
        if not (X.is_cuda and C0.is_cuda) or X.dtype != torch.float32 or C0.dtype != torch.float32:
            raise BatchedError("problems must be CUDA float32 tensors")
        X = X.contiguous()
        C = C0.clone().contiguous()
        lab = torch.empty(X.shape[0], dtype=torch.int32, device=X.device)
        keep.append((X, C, lab))
        arr[i].X = X.data_ptr()
        arr[i].n = X.shape[0]
        arr[i].d = X.shape[1]
        arr[i].C = C.data_ptr()
        arr[i].k = C.shape[0]
        arr[i].labels = lab.data_ptr()
    info = _native.kmb_batched_info()
    s = stream or torch.cuda.current_stream()
    rc = lib.kmb_batched_train(_native.KMB_F32, ctypes.cast(arr, ctypes.c_void_p), len(problems),
                               int(max_iteration_count), float(accuracy_threshold), int(bool(use_graph)),
                               ctypes.c_void_p(s.cuda_stream), ctypes.byref(info))
    if rc != _native.KMB_OK:
        raise BatchedError(f"kmb_batched_train failed: {lib.kmb_status_string(rc).decode()}")
    out = [(C, lab, int(arr[i].iterations)) for i, (X, C, lab) in enumerate(keep)]
    return out, {f: getattr(info, f) for f, _ in info._fields_}
