"""The resident plain FP32 assignment kernel against the tiled plain kernel.

Both compute every score h_j - x.c_j by FMAs in ascending feature order from zero,
so their responses, distances and recheck queues are identical, bit for bit. The
resident kernel (centroids held in shared memory, all at once or in chunks, 64-row
tiles taken in turn by two warp groups) applies to float rows with d a multiple of
4 and at most 256 whose 256 clusters fit in shared memory next to the row stages; KMB_PLAIN_RESIDENT=0 sends the same call to the
tiled kernel. The shapes cover row counts around the 64-row tile and the 128-row
step of the two groups (one group without a tile, a CTA with one tile), several
passes over 256 clusters, grids that wrap over the SMs more than once, and
centroids taken in chunks when they do not all fit (one or two row stages per
group, blocks of 4 or 8 tiles, up to 8 chunks).
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from onedal_b200 import _native

pytestmark = pytest.mark.gpu


def _infer(ctx, X, C):
    n, d = X.shape
    k = C.shape[0]
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    obj = ctypes.c_double()
    ctx.check(ctx.lib.kmb_infer(ctx.handle, _native.KMB_F32, _native.KMB_MEM_DEVICE, X.data_ptr(), n, d,
                                C.data_ptr(), k, _native.KMB_FORM_PLAIN, 1, lab.data_ptr(), ctypes.byref(obj), None))
    torch.cuda.synchronize()
    return lab.cpu().numpy(), obj.value


@pytest.mark.parametrize("n,d,k", [(1, 4, 40), (63, 64, 256), (64, 64, 256), (65, 64, 256), (127, 32, 100),
                                   (128, 64, 256), (129, 64, 256), (200, 96, 250), (4097, 64, 500),
                                   (148 * 128 * 3 + 65, 64, 256), (50000, 40, 700), (30000, 48, 96),
                                   # clusters in chunks: one or two stages per group, 4 or 8 tiles per block
                                   (1, 128, 1024), (65, 64, 1024), (3000, 128, 300), (5000, 128, 1024),
                                   (4097, 64, 1024), (2000, 100, 700), (70000, 128, 256), (20000, 96, 2000),
                                   (3000, 8, 5000)])
def test_resident_equals_tiled(n, d, k):
    ctx = _native.context(0)
    g = torch.Generator(device="cuda").manual_seed(n * 7 + d + k)
    X = torch.randn(n, d, device="cuda", generator=g) * 2.0
    C = torch.randn(k, d, device="cuda", generator=g) * 2.0
    old = os.environ.get("KMB_PLAIN_RESIDENT")
    try:
        os.environ["KMB_PLAIN_RESIDENT"] = "1"
        lab_r, obj_r = _infer(ctx, X, C)
        os.environ["KMB_PLAIN_RESIDENT"] = "0"
        lab_t, obj_t = _infer(ctx, X, C)
    finally:
        if old is None:
            os.environ.pop("KMB_PLAIN_RESIDENT", None)
        else:
            os.environ["KMB_PLAIN_RESIDENT"] = old
    assert (lab_r == lab_t).all()
    assert obj_r == obj_t
    # the resident kernel did run: its responses under C are the FP32 argmin
    Xd, Cd = X.double().cpu().numpy(), C.double().cpu().numpy()
    s = 0.5 * (Cd ** 2).sum(1)[None, :] - Xd @ Cd.T
    best = np.take_along_axis(s, lab_r[:, None].astype(np.int64), 1)[:, 0]
    assert (best <= s.min(1) + 1e-3 * (1 + np.abs(s.min(1)))).all()


def test_resident_nan_rows_take_cluster_zero():
    """NaN rows: every score is NaN, no strict '<' holds, so the row keeps cluster 0
    (the reference's strict-'<' scan) in both kernels; the other rows are unaffected."""
    ctx = _native.context(0)
    g = torch.Generator(device="cuda").manual_seed(11)
    X = torch.randn(5000, 64, device="cuda", generator=g) * 2.0
    C = torch.randn(100, 64, device="cuda", generator=g) * 2.0
    nan_rows = [3, 100, 4999]
    X[nan_rows, 5] = float("nan")
    old = os.environ.get("KMB_PLAIN_RESIDENT")
    try:
        os.environ["KMB_PLAIN_RESIDENT"] = "1"
        lab_r, _ = _infer(ctx, X, C)
        os.environ["KMB_PLAIN_RESIDENT"] = "0"
        lab_t, _ = _infer(ctx, X, C)
    finally:
        if old is None:
            os.environ.pop("KMB_PLAIN_RESIDENT", None)
        else:
            os.environ["KMB_PLAIN_RESIDENT"] = old
    assert (lab_r == lab_t).all()
    assert (lab_r[nan_rows] == 0).all()
