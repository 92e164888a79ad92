"""GPU test of kmb_infer_noalloc, the entry point for callers that cannot
allocate device memory (a plugin whose host framework owns every device
allocation, or a latency-bound loop that cannot pay for cudaMalloc/cudaFree).

It is called through the C ABI twice in a row and must match kmb_infer (the
allocating entry point) each time: responses exactly, the objective within the
1e-6 relative tolerance the parity tests use. Each result is also checked
against the FP64 oracle (restated.infer): responses equal except on rows whose
FP64 top-2 gap lies inside the stated FP32 band (none for float64), and the
objective within 1e-6 relative. Shapes cover the tiled kernel and the few-cluster
kernel (k <= 32, d <= 64). The file sorts last so that a run stopping at the
first failure has already run every other test; it also passes on its own in a
fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

from onedal_b200 import _native
from oracle import restated

pytestmark = pytest.mark.gpu

OBJ_TOL = 1e-6


def _infer_allocating(ctx, dtype, X, C):
    n, d = X.shape
    k = C.shape[0]
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    obj = ctypes.c_double()
    ctx.check(ctx.lib.kmb_infer(ctx.handle, dtype, _native.KMB_MEM_DEVICE, X.data_ptr(), n, d, C.data_ptr(), k,
                                _native.KMB_FORM_PLAIN, 1, lab.data_ptr(), ctypes.byref(obj), None))
    return lab.cpu().numpy(), obj.value


def _infer_noalloc(lib, dtype, X, C, stream):
    n, d = X.shape
    k = C.shape[0]
    lab = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    obj = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.kmb_infer_noalloc(dtype, ctypes.c_void_p(X.data_ptr()), n, d, ctypes.c_void_p(C.data_ptr()), k,
                               ctypes.c_void_p(lab.data_ptr()), ctypes.c_void_p(obj.data_ptr()),
                               ctypes.c_void_p(stream.cuda_stream))
    assert rc == _native.KMB_OK
    stream.synchronize()
    return lab.cpu().numpy(), float(obj.item())


def _fp64_labels_and_band(X, C, dt):
    """The FP64 oracle's labels and the rows whose FP64 top-2 gap lies inside the
    plain form's error band (the same bound as the parity tests)."""
    lab64, b, s = restated.assign(X.astype(np.float64), C.astype(np.float64))
    u = 2.0 ** -24 if dt == np.float32 else 2.0 ** -53
    xn = np.sqrt((X.astype(np.float64) ** 2).sum(1))
    cmax = np.sqrt((C.astype(np.float64) ** 2).sum(1)).max()
    band = 2 * 1.0625 * u * (cmax ** 2 + (X.shape[1] + 2) * xn * cmax)
    return lab64, (s - b) <= 2 * band


@pytest.mark.parametrize("n,d,k", [(50_000, 40, 300), (30_000, 20, 20)])
@pytest.mark.parametrize("torch_dtype,dtype", [(torch.float32, _native.KMB_F32), (torch.float64, _native.KMB_F64)])
def test_noalloc_matches_allocating_infer_twice(torch_dtype, dtype, n, d, k):
    g = torch.Generator(device="cpu").manual_seed(7 + k)
    centres = torch.rand(k, d, generator=g, dtype=torch.float64) * 20 - 10
    X = (centres[torch.randint(0, k, (n,), generator=g)] + torch.randn(n, d, generator=g, dtype=torch.float64))
    X = X.to(torch_dtype).cuda()
    C = X[:k].clone() + 0.25
    ctx = _native.context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ref_lab, ref_obj = _infer_allocating(ctx, dtype, X, C)
    Xh, Ch = X.cpu().numpy(), C.cpu().numpy()
    np_dt = np.float32 if dtype == _native.KMB_F32 else np.float64
    lab64, near = _fp64_labels_and_band(Xh, Ch, np_dt)
    lib = _native.load_library()
    for _ in range(2):
        lab, obj = _infer_noalloc(lib, dtype, X, C, stream)
        np.testing.assert_array_equal(lab, ref_lab)
        assert abs(obj - ref_obj) <= OBJ_TOL * abs(ref_obj)
        assert ((lab == lab64) | near).all()
        obj64 = restated.objective(Xh.astype(np.float64), Ch.astype(np.float64), lab)
        assert abs(obj - obj64) <= OBJ_TOL * abs(obj64)
    oracle_lab, oracle_obj = restated.infer(Xh.astype(np.float64), Ch.astype(np.float64), True)
    assert ((lab == oracle_lab) | near).all()
    if not near.any():
        assert abs(obj - oracle_obj) <= OBJ_TOL * abs(oracle_obj)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = _native.load_library()
    n, d, k = 4_000_000, 8, 16  # 2 * 4M * 4 bytes of row scratch alone exceeds the 24 MiB array
    X = torch.zeros(1, dtype=torch.float32, device="cuda")  # never read: the size check comes first
    lab = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.kmb_infer_noalloc(_native.KMB_F32, ctypes.c_void_p(X.data_ptr()), n, d, ctypes.c_void_p(X.data_ptr()),
                               k, ctypes.c_void_p(lab.data_ptr()), None, None)
    assert rc == _native.KMB_EINVAL
