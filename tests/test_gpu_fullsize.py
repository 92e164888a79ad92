"""The benchmark's own configurations, at their full sizes, against the FP64 oracle.

* precision configuration: n = 20,000,000 rows, d = 128, k = 1024, float32 input,
  both tensor-core forms (three split BF16 products, or one) with the FP64
  recheck, 20 Lloyd iterations from a seeded
  row sample (10 % of the rows on perpendicular bisectors of centre pairs);
* plain configuration at scale: n = 10,000,000, d = 64, k = 256, float32, plain
  FP32 form, 20 iterations.

Every iteration t of the Lloyd loop (kmb_lloyd_iterate, the benchmark's entry
point, run for t = 1, 2, ... updates from the same start -- the loop is
deterministic, so the t-th call's last update is the t-th update of the long run)
is checked against the oracle semantics of kmeans_lloyd_batch_impl.i:117-213 and
kmeans_lloyd_impl.i:137-246 on the host:

* responses: the assignment under C^(t-1) of a fixed seeded sample of 200,000
  rows plus the rows the GPU re-scored in FP64 in that pass
  (kmb_context_recheck_rows; all of them, or a seeded 200,000 when more were
  queued) equals the FP64 oracle's (restated.assign_f32_in_f64):
  exactly for the tensor-core form; for the plain form exactly outside the stated
  FP32 band (rows whose FP64 top-2 gap is below 2*1.0625*u*(cmax^2 + (d+2)||x|| cmax));
  assignment is row-independent, so a sample is a valid check;
* centroids: an FP64 pass over all n rows on the host (per-cluster sums and counts
  of the GPU's labels, restated.cluster_stats_f32) gives C^(t); the GPU's agree
  within 1e-5 relative; the number of empty clusters agrees;
* after the last update: the final responses and exact objective (kmb_infer with
  the objective, the train's final pass) -- responses as above, the objective
  within 1e-6 relative of the FP64 objective of the same labels over all rows.

Row offsets at these sizes pass 2^31 elements (20M x 128 = 2.56e9), which is what
these tests are for. They take a few minutes (the host FP64 passes dominate).
"""
import ctypes

import numpy as np
import pytest
import torch

from helpers import centroid_rel_err, rel_close
from onedal_b200 import _native, workloads
from oracle import restated

pytestmark = pytest.mark.gpu

CENTROID_TOL = 1e-5
OBJ_TOL = 1e-6
SAMPLE_ROWS = 200_000


def _band_rows(X, C, b, s, u=2.0 ** -24):
    """Rows whose FP64 top-2 score gap lies inside the plain FP32 form's band."""
    xn = np.sqrt((X.astype(np.float64) ** 2).sum(1))
    cmax = np.sqrt((C.astype(np.float64) ** 2).sum(1)).max()
    band = 2 * 1.0625 * u * (cmax ** 2 + (X.shape[1] + 2) * xn * cmax)
    return (s - b) <= 2 * band


QUEUED_ROWS = 200_000


def _recheck_rows(ctx, n, rng):
    """Rows the GPU re-scored in FP64 in its last pass (a seeded subset of
    QUEUED_ROWS of them when there are more, so the host check stays seconds)."""
    cap = n
    buf = torch.empty(cap, dtype=torch.int32, device="cuda")
    cnt = ctypes.c_int64()
    ctx.check(ctx.lib.kmb_context_recheck_rows(ctx.handle, buf.data_ptr(), cap, ctypes.byref(cnt)))
    q = buf[: min(cnt.value, cap)].cpu().numpy().astype(np.int64)
    return (np.sort(rng.choice(q, QUEUED_ROWS, replace=False)) if len(q) > QUEUED_ROWS else q), int(cnt.value)


def _check_labels(Xh, rows, gpu_lab, C_prev, exact, what):
    lab64, b, s = restated.assign_f32_in_f64(Xh[rows], C_prev)
    bad = gpu_lab[rows] != lab64
    if not exact:
        bad &= ~_band_rows(Xh[rows], C_prev, b, s)
    assert int(bad.sum()) == 0, f"{what}: {int(bad.sum())} of {len(rows)} checked responses differ from the FP64 oracle"


def _run_configuration(w, form, iterations):
    X, C0 = workloads.make(w, "cuda")
    torch.cuda.synchronize()
    n, d = X.shape
    k = C0.shape[0]
    Xh = torch.empty((n, d), dtype=torch.float32, pin_memory=True)
    Xh.copy_(X)
    Xh = Xh.numpy()
    rng = np.random.default_rng(w.seed + 99)
    sample = np.sort(rng.choice(n, SAMPLE_ROWS, replace=False))
    ctx = _native.context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    exact = form in (_native.KMB_FORM_BF16X3, _native.KMB_FORM_BF16)
    C_prev = C0.cpu().numpy()
    empties = 0
    rechecked = []
    for t in range(1, iterations + 1):
        C = C0.clone()
        p = _native.kmb_params(k, t, 0.0, form, 0)
        it = ctypes.c_int64()
        st = _native.kmb_stats()
        ctx.check(ctx.lib.kmb_lloyd_iterate(ctx.handle, _native.KMB_F32, X.data_ptr(), n, d, C.data_ptr(),
                                            ctypes.byref(p), lab.data_ptr(), ctypes.byref(it), ctypes.byref(st)))
        assert it.value == t, f"the loop stopped after {it.value} of {t} updates"
        g_lab = lab.cpu().numpy()
        g_C = C.cpu().numpy()
        rows = sample
        if exact:
            q, queued = _recheck_rows(ctx, n, rng)
            rechecked.append(queued)
            rows = np.union1d(sample, q)
        _check_labels(Xh, rows, g_lab, C_prev, exact, f"update {t}")
        sums, counts, _ = restated.cluster_stats_f32(Xh, g_lab, k)
        empty = counts == 0
        empties += int(empty.sum())
        assert st.empty_cluster_events == empties, (t, st.empty_cluster_events, empties)
        ref = np.where(empty[:, None], g_C.astype(np.float64), sums / np.maximum(counts, 1)[:, None])
        err = centroid_rel_err(ref, g_C)
        assert err < CENTROID_TOL, f"update {t}: centroid relative error {err}"
        for j in np.nonzero(empty)[0]:  # a reseeded cluster takes one of the rows
            assert (Xh == g_C[j]).all(1).any(), f"update {t}: reseeded cluster {j} is not a data row"
        C_prev = g_C
    # the train's final pass: responses and the exact objective under the last centroids
    Cd = torch.from_numpy(C_prev).cuda()
    obj = ctypes.c_double()
    ctx.check(ctx.lib.kmb_infer(ctx.handle, _native.KMB_F32, _native.KMB_MEM_DEVICE, X.data_ptr(), n, d,
                                Cd.data_ptr(), k, form, 1, lab.data_ptr(), ctypes.byref(obj), None))
    g_lab = lab.cpu().numpy()
    rows = np.union1d(sample, _recheck_rows(ctx, n, rng)[0]) if exact else sample
    _check_labels(Xh, rows, g_lab, C_prev, exact, "final responses")
    _, _, obj64 = restated.cluster_stats_f32(Xh, g_lab, k, C_prev)
    assert rel_close(obj.value, obj64, OBJ_TOL), (obj.value, obj64)
    return rechecked


@pytest.mark.parametrize("form", [_native.KMB_FORM_BF16X3, _native.KMB_FORM_BF16])
def test_precision_configuration_full_size_every_iteration(form):
    """n = 20M, d = 128, k = 1024, a tensor-core form (split or single BF16 product)
    + FP64 recheck, 20 updates: every update's responses (sample + re-scored rows)
    equal the FP64 oracle's, centroids within 1e-5 of the host FP64 update, final
    objective within 1e-6."""
    w = workloads.PRECISION
    rechecked = _run_configuration(w, form, w.iterations)
    assert min(rechecked) > 0  # the near-tie rows do reach the recheck


def test_plain_configuration_at_scale_full_size_every_iteration():
    """n = 10M, d = 64, k = 256, plain FP32 form, 20 updates: responses exact outside
    the FP32 band, centroids within 1e-5 of the host FP64 update, final objective within
    1e-6."""
    w = workloads.PLAIN_GPU
    _run_configuration(w, _native.KMB_FORM_PLAIN, w.iterations)
