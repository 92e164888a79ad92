"""Failure paths, exercised without faulting the GPU.

* A bounded device wait that runs out: the tensor-core kernel's pipeline waits
  get a short limit (KMB_TC_WAIT_LIMIT_CYCLES, read at launch); the launch must
  drain its own copies and MMAs, report KMB_ETIMEDOUT, and leave the context
  usable for a correct call afterwards.
* Host-side allocation failure (KMB_FAIL_ALLOC=1 makes every workspace growth
  fail): KMB_ENOMEM, raised as bad_alloc by the Python mirror and as oneDAL's
  host_bad_alloc by the dispatcher (backend/interop/error_converter.cpp maps
  DAAL's allocation errors the same way); the next call without the hook works.
* NaN rows: the reference's argmin starts from the first cluster's score and
  replaces it only on a strictly smaller one (kmeans_lloyd_impl.i:197-216,
  kmeans_lloyd_postprocessing.h:95-130), so a row whose scores are all NaN gets
  cluster 0; the other rows are unaffected.
"""
import os
import subprocess

import numpy as np
import pytest
import torch

from onedal_b200 import _native, kmeans
from oracle import restated

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLIENT = os.path.join(ROOT, "integration", "_build", "kmeans_client")


def _blobs(n, d, k, seed):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-5, 5, (k, d))
    X = (centres[rng.integers(0, k, n)] + rng.standard_normal((n, d))).astype(np.float32)
    return X, X[rng.choice(n, k, replace=False)].copy()


@pytest.mark.parametrize("form", [kmeans.compute_form.bf16x3, kmeans.compute_form.bf16])
def test_tensor_core_wait_limit_reports_timeout_and_context_recovers(form, monkeypatch):
    X, C = _blobs(60000, 128, 512, 31)
    desc = kmeans.descriptor(np.float32).set_cluster_count(512).set_compute_form(form)
    monkeypatch.setenv("KMB_TC_WAIT_LIMIT_CYCLES", "200")  # below one accumulator's MMA time
    with pytest.raises(kmeans.internal_error) as err:
        kmeans.infer(desc, kmeans.model(C), X)
    assert "status 4" in str(err.value)  # KMB_ETIMEDOUT
    monkeypatch.delenv("KMB_TC_WAIT_LIMIT_CYCLES")
    r = kmeans.infer(desc, kmeans.model(C), X)
    lab64, _, _ = restated.assign_f32_in_f64(X, C)
    np.testing.assert_array_equal(r.get_responses().ravel(), lab64)
    t = kmeans.train(desc.set_max_iteration_count(3), X, C)
    assert t.get_iteration_count() == 3


def test_allocation_failure_raises_bad_alloc_and_context_recovers(monkeypatch):
    X, C = _blobs(30000, 24, 40, 32)
    desc = kmeans.descriptor(np.float32).set_cluster_count(40).set_max_iteration_count(5)
    _native.context(0).lib.kmb_context_release_workspace(_native.context(0).handle)
    monkeypatch.setenv("KMB_FAIL_ALLOC", "1")
    with pytest.raises(kmeans.bad_alloc):
        kmeans.train(desc, X, C)
    monkeypatch.delenv("KMB_FAIL_ALLOC")
    r = kmeans.train(desc, X, C)
    ref = restated.train(X.astype(np.float64), C.astype(np.float64), 5, 0.0)
    assert r.get_iteration_count() == ref[3]


@pytest.mark.skipif(not os.path.exists(CLIENT), reason="integration client not built")
def test_client_maps_allocation_failure_to_host_bad_alloc(tmp_path):
    """Through dal::train: KMB_ENOMEM becomes oneDAL's host_bad_alloc, whose what()
    is std::bad_alloc's (cpp/oneapi/dal/exceptions.cpp:61-63)."""
    import json
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "gold.json")))
    X = np.asarray(g["data"], np.float64).ravel()
    C = np.asarray(g["initial_centroids"], np.float64).ravel()
    p = tmp_path / "gold.txt"
    p.write_text("%d %d %d\n%s\n%s\n" % (g["row_count"], g["column_count"], g["cluster_count"],
                                          " ".join(repr(float(v)) for v in X), " ".join(repr(float(v)) for v in C)))
    env = dict(os.environ, KMB_FAIL_ALLOC="1")
    r = subprocess.run([CLIENT, str(p), "double"], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 1, (r.stdout, r.stderr)
    assert r.stdout.strip() == "exception: std::bad_alloc", r.stdout


@pytest.mark.parametrize("dt,form", [(np.float32, kmeans.compute_form.plain), (np.float64, kmeans.compute_form.plain),
                                     (np.float32, kmeans.compute_form.bf16x3)])
def test_nan_rows_take_cluster_zero(dt, form):
    X, C = _blobs(5000, 32, 17, 33)
    X = X.astype(dt)
    C = C.astype(dt)
    nan_rows = np.array([3, 100, 4999])
    X[nan_rows, 5] = np.nan
    desc = kmeans.descriptor(dt).set_cluster_count(17).set_compute_form(form)
    r = kmeans.infer(desc, kmeans.model(C), X)
    lab = r.get_responses().ravel()
    oracle_lab, _ = restated.infer(X.astype(np.float64), C.astype(np.float64), False)
    assert (oracle_lab[nan_rows] == 0).all()
    np.testing.assert_array_equal(lab, oracle_lab)
