"""The drop-in proof: a oneDAL client compiled against the unchanged oneDAL
headers and runtime sources (integration/Makefile), whose host-policy k-means
dispatchers are integration/kmeans_dispatcher_b200.cpp. On a GPU it must
reproduce the reference's gold known-answer case (cpp/oneapi/dal/algo/kmeans/
test/fixture.hpp:156-203 with test/data.hpp) through dal::train / dal::infer,
and its smoke case (fixture.hpp:221-252) through train() without initial
centroids (the default k-means++ init);
without a GPU the dispatcher must surface the library's failure as a oneDAL
exception. The client is built only where the reference tree is present; the
built binary travels with the tree."""
import json
import os
import subprocess

import numpy as np
import pytest

from helpers import centroid_rel_err, find_match_centroids, rel_close

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLIENT = os.path.join(ROOT, "integration", "_build", "kmeans_client")

needs_client = pytest.mark.skipif(not os.path.exists(CLIENT), reason="integration client not built")


def _gold_file(tmp_path):
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "gold.json")))
    X = np.asarray(g["data"], np.float64).ravel()
    C = np.asarray(g["initial_centroids"], np.float64).ravel()
    p = tmp_path / "gold.txt"
    p.write_text("%d %d %d\n%s\n%s\n" % (g["row_count"], g["column_count"], g["cluster_count"],
                                          " ".join(repr(float(v)) for v in X), " ".join(repr(float(v)) for v in C)))
    return g, str(p)


def _parse(out):
    res = {}
    for line in out.splitlines():
        key, _, rest = line.partition(" ")
        res[key] = rest
    return res


DISPATCHER_OBJ = os.path.join(ROOT, "integration", "_build", "kmeans_dispatcher_b200.o")


@pytest.mark.skipif(not os.path.exists(DISPATCHER_OBJ), reason="integration dispatcher not built")
def test_dispatcher_exports_every_reference_instantiation():
    """The replacement keeps every symbol the reference's INSTANTIATE lines export
    (detail/train_ops.cpp:35-42: host_policy and spmd_host_policy trains,
    detail/infer_ops.cpp:37-43: host_policy infers), for both methods and types."""
    syms = subprocess.run(["nm", "-C", DISPATCHER_OBJ], capture_output=True, text=True).stdout
    defined = [ln for ln in syms.splitlines() if " W " in ln or " T " in ln]
    host = "oneapi::dal::detail::v1::host_policy"
    spmd = "oneapi::dal::detail::v1::spmd_policy<oneapi::dal::detail::v1::host_policy>"
    want = []
    for f in ("float", "double"):
        for m in ("lloyd_dense", "lloyd_csr"):
            tail = f", {f}, oneapi::dal::kmeans::method::v1::{m}, oneapi::dal::kmeans::task::v1::clustering>::operator()"
            want += [f"train_ops_dispatcher<{host}{tail}", f"infer_ops_dispatcher<{host}{tail}",
                     f"train_ops_dispatcher<{spmd}{tail}"]
    for w in want:
        assert any(w in ln for ln in defined), w


@needs_client
def test_client_links_b200_library():
    deps = subprocess.run(["ldd", CLIENT], capture_output=True, text=True).stdout
    assert "libonedal_b200_kmeans.so" in deps and "not found" not in deps


@needs_client
def test_client_reports_library_failure_as_onedal_exception(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU test covers the success path")
    _, path = _gold_file(tmp_path)
    r = subprocess.run([CLIENT, path, "double"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert r.stdout.startswith("exception: ")


@pytest.mark.gpu
@needs_client
@pytest.mark.parametrize("dtype,rtol", [("double", 1e-7), ("float", 1e-6)])
def test_client_gold_through_dal_train_infer(tmp_path, dtype, rtol):
    """Checks as the reference fixture does: centroids through the nearest-centroid
    match map (fixture.hpp:680-706), responses through the same map, objectives at
    relative 1e-7 (1e-6 for float)."""
    g, path = _gold_file(tmp_path)
    r = subprocess.run([CLIENT, path, dtype], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = _parse(r.stdout)
    cen = np.array(out["centroids"].split(), np.float64).reshape(g["cluster_count"], g["column_count"])
    exp = np.asarray(g["expected_centroids"], np.float64).reshape(cen.shape)
    m = find_match_centroids(exp, cen)
    assert centroid_rel_err(exp, cen, m) < rtol
    resp = np.array(out["responses"].split(), np.int64)
    assert (m[resp] == np.asarray(g["expected_responses"]).ravel()).all()
    assert rel_close(float(out["objective"]), g["expected_objective"], rtol)
    assert rel_close(float(out["infer_objective"]), g["expected_objective"], rtol)
    assert out.get("invalid_argument") == "ok"
    # fixture.hpp:221-252 without initial centroids: compared WITHOUT a match map
    sc = np.array(out["smoke_centroids"].split(), np.float64).reshape(2, 2)
    assert centroid_rel_err(np.array([[-1.5, -1.5], [1.5, 1.5]]), sc) < rtol
    assert out["smoke_responses"].split() == ["1", "1", "1", "1", "0", "0", "0", "0"]
    # method::lloyd_csr on a one-based csr_table (test/batch.cpp:406-480): objective 100
    assert out["csr_responses"].split() == ["0", "0", "1"]
    assert rel_close(float(out["csr_objective"]), 100.0, rtol)
    assert rel_close(float(out["csr_infer_objective"]), 100.0, rtol)
