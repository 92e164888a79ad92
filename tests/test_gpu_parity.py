"""GPU parity tests: the CUDA path (through the C ABI) against the oracle.

Cases mirror the reference suite (cpp/oneapi/dal/algo/kmeans/test/batch.cpp,
fixture.hpp) plus seeded synthetic workloads in per-iteration lock-step with
the FP64 oracle. Tolerances:
  responses   exact (plain form: exact except rows whose FP64 top-2 gap is below
              the stated bound; recheck/BF16x3 forms: exact)
  centroids   1e-5 relative (float32) / 1e-12 (float64) vs the FP64 oracle
  objective   1e-6 relative vs the FP64 oracle
"""
import os
import sys

import numpy as np
import pytest
import torch

from helpers import GOLDEN, centroid_rel_err, find_match_centroids, load_json, norm_rel_err, rel_close
from onedal_b200 import kmeans, workloads
from oracle import restated

pytestmark = pytest.mark.gpu

DTYPES = [np.float64, np.float32]
CENTROID_TOL = {np.float32: 1e-5, np.float64: 1e-12}
OBJ_TOL = 1e-6


def desc(dt, k, T=100, eps=0.0, **kw):
    d = kmeans.descriptor(dt).set_cluster_count(k).set_max_iteration_count(T).set_accuracy_threshold(eps)
    if kw.get("recheck"):
        d.set_recheck(True)
    return d


@pytest.mark.parametrize("dt", DTYPES)
def test_gold_data(dt):
    """'kmeans train/infer on gold data' (fixture.hpp:156-203)."""
    g = load_json("gold.json")
    X = np.array(g["data"], dt).reshape(100, 3)
    C0 = np.array(g["initial_centroids"], dt).reshape(3, 3)
    r = kmeans.train(desc(dt, 3, 100, 0.0), X, C0)
    C = r.get_model().get_centroids()
    exp = np.array(g["expected_centroids"]).reshape(3, 3)
    m = find_match_centroids(exp, C)
    tol = 1e-7 if dt == np.float64 else 1e-6
    assert centroid_rel_err(exp, C, m) < tol
    assert rel_close(r.get_objective_function_value(), g["expected_objective"], tol)
    inf = kmeans.infer(desc(dt, 3), r.get_model(), X)
    assert (m[inf.get_responses().ravel()] == np.array(g["expected_responses"])).all()
    assert (r.get_responses().ravel() == inf.get_responses().ravel()).all()
    ref = restated.train(X.astype(np.float64), C0.astype(np.float64), 100, 0.0)
    assert r.get_iteration_count() == ref[3]


@pytest.mark.parametrize("dt", DTYPES)
def test_empty_clusters(dt):
    """'kmeans empty clusters test' (fixture.hpp:205-219): reseed order."""
    e = load_json("empty_clusters.json")
    X = np.array(e["data"], dt).reshape(10, 1)
    C0 = np.array(e["initial_centroids"], dt).reshape(3, 1)
    r = kmeans.train(desc(dt, 3, 1, 0.0), X, C0)
    np.testing.assert_allclose(r.get_model().get_centroids().ravel(), e["expected_centroids"],
                               rtol=5 * np.finfo(dt).eps * 100)
    assert r.get_responses().ravel().tolist() == e["expected_responses"]
    assert r.get_iteration_count() == 1
    assert r.stats.empty_cluster_events == 2


@pytest.mark.parametrize("dt", DTYPES)
def test_smoke_infer(dt):
    s = load_json("smoke_infer.json")
    X = np.array(s["data"], dt).reshape(8, 2)
    C = np.array(s["centroids"], dt).reshape(2, 2)
    d = desc(dt, 2).set_result_options(kmeans.result_options.compute_exact_objective_function)
    r = kmeans.infer(d, kmeans.model(C), X)
    assert r.get_responses().ravel().tolist() == s["expected_responses"]
    assert rel_close(r.get_objective_function_value(), s["expected_objective"], s["rel_tol"])
    with pytest.raises(kmeans.domain_error):
        kmeans.infer(desc(dt, 2), kmeans.model(C), X).get_objective_function_value()


@pytest.mark.parametrize("tag,dt", [("f64", np.float64), ("f32", np.float32)])
def test_example_dataset(tag, dt):
    """The example data (k=20, 5 iterations, eps 0.001) vs recorded reference-kernel outputs."""
    z = np.load(os.path.join(GOLDEN, "example_dense.npz"))
    r = kmeans.train(desc(dt, 20, 5, 0.001), z["X"].astype(dt), z["C0"].astype(dt))
    assert r.get_iteration_count() == int(z[f"iters_{tag}"])
    assert (r.get_responses().ravel() == z[f"labels_{tag}"]).all()
    ref64 = restated.train(z["X"], z["C0"], 5, 0.001)
    assert centroid_rel_err(ref64[0], r.get_model().get_centroids()) < CENTROID_TOL[dt]
    assert rel_close(r.get_objective_function_value(), ref64[2], OBJ_TOL)


@pytest.mark.parametrize("fixture", ["daal_ref_c1.npz", "daal_ref_c1_small.npz"])
@pytest.mark.parametrize("tag,dt", [("f64", np.float64), ("f32", np.float32)])
def test_blob_workload_end_to_end(tag, dt, fixture):
    """The plain configuration (n=100,000, d=20, k=20, init = first rows, eps 0, 50
    max iterations; and its 20,000-row prefix) vs the recorded reference-kernel run.
    float64: iteration count, responses, centroids and objective as the reference's.
    float32: the reference's own FP32 labels differ from any other FP32 summation
    order on near-ties (at 100,000 rows enough to move the unconverged trajectory),
    so responses are checked against the FP64 oracle under the returned centroids
    (exact outside the rounding band) and against the reference's FP32 labels up to
    0.1 % (prefix) / 0.5 % (full size) of rows; the objective against the FP64
    objective of the returned labels (1e-6) and the reference's (1e-5)."""
    sys.path.insert(0, GOLDEN)
    from make_golden import blobs_c1
    z = np.load(os.path.join(GOLDEN, fixture))
    X = blobs_c1(int(z["n"]), int(z["seed"])).astype(dt)
    r = kmeans.train(desc(dt, 20, 50, 0.0), X, X[:20].copy())
    C = r.get_model().get_centroids()
    lab = r.get_responses().ravel()
    assert r.get_iteration_count() == int(z[f"iters_{tag}"])
    if dt == np.float64:
        assert (lab == z[f"labels_{tag}"]).all()
        assert centroid_rel_err(z[f"C_{tag}"], C) < CENTROID_TOL[dt]
        ref64 = restated.train(X, X[:20].copy(), 50, 0.0)
        assert centroid_rel_err(ref64[0], C) < CENTROID_TOL[dt]
        assert rel_close(r.get_objective_function_value(), ref64[2], OBJ_TOL)
        assert rel_close(r.get_objective_function_value(), float(z["obj_f64"]), OBJ_TOL)
    else:
        limit = 1e-3 if int(z["n"]) <= 20000 else 5e-3
        assert (lab != z[f"labels_{tag}"]).mean() < limit
        lab64, near = _fp64_gap_bound(X, C, dt)
        assert ((lab == lab64) | near).all()
        obj64 = restated.objective(X.astype(np.float64), C.astype(np.float64), lab)
        assert rel_close(r.get_objective_function_value(), obj64, OBJ_TOL)
        assert rel_close(r.get_objective_function_value(), float(z["obj_f64"]), 1e-5)


@pytest.mark.parametrize("dt", DTYPES)
def test_lockstep_plain_configuration_full_size(dt):
    """The plain configuration at its full 100,000 rows, all 50 iterations in
    lock-step with the FP64 oracle from identical C^(t) (float32 with the FP64
    recheck, so every response is exact)."""
    sys.path.insert(0, GOLDEN)
    from make_golden import blobs_c1
    X = blobs_c1(100_000, 1001).astype(dt)
    stats = _lockstep(X, X[:20].copy(), 50, dt, recheck=(dt == np.float32))
    assert all(s[0] == 0 for s in stats)


def _fp64_gap_bound(X, C, dt):
    """Rows whose FP64 top-2 score gap is below the plain form's rounding band (these
    may legitimately differ without recheck)."""
    lab64, b, s = restated.assign_f32_in_f64(X.astype(np.float32), C.astype(np.float32)) if dt == np.float32 else \
        restated.assign(X, C)
    u = 2.0 ** -24 if dt == np.float32 else 2.0 ** -53
    xn = np.sqrt((X.astype(np.float64) ** 2).sum(1))
    cmax = np.sqrt((C.astype(np.float64) ** 2).sum(1)).max()
    band = 2 * 1.0625 * u * (cmax ** 2 + (X.shape[1] + 2) * xn * cmax)
    return lab64, (s - b) <= 2 * band


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("n,d,k", [(1, 1, 1), (129, 3, 5), (1000, 7, 130), (4099, 37, 257), (3000, 130, 64),
                                   (2048, 256, 300)])
def test_infer_ragged_shapes(dt, n, d, k):
    """Ragged n, d, k (not multiples of the 128-row / 128-cluster / 8-column tiles)."""
    rng = np.random.default_rng(n + d + k)
    X = (rng.standard_normal((n, d)) * 3).astype(dt)
    C = X[rng.choice(n, k, replace=n < k)].copy() if k <= n else rng.standard_normal((k, d)).astype(dt)
    C = C + rng.standard_normal(C.shape).astype(dt) * 0.1
    dsc = desc(dt, k).set_result_options(kmeans.result_options.compute_exact_objective_function)
    r = kmeans.infer(dsc, kmeans.model(C), X)
    lab = r.get_responses().ravel()
    lab64, near = _fp64_gap_bound(X, C, dt)
    assert ((lab == lab64) | near).all()
    obj64 = restated.objective(X.astype(np.float64), C.astype(np.float64), lab)
    assert rel_close(r.get_objective_function_value(), obj64, OBJ_TOL)


@pytest.mark.parametrize("dt", DTYPES)
def test_one_cluster_means(dt):
    """'kmeans block test' (fixture.hpp:254-287): k=1, one iteration -> column means;
    objective = sum of per-column variances * (n - 1)."""
    n, d = 1 << 16, 1024 // np.dtype(dt).itemsize
    rng = np.random.default_rng(11)
    X = rng.uniform(-0.2, 0.5, (n, d)).astype(dt)
    r = kmeans.train(desc(dt, 1, 1, 0.0), X, X[:1].copy())
    mean = X.astype(np.float64).mean(0)
    assert centroid_rel_err(mean[None, :], r.get_model().get_centroids()) < CENTROID_TOL[dt]
    obj = (X.astype(np.float64).var(0, ddof=1) * (n - 1)).sum()
    assert rel_close(r.get_objective_function_value(), obj, OBJ_TOL)
    assert (r.get_responses() == 0).all()


@pytest.mark.parametrize("dt", DTYPES)
def test_partial_centroids_stress(dt):
    """'kmeans partial centroids stress test' (fixture.hpp:289-308), scaled: k = n,
    init = data, one iteration -> responses = iota, centroids = data."""
    n, d = 2048, 512
    rng = np.random.default_rng(12)
    X = rng.uniform(-0.2, 0.5, (n, d)).astype(dt)
    r = kmeans.train(desc(dt, n, 1, 0.0), X, X)
    assert (r.get_responses().ravel() == np.arange(n)).all()
    np.testing.assert_array_equal(r.get_model().get_centroids(), X)


def _lockstep(X, C0, T, dt, recheck):
    """Per-iteration comparison with the FP64 oracle from identical C^(t)."""
    from onedal_b200 import _native
    ctx = _native.context(0)
    Xd = torch.from_numpy(X).cuda()
    Cd = torch.from_numpy(C0).cuda()
    n, d = X.shape
    k = C0.shape[0]
    out = torch.empty_like(Cd)
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    shift = __import__("ctypes").c_double()
    ne = __import__("ctypes").c_int64()
    dtype = _native.KMB_F32 if dt == np.float32 else _native.KMB_F64
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    stats = []
    for t in range(T):
        C_in = Cd.cpu().numpy()
        ctx.check(ctx.lib.kmb_lloyd_step(ctx.handle, dtype, Xd.data_ptr(), n, d, Cd.data_ptr(), k,
                                         _native.KMB_FORM_PLAIN, int(recheck), out.data_ptr(), lab.data_ptr(),
                                         __import__("ctypes").byref(shift), __import__("ctypes").byref(ne)))
        torch.cuda.synchronize()
        g_lab = lab.cpu().numpy()
        g_C = out.cpu().numpy()
        C64, lab64, shift64, ne64, _ = restated.step(X.astype(np.float64), C_in.astype(np.float64))
        if recheck or dt == np.float64:
            mism = int((g_lab != lab64).sum())
        else:
            _, near = _fp64_gap_bound(X, C_in, dt)
            mism = int(((g_lab != lab64) & ~near).sum())
        assert mism == 0, f"iteration {t}: {mism} responses differ from the FP64 oracle"
        if (g_lab == lab64).all() and ne64 == 0:
            assert centroid_rel_err(C64, g_C) < CENTROID_TOL[dt], t
            # The GPU's shift is sum ||c_old - c_new||^2 over centroids rounded to F;
            # the oracle's uses its unrounded FP64 centroids. With r = ||C64 - fl_F(C64)||,
            # | ||a||^2 - ||b||^2 | <= (||a|| + ||b||) ||a - b|| <= (2 sqrt(shift64) + r) r.
            r = float(np.linalg.norm(C64 - C64.astype(dt).astype(np.float64)))
            bound = 1.01 * (2.0 * np.sqrt(max(shift64, 0.0)) + r) * r + 1e-6 * abs(shift64) + 1e-12
            assert abs(shift.value - shift64) <= bound, (t, shift.value, shift64, bound)
        stats.append((int((g_lab != lab64).sum()), ne.value))
        Cd.copy_(out)
    return stats


@pytest.mark.parametrize("recheck", [False, True])
def test_lockstep_precision_shape_f32(recheck):
    """Reduced precision-shaped workload (d=128, k=256, 10% bisector near-ties): every
    iteration in lock-step with the FP64 oracle."""
    X, C0 = workloads.make(workloads.Workload("precision", 30000, 128, 256, 3, 0.0, 5), "cpu", 30000)
    _lockstep(X.numpy(), C0.numpy(), 3, np.float32, recheck)


def test_lockstep_plain_gpu_shape_f64():
    X, C0 = workloads.make(workloads.Workload("plain_gpu", 20000, 64, 64, 3, 0.0, 6), "cpu", 20000)
    _lockstep(X.double().numpy(), C0.double().numpy(), 3, np.float64, False)


@pytest.mark.parametrize("dt", DTYPES)
def test_deterministic_repeat(dt):
    """Same inputs twice -> bit-identical centroids, responses and objective."""
    X, C0 = workloads.make(workloads.Workload("plain_gpu", 50000, 16, 40, 10, 0.0, 9), "cpu", 50000)
    X = X.numpy().astype(dt)
    C0 = C0.numpy().astype(dt)
    a = kmeans.train(desc(dt, 40, 10, 0.0), X, C0)
    b = kmeans.train(desc(dt, 40, 10, 0.0), X, C0)
    np.testing.assert_array_equal(a.get_model().get_centroids(), b.get_model().get_centroids())
    np.testing.assert_array_equal(a.get_responses(), b.get_responses())
    assert a.get_objective_function_value() == b.get_objective_function_value()
    assert a.get_iteration_count() == b.get_iteration_count()


def test_device_tensors_round_trip():
    """torch CUDA tensors in, CUDA tensors out (device-resident path)."""
    X, C0 = workloads.make(workloads.PLAIN_CPU, "cuda", 20000)
    r = kmeans.train(desc(np.float32, 20, 10, 0.0), X, C0)
    assert r.get_model().get_centroids().is_cuda and r.get_responses().is_cuda
    rh = kmeans.train(desc(np.float32, 20, 10, 0.0), X.cpu().numpy(), C0.cpu().numpy())
    np.testing.assert_array_equal(r.get_model().get_centroids().cpu().numpy(), rh.get_model().get_centroids())
    np.testing.assert_array_equal(r.get_responses().cpu().numpy(), rh.get_responses())


def test_max_iteration_zero_uses_initial_centroids():
    rng = np.random.default_rng(4)
    X = rng.standard_normal((500, 4))
    C0 = X[:6].copy()
    r = kmeans.train(desc(np.float64, 6, 0, 0.0), X, C0)
    assert r.get_iteration_count() == 0
    np.testing.assert_array_equal(r.get_model().get_centroids(), C0)
    lab, obj = restated.infer(X, C0, True)
    assert (r.get_responses().ravel() == lab).all()
    assert rel_close(r.get_objective_function_value(), obj, 1e-12)
